"""The extrapolated warm starts of the projections (incrmt_sim_set_guess 1,
linear, and 2, quadratic):
every solve stops at the same 1e-9 relative residual as with the previous
solution as the start (the reference's), so after 40 steps of the rotor and
of two falling bodies at 256^2 the fields agree with the default run to
what that tolerance carries (u, v, p to 1e-6 of their maximum; X, Y, phi to
1e-8), and the solves take fewer V-cycles; incrmt_set_field restarts the
history (the next two solves start from the previous solution).
"""
import numpy as np
import pytest

from test_coarse_refresh_gpu import _rel

pytestmark = pytest.mark.gpu


def _scene(kind, guess):
    from incrmt_b200 import capi
    g = capi.Simulation(256, 256, ntrace=0)
    if kind == "sspin":
        g.add_simple_spin()
    else:
        g.add_circle(-0.3, 0.2, 0.2, 1.0, 3.0, grav=0.6)
        g.add_ellipse(0.35, -0.1, 0.25, 0.12, 0.4, 1.0, 2.0, grav=0.5)
    g.set_guess(guess)
    dt = g.initialize()
    return g, dt


@pytest.mark.parametrize("kind", ["sspin", "bodies"])
@pytest.mark.parametrize("mode", [1, 2])
def test_extrapolated_guess(gpu, kind, mode):
    runs = {}
    for guess in (0, mode):
        g, dt = _scene(kind, guess)
        g.step(0.9 * dt, 40)
        runs[guess] = (g, g.stats())
    (g0, s0), (g1, s1) = runs[0], runs[mode]
    for f in ("u", "v", "p"):
        e = _rel(g1.get(f)[2:-2, 2:-2], g0.get(f)[2:-2, 2:-2])
        assert e <= 1e-6, (f, e)
    for k in range(g0.objects):
        for f in ("X", "Y", "phi"):
            e = _rel(g1.get(f, k)[2:-2, 2:-2], g0.get(f, k)[2:-2, 2:-2])
            assert e <= 1e-8, (f, k, e)
    vc0 = s0.vcycles_mac + s0.vcycles_fem
    vc1 = s1.vcycles_mac + s1.vcycles_fem
    assert vc1 < vc0, (vc0, vc1)
    for g, _ in runs.values():
        g.close()


def test_bad_mode_refused(gpu):
    from incrmt_b200 import capi
    g = capi.Simulation(64, 64, ntrace=0)
    with pytest.raises(capi.IncrmtError):
        g.set_guess(3)
    g.close()


def test_singular_systems_do_not_drift(gpu):
    """The rotor's walled box makes both pressure systems pure Neumann (no
    zero-pressure column): their solutions are fixed only up to a constant.
    The extrapolated starts remove the mean of their increment, so over many
    steps the quadratic start does not grow that constant (which it would
    at the square of the step count) and every solve still converges."""
    from incrmt_b200 import capi
    g = capi.Simulation(64, 64, ntrace=0)
    g.add_simple_spin()
    g.set_guess(2)
    dt = g.initialize()
    g.step(0.9 * dt, 400)
    for which in (0, 1):
        z = g.get_mg(which)
        spread = np.abs(z - z.mean()).max()
        assert abs(z.mean()) <= 10 * spread + 1e-12, (which, z.mean(), spread)
    g.close()
