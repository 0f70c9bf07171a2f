"""Per-object windows (incrmt_sim_set_windows): the same runs with the
level-set, pinning and reference-map passes restricted to each object's
windows and with every pass over the whole grid give the same state.

Four scenes: seeded circles and ellipses settling in the sediment box (many
small solids, the case the windows are for), the simple spinner (one solid
spanning most of the grid), the flag in its y-periodic channel with inflow,
and circles carried by the same inflow in a y-periodic channel, next to both
periodic ends (the windows that reach an end span the height). Compared after 30-40
steps: velocities and pressure to 1e-10 of their maximum (the projections
run to a 1e-9 residual, and the comparison allows for their summation order
only), every object's reference map and level set to 1e-10, statuses and
sweep counts exactly. Far outside a solid the windowed run leaves the
reference map's edge and slope values (never read) at older values, so
those arrays are not compared.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SED_BOX = (-0.75, 0.75, -1.5, 1.5)


def _rel(a, b):
    # a non-finite value where the other array is finite fails the comparison
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    fa, fb = np.isfinite(a), np.isfinite(b)
    if not np.array_equal(fa, fb):
        return float("inf")
    if not fb.any():
        return 0.0
    d = np.abs(a[fb] - b[fb])
    s = np.abs(b[fb]).max()
    return float(d.max() / (s if s > 0 else 1.0))


def _sediment(windows, m=128, count=12):
    from incrmt_b200 import capi, workloads
    ax, bx, ay, by = SED_BOX
    sim = capi.Simulation(m, 2 * m, ax=ax, bx=bx, ay=ay, by=by, visc=2e-3, ntrace=64)
    for o in workloads.sediment_bodies(seed=5, count=count):
        if o["kind"] == "circle":
            sim.add_circle(o["cx"], o["cy"], o["r"], 1.0, o["rhos"], grav=o["grav"])
        else:
            sim.add_ellipse(o["cx"], o["cy"], o["r"], o["b"], o["theta"], 1.0, o["rhos"], grav=o["grav"])
    sim.set_windows(windows)
    dt = sim.initialize()
    rng = np.random.default_rng(3)
    sim.set_tracers(np.stack([rng.uniform(ax, bx, 64), rng.uniform(ay, by, 64)], axis=1))
    return sim, dt, count


def _spin(windows, m=128):
    from incrmt_b200 import capi
    sim = capi.Simulation(m, m, ntrace=16)
    sim.add_simple_spin()
    sim.set_windows(windows)
    dt = sim.initialize()
    rng = np.random.default_rng(4)
    sim.set_tracers(rng.uniform(-1, 1, size=(16, 2)))
    return sim, dt, 1


def _flag(windows, n=96):
    from incrmt_b200 import capi
    w, k_B, mu, Re = 0.1, 0.1, 1.0, 100.0
    sim = capi.Simulation(3 * n, n, ax=-1.0, bx=5.0, ay=-1.0, by=1.0, visc=1.0 / Re, ntrace=0,
                          y_prd=True, horiz_flow=1.0)
    sim.add_flag(0.0, 0.0, 1.0, w, 0.25 * w, 4 * k_B / w ** 3, mu / w, ntrace=17)
    sim.set_windows(windows)
    dt = sim.initialize()
    return sim, dt, 1


def _periodic_circles(windows, m=96):
    from incrmt_b200 import capi
    sim = capi.Simulation(m, 2 * m, ax=-0.5, bx=0.5, ay=-1.0, by=1.0, visc=2e-3, ntrace=0, y_prd=True,
                          horiz_flow=0.3)
    # one a cell above the lower end, one a cell below the upper end, one in
    # the middle
    for cx, cy, r, rhos in [(-0.2, -0.91, 0.08, 2.0), (0.2, 0.92, 0.07, 2.5), (0.0, 0.1, 0.09, 1.8)]:
        sim.add_circle(cx, cy, r, 1.0, rhos, grav=(rhos - 1) / rhos)
    sim.set_windows(windows)
    dt = sim.initialize()
    return sim, dt, 3


SCENES = {"sediment": (_sediment, 40), "spin": (_spin, 30), "flag": (_flag, 30),
          "periodic_circles": (_periodic_circles, 30)}


@pytest.mark.parametrize("scene", list(SCENES))
def test_windows_match_whole_grid(gpu, scene):
    make, steps = SCENES[scene]
    b, dt_b, _ = make(False)
    a, dt, nobj = make(True)
    assert dt == dt_b
    b.step(0.9 * dt, steps)
    a.step(0.9 * dt, steps)
    sa, sb = a.stats(), b.stats()
    assert sa.march_sweeps == sb.march_sweeps and sa.extrap_sweeps == sb.extrap_sweeps
    for f in ["u", "v", "p"]:
        e = _rel(a.get(f)[2:-2, 2:-2], b.get(f)[2:-2, 2:-2])
        assert e <= 1e-10, (f, e)
    for k in range(nobj):
        for f in ["X", "Y", "phi"]:
            e = _rel(a.get(f, k), b.get(f, k))
            assert e <= 1e-10, (f, k, e)
        assert np.array_equal(a.get("status", k), b.get("status", k)), k
    if scene in ("sediment", "spin"):
        assert np.abs(a.tracers()[:, :2] - b.tracers()[:, :2]).max() <= 1e-10
    if scene == "sediment":
        # the windows cover a small part of the grid
        grid = (128 + 4) * (256 + 4) * nobj
        assert 0 < sa.window_points < 0.5 * grid, sa.window_points
        assert sb.window_points == grid
    a.close()
    b.close()
