"""GPU parity on the full-solid scenario of ftest ("full", ftest.cc:218-237)
and conv_test's type 2 (conv_test.cc:78-80, 116-120): one obj_full (phi = -1
everywhere, object.hh:83-86) filling sim_velocity_pulses' doubly periodic
[-1,1]^2, set_velocity off, no tracers, and fluid_2d::solid_prd_bc, under
which every reference map is periodic up to the box lengths
(set_boundaries_solid, edge_boundary_conditions_solid_pre / _post,
fluid_2d.cc:784-835) and the wall force and object accelerations are off
(fluid_2d.cc:1037). The oracle is the reference's own fluid_2d
(oracle/_ref, ref_pulses_create with obj_full and solid_prd_bc).

- stages: the reference state after 10 steps is copied into the GPU
  simulation, one step function runs on each, every field on the whole
  ghosted grid is compared (1e-11 relative for the explicit stages, 1e-9 for
  the projections);
- whole steps from the copied initial state: u, v, p to 1e-6 of their
  maximum, X, Y to 1e-8;
- the GPU's own initialisation: X, Y (ghosts included) identical to the
  reference's, status 0 everywhere and the level set at the reference's far
  value;
- the flag is refused on a domain that is not doubly periodic and after
  initialize.
"""
import numpy as np
import pytest

from conftest import oracle_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not oracle_available(), reason="oracle/_ref not built")]

FIELDS = "u v p rho ux uy vx vy ud vd ul vl ur vr uu vu c0 c1 c2 c3 s11 s12 s21 s22".split()
SFIELDS = "X Y nX nY Xx Xy Yx Yy Xd Yd Xl Yl Xr Yr Xu Yu".split()
PAD = (0.8, 0.4, 0.8)  # ftest's padding factors (ftest.cc:94-96)
FULL = [("full", (), 3.0, 1.0)]  # ftest's full: G 3, rho_s 1


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


def _pair(m, visc=1e-3):
    from incrmt_b200 import capi
    from oracle import refsim
    r = refsim.RefSim(m, ntrace=0, objects=FULL, visc=visc, pulses=PAD)
    g = capi.Simulation(m, m, visc=visc, ntrace=0, x_prd=True, y_prd=True, pulses=True)
    g.add_full(FULL[0][2], FULL[0][3])
    g.set_solid_prd_bc(True)
    dt_reg = g.initialize(*PAD)
    assert abs(dt_reg - r.scalars()["dt_reg"]) <= 1e-15 * dt_reg
    dt, _ = refsim.frame_dt(r.scalars()["dt_reg"])
    return r, g, dt


def _copy(r, g):
    for f in FIELDS:
        g.set(f, r.get(f))
    for f in SFIELDS + ["phi", "status"]:
        g.set(f, r.get(f, 0), 0)
    g.set_mg(0, r.mg(0))
    g.set_mg(1, r.mg(1))
    g.time = r.scalars()["time"]


@pytest.fixture(scope="module")
def evolved(gpu):
    r, g, dt = _pair(48)
    r.step(dt, 10)
    yield r, g, dt
    r.close()
    g.close()


STAGES = [
    ("normal_derivatives_velocity", ["normal_derivatives_velocity", "normal_derivatives_refmap"], 1e-11),
    ("godunov_tang", ["godunov_tang", "edge_boundary_conditions"], 1e-11),
    ("half_time_edge_velocities", ["half_time_edge_velocities", "half_time_edge_refmap"], 1e-11),
    ("godunov", ["godunov", "edge_boundary_conditions"], 1e-11),
    ("mac_projection", ["mac_projection"], 1e-9),
    ("update_reference_map", ["update_reference_map"], 1e-11),
    ("pin", ["pin"], 1e-11),
    ("set_boundaries", ["set_boundaries"], 1e-11),
    ("compute_stress", ["compute_stress"], 1e-11),
    ("compute_ustar", ["compute_ustar"], 1e-11),
    ("finite_element_projection", ["finite_element_projection", "copy_pressure"], 1e-9),
    ("update_velocity", ["update_velocity"], 1e-11),
    ("set_rho", ["set_rho"], 1e-11),
    ("step_forward", ["step_forward"], 1e-9),
]


@pytest.mark.parametrize("stage,ref_stages,tol", STAGES, ids=[s[0] for s in STAGES])
def test_stage_matches_reference(evolved, stage, ref_stages, tol):
    r, g, dt = evolved
    _copy(r, g)
    for s in ref_stages:
        r.stage(s, dt)
    g.stage(stage, dt)
    errs = {f: _rel(g.get(f), r.get(f)) for f in FIELDS}
    errs.update({"obj_" + f: _rel(g.get(f, 0), r.get(f, 0)) for f in SFIELDS + ["phi"]})
    bad = {f: e for f, e in errs.items() if e > tol}
    assert not bad, bad
    assert np.array_equal(g.get("status", 0), r.get("status", 0))


def test_initial_state(gpu):
    r, g, dt = _pair(32)
    for f in ["X", "Y"]:
        assert np.array_equal(g.get(f, 0), r.get(f, 0)), f
    # status 0 everywhere, and levelset::clean's far value below the band
    assert np.all(g.get("status", 0) == 0)
    assert np.array_equal(g.get("phi", 0), r.get("phi", 0))
    for f in ["u", "v"]:
        e = _rel(g.get(f)[2:-2, 2:-2], r.get(f)[2:-2, 2:-2])
        assert e <= 1e-13, (f, e)
    r.close()
    g.close()


def test_steps_from_initial_state(gpu):
    r, g, dt = _pair(48)
    _copy(r, g)
    r.step(dt, 20)
    g.step(dt, 20)
    for f in ["u", "v", "p"]:
        e = _rel(g.get(f)[2:-2, 2:-2], r.get(f)[2:-2, 2:-2])
        assert e <= 1e-6, (f, e)
    for f in ["X", "Y"]:
        e = _rel(g.get(f, 0), r.get(f, 0))
        assert e <= 1e-8, (f, e)
    r.close()
    g.close()


def test_solid_prd_bc_refused(gpu):
    from incrmt_b200 import capi
    g = capi.Simulation(32, 32, ntrace=0)
    g.add_full(3.0, 1.0)
    with pytest.raises(capi.IncrmtError):
        g.set_solid_prd_bc(True)
    g.close()
    g = capi.Simulation(32, 32, ntrace=0, x_prd=True, y_prd=True, pulses=True)
    g.add_full(3.0, 1.0)
    g.set_solid_prd_bc(True)
    g.initialize(*PAD)
    with pytest.raises(capi.IncrmtError):
        g.set_solid_prd_bc(False)
    g.close()
