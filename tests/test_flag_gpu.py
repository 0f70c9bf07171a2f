"""GPU parity for the flag scenario's machinery: a y-periodic channel with a
uniform inflow at the left edge and zero pressure at the right
(sim_horiz_flow, sim_type.hh:117-141, sim_type.cc:51-64) and a flag anchored
at its leading end (obj_flag, object.hh:471-505, object.cc:420-496) tracking
17 points along its length. 96 x 32 cells on [-1,5]x[-1,1] (the reference
driver's geometry, ftest.cc:335-378, at a test size). The oracle is the
reference's own fluid_2d with these classes (oracle/_ref, ref_multi_create).
Same protocol and tolerances as the other stage tests.
"""
import numpy as np
import pytest

from conftest import oracle_available

pytestmark = pytest.mark.gpu

FIELDS = "u v p rho ux uy vx vy ud vd ul vl ur vr uu vu c0 c1 c2 c3 s11 s12 s21 s22".split()
SFIELDS = "X Y nX nY Xx Xy Yx Yy Xd Yd Xl Yl Xr Yr Xu Yu".split()
GEOM = (-1.0, 5.0, -1.0, 1.0)
M, N = 96, 32
U = 1.0
# flag: length 1, width 0.25 (aspect ratio 4), anchor radius w/4; mass ratio 1
# (rho_s = L/w), bending rigidity 0.1 (G = 4 k_B / w^3), Re = 100 (visc = 0.01)
FLAG = ("flag", (0.0, 0.0, 1.0, 0.25, 0.0625, 0.0, 17), 4 * 0.1 / 0.25 ** 3, 4.0)

needs_oracle = pytest.mark.skipif(not oracle_available(), reason="oracle/_ref not built")


def _gpu_sim():
    from incrmt_b200 import capi
    g = capi.Simulation(M, N, ax=GEOM[0], bx=GEOM[1], ay=GEOM[2], by=GEOM[3], visc=0.01, ntrace=0,
                        y_prd=True, horiz_flow=U)
    cx, cy, L, w, a, pv, nt = FLAG[1]
    g.add_flag(cx, cy, L, w, a, FLAG[2], FLAG[3], perturb_v=pv, ntrace=nt)
    return g


def _pair():
    from oracle import refsim
    r = refsim.RefSim(M, ntrace=0, n=N, objects=[FLAG], geom=GEOM, visc=0.01, flow_u=U)
    g = _gpu_sim()
    dt_reg = g.initialize()
    assert abs(dt_reg - r.scalars()["dt_reg"]) <= 1e-15 * dt_reg
    dt, _ = refsim.frame_dt(r.scalars()["dt_reg"])
    return r, g, dt


def _copy(r, g):
    for f in FIELDS:
        g.set(f, r.get(f))
    for f in SFIELDS + ["phi", "status"]:
        g.set(f, r.get(f))
    g.set_mg(0, r.mg(0))
    g.set_mg(1, r.mg(1))
    g.time = r.scalars()["time"]


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


@pytest.fixture(scope="module")
def evolved(gpu):
    if not oracle_available():
        pytest.skip("oracle/_ref not built")
    r, g, dt = _pair()
    r.step(dt, 30)
    yield r, g, dt
    r.close()
    g.close()


STAGES = [
    ("normal_derivatives_velocity", ["normal_derivatives_velocity", "normal_derivatives_refmap"], 1e-11),
    ("godunov_tang", ["godunov_tang", "edge_boundary_conditions"], 1e-11),
    ("tangential_derivatives", ["tangential_derivatives"], 1e-11),
    ("half_time_edge_velocities", ["half_time_edge_velocities", "half_time_edge_refmap"], 1e-11),
    ("godunov", ["godunov", "edge_boundary_conditions"], 1e-11),
    ("mac_projection", ["mac_projection"], 1e-9),
    ("update_reference_map", ["update_reference_map"], 1e-11),
    ("pin", ["pin"], 1e-9),
    ("set_boundaries", ["set_boundaries"], 1e-11),
    ("compute_stress", ["compute_stress"], 1e-11),
    ("compute_ustar", ["compute_ustar"], 1e-11),
    ("finite_element_projection", ["finite_element_projection", "copy_pressure"], 1e-9),
    ("update_velocity", ["update_velocity"], 1e-11),
    ("set_rho", ["set_rho"], 1e-11),
    ("build_band", ["build_band"], 1e-9),
    ("extrapolate", ["extrapolate"], 1e-11),
    ("step_forward", ["step_forward"], 1e-9),
]


@needs_oracle
@pytest.mark.parametrize("stage,ref_stages,tol", STAGES, ids=[s[0] for s in STAGES])
def test_stage_matches_reference(evolved, stage, ref_stages, tol):
    r, g, dt = evolved
    _copy(r, g)
    for s in ref_stages:
        r.stage(s, dt)
    g.stage(stage, dt)
    errs = {f: _rel(g.get(f), r.get(f)) for f in FIELDS + SFIELDS + ["phi"]}
    bad = {f: e for f, e in errs.items() if e > tol}
    assert not bad, bad
    assert np.array_equal(g.get("status"), r.get("status"))


@needs_oracle
def test_steps_from_initial_state(gpu):
    """40 whole steps from the reference's initial state, including the
    tracked points along the flag (every 100 steps the reference records
    them; here their positions after the steps are compared)."""
    r, g, dt = _pair()
    _copy(r, g)
    r.step(dt, 40)
    g.step(dt, 40)
    for f, tol in [("u", 1e-6), ("v", 1e-6), ("p", 1e-6)]:
        e = _rel(g.get(f)[2:-2, 2:-2], r.get(f)[2:-2, 2:-2])
        assert e <= tol, (f, e)
    for f in ["X", "Y", "phi"]:
        e = _rel(g.get(f)[2:-2, 2:-2], r.get(f)[2:-2, 2:-2])
        assert e <= 1e-8, (f, e)
    a, b = g.object_tracers(), r.obj_tracers()
    assert a.shape == b.shape == (17, 6)
    assert np.abs(a[:, :2] - b[:, :2]).max() <= 1e-9
    r.close()
    g.close()


@needs_oracle
def test_initial_state(gpu):
    """Initialisation: level set (see below and the multi-solid tests),
    statuses, the flag's tracked points, and the velocity: (U, 0) in the
    fluid, blended with the solid's by its smoothed Heaviside, so that near
    the flag's rounded ends the level-set difference moves u by up to
    ~0.03 dx / eps of U."""
    r, g, dt = _pair()
    far = np.abs(r.get("phi")) > 0.2
    assert _rel(g.get("u")[far], r.get("u")[far]) <= 1e-12
    assert _rel(g.get("u")[2:-2, 2:-2], r.get("u")[2:-2, 2:-2]) <= 0.05
    # The initial flag is symmetric about y = 0 and aligned with the grid, so
    # the march meets many exactly equal values, whose acceptance order in the
    # reference's heap decides their neighbours' stencils: 0.15 dx.
    assert np.abs(g.get("phi") - r.get("phi")).max() <= 0.15 * (2.0 / N)
    assert np.array_equal(g.get("status"), r.get("status"))
    # Columns 2,3 (the stage velocity) are not set until the first step; the
    # reference leaves them uninitialised (obj_track, object.hh:314-318).
    a, b = g.object_tracers(), r.obj_tracers()
    assert np.abs(a[:, [0, 1, 4, 5]] - b[:, [0, 1, 4, 5]]).max() <= 1e-15
    r.close()
    g.close()


def test_periodic_without_outlet_rejected(gpu):
    """A y-periodic channel needs the zero-pressure outlet: walls in x with y
    periodicity alone leave singular periodic pressure systems, which the
    simulation refuses at creation."""
    from incrmt_b200 import capi
    with pytest.raises(capi.IncrmtError):
        capi.Simulation(64, 64, y_prd=True)
