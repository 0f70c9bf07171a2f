"""GPU parity with several solids falling under gravity in a walled 64 x 96
box, in two scenes:
  - "circles_rod": two circles close enough for the collision stress
    (fluid_2d::collision_stress, fluid_2d.cc:541-598) and a rounded rod
    (obj_rounded_rod, object.hh:218-241);
  - "ellipses": the sediment workload's bodies, two rotated ellipses and a
    circle. The reference has no ellipse; the oracle's is the harness-side
    obj_ellipse (oracle/harness/ref_capi.cc), a subclass of the reference's
    obj_standard with the GPU ellipse's level set and obj_circle's gravity,
    compiled against the unmodified reference.
The oracle is the reference's own fluid_2d with these objects (oracle/_ref,
ref_multi_create). Same protocol and tolerances as the single-solid stage
tests: the evolved reference state is copied into the GPU simulation, one
step function runs on each, and every field of every object is compared.
"""
import numpy as np
import pytest

from conftest import oracle_available

pytestmark = pytest.mark.gpu

FIELDS = "u v p rho ux uy vx vy ud vd ul vl ur vr uu vu c0 c1 c2 c3 s11 s12 s21 s22".split()
SFIELDS = "X Y nX nY Xx Xy Yx Yy Xd Yd Xl Yl Xr Yr Xu Yu".split()
GEOM = (-1.0, 1.0, -1.5, 1.5)
M, N = 64, 96
# (kind, params, G, rhos)
SCENES = {
    # the circles' transition zones (eps = 2.5 dx) overlap
    "circles_rod": [
        ("circle", (0.0, 0.3, 0.2, 0.0, 0.0, 0.0, 0.5), 10.0, 2.0),
        ("circle", (0.0, -0.12, 0.2, 0.0, 0.0, 0.0, 0.6), 10.0, 2.5),
        ("rod", (0.55, 0.0, 0.08, 0.25, 0.3), 10.0, 1.5),
    ],
    # ellipse params (cx, cy, a, b, theta, grav); gravity (rho_s - 1)/rho_s
    "ellipses": [
        ("ellipse", (-0.35, 0.45, 0.25, 0.12, 0.4, 0.5), 10.0, 2.0),
        ("ellipse", (0.3, -0.35, 0.2, 0.09, -0.9, 0.6), 10.0, 2.5),
        ("circle", (0.35, 0.75, 0.12, 0.0, 0.0, 0.0, 1.0 / 3.0), 10.0, 1.5),
    ],
}

needs_oracle = pytest.mark.skipif(not oracle_available(), reason="oracle/_ref not built")


@pytest.fixture(scope="module", params=sorted(SCENES))
def scene(request):
    return request.param


def _gpu_sim(objects, ntrace=16):
    from incrmt_b200 import capi
    g = capi.Simulation(M, N, ax=GEOM[0], bx=GEOM[1], ay=GEOM[2], by=GEOM[3], ntrace=ntrace)
    for kind, p, G, rhos in objects:
        if kind == "circle":
            cx, cy, cr, uu, vv, om, grav = p
            g.add_circle(cx, cy, cr, G, rhos, grav=grav, uu=uu, vv=vv, omega=om)
        elif kind == "ellipse":
            cx, cy, a, b, th, grav = p
            g.add_ellipse(cx, cy, a, b, th, G, rhos, grav=grav)
        else:
            cx, cy, cr, cl, grav = p
            g.add_rounded_rod(cx, cy, cr, cl, G, rhos, grav=grav)
    return g


def _pair(objects, ntrace=16):
    from oracle import refsim
    r = refsim.RefSim(M, ntrace=ntrace, n=N, objects=objects, geom=GEOM)
    g = _gpu_sim(objects, ntrace)
    dt_reg = g.initialize()
    assert abs(dt_reg - r.scalars()["dt_reg"]) <= 1e-15 * dt_reg
    g.set_tracers(r.tracers()[:, :2])
    dt, _ = refsim.frame_dt(r.scalars()["dt_reg"])
    return r, g, dt


def _copy(r, g):
    for f in FIELDS:
        g.set(f, r.get(f))
    for k in range(g.objects):
        for f in SFIELDS + ["phi", "status"]:
            g.set(f, r.get(f, k), k)
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
def evolved(gpu, scene):
    if not oracle_available():
        pytest.skip("oracle/_ref not built")
    r, g, dt = _pair(SCENES[scene])
    r.step(dt, 30)
    yield r, g, dt
    r.close()
    g.close()


# The stages of one step in the order of fluid_2d::step_forward
# (fluid_2d.cc:298-369): the module's oracle advances through them, so each
# stage starts from the state the previous ones left, as in a real step (the
# MAC projection's source is only compatible with the walls once the edge
# values have been through the second Godunov pass).
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
    errs = {f: _rel(g.get(f), r.get(f)) for f in FIELDS}
    for k in range(g.objects):
        for f in SFIELDS + ["phi"]:
            errs[f"{f}[{k}]"] = _rel(g.get(f, k), r.get(f, k))
    bad = {f: e for f, e in errs.items() if e > tol}
    assert not bad, bad
    for k in range(g.objects):
        assert np.array_equal(g.get("status", k), r.get("status", k)), k


def test_collision_stress_active(evolved, scene):
    """The first scene exercises the collision term: the two circles'
    transition zones overlap somewhere on the grid."""
    if scene != "circles_rod":
        pytest.skip("the collision scene only")
    r, _, _ = evolved
    eps = r.scalars()["eps"]
    p0, p1 = r.get("phi", 0), r.get("phi", 1)
    assert np.any((p0 < eps) & (p1 < eps))


@needs_oracle
def test_initial_band(gpu, scene):
    """The bands built at initialisation agree to a fraction of dx: where the
    second-order march is not causal (a point accepted below an already
    accepted neighbour) or meets exactly tied values (grid-aligned circles),
    the reference's heap order and the fixed point differ. Measured: 0.03 dx
    with identical statuses (circles_rod); 0.038 dx at the small circle of
    the ellipses scene, where the far/trial status of a few neighbours of
    the differing points changes with them; the first pinning of the next step
    rebuilds the band from the reference map, and the simple spin's end state
    at t = 2 pi (test_endstate_gpu.py) shows no trace of such differences."""
    r, g, dt = _pair(SCENES[scene])
    dx = 2.0 / M
    tol = {"circles_rod": 0.03, "ellipses": 0.05}[scene]
    for k in range(g.objects):
        pg, pr = g.get("phi", k), r.get("phi", k)
        assert np.abs(pg - pr).max() <= tol * dx, k
        sg, sr = g.get("status", k), r.get("status", k)
        if scene == "circles_rod":
            assert np.array_equal(sg, sr), k
            continue
        # A band-edge point whose value falls below the cap in one solution
        # only is accepted there (status 5 / 2) and its far neighbours become
        # trial (6 / 1): the only status change allowed where the values agree
        # is far <-> trial, next to a point whose value differs.
        differ = np.abs(pg - pr) > 1e-12 * dx
        near = differ.copy()
        near[1:, :] |= differ[:-1, :]
        near[:-1, :] |= differ[1:, :]
        near[:, 1:] |= differ[:, :-1]
        near[:, :-1] |= differ[:, 1:]
        moved = (sg != sr) & ~differ
        pair = np.minimum(sg, sr) * 8 + np.maximum(sg, sr)
        assert np.all(near[moved]), (k, int(moved.sum()), int((moved & ~near).sum()))
        assert np.all(np.isin(pair[moved], [0 * 8 + 1, 6 * 8 + 7])), (k, np.unique(pair[moved]))
    r.close()
    g.close()


@needs_oracle
def test_steps_from_initial_state(gpu, scene):
    """25 whole steps from the reference's initial state (copied, so the
    initial-band difference above is excluded)."""
    r, g, dt = _pair(SCENES[scene])
    _copy(r, g)
    r.step(dt, 25)
    g.step(dt, 25)
    for f, tol in [("u", 1e-6), ("v", 1e-6), ("p", 1e-6)]:
        e = _rel(g.get(f)[2:-2, 2:-2], r.get(f)[2:-2, 2:-2])
        assert e <= tol, (f, e)
    for k in range(g.objects):
        for f in ["X", "Y", "phi"]:
            e = _rel(g.get(f, k)[2:-2, 2:-2], r.get(f, k)[2:-2, 2:-2])
            assert e <= 1e-8, (f, k, e)
    assert np.abs(g.tracers()[:, :2] - r.tracers()[:, :2]).max() <= 1e-9
    r.close()
    g.close()


def test_ellipse_object_runs(gpu):
    """The ellipse (no reference counterpart) initialises to a signed distance
    whose zero contour is the ellipse, and steps without error."""
    from incrmt_b200 import capi
    from oracle import refsim
    g = capi.Simulation(M, N, ax=GEOM[0], bx=GEOM[1], ay=GEOM[2], by=GEOM[3], ntrace=0)
    a, b, th = 0.3, 0.15, 0.4
    g.add_ellipse(0.0, 0.0, a, b, th, 10.0, 2.0, grav=0.5)
    dt, _ = refsim.frame_dt(g.initialize())
    phi = g.get("phi")[2:-2, 2:-2]
    dx = 2.0 / M
    x = GEOM[0] + (np.arange(M) + 0.5) * dx
    y = GEOM[2] + (np.arange(N) + 0.5) * (3.0 / N)
    X, Y = np.meshgrid(x, y)
    xb, yb = np.cos(th) * X + np.sin(th) * Y, -np.sin(th) * X + np.cos(th) * Y
    inside = (xb / a) ** 2 + (yb / b) ** 2 < 1
    band = (np.abs(phi) > 0.25 * dx) & (np.abs(phi) < 2 * dx)
    assert band.sum() > 50
    assert np.all((phi[band] < 0) == inside[band])
    g.step(dt, 5)
    assert np.isfinite(g.get("u")).all()
    g.close()
