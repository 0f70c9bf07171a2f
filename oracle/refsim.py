"""ctypes access to the compiled reference (oracle/_ref/libincrmt_ref.so).

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py). Field ids follow the
member order of the reference's structs: 0..23 = struct field
(fields.hh:7-49: u,v,p,rho,ux,uy,vx,vy,ud,vd,ul,vl,ur,vr,uu,vu,c0..c3,
s11,s12,s21,s22), 100..119 = struct s_field of object k (fields.hh:51-79:
X,Y,nX,nY,Xx,Xy,Yx,Yy,Xd,Yd,Xl,Yl,Xr,Yr,Xu,Yu,r0..r3), 200 = phi, 201 =
level-set status.
"""
import ctypes
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libincrmt_ref.so")
RUN = os.path.join(HERE, "_ref", "ref_run")
FTEST = os.path.join(HERE, "_ref", "ref_ftest")

FIELD = {n: k for k, n in enumerate(
    "u v p rho ux uy vx vy ud vd ul vl ur vr uu vu c0 c1 c2 c3 s11 s12 s21 s22".split())}
SFIELD = {n: 100 + k for k, n in enumerate(
    "X Y nX nY Xx Xy Yx Yy Xd Yd Xl Yl Xr Yr Xu Yu r0 r1 r2 r3".split())}
PHI, STATUS = 200, 201

STAGES = {n: k for k, n in enumerate([
    "tracers1", "normal_derivatives_velocity", "normal_derivatives_refmap",
    "godunov_tang", "edge_boundary_conditions", "tangential_derivatives",
    "half_time_edge_velocities", "half_time_edge_refmap", "godunov",
    "mac_projection", "update_reference_map", "pin", "set_boundaries",
    "compute_stress", "compute_ustar", "finite_element_projection",
    "copy_pressure", "update_velocity", "tracers2", "set_rho", "step_forward",
    "build_band", "extrapolate"])}

_lib = None


def available():
    return os.path.exists(LIB)


def build(ref_root=None):
    """Builds oracle/_ref from the reference sources (needs the reference
    tree: ref_root, else $INCRMT_REFERENCE, else the build container's
    checkout)."""
    if ref_root is None:
        ref_root = os.environ.get("INCRMT_REFERENCE", "/root/reference")
    subprocess.run(["make", "-C", HERE, f"REF={ref_root}", "-j8"], check=True,
                   stdout=subprocess.DEVNULL)


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not available():
        raise FileNotFoundError(f"{LIB} is not built (make -C oracle)")
    L = ctypes.CDLL(LIB)
    P, I, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    dp = ctypes.POINTER(ctypes.c_double)
    ip = ctypes.POINTER(ctypes.c_int)
    L.ref_sspin_create.argtypes = [I, I, ctypes.c_char_p]
    L.ref_sspin_create.restype = P
    L.ref_destroy.argtypes = [P]
    L.ref_multi_create.argtypes = [I, I, dp, I, I, D, D, I, I, ip, dp, dp, ctypes.c_char_p, D]
    L.ref_multi_create.restype = P
    L.ref_pulses_create.argtypes = [I, D, D, I, I, ip, dp, dp, D, D, D, ctypes.c_char_p, I]
    L.ref_pulses_create.restype = P
    L.ref_l_comparison.argtypes = [P, P, dp]
    L.ref_l_comparison.restype = None
    L.ref_obj_track_count.argtypes = [P, I]
    L.ref_obj_track_count.restype = I
    L.ref_dims.argtypes = [P, ip]
    L.ref_scalars.argtypes = [P, dp]
    L.ref_set_time.argtypes = [P, D]
    L.ref_get.argtypes = [P, I, I, dp]
    L.ref_set.argtypes = [P, I, I, dp]
    L.ref_band.argtypes = [P, I, ip, I]
    L.ref_get_tracers.argtypes = [P, dp]
    L.ref_set_tracers.argtypes = [P, dp]
    L.ref_get_obj_tracers.argtypes = [P, I, dp]
    L.ref_get_mg.argtypes = [P, I, dp]
    L.ref_set_mg.argtypes = [P, I, dp]
    L.ref_vcycles.argtypes = [P, I, I]
    L.ref_stage.argtypes = [P, I, D]
    L.ref_steps.argtypes = [P, I, D]
    L.ref_mg_solve.argtypes = [I, I, I, D, D, D, D, I, I, I, dp, dp, dp, dp]
    L.ref_mg_apply.argtypes = [I, I, I, D, D, D, D, I, I, I, dp, dp, dp]
    _lib = L
    return L


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def mg_solve(sys, m, n, rho, b, z0=None, ax=-1., bx=1., ay=-1., by=1.,
             x_prd=False, y_prd=False, zpr=False):
    """Reference solve (mgs_*_varying_rho + shim). Returns (z, b_used, stats)
    with stats = (vcycles, rel_res, seconds); raises if it did not converge."""
    rho = np.ascontiguousarray(rho, dtype=np.float64).ravel()
    b = np.array(b, dtype=np.float64).ravel()
    z = np.zeros_like(b) if z0 is None else np.array(z0, dtype=np.float64).ravel()
    st = np.zeros(3)
    r = lib().ref_mg_solve(sys, m, n, ax, bx, ay, by, int(x_prd), int(y_prd), int(zpr),
                           _dp(rho), _dp(b), _dp(z), _dp(st))
    if r != 0:
        raise RuntimeError("reference multigrid did not converge")
    return z, b, (int(st[0]), st[1], st[2])


def mg_apply(sys, m, n, rho, z, ax=-1., bx=1., ay=-1., by=1., x_prd=False, y_prd=False, zpr=False):
    """A z through the reference's own a_cc/mul_a callbacks."""
    rho = np.ascontiguousarray(rho, dtype=np.float64).ravel()
    z = np.ascontiguousarray(z, dtype=np.float64).ravel()
    out = np.empty_like(z)
    lib().ref_mg_apply(sys, m, n, ax, bx, ay, by, int(x_prd), int(y_prd), int(zpr),
                       _dp(rho), _dp(z), _dp(out))
    return out


# object kinds of ref_multi_create (oracle/harness/ref_capi.cc make_multi)
OBJECT_TYPES = {"circle": 1, "rod": 2, "flag": 3, "square": 5, "star": 6, "flapper": 7, "piston": 8,
                "circle_track": 9, "triangle": 11, "lamprey": 12, "hoop": 13, "ellipse": 14}


class RefSim:
    """A reference fluid_2d simulation: the simple-spin scenario, or with
    `objects` a domain of circles and rounded rods.

    objects: list of ("circle", (cx, cy, cr, uu, vv, omega, grav), G, rhos),
    ("rod", (cx, cy, cr, cl, grav), G, rhos), ("ellipse", (cx, cy, a, b, theta,
    grav), G, rhos) or ("flag", (cx, cy, flag_l, flag_w, flag_a, perturb_v,
    ntrace), G, rhos); geom = (ax, bx, ay, by);
    flow_u > 0 makes the domain sim_horiz_flow (y-periodic with inflow)."""

    def __init__(self, m, ntrace=512, workdir=None, n=None, objects=None, geom=(-1., 1., -1., 1.),
                 visc=1e-2, rhof=1.0, periodic=(False, False), flow_u=0.0, pulses=None):
        self._tmp = None
        if workdir is None:
            self._tmp = tempfile.TemporaryDirectory()
            workdir = self._tmp.name
        if pulses is not None:
            # conv_test's scenario: pulses = (ev_mult, dt_pad, dt_ev_pad);
            # a ("full", (), G, rhos) object also sets solid_prd_bc, as
            # conv_test's type 2 and ftest's "full" do.
            objects = objects or []
            k = len(objects)
            types = (ctypes.c_int * max(k, 1))(*[{"circle": 1, "square": 5, "full": 10}[o[0]] for o in objects])
            solid_prd = int(any(o[0] == "full" for o in objects))
            params = np.zeros((max(k, 1), 12))
            mats = np.zeros((max(k, 1), 2))
            for q, (kind, p, G, rhos) in enumerate(objects):
                params[q, :len(p)] = p
                mats[q] = (G, rhos)
            base = os.path.join(workdir, f"pulses_{m}").encode()
            self.h = lib().ref_pulses_create(m, visc, rhof, ntrace, k, types, _dp(params), _dp(mats),
                                             float(pulses[0]), float(pulses[1]), float(pulses[2]), base,
                                             solid_prd)
        elif objects is None:
            base = os.path.join(workdir, f"sspin_{m}").encode()
            self.h = lib().ref_sspin_create(m, ntrace, base)
        else:
            n = m if n is None else n
            k = len(objects)
            types = (ctypes.c_int * k)(*[OBJECT_TYPES[o[0]] for o in objects])
            params = np.zeros((k, 12))
            mats = np.zeros((k, 2))
            for q, (kind, p, G, rhos) in enumerate(objects):
                params[q, :len(p)] = p
                mats[q] = (G, rhos)
            g = np.array(geom, dtype=np.float64)
            base = os.path.join(workdir, f"multi_{m}").encode()
            self.h = lib().ref_multi_create(m, n, _dp(g), int(periodic[0]), int(periodic[1]), visc, rhof,
                                            ntrace, k, types, _dp(params), _dp(mats), base, float(flow_u))
        d = (ctypes.c_int * 7)()
        lib().ref_dims(self.h, d)
        self.m, self.n, self.ml, self.nl, self.n_obj, self.m_fem, self.n_fem = list(d)
        self.ntrace = ntrace

    def l_comparison(self, fine):
        """fluid_2d::l_comparison of this (coarse) simulation against `fine`:
        the 32 error norms (fluid_2d_io.cc:186-281)."""
        err = np.zeros(32)
        lib().ref_l_comparison(self.h, fine.h, _dp(err))
        return err

    def scalars(self):
        s = np.zeros(6)
        lib().ref_scalars(self.h, _dp(s))
        return dict(dt_reg=s[0], time=s[1], dx=s[2], dy=s[3], eps=s[4], K_stiff=s[5])

    def get(self, name_or_id, k=0):
        fid = name_or_id if isinstance(name_or_id, int) else \
            FIELD.get(name_or_id, SFIELD.get(name_or_id, {"phi": PHI, "status": STATUS}.get(name_or_id)))
        out = np.empty(self.ml * self.nl)
        if lib().ref_get(self.h, fid, k, _dp(out)) != 0:
            raise KeyError(name_or_id)
        return out.reshape(self.nl, self.ml)

    def set(self, name_or_id, arr, k=0):
        fid = name_or_id if isinstance(name_or_id, int) else \
            FIELD.get(name_or_id, SFIELD.get(name_or_id, {"phi": PHI, "status": STATUS}.get(name_or_id)))
        a = np.ascontiguousarray(arr, dtype=np.float64).ravel()
        if lib().ref_set(self.h, fid, k, _dp(a)) != 0:
            raise KeyError(name_or_id)

    def band(self, k=0):
        cap = self.ml * self.nl
        out = (ctypes.c_int * cap)()
        c = lib().ref_band(self.h, k, out, cap)
        return np.frombuffer(out, dtype=np.int32)[:c].copy()

    def tracers(self):
        out = np.empty(4 * self.ntrace)
        lib().ref_get_tracers(self.h, _dp(out))
        return out.reshape(self.ntrace, 4)

    def obj_tracers(self, k=0):
        out = np.empty(6 * 64)
        c = lib().ref_get_obj_tracers(self.h, k, _dp(out))
        return out[:6 * c].reshape(c, 6)

    def obj_track_count(self, k=0):
        """obj_track::count of object k: steps since its last record."""
        return lib().ref_obj_track_count(self.h, k)

    def mg(self, which):
        nv = lib().ref_get_mg(self.h, which, None)
        out = np.empty(nv)
        lib().ref_get_mg(self.h, which, _dp(out))
        return out

    def vcycles(self, which, reset=True):
        return lib().ref_vcycles(self.h, which, int(reset))

    def set_time(self, t):
        lib().ref_set_time(self.h, t)

    def stage(self, name, dt=0.0):
        if lib().ref_stage(self.h, STAGES[name], dt) != 0:
            raise KeyError(name)

    def step(self, dt, steps=1):
        lib().ref_steps(self.h, steps, dt)

    def close(self):
        if self.h:
            lib().ref_destroy(self.h)
            self.h = None
        if self._tmp is not None:
            self._tmp.cleanup()
            self._tmp = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def frame_dt(dt_reg, duration=2 * np.pi, frames=120):
    """Step size and steps per frame that fluid_2d::solve chooses
    (timestep_select, fluid_2d.hh:173-177)."""
    interval = duration / frames
    l = int(interval / dt_reg) + 1
    return interval / l, l
