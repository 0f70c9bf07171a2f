"""ctypes binding of libincrmt_gpu.so (include/incrmt.h).

Mirrors the reference's multigrid-system interface: an MGSolver stands for
an mgs_mac_varying_rho / mgs_fem_varying_rho object (mgs_mac.hh:64-102,
mgs_fem.hh:86-136). set_density plays fluid_2d::set_edge_irho /
set_corner_irho followed by tgmg::setup, and solve plays
mgs_*::solve_internal's V-cycle loop, returning the V-cycle count. Errors
raise IncrmtError carrying the library's status code and message, where the
reference would print and exit(1) (mgs_mac.cc:31-34).
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(HERE, "libincrmt_gpu.so")

OK = 0
ERR_NOCONV = -1
ERR_NONFINITE = -2
ERR_NEWTON = -3
ERR_EXTRAP_SINGULAR = -4
ERR_OOM = -5
ERR_BADARG = -6
ERR_CUDA = -7

SYS_MAC = 0
SYS_FEM = 1
PREC_FP64 = 0
PREC_MIXED = 1


class IncrmtError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"incrmt status {code}: {msg}")
        self.code = code


class MGOpts(ctypes.Structure):
    _fields_ = [("rel_tol", ctypes.c_double), ("max_vcycles", ctypes.c_int),
                ("precision", ctypes.c_int)]


class MGStats(ctypes.Structure):
    _fields_ = [("vcycles", ctypes.c_int), ("rel_res", ctypes.c_double),
                ("device_ms", ctypes.c_double)]


_lib = None


def lib_path():
    return _LIB_PATH


def lib():
    """Loads libincrmt_gpu.so; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        raise ImportError(
            f"{_LIB_PATH} is missing: build it with `python -m incrmt_b200.build` "
            "(there is no CPU fallback)")
    L = ctypes.CDLL(_LIB_PATH)
    P = ctypes.c_void_p
    D = ctypes.c_double
    I = ctypes.c_int
    dp = ctypes.POINTER(ctypes.c_double)
    L.incrmt_last_error.restype = ctypes.c_char_p
    L.incrmt_mg_create.argtypes = [I, I, I, D, D, D, D, I, I, I, ctypes.POINTER(P)]
    L.incrmt_mg_size.argtypes = [P, ctypes.POINTER(I), ctypes.POINTER(I)]
    L.incrmt_mg_set_density.argtypes = [P, dp]
    L.incrmt_mg_set_density_device.argtypes = [P, P]
    L.incrmt_mg_solve.argtypes = [P, dp, dp, ctypes.POINTER(MGOpts), ctypes.POINTER(MGStats)]
    L.incrmt_mg_solve_device.argtypes = [P, P, P, ctypes.POINTER(MGOpts), ctypes.POINTER(MGStats)]
    L.incrmt_mg_apply.argtypes = [P, dp, dp]
    L.incrmt_mg_vcycle_device.argtypes = [P, P, P]
    L.incrmt_mg_set_profiling.argtypes = [P, I]
    L.incrmt_mg_set_tiles.argtypes = [P, I]
    L.incrmt_mg_set_coarse_refresh.argtypes = [P, I]
    L.incrmt_mg_set_krylov.argtypes = [P, I]
    L.incrmt_mg_krylov_fallbacks.argtypes = [P]
    L.incrmt_mg_krylov_fallbacks.restype = ctypes.c_longlong
    L.incrmt_mg_coarse_builds.argtypes = [P, ctypes.POINTER(ctypes.c_longlong)]
    L.incrmt_mg_coarse_builds.restype = ctypes.c_longlong
    L.incrmt_mg_mixed_fallbacks.argtypes = [P]
    L.incrmt_mg_mixed_fallbacks.restype = ctypes.c_longlong
    L.incrmt_mg_profile.argtypes = [P, ctypes.POINTER(D), ctypes.POINTER(D), ctypes.POINTER(ctypes.c_longlong)]
    L.incrmt_mg_stream.argtypes = [P]
    L.incrmt_mg_stream.restype = P
    L.incrmt_mg_levels.argtypes = [P]
    L.incrmt_mg_launches.argtypes = [P]
    L.incrmt_mg_launches.restype = ctypes.c_longlong
    L.incrmt_mg_destroy.argtypes = [P]
    L.incrmt_mg_destroy.restype = None
    L.incrmt_mg_apply_noalloc.argtypes = [I, I, I, D, D, D, D, I, P, P, P, P]
    _lib = L
    return L


def check(code):
    if code != OK:
        raise IncrmtError(code, lib().incrmt_last_error().decode())
    return code


def _dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def mg_apply_noalloc(sys, m, n, rho_ptr, z_ptr, out_ptr, ax=-1.0, bx=1.0, ay=-1.0, by=1.0,
                     zpr=False, stream=0):
    """out = A z with device pointers and no device allocation
    (incrmt_mg_apply_noalloc); returns once the work is queued on `stream`."""
    check(lib().incrmt_mg_apply_noalloc(sys, m, n, ax, bx, ay, by, int(zpr), ctypes.c_void_p(rho_ptr),
                                        ctypes.c_void_p(z_ptr), ctypes.c_void_p(out_ptr),
                                        ctypes.c_void_p(stream)))


class MGSolver:
    """A pressure system (MAC or FEM) on an m x n cell grid, solved on the GPU."""

    def __init__(self, sys, m, n, ax=-1.0, bx=1.0, ay=-1.0, by=1.0,
                 x_prd=False, y_prd=False, zpr=False):
        L = lib()
        h = ctypes.c_void_p()
        check(L.incrmt_mg_create(sys, m, n, ax, bx, ay, by, int(x_prd), int(y_prd),
                                 int(zpr), ctypes.byref(h)))
        self._h = h
        self.sys, self.m, self.n = sys, m, n
        ms, ns = ctypes.c_int(), ctypes.c_int()
        check(L.incrmt_mg_size(h, ctypes.byref(ms), ctypes.byref(ns)))
        self.m_sys, self.n_sys = ms.value, ns.value
        self.last_stats = None

    @property
    def handle(self):
        return self._h

    def stream(self):
        """The handle's cudaStream_t as an integer."""
        return lib().incrmt_mg_stream(self._h)

    def levels(self):
        return lib().incrmt_mg_levels(self._h)

    def launches(self):
        return lib().incrmt_mg_launches(self._h)

    def set_density(self, rho):
        """rho: (n+4, m+4) ghosted cell densities (fluid_2d field layout)."""
        rho = np.ascontiguousarray(rho, dtype=np.float64)
        if rho.size != (self.m + 4) * (self.n + 4):
            raise ValueError("rho must hold (m+4)*(n+4) values")
        check(lib().incrmt_mg_set_density(self._h, _dptr(rho)))

    def set_density_device(self, ptr):
        check(lib().incrmt_mg_set_density_device(self._h, ctypes.c_void_p(ptr)))

    def solve(self, b, z, rel_tol=1e-9, max_vcycles=200, precision=PREC_FP64):
        """Solves A z = b in place on host arrays; returns MGStats."""
        b = np.ascontiguousarray(b, dtype=np.float64)
        if z.dtype != np.float64 or not z.flags.c_contiguous:
            raise ValueError("z must be a C-contiguous float64 array")
        o = MGOpts(rel_tol, max_vcycles, precision)
        s = MGStats()
        check(lib().incrmt_mg_solve(self._h, _dptr(b), _dptr(z), ctypes.byref(o), ctypes.byref(s)))
        self.last_stats = s
        return s

    def solve_device(self, b_ptr, z_ptr, rel_tol=1e-9, max_vcycles=200, precision=PREC_FP64):
        o = MGOpts(rel_tol, max_vcycles, precision)
        s = MGStats()
        check(lib().incrmt_mg_solve_device(self._h, ctypes.c_void_p(b_ptr), ctypes.c_void_p(z_ptr),
                                           ctypes.byref(o), ctypes.byref(s)))
        self.last_stats = s
        return s

    def vcycle_device(self, b_ptr, z_ptr):
        check(lib().incrmt_mg_vcycle_device(self._h, ctypes.c_void_p(b_ptr), ctypes.c_void_p(z_ptr)))

    def set_profiling(self, on=True):
        check(lib().incrmt_mg_set_profiling(self._h, int(on)))

    def set_tiles(self, on=True):
        """Tile-fused smoothing (incrmt_mg_set_tiles); off runs one launch
        per colour."""
        check(lib().incrmt_mg_set_tiles(self._h, int(on)))

    def set_coarse_refresh(self, every):
        """Rebuild the Galerkin coarse levels every `every` density changes
        (incrmt_mg_set_coarse_refresh; 1 rebuilds on every change)."""
        check(lib().incrmt_mg_set_coarse_refresh(self._h, int(every)))

    def set_krylov(self, on=True):
        """Flexible conjugate gradients with the V-cycle as preconditioner
        (incrmt_mg_set_krylov); off runs plain V-cycles."""
        check(lib().incrmt_mg_set_krylov(self._h, int(on)))

    def krylov_fallbacks(self):
        """Solves whose flexible CG handed over to plain FP64 V-cycles."""
        return int(lib().incrmt_mg_krylov_fallbacks(self._h))

    def mixed_fallbacks(self):
        """Mixed-precision solves that finished with FP64 V-cycles."""
        return int(lib().incrmt_mg_mixed_fallbacks(self._h))

    def coarse_builds(self):
        """(hierarchy rebuilds, solves repeated after a rebuild of lagged
        coarse levels) since creation."""
        r = ctypes.c_longlong()
        b = lib().incrmt_mg_coarse_builds(self._h, ctypes.byref(r))
        return int(b), int(r.value)

    def profile(self):
        """(device ms, algorithmic bytes, launches) of the timed fine-level sweeps."""
        ms, by, nl = ctypes.c_double(), ctypes.c_double(), ctypes.c_longlong()
        check(lib().incrmt_mg_profile(self._h, ctypes.byref(ms), ctypes.byref(by), ctypes.byref(nl)))
        return ms.value, by.value, nl.value

    def apply(self, z):
        z = np.ascontiguousarray(z, dtype=np.float64)
        out = np.empty_like(z)
        check(lib().incrmt_mg_apply(self._h, _dptr(z), _dptr(out)))
        return out

    def close(self):
        if self._h:
            lib().incrmt_mg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# Simulation handle (include/incrmt_sim.h): the fluid_2d replacement.

OBJ_SIMPLE_SPIN = 0
OBJ_CIRCLE = 1
OBJ_ROUNDED_ROD = 2
OBJ_ELLIPSE = 3
OBJ_FLAG = 4
OBJ_SQUARE = 5
OBJ_SEVEN_POINT = 6
OBJ_FLAPPER = 7
OBJ_PISTON = 8
OBJ_CIRCLE_TRACK = 9
OBJ_FULL = 10
OBJ_TRIANGLE = 11
OBJ_LAMPREY = 12
OBJ_HOOP = 13
FIELD_PHI = 200
FIELD_STATUS = 201
FIELDS = {n: k for k, n in enumerate(
    "u v p rho ux uy vx vy ud vd ul vl ur vr uu vu c0 c1 c2 c3 s11 s12 s21 s22".split())}
SFIELDS = {n: 100 + k for k, n in enumerate(
    "X Y nX nY Xx Xy Yx Yy Xd Yd Xl Yl Xr Yr Xu Yu".split())}
STAGES = {n: k for k, n in enumerate([
    "tracers1", "normal_derivatives_velocity", "normal_derivatives_refmap",
    "godunov_tang", "edge_boundary_conditions", "tangential_derivatives",
    "half_time_edge_velocities", "half_time_edge_refmap", "godunov",
    "mac_projection", "update_reference_map", "pin", "set_boundaries",
    "compute_stress", "compute_ustar", "finite_element_projection",
    "copy_pressure", "update_velocity", "tracers2", "set_rho", "step_forward",
    "build_band", "extrapolate"])}


class Grid(ctypes.Structure):
    _fields_ = [("m", ctypes.c_int), ("n", ctypes.c_int), ("ax", ctypes.c_double),
                ("bx", ctypes.c_double), ("ay", ctypes.c_double), ("by", ctypes.c_double),
                ("x_prd", ctypes.c_int), ("y_prd", ctypes.c_int)]


class Phys(ctypes.Structure):
    _fields_ = [("visc", ctypes.c_double), ("rhof", ctypes.c_double), ("tw", ctypes.c_double),
                ("pinw", ctypes.c_double), ("w_scale", ctypes.c_double), ("w_force", ctypes.c_double),
                ("ntrace", ctypes.c_int), ("zpr", ctypes.c_int), ("precision", ctypes.c_int),
                ("mg_rel_tol", ctypes.c_double), ("horiz_flow", ctypes.c_int), ("flow_u", ctypes.c_double),
                ("pulses", ctypes.c_int)]


def _params(*p):
    """The object parameter array of incrmt_object_desc (12 doubles)."""
    return (ctypes.c_double * 12)(*p)


class ObjectDesc(ctypes.Structure):
    _fields_ = [("type", ctypes.c_int), ("G", ctypes.c_double), ("rhos", ctypes.c_double),
                ("ev_trans_mult", ctypes.c_double), ("set_velocity", ctypes.c_int),
                ("params", ctypes.c_double * 12)]


class SimStats(ctypes.Structure):
    _fields_ = [("steps", ctypes.c_longlong), ("vcycles_mac", ctypes.c_longlong),
                ("vcycles_fem", ctypes.c_longlong), ("solves_mac", ctypes.c_longlong),
                ("solves_fem", ctypes.c_longlong), ("march_sweeps", ctypes.c_longlong),
                ("extrap_sweeps", ctypes.c_longlong), ("launches", ctypes.c_longlong),
                ("dt_reg", ctypes.c_double), ("time", ctypes.c_double),
                ("march_monotone", ctypes.c_longlong), ("window_points", ctypes.c_longlong),
                ("coarse_builds", ctypes.c_longlong), ("coarse_retries", ctypes.c_longlong),
                ("mixed_fallbacks", ctypes.c_longlong), ("krylov_fallbacks", ctypes.c_longlong)]


def _sim_sigs(L):
    P, I, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    dp = ctypes.POINTER(ctypes.c_double)
    L.incrmt_create.argtypes = [ctypes.POINTER(Grid), ctypes.POINTER(Phys), ctypes.POINTER(P)]
    L.incrmt_add_object.argtypes = [P, ctypes.POINTER(ObjectDesc)]
    L.incrmt_initialize.argtypes = [P, D, D, D, dp]
    L.incrmt_set_tracers.argtypes = [P, dp]
    L.incrmt_step.argtypes = [P, D]
    L.incrmt_steps.argtypes = [P, D, I]
    L.incrmt_stage.argtypes = [P, I, D]
    L.incrmt_get_field.argtypes = [P, I, I, dp]
    L.incrmt_set_field.argtypes = [P, I, I, dp]
    L.incrmt_get_mg.argtypes = [P, I, dp]
    L.incrmt_set_mg.argtypes = [P, I, dp]
    L.incrmt_get_time.argtypes = [P, dp]
    L.incrmt_set_time.argtypes = [P, D]
    L.incrmt_get_tracers.argtypes = [P, dp]
    L.incrmt_get_object_tracers.argtypes = [P, dp, ctypes.POINTER(I)]
    L.incrmt_track_records.argtypes = [P, dp, I, ctypes.POINTER(I), I]
    L.incrmt_record_track.argtypes = [P]
    L.incrmt_get_stats.argtypes = [P, ctypes.POINTER(SimStats)]
    L.incrmt_sim_set_profiling.argtypes = [P, I]
    L.incrmt_sim_set_windows.argtypes = [P, I]
    L.incrmt_set_solid_prd_bc.argtypes = [P, I]
    L.incrmt_sim_set_coarse_refresh.argtypes = [P, I]
    L.incrmt_sim_set_krylov.argtypes = [P, I]
    L.incrmt_sim_set_guess.argtypes = [P, I]
    L.incrmt_set_object_tracers.argtypes = [P, dp, I, I]
    L.incrmt_l_comparison.argtypes = [P, P, dp]
    L.incrmt_sim_profile.argtypes = [P, dp]
    L.incrmt_sim_mg_profile.argtypes = [P, I, dp, dp, ctypes.POINTER(ctypes.c_longlong)]
    L.incrmt_solid_bound.argtypes = [P, ctypes.POINTER(I)]
    L.incrmt_frame.argtypes = [P, I, ctypes.POINTER(I), ctypes.POINTER(ctypes.c_float)]
    L.incrmt_sim_stream.argtypes = [P]
    L.incrmt_sim_stream.restype = P
    L.incrmt_destroy.argtypes = [P]
    L.incrmt_destroy.restype = None


class Simulation:
    """A fluid_2d on the GPU (fluid_2d.hh:131-177) through the C ABI."""

    def __init__(self, m, n, ax=-1.0, bx=1.0, ay=-1.0, by=1.0, visc=1e-2, rhof=1.0, tw=2.5,
                 pinw=2.5, ntrace=512, zpr=False, precision=PREC_FP64, rel_tol=1e-9, y_prd=False,
                 horiz_flow=None, x_prd=False, pulses=False):
        """horiz_flow=U selects sim_horiz_flow: inflow of speed U at the left
        edge, zero pressure at the right, fluid starting at (U, 0).
        pulses=True with x_prd=y_prd=True on [-1,1]^2 is conv_test's
        sim_velocity_pulses."""
        L = lib()
        if not hasattr(L, "_sim_ready"):
            _sim_sigs(L)
            L._sim_ready = True
        g = Grid(m, n, ax, bx, ay, by, int(x_prd), int(y_prd))
        p = Phys(visc, rhof, tw, pinw, 0.0, 0.0, ntrace, int(zpr), precision, rel_tol,
                 int(horiz_flow is not None), float(horiz_flow or 0.0), int(pulses))
        h = ctypes.c_void_p()
        check(L.incrmt_create(ctypes.byref(g), ctypes.byref(p), ctypes.byref(h)))
        self._h = h
        self.m, self.n, self.ml, self.nl, self.ntrace = m, n, m + 4, n + 4, ntrace
        self.dt_reg = None
        self.objects = 0

    def _add(self, d):
        check(lib().incrmt_add_object(self._h, ctypes.byref(d)))
        self.objects += 1

    def add_simple_spin(self, r_scale=0.8, a1=0.5, a2=0.125, piv_r=0.2, th_max=np.pi, omega=1.0,
                        G=48.0, rhos=3.0, ev_trans_mult=1.0):
        d = ObjectDesc(OBJ_SIMPLE_SPIN, G, rhos, ev_trans_mult, 1,
                       _params(r_scale, a1, a2, piv_r, th_max, omega, 0, 0))
        self._add(d)

    def add_circle(self, cx, cy, cr, G, rhos, grav=0.0, uu=0.0, vv=0.0, omega=0.0, ev_trans_mult=1.0,
                   set_velocity=True):
        """set_velocity is mat_const::set_velocity: whether the solid's own
        velocity replaces the scenario's fluid velocity at initialisation."""
        d = ObjectDesc(OBJ_CIRCLE, G, rhos, ev_trans_mult, int(set_velocity),
                       _params(cx, cy, cr, uu, vv, omega, grav, 0))
        self._add(d)

    def add_square(self, cx, cy, cr, G, rhos, grav=0.0, uu=0.0, vv=0.0, omega=0.0, ev_trans_mult=1.0,
                   set_velocity=True):
        d = ObjectDesc(OBJ_SQUARE, G, rhos, ev_trans_mult, int(set_velocity),
                       _params(cx, cy, cr, uu, vv, omega, grav, 0))
        self._add(d)

    def add_seven_point(self, cx, cy, cr, piv_r, th_max, omega, G, rhos, ev_trans_mult=1.0, set_velocity=True):
        """obj_seven_point: a seven-pointed star spun by an anchor."""
        self._add(ObjectDesc(OBJ_SEVEN_POINT, G, rhos, ev_trans_mult, int(set_velocity),
                             _params(cx, cy, cr, piv_r, th_max, omega)))

    def add_flapper(self, cx, cy, cr, cl, ar, al, theta, m_stretch, T, G, rhos, ev_trans_mult=1.0,
                    set_velocity=True):
        """obj_flapper: a rod swimming by contracting its actuated core."""
        self._add(ObjectDesc(OBJ_FLAPPER, G, rhos, ev_trans_mult, int(set_velocity),
                             _params(cx, cy, cr, cl, ar, al, theta, m_stretch, T)))

    def add_piston(self, lx, ly, cx, y_start, y_end, duration, anch_r, G, rhos, ev_trans_mult=1.0,
                   set_velocity=True):
        """obj_piston: a block dragged by a moving anchor, tracking one point."""
        self._add(ObjectDesc(OBJ_PISTON, G, rhos, ev_trans_mult, int(set_velocity),
                             _params(lx, ly, cx, y_start, y_end, duration, anch_r)))

    def add_circle_track(self, cx, cy, cr, uu, vv, omega, G, rhos, ev_trans_mult=1.0, set_velocity=True):
        """obj_circle_track: a moving circle tracking two points."""
        self._add(ObjectDesc(OBJ_CIRCLE_TRACK, G, rhos, ev_trans_mult, int(set_velocity),
                             _params(cx, cy, cr, uu, vv, omega)))

    def add_triangle(self, cx, cy, cr, theta, G, rhos, grav=0.0, ev_trans_mult=1.0, set_velocity=True):
        """obj_triangle: an equilateral triangle under gravity."""
        self._add(ObjectDesc(OBJ_TRIANGLE, G, rhos, ev_trans_mult, int(set_velocity),
                             _params(cx, cy, cr, theta, grav)))

    def add_lamprey(self, cx, cy, theta, le, dis, w1, w2, T, mlam, G, rhos, ev_trans_mult=1.0,
                    set_velocity=True):
        """obj_lamprey: a swimmer actuated by a travelling contraction wave."""
        self._add(ObjectDesc(OBJ_LAMPREY, G, rhos, ev_trans_mult, int(set_velocity),
                             _params(cx, cy, theta, le, dis, w1, w2, T, mlam)))

    def add_hoop(self, r_in, r_out, G, rhos, grav=0.0, ev_trans_mult=1.0, set_velocity=True):
        """obj_hoop: a ring about the origin."""
        self._add(ObjectDesc(OBJ_HOOP, G, rhos, ev_trans_mult, int(set_velocity), _params(r_in, r_out, grav)))

    def add_full(self, G, rhos, ev_trans_mult=1.0, set_velocity=False):
        """obj_full: a solid filling the whole domain (with set_solid_prd_bc)."""
        self._add(ObjectDesc(OBJ_FULL, G, rhos, ev_trans_mult, int(set_velocity), _params()))

    def set_solid_prd_bc(self, on=True):
        """fluid_2d::solid_prd_bc: reference maps periodic up to the box
        lengths, no wall force; doubly periodic domains, before initialize."""
        check(lib().incrmt_set_solid_prd_bc(self._h, int(on)))

    def add_rounded_rod(self, cx, cy, cr, cl, G, rhos, grav=0.0, ev_trans_mult=1.0):
        d = ObjectDesc(OBJ_ROUNDED_ROD, G, rhos, ev_trans_mult, 1,
                       _params(cx, cy, cr, cl, grav, 0, 0, 0))
        self._add(d)

    def add_ellipse(self, cx, cy, a, b, theta, G, rhos, grav=0.0, ev_trans_mult=1.0):
        d = ObjectDesc(OBJ_ELLIPSE, G, rhos, ev_trans_mult, 1,
                       _params(cx, cy, a, b, theta, grav, 0, 0))
        self._add(d)

    def add_flag(self, cx, cy, flag_l, flag_w, flag_a, G, rhos, perturb_v=0.0, ntrace=17, ev_trans_mult=1.0):
        d = ObjectDesc(OBJ_FLAG, G, rhos, ev_trans_mult, 1,
                       _params(cx, cy, flag_l, flag_w, flag_a, perturb_v, ntrace, 0))
        self._add(d)

    def initialize(self, ev_mult=0.8, dt_pad=0.4, dt_ev_pad=0.8):
        dt = ctypes.c_double()
        check(lib().incrmt_initialize(self._h, ev_mult, dt_pad, dt_ev_pad, ctypes.byref(dt)))
        self.dt_reg = dt.value
        return self.dt_reg

    def set_tracers(self, xy):
        xy = np.ascontiguousarray(xy, dtype=np.float64).ravel()
        check(lib().incrmt_set_tracers(self._h, _dptr(xy)))

    def step(self, dt, steps=1):
        check(lib().incrmt_steps(self._h, dt, steps))

    def stage(self, name, dt=0.0):
        check(lib().incrmt_stage(self._h, STAGES[name], dt))

    def _fid(self, name):
        if isinstance(name, int):
            return name
        return FIELDS.get(name, SFIELDS.get(name, {"phi": FIELD_PHI, "status": FIELD_STATUS}.get(name)))

    def get(self, name, k=0, out=None):
        """A field on the ghosted grid (incrmt_get_field). `out`, if given,
        is a C-contiguous float64 array of nl x ml elements to fill (e.g. a
        view of pinned host memory, which the copy then reaches at full
        PCIe bandwidth)."""
        if out is None:
            out = np.empty(self.ml * self.nl)
        elif out.dtype != np.float64 or out.size != self.ml * self.nl or not out.flags["C_CONTIGUOUS"]:
            raise ValueError("out must be a contiguous float64 array of nl x ml elements")
        check(lib().incrmt_get_field(self._h, self._fid(name), k, _dptr(out)))
        return out.reshape(self.nl, self.ml)

    def set(self, name, arr, k=0):
        a = np.ascontiguousarray(arr, dtype=np.float64).ravel()
        check(lib().incrmt_set_field(self._h, self._fid(name), k, _dptr(a)))

    def get_mg(self, which):
        n = self.m * self.n if which in (0, 2) else (self.m + 1) * (self.n + 1)
        out = np.empty(n)
        check(lib().incrmt_get_mg(self._h, which, _dptr(out)))
        return out

    def set_mg(self, which, arr):
        a = np.ascontiguousarray(arr, dtype=np.float64).ravel()
        check(lib().incrmt_set_mg(self._h, which, _dptr(a)))

    @property
    def time(self):
        t = ctypes.c_double()
        check(lib().incrmt_get_time(self._h, ctypes.byref(t)))
        return t.value

    @time.setter
    def time(self, t):
        check(lib().incrmt_set_time(self._h, t))

    def tracers(self):
        out = np.empty(4 * max(self.ntrace, 1))
        check(lib().incrmt_get_tracers(self._h, _dptr(out)))
        return out[:4 * self.ntrace].reshape(self.ntrace, 4)

    def set_object_tracers(self, recs, track_count=1):
        """Sets the tracked points (records of 6 doubles) and the counter
        of their recording (incrmt_set_object_tracers)."""
        recs = np.ascontiguousarray(recs, dtype=np.float64)
        check(lib().incrmt_set_object_tracers(self._h, _dptr(recs), recs.shape[0], int(track_count)))

    def object_tracers(self):
        c = ctypes.c_int()
        check(lib().incrmt_get_object_tracers(self._h, None, ctypes.byref(c)))
        out = np.empty(6 * max(c.value, 1))
        check(lib().incrmt_get_object_tracers(self._h, _dptr(out), ctypes.byref(c)))
        return out[:6 * c.value].reshape(c.value, 6)

    def track_records(self, clear=False):
        """Records of 1 + 4*K doubles: time, then (x, y) before and after the
        correction for each of the K object tracers."""
        rec = 1 + 4 * len(self.object_tracers())
        c = ctypes.c_int()
        check(lib().incrmt_track_records(self._h, None, 0, ctypes.byref(c), 0))
        out = np.empty(rec * max(c.value, 1))
        check(lib().incrmt_track_records(self._h, _dptr(out), c.value, ctypes.byref(c), int(clear)))
        return out[:rec * c.value].reshape(c.value, rec)

    def record_track(self):
        check(lib().incrmt_record_track(self._h))

    def stats(self):
        s = SimStats()
        check(lib().incrmt_get_stats(self._h, ctypes.byref(s)))
        return s

    PHASES = ["tracers", "advection", "mac", "refmap", "extrapolation", "pin_and_band", "stress",
              "fem", "mg_setup"]

    def set_learned(self, sys, net, factor=8, rule=0):
        """Learned warm start of the MAC (sys=SYS_MAC) or FEM (SYS_FEM)
        projection (incrmt_sim_set_learned); net=None turns it off. rule 0
        falls back to the previous solution when the guess raises the
        residual, rule 1 only when alpha <= 0."""
        self._nets = getattr(self, "_nets", {})
        self._nets[sys] = net  # keep the network alive while the simulation uses it
        check(_ulib().incrmt_sim_set_learned(self._h, sys, net.handle if net is not None else None, factor, rule))

    def learned_grid(self, sys, factor):
        H, W = ctypes.c_int(), ctypes.c_int()
        check(_ulib().incrmt_sim_learned_grid(self._h, sys, factor, ctypes.byref(H), ctypes.byref(W)))
        return H.value, W.value

    def learned_capture(self, sys, factor, in_ptr, target_ptr, cap):
        """Captures the next `cap` projections of system sys as training
        samples into device buffers (incrmt_sim_learned_capture)."""
        check(_ulib().incrmt_sim_learned_capture(self._h, sys, factor, ctypes.c_void_p(in_ptr),
                                                 ctypes.c_void_p(target_ptr), cap))

    def learned_stats(self, sys):
        st = SimLearnedStats()
        check(_ulib().incrmt_sim_get_learned_stats(self._h, sys, ctypes.byref(st)))
        return st

    def l_comparison(self, fine):
        """The 32 error norms of this simulation against a finer one
        (incrmt_l_comparison)."""
        err = np.zeros(32)
        check(lib().incrmt_l_comparison(self._h, fine._h, _dptr(err)))
        return err

    def set_windows(self, on=True):
        """Per-object windows of the level-set and reference-map passes
        (on by default); off runs every pass over the whole grid."""
        check(lib().incrmt_sim_set_windows(self._h, int(on)))

    def set_coarse_refresh(self, every):
        """Rebuild the projections' Galerkin coarse operators every `every`
        projections (1 = every density change)."""
        check(lib().incrmt_sim_set_coarse_refresh(self._h, int(every)))

    def set_krylov(self, on=True):
        """Flexible conjugate gradients around the V-cycle in both
        projections (incrmt_sim_set_krylov)."""
        check(lib().incrmt_sim_set_krylov(self._h, int(on)))

    def set_guess(self, mode):
        """Warm start of the projections (incrmt_sim_set_guess): 0 the
        previous solution, 1 the extrapolation 2 z(n-1) - z(n-2), 2 the
        quadratic 3 z(n-1) - 3 z(n-2) + z(n-3)."""
        check(lib().incrmt_sim_set_guess(self._h, int(mode)))

    def set_profiling(self, on=True, smoothers=False):
        """Phase timing (on) and per-launch timing of the projections'
        fine-level smoothing (smoothers; V-cycles then run without graphs)."""
        check(lib().incrmt_sim_set_profiling(self._h, (1 if on else 0) | (2 if smoothers else 0)))

    def profile(self):
        """Device ms per step phase since profiling was turned on."""
        out = np.zeros(len(self.PHASES))
        check(lib().incrmt_sim_profile(self._h, _dptr(out)))
        return dict(zip(self.PHASES, out.tolist()))

    def solid_bound(self):
        """Ghosted index box [li, ui, lj, uj] of all points with level-set
        status below 4 (obj_field::bound)."""
        b = (ctypes.c_int * 4)()
        check(lib().incrmt_solid_bound(self._h, b))
        return list(b)

    def frame(self, mode, box):
        """Output frame of field code `mode` over the ghosted box as the
        float32 gnuplot matrix fluid_2d::output writes."""
        b = (ctypes.c_int * 4)(*box)
        si, sj = box[1] - box[0], box[3] - box[2]
        out = np.empty((sj + 1, si + 1), dtype=np.float32)
        check(lib().incrmt_frame(self._h, mode, b, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
        return out

    def smoother_profile(self, which):
        """(ms, algorithmic bytes, launches) of the fine-level smoothing of
        projection `which` (SYS_MAC or SYS_FEM) since profiling was set."""
        ms, by, n = ctypes.c_double(), ctypes.c_double(), ctypes.c_longlong()
        check(lib().incrmt_sim_mg_profile(self._h, which, ctypes.byref(ms), ctypes.byref(by), ctypes.byref(n)))
        return ms.value, by.value, n.value

    def stream(self):
        return lib().incrmt_sim_stream(self._h)

    def close(self):
        if self._h:
            lib().incrmt_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# Learned initial guess (include/incrmt_unet.h).

class LearnedStats(ctypes.Structure):
    _fields_ = [("res_before", ctypes.c_double), ("res_after", ctypes.c_double), ("alpha", ctypes.c_double),
                ("used", ctypes.c_int)]


class SimLearnedStats(ctypes.Structure):
    _fields_ = [("applied", ctypes.c_longlong), ("fallback", ctypes.c_longlong), ("captured", ctypes.c_longlong),
                ("skipped", ctypes.c_longlong)]


def _unet_sigs(L):
    P, I, D, F = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_float
    fp = ctypes.POINTER(ctypes.c_float)
    L.incrmt_unet_create.argtypes = [I, I, ctypes.c_ulonglong, ctypes.POINTER(P)]
    L.incrmt_unet_num_params.argtypes = [P]
    L.incrmt_unet_num_params.restype = ctypes.c_longlong
    L.incrmt_unet_get_params.argtypes = [P, fp]
    L.incrmt_unet_set_params.argtypes = [P, fp]
    L.incrmt_unet_forward.argtypes = [P, I, I, I, P, P, P]
    L.incrmt_unet_train_step.argtypes = [P, I, I, I, P, P, P, F, fp, P]
    L.incrmt_unet_gradients.argtypes = [P, I, I, I, P, P, P, fp, fp, P]
    L.incrmt_conv_bf16.argtypes = [P, I, I, I, I, P, I, I, I, P, I, P, P]
    L.incrmt_conv_status.argtypes = []
    L.incrmt_conv_set_variant.argtypes = [I]
    L.incrmt_conv_wgrad_workspace.argtypes = [I, I, I, I, I, I]
    L.incrmt_conv_wgrad_workspace.restype = ctypes.c_longlong
    L.incrmt_conv_wgrad_bf16.argtypes = [P, P, I, I, I, I, I, I, P, P, ctypes.c_longlong, P]
    L.incrmt_unet_launches.argtypes = [P]
    L.incrmt_unet_launches.restype = ctypes.c_longlong
    L.incrmt_unet_destroy.argtypes = [P]
    L.incrmt_unet_destroy.restype = None
    L.incrmt_mg_learned_guess.argtypes = [P, P, P, P, I, ctypes.POINTER(LearnedStats)]
    L.incrmt_mg_learned_input.argtypes = [P, P, P, I, P, I, I]
    ip = ctypes.POINTER(ctypes.c_int)
    L.incrmt_sim_set_learned.argtypes = [P, I, P, I, I]
    L.incrmt_sim_learned_grid.argtypes = [P, I, I, ip, ip]
    L.incrmt_sim_learned_capture.argtypes = [P, I, I, P, P, I]
    L.incrmt_sim_get_learned_stats.argtypes = [P, I, ctypes.POINTER(SimLearnedStats)]


def _ulib():
    L = lib()
    if not hasattr(L, "_unet_ready"):
        _unet_sigs(L)
        L._unet_ready = True
    return L


def learned_grid(m, n, factor):
    """Network grid (H, W) of an m x n solve restricted by `factor`."""
    return ((n + factor - 1) // factor + 15) // 16 * 16, ((m + factor - 1) // factor + 15) // 16 * 16


class UNet:
    """The BF16 U-Net of the learned initial guess (include/incrmt_unet.h).
    Device arrays are passed as integer pointers (e.g. torch data_ptr())."""

    def __init__(self, levels=4, base=16, seed=1):
        h = ctypes.c_void_p()
        check(_ulib().incrmt_unet_create(levels, base, seed, ctypes.byref(h)))
        self._h = h
        self.levels, self.base = levels, base

    @property
    def handle(self):
        return self._h

    def num_params(self):
        return int(_ulib().incrmt_unet_num_params(self._h))

    def get_params(self):
        out = np.empty(self.num_params(), dtype=np.float32)
        check(_ulib().incrmt_unet_get_params(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
        return out

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        check(_ulib().incrmt_unet_set_params(self._h, p.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))

    def forward(self, batch, H, W, in_ptr, out_ptr, stream=0):
        check(_ulib().incrmt_unet_forward(self._h, batch, H, W, ctypes.c_void_p(in_ptr), ctypes.c_void_p(out_ptr),
                                          ctypes.c_void_p(stream)))

    def train_step(self, batch, H, W, in_ptr, target_ptr, valid_ptr, lr, stream=0):
        loss = ctypes.c_float()
        check(_ulib().incrmt_unet_train_step(self._h, batch, H, W, ctypes.c_void_p(in_ptr), ctypes.c_void_p(target_ptr),
                                             ctypes.c_void_p(valid_ptr), lr, ctypes.byref(loss), ctypes.c_void_p(stream)))
        return loss.value

    def gradients(self, batch, H, W, in_ptr, target_ptr, valid_ptr, stream=0):
        g = np.empty(self.num_params(), dtype=np.float32)
        loss = ctypes.c_float()
        check(_ulib().incrmt_unet_gradients(self._h, batch, H, W, ctypes.c_void_p(in_ptr), ctypes.c_void_p(target_ptr),
                                            ctypes.c_void_p(valid_ptr), ctypes.byref(loss),
                                            g.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), ctypes.c_void_p(stream)))
        return loss.value, g

    def launches(self):
        return int(_ulib().incrmt_unet_launches(self._h))

    def close(self):
        if getattr(self, "_h", None):
            _ulib().incrmt_unet_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def conv_bf16(x_ptr, batch, H, W, cin, wk_ptr, taps, cout, y_ptr, bias_ptr=0, relu=False, flip=False, stream=0):
    """One tensor-core convolution (incrmt_conv_bf16): NHWC BF16 activations,
    weights BF16 [tap][cout][cin]; device pointers as integers."""
    check(_ulib().incrmt_conv_bf16(ctypes.c_void_p(x_ptr), batch, H, W, cin, ctypes.c_void_p(wk_ptr), taps, cout,
                                   int(flip), ctypes.c_void_p(bias_ptr or None), int(relu), ctypes.c_void_p(y_ptr),
                                   ctypes.c_void_p(stream)))


def conv_wgrad_workspace(batch, H, W, cin, cout, taps):
    """Floats of workspace the tensor-core weight gradient needs."""
    return int(_ulib().incrmt_conv_wgrad_workspace(batch, H, W, cin, cout, taps))


def conv_wgrad_bf16(x_ptr, dy_ptr, batch, H, W, cin, cout, taps, dw_ptr, work_ptr, work_floats, stream=0):
    """dW += the weight gradient of one convolution (incrmt_conv_wgrad_bf16)."""
    check(_ulib().incrmt_conv_wgrad_bf16(ctypes.c_void_p(x_ptr), ctypes.c_void_p(dy_ptr), batch, H, W, cin, cout,
                                         taps, ctypes.c_void_p(dw_ptr), ctypes.c_void_p(work_ptr), int(work_floats),
                                         ctypes.c_void_p(stream)))


def conv_status():
    """Raises if a tensor-core convolution gave up a pipeline wait
    (incrmt_conv_status; synchronises the device)."""
    check(_ulib().incrmt_conv_status())


def conv_set_variant(variant):
    """3x3 kernel choice for the process (incrmt_conv_set_variant): 0
    automatic, 1 one tap per stage, 2 row reuse, 3 resident weights, 4 two
    128-pixel halves per CTA."""
    check(_ulib().incrmt_conv_set_variant(int(variant)))


def learned_guess(solver, net, b_ptr, z_ptr, factor=1, stats=True):
    """z += alpha d from the network (incrmt_mg_learned_guess); returns the
    LearnedStats when stats is set (that synchronises the solver's stream)."""
    st = LearnedStats() if stats else None
    check(_ulib().incrmt_mg_learned_guess(solver.handle, net.handle, ctypes.c_void_p(b_ptr), ctypes.c_void_p(z_ptr),
                                          factor, ctypes.byref(st) if st is not None else None))
    return st


def learned_input(solver, b_ptr, z_ptr, factor, in_ptr):
    """The network input of a guess from (b, z) (for training data)."""
    H, W = learned_grid(solver.m_sys, solver.n_sys, factor)
    check(_ulib().incrmt_mg_learned_input(solver.handle, ctypes.c_void_p(b_ptr), ctypes.c_void_p(z_ptr), factor,
                                          ctypes.c_void_p(in_ptr), H, W))
    return H, W
