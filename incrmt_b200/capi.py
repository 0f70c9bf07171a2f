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
    L.incrmt_mg_profile.argtypes = [P, ctypes.POINTER(D), ctypes.POINTER(D), ctypes.POINTER(ctypes.c_longlong)]
    L.incrmt_mg_stream.argtypes = [P]
    L.incrmt_mg_stream.restype = P
    L.incrmt_mg_levels.argtypes = [P]
    L.incrmt_mg_launches.argtypes = [P]
    L.incrmt_mg_launches.restype = ctypes.c_longlong
    L.incrmt_mg_destroy.argtypes = [P]
    L.incrmt_mg_destroy.restype = None
    _lib = L
    return L


def check(code):
    if code != OK:
        raise IncrmtError(code, lib().incrmt_last_error().decode())
    return code


def _dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


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
