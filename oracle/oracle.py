"""ctypes wrapper of the CPU oracle (oracle/_build/liboracle.so) -- TEST INFRASTRUCTURE ONLY.

Only tests/, the smoke check and bench.py's CPU-baseline leg import this module;
it is the checker, never the product.  Each function restates the reference
single-task arithmetic listed in oracle.h (ParisPencil.cpp, FishFry.hpp).
"""
import ctypes
import math
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None


class Mode(ctypes.Structure):
    _fields_ = [("kx", ctypes.c_int), ("ky", ctypes.c_int), ("kz", ctypes.c_int),
                ("a", ctypes.c_double), ("theta", ctypes.c_double)]


def build():
    """Compile the oracle with its Makefile (g++ -fopenmp)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        L.orc_fft1d.argtypes = [ctypes.c_int, ctypes.c_int, dp, dp]
        L.orc_solve.argtypes = [ctypes.c_int] * 3 + [dp, dp, dp, dp]
        L.orc_forward_spectrum.argtypes = [ctypes.c_int] * 3 + [dp, dp]
        for name in ("orc_init_f", "orc_phi_exact"):
            getattr(L, name).argtypes = [ctypes.c_int] * 3 + [dp, dp, ctypes.c_int, ctypes.c_void_p, dp]
            getattr(L, name).restype = None
        for name in ("orc_diff_sums", "orc_rel_norms"):
            getattr(L, name).argtypes = ([ctypes.c_int] * 3 + [dp, dp, ctypes.c_int, ctypes.c_void_p,
                                                                ctypes.c_void_p, dp])
            getattr(L, name).restype = None
        L.orc_modes_generate.argtypes = [ctypes.c_uint64, ctypes.c_int, ctypes.c_int,
                                         ctypes.POINTER(ctypes.c_int), ctypes.c_double, ctypes.c_void_p]
        L.orc_modes_generate.restype = None
        L.orc_set_threads.argtypes = [ctypes.c_int]
        L.orc_get_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _d3(v):
    return (ctypes.c_double * 3)(*[float(x) for x in v])


def set_threads(n):
    lib().orc_set_threads(int(n))


def get_threads():
    return lib().orc_get_threads()


def reference_domain(n):
    """lo, hi, xlo, dx of the harness for a single task (FishFry.hpp:109-111,133-139)."""
    dx = [2.0 * math.pi / n[a] for a in range(3)]
    lo = [-math.pi] * 3
    hi = [math.pi - dx[a] for a in range(3)]
    return lo, hi, list(lo), dx


def fft1d(x, sign=-1):
    x = np.ascontiguousarray(x, dtype=np.complex128)
    out = np.empty_like(x)
    rc = lib().orc_fft1d(x.size, sign, _dp(x.view(np.float64)), _dp(out.view(np.float64)))
    if rc:
        raise ValueError("orc_fft1d failed")
    return out


def solve(f, lo=None, hi=None):
    f = np.ascontiguousarray(f, dtype=np.float64)
    ni, nj, nk = f.shape
    if lo is None:
        lo, hi, _, _ = reference_domain((ni, nj, nk))
    phi = np.empty_like(f)
    rc = lib().orc_solve(ni, nj, nk, _d3(lo), _d3(hi), _dp(f), _dp(phi))
    if rc:
        raise ValueError("orc_solve failed")
    return phi


def forward_spectrum(f):
    f = np.ascontiguousarray(f, dtype=np.float64)
    ni, nj, nk = f.shape
    spec = np.empty((ni, nj, nk // 2 + 1), dtype=np.complex128)
    rc = lib().orc_forward_spectrum(ni, nj, nk, _dp(f), _dp(spec.view(np.float64)))
    if rc:
        raise ValueError("orc_forward_spectrum failed")
    return spec


def _modes_arg(modes):
    if modes is None or len(modes) == 0:
        return 0, None, None
    arr = (Mode * len(modes))()
    for q, m in enumerate(modes):
        arr[q] = Mode(int(m[0]), int(m[1]), int(m[2]), float(m[3]), float(m[4]))
    return len(modes), ctypes.cast(arr, ctypes.c_void_p), arr


def init_f(n, modes=None):
    _, _, xlo, dx = reference_domain(n)
    f = np.empty(tuple(n), dtype=np.float64)
    nm, p, keep = _modes_arg(modes)
    lib().orc_init_f(n[0], n[1], n[2], _d3(xlo), _d3(dx), nm, p, _dp(f))
    return f


def phi_exact(n, modes=None):
    _, _, xlo, dx = reference_domain(n)
    phi = np.empty(tuple(n), dtype=np.float64)
    nm, p, keep = _modes_arg(modes)
    lib().orc_phi_exact(n[0], n[1], n[2], _d3(xlo), _d3(dx), nm, p, _dp(phi))
    return phi


def diff_sums(phi, modes=None):
    n = phi.shape
    _, _, xlo, dx = reference_domain(n)
    phi = np.ascontiguousarray(phi, dtype=np.float64)
    out = np.zeros(3)
    nm, p, keep = _modes_arg(modes)
    lib().orc_diff_sums(n[0], n[1], n[2], _d3(xlo), _d3(dx), nm, p,
                        phi.ctypes.data_as(ctypes.c_void_p), _dp(out))
    return out


def rel_norms(phi, modes=None):
    """Relative L1, L2, Linf of phi against the analytic solution (FishFry.hpp:198)."""
    n = phi.shape
    _, _, xlo, dx = reference_domain(n)
    phi = np.ascontiguousarray(phi, dtype=np.float64)
    out = np.zeros(3)
    nm, p, keep = _modes_arg(modes)
    lib().orc_rel_norms(n[0], n[1], n[2], _d3(xlo), _d3(dx), nm, p,
                        phi.ctypes.data_as(ctypes.c_void_p), _dp(out))
    return out


def modes_generate(seed, count, kmax, kaxis, sigma=0.1):
    arr = (Mode * count)()
    ka = (ctypes.c_int * 3)(*[int(k) for k in kaxis])
    lib().orc_modes_generate(ctypes.c_uint64(seed), count, kmax, ka, float(sigma),
                             ctypes.cast(arr, ctypes.c_void_p))
    return [(m.kx, m.ky, m.kz, m.a, m.theta) for m in arr]
