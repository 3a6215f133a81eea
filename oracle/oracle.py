"""ctypes wrapper around the CPU oracle (``oracle/mt_oracle.c``).

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``__graft_entry__.smoke()``
and the ``cpu_baseline`` leg of ``bench.py`` as the checker.  The product
(``magtense_b200``) never imports it.

The C file restates the reference Fortran path; every function there cites the
reference file:line it follows.  This module only marshals NumPy arrays.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
_LIB_PATH = _HERE / "_build" / "liboracle.so"
_lib = None

D = C.POINTER(C.c_double)
F = C.POINTER(C.c_float)
I = C.POINTER(C.c_int)


class Stats(C.Structure):
    _fields_ = [
        ("f_evals", C.c_long),
        ("steps", C.c_long),
        ("bad_steps", C.c_long),
        ("n_flag3", C.c_long),
        ("n_flag4", C.c_long),
        ("n_out", C.c_long),
        ("status", C.c_int),
        ("converged_at", C.c_int),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


def build() -> Path:
    """Compile the oracle with its Makefile (gcc, no FMA contraction)."""
    subprocess.run(["make", "-s", "-C", str(_HERE)], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not _LIB_PATH.exists():
            build()
        _lib = C.CDLL(str(_LIB_PATH))
        L = _lib
        L.or_prism_tensor.argtypes = [C.c_double] * 6 + [D]
        L.or_grid.argtypes = [C.c_int] * 3 + [C.c_double] * 3 + [D, D]
        L.or_assemble.argtypes = [C.c_int] * 3 + [C.c_double] * 3 + [I, C.c_int, F, D]
        L.or_problem_create.restype = C.c_void_p
        L.or_problem_create.argtypes = ([C.c_int] * 3 + [C.c_double] * 3 + [C.c_int, C.c_int, C.c_double, D, D, D,
                                        C.c_double, C.c_double, D, C.c_int, D, C.c_int])
        L.or_problem_set_tensor.argtypes = [C.c_void_p, F, D]
        L.or_problem_set_hext_ind.argtypes = [C.c_void_p, C.c_int]
        L.or_problem_set_renorm.argtypes = [C.c_void_p, C.c_int]
        L.or_problem_set_alpha0.argtypes = [C.c_void_p, C.c_double]
        L.or_problem_nrhs.argtypes = [C.c_void_p]
        L.or_problem_nrhs.restype = C.c_long
        L.or_problem_destroy.argtypes = [C.c_void_p]
        L.or_problem_range_err.argtypes = [C.c_void_p]
        L.or_problem_range_err.restype = C.c_int
        L.or_fields.argtypes = [C.c_void_p, C.c_double, D, D, D, D, D]
        L.or_rhs.argtypes = [C.c_void_p, C.c_double, D, D]
        L.or_interp1.argtypes = [D, C.c_int, C.c_int, C.c_int, C.c_double]
        L.or_interp1.restype = C.c_double
        L.or_solve.argtypes = [C.c_void_p, D, C.c_int, D, C.c_double, C.c_double, D, C.c_int, C.c_double,
                               D, D, I, C.POINTER(Stats)]
        L.or_solve_linear.argtypes = [C.c_int, D, D, C.c_int, D, C.c_double, C.c_double, D, D, I,
                                      C.POINTER(Stats)]
        L.or_demag_rows.argtypes = [F, D, C.c_int, C.c_int, D, D, C.c_int, D]
        L.or_threshold_fraction.argtypes = [F, C.c_int, C.c_float]
        L.or_threshold_fraction.restype = C.c_float
        L.or_problem_set_threshold.argtypes = [C.c_void_p, C.c_float]
        L.or_problem_set_threshold.restype = C.c_longlong
        L.or_stats_size.restype = C.c_int
        assert L.or_stats_size() == C.sizeof(Stats), "oracle stats layout mismatch"
    return _lib


def _d(a):
    return a.ctypes.data_as(D)


def _f(a):
    return a.ctypes.data_as(F)


def _i(a):
    return a.ctypes.data_as(I)


def prism_tensor(a, b, c, x, y, z) -> np.ndarray:
    """(xx, xy, xz, yy, yz, zz) of a prism (a,b,c) at offset (x,y,z), reference sign."""
    out = np.zeros(6)
    lib().or_prism_tensor(a, b, c, x, y, z, _d(out))
    return out


def grid(res, L):
    nx, ny, nz = (int(v) for v in res)
    n = nx * ny * nz
    pts = np.zeros((n, 3))
    d = np.zeros(3)
    lib().or_grid(nx, ny, nz, float(L[0]), float(L[1]), float(L[2]), _d(pts), _d(d))
    return pts, d


def assemble(res, L, rows=None, fp32=True, fp64=False):
    """Dense tensor rows K[c][r][j] (c = xx,xy,xz,yy,yz,zz) for receivers ``rows``."""
    nx, ny, nz = (int(v) for v in res)
    n = nx * ny * nz
    nr = n if rows is None else len(rows)
    K32 = np.zeros((6, nr, n), dtype=np.float32) if fp32 else None
    K64 = np.zeros((6, nr, n), dtype=np.float64) if fp64 else None
    rws = None if rows is None else np.ascontiguousarray(rows, dtype=np.int32)
    lib().or_assemble(nx, ny, nz, float(L[0]), float(L[1]), float(L[2]),
                      None if rws is None else _i(rws), nr,
                      None if K32 is None else _f(K32), None if K64 is None else _d(K64))
    return K32, K64


def demag_rows(K32, K64, m, Ms_rows, mode=0):
    """Internal demag field H = -Ms K m at the receivers whose rows are given."""
    nr = (K32 if K32 is not None else K64).shape[1]
    n = (K32 if K32 is not None else K64).shape[2]
    m = np.ascontiguousarray(m, dtype=np.float64).reshape(3 * n)
    Ms_rows = np.ascontiguousarray(np.broadcast_to(Ms_rows, (nr,)), dtype=np.float64)
    out = np.zeros((3, nr))
    lib().or_demag_rows(None if K32 is None else _f(np.ascontiguousarray(K32)),
                        None if K64 is None else _d(np.ascontiguousarray(K64)),
                        nr, n, _d(m), _d(Ms_rows), mode, _d(out))
    return out


def threshold_fraction(K32, frac):
    """FindThresholdFraction's threshold for the tensor K32[c][i][j] (FP32)."""
    K32 = np.ascontiguousarray(K32, dtype=np.float32)
    return float(lib().or_threshold_fraction(_f(K32), K32.shape[1], float(frac)))


def interp1(table, col, x):
    table = np.ascontiguousarray(table, dtype=np.float64)
    return lib().or_interp1(_d(table), table.shape[1], col, table.shape[0], float(x))


class Problem:
    """Oracle counterpart of one micromagnetic problem (uniform grid).

    mode 0 ("ref"): FP32 tensor and FP32 demag product, as the reference.
    mode 1 ("fp64"): FP64 tensor and FP64 product.
    mode 2 ("int8"): the exact fixed-point product of the int8 backend, from
    the FP32 tensor (32-bit rows, m as rint(m 2^30), sixteen limb products).
    """

    def __init__(self, res, L, *, solver=2, mode=0, A0=1.3e-11, Ms=8e5, K0=0.0, u_ea=None,
                 gamma=0.0, alpha=0.02, alpha_tab=None, hext=None, K32=None, K64=None):
        nx, ny, nz = (int(v) for v in res)
        self.res = (nx, ny, nz)
        self.L = tuple(float(v) for v in L)
        n = nx * ny * nz
        self.n = n
        self.mode = mode
        Ms = np.ascontiguousarray(np.broadcast_to(np.asarray(Ms, dtype=np.float64), (n,)))
        K0 = np.ascontiguousarray(np.broadcast_to(np.asarray(K0, dtype=np.float64), (n,)))
        u = np.zeros((n, 3)) if u_ea is None else np.ascontiguousarray(u_ea, dtype=np.float64).reshape(n, 3)
        at = np.zeros((1, 2)) if alpha_tab is None else np.ascontiguousarray(alpha_tab, dtype=np.float64)
        he = np.zeros((2, 4)) if hext is None else np.ascontiguousarray(hext, dtype=np.float64)
        self._keep = (Ms, K0, u, at, he)
        self.Ms = Ms
        self.h = lib().or_problem_create(nx, ny, nz, *self.L, solver, mode, float(A0), _d(Ms), _d(K0), _d(u),
                                         float(gamma), float(alpha), _d(at), at.shape[0], _d(he), he.shape[0])
        if mode in (0, 2) and K32 is None:
            K32, _ = assemble(res, L, fp32=True)
        if mode == 1 and K64 is None:
            _, K64 = assemble(res, L, fp32=False, fp64=True)
        self.K32 = None if K32 is None else np.ascontiguousarray(K32, dtype=np.float32)
        self.K64 = None if K64 is None else np.ascontiguousarray(K64, dtype=np.float64)
        lib().or_problem_set_tensor(self.h, None if self.K32 is None else _f(self.K32),
                                    None if self.K64 is None else _d(self.K64))

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            lib().or_problem_destroy(h)
            self.h = None

    def set_hext_ind(self, i):
        lib().or_problem_set_hext_ind(self.h, int(i))

    def set_threshold(self, thr):
        """mode 0: keep only the tensor entries with |K| > thr (FP32); returns their count."""
        return int(lib().or_problem_set_threshold(self.h, float(thr)))

    def set_renorm(self, on):
        lib().or_problem_set_renorm(self.h, int(bool(on)))

    def set_alpha0(self, a):
        lib().or_problem_set_alpha0(self.h, float(a))

    @property
    def range_err(self):
        """mode 2: a component of m outside (-1.96, 1.96) was met"""
        return bool(lib().or_problem_range_err(self.h))

    @property
    def nrhs(self):
        return lib().or_problem_nrhs(self.h)

    def fields(self, t, m):
        n = self.n
        m = np.ascontiguousarray(m, dtype=np.float64).reshape(3 * n)
        out = [np.zeros(3 * n) for _ in range(4)]
        lib().or_fields(self.h, float(t), _d(m), *(_d(o) for o in out))
        return tuple(o.reshape(3, n) for o in out)   # Hj, Hh, Hk, Hm

    def rhs(self, t, m):
        n = self.n
        m = np.ascontiguousarray(m, dtype=np.float64).reshape(3 * n)
        out = np.zeros(3 * n)
        lib().or_rhs(self.h, float(t), _d(m), _d(out))
        return out

    def solve(self, t, m0, tol=1e-4, thres=1e-6, t_conv=None, conv_tol=1e-4):
        """MagTense_ODE_RKSuite: returns (t_out, y_out[nt, 3n], flags[nt], stats)."""
        t = np.ascontiguousarray(t, dtype=np.float64)
        nt = t.shape[0]
        m0 = np.ascontiguousarray(m0, dtype=np.float64).reshape(3 * self.n)
        tc = np.zeros(1) if t_conv is None else np.ascontiguousarray(t_conv, dtype=np.float64)
        t_out = np.zeros(nt)
        y_out = np.zeros((nt, 3 * self.n))
        flags = np.zeros(nt, dtype=np.int32)
        st = Stats()
        lib().or_solve(self.h, _d(t), nt, _d(m0), float(tol), float(thres), _d(tc), tc.shape[0],
                       float(conv_tol), _d(t_out), _d(y_out), _i(flags), C.byref(st))
        return t_out, y_out, flags, st.as_dict()


def solve_linear(lam, t, y0, tol=1e-6, thres=1e-6):
    lam = np.ascontiguousarray(lam, dtype=np.float64)
    t = np.ascontiguousarray(t, dtype=np.float64)
    y0 = np.ascontiguousarray(y0, dtype=np.float64)
    n = lam.shape[0]
    nt = t.shape[0]
    t_out = np.zeros(nt)
    y_out = np.zeros((nt, n))
    flags = np.zeros(nt, dtype=np.int32)
    st = Stats()
    lib().or_solve_linear(n, _d(lam), _d(t), nt, _d(y0), float(tol), float(thres), _d(t_out), _d(y_out),
                          _i(flags), C.byref(st))
    return t_out, y_out, flags, st.as_dict()


def threads() -> int:
    return int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
