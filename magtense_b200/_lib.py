"""ctypes binding of libmagtense_b200.so (C ABI in include/magtense_b200.h).

The library is built in-tree by ``make -C magtense_b200/csrc``.  There is no
fallback: if the library is missing or no CUDA device is present, every entry
point raises.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "libmagtense_b200.so"
_lib = None

MT_OK = 0
ERRORS = {
    -1: "invalid argument",
    -2: "CUDA error",
    -3: "device out of memory",
    -4: "call out of order",
    -5: "not supported on this path",
    -6: "integrator stopped",
    -7: "bounded device wait gave up",
}

D = C.POINTER(C.c_double)
F = C.POINTER(C.c_float)
I = C.POINTER(C.c_int)
VP = C.c_void_p


class MTError(RuntimeError):
    def __init__(self, code, where, msg):
        super().__init__(f"{where}: {ERRORS.get(code, code)} ({code}): {msg}")
        self.code = code


class Grid(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("Lx", C.c_double), ("Ly", C.c_double), ("Lz", C.c_double)]


class Stats(C.Structure):
    _fields_ = [("f_evals", C.c_longlong), ("steps", C.c_longlong), ("bad_steps", C.c_longlong),
                ("n_flag3", C.c_longlong), ("n_flag4", C.c_longlong), ("n_out", C.c_longlong),
                ("status", C.c_int), ("converged_at", C.c_int), ("launches", C.c_longlong),
                ("kernel_ms", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


# name -> argtypes (all return int status unless listed in _RESTYPE)
SIGNATURES = {
    "mt_create": [C.POINTER(Grid), C.POINTER(VP)],
    "mt_destroy": [VP],
    "mt_last_error": [],
    "mt_version": [],
    "mt_set_material": [VP, C.c_double, D, D, D],
    "mt_set_dynamics": [VP, C.c_int, C.c_double, C.c_double, D, C.c_int, D, C.c_int, C.c_int, C.c_int],
    "mt_assemble_demag": [VP, VP],
    "mt_load_demag_colmajor": [VP, F, F, F, F, F, F],
    "mt_get_demag_colmajor": [VP, F, F, F, F, F, F],
    "mt_demag_field": [VP, VP, VP, VP],
    "mt_fields": [VP, C.c_double, VP, VP, VP, VP, VP, VP],
    "mt_rhs": [VP, C.c_double, VP, VP, VP],
    "mt_rhs_vjp": [VP, C.c_double, VP, VP, VP, VP, VP, VP],
    "mt_rhs_noalloc": [VP, C.c_double, VP, VP, VP],
    "mt_integrate_ragged": [C.POINTER(VP), C.c_int, D, C.c_int, C.POINTER(VP), C.c_double, C.c_double, D,
                            C.POINTER(VP), I, C.POINTER(Stats), C.c_int, VP],
    "mt_integrate": [VP, D, C.c_int, VP, C.c_double, C.c_double, D, C.c_int, C.c_double, D, VP, I,
                     C.POINTER(Stats), VP],
    "mt_set_row_shard": [VP, C.c_int, C.c_int],
    "mt_shard_region": [VP, C.POINTER(VP), C.POINTER(C.c_size_t)],
    "mt_shard_ipc_handle": [VP, VP],
    "mt_shard_open_peers": [VP, VP],
    "mt_shard_set_peers": [VP, C.POINTER(VP)],
    "mt_integrate_shards_local": [C.POINTER(VP), C.c_int, D, C.c_int, VP, C.c_double, C.c_double, D, C.c_int,
                                  C.c_double, D, VP, I, C.POINTER(Stats), VP],
    "mt_batch_create": [C.POINTER(Grid), C.c_int, C.c_int, C.POINTER(VP)],
    "mt_batch_destroy": [VP],
    "mt_batch_set_material": [VP, C.c_double, D, D, D],
    "mt_batch_set_dynamics": [VP, C.c_int, C.c_double, D, D, C.c_int, C.c_int],
    "mt_batch_set_alpha_table": [VP, D, C.c_int],
    "mt_batch_tune": [VP, VP],
    "mt_batch_get_schedule": [VP, I, I, C.c_int, I],
    "mt_batch_set_schedule": [VP, I, I, C.c_int],
    "mt_batch_assemble_demag": [VP, VP],
    "mt_batch_integrate": [VP, D, C.c_int, VP, C.c_double, C.c_double, D, C.c_int, C.c_double, D, VP, I,
                           C.POINTER(Stats), VP],
    "mt_batch_integrate_host": [VP, D, C.c_int, VP, C.c_double, C.c_double, D, C.c_int, C.c_double, D, VP, VP,
                                I, C.POINTER(Stats), VP],
    "mt_batch_demag_field": [VP, VP, VP, VP],
    "icl_initDemagMatrices": [F, F, F, F, F, F, I],
    "icl_MVMult_GetH": [F, F, F, F, F, F, I, F],
    "icl_destroy": [],
    "mt_set_demag_threshold": [VP, C.c_int, C.c_double, C.POINTER(C.c_longlong), F, VP],
    "icl_initDemagMatrices_sparse": [I, I, I, F, I, I],
    "icl_MVMult_GetH_sparse": [F, F, F, F, F, F, I, F],
}
_RESTYPE = {"mt_last_error": C.c_char_p, "mt_version": C.c_char_p}


def build(quiet: bool = True) -> Path:
    """Compile the CUDA sources for sm_100a into magtense_b200/libmagtense_b200.so."""
    cmd = ["make", "-C", str(_HERE / "csrc")]
    if quiet:
        cmd.insert(1, "-s")
    subprocess.run(cmd, check=True)
    return LIB_PATH


def lib():
    """The loaded library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C {_HERE / 'csrc'}`")
        L = C.CDLL(str(LIB_PATH))
        for name, args in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = _RESTYPE.get(name, C.c_int)
        _lib = L
    return _lib


def check(rc: int, where: str):
    if rc != MT_OK:
        raise MTError(rc, where, lib().mt_last_error().decode(errors="replace"))
