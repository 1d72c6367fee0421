"""ctypes binding of libedk.so (the C ABI declared in include/edk.h).

The library is loaded from this directory.  There is no fallback: if the
shared object is missing or cannot be loaded, every call raises.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libedk.so")

# edk_status
OK, INVALID_ARG, NOT_HERMITIAN, OOM, CUDA_ERROR, TIMEOUT, NOT_CONVERGED, UNSUPPORTED, \
    ZERO_NORM, BACKWARD_TIME = range(10)
# edk_dtype
F64, C128, F32, C64 = range(4)
HOST, DEVICE = 0, 1
TENSOR, PROJECTED, TRANSLATIONAL, TRANSPARITY, ABELIAN, TRANSFLIP = range(6)
PREC_FP64, PREC_MIXED = 0, 1

EXPORTS = [
    "edk_basis_create", "edk_basis_destroy", "edk_basis_dim", "edk_basis_export",
    "edk_basis_index", "edk_basis_index_noalloc", "edk_operator_create", "edk_operator_destroy", "edk_operator_info",
    "edk_operator_materialize", "edk_operator_configure", "edk_operator_autotune",
    "edk_basis_set_search", "edk_basis_get_search", "edk_block_lanczos", "edk_lanczos_ground_state",
    "edk_schmidt", "edk_ent_spec", "edk_ent_S", "edk_double_basis_apply", "edk_symmetrizer",
    "edk_block_tridiag_lowest",
    "edk_block_lanczos_default_opts",
    "edk_apply", "edk_apply_async", "edk_lanczos_e0", "edk_krylov_default_opts",
    "edk_krylov_evolve", "edk_batch_lanczos_e0", "edk_tridiag_eigen", "edk_last_error",
    "edk_version", "edk_krylov_cache_create", "edk_krylov_cache_evolve", "edk_krylov_cache_info",
    "edk_krylov_cache_destroy", "edk_selftest_bounded_wait",
]


class EDKError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(msg)
        self.status = status


class BasisDesc(C.Structure):
    _fields_ = [
        ("kind", C.c_int32), ("L", C.c_int32), ("base", C.c_int32), ("a", C.c_int32),
        ("k", C.c_int32), ("p", C.c_int32), ("N", C.c_int32), ("ngen", C.c_int32),
        ("gen_order", C.c_void_p), ("gen_q", C.c_void_p), ("gen_perm", C.c_void_p),
        ("gen_inv", C.c_void_p), ("allow", C.c_void_p), ("D", C.c_int64), ("I", C.c_void_p),
        ("R", C.c_void_p),
    ]


class LanczosOpts(C.Structure):
    _fields_ = [
        ("max_steps", C.c_int32), ("nev", C.c_int32), ("tol", C.c_double),
        ("check_every", C.c_int32), ("precision", C.c_int32), ("refine_steps", C.c_int32),
        ("reorth", C.c_int32), ("complex_vectors", C.c_int32),
    ]


class LanczosDiag(C.Structure):
    _fields_ = [
        ("steps", C.c_int32), ("steps_low", C.c_int32), ("matvecs", C.c_int32),
        ("breakdown", C.c_int32), ("seconds", C.c_double), ("seconds_matvec", C.c_double),
        ("seconds_reorth", C.c_double), ("residual", C.c_double),
        ("seconds_setup", C.c_double), ("seconds_stage1", C.c_double),
        ("seconds_refine", C.c_double), ("refine_rounds", C.c_int32), ("checks", C.c_int32),
    ]


class KrylovOpts(C.Structure):
    _fields_ = [
        ("tol", C.c_double), ("m_init", C.c_int32), ("m_max", C.c_int32),
        ("extend_step", C.c_int32), ("nsample", C.c_int32), ("bisect_iters", C.c_int32),
        ("reuse_basis", C.c_int32), ("extend_basis", C.c_int32),
        ("normalize_output", C.c_int32), ("precision", C.c_int32),
    ]


class KrylovDiag(C.Structure):
    _fields_ = [
        ("basis_builds", C.c_int32), ("basis_extensions", C.c_int32), ("restarts", C.c_int32),
        ("matvecs", C.c_int32), ("total_times_served", C.c_int32), ("max_dim_used", C.c_int32),
        ("n_intervals", C.c_int32), ("accepted_intervals", C.c_double * 64),
        ("seconds", C.c_double),
    ]


class BlockLanczosOpts(C.Structure):
    _fields_ = [
        ("block", C.c_int32), ("max_steps", C.c_int32), ("nev", C.c_int32), ("tol", C.c_double),
        ("check_every", C.c_int32), ("seed", C.c_uint64),
    ]


class BlockLanczosDiag(C.Structure):
    _fields_ = [
        ("steps", C.c_int32), ("matvecs", C.c_int64), ("breakdowns", C.c_int32),
        ("converged", C.c_int32), ("seconds", C.c_double), ("seconds_spmm", C.c_double),
        ("seconds_orth", C.c_double), ("seconds_eig", C.c_double),
    ]


TUNE_MAX = 24
KERNEL_FAST, KERNEL_GENERIC, KERNEL_MATERIALIZED, KERNEL_MATERIALIZED_STAGED = 0, 1, 2, 3
SEARCH_HASH, SEARCH_SORTED = 0, 1
TUNE_MATERIALIZE = 1


class TuneResult(C.Structure):
    _fields_ = [
        ("kernel", C.c_int32), ("search", C.c_int32), ("tps", C.c_int32), ("block", C.c_int32),
        ("ms", C.c_double), ("ncand", C.c_int32), ("cand_kernel", C.c_int32 * TUNE_MAX),
        ("cand_search", C.c_int32 * TUNE_MAX), ("cand_tps", C.c_int32 * TUNE_MAX),
        ("cand_block", C.c_int32 * TUNE_MAX), ("cand_ms", C.c_double * TUNE_MAX),
    ]


_lib = None


def load():
    """Load libedk.so; raises if it is absent (no CPU fallback exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise EDKError(-1, f"libedk.so not built ({LIB_PATH}); run __graft_entry__.build()")
    L = C.CDLL(LIB_PATH)
    vp, i32, i64, dp = C.c_void_p, C.c_int32, C.c_int64, C.POINTER(C.c_double)
    st = C.c_int
    sig = {
        "edk_basis_create": (st, [C.POINTER(BasisDesc), C.POINTER(vp)]),
        "edk_basis_destroy": (st, [vp]),
        "edk_basis_dim": (st, [vp, C.POINTER(i64)]),
        "edk_basis_export": (st, [vp, vp, vp]),
        "edk_basis_index": (st, [vp, i64, vp, vp, vp, i32]),
        "edk_basis_index_noalloc": (st, [vp, i64, vp, vp, vp]),
        "edk_operator_create": (st, [vp, i32, vp, vp, vp, vp, vp, vp, C.POINTER(vp)]),
        "edk_operator_destroy": (st, [vp]),
        "edk_operator_materialize": (st, [vp, i32, C.POINTER(i64)]),
        "edk_operator_configure": (st, [vp, i32, i32, i32]),
        "edk_operator_autotune": (st, [vp, i32, i64, i32, C.POINTER(TuneResult)]),
        "edk_basis_set_search": (st, [vp, i32]),
        "edk_block_lanczos_default_opts": (None, [C.POINTER(BlockLanczosOpts)]),
        "edk_block_lanczos": (st, [i32, vp, C.POINTER(BlockLanczosOpts), vp, vp,
                                   C.POINTER(BlockLanczosDiag)]),
        "edk_basis_get_search": (st, [vp, C.POINTER(i32)]),
        "edk_operator_info": (st, [vp, C.POINTER(i32), C.POINTER(i32), C.POINTER(i32),
                                   C.POINTER(i32)]),
        "edk_apply": (st, [vp, i32, vp, vp, i64, i64, i64, i32, i32]),
        "edk_apply_async": (st, [vp, i32, vp, vp, i64, i64, i64, i32, vp]),
        "edk_lanczos_e0": (st, [vp, C.POINTER(LanczosOpts), vp, i32, i32, vp, vp, vp,
                                C.POINTER(LanczosDiag)]),
        "edk_block_tridiag_lowest": (st, [i32, i32, vp, vp, i32, vp]),
        "edk_lanczos_ground_state": (st, [vp, C.POINTER(LanczosOpts), vp, i32, i32, vp, vp, i32,
                                          C.POINTER(LanczosDiag)]),
        "edk_krylov_default_opts": (None, [C.POINTER(KrylovOpts)]),
        "edk_krylov_evolve": (st, [vp, C.POINTER(KrylovOpts), vp, vp, i64, vp, i32,
                                   C.POINTER(KrylovDiag)]),
        "edk_krylov_cache_create": (st, [vp, C.POINTER(KrylovOpts), vp, i32, C.POINTER(vp)]),
        "edk_krylov_cache_evolve": (st, [vp, vp, i64, vp, i32]),
        "edk_krylov_cache_info": (st, [vp, dp, dp, C.POINTER(i32), C.POINTER(KrylovDiag)]),
        "edk_krylov_cache_destroy": (st, [vp]),
        "edk_selftest_bounded_wait": (st, [C.c_uint32]),
        "edk_batch_lanczos_e0": (st, [i32, vp, C.POINTER(LanczosOpts), vp, i32, vp,
                                      C.POINTER(LanczosDiag)]),
        "edk_tridiag_eigen": (C.c_int, [C.c_int, vp, vp, vp, vp]),
        "edk_schmidt": (st, [vp, i32, vp, i32, vp, vp, i32, i32]),
        "edk_ent_spec": (st, [vp, i32, vp, i32, vp, vp, C.POINTER(i64), i32]),
        "edk_ent_S": (st, [vp, i32, vp, i32, vp, C.c_double, C.c_double, dp, i32]),
        "edk_double_basis_apply": (st, [vp, vp, i32, vp, vp, i32]),
        "edk_symmetrizer": (st, [vp, vp, vp, i32]),
        "edk_last_error": (C.c_char_p, []),
        "edk_version": (C.c_char_p, []),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def check(status):
    if status != OK:
        msg = load().edk_last_error().decode(errors="replace")
        raise EDKError(status, msg or f"libedk status {status}")


def ptr(a):
    """Raw address of a numpy array or torch tensor."""
    if hasattr(a, "data_ptr"):
        return C.c_void_p(a.data_ptr())
    return a.ctypes.data_as(C.c_void_p)
