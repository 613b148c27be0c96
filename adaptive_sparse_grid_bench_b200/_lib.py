"""Loader and ctypes signatures for libsgb200.so (the C ABI of include/sgrid.h).

The shared library is built in-tree by ``make -C adaptive_sparse_grid_bench_b200/csrc``
(or ``__graft_entry__.build()``).  There is no Python or CPU fallback: if the
library is missing, importing the bindings raises.
"""
from __future__ import annotations

import ctypes as C
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsgb200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "sgrid.h")

SG_OK = 0
SG_ERR_ARG = -1
SG_ERR_RANGE = -2
SG_ERR_CUDA = -3
SG_ERR_NOMEM = -4
SG_ERR_STATE = -5
SG_ERR_TIMEOUT = -6

SG_HIER_FP32 = 0
SG_HIER_FP64 = 1

SG_OPT_HIER_PRECISION = 1
SG_OPT_EVAL_SORT = 2
SG_OPT_EVAL_PPT = 3
SG_OPT_HIER_KERNEL = 5
SG_OPT_PROFILE = 6
SG_OPT_USE_GRAPH = 7
SG_OPT_SWEEP_GROUP = 8
SG_OPT_TEST_WAIT = 9
SG_OPT_EVAL_BLOCKING = 10
SG_EVAL_BLOCKINGS = 2
SG_SRV_OPT_ZERO_COPY = 1
SG_SRV_OPT_HEAVY_PAIRS = 2
SG_SRV_OPT_LIGHT_SLOTS = 3
SG_SRV_OPT_SORT_HEAVY = 4
SG_NUM_PHASES = 3

SG_FN_REFERENCE = 0
SG_FN_PROD4 = 1
SG_FN_GAUSS = 2
SG_FN_BUMP = 3
SG_FN_QUAD = 4

SG_MAX_DIMS = 20
SG_TUNE_TIMINGS = 8
SG_BATCH_TUNE_TIMINGS = 4 * (SG_MAX_DIMS + 1)
SG_MAX_LEVELS = 16
SG_NOALLOC_MAX_POINTS = 1 << 18
SG_NOALLOC_SCRATCH_BYTES = 24 << 20

_i = C.c_int
_i64 = C.c_int64
_p = C.c_void_p
_pi64 = C.POINTER(C.c_int64)

# name -> (restype, argtypes)
SIGNATURES = {
    "sg_create": (_i, [_i, _i, _p, C.POINTER(_p)]),
    "sg_destroy": (_i, [_p]),
    "sg_num_points": (_i, [_p, _pi64]),
    "sg_num_subspaces": (_i, [_p, _pi64]),
    "sg_dims": (_i, [_p, _p, _p, _p]),
    "sg_tables": (_i, [_p, _p, _p]),
    "sg_gp2idx": (_i, [_p, _p, _p, _pi64]),
    "sg_idx2gp": (_i, [_p, _i64, _p, _p]),
    "sg_l2idx": (_i, [_p, _p, _pi64]),
    "sg_idx2l": (_i, [_p, _i64, _i, _p]),
    "sg_set_values": (_i, [_p, _p]),
    "sg_get_values": (_i, [_p, _p]),
    "sg_hierarchize": (_i, [_p]),
    "sg_evaluate": (_i, [_p, _p, _p, _i64]),
    "sg_set_values_device": (_i, [_p, _p, _p]),
    "sg_get_values_device": (_i, [_p, _p, _p]),
    "sg_hierarchize_async": (_i, [_p, _p]),
    "sg_evaluate_device": (_i, [_p, _p, _p, _i64, _p]),
    "sg_evaluate_device_noalloc": (_i, [_p, _p, _p, _i64, _p]),
    "sg_sync": (_i, [_p, _p]),
    "sg_autotune": (_i, [_p, _p, _p, _i64, _p, _p]),
    "sg_idx2gp_device": (_i, [_p, _p, _p, _p, _i64, _p]),
    "sg_gp2idx_device": (_i, [_p, _p, _p, _p, _i64, _p]),
    "sg_set_option": (_i, [_p, _i, _i64]),
    "sg_get_option": (_i, [_p, _i, _pi64]),
    "sg_device_bytes": (_i, [_p, _pi64]),
    "sg_timings": (_i, [_p, _p]),
    "sg_kernel_launches": (_i, [_pi64]),
    "sg_sample_function": (_i, [_p, _i, _p, _i, _p]),
    "sg_subspace_maxabs": (_i, [_p, _p]),
    "sg_refine_step": (_i, [_i, _i, _p, _p, C.c_double, _i, _p, _p, _p]),
    "sg_refine": (_i, [_i, _i, _p, _i, _p, _i, C.c_double, _i, _i64, _i, _i, C.POINTER(_p), _p]),
    "sg_batch_create": (_i, [_i, _p, _p, _p, C.POINTER(_p)]),
    "sg_batch_destroy": (_i, [_p]),
    "sg_batch_num_grids": (_i, [_p, _p]),
    "sg_batch_offsets": (_i, [_p, _p]),
    "sg_batch_set_values": (_i, [_p, _p]),
    "sg_batch_set_values_device": (_i, [_p, _p, _p]),
    "sg_batch_get_values": (_i, [_p, _p]),
    "sg_batch_get_values_device": (_i, [_p, _p, _p]),
    "sg_batch_sample_function": (_i, [_p, _i, _p, _i, _p]),
    "sg_batch_hierarchize_async": (_i, [_p, _p]),
    "sg_batch_hierarchize": (_i, [_p]),
    "sg_batch_evaluate_device": (_i, [_p, _p, _p, _p, _p]),
    "sg_batch_sync": (_i, [_p, _p]),
    "sg_batch_set_option": (_i, [_p, _i, _i64]),
    "sg_batch_device_bytes": (_i, [_p, _pi64]),
    "sg_batch_autotune": (_i, [_p, _p, _p, _p, _p, _p]),
    "sg_server_create": (_i, [_i64, _i64, C.POINTER(_p)]),
    "sg_server_destroy": (_i, [_p]),
    "sg_server_add_grid": (_i, [_p, _i, _i, _p, _i, _p, _i, _pi64]),
    "sg_server_submit": (_i, [_p, _i64, _p, _i64, _p, _pi64]),
    "sg_server_wait": (_i, [_p, _i64, C.POINTER(C.c_double)]),
    "sg_server_wait_detail": (_i, [_p, _i64, _p]),
    "sg_server_set_option": (_i, [_p, _i, _i64]),
    "sg_server_stats": (_i, [_p, _p]),
    "sg_server_evaluate_now": (_i, [_p, _i64, _p, _i64, _p]),
    "sg_last_error": (C.c_char_p, []),
    "sg_version": (C.c_char_p, []),
}

_lib = None


def header_functions(path: str = HEADER) -> list[str]:
    """Names of the functions declared in include/sgrid.h."""
    text = open(path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sg_\w+)\s*\(", text)))


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is not built; run `make -C {os.path.join(HERE, 'csrc')}` "
                "(there is no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def kernel_launches() -> int:
    """Kernels launched by libsgb200.so so far in this process."""
    v = C.c_int64()
    check(lib().sg_kernel_launches(C.byref(v)))
    return v.value


class SgError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def check(code: int) -> None:
    if code != SG_OK:
        raise SgError(code, lib().sg_last_error().decode(errors="replace"))
