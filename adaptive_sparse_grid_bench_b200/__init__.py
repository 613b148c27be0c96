"""B200-native compact sparse grids: index bijection, hierarchization and
evaluation on sm_100a behind the C ABI of include/sgrid.h.

The compute lives in libsgb200.so (CUDA kernels + C host code); this package
only binds it (`Grid`) and generates seeded inputs (`inputs`).
"""
from ._lib import (SG_HIER_FP32, SG_HIER_FP64, SG_OPT_EVAL_BLOCKING, SG_OPT_EVAL_PPT,  # noqa: F401
                   SG_OPT_EVAL_SORT, SG_OPT_HIER_KERNEL, SG_OPT_HIER_PRECISION, SG_OPT_PROFILE, SgError,
                   header_functions, lib)
from .batch import Batch  # noqa: F401
from .grid import Grid  # noqa: F401
from .refine import refine, refine_step  # noqa: F401
from .server import Server  # noqa: F401

__all__ = ["Grid", "Batch", "Server", "SgError", "lib", "header_functions", "refine", "refine_step"]
