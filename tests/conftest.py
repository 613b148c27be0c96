import glob
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def golden_cases():
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz")))


def load_golden(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    return {k: z[k] for k in z.files}


# Evaluation tolerance against the FP64 oracle, used by the GPU tests:
#   norm-wise   |u - u64| <= EVAL_RTOL_NORM max|u64| + EVAL_ATOL
#   per point   |u - u64| <= EVAL_RTOL_POINT max(|u64|, EVAL_FLOOR max|u64|)
#               (smooth test functions: the benchmark's configurations)
# (relative error 1e-5 per point; the floor bounds points where u64 crosses
# zero absolutely, at 1e-7 of the largest value).
EVAL_RTOL_NORM, EVAL_ATOL = 1e-5, 2e-7
EVAL_RTOL_POINT, EVAL_FLOOR = 1e-5, 1e-2


def check_eval(got, ref64, what="", per_point=True):
    """Asserts the norm-wise bound and, for smooth test functions
    (per_point), the per-point bound; returns the per-point relative error.
    Grids holding random nodal values have surpluses far larger than the
    interpolant, so FP32 rounding is bounded relative to max|u| only."""
    ref64 = np.asarray(ref64, np.float64)
    scale = max(float(np.max(np.abs(ref64))), 1e-30)
    err = np.abs(np.asarray(got, np.float64) - ref64)
    assert np.all(err <= EVAL_RTOL_NORM * scale + EVAL_ATOL), f"{what}: norm-wise {err.max() / scale:.3e}"
    rel = err / np.maximum(np.abs(ref64), EVAL_FLOOR * scale)
    if per_point:
        assert rel.max() <= EVAL_RTOL_POINT, f"{what}: per-point relative {rel.max():.3e}"
    return float(rel.max())


@pytest.fixture(scope="session")
def cuda():
    """The GPU tests' device; fails (does not skip) when there is none, so a
    GPU run can never pass on a silent fallback."""
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch.device("cuda:0")
