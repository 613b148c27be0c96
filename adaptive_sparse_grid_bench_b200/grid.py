"""Python mirror of the reference benchmark's grid operations over the C ABI.

Names and argument meanings follow adaptive_sparse_grid_bench.c: a grid is
created from (num_dims, num_levels, limits) as ``init()`` does (c:101-140),
``hierarchize()`` works in place (c:557-1233), ``evaluate(coord_mat)`` returns
one value per row (c:1237-1722), and ``gp2idx``/``idx2gp`` are the bijection
(c:187-243).  Every call goes to libsgb200.so; errors raise `SgError`
instead of asserting.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from ._lib import check


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def _stream_handle(stream) -> int | None:
    """Accepts None, an int handle, or a torch.cuda.Stream."""
    if stream is None:
        return None
    if isinstance(stream, int):
        return stream
    return int(stream.cuda_stream)


class Grid:
    """A compact sparse grid resident on the GPU (one sg_grid handle)."""

    def __init__(self, num_dims: int, num_levels: int, limits=None):
        lib = L.lib()
        h = C.c_void_p()
        lim = None
        if limits is not None:
            self._lim_buf = np.ascontiguousarray(limits, dtype=np.int32)
            if self._lim_buf.shape != (num_dims,):
                raise ValueError("limits must have num_dims entries")
            lim = _ptr(self._lim_buf)
        check(lib.sg_create(num_dims, num_levels, lim, C.byref(h)))
        self._adopt(h)

    @classmethod
    def from_handle(cls, h: C.c_void_p) -> "Grid":
        """Wraps an sg_grid handle made by the library (e.g. by sg_refine);
        the Grid owns it from then on."""
        g = cls.__new__(cls)
        g._adopt(h)
        return g

    def _adopt(self, h: C.c_void_p) -> None:
        lib = L.lib()
        self._h = h
        d, n = C.c_int(), C.c_int()
        check(lib.sg_dims(h, C.byref(d), C.byref(n), None))
        num_dims, num_levels = d.value, n.value
        self.d = num_dims
        self.n = num_levels
        v = C.c_int64()
        check(lib.sg_num_points(h, C.byref(v)))
        self.num_points = v.value
        check(lib.sg_num_subspaces(h, C.byref(v)))
        self.num_subspaces = v.value
        lim_out = np.zeros(num_dims, np.int32)
        check(lib.sg_dims(h, None, None, _ptr(lim_out)))
        self.limits = lim_out

    # -- lifetime -----------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            L.lib().sg_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    # -- tables and bijection (host) ----------------------------------------
    def tables(self):
        dp = np.zeros(self.d * self.n, np.int64)
        lidx = np.zeros(self.n + 1, np.int64)
        check(L.lib().sg_tables(self._h, _ptr(dp), _ptr(lidx)))
        return dp.reshape(self.d, self.n), lidx

    def gp2idx(self, levels, indices) -> int:
        lv = np.ascontiguousarray(levels, np.int32)
        ix = np.ascontiguousarray(indices, np.int32)
        out = C.c_int64()
        check(L.lib().sg_gp2idx(self._h, _ptr(lv), _ptr(ix), C.byref(out)))
        return out.value

    def idx2gp(self, index: int):
        lv = np.zeros(self.d, np.int32)
        ix = np.zeros(self.d, np.int32)
        check(L.lib().sg_idx2gp(self._h, int(index), _ptr(lv), _ptr(ix)))
        return lv, ix

    def l2idx(self, levels) -> int:
        lv = np.ascontiguousarray(levels, np.int32)
        out = C.c_int64()
        check(L.lib().sg_l2idx(self._h, _ptr(lv), C.byref(out)))
        return out.value

    def idx2l(self, position: int, level_sum: int):
        lv = np.zeros(self.d, np.int32)
        check(L.lib().sg_idx2l(self._h, int(position), int(level_sum), _ptr(lv)))
        return lv

    def subspaces(self):
        """Level vectors of all subspaces in memory order, shape (S, d)."""
        dp, _ = self.tables()
        out = np.zeros((self.num_subspaces, self.d), np.int32)
        r = 0
        for s in range(self.n):
            for pos in range(int(dp[self.d - 1, s])):
                out[r] = self.idx2l(pos, s)
                r += 1
        return out

    # -- options --------------------------------------------------------------
    def set_option(self, option: int, value: int) -> None:
        check(L.lib().sg_set_option(self._h, option, int(value)))

    def get_option(self, option: int) -> int:
        v = C.c_int64()
        check(L.lib().sg_get_option(self._h, option, C.byref(v)))
        return v.value

    @property
    def precision(self) -> str:
        return "fp64" if self.get_option(L.SG_OPT_HIER_PRECISION) == L.SG_HIER_FP64 else "fp32"

    @precision.setter
    def precision(self, p: str) -> None:
        self.set_option(L.SG_OPT_HIER_PRECISION, L.SG_HIER_FP64 if p == "fp64" else L.SG_HIER_FP32)

    def timings(self) -> dict:
        """Device milliseconds of the phases of the latest profiled calls."""
        ms = np.zeros(L.SG_NUM_PHASES, np.float64)
        check(L.lib().sg_timings(self._h, _ptr(ms)))
        return {"hierarchize": ms[0], "sort": ms[1], "evaluate": ms[2]}

    def device_bytes(self) -> int:
        v = C.c_int64()
        check(L.lib().sg_device_bytes(self._h, C.byref(v)))
        return v.value

    # -- host-buffer calls (synchronous) -------------------------------------
    def set_values(self, values) -> None:
        v = np.ascontiguousarray(values, np.float32)
        if v.shape != (self.num_points,):
            raise ValueError(f"expected {self.num_points} values, got {v.shape}")
        check(L.lib().sg_set_values(self._h, _ptr(v)))

    def get_values(self) -> np.ndarray:
        out = np.empty(self.num_points, np.float32)
        check(L.lib().sg_get_values(self._h, _ptr(out)))
        return out

    def hierarchize(self) -> None:
        check(L.lib().sg_hierarchize(self._h))

    def subspace_maxabs(self) -> np.ndarray:
        """max |value| per subspace (compact subspace order), S floats."""
        out = np.empty(self.num_subspaces, np.float32)
        check(L.lib().sg_subspace_maxabs(self._h, _ptr(out)))
        return out

    def evaluate(self, coord_mat) -> np.ndarray:
        X = np.ascontiguousarray(coord_mat, np.float32).reshape(-1, self.d)
        out = np.empty(X.shape[0], np.float32)
        check(L.lib().sg_evaluate(self._h, _ptr(X), _ptr(out), X.shape[0]))
        return out

    # -- device-pointer calls (asynchronous; torch tensors or raw pointers) ---
    @staticmethod
    def _dptr(t) -> int:
        return t if isinstance(t, int) else int(t.data_ptr())

    def set_values_device(self, values, stream=None) -> None:
        check(L.lib().sg_set_values_device(self._h, self._dptr(values), _stream_handle(stream)))

    def get_values_device(self, values, stream=None) -> None:
        check(L.lib().sg_get_values_device(self._h, self._dptr(values), _stream_handle(stream)))

    def hierarchize_async(self, stream=None) -> None:
        check(L.lib().sg_hierarchize_async(self._h, _stream_handle(stream)))

    def evaluate_device(self, coords, out, num_evals: int | None = None, stream=None) -> None:
        if num_evals is None:
            num_evals = int(coords.shape[0])
        check(L.lib().sg_evaluate_device(self._h, self._dptr(coords), self._dptr(out), int(num_evals),
                                         _stream_handle(stream)))

    def sample_function(self, fn: int, params=(), stream=None) -> None:
        """Fill the grid on the device with a built-in function (SG_FN_*)."""
        p = np.ascontiguousarray(params, np.float64)
        check(L.lib().sg_sample_function(self._h, int(fn), _ptr(p) if p.size else None, int(p.size),
                                         _stream_handle(stream)))

    def evaluate_device_noalloc(self, coords, out, num_evals: int | None = None, stream=None) -> None:
        """sg_evaluate_device_noalloc: the same evaluation without any device
        allocation (fixed scratch; at most SG_NOALLOC_MAX_POINTS points)."""
        if num_evals is None:
            num_evals = int(coords.shape[0])
        check(L.lib().sg_evaluate_device_noalloc(self._h, self._dptr(coords), self._dptr(out), int(num_evals),
                                                 _stream_handle(stream)))

    def sync(self, stream=None) -> None:
        check(L.lib().sg_sync(self._h, _stream_handle(stream)))

    def autotune(self, coords, out, num_evals: int | None = None, stream=None) -> dict:
        """sg_autotune: times the evaluation settings and sweep kernels on these
        device buffers, keeps the fastest; returns the timings (ms, -1 = n/a)."""
        if num_evals is None:
            num_evals = int(coords.shape[0])
        ms = np.zeros(L.SG_TUNE_TIMINGS, np.float64)
        check(L.lib().sg_autotune(self._h, self._dptr(coords), self._dptr(out), int(num_evals),
                                  _stream_handle(stream), _ptr(ms)))
        return {"eval_ppt1_unsorted": ms[0], "eval_ppt1_sorted": ms[1], "eval_ppt2_unsorted": ms[2],
                "eval_ppt2_sorted": ms[3], "hier_chains": ms[4], "hier_gather": ms[5],
                "eval_blocking_wide": ms[6], "eval_blocking_medium": ms[7]}

    def idx2gp_device(self, index, levels, indices, count: int, stream=None) -> None:
        check(L.lib().sg_idx2gp_device(self._h, self._dptr(index), self._dptr(levels), self._dptr(indices),
                                       int(count), _stream_handle(stream)))

    def gp2idx_device(self, levels, indices, index, count: int, stream=None) -> None:
        check(L.lib().sg_gp2idx_device(self._h, self._dptr(levels), self._dptr(indices), self._dptr(index),
                                       int(count), _stream_handle(stream)))
