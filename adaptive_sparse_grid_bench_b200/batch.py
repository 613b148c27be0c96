"""Batches of independent grids over the C ABI (sg_batch_*): many grids of
mixed d, n and limits hierarchized and evaluated with a fixed set of launches
replayed as CUDA graphs.  Values cross the boundary as the grids' compact
arrays concatenated in grid order."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from ._lib import check
from .grid import _stream_handle


class Batch:
    def __init__(self, dims, levels, limits=None):
        self.dims = np.ascontiguousarray(dims, np.int32)
        self.levels = np.ascontiguousarray(levels, np.int32)
        if self.dims.shape != self.levels.shape or self.dims.ndim != 1:
            raise ValueError("dims and levels must be equal-length 1-D arrays")
        lim = None
        if limits is not None:
            self._lim = np.ascontiguousarray(np.concatenate([np.asarray(x, np.int32) for x in limits]), np.int32)
            if self._lim.size != int(self.dims.sum()):
                raise ValueError("limits must hold d entries per grid")
            lim = self._lim.ctypes.data
        h = C.c_void_p()
        check(L.lib().sg_batch_create(len(self.dims), self.dims.ctypes.data, self.levels.ctypes.data, lim,
                                      C.byref(h)))
        self._h = h
        self.num_grids = len(self.dims)
        off = np.zeros(self.num_grids + 1, np.int64)
        check(L.lib().sg_batch_offsets(h, off.ctypes.data))
        self.value_offsets = off
        self.num_values = int(off[-1])

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            L.lib().sg_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def set_option(self, option: int, value: int) -> None:
        check(L.lib().sg_batch_set_option(self._h, option, int(value)))

    def set_values(self, values) -> None:
        v = np.ascontiguousarray(values, np.float32)
        if v.shape != (self.num_values,):
            raise ValueError(f"expected {self.num_values} values")
        check(L.lib().sg_batch_set_values(self._h, v.ctypes.data))

    def set_values_device(self, values, stream=None) -> None:
        check(L.lib().sg_batch_set_values_device(self._h, int(values.data_ptr()), _stream_handle(stream)))

    def get_values(self) -> np.ndarray:
        out = np.empty(self.num_values, np.float32)
        check(L.lib().sg_batch_get_values(self._h, out.ctypes.data))
        return out

    def get_values_device(self, values, stream=None) -> None:
        check(L.lib().sg_batch_get_values_device(self._h, int(values.data_ptr()), _stream_handle(stream)))

    def grid_values(self, all_values, g: int) -> np.ndarray:
        return all_values[self.value_offsets[g]:self.value_offsets[g + 1]]

    def sample_function(self, fn: int, params=None, stream=None) -> None:
        if params is None:
            ptr, per = None, 0
        else:
            p = np.ascontiguousarray(params, np.float64)
            self._params = p
            ptr, per = p.ctypes.data, p.shape[1]
        check(L.lib().sg_batch_sample_function(self._h, int(fn), ptr, int(per), _stream_handle(stream)))

    def hierarchize(self) -> None:
        check(L.lib().sg_batch_hierarchize(self._h))

    def hierarchize_async(self, stream=None) -> None:
        check(L.lib().sg_batch_hierarchize_async(self._h, _stream_handle(stream)))

    def evaluate_device(self, point_offsets, coords, out, stream=None) -> None:
        po = np.ascontiguousarray(point_offsets, np.int64)
        if po.shape != (self.num_grids + 1,):
            raise ValueError("point_offsets needs num_grids + 1 entries")
        self._po = po
        check(L.lib().sg_batch_evaluate_device(self._h, po.ctypes.data, int(coords.data_ptr()),
                                               int(out.data_ptr()), _stream_handle(stream)))

    def sync(self, stream=None) -> None:
        check(L.lib().sg_batch_sync(self._h, _stream_handle(stream)))

    def autotune(self, point_offsets, coords, out, stream=None) -> np.ndarray:
        """sg_batch_autotune: per dimension, the fastest pair of points per
        thread (1, 2) and subspace blocking (1 wide, 2 medium) on
        these buffers; returns ms[blocking-1][ppt-1][d] (-1 = no grid of d)."""
        po = np.ascontiguousarray(point_offsets, np.int64)
        if po.shape != (self.num_grids + 1,):
            raise ValueError("point_offsets needs num_grids + 1 entries")
        self._po = po
        ms = np.zeros((L.SG_EVAL_BLOCKINGS, 2, L.SG_MAX_DIMS + 1), np.float64)
        check(L.lib().sg_batch_autotune(self._h, po.ctypes.data, int(coords.data_ptr()), int(out.data_ptr()),
                                        _stream_handle(stream), ms.ctypes.data))
        return ms

    def device_bytes(self) -> int:
        v = C.c_int64()
        check(L.lib().sg_batch_device_bytes(self._h, C.byref(v)))
        return v.value
