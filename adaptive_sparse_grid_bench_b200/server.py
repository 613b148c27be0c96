"""The serving loop over the C ABI (sg_server_*): resident grids under an HBM
cap with LRU eviction, and a dispatcher thread in the library that batches
evaluate requests continuously.  Requests are host numpy arrays; submit()
returns a ticket, wait() the latency in milliseconds."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from ._lib import check

STATS = ("batches", "requests", "points", "evictions", "resident_grids", "bytes_in_use", "failed")


class Server:
    def __init__(self, hbm_cap_bytes: int, max_batch_points: int = 1 << 20):
        h = C.c_void_p()
        check(L.lib().sg_server_create(int(hbm_cap_bytes), int(max_batch_points), C.byref(h)))
        self._h = h
        self._keep = {}  # ticket -> (coords, out): buffers stay alive until waited

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            L.lib().sg_server_destroy(self._h)
            self._h = C.c_void_p()
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_option(self, option: int, value: int) -> None:
        check(L.lib().sg_server_set_option(self._h, int(option), int(value)))

    def add_grid(self, d: int, n: int, fn: int, params=(), limits=None) -> int:
        p = np.ascontiguousarray(params, np.float64)
        lim = None if limits is None else np.ascontiguousarray(limits, np.int32)
        gid = C.c_int64()
        check(L.lib().sg_server_add_grid(self._h, int(d), int(n), lim.ctypes.data if lim is not None else None,
                                         int(fn), p.ctypes.data if p.size else None, int(p.size), C.byref(gid)))
        return gid.value

    def submit(self, grid_id: int, coords: np.ndarray, out: np.ndarray | None = None) -> int:
        x = np.ascontiguousarray(coords, np.float32)
        m = x.shape[0]
        if out is None:
            out = np.empty(m, np.float32)
        t = C.c_int64()
        check(L.lib().sg_server_submit(self._h, int(grid_id), x.ctypes.data, int(m), out.ctypes.data, C.byref(t)))
        self._keep[t.value] = (x, out)
        return t.value

    def wait(self, ticket: int):
        lat = C.c_double()
        try:
            check(L.lib().sg_server_wait(self._h, int(ticket), C.byref(lat)))
        finally:
            _, out = self._keep.pop(ticket, (None, None))
        return out, lat.value

    def wait_detail(self, ticket: int):
        """(results, timeline): timeline = ms from submit to taken into a
        batch, to launches issued, to completion seen, to results delivered,
        and the request's point x subspace pairs."""
        ms = np.zeros(5, np.float64)
        try:
            check(L.lib().sg_server_wait_detail(self._h, int(ticket), ms.ctypes.data))
        finally:
            _, out = self._keep.pop(ticket, (None, None))
        return out, {"take_ms": ms[0], "launch_ms": ms[1], "gpu_ms": ms[2], "pairs": ms[3], "latency_ms": ms[4]}

    def evaluate_now(self, grid_id: int, coords: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(coords, np.float32)
        out = np.empty(x.shape[0], np.float32)
        check(L.lib().sg_server_evaluate_now(self._h, int(grid_id), x.ctypes.data, x.shape[0], out.ctypes.data))
        return out

    def stats(self) -> dict:
        v = np.zeros(len(STATS), np.int64)
        check(L.lib().sg_server_stats(self._h, v.ctypes.data))
        return dict(zip(STATS, (int(x) for x in v)))
