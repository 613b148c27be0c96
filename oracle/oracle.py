"""ctypes bindings for the CPU checkers (TEST INFRASTRUCTURE ONLY).

`Oracle` wraps this project's C restatement (``liboracle.so`` built from
``sg_oracle.c``); `Reference` wraps the reference benchmark's own C code
compiled in place (``_ref/libasgb_ref.so``).  Only the test suite, the smoke
check and the benchmark's CPU-baseline leg import this module; the product
library never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libasgb_ref.so")
REFCUDA_SO = os.path.join(HERE, "_ref", "libasgb_refcuda.so")

_i64 = C.c_int64
_fp = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


def build() -> None:
    """Compile the checkers (`make -C oracle`)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def _load(path: str) -> C.CDLL:
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is not built; run `make -C oracle`")
    return C.CDLL(path)


class Oracle:
    """The C restatement of the reference algorithm, one layout per object."""

    _lib = None

    @classmethod
    def lib(cls) -> C.CDLL:
        if cls._lib is None:
            lib = _load(ORACLE_SO)
            lib.or_layout_size.restype = C.c_int
            lib.or_layout_init.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p]
            lib.or_layout_init.restype = C.c_int
            lib.or_gp2idx.argtypes = [C.c_void_p, _ip, _ip]
            lib.or_gp2idx.restype = _i64
            lib.or_idx2gp.argtypes = [C.c_void_p, _i64, _ip, _ip]
            lib.or_idx2gp.restype = C.c_int
            lib.or_l2idx.argtypes = [C.c_void_p, _ip]
            lib.or_l2idx.restype = _i64
            lib.or_idx2l.argtypes = [C.c_void_p, _i64, C.c_int, _ip]
            lib.or_hierarchize_f32.argtypes = [C.c_void_p, _fp]
            lib.or_hierarchize_f64.argtypes = [C.c_void_p, _dp]
            lib.or_hierarchize_f64_fast.argtypes = [C.c_void_p, _dp]
            lib.or_evaluate_f32.argtypes = [C.c_void_p, _fp, _fp, _fp, _i64]
            lib.or_evaluate_f64.argtypes = [C.c_void_p, _dp, _fp, _dp, _i64]
            lib.or_evaluate_f64_par.argtypes = [C.c_void_p, _dp, _fp, _dp, _i64]
            lib.or_evaluate_f64_par.restype = C.c_int
            lib.or_grid_points.argtypes = [C.c_void_p, _fp]
            cls._lib = lib
        return cls._lib

    def __init__(self, d: int, n: int, limits=None):
        lib = self.lib()
        self._buf = C.create_string_buffer(lib.or_layout_size())
        lim = None
        if limits is not None:
            self._lim = np.ascontiguousarray(limits, dtype=np.int32)
            lim = self._lim.ctypes.data
        if lib.or_layout_init(self._buf, d, n, lim) != 0:
            raise ValueError(f"bad layout d={d} n={n} limits={limits}")
        self.d, self.n = d, n
        # or_layout: int d, n; int lim[32]; int64 dp[32][32]; int64 lidx[33]; int64 N, S
        raw = np.frombuffer(self._buf, dtype=np.uint8)
        off = 8 + 4 * 32
        self.dp = np.frombuffer(raw[off:off + 8 * 32 * 32].tobytes(), dtype=np.int64).reshape(32, 32)[:d, :n].copy()
        off += 8 * 32 * 32
        self.lidx = np.frombuffer(raw[off:off + 8 * 33].tobytes(), dtype=np.int64)[: n + 1].copy()
        off += 8 * 33
        self.N, self.S = (int(v) for v in np.frombuffer(raw[off:off + 16].tobytes(), dtype=np.int64))

    def gp2idx(self, lv, ix) -> int:
        return int(self.lib().or_gp2idx(self._buf, np.ascontiguousarray(lv, np.int32), np.ascontiguousarray(ix, np.int32)))

    def idx2gp(self, idx: int):
        lv = np.zeros(self.d, np.int32)
        ix = np.zeros(self.d, np.int32)
        if self.lib().or_idx2gp(self._buf, idx, lv, ix) != 0:
            raise IndexError(idx)
        return lv, ix

    def idx2l(self, pos: int, s: int):
        lv = np.zeros(self.d, np.int32)
        self.lib().or_idx2l(self._buf, pos, s, lv)
        return lv

    def l2idx(self, lv) -> int:
        return int(self.lib().or_l2idx(self._buf, np.ascontiguousarray(lv, np.int32)))

    def grid_points(self) -> np.ndarray:
        X = np.zeros((self.N, self.d), np.float32)
        self.lib().or_grid_points(self._buf, X)
        return X

    def hierarchize_f32(self, vals) -> np.ndarray:
        a = np.array(vals, dtype=np.float32, copy=True)
        self.lib().or_hierarchize_f32(self._buf, a)
        return a

    def hierarchize_f64(self, vals, fast: bool = True) -> np.ndarray:
        a = np.array(vals, dtype=np.float64, copy=True)
        (self.lib().or_hierarchize_f64_fast if fast else self.lib().or_hierarchize_f64)(self._buf, a)
        return a

    def evaluate_f32(self, surplus, X) -> np.ndarray:
        X = np.ascontiguousarray(X, np.float32).reshape(-1, self.d)
        out = np.zeros(X.shape[0], np.float32)
        self.lib().or_evaluate_f32(self._buf, np.ascontiguousarray(surplus, np.float32), X, out, X.shape[0])
        return out

    def evaluate_f64(self, surplus64, X, parallel: bool = True) -> np.ndarray:
        """FP64 interpolant at the rows of X; `parallel` splits the points
        over OpenMP threads with the subspaces' level vectors computed once
        (bit-identical to the serial restatement)."""
        X = np.ascontiguousarray(X, np.float32).reshape(-1, self.d)
        out = np.zeros(X.shape[0], np.float64)
        a = np.ascontiguousarray(surplus64, np.float64)
        if parallel and X.shape[0] > 1:
            if self.lib().or_evaluate_f64_par(self._buf, a, X, out, X.shape[0]) != 0:
                raise MemoryError("or_evaluate_f64_par")
        else:
            self.lib().or_evaluate_f64(self._buf, a, X, out, X.shape[0])
        return out


class Reference:
    """The reference benchmark's own C code (global state: one grid at a time)."""

    _lib = None

    @classmethod
    def available(cls) -> bool:
        return os.path.exists(REF_SO)

    @classmethod
    def lib(cls) -> C.CDLL:
        if cls._lib is None:
            lib = _load(REF_SO)
            lib.ref_init.argtypes = [C.c_int, C.c_int, C.c_void_p]
            lib.ref_tables.argtypes = [_ip, _ip]
            lib.ref_get_values.argtypes = [_fp]
            lib.ref_set_values.argtypes = [_fp]
            lib.ref_gp2idx.argtypes = [_ip, _ip]
            lib.ref_idx2gp.argtypes = [C.c_int, _ip, _ip]
            lib.ref_hierarchize.argtypes = [C.c_int]
            lib.ref_evaluate.argtypes = [C.c_int, _fp, _fp, C.c_int]
            cls._lib = lib
        return cls._lib

    def __init__(self, d: int, n: int, limits=None):
        lib = self.lib()
        lim = None
        if limits is not None:
            self._lim = np.ascontiguousarray(limits, dtype=np.int32)
            lim = self._lim.ctypes.data
        lib.ref_init(d, n, lim)
        self.d, self.n = d, n
        self.N = lib.ref_num_points()
        self.S = lib.ref_num_subspaces()

    def tables(self):
        dp = np.zeros(self.d * self.n, np.int32)
        lidx = np.zeros(self.n, np.int32)
        self.lib().ref_tables(dp, lidx)
        return dp.reshape(self.d, self.n), lidx

    def values(self) -> np.ndarray:
        v = np.zeros(self.N, np.float32)
        self.lib().ref_get_values(v)
        return v

    def set_values(self, v) -> None:
        self.lib().ref_set_values(np.ascontiguousarray(v, np.float32))

    def gp2idx(self, lv, ix) -> int:
        return int(self.lib().ref_gp2idx(np.array(lv, np.int32), np.array(ix, np.int32)))

    def idx2gp(self, idx: int):
        lv = np.zeros(self.d, np.int32)
        ix = np.zeros(self.d, np.int32)
        self.lib().ref_idx2gp(int(idx), lv, ix)
        return lv, ix

    def hierarchize(self, variant: int = 0) -> None:
        if self.lib().ref_hierarchize(variant) != 0:
            raise ValueError(variant)

    def evaluate(self, X, variant: int = 0, chunk: int = 16384) -> np.ndarray:
        X = np.ascontiguousarray(X, np.float32).reshape(-1, self.d)
        out = np.zeros(X.shape[0], np.float32)
        for s in range(0, X.shape[0], chunk):
            xs = np.ascontiguousarray(X[s:s + chunk])
            o = np.zeros(xs.shape[0], np.float32)
            self.lib().ref_evaluate(variant, xs, o, xs.shape[0])
            out[s:s + chunk] = o
        return out


class ReferenceCUDA:
    """The reference's CUDA kernels evaluate5 (adaptive_sparse_grid_bench_cuda.cu:1522)
    and hierarchize7 (cu:1053, with the warp barriers it lacks added by
    ``patch_ref_cuda.py``), compiled into ``_ref/libasgb_refcuda.so``; timed
    next to this project's kernels.  The harness refuses sizes outside each
    kernel's safe launch conditions before touching the GPU: for evaluate5
    P a multiple of 32, points a multiple of 8 P, n <= 10, d <= 20,
    coordinates in [0,1); for hierarchize7 6 <= n <= 10, d <= 20."""

    _lib = None

    @classmethod
    def available(cls) -> bool:
        return os.path.exists(REFCUDA_SO)

    @classmethod
    def lib(cls) -> C.CDLL:
        if cls._lib is None:
            lib = _load(REFCUDA_SO)
            lib.refcuda_evaluate5.argtypes = [C.c_int, C.c_int, _fp, C.c_int, _fp, C.c_int, C.c_int, C.c_int, _fp,
                                              C.POINTER(C.c_float), C.POINTER(C.c_float)]
            lib.refcuda_evaluate5.restype = C.c_int
            lib.refcuda_hierarchize7.argtypes = [C.c_int, C.c_int, _fp, C.c_int, C.c_int, _fp,
                                                 C.POINTER(C.c_float), C.POINTER(C.c_float)]
            lib.refcuda_hierarchize7.restype = C.c_int
            cls._lib = lib
        return cls._lib

    @classmethod
    def evaluate5(cls, d: int, n: int, surplus, X, points_per_warp: int, reps: int = 1):
        """Returns (out, fastest kernel ms, fastest copy-inclusive ms)."""
        a = np.ascontiguousarray(surplus, np.float32)
        X = np.ascontiguousarray(X, np.float32).reshape(-1, d)
        out = np.zeros(X.shape[0], np.float32)
        tk, tt = C.c_float(), C.c_float()
        r = cls.lib().refcuda_evaluate5(d, n, a, a.size, X, X.shape[0], points_per_warp, reps, out, C.byref(tk),
                                        C.byref(tt))
        if r != 0:
            raise RuntimeError(f"refcuda_evaluate5 returned {r}")
        return out, tk.value, tt.value

    @classmethod
    def hierarchize7(cls, d: int, n: int, values, reps: int = 1):
        """Hierarchizes the nodal values (compact order) with the reference's
        hierarchize7, one launch per dimension as its main() does.  Returns
        (surpluses, fastest kernel ms, fastest ms with the copy in)."""
        a = np.ascontiguousarray(values, np.float32)
        out = np.zeros(a.size, np.float32)
        tk, tt = C.c_float(), C.c_float()
        r = cls.lib().refcuda_hierarchize7(d, n, a, a.size, reps, out, C.byref(tk), C.byref(tt))
        if r != 0:
            raise RuntimeError(f"refcuda_hierarchize7 returned {r}")
        return out, tk.value, tt.value
