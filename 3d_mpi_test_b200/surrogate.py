"""Surrogate network host API (C ABI in include/fdtd_surrogate.h).

:class:`Net` is one ReLU MLP trained and evaluated on the device by the
library's own tensor-core kernels (bf16 weights and activations, FP32
accumulation, FP32 Adam masters). :func:`tc_gemm` exposes the tensor-core
GEMM with its epilogues on device buffers (torch CUDA tensors). There is
no CPU path: without the native library every call fails.
"""

from __future__ import annotations

import ctypes
from typing import Optional, Tuple

import numpy as np

from . import FDTD_ERR_ARG, FdtdError, load_library

EPI_F32, EPI_BIAS_RELU_T, EPI_BIAS_F32, EPI_RELU_GRAD_T, EPI_BIAS_RELU = 0, 1, 2, 3, 4

_FP = ctypes.POINTER(ctypes.c_float)


def _declare(L) -> None:
    if getattr(L, "_surrogate_declared", False):
        return
    vp, i, f, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.POINTER(ctypes.c_double)
    ull, ll = ctypes.c_ulonglong, ctypes.POINTER(ctypes.c_longlong)
    sig = {
        "fdtd_tc_gemm": ([i, i, i, i, i, vp, vp, vp, vp, vp, vp, vp], i),
        "fdtd_net_create": ([i, i, i, i, i, i, ull, ctypes.POINTER(vp)], i),
        "fdtd_net_destroy": ([vp], i),
        "fdtd_net_n_params": ([vp, ctypes.POINTER(i)], i),
        "fdtd_net_get_params": ([vp, _FP], i),
        "fdtd_net_set_params": ([vp, _FP], i),
        "fdtd_net_set_data": ([vp, _FP, _FP, i], i),
        "fdtd_net_get_normalization": ([vp, _FP, _FP, _FP, _FP], i),
        "fdtd_net_set_normalization": ([vp, _FP, _FP, _FP, _FP], i),
        "fdtd_net_train": ([vp, i, f, f, ull, i, d], i),
        "fdtd_net_gradients": ([vp, _FP, d], i),
        "fdtd_net_predict": ([vp, _FP, i, _FP], i),
        "fdtd_net_predict_device": ([vp, vp, i, vp, vp], i),
        "fdtd_net_info": ([vp, ll, d], i),
    }
    for name, (args, res) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    L._surrogate_declared = True


def _lib(lib_path: Optional[str] = None):
    L = load_library(lib_path)
    _declare(L)
    return L


def _check(L, rc: int) -> None:
    if rc < 0:
        raise FdtdError(rc, L.fdtd_last_error().decode())


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


def _fp(a: np.ndarray):
    return a.ctypes.data_as(_FP)


def tc_gemm(epilogue: int, A, B, out, bias=None, mask=None, outT=None, device: int = 0,
            lib_path: Optional[str] = None) -> None:
    """out = epilogue(A . B^T) on device tensors: A [M][K], B [N][K] bf16
    contiguous; out [M][N] (FP32 for EPI_F32 / EPI_BIAS_F32, else bf16);
    outT [N][M] bf16; bias [N] FP32; mask [M][N] bf16."""
    L = _lib(lib_path)
    M, K = A.shape
    N = B.shape[0]
    if B.shape[1] != K:
        raise FdtdError(FDTD_ERR_ARG, "A and B disagree on K")
    ptr = (lambda t: ctypes.c_void_p(t.data_ptr()) if t is not None else None)
    _check(L, L.fdtd_tc_gemm(device, epilogue, M, N, K, ptr(A), ptr(B), ptr(bias), ptr(mask), ptr(out), ptr(outT),
                             None))


class Net:
    """One surrogate network: n_in -> hidden x width (ReLU) -> n_out."""

    def __init__(self, n_in: int, n_out: int, width: int = 512, hidden: int = 4, batch: int = 256, seed: int = 0,
                 device: int = 0, lib_path: Optional[str] = None):
        self._L = _lib(lib_path)
        self._h = ctypes.c_void_p()
        _check(self._L, self._L.fdtd_net_create(device, n_in, width, hidden, n_out, batch, seed,
                                                ctypes.byref(self._h)))
        self.n_in, self.n_out, self.width, self.hidden, self.batch = n_in, n_out, width, hidden, batch
        n = ctypes.c_int()
        _check(self._L, self._L.fdtd_net_n_params(self._h, ctypes.byref(n)))
        self.n_params = n.value

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            self._L.fdtd_net_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def dims(self):
        """(N, K) of every layer's weight matrix."""
        return [(self.n_out if l == self.hidden else self.width, self.n_in if l == 0 else self.width)
                for l in range(self.hidden + 1)]

    def params(self) -> np.ndarray:
        p = np.empty(self.n_params, np.float32)
        _check(self._L, self._L.fdtd_net_get_params(self._h, _fp(p)))
        return p

    def set_params(self, p) -> None:
        p = _f32(p)
        if p.size != self.n_params:
            raise FdtdError(FDTD_ERR_ARG, "parameter count mismatch")
        _check(self._L, self._L.fdtd_net_set_params(self._h, _fp(p)))

    def set_data(self, X, T) -> None:
        X, T = _f32(X), _f32(T)
        if X.ndim != 2 or X.shape[1] != self.n_in or T.shape != (X.shape[0], self.n_out):
            raise FdtdError(FDTD_ERR_ARG, "data must be X [n][n_in], T [n][n_out]")
        _check(self._L, self._L.fdtd_net_set_data(self._h, _fp(X), _fp(T), X.shape[0]))

    def normalization(self) -> Tuple[np.ndarray, np.ndarray, np.ndarray, np.ndarray]:
        im, is_ = np.empty(self.n_in, np.float32), np.empty(self.n_in, np.float32)
        om, os_ = np.empty(self.n_out, np.float32), np.empty(self.n_out, np.float32)
        _check(self._L, self._L.fdtd_net_get_normalization(self._h, _fp(im), _fp(is_), _fp(om), _fp(os_)))
        return im, is_, om, os_

    def set_normalization(self, in_mean, in_std, out_mean, out_std) -> None:
        a, b, c, d = _f32(in_mean), _f32(in_std), _f32(out_mean), _f32(out_std)
        _check(self._L, self._L.fdtd_net_set_normalization(self._h, _fp(a), _fp(b), _fp(c), _fp(d)))

    def train(self, steps: int, lr: float = 1e-3, lr_final: float = 1e-5, seed: int = 0, report: int = 100) -> float:
        loss = ctypes.c_double()
        _check(self._L, self._L.fdtd_net_train(self._h, steps, lr, lr_final, seed, report, ctypes.byref(loss)))
        return loss.value

    def gradients(self) -> Tuple[float, np.ndarray]:
        g = np.empty(self.n_params, np.float32)
        loss = ctypes.c_double()
        _check(self._L, self._L.fdtd_net_gradients(self._h, _fp(g), ctypes.byref(loss)))
        return loss.value, g

    def predict(self, X) -> np.ndarray:
        X = _f32(np.atleast_2d(X))
        Y = np.empty((X.shape[0], self.n_out), np.float32)
        _check(self._L, self._L.fdtd_net_predict(self._h, _fp(X), X.shape[0], _fp(Y)))
        return Y

    def predict_device(self, X_ptr: int, n: int, Y_ptr: int, stream: int = 0) -> None:
        """Inference on device buffers X [n][n_in], Y [n][n_out] (FP32)."""
        _check(self._L, self._L.fdtd_net_predict_device(self._h, ctypes.c_void_p(X_ptr), n, ctypes.c_void_p(Y_ptr),
                                                        ctypes.c_void_p(stream) if stream else None))

    def info(self) -> dict:
        n, ms = ctypes.c_longlong(), ctypes.c_double()
        _check(self._L, self._L.fdtd_net_info(self._h, ctypes.byref(n), ctypes.byref(ms)))
        return {"launches": n.value, "last_device_ms": ms.value}
