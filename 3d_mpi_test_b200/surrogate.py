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
from .surrogate_data import N_REC, PARAMS, features

# query-row geometry of the ray features: (n_par, col_hs, col_hr, col_range, n_rec)
RAYS = (len(PARAMS), PARAMS.index("source_height"), PARAMS.index("receiver_height"), PARAMS.index("range"), N_REC)

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
        "fdtd_net_train": ([vp, i, f, f, f, ull, i, d], i),
        "fdtd_net_gradients": ([vp, _FP, d], i),
        "fdtd_net_predict": ([vp, _FP, i, _FP], i),
        "fdtd_net_predict_device": ([vp, vp, i, vp, vp], i),
        "fdtd_net_info": ([vp, ll, d], i),
        "fdtd_net_set_fused": ([vp, i, ctypes.POINTER(i)], i),
        "fdtd_net_ensemble_predict": ([ctypes.POINTER(vp), i, _FP, i, _FP, _FP], i),
        "fdtd_ray_features": ([vp, i, i, i, i, i, i, vp, vp], i),
        "fdtd_net_ensemble_predict_rays": ([ctypes.POINTER(vp), i, _FP, i, i, i, i, i, i, _FP, _FP], i),
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


def ray_features(P_ptr: int, n: int, F_ptr: int, stream: int = 0, lib_path: Optional[str] = None) -> None:
    """Network inputs F [n][27] (device) of query rows P [n][11] (device):
    ``surrogate_data.features`` formed on the device, on a stream."""
    L = _lib(lib_path)
    _check(L, L.fdtd_ray_features(P_ptr, n, *RAYS, F_ptr, stream))


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

    def train(self, steps: int, lr: float = 1e-3, lr_final: float = 1e-5, seed: int = 0, report: int = 100,
              weight_decay: float = 0.0) -> float:
        loss = ctypes.c_double()
        _check(self._L, self._L.fdtd_net_train(self._h, steps, lr, lr_final, weight_decay, seed, report,
                                               ctypes.byref(loss)))
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

    def set_fused(self, on: bool = True) -> bool:
        """Inference by one fused kernel for all layers (default) or one GEMM
        per layer; returns whether the fused kernel serves this network."""
        served = ctypes.c_int()
        _check(self._L, self._L.fdtd_net_set_fused(self._h, int(on), ctypes.byref(served)))
        return bool(served.value)

    def info(self) -> dict:
        n, ms = ctypes.c_longlong(), ctypes.c_double()
        _check(self._L, self._L.fdtd_net_info(self._h, ctypes.byref(n), ctypes.byref(ms)))
        return {"launches": n.value, "last_device_ms": ms.value}


class Surrogate:
    """Ensemble of networks that answers excess-attenuation queries, with
    the FDTD solver as its fallback.

    Inputs: the 11 parameters of ``surrogate_data.PARAMS`` (flow
    resistivity as log10, porosity, tortuosity, layer depth, source and
    receiver heights, range, hill height and half-width, u*, z0); the
    networks see them with the receivers' ray geometry appended
    (``surrogate_data.features``, 27 inputs). Outputs: excess attenuation
    [n_rec][n_band] in dB (``surrogate_data`` layout).
    Each member is trained on a bootstrap resample of the data from its own
    initialisation. A query is answered by the FDTD solver instead of the
    networks when it lies outside the training hull (the per-parameter
    range of the training inputs) or when the members disagree: the root
    mean square over the outputs of the standard deviation across members
    exceeds ``tol_db``.
    """

    def __init__(self, members: int = 5, width: int = 512, hidden: int = 4, batch: int = 256, seed: int = 0,
                 device: int = 0, lib_path: Optional[str] = None):
        self.members, self.width, self.hidden, self.batch = members, width, hidden, batch
        self.seed, self.device, self._lib_path = seed, device, lib_path
        self.nets = []
        self.lo = self.hi = None

    def close(self) -> None:
        for n in self.nets:
            n.close()
        self.nets = []

    def fit(self, X, EA, steps: int = 12000, lr: float = 2e-3, lr_final: float = 2e-5,
            weight_decay: float = 0.1) -> list:
        """Trains every member; returns their final training losses (mean
        squared error of the normalised outputs)."""
        X = np.asarray(X, np.float32)
        EA = np.asarray(EA, np.float32)
        ok = np.isfinite(EA).all(axis=1) & np.isfinite(X).all(axis=1)
        X, EA = X[ok], EA[ok]
        self.lo, self.hi = X.min(axis=0), X.max(axis=0)
        F = features(X)
        self.close()
        losses = []
        rng = np.random.default_rng(self.seed)
        for m in range(self.members):
            net = Net(F.shape[1], EA.shape[1], width=self.width, hidden=self.hidden, batch=self.batch,
                      seed=self.seed * 1000 + m, device=self.device, lib_path=self._lib_path)
            pick = rng.integers(0, len(X), len(X))  # bootstrap resample
            net.set_data(F[pick], EA[pick])
            losses.append(net.train(steps, lr=lr, lr_final=lr_final, seed=self.seed * 1000 + m, report=100,
                                    weight_decay=weight_decay))
            self.nets.append(net)
        return losses

    def in_hull(self, X) -> np.ndarray:
        X = np.atleast_2d(np.asarray(X, np.float32))
        return np.all((X >= self.lo) & (X <= self.hi), axis=1)

    def predict(self, X) -> Tuple[np.ndarray, np.ndarray]:
        """Member mean [n][outputs] and the disagreement [n] (root mean
        square over the outputs of the standard deviation across members, dB)
        of the parameter rows X [n][11]."""
        if not self.nets or not isinstance(self.nets[0], Net):  # stand-in members (tests) see the parameters
            ys = np.stack([n.predict(X) for n in self.nets])
            return ys.mean(axis=0), np.sqrt(ys.var(axis=0).mean(axis=1))
        X = _f32(np.atleast_2d(X))
        if X.shape[1] != len(PARAMS):
            raise FdtdError(FDTD_ERR_ARG, f"queries need {len(PARAMS)} parameters per row")
        net0 = self.nets[0]
        mean = np.empty((X.shape[0], net0.n_out), np.float32)
        spread = np.empty(X.shape[0], np.float32)
        arr = (ctypes.c_void_p * len(self.nets))(*[n._h.value for n in self.nets])
        _check(net0._L, net0._L.fdtd_net_ensemble_predict_rays(arr, len(self.nets), _fp(X), X.shape[0], *RAYS,
                                                               _fp(mean), _fp(spread)))
        return mean, spread

    def query(self, X, tol_db: float = 1.0, fdtd=None) -> Tuple[np.ndarray, np.ndarray]:
        """Answers [n][outputs] and the source of each answer: 0 network,
        1 FDTD (outside the hull), 2 FDTD (members disagree). ``fdtd`` maps
        inputs [k][11] to excess attenuation [k][outputs]; the default runs
        ``surrogate_data.solve``."""
        X = np.atleast_2d(np.asarray(X, np.float32))
        y, spread = self.predict(X)
        src = np.zeros(len(X), np.int8)
        src[spread > tol_db] = 2
        src[~self.in_hull(X)] = 1
        fall = np.nonzero(src)[0]
        if len(fall):
            if fdtd is None:
                from .surrogate_data import solve

                def fdtd(xs):
                    return solve(xs, device=self.device)
            y[fall] = fdtd(X[fall])
        return y, src
