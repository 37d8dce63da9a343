"""CPU restatement of the surrogate network -- TEST INFRASTRUCTURE ONLY.

Only the tests, ``__graft_entry__.smoke()`` and the CPU baseline of the
benchmark may use this module, as the checker of the device network
(3d_mpi_test_b200/csrc/mlp.cu, mlp_tc.cuh). The reference repository has no
network, so there is nothing to pin it to. This restatement is checked
instead by central finite differences of its own loss (exact float64
arithmetic, ``emulate=False``).

With ``emulate=True`` it rounds to bf16 where the device does:
- the normalised inputs;
- the weights;
- the hidden activations after the ReLU;
- the loss gradient dY and every masked hidden gradient dZ.
Accumulations run in float64, against the device's FP32 accumulation in
tensor memory.

Network: h_0 = x; h_{l+1} = relu(W_l h_l + b_l) for the hidden layers;
y = W_L h_L + b_L. Loss = mean over the batch and the n_out outputs of
(y - t)^2. Parameters flat, layer by layer: W [N][K] row-major, then b [N]
(the order of fdtd_net_get_params).
"""

from __future__ import annotations

import numpy as np


def bf16(x: np.ndarray) -> np.ndarray:
    """Round float32 values to the nearest bf16 (ties to even), returned as
    float32."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32).copy()
    nan = np.isnan(a)
    out[nan] = a[nan]
    return out


def layer_dims(n_in: int, width: int, hidden: int, n_out: int):
    dims = []
    for l in range(hidden + 1):
        k = n_in if l == 0 else width
        n = n_out if l == hidden else width
        dims.append((n, k))
    return dims


def unpack(p: np.ndarray, dims):
    Ws, bs, o = [], [], 0
    for n, k in dims:
        Ws.append(np.asarray(p[o:o + n * k], dtype=np.float64).reshape(n, k))
        o += n * k
        bs.append(np.asarray(p[o:o + n], dtype=np.float64))
        o += n
    assert o == len(p)
    return Ws, bs


def pack(Ws, bs) -> np.ndarray:
    return np.concatenate([np.concatenate([W.ravel(), b]) for W, b in zip(Ws, bs)])


def _r(x, emulate):
    """bf16 rounding of float32 x when emulating the device; exact float64
    otherwise."""
    return bf16(np.asarray(x, np.float32)).astype(np.float64) if emulate else np.asarray(x, dtype=np.float64)


def forward(p, dims, Xn, emulate=True):
    """Outputs y [B][n_out] and the hidden activations (bf16-rounded when
    emulating) for normalised inputs Xn [B][n_in]."""
    Ws, bs = unpack(p, dims)
    h = _r(Xn, emulate)
    hs = [h]
    for l in range(len(dims) - 1):
        z = h @ _r(Ws[l], emulate).T + bs[l]
        h = _r(np.maximum(z, 0.0), emulate)
        hs.append(h)
    y = h @ _r(Ws[-1], emulate).T + bs[-1]
    return y, hs


def loss_and_grads(p, dims, Xn, Tn, emulate=True):
    """Mean squared error and its gradient with respect to the flat
    parameters (backward pass in the device's order and rounding)."""
    Ws, bs = unpack(p, dims)
    y, hs = forward(p, dims, Xn, emulate)
    B, nout = Tn.shape
    d = y - Tn
    loss = float(np.sum(d * d) / (B * nout))
    g = 2.0 * d / (B * nout)
    g = _r(g, emulate)
    gW, gb = [None] * len(dims), [None] * len(dims)
    for l in range(len(dims) - 1, -1, -1):
        gW[l] = g.T @ hs[l]
        gb[l] = g.sum(axis=0)
        if l > 0:
            dh = g @ _r(Ws[l], emulate)
            g = _r(dh * (hs[l] > 0), emulate)
    return loss, pack(gW, gb)


def finite_difference(p, dims, Xn, Tn, idx, eps=1e-6):
    """Central differences of the exact (float64) loss at parameters idx."""
    out = []
    for i in idx:
        q = np.array(p, dtype=np.float64)
        q[i] += eps
        lp, _ = loss_and_grads(q, dims, Xn, Tn, emulate=False)
        q[i] -= 2 * eps
        lm, _ = loss_and_grads(q, dims, Xn, Tn, emulate=False)
        out.append((lp - lm) / (2 * eps))
    return np.array(out)


def normalise(X, mean, std):
    return ((np.asarray(X, np.float32) - np.asarray(mean, np.float32)) * (np.float32(1) / np.asarray(std, np.float32))
            ).astype(np.float32)
