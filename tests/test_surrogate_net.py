"""Surrogate network kernels: the tcgen05 GEMM with its epilogues, forward,
backward and Adam training on the device, against the CPU oracle
(oracle/mlp_oracle.py).

CPU: the oracle's analytic gradients against central finite differences
(float64), its bf16 rounding, and argument checks of the C ABI.
GPU: every GEMM epilogue against numpy on bf16 inputs; device gradients
against the oracle on the same parameters and data (bf16 rounding
emulated); training lowers the loss; device predictions against the
oracle's forward pass."""

from __future__ import annotations

import ctypes
import importlib

import numpy as np
import pytest

import mlp_oracle as mo

pkg = importlib.import_module("3d_mpi_test_b200")
sur = importlib.import_module("3d_mpi_test_b200.surrogate")


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-300))


# ------------------------------------------------------------------ CPU
def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    dims = mo.layer_dims(5, 8, 2, 3)
    p = rng.standard_normal(sum(n * k + n for n, k in dims)) * 0.5
    X, T = rng.standard_normal((6, 5)), rng.standard_normal((6, 3))
    _, g = mo.loss_and_grads(p, dims, X, T, emulate=False)
    idx = rng.choice(len(p), 40, replace=False)
    fd = mo.finite_difference(p, dims, X, T, idx)
    np.testing.assert_allclose(g[idx], fd, rtol=1e-6, atol=1e-9)


def test_bf16_rounding():
    x = np.array([1.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -9, -2.5, 1e-40, 3.0e38], np.float32)
    r = mo.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0  # tie to even
    assert r[2] == np.float32(1.0 + 2.0 ** -7)
    assert r[3] == -2.5 and np.isfinite(r[5])
    assert np.all(mo.bf16(r) == r)


def test_surrogate_argument_checks():
    L = sur._lib()
    assert L.fdtd_net_create(0, 11, 512, 4, 136, 256, 0, None) == pkg.FDTD_ERR_ARG
    assert L.fdtd_net_destroy(None) == pkg.FDTD_OK
    # sizes are checked before any device work
    assert L.fdtd_tc_gemm(0, 0, 100, 64, 64, ctypes.c_void_p(16), ctypes.c_void_p(16), None, None,
                          ctypes.c_void_p(16), None, None) == pkg.FDTD_ERR_ARG
    assert L.fdtd_tc_gemm(0, 1, 128, 64, 64, ctypes.c_void_p(16), ctypes.c_void_p(16), None, None,
                          ctypes.c_void_p(16), None, None) == pkg.FDTD_ERR_ARG  # bias missing


# ------------------------------------------------------------------ GPU
def _bf(t):
    import torch

    return torch.from_numpy(t).to(torch.bfloat16).cuda()


@pytest.mark.gpu
@pytest.mark.parametrize("M,N,K", [(128, 64, 64), (256, 128, 128), (384, 192, 320), (128, 512, 512),
                                   (1024, 256, 576), (8192, 512, 512), (32768, 512, 64), (20480, 192, 128)])
def test_tc_gemm_matches_numpy(M, N, K):
    """Small and large products: from one tile per CTA up to several tiles
    per persistent CTA (both tensor-memory accumulators, wrapped phases)."""
    import torch

    rng = np.random.default_rng(M + N + K)
    A = mo.bf16(rng.standard_normal((M, K)).astype(np.float32))
    B = mo.bf16(rng.standard_normal((N, K)).astype(np.float32))
    bias = rng.standard_normal(N).astype(np.float32)
    ref = A.astype(np.float64) @ B.astype(np.float64).T
    At, Bt, bt = _bf(A), _bf(B), torch.from_numpy(bias).cuda()
    out = torch.empty((M, N), dtype=torch.float32, device="cuda")
    sur.tc_gemm(sur.EPI_F32, At, Bt, out)
    assert rel(out.cpu().numpy(), ref) < 1e-5
    sur.tc_gemm(sur.EPI_BIAS_F32, At, Bt, out, bias=bt)
    assert rel(out.cpu().numpy(), ref + bias) < 1e-5
    h = torch.empty((M, N), dtype=torch.bfloat16, device="cuda")
    hT = torch.empty((N, M), dtype=torch.bfloat16, device="cuda")
    sur.tc_gemm(sur.EPI_BIAS_RELU_T, At, Bt, h, bias=bt, outT=hT)
    want = np.maximum(ref + bias, 0)
    hn = h.float().cpu().numpy()
    assert rel(hn, want) < 5e-3  # bf16 output
    assert np.array_equal(hT.float().cpu().numpy(), hn.T)
    h2 = torch.empty_like(h)
    sur.tc_gemm(sur.EPI_BIAS_RELU, At, Bt, h2, bias=bt)
    assert torch.equal(h, h2)
    mask = _bf(mo.bf16(rng.standard_normal((M, N)).astype(np.float32)))
    g = torch.empty_like(h)
    gT = torch.empty_like(hT)
    sur.tc_gemm(sur.EPI_RELU_GRAD_T, At, Bt, g, mask=mask, outT=gT)
    want = ref * (mask.float().cpu().numpy() > 0)
    gn = g.float().cpu().numpy()
    assert rel(gn, want) < 5e-3 and np.all(gn[mask.float().cpu().numpy() <= 0] == 0)
    assert np.array_equal(gT.float().cpu().numpy(), gn.T)


def _data(n, n_in, n_out, seed):
    rng = np.random.default_rng(seed)
    X = rng.uniform(-1, 1, (n, n_in)).astype(np.float32) * np.linspace(1, 5, n_in, dtype=np.float32) + 2.0
    Wt = rng.standard_normal((n_in, n_out)).astype(np.float32)
    T = (np.sin(X @ Wt * 0.3) + 0.1 * (X ** 2) @ Wt[:, ::-1] * 0.05).astype(np.float32)
    return X, T


@pytest.mark.gpu
@pytest.mark.parametrize("width,hidden,n_out", [(128, 1, 10), (256, 3, 136), (512, 4, 136)])
def test_device_gradients_match_oracle(width, hidden, n_out):
    X, T = _data(256, 11, n_out, 1)
    with sur.Net(11, n_out, width=width, hidden=hidden, batch=128, seed=3) as net:
        net.set_data(X, T)
        im, is_, om, os_ = net.normalization()
        loss, g = net.gradients()
        p = net.params()
    dims = mo.layer_dims(11, width, hidden, n_out)
    Xn = mo.normalise(X[:128], im, is_)
    Tn = ((T[:128] - om) / os_).astype(np.float32)
    lo, go = mo.loss_and_grads(p, dims, Xn, Tn, emulate=True)
    assert loss == pytest.approx(lo, rel=2e-3)
    o = 0
    for n, k in dims:
        gw, gb = g[o:o + n * k], g[o + n * k:o + n * k + n]
        ow, ob = go[o:o + n * k], go[o + n * k:o + n * k + n]
        assert rel(gw, ow) < 2e-2, (n, k, rel(gw, ow))
        assert rel(gb, ob) < 2e-2, (n, rel(gb, ob))
        o += n * k + n


@pytest.mark.gpu
def test_training_lowers_loss_and_predictions_match_oracle():
    import torch

    X, T = _data(4096, 11, 136, 2)
    with sur.Net(11, 136, width=512, hidden=4, batch=256, seed=5) as net:
        net.set_data(X, T)
        first = net.train(1, lr=1e-3, lr_final=1e-3, report=1)
        net.set_data(X, T)
        last = net.train(600, lr=2e-3, lr_final=1e-4, seed=1, report=50)
        assert last < 0.2 * first, (first, last)
        Xq = X[:1000] + 0.01
        Y = net.predict(Xq)
        im, is_, om, os_ = net.normalization()
        p = net.params()
        yo, _ = mo.forward(p, mo.layer_dims(11, 512, 4, 136), mo.normalise(Xq, im, is_), emulate=True)
        yo = yo * os_ + om
        assert rel(Y, yo) < 1e-2
        # device-buffer path agrees with the host path
        xd = torch.from_numpy(Xq).cuda()
        yd = torch.empty((1000, 136), dtype=torch.float32, device="cuda")
        net.predict_device(xd.data_ptr(), 1000, yd.data_ptr())
        torch.cuda.synchronize()
        assert np.array_equal(yd.cpu().numpy(), Y)
        info = net.info()
        assert info["launches"] > 600 and info["last_device_ms"] > 0


@pytest.mark.gpu
def test_inference_across_chunks_matches_single_rows():
    """Queries spanning several inference passes (65,536 rows each) and a
    ragged last pass give the same answers as the same rows on their own."""
    X, T = _data(2048, 11, 136, 4)
    with sur.Net(11, 136, width=512, hidden=4, batch=256, seed=9) as net:
        net.set_data(X, T)
        net.train(50, lr=1e-3, lr_final=1e-3)
        Xq = np.tile(X, (70000 // len(X) + 1, 1))[:70000] + np.linspace(0, 1, 70000, dtype=np.float32)[:, None]
        Y = net.predict(Xq)
        for r0 in (0, 65530, 69990):
            np.testing.assert_array_equal(net.predict(Xq[r0:r0 + 10]), Y[r0:r0 + 10])
        assert net.predict(np.zeros((0, 11), np.float32)).shape == (0, 136)


@pytest.mark.gpu
@pytest.mark.parametrize("hidden", [4, 2])
def test_fused_inference_matches_layer_gemms(hidden):
    """The fused inference kernel (all layers in one persistent launch,
    activations in shared and tensor memory) gives the answers of the
    per-layer GEMMs: the same bf16 rounding points and the same K order."""
    X, T = _data(2048, 11, 136, 5)
    with sur.Net(11, 136, width=512, hidden=hidden, batch=256, seed=3) as net:
        net.set_data(X, T)
        net.train(40, lr=1e-3, lr_final=1e-3)
        Xq = np.tile(X, (9000 // len(X) + 1, 1))[:9000] + np.linspace(0, 1, 9000, dtype=np.float32)[:, None]
        assert net.set_fused(False)  # the shapes fit the fused kernel
        l0 = net.info()["launches"]
        Y_layers = net.predict(Xq)
        per_layers = net.info()["launches"] - l0
        net.set_fused(True)
        l0 = net.info()["launches"]
        Y_fused = net.predict(Xq)
        per_fused = net.info()["launches"] - l0
    assert per_fused == 2 and per_layers == 2 + hidden + 1  # pack + network (+ denormalise)
    scale = np.abs(Y_layers).max()
    assert np.abs(Y_fused - Y_layers).max() <= 1e-5 * scale, np.abs(Y_fused - Y_layers).max()


@pytest.mark.gpu
def test_fused_inference_declines_other_shapes():
    X, T = _data(512, 11, 20, 6)
    with sur.Net(11, 20, width=256, hidden=2, batch=256, seed=4) as net:
        net.set_data(X, T)
        assert not net.set_fused(True)  # width 256: the per-layer GEMMs serve it
        Y = net.predict(X[:300])
        assert Y.shape == (300, 20) and np.all(np.isfinite(Y))
