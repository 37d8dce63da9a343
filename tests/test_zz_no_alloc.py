"""The allocation-free entry point fdtd_fb_step_noalloc, for callers that
cannot allocate device memory themselves (for example a host that owns all
device memory through its own pool and hands the library finished buffers).

It must reproduce the handle-based path (fdtd_create + fdtd_step_pressure +
fdtd_step_velocity) on the same rigid-box case, on two calls in a row, within
the parity tolerances used elsewhere (FP64 relative L2 <= 1e-10, FP32 <=
1e-4), and in FP64 the oracle's fields after the two steps.  The test allocates the caller's buffers itself (with torch); the
entry point allocates nothing.  This file is collected last on purpose."""

import ctypes
import importlib

import numpy as np
import pytest

import cases
import oracle

pkg = importlib.import_module("3d_mpi_test_b200")

pytestmark = pytest.mark.gpu


def rel_l2(x, y):
    n = np.linalg.norm(y)
    return float(np.linalg.norm(x - y) / n) if n > 0 else float(np.linalg.norm(x - y))


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


@pytest.mark.parametrize("precision,tol", [("f64", 1e-10), ("f32", 1e-4)])
def test_noalloc_matches_handle_path_on_two_calls(precision, tol, tmp_path):
    import torch

    L = pkg.load_library()
    case, _ = cases.all_rigid()
    d = str(tmp_path / "box")
    case.write(d)
    tdt = torch.float64 if precision == "f64" else torch.float32
    ndt = np.float64 if precision == "f64" else np.float32
    prec = pkg.F64 if precision == "f64" else pkg.F32
    X = np.ascontiguousarray(case.X, dtype=np.float64)
    Y = np.ascontiguousarray(case.Y, dtype=np.float64)
    Z = np.ascontiguousarray(case.Z, dtype=np.float64)
    dx, dy, dz = case.spacing()

    with pkg.Airpore(d, precision) as ref:
        ref.reset(4)
        n = ref.state_elems()
        state = np.zeros(4 * n, dtype=ndt)
        ref.copy_state(state, to_device=False)  # initial u v w p, native layout
        bufs = [[torch.empty(n, dtype=tdt, device="cuda") for _ in range(4)] for _ in range(2)]
        for c in range(4):
            bufs[0][c].copy_(torch.from_numpy(state[c * n:(c + 1) * n]))
        torch.cuda.synchronize()
        stream = torch.cuda.current_stream().cuda_stream
        for call in range(2):
            src, dst = bufs[call % 2], bufs[1 - call % 2]
            rc = L.fdtd_fb_step_noalloc(prec, case.NI, case.NJ, case.NK, _dp(X), _dp(Y), _dp(Z), dx, dy, dz,
                                        case.dt, case.gamma, case.P0, case.c0,
                                        *[t.data_ptr() for t in src], *[t.data_ptr() for t in dst], stream)
            assert rc == pkg.FDTD_OK, L.fdtd_last_error()
            ref.Cal_pressure()
            ref.Cal_velocity()
            expect = np.zeros(4 * n, dtype=ndt)
            ref.copy_state(expect, to_device=False)
            got = torch.cat(dst).cpu().numpy()
            for c, name in enumerate("uvwp"):
                e = rel_l2(got[c * n:(c + 1) * n].astype(np.float64), expect[c * n:(c + 1) * n].astype(np.float64))
                assert e <= tol, (call, name, e)
            assert np.abs(got[3 * n:]).max() > 1e-3  # the pulse is really there
        if precision == "f64":  # and directly against the oracle after the two steps
            ref_o = oracle.run_case(d, [], 2)
            njp = n // (case.NI * case.NK)
            for c, name in enumerate("uvwp"):
                f = got[c * n:(c + 1) * n].reshape(case.NK, case.NI, njp)[:, :, :case.NJ].transpose(1, 2, 0)
                assert rel_l2(f, ref_o[name]) <= 1e-10, name


def test_noalloc_rejects_oversized_axis():
    L = pkg.load_library()
    big = np.zeros(5000, dtype=np.float64)
    small = np.zeros(8, dtype=np.float64)
    dummy = ctypes.c_void_p(1)
    rc = L.fdtd_fb_step_noalloc(pkg.F64, 8, 5000, 8, _dp(small), _dp(big), _dp(small), 0.05, 0.05, 0.05, 1e-4,
                                1.4, 1e5, 343.0, *([dummy] * 8), None)
    assert rc == pkg.FDTD_ERR_ARG
    assert b"4096" in L.fdtd_last_error()
