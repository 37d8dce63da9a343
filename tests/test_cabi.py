"""C ABI surface checks that need no GPU: the library loads, exports every
function include/*.h declares, and rejects bad case directories
before touching the device."""

import ctypes
import importlib
import os
import re

import pytest

import cases

pkg = importlib.import_module("3d_mpi_test_b200")
build = importlib.import_module("3d_mpi_test_b200.build")

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    inc = os.path.join(ROOT, "include")
    for h in sorted(os.listdir(inc)):
        if h.endswith(".h"):
            txt = re.sub(r"/\*.*?\*/", "", open(os.path.join(inc, h)).read(), flags=re.S)
            names |= set(re.findall(r"\b(fdtd_[a-z0-9_]+)\s*\(", txt))
    return sorted(names)


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(pkg.LIB_PATH):
        build.build()
    return pkg.load_library()


def test_every_declared_symbol_is_exported(lib):
    names = declared_functions()
    assert len(names) >= 15
    assert set(names) == set(pkg.EXPORTS)
    for n in names:
        assert hasattr(lib, n), n


def test_library_is_sm100a_only():
    # the fatbin is built for sm_100a alone (no PTX for JIT to other archs)
    assert "arch=compute_100a,code=sm_100a" in " ".join(build.ARCH)


def test_missing_case_is_input_error(lib, tmp_path):
    h = ctypes.c_void_p()
    rc = lib.fdtd_create(str(tmp_path / "nope").encode(), 0, 0, ctypes.byref(h))
    assert rc == pkg.FDTD_ERR_INPUT
    assert b"input.txt" in lib.fdtd_last_error()
    assert not h.value


def test_malformed_axis_file_is_input_error(lib, tmp_path):
    c, _ = cases.pml_rigid()
    d = str(tmp_path / "bad")
    c.write(d)
    with open(os.path.join(d, "coordi_air3.dat"), "w") as f:
        f.write("0 0.05\n")  # far fewer Z nodes than the header promises
    h = ctypes.c_void_p()
    rc = lib.fdtd_create(d.encode(), 0, 0, ctypes.byref(h))
    assert rc == pkg.FDTD_ERR_INPUT
    assert b"Z coordinates" in lib.fdtd_last_error()


def test_null_arguments(lib):
    assert lib.fdtd_create(None, 0, 0, None) == pkg.FDTD_ERR_ARG
    assert lib.fdtd_destroy(None) == pkg.FDTD_OK
    assert lib.fdtd_state_elems(None) == 0


def test_ray_feature_arguments_are_checked_before_any_device_work(lib):
    fn = lib.fdtd_ray_features
    fn.argtypes = [ctypes.c_void_p] + [ctypes.c_int] * 6 + [ctypes.c_void_p, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    buf = ctypes.c_void_p(16)  # never dereferenced: every call below is rejected first
    assert fn(None, 1, 11, 4, 5, 6, 8, buf, None) == pkg.FDTD_ERR_ARG  # null rows
    assert fn(buf, -1, 11, 4, 5, 6, 8, buf, None) == pkg.FDTD_ERR_ARG  # negative count
    assert fn(buf, 1, 11, 4, 5, 11, 8, buf, None) == pkg.FDTD_ERR_ARG  # range column outside the row
    assert fn(buf, 1, 11, 4, 5, 6, 0, buf, None) == pkg.FDTD_ERR_ARG  # no receivers
    assert b"ray features" in lib.fdtd_last_error()
    assert fn(None, 0, 11, 4, 5, 6, 8, None, None) == pkg.FDTD_OK  # nothing to do


def test_package_fails_loudly_without_library(tmp_path):
    with pytest.raises(pkg.FdtdError) as e:
        pkg.load_library(str(tmp_path / "libfdtd_b200.so"))
    assert e.value.code == pkg.FDTD_ERR_CUDA


def test_noalloc_rejects_overlapping_buffers_before_any_device_work(lib):
    # the step cannot run in place: every output must be disjoint from every
    # input and from the other outputs; the check comes before any CUDA call
    import numpy as np

    fn = lib.fdtd_fb_step_noalloc
    NI, NJ, NK = 4, 8, 4
    X, Y, Z = (np.arange(n, dtype=np.float64) * 0.05 for n in (NI, NJ, NK))
    dp = ctypes.POINTER(ctypes.c_double)
    nb = NI * NJ * NK * 8
    base = 1 << 40  # never dereferenced: every call below is rejected first
    bufs = [ctypes.c_void_p(base + q * 4 * nb) for q in range(8)]  # disjoint address ranges

    def call(u_o, v_o, w_o, p_o):
        return fn(0, NI, NJ, NK, X.ctypes.data_as(dp), Y.ctypes.data_as(dp), Z.ctypes.data_as(dp), 0.05, 0.05,
                  0.05, 1e-5, 1.4, 1e5, 343.0, bufs[0], bufs[1], bufs[2], bufs[3], u_o, v_o, w_o, p_o, None)

    assert call(bufs[0], bufs[5], bufs[6], bufs[7]) == pkg.FDTD_ERR_ARG  # u in place
    assert b"overlaps an input" in lib.fdtd_last_error()
    assert call(bufs[4], bufs[5], bufs[6], ctypes.c_void_p(base + 3 * 4 * nb + 8)) == pkg.FDTD_ERR_ARG
    assert call(bufs[4], bufs[4], bufs[6], bufs[7]) == pkg.FDTD_ERR_ARG  # two outputs share memory
    assert b"two output buffers" in lib.fdtd_last_error()
