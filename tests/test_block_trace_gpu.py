"""Block timeline of the tiled kernel (fdtd_set_block_trace /
fdtd_get_block_trace): recording changes no result, every step of the last
advance holds every block of every tile kind, and the spans are ordered."""

import importlib

import numpy as np
import pytest

import cases

pkg = importlib.import_module("3d_mpi_test_b200")

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def hill_dir(tmp_path_factory):
    c, rec = cases.hill_porous()
    d = tmp_path_factory.mktemp("trace") / "hill_porous"
    c.write(str(d))
    return str(d), rec


def _fields(a):
    out = {f: a.field(f) for f in "puvw"}
    out.update({"pore_" + f: a.field(f, "pore") for f in "puvw"})
    return out


@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_block_trace_records_every_block(precision, hill_dir):
    d, rec = hill_dir
    n = 40
    with pkg.Airpore(d, precision) as a:
        a.set_receivers(rec)
        r0 = a.get_output(n)
        f0 = _fields(a)
    with pkg.Airpore(d, precision) as a:
        with pytest.raises(pkg.FdtdError):
            a.block_trace()
        a.set_block_trace(True)
        a.set_receivers(rec)
        r1 = a.get_output(n)
        f1 = _fields(a)
        tr = a.block_trace()
        shape = a.tile_shape()
    np.testing.assert_array_equal(r1, r0)
    for k in f0:
        np.testing.assert_array_equal(f1[k], f0[k], err_msg=k)
    none = np.iinfo(np.uint64).max
    blocks = tr[:, :, 3]
    assert int((blocks.sum(axis=1) > 0).sum()) == n  # one slot per step
    live = blocks[blocks.sum(axis=1) > 0]
    assert (live[:, 0] == shape["full"]["tiles"]).all()
    assert (live[:, 1] == shape["lean"]["tiles"]).all()
    assert (live[:, 2:].sum(axis=1) == shape["pml"]["tiles"]).all()
    ran = tr[:, :, 3] > 0
    assert (tr[:, :, 0][ran] <= tr[:, :, 1][ran]).all()
    assert (tr[:, :, 0][~ran] == none).all()
    assert (tr[:, :, 2][ran] > 0).all()
