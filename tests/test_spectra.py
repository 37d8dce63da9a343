"""Receiver spectra: the reference's FFT post-processing (airpore::get_FFT_y1,
FFT.cpp) on the GPU, band levels and excess attenuation.

CPU: the oracle's FFT restatement against the compiled reference and the
golden vectors the reference produced; argument errors of the C ABI.
GPU: the device FFT bit for bit against the golden vectors and the oracle,
spectra of solver runs against the oracle's, band levels, excess
attenuation."""

from __future__ import annotations

import importlib
import os

import numpy as np
import pytest

import oracle
import cases

pkg = importlib.import_module("3d_mpi_test_b200")
HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = np.load(os.path.join(HERE, "golden", "fft_ref.npz"))
TAGS = ("a", "b", "c")


def _padded(t: np.ndarray, m: int) -> np.ndarray:
    n = 1 << m
    x = np.zeros(n)
    k = min(len(t), n)
    x[:k] = t[:k]
    return x


# ------------------------------------------------------------------ CPU
@pytest.mark.parametrize("tag", TAGS)
def test_oracle_fft_matches_reference_golden(tag):
    m = int(GOLDEN[f"{tag}_m"])
    for r, t in enumerate(GOLDEN[f"{tag}_traces"]):
        x = _padded(t, m)
        re, im = oracle.fft(x, np.zeros_like(x), 1)
        assert np.array_equal(re, GOLDEN[f"{tag}_re"][r]) and np.array_equal(im, GOLDEN[f"{tag}_im"][r])


def test_oracle_fft_matches_compiled_reference(ref_harness):
    refio = importlib.import_module("refio")
    if not os.path.exists(refio.REF_FFT):
        pytest.skip("oracle/_ref/ref_fft not built")
    rng = np.random.default_rng(7)
    for m in (1, 2, 9, 14):
        x, y = rng.standard_normal(1 << m), rng.standard_normal(1 << m)
        for d in (1, -1):
            a = oracle.fft(x, y, d)
            b = refio.run_reference_fft(x, y, d)
            assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]), (m, d)


def test_oracle_spectrum_is_a_scaled_dft():
    rng = np.random.default_rng(3)
    t = rng.standard_normal(300)
    f, mag = oracle.spectrum(t, 9, 1e-4)
    ref = np.abs(np.fft.rfft(_padded(t, 9))) / 512
    assert np.allclose(mag, ref, rtol=1e-10, atol=1e-14)
    assert f[1] == pytest.approx(1.0 / (1e-4 * 512)) and len(f) == 257


def test_spectrum_arguments_are_checked():
    t = np.zeros((2, 10))
    for fn, args in ((pkg.fft, (t, 0)), (pkg.fft, (t, 25)), (pkg.spectrum, (t, 4, 1e-3, 0, 20)),
                     (pkg.band_levels, (t, 4, 0.0)), (pkg.band_levels, (t, 4, 1e-3, (100.0, -1.0)))):
        with pytest.raises(pkg.FdtdError) as e:
            fn(*args)
        assert e.value.code == pkg.FDTD_ERR_ARG


# ------------------------------------------------------------------ GPU
@pytest.mark.gpu
@pytest.mark.parametrize("tag", TAGS)
def test_gpu_fft_is_bit_exact_with_reference(tag):
    m = int(GOLDEN[f"{tag}_m"])
    re, im = pkg.fft(GOLDEN[f"{tag}_traces"], m)
    assert np.array_equal(re, GOLDEN[f"{tag}_re"]) and np.array_equal(im, GOLDEN[f"{tag}_im"])


@pytest.mark.gpu
@pytest.mark.parametrize("m", [1, 7, 13, 17])
def test_gpu_fft_is_bit_exact_with_oracle(m):
    rng = np.random.default_rng(m)
    traces = rng.standard_normal((3, (1 << m) * 3 // 4 + 1))
    re, im = pkg.fft(traces, m)
    for r in range(3):
        x = _padded(traces[r], m)
        a = oracle.fft(x, np.zeros_like(x), 1)
        assert np.array_equal(re[r], a[0]) and np.array_equal(im[r], a[1])


@pytest.mark.gpu
def test_gpu_spectrum_bins_and_band_levels():
    rng = np.random.default_rng(11)
    traces = rng.standard_normal((2, 3000))
    m, dt = 13, 7.2886e-5
    f, mag = pkg.spectrum(traces, m, dt)
    f2, sub = pkg.spectrum(traces, m, dt, k0=100, nk=50)
    for r in range(2):
        fo, mo = oracle.spectrum(traces[r], m, dt)
        np.testing.assert_allclose(mag[r], mo, rtol=1e-15, atol=0)
        np.testing.assert_allclose(sub[r], mo[100:150], rtol=1e-15, atol=0)
        np.testing.assert_array_equal(f, fo)
    np.testing.assert_array_equal(f2, f[100:150])
    levels = pkg.band_levels(traces, m, dt)
    e = 2.0 ** (1 / 6)
    for r in range(2):
        for b, fc in enumerate(pkg.THIRD_OCTAVE_50_2K):
            sel = (f >= fc / e) & (f < fc * e)
            want = 10 * np.log10(np.sum(mag[r][sel] ** 2))
            assert levels[r, b] == pytest.approx(want, rel=1e-12, abs=1e-9)


@pytest.mark.gpu
def test_solver_receiver_spectra_match_oracle(tmp_path):
    """Receiver histories of a GPU run, through the GPU spectrum, agree with
    the oracle run through the oracle's FFT (FP64 tolerance of the solve)."""
    c, rec = cases.CASES["porous_tdbc_fine_pore"]()
    d = str(tmp_path / "case")
    c.write(d)
    n = c.time_domain
    ref = oracle.run_case(d, rec, n)
    with pkg.Airpore(d, "f64") as a:
        a.set_receivers(rec)
        got = a.get_output(n)
    m, dt = 7, c.dt
    _, mag = pkg.spectrum(got.T, m, dt)
    for r in range(len(rec)):
        _, mo = oracle.spectrum(ref["receivers"][:, r], m, dt)
        assert np.linalg.norm(mag[r] - mo) <= 1e-10 * np.linalg.norm(mo)


@pytest.mark.gpu
def test_excess_attenuation_of_ground_against_free_field(tmp_path):
    """Band levels of a rigid-ground solve minus those of the same source and
    receivers with every face absorbing: finite, and zero for identical runs."""
    base = cases._base(nk=18, steps=120)
    rec = [(0.5, 1.05, 0.15)]
    dirs = {}
    for name, bc in (("ground", (cases.PML, cases.RIGID, cases.PML, cases.PML, cases.PML, cases.PML)),
                     ("free", (cases.PML,) * 6)):
        c = cases._base(nk=18, steps=120, bc=bc, pml_nodes=(5, 5, 5, 5, 5 if bc[1] == cases.PML else 0, 5))
        c.source = (0.5, 0.55, 0.3)
        dirs[name] = str(tmp_path / name)
        c.write(dirs[name])
    traces = {}
    for name, d in dirs.items():
        with pkg.Airpore(d, "f64") as a:
            a.set_receivers(rec)
            traces[name] = a.get_output(120).T
    dt = base.dt
    ea = pkg.excess_attenuation(traces["ground"], traces["free"], 12, dt)
    assert ea.shape == (1, 17) and np.all(np.isfinite(ea))
    assert np.all(pkg.excess_attenuation(traces["ground"], traces["ground"], 12, dt) == 0)
