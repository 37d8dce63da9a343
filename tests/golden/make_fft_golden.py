"""Golden vectors for the receiver-spectrum path, produced by the reference
itself: seeded traces transformed by the reference's own FFT() (FFT.cpp,
compiled under oracle/_ref/ by oracle/Makefile as ref_fft).

    python tests/golden/make_fft_golden.py      # writes tests/golden/fft_ref.npz
"""

from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
import refio  # noqa: E402


def main() -> None:
    rng = np.random.default_rng(20251203)
    out = {}
    # (m, nrec, nt): padded (nt < 2^m), exact (nt = 2^m) and cut (nt > 2^m) traces
    for tag, (m, nrec, nt) in {"a": (6, 3, 40), "b": (10, 2, 1024), "c": (11, 2, 3000)}.items():
        t = np.cumsum(rng.standard_normal((nrec, nt)), axis=1) * 1e-3  # pressure-like random walks
        n = 1 << m
        re = np.empty((nrec, n))
        im = np.empty((nrec, n))
        for r in range(nrec):
            x = np.zeros(n)
            k = min(nt, n)
            x[:k] = t[r, :k]
            re[r], im[r] = refio.run_reference_fft(x, np.zeros(n), 1)
        out[f"{tag}_traces"] = t
        out[f"{tag}_m"] = np.array(m)
        out[f"{tag}_re"] = re
        out[f"{tag}_im"] = im
    np.savez_compressed(os.path.join(HERE, "fft_ref.npz"), **out)


if __name__ == "__main__":
    main()
