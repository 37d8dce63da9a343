"""Reader for the full-precision dumps written by ``oracle/_ref/ref_harness``
(the unmodified reference solver driven through its own airpore loop).
Test infrastructure only."""

from __future__ import annotations

import os
import subprocess
from typing import Dict, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_HARNESS = os.path.join(HERE, "_ref", "ref_harness")
REF_FFT = os.path.join(HERE, "_ref", "ref_fft")

SLAB_NAMES = {0: "x1", 1: "x2", 2: "y1", 3: "y2", 4: "z1", 5: "z2"}


def read_dump(path: str) -> Dict[str, object]:
    with open(path, "rb") as f:
        buf = f.read()
    if buf[:8] != b"FDTDREF1":
        raise ValueError(f"{path}: not a reference dump")
    off = 8
    hdr = np.frombuffer(buf, dtype="<i4", count=10, offset=off)
    off += 40
    nrec, nsteps, I, J, K, has_pore, pI, pJ, pK, nslab = (int(v) for v in hdr)
    out: Dict[str, object] = {"I": I, "J": J, "K": K, "nsteps": nsteps}
    idx = np.frombuffer(buf, dtype="<i4", count=3 * nrec, offset=off).reshape(nrec, 3)
    off += 12 * nrec
    out["rec_index"] = idx.copy()

    def take(n, shape):
        nonlocal off
        a = np.frombuffer(buf, dtype="<f8", count=n, offset=off).reshape(shape).copy()
        off += 8 * n
        return a

    out["receivers"] = take(nsteps * nrec, (nsteps, nrec)) if nrec else np.zeros((nsteps, 0))
    for name in ("p", "u", "v", "w"):
        out[name] = take(I * J * K, (I, J, K))
    if has_pore:
        for name in ("p", "u", "v", "w"):
            out["pore_" + name] = take(pI * pJ * pK, (pI, pJ, pK))
    out["psi"] = take(I * K * 6, (I, K, 6))
    slabs = {}
    for _ in range(nslab):
        sid, d0, d1, d2 = (int(v) for v in np.frombuffer(buf, dtype="<i4", count=4, offset=off))
        off += 16
        q = {}
        for comp in ("u", "v", "w", "p"):
            q[comp] = take(d0 * d1 * d2, (d0, d1, d2))
        slabs[SLAB_NAMES[sid]] = q
    out["slabs"] = slabs
    return out


def run_reference(case_dir: str, out_path: str, receivers_file: Optional[str] = None,
                  steps: Optional[int] = None, harness: str = REF_HARNESS) -> Dict[str, object]:
    cmd = [harness, case_dir, "--out", out_path]
    if receivers_file:
        cmd += ["--receivers", receivers_file]
    if steps is not None:
        cmd += ["--steps", str(steps)]
    subprocess.run(cmd, check=True)
    return read_dump(out_path)


def run_reference_fft(re, im, direction: int = 1, exe: str = REF_FFT):
    """The compiled reference FFT() on copies of re, im (length 2^m)."""
    n = len(re)
    m = n.bit_length() - 1
    buf = np.concatenate([np.asarray(re, np.float64), np.asarray(im, np.float64)]).tobytes()
    out = subprocess.run([exe, str(m), str(direction)], input=buf, capture_output=True, check=True).stdout
    a = np.frombuffer(out, dtype=np.float64)
    return a[:n].copy(), a[n:].copy()
