"""ctypes wrapper of the plain-C oracle (``oracle/_ref/liboracle.so``, built
from ``oracle/fdtd_oracle.c`` by ``oracle/Makefile``).

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``__graft_entry__.smoke``
and ``bench.py``'s cpu_baseline leg as the checker.  The product path never
imports it.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Dict, Optional, Sequence, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "liboracle.so")

_lib = None


def build(force: bool = False) -> str:
    """Compile the C restatement (gcc only; no reference sources needed)."""
    if force or not os.path.exists(LIB_PATH) or (
        os.path.getmtime(LIB_PATH) < os.path.getmtime(os.path.join(HERE, "fdtd_oracle.c"))
    ):
        subprocess.run(["make", "-C", HERE, "restatement"], check=True, stdout=subprocess.DEVNULL)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB_PATH)
        L.orc_create.restype = ctypes.c_void_p
        L.orc_create.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int]
        L.orc_destroy.argtypes = [ctypes.c_void_p]
        L.orc_dims.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]
        L.orc_set_receivers.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                        ctypes.POINTER(ctypes.c_int)]
        L.orc_run.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
        L.orc_get_field.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
        L.orc_set_field.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
        L.orc_get_psi.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]
        L.orc_get_ground_psi.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]
        L.orc_get_slab.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                   ctypes.POINTER(ctypes.c_int)]
        L.orc_get_wind.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
        L.orc_fft.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
        L.orc_fft.restype = None
        _lib = L
    return _lib


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class OracleCase:
    """One reference-solver instance restated in C, built from a case dir."""

    SLABS = ("x1", "x2", "y1", "y2", "z1", "z2")

    def __init__(self, case_dir: str):
        L = lib()
        err = ctypes.create_string_buffer(512)
        h = L.orc_create(case_dir.encode(), err, 512)
        if not h:
            raise RuntimeError(f"oracle: {err.value.decode()}")
        self._h = h
        d = (ctypes.c_int * 10)()
        L.orc_dims(h, d)
        self.I, self.J, self.K, self.has_pore, self.pI, self.pJ, self.pK, self.time_domain, self.scheme, _ = list(d)
        self.nrec = 0

    def close(self):
        if self._h:
            lib().orc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_receivers(self, xyz: Sequence[Tuple[float, float, float]]) -> np.ndarray:
        a = np.ascontiguousarray(np.asarray(xyz, dtype=np.float64).reshape(-1, 3))
        idx = np.zeros((a.shape[0], 3), dtype=np.int32)
        lib().orc_set_receivers(self._h, a.shape[0], _dp(a), idx.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
        self.nrec = a.shape[0]
        return idx

    def run(self, nsteps: int) -> np.ndarray:
        out = np.zeros((nsteps, max(self.nrec, 1)), dtype=np.float64)
        n = lib().orc_run(self._h, nsteps, _dp(out))
        if n < 0:
            raise RuntimeError(f"oracle run failed ({n})")
        return out[:, : self.nrec]

    def field(self, name: str, medium: int = 0) -> np.ndarray:
        comp = {"p": 0, "u": 1, "v": 2, "w": 3}[name]
        shape = (self.I, self.J, self.K) if medium == 0 else (self.pI, self.pJ, self.pK)
        out = np.zeros(shape, dtype=np.float64)
        if lib().orc_get_field(self._h, medium, comp, _dp(out)) != 0:
            raise ValueError("no such medium")
        return out

    def set_field(self, name: str, arr: np.ndarray, medium: int = 0) -> None:
        comp = {"p": 0, "u": 1, "v": 2, "w": 3}[name]
        a = np.ascontiguousarray(arr, dtype=np.float64)
        lib().orc_set_field(self._h, medium, comp, _dp(a))

    def psi(self) -> np.ndarray:
        out = np.zeros((self.I, self.K, 6), dtype=np.float64)
        lib().orc_get_psi(self._h, _dp(out))
        return out

    def ground_psi(self) -> Optional[np.ndarray]:
        """Impedance-ground TDBC state [i][j][6], None without tdbc_ground.dat."""
        out = np.zeros((self.I, self.J, 6), dtype=np.float64)
        return out if lib().orc_get_ground_psi(self._h, _dp(out)) == 0 else None

    def slabs(self) -> Dict[str, Dict[str, np.ndarray]]:
        res: Dict[str, Dict[str, np.ndarray]] = {}
        for sid, name in enumerate(self.SLABS):
            dims = (ctypes.c_int * 3)()
            if not lib().orc_get_slab(self._h, sid, 0, None, dims):
                continue
            q = {}
            for comp, cname in enumerate("uvwp"):
                a = np.zeros(tuple(dims), dtype=np.float64)
                lib().orc_get_slab(self._h, sid, comp, _dp(a), dims)
                q[cname] = a
            res[name] = q
        return res

    def wind(self) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
        outs = []
        for comp in range(3):
            a = np.zeros((self.I, self.J, self.K), dtype=np.float64)
            lib().orc_get_wind(self._h, comp, _dp(a))
            outs.append(a)
        return tuple(outs)


def run_case(case_dir: str, receivers: Sequence[Tuple[float, float, float]], nsteps: Optional[int] = None):
    """Convenience: run a case and return a dict shaped like refio.read_dump()."""
    oc = OracleCase(case_dir)
    idx = oc.set_receivers(receivers) if len(receivers) else np.zeros((0, 3), np.int32)
    n = oc.time_domain if nsteps is None else nsteps
    rec = oc.run(n)
    out = {"receivers": rec, "rec_index": idx, "I": oc.I, "J": oc.J, "K": oc.K, "nsteps": n}
    for f in "puvw":
        out[f] = oc.field(f)
        if oc.has_pore:
            out["pore_" + f] = oc.field(f, 1)
    out["psi"] = oc.psi()
    out["slabs"] = oc.slabs()
    oc.close()
    return out


def fft(re: np.ndarray, im: np.ndarray, direction: int = 1) -> Tuple[np.ndarray, np.ndarray]:
    """The reference's radix-2 FFT (FFT.cpp:15-83) on copies of re, im
    (length 2^m); direction 1 is forward and scaled by 1/2^m."""
    n = len(re)
    m = n.bit_length() - 1
    if n != 1 << m or len(im) != n:
        raise ValueError("length must be a power of two")
    r = np.ascontiguousarray(re, dtype=np.float64).copy()
    i = np.ascontiguousarray(im, dtype=np.float64).copy()
    lib().orc_fft(direction, m, _dp(r), _dp(i))
    return r, i


def spectrum(trace: np.ndarray, m: int, dt: float) -> Tuple[np.ndarray, np.ndarray]:
    """airpore::get_FFT_y1 + FFT_output (airpore.cpp:966-1011, FFT.cpp:86-120):
    zero-pad the trace to 2^m points, forward FFT, and return the bin
    frequencies k / (dt 2^m) and magnitudes |X_k| for k = 0 .. 2^(m-1)."""
    n = 1 << m
    re = np.zeros(n)
    re[:min(len(trace), n)] = trace[:n]
    r, i = fft(re, np.zeros(n), 1)
    k = np.arange(n // 2 + 1)
    return k / dt / n, np.hypot(r[: n // 2 + 1], i[: n // 2 + 1])
