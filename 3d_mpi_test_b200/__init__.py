"""B200-native time-marching path of the azhang22/3D_MPI_TEST outdoor-sound
FDTD solver (linearized Euler with mean wind, Zwikker-Kosten porous ground,
PML, 6-pole TDBC, moving frame), behind the C ABI in include/fdtd_b200.h.

Python here is a thin host mirror of the reference's ``airpore`` driver
(airpore.h:24-68): :class:`Airpore` is built from a reference case directory
(``input.txt`` + ``coordi_*.dat``) and exposes ``get_output`` (the time loop,
airpore.cpp:400-641), ``Cal_pressure`` / ``Cal_velocity`` (the half steps,
airpore.cpp:324-398) and field read-out.  All compute runs in the native
library ``lib/libfdtd_b200.so`` on an sm_100a device; there is no CPU path.
"""

from __future__ import annotations

import ctypes
import os
from typing import Optional, Sequence, Tuple

import numpy as np

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG_DIR, "lib", "libfdtd_b200.so")

FDTD_OK = 0
FDTD_ERR_INPUT = -1
FDTD_ERR_UNSUPPORTED = -2
FDTD_ERR_CUDA = -3
FDTD_ERR_NONFINITE = -4
FDTD_ERR_ARG = -5
FDTD_ERR_STATE = -6
FDTD_ERR_TIMEOUT = -7
F64, F32 = 0, 1

# Every function declared in include/*.h.
EXPORTS = (
    "fdtd_create", "fdtd_destroy", "fdtd_dims", "fdtd_last_error", "fdtd_set_receivers", "fdtd_reset",
    "fdtd_run", "fdtd_advance", "fdtd_step_pressure", "fdtd_step_velocity", "fdtd_get_field",
    "fdtd_set_field", "fdtd_get_psi", "fdtd_get_ground_psi", "fdtd_get_slab", "fdtd_state_elems", "fdtd_copy_state",
    "fdtd_launch_count", "fdtd_last_device_ms", "fdtd_fb_step_noalloc", "fdtd_set_tiling", "fdtd_autotune",
    "fdtd_fft", "fdtd_spectrum", "fdtd_band_levels", "fdtd_save_restart", "fdtd_load_restart",
    "fdtd_write_contour", "fdtd_get_receivers", "fdtd_set_wait_limit", "fdtd_ensemble_create",
    "fdtd_ensemble_destroy", "fdtd_ensemble_advance", "fdtd_ensemble_autotune", "fdtd_ensemble_info",
    "fdtd_ensemble_last_device_ms", "fdtd_ensemble_set_mode", "fdtd_set_tile_shape", "fdtd_get_tile_shape",
    "fdtd_set_block_trace", "fdtd_get_block_trace",
    # include/fdtd_surrogate.h (signatures in surrogate.py)
    "fdtd_tc_gemm", "fdtd_net_create", "fdtd_net_destroy", "fdtd_net_n_params", "fdtd_net_get_params",
    "fdtd_net_set_params", "fdtd_net_set_data", "fdtd_net_get_normalization", "fdtd_net_set_normalization",
    "fdtd_net_train", "fdtd_net_gradients", "fdtd_net_predict", "fdtd_net_predict_device", "fdtd_net_set_fused", "fdtd_net_info",
    "fdtd_net_ensemble_predict", "fdtd_ray_features", "fdtd_net_ensemble_predict_rays",
)


class FdtdError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


_LIBS = {}


def load_library(path: Optional[str] = None) -> ctypes.CDLL:
    """Load the native library and declare the C ABI signatures.  Raises if
    the library has not been built: there is no fallback implementation."""
    path = path or LIB_PATH
    if path in _LIBS:
        return _LIBS[path]
    if not os.path.exists(path):
        raise FdtdError(FDTD_ERR_CUDA, f"native library missing: {path} (run __graft_entry__.build())")
    L = ctypes.CDLL(path)
    vp, ip, dp, i, cp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double), \
        ctypes.c_int, ctypes.c_char_p
    sig = {
        "fdtd_create": ([cp, i, i, ctypes.POINTER(vp)], i),
        "fdtd_destroy": ([vp], i),
        "fdtd_dims": ([vp, ip], i),
        "fdtd_last_error": ([], cp),
        "fdtd_set_receivers": ([vp, i, dp, ip], i),
        "fdtd_reset": ([vp, i], i),
        "fdtd_run": ([vp, i, dp], i),
        "fdtd_advance": ([vp, i, dp], i),
        "fdtd_step_pressure": ([vp], i),
        "fdtd_step_velocity": ([vp], i),
        "fdtd_get_field": ([vp, i, i, dp], i),
        "fdtd_set_field": ([vp, i, i, dp], i),
        "fdtd_get_psi": ([vp, dp], i),
        "fdtd_get_ground_psi": ([vp, dp], i),
        "fdtd_get_slab": ([vp, i, i, dp, ip], i),
        "fdtd_state_elems": ([vp], ctypes.c_size_t),
        "fdtd_copy_state": ([vp, i, vp], i),
        "fdtd_launch_count": ([vp], ctypes.c_longlong),
        "fdtd_last_device_ms": ([vp, dp], i),
        "fdtd_fb_step_noalloc": ([i, i, i, i, dp, dp, dp] + [ctypes.c_double] * 7 + [vp] * 9, i),
        "fdtd_set_tiling": ([vp, i, i, i, i, i], i),
        "fdtd_autotune": ([vp, i, ip], i),
        "fdtd_set_tile_shape": ([vp, i, i, i, i, i], i),
        "fdtd_get_tile_shape": ([vp, ip], i),
        "fdtd_set_block_trace": ([vp, i], i),
        "fdtd_get_block_trace": ([vp, ctypes.POINTER(ctypes.c_ulonglong)], i),
        "fdtd_fft": ([i, dp, i, i, i, dp, dp], i),
        "fdtd_spectrum": ([i, dp, i, i, i, ctypes.c_longlong, ctypes.c_longlong, dp], i),
        "fdtd_band_levels": ([i, dp, i, i, i, ctypes.c_double, i, dp, dp], i),
        "fdtd_save_restart": ([vp, cp], i),
        "fdtd_load_restart": ([vp, cp, i], i),
        "fdtd_write_contour": ([vp, cp, i], i),
        "fdtd_get_receivers": ([vp, i, i, dp], i),
        "fdtd_set_wait_limit": ([vp, ctypes.c_longlong], i),
        "fdtd_ensemble_create": ([ctypes.POINTER(vp), i, ctypes.POINTER(vp)], i),
        "fdtd_ensemble_destroy": ([vp], i),
        "fdtd_ensemble_advance": ([vp, i, ip], i),
        "fdtd_ensemble_autotune": ([vp, i, ip], i),
        "fdtd_ensemble_info": ([vp, ctypes.POINTER(ctypes.c_longlong)], i),
        "fdtd_ensemble_last_device_ms": ([vp, dp], i),
        "fdtd_ensemble_set_mode": ([vp, i], i),
    }
    for name, (args, res) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    _LIBS[path] = L
    return L


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


_COMP = {"p": 0, "u": 1, "v": 2, "w": 3}
_SLABS = ("x1", "x2", "y1", "y2", "z1", "z2")


class Airpore:
    """Host mirror of the reference's ``airpore`` object on one device.

    ``precision``: "f64" (parity path) or "f32" (FP32 fields and stencil,
    FP64 TDBC state and receiver series)."""

    def __init__(self, case_dir: str, precision: str = "f64", device: int = 0, lib_path: Optional[str] = None):
        self._L = load_library(lib_path)
        self._h = ctypes.c_void_p()
        prec = {"f64": F64, "f32": F32}[precision]
        self._check(self._L.fdtd_create(case_dir.encode(), prec, device, ctypes.byref(self._h)))
        self.precision = precision
        d = (ctypes.c_int * 12)()
        self._check(self._L.fdtd_dims(self._h, d))
        (self.I, self.J, self.K, self.has_pore, self.pI, self.pJ, self.pK, self.NG, self.time_domain, _,
         self.scheme, _) = list(d)
        self.nrec = 0

    # ------------------------------------------------------------------
    def _check(self, rc: int) -> int:
        if rc < 0:
            raise FdtdError(rc, self._L.fdtd_last_error().decode())
        return rc

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            self._L.fdtd_destroy(self._h)
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

    # ------------------------------------------------------------------
    def set_receivers(self, xyz: Sequence[Tuple[float, float, float]]) -> np.ndarray:
        """calculation_2D::get_position for each (X, Y, Z); returns indices."""
        a = np.ascontiguousarray(np.asarray(xyz, dtype=np.float64).reshape(-1, 3))
        idx = np.zeros((a.shape[0], 3), dtype=np.int32)
        self._check(self._L.fdtd_set_receivers(self._h, a.shape[0], _dp(a),
                                               idx.ctypes.data_as(ctypes.POINTER(ctypes.c_int))))
        self.nrec = a.shape[0]
        return idx

    def reset(self, horizon: int = 0) -> None:
        self._check(self._L.fdtd_reset(self._h, horizon))

    def get_output(self, nsteps: Optional[int] = None) -> np.ndarray:
        """The reference time loop (airpore::get_output) for ``nsteps`` steps
        (default: input.txt's time_domain) from t = 0; returns receiver p(t)
        as [nsteps, n_receivers] FP64."""
        n = self.time_domain if nsteps is None else nsteps
        out = np.zeros((n, max(self.nrec, 1)), dtype=np.float64)
        self._check(self._L.fdtd_run(self._h, n, _dp(out)))
        return out[:, : self.nrec]

    def advance(self, nsteps: int) -> np.ndarray:
        out = np.zeros((nsteps, max(self.nrec, 1)), dtype=np.float64)
        self._check(self._L.fdtd_advance(self._h, nsteps, _dp(out)))
        return out[:, : self.nrec]

    def Cal_pressure(self) -> None:
        self._check(self._L.fdtd_step_pressure(self._h))

    def Cal_velocity(self) -> None:
        self._check(self._L.fdtd_step_velocity(self._h))

    # ------------------------------------------------------------------
    def field(self, name: str, medium: str = "air", level: str = "n") -> np.ndarray:
        m = {"air": 0, "pore": 1}[medium]
        comp = _COMP[name] + (4 if level == "nn" else 0)
        shape = (self.I, self.J, self.K) if m == 0 else (self.pI, self.pJ, self.pK)
        out = np.zeros(shape, dtype=np.float64)
        self._check(self._L.fdtd_get_field(self._h, m, comp, _dp(out)))
        return out

    def set_field(self, name: str, arr: np.ndarray, medium: str = "air") -> None:
        m = {"air": 0, "pore": 1}[medium]
        a = np.ascontiguousarray(arr, dtype=np.float64)
        self._check(self._L.fdtd_set_field(self._h, m, _COMP[name], _dp(a)))

    def psi(self) -> np.ndarray:
        out = np.zeros((self.I, self.K, 6), dtype=np.float64)
        self._check(self._L.fdtd_get_psi(self._h, _dp(out)))
        return out

    def ground_psi(self) -> np.ndarray:
        """Impedance-ground TDBC state [i][j][6] (tdbc_ground.dat), FP64."""
        out = np.zeros((self.I, self.J, 6), dtype=np.float64)
        self._check(self._L.fdtd_get_ground_psi(self._h, _dp(out)))
        return out

    def slabs(self):
        res = {}
        for s, name in enumerate(_SLABS):
            dims = (ctypes.c_int * 3)()
            if not self._check(self._L.fdtd_get_slab(self._h, s, 0, None, dims)):
                continue
            q = {}
            for c, cname in enumerate("uvwp"):
                a = np.zeros(tuple(dims), dtype=np.float64)
                self._check(self._L.fdtd_get_slab(self._h, s, c, _dp(a), dims))
                q[cname] = a
            res[name] = q
        return res

    def state_elems(self) -> int:
        return int(self._L.fdtd_state_elems(self._h))

    def copy_state(self, host: np.ndarray, to_device: bool) -> None:
        self._check(self._L.fdtd_copy_state(self._h, 1 if to_device else 0, host.ctypes.data_as(ctypes.c_void_p)))

    def get_data_contour(self, path: str, binary: bool = False) -> None:
        """airpore::get_data_contour: the pressure contour of the current state
        (every 4th node plus the last) as the reference's Tecplot file, or
        the binary variant."""
        self._check(self._L.fdtd_write_contour(self._h, os.fsencode(path), 1 if binary else 0))

    def Save_restart(self, path: str) -> None:
        """airpore::Save_restart: the state in the reference's restart layout
        plus the frame counters and TDBC state."""
        self._check(self._L.fdtd_save_restart(self._h, os.fsencode(path)))

    def Read_restart(self, path: str, reference_semantics: bool = False) -> None:
        """airpore::Read_restart: load a restart file (this library's or the
        reference's) for the same case; continue with advance. With
        reference_semantics the PML integrals and TDBC state restart from zero,
        as the reference's own restart continues."""
        self._check(self._L.fdtd_load_restart(self._h, os.fsencode(path), 1 if reference_semantics else 0))

    def set_tiling(self, rows_per_block: int, planes_per_block: int, threads_per_block: int,
                   vector_width: int = 0, ring_stages: int = 0) -> None:
        """Tile of the single-pass marching kernel: rows, planes and threads per
        block (threads round down to whole rows of column-vector threads),
        columns per thread (0: 16 bytes of columns) and staging-ring planes
        (0: the minimum)."""
        self._check(self._L.fdtd_set_tiling(self._h, rows_per_block, planes_per_block, threads_per_block,
                                            vector_width, ring_stages))

    def set_tile_shape(self, kind: int, rows: int, vectors: int, planes: int, ring_stages: int = 4) -> None:
        """Largest tile of the tiled kernel for kind 0 (full tiles: faces,
        PML edges and corners, TDBC), 1 (lean interior tiles) or 2 (tiles
        inside one PML layer): rows, 16-byte column vectors and planes per
        tile, TMA ring stages; selects the tiled kernel."""
        self._check(self._L.fdtd_set_tile_shape(self._h, kind, rows, vectors, planes, ring_stages))

    def tile_shape(self) -> dict:
        out = (ctypes.c_int * 19)()
        self._check(self._L.fdtd_get_tile_shape(self._h, out))
        keys = ("rows", "vectors", "planes", "stages", "threads", "tiles")
        return {"full": dict(zip(keys, out[0:6])), "lean": dict(zip(keys, out[6:12])),
                "pml": dict(zip(keys, out[12:18])), "tiled": bool(out[18])}

    def set_block_trace(self, on: bool) -> None:
        """Record the block timeline of the tiled kernel from the next advance
        on (a profiling aid; one global-timer read per block when off)."""
        self._check(self._L.fdtd_set_block_trace(self._h, 1 if on else 0))

    def block_trace(self) -> np.ndarray:
        """uint64 [64 step slots, 10 tile kinds, 4]: earliest block start,
        latest block end (global timer, ns; start 2^64-1 where the kind did
        not run), summed block durations (ns), blocks. Kinds: 0 full, 1
        lean, 2 + LM PML / face with layer set LM (bit 0 x, 1 y, 2 z)."""
        out = np.zeros(64 * 10 * 4, dtype=np.uint64)
        self._check(self._L.fdtd_get_block_trace(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_ulonglong))))
        return out.reshape(64, 10, 4)

    def autotune(self, nsteps: int = 20) -> Tuple[int, int, int, int, int]:
        best = (ctypes.c_int * 5)()
        self._check(self._L.fdtd_autotune(self._h, nsteps, best))
        return tuple(best)

    def launch_count(self) -> int:
        return int(self._L.fdtd_launch_count(self._h))

    def last_device_ms(self) -> float:
        v = ctypes.c_double()
        self._check(self._L.fdtd_last_device_ms(self._h, ctypes.byref(v)))
        return v.value

    def receivers(self, first_step: int, nsteps: int) -> np.ndarray:
        """Receiver pressure of steps [first_step, first_step + nsteps) already
        taken (by ``advance`` or an :class:`Ensemble`): [nsteps][nrec]."""
        out = np.zeros((nsteps, max(self.nrec, 1)))
        self._check(self._L.fdtd_get_receivers(self._h, first_step, nsteps, _dp(out)))
        return out[:, : self.nrec]

    def set_wait_limit(self, polls: int) -> None:
        """Polls a staged-copy wait of the marching kernel makes before the
        step reports FDTD_ERR_TIMEOUT (0: at the first wait; < 0: default)."""
        self._check(self._L.fdtd_set_wait_limit(self._h, polls))


class Ensemble:
    """Independent :class:`Airpore` solves of one precision on one device
    stepped together: one batched marching launch per group of members per
    step, the time loop in a CUDA graph. Members keep their own receivers,
    horizon (``reset``) and read-out, and must stay open while the ensemble
    is used."""

    def __init__(self, members: Sequence[Airpore], lib_path: Optional[str] = None, mode: int = 1):
        if not members:
            raise FdtdError(FDTD_ERR_ARG, "an ensemble needs at least one member")
        self._L = members[0]._L if lib_path is None else load_library(lib_path)
        self.members = list(members)
        arr = (ctypes.c_void_p * len(members))(*[m._h.value for m in members])
        self._h = ctypes.c_void_p()
        self._check(self._L.fdtd_ensemble_create(arr, len(members), ctypes.byref(self._h)))
        self._check(self._L.fdtd_ensemble_set_mode(self._h, mode))

    def _check(self, rc: int) -> None:
        if rc < 0:
            raise FdtdError(rc, self._L.fdtd_last_error().decode())

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            self._L.fdtd_ensemble_destroy(self._h)
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

    def advance(self, nsteps: int) -> int:
        """Lock-step steps of every member; returns the steps taken (bounded by
        the nearest member horizon)."""
        n = ctypes.c_int()
        self._check(self._L.fdtd_ensemble_advance(self._h, nsteps, ctypes.byref(n)))
        return n.value

    def autotune(self, nsteps: int = 10) -> Tuple[int, int]:
        """One tile rule (rows, planes per block) for all members, timed on the
        whole ensemble; members end reset to t = 0."""
        best = (ctypes.c_int * 2)()
        self._check(self._L.fdtd_ensemble_autotune(self._h, nsteps, best))
        return best[0], best[1]

    def info(self) -> dict:
        v = (ctypes.c_longlong * 3)()
        self._check(self._L.fdtd_ensemble_info(self._h, v))
        return {"launches": v[0], "groups": v[1], "blocks_per_step": v[2]}

    def last_device_ms(self) -> float:
        v = ctypes.c_double()
        self._check(self._L.fdtd_ensemble_last_device_ms(self._h, ctypes.byref(v)))
        return v.value


# --------------------------------------------------------------- spectra
# Base-2 third-octave centres 1000 * 2^(n/3) Hz from 50 Hz to 2 kHz (17 bands).
THIRD_OCTAVE_50_2K = tuple(1000.0 * 2.0 ** (n / 3.0) for n in range(-13, 4))


def _check_rc(L, rc: int) -> None:
    if rc != FDTD_OK:
        raise FdtdError(rc, L.fdtd_last_error().decode())


def _fft_m(fft_m: int) -> int:
    if not 1 <= fft_m <= 24:
        raise FdtdError(FDTD_ERR_ARG, "fft_m must be 1..24")
    return 1 << fft_m


def _traces(traces) -> np.ndarray:
    a = np.ascontiguousarray(np.atleast_2d(np.asarray(traces, dtype=np.float64)))
    if a.ndim != 2 or a.shape[1] < 1:
        raise FdtdError(FDTD_ERR_ARG, "traces must be [nrec][nt]")
    return a


def fft(traces, fft_m: int, device: int = 0, lib_path: Optional[str] = None) -> Tuple[np.ndarray, np.ndarray]:
    """The reference's post-processing transform (airpore::get_FFT_y1 with
    FFT(1, m, ...)) of every receiver trace on the GPU: zero-padded to 2^m
    points, forward, scaled by 1/2^m. Returns re, im [nrec][2^m]."""
    L = load_library(lib_path)
    t = _traces(traces)
    n = _fft_m(fft_m)
    re = np.empty((t.shape[0], n))
    im = np.empty((t.shape[0], n))
    _check_rc(L, L.fdtd_fft(device, _dp(t), t.shape[0], t.shape[1], fft_m, _dp(re), _dp(im)))
    return re, im


def spectrum(traces, fft_m: int, dt: float, k0: int = 0, nk: Optional[int] = None, device: int = 0,
             lib_path: Optional[str] = None) -> Tuple[np.ndarray, np.ndarray]:
    """FFT_output's spectrum: frequencies k / (dt 2^m) and magnitudes |X_k|
    [nrec][nk] for k = k0 .. k0+nk-1 (default: all 2^(m-1)+1 bins)."""
    L = load_library(lib_path)
    t = _traces(traces)
    n = _fft_m(fft_m)
    if nk is None:
        nk = n // 2 + 1 - k0
    mag = np.empty((t.shape[0], nk))
    _check_rc(L, L.fdtd_spectrum(device, _dp(t), t.shape[0], t.shape[1], fft_m, k0, nk, _dp(mag)))
    return (k0 + np.arange(nk)) / (dt * n), mag


def band_levels(traces, fft_m: int, dt: float, centres=THIRD_OCTAVE_50_2K, device: int = 0,
                lib_path: Optional[str] = None) -> np.ndarray:
    """Band levels 10 log10(sum |X_k|^2) over each band [fc 2^-1/6, fc 2^1/6)
    per receiver trace: [nrec][nband] dB."""
    L = load_library(lib_path)
    t = _traces(traces)
    fc = np.ascontiguousarray(centres, dtype=np.float64)
    out = np.empty((t.shape[0], len(fc)))
    _check_rc(L, L.fdtd_band_levels(device, _dp(t), t.shape[0], t.shape[1], fft_m, dt, len(fc), _dp(fc), _dp(out)))
    return out


def excess_attenuation(traces, free_field_traces, fft_m: int, dt: float, centres=THIRD_OCTAVE_50_2K,
                       device: int = 0, lib_path: Optional[str] = None) -> np.ndarray:
    """Excess attenuation per band [nrec][nband] dB: the band levels of the
    solve with ground (and terrain, wind) minus those of the same source and
    receivers in a free field (all faces absorbing)."""
    return band_levels(traces, fft_m, dt, centres, device, lib_path) - \
        band_levels(free_field_traces, fft_m, dt, centres, device, lib_path)

