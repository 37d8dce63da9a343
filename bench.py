#!/usr/bin/env python
"""Throughput benchmark of the B200 FDTD time-marching path.

Workload (N=1): porous ground under air over an analytic hill, 256 (range,
Y/j) x 128 (X/i) x 96 (Z/k) air nodes over a 16-cell Zwikker-Kosten layer
(sigma 200 kPa s/m^2, porosity 0.3, tortuosity 1.8) with the two-plane
airpore interface, the hill z_g = h exp(-(y - y0)^2 / 2w^2) (h = 0.5 m,
w = 1 m, y0 mid-range) on a terrain-following grid stretched vertically
(metrics in FP64 on the host), 20-node PML on the five air faces, FB_p_v,
source height above the ground drawn from a seed, 8 receivers 1 m above the
ground; synthetic setup generated from a seed (``--flat``: the same domain
on flat ground).  One bench step = ``--inner`` forward-backward time steps of
the whole domain with the state resident in HBM; L2 is flushed (a 512 MB
write) between bench steps.  The headline ``value`` is FP32; the FP64 path
is reported beside it.

``--impl reference`` times the reference solver itself (the unmodified
sources compiled under oracle/_ref/, driven through airpore's own loop) on
the host cores: one independent single-rank process per core (the
reference's MPI decomposition has no MPI here), aggregate throughput. The
reference has no terrain-following grid (it ignores terrain.dat and runs
the domain on flat ground); its per-step work is the same, since it
evaluates all nine metric terms at every node either way.

Multi-GPU: replicas only -- each rank runs its own independent solve, no
collective on the data path; value = all ranks' cell updates / max time.

The domain line carries a ``surrogate`` section (skip with
``--no-surrogate``; alone with ``--workload surrogate``): a 5-network bf16
ensemble trained on the committed FDTD dataset, its held-out error and
fallback rate, its inference throughput on 1 M queries in HBM against the
bf16 tensor roofline, and the speed-up over the FDTD solves it replaces.

``--workload ensemble`` measures the batched ensemble instead: ``--members``
independent FP32 solves drawn by casegen.ensemble_member (seed = rank),
stepped by batched marching launches in a graph-captured loop, tile rule
from the ensemble autotuner; value = all members' cell updates / device
time. Every member (or the first ``--check-members``) is then checked
against its own FP64 single solve (receiver relative L2 over
``--check-steps`` steps).
"""

from __future__ import annotations

import argparse
import importlib
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Gcell-upd/s & % HBM peak, FP32 vs FP64 at <=1e-4 rel err; surrogate speedup"
UNIT = "Gcell-upd/s"
WORKLOAD = ("porous ground under a Gaussian hill (h 0.5 m, w 1 m) on a terrain-following grid + 20-node PML, "
            "256x128x96 air + 256x128x18 porous nodes, FB_p_v")
FLAT_WORKLOAD = "porous ground + 20-node PML, 256x128x96 air + 256x128x18 porous nodes, FB_p_v"
FLAT = "--flat" in sys.argv


def make_case(tmp: str):
    casegen = importlib.import_module("3d_mpi_test_b200.casegen")
    make = casegen.porous_ground if FLAT else casegen.porous_hill
    case, rec = make(ni=128, nj=256, nk=96, layer=16, d=0.05, steps=4000, pml=20, seed=0)
    d = os.path.join(tmp, "porous_ground" if FLAT else "porous_hill")
    case.write(d)
    casegen.write_receivers(os.path.join(d, "rec.txt"), rec)
    air = case.NI * case.NJ * case.NK
    pore = case.NI * case.NJ * len(case.pore_Z)
    return d, rec, air + pore, case


def algorithmic_bytes(case, word: int) -> dict:
    """Per FB step: every node's u,v,w,p read once and written once (8 words),
    plus 8 words (Qu,Qv,Qw,Qp read+write) per PML slab storage node, plus
    the TDBC state and receiver words."""
    I, J, K = case.NI, case.NJ, case.NK
    I1, I2, J1, J2, K1, K2 = case.pml_nodes
    cells = I * J * K + I * J * len(case.pore_Z or [])
    slab = 0
    slab += (I1 + 1) * J * K if I1 else 0
    slab += (I2 + 1) * J * K if I2 else 0
    slab += I * (J1 + 1) * K if J1 else 0
    slab += I * (J2 + 1) * K if J2 else 0
    slab += I * J * (K2 + 1) if K2 else 0
    tdbc = I * K if case.bc[2] == 5 else 0
    b = cells * 8 * word + slab * 8 * word + tdbc * 12 * 8 + 8 * 8
    return {"bytes_per_step": b, "cells": cells, "slab_nodes": slab}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        if shutil.which("nvidia-smi"):
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        return self

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[4:8]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ---------------------------------------------------------------- CPU side
def ref_harness_path():
    p = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
    return p if os.path.exists(p) else None


def time_reference(case_dir: str, cells: int, steps: int, warmup: int, replicas: int):
    """Run `replicas` independent reference processes; returns aggregate
    Gcell-upd/s and the per-process ms/step."""
    exe = ref_harness_path()
    if exe is None:
        return None
    procs = [subprocess.Popen([exe, case_dir, "--time", str(warmup), str(steps)], stdout=subprocess.PIPE,
                              stderr=subprocess.DEVNULL, text=True) for _ in range(replicas)]
    ms = []
    for p in procs:
        out, _ = p.communicate()
        for ln in out.splitlines():
            if ln.startswith("{"):
                ms.append(json.loads(ln)["ms_per_step"])
    if len(ms) != replicas:
        return None
    worst = max(ms)
    return {"value": replicas * cells / (worst * 1e-3) / 1e9, "ms_per_step": worst, "cores": replicas}


def host_replicas(bytes_per_process=700e6) -> int:
    n = os.cpu_count() or 1
    try:
        with open("/proc/meminfo") as f:
            for ln in f:
                if ln.startswith("MemAvailable"):
                    avail = float(ln.split()[1]) * 1024
                    n = max(1, min(n, int(0.6 * avail / bytes_per_process)))
    except OSError:
        pass
    return n


def cpu_baseline(case_dir: str, cells: int):
    """Bounded sample on rank 0: the reference (or, if its build is absent,
    the oracle restatement) over 3 steps after 1 warm-up step, all cores."""
    reps = host_replicas()
    r = time_reference(case_dir, cells, steps=3, warmup=1, replicas=reps)
    if r is not None:
        return {"value": round(r["value"], 6), "unit": UNIT, "cores": r["cores"], "kind": "reference",
                "sample": f"{reps} independent single-rank reference processes x 3 FB steps of the bench workload "
                          f"(after 1 warm-up step; the reference runs it on flat ground, same per-step work); "
                          f"{r['ms_per_step']:.0f} ms/step each"}
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle  # the checker's own CPU restatement, timed only as the baseline

    oc = oracle.OracleCase(case_dir)
    oc.run(1)
    t0 = time.perf_counter()
    oc.run(3)
    dt = (time.perf_counter() - t0) / 3
    return {"value": round(cells / dt / 1e9, 6), "unit": UNIT, "cores": 1, "kind": "port",
            "sample": "oracle restatement, 1 core, 3 FB steps of the bench workload"}


# ---------------------------------------------------------------- GPU side
ENS_WORKLOAD = ("batched ensemble: seeded members, NJ U[64,512] x NK U[32,192], NI 3 (2D) for half and "
                "U[32,96] else, porous ground 8 cells, porous hill, log wind, 10-node PML, FP32")


def run_ensemble(args, rank, world, local_rank):
    import numpy as np
    import torch

    pkg = importlib.import_module("3d_mpi_test_b200")
    casegen = importlib.import_module("3d_mpi_test_b200.casegen")
    replicas = importlib.import_module("3d_mpi_test_b200.replicas")
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist  # noqa: F811
    group = replicas.ReplicaGroup(dist, "cuda")
    tmp = tempfile.mkdtemp(prefix=f"bench_ens_r{rank}_")
    inner = args.inner
    horizon = (args.warmup + args.steps) * inner + 8
    specs, cells, mem = [], 0, []
    t_setup = time.perf_counter()
    for i in range(args.members):
        c, rec, p = casegen.ensemble_member(rank, i, steps=horizon, wind="reference" if args.ens_mode == 0 else "loglaw")
        d = c.write(os.path.join(tmp, f"m{i:03d}"))
        specs.append((d, rec, p))
        cells += c.NI * c.NJ * (c.NK + len(c.pore_Z))
        a = pkg.Airpore(d, "f32", device=local_rank)
        a.set_receivers(rec)
        a.reset(horizon)
        mem.append(a)
    ens = pkg.Ensemble(mem, mode=args.ens_mode)
    # the project's ensemble autotuner: mode 0 tunes the batched row
    # marching kernel's tiles, mode 1 one set of tile shapes for every
    # member's tiled kernels (timing whole-ensemble steps)
    tile = ens.autotune(3)
    for a in mem:
        a.reset(horizon)
    setup_s = time.perf_counter() - t_setup
    for _ in range(args.warmup):
        ens.advance(inner)
    group.barrier()
    torch.cuda.synchronize()
    launches0 = ens.info()["launches"]
    dev_ms = 0.0
    sampler = ClockSampler(local_rank)
    with sampler:
        for _ in range(args.steps):
            ens.advance(inner)  # inputs (hundreds of MB per member set) are far larger than L2
            dev_ms += ens.last_device_ms()
    torch.cuda.synchronize()
    group.barrier()
    info = ens.info()
    steps_total = args.steps * inner
    gcell = group.throughput(cells, steps_total, dev_ms)
    dev_ms = group.max_over_ranks(dev_ms)
    # end to end: each bench step starts every member from its initial
    # condition (host-side Gaussian, H2D upload), steps it and reads all
    # receiver series back
    h2d = sum(a.state_elems() for a in mem) * 4  # the initial FP32 pressure field of each member
    e2e_n = 2
    t1 = time.perf_counter()
    nrec_words = 0
    for _ in range(e2e_n):
        for a in mem:
            a.reset(horizon)
        ens.advance(inner)
        nrec_words = 0
        for a in mem:
            nrec_words += a.receivers(0, inner).size
    torch.cuda.synchronize()
    e2e_s = group.max_over_ranks(time.perf_counter() - t1)
    e2e = {"value": round(world * cells * inner * e2e_n / e2e_s / 1e9, 3), "unit": UNIT,
           "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(nrec_words * 8)}
    # every member against its own FP64 single solve
    nchk = min(args.check_members, len(mem)) if args.check_members >= 0 else len(mem)
    for a in mem:
        a.reset(horizon)
    ens.advance(args.check_steps)
    errs = []
    for (d, rec, p), a in zip(specs[:nchk], mem[:nchk]):
        r32 = a.receivers(0, args.check_steps)
        with pkg.Airpore(d, "f64", device=local_rank) as b:
            b.set_receivers(rec)
            r64 = b.get_output(args.check_steps)
        errs.append(float(np.linalg.norm(r32 - r64) / np.linalg.norm(r64)))
    ens.close()
    for a in mem:
        a.close()
    shutil.rmtree(tmp, ignore_errors=True)
    if rank != 0:
        return None
    return {
        "metric": "Gcell-upd/s of a batched ensemble (FP32), each member checked against its FP64 single solve",
        "value": round(gcell, 3), "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(dev_ms / args.steps, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded ensemble generator)",
        "config": {"workload": ENS_WORKLOAD, "members": args.members, "cells_per_fb_step": cells,
                   "inner_fb_steps_per_bench_step": inner, "l2": "inputs larger than L2",
                   "tile_rows_planes": list(tile), "launch_groups": info["groups"],
                   "launch_mode": ["one batched launch per group per step",
                                   "each member's own launch, 16 streams"][args.ens_mode],
                   "blocks_per_fb_step": info["blocks_per_step"], "setup_s": round(setup_s, 1),
                   "parallelism": f"replicas x{world}" if world > 1 else "one device"},
        "check": {"members": nchk, "steps": args.check_steps, "max_rel_l2_receivers_vs_fp64": max(errs),
                  "median_rel_l2": statistics.median(errs)},
        "e2e": e2e,
        "gpu_launches": int(info["launches"] - launches0),
        "clocks": sampler.summary(),
    }


WINDOW_WORKLOAD = ("moving window 256 (i) x 1024 (j) x 192 (k) = 50.3 M nodes over an 11264-node range, "
                   "frames of 10 cells following the pulse at c0, log-law wind u*=0.4 m/s kappa=0.41 z0=0.01 m "
                   "(upwind advection), 6-pole TDBC ground fitted to Miki at 50 kPa s/m^2, 20-node PML on top, "
                   "front and back, rigid leading and trailing faces, FP32 fields, FP64 TDBC state")


def run_window(args, rank, world, local_rank):
    """The long-range configuration's shape: a 50.3 M-node window moving
    over the range (frame shifts inside the timed region)."""
    import torch

    pkg = importlib.import_module("3d_mpi_test_b200")
    casegen = importlib.import_module("3d_mpi_test_b200.casegen")
    replicas = importlib.import_module("3d_mpi_test_b200.replicas")
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist  # noqa: F811
    group = replicas.ReplicaGroup(dist, "cuda")
    tmp = tempfile.mkdtemp(prefix=f"bench_win_r{rank}_")
    case, rec = casegen.moving_window()
    d = case.write(os.path.join(tmp, "window"))
    cells = case.NI * 1024 * case.NK
    hbm_peak, peak_kind = peaks()
    inner = args.inner
    a = pkg.Airpore(d, "f32", device=local_rank)
    a.set_receivers(rec)
    a.reset((args.warmup + args.steps) * inner + 8)
    for _ in range(args.warmup):
        a.advance(inner)
    group.barrier()
    l0 = a.launch_count()
    ms = 0.0
    sampler = ClockSampler(local_rank)
    with sampler:
        for _ in range(args.steps):
            a.advance(inner)  # 1.7 GB of FP32 state: far larger than L2
            ms += a.last_device_ms()
    torch.cuda.synchronize()
    group.barrier()
    launches = a.launch_count() - l0
    steps_total = args.steps * inner
    gcell = group.throughput(cells, steps_total, ms)
    ms = group.max_over_ranks(ms)
    slab = 2 * 21 * 1024 * 192 + 256 * 1024 * 21  # x1 x2 z2 storage nodes
    bytes_step = cells * 8 * 4 + slab * 8 * 4
    achieved = bytes_step / (ms * 1e-3 / steps_total) / 1e9
    a.close()
    shutil.rmtree(tmp, ignore_errors=True)
    if rank != 0:
        return None
    return {
        "metric": "Gcell-upd/s of the moving-window configuration (FP32)", "value": round(gcell, 3), "unit": UNIT,
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded case generator)",
        "config": {"workload": WINDOW_WORKLOAD, "inner_fb_steps_per_bench_step": inner, "cells_per_fb_step": cells,
                   "frame_shifts_in_timed_region": int(steps_total // 20), "l2": "inputs larger than L2"},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": hbm_peak, "unit": "GB/s",
                     "frac": round(achieved / hbm_peak, 4), "peak_kind": peak_kind,
                     "algorithmic_bytes_per_step": bytes_step},
        "gpu_launches": int(launches), "clocks": sampler.summary(),
    }


def run_window_full(args, local_rank):
    """The long-range configuration run end to end once per precision:
    `--window-steps` steps (20000) of the moving window with its wind and
    ground, receivers every 5 m to 100 m at 1.5 m. Reports each run's
    device rate, the FP32 receiver error against FP64 (rel L2 of p(t) and
    dB per third-octave band, 50 Hz - 2 kHz), the peak pressure and the
    FP64 band levels per receiver (written to --window-out as .npz)."""
    import numpy as np
    import torch

    pkg = importlib.import_module("3d_mpi_test_b200")
    casegen = importlib.import_module("3d_mpi_test_b200.casegen")
    torch.cuda.set_device(local_rank)
    tmp = tempfile.mkdtemp(prefix="bench_winfull_")
    n = args.window_steps
    case, rec = casegen.moving_window(steps=n)
    d = case.write(os.path.join(tmp, "window"))
    cells = case.NI * 1024 * case.NK
    runs = {}
    for prec in ("f32", "f64"):
        a = pkg.Airpore(d, prec, device=local_rank)
        a.set_receivers(rec)
        a.reset(n)
        sampler = ClockSampler(local_rank)
        t0 = time.perf_counter()
        with sampler:
            r = a.advance(n)
        wall = time.perf_counter() - t0
        ms = a.last_device_ms()
        p = a.field("p")
        runs[prec] = {"rec": np.asarray(r), "ms": ms, "wall_s": wall, "gcell": cells * n / (ms * 1e-3) / 1e9,
                      "p_max": float(np.abs(p).max()), "finite": bool(np.all(np.isfinite(p))),
                      "clocks": sampler.summary(), "launches": a.launch_count()}
        a.close()
    fft_m = int(np.ceil(np.log2(n)))
    lv = {k: pkg.band_levels(v["rec"].T, fft_m, case.dt) for k, v in runs.items()}
    dl = np.abs(lv["f32"] - lv["f64"])
    r32, r64 = runs["f32"]["rec"], runs["f64"]["rec"]
    per_rec = np.linalg.norm(r32 - r64, axis=0) / np.maximum(np.linalg.norm(r64, axis=0), 1e-300)
    if args.window_out:
        np.savez(args.window_out, rec_f32=r32, rec_f64=r64, levels_f32=lv["f32"], levels_f64=lv["f64"],
                 centres=np.asarray(pkg.THIRD_OCTAVE_50_2K), ranges=np.asarray([x[1] for x in rec]))
    shutil.rmtree(tmp, ignore_errors=True)
    return {
        "metric": "Gcell-upd/s of the long-range configuration run end to end (FP32)",
        "value": round(runs["f32"]["gcell"], 3), "unit": UNIT, "n_gpus": 1, "steps": n, "warmup": 0,
        "higher_is_better": True, "dtype": "f32", "data": "synthetic (seeded case generator)",
        "config": {"workload": WINDOW_WORKLOAD, "fb_steps": n, "receivers_m": [x[1] for x in rec]},
        "f64_gcell": round(runs["f64"]["gcell"], 3),
        "device_s": {k: round(v["ms"] / 1e3, 3) for k, v in runs.items()},
        "wall_s": {k: round(v["wall_s"], 3) for k, v in runs.items()},
        "finite": {k: v["finite"] for k, v in runs.items()},
        "p_max_final": {k: v["p_max"] for k, v in runs.items()},
        "rec_p_max": float(np.abs(r64).max()),
        "fp32_error": {"rel_l2_all": float(np.linalg.norm(r32 - r64) / np.linalg.norm(r64)),
                       "rel_l2_per_receiver_max": float(per_rec.max()),
                       "band_db_max": float(dl.max()), "band_db_mean": float(dl.mean())},
        "clocks": {k: v["clocks"] for k, v in runs.items()},
    }


def bf16_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["bf16_tflops"]), "measured (burst cuBLAS bf16)"
    return 1590.0, "fallback"


def run_surrogate(queries: int = 1_000_000, members: int = 5, steps: int = 12000, device: int = 0) -> dict:
    """The learned surrogate on this GPU: a `members`-network bf16 ensemble
    trained on the committed FDTD dataset (3d_mpi_test_b200/data), its
    held-out error and FDTD fallback rate, its inference throughput on
    `queries` seeded queries resident in HBM (CUDA events), the end-to-end
    rate from host arrays, and the time per query of the FDTD solves it
    replaces (ground + free-field pair through the batched ensemble)."""
    import numpy as np
    import torch

    sur = importlib.import_module("3d_mpi_test_b200.surrogate")
    sd = importlib.import_module("3d_mpi_test_b200.surrogate_data")
    Xtr, Etr, Xte, Ete = sd.load_dataset()
    s = sur.Surrogate(members=members, seed=1)
    t0 = time.perf_counter()
    losses = s.fit(Xtr, Etr, steps=steps)
    train_s = time.perf_counter() - t0
    train_ms = sum(n.info()["last_device_ms"] for n in s.nets)
    y, spread = s.predict(Xte)
    err = np.abs(y - Ete)
    kept = spread <= 1.0
    per_band = err.reshape(len(Xte), sd.N_REC, len(sd.BANDS)).mean(axis=(0, 1))
    # inference: query rows resident in HBM; the ray-feature kernel (CUDA
    # events on its stream) and every member (CUDA events inside the library)
    Xq = sd.draw(99, queries).astype(np.float32)
    pq = torch.from_numpy(Xq).cuda(device)
    xd = torch.empty((queries, sd.N_FEATURES), dtype=torch.float32, device=f"cuda:{device}")
    yd = torch.empty((queries, Etr.shape[1]), dtype=torch.float32, device=f"cuda:{device}")
    st = torch.cuda.current_stream(device)
    sur.ray_features(pq.data_ptr(), 4096, xd.data_ptr(), st.cuda_stream)  # warm-up
    for n in s.nets:
        n.predict_device(xd.data_ptr(), 4096, yd.data_ptr())  # warm-up
    l0 = sum(n.info()["launches"] for n in s.nets)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(device)
    ev0.record(st)
    sur.ray_features(pq.data_ptr(), queries, xd.data_ptr(), st.cuda_stream)
    ev1.record(st)
    torch.cuda.synchronize(device)
    ms = ev0.elapsed_time(ev1)
    for n in s.nets:
        n.predict_device(xd.data_ptr(), queries, yd.data_ptr())
        ms += n.info()["last_device_ms"]
    launches = sum(n.info()["launches"] for n in s.nets) - l0 + 1  # + the ray-feature kernel
    width, K0, NO = 512, 64, 256  # padded GEMM shapes of one member
    flop_padded = 2.0 * (K0 * width + 3 * width * width + width * NO)
    flop_alg = 2.0 * (sd.N_FEATURES * width + 3 * width * width + width * Etr.shape[1])
    peak, peak_kind = bf16_peak()
    tflops = members * queries * flop_padded / (ms * 1e-3) / 1e12
    # end to end from host parameter arrays: features, H2D of the inputs, D2H of the answers
    t0 = time.perf_counter()
    s.predict(Xq)
    e2e_s = time.perf_counter() - t0
    # the method without the network: an FDTD solve pair per query
    nf = 16
    t0 = time.perf_counter()
    sd.solve(Xte[:nf])
    fdtd_s = (time.perf_counter() - t0) / nf
    s.close()
    return {
        "members": members, "layers": "11 parameters + 16 ray-geometry features -> 4 x 512 ReLU -> 136 (17 bands x 8 receivers), "
                                    "bf16 weights, FP32 accumulate",
        "train": {"samples": int(len(Xtr)), "steps_per_member": steps, "batch": 256, "wall_s": round(train_s, 2),
                  "device_ms": round(train_ms, 1), "final_loss_normalised": [round(float(v), 5) for v in losses]},
        "held_out": {"samples": int(len(Xte)), "mae_db": round(float(err.mean()), 3),
                     "rmse_db": round(float(np.sqrt((err ** 2).mean())), 3),
                     "mae_db_per_band": [round(float(v), 2) for v in per_band],
                     "fdtd_fallback_fraction_at_1db": round(float(1 - kept.mean()), 3),
                     "mae_db_answered_by_network": round(float(err[kept].mean()), 3) if kept.any() else None},
        "inference": {"queries": queries, "queries_per_s": round(queries / (ms * 1e-3), 1), "ms": round(ms, 3),
                      "gpu_launches": int(launches),
                      "roofline": {"bound": "tensor", "achieved": round(tflops, 1), "peak": peak, "unit": "TFLOP/s",
                                   "frac": round(tflops / peak, 4), "peak_kind": peak_kind,
                                   "flop_per_query_member_padded": flop_padded,
                                   "flop_per_query_member_algorithmic": flop_alg}},
        "e2e_queries_per_s": round(queries / e2e_s, 1),
        "fdtd_s_per_query": round(fdtd_s, 5),
        "speedup_vs_fdtd": round(fdtd_s / (e2e_s / queries), 1),
    }


def run_profile(args, local_rank):
    """One precision of the headline workload for a profiler: autotuned
    tiles (or --tile-shapes), two warm-up FB steps, then --profile-steps FB
    steps between cudaProfilerStart and cudaProfilerStop (ncu
    --profile-from-start off captures just those). Prints the tile shapes
    and the device time of the profiled steps."""
    import torch

    pkg = importlib.import_module("3d_mpi_test_b200")
    torch.cuda.set_device(local_rank)
    tmp = tempfile.mkdtemp(prefix="bench_prof_")
    case_dir, rec, cells, case = make_case(tmp)
    a = pkg.Airpore(case_dir, args.profile_prec, device=local_rank)
    if args.tile_shapes:
        for kind, spec in enumerate(args.tile_shapes.split(";")):
            if spec:
                a.set_tile_shape(kind, *(int(x) for x in spec.split(",")))
    else:
        a.autotune(10)
    a.set_receivers(rec)
    a.reset(args.profile_steps + 8)
    if args.block_trace:
        if args.profile_steps > 64:
            raise SystemExit("--block-trace keeps at most 64 steps apart")
        a.set_block_trace(True)
    a.advance(2)
    torch.cuda.synchronize()
    torch.cuda.profiler.start()
    a.advance(args.profile_steps)
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    ms = a.last_device_ms()
    out = {"profile": args.profile_prec, "fb_steps": args.profile_steps, "device_ms": round(ms, 4),
           "gcell": round(cells * args.profile_steps / (ms * 1e-3) / 1e9, 3), "tile_shapes": a.tile_shape(),
           "workload": FLAT_WORKLOAD if FLAT else WORKLOAD}
    if args.block_trace:
        out["block_trace"] = block_trace_summary(a.block_trace())
    a.close()
    shutil.rmtree(tmp, ignore_errors=True)
    return out


TRACE_KINDS = ("full", "lean", "pml_none", "pml_x", "pml_y", "pml_xy", "pml_z", "pml_xz", "pml_yz", "pml_xyz")


def block_trace_summary(tr):
    """Per tile kind over the traced steps: median start and end of its
    blocks relative to the step's first block (us), mean block duration (us)
    and blocks per step; and the median span of a step (first block start
    to last block end)."""
    import numpy as np

    none = np.iinfo(np.uint64).max
    steps = [s for s in range(tr.shape[0]) if (tr[s, :, 3] > 0).any()]
    per, spans = {}, []
    for s in steps:
        live = [k for k in range(tr.shape[1]) if tr[s, k, 3] > 0 and tr[s, k, 0] != none]
        t0 = min(int(tr[s, k, 0]) for k in live)
        spans.append((max(int(tr[s, k, 1]) for k in live) - t0) * 1e-3)
        for k in live:
            q = per.setdefault(TRACE_KINDS[k], {"start": [], "end": [], "block": [], "blocks": int(tr[s, k, 3])})
            q["start"].append((int(tr[s, k, 0]) - t0) * 1e-3)
            q["end"].append((int(tr[s, k, 1]) - t0) * 1e-3)
            q["block"].append(int(tr[s, k, 2]) / int(tr[s, k, 3]) * 1e-3)
    kinds = {k: {"start_us": round(float(np.median(q["start"])), 1), "end_us": round(float(np.median(q["end"])), 1),
                 "block_us": round(float(np.mean(q["block"])), 2), "blocks": q["blocks"]}
             for k, q in sorted(per.items(), key=lambda kv: np.median(kv[1]["start"]))}
    return {"steps": len(steps), "step_span_us": round(float(np.median(spans)), 1) if spans else None, "kinds": kinds}


def run_ensemble_profile(args, local_rank):
    """The ensemble workload for a profiler: every member set up, two
    warm-up steps, then --profile-steps steps of all members between
    cudaProfilerStart and cudaProfilerStop (mode 1, default tiles)."""
    import torch

    pkg = importlib.import_module("3d_mpi_test_b200")
    casegen = importlib.import_module("3d_mpi_test_b200.casegen")
    torch.cuda.set_device(local_rank)
    tmp = tempfile.mkdtemp(prefix="bench_ensprof_")
    horizon = args.profile_steps + 8
    mem, cells = [], 0
    for i in range(args.members):
        c, rec, p = casegen.ensemble_member(0, i, steps=horizon)
        d = c.write(os.path.join(tmp, f"m{i:03d}"))
        cells += c.NI * c.NJ * (c.NK + len(c.pore_Z))
        a = pkg.Airpore(d, "f32", device=local_rank)
        a.set_receivers(rec)
        a.reset(horizon)
        mem.append(a)
    ens = pkg.Ensemble(mem, mode=args.ens_mode)
    ens.advance(2)
    torch.cuda.synchronize()
    torch.cuda.profiler.start()
    ens.advance(args.profile_steps)
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    ms = ens.last_device_ms()
    out = {"profile": "ensemble", "members": args.members, "fb_steps": args.profile_steps, "device_ms": round(ms, 4),
           "gcell": round(cells * args.profile_steps / (ms * 1e-3) / 1e9, 3), "launches": ens.info()["launches"]}
    ens.close()
    for a in mem:
        a.close()
    shutil.rmtree(tmp, ignore_errors=True)
    return out


def run_gpu(args, rank, world, local_rank):
    import numpy as np
    import torch

    pkg = importlib.import_module("3d_mpi_test_b200")
    replicas = importlib.import_module("3d_mpi_test_b200.replicas")
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist  # noqa: F811
    group = replicas.ReplicaGroup(dist, "cuda")
    tmp = tempfile.mkdtemp(prefix=f"bench_r{rank}_")
    case_dir, rec, cells, case = make_case(tmp)
    inner = args.inner
    horizon = max(4000, (args.warmup + args.steps + 2) * inner + 10)
    flush = torch.empty(128 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 512 MB > L2
    hbm_peak, peak_kind = peaks()

    def barrier():
        torch.cuda.synchronize()
        group.barrier()

    max_over_ranks = group.max_over_ranks

    results = {}
    for prec in ("f32", "f64"):
        word = 4 if prec == "f32" else 8
        a = pkg.Airpore(case_dir, prec, device=local_rank)
        tile = None
        if args.tile:
            tile = tuple(int(x) for x in args.tile.split(","))
            try:
                a.set_tiling(*tile)
            except pkg.FdtdError as e:
                print(f"tile {tile} rejected for {prec} ({e}); autotuning", file=sys.stderr)
                tile = None
        if tile is None:
            tile = a.autotune(10)  # the project's tile autotuner, on this domain
        shape = a.tile_shape()
        a.set_receivers(rec)
        a.reset(horizon)
        for _ in range(args.warmup):
            flush.zero_()
            torch.cuda.synchronize()
            a.advance(inner)
        barrier()
        launches0 = a.launch_count()
        dev_ms = 0.0
        t0 = time.perf_counter()
        sampler = ClockSampler(local_rank) if prec == "f32" else None
        if sampler:
            sampler.__enter__()
        try:
            for _ in range(args.steps):
                flush.zero_()
                torch.cuda.synchronize()
                a.advance(inner)
                dev_ms += a.last_device_ms()
        finally:
            if sampler:
                sampler.__exit__(None, None, None)
        barrier()
        wall = time.perf_counter() - t0
        launches = a.launch_count() - launches0
        steps_total = args.steps * inner
        gcell = group.throughput(cells, steps_total, dev_ms)  # whole job: all ranks' cells / slowest rank
        dev_ms = max_over_ranks(dev_ms)
        ab = algorithmic_bytes(case, word)
        achieved = ab["bytes_per_step"] / (dev_ms * 1e-3 / steps_total) / 1e9
        results[prec] = {"gcell": gcell, "ms_per_bench_step": dev_ms / args.steps, "wall_s": wall, "tile": tile,
                         "shape": shape,
                         "launches": launches, "achieved_gbs": achieved, "bytes_per_step": ab["bytes_per_step"],
                         "clocks": sampler.summary() if sampler else None}
        # the error statement: receiver p(t) over the workload's full 4000
        # steps from t = 0, this precision's path with the tuned tile
        results["trace_" + prec] = a.get_output(case.time_domain).T.copy()
        # end to end through the public API with host buffers (FP32 headline only)
        if prec == "f32":
            n = a.state_elems()
            host = torch.empty(4 * n, dtype=torch.float32, pin_memory=True)
            a.copy_state(host.numpy(), to_device=False)
            a.reset(horizon)
            barrier()
            t1 = time.perf_counter()
            for _ in range(args.steps):
                a.copy_state(host.numpy(), to_device=True)  # H2D: the step's input state
                r = a.advance(inner)  # receivers come back D2H inside the call
            torch.cuda.synchronize()
            e2e_s = max_over_ranks(time.perf_counter() - t1)
            results["e2e"] = {"value": world * cells * steps_total / e2e_s / 1e9, "unit": UNIT,
                              "h2d_bytes_per_step": int(host.numel() * 4),
                              "d2h_bytes_per_step": int(r.size * 8)}
        a.close()
    shutil.rmtree(tmp, ignore_errors=True)

    if rank != 0:
        return None
    f32, f64 = results["f32"], results["f64"]
    roof = {"bound": "hbm", "achieved": round(f32["achieved_gbs"], 1), "peak": hbm_peak, "unit": "GB/s",
            "frac": round(f32["achieved_gbs"] / hbm_peak, 4), "traffic": None,
            "peak_kind": peak_kind,
            "kernel": ("k_tile + k_tile_pml_calm: full, lean and PML-layer-set tile launches, together one FB step "
                       "of the whole domain, FP32"
                       if f32["shape"]["tiled"] else "k_march (one launch = one FB step of the whole domain), FP32"),
            "tile_shapes": f32["shape"] if f32["shape"]["tiled"] else list(f32["tile"]),
            "algorithmic_bytes_per_step": f32["bytes_per_step"]}
    fp32_error = fp32_error_statement(results["trace_f32"], results["trace_f64"], case.dt, local_rank)
    prof = os.path.join(ROOT, "profiles", "traffic.txt")
    if os.path.exists(prof):
        with open(prof) as fh:
            for ln in fh:
                if ln.startswith("f32_bytes_per_step:"):
                    roof["traffic"] = int(ln.split(":")[1])
    line = {
        "metric": METRIC, "value": round(f32["gcell"], 3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(f32["ms_per_bench_step"], 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded case generator)",
        "config": {"workload": FLAT_WORKLOAD if FLAT else WORKLOAD, "inner_fb_steps_per_bench_step": args.inner,
                   "cells_per_fb_step": cells, "l2": "flushed (512 MB write) between bench steps",
                   "parallelism": f"replicas x{world}" if world > 1 else "single device-resident domain"},
        "fp64": {"value": round(f64["gcell"], 3), "ms_per_step": round(f64["ms_per_bench_step"], 4),
                 "tile_shapes": f64["shape"] if f64["shape"]["tiled"] else list(f64["tile"]),
                 "achieved_gbs": round(f64["achieved_gbs"], 1),
                 "frac": round(f64["achieved_gbs"] / hbm_peak, 4),
                 "fp32_speedup": round(f32["gcell"] / f64["gcell"], 3)},
        "fp32_error": fp32_error,
        "roofline": roof,
        "e2e": {k: (round(v, 3) if isinstance(v, float) else v) for k, v in results["e2e"].items()},
        "gpu_launches": int(f32["launches"]),
        "clocks": f32["clocks"],
    }
    if world == 1 and not args.no_surrogate:
        line["surrogate"] = run_surrogate(args.sur_queries, steps=args.sur_train_steps, device=local_rank)
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(case_dir_for_cpu(), cells)
    return line


def fp32_error_statement(tr32, tr64, dt: float, device: int) -> dict:
    """FP32 against FP64 on the device for the same workload: relative L2
    of every receiver's p(t) over the whole run, and the band-level error
    per third-octave band (50 Hz - 2 kHz) from the receivers' spectra."""
    import numpy as np

    pkg = importlib.import_module("3d_mpi_test_b200")
    nt = tr64.shape[1]
    fft_m = max(1, int(np.ceil(np.log2(nt))))
    l32 = pkg.band_levels(tr32, fft_m, dt, device=device)
    l64 = pkg.band_levels(tr64, fft_m, dt, device=device)
    db = np.abs(l32 - l64)
    per_rec = [float(np.linalg.norm(a - b) / np.linalg.norm(b)) for a, b in zip(tr32, tr64)]
    return {"steps": int(nt), "receivers": int(tr64.shape[0]),
            "rel_l2_receivers": float(np.linalg.norm(tr32 - tr64) / np.linalg.norm(tr64)),
            "rel_l2_worst_receiver": max(per_rec),
            "band_db_error_max": float(db.max()), "band_db_error_mean": float(db.mean()),
            "band_db_error_max_per_band": [round(float(v), 7) for v in db.max(axis=0)],
            "bands_hz": [round(f, 1) for f in pkg.THIRD_OCTAVE_50_2K], "fft_m": fft_m,
            "within_1e-4": bool(float(np.linalg.norm(tr32 - tr64) / np.linalg.norm(tr64)) <= 1e-4)}


def case_dir_for_cpu():
    tmp = tempfile.mkdtemp(prefix="bench_cpu_")
    return make_case(tmp)[0]


def run_reference_arm(args, world, rank):
    if rank != 0:
        return None
    tmp = tempfile.mkdtemp(prefix="bench_ref_")
    case_dir, rec, cells, case = make_case(tmp)
    exe = ref_harness_path()
    if exe is None:
        return {"impl": "reference", "unavailable": "oracle/_ref/ref_harness not built (needs the reference sources)"}
    reps = host_replicas()
    t0 = time.perf_counter()
    r = time_reference(case_dir, cells, steps=args.steps, warmup=args.warmup, replicas=reps)
    wall = time.perf_counter() - t0
    if r is None:
        return {"impl": "reference", "unavailable": "reference harness failed"}
    v = round(r["value"], 6)
    return {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(r["ms_per_step"], 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded case generator)",
        "config": {"workload": FLAT_WORKLOAD if FLAT else WORKLOAD, "inner_fb_steps_per_bench_step": 1,
                   "cells_per_fb_step": cells,
                   "parallelism": f"{reps} single-rank host processes"},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": reps, "kind": "reference",
                         "sample": f"{reps} independent single-rank reference processes, {args.steps} timed FB steps "
                                   f"each after {args.warmup} warm-up steps ({wall:.0f} s wall)"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--inner", type=int, default=200)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--tile", default="", help="rows,planes,threads,vector-width,ring-stages of the marching kernel (default: autotune)")
    ap.add_argument("--workload", default="domain", choices=["domain", "ensemble", "surrogate", "window"])
    ap.add_argument("--window-steps", type=int, default=0,
                    help="--workload window: run the configuration end to end for this many steps per precision "
                         "instead of timing bench steps")
    ap.add_argument("--window-out", default="", help="npz for the end-to-end window run's traces and band levels")
    ap.add_argument("--profile-steps", type=int, default=0,
                    help="run this many FB steps of the headline workload (or, with --workload ensemble, of the "
                         "ensemble) between cudaProfilerStart/Stop and exit")
    ap.add_argument("--profile-prec", default="f32", choices=["f32", "f64"])
    ap.add_argument("--block-trace", action="store_true",
                    help="with --profile-steps (<= 64): per tile kind, when its blocks run inside a step")
    ap.add_argument("--tile-shapes", default="",
                    help="--profile-steps: 'rows,vectors,planes,stages' per tile kind (full;lean;pml) instead of autotuning")
    ap.add_argument("--no-surrogate", action="store_true", help="skip the surrogate section of the domain line")
    ap.add_argument("--flat", action="store_true", help="the domain workload on flat ground (no hill)")
    ap.add_argument("--sur-queries", type=int, default=1_000_000, help="surrogate inference queries")
    ap.add_argument("--sur-train-steps", type=int, default=12000, help="training steps per surrogate member")
    ap.add_argument("--members", type=int, default=256, help="ensemble members (--workload ensemble)")
    ap.add_argument("--check-members", type=int, default=-1, help="members checked against FP64 (-1: all)")
    ap.add_argument("--check-steps", type=int, default=200)
    ap.add_argument("--ens-mode", type=int, default=1, choices=[0, 1], help="ensemble launch mode")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        line = run_reference_arm(args, world, rank)
        if line is not None:
            print(json.dumps(line), flush=True)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        if args.profile_steps > 0 and args.workload == "ensemble":
            line = run_ensemble_profile(args, local_rank) if rank == 0 else None
        elif args.profile_steps > 0:
            line = run_profile(args, local_rank) if rank == 0 else None
        elif args.workload == "ensemble":
            line = run_ensemble(args, rank, world, local_rank)
        elif args.workload == "window" and args.window_steps > 0:
            line = run_window_full(args, local_rank) if rank == 0 else None
        elif args.workload == "window":
            line = run_window(args, rank, world, local_rank)
        elif args.workload == "surrogate":
            line = {"workload": "surrogate", **run_surrogate(args.sur_queries, steps=args.sur_train_steps,
                                                              device=local_rank)} if rank == 0 else None
        else:
            line = run_gpu(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
