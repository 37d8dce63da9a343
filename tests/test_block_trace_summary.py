"""bench.py's block-timeline summary on a synthetic record (host logic, no
GPU): per-kind medians relative to each step's first block, mean block
durations, skipped kinds and the median step span."""

import importlib
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
bench = importlib.import_module("bench")


def test_block_trace_summary_synthetic():
    none = np.iinfo(np.uint64).max
    tr = np.zeros((64, 10, 4), dtype=np.uint64)
    tr[:, :, 0] = none
    base = 1_000_000
    for s in range(3):  # three steps, 100 us apart
        t0 = base + 100_000 * s
        # lean kind (1): starts 50 us in, ends 90 us in, 4 blocks of 10 us
        tr[s, 1] = [t0 + 50_000, t0 + 90_000, 40_000, 4]
        # x-layer kind (2 + 1): starts with the step, ends 60 us in, 2 blocks of 20 us
        tr[s, 3] = [t0, t0 + 60_000, 40_000, 2]
    out = bench.block_trace_summary(tr)
    assert out["steps"] == 3
    assert out["step_span_us"] == 90.0
    kinds = out["kinds"]
    assert list(kinds) == ["pml_x", "lean"]  # ordered by start
    assert kinds["pml_x"] == {"start_us": 0.0, "end_us": 60.0, "block_us": 20.0, "blocks": 2}
    assert kinds["lean"] == {"start_us": 50.0, "end_us": 90.0, "block_us": 10.0, "blocks": 4}


def test_block_trace_summary_empty():
    tr = np.zeros((64, 10, 4), dtype=np.uint64)
    tr[:, :, 0] = np.iinfo(np.uint64).max
    out = bench.block_trace_summary(tr)
    assert out == {"steps": 0, "step_span_us": None, "kinds": {}}
