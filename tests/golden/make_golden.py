"""Regenerates the golden fixtures in tests/golden/ from the UNMODIFIED
reference solver (oracle/_ref/ref_harness, built by oracle/Makefile from the
reference sources).  Each fixture stores the reference's full-precision
receiver series and final-field data for one generated case.

Usage: python tests/golden/make_golden.py   (needs oracle/_ref/ref_harness)
"""

import importlib
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")]

import cases  # noqa: E402
import refio  # noqa: E402

casegen = importlib.import_module("3d_mpi_test_b200.casegen")

SMALL = ["pml_rigid", "tdbc_east", "porous_ground", "moving_frame", "hill5", "wind_log", "fb_v_p"]


def field_summary(a: np.ndarray) -> np.ndarray:
    return np.array([np.linalg.norm(a), a.sum(), np.abs(a).max()])


def main():
    if not os.path.exists(refio.REF_HARNESS):
        sys.exit("build oracle/_ref/ref_harness first (make -C oracle ref)")
    builders = {n: cases.CASES[n] for n in SMALL}
    builders["plain_box"] = casegen.plain_box
    with tempfile.TemporaryDirectory() as tmp:
        for name, fn in builders.items():
            c, rec = fn()
            d = os.path.join(tmp, name)
            c.write(d)
            casegen.write_receivers(os.path.join(d, "rec.txt"), rec)
            r = refio.run_reference(d, os.path.join(d, "ref.bin"), os.path.join(d, "rec.txt"))
            out = {"steps": np.int64(c.time_domain), "receivers": r["receivers"], "rec_index": r["rec_index"]}
            for f in "puvw":
                out["sum_" + f] = field_summary(r[f])
                if "pore_" + f in r:
                    out["sum_pore_" + f] = field_summary(r["pore_" + f])
            if name == "plain_box":
                out["p_plane_k6"] = r["p"][:, :, 6]  # the receivers' height plane
            else:
                out["p"] = r["p"]
            np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
            print(name, {k: getattr(v, "shape", v) for k, v in out.items()})


if __name__ == "__main__":
    main()
