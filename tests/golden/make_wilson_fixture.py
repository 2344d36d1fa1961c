"""Writes tests/golden/hot_48x48x48x96_wloops.json from the FP64 oracle.

    python tests/golden/make_wilson_fixture.py [--threads N]

The 48^3 x 96 lattice of the Wilson-loop workload at its full size: a Haar hot
start from Philox seed 6 (``gen_hot``, which the GPU's ``mag_gauge_hot_start``
reproduces to rounding) and, on it, the oracle's plaquette and rectangle sums,
the average plaquette, the constrained plaquette for mag = 2, the planar Wilson
loops avg_wilson_loop((R, 0, 0), T) for R, T in {1, 2, 4, 8} and two off-axis
loops.  No field is stored.  About ten minutes on 2 threads; 6.1 GB of host
memory for the links.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

DIMS = (48, 48, 48, 96)
HOT_SEED = 6
RT = (1, 2, 4, 8)
OFF_AXIS = (((1, 1, 0), 2), ((2, 1, 0), 3))


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--threads", type=int, default=0)
    ap.add_argument("--out", default=os.path.join(HERE, "hot_48x48x48x96_wloops.json"))
    a = ap.parse_args()
    import oracle as O

    O.build()
    if a.threads:
        O.set_threads(a.threads)
    t0 = time.perf_counter()
    U = O.gen_hot(DIMS, HOT_SEED)
    plaq, rect = O.plaq_rect(DIMS, U)
    out = {"dims": list(DIMS), "hot_seed": HOT_SEED, "plaq_sum": plaq, "rect_sum": rect,
           "avg_plaquette": O.avg_plaquette(DIMS, U), "constrained_plaquette_mag2": O.constrained_plaquette(DIMS, U, 2),
           "planar": [], "off_axis": []}
    for R in RT:
        for T in RT:
            out["planar"].append({"R": R, "T": T, "w": O.wilson_loop(DIMS, U, (R, 0, 0), T)})
            print(R, T, out["planar"][-1]["w"], f"{time.perf_counter() - t0:.0f} s", flush=True)
    for r, T in OFF_AXIS:
        out["off_axis"].append({"r": list(r), "T": T, "w": O.wilson_loop(DIMS, U, r, T)})
    with open(a.out, "w") as f:
        json.dump(out, f, indent=1)
    print("written", a.out, f"{time.perf_counter() - t0:.0f} s")


if __name__ == "__main__":
    main()
