"""Small, self-contained SCFT run for kernel profiling.

Runs the diblock workload's kernels on an n^3 grid with a short contour
(Ns = 20 by default: 7 + 13 steps per sweep), so a profiler capture holds
well under a few GB on the device while every kernel sees full-size grids.

    python -m polyswift_plusplus_b200.profile_case --n 128 --ns 20 --precision mixed --iters 3
"""
from __future__ import annotations

import argparse

from . import workloads as W
from .config import Updater
from .scft import ScftSolver


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--ns", type=int, default=20)
    ap.add_argument("--precision", choices=["mixed", "fp64"], default="mixed")
    ap.add_argument("--iters", type=int, default=3)
    ap.add_argument("--anderson", action="store_true")
    ap.add_argument("--variant", type=int, default=-1, help="kernel variant (-1: autotune)")
    a = ap.parse_args()
    upd = (Updater(kind="andersonMixing", relaxlambdas=(0.1, 0.05), anderson_depth=10,
                   anderson_mix=0.5, anderson_start=0) if a.anderson
           else Updater(kind="steepestDescent", relaxlambdas=(0.1, 0.05)))
    cfg = W.diblock_config(a.n, 8.0 * a.n / 128, 0.35, 25.0, a.ns, upd, a.precision)
    s = W.hex_seed(cfg)
    w = W.random_fields(cfg, 0.05)
    g = ScftSolver(cfg)
    if a.variant >= 0:
        g.set_variant(a.variant)
    g.restore([w[0] + s, w[1] - s])
    g.update(a.iters)
    sc = g.scalars()
    print(f"n={a.n} ns={a.ns} {a.precision}: F={sc['free_energy']:.12g} Q={sc['q'][0]:.12g} "
          f"launches/iteration={g.launches_per_iteration}")
    g.close()


if __name__ == "__main__":
    main()
