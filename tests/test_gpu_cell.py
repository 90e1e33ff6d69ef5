"""Variable-cell SCFT: the stress dF/dL_box from the adjoint drives the box.

The stress is checked against central differences of F (the reference free
energy on fixed fields) and a lamellar diblock, started in a box away from
its preferred period, must relax the box length normal to the lamellae until
that stress component has shrunk.
"""
import dataclasses
import math

import numpy as np
import pytest

from polyswift_plusplus_b200 import workloads as W
from polyswift_plusplus_b200.cell import VariableCellRun, stress, with_box
from polyswift_plusplus_b200.config import Updater
from polyswift_plusplus_b200.scft import ScftSolver

pytestmark = pytest.mark.gpu


def lamellar_case(box=4.0, n=32):
    cfg = W.diblock_config(n, box, 0.40, 30.0, 100,
                           Updater(kind="andersonMixing", relaxlambdas=(0.1, 0.05), anderson_depth=10,
                                   anderson_mix=0.5, anderson_start=40), "fp64")
    x, _, _ = W.coords(cfg)
    c = np.cos(2 * math.pi * x / cfg.box[0]).reshape(-1)
    w = W.random_fields(cfg, 0.05)
    return cfg, [w[0] + 2.0 * c, w[1] - 2.0 * c]


def test_stress_matches_finite_differences_of_F(gpu):
    cfg, w = lamellar_case()
    s = ScftSolver(cfg)
    s.restore(w)
    s.update(150)
    wc = [s.w(0), s.w(1)]
    s.close()
    F0, g = stress(cfg, wc)
    box = np.array(cfg.box)
    h = 1e-6 * box[0]
    Fp, _ = stress(with_box(cfg, box + [h, 0, 0]), wc)
    Fm, _ = stress(with_box(cfg, box - [h, 0, 0]), wc)
    fd = (Fp - Fm) / (2 * h)
    print(f"dF/dL_x adjoint {g[0]:.10e} central difference {fd:.10e}; dF/dL_y,z {g[1]:.2e} {g[2]:.2e}")
    assert abs(g[0] - fd) <= 1e-5 * abs(fd)
    assert abs(g[0]) > 100 * max(abs(g[1]), abs(g[2]))  # lamellae along x carry the stress


def test_variable_cell_relaxes_the_lamellar_period(gpu):
    cfg, w = lamellar_case(box=3.4)
    r = VariableCellRun(cfg, w, period=100, eta=5.0, max_step=0.03, axes=(0,))
    hist = r.run(1000)
    r.close()
    for e in hist:
        print(e["iteration"], np.round(e["box"], 4), f"F {e['F']:.8f}", f"dF/dLx {e['stress'][0]:.3e}")
    first, last = hist[1], hist[-1]  # hist[0]: fields still forming
    assert abs(last["stress"][0]) < 0.5 * abs(first["stress"][0])
    assert np.sign(last["box"][0] - hist[0]["box"][0]) == -np.sign(hist[0]["stress"][0])
