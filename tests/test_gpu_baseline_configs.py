"""GPU parity on the benchmark configurations themselves, against the FP64 oracle.

* diblock32: the plain-method case (32^3, box 4.0 Rg, f_A 0.30, chiN 20, Ns 100,
  steepest descent with the pressure field, lambda (0.1, 0.05)) run for its full
  500 iterations in FP64; F, Q, max|phi_A + phi_B - 1|, w and phi at 1e-10.
* diblock128: the precision case at full size (128^3, box 8.0 Rg, f_A 0.35,
  chiN 25, Ns 200, hexagonal seed), three iterations:
  - the FP64 device path at 1e-10;
  - the FP32 production kernels (variant 11: fused real-space step in the
    128^2 plane pass, fused k^2 pencil pass, the sweeps as concurrent launch
    chains) at the mixed-path bounds: F to 1e-5 absolute, phi to 1e-4.

The reference loop these follow is PsDomain::update (pstrol/PsDomain.cpp:332-372)
driven for nsteps by polyswift/polyswift.cxx:544-588; Q and phi are
PsBlock::calcBigQ / setCalcQQTIntegral (pspolymer/PsBlock.cpp:205-380).
"""
import numpy as np
import pytest

import oracle as O
from polyswift_plusplus_b200 import workloads as W
from polyswift_plusplus_b200.scft import ScftSolver

pytestmark = pytest.mark.gpu
TOL64 = 1e-10


def rel(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def check_scalars(sg, so, tol):
    assert abs(sg["free_energy"] - so["free_energy"]) <= tol * max(abs(so["free_energy"]), 1e-2)
    assert sg["q"][0] == pytest.approx(so["q"][0], rel=tol)
    assert abs(sg["max_incomp"] - so["max_incomp"]) <= tol * max(so["max_incomp"], 1e-3)


def test_diblock32_500_iterations_fp64(gpu, oracle_lib):
    cfg, w = W.diblock32()
    o = O.Oracle(cfg)
    o.restore(w)
    hist = o.update(500)
    g = ScftSolver(cfg)
    g.restore(w)
    for block in range(5):
        g.update(100)
        check_scalars(g.scalars(), hist[100 * block + 99], TOL64)
    for i in range(2):
        assert rel(g.w(i), o.w(i)) < TOL64
        assert rel(g.phi(i), o.phi(i)) < TOL64
    assert rel(g.pressure(), o.pressure()) < 10 * TOL64
    # the run has ordered: the lamellar seed grew and the melt is near incompressible
    assert hist[-1]["max_incomp"] < 0.05 < hist[0]["max_incomp"]
    g.close()


@pytest.fixture(scope="module")
def diblock128_oracle(oracle_lib):
    """Three FP64 oracle iterations of the full-size precision case (about half
    a minute of host time on all cores)."""
    cfg, w = W.diblock128(precision="fp64")
    o = O.Oracle(cfg)
    o.restore(w)
    hist = o.update(3)
    res = dict(w=w, hist=hist, w_out=[o.w(i) for i in range(2)],
               phi=[o.phi(i) for i in range(2)], p=o.pressure())
    o.close()
    return res


def test_diblock128_full_size_fp64(gpu, diblock128_oracle):
    ref = diblock128_oracle
    cfg, _ = W.diblock128(precision="fp64")
    g = ScftSolver(cfg)
    g.restore(ref["w"])
    for it in range(3):
        g.update(1)
        check_scalars(g.scalars(), ref["hist"][it], TOL64)
    for i in range(2):
        assert rel(g.w(i), ref["w_out"][i]) < TOL64
        assert rel(g.phi(i), ref["phi"][i]) < TOL64
    assert rel(g.pressure(), ref["p"]) < 10 * TOL64
    g.close()


def test_diblock128_full_size_mixed_variant11(gpu, diblock128_oracle):
    ref = diblock128_oracle
    cfg, _ = W.diblock128(precision="mixed")
    g = ScftSolver(cfg)
    g.set_variant(11)
    g.restore(ref["w"])
    for it in range(3):
        g.update(1)
        s = g.scalars()
        assert abs(s["free_energy"] - ref["hist"][it]["free_energy"]) < 1e-5
        assert s["q"][0] == pytest.approx(ref["hist"][it]["q"][0], rel=1e-5)
    for i in range(2):
        assert np.abs(g.phi(i) - ref["phi"][i]).max() < 1e-4
        assert rel(g.w(i), ref["w_out"][i]) < 1e-5
    g.close()


def test_mean_mode_carry_reduces_fp32_error(gpu):
    """FP32 sweeps carry the k = 0 coefficient of every step in FP64 (PlaneWork's
    mean-mode carry, with the rounding of the added mean fed back into the next
    step).  At full size, after one iteration Q of the FP32 sweeps must be
    within 1.5e-7 of the FP64 device path's and at most 0.3 times the error
    without the carry (measured on a B200: 6.7e-8 with, 7.7e-7 without)."""
    import os
    cfg64, w = W.diblock128(precision="fp64")
    g = ScftSolver(cfg64)
    g.restore(w)
    g.update(1)
    q64 = g.scalars()["q"][0]
    g.close()
    errs = {}
    for carry in ("1", "0"):
        os.environ["PSB_DC_CARRY"] = carry
        try:
            cfg, _ = W.diblock128(precision="mixed")
            m = ScftSolver(cfg)
            m.set_variant(11)
            m.restore(w)
            m.update(1)
            errs[carry] = abs(m.scalars()["q"][0] - q64) / q64
            m.close()
        finally:
            os.environ.pop("PSB_DC_CARRY", None)
    assert errs["1"] < 1.5e-7, errs
    assert errs["1"] < 0.3 * errs["0"], errs
