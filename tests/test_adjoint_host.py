"""CPU tests of the torch restatements the adjoint's losses build on.

`free_energy` and `dens_avg` (polyswift_plusplus_b200/adjoint.py) restate the
reference's free energy (pseffhamil/PsPolymerUpdater.cpp:173-226,
pseffhamil/PsFloryInteraction.cpp:275-321) and density averages; here they are
put against one oracle iteration of a blend with a solvent: F of an iteration
is evaluated on the densities and ln Q of the fields going in and the fields
coming out of the update (the reference's order).
"""
import dataclasses

import numpy as np
import pytest
import torch

import oracle as O
from polyswift_plusplus_b200 import workloads as W
from polyswift_plusplus_b200.adjoint import dens_avg, free_energy
from polyswift_plusplus_b200.config import Solvent, Updater


def blend_with_solvent():
    """AB diblock (vf 0.75) + A homopolymer (vf 0.15, half length) + solvent on B (vf 0.1), FP64,
    steepest descent, an 8^3 grid."""
    cfg = W.blend(8, 18.0, 0.375, 0.15, precision="fp64", ns=16, anderson=False)
    cfg.polymers[0].volfrac = 0.75
    cfg = dataclasses.replace(cfg, cell=(0.21, 0.19, 0.2), solvents=[Solvent("solv", "B", 0.1)],
                              updater=Updater(kind="steepestDescent", relaxlambdas=(0.1, 0.05)))
    _, _, z = W.coords(cfg)
    c = np.cos(2 * np.pi * z / cfg.box[2]).reshape(-1)
    w = W.random_fields(cfg, 0.3)
    return cfg, [w[0] + c, w[1] - c]


def test_dens_avg_of_a_blend_with_solvent():
    cfg, _ = blend_with_solvent()
    a = dens_avg(cfg)
    # A: diblock 0.75 * 0.375 + homopolymer 0.15; B: diblock 0.75 * 0.625 + solvent 0.1
    assert a[0] == pytest.approx(0.75 * 0.375 + 0.15, rel=1e-15)
    assert a[1] == pytest.approx(0.75 * 0.625 + 0.1, rel=1e-15)


def test_free_energy_matches_oracle_iteration(oracle_lib):
    cfg, w = blend_with_solvent()
    o = O.Oracle(cfg)
    o.restore(w)
    hist = o.update(1)[0]
    phi = torch.tensor(np.stack([o.phi(i) for i in range(2)]))
    w_new = torch.tensor(np.stack([o.w(i) for i in range(2)]))
    L0 = float(cfg.polymers[0].length)
    # the solvent's ln Q from the fields going in (pssolvent/PsSimpleSolvent.cpp:86-140)
    lnq_s = float(np.log(np.mean(np.exp(-w[1] / L0))))
    lnq = torch.tensor(list(hist["log_q"][:2]) + [lnq_s], dtype=torch.float64)
    vf = [p.volfrac for p in cfg.polymers] + [0.1]
    al = [p.length / L0 for p in cfg.polymers] + [1.0 / L0]
    chin = cfg.interactions[0].chi * L0
    F = float(free_energy(w_new, phi, lnq, chin, dens_avg(cfg), vf, al))
    assert F == pytest.approx(hist["free_energy"], rel=1e-12, abs=1e-14)
    # one species, scalar form: the diblock alone is the same expression with one term
    F1 = float(free_energy(w_new, phi, lnq[0], chin, dens_avg(cfg), vf[0], al[0]))
    Fv = float(free_energy(w_new, phi, lnq[:1], chin, dens_avg(cfg), vf[:1], al[:1]))
    assert F1 == pytest.approx(Fv, rel=1e-15)


def test_steepest_descent_step_matches_oracle_iteration(oracle_lib):
    """The torch steepest-descent update (two fields, pressure rebuilt and shifted to zero mean)
    against the oracle's update of one iteration (pseffhamil/PsSteepDUpdater.cpp:159-203,
    psphysf/PsConstraint.cpp:184-262), from the densities of the fields going in."""
    from polyswift_plusplus_b200.adjoint import steepest_descent_step
    cfg = W.diblock_config(8, 2.0, 0.375, 18.0, 16, Updater(kind="steepestDescent", relaxlambdas=(0.1, 0.05)),
                           "fp64")
    _, _, z = W.coords(cfg)
    c = np.cos(2 * np.pi * z / cfg.box[2]).reshape(-1)
    w = W.random_fields(cfg, 0.3)
    w = [w[0] + c, w[1] - c]
    p0 = 0.05 * np.sin(2 * np.pi * z / cfg.box[2]).reshape(-1)
    o = O.Oracle(cfg)
    o.restore(w, p0)
    o.update(1)
    phi = torch.tensor(np.stack([o.phi(i) for i in range(2)]))
    chin = cfg.interactions[0].chi * cfg.polymers[0].length
    w1, p1 = steepest_descent_step(torch.tensor(np.stack(w)), torch.tensor(p0), phi, chin, dens_avg(cfg),
                                   cfg.updater.relaxlambdas)
    for i in range(2):
        assert np.abs(w1[i].numpy() - o.w(i)).max() <= 1e-12 * np.abs(o.w(i)).max()
    assert np.abs(p1.numpy() - o.pressure()).max() <= 1e-12 * np.abs(o.pressure()).max()
