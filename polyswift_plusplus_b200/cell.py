"""Variable-cell SCFT: the box lengths follow the stress dF/dL_box.

The stress comes from the FP64 adjoint of the propagator sweeps
(``adjoint.DifferentiableChain``): the reference free energy (pseffhamil/
PsPolymerUpdater.cpp:173-226, pseffhamil/PsFloryInteraction.cpp:275-321)
evaluated on the current fields, differentiated with respect to the three
box lengths L_d = n_d * cell_d through the k^2 operator of every contour step.

``VariableCellRun`` iterates an ``ScftSolver`` (any precision) and every
``period`` iterations takes a bounded steepest-descent step on the box,
L_d <- L_d - eta_d * dF/dL_d with |dL_d| <= max_step * L_d; eta_d halves
whenever the stress along d changes sign (the box overshot the minimum).  The
solver is then rebuilt on the new cell from the current w and p; the Anderson
history starts again (it is a history of the old operator).
"""
from __future__ import annotations

import dataclasses

import numpy as np
import torch

from .adjoint import DifferentiableChain, dens_avg, free_energy
from .config import ScftConfig
from .scft import ScftSolver


def interaction_pairs(cfg: ScftConfig) -> list:
    """(i, j, chiN_ij) of every Flory interaction; chiN = chi * length of polymer 0."""
    scale = float(cfg.polymers[0].length)
    return [(cfg.field_index(it.scfields[0]), cfg.field_index(it.scfields[1]), it.chi * scale)
            for it in cfg.interactions]


def with_box(cfg: ScftConfig, box) -> ScftConfig:
    return dataclasses.replace(cfg, cell=tuple(float(box[d]) / cfg.n[d] for d in range(3)))


def stress(cfg: ScftConfig, w, checkpoint: int = 0, device: int = 0):
    """(F, dF/dL_box) of the fields w (n_fields x N) on cfg's box, from the FP64 adjoint."""
    chain = DifferentiableChain(cfg, checkpoint)
    try:
        dev = torch.device("cuda", device)
        wt = torch.as_tensor(np.asarray(w, dtype=np.float64).reshape(len(cfg.fields), -1), device=dev)
        box = torch.tensor(chain.box0, dtype=torch.float64, requires_grad=True)
        ds = torch.tensor(chain.ds0, dtype=torch.float64)
        phi, lnq = chain(wt, box, ds)
        p = cfg.polymers[0]
        F = free_energy(wt, phi, lnq, None, dens_avg(cfg), vf=p.volfrac, alpha=chain.alpha,
                        pairs=interaction_pairs(cfg))
        F.backward()
        return float(F.detach()), box.grad.numpy().copy()
    finally:
        chain.close()


class VariableCellRun:
    def __init__(self, cfg: ScftConfig, w, p=None, period: int = 50, eta: float = 1.0,
                 max_step: float = 0.02, axes=(0, 1, 2), checkpoint: int = 0):
        self.cfg = cfg
        self.period = int(period)
        self.eta = float(eta)
        self.max_step = float(max_step)
        self.axes = tuple(axes)
        self.checkpoint = checkpoint
        self.box = np.array(cfg.box, dtype=np.float64)
        self.eta_d = np.full(3, self.eta)
        self.last_g = np.zeros(3)
        self.solver = ScftSolver(cfg)
        self.solver.restore(w, p)
        self.history: list[dict] = []
        self.iterations = 0

    def _fields(self):
        s = self.solver
        return [s.w(i) for i in range(len(self.cfg.fields))], s.pressure()

    def cell_step(self) -> dict:
        w, p = self._fields()
        F, g = stress(self.cfg, w, self.checkpoint, self.cfg.device)
        step = np.zeros(3)
        for d in self.axes:
            if g[d] * self.last_g[d] < 0.0:
                self.eta_d[d] *= 0.5
            cap = self.max_step * self.box[d]
            step[d] = np.clip(-self.eta_d[d] * g[d], -cap, cap)
        self.last_g = g.copy()
        rec = {"iteration": self.iterations, "box": self.box.copy(), "F": F, "stress": g.copy(),
               "scft_free_energy": self.solver.scalars()["free_energy"]}
        self.history.append(rec)
        if np.any(step != 0.0):
            self.box = self.box + step
            self.cfg = with_box(self.cfg, self.box)
            self.solver.close()
            self.solver = ScftSolver(self.cfg)
            self.solver.restore(w, p)
        return rec

    def run(self, iters: int) -> list[dict]:
        done = 0
        while done < iters:
            n = min(self.period, iters - done)
            self.solver.update(n)
            done += n
            self.iterations += n
            if n == self.period:
                self.cell_step()
        return self.history

    def close(self) -> None:
        self.solver.close()
