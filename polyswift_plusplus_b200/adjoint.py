"""Differentiable SCFT pieces: the adjoint of the propagator sweeps in torch.autograd.

``ChainAdjoint`` wraps the native FP64 adjoint (``ps_adj_*``) of one linear
block copolymer melt: ``forward(w)`` gives the monomer densities phi and ln Q
(the same sweeps, contour quadrature and Q as one reference iteration,
PsBlockCopolymer::update, pspolymer/PsBlockCopolymer.cpp:189-239), and
``backward(g_phi, g_lnQ)`` runs the adjoint sweeps (propagator slices
checkpointed every C ~ sqrt(Ns) contour steps) for dL/dw, dL/dL_box and
dL/d(ds) of every block.

``DifferentiableChain`` exposes that as a ``torch.autograd.Function`` of
(w, box lengths, per-block contour steps): block lengths enter through
ds_b = f_b / steps_b with the step counts fixed, so dL/df follows by the chain
rule.  ``free_energy`` and ``steepest_descent_step`` restate the reference's
free energy (pseffhamil/PsPolymerUpdater.cpp:173-226) and field update
(pseffhamil/PsSteepDUpdater.cpp:159-203) in torch for two fields, so a loss
can depend on chiN through F or through updated fields.  Nothing here falls
back to the CPU: every sweep runs in the native library.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import math

import numpy as np
import torch

from . import _abi as A
from .config import ScftConfig


def _chk(lib, rc, handle):
    if rc != A.PS_OK:
        raise A.PsError(rc, (lib.ps_adj_last_error(handle) or b"").decode(errors="replace"))


class ChainAdjoint:
    """Native forward/adjoint pair for one FP64 configuration (fixed box and ds).

    ``polymer=None``: ``cfg`` is a one-polymer melt.  ``polymer=i``: the chain
    is polymer i of ``cfg`` (a blend; quadrature chain ``chain`` of a
    polyDisperseBCP) and ``forward`` gives its contribution to phi and its
    ln Q."""

    def __init__(self, cfg: ScftConfig, checkpoint: int = 0, polymer: int | None = None, chain: int = 0):
        if cfg.precision != "fp64":
            cfg = dataclasses.replace(cfg, precision="fp64")
        self.cfg = cfg
        self._lib = A.load_library()
        self._pc = cfg.to_ps_config()
        h = C.c_void_p()
        if polymer is None:
            rc = self._lib.ps_adj_create(C.byref(self._pc), int(checkpoint), C.byref(h))
        else:
            rc = self._lib.ps_adj_create_polymer(C.byref(self._pc), int(polymer), int(chain), int(checkpoint),
                                                 C.byref(h))
        _chk(self._lib, rc, None)
        self._h = h
        self.polymer = 0 if polymer is None else int(polymer)
        self.N = cfg.n_total
        self.nf = len(cfg.fields)
        self.nb = len(cfg.polymers[self.polymer].blocks)
        steps, ck, nbytes = C.c_int(), C.c_int(), C.c_size_t()
        _chk(self._lib, self._lib.ps_adj_info(h, C.byref(steps), C.byref(ck), C.byref(nbytes)), h)
        self.contour_steps, self.checkpoint, self.slice_bytes = steps.value, ck.value, nbytes.value
        self.forward_count = 0

    def forward(self, w: torch.Tensor):
        """w: (n_fields, N) float64 CUDA tensor -> (phi (n_fields, N), ln Q)."""
        w = w.detach().to(torch.float64).contiguous()
        if not w.is_cuda or w.numel() != self.nf * self.N:
            raise ValueError("w must be a CUDA float64 tensor of n_fields * N values")
        phi = torch.empty_like(w)
        lnq = C.c_double()
        torch.cuda.current_stream(w.device).synchronize()
        _chk(self._lib, self._lib.ps_adj_forward(self._h, C.c_void_p(w.data_ptr()), C.c_void_p(phi.data_ptr()),
                                                 C.byref(lnq)), self._h)
        self.forward_count += 1
        return phi.view(self.nf, self.N), lnq.value

    def backward(self, g_phi: torch.Tensor, g_lnq: float):
        """Gradients for the last forward: (dL/dw (n_fields, N), dL/dL_box (3,), dL/dds (n_blocks,))."""
        g_phi = g_phi.detach().to(torch.float64).contiguous()
        gw = torch.empty_like(g_phi)
        gbox = (C.c_double * 3)()
        gds = (C.c_double * self.nb)()
        torch.cuda.current_stream(g_phi.device).synchronize()
        _chk(self._lib, self._lib.ps_adj_backward(self._h, C.c_void_p(g_phi.data_ptr()), float(g_lnq),
                                                  C.c_void_p(gw.data_ptr()), gbox, gds), self._h)
        return (gw.view(self.nf, self.N), np.array([gbox[i] for i in range(3)]),
                np.array([gds[i] for i in range(self.nb)]))

    def set_potential(self, psi: torch.Tensor) -> None:
        """Charged systems: the potential (n_charges, N) float64 CUDA tensor, held fixed."""
        psi = psi.detach().to(torch.float64).contiguous()
        torch.cuda.current_stream(psi.device).synchronize()
        _chk(self._lib, self._lib.ps_adj_set_potential(self._h, C.c_void_p(psi.data_ptr())), self._h)
        self._psi = psi  # kept alive until the copy on the handle's stream has run
        self.forward_count += 1

    def potential_grad(self, n_charges: int) -> torch.Tensor:
        """dL/dpsi of the last backward, (n_charges, N)."""
        g = torch.empty((n_charges, self.N), dtype=torch.float64, device="cuda")
        _chk(self._lib, self._lib.ps_adj_potential_grad(self._h, C.c_void_p(g.data_ptr())), self._h)
        return g

    def species(self) -> tuple[float, float, list]:
        """(free-energy weight, length ratio, average density of each field of the configuration)."""
        wt, lr = C.c_double(), C.c_double()
        avg = (C.c_double * self.nf)()
        _chk(self._lib, self._lib.ps_adj_species(self._h, C.byref(wt), C.byref(lr), avg), self._h)
        return wt.value, lr.value, [avg[i] for i in range(self.nf)]

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.ps_adj_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class _ChainFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, w, box, ds, chain):
        solver = chain.solver(box, ds)
        phi, lnq = solver.forward(w)
        ctx.solver = solver
        ctx.token = solver.forward_count
        ctx.save_for_backward(w)
        return phi, torch.tensor(lnq, dtype=torch.float64, device=w.device)

    @staticmethod
    def backward(ctx, g_phi, g_lnq):
        (w,) = ctx.saved_tensors
        s = ctx.solver
        if s.forward_count != ctx.token:  # another forward ran on this solver since
            s.forward(w)
        if g_phi is None:
            g_phi = torch.zeros((s.nf, s.N), dtype=torch.float64, device=w.device)
        gl = 0.0 if g_lnq is None else float(g_lnq)
        gw, gbox, gds = s.backward(g_phi, gl)
        return (gw.view_as(w), torch.as_tensor(gbox, dtype=torch.float64),
                torch.as_tensor(gds, dtype=torch.float64), None)


class DifferentiableChain:
    """phi, ln Q = chain(w, box, ds) for one linear block copolymer melt.

    ``box`` holds the three box lengths (Rg) and ``ds`` the contour step of
    each block (CPU float64 tensors); the step counts are those of ``cfg``.
    A native solver is built per distinct (box, ds) and cached.
    """

    def __init__(self, cfg: ScftConfig, checkpoint: int = 0, cache: int = 8):
        self.cfg = dataclasses.replace(cfg, precision="fp64")
        self.checkpoint = checkpoint
        self._cache: dict = {}
        self._order: list = []
        self._max = cache
        base = ChainAdjoint(self.cfg, checkpoint)
        p = self.cfg.polymers[0]
        scale = float(p.length)
        self.alpha = p.length / scale
        self.steps = [max(4, int(math.floor(self.alpha * b.lengthfrac / b.ds + 0.5))) if b.force_block_steps
                      else int(round(self.alpha * b.lengthfrac / b.ds)) for b in p.blocks]
        self.box0 = tuple(self.cfg.n[d] * self.cfg.cell[d] for d in range(3))
        self.ds0 = tuple(b.ds for b in p.blocks)
        self._put((self.box0, self.ds0), base)

    def _put(self, key, solver):
        self._cache[key] = solver
        self._order.append(key)
        while len(self._order) > self._max:
            old = self._order.pop(0)
            self._cache.pop(old).close()

    def config_for(self, box, ds) -> ScftConfig:
        p = self.cfg.polymers[0]
        blocks = [dataclasses.replace(b, ds=float(d), lengthfrac=float(d) * s / self.alpha,
                                      force_block_steps=True)
                  for b, d, s in zip(p.blocks, ds, self.steps)]
        cell = tuple(float(box[d]) / self.cfg.n[d] for d in range(3))
        return dataclasses.replace(self.cfg, cell=cell,
                                   polymers=[dataclasses.replace(p, blocks=blocks)])

    def solver(self, box, ds) -> ChainAdjoint:
        key = (tuple(float(x) for x in box), tuple(float(x) for x in ds))
        if key not in self._cache:
            self._put(key, ChainAdjoint(self.config_for(key[0], key[1]), self.checkpoint))
        return self._cache[key]

    def __call__(self, w, box=None, ds=None):
        box = torch.tensor(self.box0, dtype=torch.float64) if box is None else box
        ds = torch.tensor(self.ds0, dtype=torch.float64) if ds is None else ds
        return _ChainFn.apply(w, box, ds, self)

    def close(self):
        for s in self._cache.values():
            s.close()
        self._cache.clear()
        self._order.clear()


class _PolymerFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, w, box, blend, ip):
        solver = blend.solvers(box)[ip]
        phi, lnq = solver.forward(w)
        ctx.solver = solver
        ctx.token = solver.forward_count
        ctx.save_for_backward(w)
        return phi, torch.tensor(lnq, dtype=torch.float64, device=w.device)

    @staticmethod
    def backward(ctx, g_phi, g_lnq):
        (w,) = ctx.saved_tensors
        s = ctx.solver
        if s.forward_count != ctx.token:
            s.forward(w)
        if g_phi is None:
            g_phi = torch.zeros((s.nf, s.N), dtype=torch.float64, device=w.device)
        gl = 0.0 if g_lnq is None else float(g_lnq)
        gw, gbox, _ = s.backward(g_phi, gl)
        return gw.view_as(w), torch.as_tensor(gbox, dtype=torch.float64), None, None


class DifferentiableBlend:
    """phi, ln Q = blend(w, box) for a blend of block copolymers (linear, mirror-symmetric,
    branched or polydisperse) and simple solvents.

    phi (n_fields, N) is the sum of every species' density and ln Q holds the polymers' chains'
    ln Q in configuration order (n_g entries for a polyDisperseBCP), then the solvents'.  Each
    chain runs the native adjoint (``ps_adj_create_polymer``); a simple solvent is closed form
    (pssolvent/PsSimpleSolvent.cpp:86-140): wf = exp(-w_f / L_0), Q_s = mean(wf),
    phi_f += vf_s wf / Q_s, with L_0 the length of polymer 0, differentiated by torch.  ``box``
    holds the three box lengths (CPU float64); contour steps are fixed.  Native solvers are built
    per distinct box and cached.
    """

    def __init__(self, cfg: ScftConfig, checkpoint: int = 0, cache: int = 4):
        self.cfg = dataclasses.replace(cfg, precision="fp64")
        for sv in self.cfg.solvents:
            if sv.kind != "simpleSolvent":
                raise ValueError("the blend adjoint takes simple solvents only")
        self.checkpoint = checkpoint
        self.scale = float(self.cfg.polymers[0].length)
        self.box0 = tuple(self.cfg.n[d] * self.cfg.cell[d] for d in range(3))
        self._cache: dict = {}
        self._order: list = []
        self._max = cache
        self.solvers(self.box0)

    def chains(self) -> list:
        """(polymer, quadrature chain) of each entry of the polymers' part of ln Q."""
        return [(i, k) for i, p in enumerate(self.cfg.polymers) for k in range(p.n_chains)]

    def solvers(self, box) -> list:
        key = tuple(float(x) for x in box)
        if key not in self._cache:
            cell = tuple(key[d] / self.cfg.n[d] for d in range(3))
            c = dataclasses.replace(self.cfg, cell=cell)
            self._cache[key] = [ChainAdjoint(c, self.checkpoint, polymer=i, chain=k) for i, k in self.chains()]
            self._order.append(key)
            while len(self._order) > self._max:
                for s in self._cache.pop(self._order.pop(0)):
                    s.close()
        return self._cache[key]

    def __call__(self, w, box=None):
        box = torch.tensor(self.box0, dtype=torch.float64) if box is None else box
        phi, lnqs = None, []
        for ip in range(len(self.chains())):
            p, q = _PolymerFn.apply(w, box, self, ip)
            phi = p if phi is None else phi + p
            lnqs.append(q)
        for sv in self.cfg.solvents:
            f = self.cfg.field_index(sv.scfield)
            wf = torch.exp(-w[f] / self.scale)
            q = wf.mean()
            add = torch.zeros_like(phi)
            add[f] = (sv.volfrac / q) * wf
            phi = phi + add
            lnqs.append(torch.log(q))
        return phi, torch.stack(lnqs)

    def species_weights(self) -> tuple[list, list]:
        """(vf, alpha) per entry of ln Q for free_energy: a chain's volfrac times its polydisperse
        density weight and its length ratio L / L_0; vf and 1 / L_0 for a solvent
        (pseffhamil/PsPolymerUpdater.cpp:173-226)."""
        sp = [s.species() for s in self.solvers(self.box0)]
        vf = [x[0] for x in sp] + [sv.volfrac for sv in self.cfg.solvents]
        al = [x[1] for x in sp] + [1.0 / self.scale for _ in self.cfg.solvents]
        return vf, al

    def dens_avg(self) -> list:
        """The configuration's average density of each field (the disorder reference of F)."""
        return self.solvers(self.box0)[0].species()[2]

    def close(self):
        for ss in self._cache.values():
            for s in ss:
                s.close()
        self._cache.clear()
        self._order.clear()


def dens_avg(cfg: ScftConfig, f: torch.Tensor | None = None) -> list:
    """Average density of each field: sum over polymers of vf * (length fraction of its blocks),
    plus each solvent's vf on its field.  ``f`` overrides polymer 0's block fractions."""
    out = [0.0] * len(cfg.fields)
    for ip, p in enumerate(cfg.polymers):
        for i, b in enumerate(p.blocks):
            frac = b.lengthfrac if (f is None or ip > 0) else f[i]
            out[cfg.field_index(b.scfield)] = out[cfg.field_index(b.scfield)] + p.volfrac * frac
    for sv in cfg.solvents:
        out[cfg.field_index(sv.scfield)] = out[cfg.field_index(sv.scfield)] + sv.volfrac
    return out


def free_energy(w, phi, lnq, chin, avg, vf=1.0, alpha=1.0, pairs=None):
    """F = -sum_species vf ln Q / alpha + mean_r[-sum_i phi_i w_i + sum_pairs chiN_ij (phi_i phi_j
    - avg_i avg_j)] (pseffhamil/PsPolymerUpdater.cpp:173-226, pseffhamil/PsFloryInteraction.cpp:275-321,
    disorder term subtracted).  One species: scalar ``lnq``, ``vf``, ``alpha``; a blend: ``lnq`` a
    1-d tensor and ``vf``, ``alpha`` sequences (``DifferentiableBlend.species_weights``).  Two
    fields: ``chin`` is the A-B chiN; otherwise ``pairs`` lists (i, j, chiN_ij) and ``chin`` is
    ignored."""
    if pairs is None:
        pairs = [(0, 1, chin)]
    inter = 0.0
    for i, j, c in pairs:
        inter = inter + c * (phi[i] * phi[j] - avg[i] * avg[j])
    field = (-(phi * w).sum(0) + inter).mean()
    if torch.is_tensor(lnq) and lnq.dim() > 0:
        species = 0.0
        for k in range(lnq.shape[0]):
            species = species - vf[k] * lnq[k] / alpha[k]
        return species + field
    return -vf * lnq / alpha + field


def steepest_descent_step(w, p, phi, chin, avg, lambdas=(0.1, 0.05)):
    """One reference steepest-descent update of two fields and the pressure
    (pseffhamil/PsSteepDUpdater.cpp:159-203, :264-278; psphysf/PsConstraint.cpp:184-262):
    dH_i = p - w_i + chiN (phi_j - avg_j), w_i += l0 (dH_i - l1 dH_j), p = mean-free (w_A + w_B)/2."""
    l0, l1 = lambdas
    dh_a = p - w[0] + chin * (phi[1] - avg[1])
    dh_b = p - w[1] + chin * (phi[0] - avg[0])
    wa = w[0] + l0 * (dh_a - l1 * dh_b)
    wb = w[1] + l0 * (dh_b - l1 * dh_a)
    pn = 0.5 * (wa + wb)
    return torch.stack([wa, wb]), pn - pn.mean()
