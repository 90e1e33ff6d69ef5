"""Adjoint of the propagator sweeps against FP64 central finite differences.

The adjoint (ps_adj_*) must reproduce the densities of one engine iteration,
give gradients that agree with central differences (step 1e-6 relative) to
1e-5, and give the same result for every checkpoint interval (full storage,
square-root checkpointing, an uneven interval).  The last test runs the
differentiation workload: a 64^3, Ns = 128 diblock at a lamellar state, loss
sum (phi_A - phi_target)^2 after one self-consistent field update, external
field h on w_A, gradients in w, h, chiN, f_A and the box, and the stress
dF/dL_box.
"""
import dataclasses
import math

import numpy as np
import pytest
import torch

from polyswift_plusplus_b200 import workloads as W
from polyswift_plusplus_b200.adjoint import (ChainAdjoint, DifferentiableChain, dens_avg, free_energy,
                                             steepest_descent_step)
from polyswift_plusplus_b200.config import Updater
from polyswift_plusplus_b200.scft import ScftSolver

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
TOL = 1e-5


def small_case(n=16, ns=32, cell=(0.2, 0.19, 0.21)):
    cfg = W.diblock_config(n, 3.0, 0.40, 18.0, ns, Updater(kind="steepestDescent", relaxlambdas=(0.1, 0.05)),
                           "fp64", force=True)
    cfg = dataclasses.replace(cfg, cell=cell)
    _, _, z = W.coords(cfg)
    c = np.cos(2 * math.pi * z / cfg.box[2]).reshape(-1)
    w = W.random_fields(cfg, 0.5)
    return cfg, np.stack([w[0] + c, w[1] - c])


def loss_terms(cfg, seed=5):
    rng = np.random.default_rng(seed)
    t = torch.tensor(rng.uniform(0.2, 0.8, cfg.n_total), device=DEV)
    r = torch.tensor(rng.standard_normal(cfg.n_total), device=DEV)

    def L(phi, lnq):
        return ((phi[0] - t) ** 2).sum() + 0.5 * (phi[1] * r).sum() + 0.3 * lnq
    return L


def eval_loss(adj, w, L):
    phi, lnq = adj.forward(w)
    return float(L(phi, torch.tensor(lnq, dtype=torch.float64, device=DEV)))


def grads(adj, w, L):
    phi, lnq = adj.forward(w)
    phi = phi.clone().requires_grad_(True)
    lq = torch.tensor(lnq, dtype=torch.float64, device=DEV, requires_grad=True)
    L(phi, lq).backward()
    return adj.backward(phi.grad, float(lq.grad))


def test_adjoint_forward_matches_engine(gpu):
    cfg, w = small_case()
    s = ScftSolver(cfg)
    s.restore(list(w))
    s.update(1)  # phi of the first iteration is phi(w0)
    adj = ChainAdjoint(cfg, checkpoint=1)
    phi, lnq = adj.forward(torch.tensor(w, device=DEV))
    for i in range(2):
        ref = s.phi(i)
        assert np.abs(phi[i].cpu().numpy() - ref).max() <= 1e-12 * np.abs(ref).max()
    assert lnq == pytest.approx(s.scalars()["log_q"][0], rel=1e-13, abs=1e-13)
    assert adj.contour_steps == 32


def test_adjoint_field_gradient_matches_finite_differences(gpu):
    cfg, w = small_case()
    L = loss_terms(cfg)
    adj = ChainAdjoint(cfg)  # square-root checkpointing
    wt = torch.tensor(w, device=DEV)
    gw, _, _ = grads(adj, wt, L)
    rng = np.random.default_rng(11)
    for k in range(3):
        d = torch.tensor(rng.standard_normal(w.shape), device=DEV)
        if k == 2:  # a localised direction
            d = torch.zeros_like(wt)
            d[0, 1234] = 1.0
            d[1, 77] = -0.5
        eps = 1e-6
        fd = (eval_loss(adj, wt + eps * d, L) - eval_loss(adj, wt - eps * d, L)) / (2 * eps)
        an = float((gw * d).sum())
        print(f"dL/dw direction {k}: adjoint {an:.12e} central difference {fd:.12e}")
        assert abs(an - fd) <= TOL * abs(fd), (k, an, fd)


def test_adjoint_box_and_ds_gradients_match_finite_differences(gpu):
    cfg, w = small_case()
    L = loss_terms(cfg, seed=7)
    chain = DifferentiableChain(cfg)
    wt = torch.tensor(w, device=DEV)
    box = torch.tensor(chain.box0, dtype=torch.float64, requires_grad=True)
    ds = torch.tensor(chain.ds0, dtype=torch.float64, requires_grad=True)
    phi, lnq = chain(wt, box, ds)
    L(phi, lnq).backward()

    def at(b, d):
        with torch.no_grad():
            p, q = chain(wt, torch.tensor(b, dtype=torch.float64), torch.tensor(d, dtype=torch.float64))
            return float(L(p, q))
    for dim in range(3):
        h = 1e-6 * chain.box0[dim]
        bp, bm = list(chain.box0), list(chain.box0)
        bp[dim] += h
        bm[dim] -= h
        fd = (at(bp, chain.ds0) - at(bm, chain.ds0)) / (2 * h)
        print(f"dL/dL_{dim}: adjoint {box.grad[dim].item():.12e} central difference {fd:.12e}")
        assert abs(box.grad[dim].item() - fd) <= TOL * abs(fd), (dim, box.grad[dim].item(), fd)
    for b in range(2):
        h = 1e-6 * chain.ds0[b]
        dp, dm = list(chain.ds0), list(chain.ds0)
        dp[b] += h
        dm[b] -= h
        fd = (at(chain.box0, dp) - at(chain.box0, dm)) / (2 * h)
        print(f"dL/dds_{b}: adjoint {ds.grad[b].item():.12e} central difference {fd:.12e}")
        assert abs(ds.grad[b].item() - fd) <= TOL * abs(fd), (b, ds.grad[b].item(), fd)
    chain.close()


def test_adjoint_checkpoint_interval_does_not_change_results(gpu):
    cfg, w = small_case(n=16, ns=40)
    L = loss_terms(cfg)
    wt = torch.tensor(w, device=DEV)
    out = []
    for ck in (1, 0, 7):  # full storage, ceil(sqrt(40)) = 7, uneven 7 -> 6 segments
        adj = ChainAdjoint(cfg, checkpoint=ck)
        phi, lnq = adj.forward(wt)
        gw, gbox, gds = grads(adj, wt, L)
        out.append((phi.cpu().numpy(), lnq, gw.cpu().numpy(), gbox, gds, adj.slice_bytes))
        adj.close()
    for o in out[1:]:
        assert np.array_equal(o[0], out[0][0]) and o[1] == out[0][1]
        assert np.array_equal(o[2], out[0][2])
        assert np.array_equal(o[3], out[0][3]) and np.array_equal(o[4], out[0][4])
    assert out[1][5] < out[0][5] / 2  # checkpointing stores far fewer slices


def test_differentiation_workload_64cubed(gpu):
    """cfg: 64^3, box 6.0, f_A 0.40 (51 + 77 steps), chiN 18, Ns 128, FP64, lamellar
    state.  L = sum (phi_A[w'] - 0.5 - 0.4 cos(2 pi z / L))^2, w' = one steepest-descent
    update of (w_A + h, w_B) with phi[w + h]; gradients vs central differences."""
    cfg, w0 = W.diblock64_adjoint()
    s = ScftSolver(cfg)
    s.restore(w0)
    s.update(60)  # relax towards the lamellar saddle point
    w = torch.tensor(np.stack([s.w(0), s.w(1)]), device=DEV)
    p = torch.tensor(s.pressure(), device=DEV)
    s.close()
    rng = np.random.default_rng(2024)
    h = torch.tensor(rng.normal(0.0, 0.05, cfg.n_total), device=DEV)
    _, _, z = W.coords(cfg)
    target = torch.tensor(0.5 + 0.4 * np.cos(2 * math.pi * z / cfg.box[2]).reshape(-1), device=DEV)
    chain = DifferentiableChain(cfg)
    assert chain.steps == [51, 77]
    assert chain.solver(chain.box0, chain.ds0).checkpoint == 12

    def objective(w, h, chin, f, box):
        ds = torch.stack([f / 51.0, (1.0 - f) / 77.0])
        avg = [f, 1.0 - f]
        wh = torch.stack([w[0] + h, w[1]])
        phi, lnq = chain(wh, box, ds)
        w1, _ = steepest_descent_step(wh, p, phi, chin, avg)
        phi1, _ = chain(w1, box, ds)
        loss = ((phi1[0] - target) ** 2).sum()
        F = free_energy(wh, phi, lnq, chin, avg)
        return loss, F

    wv = w.clone().requires_grad_(True)
    hv = h.clone().requires_grad_(True)
    chin = torch.tensor(18.0, dtype=torch.float64, requires_grad=True)
    f = torch.tensor(0.40, dtype=torch.float64, requires_grad=True)
    box = torch.tensor(chain.box0, dtype=torch.float64, requires_grad=True)
    loss, F = objective(wv, hv, chin, f, box)
    g_w, g_h, g_chin, g_f, _ = torch.autograd.grad(loss, [wv, hv, chin, f, box], retain_graph=True)
    dF_dbox = torch.autograd.grad(F, box)[0]

    def val(which, **kw):
        args = dict(w=w, h=h, chin=torch.tensor(18.0, dtype=torch.float64),
                    f=torch.tensor(0.40, dtype=torch.float64), box=torch.tensor(chain.box0, dtype=torch.float64))
        args.update(kw)
        with torch.no_grad():
            lo, Fv = objective(**args)
        return float(lo if which == "L" else Fv)

    def check(an, plus, minus, eps, what):
        fd = (plus - minus) / (2 * eps)
        print(f"{what}: adjoint {an:.12e} central difference {fd:.12e} rel {abs(an - fd) / abs(fd):.2e}")
        assert abs(an - fd) <= TOL * abs(fd), (what, an, fd)

    d = torch.tensor(rng.standard_normal(w.shape), device=DEV)
    check(float((g_w * d).sum()), val("L", w=w + 1e-6 * d), val("L", w=w - 1e-6 * d), 1e-6, "dL/dw.d")
    dh = torch.tensor(rng.standard_normal(cfg.n_total), device=DEV)
    check(float((g_h * dh).sum()), val("L", h=h + 1e-6 * dh), val("L", h=h - 1e-6 * dh), 1e-6, "dL/dh.d")
    e = 18.0 * 1e-6
    check(g_chin.item(), val("L", chin=torch.tensor(18.0 + e, dtype=torch.float64)),
          val("L", chin=torch.tensor(18.0 - e, dtype=torch.float64)), e, "dL/dchiN")
    e = 0.4 * 1e-6
    check(g_f.item(), val("L", f=torch.tensor(0.4 + e, dtype=torch.float64)),
          val("L", f=torch.tensor(0.4 - e, dtype=torch.float64)), e, "dL/df_A")
    # The stress is checked as a vector: each component to 1e-5 of the largest
    # one.  Along x and y (in the lamellar planes) it is about 1e-6 of F, below
    # what a central difference of F can resolve at this step.
    an, fd = [], []
    for dim in range(3):
        e = chain.box0[dim] * 1e-6
        bp = torch.tensor(chain.box0, dtype=torch.float64)
        bm = bp.clone()
        bp[dim] += e
        bm[dim] -= e
        an.append(dF_dbox[dim].item())
        fd.append((val("F", box=bp) - val("F", box=bm)) / (2 * e))
        print(f"dF/dL_{'xyz'[dim]}: adjoint {an[-1]:.12e} central difference {fd[-1]:.12e}")
    scale = max(abs(x) for x in fd)
    assert abs(fd[2]) == scale
    for a_, f_ in zip(an, fd):
        assert abs(a_ - f_) <= TOL * scale, (an, fd)
    chain.close()


def test_adjoint_on_split_plane_grid(gpu):
    """8 x 16 x 32: y-z planes without a fused kernel, so the adjoint runs the
    row + y-pencil passes (the 256^3 path); checkpointing invariance and a
    directional derivative against central differences."""
    cfg, w = small_case(n=16, ns=30)
    cfg = dataclasses.replace(cfg, n=(8, 16, 32), cell=(0.4, 0.2, 0.1))
    w = np.stack(W.random_fields(cfg, 0.5))
    L = loss_terms(cfg, seed=9)
    wt = torch.tensor(w, device=DEV)
    full = ChainAdjoint(cfg, checkpoint=1)
    gw1, gb1, gd1 = grads(full, wt, L)
    ck = ChainAdjoint(cfg)
    gw2, gb2, gd2 = grads(ck, wt, L)
    assert np.array_equal(gw1.cpu().numpy(), gw2.cpu().numpy()) and np.array_equal(gb1, gb2)
    # along the gradient (a well-conditioned central difference) and a localised direction
    loc = torch.zeros_like(wt)
    loc[0, 321] = 1.0
    loc[1, 2222] = -0.7
    for d in (gw2 / gw2.norm(), loc):
        fd = (eval_loss(ck, wt + 1e-6 * d, L) - eval_loss(ck, wt - 1e-6 * d, L)) / 2e-6
        an = float((gw2 * d).sum())
        print(f"split-plane dL/dw: adjoint {an:.12e} central difference {fd:.12e}")
        assert abs(an - fd) <= TOL * abs(fd), (an, fd)


def blend_case(n=16, ns=32):
    """AB diblock (vf 0.75, f_A = 12/32) + A homopolymer (vf 0.15, half length: a
    mirror-symmetric chain) + simple solvent on B (vf 0.1), FP64."""
    from polyswift_plusplus_b200.config import Solvent
    cfg = W.blend(n, 18.0, 0.375, 0.15, precision="fp64", ns=ns, anderson=False)
    cfg.polymers[0].volfrac = 0.75
    cfg = dataclasses.replace(cfg, cell=(0.13, 0.12, 0.125), solvents=[Solvent("solv", "B", 0.1)])
    _, _, z = W.coords(cfg)
    c = np.cos(2 * math.pi * z / cfg.box[2]).reshape(-1)
    w = W.random_fields(cfg, 0.5)
    return cfg, np.stack([w[0] + c, w[1] - c])


def blend_loss(cfg, seed=5):
    rng = np.random.default_rng(seed)
    t = torch.tensor(rng.uniform(0.2, 0.8, cfg.n_total), device=DEV)
    r = torch.tensor(rng.standard_normal(cfg.n_total), device=DEV)
    c = torch.tensor([0.3, -0.2, 0.1], dtype=torch.float64, device=DEV)

    def L(phi, lnq):
        return ((phi[0] - t) ** 2).sum() + 0.5 * (phi[1] * r).sum() + (c * lnq).sum()
    return L


def test_blend_adjoint_forward_matches_engine(gpu):
    """DifferentiableBlend's phi (sum of the diblock's and the homopolymer's native adjoint
    forwards and the solvent's closed form) and the polymers' ln Q against one engine
    iteration."""
    from polyswift_plusplus_b200.adjoint import DifferentiableBlend
    cfg, w = blend_case()
    s = ScftSolver(cfg)
    s.restore(list(w))
    s.update(1)
    blend = DifferentiableBlend(cfg, checkpoint=1)
    with torch.no_grad():
        phi, lnq = blend(torch.tensor(w, device=DEV))
    for i in range(2):
        ref = s.phi(i)
        assert np.abs(phi[i].cpu().numpy() - ref).max() <= 1e-12 * np.abs(ref).max()
    for ip in range(2):
        assert float(lnq[ip]) == pytest.approx(s.scalars()["log_q"][ip], rel=1e-13, abs=1e-13)
    blend.close()


def test_blend_adjoint_gradients_match_finite_differences(gpu):
    """dL/dw and dL/dL_box of a loss over the blend's phi and every species' ln Q, and the
    stress dF/dL_box of its free energy, against central differences."""
    from polyswift_plusplus_b200.adjoint import DifferentiableBlend
    cfg, w = blend_case()
    L = blend_loss(cfg)
    blend = DifferentiableBlend(cfg)  # square-root checkpointing
    wt = torch.tensor(w, device=DEV, requires_grad=True)
    box = torch.tensor(blend.box0, dtype=torch.float64, requires_grad=True)
    phi, lnq = blend(wt, box)
    L(phi, lnq).backward()
    gw, gbox = wt.grad.detach(), box.grad.detach().clone()

    def at(wv, b):
        with torch.no_grad():
            p, q = blend(wv, torch.tensor(b, dtype=torch.float64))
            return float(L(p, q))
    w0 = wt.detach()
    rng = np.random.default_rng(11)
    for k in range(3):
        d = torch.tensor(rng.standard_normal(w.shape), device=DEV)
        if k == 2:
            d = torch.zeros_like(w0)
            d[0, 1234] = 1.0
            d[1, 77] = -0.5
        eps = 1e-6
        fd = (at(w0 + eps * d, blend.box0) - at(w0 - eps * d, blend.box0)) / (2 * eps)
        an = float((gw * d).sum())
        print(f"blend dL/dw direction {k}: adjoint {an:.12e} central difference {fd:.12e}")
        assert abs(an - fd) <= TOL * abs(fd), (k, an, fd)
    for dim in range(3):
        h = 1e-6 * blend.box0[dim]
        bp, bm = list(blend.box0), list(blend.box0)
        bp[dim] += h
        bm[dim] -= h
        fd = (at(w0, bp) - at(w0, bm)) / (2 * h)
        print(f"blend dL/dL_{dim}: adjoint {gbox[dim].item():.12e} central difference {fd:.12e}")
        assert abs(gbox[dim].item() - fd) <= TOL * abs(fd), (dim, gbox[dim].item(), fd)
    # stress of the free energy (fields fixed): F over every species
    from polyswift_plusplus_b200.adjoint import dens_avg, free_energy
    avg = blend.dens_avg()
    assert avg == pytest.approx(dens_avg(cfg), rel=1e-15, abs=1e-15)
    vf, al = blend.species_weights()
    chin = cfg.interactions[0].chi * cfg.polymers[0].length
    box = torch.tensor(blend.box0, dtype=torch.float64, requires_grad=True)
    phi, lnq = blend(w0, box)
    free_energy(w0, phi, lnq, chin, avg, vf, al).backward()

    def F_at(b):
        with torch.no_grad():
            p, q = blend(w0, torch.tensor(b, dtype=torch.float64))
            return float(free_energy(w0, p, q, chin, avg, vf, al))
    fds = []
    for dim in range(3):
        h = 1e-6 * blend.box0[dim]
        bp, bm = list(blend.box0), list(blend.box0)
        bp[dim] += h
        bm[dim] -= h
        fds.append((F_at(bp) - F_at(bm)) / (2 * h))
        print(f"blend dF/dL_{dim}: adjoint {box.grad[dim].item():.12e} central difference {fds[-1]:.12e}")
    # the stress across the pattern (z) is the large component; the others sit at the
    # resolution of a central difference of F and are checked against it
    big = max(abs(x) for x in fds)
    for dim in range(3):
        assert abs(box.grad[dim].item() - fds[dim]) <= TOL * big, (dim, box.grad[dim].item(), fds[dim])
    blend.close()


def test_adjoint_mirror_symmetric_chain(gpu):
    """A symmetric ABA triblock melt (identical sweeps from both ends, aliased in the engine)
    through ps_adj_create: forward against the engine, dL/dw against central differences."""
    from polyswift_plusplus_b200.config import Block, Polymer
    cfg, w = small_case()
    ds = cfg.polymers[0].blocks[0].ds
    cfg.polymers[0] = Polymer(name="aba", volfrac=1.0, length=cfg.polymers[0].length, blocks=[
        Block("aba_A1", "A", ds, 0.25, ["freeEnd"], ["aba_B"], force_block_steps=True),
        Block("aba_B", "B", ds, 0.5, ["aba_A1"], ["aba_A2"], force_block_steps=True),
        Block("aba_A2", "A", ds, 0.25, ["aba_B"], ["freeEnd"], force_block_steps=True)])
    s = ScftSolver(cfg)
    s.restore(list(w))
    s.update(1)
    adj = ChainAdjoint(cfg)
    wt = torch.tensor(w, device=DEV)
    phi, lnq = adj.forward(wt)
    for i in range(2):
        ref = s.phi(i)
        assert np.abs(phi[i].cpu().numpy() - ref).max() <= 1e-12 * np.abs(ref).max()
    assert lnq == pytest.approx(s.scalars()["log_q"][0], rel=1e-13, abs=1e-13)
    L = loss_terms(cfg, seed=9)
    gw, _, _ = grads(adj, wt, L)
    rng = np.random.default_rng(3)
    for k in range(2):
        d = torch.tensor(rng.standard_normal(w.shape), device=DEV)
        eps = 1e-6
        fd = (eval_loss(adj, wt + eps * d, L) - eval_loss(adj, wt - eps * d, L)) / (2 * eps)
        an = float((gw * d).sum())
        print(f"ABA dL/dw direction {k}: adjoint {an:.12e} central difference {fd:.12e}")
        assert abs(an - fd) <= TOL * abs(fd), (k, an, fd)
    adj.close()


def branched_case(kind):
    """A three-arm ABC star, or the two-junction H-shaped tree (arms A, B and backbone C at one
    junction, C, D, E at the other), FP64 at 16^3."""
    from polyswift_plusplus_b200.config import Block, Interaction, Polymer, ScftConfig
    if kind == "star3":
        return W.star_abc(n=16)
    ds = 0.01
    blocks = [Block("a", "A", ds, 0.15, ["freeEnd"], ["b", "c"]),
              Block("b", "B", ds, 0.15, ["freeEnd"], ["a", "c"]),
              Block("c", "C", ds, 0.40, ["a", "b"], ["d", "e"]),
              Block("d", "A", ds, 0.15, ["freeEnd"], ["c", "e"]),
              Block("e", "B", ds, 0.15, ["freeEnd"], ["c", "d"])]
    cfg = ScftConfig(n=(16, 16, 16), cell=(0.2, 0.19, 0.21), fields=["A", "B", "C"],
                     polymers=[Polymer("h", 1.0, 100, blocks)],
                     interactions=[Interaction("AB", 0.12, ["A", "B"]), Interaction("BC", 0.12, ["B", "C"]),
                                   Interaction("AC", 0.15, ["A", "C"])],
                     updater=Updater(relaxlambdas=(0.05, 0.025)), seed=77, precision="fp64")
    return cfg, W.random_fields(cfg, 0.4)


@pytest.mark.parametrize("kind", ["star3", "tree_h"])
def test_adjoint_branched_chain(gpu, kind):
    """Branched chains (every slice stored; junction products differentiated back to the
    arriving sweeps): forward against the engine, dL/dw, dL/dL_box and dL/d(ds) against
    central differences."""
    cfg, w = branched_case(kind)
    w = np.stack(w)
    s = ScftSolver(cfg)
    s.restore(list(w))
    s.update(1)
    adj = ChainAdjoint(cfg)
    assert adj.checkpoint == 1
    wt = torch.tensor(w, device=DEV)
    phi, lnq = adj.forward(wt)
    for i in range(len(cfg.fields)):
        ref = s.phi(i)
        assert np.abs(phi[i].cpu().numpy() - ref).max() <= 1e-12 * np.abs(ref).max()
    assert lnq == pytest.approx(s.scalars()["log_q"][0], rel=1e-13, abs=1e-13)
    L = loss_terms(cfg, seed=13)
    gw, _, _ = grads(adj, wt, L)
    rng = np.random.default_rng(17)
    n = cfg.n
    for k in range(3):
        d = torch.tensor(rng.standard_normal(w.shape), device=DEV)
        if k == 2:
            # localised: a 4^3 patch of field A and one of field C (a single point's derivative is
            # at the roundoff floor of a central difference of this loss)
            d = torch.zeros((len(cfg.fields),) + tuple(n), dtype=torch.float64, device=DEV)
            d[0, 2:6, 3:7, 4:8] = 1.0
            d[2, 9:13, 10:14, 1:5] = -0.5
            d = d.reshape(len(cfg.fields), -1)
        an = float((gw * d).sum())
        for eps in (1e-6, 1e-5):
            fd = (eval_loss(adj, wt + eps * d, L) - eval_loss(adj, wt - eps * d, L)) / (2 * eps)
            print(f"{kind} dL/dw direction {k} (step {eps:g}): adjoint {an:.12e} central difference {fd:.12e}")
        assert abs(an - fd) <= TOL * abs(fd), (k, an, fd)
    adj.close()
    chain = DifferentiableChain(cfg)
    box = torch.tensor(chain.box0, dtype=torch.float64, requires_grad=True)
    ds = torch.tensor(chain.ds0, dtype=torch.float64, requires_grad=True)
    phi, lnq = chain(wt, box, ds)
    L(phi, lnq).backward()

    def at(b, dd):
        with torch.no_grad():
            p, q = chain(wt, torch.tensor(b, dtype=torch.float64), torch.tensor(dd, dtype=torch.float64))
            return float(L(p, q))
    # relative steps of 1e-5: with 1e-6 the roundoff of L (about 400) is 5e-7 in a difference
    for dim in range(3):
        h = 1e-5 * chain.box0[dim]
        bp, bm = list(chain.box0), list(chain.box0)
        bp[dim] += h
        bm[dim] -= h
        fd = (at(bp, chain.ds0) - at(bm, chain.ds0)) / (2 * h)
        print(f"{kind} dL/dL_{dim}: adjoint {box.grad[dim].item():.12e} central difference {fd:.12e}")
        assert abs(box.grad[dim].item() - fd) <= TOL * abs(fd), (dim, box.grad[dim].item(), fd)
    for b in (0, len(chain.ds0) - 1):
        h = 1e-5 * chain.ds0[b]
        dp, dm = list(chain.ds0), list(chain.ds0)
        dp[b] += h
        dm[b] -= h
        fd = (at(chain.box0, dp) - at(chain.box0, dm)) / (2 * h)
        print(f"{kind} dL/dds_{b}: adjoint {ds.grad[b].item():.12e} central difference {fd:.12e}")
        assert abs(ds.grad[b].item() - fd) <= TOL * abs(fd), (b, ds.grad[b].item(), fd)
    chain.close()


def test_blend_adjoint_polydisperse(gpu):
    """An A homopolymer (first, so the polydisperse polymer's quadrature chains sit at shifted
    engine indices) blended with a polyDisperseBCP diblock of three Gauss-Laguerre chains: the
    blend's phi against the engine, dL/dw against central differences, and F against the
    engine's free-energy formula through the chains' weights."""
    from polyswift_plusplus_b200.adjoint import DifferentiableBlend, free_energy
    from polyswift_plusplus_b200.config import Block, Polymer
    cfg, w = W.polydisperse_diblock(n=(16, 16, 16), n_g=3)
    pd = dataclasses.replace(cfg.polymers[0], volfrac=0.85)
    homo = Polymer(name="homoA", volfrac=0.15, length=50,
                   blocks=[Block(name="hA", scfield="A", ds=0.02, lengthfrac=1.0)])
    cfg = dataclasses.replace(cfg, polymers=[homo, pd])
    w = np.stack(w)
    s = ScftSolver(cfg)
    s.restore(list(w))
    s.update(1)
    blend = DifferentiableBlend(cfg)
    assert blend.chains() == [(0, 0), (1, 0), (1, 1), (1, 2)]
    wt = torch.tensor(w, device=DEV, requires_grad=True)
    phi, lnq = blend(wt)
    for i in range(2):
        ref = s.phi(i)
        assert np.abs(phi[i].detach().cpu().numpy() - ref).max() <= 1e-12 * np.abs(ref).max()
    assert float(lnq[0].detach()) == pytest.approx(s.scalars()["log_q"][0], rel=1e-13, abs=1e-13)
    L = blend_loss(cfg, seed=21)
    c = torch.tensor([0.3, -0.2, 0.1, 0.25], dtype=torch.float64, device=DEV)
    rng = np.random.default_rng(5)
    t = torch.tensor(rng.uniform(0.2, 0.8, cfg.n_total), device=DEV)

    def Lp(p, q):
        return ((p[0] - t) ** 2).sum() + 0.5 * p[1].sum() + (c * q).sum()
    Lp(phi, lnq).backward()
    gw = wt.grad.detach()
    w0 = wt.detach()

    def at(wv):
        with torch.no_grad():
            p, q = blend(wv)
            return float(Lp(p, q))
    for k in range(2):
        d = torch.tensor(rng.standard_normal(w.shape), device=DEV)
        if k == 1:
            d = torch.zeros((2, 16, 16, 16), dtype=torch.float64, device=DEV)
            d[0, 2:6, 3:7, 4:8] = 1.0
            d[1, 9:13, 10:14, 1:5] = -0.5
            d = d.reshape(2, -1)
        eps = 1e-5
        fd = (at(w0 + eps * d) - at(w0 - eps * d)) / (2 * eps)
        an = float((gw * d).sum())
        print(f"polydisperse blend dL/dw direction {k}: adjoint {an:.12e} central difference {fd:.12e}")
        assert abs(an - fd) <= TOL * abs(fd), (k, an, fd)
    # the chains' free-energy weights reproduce the engine's -vf sum_k (w_k / Gamma) ln Q_k / alpha
    # term: F of the blend's phi and ln Q at the engine's post-update fields equals the engine's F
    vf, al = blend.species_weights()
    wn = torch.tensor(np.stack([s.w(0), s.w(1)]), device=DEV)
    with torch.no_grad():
        F = float(free_energy(wn, phi.detach(), lnq.detach(), cfg.interactions[0].chi * cfg.polymers[0].length,
                              blend.dens_avg(), vf, al))
    print(f"polydisperse blend F: torch {F:.15f} engine {s.scalars()['free_energy']:.15f}")
    assert F == pytest.approx(s.scalars()["free_energy"], rel=1e-12, abs=1e-12)
    blend.close()


def test_adjoint_charged_chain_at_fixed_potential(gpu):
    """A charged diblock (chargeFlexPseudoSpec block A, counter-ions): with the potential psi set,
    the adjoint's phi against the engine's first iteration, and dL/dw and dL/dpsi against
    central differences (psi enters the charged block's Boltzmann factor next to w)."""
    from polyswift_plusplus_b200 import _abi as A
    cfg, w, psi = W.charged_diblock(n=(16, 16, 16), poisson_every=5)
    w = np.stack(w)
    s = ScftSolver(cfg)
    s.restore(list(w))
    s.set_field(A.PS_FIELD_POTENTIAL, 0, psi)
    s.update(1)
    adj = ChainAdjoint(cfg, polymer=0)
    nq = 2
    pt = torch.zeros((nq, cfg.n_total), dtype=torch.float64, device=DEV)
    pt[0] = torch.tensor(psi, device=DEV)
    adj.set_potential(pt)
    wt = torch.tensor(w, device=DEV)
    phi, lnq = adj.forward(wt)
    for i in range(2):
        ref = s.phi(i)
        assert np.abs(phi[i].cpu().numpy() - ref).max() <= 1e-12 * np.abs(ref).max()
    assert lnq == pytest.approx(s.scalars()["log_q"][0], rel=1e-13, abs=1e-13)
    L = loss_terms(cfg, seed=23)
    gw, _, _ = grads(adj, wt, L)
    gpsi = adj.potential_grad(nq)
    assert float(gpsi[1].abs().max()) == 0.0  # no block is charged through the counter-ion field
    rng = np.random.default_rng(29)
    eps = 1e-5
    for k in range(2):
        d = torch.tensor(rng.standard_normal(w.shape), device=DEV)
        fd = (eval_loss(adj, wt + eps * d, L) - eval_loss(adj, wt - eps * d, L)) / (2 * eps)
        an = float((gw * d).sum())
        print(f"charged dL/dw direction {k}: adjoint {an:.12e} central difference {fd:.12e}")
        assert abs(an - fd) <= TOL * abs(fd), (k, an, fd)
    for k in range(2):
        d = torch.zeros_like(pt)
        d[0] = torch.tensor(rng.standard_normal(cfg.n_total), device=DEV)

        def at(p):
            adj.set_potential(p)
            return eval_loss(adj, wt, L)
        fd = (at(pt + eps * d) - at(pt - eps * d)) / (2 * eps)
        an = float((gpsi * d).sum())
        print(f"charged dL/dpsi direction {k}: adjoint {an:.12e} central difference {fd:.12e}")
        assert abs(an - fd) <= TOL * abs(fd), (k, an, fd)
    adj.close()
