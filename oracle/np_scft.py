"""Independent numpy restatement of the SCFT iteration (TEST INFRASTRUCTURE).

A second, separately written FP64 restatement of the same reference sources as
oracle/scft.c, using numpy.fft instead of the project FFT and whole-array
operations instead of point loops.  Tests use it to cross-check the C oracle
on small grids; tests/golden/make_golden.py uses it to write the committed
golden fixtures.  Linear block sequences only.

Reference order of one update (pstrol/PsDomain.cpp:332-372):
  propagators  pspolymer/PsFlexPseudoSpec.cpp:158-293, psfft/PsFFTW.cpp:196-224
  Q            pspolymer/PsBlock.cpp:204-237
  quadrature   pspolymer/PsBlock.cpp:255-380 (0.33333 Simpson factor)
  densities    pspolymer/PsBlock.cpp:153-196
  update       pseffhamil/PsSteepDUpdater.cpp:159-453, psphysf/PsConstraint.cpp:184-262
  free energy  pseffhamil/PsPolymerUpdater.cpp:172-226, pseffhamil/PsFloryInteraction.cpp:274-321
  charges      psphysf/PsChargeDens.cpp:180-190, pssolvent/PsSimpleIons.cpp:90-160,
               pspolymer/PsChargeFlexPseudoSpec.cpp:97-165, pseffhamil/PsPoissonUpdater.cpp:140-262
"""
from __future__ import annotations

import math

import numpy as np

from polyswift_plusplus_b200.config import ScftConfig


def block_steps(bs: float, force: bool) -> int:
    """psbase/PsBlockBase.cpp:252-326"""
    if force:
        v = math.floor(bs + 0.5)
    else:
        frac = bs - float(int(bs))
        if 0.0001 < frac < 0.9999:
            raise ValueError(f"non-integer # of block steps {bs}")
        c, f = math.ceil(bs), math.floor(bs)
        v = c if (c == f or abs(bs - c) < abs(bs - f)) else f
    if v < 4:
        raise ValueError("# of block steps too small")
    return int(v)


def k_squared(cfg: ScftConfig) -> np.ndarray:
    """psbase/PsGridField.cpp:66-104"""
    ks = []
    for d in range(3):
        n = cfg.n[d]
        i = np.arange(n, dtype=np.float64)
        nk = n / 2.0 - np.abs(i - n / 2.0)
        ks.append((2.0 * math.pi * nk / n) / cfg.cell[d])
    kx, ky, kz = np.meshgrid(*ks, indexing="ij")
    return kx * kx + ky * ky + kz * kz


def k2_operator(cfg: ScftConfig, ds: float, bseg: float) -> np.ndarray:
    """pspolymer/PsFlexPseudoSpec.cpp:188-206"""
    return np.exp(-1.0 * ds * k_squared(cfg) * bseg * bseg)


def coulomb_operator(cfg: ScftConfig, bjerrum_len: float) -> np.ndarray:
    """PsPoissonUpdater::build_k2 (pseffhamil/PsPoissonUpdater.cpp:140-175)."""
    k2 = k_squared(cfg)
    with np.errstate(divide="ignore"):
        return np.where(k2 < 0.000000001, 0.0, (4.0 * 3.1415 * bjerrum_len) / k2)


def chain_order(poly) -> list[tuple[int, int]]:
    """(block, from_end) along the chain from its first free end; 0 = HEAD."""
    names = [b.name for b in poly.blocks]
    def conn(b, e):
        lst = poly.blocks[b].headjoined if e == 0 else poly.blocks[b].tailjoined
        return [names.index(x) for x in lst if x != "freeEnd"]
    start = None
    for b in range(len(names)):
        if not conn(b, 0):
            start = (b, 0)
            break
        if not conn(b, 1):
            start = (b, 1)
            break
    order, (b, e) = [], start
    while True:
        order.append((b, e))
        o = 1 - e
        c = conn(b, o)
        if not c:
            break
        nb = c[0]
        e = 1 if names[b] in poly.blocks[nb].tailjoined else 0
        b = nb
    return order


class NpScft:
    def __init__(self, cfg: ScftConfig):
        self.cfg = cfg
        self.shape = tuple(cfg.n)
        self.N = cfg.n_total
        self.nf = len(cfg.fields)
        self.L0 = float(cfg.polymers[0].length)
        self.alpha = [p.length / self.L0 for p in cfg.polymers]
        self.chin = [it.chi * self.L0 for it in cfg.interactions]
        self.ia = [(cfg.field_index(it.scfields[0]), cfg.field_index(it.scfields[1]))
                   for it in cfg.interactions]
        self.avg = [0.0] * self.nf
        self.steps = []
        self.pd = {}
        for ip, P in enumerate(cfg.polymers):
            if P.kind == "polyDisperseBCP":
                self.pd[ip] = self._polydisperse(ip, P)
                continue
            st = []
            for B in P.blocks:
                f = cfg.field_index(B.scfield)
                self.avg[f] = self.avg[f] + 1.0 * B.lengthfrac * P.volfrac
                st.append(block_steps(self.alpha[ip] * B.lengthfrac / B.ds, B.force_block_steps))
            self.steps.append(st)
        for S in getattr(cfg, "solvents", []):  # PsSimpleSolvent::buildSolvers: addToDensAverage
            if S.kind == "simpleIons":
                continue
            f = cfg.field_index(S.scfield)
            self.avg[f] = self.avg[f] + S.volfrac
        self.nq = len(getattr(cfg, "charge_fields", []))
        self.rho = [np.zeros(tuple(cfg.n)) for _ in range(self.nq)]
        self.psi = [np.zeros(tuple(cfg.n)) for _ in range(self.nq)]
        self.t = 0
        if getattr(cfg, "spec_filter", None) is not None:
            raise NotImplementedError("the numpy restatement has no spectral filter")
        self.w = [np.zeros(self.shape) for _ in range(self.nf)]
        self.p = np.zeros(self.shape)
        self.phi = [np.zeros(self.shape) for _ in range(self.nf)]
        self.k2 = {}

    def _polydisperse(self, ip, P):
        """PsPolyDisperseBCP (pspolymer/PsPolyDisperseBCP.cpp:41-455): quadrature chains of the
        seed blocks with the Schulz-distributed block's lengthfrac at the Gauss-Laguerre nodes
        (scipy's generalized Gauss-Laguerre rule for x^(alpha-1) e^-x)."""
        from scipy.special import gamma, roots_genlaguerre
        x, wq = roots_genlaguerre(P.n_g, P.schulz_alpha - 1.0)
        galpha = float(gamma(P.schulz_alpha))
        names = [b.name for b in P.blocks]
        pb = names.index(P.polyblock)
        nlen = float(P.length)
        const_frac = 1.0 - P.blocks[pb].lengthfrac
        ncl = const_frac * nlen
        n_b = (nlen - ncl) / P.schulz_alpha
        fmk = [((xk * n_b + ncl) / nlen) - const_frac for xk in x]
        chains = []
        for k in range(P.n_g):
            fr = [fmk[k] if b == pb else B.lengthfrac for b, B in enumerate(P.blocks)]
            st = [block_steps(self.alpha[ip] * fr[b] / B.ds, B.force_block_steps)
                  for b, B in enumerate(P.blocks)]
            lwt = [wq[k] / galpha if b == pb else 1.0 / P.n_g for b in range(len(P.blocks))]
            chains.append({"frac": fr, "steps": st, "lwt": lwt, "dwt": wq[k] / galpha, "w": wq[k]})
        for b, B in enumerate(P.blocks):  # seed-major block order
            f = self.cfg.field_index(B.scfield)
            for ch in chains:
                self.avg[f] = self.avg[f] + ch["lwt"][b] * ch["frac"][b] * P.volfrac
        self.steps.append(None)
        return {"chains": chains, "galpha": galpha}

    def restore(self, w, p=None):
        self.w = [np.asarray(x, dtype=np.float64).reshape(self.shape).copy() for x in w]
        self.p = np.zeros(self.shape) if p is None else np.asarray(p).reshape(self.shape).copy()

    def _solve(self, q0, wfac, k2, steps):
        out = [q0]
        q = q0
        for _ in range(steps):
            qw = q * wfac
            res = np.fft.ifftn(np.fft.fftn(qw) * k2).real * self.N
            q = (1.0 / self.N) * (res * wfac)
            out.append(q)
        return out

    def _chain(self, P, steps_of):
        order = chain_order(P)
        qs = {}
        for direction in (order, [(b, 1 - e) for b, e in reversed(order)]):
            q = np.ones(self.shape)
            for b, e in direction:
                B = P.blocks[b]
                f = self.cfg.field_index(B.scfield)
                wfac = np.exp(-0.5 * B.ds * self.w[f])
                key = (B.ds, B.bseg_ratio)
                if key not in self.k2:
                    self.k2[key] = k2_operator(self.cfg, B.ds, B.bseg_ratio)
                sl = self._solve(q, wfac, self.k2[key], steps_of[b])
                qs[(b, e)] = sl
                q = sl[-1]
        return qs

    def _qqt(self, a, t, ds):
        num = len(a)
        even = num % 2 == 0
        tail = num - 1 - (3 if even else 2)
        acc = np.zeros(self.shape)
        for n in range(0, tail + 1, 2):
            acc = acc + a[n] * t[num - n - 1]
            acc = acc + (a[n + 1] * t[num - n - 2]) * 4.0
            acc = acc + a[n + 2] * t[num - n - 3]
        acc = acc * (0.33333 * ds)
        if even:
            acc = acc + (a[num - 2] * t[1] + a[num - 1] * t[0]) * (ds * 0.5)
        return acc

    def polymer_pd(self, ip):
        """PsPolyDisperseBCP::update and getLogBigQ (pspolymer/PsPolyDisperseBCP.cpp:282-377):
        per-block Q normalisation, densities weighted by w_k / Gamma(alpha)."""
        P = self.cfg.polymers[ip]
        pdm = self.pd[ip]
        res = []
        for ch in pdm["chains"]:
            qs = self._chain(P, ch["steps"])
            res.append(qs)
        logq = 0.0
        for k, ch in enumerate(pdm["chains"]):
            Q0 = float(np.sum(res[k][(0, 0)][0] * res[k][(0, 1)][-1])) / self.N
            logq = logq + (math.log(Q0) * ch["w"]) / pdm["galpha"]
        for b, B in enumerate(P.blocks):
            f = self.cfg.field_index(B.scfield)
            for k, ch in enumerate(pdm["chains"]):
                a, t = res[k][(b, 0)], res[k][(b, 1)]
                Qb = float(np.sum(a[0] * t[-1])) / self.N
                acc = self._qqt(a, t, B.ds)
                self.phi[f] = self.phi[f] + (ch["dwt"] * P.volfrac / self.alpha[ip]) * ((1.0 / Qb) * acc)
        return math.exp(logq), logq

    def polymer(self, ip):
        P = self.cfg.polymers[ip]
        order = chain_order(P)
        qs = {}
        for direction in (order, [(b, 1 - e) for b, e in reversed(order)]):
            q = np.ones(self.shape)
            for b, e in direction:
                B = P.blocks[b]
                f = self.cfg.field_index(B.scfield)
                wfac = np.exp(-0.5 * B.ds * self.w[f])
                if B.chargefield is not None:
                    c = self.cfg.charge_index(B.chargefield)
                    wfac = wfac * np.exp((B.za * B.alpha * self.L0) * (-0.5 * B.ds) * self.psi[c])
                key = (B.ds, B.bseg_ratio)
                if key not in self.k2:
                    self.k2[key] = k2_operator(self.cfg, B.ds, B.bseg_ratio)
                sl = self._solve(q, wfac, self.k2[key], self.steps[ip][b])
                qs[(b, e)] = sl
                q = sl[-1]
        # Q from block 0: qHeadInitial * qHeadFinal
        Q = float(np.sum(qs[(0, 0)][0] * qs[(0, 1)][-1])) / self.N
        for b, B in enumerate(P.blocks):
            f = self.cfg.field_index(B.scfield)
            a, t = qs[(b, 0)], qs[(b, 1)]
            num = len(a)
            even = num % 2 == 0
            tail = num - 1 - (3 if even else 2)
            acc = np.zeros(self.shape)
            for n in range(0, tail + 1, 2):
                acc = acc + a[n] * t[num - n - 1]
                acc = acc + (a[n + 1] * t[num - n - 2]) * 4.0
                acc = acc + a[n + 2] * t[num - n - 3]
            acc = acc * (0.33333 * B.ds)
            if even:
                acc = acc + (a[num - 2] * t[1] + a[num - 1] * t[0]) * (B.ds * 0.5)
            self.phi[f] = self.phi[f] + (1.0 * P.volfrac / self.alpha[ip]) * ((1.0 / Q) * acc)
            if B.chargefield is not None:
                c = self.cfg.charge_index(B.chargefield)
                self.rho[c] = self.rho[c] + (self.phi[f] * B.alpha) * B.za
        return Q, qs

    def solvent(self, S):
        """PsSimpleSolvent::setPhysFields (pssolvent/PsSimpleSolvent.cpp:86-140)."""
        f = self.cfg.field_index(S.scfield)
        wfactor = np.exp(self.w[f] * (-1.0 / self.L0))
        Q = float(np.sum(wfactor)) / self.N
        self.phi[f] = self.phi[f] + wfactor * (S.volfrac / Q)
        return Q

    def ions(self, S):
        """PsSimpleIons::setPhysFields (pssolvent/PsSimpleIons.cpp:90-160)."""
        c = self.cfg.charge_index(S.chargefield)
        e = np.exp(self.psi[c] * (-1.0 * S.zc))
        Q = float(np.sum(e)) / self.N
        e = e * (-S.neutral_factor / (Q * S.zc))
        if S.blockfield is not None:
            self.rho[self.cfg.charge_index(S.blockfield)] = e.copy()
        self.rho[c] = self.rho[c] + e * S.zc
        return Q

    def poisson(self, P):
        """PsPoissonUpdater::update (pseffhamil/PsPoissonUpdater.cpp:196-262)."""
        kc = coulomb_operator(self.cfg, P.bjerrum_len)
        for name in P.updatefields:
            c = self.cfg.charge_index(name)
            self.rho[c] = self.rho[c] + (-1.0 * (float(np.sum(self.rho[c])) / self.N))
            res = np.fft.ifftn(np.fft.fftn(self.rho[c]) * kc).real * self.N
            psi0 = self.psi[c]
            with np.errstate(divide="ignore", invalid="ignore"):
                frac = np.abs((res * (1.0 / self.N) - psi0) / psi0)
            res = np.where(frac > 0.2, psi0 * 1.2, res)
            self.psi[c] = res * (1.0 / self.N)

    def iterate(self):
        self.phi = [np.zeros(self.shape) for _ in range(self.nf)]
        self.rho = [np.zeros(self.shape) for _ in range(self.nq)]
        solvents = list(getattr(self.cfg, "solvents", []))
        Qsol = [self.ions(S) if S.kind == "simpleIons" else self.solvent(S) for S in solvents]
        Qs, logQs = [], []
        for ip in range(len(self.cfg.polymers)):
            if ip in self.pd:
                q, lq = self.polymer_pd(ip)
            else:
                q = self.polymer(ip)[0]
                lq = math.log(q)
            Qs.append(q)
            logQs.append(lq)
        nf = self.nf
        dh = []
        for i in range(nf):
            d = self.p - self.w[i]
            for it, (a, b) in enumerate(self.ia):
                if i in (a, b):
                    o = b if i == a else a
                    d = d + (self.phi[o] - self.avg[o]) * self.chin[it]
            dh.append(d)
        lam0, lam1 = self.cfg.updater.relaxlambdas
        if self.cfg.updater.kind.replace("GPU", "") != "steepestDescent":
            raise NotImplementedError("the numpy restatement covers steepest descent only")
        for i in range(nf):
            x = sum((dh[j] for j in range(nf) if j != i), np.zeros(self.shape)) * (-1.0 * lam1) + dh[i]
            self.w[i] = self.w[i] + x * lam0
        pr = sum(self.w, np.zeros(self.shape))
        if nf == 2:
            pr = 0.5 * pr
        else:
            for it, (a, b) in enumerate(self.ia):
                for n in range(nf):
                    if n not in (a, b):
                        pr = pr + (self.phi[n] - self.avg[n]) * self.chin[it]
            pr = (1.0 / 3.0) * pr
        self.p = pr - np.sum(pr) / self.N
        fe = -sum(P.volfrac * lq / a for P, lq, a in zip(self.cfg.polymers, logQs, self.alpha))
        fe -= sum(S.volfrac * math.log(Q) * self.L0 for S, Q in zip(solvents, Qsol))
        dens = -sum(self.phi[i] * self.w[i] for i in range(nf))
        for it, (a, b) in enumerate(self.ia):
            dens = dens + self.chin[it] * (self.phi[a] * self.phi[b] - self.avg[a] * self.avg[b])
        fe += float(np.sum(dens)) / self.N
        inc = float(np.max(np.abs(sum(self.phi, np.zeros(self.shape)) - 1.0)))
        P = getattr(self.cfg, "poisson", None)
        if P is not None and self.t >= P.apply_start and (P.apply_end < 0 or self.t <= P.apply_end) \
                and (self.t - P.apply_start) % P.apply_frequency == 0:
            self.poisson(P)
        self.t += 1
        return {"free_energy": fe, "q": Qs, "max_incomp": inc}
