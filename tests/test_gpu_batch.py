"""Batched instances (ps_gpu_batch_*) against the same instances run alone.

A batch merges the propagator sweeps of every instance of one grid size into
one launch per contour step and runs the field updates as parallel graph
branches.  With the kernel variant pinned, every instance of the batch must
be bit-identical to ps_gpu_iterate on that instance alone; with per-class
autotuning the variants differ only in rounding (FP64: 1e-10).  One FP64
instance is also checked against the oracle at 1e-10.
"""
import dataclasses

import numpy as np
import pytest

import oracle as O
from polyswift_plusplus_b200 import _abi as A
from polyswift_plusplus_b200 import workloads as W
from polyswift_plusplus_b200.scft import ScftBatch, ScftSolver

pytestmark = pytest.mark.gpu


def rel(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _anderson_early(cfg, start=2):
    return dataclasses.replace(cfg, updater=dataclasses.replace(cfg.updater, anderson_start=start))


def _mixed_batch():
    """Uneven grids, chiN, f_A and homopolymer fractions, both precisions."""
    specs = [(16, 15.0, 0.30, 0.10, "fp64"), (16, 25.0, 0.45, 0.0, "fp64"),
             (24, 20.0, 0.35, 0.15, "fp64"), (16, 18.0, 0.40, 0.05, "mixed"),
             (32, 22.0, 0.25, 0.12, "mixed"), (16, 12.5, 0.50, 0.20, "fp64")]
    out = []
    for i, (n, chin, f, ph, prec) in enumerate(specs):
        cfg = _anderson_early(W.blend(n, chin, f, ph, precision=prec, seed=100 + i))
        x, _, _ = W.coords(cfg)
        c = np.cos(2 * np.pi * x / cfg.box[0]).reshape(-1)
        w = W.random_fields(cfg, 0.1)
        out.append((cfg, [w[0] + c, w[1] - c]))
    return out


def _run_single(cfg, w, iters, variant):
    s = ScftSolver(cfg)
    if variant is not None:
        s.set_variant(variant)
    s.restore(w)
    s.update(iters)
    return s


@pytest.mark.parametrize("noise", [0.0, 0.01])
@pytest.mark.parametrize("variant", [0, 2, 10])
def test_batch_bit_identical_to_single_instances(gpu, variant, noise):
    """variant 10 (bit 3): every instance's sweeps as its own concurrent launch
    chains inside the batch graph, instead of shared launches per step."""
    items = _mixed_batch()
    if noise:  # every other instance draws updater noise on the device
        items = [(dataclasses.replace(c, updater=dataclasses.replace(c.updater, noise=noise)) if i % 2 else c, w)
                 for i, (c, w) in enumerate(items)]
    iters = 6  # eager first iteration, graph replays, Anderson from iteration 2
    with ScftBatch([c for c, _ in items]) as b:
        b.set_variant(variant)
        for i, (_, w) in enumerate(items):
            b.instance(i).restore(w)
        b.update(2)
        b.update(iters - 2)
        class_of, variants = b.classes()
        assert len(set(class_of)) == 4  # (16, fp64), (24, fp64), (16, mixed), (32, mixed)
        assert b.launches_per_iteration > 0
        for i, (cfg, w) in enumerate(items):
            s = _run_single(cfg, w, iters, variant)
            v = b.instance(i)
            assert v.scalars()["iteration"] == s.scalars()["iteration"] == iters
            assert v.scalars()["free_energy"] == s.scalars()["free_energy"]
            for f in range(2):
                assert np.array_equal(v.w(f), s.w(f))
                assert np.array_equal(v.phi(f), s.phi(f))
            assert np.array_equal(v.pressure(), s.pressure())
            s.close()


def test_batch_autotuned_matches_oracle(gpu, oracle_lib):
    # steepest descent: Anderson this early amplifies rounding differences far
    # beyond 1e-10 (its own trajectory test uses 1e-6)
    items = [(dataclasses.replace(c, updater=dataclasses.replace(c.updater, kind="steepestDescent")), w)
             for c, w in _mixed_batch()]
    iters = 5
    with ScftBatch([c for c, _ in items]) as b:
        for i, (_, w) in enumerate(items):
            b.instance(i).restore(w)
        b.update(iters)
        _, variants = b.classes()
        assert all(0 <= v < 8 for v in variants)
        for i in (0, 2):  # FP64 instances against the oracle
            cfg, w = items[i]
            o = O.Oracle(cfg)
            o.restore(w)
            ho = o.update(iters)
            sc = b.instance(i).scalars()
            assert abs(sc["free_energy"] - ho[-1]["free_energy"]) <= 1e-10 * max(abs(ho[-1]["free_energy"]), 1e-2)
            for f in range(2):
                assert rel(b.instance(i).w(f), o.w(f)) < 1e-10
                assert rel(b.instance(i).phi(f), o.phi(f)) < 1e-10


def test_batch_blend_workload_matches_single(gpu):
    """Eight instances of the batched blend workload (grids 32..96, FP32 sweeps),
    autotuned per size class, against the same instances run one by one (each
    autotuned on its own: variants may differ, so agreement is to FP32 rounding)."""
    items = W.blend_instances(count=8)
    iters = 12
    with ScftBatch([c for c, _ in items]) as b:
        for i, (_, w) in enumerate(items):
            b.instance(i).restore(w)
        b.update(iters)
        got = b.scalars()
    for (cfg, w), sb in zip(items, got):
        s = _run_single(cfg, w, iters, None)
        ss = s.scalars()
        s.close()
        assert sb["iteration"] == ss["iteration"] == iters
        assert np.isfinite(sb["free_energy"])
        assert abs(sb["free_energy"] - ss["free_energy"]) < 1e-5 * max(abs(ss["free_energy"]), 1.0)
        for ip in range(len(cfg.polymers)):
            assert sb["q"][ip] == pytest.approx(ss["q"][ip], rel=1e-5)


def test_batch_rejects_bad_instances(gpu):
    cfg = W.blend(16, 15.0, 0.3, 0.1, precision="fp64")
    bad = dataclasses.replace(cfg, n=(20, 16, 16))
    with pytest.raises(A.PsError) as e:
        ScftBatch([cfg, bad])
    assert e.value.code == A.PS_INPUT_ERR


def test_batch_instance_precision_is_fixed(gpu):
    cfg = W.blend(16, 15.0, 0.3, 0.1, precision="mixed")
    with ScftBatch([cfg]) as b:
        with pytest.raises(A.PsError) as e:
            b.instance(0).set_precision("fp64")
        assert e.value.code == A.PS_ATTRIB_ERR


@pytest.mark.parametrize("poisson", [False, True])
def test_batch_with_charged_instances_bit_identical(gpu, poisson):
    """Charged diblocks (ions + charged block; with and without their Poisson
    updater, which runs between batch iterations) batched with a plain diblock:
    bit-identical to single runs."""
    items = []
    for i, n in enumerate(((16, 16, 16), (16, 16, 16))):
        cfg, w, psi = W.charged_diblock(n=n, seed=300 + i, poisson_every=2)
        if not poisson:
            cfg.poisson = None
        items.append((cfg, w, psi))
    plain, wp = W.diblock32(n=16)
    with ScftBatch([c for c, _, _ in items] + [plain]) as b:
        b.set_variant(0)
        for i, (_, w, psi) in enumerate(items):
            b.instance(i).restore(w)
            b.instance(i).set_field(A.PS_FIELD_POTENTIAL, 0, psi)
        b.instance(2).restore(wp)
        b.update(4)
        for i, (cfg, w, psi) in enumerate(items):
            s = ScftSolver(cfg)
            s.set_variant(0)
            s.restore(w)
            s.set_field(A.PS_FIELD_POTENTIAL, 0, psi)
            s.update(4)
            v = b.instance(i)
            assert v.scalars()["free_energy"] == s.scalars()["free_energy"]
            for c in range(2):
                assert np.array_equal(v.rho(c), s.rho(c))
            assert np.array_equal(v.w(0), s.w(0))
            s.close()


def test_batch_with_filtered_instances_bit_identical(gpu):
    """Spectral filters (simple and multi) on batch instances run at their scheduled
    steps between batch iterations: each instance bit-identical to its single run."""
    from polyswift_plusplus_b200.config import SpecFilter
    items = []
    for i, kind in enumerate(("simple", "multi", None)):
        cfg, w = W.diblock32(n=16, precision="fp64" if i != 1 else "mixed")
        if kind is not None:
            cfg = dataclasses.replace(cfg, spec_filter=SpecFilter(
                updatefields=["A", "B"], cutoff_factor=0.02, filter_strength=0.5, apply_start=1,
                apply_frequency=2, apply_end=9, spec_cells=(4, 4, 4) if kind == "multi" else None))
        items.append((cfg, w))
    iters = 7
    with ScftBatch([c for c, _ in items]) as b:
        b.set_variant(0)
        for i, (_, w) in enumerate(items):
            b.instance(i).restore(w)
        b.update(3)
        b.update(iters - 3)
        for i, (cfg, w) in enumerate(items):
            s = ScftSolver(cfg)
            s.set_variant(0)
            s.restore(w)
            s.update(iters)
            v = b.instance(i)
            assert v.scalars()["free_energy"] == s.scalars()["free_energy"]
            for f in range(2):
                assert np.array_equal(v.w(f), s.w(f))
            s.close()


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_batch_class_with_cluster_plane_pass(gpu, precision):
    """A size class of 8 x 256 x 256 instances with the cluster plane pass forced
    (variant 16: one merged plane launch covers every member's sweeps; eight CTAs
    per plane): each instance bit-identical to its single run with the same
    variant."""
    items = []
    for i in range(3):
        cfg, _ = W.diblock32(n=16, precision=precision)
        cfg = dataclasses.replace(cfg, n=(8, 256, 256), cell=(0.5, 0.03125, 0.03125), seed=700 + i)
        items.append((cfg, W.random_fields(cfg, 0.3)))
    iters = 3
    with ScftBatch([c for c, _ in items]) as b:
        b.set_variant(16)
        for i, (_, w) in enumerate(items):
            b.instance(i).restore(w)
        b.update(iters)
        _, variants = b.classes()
        assert variants == [16]
        for i, (cfg, w) in enumerate(items):
            s = ScftSolver(cfg)
            s.set_variant(16)
            s.restore(w)
            s.update(iters)
            v = b.instance(i)
            assert v.scalars()["free_energy"] == s.scalars()["free_energy"]
            for f in range(2):
                assert np.array_equal(v.phi(f), s.phi(f))
            s.close()
