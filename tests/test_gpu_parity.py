"""GPU parity: the sm_100a path through the C-ABI against the FP64 oracle.

Tolerances: FP64 device path 1e-10 relative (fields: 1e-10 of the field's max
magnitude); mixed path |dF/F| < 1e-6.
"""
import math
from pathlib import Path

import numpy as np
import pytest

import oracle as O
from polyswift_plusplus_b200 import _abi as A
from polyswift_plusplus_b200 import workloads as W
from polyswift_plusplus_b200.config import Block, Interaction, Polymer, ScftConfig, Updater
from polyswift_plusplus_b200.scft import B200FFT, ScftSolver

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden"
TOL64 = 1e-10


def rel(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def run_both(cfg, w, iters, p=None):
    g = ScftSolver(cfg)
    g.restore(w, p)
    o = O.Oracle(cfg)
    o.restore(w, p)
    hist_o = o.update(iters)
    hist_g = []
    for _ in range(iters):
        g.update(1)
        hist_g.append(g.scalars())
    return g, o, hist_g, hist_o


def assert_parity(cfg, g, o, hist_g, hist_o, tol=TOL64):
    for hg, ho in zip(hist_g, hist_o):
        assert abs(hg["free_energy"] - ho["free_energy"]) <= tol * max(abs(ho["free_energy"]), 1e-2)
        for ip in range(len(cfg.polymers)):
            assert hg["q"][ip] == pytest.approx(ho["q"][ip], rel=tol)
        assert abs(hg["max_incomp"] - ho["max_incomp"]) <= tol * max(ho["max_incomp"], 1e-3)
    for i in range(len(cfg.fields)):
        assert rel(g.w(i), o.w(i)) < tol
        assert rel(g.phi(i), o.phi(i)) < tol
    assert rel(g.pressure(), o.pressure()) < tol * 10


@pytest.mark.parametrize("shape", [(8, 8, 8), (16, 16, 16), (12, 12, 12), (32, 32, 32),
                                   (24, 48, 48), (16, 64, 1), (8, 4, 256), (4, 16, 32),
                                   (64, 64, 64)])
def test_fft_plugin_matches_oracle(gpu, oracle_lib, shape):
    rng = np.random.default_rng(3)
    d = rng.standard_normal(shape)
    k = rng.standard_normal(shape)  # non-symmetric kdata: exercises the c2c real-part semantics
    f = B200FFT(shape)
    assert f.getFFTSize() == d.size
    got = f.scaledFFTPair(d, k).reshape(shape)
    ref = O.scaled_fft_pair(d, k)
    assert rel(got, ref) < 1e-12


@pytest.mark.parametrize("shape", [(8, 8, 8), (12, 16, 24), (32, 32, 32), (24, 48, 48),
                                   (16, 64, 1), (8, 4, 256), (1, 16, 32), (64, 1, 1),
                                   (64, 64, 64), (128, 128, 128)])
def test_fft_plugin_interface_matches_oracle(gpu, oracle_lib, shape):
    """Every other transform of PsFFTBase<double,3> (psbase/PsFFTBase.h:83-134):
    scaledFFTPairIm, convolveRe, forwardFFTAbs, calcForwardFFT and
    calcBackwardFFT against the oracle's c2c restatement of PsFFTW, on fused
    planes, row-pass grids (256-point z rows) and degenerate axes."""
    rng = np.random.default_rng(11)
    d = rng.standard_normal(shape)
    d2 = rng.standard_normal(shape)
    k = rng.standard_normal(shape)  # no symmetry: the odd part drives scaledFFTPairIm
    f = B200FFT(shape)
    assert f.getGrid() == tuple(shape)
    r = lambda a: a.reshape(shape)
    assert rel(r(f.scaledFFTPairIm(d, k)), O.scaled_fft_pair_im(d, k)) < 1e-12
    assert rel(r(f.convolveRe(d, d2)), O.convolve_re(d, d2)) < 1e-12
    assert rel(r(f.forwardFFTAbs(d)), O.forward_fft_abs(d)) < 1e-12
    assert rel(r(f.calcForwardFFT(d)), O.calc_forward_fft(d)) < 1e-12
    assert rel(r(f.calcBackwardFFT(d)), O.calc_backward_fft(d)) < 1e-12
    # the handle's buffers are reused: a second call with other inputs
    assert rel(r(f.convolveRe(d2, k)), O.convolve_re(d2, k)) < 1e-12
    assert rel(r(f.scaledFFTPair(d, k)), O.scaled_fft_pair(d, k)) < 1e-12
    f.close()


def test_fft_plugin_interface_known_answers(gpu):
    """Known answers independent of the oracle: the transforms of a single
    cosine mode and a delta function."""
    n = (16, 8, 12)
    N = n[0] * n[1] * n[2]
    x, y, z = np.meshgrid(*[np.arange(v) for v in n], indexing="ij")
    c = np.cos(2 * np.pi * (2 * x / n[0] + 3 * z / n[2]))
    f = B200FFT(n)
    pw = f.forwardFFTAbs(c).reshape(n)
    exp = np.zeros(n)
    exp[2, 0, 3] = exp[-2, 0, -3] = (N / 2) ** 2
    assert np.abs(pw - exp).max() < 1e-9 * N * N
    delta = np.zeros(n)
    delta[0, 0, 0] = 1.0
    # FFT of a delta at the origin is 1 everywhere; convolving with it gives N times
    # the input (both transforms unnormalised)
    assert np.abs(f.calcForwardFFT(delta) - 1.0).max() < 1e-14
    assert np.abs(f.convolveRe(c, delta).reshape(n) - N * c).max() < 1e-12 * N
    # scaledFFTPairIm with an odd kdata i*sign(kx): a Hilbert-like transform of the cosine
    kx = np.fft.fftfreq(n[0])[:, None, None] * np.ones(n)
    res = f.scaledFFTPairIm(c, np.sign(kx)).reshape(n)
    ref = np.fft.ifftn(np.fft.fftn(1j * c) * np.sign(kx)).real * N
    assert np.abs(res - ref).max() < 1e-10
    f.close()


@pytest.mark.parametrize("shape", [(1, 16, 32), (16, 1, 32), (64, 1, 1), (1, 1, 64), (1, 64, 1)])
def test_fft_plugin_degenerate_axes(gpu, oracle_lib, shape):
    """Grids with extent-1 axes (1-D and 2-D runs in any orientation)."""
    rng = np.random.default_rng(5)
    d = rng.standard_normal(shape)
    k = rng.standard_normal(shape)
    got = B200FFT(shape).scaledFFTPair(d, k).reshape(shape)
    assert rel(got, O.scaled_fft_pair(d, k)) < 1e-12


@pytest.mark.parametrize("shape", [(64, 1, 1), (1, 1, 64), (1, 32, 32)])
def test_fp64_low_dimensional_grids(gpu, oracle_lib, shape):
    """One- and two-dimensional SCFT (lamellae along the one long axis)."""
    cfg, _ = W.diblock32(n=8)
    cfg.n = shape
    cfg.cell = tuple(4.0 / s if s > 1 else 0.125 for s in shape)
    w = W.random_fields(cfg, 0.3)
    ax = [i for i, s in enumerate(shape) if s > 1][0]
    x = W.coords(cfg)[ax].reshape(-1)
    c = np.cos(2 * math.pi * x / cfg.box[ax])
    w = [w[0] + c, w[1] - c]
    g, o, hg, ho = run_both(cfg, w, 8)
    assert_parity(cfg, g, o, hg, ho)


def test_mixed_long_x_axis(gpu, oracle_lib):
    """FP32 sweeps on a 256 x 8 x 8 grid (x pencils of length 256) against the
    FP64 oracle at the mixed-path tolerance."""
    cfg, _ = W.diblock32(n=8, precision="mixed")
    cfg.n = (256, 8, 8)
    cfg.cell = (8.0 / 256, 0.25, 0.25)
    x = W.coords(cfg)[0].reshape(-1)
    c = np.cos(2 * math.pi * x / cfg.box[0])
    w = W.random_fields(cfg, 0.2)
    w = [w[0] + c, w[1] - c]
    g = ScftSolver(cfg)
    g.restore(w)
    g.update(4)
    o = O.Oracle(cfg)
    o.restore(w)
    ho = o.update(4)
    assert abs(g.scalars()["free_energy"] - ho[-1]["free_energy"]) < 1e-5
    for i in range(2):
        assert rel(g.phi(i), o.phi(i)) < 1e-4


@pytest.mark.parametrize("n", [16, 32])
def test_fp64_diblock_parity(gpu, oracle_lib, n):
    cfg, w = W.diblock32(n=n)
    g, o, hg, ho = run_both(cfg, w, 12 if n == 32 else 25)
    assert_parity(cfg, g, o, hg, ho)
    assert g.launches_per_iteration > 0


@pytest.mark.parametrize("variant", list(range(8)) + [8, 9, 10, 11, 14])
@pytest.mark.parametrize("n", [16, 32])
def test_every_kernel_variant_matches_oracle(gpu, oracle_lib, variant, n):
    cfg, w = W.diblock32(n=n)
    g = ScftSolver(cfg)
    g.set_variant(variant)
    g.restore(w)
    o = O.Oracle(cfg)
    o.restore(w)
    ho = o.update(4)
    hg = []
    for _ in range(4):
        g.update(1)
        hg.append(g.scalars())
    assert g.variant()[0] == variant
    assert_parity(cfg, g, o, hg, ho)


def _slab256(precision):
    """A diblock on an 8 x 256 x 256 grid: 256 x 256 y-z planes (the cluster plane
    pass) at a size the FP64 oracle runs in seconds."""
    cfg, _ = W.diblock32(n=16, precision=precision)
    cfg.n = (8, 256, 256)
    cfg.cell = (0.5, 0.03125, 0.03125)
    x, y, z = W.coords(cfg)
    c = np.cos(2 * math.pi * z / cfg.box[2]).reshape(-1) + 0.5 * np.cos(2 * math.pi * y / cfg.box[1]).reshape(-1)
    w = W.random_fields(cfg, 0.1)
    return cfg, [w[0] + c, w[1] - c]


@pytest.mark.parametrize("base", [0, 8])
def test_cluster_plane_pass_256(gpu, oracle_lib, base):
    """Variant bit 4: FP32 256 x 256 y-z planes as one plane pass on a cluster of
    eight CTAs (column eighths for the y FFTs, row eighths for the z passes,
    exchanged through distributed shared memory), instead of a row pass and
    two y pencil passes.  Against the same variant without the bit (the FFT
    decomposition differs, so FP32 rounding does) and against the FP64 oracle
    at the mixed-path tolerance."""
    cfg, w = _slab256("mixed")
    iters = 3
    runs = {}
    for v in (base, base | 16):
        g = ScftSolver(cfg)
        g.set_variant(v)
        g.restore(w)
        g.update(iters)
        assert g.variant()[0] == v
        runs[v] = (g.scalars(), [g.w(i) for i in range(2)], [g.phi(i) for i in range(2)],
                   g.propagator(0, 1, A.PS_FROM_HEAD, 20))
        g.close()
    o = O.Oracle(cfg)
    o.restore(w)
    ho = o.update(iters)
    a, b = runs[base], runs[base | 16]
    fo = ho[-1]["free_energy"]
    print(f"F: cluster {b[0]['free_energy']:.10f}, rows {a[0]['free_energy']:.10f}, oracle {fo:.10f}; "
          f"phi vs oracle: cluster {max(rel(b[2][i], o.phi(i)) for i in range(2)):.2e}, "
          f"rows {max(rel(a[2][i], o.phi(i)) for i in range(2)):.2e}; "
          f"cluster vs rows: w {max(rel(b[1][i], a[1][i]) for i in range(2)):.2e}, q {rel(b[3], a[3]):.2e}")
    # FP32 sweeps: F within the mixed path's floor of a few 1e-6, fields to ~1e-5
    assert abs(b[0]["free_energy"] - fo) < 1e-5
    assert abs(b[0]["free_energy"] - a[0]["free_energy"]) < 1e-5
    assert b[0]["q"][0] == pytest.approx(ho[-1]["q"][0], rel=1e-5)
    for i in range(2):
        assert rel(b[1][i], a[1][i]) < 1e-4
        assert rel(b[2][i], o.phi(i)) < 1e-4
    assert rel(b[3], a[3]) < 1e-4


@pytest.mark.parametrize("base", [0, 8])
def test_cluster_plane_pass_256_fp64(gpu, oracle_lib, base):
    """Variant bit 4 in FP64: 256 x 256 y-z planes (528 KB as a half plane) as one
    plane pass on a cluster of eight CTAs (column eighths for the y FFTs, row
    eighths for the z passes), against the FP64 oracle at the FP64 tolerance
    over three iterations, and against the row + y-pencil design."""
    cfg, w = _slab256("fp64")
    iters = 3
    o = O.Oracle(cfg)
    o.restore(w)
    ho = o.update(iters)
    runs = {}
    for v in (base, base | 16):
        g = ScftSolver(cfg)
        g.set_variant(v)
        g.restore(w)
        hg = []
        for _ in range(iters):
            g.update(1)
            hg.append(g.scalars())
        assert g.variant()[0] == v
        if v & 16:
            assert_parity(cfg, g, o, hg, ho)
        runs[v] = ([g.w(i) for i in range(2)], g.propagator(0, 1, A.PS_FROM_HEAD, 20),
                   hg[-1]["free_energy"])
        g.close()
    a, b = runs[base], runs[base | 16]
    print(f"FP64 cluster vs rows: w {max(rel(b[0][i], a[0][i]) for i in range(2)):.2e}, "
          f"q {rel(b[1], a[1]):.2e}, dF {abs(b[2] - a[2]):.2e}")
    for i in range(2):
        assert rel(b[0][i], a[0][i]) < 1e-11
    assert rel(b[1], a[1]) < 1e-11


@pytest.mark.parametrize("prec,tol", [("mixed", 1e-5), ("fp64", 1e-11)])
def test_cluster_plane_pass_full_256_cubed(gpu, prec, tol):
    """The cluster plane pass at full size: the 256^3 ABC triblock (its box and chiN, Ns = 20)
    over two iterations with the cluster pass (variant 26) and with the row + y-pencil design
    (variant 10); the two decompositions agree to FP64 roundoff, and to FP32 rounding for FP32
    sweeps."""
    import dataclasses
    cfg, w = W.triblock256(precision=prec)
    p = cfg.polymers[0]
    cfg = dataclasses.replace(cfg, polymers=[dataclasses.replace(
        p, blocks=[dataclasses.replace(b, ds=0.05) for b in p.blocks])])
    runs = {}
    for v in (10, 26):
        g = ScftSolver(cfg)
        g.set_variant(v)
        g.restore(w)
        g.update(2)
        assert g.variant()[0] == v
        runs[v] = ([g.phi(i) for i in range(3)], g.scalars()["free_energy"], g.block_steps(0, 1))
        g.close()
    (pr, fr, nb), (pc, fc, _) = runs[10], runs[26]
    assert nb == 8
    d = max(rel(pc[i], pr[i]) for i in range(3))
    print(f"256^3 {prec}: cluster vs rows: phi {d:.2e}, F {fc:.12e} / {fr:.12e}")
    assert d < tol
    assert abs(fc - fr) <= tol * max(abs(fr), 1e-3)


def test_cluster_variant_only_where_it_exists(gpu):
    for prec, n in (("mixed", 16), ("fp64", 16)):
        cfg, _ = W.diblock32(n=n, precision=prec)
        g = ScftSolver(cfg)
        with pytest.raises(A.PsError) as e:
            g.set_variant(16)
        assert e.value.code == A.PS_ATTRIB_ERR
        g.close()
    for prec in ("mixed", "fp64"):  # eight CTAs per plane in both precisions
        cfg, _ = _slab256(prec)
        g = ScftSolver(cfg)
        g.set_variant(16)
        assert g.variant()[0] == 16
        g.close()


def test_autotune_picks_a_measured_variant(gpu):
    cfg, w = W.diblock32(n=32, precision="mixed")
    g = ScftSolver(cfg)
    g.restore(w)
    g.update(3)
    v, ms = g.variant()
    timed = [t for t in ms if t > 0]
    assert 0 <= v < 32 and len(timed) >= 8
    assert ms[v] == min(timed)


def test_xy_design_mixed_and_blend(gpu, oracle_lib):
    """The row + x-y plane design on a blend (3 sweeps, one aliased) in both precisions."""
    for prec, tol in (("fp64", TOL64), ("mixed", None)):
        cfg = W.blend(16, 18.0, 0.35, 0.15, precision=prec, seed=12, anderson=False)
        w = W.random_fields(cfg, 0.3)
        g = ScftSolver(cfg)
        g.set_variant(6)
        g.restore(w)
        o = O.Oracle(cfg)
        o.restore(w)
        ho = o.update(5)
        hg = []
        for _ in range(5):
            g.update(1)
            hg.append(g.scalars())
        if tol:
            assert_parity(cfg, g, o, hg, ho)
        else:
            assert abs(hg[-1]["free_energy"] - ho[-1]["free_energy"]) < 1e-5


def test_fp64_propagator_slices(gpu, oracle_lib):
    cfg, w = W.diblock32(n=16)
    g, o, _, _ = run_both(cfg, w, 2)
    for ib, steps in ((0, 30), (1, 70)):
        for end in (A.PS_FROM_HEAD, A.PS_FROM_TAIL):
            for n in (0, 1, steps // 2, steps):
                assert rel(g.propagator(0, ib, end, n), o.propagator(0, ib, end, n)) < TOL64


@pytest.mark.parametrize("name", ["diblock8", "triblock8", "blend8"])
def test_gpu_matches_golden(gpu, name):
    import sys
    sys.path.insert(0, str(GOLD))
    from make_golden import small_configs
    cfg, _ = small_configs()[name]
    gd = np.load(GOLD / f"scft_{name}.npz")
    g = ScftSolver(cfg)
    g.restore(list(gd["w0"]))
    fe = []
    for _ in range(len(gd["free_energy"])):
        g.update(1)
        fe.append(g.scalars()["free_energy"])
    assert np.allclose(fe, gd["free_energy"], rtol=TOL64, atol=1e-12)
    for i in range(len(cfg.fields)):
        assert rel(g.w(i), gd["w"][i]) < TOL64
        assert rel(g.phi(i), gd["phi"][i]) < TOL64


def test_fp64_triblock_three_fields(gpu, oracle_lib):
    ds = 0.02
    tri = Polymer("abc", 1.0, 100, [Block("a", "A", ds, 0.3, ["freeEnd"], ["b"]),
                                    Block("b", "B", ds, 0.4, ["a"], ["c"]),
                                    Block("c", "C", ds, 0.3, ["b"], ["freeEnd"])])
    cfg = ScftConfig(n=(16, 16, 16), cell=(0.25,) * 3, fields=["A", "B", "C"], polymers=[tri],
                     interactions=[Interaction("AB", 0.3, ["A", "B"]),
                                   Interaction("BC", 0.3, ["B", "C"]),
                                   Interaction("AC", 0.45, ["A", "C"])],
                     updater=Updater(relaxlambdas=(0.05, 0.025)), seed=91)
    w = W.random_fields(cfg, 0.3)
    g, o, hg, ho = run_both(cfg, w, 10)
    assert_parity(cfg, g, o, hg, ho)


def test_fp64_triblock_three_fields_anderson(gpu, oracle_lib):
    """Anderson mixing on three fields (the nf = 3 update kernels) against the
    oracle; as for the diblock trajectory test, the Gram entries cancel, so 1e-6."""
    ds = 0.02
    tri = Polymer("abc", 1.0, 100, [Block("a", "A", ds, 0.3, ["freeEnd"], ["b"]),
                                    Block("b", "B", ds, 0.4, ["a"], ["c"]),
                                    Block("c", "C", ds, 0.3, ["b"], ["freeEnd"])])
    cfg = ScftConfig(n=(16, 16, 16), cell=(0.25,) * 3, fields=["A", "B", "C"], polymers=[tri],
                     interactions=[Interaction("AB", 0.3, ["A", "B"]),
                                   Interaction("BC", 0.3, ["B", "C"]),
                                   Interaction("AC", 0.45, ["A", "C"])],
                     updater=Updater(kind="andersonMixing", relaxlambdas=(0.05, 0.025), anderson_depth=4,
                                     anderson_mix=0.1, anderson_start=3), seed=91)
    w = W.random_fields(cfg, 0.3)
    g, o, hg, ho = run_both(cfg, w, 12)
    assert_parity(cfg, g, o, hg, ho, tol=1e-6)


def test_fp64_blend_with_homopolymer(gpu, oracle_lib):
    cfg = W.blend(16, 18.0, 0.35, 0.15, precision="fp64", seed=12, anderson=False)
    w = W.random_fields(cfg, 0.3)
    g, o, hg, ho = run_both(cfg, w, 10)
    assert_parity(cfg, g, o, hg, ho)
    # homopolymer: forward and backward propagators coincide
    assert rel(g.propagator(1, 0, A.PS_FROM_HEAD, 17), o.propagator(1, 0, A.PS_FROM_TAIL, 17)) < TOL64


def test_fp64_anderson_trajectory_parity(gpu, oracle_lib):
    """Anderson mixing, iteration by iteration, on a short well-conditioned
    horizon.  The normal equations come from a Gram matrix whose entries cancel
    (U_ab = G00 - G0a - G0b + Gab), so summation-order differences of the FP64
    dot products (tree on the GPU, sequential in the oracle) are amplified by
    the condition number (observed: 1e-11 in F, 6e-8 relative in
    max|sum phi - 1| after 20 iterations): tolerance 1e-6 here; the converged
    state is compared at 1e-10 below."""
    cfg, w = W.diblock32(n=16)
    cfg.updater = Updater(kind="andersonMixing", relaxlambdas=(0.1, 0.05), anderson_depth=5,
                          anderson_mix=0.1, anderson_start=4)
    g, o, hg, ho = run_both(cfg, w, 20)
    assert_parity(cfg, g, o, hg, ho, tol=1e-6)


def test_fp64_anderson_converged_state_parity(gpu, oracle_lib):
    """Over long horizons the Anderson iteration is chaotic where the history is
    first used (a 1e-13 change of the input moves F by 1e-2 at that step, in
    the oracle alone), so both runs are compared at their common converged
    saddle point: F and Q to 1e-10 and the translation-invariant |FFT(phi)|."""
    cfg, w = W.diblock32(n=16)
    cfg.updater = Updater(kind="andersonMixing", relaxlambdas=(0.1, 0.05), anderson_depth=10,
                          anderson_mix=1.0, anderson_start=100)
    g = ScftSolver(cfg)
    g.restore(w)
    g.update(400)
    sg = g.scalars()
    o = O.Oracle(cfg)
    o.restore(w)
    so = o.update(400)[-1]
    assert sg["dh_norm"] < 1e-9 and so["dh_norm"] < 1e-9
    assert sg["free_energy"] == pytest.approx(so["free_energy"], rel=1e-10)
    assert sg["q"][0] == pytest.approx(so["q"][0], rel=1e-10)
    for i in range(2):
        a = np.abs(np.fft.fftn(g.phi(i).reshape(cfg.n)))
        b = np.abs(np.fft.fftn(o.phi(i).reshape(cfg.n)))
        assert rel(a, b) < 1e-8


def test_fp64_split_plane_path(gpu, oracle_lib):
    """(ny, nz) planes without a fused kernel run as row + y-pencil passes."""
    cfg, _ = W.diblock32(n=8)
    cfg.n = (8, 4, 256)
    cfg.cell = (0.5, 0.5, 0.03125)
    w = W.random_fields(cfg, 0.5)
    g, o, hg, ho = run_both(cfg, w, 4)
    assert_parity(cfg, g, o, hg, ho)


def test_fp64_two_dimensional_grid(gpu, oracle_lib):
    cfg, _ = W.diblock32(n=8)
    cfg.n = (64, 64, 1)
    cfg.cell = (0.1, 0.1, 0.1)
    w = W.random_fields(cfg, 0.5)
    g, o, hg, ho = run_both(cfg, w, 6)
    assert_parity(cfg, g, o, hg, ho)


def test_reference_random_init_and_noise(gpu, oracle_lib):
    cfg, _ = W.diblock32(n=16)
    cfg.updater.noise = 0.002
    g = ScftSolver(cfg)
    g.initialize()
    o = O.Oracle(cfg)
    o.initialize()
    for i in range(2):
        assert np.array_equal(g.w(i), o.w(i))
    ho = o.update(3)
    g.update(3)
    hg = g.scalars()
    assert hg["free_energy"] == pytest.approx(ho[-1]["free_energy"], rel=TOL64)
    for i in range(2):
        assert rel(g.w(i), o.w(i)) < TOL64


@pytest.mark.parametrize("case", ["diblock_sd_fp64", "diblock_am_fp64", "diblock_sd_mixed",
                                  "star_abc_fp64"])
def test_device_noise_follows_the_host_stream(gpu, oracle_lib, case):
    """Updater noise is drawn on the device from the MT19937 stream the host
    generator continues: after noisy iterations (the first eager, the rest
    graph replays) the fields follow the oracle, and a random initialisation
    drawn afterwards is bit-identical, so the device left the stream at exactly
    the oracle's position."""
    if case == "diblock_sd_fp64":
        cfg, _ = W.diblock32(n=16)
        iters, tol = 7, TOL64
    elif case == "diblock_am_fp64":
        # Anderson's Gram entries cancel: 1e-6 as in the noiseless trajectory test
        cfg, _ = W.diblock32(n=16)
        cfg.updater = Updater(kind="andersonMixing", relaxlambdas=(0.1, 0.05), anderson_depth=4,
                              anderson_mix=0.1, anderson_start=2)
        iters, tol = 6, 1e-6
    elif case == "diblock_sd_mixed":
        # FP32 sweeps: the fields follow the FP64 oracle to about 1e-5
        cfg, _ = W.diblock32(n=32, precision="mixed")
        iters, tol = 5, 1e-4
    else:
        cfg, _ = W.star_abc(n=16)
        iters, tol = 4, TOL64
    cfg.updater.noise = 0.01
    g = ScftSolver(cfg)
    o = O.Oracle(cfg)
    g.initialize()
    o.initialize()
    ho = o.update(iters)
    g.update(iters)
    hg = g.scalars()
    assert hg["iteration"] == iters
    assert abs(hg["free_energy"] - ho[-1]["free_energy"]) <= tol * max(abs(ho[-1]["free_energy"]), 1.0)
    for i in range(g.nf):
        assert rel(g.w(i), o.w(i)) < tol
    g.initialize()
    o.initialize()
    for i in range(g.nf):
        assert np.array_equal(g.w(i), o.w(i))
    # and the stream carries on from there on the device
    ho = o.update(2)
    g.update(2)
    for i in range(g.nf):
        assert rel(g.w(i), o.w(i)) < tol


def test_mixed_precision_close_to_fp64_at_convergence(gpu):
    """Mixed (FP32 sweeps) against FP64 at a converged state of a 32^3, Ns = 100
    diblock.  F is stationary in w and phi at the saddle point, but -ln Q enters
    F at first order, and Q from FP32 FFT sweeps carries the round-off of 2 Ns
    transforms: about 1e-6 relative, varying from iteration to iteration (a
    single-precision numpy/pocketfft sweep of the same fields gives 6e-7 over
    100 steps).  That puts a floor of about 5e-6 (absolute) on F: about 1.5e-5
    relative to the disorder-subtracted F of -0.33 here and about 1.5e-6
    relative to the total F (without the disorder subtraction, 3.87 here)."""
    out = {}
    for prec in ("fp64", "mixed"):
        cfg, w = W.diblock32(n=32, precision=prec)
        cfg.updater = Updater(kind="andersonMixing", relaxlambdas=(0.1, 0.05), anderson_depth=10,
                              anderson_mix=1.0, anderson_start=100)
        g = ScftSolver(cfg)
        g.restore(w)
        g.update(300)
        out[prec] = (g.scalars(), [g.phi(i) for i in range(2)])
    s64, phi64 = out["fp64"]
    s32, phi32 = out["mixed"]
    assert s64["dh_norm"] < 1e-6
    dfe = abs(s32["free_energy"] - s64["free_energy"]) / abs(s64["free_energy"])
    dfe_tot = (abs(s32["free_energy_nodis"] - s64["free_energy_nodis"])
               / abs(s64["free_energy_nodis"]))
    dphi = max(np.abs(a - b).max() for a, b in zip(phi32, phi64))
    print(f"mixed vs fp64 at convergence: |dF/F| = {dfe:.3e} (total F: {dfe_tot:.3e}), "
          f"max|dphi| = {dphi:.3e}")
    assert dfe < 1e-4
    assert dfe_tot < 1e-5
    # the lamellae may translate by a fraction of a cell under FP32 noise (a zero
    # mode of the saddle point), so max|dphi| is reported and only sanity-bounded
    assert dphi < 1e-2


def test_kat_uniform_field_gpu(gpu):
    cfg, _ = W.diblock32(n=16)
    g = ScftSolver(cfg)
    c = 0.7
    g.restore([np.full(cfg.n_total, c)] * 2)
    g.update(1)
    s = g.scalars()
    assert s["q"][0] == pytest.approx(math.exp(-c), rel=1e-13)
    for n in (0, 10, 30):
        assert np.allclose(g.propagator(0, 0, A.PS_FROM_HEAD, n), math.exp(-c * 0.01 * n), rtol=1e-13)
    g2 = ScftSolver(cfg)
    g2.restore([np.zeros(cfg.n_total)] * 2)
    g2.update(1)
    assert np.allclose(g2.phi(0), 0.33333 * 0.01 * 90, rtol=1e-13)


def test_kat_q_independent_of_s_gpu(gpu):
    cfg, w = W.diblock32(n=16)
    g = ScftSolver(cfg)
    g.restore(w)
    g.update(1)
    Q = g.scalars()["q"][0]
    for ib, steps in ((0, 30), (1, 70)):
        for n in (0, 9, steps):
            qs = g.propagator(0, ib, A.PS_FROM_HEAD, n)
            qt = g.propagator(0, ib, A.PS_FROM_TAIL, steps - n)
            assert np.mean(qs * qt) == pytest.approx(Q, rel=1e-12)


def test_graph_replay_is_deterministic(gpu):
    """Same variant, same inputs: bitwise the same results, whether the
    iterations come from one graph replay loop or one call each.  (Variants
    differ from each other in rounding, so the autotuned choice is pinned.)"""
    cfg, w = W.diblock32(n=16)
    a, b = ScftSolver(cfg), ScftSolver(cfg)
    a.set_variant(2)
    b.set_variant(2)
    a.restore(w)
    b.restore(w)
    a.update(6)
    for _ in range(6):
        b.update(1)
    assert a.scalars()["free_energy"] == b.scalars()["free_energy"]
    assert np.array_equal(a.w(0), b.w(0))


def test_errors_are_status_codes(gpu):
    cfg, w = W.diblock32(n=8)
    g = ScftSolver(cfg)
    bad = w[0].copy()
    bad[5] = np.nan
    g.restore([bad, w[1]])
    with pytest.raises(A.PsError) as e:
        g.update(1)
    assert e.value.code == A.PS_RUN_ERR
    cfg2, _ = W.diblock32(n=8)
    cfg2.n = (10, 10, 10)
    with pytest.raises(A.PsError) as e:
        ScftSolver(cfg2)
    assert e.value.code == A.PS_INPUT_ERR
    cfg3, _ = W.diblock32(n=8)
    cfg3.polymers[0].blocks[0].ds = 0.013
    cfg3.polymers[0].blocks[1].ds = 0.013
    with pytest.raises(A.PsError) as e:
        ScftSolver(cfg3)
    assert e.value.code == A.PS_INPUT_ERR


def test_precision_switch_carries_state(gpu):
    """Switching the sweeps from FP32 to FP64 between iterations keeps w, p and
    phi: with steepest descent (no history) the switched handle then runs
    exactly like an FP64 handle restored from the same fields."""
    cfg, w = W.diblock32(n=16, precision="mixed")
    g = ScftSolver(cfg)
    g.set_variant(0)
    g.restore(w)
    g.update(3)
    w3 = [g.w(0), g.w(1)]
    p3 = g.pressure()
    g.set_precision("fp64")
    g.set_variant(0)
    g.update(4)
    cfg64, _ = W.diblock32(n=16, precision="fp64")
    f = ScftSolver(cfg64)
    f.set_variant(0)
    f.restore(w3, p3)
    f.update(4)
    for i in range(2):
        assert np.array_equal(g.w(i), f.w(i))
        assert np.array_equal(g.phi(i), f.phi(i))
    assert g.scalars()["free_energy"] == f.scalars()["free_energy"]
    assert g.scalars()["iteration"] == 7
    g.set_precision("mixed")  # back again: buffers are kept, the run continues
    g.update(2)
    assert np.isfinite(g.scalars()["free_energy"])


def test_precision_escalation_meets_fp64(gpu):
    """Anderson run mostly in mixed precision, last 20 iterations in FP64 (the
    history carries over): F lands within 1e-7 of the all-FP64 run, below the
    FP32 noise floor of the mixed-only run."""
    iters, finish = 300, 20
    out = {}
    for mode in ("fp64", "escalated"):
        cfg, w = W.diblock32(n=32, precision="fp64" if mode == "fp64" else "mixed")
        cfg.updater = Updater(kind="andersonMixing", relaxlambdas=(0.1, 0.05), anderson_depth=10,
                              anderson_mix=1.0, anderson_start=100)
        g = ScftSolver(cfg)
        g.restore(w)
        if mode == "fp64":
            g.update(iters)
        else:
            g.update(iters - finish)
            g.set_precision("fp64")
            g.update(finish)
        out[mode] = g.scalars()
        g.close()
    a, b = out["fp64"], out["escalated"]
    assert a["iteration"] == b["iteration"] == iters
    assert abs(b["free_energy"] - a["free_energy"]) < 1e-7 * abs(a["free_energy"])
    assert abs(b["free_energy_nodis"] - a["free_energy_nodis"]) < 1e-7 * abs(a["free_energy_nodis"])


@pytest.mark.parametrize("variant", [0, 1, 2, 3, 9, 11])
def test_128_square_plane_variants_match_oracle(gpu, oracle_lib, variant):
    """8 x 128 x 128 grid: the 128 x 128 y-z plane kernel, whose z passes fold the
    real-transform pre/post-processing into the first/last pass and (bit 0) fuse
    the real-space step into the middle pass; FP64 against the oracle at 1e-10."""
    import dataclasses
    cfg, _ = W.diblock32(n=16)
    cfg = dataclasses.replace(cfg, n=(8, 128, 128), cell=(0.5, 4.0 / 128, 4.0 / 128))
    _, y, z = W.coords(cfg)
    w = W.random_fields(cfg, 0.2)
    c = (np.cos(2 * math.pi * z / cfg.box[2]) * np.cos(2 * math.pi * y / cfg.box[1])).reshape(-1)
    w = [w[0] + c, w[1] - c]
    g = ScftSolver(cfg)
    g.set_variant(variant)
    g.restore(w)
    o = O.Oracle(cfg)
    o.restore(w)
    ho = o.update(3)
    hg = []
    for _ in range(3):
        g.update(1)
        hg.append(g.scalars())
    assert_parity(cfg, g, o, hg, ho)


@pytest.mark.parametrize("variant", [0, 11])
def test_fp64_solvent_blend_parity(gpu, oracle_lib, variant):
    """Diblock + simpleSolvent on the A field (pssolvent/PsSimpleSolvent.cpp:86-140):
    the solvent's Q and density on the device, and its -vf L ln Q term in F, against the
    oracle at 1e-10."""
    import dataclasses
    from polyswift_plusplus_b200.config import Solvent
    cfg, w = W.diblock32(n=16)
    cfg.polymers[0].volfrac = 0.8
    cfg = dataclasses.replace(cfg, solvents=[Solvent("solv", "A", 0.2)])
    g = ScftSolver(cfg)
    g.set_variant(variant)
    g.restore(w)
    o = O.Oracle(cfg)
    o.restore(w)
    ho = o.update(8)
    hg = []
    for _ in range(8):
        g.update(1)
        hg.append(g.scalars())
    assert_parity(cfg, g, o, hg, ho)


def test_mixed_solvent_blend_close_to_fp64(gpu):
    import dataclasses
    from polyswift_plusplus_b200.config import Solvent
    out = []
    for prec in ("fp64", "mixed"):
        cfg, w = W.diblock32(n=16, precision=prec)
        cfg.polymers[0].volfrac = 0.8
        cfg = dataclasses.replace(cfg, solvents=[Solvent("solv", "B", 0.2)])
        g = ScftSolver(cfg)
        g.restore(w)
        g.update(20)
        out.append(g.scalars()["free_energy"])
    assert abs(out[1] - out[0]) < 1e-5 * max(abs(out[0]), 1.0)


def test_dump_restore_continues_a_run_exactly(gpu, tmp_path):
    """Steepest descent (no history): 5 iterations, dump, restore into a fresh solver,
    5 more, equals 10 uninterrupted iterations bit for bit."""
    from polyswift_plusplus_b200.dump import dump, restore
    cfg, w = W.diblock32(n=16)
    a = ScftSolver(cfg)
    a.set_variant(0)
    a.restore(w)
    a.update(5)
    dump(a, tmp_path / "ck.npz", history=[a.scalars()["free_energy"]])
    a.update(5)
    b = ScftSolver(cfg)
    b.set_variant(0)
    meta = restore(b, tmp_path / "ck.npz")
    assert meta["iteration"] == 5
    b.update(5)
    for i in range(2):
        assert np.array_equal(a.w(i), b.w(i))
        assert np.array_equal(a.phi(i), b.phi(i))
    assert a.scalars()["free_energy"] == b.scalars()["free_energy"]


def _spec_filter(fields, cutoff, strength, start=0, freq=1, end=-1):
    from polyswift_plusplus_b200.config import SpecFilter
    return SpecFilter(updatefields=list(fields), cutoff_factor=cutoff, filter_strength=strength,
                      apply_start=start, apply_frequency=freq, apply_end=end)


@pytest.mark.parametrize("shape", [(16, 16, 16), (32, 32, 32), (8, 4, 256), (64, 64, 1),
                                   (24, 48, 48), (128, 128, 128)])
def test_spectral_filter_matches_oracle(gpu, oracle_lib, shape):
    """simpleSpecFilter on the device (fused plane and split-plane FFT paths, a 2-D grid)
    against the oracle: w after one application at 1e-12 of max|w|."""
    cfg, _ = W.diblock32(n=8)
    cfg.n = shape
    rng = np.random.default_rng(11)
    w = [rng.standard_normal(cfg.n_total) + 0.3, rng.standard_normal(cfg.n_total) - 0.2]
    f = _spec_filter(["B", "A"], 0.25, 0.1)
    g = ScftSolver(cfg)
    g.restore(w)
    g.set_spectral_filter(f)
    g.apply_spectral_filter()
    o = O.Oracle(cfg)
    o.restore(w)
    o.set_spectral_filter(f)
    o.apply_spectral_filter()
    for i in range(2):
        assert rel(g.w(i), o.w(i)) < 1e-12
        assert abs(g.w(i).mean()) < 1e-12


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_spectral_filter_scheduled_in_iterations(gpu, oracle_lib, precision):
    """The filter runs after the field update of the scheduled steps (PsUpdater::update);
    FP64 sweeps: parity with the oracle at 1e-10 over the run; mixed sweeps: the filter
    itself stays FP64 and F tracks the FP64 run."""
    import dataclasses
    cfg, w = W.diblock32(n=16, precision=precision)
    cfg = dataclasses.replace(cfg, spec_filter=_spec_filter(["A", "B"], 0.02, 0.5, start=1, freq=2, end=9))
    g = ScftSolver(cfg)
    g.restore(w)
    if precision == "fp64":
        cfgo = dataclasses.replace(cfg, precision="fp64")
        o = O.Oracle(cfgo)
        o.restore(w)
        ho = o.update(12)
        hg = []
        for _ in range(12):
            g.update(1)
            hg.append(g.scalars())
        assert_parity(cfg, g, o, hg, ho)
    else:
        g.update(12)
        c64, _ = W.diblock32(n=16)
        c64 = dataclasses.replace(c64, spec_filter=cfg.spec_filter)
        g64 = ScftSolver(c64)
        g64.restore(w)
        g64.update(12)
        f32, f64 = g.scalars()["free_energy"], g64.scalars()["free_energy"]
        assert abs(f32 - f64) < 1e-5 * max(abs(f64), 1.0)


def test_spectral_filter_errors(gpu):
    cfg, w = W.diblock32(n=16)
    g = ScftSolver(cfg)
    g.restore(w)
    with pytest.raises(A.PsError):
        g.apply_spectral_filter()            # none installed
    with pytest.raises(A.PsError):
        g.set_spectral_filter(_spec_filter(["A"], 0.1, 0.0, start=5, end=5))
    with pytest.raises(A.PsError):
        g.set_spectral_filter(_spec_filter(["A"], 0.1, 0.0, start=0, freq=10, end=10))
    g.set_spectral_filter(_spec_filter(["A"], 0.1, 0.0))
    g.set_spectral_filter(None)              # removed again
    g.update(2)
    assert math.isfinite(g.scalars()["free_energy"])


@pytest.mark.parametrize("shape,cells", [((16, 16, 16), (4, 4, 1)), ((32, 32, 32), (8, 8, 8)),
                                         ((24, 48, 48), (4, 8, 6)), ((64, 64, 1), (8, 4, 1)),
                                         ((8, 4, 256), (2, 2, 16)), ((128, 128, 128), (4, 4, 1))])
def test_multi_spectral_filter_matches_oracle(gpu, oracle_lib, shape, cells):
    """multiSpecFilter: the per-region cutoff and the serial (y, x, z) region map on the
    half spectrum (symmetrised mask) against the oracle's full complex spectrum, 1e-12.
    (128, 128, 128) with 4x4x1 cells has 131072 regions (global atomics); the others
    reduce in shared memory first."""
    cfg, _ = W.diblock32(n=8)
    cfg.n = shape
    rng = np.random.default_rng(17)
    w = [rng.standard_normal(cfg.n_total), rng.standard_normal(cfg.n_total) + 0.5]
    f = _spec_filter(["A", "B"], 0.6, 0.05)
    f.spec_cells = cells
    g = ScftSolver(cfg)
    g.restore(w)
    g.set_spectral_filter(f)
    g.apply_spectral_filter()
    o = O.Oracle(cfg)
    o.restore(w)
    o.set_spectral_filter(f)
    o.apply_spectral_filter()
    for i in range(2):
        assert rel(g.w(i), o.w(i)) < 1e-12


def test_multi_spectral_filter_scheduled_parity(gpu, oracle_lib):
    import dataclasses
    cfg, w = W.diblock32(n=16)
    f = _spec_filter(["A", "B"], 0.3, 0.0, start=2, freq=3, end=11)
    f.spec_cells = (4, 4, 1)
    cfg = dataclasses.replace(cfg, spec_filter=f)
    g, o, hg, ho = run_both(cfg, w, 12)
    assert_parity(cfg, g, o, hg, ho)


# ---------------------------------------------------------------------------
# Charged systems

def _charged_both(n, every=2, precision="fp64"):
    cfg, w, psi = W.charged_diblock(n=n, poisson_every=every, precision=precision)
    g = ScftSolver(cfg)
    g.restore(w)
    g.set_field(A.PS_FIELD_POTENTIAL, 0, psi)
    import dataclasses
    o = O.Oracle(dataclasses.replace(cfg, precision="fp64"))
    o.restore(w)
    o.set_field(A.PS_FIELD_POTENTIAL, 0, psi)
    return cfg, g, o


@pytest.mark.parametrize("n", [(16, 16, 16), (32, 32, 32), (16, 12, 1), (8, 4, 256)])
def test_fp64_charged_diblock_parity(gpu, oracle_lib, n):
    """chargeFlexPseudoSpec block, simpleIons counter-ions and the Poisson updater every
    2 steps on the device against the oracle: F, Q, w, phi at 1e-10; rho and psi at 1e-10
    of their magnitude."""
    cfg, g, o = _charged_both(n)
    ho = o.update(7)
    hg = []
    for _ in range(7):
        g.update(1)
        hg.append(g.scalars())
    assert_parity(cfg, g, o, hg, ho)
    for c in range(2):
        assert rel(g.rho(c), o.rho(c)) < TOL64
        assert np.abs(g.psi(c) - o.psi(c)).max() <= TOL64 * max(np.abs(o.psi(c)).max(), 1e-300)


def test_fp64_charged_diblock_on_cluster_plane_pass(gpu, oracle_lib):
    """The charged diblock (charged Boltzmann factors, counter-ions, the Poisson updater every
    2 steps) on an 8 x 256 x 256 grid with the cluster plane pass forced (variant 24), against
    the oracle at 1e-10 over 4 iterations.  On this grid the Poisson clamp shrinks psi to about
    1e-8, so psi is checked at 1e-10 of the seeded potential's magnitude."""
    cfg, g, o = _charged_both((8, 256, 256))
    _, _, psi0 = W.charged_diblock(n=(8, 256, 256), poisson_every=2)
    g.set_variant(24)
    ho = o.update(4)
    hg = []
    for _ in range(4):
        g.update(1)
        hg.append(g.scalars())
    assert g.variant()[0] == 24
    assert_parity(cfg, g, o, hg, ho)
    for c in range(2):
        assert rel(g.rho(c), o.rho(c)) < TOL64
        scale = max(np.abs(o.psi(c)).max(), np.abs(psi0).max())
        assert np.abs(g.psi(c) - o.psi(c)).max() <= TOL64 * scale


def test_poisson_single_apply_matches_oracle(gpu, oracle_lib):
    """One Poisson application on a random charge density with the old potential near the
    answer (no clamping) and far from it (clamping), device vs oracle at 1e-12."""
    from polyswift_plusplus_b200.config import PoissonUpdater
    cfg, w, _ = W.charged_diblock(n=(32, 32, 32))
    cfg.poisson = None
    rng = np.random.default_rng(4)
    rho = rng.standard_normal(cfg.n_total) + 0.2
    pu = PoissonUpdater(updatefields=["charge"], bjerrum_len=3.0)
    o = O.Oracle(cfg)
    o.set_field(A.PS_FIELD_CHARGE, 0, rho)
    o.set_poisson(pu)
    o.apply_poisson()
    exact = o.psi(0)  # psi = 0 before: every changed point clamps to 0
    assert not np.any(exact)
    for psi0 in (1.05 * rng.standard_normal(cfg.n_total), None):
        o.set_field(A.PS_FIELD_CHARGE, 0, rho)
        g = ScftSolver(cfg)
        g.set_field(A.PS_FIELD_CHARGE, 0, rho)
        if psi0 is None:  # start near the answer: take the unclamped result as the old potential
            from oracle.np_scft import coulomb_operator
            r = (rho - rho.mean()).reshape(cfg.n)
            psi0 = 1.1 * np.fft.ifftn(np.fft.fftn(r) * coulomb_operator(cfg, 3.0)).real.reshape(-1)
        o.set_field(A.PS_FIELD_POTENTIAL, 0, psi0)
        g.set_field(A.PS_FIELD_POTENTIAL, 0, psi0)
        g.set_poisson(pu)
        g.apply_poisson()
        o.apply_poisson()
        assert rel(g.psi(0), o.psi(0)) < 1e-12
        assert rel(g.rho(0), o.rho(0)) < 1e-12


def test_mixed_charged_diblock_close_to_fp64(gpu):
    out = []
    for prec in ("fp64", "mixed"):
        cfg, g, _ = _charged_both((16, 16, 16), precision=prec)
        g.update(12)
        out.append(g.scalars()["free_energy"])
    assert abs(out[1] - out[0]) < 1e-5 * max(abs(out[0]), 1.0)


def test_charged_errors(gpu):
    import dataclasses
    from polyswift_plusplus_b200.config import PoissonUpdater, Solvent
    cfg, _, _ = W.charged_diblock(n=(16, 16, 16))
    cfg.polymers[0].volfrac = 0.9
    bad = dataclasses.replace(cfg, solvents=cfg.solvents + [Solvent("s", "A", 0.1)])
    with pytest.raises(A.PsError):
        ScftSolver(bad)
    cfg, _, _ = W.charged_diblock(n=(16, 16, 16))
    g = ScftSolver(cfg)
    with pytest.raises(A.PsError):
        g.set_poisson(PoissonUpdater(updatefields=["charge"], apply_start=4, apply_end=4))
    g.set_poisson(None)
    with pytest.raises(A.PsError):
        g.apply_poisson()
    with pytest.raises(ValueError):
        g.set_poisson(PoissonUpdater(updatefields=["nope"]))
    with pytest.raises(A.PsError):
        g.get_field(A.PS_FIELD_POTENTIAL, 2)


# ---------------------------------------------------------------------------
# polyDisperseBCP

@pytest.mark.parametrize("n", [(16, 16, 16), (16, 12, 1), (8, 4, 256)])
def test_fp64_polydisperse_parity(gpu, oracle_lib, n):
    """n_g = 4 quadrature chains on the device (the library's Golub-Welsch nodes) against
    the oracle (its own root-bracketing nodes, per-block Q): 1e-10; block steps and
    propagators indexed the reference's way (seed-major quadrature blocks)."""
    cfg, w = W.polydisperse_diblock(n=n)
    g, o, hg, ho = run_both(cfg, w, 6)
    assert_parity(cfg, g, o, hg, ho)
    for b in range(8):
        assert g.block_steps(0, b) == o.block_steps(0, b)
    for b in (0, 3, 5, 7):
        steps = o.block_steps(0, b)
        for end in (A.PS_FROM_HEAD, A.PS_FROM_TAIL):
            for s in (0, steps // 2, steps):
                assert rel(g.propagator(0, b, end, s), o.propagator(0, b, end, s)) < TOL64


def test_mixed_polydisperse_close_to_fp64(gpu):
    out = []
    for prec in ("fp64", "mixed"):
        cfg, w = W.polydisperse_diblock(n=(16, 16, 16), precision=prec)
        g = ScftSolver(cfg)
        g.restore(w)
        g.update(15)
        out.append(g.scalars()["free_energy"])
    assert abs(out[1] - out[0]) < 1e-5 * max(abs(out[0]), 1.0)


def test_polydisperse_blend_with_homopolymer(gpu, oracle_lib):
    """A polydisperse diblock (n_g 3) blended with an A homopolymer: chains of both
    polymers in one graph, F and fields at 1e-10."""
    import dataclasses
    from polyswift_plusplus_b200.config import Block, Polymer
    cfg, w = W.polydisperse_diblock(n=(16, 16, 16), n_g=3)
    pd = dataclasses.replace(cfg.polymers[0], volfrac=0.85)
    homo = Polymer(name="homoA", volfrac=0.15, length=50,
                   blocks=[Block(name="hA", scfield="A", ds=0.02, lengthfrac=1.0)])
    cfg = dataclasses.replace(cfg, polymers=[pd, homo])
    g, o, hg, ho = run_both(cfg, w, 5)
    assert_parity(cfg, g, o, hg, ho)


@pytest.mark.parametrize("axis", [0, 2])
def test_kat7_debye_response_gpu(gpu, axis):
    """The device's weak-segregation response against the Debye functions (see the
    oracle's KAT7), FP64: 1e-4."""
    import sys
    sys.path.insert(0, str(Path(__file__).resolve().parent))
    from test_oracle import mode_amplitude, rpa_case
    cfg, w, k, eps, (gaa, gab) = rpa_case(axis)
    g = ScftSolver(cfg)
    g.restore(w)
    g.update(1)
    assert mode_amplitude(g.phi(0), cfg, axis) == pytest.approx(-eps * gaa, rel=1e-4)
    assert mode_amplitude(g.phi(1), cfg, axis) == pytest.approx(-eps * gab, rel=1e-4)


# ---------------------------------------------------------------------------
# Branched polymers

def _tree_h(n=16):
    """Two junctions: arms A, B and the backbone C meet at one, C, D, E at the other."""
    ds = 0.01
    blocks = [Block("a", "A", ds, 0.15, ["freeEnd"], ["b", "c"]),
              Block("b", "B", ds, 0.15, ["freeEnd"], ["a", "c"]),
              Block("c", "C", ds, 0.40, ["a", "b"], ["d", "e"]),
              Block("d", "A", ds, 0.15, ["freeEnd"], ["c", "e"]),
              Block("e", "B", ds, 0.15, ["freeEnd"], ["c", "d"])]
    cfg = ScftConfig(n=(n, n, n), cell=(0.2,) * 3, fields=["A", "B", "C"],
                     polymers=[Polymer("h", 1.0, 100, blocks)],
                     interactions=[Interaction("AB", 0.12, ["A", "B"]), Interaction("BC", 0.12, ["B", "C"]),
                                   Interaction("AC", 0.15, ["A", "C"])],
                     updater=Updater(relaxlambdas=(0.05, 0.025)), seed=77)
    return cfg, W.random_fields(cfg, 0.2)


def _star4(n=16):
    from polyswift_plusplus_b200.workloads import star
    cfg = ScftConfig(n=(n, n, n), cell=(0.2,) * 3, fields=["A", "B", "C"],
                     polymers=[star((0.2, 0.3, 0.25, 0.25), fields=("A", "B", "C", "A"))],
                     interactions=[Interaction("AB", 0.15, ["A", "B"]), Interaction("BC", 0.15, ["B", "C"]),
                                   Interaction("AC", 0.15, ["A", "C"])],
                     updater=Updater(relaxlambdas=(0.05, 0.025)), seed=78)
    return cfg, W.random_fields(cfg, 0.2)


@pytest.mark.parametrize("variant", [16, 24])
def test_fp64_branched_polymer_on_cluster_plane_pass(gpu, oracle_lib, variant):
    """A three-arm star on an 8 x 256 x 256 grid with the cluster plane pass (lockstep sweeps
    with junction launches, variant 16, and dependent launch chains, variant 24) against the
    oracle at 1e-10, block propagators from both ends included."""
    cfg, _ = W.star_abc(n=16)
    cfg.n, cfg.cell = (8, 256, 256), (0.4, 0.0125, 0.0125)
    w = W.random_fields(cfg, 0.2)
    g = ScftSolver(cfg)
    g.set_variant(variant)
    g.restore(w)
    o = O.Oracle(cfg)
    o.restore(w)
    ho = o.update(2)
    hg = []
    for _ in range(2):
        g.update(1)
        hg.append(g.scalars())
    assert g.variant()[0] == variant
    assert_parity(cfg, g, o, hg, ho)
    for b in range(3):
        steps = o.block_steps(0, b)
        for end in (A.PS_FROM_HEAD, A.PS_FROM_TAIL):
            assert rel(g.propagator(0, b, end, steps), o.propagator(0, b, end, steps)) < TOL64
    g.close()


@pytest.mark.parametrize("case", ["star3", "star3_split_plane", "star4", "tree_h"])
def test_fp64_branched_polymer_parity(gpu, oracle_lib, case):
    """Branched polymers (PsBlockCopolymer's dependency-driven solve order) on the device:
    sweeps from free ends, junction products, sweeps from junctions, against the oracle's
    general block scheduler at 1e-10, with every block's propagators from both ends."""
    if case.startswith("star3"):
        cfg, w = W.star_abc(n=16)
        if case == "star3_split_plane":
            cfg.n, cfg.cell = (8, 4, 256), (0.4, 0.4, 0.0125)
            w = W.random_fields(cfg, 0.2)
    elif case == "star4":
        cfg, w = _star4()
    else:
        cfg, w = _tree_h()
    g, o, hg, ho = run_both(cfg, w, 6)
    assert_parity(cfg, g, o, hg, ho)
    for b in range(len(cfg.polymers[0].blocks)):
        steps = o.block_steps(0, b)
        assert g.block_steps(0, b) == steps
        for end in (A.PS_FROM_HEAD, A.PS_FROM_TAIL):
            for s in (0, steps):
                assert rel(g.propagator(0, b, end, s), o.propagator(0, b, end, s)) < TOL64


def test_kat7_star_debye_response_gpu(gpu):
    """The star's weak-segregation response on the device (see the oracle's KAT7)."""
    import sys
    sys.path.insert(0, str(Path(__file__).resolve().parent))
    from test_oracle import debye, mode_amplitude
    fr = (0.3, 0.3, 0.4)
    cfg = ScftConfig(n=(32, 4, 4), cell=(4.0 / 32, 0.1, 0.1), fields=["A", "B", "C"],
                     polymers=[W.star(fr)], interactions=[Interaction("AB", 0.15, ["A", "B"])],
                     updater=Updater(relaxlambdas=(0.05, 0.025)))
    x = W.coords(cfg)[0]
    k = 2 * math.pi / cfg.box[0]
    eps = 1e-4
    wa = (eps * np.cos(k * x)).reshape(-1)
    g = ScftSolver(cfg)
    g.restore([wa, np.zeros_like(wa), np.zeros_like(wa)])
    g.update(1)
    kk = k * k
    want = [debye(fr[0], kk)] + [0.5 * (debye(fr[0] + f, kk) - debye(fr[0], kk) - debye(f, kk)) for f in fr[1:]]
    for i in range(3):
        assert mode_amplitude(g.phi(i), cfg, 0) == pytest.approx(-eps * want[i], rel=1e-4)


@pytest.mark.parametrize("case", ["star3", "star4", "tree_h"])
@pytest.mark.parametrize("variant", [0, 3, 11])
def test_branched_polymer_every_variant(gpu, oracle_lib, case, variant):
    """Branched sweeps in shared (lockstep) launches, each leaving-junction sweep
    offset to start one step after the last arriving sweep with its junction
    product launched in between (variants 0, 3), and as dependent launch chains
    (variant 11), all against the oracle at 1e-10."""
    cfg, w = {"star3": lambda: W.star_abc(n=16), "star4": _star4, "tree_h": _tree_h}[case]()
    g = ScftSolver(cfg)
    g.set_variant(variant)
    g.restore(w)
    o = O.Oracle(cfg)
    o.restore(w)
    ho = o.update(5)
    hg = []
    for _ in range(5):
        g.update(1)
        hg.append(g.scalars())
    assert_parity(cfg, g, o, hg, ho)


def test_branched_polymer_mixed(gpu):
    """Mixed-precision star within 1e-5 of FP64."""
    out = []
    for prec in ("fp64", "mixed"):
        cfg, w = W.star_abc(n=16, precision=prec)
        g = ScftSolver(cfg)
        g.restore(w)
        g.update(10)
        out.append(g.scalars()["free_energy"])
    assert abs(out[1] - out[0]) < 1e-5 * max(abs(out[0]), 1.0)


@pytest.mark.parametrize("variant", [0, 3])
def test_branched_polymers_in_a_batch(gpu, variant):
    """Stars and a two-junction tree batched with a diblock blend of the same grid:
    each instance bit-identical to its single run with the same variant."""
    from polyswift_plusplus_b200.scft import ScftBatch
    items = [W.star_abc(n=16), _star4(), _tree_h(), W.star_abc(n=16, precision="mixed")]
    cfg_b = W.blend(16, 15.0, 0.3, 0.1, precision="fp64", seed=5)
    items.append((cfg_b, W.random_fields(cfg_b, 0.1)))
    with ScftBatch([c for c, _ in items]) as b:
        b.set_variant(variant)
        for i, (_, w) in enumerate(items):
            b.instance(i).restore(w)
        b.update(4)
        for i, (cfg, w) in enumerate(items):
            s = ScftSolver(cfg)
            s.set_variant(variant)
            s.restore(w)
            s.update(4)
            v = b.instance(i)
            assert v.scalars()["free_energy"] == s.scalars()["free_energy"]
            for f in range(len(cfg.fields)):
                assert np.array_equal(v.phi(f), s.phi(f))
                assert np.array_equal(v.w(f), s.w(f))
            s.close()


def test_async_field_readback_matches_blocking_read(gpu):
    """ps_gpu_get_fields_async: the snapshot taken at the call reaches the host
    buffer by ps_gpu_fields_wait, while later iterations run; a second read of
    the same field into another buffer waits for the first copy."""
    import torch
    cfg, w = W.diblock32(n=32)
    g = ScftSolver(cfg)
    g.restore(w)
    g.update(2)
    N = cfg.n_total
    bufs = [torch.empty(N, dtype=torch.float64).pin_memory() for _ in range(4)]
    g.get_field_async(A.PS_FIELD_W, 0, bufs[0])
    g.get_field_async(A.PS_FIELD_PHI, 1, bufs[1])
    w0, phi1 = g.w(0), g.phi(1)
    g.update(1)  # runs while the copies may still be in flight
    g.get_field_async(A.PS_FIELD_W, 0, bufs[2])
    host_p = np.empty(N)
    g.get_field_async(A.PS_FIELD_PRES, 0, host_p)  # pageable numpy memory also works
    g.fields_wait()
    assert np.array_equal(bufs[0].numpy(), w0)
    assert np.array_equal(bufs[1].numpy(), phi1)
    assert np.array_equal(bufs[2].numpy(), g.w(0))
    assert not np.array_equal(bufs[2].numpy(), w0)
    assert np.array_equal(host_p, g.pressure())
    with pytest.raises(A.PsError):
        g.get_field_async(A.PS_FIELD_W, 7, bufs[3])
    g.close()


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_async_field_upload_matches_blocking_upload(gpu, prec):
    """ps_gpu_set_fields_async: iterations fed by asynchronous uploads (w on the handle
    stream, p on the upload stream with the field update waiting for it inside the captured
    graph) are bit-identical to iterations fed by blocking uploads, step by step, with new
    host values every step; a blocking read of p right after its asynchronous upload sees
    the uploaded values."""
    import torch
    cfg, w = W.diblock32(n=32, precision=prec)
    N = cfg.n_total
    rng = np.random.default_rng(41)
    steps = [([w[0] + 0.01 * rng.standard_normal(N), w[1] + 0.01 * rng.standard_normal(N)],
              0.05 * rng.standard_normal(N)) for _ in range(4)]
    runs = []
    for mode in ("blocking", "async"):
        g = ScftSolver(cfg)
        g.restore(w)
        g.update(3)  # eager iterations, then the captured graph
        host_w = [torch.empty(N, dtype=torch.float64).pin_memory() for _ in range(2)]
        host_p = torch.empty(N, dtype=torch.float64).pin_memory()
        hist = []
        for ws, p in steps:
            for i in range(2):
                host_w[i].copy_(torch.from_numpy(ws[i]))
            host_p.copy_(torch.from_numpy(p))
            if mode == "blocking":
                for i in range(2):
                    g.set_field(A.PS_FIELD_W, i, host_w[i])
                g.set_field(A.PS_FIELD_PRES, 0, host_p)
            else:
                for i in range(2):
                    g.set_field_async(A.PS_FIELD_W, i, host_w[i])
                g.set_field_async(A.PS_FIELD_PRES, 0, host_p)
            g.update(1)
            hist.append(g.scalars())  # the host buffers are free again after this
        runs.append((hist, [g.w(i) for i in range(2)], g.pressure()))
        if mode == "async":
            q = np.arange(N, dtype=np.float64)
            g.set_field_async(A.PS_FIELD_PRES, 0, q)
            assert np.array_equal(g.pressure(), q)
            qd = torch.full((N,), 0.25, dtype=torch.float64, device="cuda")  # a device source
            g.set_field_async(A.PS_FIELD_W, 1, qd)
            g.set_field_async(A.PS_FIELD_PRES, 0, qd)
            g.fields_wait()
            assert np.array_equal(g.w(1), qd.cpu().numpy()) and np.array_equal(g.pressure(), qd.cpu().numpy())
        g.close()
    (ha, wa, pa), (hb, wb, pb) = runs
    for a, b in zip(ha, hb):
        assert a["free_energy"] == b["free_energy"] and a["q"][0] == b["q"][0]
    for i in range(2):
        assert np.array_equal(wa[i], wb[i])
    assert np.array_equal(pa, pb)
