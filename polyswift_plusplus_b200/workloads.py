"""Named SCFT workloads and their seeded initial fields.

Each workload is a synthetic input with the shapes, sizes and parameters of
one benchmark configuration (there is no public dataset for this path).
Initial fields are drawn from MT19937 (``init_genrand(seed)``, ``real() =
u32 / 2^32``: the reference's PsRandom conventions) field by field, point by
point in row-major order, plus the deterministic seeds described per workload.

* ``diblock32``   32^3, box 4.0 Rg, f_A 0.30, chiN 20, Ns 100, steepest descent
                  lambda = (0.1, 0.05); w = U(-0.1, 0.1) +/- cos(2 pi x / L).
* ``diblock128``  128^3, box 8.0 Rg, f_A 0.35, chiN 25, Ns 200, Anderson depth 10
                  (mixing 0.5 after 100 steepest-descent steps, which let the melt order
                  first; started earlier the history pulls it to the disordered saddle);
                  w = U(-0.05, 0.05) +/- hexagonal seed (three cosines with integer
                  wave vectors (2,0), (-1,2), (-1,-2) x 2 pi / L in the x-y plane:
                  the periodic box's nearest match to 120 degrees).
* ``diblock64_adjoint`` 64^3, box 6.0 Rg, f_A 0.40, chiN 18, Ns 128 (forceBlockSteps:
                  51 + 77 steps), FP64; lamellar start cos(2 pi z / L) + U(-0.1, 0.1).
* ``triblock256`` 256^3, box 16 Rg, ABC (0.3, 0.4, 0.3), chiN AB 30, BC 30, AC 45,
                  Ns 400, Anderson depth 20, mixed precision; w = U(-0.05, 0.05).
* ``blend_batch`` 64 diblock / A-homopolymer blend instances (see ``blend_instances``).
* ``polydisperse_diblock`` the polydisperse example's model: A block (f 0.7, ds 0.02) and
                  a Schulz-distributed B block (average f 0.3, ds 0.01, alpha 1.5, n_g 4
                  Gauss-Laguerre points, forceBlockSteps), length 100, chiN 12 (the example
                  ramps chi with an STFunc; a constant chi stands in), steepest descent
                  lambda (0.2, 0.1); w = U(-0.1, 0.1) +/- cos(2 pi x / L).
* ``star_abc``    a three-arm ABC star (the reference's star example: every arm's head free,
                  the tails joined at one junction), chiN 15 for each pair, ds 0.01;
                  w = U(-0.2, 0.2).
* ``charged_diblock`` the charged-diblock test deck's model (chargeFlexPseudoSpec A block,
                  za 1, alpha 0.01, length 1000, f_A 0.5, ds 0.05, chi = 1/(20 (3.1415) 1.4),
                  bjerrumLen = 1/(4 (3.1415) 0.01 1.4), simpleIons counter-ions zc -1 with
                  neutralFactor za alpha f_A, a poissonUpdater every 5 steps), on a chosen
                  grid; w = U(-0.1, 0.1) +/- cos(2 pi x / L), and a small seeded potential
                  psi (the reference starts from psi = 0, which its Poisson clamp keeps at 0).
"""
from __future__ import annotations

import math

import numpy as np

from .config import Block, Interaction, Polymer, ScftConfig, Updater


def mt_reals(seed: int, n: int) -> np.ndarray:
    """n draws of PsRandom::real() from MT19937 init_genrand(seed)."""
    bg = np.random.MT19937(0)
    bg._legacy_seeding(int(seed) & 0xFFFFFFFF)
    return bg.random_raw(n).astype(np.float64) * (1.0 / 4294967296.0)


def diblock(name_a="A", name_b="B", f_a=0.5, ds=0.01, length=100, volfrac=1.0,
            force=False, pname="diblock") -> Polymer:
    return Polymer(name=pname, volfrac=volfrac, length=length, blocks=[
        Block(name=pname + "_A", scfield=name_a, ds=ds, lengthfrac=f_a,
              headjoined=["freeEnd"], tailjoined=[pname + "_B"], force_block_steps=force),
        Block(name=pname + "_B", scfield=name_b, ds=ds, lengthfrac=1.0 - f_a,
              headjoined=[pname + "_A"], tailjoined=["freeEnd"], force_block_steps=force),
    ])


def diblock_config(n, box, f_a, chin, ns, updater: Updater, precision="fp64", seed=38383,
                   length=100, force=False) -> ScftConfig:
    ds = 1.0 / ns
    return ScftConfig(
        n=(n, n, n), cell=(box / n, box / n, box / n), fields=["A", "B"],
        polymers=[diblock(f_a=f_a, ds=ds, length=length, force=force)],
        interactions=[Interaction(name="AB", chi=chin / length, scfields=["A", "B"])],
        updater=updater, seed=seed, precision=precision)


def coords(cfg: ScftConfig):
    """Cell coordinates (x, y, z) as 3D arrays (x slowest)."""
    axes = [np.arange(cfg.n[d]) * cfg.cell[d] for d in range(3)]
    return np.meshgrid(*axes, indexing="ij")


def random_fields(cfg: ScftConfig, amp: float, seed: int | None = None) -> list[np.ndarray]:
    """w_i = 2*amp*(U - 0.5), fields drawn in declaration order."""
    N = cfg.n_total
    u = mt_reals(cfg.seed if seed is None else seed, N * len(cfg.fields))
    return [2.0 * amp * (u[i * N:(i + 1) * N] - 0.5) for i in range(len(cfg.fields))]


def diblock32(precision="fp64", n=32) -> tuple[ScftConfig, list[np.ndarray]]:
    cfg = diblock_config(n, 4.0, 0.30, 20.0, 100,
                         Updater(kind="steepestDescent", relaxlambdas=(0.1, 0.05)), precision)
    x, _, _ = coords(cfg)
    L = cfg.box[0]
    c = np.cos(2 * math.pi * x / L).reshape(-1)
    w = random_fields(cfg, 0.1)
    return cfg, [w[0] + 1.0 * c, w[1] - 1.0 * c]


def hex_seed(cfg: ScftConfig) -> np.ndarray:
    x, y, _ = coords(cfg)
    L = cfg.box[0]
    k = 2 * math.pi / L
    s = (np.cos(k * (2 * x)) + np.cos(k * (-x + 2 * y)) + np.cos(k * (-x - 2 * y))) / 3.0
    return s.reshape(-1)


def diblock128(precision="mixed", n=128, anderson=True) -> tuple[ScftConfig, list[np.ndarray]]:
    upd = (Updater(kind="andersonMixing", relaxlambdas=(0.1, 0.05), anderson_depth=10,
                   anderson_mix=0.5, anderson_start=100) if anderson
           else Updater(kind="steepestDescent", relaxlambdas=(0.1, 0.05)))
    cfg = diblock_config(n, 8.0 * n / 128, 0.35, 25.0, 200, upd, precision)
    s = hex_seed(cfg)
    w = random_fields(cfg, 0.05)
    return cfg, [w[0] + 1.0 * s, w[1] - 1.0 * s]


def diblock64_adjoint(n=64) -> tuple[ScftConfig, list[np.ndarray]]:
    cfg = diblock_config(n, 6.0 * n / 64, 0.40, 18.0, 128,
                         Updater(kind="steepestDescent", relaxlambdas=(0.1, 0.05)), "fp64",
                         force=True)
    _, _, z = coords(cfg)
    c = np.cos(2 * math.pi * z / cfg.box[2]).reshape(-1)
    w = random_fields(cfg, 0.1)
    return cfg, [w[0] + 1.0 * c, w[1] - 1.0 * c]


def triblock256(precision="mixed", n=256) -> tuple[ScftConfig, list[np.ndarray]]:
    ds = 1.0 / 400
    length = 100
    poly = Polymer(name="abc", volfrac=1.0, length=length, blocks=[
        Block("abc_A", "A", ds, 0.3, ["freeEnd"], ["abc_B"]),
        Block("abc_B", "B", ds, 0.4, ["abc_A"], ["abc_C"]),
        Block("abc_C", "C", ds, 0.3, ["abc_B"], ["freeEnd"]),
    ])
    box = 16.0 * n / 256
    cfg = ScftConfig(n=(n, n, n), cell=(box / n,) * 3, fields=["A", "B", "C"], polymers=[poly],
                     interactions=[Interaction("AB", 30.0 / length, ["A", "B"]),
                                   Interaction("BC", 30.0 / length, ["B", "C"]),
                                   Interaction("AC", 45.0 / length, ["A", "C"])],
                     updater=Updater(kind="andersonMixing", relaxlambdas=(0.05, 0.025),
                                     anderson_depth=20, anderson_mix=0.5, anderson_start=200),
                     seed=38383, precision=precision)
    return cfg, random_fields(cfg, 0.05)


def blend(n: int, chin: float, f_a: float, phi_h: float, precision="mixed", seed=1,
          ns=100, anderson=True) -> ScftConfig:
    """AB diblock (length 100) + A homopolymer (length 50, alpha = 0.5) blend."""
    ds = 1.0 / ns
    length = 100
    polymers = [diblock(f_a=f_a, ds=ds, length=length, volfrac=1.0 - phi_h)]
    if phi_h > 0.0:
        polymers.append(Polymer(name="homoA", volfrac=phi_h, length=length // 2, blocks=[
            Block("homoA_A", "A", ds, 1.0, ["freeEnd"], ["freeEnd"])]))
    upd = (Updater(kind="andersonMixing", relaxlambdas=(0.1, 0.05), anderson_depth=10,
                   anderson_mix=0.5, anderson_start=100) if anderson
           else Updater(kind="steepestDescent", relaxlambdas=(0.1, 0.05)))
    box = 4.0 * n / 32
    return ScftConfig(n=(n, n, n), cell=(box / n,) * 3, fields=["A", "B"], polymers=polymers,
                      interactions=[Interaction("AB", chin / length, ["A", "B"])], updater=upd,
                      seed=seed, precision=precision)


def blend_instances(count=64, seed=2024, ns=100, sizes=(32, 48, 64, 96), precision="mixed"):
    """Instances of the batched workload: grid from {32,48,64,96}^3, chiN ~ U[12,30],
    f_A ~ U[0.2,0.5] quantised to 1/Ns, homopolymer fraction ~ U[0,0.2]."""
    u = mt_reals(seed, 4 * count)
    out = []
    for i in range(count):
        n = sizes[int(u[4 * i] * len(sizes)) % len(sizes)]
        chin = 12.0 + 18.0 * u[4 * i + 1]
        f_a = round((0.2 + 0.3 * u[4 * i + 2]) * ns) / ns
        phi_h = round(0.2 * u[4 * i + 3], 6)
        cfg = blend(n, chin, f_a, phi_h, precision=precision, seed=seed + 1 + i, ns=ns)
        x, _, _ = coords(cfg)
        c = np.cos(2 * math.pi * x / cfg.box[0]).reshape(-1)
        w = random_fields(cfg, 0.1)
        out.append((cfg, [w[0] + c, w[1] - c]))
    return out


def charged_diblock(n=(16, 16, 16), cell=0.05, precision="fp64", poisson_every=5, seed=38383):
    """(cfg, w, psi) for a charged diblock with counter-ions and a Poisson updater."""
    from .config import PoissonUpdater, Solvent
    za, alpha, f_a, length, ds, red_t = 1.0, 0.01, 0.5, 1000, 0.05, 1.4
    blocks = [Block(name="blockA", scfield="A", ds=ds, lengthfrac=f_a, headjoined=["freeEnd"],
                    tailjoined=["blockB"], kind="chargeFlexPseudoSpec", chargefield="charge",
                    za=za, alpha=alpha),
              Block(name="blockB", scfield="B", ds=ds, lengthfrac=1.0 - f_a, headjoined=["blockA"],
                    tailjoined=["freeEnd"])]
    cfg = ScftConfig(
        n=tuple(n), cell=(cell, cell, cell), fields=["A", "B"],
        polymers=[Polymer(name="diblock1", volfrac=1.0, length=length, blocks=blocks)],
        interactions=[Interaction(name="AB", chi=1.0 / (20.0 * 3.1415 * red_t), scfields=["A", "B"])],
        updater=Updater(kind="steepestDescent", relaxlambdas=(0.2, 0.1)), seed=seed,
        precision=precision,
        solvents=[Solvent(name="counterIons", scfield="A", volfrac=0.0, kind="simpleIons",
                          chargefield="charge", blockfield="counterIon", zc=-1.0,
                          neutral_factor=za * alpha * f_a)],
        charge_fields=["charge", "counterIon"],
        poisson=PoissonUpdater(name="ePotential", updatefields=["charge"],
                               bjerrum_len=1.0 / (4.0 * 3.1415 * alpha * red_t), relaxlambda=1.0,
                               apply_frequency=poisson_every))
    x, _, _ = coords(cfg)
    c = np.cos(2 * math.pi * x / cfg.box[0]).reshape(-1)
    w = random_fields(cfg, 0.1)
    u = mt_reals(seed + 1, cfg.n_total)
    psi = 0.05 * c + 0.01 * (u - 0.5)
    return cfg, [w[0] + 1.0 * c, w[1] - 1.0 * c], psi


def polydisperse_diblock(n=(16, 16, 16), cell=0.2, n_g=4, schulz_alpha=1.5, precision="fp64",
                         seed=38383):
    """(cfg, w) for a diblock whose B block follows a Schulz length distribution."""
    blocks = [Block(name="blockA", scfield="A", ds=0.02, lengthfrac=0.7, headjoined=["freeEnd"],
                    tailjoined=["blockB"], force_block_steps=True),
              Block(name="blockB", scfield="B", ds=0.01, lengthfrac=0.3, headjoined=["blockA"],
                    tailjoined=["freeEnd"], force_block_steps=True)]
    cfg = ScftConfig(
        n=tuple(n), cell=(cell, cell, cell), fields=["A", "B"],
        polymers=[Polymer(name="diblock1", volfrac=1.0, length=100, blocks=blocks,
                          kind="polyDisperseBCP", n_g=n_g, schulz_alpha=schulz_alpha,
                          polyblock="blockB")],
        interactions=[Interaction(name="AB", chi=0.12, scfields=["A", "B"])],
        updater=Updater(kind="steepestDescent", relaxlambdas=(0.2, 0.1)), seed=seed,
        precision=precision)
    x, _, _ = coords(cfg)
    c = np.cos(2 * math.pi * x / cfg.box[0]).reshape(-1)
    w = random_fields(cfg, 0.1)
    return cfg, [w[0] + 1.0 * c, w[1] - 1.0 * c]


def star(fracs=(0.3, 0.3, 0.4), fields=("A", "B", "C"), ds=0.01, length=100, name="star"):
    """An arm-star: arm i has a free head and its tail at the one junction."""
    arms = [f"{name}_{k}" for k in range(len(fracs))]
    blocks = [Block(name=arms[k], scfield=fields[k], ds=ds, lengthfrac=fracs[k], headjoined=["freeEnd"],
                    tailjoined=[a for a in arms if a != arms[k]]) for k in range(len(fracs))]
    return Polymer(name=name, volfrac=1.0, length=length, blocks=blocks)


def star_abc(n=16, box=3.2, precision="fp64", fracs=(0.3, 0.3, 0.4), seed=515):
    """(cfg, w) for a three-arm ABC star melt."""
    cfg = ScftConfig(
        n=(n, n, n), cell=(box / n,) * 3, fields=["A", "B", "C"], polymers=[star(fracs)],
        interactions=[Interaction("AB", 0.15, ["A", "B"]), Interaction("BC", 0.15, ["B", "C"]),
                      Interaction("AC", 0.15, ["A", "C"])],
        updater=Updater(kind="steepestDescent", relaxlambdas=(0.05, 0.025)), seed=seed,
        precision=precision)
    return cfg, random_fields(cfg, 0.2)
