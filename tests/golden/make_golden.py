"""Write the golden fixtures of tests/golden/ (run from the repository root).

The reference (PolySwift++) cannot be built or imported here and ships no
golden outputs, so these fixtures come from code that is independent of the C
oracle: numpy's MT19937 (legacy init_genrand seeding) with the reference's
real() and polar-Gaussian conversions written out below, and the numpy
restatement oracle/np_scft.py (numpy.fft).  The C oracle and the GPU path are
checked against them.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import math
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle.np_scft import NpScft  # noqa: E402
from polyswift_plusplus_b200 import workloads as W  # noqa: E402
from polyswift_plusplus_b200.config import Block, Interaction, Polymer, ScftConfig, Updater  # noqa: E402

OUT = Path(__file__).resolve().parent


def u32(seed, n):
    bg = np.random.MT19937(0)
    bg._legacy_seeding(seed)
    return bg.random_raw(n).astype(np.uint64)


def polar_gauss(reals, count):
    """psRandomGaussian: Marsaglia polar method, second value cached."""
    out, i = [], 0
    while len(out) < count:
        while True:
            v1 = 2.0 * reals[i] - 1.0
            v2 = 2.0 * reals[i + 1] - 1.0
            i += 2
            r = v1 * v1 + v2 * v2
            if 0.0 < r < 1.0:
                break
        fac = math.sqrt(-2.0 * math.log(r) / r)
        out.append(v2 * fac)
        out.append(v1 * fac)
    return np.array(out[:count])


def mt_fixture():
    seed = 38383
    raw = u32(seed, 6000)
    reals = raw.astype(np.float64) * (1.0 / 4294967296.0)
    np.savez_compressed(OUT / "mt19937_seed38383.npz", u32=raw[:1000].astype(np.uint32),
                        reals=reals[:2000], gauss=polar_gauss(reals, 1000))


def small_configs():
    cfgs = {}
    cfg, w = W.diblock32(n=8)
    cfgs["diblock8"] = (cfg, w)
    ds = 0.05
    tri = Polymer("abc", 1.0, 100, [Block("a", "A", ds, 0.25, ["freeEnd"], ["b"]),
                                    Block("b", "B", ds, 0.5, ["a"], ["c"]),
                                    Block("c", "C", ds, 0.25, ["b"], ["freeEnd"])])
    cfg = ScftConfig(n=(8, 8, 8), cell=(0.4, 0.4, 0.4), fields=["A", "B", "C"], polymers=[tri],
                     interactions=[Interaction("AB", 0.2, ["A", "B"]),
                                   Interaction("BC", 0.15, ["B", "C"]),
                                   Interaction("AC", 0.3, ["A", "C"])],
                     updater=Updater(relaxlambdas=(0.05, 0.02)), seed=77)
    cfgs["triblock8"] = (cfg, W.random_fields(cfg, 0.3))
    cfg = W.blend(8, 15.0, 0.4, 0.15, precision="fp64", seed=5, ns=20, anderson=False)
    cfgs["blend8"] = (cfg, W.random_fields(cfg, 0.3))
    return cfgs


def scft_fixtures(iters=4):
    for name, (cfg, w) in small_configs().items():
        s = NpScft(cfg)
        s.restore(w)
        hist = [s.iterate() for _ in range(iters)]
        np.savez_compressed(
            OUT / f"scft_{name}.npz",
            w0=np.array(w), free_energy=np.array([h["free_energy"] for h in hist]),
            q=np.array([h["q"] for h in hist]), max_incomp=np.array([h["max_incomp"] for h in hist]),
            w=np.array([x.reshape(-1) for x in s.w]), phi=np.array([x.reshape(-1) for x in s.phi]),
            p=s.p.reshape(-1))


if __name__ == "__main__":
    mt_fixture()
    scft_fixtures()
    print("written to", OUT)
