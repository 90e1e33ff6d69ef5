"""Build the oracle's C restatement into ``oracle/liboracle.so`` (TEST INFRASTRUCTURE).

gcc, FP64, no FMA contraction (-ffp-contract=off) so the arithmetic follows the
written evaluation order; OpenMP for the FFT and point loops.  The reference
itself is not built: it needs txbase, txutils, FFTW 2, HDF5, Boost and MPI,
none of which exist here.
"""
from __future__ import annotations

import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
SRCS = ["mt19937.c", "fft.c", "scft.c"]


def build(force: bool = False) -> Path:
    srcs = [HERE / s for s in SRCS]
    hdrs = [HERE / "oracle.h", HERE / "mt19937.h", HERE.parent / "include" / "pswift.h"]
    newest = max(p.stat().st_mtime for p in srcs + hdrs)
    if not force and LIB.exists() and LIB.stat().st_mtime >= newest:
        return LIB
    cmd = ["gcc", "-O3", "-march=x86-64-v3", "-ffp-contract=off", "-fopenmp", "-fPIC", "-shared",
           "-std=c11", "-o", str(LIB) + ".tmp"] + [str(s) for s in srcs] + ["-lm"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{r.stderr}")
    Path(str(LIB) + ".tmp").replace(LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
