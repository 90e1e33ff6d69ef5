"""Build the in-tree native library ``_native/libpswift_b200.so`` for sm_100a.

Every ``csrc/*.cu`` file is compiled by nvcc with
``-gencode arch=compute_100a,code=sm_100a -lineinfo`` into ``_build/`` and
linked into one shared library.  nvcc cross-compiles, so this runs on a host
without a GPU.  Objects are rebuilt only when a source or header is newer.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG.parent / "_build" / "native"
OUT_DIR = PKG / "_native"
LIB_NAME = "libpswift_b200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found; the CUDA toolkit is required to build the library")


def _flags(extra: list[str] | None = None) -> list[str]:
    f = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3",
                "--expt-relaxed-constexpr", "-I", str(PKG.parent / "include")]
    return f + (extra or [])


def _newest_header() -> float:
    hs = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + [PKG.parent / "include" / "pswift.h"]
    return max(h.stat().st_mtime for h in hs)


def _compile(src: Path, obj: Path, ptxas_verbose: bool) -> tuple[Path, str]:
    cmd = [nvcc_path(), "-c", str(src), "-o", str(obj)] + _flags(
        ["-Xptxas", "-v"] if ptxas_verbose else None)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src.name}:\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(force: bool = False, ptxas_verbose: bool = False, jobs: int | None = None) -> Path:
    BUILD.mkdir(parents=True, exist_ok=True)
    OUT_DIR.mkdir(parents=True, exist_ok=True)
    srcs = sorted(CSRC.glob("*.cu"))
    hdr_t = _newest_header()
    todo = []
    objs = []
    for s in srcs:
        o = BUILD / (s.stem + ".o")
        objs.append(o)
        if force or ptxas_verbose or not o.exists() or o.stat().st_mtime < max(s.stat().st_mtime, hdr_t):
            todo.append((s, o))
    logs = []
    if todo:
        with cf.ThreadPoolExecutor(max_workers=jobs or min(len(todo), os.cpu_count() or 4)) as ex:
            for obj, log in ex.map(lambda a: _compile(a[0], a[1], ptxas_verbose), todo):
                logs.append((obj.name, log))
    lib = OUT_DIR / LIB_NAME
    if todo or not lib.exists():
        tmp = lib.with_suffix(".so.tmp")
        cmd = [nvcc_path(), "-shared", "-o", str(tmp)] + ARCH + [str(o) for o in objs]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
        os.replace(tmp, lib)
    if ptxas_verbose:
        for name, log in logs:
            sys.stderr.write(f"== {name}\n{log}\n")
    return lib


if __name__ == "__main__":
    build(force="--force" in sys.argv, ptxas_verbose="-v" in sys.argv)
    print(OUT_DIR / LIB_NAME)
