"""Failure detection on the GPU without a GPU fault.

* A bulk-copy wait that runs out: the plane pass's first wait on its spectrum
  copy is given a limit of 0 polls through ps_gpu_set_bulk_wait_limit, so every
  plane CTA takes the timeout path (set status bit 2, drain the copy still in
  flight under the full bound, return).  The handle reports PS_GPU_ERR with the
  timeout message and the context stays usable: a new handle runs and matches
  the oracle.
* A configuration whose propagator storage exceeds device memory: create fails
  with PS_GPU_ERR and a message, and nothing is left behind (a small handle
  created next runs normally).

The reference reports failures through its exit codes
(polyswift/polyswift/polyswift.cxx:115-125); the ABI returns the same numbers.
"""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from polyswift_plusplus_b200 import _abi as A
from polyswift_plusplus_b200 import workloads as W
from polyswift_plusplus_b200.scft import ScftSolver

pytestmark = pytest.mark.gpu


def small_run_matches_oracle():
    cfg, w = W.diblock32(n=16)
    g = ScftSolver(cfg)
    g.restore(w)
    g.update(2)
    o = O.Oracle(cfg)
    o.restore(w)
    ho = o.update(2)
    fe = g.scalars()["free_energy"]
    g.close()
    assert abs(fe - ho[-1]["free_energy"]) <= 1e-10 * abs(ho[-1]["free_energy"])


def test_bulk_copy_wait_timeout_is_reported(gpu, oracle_lib):
    cfg, w = W.diblock32(n=16)
    g = ScftSolver(cfg)
    g.set_variant(0)  # fused y-z plane pass: its spectrum arrives by bulk copy
    g.restore(w)
    assert gpu.ps_gpu_set_bulk_wait_limit(0) == A.PS_OK
    try:
        with pytest.raises(A.PsError) as ei:
            g.update(1)
    finally:
        assert gpu.ps_gpu_set_bulk_wait_limit(0xFFFFFFFF) == A.PS_OK
    assert ei.value.code == A.PS_GPU_ERR
    assert "wait limit" in str(ei.value)
    sc = A.ps_scalars()
    gpu.ps_gpu_get_scalars(g._h, C.byref(sc))
    assert sc.error_flags & 4
    g.close()
    small_run_matches_oracle()


def test_propagator_storage_beyond_device_memory(gpu, oracle_lib):
    import torch
    free, total = torch.cuda.mem_get_info(0)
    # 256^3 FP64 slices are 134 MB each: one sweep of this diblock stores
    # more slices than the whole device holds, so its single allocation fails
    ns = 2 * (int(total / (256 ** 3 * 8)) // 2 + 50)  # even: f_A = 0.5 gives whole block steps
    cfg = W.diblock_config(256, 16.0, 0.5, 10.0, ns, W.Updater(kind="steepestDescent",
                                                              relaxlambdas=(0.1, 0.05)), "fp64")
    with pytest.raises(A.PsError) as ei:
        ScftSolver(cfg)
    assert ei.value.code == A.PS_GPU_ERR
    assert "cudaMalloc" in str(ei.value)
    assert torch.cuda.mem_get_info(0)[0] >= free - (64 << 20)
    small_run_matches_oracle()
