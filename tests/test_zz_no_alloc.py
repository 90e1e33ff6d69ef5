"""ps_fft_scaled_pair_noalloc: the scaledFFTPair entry point that allocates nothing.

It exists for callers that cannot call cudaMalloc at the time they need the
transform (their device memory belongs to another allocator, or their solver
loop must not allocate once running).  They hand in device buffers, and the
library works in one fixed 4 MiB device array per GPU.  These tests call it
through the C-ABI on torch-owned device buffers and compare it with the
allocating plugin ps_fft_scaled_pair, whose own parity with the oracle is
tested elsewhere, at the same 1e-12 relative tolerance.  Two calls in a row
with different inputs check that whatever the shared array keeps from a call
does not leak into the next.  This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

from polyswift_plusplus_b200 import _abi as A
from polyswift_plusplus_b200.scft import B200FFT

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _noalloc(lib, shape, d, k):
    """One call of the allocation-free entry point; returns res on the host."""
    import torch
    dev = torch.device("cuda", 0)
    td = torch.from_numpy(d).to(dev)
    tk = torch.from_numpy(k).to(dev)
    tr = torch.full(d.shape, float("nan"), dtype=torch.float64, device=dev)
    n = (C.c_int * 3)(*shape)
    stream = torch.cuda.current_stream(dev)
    rc = lib.ps_fft_scaled_pair_noalloc(n, C.c_void_p(td.data_ptr()), C.c_void_p(tk.data_ptr()),
                                        C.c_void_p(tr.data_ptr()), C.c_void_p(stream.cuda_stream))
    assert rc == A.PS_OK, lib.ps_fft_noalloc_last_error().decode()
    stream.synchronize()
    return tr.cpu().numpy()


def _plugin(shape, d, k):
    f = B200FFT(shape)
    try:
        return f.scaledFFTPair(d, k).reshape(shape)
    finally:
        f.close()


def _inputs(shape, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal(shape), rng.standard_normal(shape)


def test_noalloc_two_calls_match_plugin_at_64cubed(gpu):
    shape = (64, 64, 64)  # the largest cube the 4 MiB scratch holds
    for seed in (11, 12):
        d, k = _inputs(shape, seed)
        got = _noalloc(gpu, shape, d, k)
        assert np.isfinite(got).all()
        assert _rel(got, _plugin(shape, d, k)) < TOL


def test_noalloc_matches_the_oracle_directly(gpu, oracle_lib):
    """The same check without the indirection through the allocating plugin:
    the CPU restatement of PsFFTW::scaledFFTPair, on a fused-plane grid."""
    import oracle as O
    shape = (32, 32, 32)
    d, k = _inputs(shape, 31)
    assert _rel(_noalloc(gpu, shape, d, k), O.scaled_fft_pair(d, k)) < TOL


def test_noalloc_two_calls_of_different_shapes(gpu):
    # a fused-plane grid and a row-kernel grid back to back on the same scratch
    for shape, seed in (((24, 48, 48), 21), ((8, 4, 256), 22), ((32, 32, 32), 23)):
        d, k = _inputs(shape, seed)
        got = _noalloc(gpu, shape, d, k)
        assert _rel(got, _plugin(shape, d, k)) < TOL


def test_noalloc_rejects_oversize_and_misaligned(gpu):
    import torch
    assert gpu.ps_fft_noalloc_scratch_bytes() == 4 << 20
    buf = torch.zeros(96 ** 3 + 2, dtype=torch.float64, device="cuda:0")
    p = buf.data_ptr()
    big = (C.c_int * 3)(96, 96, 96)
    rc = gpu.ps_fft_scaled_pair_noalloc(big, C.c_void_p(p), C.c_void_p(p), C.c_void_p(p), None)
    assert rc == A.PS_INPUT_ERR
    assert b"scratch" in gpu.ps_fft_noalloc_last_error()
    small = (C.c_int * 3)(8, 8, 8)
    rc = gpu.ps_fft_scaled_pair_noalloc(small, C.c_void_p(p + 8), C.c_void_p(p), C.c_void_p(p),
                                        None)
    assert rc == A.PS_ATTRIB_ERR
    torch.cuda.synchronize()
