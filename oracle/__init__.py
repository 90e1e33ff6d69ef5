"""ctypes front end of the FP64 CPU oracle (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this package, as the checker or the timed CPU baseline.  Parity is unpinned:
see oracle/oracle.h.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from polyswift_plusplus_b200 import _abi as A
from polyswift_plusplus_b200.config import ScftConfig

from .build import LIB, build

_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = C.CDLL(str(LIB))
        vp, dp = C.c_void_p, C.POINTER(C.c_double)
        L.oracle_set_threads.restype = C.c_int
        L.oracle_set_threads.argtypes = [C.c_int]
        L.oracle_mt_reals.argtypes = [C.c_ulonglong, C.c_long, vp]
        L.oracle_mt_gauss.argtypes = [C.c_ulonglong, C.c_long, vp]
        L.oracle_mt_u32.argtypes = [C.c_ulonglong, C.c_long, vp]
        L.oracle_fft3d.argtypes = [C.POINTER(C.c_int), vp, vp, C.c_int]
        L.oracle_scaled_fft_pair.argtypes = [C.POINTER(C.c_int), vp, vp, vp]
        L.oracle_scaled_fft_pair_im.argtypes = [C.POINTER(C.c_int), vp, vp, vp]
        L.oracle_convolve_re.argtypes = [C.POINTER(C.c_int), vp, vp, vp]
        L.oracle_forward_fft_abs.argtypes = [C.POINTER(C.c_int), vp, vp]
        L.oracle_calc_forward_fft.argtypes = [C.POINTER(C.c_int), vp, vp]
        L.oracle_calc_backward_fft.argtypes = [C.POINTER(C.c_int), vp, vp]
        L.oracle_create.restype = C.c_int
        L.oracle_create.argtypes = [C.POINTER(A.ps_config), C.POINTER(vp), C.c_char_p, C.c_int]
        L.oracle_destroy.argtypes = [vp]
        L.oracle_block_steps.restype = C.c_int
        L.oracle_block_steps.argtypes = [vp, C.c_int, C.c_int]
        L.oracle_init_random.argtypes = [vp]
        L.oracle_set_field.argtypes = [vp, C.c_int, C.c_int, vp]
        L.oracle_set_filter.restype = C.c_int
        L.oracle_set_filter.argtypes = [vp, C.POINTER(A.ps_filter_config)]
        L.oracle_apply_filter.argtypes = [vp]
        L.oracle_set_poisson.restype = C.c_int
        L.oracle_set_poisson.argtypes = [vp, C.POINTER(A.ps_poisson_config)]
        L.oracle_apply_poisson.argtypes = [vp]
        L.oracle_gauss_laguerre.restype = C.c_int
        L.oracle_gauss_laguerre.argtypes = [C.c_int, C.c_double, vp, vp]
        L.oracle_get_field.argtypes = [vp, C.c_int, C.c_int, vp]
        L.oracle_iterate.restype = C.c_int
        L.oracle_iterate.argtypes = [vp, C.c_int, C.POINTER(A.ps_scalars)]
        L.oracle_get_propagator.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int, vp]
        L.oracle_get_k2.argtypes = [vp, C.c_int, C.c_int, vp]
        L.oracle_last_timing.argtypes = [vp, dp, dp]
        L.oracle_propagate_sample.restype = C.c_double
        L.oracle_propagate_sample.argtypes = [vp, C.c_int]
        _lib = L
    return _lib


def set_threads(n: int) -> int:
    return lib().oracle_set_threads(int(n))


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def mt_reals(seed: int, n: int) -> np.ndarray:
    out = np.empty(n)
    lib().oracle_mt_reals(seed, n, _ptr(out))
    return out


def mt_gauss(seed: int, n: int) -> np.ndarray:
    out = np.empty(n)
    lib().oracle_mt_gauss(seed, n, _ptr(out))
    return out


def mt_u32(seed: int, n: int) -> np.ndarray:
    out = np.empty(n, dtype=np.uint32)
    lib().oracle_mt_u32(seed, n, _ptr(out))
    return out


def fft3d(x: np.ndarray, sign: int = -1) -> np.ndarray:
    n = (C.c_int * 3)(*x.shape)
    re = np.ascontiguousarray(x.real, dtype=np.float64).copy()
    im = np.ascontiguousarray(x.imag, dtype=np.float64).copy()
    lib().oracle_fft3d(n, _ptr(re), _ptr(im), sign)
    return re + 1j * im


def scaled_fft_pair(data: np.ndarray, kdata: np.ndarray) -> np.ndarray:
    n = (C.c_int * 3)(*data.shape)
    d = np.ascontiguousarray(data, dtype=np.float64)
    k = np.ascontiguousarray(kdata, dtype=np.float64)
    res = np.empty_like(d)
    lib().oracle_scaled_fft_pair(n, _ptr(d), _ptr(k), _ptr(res))
    return res


def _two_input(fn: str, a: np.ndarray, b: np.ndarray) -> np.ndarray:
    n = (C.c_int * 3)(*a.shape)
    x = np.ascontiguousarray(a, dtype=np.float64)
    y = np.ascontiguousarray(b, dtype=np.float64)
    res = np.empty_like(x)
    getattr(lib(), fn)(n, _ptr(x), _ptr(y), _ptr(res))
    return res


def _one_input(fn: str, a: np.ndarray) -> np.ndarray:
    n = (C.c_int * 3)(*a.shape)
    x = np.ascontiguousarray(a, dtype=np.float64)
    res = np.empty_like(x)
    getattr(lib(), fn)(n, _ptr(x), _ptr(res))
    return res


def scaled_fft_pair_im(data: np.ndarray, kdata: np.ndarray) -> np.ndarray:
    """PsFFTW::scaledFFTPairIm: Re(IFFT(kdata * FFT(i*data)))."""
    return _two_input("oracle_scaled_fft_pair_im", data, kdata)


def convolve_re(data1: np.ndarray, data2: np.ndarray) -> np.ndarray:
    """PsFFTW::convolveRe: Re(IFFT(FFT(data1) * FFT(data2)))."""
    return _two_input("oracle_convolve_re", data1, data2)


def forward_fft_abs(data: np.ndarray) -> np.ndarray:
    """PsFFTW::forwardFFTAbs: |FFT(data)|^2 elementwise."""
    return _one_input("oracle_forward_fft_abs", data)


def calc_forward_fft(data: np.ndarray) -> np.ndarray:
    """PsFFTW::calcForwardFFT: Re(FFT(data))."""
    return _one_input("oracle_calc_forward_fft", data)


def calc_backward_fft(data: np.ndarray) -> np.ndarray:
    """PsFFTW::calcBackwardFFT: Re(IFFT(data)), unnormalised."""
    return _one_input("oracle_calc_backward_fft", data)


def gauss_laguerre(n: int, a: float):
    """The oracle's generalized Gauss-Laguerre rule (root bracketing + bisection)."""
    x = np.zeros(n)
    w = np.zeros(n)
    rc = lib().oracle_gauss_laguerre(int(n), float(a), _ptr(x), _ptr(w))
    if rc != A.PS_OK:
        raise A.PsError(rc, "bad Gauss-Laguerre arguments")
    return x, w


class Oracle:
    """The CPU restatement of one SCFT instance (FP64)."""

    def __init__(self, cfg: ScftConfig):
        self.cfg = cfg
        self._pc = cfg.to_ps_config()
        h = C.c_void_p()
        err = C.create_string_buffer(512)
        rc = lib().oracle_create(C.byref(self._pc), C.byref(h), err, 512)
        if rc != A.PS_OK:
            raise A.PsError(rc, err.value.decode())
        self._h = h
        self.N = cfg.n_total
        self.nf = len(cfg.fields)
        for kind, u in cfg.post_updaters():
            if kind == "filter":
                self.set_spectral_filter(u)
            else:
                self.set_poisson(u)

    def close(self):
        if getattr(self, "_h", None):
            lib().oracle_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def block_steps(self, ip: int, ib: int) -> int:
        return lib().oracle_block_steps(self._h, ip, ib)

    def initialize(self):
        lib().oracle_init_random(self._h)

    def restore(self, w, p=None):
        for i, x in enumerate(w):
            self.set_field(A.PS_FIELD_W, i, x)
        self.set_field(A.PS_FIELD_PRES, 0, np.zeros(self.N) if p is None else p)

    def set_spectral_filter(self, spec_filter):
        """spec_filter: a config.SpecFilter, or None to remove the updater."""
        self._fcfg = spec_filter.to_ps(self.cfg) if spec_filter is not None else None
        rc = lib().oracle_set_filter(self._h, C.byref(self._fcfg) if self._fcfg is not None else None)
        if rc != A.PS_OK:
            raise A.PsError(rc, "bad spectral filter")

    def apply_spectral_filter(self):
        lib().oracle_apply_filter(self._h)

    def set_poisson(self, poisson):
        """poisson: a config.PoissonUpdater, or None to remove the updater."""
        self._ppcfg = poisson.to_ps(self.cfg) if poisson is not None else None
        rc = lib().oracle_set_poisson(self._h, C.byref(self._ppcfg) if self._ppcfg is not None else None)
        if rc != A.PS_OK:
            raise A.PsError(rc, "bad poisson updater")

    def apply_poisson(self):
        lib().oracle_apply_poisson(self._h)

    def rho(self, c):
        return self.get_field(A.PS_FIELD_CHARGE, c)

    def psi(self, c):
        return self.get_field(A.PS_FIELD_POTENTIAL, c)

    def set_field(self, which, index, data):
        x = np.ascontiguousarray(data, dtype=np.float64).reshape(-1)
        assert x.size == self.N
        lib().oracle_set_field(self._h, which, index, _ptr(x))

    def get_field(self, which, index=0):
        x = np.empty(self.N)
        lib().oracle_get_field(self._h, which, index, _ptr(x))
        return x

    def w(self, i):
        return self.get_field(A.PS_FIELD_W, i)

    def phi(self, i):
        return self.get_field(A.PS_FIELD_PHI, i)

    def pressure(self):
        return self.get_field(A.PS_FIELD_PRES, 0)

    def update(self, n: int = 1) -> list[dict]:
        hist = (A.ps_scalars * max(n, 1))()
        rc = lib().oracle_iterate(self._h, n, hist)
        if rc != A.PS_OK:
            raise A.PsError(rc, "oracle iteration failed")
        return [hist[i].as_dict(len(self.cfg.polymers)) for i in range(n)]

    def propagator(self, ip, ib, end, n):
        x = np.empty(self.N)
        lib().oracle_get_propagator(self._h, ip, ib, end, n, _ptr(x))
        return x

    def k2(self, ip, ib):
        x = np.empty(self.N)
        lib().oracle_get_k2(self._h, ip, ib, _ptr(x))
        return x

    def last_timing(self) -> tuple[float, float]:
        """(seconds in the propagator sweeps, seconds in total) of the last iteration."""
        a, b = C.c_double(), C.c_double()
        lib().oracle_last_timing(self._h, C.byref(a), C.byref(b))
        return a.value, b.value

    def propagate_sample(self, nsteps: int) -> float:
        """Wall seconds of nsteps propagator steps (bounded sample of the sweep work)."""
        return float(lib().oracle_propagate_sample(self._h, int(nsteps)))
