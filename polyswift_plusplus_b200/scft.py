"""Python mirror of the reference's domain / plugin interfaces over the C-ABI.

``ScftSolver`` follows the PsDomain build cycle (pstrol/PsDomain.cpp:64-372):
construction = setAttrib + buildData + buildSolvers (``ps_gpu_create``), then
``initialize()`` (the reference's "random" monomerDens initialisation) or
``restore(w, p)`` (dump/restart of (dens, conj) fields), then ``update(t)``
iterations, and scalars equal to what the reference's free-energy history and
``getLogBigQ`` report.  ``B200FFT`` is the ``PsFFTBase::scaledFFTPair`` plugin.
All computation runs on the GPU through the native library; nothing here falls
back to the CPU.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi as A
from .config import ScftConfig


class ScftSolver:
    def __init__(self, cfg: ScftConfig, _handle=None):
        self.cfg = cfg
        self._lib = A.load_library()
        self._owned = _handle is None
        if _handle is None:
            self._pc = cfg.to_ps_config()
            h = C.c_void_p()
            A.check(self._lib.ps_gpu_create(C.byref(self._pc), C.byref(h)), None)
            self._h = h
        else:
            self._h = C.c_void_p(_handle)
        self.N = cfg.n_total
        self.nf = len(cfg.fields)
        self.t = 0
        if self._owned:
            # updaters after the field updater, installed in updaterSequence order
            for kind, u in cfg.post_updaters():
                if kind == "filter":
                    self.set_spectral_filter(u)
                else:
                    self.set_poisson(u)

    # -- lifetime ---------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None):
            if self._owned:
                self._lib.ps_gpu_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int) -> None:
        A.check(rc, self._h)

    # -- build cycle ------------------------------------------------------
    def block_steps(self, polymer: int, block: int) -> int:
        v = C.c_int()
        self._check(self._lib.ps_gpu_block_steps(self._h, polymer, block, C.byref(v)))
        return v.value

    def initialize(self) -> None:
        """PsMonomerDens::initialize "random": w_i = U[0,1) - 0.5, p = 0."""
        self._check(self._lib.ps_gpu_init_random(self._h))

    def restore(self, w, p=None) -> None:
        """Set the conjugate fields (nf x N, or a list) and optionally the pressure."""
        w = [np.ascontiguousarray(x, dtype=np.float64).reshape(-1) for x in w]
        if len(w) != self.nf:
            raise ValueError(f"expected {self.nf} fields")
        for i, x in enumerate(w):
            self.set_field(A.PS_FIELD_W, i, x)
        if p is not None:
            self.set_field(A.PS_FIELD_PRES, 0, p)
        else:
            self.set_field(A.PS_FIELD_PRES, 0, np.zeros(self.N))

    def set_field(self, which: int, index: int, data) -> None:
        if hasattr(data, "data_ptr"):  # torch tensor: on the handle's device, or (pinned) host
            t = data
            if t.dtype != __import__("torch").float64 or not t.is_contiguous():
                raise ValueError("tensors must be contiguous float64")
            if t.numel() != self.N:
                raise ValueError("wrong field size")
            self._check(self._lib.ps_gpu_set_fields(self._h, which, index, C.c_void_p(t.data_ptr()),
                                                    1 if t.is_cuda else 0))
            return
        x = np.ascontiguousarray(data, dtype=np.float64).reshape(-1)
        if x.size != self.N:
            raise ValueError("wrong field size")
        self._check(self._lib.ps_gpu_set_fields(self._h, which, index, x.ctypes.data_as(C.c_void_p), 0))

    def get_field(self, which: int, index: int = 0, out=None):
        if out is not None and hasattr(out, "data_ptr"):  # torch tensor: device or (pinned) host
            if out.dtype != __import__("torch").float64 or not out.is_contiguous() or out.numel() != self.N:
                raise ValueError("out must be a contiguous float64 tensor of N values")
            self._check(self._lib.ps_gpu_get_fields(self._h, which, index, C.c_void_p(out.data_ptr()),
                                                    1 if out.is_cuda else 0))
            return out
        x = np.empty(self.N, dtype=np.float64) if out is None else out
        self._check(self._lib.ps_gpu_get_fields(self._h, which, index, x.ctypes.data_as(C.c_void_p), 0))
        return x

    def get_field_async(self, which: int, index: int, out) -> None:
        """Start reading a field into `out` (a pinned host float64 tensor or a numpy
        array of N values) without waiting; `out` holds it after fields_wait()."""
        if hasattr(out, "data_ptr"):
            if out.is_cuda or out.dtype != __import__("torch").float64 or out.numel() != self.N:
                raise ValueError("out must be a host float64 tensor of N values")
            ptr = C.c_void_p(out.data_ptr())
        else:
            if out.dtype != np.float64 or out.size != self.N or not out.flags.c_contiguous:
                raise ValueError("out must be a contiguous float64 array of N values")
            ptr = out.ctypes.data_as(C.c_void_p)
        self._check(self._lib.ps_gpu_get_fields_async(self._h, which, index, ptr))

    def set_field_async(self, which: int, index: int, data) -> None:
        """Start copying a field in from `data` (a pinned host or device float64 tensor, or a
        numpy array of N values) without waiting; `data` must stay unchanged until
        fields_wait(), synchronize() or scalars() returns.  The pressure field's copy overlaps
        the next iteration's sweeps."""
        if hasattr(data, "data_ptr"):
            if data.dtype != __import__("torch").float64 or data.numel() != self.N or not data.is_contiguous():
                raise ValueError("data must be a contiguous float64 tensor of N values")
            ptr = C.c_void_p(data.data_ptr())
        else:
            if data.dtype != np.float64 or data.size != self.N or not data.flags.c_contiguous:
                raise ValueError("data must be a contiguous float64 array of N values")
            ptr = data.ctypes.data_as(C.c_void_p)
        self._check(self._lib.ps_gpu_set_fields_async(self._h, which, index, ptr))

    def fields_wait(self) -> None:
        self._check(self._lib.ps_gpu_fields_wait(self._h))

    def w(self, i: int) -> np.ndarray:
        return self.get_field(A.PS_FIELD_W, i)

    def phi(self, i: int) -> np.ndarray:
        return self.get_field(A.PS_FIELD_PHI, i)

    def pressure(self) -> np.ndarray:
        return self.get_field(A.PS_FIELD_PRES, 0)

    def rho(self, c: int) -> np.ndarray:
        """Charge density of chargeDens field c."""
        return self.get_field(A.PS_FIELD_CHARGE, c)

    def psi(self, c: int) -> np.ndarray:
        """Electric potential of chargeDens field c."""
        return self.get_field(A.PS_FIELD_POTENTIAL, c)

    # -- iterations -------------------------------------------------------
    def update(self, n: int = 1) -> None:
        """Run n SCFT iterations (PsDomain::update order)."""
        self._check(self._lib.ps_gpu_iterate(self._h, int(n)))
        self.t += n

    def scalars(self) -> dict:
        s = A.ps_scalars()
        self._check(self._lib.ps_gpu_get_scalars(self._h, C.byref(s)))
        return s.as_dict(len(self.cfg.polymers))

    def propagator(self, polymer: int, block: int, end: int, n: int) -> np.ndarray:
        x = np.empty(self.N, dtype=np.float64)
        self._check(self._lib.ps_gpu_get_propagator(self._h, polymer, block, end, n,
                                                    x.ctypes.data_as(C.c_void_p)))
        return x

    def synchronize(self) -> None:
        self._check(self._lib.ps_gpu_synchronize(self._h))

    @property
    def launches_per_iteration(self) -> int:
        return int(self._lib.ps_gpu_launches_per_iteration(self._h))

    @property
    def stream_ptr(self) -> int:
        """The handle's cudaStream_t (e.g. for torch.cuda.ExternalStream)."""
        return int(self._lib.ps_gpu_stream(self._h) or 0)

    def set_variant(self, variant: int) -> None:
        """Force a kernel variant (0..31) or re-enable autotuning (-1)."""
        self._check(self._lib.ps_gpu_set_variant(self._h, int(variant)))

    def set_spectral_filter(self, spec_filter) -> None:
        """Install a simpleSpecFilter updater (config.SpecFilter) or remove it (None)."""
        if spec_filter is None:
            self._check(self._lib.ps_gpu_set_spectral_filter(self._h, None))
            return
        self._fcfg = spec_filter.to_ps(self.cfg)
        self._check(self._lib.ps_gpu_set_spectral_filter(self._h, C.byref(self._fcfg)))

    def apply_spectral_filter(self) -> None:
        self._check(self._lib.ps_gpu_apply_spectral_filter(self._h))

    def set_poisson(self, poisson) -> None:
        """Install a poissonUpdater (config.PoissonUpdater) or remove it (None)."""
        if poisson is None:
            self._check(self._lib.ps_gpu_set_poisson(self._h, None))
            return
        self._pcfg = poisson.to_ps(self.cfg)
        self._check(self._lib.ps_gpu_set_poisson(self._h, C.byref(self._pcfg)))

    def apply_poisson(self) -> None:
        self._check(self._lib.ps_gpu_apply_poisson(self._h))

    def set_precision(self, precision: str) -> None:
        """Switch the sweeps to "fp64" or "mixed" between iterations; fields and
        the Anderson history carry over (precision escalation)."""
        code = {"fp64": A.PS_PREC_FP64, "mixed": A.PS_PREC_MIXED}[precision]
        self._check(self._lib.ps_gpu_set_precision(self._h, code))

    def variant(self):
        """(chosen variant or -1 before tuning, measured sweep ms of each variant;
        -1 for variants that were not timed)."""
        v = C.c_int()
        t = (C.c_float * 32)()
        self._check(self._lib.ps_gpu_get_variant(self._h, C.byref(v), t, 32))
        return v.value, [t[i] for i in range(32)]

    def enable_sweep_timing(self, max_samples: int) -> None:
        self._check(self._lib.ps_gpu_enable_sweep_timing(self._h, int(max_samples)))

    def sweep_timing(self, max_out: int = 4096):
        """(per-iteration sweep durations in ms, algorithmic bytes per iteration's
        sweeps, propagator steps per iteration); clears the samples."""
        buf = (C.c_double * max_out)()
        n = C.c_int()
        b = C.c_double()
        s = C.c_longlong()
        self._check(self._lib.ps_gpu_sweep_timing(self._h, buf, max_out, C.byref(n), C.byref(b),
                                                  C.byref(s)))
        return [buf[i] for i in range(min(n.value, max_out))], b.value, s.value


class ScftBatch:
    """Many independent SCFT instances advanced together (``ps_gpu_batch_*``).

    ``instance(i)`` is a ``ScftSolver`` view of instance i (restore, fields,
    scalars); ``update(n)`` runs n iterations of every instance in one captured
    graph per iteration, with each size class's propagator sweeps merged into
    one launch per contour step.
    """

    def __init__(self, cfgs):
        self.cfgs = list(cfgs)
        self._lib = A.load_library()
        self._pcs = (A.ps_config * len(self.cfgs))(*[c.to_ps_config() for c in self.cfgs])
        b = C.c_void_p()
        A.check(self._lib.ps_gpu_batch_create(self._pcs, len(self.cfgs), C.byref(b)),
                batch=C.c_void_p())
        self._b = b
        self._views = [ScftSolver(c, _handle=self._lib.ps_gpu_batch_instance(b, i))
                       for i, c in enumerate(self.cfgs)]
        # updaters after the field updater, installed in updaterSequence order
        for v, c in zip(self._views, self.cfgs):
            for kind, u in c.post_updaters():
                if kind == "filter":
                    v.set_spectral_filter(u)
                else:
                    v.set_poisson(u)
        self.t = 0

    def __len__(self) -> int:
        return len(self.cfgs)

    def instance(self, i: int) -> ScftSolver:
        return self._views[i]

    def update(self, n: int = 1) -> None:
        A.check(self._lib.ps_gpu_batch_iterate(self._b, int(n)), batch=self._b)
        self.t += n
        for v in self._views:
            v.t += n

    def scalars(self) -> list[dict]:
        return [v.scalars() for v in self._views]

    def set_variant(self, variant: int) -> None:
        A.check(self._lib.ps_gpu_batch_set_variant(self._b, int(variant)), batch=self._b)

    def classes(self):
        """(class index of each instance, kernel variant of each class)."""
        n = C.c_int()
        k = len(self.cfgs)
        co = (C.c_int * k)()
        va = (C.c_int * k)()
        A.check(self._lib.ps_gpu_batch_classes(self._b, C.byref(n), co, k, va, k), batch=self._b)
        return [co[i] for i in range(k)], [va[c] for c in range(n.value)]

    @property
    def launches_per_iteration(self) -> int:
        return int(self._lib.ps_gpu_batch_launches_per_iteration(self._b))

    @property
    def stream_ptr(self) -> int:
        return int(self._lib.ps_gpu_batch_stream(self._b) or 0)

    def close(self) -> None:
        if getattr(self, "_b", None):
            for v in self._views:
                v.close()
            self._lib.ps_gpu_batch_destroy(self._b)
            self._b = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class B200FFT:
    """PsFFTBase<double,3> plugin (psbase/PsFFTBase.h:40-134): every transform
    of the interface, host arrays in and out, FFTW-2 c2c semantics on real data
    (psfft/PsFFTW.cpp:122-297).  Each method returns a new flat array of
    getFFTSize() doubles."""

    def __init__(self, n, device: int = 0):
        self._lib = A.load_library()
        arr = (C.c_int * 3)(*[int(v) for v in n])
        h = C.c_void_p()
        A.check(self._lib.ps_fft_create(arr, A.PS_PREC_FP64, device, C.byref(h)), fft=True)
        self._h = h
        self.n = tuple(int(v) for v in n)
        self.N = self.n[0] * self.n[1] * self.n[2]

    def getFFTSize(self) -> int:
        v = C.c_size_t()
        A.check(self._lib.ps_fft_size(self._h, C.byref(v)), fft=True)
        return int(v.value)

    def getGrid(self) -> tuple:
        """The grid extents (PsFFTBase::getGrid reduced to what the transforms use)."""
        n = (C.c_int * 3)()
        A.check(self._lib.ps_fft_get_grid(self._h, n), fft=True)
        return tuple(int(v) for v in n)

    def _flat(self, a, name: str) -> np.ndarray:
        a = np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
        if a.size != self.N:
            raise ValueError(f"{name} size must equal getFFTSize()")
        return a

    def _call(self, fn: str, *arrays) -> np.ndarray:
        res = np.empty(self.N, dtype=np.float64)
        ptrs = [a.ctypes.data_as(C.c_void_p) for a in arrays]
        A.check(getattr(self._lib, fn)(self._h, *ptrs, res.ctypes.data_as(C.c_void_p)), fft=True)
        return res

    def scaledFFTPair(self, data, kdata) -> np.ndarray:
        """Re(IFFT(kdata * FFT(data)))."""
        return self._call("ps_fft_scaled_pair", self._flat(data, "data"), self._flat(kdata, "kdata"))

    def scaledFFTPairIm(self, data, kdata) -> np.ndarray:
        """Re(IFFT(kdata * FFT(i * data))): data is the imaginary part of the input."""
        return self._call("ps_fft_scaled_pair_im", self._flat(data, "data"), self._flat(kdata, "kdata"))

    def convolveRe(self, data1, data2) -> np.ndarray:
        """Re(IFFT(FFT(data1) * FFT(data2)))."""
        return self._call("ps_fft_convolve_re", self._flat(data1, "data1"), self._flat(data2, "data2"))

    def forwardFFTAbs(self, data) -> np.ndarray:
        """|FFT(data)|^2 elementwise (re^2 + im^2, as the reference computes it)."""
        return self._call("ps_fft_forward_abs", self._flat(data, "data"))

    def calcForwardFFT(self, data) -> np.ndarray:
        """Re(FFT(data))."""
        return self._call("ps_fft_forward", self._flat(data, "data"))

    def calcBackwardFFT(self, data) -> np.ndarray:
        """Re(IFFT(data)) of real data, unnormalised."""
        return self._call("ps_fft_backward", self._flat(data, "data"))

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.ps_fft_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
