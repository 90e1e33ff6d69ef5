"""ctypes mirror of ``include/pswift.h`` and the loader of the native library.

The library is the in-tree ``_native/libpswift_b200.so`` built by
``build_native.py``.  There is no fallback: if it is missing or fails to load,
every entry point raises.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

PS_MAX_BLOCKS = 8
PS_MAX_JOINS = 4
PS_MAX_POLYMERS = 16
PS_MAX_FIELDS = 4
PS_MAX_INTERACTIONS = 6
PS_MAX_SOLVENTS = 2
PS_MAX_CHARGES = 2

PS_OK = 0
PS_ATTRIB_ERR = 3
PS_RUN_ERR = 4
PS_INPUT_ERR = 6
PS_GPU_ERR = 7

PS_PREC_FP64 = 0
PS_PREC_MIXED = 1
PS_UPD_STEEPEST = 0
PS_UPD_ANDERSON = 1
PS_FIELD_W = 0
PS_FIELD_PHI = 1
PS_FIELD_PRES = 2
PS_FIELD_CHARGE = 3
PS_FIELD_POTENTIAL = 4
PS_SOLV_SIMPLE = 0
PS_SOLV_IONS = 1
PS_FROM_HEAD = 0
PS_FROM_TAIL = 1

ERROR_NAMES = {PS_OK: "PS_OK", PS_ATTRIB_ERR: "PS_ATTRIB_ERR", PS_RUN_ERR: "PS_RUN_ERR",
               PS_INPUT_ERR: "PS_INPUT_ERR", PS_GPU_ERR: "PS_GPU_ERR"}


class ps_block_config(C.Structure):
    _fields_ = [("field", C.c_int), ("lengthfrac", C.c_double), ("ds", C.c_double),
                ("bseg_ratio", C.c_double), ("force_block_steps", C.c_int),
                ("n_head", C.c_int), ("n_tail", C.c_int),
                ("head_joined", C.c_int * PS_MAX_JOINS), ("tail_joined", C.c_int * PS_MAX_JOINS)]


class ps_polymer_config(C.Structure):
    _fields_ = [("volfrac", C.c_double), ("length", C.c_int), ("n_blocks", C.c_int),
                ("blocks", ps_block_config * PS_MAX_BLOCKS)]


class ps_polydisperse_config(C.Structure):
    _fields_ = [("enabled", C.c_int), ("poly_block", C.c_int), ("n_g", C.c_int),
                ("alpha", C.c_double)]


class ps_interaction_config(C.Structure):
    _fields_ = [("field_a", C.c_int), ("field_b", C.c_int), ("chi", C.c_double)]


class ps_updater_config(C.Structure):
    _fields_ = [("kind", C.c_int), ("lambda0", C.c_double), ("lambda1", C.c_double),
                ("noise", C.c_double), ("anderson_depth", C.c_int), ("anderson_mix", C.c_double),
                ("anderson_start", C.c_int)]


class ps_solvent_config(C.Structure):
    _fields_ = [("field", C.c_int), ("volfrac", C.c_double), ("kind", C.c_int),
                ("charge_field", C.c_int), ("has_block_field", C.c_int), ("block_field", C.c_int),
                ("zc", C.c_double), ("neutral_factor", C.c_double)]


class ps_block_charge(C.Structure):
    _fields_ = [("charged", C.c_int), ("charge_field", C.c_int), ("za", C.c_double),
                ("alpha", C.c_double)]


class ps_config(C.Structure):
    _fields_ = [("n", C.c_int * 3), ("cell", C.c_double * 3), ("precision", C.c_int),
                ("n_fields", C.c_int), ("n_polymers", C.c_int),
                ("polymers", ps_polymer_config * PS_MAX_POLYMERS),
                ("n_interactions", C.c_int),
                ("interactions", ps_interaction_config * PS_MAX_INTERACTIONS),
                ("updater", ps_updater_config), ("seed", C.c_ulonglong),
                ("calc_disorder", C.c_int), ("device", C.c_int),
                ("n_solvents", C.c_int), ("solvents", ps_solvent_config * PS_MAX_SOLVENTS),
                ("n_charges", C.c_int),
                ("block_charge", (ps_block_charge * PS_MAX_BLOCKS) * PS_MAX_POLYMERS),
                ("polydisperse", ps_polydisperse_config * PS_MAX_POLYMERS)]


class ps_filter_config(C.Structure):
    _fields_ = [("n_fields", C.c_int), ("fields", C.c_int * PS_MAX_FIELDS),
                ("cutoff_factor", C.c_double), ("filter_strength", C.c_double),
                ("apply_start", C.c_longlong), ("apply_frequency", C.c_longlong),
                ("apply_end", C.c_longlong), ("spec_cells", C.c_int * 3), ("pad", C.c_int)]


class ps_poisson_config(C.Structure):
    _fields_ = [("n_fields", C.c_int), ("fields", C.c_int * PS_MAX_CHARGES),
                ("bjerrum_len", C.c_double), ("relaxlambda", C.c_double),
                ("apply_start", C.c_longlong), ("apply_frequency", C.c_longlong),
                ("apply_end", C.c_longlong)]


class ps_scalars(C.Structure):
    _fields_ = [("free_energy", C.c_double), ("free_energy_nodis", C.c_double),
                ("log_q", C.c_double * PS_MAX_POLYMERS), ("q", C.c_double * PS_MAX_POLYMERS),
                ("max_incomp", C.c_double), ("dh_norm", C.c_double),
                ("pressure_mean", C.c_double), ("iteration", C.c_longlong),
                ("error_flags", C.c_int)]

    def as_dict(self, n_polymers: int = PS_MAX_POLYMERS) -> dict:
        return {"free_energy": self.free_energy, "free_energy_nodis": self.free_energy_nodis,
                "log_q": list(self.log_q)[:n_polymers], "q": list(self.q)[:n_polymers],
                "max_incomp": self.max_incomp, "dh_norm": self.dh_norm,
                "pressure_mean": self.pressure_mean, "iteration": self.iteration,
                "error_flags": self.error_flags}


PKG_DIR = Path(__file__).resolve().parent
LIB_PATH = PKG_DIR / "_native" / "libpswift_b200.so"

# Every exported entry point of the C-ABI with (restype, argtypes).
_dbl_p = C.POINTER(C.c_double)
_vp = C.c_void_p
SIGNATURES = {
    "ps_version": (C.c_char_p, []),
    "ps_gpu_last_error": (C.c_char_p, [_vp]),
    "ps_gpu_create": (C.c_int, [C.POINTER(ps_config), C.POINTER(_vp)]),
    "ps_gpu_destroy": (C.c_int, [_vp]),
    "ps_gpu_block_steps": (C.c_int, [_vp, C.c_int, C.c_int, C.POINTER(C.c_int)]),
    "ps_gpu_set_fields": (C.c_int, [_vp, C.c_int, C.c_int, _vp, C.c_int]),
    "ps_gpu_get_fields": (C.c_int, [_vp, C.c_int, C.c_int, _vp, C.c_int]),
    "ps_gpu_init_random": (C.c_int, [_vp]),
    "ps_gpu_iterate": (C.c_int, [_vp, C.c_int]),
    "ps_gpu_get_scalars": (C.c_int, [_vp, C.POINTER(ps_scalars)]),
    "ps_gpu_get_propagator": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, C.c_int, _vp]),
    "ps_gpu_synchronize": (C.c_int, [_vp]),
    "ps_gpu_launches_per_iteration": (C.c_longlong, [_vp]),
    "ps_gpu_enable_sweep_timing": (C.c_int, [_vp, C.c_int]),
    "ps_gpu_stream": (_vp, [_vp]),
    "ps_gpu_set_variant": (C.c_int, [_vp, C.c_int]),
    "ps_gpu_get_variant": (C.c_int, [_vp, C.POINTER(C.c_int), C.POINTER(C.c_float), C.c_int]),
    "ps_gpu_set_precision": (C.c_int, [_vp, C.c_int]),
    "ps_gpu_set_spectral_filter": (C.c_int, [_vp, C.POINTER(ps_filter_config)]),
    "ps_gpu_apply_spectral_filter": (C.c_int, [_vp]),
    "ps_gpu_set_poisson": (C.c_int, [_vp, C.POINTER(ps_poisson_config)]),
    "ps_gpu_apply_poisson": (C.c_int, [_vp]),
    "ps_gpu_sweep_timing": (C.c_int, [_vp, _dbl_p, C.c_int, C.POINTER(C.c_int), _dbl_p,
                                      C.POINTER(C.c_longlong)]),
    "ps_gpu_batch_create": (C.c_int, [C.POINTER(ps_config), C.c_int, C.POINTER(_vp)]),
    "ps_gpu_batch_destroy": (C.c_int, [_vp]),
    "ps_gpu_batch_size": (C.c_int, [_vp]),
    "ps_gpu_batch_instance": (_vp, [_vp, C.c_int]),
    "ps_gpu_batch_iterate": (C.c_int, [_vp, C.c_int]),
    "ps_gpu_batch_set_variant": (C.c_int, [_vp, C.c_int]),
    "ps_gpu_batch_classes": (C.c_int, [_vp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_int,
                                       C.POINTER(C.c_int), C.c_int]),
    "ps_gpu_batch_launches_per_iteration": (C.c_longlong, [_vp]),
    "ps_gpu_batch_stream": (_vp, [_vp]),
    "ps_gpu_batch_last_error": (C.c_char_p, [_vp]),
    "ps_adj_create": (C.c_int, [C.POINTER(ps_config), C.c_int, C.POINTER(_vp)]),
    "ps_adj_create_polymer": (C.c_int, [C.POINTER(ps_config), C.c_int, C.c_int, C.c_int, C.POINTER(_vp)]),
    "ps_adj_species": (C.c_int, [_vp, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "ps_adj_set_potential": (C.c_int, [_vp, _vp]),
    "ps_adj_potential_grad": (C.c_int, [_vp, _vp]),
    "ps_adj_destroy": (C.c_int, [_vp]),
    "ps_adj_forward": (C.c_int, [_vp, _vp, _vp, _dbl_p]),
    "ps_adj_backward": (C.c_int, [_vp, _vp, C.c_double, _vp, _dbl_p, _dbl_p]),
    "ps_adj_info": (C.c_int, [_vp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_size_t)]),
    "ps_adj_stream": (_vp, [_vp]),
    "ps_adj_last_error": (C.c_char_p, [_vp]),
    "ps_fft_create": (C.c_int, [C.POINTER(C.c_int), C.c_int, C.c_int, C.POINTER(_vp)]),
    "ps_fft_destroy": (C.c_int, [_vp]),
    "ps_fft_size": (C.c_int, [_vp, C.POINTER(C.c_size_t)]),
    "ps_gpu_set_bulk_wait_limit": (C.c_int, [C.c_uint]),
    "ps_gpu_get_fields_async": (C.c_int, [_vp, C.c_int, C.c_int, _vp]),
    "ps_gpu_set_fields_async": (C.c_int, [_vp, C.c_int, C.c_int, _vp]),
    "ps_gpu_fields_wait": (C.c_int, [_vp]),
    "ps_fft_get_grid": (C.c_int, [_vp, C.POINTER(C.c_int)]),
    "ps_fft_scaled_pair": (C.c_int, [_vp, _vp, _vp, _vp]),
    "ps_fft_scaled_pair_im": (C.c_int, [_vp, _vp, _vp, _vp]),
    "ps_fft_convolve_re": (C.c_int, [_vp, _vp, _vp, _vp]),
    "ps_fft_forward_abs": (C.c_int, [_vp, _vp, _vp]),
    "ps_fft_forward": (C.c_int, [_vp, _vp, _vp]),
    "ps_fft_backward": (C.c_int, [_vp, _vp, _vp]),
    "ps_gauss_laguerre": (C.c_int, [C.c_int, C.c_double, _vp, _vp]),
    "ps_fft_last_error": (C.c_char_p, []),
    "ps_fft_scaled_pair_noalloc": (C.c_int, [C.POINTER(C.c_int), _vp, _vp, _vp, _vp]),
    "ps_fft_noalloc_scratch_bytes": (C.c_size_t, []),
    "ps_fft_noalloc_last_error": (C.c_char_p, []),
}

_lib = None


class PsError(RuntimeError):
    """A non-zero status from the C-ABI (code = the PS_* status)."""

    def __init__(self, code: int, message: str):
        super().__init__(f"{ERROR_NAMES.get(code, code)}: {message}")
        self.code = code


def load_library(path: Path | None = None) -> C.CDLL:
    """Load the native library (once).  Raises if it is missing: there is no CPU fallback."""
    global _lib
    if _lib is not None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise RuntimeError(f"native library {p} is missing; build it with "
                           "`python -m polyswift_plusplus_b200.build_native` or __graft_entry__.build()")
    lib = C.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(rc: int, handle=None, fft: bool = False, batch=None) -> None:
    if rc == PS_OK:
        return
    lib = load_library()
    if fft:
        msg = lib.ps_fft_last_error()
    elif batch is not None:
        msg = lib.ps_gpu_batch_last_error(batch)
    else:
        msg = lib.ps_gpu_last_error(handle)
    raise PsError(rc, (msg or b"").decode(errors="replace"))
