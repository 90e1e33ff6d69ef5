"""B200-native SCFT inner loop with the capabilities of PolySwift++'s hot path.

The propagator sweeps, contour quadrature, Q, free energy and field updates run
as hand-written sm_100a CUDA kernels in ``_native/libpswift_b200.so`` behind the
C-ABI of ``include/pswift.h``; this package is the Python side of that ABI.
"""
from . import _abi
from .config import (Block, Interaction, Polymer, ScftConfig, Solvent, Updater, config_from_file,
                     config_from_text)
from .scft import B200FFT, ScftBatch, ScftSolver

__all__ = ["Block", "Interaction", "Polymer", "ScftConfig", "Updater", "config_from_file",
           "config_from_text", "Solvent", "ScftSolver", "ScftBatch", "B200FFT", "_abi"]
