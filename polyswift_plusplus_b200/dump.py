"""Dump and restore of the SCFT state (PsPhysFldFuncs::dump / ::restore).

The reference writes, per PhysField, its density and conjugate field
(psphysf/PsPhysFldFuncs.cpp:116-166): "MonomerDensity" and "ConjugateDensity"
for a monomerDens field (psphysf/PsMonomerDens.cpp:22-26), "MonomerDensity"
and "PressureField" for the constraint (psphysf/PsConstraint.cpp:20-26), and
the free-energy History (pshist/PsHistHldr.cpp:124-164).  Its container is
HDF5 through txbase's TxIoBase, which is not part of this tree; here the same
datasets, keyed "<PhysField>/<dataset>" with the grid as (nx, ny, nz) arrays,
go into a numpy .npz file together with the grid, the cell sizes, the
iteration count and the free-energy history.

    from polyswift_plusplus_b200.dump import dump, restore
    dump(solver, "run_0100.npz", history=fe_history)
    restore(solver2, "run_0100.npz")        # same grid and fields
"""
from __future__ import annotations

from pathlib import Path

import numpy as np

from . import _abi as A

MONO_DENS = "MonomerDensity"
MONO_CONJ = "ConjugateDensity"
PRES = "PressureField"


def dump(solver, path, history=None, pressure_field: str = "defaultPressure") -> Path:
    """Write the fields of `solver` (an ScftSolver or a view of a batch instance)."""
    cfg = solver.cfg
    shape = tuple(int(v) for v in cfg.n)
    data = {"numCellsGlobal": np.array(shape, dtype=np.int64),
            "cellSizes": np.array(cfg.cell, dtype=np.float64),
            "physFields": np.array(list(cfg.fields) + [pressure_field]),
            "iteration": np.array(int(solver.scalars()["iteration"]), dtype=np.int64)}
    for i, name in enumerate(cfg.fields):
        data[f"{name}/{MONO_DENS}"] = np.asarray(solver.phi(i)).reshape(shape)
        data[f"{name}/{MONO_CONJ}"] = np.asarray(solver.w(i)).reshape(shape)
    data[f"{pressure_field}/{MONO_DENS}"] = np.zeros(shape)  # bulk: no wall density
    data[f"{pressure_field}/{PRES}"] = np.asarray(solver.pressure()).reshape(shape)
    if history is not None:
        data["freeEnergy"] = np.asarray(history, dtype=np.float64)
    path = Path(path)
    with open(path, "wb") as f:
        np.savez(f, **data)
    return path


class DumpError(ValueError):
    """A dump that cannot be restored: unreadable, truncated, or not this grid."""


def _read_dump(path, cfg, pressure_field: str) -> dict:
    """Read and check every dataset restore needs before anything is set."""
    shape = tuple(int(v) for v in cfg.n)
    out = {"w": [], "phi": []}
    try:
        with np.load(Path(path)) as d:
            if "numCellsGlobal" not in d:
                raise DumpError(f"{path}: no numCellsGlobal dataset")
            got = tuple(int(v) for v in d["numCellsGlobal"])
            if got != shape:
                raise DumpError(f"dump grid {got} does not match the solver grid {shape}")

            def field(key):
                a = np.asarray(d[key], dtype=np.float64)
                if a.shape != shape:
                    raise DumpError(f"{path}: {key} has shape {a.shape}, the grid is {shape}")
                if not np.all(np.isfinite(a)):
                    raise DumpError(f"{path}: {key} holds non-finite values")
                return a.reshape(-1).copy()

            for name in cfg.fields:
                key = f"{name}/{MONO_CONJ}"
                if key not in d:
                    raise DumpError(f"dump has no {key}")
                out["w"].append(field(key))
                dk = f"{name}/{MONO_DENS}"
                out["phi"].append(field(dk) if dk in d else None)
            pkey = f"{pressure_field}/{PRES}"
            out["p"] = field(pkey) if pkey in d else np.zeros(int(np.prod(shape)))
            out["meta"] = {
                "iteration": int(d["iteration"]) if "iteration" in d else 0,
                "freeEnergy": d["freeEnergy"].copy() if "freeEnergy" in d else None,
                "cellSizes": tuple(float(v) for v in d["cellSizes"]) if "cellSizes" in d else None}
    except DumpError:
        raise
    except Exception as e:  # truncated or corrupt container (zip, npy header, data)
        raise DumpError(f"{path}: unreadable dump ({type(e).__name__}: {e})") from e
    return out


def restore(solver, path, pressure_field: str = "defaultPressure") -> dict:
    """Set the conjugate fields, densities and pressure of `solver` from a dump;
    returns the dump's metadata (iteration, free-energy history).

    The whole file is read and checked first (grid, dataset shapes, finite
    values); an unreadable, truncated or mismatched dump raises DumpError and
    leaves the solver's fields as they were (PsPhysFldFuncs::restore,
    psphysf/PsPhysFldFuncs.cpp:150-166, reads each dataset of the dump)."""
    data = _read_dump(path, solver.cfg, pressure_field)
    for i in range(len(solver.cfg.fields)):
        solver.set_field(A.PS_FIELD_W, i, data["w"][i])
        if data["phi"][i] is not None:
            solver.set_field(A.PS_FIELD_PHI, i, data["phi"][i])
    solver.set_field(A.PS_FIELD_PRES, 0, data["p"])
    return data["meta"]
