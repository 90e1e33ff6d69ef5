"""The C-ABI library loads and exports every entry point include/pswift.h declares
(no compute calls: this runs without a GPU)."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import pytest

from polyswift_plusplus_b200 import _abi as A

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    names = []
    for h in sorted((ROOT / "include").glob("*.h")):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(ps_\w+)\s*\(", text, flags=re.M):
            names.append(m.group(1))
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ("ps_gpu_create", "ps_gpu_iterate", "ps_gpu_get_scalars", "ps_fft_scaled_pair"):
        assert must in names


def test_every_fft_interface_method_is_exported(native_lib):
    """Each pure virtual of PsFFTBase<T,3> (psbase/PsFFTBase.h:58-134) that
    computes something has a C-ABI entry point; buildData/buildSolvers map to
    ps_fft_create.  B200FFT exposes the same method names."""
    from polyswift_plusplus_b200.scft import B200FFT
    methods = {
        "getGrid": "ps_fft_get_grid",
        "getFFTSize": "ps_fft_size",
        "forwardFFTAbs": "ps_fft_forward_abs",
        "convolveRe": "ps_fft_convolve_re",
        "scaledFFTPair": "ps_fft_scaled_pair",
        "scaledFFTPairIm": "ps_fft_scaled_pair_im",
        "calcForwardFFT": "ps_fft_forward",
        "calcBackwardFFT": "ps_fft_backward",
        "buildSolvers": "ps_fft_create",
    }
    names = declared_functions()
    for method, sym in methods.items():
        assert sym in names, sym
        assert hasattr(native_lib, sym), sym
        if method != "buildSolvers":
            assert callable(getattr(B200FFT, method)), method


def test_library_exports_every_declared_symbol(native_lib):
    out = subprocess.run(["nm", "-D", "--defined-only", str(A.LIB_PATH)], capture_output=True,
                         text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = [n for n in declared_functions() if n not in exported]
    assert not missing, f"declared but not exported: {missing}"
    for n in declared_functions():
        assert hasattr(native_lib, n)
        assert n in A.SIGNATURES, f"{n} has no ctypes signature"


def test_version_string(native_lib):
    assert b"sm_100a" in native_lib.ps_version()


def test_struct_layout_matches_header(tmp_path):
    """Every ctypes field offset and struct size equals gcc's offsetof/sizeof."""
    structs = [A.ps_block_config, A.ps_polymer_config, A.ps_interaction_config,
               A.ps_updater_config, A.ps_solvent_config, A.ps_block_charge, A.ps_config,
               A.ps_filter_config, A.ps_poisson_config, A.ps_scalars]
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "pswift.h"', 'int main(void){']
    for s in structs:
        n = s.__name__
        lines.append(f'printf("{n} size %zu\\n", sizeof({n}));')
        for f in s._fields_:
            lines.append(f'printf("{n} {f[0]} %zu\\n", offsetof({n}, {f[0]}));')
    lines.append("return 0;}")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    got = {}
    for line in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines():
        a, b, c = line.split()
        got[(a, b)] = int(c)
    for s in structs:
        n = s.__name__
        assert got[(n, "size")] == C.sizeof(s), n
        for f in s._fields_:
            assert got[(n, f[0])] == getattr(s, f[0]).offset, (n, f[0])


def test_config_parser_reads_reference_style_input():
    from polyswift_plusplus_b200.config import config_from_text
    text = """
$ NX = 16
$ DX = 0.25
nsteps = 20
randomSeed = 38383
setupPS(NX, NX, NX, DX, DX, DX, "'off'")
<EffHamil mainHamil>
  kind = canonicalMF
  updaterSequence = [wAwB]
  <Updater wAwB>
    kind = steepestDescent
    relaxlambdas = [0.40 0.20]
    noise = 0.0
    updatefields = [totA totB]
    interactions = [AB]
  </Updater>
  <Interaction AB>
    kind = flory
    chi = 0.12
    scfields = [totA totB]
  </Interaction>
</EffHamil>
<PhysField totA>
  kind = monomerDens
  type = fieldD3R
</PhysField>
<PhysField totB>
  kind = monomerDens
  type = fieldD3R
</PhysField>
<PhysField defaultPressure>
  kind = constraint
  type = fieldD3R
</PhysField>
<Polymer diblock1>
  kind = blockCopolymer
  volfrac = 1.0
  length = 100
  <Block blockA>
    kind = flexPseudoSpec
    scfield = totA
    ds = 0.05
    lengthfrac = 0.5
    headjoined = [freeEnd]
    tailjoined = [blockB]
  </Block>
  <Block blockB>
    kind = flexPseudoSpec
    scfield = totB
    ds = 0.05
    lengthfrac = 0.5
    headjoined = [blockA]
    tailjoined = [freeEnd]
  </Block>
</Polymer>
<History freeE1>
  kind = freeEnergy
  updaterName = wAwB
</History>
"""
    cfg = config_from_text(text)
    assert cfg.n == (16, 16, 16) and cfg.cell == (0.25, 0.25, 0.25)
    assert cfg.fields == ["totA", "totB"] and cfg.seed == 38383 and cfg.nsteps == 20
    assert cfg.updater.relaxlambdas == (0.40, 0.20)
    pc = cfg.to_ps_config()
    assert pc.polymers[0].blocks[1].n_head == 1 and pc.polymers[0].blocks[1].head_joined[0] == 0
    assert pc.interactions[0].chi == pytest.approx(0.12)


def test_config_parser_reads_simple_solvent():
    """<Solvent name> kind = simpleSolvent (psbase/PsSolvent.cpp:40-60) with its
    scfield and volfrac reaches ps_config.solvents."""
    from polyswift_plusplus_b200.config import config_from_text
    text = """
setupPS(8, 8, 8, 0.25, 0.25, 0.25, "'off'")
<EffHamil h>
  <Updater u>
    kind = steepestDescent
    relaxlambdas = [0.1 0.05]
  </Updater>
  <Interaction AB>
    kind = flory
    chi = 0.2
    scfields = [A B]
  </Interaction>
</EffHamil>
<PhysField A>
  kind = monomerDens
</PhysField>
<PhysField B>
  kind = monomerDens
</PhysField>
<PhysField defaultPressure>
  kind = constraint
</PhysField>
<Polymer homoB>
  kind = blockCopolymer
  volfrac = 0.7
  length = 100
  <Block b>
    scfield = B
    ds = 0.01
    lengthfrac = 1.0
    headjoined = [freeEnd]
    tailjoined = [freeEnd]
  </Block>
</Polymer>
<Solvent solvA>
  kind = simpleSolvent
  scfield = A
  volfrac = 0.3
</Solvent>
"""
    cfg = config_from_text(text)
    assert len(cfg.solvents) == 1 and cfg.solvents[0].scfield == "A"
    pc = cfg.to_ps_config()
    assert pc.n_solvents == 1 and pc.solvents[0].field == 0
    assert pc.solvents[0].volfrac == pytest.approx(0.3)


def test_dump_restore_round_trip_on_host(tmp_path):
    """The dump keeps the reference's per-PhysField datasets and restore puts every
    field back (a host-side stand-in for the solver: no GPU needed)."""
    import numpy as np

    from polyswift_plusplus_b200 import workloads as W
    from polyswift_plusplus_b200.dump import dump, restore

    class Stub:
        def __init__(self, cfg, seed):
            rng = np.random.default_rng(seed)
            self.cfg = cfg
            self.f = {A.PS_FIELD_W: [rng.standard_normal(cfg.n_total) for _ in cfg.fields],
                      A.PS_FIELD_PHI: [rng.random(cfg.n_total) for _ in cfg.fields],
                      A.PS_FIELD_PRES: [rng.standard_normal(cfg.n_total)]}

        def w(self, i): return self.f[A.PS_FIELD_W][i]
        def phi(self, i): return self.f[A.PS_FIELD_PHI][i]
        def pressure(self): return self.f[A.PS_FIELD_PRES][0]
        def scalars(self): return {"iteration": 42}
        def set_field(self, which, i, x): self.f[which][i] = np.array(x)

    cfg, _ = W.diblock32(n=8)
    a, b = Stub(cfg, 1), Stub(cfg, 2)
    p = dump(a, tmp_path / "d.npz", history=[1.0, 0.5])
    with np.load(p) as d:
        assert "A/MonomerDensity" in d and "B/ConjugateDensity" in d
        assert "defaultPressure/PressureField" in d and d["A/ConjugateDensity"].shape == (8, 8, 8)
    meta = restore(b, p)
    assert meta["iteration"] == 42 and list(meta["freeEnergy"]) == [1.0, 0.5]
    for which in a.f:
        for x, y in zip(a.f[which], b.f[which]):
            assert np.array_equal(x, y)


def test_bad_dumps_raise_and_leave_the_solver_untouched(tmp_path):
    """A truncated file, a corrupt byte range, another grid, a missing dataset,
    a wrongly shaped or non-finite dataset: each raises DumpError before any
    field is set (the reference's restore reads every dataset it needs,
    psphysf/PsPhysFldFuncs.cpp:150-166)."""
    import numpy as np

    from polyswift_plusplus_b200 import workloads as W
    from polyswift_plusplus_b200.dump import DumpError, dump, restore

    class Stub:
        def __init__(self, cfg, seed):
            rng = np.random.default_rng(seed)
            self.cfg = cfg
            self.sets = 0
            self.f = {A.PS_FIELD_W: [rng.standard_normal(cfg.n_total) for _ in cfg.fields],
                      A.PS_FIELD_PHI: [rng.random(cfg.n_total) for _ in cfg.fields],
                      A.PS_FIELD_PRES: [rng.standard_normal(cfg.n_total)]}

        def w(self, i): return self.f[A.PS_FIELD_W][i]
        def phi(self, i): return self.f[A.PS_FIELD_PHI][i]
        def pressure(self): return self.f[A.PS_FIELD_PRES][0]
        def scalars(self): return {"iteration": 7}

        def set_field(self, which, i, x):
            self.sets += 1
            self.f[which][i] = np.array(x)

    cfg, _ = W.diblock32(n=8)
    good = dump(Stub(cfg, 1), tmp_path / "good.npz")
    raw = good.read_bytes()
    bad = {}
    bad["truncated"] = tmp_path / "trunc.npz"
    bad["truncated"].write_bytes(raw[: len(raw) // 2])
    bad["corrupt"] = tmp_path / "corrupt.npz"
    bad["corrupt"].write_bytes(raw[:200] + bytes(1000) + raw[1200:])
    bad["empty"] = tmp_path / "empty.npz"
    bad["empty"].write_bytes(b"")
    cfg16, _ = W.diblock32(n=16)
    bad["grid"] = dump(Stub(cfg16, 2), tmp_path / "grid.npz")
    with np.load(good) as d:
        items = {k: d[k] for k in d.files}
    drop = dict(items)
    del drop["B/ConjugateDensity"]
    bad["missing"] = tmp_path / "missing.npz"
    np.savez(bad["missing"], **drop)
    shaped = dict(items)
    shaped["B/ConjugateDensity"] = shaped["B/ConjugateDensity"][:4]
    bad["shape"] = tmp_path / "shape.npz"
    np.savez(bad["shape"], **shaped)
    nonfin = dict(items)
    nonfin["defaultPressure/PressureField"] = nonfin["defaultPressure/PressureField"].copy()
    nonfin["defaultPressure/PressureField"][1, 2, 3] = np.nan
    bad["nan"] = tmp_path / "nan.npz"
    np.savez(bad["nan"], **nonfin)
    bad["absent"] = tmp_path / "no_such_file.npz"

    target = Stub(cfg, 3)
    before = {k: [x.copy() for x in v] for k, v in target.f.items()}
    for name, path in bad.items():
        with pytest.raises(DumpError):
            restore(target, path)
        assert target.sets == 0, name
    for which in before:
        for x, y in zip(before[which], target.f[which]):
            assert np.array_equal(x, y)
    restore(target, good)  # the same target still takes a good dump
    assert target.sets == 2 * len(cfg.fields) + 1


_SPEC_FILTER_DECK = """
setupPS(8, 8, 8, 0.25, 0.25, 0.25, "'off'")
<EffHamil h>
  <Updater u>
    kind = steepestDescent
    relaxlambdas = [0.1 0.05]
  </Updater>
  <Updater filt>
    kind = simpleSpecFilter
    updatefields = [B A]
    cutoffFactor = 0.02
    filterStrength = 0.1
    applyStart = 5
    applyFrequency = 10
    applyEnd = 200
    fftKind = fftw3
  </Updater>
  <Interaction AB>
    kind = flory
    chi = 0.2
    scfields = [A B]
  </Interaction>
</EffHamil>
<PhysField A>
  kind = monomerDens
</PhysField>
<PhysField B>
  kind = monomerDens
</PhysField>
<PhysField defaultPressure>
  kind = constraint
</PhysField>
<Polymer di>
  kind = blockCopolymer
  volfrac = 1.0
  length = 100
  <Block a>
    kind = flexPseudoSpec
    scfield = A
    ds = 0.05
    lengthfrac = 0.3
    headjoined = [freeEnd]
    tailjoined = [b]
  </Block>
  <Block b>
    kind = flexPseudoSpec
    scfield = B
    ds = 0.05
    lengthfrac = 0.7
    headjoined = [a]
    tailjoined = [freeEnd]
  </Block>
</Polymer>
"""


def test_config_parser_reads_simple_spec_filter():
    """<Updater name> kind = simpleSpecFilter (pseffhamil/PsSpecFilterUpdater.cpp:55-90 and
    psbase/PsUpdater.cpp:55-110) beside the field updater."""
    from polyswift_plusplus_b200.config import config_from_text
    text = _SPEC_FILTER_DECK
    cfg = config_from_text(text)
    assert cfg.updater.kind == "steepestDescent"
    f = cfg.spec_filter
    assert f.updatefields == ["B", "A"]
    assert (f.cutoff_factor, f.filter_strength) == (0.02, 0.1)
    assert (f.apply_start, f.apply_frequency, f.apply_end) == (5, 10, 200)
    pf = f.to_ps(cfg)
    assert pf.n_fields == 2 and list(pf.fields[:2]) == [1, 0]


def test_config_parser_multi_spec_filter_and_updater_sequence():
    """multiSpecFilter with specCellSizes (pseffhamil/PsMultiSpecFilter.cpp:50-67); a filter
    runs only when updaterSequence names it (pseffhamil/PsEffHamil.cpp:190-203)."""
    from polyswift_plusplus_b200.config import InputError, config_from_text
    base = _SPEC_FILTER_DECK
    deck = base.replace("kind = simpleSpecFilter", "kind = multiSpecFilter\n    specCellSizes = [4 4 1]")
    cfg = config_from_text(deck.replace("<EffHamil h>", "<EffHamil h>\n  updaterSequence = [u filt]"))
    assert cfg.spec_filter.spec_cells == (4, 4, 1)
    pf = cfg.spec_filter.to_ps(cfg)
    assert list(pf.spec_cells) == [4, 4, 1]
    cfg = config_from_text(deck.replace("<EffHamil h>", "<EffHamil h>\n  updaterSequence = [u]"))
    assert cfg.spec_filter is None
    with pytest.raises(InputError):
        config_from_text(deck.replace("<EffHamil h>", "<EffHamil h>\n  updaterSequence = [filt u]"))
    with pytest.raises(InputError):
        config_from_text(base.replace("kind = simpleSpecFilter", "kind = multiSpecFilter"))


def test_config_parser_reads_charged_deck():
    """chargeDens PhysFields, a chargeFlexPseudoSpec block, simpleIons and a
    poissonUpdater after the field updater, as in the reference's charged test deck."""
    from polyswift_plusplus_b200.config import config_from_text
    text = """
setupPS(16, 16, 1, 0.05, 0.05, 0.05, "'off'")
<EffHamil mainHamil>
  updaterSequence = [wAwB ePotential]
  <Updater ePotential>
    kind = poissonUpdater
    fftKind = fftWObj
    applyFrequency = 5
    relaxlambda = 1.0
    bjerrumLen = 5.68
    updatefields = [ totChargeDens ]
  </Updater>
  <Updater wAwB>
    kind = steepestDescent
    relaxlambdas = [0.20 0.10]
    updatefields = [totStyrDens totEthyDens]
  </Updater>
  <Interaction StyrEthy>
     kind = flory
     chi = 0.0114
     scfields = [totStyrDens totEthyDens]
  </Interaction>
</EffHamil>
<PhysField totStyrDens>
   kind = monomerDens
</PhysField>
<PhysField totEthyDens>
   kind = monomerDens
</PhysField>
<PhysField totChargeDens>
   kind = chargeDens
</PhysField>
<PhysField counterIonDens>
   kind = chargeDens
</PhysField>
<PhysField defaultPressure>
   kind = constraint
</PhysField>
<Solvent counterIons>
  kind = simpleIons
  volfrac = 0.0
  zc = -1.0
  neutralFactor = 0.005
  scfield = totStyrDens
  chargefield = totChargeDens
  blockfield = counterIonDens
</Solvent>
<Polymer diblock1>
  kind = blockCopolymer
  volfrac = 1.0
  length = 1000
  <Block blockA>
    kind = chargeFlexPseudoSpec
    scfield = totStyrDens
    chargefield = totChargeDens
    za = 1.0
    alpha = 0.01
    ds = 0.05
    lengthfrac = 0.5
    headjoined = [freeEnd]
    tailjoined = [blockB]
  </Block>
  <Block blockB>
    kind = flexPseudoSpec
    scfield = totEthyDens
    ds = 0.05
    lengthfrac = 0.50
    headjoined = [blockA]
    tailjoined = [freeEnd]
  </Block>
</Polymer>
"""
    cfg = config_from_text(text)
    assert cfg.charge_fields == ["totChargeDens", "counterIonDens"]
    assert cfg.poisson.updatefields == ["totChargeDens"] and cfg.poisson.apply_frequency == 5
    assert [k for k, _ in cfg.post_updaters()] == ["poisson"]
    pc = cfg.to_ps_config()
    assert pc.n_charges == 2
    z = pc.block_charge[0][0]
    assert (z.charged, z.charge_field, z.za, z.alpha) == (1, 0, 1.0, 0.01)
    assert pc.block_charge[0][1].charged == 0
    s = pc.solvents[0]
    assert (s.kind, s.charge_field, s.has_block_field, s.block_field) == (A.PS_SOLV_IONS, 0, 1, 1)
    assert (s.zc, s.neutral_factor) == (-1.0, 0.005)
    pp = cfg.poisson.to_ps(cfg)
    assert pp.n_fields == 1 and pp.fields[0] == 0 and pp.bjerrum_len == 5.68


def test_config_parser_reads_polydisperse_polymer():
    """<Polymer> kind = polyDisperseBCP with alpha, n_g and polyblock
    (pspolymer/PsPolyDisperseBCP.cpp:41-100)."""
    from polyswift_plusplus_b200.config import config_from_text
    text = """
setupPS(16, 16, 1, 0.2, 0.2, 0.2, "'off'")
<EffHamil mainHamil>
  updaterSequence = [wAwB]
  <Updater wAwB>
    kind = steepestDescent
    relaxlambdas = [0.20 0.10]
    updatefields = [totStyrDens totEthyDens]
  </Updater>
  <Interaction StyrEthy>
    kind = flory
    chi = 0.12
    scfields = [totStyrDens totEthyDens]
  </Interaction>
</EffHamil>
<PhysField totStyrDens>
  kind = monomerDens
</PhysField>
<PhysField totEthyDens>
  kind = monomerDens
</PhysField>
<PhysField defaultPressure>
  kind = constraint
</PhysField>
<Polymer diblock1>
  kind = polyDisperseBCP
  n_g = 4
  alpha = 1.5
  polyblock = blockB
  volfrac = 1.0
  length = 100
  <Block blockA>
    kind = flexPseudoSpec
    scfield = totStyrDens
    forceBlockSteps = true
    ds = 0.02
    lengthfrac = 0.7
    headjoined = [freeEnd]
    tailjoined = [blockB]
  </Block>
  <Block blockB>
    kind = flexPseudoSpec
    scfield = totEthyDens
    ds = 0.01
    forceBlockSteps = true
    lengthfrac = 0.3
    headjoined = [blockA]
    tailjoined = [freeEnd]
  </Block>
</Polymer>
"""
    cfg = config_from_text(text)
    P = cfg.polymers[0]
    assert (P.kind, P.n_g, P.schulz_alpha, P.polyblock) == ("polyDisperseBCP", 4, 1.5, "blockB")
    pc = cfg.to_ps_config()
    d = pc.polydisperse[0]
    assert (d.enabled, d.poly_block, d.n_g, d.alpha) == (1, 1, 4, 1.5)


def test_config_parser_reads_star_polymer():
    """The reference's three-arm star: every arm's tail lists the two others."""
    from polyswift_plusplus_b200.config import config_from_text
    text = """
setupPS(8, 8, 8, 0.25, 0.25, 0.25, "'off'")
<EffHamil h>
  <Updater u>
    kind = steepestDescent
    relaxlambdas = [0.1 0.05]
  </Updater>
  <Interaction AB>
    kind = flory
    chi = 0.15
    scfields = [A B]
  </Interaction>
</EffHamil>
<PhysField A>
  kind = monomerDens
</PhysField>
<PhysField B>
  kind = monomerDens
</PhysField>
<PhysField C>
  kind = monomerDens
</PhysField>
<PhysField defaultPressure>
  kind = constraint
</PhysField>
<Polymer threeArmABC>
  kind = blockCopolymer
  volfrac = 1.0
  length = 100
  <Block blockA>
    kind = flexPseudoSpec
    scfield = A
    ds = 0.01
    lengthfrac = 0.3
    headjoined = [freeEnd]
    tailjoined = [blockB blockC]
  </Block>
  <Block blockB>
    kind = flexPseudoSpec
    scfield = B
    ds = 0.01
    lengthfrac = 0.3
    headjoined = [freeEnd]
    tailjoined = [blockA blockC]
  </Block>
  <Block blockC>
    kind = flexPseudoSpec
    scfield = C
    ds = 0.01
    lengthfrac = 0.4
    headjoined = [freeEnd]
    tailjoined = [blockA blockB]
  </Block>
</Polymer>
"""
    cfg = config_from_text(text)
    pc = cfg.to_ps_config()
    blocks = pc.polymers[0].blocks
    assert [(b.n_head, b.n_tail) for b in list(blocks)[:3]] == [(0, 2), (0, 2), (0, 2)]
    assert list(blocks[0].tail_joined[:2]) == [1, 2] and list(blocks[2].tail_joined[:2]) == [0, 1]
