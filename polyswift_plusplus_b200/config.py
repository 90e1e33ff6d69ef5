"""SCFT instance description, mirroring the reference's input-file blocks.

The reference reads a txpp-expanded input file into a hierarchical attribute
set (``<Polymer name> ... </Polymer>`` etc.) and builds objects through its
maker maps.  The same blocks and keys are accepted here:

* ``<Grid>``: ``numCellsGlobal``, ``cellSizes`` (psgrid/PsUniCartGrid.cpp:30-43); the
  ``setupPS(nx, ny, nz, dx, dy, dz, debug)`` macro line of
  polyswift/psutils/macros/pseudoSpecSetup.mac:34-98 is expanded to it.
* ``<PhysField name> kind = monomerDens | constraint`` (psphysf/).
* ``<Polymer name> kind = blockCopolymer``: ``volfrac``, ``length``
  (psbase/PsPolymer.cpp:42-73) with ``<Block name> kind = flexPseudoSpec``:
  ``scfield``, ``ds``, ``lengthfrac``, ``headjoined``, ``tailjoined``,
  ``bSegRatio``, ``forceBlockSteps`` (psbase/PsBlockBase.cpp:67-145,
  pspolymer/PsFlexPseudoSpec.cpp:58-82).
* ``<EffHamil>`` with ``<Updater name> kind = steepestDescent``: ``relaxlambdas``,
  ``noise``, ``updatefields``, ``interactions`` (pseffhamil/PsSteepDUpdater.cpp:47-76)
  and ``<Interaction name> kind = flory``: ``chi``, ``scfields``
  (pseffhamil/PsFloryInteraction.cpp:65-89).
* top level: ``randomSeed``, ``nsteps``.

Added keys: ``kind = andersonMixing`` for ``<Updater>`` (``andersonDepth``,
``andersonMix``, ``andersonStart``), and top-level ``precision = fp64 | mixed``
and ``device``.  ``kind`` aliases ``blockCopolymerGPU`` / ``steepestDescentGPU`` /
``andersonGPU`` select the same device path.
"""
from __future__ import annotations

import ctypes as C
import math
import re
from dataclasses import dataclass, field
from pathlib import Path

from . import _abi as A


@dataclass
class Block:
    name: str
    scfield: str
    ds: float
    lengthfrac: float
    headjoined: list[str] = field(default_factory=lambda: ["freeEnd"])
    tailjoined: list[str] = field(default_factory=lambda: ["freeEnd"])
    bseg_ratio: float = 1.0
    force_block_steps: bool = False
    kind: str = "flexPseudoSpec"
    # chargeFlexPseudoSpec (pspolymer/PsChargeFlexPseudoSpec.cpp:42-75)
    chargefield: str | None = None
    za: float = 0.0
    alpha: float = 0.0


@dataclass
class Polymer:
    name: str
    volfrac: float
    length: int
    blocks: list[Block]
    kind: str = "blockCopolymer"
    # polyDisperseBCP (pspolymer/PsPolyDisperseBCP.cpp:41-100): Schulz exponent alpha,
    # n_g Gauss-Laguerre points, the polydisperse block's name
    n_g: int = 0
    schulz_alpha: float = 0.0
    polyblock: str | None = None

    @property
    def n_chains(self) -> int:
        return self.n_g if self.kind == "polyDisperseBCP" else 1


@dataclass
class Interaction:
    name: str
    chi: float
    scfields: list[str]
    kind: str = "flory"


@dataclass
class Solvent:
    """<Solvent name> kind = simpleSolvent | simpleIons (psbase/PsSolvent.cpp:40-60,
    pssolvent/PsSimpleIons.cpp:30-60)."""
    name: str
    scfield: str
    volfrac: float
    kind: str = "simpleSolvent"
    # simpleIons
    chargefield: str | None = None
    blockfield: str | None = None
    zc: float = 0.0
    neutral_factor: float = 0.0


@dataclass
class PoissonUpdater:
    """<Updater name> kind = poissonUpdater (pseffhamil/PsPoissonUpdater.cpp:50-95,
    psbase/PsUpdater.cpp:60-120)."""
    name: str = "poisson"
    updatefields: list = field(default_factory=list)   # chargeDens PhysFields
    bjerrum_len: float = 1.0
    relaxlambda: float = 1.0
    apply_start: int = 0
    apply_frequency: int = 1
    apply_end: int = -1

    def to_ps(self, cfg: "ScftConfig") -> A.ps_poisson_config:
        p = A.ps_poisson_config()
        if not 1 <= len(self.updatefields) <= A.PS_MAX_CHARGES:
            raise ValueError("poissonUpdater: updatefields out of range")
        p.n_fields = len(self.updatefields)
        for i, name in enumerate(self.updatefields):
            p.fields[i] = cfg.charge_index(name)
        p.bjerrum_len = float(self.bjerrum_len)
        p.relaxlambda = float(self.relaxlambda)
        p.apply_start = int(self.apply_start)
        p.apply_frequency = int(self.apply_frequency)
        p.apply_end = int(self.apply_end)
        return p


@dataclass
class SpecFilter:
    """<Updater name> kind = simpleSpecFilter | multiSpecFilter
    (pseffhamil/PsSpecFilterUpdater.cpp:56-90, pseffhamil/PsMultiSpecFilter.cpp:50-67,
    psbase/PsUpdater.cpp:60-120).  ``spec_cells`` (specCellSizes) is None for
    simpleSpecFilter."""
    name: str = "filter"
    spec_cells: tuple | None = None
    updatefields: list = field(default_factory=list)
    cutoff_factor: float = 0.0
    filter_strength: float = 0.0
    apply_start: int = 0
    apply_frequency: int = 1
    apply_end: int = -1

    def to_ps(self, cfg: "ScftConfig") -> A.ps_filter_config:
        f = A.ps_filter_config()
        f.n_fields = len(self.updatefields)
        for i, name in enumerate(self.updatefields):
            f.fields[i] = cfg.field_index(name)
        f.cutoff_factor = float(self.cutoff_factor)
        f.filter_strength = float(self.filter_strength)
        f.apply_start = int(self.apply_start)
        f.apply_frequency = int(self.apply_frequency)
        f.apply_end = int(self.apply_end)
        if self.spec_cells is not None:
            cells = [int(x) for x in self.spec_cells] + [1] * (3 - len(self.spec_cells))
            for d in range(3):
                f.spec_cells[d] = cells[d]
        return f


@dataclass
class Updater:
    name: str = "updater"
    kind: str = "steepestDescent"
    relaxlambdas: tuple[float, float] = (0.1, 0.05)
    noise: float = 0.0
    anderson_depth: int = 10
    anderson_mix: float = 0.1
    anderson_start: int = 0


@dataclass
class ScftConfig:
    n: tuple[int, int, int]
    cell: tuple[float, float, float]
    fields: list[str]                 # monomerDens PhysFields in declaration order
    polymers: list[Polymer]
    interactions: list[Interaction]
    updater: Updater = field(default_factory=Updater)
    seed: int = 0
    precision: str = "fp64"           # "fp64" or "mixed"
    nsteps: int = 1
    device: int = 0
    solvents: list = field(default_factory=list)  # Solvent entries
    spec_filter: "SpecFilter | None" = None       # simpleSpecFilter updater
    charge_fields: list = field(default_factory=list)  # chargeDens PhysFields in declaration order
    poisson: "PoissonUpdater | None" = None
    updater_sequence: list | None = None         # names; None: filter, then Poisson

    def post_updaters(self) -> list:
        """The updaters that run after the field updater, in updaterSequence order
        (pseffhamil/PsEffHamil.cpp:190-203): ("filter", SpecFilter) / ("poisson", PoissonUpdater)."""
        items = [(u.name, k, u) for k, u in (("filter", self.spec_filter), ("poisson", self.poisson))
                 if u is not None]
        if self.updater_sequence is not None:
            seq = list(self.updater_sequence)
            items = sorted((t for t in items if t[0] in seq), key=lambda t: seq.index(t[0]))
        return [(k, u) for _, k, u in items]

    def charge_index(self, name: str) -> int:
        try:
            return self.charge_fields.index(name)
        except ValueError as e:
            raise ValueError(f"unknown chargeDens PhysField {name!r}; declared: {self.charge_fields}") from e

    @property
    def n_total(self) -> int:
        return self.n[0] * self.n[1] * self.n[2]

    @property
    def box(self) -> tuple[float, float, float]:
        return tuple(self.n[d] * self.cell[d] for d in range(3))

    def field_index(self, name: str) -> int:
        try:
            return self.fields.index(name)
        except ValueError as e:
            raise ValueError(f"unknown PhysField {name!r}; declared: {self.fields}") from e

    def to_ps_config(self) -> A.ps_config:
        c = A.ps_config()
        for d in range(3):
            c.n[d] = int(self.n[d])
            c.cell[d] = float(self.cell[d])
        if self.precision not in ("fp64", "mixed"):
            raise ValueError("precision must be 'fp64' or 'mixed'")
        c.precision = A.PS_PREC_FP64 if self.precision == "fp64" else A.PS_PREC_MIXED
        c.n_fields = len(self.fields)
        if not 1 <= sum(P.n_chains for P in self.polymers) <= A.PS_MAX_POLYMERS:
            raise ValueError("number of polymers (counting polydisperse quadrature chains) out of range")
        c.n_polymers = len(self.polymers)
        for ip, P in enumerate(self.polymers):
            cp = c.polymers[ip]
            cp.volfrac = float(P.volfrac)
            cp.length = int(P.length)
            if not 1 <= len(P.blocks) <= A.PS_MAX_BLOCKS:
                raise ValueError(f"polymer {P.name}: number of blocks out of range")
            cp.n_blocks = len(P.blocks)
            names = [b.name for b in P.blocks]
            if P.kind == "polyDisperseBCP":
                d = c.polydisperse[ip]
                d.enabled = 1
                d.poly_block = names.index(P.polyblock)
                d.n_g = int(P.n_g)
                d.alpha = float(P.schulz_alpha)
            for ib, B in enumerate(P.blocks):
                cb = cp.blocks[ib]
                cb.field = self.field_index(B.scfield)
                cb.lengthfrac = float(B.lengthfrac)
                cb.ds = float(B.ds)
                cb.bseg_ratio = float(B.bseg_ratio)
                cb.force_block_steps = int(bool(B.force_block_steps))
                heads = [names.index(x) for x in B.headjoined if x != "freeEnd"]
                tails = [names.index(x) for x in B.tailjoined if x != "freeEnd"]
                if len(heads) > A.PS_MAX_JOINS or len(tails) > A.PS_MAX_JOINS:
                    raise ValueError("too many junctions on one block end")
                cb.n_head = len(heads)
                cb.n_tail = len(tails)
                for k, v in enumerate(heads):
                    cb.head_joined[k] = v
                for k, v in enumerate(tails):
                    cb.tail_joined[k] = v
                if B.chargefield is not None:
                    z = c.block_charge[ip][ib]
                    z.charged = 1
                    z.charge_field = self.charge_index(B.chargefield)
                    z.za = float(B.za)
                    z.alpha = float(B.alpha)
        if len(self.interactions) > A.PS_MAX_INTERACTIONS:
            raise ValueError("too many interactions")
        c.n_interactions = len(self.interactions)
        for it, I in enumerate(self.interactions):
            c.interactions[it].field_a = self.field_index(I.scfields[0])
            c.interactions[it].field_b = self.field_index(I.scfields[1])
            c.interactions[it].chi = float(I.chi)
        U = self.updater
        kind = U.kind.replace("GPU", "")
        if kind in ("steepestDescent",):
            c.updater.kind = A.PS_UPD_STEEPEST
        elif kind in ("andersonMixing", "anderson"):
            c.updater.kind = A.PS_UPD_ANDERSON
        else:
            raise ValueError(f"unknown updater kind {U.kind!r}")
        c.updater.lambda0 = float(U.relaxlambdas[0])
        c.updater.lambda1 = float(U.relaxlambdas[1]) if len(U.relaxlambdas) > 1 else 0.0
        c.updater.noise = float(U.noise)
        c.updater.anderson_depth = int(U.anderson_depth)
        c.updater.anderson_mix = float(U.anderson_mix)
        c.updater.anderson_start = int(U.anderson_start)
        if len(self.solvents) > A.PS_MAX_SOLVENTS:
            raise ValueError("too many solvents")
        c.n_solvents = len(self.solvents)
        if len(self.charge_fields) > A.PS_MAX_CHARGES:
            raise ValueError("too many chargeDens PhysFields")
        c.n_charges = len(self.charge_fields)
        for i_s, S in enumerate(self.solvents):
            cs = c.solvents[i_s]
            cs.field = self.field_index(S.scfield)
            cs.volfrac = float(S.volfrac)
            if S.kind in ("simpleSolvent", "simpleSolventGPU"):
                cs.kind = A.PS_SOLV_SIMPLE
            elif S.kind == "simpleIons":
                cs.kind = A.PS_SOLV_IONS
                cs.charge_field = self.charge_index(S.chargefield)
                if S.blockfield is not None:
                    cs.has_block_field = 1
                    cs.block_field = self.charge_index(S.blockfield)
                cs.zc = float(S.zc)
                cs.neutral_factor = float(S.neutral_factor)
            else:
                raise ValueError(f"Solvent kind {S.kind!r} is not on the device path")
        c.seed = int(self.seed) & 0xFFFFFFFFFFFFFFFF
        c.calc_disorder = 1
        c.device = int(self.device)
        return c


# ---------------------------------------------------------------------------
# Input-file parser (expanded .pre / .in subset)
# ---------------------------------------------------------------------------
_OPEN = re.compile(r"^<\s*(\w+)\s+(\w+)\s*>$")
_CLOSE = re.compile(r"^</\s*(\w+)\s*>$")
_SETUPPS = re.compile(r"^setupPS\s*\((.*)\)\s*$")


class InputError(ValueError):
    pass


def _value(tok: str, env: dict):
    tok = tok.strip()
    if tok.startswith("[") and tok.endswith("]"):
        return [_value(t, env) for t in tok[1:-1].split()]
    if tok in env:
        return env[tok]
    t = tok.strip("'\"")
    for conv in (int, float):
        try:
            return conv(t)
        except ValueError:
            pass
    return t


def parse_blocks(text: str) -> dict:
    """Parse into a nested dict {'attrs': {...}, 'blocks': [(type, name, node), ...]}."""
    env: dict = {}
    root = {"attrs": {}, "blocks": []}
    stack = [root]
    for raw in text.splitlines():
        line = raw.split("#", 1)[0].strip()
        if not line:
            continue
        if line.startswith("$"):
            body = line[1:].strip()
            if body.startswith("import"):
                continue
            if "=" in body:
                k, v = body.split("=", 1)
                env[k.strip()] = _value(v.strip().strip('"'), env)
            continue
        m = _SETUPPS.match(line)
        if m:
            args = [_value(a, env) for a in m.group(1).split(",")]
            if len(args) < 6:
                raise InputError("setupPS needs nx, ny, nz, dx, dy, dz")
            node = {"attrs": {"kind": "uniCartGrid",
                              "numCellsGlobal": [int(a) for a in args[:3]],
                              "cellSizes": [float(a) for a in args[3:6]]}, "blocks": []}
            stack[-1]["blocks"].append(("Grid", "mainGrid", node))
            continue
        m = _OPEN.match(line)
        if m:
            node = {"attrs": {}, "blocks": []}
            stack[-1]["blocks"].append((m.group(1), m.group(2), node))
            stack.append(node)
            continue
        m = _CLOSE.match(line)
        if m:
            if len(stack) == 1:
                raise InputError(f"unbalanced </{m.group(1)}>")
            stack.pop()
            continue
        if "=" in line:
            k, v = line.split("=", 1)
            stack[-1]["attrs"][k.strip()] = _value(v.strip(), env)
            continue
        raise InputError(f"cannot parse line: {raw!r}")
    if len(stack) != 1:
        raise InputError("unterminated block")
    return root


def _find(node: dict, typ: str) -> list:
    return [(n, b) for t, n, b in node["blocks"] if t == typ]


def config_from_text(text: str) -> ScftConfig:
    root = parse_blocks(text)
    ra = root["attrs"]
    grids = _find(root, "Grid")
    if not grids:
        raise InputError("no <Grid> block or setupPS(...) line")
    g = grids[0][1]["attrs"]
    n = tuple(int(v) for v in g["numCellsGlobal"])
    cell = tuple(float(v) for v in g["cellSizes"])
    fields, charge_fields, has_pressure = [], [], False
    for name, node in _find(root, "PhysField"):
        kind = node["attrs"].get("kind", "")
        if kind == "monomerDens":
            fields.append(name)
        elif kind == "chargeDens":
            charge_fields.append(name)
        elif kind == "constraint":
            has_pressure = True
        else:
            raise InputError(f"PhysField kind {kind!r} is not on the device path")
    if not has_pressure:
        raise InputError("a <PhysField defaultPressure> kind = constraint is required")
    polymers = []
    for pname, pnode in _find(root, "Polymer"):
        pa = pnode["attrs"]
        pkind = str(pa.get("kind", "blockCopolymer"))
        if pkind not in ("blockCopolymer", "blockCopolymerGPU", "polyDisperseBCP"):
            raise InputError(f"Polymer kind {pa.get('kind')!r} is not on the device path")
        pd = {}
        if pkind == "polyDisperseBCP":
            for key in ("alpha", "n_g", "polyblock"):
                if key not in pa:
                    raise InputError(f"PsPolyDisperseBCP::setAttrib: {key} not set in <Polymer {pname}>")
            pd = dict(kind=pkind, n_g=int(pa["n_g"]), schulz_alpha=float(pa["alpha"]),
                      polyblock=str(pa["polyblock"]))
        blocks = []
        for bname, bnode in _find(pnode, "Block"):
            ba = bnode["attrs"]
            bkind = str(ba.get("kind", "flexPseudoSpec"))
            if bkind not in ("flexPseudoSpec", "flexPseudoSpecGPU", "chargeFlexPseudoSpec"):
                raise InputError(f"Block kind {ba.get('kind')!r} is not on the device path")
            charge = {}
            if bkind == "chargeFlexPseudoSpec":
                for key in ("za", "alpha", "chargefield"):
                    if key not in ba:
                        raise InputError(f"PsChargeFlexPseudoSpec::setAttrib: {key} not set in <Block {bname}>")
                charge = dict(chargefield=str(ba["chargefield"]), za=float(ba["za"]),
                              alpha=float(ba["alpha"]))
            if "ds" not in ba:
                raise InputError(f"PsBlockBase::setAttrib: ds not set in <Block {bname}>")
            if "headjoined" not in ba or "tailjoined" not in ba:
                raise InputError(f"headjoined/tailjoined not set in <Block {bname}>")
            hj = ba["headjoined"] if isinstance(ba["headjoined"], list) else [ba["headjoined"]]
            tj = ba["tailjoined"] if isinstance(ba["tailjoined"], list) else [ba["tailjoined"]]
            fbs = ba.get("forceBlockSteps", 0)
            blocks.append(Block(name=bname, scfield=str(ba["scfield"]), ds=float(ba["ds"]),
                                lengthfrac=float(ba.get("lengthfrac", 0.0)),
                                headjoined=[str(x) for x in hj], tailjoined=[str(x) for x in tj],
                                bseg_ratio=float(ba.get("bSegRatio", 1.0)),
                                force_block_steps=fbs in (1, "on", "true", "1"), kind=bkind,
                                **charge))
        polymers.append(Polymer(name=pname, volfrac=float(pa.get("volfrac", 1.0)),
                                length=int(pa.get("length", 1)), blocks=blocks, **pd))
    solvents = []
    for sname, snode in _find(root, "Solvent"):
        sa = snode["attrs"]
        kind = str(sa.get("kind", "simpleSolvent"))
        if kind not in ("simpleSolvent", "simpleSolventGPU", "simpleIons"):
            raise InputError(f"Solvent kind {kind!r} is not on the device path")
        ions = {}
        if kind == "simpleIons":
            for key in ("zc", "neutralFactor", "chargefield"):
                if key not in sa:
                    raise InputError(f"PsSimpleIons::setAttrib: {key} not set in <Solvent {sname}>")
            ions = dict(chargefield=str(sa["chargefield"]), zc=float(sa["zc"]),
                        neutral_factor=float(sa["neutralFactor"]),
                        blockfield=str(sa["blockfield"]) if "blockfield" in sa else None)
        solvents.append(Solvent(name=sname, scfield=str(sa["scfield"]),
                                volfrac=float(sa.get("volfrac", 0.0)), kind=kind, **ions))
    interactions, updater, spec_filter, poisson, sequence = [], None, None, None, None
    for hname, hnode in _find(root, "EffHamil"):
        for iname, inode in _find(hnode, "Interaction"):
            ia = inode["attrs"]
            if ia.get("kind", "flory") != "flory":
                raise InputError(f"Interaction kind {ia.get('kind')!r} is not on the device path")
            interactions.append(Interaction(name=iname, chi=float(ia.get("chi", 0.01)),
                                            scfields=[str(x) for x in ia["scfields"]]))
        ups = _find(hnode, "Updater")
        fkinds = ("simpleSpecFilter", "multiSpecFilter")
        filters = [(n, u) for n, u in ups if str(u["attrs"].get("kind", "")) in fkinds]
        poissons = [(n, u) for n, u in ups if str(u["attrs"].get("kind", "")) == "poissonUpdater"]
        ups = [(n, u) for n, u in ups
               if str(u["attrs"].get("kind", "")) not in fkinds + ("poissonUpdater",)]
        # PsEffHamil::update runs the updaters named in updaterSequence, in its order
        # (pseffhamil/PsEffHamil.cpp:190-203)
        seq = hnode["attrs"].get("updaterSequence")
        seq = [str(x) for x in (seq if isinstance(seq, list) else [seq])] if seq is not None else None
        if seq is not None:
            sequence = seq
            filters = [(n, u) for n, u in filters if n in seq]
            poissons = [(n, u) for n, u in poissons if n in seq]
            if ups and ups[0][0] in seq:
                for uname_, _u in filters + poissons:
                    if seq.index(uname_) < seq.index(ups[0][0]):
                        raise InputError(f"updater {uname_!r} before the field updater in updaterSequence "
                                         "is not on the device path")
        if len(filters) > 1:
            raise InputError("one spectral filter per run is on the device path")
        if len(poissons) > 1:
            raise InputError("one poissonUpdater per run is on the device path")
        if poissons:
            pname, pnode = poissons[0]
            pa = pnode["attrs"]
            for key in ("relaxlambda", "bjerrumLen"):
                if key not in pa:
                    raise InputError(f"PsPoissonUpdater::setAttrib: {key} not set")
            upf = pa.get("updatefields", [])
            poisson = PoissonUpdater(name=pname, updatefields=[str(x) for x in (upf if isinstance(upf, list) else [upf])],
                                     bjerrum_len=float(pa["bjerrumLen"]),
                                     relaxlambda=float(pa["relaxlambda"]),
                                     apply_start=int(pa.get("applyStart", 0)),
                                     apply_frequency=int(pa.get("applyFrequency", 1)),
                                     apply_end=int(pa.get("applyEnd", -1)))
        if filters:
            fname, fnode = filters[0]
            fa = fnode["attrs"]
            upf = fa.get("updatefields", [])
            cells = None
            if str(fa["kind"]) == "multiSpecFilter":
                if "specCellSizes" not in fa:
                    raise InputError("PsMultiSpecFilter::setAttrib: specCellSizes not set")
                cells = tuple(int(x) for x in fa["specCellSizes"])
            spec_filter = SpecFilter(name=fname, updatefields=[str(x) for x in (upf if isinstance(upf, list) else [upf])],
                                     cutoff_factor=float(fa.get("cutoffFactor", 0.0)),
                                     filter_strength=float(fa.get("filterStrength", 0.0)),
                                     apply_start=int(fa.get("applyStart", 0)),
                                     apply_frequency=int(fa.get("applyFrequency", 1)),
                                     apply_end=int(fa.get("applyEnd", -1)), spec_cells=cells)
        if ups:
            uname, unode = ups[0]
            ua = unode["attrs"]
            lam = ua.get("relaxlambdas", [0.1, 0.05])
            updater = Updater(name=uname, kind=str(ua.get("kind", "steepestDescent")),
                              relaxlambdas=tuple(float(x) for x in lam),
                              noise=float(ua.get("noise", 0.0)),
                              anderson_depth=int(ua.get("andersonDepth", 10)),
                              anderson_mix=float(ua.get("andersonMix", 0.1)),
                              anderson_start=int(ua.get("andersonStart", 0)))
            upf = ua.get("updatefields")
            if upf is not None and [str(x) for x in upf] != fields:
                raise InputError("updatefields must list the monomerDens PhysFields in declaration order")
            names = [i.name for i in interactions]
            wanted = ua.get("interactions")
            if wanted is not None:
                interactions = [interactions[names.index(str(x))] for x in wanted]
    if updater is None:
        raise InputError("no <Updater> found")
    return ScftConfig(n=n, cell=cell, fields=fields, polymers=polymers, interactions=interactions,
                      updater=updater, seed=int(ra.get("randomSeed", 0)),
                      precision=str(ra.get("precision", "fp64")), nsteps=int(ra.get("nsteps", 1)),
                      device=int(ra.get("device", 0)), solvents=solvents, spec_filter=spec_filter,
                      charge_fields=charge_fields, poisson=poisson, updater_sequence=sequence)


def config_from_file(path: str | Path) -> ScftConfig:
    return config_from_text(Path(path).read_text())
