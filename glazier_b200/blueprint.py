"""The Blueprint reader: a JSON model description to a model and a start.

This is the host half of the drop-in boundary. It reads the same files the
reference engine reads and states what they mean the same way
(glazier-core/src/blueprint.rs), so a description runs unchanged on the
device engine:

- serde defaults and the cross-checks of ``Blueprint::from_json``
  (blueprint.rs:385-447),
- the adhesion fold of ``effective_contact`` (blueprint.rs:201-239),
- the in-order type shares of ``initial_types`` (blueprint.rs:247-261),
- the engine model of ``model`` (blueprint.rs:265-325),
- the start of ``simulation``: squares laid down from the origin, or a
  ``.npy`` label field (blueprint.rs:336-376, lattice.rs:169-196,
  cpu.rs:122-175).

Nothing here touches the device; the engine takes the flat arrays
``Model.flat()`` returns.
"""

from __future__ import annotations

import json
import math
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np


class BlueprintError(ValueError):
    """A description this reader refuses, with the reason."""


@dataclass
class CellType:
    """One cell type's parameters (model.rs:9-41). Every term is off at zero."""

    target_volume: float = 0.0
    lambda_volume: float = 0.0
    target_surface: float = 0.0
    lambda_surface: float = 0.0
    division_volume: float = 0.0
    death_rate: float = 0.0
    target_length: float = 0.0
    lambda_length: float = 0.0
    connected: bool = False
    max_activity: float = 0.0
    lambda_activity: float = 0.0
    external: tuple = (0.0, 0.0, 0.0)
    lambda_nematic: float = 0.0


@dataclass
class Species:
    """One diffusing species (field.rs:15-25)."""

    name: str
    diffusion: float
    decay: float = 0.0
    initial: float = 0.0


@dataclass
class Model:
    """The engine-facing model (model.rs:44-76), index 0 of every per-type
    list the medium."""

    width: int = 1
    height: int = 1
    depth: int = 1
    contact: list = field(default_factory=lambda: [0.0])
    types: list = field(default_factory=lambda: [CellType()])
    temperature: float = 10.0
    neighbour_order: int = 2
    seed: int = 0
    species: list = field(default_factory=list)
    secretion: list = field(default_factory=list)  # [type][species]
    uptake: list = field(default_factory=list)  # [type][species]
    chemotaxis: list = field(default_factory=list)  # [type][species]
    nematic: np.ndarray | None = None  # (sites, 2) float64 or None

    @property
    def n_types(self) -> int:
        return len(self.types)

    @property
    def sites(self) -> int:
        return self.width * self.height * self.depth

    def dimensions(self) -> int:
        return 3 if self.depth > 1 else 2

    def has_connectivity(self) -> bool:
        return any(t.connected for t in self.types)

    def has_length_constraint(self) -> bool:
        return any(t.lambda_length != 0.0 for t in self.types)

    def has_nematic(self) -> bool:
        return self.nematic is not None and any(t.lambda_nematic != 0.0 for t in self.types)

    def has_motility(self) -> bool:
        return any(t.lambda_activity != 0.0 and t.max_activity > 0.0 for t in self.types)

    def has_external_potential(self) -> bool:
        return any(any(v != 0.0 for v in t.external) for t in self.types)

    def has_population_events(self) -> bool:
        return any(t.division_volume > 0.0 or t.death_rate > 0.0 for t in self.types)

    def validate(self) -> None:
        """model.rs:160-232."""
        n = self.n_types
        if n == 0:
            raise BlueprintError("a model needs at least the medium type")
        if len(self.contact) != n * n:
            raise BlueprintError(f"contact matrix is {len(self.contact)} entries for {n} types, want {n * n}")
        for a in range(n):
            for b in range(n):
                if abs(self.contact[a * n + b] - self.contact[b * n + a]) > 1e-12:
                    raise BlueprintError(f"contact matrix is asymmetric at ({a}, {b})")
        if self.width == 0 or self.height == 0 or self.depth == 0:
            raise BlueprintError("the lattice has a zero dimension")
        if self.neighbour_order not in (1, 2, 3):
            raise BlueprintError(f"neighbour order {self.neighbour_order} is outside the range one to three")
        if self.temperature <= 0.0:
            raise BlueprintError("the temperature must be positive")
        if self.nematic is not None and len(self.nematic) != self.sites:
            raise BlueprintError(
                f"the nematic field has {len(self.nematic)} sites for a lattice of {self.sites}"
            )

    def per_type(self, name: str) -> np.ndarray:
        return np.array([getattr(t, name) for t in self.types], dtype=np.float64)

    def table(self, rows: list) -> np.ndarray:
        """A [type][species] table as a dense float64 array, missing entries 0."""
        out = np.zeros((self.n_types, len(self.species)), dtype=np.float64)
        for t, row in enumerate(rows[: self.n_types]):
            for s, v in enumerate(row[: len(self.species)]):
                out[t, s] = v
        return out


# ---------------------------------------------------------------- the file


_TYPE_DEFAULTS = {
    "secretion": {},
    "uptake": {},
    "chemotaxis": {},
    "presents": {},
    "target_surface": 0.0,
    "lambda_surface": 0.0,
    "division_volume": 0.0,
    "death_rate": 0.0,
    "target_length": 0.0,
    "lambda_length": 0.0,
    "connected": False,
    "max_activity": 0.0,
    "lambda_activity": 0.0,
    "external": [0.0, 0.0, 0.0],
    "lambda_nematic": 0.0,
}
_TYPE_REQUIRED = ("name", "target_volume", "lambda_volume")
_TOP_REQUIRED = (
    "name",
    "width",
    "height",
    "types",
    "contact",
    "temperature",
    "neighbour_order",
    "seed",
    "steps",
    "dump_every",
    "initial",
    "units",
)


def _require(obj: dict, keys, where: str) -> None:
    for k in keys:
        if k not in obj:
            raise BlueprintError(f"missing field `{k}` in {where}")


@dataclass
class Blueprint:
    """A parsed description (blueprint.rs:152-193)."""

    raw: dict

    @property
    def name(self) -> str:
        return self.raw["name"]

    @property
    def width(self) -> int:
        return int(self.raw["width"])

    @property
    def height(self) -> int:
        return int(self.raw["height"])

    @property
    def depth(self) -> int:
        return int(self.raw.get("depth", 1))

    @property
    def types(self) -> list:
        return self.raw["types"]

    @property
    def fields(self) -> list:
        return self.raw.get("fields", [])

    @property
    def steps(self) -> int:
        return int(self.raw["steps"])

    @property
    def dump_every(self) -> int:
        return int(self.raw["dump_every"])

    @property
    def initial(self) -> dict:
        return self.raw["initial"]

    @property
    def nematic_field(self):
        return self.raw.get("nematic_field")

    def infection_rule(self):
        """The optional `infection` object, an extension glazier's reader does
        not have: ``{"field": name, "from": type, "to": type, "threshold": x}``
        as (field index, from type, to type, threshold) in the engine's
        indices (type 0 the medium), or None."""
        spec = self.raw.get("infection")
        if spec is None:
            return None
        fields = [f["name"] for f in self.fields]
        names = [t["name"] for t in self.types]
        return (fields.index(spec["field"]), names.index(spec["from"]) + 1, names.index(spec["to"]) + 1,
                float(spec["threshold"]))

    @classmethod
    def from_json(cls, text: str) -> "Blueprint":
        """blueprint.rs:385-447: parse, fill serde defaults, cross-check."""
        try:
            raw = json.loads(text)
        except json.JSONDecodeError as e:
            raise BlueprintError(str(e)) from e
        if not isinstance(raw, dict):
            raise BlueprintError("a description is a JSON object")
        _require(raw, _TOP_REQUIRED, "the description")
        raw.setdefault("depth", 1)
        raw.setdefault("fields", [])
        raw.setdefault("adhesion", None)
        raw.setdefault("nematic_field", None)
        for spec in raw["types"]:
            _require(spec, _TYPE_REQUIRED, "a type")
            for k, v in _TYPE_DEFAULTS.items():
                spec.setdefault(k, json.loads(json.dumps(v)))
        for f in raw["fields"]:
            _require(f, ("name", "diffusion"), "a field")
            f.setdefault("decay", 0.0)
            f.setdefault("initial", 0.0)
        init = raw["initial"]
        _require(init, ("side", "nx", "ny"), "the initial condition")
        init.setdefault("nz", 1)
        init.setdefault("fractions", {})
        init.setdefault("labels", None)
        _require(raw["units"], ("micron_per_site", "minute_per_step"), "the units")

        bp = cls(raw)
        names = [t["name"] for t in bp.types]
        for name in init["fractions"]:
            if name not in names:
                raise BlueprintError(
                    f"the initial condition names the type {name}, which the description does not state"
                )
        adhesion = raw["adhesion"]
        if adhesion is not None:
            n = len(adhesion["molecules"])
            if len(adhesion["binding"]) != n * n:
                raise BlueprintError(
                    f"the binding matrix is {len(adhesion['binding'])} entries for {n} molecules, want {n * n}"
                )
            for spec in bp.types:
                for name in spec["presents"]:
                    if name not in adhesion["molecules"]:
                        raise BlueprintError(
                            f"type {spec['name']} presents {name}, which is not a molecule this description declares"
                        )
        else:
            for spec in bp.types:
                if spec["presents"]:
                    raise BlueprintError(
                        f"type {spec['name']} presents adhesion molecules, and the description declares none"
                    )
        known = [f["name"] for f in bp.fields]
        for spec in bp.types:
            for what in ("secretion", "uptake", "chemotaxis"):
                for name in spec[what]:
                    if name not in known:
                        raise BlueprintError(
                            f"type {spec['name']} states {what} of {name}, which is not a field this description declares"
                        )
        infection = raw.get("infection")
        if infection is not None:
            _require(infection, ("field", "from", "to", "threshold"), "the infection rule")
            if infection["field"] not in known:
                raise BlueprintError(f"the infection rule names the field {infection['field']}, which the description does not declare")
            for key in ("from", "to"):
                if infection[key] not in names:
                    raise BlueprintError(f"the infection rule names the type {infection[key]}, which the description does not state")
            if infection["from"] == infection["to"]:
                raise BlueprintError("the infection rule switches a type to itself")
            threshold = infection["threshold"]
            if not isinstance(threshold, (int, float)) or not threshold >= 0:
                raise BlueprintError("the infection threshold must be a number >= 0")
        bp.model().validate()
        return bp

    def effective_contact(self) -> list:
        """blueprint.rs:201-239: the contact matrix less what molecules bind."""
        contact = [float(v) for v in self.raw["contact"]]
        adhesion = self.raw.get("adhesion")
        if adhesion is None:
            return contact
        n_types = len(self.types) + 1
        mols = adhesion["molecules"]
        n = len(mols)

        def presented(index: int) -> list:
            if index == 0:
                return [0.0] * n
            return [float(self.types[index - 1]["presents"].get(m, 0.0)) for m in mols]

        molecules = [presented(i) for i in range(n_types)]
        for a in range(n_types):
            for b in range(n_types):
                bound = 0.0
                for i in range(n):
                    for j in range(n):
                        bound += adhesion["binding"][i * n + j] * molecules[a][i] * molecules[b][j]
                contact[a * n_types + b] -= bound
        return contact

    def initial_types(self, cells: int) -> np.ndarray:
        """blueprint.rs:247-261: each named type takes its rounded share, in order."""
        types = np.ones(cells, dtype=np.uint8)
        nxt = 0
        fractions = self.initial["fractions"]
        for index, spec in enumerate(self.types):
            if spec["name"] not in fractions:
                continue
            share = min(int(_round_half_away(fractions[spec["name"]] * cells)), cells - nxt)
            types[nxt : nxt + share] = index + 1
            nxt += share
        return types

    def model(self) -> Model:
        """blueprint.rs:265-325."""
        types = [CellType()]
        for t in self.types:
            types.append(
                CellType(
                    target_volume=float(t["target_volume"]),
                    lambda_volume=float(t["lambda_volume"]),
                    target_surface=float(t["target_surface"]),
                    lambda_surface=float(t["lambda_surface"]),
                    division_volume=float(t["division_volume"]),
                    death_rate=float(t["death_rate"]),
                    target_length=float(t["target_length"]),
                    lambda_length=float(t["lambda_length"]),
                    connected=bool(t["connected"]),
                    max_activity=float(t["max_activity"]),
                    lambda_activity=float(t["lambda_activity"]),
                    external=tuple(float(v) for v in t["external"]),
                    lambda_nematic=float(t["lambda_nematic"]),
                )
            )
        species = [
            Species(f["name"], float(f["diffusion"]), float(f["decay"]), float(f["initial"])) for f in self.fields
        ]

        def rates(m: dict) -> list:
            return [float(m.get(s.name, 0.0)) for s in species]

        secretion = [[0.0] * len(species)] + [rates(t["secretion"]) for t in self.types]
        uptake = [[0.0] * len(species)] + [rates(t["uptake"]) for t in self.types]
        chemotaxis = [[0.0] * len(species)] + [rates(t["chemotaxis"]) for t in self.types]
        return Model(
            width=self.width,
            height=self.height,
            depth=self.depth,
            contact=self.effective_contact(),
            types=types,
            temperature=float(self.raw["temperature"]),
            neighbour_order=int(self.raw["neighbour_order"]),
            seed=int(self.raw["seed"]),
            species=species,
            secretion=secretion,
            uptake=uptake,
            chemotaxis=chemotaxis,
        )

    def start(self, base: str | Path = ".") -> "Start":
        """blueprint.rs:336-376: the model with its nematic field read, the
        initial lattice and the type of every label."""
        base = Path(base)

        def resolve(name: str) -> Path:
            p = Path(name)
            return p if p.is_absolute() else base / p

        model = self.model()
        if self.nematic_field is not None:
            path = resolve(self.nematic_field)
            pairs = np.load(path).astype(np.float64)
            if pairs.shape[-1] != 2:
                raise BlueprintError(f"{path}: the last axis is {pairs.shape[-1]}, want 2")
            pairs = pairs.reshape(-1, 2)
            if len(pairs) != model.sites:
                raise BlueprintError(f"{path}: holds {len(pairs)} sites for a lattice of {model.sites}")
            model.nematic = pairs
        if self.initial["labels"] is not None:
            path = resolve(self.initial["labels"])
            arr = np.load(path)
            if arr.dtype.kind == "i" and (arr < 0).any():
                raise BlueprintError(f"{path}: a negative label")
            labels = arr.reshape(-1).astype(np.uint32)
            start = Start.from_labels(model, labels)
        else:
            init = self.initial
            start = Start.tiled_grid(model, int(init["side"]), int(init["nx"]), int(init["ny"]), int(init["nz"]))
        start.set_cell_types(self.initial_types(start.n_cells))
        return start


def _round_half_away(v: float) -> float:
    """Rust's f64::round: halves round away from zero."""
    return math.floor(v + 0.5) if v >= 0 else -math.floor(-v + 0.5)


@dataclass
class Start:
    """An initial lattice and the type of every label, index 0 the medium.

    The state ``Simulation::assemble`` (cpu.rs:178-217) builds before a run;
    volumes and surfaces are counted by the engine itself from the labels.
    """

    model: Model
    labels: np.ndarray  # uint32[sites], x fastest
    cell_type: np.ndarray  # uint8[n_labels]

    @property
    def n_cells(self) -> int:
        return len(self.cell_type) - 1

    @classmethod
    def tiled_grid(cls, model: Model, side: int, nx: int, ny: int, nz: int = 1) -> "Start":
        """cpu.rs:122-141 and lattice.rs:169-196: ``nx`` by ``ny`` (by ``nz``)
        squares of ``side`` from the origin, numbered x fastest, medium
        elsewhere."""
        model.validate()
        if model.n_types < 2:
            raise BlueprintError("a tiled start needs a cell type beside the medium")
        w, h, d = model.width, model.height, model.depth
        nx = min(nx, w // side)
        ny = min(ny, h // side)
        nz = 1 if d == 1 else min(nz, d // side)
        side_z = 1 if d == 1 else side
        labels = np.zeros((d, h, w), dtype=np.uint32)
        nxt = 1
        for bz in range(nz):
            for by in range(ny):
                for bx in range(nx):
                    labels[bz * side_z : (bz + 1) * side_z, by * side : (by + 1) * side, bx * side : (bx + 1) * side] = nxt
                    nxt += 1
        return cls(model, labels.reshape(-1), np.ones(nxt, dtype=np.uint8))

    @classmethod
    def tiled(cls, model: Model, side: int) -> "Start":
        """cpu.rs:109-116: as many squares as fit."""
        return cls.tiled_grid(model, side, model.width // side, model.height // side, max(model.depth // side, 1))

    @classmethod
    def from_labels(cls, model: Model, labels) -> "Start":
        """cpu.rs:151-175: every label from one to the largest is a cell of type 1."""
        model.validate()
        if model.n_types < 2:
            raise BlueprintError("a labelled start needs a cell type beside the medium")
        labels = np.ascontiguousarray(labels, dtype=np.uint32).reshape(-1)
        if len(labels) != model.sites:
            raise BlueprintError(f"the label field has {len(labels)} sites for a lattice of {model.sites}")
        n = int(labels.max()) if len(labels) else 0
        if n == 0:
            raise BlueprintError("the label field holds no cells")
        return cls(model, labels, np.ones(n + 1, dtype=np.uint8))

    def set_cell_types(self, types) -> None:
        """cpu.rs:220-224: the type of each cell in label order, from label 1."""
        types = np.asarray(types, dtype=np.uint8)
        k = min(len(types), self.n_cells)
        self.cell_type[1 : 1 + k] = types[:k]


def parse_dict(bp: Blueprint) -> dict:
    """What this engine read from a description: the keys and values of
    glazier-py's ``_native.parse`` (glazier-py/src/lib.rs:18-146)."""
    m = bp.model()
    per = lambda name: [getattr(t, name) for t in m.types]  # noqa: E731
    return {
        "name": bp.name,
        "width": m.width,
        "height": m.height,
        "depth": m.depth,
        "n_types": m.n_types,
        "contact": list(m.contact),
        "target_volume": per("target_volume"),
        "lambda_volume": per("lambda_volume"),
        "target_surface": per("target_surface"),
        "lambda_surface": per("lambda_surface"),
        "target_length": per("target_length"),
        "lambda_length": per("lambda_length"),
        "chemotaxis": [list(r) for r in m.chemotaxis],
        "division_volume": per("division_volume"),
        "death_rate": per("death_rate"),
        "species": [s.name for s in m.species],
        "diffusion": [s.diffusion for s in m.species],
        "decay": [s.decay for s in m.species],
        "secretion": [list(r) for r in m.secretion],
        "uptake": [list(r) for r in m.uptake],
        "lambda_nematic": per("lambda_nematic"),
        "nematic_field": bp.nematic_field,
        "temperature": m.temperature,
        "neighbour_order": m.neighbour_order,
        "seed": m.seed,
        "steps": bp.steps,
        "initial": [int(bp.initial["side"]), int(bp.initial["nx"]), int(bp.initial["ny"]), int(bp.initial["nz"])],
        "micron_per_site": float(bp.raw["units"]["micron_per_site"]),
        "minute_per_step": float(bp.raw["units"]["minute_per_step"]),
    }
