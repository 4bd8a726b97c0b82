"""scene.yaml loading and validation (the schema of chatcarlo/scene.py).

Checks the parts of the schema the transport path reads: the source
(explicit spectrum or kvp 20-150, focus position and direction, rect /
cone / parallel field, rotation), the geometry list (box / sphere /
cylinder with positive sizes, axis x/y/z, a known material; plus the
axis-aligned ``ellipsoid`` with ``semi_axes_cm``, an extension) and the
physics.fluorescence switch (scene.py:52-309).  Errors carry the path of
the offending entry, like ChatCarlo's SceneError.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import yaml

from . import tables as tb

VALID_SHAPES = {"box", "cylinder", "sphere", "ellipsoid"}
VALID_AXES = {"x", "y", "z"}
VALID_FIELDS = {"rect", "cone", "parallel"}


@dataclass
class SceneError:
    path: str
    message: str

    def __str__(self) -> str:
        return f"{self.path}: {self.message}"


@dataclass
class Scene:
    raw: dict
    errors: list = field(default_factory=list)
    warnings: list = field(default_factory=list)

    @property
    def ok(self) -> bool:
        return not self.errors


def _num(x) -> bool:
    return isinstance(x, (int, float)) and not isinstance(x, bool)


def _vec3(v, path, errors):
    if not (isinstance(v, (list, tuple)) and len(v) == 3 and all(_num(x) for x in v)):
        errors.append(SceneError(path, "expected a list of three numbers"))
        return None
    return [float(x) for x in v]


def _positive(g, key, path, errors):
    v = g.get(key)
    if not (_num(v) and v > 0):
        errors.append(SceneError(f"{path}.{key}", "must be a positive number"))


def load_scene(path: str) -> Scene:
    with open(path, encoding="utf-8") as f:
        raw = yaml.safe_load(f)
    return validate_scene(raw)


def validate_scene(raw) -> Scene:
    errors: list = []
    warnings: list = []
    scene = Scene(raw=raw, errors=errors, warnings=warnings)
    if not isinstance(raw, dict):
        errors.append(SceneError("(root)", "the YAML top level must be a mapping"))
        return scene
    src = raw.get("source")
    if src is None:
        errors.append(SceneError("source", "missing source section"))
    else:
        spectrum = src.get("spectrum")
        if spectrum is not None:
            if not (isinstance(spectrum, list) and spectrum and all(
                    isinstance(s, dict) and _num(s.get("energy_keV")) and s["energy_keV"] > 0
                    and _num(s.get("weight")) and s["weight"] > 0 for s in spectrum)):
                errors.append(SceneError("source.spectrum",
                                         "expected [{energy_keV: >0, weight: >0}, ...]"))
            elif any(s["energy_keV"] > tb.XS_GRID_MAX_KEV for s in spectrum):
                errors.append(SceneError("source.spectrum", "energy_keV above the 150 keV table limit"))
            for key in ("kvp", "mas", "ctdi_vol_mGy", "heel_effect"):
                if src.get(key):
                    errors.append(SceneError("source", f"source.spectrum cannot be combined with {key}"))
        else:
            kvp = src.get("kvp")
            if not (_num(kvp) and 20 <= kvp <= 150):
                errors.append(SceneError("source.kvp", f"kvp={kvp!r}: give a number in 20..150 or a spectrum"))
        _vec3(src.get("position"), "source.position", errors)
        d = _vec3(src.get("direction"), "source.direction", errors)
        if d is not None:
            n = math.sqrt(sum(x * x for x in d))
            if n < 1e-9:
                errors.append(SceneError("source.direction", "zero direction vector"))
            else:
                src["direction"] = [x / n for x in d]
        fld = src.get("field")
        if not isinstance(fld, dict):
            errors.append(SceneError("source.field", "missing field mapping"))
        else:
            shape = fld.get("shape", "rect")
            if shape not in VALID_FIELDS:
                errors.append(SceneError("source.field.shape", f"one of {sorted(VALID_FIELDS)}"))
            elif shape == "cone":
                _positive(fld, "diameter_cm", "source.field", errors)
                _positive(fld, "sid_cm", "source.field", errors)
            else:
                sz = fld.get("size_cm")
                if not (isinstance(sz, (list, tuple)) and len(sz) == 2 and all(_num(x) and x > 0 for x in sz)):
                    errors.append(SceneError("source.field.size_cm", "expected two positive numbers"))
                if shape == "rect":
                    _positive(fld, "sid_cm", "source.field", errors)
        rot = src.get("rotation")
        if rot is not None:
            if not isinstance(rot, dict):
                errors.append(SceneError("source.rotation", "expected a mapping"))
            else:
                _vec3(rot.get("isocenter"), "source.rotation.isocenter", errors)
                if rot.get("axis", "z") not in VALID_AXES:
                    errors.append(SceneError("source.rotation.axis", "x, y or z"))
    geoms = raw.get("geometry")
    if not isinstance(geoms, list) or not geoms:
        errors.append(SceneError("geometry", "expected a non-empty list of objects"))
    else:
        for i, g in enumerate(geoms):
            path = f"geometry[{i}]"
            if not isinstance(g, dict):
                errors.append(SceneError(path, "expected a mapping"))
                continue
            shape = g.get("shape")
            if shape not in VALID_SHAPES:
                errors.append(SceneError(f"{path}.shape", f"one of {sorted(VALID_SHAPES)}"))
                continue
            _vec3(g.get("center"), f"{path}.center", errors)
            if shape == "box":
                sz = g.get("size_cm")
                if not (isinstance(sz, (list, tuple)) and len(sz) == 3 and all(_num(x) and x > 0 for x in sz)):
                    errors.append(SceneError(f"{path}.size_cm", "expected three positive numbers"))
            elif shape == "ellipsoid":
                sa = g.get("semi_axes_cm")
                if not (isinstance(sa, (list, tuple)) and len(sa) == 3 and all(_num(x) and x > 0 for x in sa)):
                    errors.append(SceneError(f"{path}.semi_axes_cm", "expected three positive numbers"))
            else:
                _positive(g, "radius_cm", path, errors)
                if shape == "cylinder":
                    _positive(g, "height_cm", path, errors)
                    if g.get("axis", "z") not in VALID_AXES:
                        errors.append(SceneError(f"{path}.axis", "x, y or z"))
            mat = g.get("material")
            try:
                tb.resolve(str(mat))
            except ValueError as e:
                errors.append(SceneError(f"{path}.material", str(e)))
    phys = raw.get("physics")
    if phys is not None:
        if not isinstance(phys, dict):
            errors.append(SceneError("physics", "expected a mapping"))
        elif "fluorescence" in phys and not isinstance(phys["fluorescence"], bool):
            errors.append(SceneError("physics.fluorescence", "true or false"))
    return scene
