"""Scene geometry on the host: primitives in list order, world box, packing.

Mirrors ChatCarlo's ``Geometry`` (chatcarlo/geometry.py:121-231): box,
sphere and finite cylinder (axis x/y/z) primitives, plus an axis-aligned
``ellipsoid`` (``semi_axes_cm``) that the reference does not have and the
learned-denoiser phantoms need; where they overlap the
later one in the list wins; everything else is the background material;
the world is the bounding box of all primitives grown by bbox_margin_cm
(geometry.py:137-164).  Ray tracing happens in the engine; the host keeps
point location for post-processing (dose per voxel centre) and packs the
primitives for the device.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import _native as N

AXES = {"x": 0, "y": 1, "z": 2}
SHAPES = {"box": N.CC_SHAPE_BOX, "sphere": N.CC_SHAPE_SPHERE, "cylinder": N.CC_SHAPE_CYLINDER,
          "ellipsoid": N.CC_SHAPE_ELLIPSOID}


def shape_bbox(g: dict) -> tuple[np.ndarray, np.ndarray]:
    c = np.asarray(g["center"], dtype=float)
    shape = g["shape"]
    if shape == "box":
        half = np.asarray(g["size_cm"], dtype=float) / 2
        return c - half, c + half
    if shape == "sphere":
        r = g["radius_cm"]
        return c - r, c + r
    if shape == "ellipsoid":
        s = np.asarray(g["semi_axes_cm"], dtype=float)
        return c - s, c + s
    if shape == "cylinder":
        ai = AXES[g.get("axis", "z")]
        r, h = g["radius_cm"], g["height_cm"]
        lo, hi = c.copy(), c.copy()
        for k in range(3):
            ext = h / 2 if k == ai else r
            lo[k] -= ext
            hi[k] += ext
        return lo, hi
    raise ValueError(f"unknown shape: {shape}")


def contains(g: dict, points: np.ndarray) -> np.ndarray:
    c = np.asarray(g["center"], dtype=float)
    shape = g["shape"]
    if shape == "box":
        half = np.asarray(g["size_cm"], dtype=float) / 2
        return np.all((points >= c - half) & (points <= c + half), axis=1)
    if shape == "sphere":
        return np.sum((points - c) ** 2, axis=1) <= g["radius_cm"] ** 2
    if shape == "ellipsoid":
        return np.sum(((points - c) / np.asarray(g["semi_axes_cm"], dtype=float)) ** 2, axis=1) <= 1.0
    if shape == "cylinder":
        ai = AXES[g.get("axis", "z")]
        oi = [k for k in range(3) if k != ai]
        r2 = (points[:, oi[0]] - c[oi[0]]) ** 2 + (points[:, oi[1]] - c[oi[1]]) ** 2
        return (r2 <= g["radius_cm"] ** 2) & (np.abs(points[:, ai] - c[ai]) <= g["height_cm"] / 2)
    raise ValueError(f"unknown shape: {shape}")


@dataclass
class Geometry:
    geoms: list
    background: str = "air"
    bbox_margin_cm: float = 50.0
    bbox_min: np.ndarray = field(init=False)
    bbox_max: np.ndarray = field(init=False)

    def __post_init__(self):
        if not self.geoms:
            raise ValueError("geometry needs at least one primitive")
        los, his = zip(*(shape_bbox(g) for g in self.geoms))
        self.bbox_min = np.min(np.stack(los), axis=0) - self.bbox_margin_cm
        self.bbox_max = np.max(np.stack(his), axis=0) + self.bbox_margin_cm

    def materials(self) -> list[str]:
        """Materials in first-use order, the background first."""
        names = [self.background]
        for g in self.geoms:
            if g["material"] not in names:
                names.append(g["material"])
        return names

    def material_at(self, points: np.ndarray) -> np.ndarray:
        mat = np.full(points.shape[0], self.background, dtype=object)
        for g in self.geoms:
            m = contains(g, points)
            if np.any(m):
                mat[m] = g["material"]
        return mat

    def nearest_object_distance_cm(self, point) -> float | None:
        pos = np.asarray(point, dtype=float)
        dists = []
        for g in self.geoms:
            lo, hi = shape_bbox(g)
            dists.append(float(np.linalg.norm(pos - np.clip(pos, lo, hi))))
        return min(dists) if dists else None

    def primitives(self, material_index: dict) -> "N.Primitive * n":
        arr = (N.Primitive * len(self.geoms))()
        for i, g in enumerate(self.geoms):
            p = arr[i]
            if g["shape"] not in SHAPES:
                raise ValueError(f"unknown shape: {g['shape']}")
            p.type = SHAPES[g["shape"]]
            p.material = material_index[g["material"]]
            p.axis = AXES[g.get("axis", "z")]
            for k in range(3):
                p.center[k] = float(g["center"][k])
            if g["shape"] == "box":
                for k in range(3):
                    p.size[k] = float(g["size_cm"][k])
            elif g["shape"] == "ellipsoid":
                for k in range(3):
                    p.size[k] = 2.0 * float(g["semi_axes_cm"][k])
            else:
                p.radius = float(g["radius_cm"])
                if g["shape"] == "cylinder":
                    p.height = float(g["height_cm"])
        return arr
