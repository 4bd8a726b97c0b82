"""Denoiser phantoms: random water/bone/lead/air ellipsoid mixtures.

Each phantom is a scene (in the scene.yaml schema, with the ``ellipsoid``
extension primitive) on a cubic grid of ``side`` voxels:

* a water body ellipsoid with semi-axes U(0.55, 0.9) x half the grid side;
* 2-7 inner ellipsoids, each bone, air or lead (bone and air with semi-axes
  U(0.06, 0.25) x half side, lead U(0.01, 0.04) x half side), placed inside
  the body's bounding box and listed after it (so they win);
* a cone beam from a focus 1.5 grid sides from the centre along a random
  axis direction (+-x, +-y, +-z), diameter covering the grid, with a 60-120
  kVp tungsten spectrum (the Kramers model of spectrum.py:55-62, 1 keV
  bins, 2.5 mm Al).

``voxel_maps`` gives the material index (air 0, water 1, bone 2, lead 3)
and density at every voxel centre, from the same point location the
engine uses.
"""
from __future__ import annotations

import numpy as np

from .geometry import Geometry, contains
from .source import kramers_spectrum
from . import tables as tb

MATERIALS = ["air", "water", "bone", "lead"]


def phantom(rng: np.random.Generator, side: int = 64, voxel_cm: float = 0.5) -> tuple[dict, dict]:
    half = 0.5 * side * voxel_cm
    geoms = [{"name": "body", "shape": "ellipsoid", "material": "water", "center": [0.0, 0.0, 0.0],
              "semi_axes_cm": [float(x) for x in rng.uniform(0.55, 0.9, 3) * half]}]
    body = np.array(geoms[0]["semi_axes_cm"])
    for i in range(int(rng.integers(2, 8))):
        mat = str(rng.choice(["bone", "bone", "air", "lead"]))
        lo, hi = (0.01, 0.04) if mat == "lead" else (0.06, 0.25)
        semi = rng.uniform(lo, hi, 3) * half
        c = rng.uniform(-0.6, 0.6, 3) * body
        geoms.append({"name": f"inner{i}", "shape": "ellipsoid", "material": mat,
                      "center": [float(x) for x in c], "semi_axes_cm": [float(x) for x in semi]})
    axis = int(rng.integers(0, 3))
    sign = float(rng.choice([-1.0, 1.0]))
    d = np.zeros(3)
    d[axis] = -sign
    pos = -d * 3.0 * half
    kvp = float(rng.uniform(60.0, 120.0))
    e, w = kramers_spectrum(kvp, 2.5, n_bins=None)
    src = {"position": [float(x) for x in pos], "direction": [float(x) for x in d],
           "field": {"shape": "cone", "diameter_cm": float(2.0 * half * 1.5), "sid_cm": float(3.0 * half)},
           "spectrum": [{"energy_keV": float(a), "weight": float(b)} for a, b in zip(e, w)]}
    scene = {"source": src, "geometry": geoms, "physics": {"fluorescence": True}}
    grid = {"origin": (-half, -half, -half), "shape": (side, side, side), "voxel_cm": voxel_cm}
    return scene, grid


def phantoms(n: int, seed: int, side: int = 64, voxel_cm: float = 0.5):
    rng = np.random.default_rng(seed)
    out = [phantom(rng, side, voxel_cm) for _ in range(n)]
    return [s for s, _ in out], [g for _, g in out]


def voxel_maps(scene: dict, grid: dict, materials: list[str] | None = None) -> tuple[np.ndarray, np.ndarray]:
    """(material index uint8 into ``materials``, default MATERIALS; density
    float32) at the voxel centres, shaped (nx, ny, nz) like the kerma grid."""
    mats = MATERIALS if materials is None else materials
    nx, ny, nz = grid["shape"]
    h = grid["voxel_cm"]
    o = np.asarray(grid["origin"], dtype=float)
    ix, iy, iz = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    pts = np.stack([o[0] + (ix + 0.5) * h, o[1] + (iy + 0.5) * h, o[2] + (iz + 0.5) * h], axis=-1).reshape(-1, 3)
    idx = np.full(pts.shape[0], mats.index(Geometry(scene["geometry"]).background), dtype=np.uint8)
    for g in scene["geometry"]:                      # later primitives win (geometry.py:205-212)
        idx[contains(g, pts)] = mats.index(g["material"])
    idx = idx.reshape(nx, ny, nz)
    dens = np.array([tb.density(m) for m in mats], dtype=np.float32)[idx]
    return idx, dens
