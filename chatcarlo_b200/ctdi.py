"""CTDIvol calibration on the engine (chatcarlo/ctdi.py).

A CT console's CTDIvol [mGy] is the absolute anchor: the source of the scene
(kVp, filtration, rotation, field) irradiates the standard PMMA CTDI phantom
(body 32 cm or head 16 cm diameter, 15 cm long, on the isocentre), whose
CTDIw-like quantity per history,

    CTDIw = D_center / 3 + 2 D_periphery / 3,

comes from the kerma-derived dose in the voxels of the ionisation chambers'
positions (on the axis, and 1 cm under the surface, 100 mm long) on a 1 cm
grid (ctdi.py:53-100).  The measured CTDIvol divided by it is the effective
photon count that turns per-history results into absolute ones
(ctdi.py:103-108), reported as ``TransportResult.n_photons_real``.

The histories run through the engine's ``run_transport`` (sources sampled
on the device) instead of host-sampled batches through transport_photons;
the estimator is the same.
"""
from __future__ import annotations

import numpy as np

from .geometry import Geometry
from .tally import VoxelGrid
from . import tables as tb

PHANTOM_DIAMETER_CM = {"body": 32.0, "head": 16.0}       # ctdi.py:35
PHANTOM_LENGTH_CM = 15.0
CHAMBER_LENGTH_CM = 10.0
GRID_RESOLUTION_CM = 1.0


def ctdi_phantom_geometry(rot: dict, phantom: str = "body") -> Geometry:
    """The PMMA cylinder on the isocentre, along the rotation axis (ctdi.py:41-52)."""
    return Geometry([_phantom_prim(rot, phantom)])


def _phantom_prim(rot: dict, phantom: str) -> dict:
    return {"name": f"ctdi_phantom_{phantom}", "shape": "cylinder", "material": "pmma",
            "axis": rot.get("axis", "z"), "radius_cm": PHANTOM_DIAMETER_CM[phantom] / 2.0,
            "height_cm": PHANTOM_LENGTH_CM, "center": [float(x) for x in rot["isocenter"]]}


def phantom_grid(rot: dict, phantom: str = "body") -> VoxelGrid:
    """1 cm grid over the phantom with a 2 cm margin (ctdi.py:71-77)."""
    radius = PHANTOM_DIAMETER_CM[phantom] / 2.0
    iso = np.asarray(rot["isocenter"], dtype=float)
    ax = {"x": 0, "y": 1, "z": 2}[rot.get("axis", "z")]
    margin = 2.0
    lo, hi = iso - radius - margin, iso + radius + margin
    lo[ax] = iso[ax] - PHANTOM_LENGTH_CM / 2.0 - margin
    hi[ax] = iso[ax] + PHANTOM_LENGTH_CM / 2.0 + margin
    return VoxelGrid.from_bbox(lo, hi, GRID_RESOLUTION_CM)


def chamber_masks(grid: VoxelGrid, rot: dict, phantom: str = "body"):
    """Centre (r < 2 cm) and periphery (R-2 <= r <= R-1 cm) voxels within
    +-5 cm of the isocentre along the axis (ctdi.py:89-95)."""
    radius = PHANTOM_DIAMETER_CM[phantom] / 2.0
    iso = np.asarray(rot["isocenter"], dtype=float)
    ax = {"x": 0, "y": 1, "z": 2}[rot.get("axis", "z")]
    plane = [k for k in range(3) if k != ax]
    c = grid.voxel_centers().reshape(*grid.shape, 3)
    r = np.sqrt((c[..., plane[0]] - iso[plane[0]]) ** 2 + (c[..., plane[1]] - iso[plane[1]]) ** 2)
    z_ok = np.abs(c[..., ax] - iso[ax]) <= CHAMBER_LENGTH_CM / 2.0
    return z_ok & (r < 2.0), z_ok & (r >= radius - 2.0) & (r <= radius - 1.0)


def dose_map_Gy(grid: VoxelGrid, geometry: Geometry) -> np.ndarray:
    """Kerma to dose with the density of the material at each voxel centre
    (diagnostics.py:16-26)."""
    mats = geometry.material_at(grid.voxel_centers())
    dens = np.array([tb.density(m) for m in mats]).reshape(grid.shape)
    return grid.dose_map_Gy(dens)


def ctdi_per_history_Gy(src: dict, phantom: str = "body", n_histories: int = 200_000, seed: int | None = None,
                        engine=None) -> tuple[float, float, float]:
    """(CTDIw, D_center, D_periphery) in Gy per history (ctdi.py:53-100)."""
    from .transport import run_transport
    rot = src.get("rotation")
    if rot is None:
        raise ValueError("CTDIvol calibration needs source.rotation (a gantry rotation)")
    prim = _phantom_prim(rot, phantom)
    grid = phantom_grid(rot, phantom)
    scene = {"source": {k: v for k, v in src.items() if k not in ("ctdi_vol_mGy", "ctdi_phantom", "mas")},
             "geometry": [prim]}
    run_transport(scene, n_histories=n_histories, seed=seed, dose_grid=True, grid=grid, track_uncertainty=False,
                  engine=engine)
    dose = dose_map_Gy(grid, Geometry([prim])) / n_histories
    center, periph = chamber_masks(grid, rot, phantom)
    d_center = float(dose[center].mean())
    d_periph = float(dose[periph].mean())
    return d_center / 3.0 + 2.0 * d_periph / 3.0, d_center, d_periph


def effective_histories_from_ctdi(src: dict, seed: int | None = None, engine=None,
                                  n_histories: int = 200_000) -> float:
    """Measured CTDIvol [mGy] / CTDIw [Gy per history] (ctdi.py:103-108)."""
    ctdi_vol_mGy = float(src["ctdi_vol_mGy"])
    ctdiw, _, _ = ctdi_per_history_Gy(src, phantom=src.get("ctdi_phantom", "body"), n_histories=n_histories,
                                      seed=seed, engine=engine)
    return ctdi_vol_mGy * 1e-3 / ctdiw
