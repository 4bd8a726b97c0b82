"""Synthetic scenes of the benchmark configurations, as scene.yaml dicts.

* ``plain_mc``: monoenergetic 60 keV pencil beam along +z into a 30x30x20 cm
  water box centred in a 200 cm air cube; kerma on 60x60x40 voxels of 0.5 cm
  covering the water box.
* ``room``: 400x400x300 cm air room; water torso box 35x25x20 cm with two
  cortical-bone cylinders (r 1.5 cm, length 20 cm) inside; 0.05 cm lead
  sheet 30x30 cm 150 cm from the focus; 20 cm concrete wall.  80 kVp
  tungsten-anode spectrum with 2.5 mm Al in 1 keV bins from the Kramers
  model ChatCarlo falls back to without SpekPy (spectrum.py:55-62), rect
  field 35x43 cm at SID 180 cm.  Kerma and H*(10) on 5 cm voxels over the
  whole room (80x80x60).
* ``ct``: the CT dosimetry configuration (PMMA phantom with five holes,
  helical 120 kVp fan beam, kerma on 320x320x150 voxels of 1 mm).

Positions are fixed here (the configuration leaves them open) and the same
dicts feed the engine and the CPU oracle.
"""
from __future__ import annotations

import numpy as np

from .source import kramers_spectrum


def plain_mc() -> dict:
    return {
        "source": {
            "position": [0.0, 0.0, -100.0],
            "direction": [0.0, 0.0, 1.0],
            "field": {"shape": "parallel", "size_cm": [1e-4, 1e-4]},
            "spectrum": [{"energy_keV": 60.0, "weight": 1.0}],
        },
        "geometry": [
            {"name": "air_cube", "shape": "box", "material": "air", "center": [0.0, 0.0, 0.0],
             "size_cm": [200.0, 200.0, 200.0]},
            {"name": "water_box", "shape": "box", "material": "water", "center": [0.0, 0.0, 0.0],
             "size_cm": [30.0, 30.0, 20.0]},
        ],
        "physics": {"fluorescence": True},
    }


PLAIN_MC_GRID = {"origin": (-15.0, -15.0, -10.0), "shape": (60, 60, 40), "voxel_cm": 0.5}


def room_spectrum() -> list[dict]:
    e, w = kramers_spectrum(80.0, 2.5, n_bins=75)
    return [{"energy_keV": float(a), "weight": float(b)} for a, b in zip(e, w)]


def room() -> dict:
    return {
        "source": {
            "position": [0.0, 0.0, 190.0],
            "direction": [0.0, 0.0, -1.0],
            "field": {"shape": "rect", "size_cm": [35.0, 43.0], "sid_cm": 180.0},
            "spectrum": room_spectrum(),
        },
        "geometry": [
            {"name": "room_air", "shape": "box", "material": "air", "center": [0.0, 0.0, 150.0],
             "size_cm": [400.0, 400.0, 300.0]},
            {"name": "torso", "shape": "box", "material": "water", "center": [0.0, 0.0, 100.0],
             "size_cm": [35.0, 25.0, 20.0]},
            {"name": "bone_left", "shape": "cylinder", "material": "bone", "axis": "y",
             "center": [-8.0, 0.0, 100.0], "radius_cm": 1.5, "height_cm": 20.0},
            {"name": "bone_right", "shape": "cylinder", "material": "bone", "axis": "y",
             "center": [8.0, 0.0, 100.0], "radius_cm": 1.5, "height_cm": 20.0},
            {"name": "lead_sheet", "shape": "box", "material": "lead", "center": [0.0, 0.0, 40.0],
             "size_cm": [30.0, 30.0, 0.05]},
            {"name": "wall", "shape": "box", "material": "concrete", "center": [190.0, 0.0, 150.0],
             "size_cm": [20.0, 400.0, 300.0]},
        ],
        "physics": {"fluorescence": True},
    }


ROOM_GRID = {"origin": (-200.0, -200.0, 0.0), "shape": (80, 80, 60), "voxel_cm": 5.0}


def ct() -> dict:
    """CT dosimetry: PMMA body CTDI-type phantom (32 cm diameter, 15 cm long,
    axis z on the isocentre) with five 1.3 cm air holes (centre, and 1 cm
    under the surface at 0/90/180/270 degrees; listed after the cylinder so
    they win); 120 kVp tungsten spectrum with 6.8 mm Al (the Kramers model
    of spectrum.py:55-62, 1 keV bins); focus 60 cm from the isocentre, fan
    50x4 cm at SID 60 cm, continuous rotation about z with a 30 cm helical
    scan length."""
    holes = [(0.0, 0.0), (15.0, 0.0), (0.0, 15.0), (-15.0, 0.0), (0.0, -15.0)]
    geoms = [{"name": "pmma_body", "shape": "cylinder", "material": "pmma", "axis": "z",
              "center": [0.0, 0.0, 0.0], "radius_cm": 16.0, "height_cm": 15.0}]
    geoms += [{"name": f"hole{i}", "shape": "cylinder", "material": "air", "axis": "z",
               "center": [x, y, 0.0], "radius_cm": 0.65, "height_cm": 15.0} for i, (x, y) in enumerate(holes)]
    e, w = kramers_spectrum(120.0, 6.8, n_bins=None)
    return {"source": {"position": [0.0, -60.0, 0.0], "direction": [0.0, 1.0, 0.0],
                       "field": {"shape": "rect", "size_cm": [50.0, 4.0], "sid_cm": 60.0},
                       "rotation": {"isocenter": [0.0, 0.0, 0.0], "axis": "z", "scan_length_cm": 30.0},
                       "spectrum": [{"energy_keV": float(a), "weight": float(b)} for a, b in zip(e, w)]},
            "geometry": geoms, "physics": {"fluorescence": True}}


CT_GRID = {"origin": (-16.0, -16.0, -7.5), "shape": (320, 320, 150), "voxel_cm": 0.1}


def make_grid(spec: dict, track_uncertainty: bool = True, pinned: bool = False):
    from .tally import VoxelGrid
    return VoxelGrid(origin_cm=np.asarray(spec["origin"], dtype=float), shape=spec["shape"],
                     voxel_size_cm=spec["voxel_cm"], track_uncertainty=track_uncertainty, pinned=pinned)


def pencil_beam_arrays(n: int, start, direction, energy_kev: float):
    pos = np.tile(np.asarray(start, dtype=float), (n, 1))
    dirv = np.tile(np.asarray(direction, dtype=float), (n, 1))
    return pos, dirv, np.full(n, float(energy_kev))


BATCH_MATERIALS = ["air", "water", "bone", "muscle", "pmma", "lead", "concrete"]


def batched_scenes(n_scenes: int = 256, seed: int = 2026, hist_lo: float = 1e5, hist_hi: float = 1e7):
    """The batched configuration: n_scenes random scenes.

    Per scene: 1-12 primitives of a uniformly drawn type (box / cylinder /
    sphere) with dimensions U(1, 50) cm, materials drawn from
    {air, water, ICRU bone, muscle, PMMA, lead, concrete} (a lead primitive
    gets one dimension U(0.01, 0.2) cm); a source that is monoenergetic
    U(20, 140) keV or a 60-140 kVp tungsten spectrum with 2-4 mm Al (the
    Kramers model of spectrum.py:55-62 in 1 keV bins); its own 64^3 kerma
    grid of U(0.5, 2) cm voxels centred on the scene; history counts
    log-uniform in [hist_lo, hist_hi].  Returns (scenes, grid specs, counts).
    """
    rng = np.random.default_rng(seed)
    scenes, grids, counts = [], [], []
    for s in range(n_scenes):
        voxel = float(rng.uniform(0.5, 2.0))
        half = 32 * voxel
        shape = str(rng.choice(["box", "cylinder", "sphere"]))
        geoms = []
        for i in range(int(rng.integers(1, 13))):
            mat = str(rng.choice(BATCH_MATERIALS))
            c = [float(x) for x in rng.uniform(-0.6 * half, 0.6 * half, 3)]
            g = {"name": f"p{i}", "shape": shape, "material": mat, "center": c}
            if shape == "box":
                size = [float(x) for x in rng.uniform(1.0, 50.0, 3)]
                if mat == "lead":
                    size[int(rng.integers(0, 3))] = float(rng.uniform(0.01, 0.2))
                g["size_cm"] = size
            elif shape == "cylinder":
                g["axis"] = str(rng.choice(["x", "y", "z"]))
                g["radius_cm"] = float(rng.uniform(1.0, 50.0)) / 2.0
                g["height_cm"] = float(rng.uniform(1.0, 50.0))
                if mat == "lead":
                    g["height_cm"] = float(rng.uniform(0.01, 0.2))
            else:
                g["radius_cm"] = float(rng.uniform(1.0, 50.0)) / 2.0
                if mat == "lead":
                    g["radius_cm"] = float(rng.uniform(0.01, 0.2))
            geoms.append(g)
        sid = 100.0 + half
        src = {"position": [0.0, 0.0, -sid], "direction": [0.0, 0.0, 1.0],
               "field": {"shape": "rect", "size_cm": [2 * half, 2 * half], "sid_cm": sid}}
        if rng.random() < 0.5:
            src["spectrum"] = [{"energy_keV": float(rng.uniform(20.0, 140.0)), "weight": 1.0}]
        else:
            e, w = kramers_spectrum(float(rng.uniform(60.0, 140.0)), float(rng.uniform(2.0, 4.0)),
                                    n_bins=None)
            src["spectrum"] = [{"energy_keV": float(a), "weight": float(b)} for a, b in zip(e, w)]
        scenes.append({"source": src, "geometry": geoms, "physics": {"fluorescence": True}})
        grids.append({"origin": (-half, -half, -half), "shape": (64, 64, 64), "voxel_cm": voxel})
        counts.append(int(round(float(np.exp(rng.uniform(np.log(hist_lo), np.log(hist_hi)))))))
    return scenes, grids, counts
