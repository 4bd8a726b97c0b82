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


def make_grid(spec: dict, track_uncertainty: bool = True):
    from .tally import VoxelGrid
    return VoxelGrid(origin_cm=np.asarray(spec["origin"], dtype=float), shape=spec["shape"],
                     voxel_size_cm=spec["voxel_cm"], track_uncertainty=track_uncertainty)


def pencil_beam_arrays(n: int, start, direction, energy_kev: float):
    pos = np.tile(np.asarray(start, dtype=float), (n, 1))
    dirv = np.tile(np.asarray(direction, dtype=float), (n, 1))
    return pos, dirv, np.full(n, float(energy_kev))
