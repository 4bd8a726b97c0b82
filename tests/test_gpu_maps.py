"""Output maps on the device (cc_grid_maps) and the grid's host transfers.

The dose, H*(10) and relative-error maps of chatcarlo/__main__.py:198-209
(diagnostics.py:16-26, tally.py:96-132) computed on the device must equal,
bit for bit, the reference's own host computation (tests/golden/maps.npz,
made by running the reference) and the oracle's restatement of it on grids
that the engine filled.
"""
import numpy as np
import pytest

import cc_oracle as O
from chatcarlo_b200 import workloads as W
from chatcarlo_b200.geometry import Geometry
from chatcarlo_b200.tally import VoxelGrid

pytestmark = pytest.mark.gpu

GEOMS = [
    {"name": "room", "shape": "box", "material": "air", "center": [0, 0, 0], "size_cm": [120, 100, 90]},
    {"name": "slab", "shape": "box", "material": "water", "center": [0, 0, 0], "size_cm": [30, 30, 20]},
    {"name": "ball", "shape": "sphere", "material": "bone", "center": [5, -3, 2], "radius_cm": 6},
    {"name": "rodx", "shape": "cylinder", "material": "lead", "axis": "x", "center": [0, 8, -4],
     "radius_cm": 1.5, "height_cm": 25},
    {"name": "rody", "shape": "cylinder", "material": "concrete", "axis": "y", "center": [-9, 0, 5],
     "radius_cm": 2.0, "height_cm": 18},
    {"name": "rodz", "shape": "cylinder", "material": "pmma", "axis": "z", "center": [10, 10, 0],
     "radius_cm": 3.0, "height_cm": 12},
]


@pytest.fixture(scope="module")
def engine():
    from chatcarlo_b200.transport import default_engine
    return default_engine()


def _golden_grid(g, n_batches=None):
    grid = VoxelGrid(origin_cm=g["origin"], shape=tuple(g["shape"]), voxel_size_cm=float(g["voxel_cm"]),
                     track_uncertainty=True)
    grid.kerma_keV[...] = g["kerma"]
    grid.h10_track_pSv_cm3[...] = g["h10"]
    grid.kerma_sum2[...] = g["k2"]
    grid.h10_sum2[...] = g["h2"]
    grid.n_batches_hit[...] = g["nhit"]
    grid.n_batches = int(g["nb"]) if n_batches is None else n_batches
    grid.n_histories = int(g["nh"])
    return grid


def test_device_maps_equal_the_reference(engine, golden):
    import torch
    from chatcarlo_b200.transport import DeviceGrid
    g = golden("maps")
    grid = _golden_grid(g)
    dg = DeviceGrid(engine, grid, stats=True)
    try:
        dg.upload(grid)
        back = VoxelGrid(origin_cm=g["origin"], shape=tuple(g["shape"]), voxel_size_cm=1.0, track_uncertainty=True)
        dg.download(back)
        for a in ("kerma_keV", "h10_track_pSv_cm3", "kerma_sum2", "h10_sum2", "n_batches_hit"):
            np.testing.assert_array_equal(getattr(back, a), getattr(grid, a))
        assert (back.n_batches, back.n_histories) == (grid.n_batches, grid.n_histories)
        nh = int(g["nh"])
        m = dg.maps(Geometry(GEOMS), divisor=nh, rel=True)
        np.testing.assert_array_equal(m["dose_Gy"], g["dose"])
        np.testing.assert_array_equal(m["h10_pSv"], g["h10map"])
        np.testing.assert_array_equal(m["kerma_rel"], g["krel"])
        np.testing.assert_array_equal(m["h10_rel"], g["hrel"])
        # the same maps left on the device
        out = {k: torch.empty(tuple(g["shape"]), dtype=torch.float64, device="cuda")
               for k in ("dose_Gy", "h10_pSv", "kerma_rel", "h10_rel")}
        md = dg.maps(Geometry(GEOMS), divisor=nh, rel=True, out=out)
        torch.cuda.synchronize()
        for k in out:
            np.testing.assert_array_equal(md[k].cpu().numpy(), m[k])
        # fewer than two batches: no relative error anywhere
        dg.upload(_golden_grid(g, n_batches=1))
        m1 = dg.maps(Geometry(GEOMS), divisor=nh, dose=False, h10=False, rel=True)
        np.testing.assert_array_equal(m1["kerma_rel"], g["krel_m1"])
    finally:
        dg.close()


def test_run_transport_maps_equal_the_oracle_on_the_engines_grid(engine):
    """A real run: the per-history maps run_transport(maps=True) computes on
    the device equal the oracle's maps of the downloaded grid, bit for bit
    (voxel centres on integer coordinates put some of them on surfaces)."""
    from chatcarlo_b200 import tables as tb
    from chatcarlo_b200.transport import run_transport
    scene = {"source": {"position": [0.0, 0.0, -60.0], "direction": [0.0, 0.0, 1.0],
                        "field": {"shape": "cone", "diameter_cm": 40.0, "sid_cm": 60.0},
                        "spectrum": [{"energy_keV": 60.0, "weight": 1.0}, {"energy_keV": 80.0, "weight": 0.5}]},
             "geometry": GEOMS}
    grid = VoxelGrid(origin_cm=np.array([-20.5, -16.5, -14.5]), shape=(41, 33, 29), voxel_size_cm=1.0,
                     track_uncertainty=True)
    n = 400_000
    res = run_transport(scene, n_histories=n, seed=5, batch_size=50_000, dose_grid=True, grid=grid,
                        engine=engine, maps=True)
    g = res.grid
    assert g.n_batches == 8 and res.maps is not None
    dose = O.dose_map_Gy(g.kerma_keV, g.origin_cm, g.voxel_size_cm, O.OracleGeometry(GEOMS), tb.density) / n
    np.testing.assert_array_equal(res.maps["dose_per_history_Gy"], dose)
    np.testing.assert_array_equal(res.maps["h10_per_history_pSv"], O.h10_map_pSv(g.h10_track_pSv_cm3, 1.0) / n)
    np.testing.assert_array_equal(res.maps["kerma_rel"],
                                  O.relative_error(g.kerma_keV, g.kerma_sum2, g.n_batches, g.n_histories))
    np.testing.assert_array_equal(res.maps["h10_rel"],
                                  O.relative_error(g.h10_track_pSv_cm3, g.h10_sum2, g.n_batches, g.n_histories))
    assert np.count_nonzero(dose) > 1000


def test_download_into_pinned_and_pageable_grids_agree(engine):
    """The device writes a page-locked VoxelGrid's arrays directly; a
    pageable one goes through the staging copy; both hold the same run."""
    from chatcarlo_b200.transport import run_transport
    raw = W.room()
    spec = W.ROOM_GRID
    grids = [W.make_grid(spec, track_uncertainty=True, pinned=p) for p in (True, False)]
    import torch
    assert grids[0].kerma_keV.ctypes.data and torch.cuda.is_available()
    for gr in grids:
        run_transport(raw, n_histories=300_000, seed=8, batch_size=100_000, dose_grid=True, grid=gr, engine=engine)
    for a in ("kerma_keV", "h10_track_pSv_cm3", "kerma_sum2", "h10_sum2", "n_batches_hit"):
        np.testing.assert_allclose(getattr(grids[0], a), getattr(grids[1], a), rtol=1e-9, atol=1e-12)
    assert grids[0].n_batches == grids[1].n_batches == 3
