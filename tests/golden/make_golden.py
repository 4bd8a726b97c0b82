"""Generate the golden vectors that pin the CPU oracle to ChatCarlo itself.

Run in an environment that has the reference checkout, naming its path
in $CHATCARLO_REFERENCE (required):

    CHATCARLO_REFERENCE=<path to the chatcarlo checkout> python tests/golden/make_golden.py

The reference's modules are imported unmodified, with the stand-in data
module oracle/xraylib_standin first on sys.path in place of the absent
third-party ``xraylib``.  Every case records its inputs, the seed and the
reference's outputs in tests/golden/*.npz; tests/test_oracle_golden.py
replays the same cases through the oracle and demands identical results.
"""
from __future__ import annotations

import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent
if not os.environ.get("CHATCARLO_REFERENCE"):
    sys.exit("set CHATCARLO_REFERENCE to the path of the chatcarlo checkout")
REF = Path(os.environ["CHATCARLO_REFERENCE"])

sys.dont_write_bytecode = True
sys.path.insert(0, str(REPO / "oracle" / "xraylib_standin"))
sys.path.insert(0, str(REF))
sys.path.insert(0, str(REPO))

from chatcarlo import geometry as rgeom  # noqa: E402
from chatcarlo import materials as rmat  # noqa: E402
from chatcarlo import physics as rphys  # noqa: E402
from chatcarlo import source as rsrc  # noqa: E402
from chatcarlo import tally as rtally  # noqa: E402
from chatcarlo import transport as rtr  # noqa: E402
from chatcarlo.dose_coefficients import h_star_10_per_fluence  # noqa: E402
from chatcarlo.scene import validate_scene  # noqa: E402

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

MATERIALS = ["water", "air", "bone", "lead", "concrete", "pmma", "soft_tissue", "lung", "aluminum",
             "copper", "iron"]


def unit(v):
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def case_geometry():
    rng = np.random.default_rng(101)
    n = 3000
    o = rng.uniform(-40, 40, (n, 3))
    d = unit(rng.normal(size=(n, 3)))
    # a share of axis-parallel rays exercise the parallel-slab branches
    d[:300] = np.eye(3)[rng.integers(0, 3, 300)] * rng.choice([-1.0, 1.0], (300, 1))
    g = rgeom.Geometry(GEOMS)
    mat = g.material_at(o)
    t, esc = g.next_boundary(o, d)
    return {"o": o, "d": d, "mat": mat.astype(str), "t": t, "escape": esc,
            "bbox_min": g.bbox_min, "bbox_max": g.bbox_max}


def case_materials():
    rng = np.random.default_rng(202)
    e = np.exp(rng.uniform(0.0, np.log(150.0), 400))
    out = {"e": e}
    for m in MATERIALS:
        p = rmat.mu_rho_parts(m, e)
        out[f"{m}__photo"] = p["photoelectric"]
        out[f"{m}__compt"] = p["compton"]
        out[f"{m}__rayl"] = p["rayleigh"]
        out[f"{m}__muen"] = rmat.mu_en_rho(m, e)
        out[f"{m}__density"] = np.array(rmat.density(m))
    eh = np.exp(rng.uniform(np.log(1.0), np.log(2e4), 200))
    out["eh"] = eh
    out["h10"] = h_star_10_per_fluence(eh)
    for z in (1, 8, 20, 26, 29, 74, 82):
        ed, om, le, lp = rmat.fluorescence_k_data(z)
        out[f"k{z}"] = np.concatenate([[ed, om], le, lp])
        q, f = rmat.rayleigh_form_factor_table(z)
        x, a = rmat.rayleigh_cumulative_table(z)
        qs, s = rmat.incoherent_sq_table(z)
        out[f"ff{z}"] = f
        out[f"ra{z}"] = a
        out[f"sq{z}"] = s
        out[f"grid{z}"] = rmat._element_energy_grid_kev(z)
    return out


def case_samplers():
    out = {}
    rng = np.random.default_rng(303)
    n = 4000
    for m, e0 in (("water", 60.0), ("bone", 40.0), ("lead", 120.0)):
        mats = np.full(n, m, dtype=object)
        e = np.full(n, e0)
        eps, cos = rphys.sample_compton_bound(mats, e, np.random.default_rng(11))
        out[f"compton_{m}"] = np.stack([eps, cos])
        z = rphys.sample_rayleigh_element(mats, e, np.random.default_rng(12))
        out[f"rayl_el_{m}"] = z
        out[f"rayl_cos_{m}"] = rphys.sample_rayleigh_cos_theta(z, e, np.random.default_rng(13))
        emit, el = rphys.sample_fluorescence(mats, np.full(n, 100.0), np.random.default_rng(14))
        out[f"fluor_{m}"] = np.stack([emit.astype(float), el])
    e = rng.uniform(10, 150, n)
    out["kn_e"] = e
    out["kn"] = np.stack(rphys.sample_klein_nishina(e, np.random.default_rng(15)))
    zs = rng.choice([1, 8, 20, 82], n)
    out["ru_z"] = zs
    out["ru_e"] = e
    out["ru"] = rphys._sample_rayleigh_cos_theta_uniform(zs, np.full(n, 30.0), np.random.default_rng(16))
    d = unit(rng.normal(size=(n, 3)))
    d[:50] = [0.0, 0.0, 1.0]
    c = rng.uniform(-1, 1, n)
    out["sd_d"] = d
    out["sd_c"] = c
    out["sd"] = rphys.scatter_direction(d, c, np.random.default_rng(17))
    out["iso"] = rphys.isotropic_direction(n, np.random.default_rng(18))
    return out


def case_tally():
    rng = np.random.default_rng(404)
    n = 500
    grid = rtally.VoxelGrid(origin_cm=np.array([-10.0, -8.0, -6.0]), shape=(20, 16, 12), voxel_size_cm=1.0)
    o = rng.uniform(-14, 14, (n, 3))
    d = unit(rng.normal(size=(n, 3)))
    L = rng.exponential(8.0, n)
    w = rng.uniform(0.5, 2.0, n)
    target = np.zeros(grid.shape)
    rtally.accumulate_track_length(target, grid, o, d, L, w, np.random.default_rng(19))
    return {"o": o, "d": d, "L": L, "w": w, "target": target}


def _tp(geoms, start, direction, e0, n, seed, grid_res=None, fluor=True, margin=50.0):
    g = rgeom.Geometry(geoms, bbox_margin_cm=margin)
    pos = np.tile(np.asarray(start, dtype=float), (n, 1))
    dirv = np.tile(np.asarray(direction, dtype=float), (n, 1))
    en = np.full(n, float(e0))
    grid = None
    if grid_res is not None:
        grid = rtally.VoxelGrid.from_bbox(g.bbox_min, g.bbox_max, grid_res)
    r = rtr.transport_photons(pos, dirv, en, g, np.random.default_rng(seed), grid=grid,
                              fluorescence_enabled=fluor)
    out = {"pos": pos, "dir": dirv, "energy": en, "n_scatter": r.n_scatter, "absorbed": r.absorbed,
           "escaped": r.escaped, "n_fluor": np.array(r.n_fluorescence),
           "dep_names": np.array(sorted(r.energy_deposited)),
           "dep": np.array([r.energy_deposited[k] for k in sorted(r.energy_deposited)])}
    if grid is not None:
        out["kerma"] = grid.kerma_keV
        out["h10"] = grid.h10_track_pSv_cm3
    return out


def case_transport():
    out = {}
    water = [{"name": "slab", "shape": "box", "material": "water", "center": [0, 0, 0],
              "size_cm": [10.0, 100.0, 100.0]}]
    for k, v in _tp(water, [-15, 0, 0], [1, 0, 0], 60.0, 3000, 1).items():
        out[f"water_{k}"] = v
    lead = [{"name": "slab", "shape": "box", "material": "lead", "center": [0, 0, 0],
             "size_cm": [0.5, 50.0, 50.0]}]
    for k, v in _tp(lead, [-5.25, 0, 0], [1, 0, 0], 100.0, 3000, 42, grid_res=10.0).items():
        out[f"lead_{k}"] = v
    for k, v in _tp(GEOMS, [-55, 1, 2], unit(np.array([[1.0, 0.05, 0.02]]))[0], 80.0, 2000, 7,
                    grid_res=15.0).items():
        out[f"mixed_{k}"] = v
    return out


def scene_small():
    return {
        "source": {"position": [0, 0, 120], "direction": [0, 0, -1],
                   "field": {"shape": "rect", "size_cm": [20, 25], "sid_cm": 150},
                   "spectrum": [{"energy_keV": float(e), "weight": float(w)}
                                for e, w in zip(*rsrc_kramers())]},
        "geometry": [
            {"name": "air", "shape": "box", "material": "air", "center": [0, 0, 30], "size_cm": [150, 150, 150]},
            {"name": "body", "shape": "box", "material": "water", "center": [0, 0, 20], "size_cm": [30, 20, 20]},
            {"name": "bone", "shape": "cylinder", "material": "bone", "axis": "y", "center": [4, 0, 20],
             "radius_cm": 1.5, "height_cm": 18},
            {"name": "pb", "shape": "box", "material": "lead", "center": [0, 0, -20], "size_cm": [30, 30, 0.05]},
        ],
        "physics": {"fluorescence": True},
    }


def rsrc_kramers():
    from chatcarlo.spectrum import _kramers_fallback_spectrum
    return _kramers_fallback_spectrum(80.0, 2.5, n_bins=75)


def case_run():
    raw = scene_small()
    sc = validate_scene(raw)
    assert sc.ok, sc.errors
    res = rtr.run_transport(sc, n_histories=12000, seed=5, batch_size=3000, dose_grid=True,
                            grid_resolution_cm=20.0, n_workers=1, track_uncertainty=True)
    g = res.grid
    names = sorted(res.energy_deposited_MeV)
    return {"kerma": g.kerma_keV, "h10": g.h10_track_pSv_cm3, "kerma_sum2": g.kerma_sum2,
            "h10_sum2": g.h10_sum2, "n_hit": g.n_batches_hit, "n_batches": np.array(g.n_batches),
            "origin": g.origin_cm, "shape": np.array(g.shape),
            "scalars": np.array([res.fraction_absorbed, res.fraction_escaped, res.mean_scatter_events,
                                 res.n_fluorescence, res.n_batches]),
            "dep_names": np.array(names), "dep": np.array([res.energy_deposited_MeV[k] for k in names]),
            "sem": np.array([res.energy_deposited_sem_MeV[k] for k in names]),
            "kramers": np.stack(rsrc_kramers())}


def case_source():
    out = {}
    base = {"position": [0, -100, 50], "direction": [0, 1, 0], "spectrum": [
        {"energy_keV": 30.0, "weight": 1.0}, {"energy_keV": 60.0, "weight": 3.0}, {"energy_keV": 90.0, "weight": 2.0}]}
    variants = {
        "rect": {"field": {"shape": "rect", "size_cm": [30, 40], "sid_cm": 100}},
        "cone": {"field": {"shape": "cone", "diameter_cm": 25, "sid_cm": 100}},
        "parallel": {"field": {"shape": "parallel", "size_cm": [10, 12]}},
        "rot": {"field": {"shape": "rect", "size_cm": [50, 4], "sid_cm": 100},
                "rotation": {"isocenter": [0, 0, 50], "axis": "z", "scan_length_cm": 30}},
        "rotn": {"field": {"shape": "cone", "diameter_cm": 20, "sid_cm": 100},
                 "rotation": {"isocenter": [0, 0, 50], "axis": "x", "n_angles": 8}},
    }
    for k, extra in variants.items():
        src = dict(base, **extra)
        p, d, e = rsrc.sample_source_photons(src, 2000, np.random.default_rng(21))
        out[f"{k}_pos"], out[f"{k}_dir"], out[f"{k}_e"] = p, d, e
    return out


HEEL_VARIANTS = {
    "rect": {"field": {"shape": "rect", "size_cm": [35, 43], "sid_cm": 100}, "anode_direction": [1.0, 0.3, 0.0]},
    "cone": {"field": {"shape": "cone", "diameter_cm": 30, "sid_cm": 100}, "anode_direction": [0.0, 1.0, 0.2]},
    "rot": {"field": {"shape": "rect", "size_cm": [50, 4], "sid_cm": 100}, "anode_direction": [1.0, 0.0, 0.0],
            "rotation": {"isocenter": [0, 0, 50], "axis": "y", "scan_length_cm": 20}},
}


def heel_bins(span_cm, n_bins=15):
    """Fixed heel-axis bins standing in for SpekPy's off-axis spectra: the
    reference's bin centres (spectrum.py:103), relative fluence falling
    towards the anode side with its last bin cut off (zero), and Kramers
    spectra (the reference's own fallback, spectrum.py:55-62) hardened by
    0.4 mm Al more per bin towards the anode."""
    from chatcarlo.spectrum import _kramers_fallback_spectrum
    centers = (np.arange(n_bins) + 0.5) / n_bins * 2.0 * span_cm - span_cm
    rel = np.clip(1.0 - 0.9 * (np.arange(n_bins) / (n_bins - 1)) ** 2, 0.0, None)
    rel[-1] = 0.0
    spectra = tuple(_kramers_fallback_spectrum(80.0, 2.5 + 0.4 * i, n_bins=75) for i in range(n_bins))
    return centers, spectra, rel, rel * 1e6


def case_heel():
    """source.py:130-149,195-207 run by the reference itself, with its
    SpekPy-only heel_spectra_for_source replaced by fixed bins; the bins are
    stored with the outputs."""
    out = {}
    base = {"position": [0, -100, 50], "direction": [0, 1, 0], "heel_effect": True, "kvp": 80}
    saved = rsrc.heel_spectra_for_source
    try:
        for k, extra in HEEL_VARIANTS.items():
            src = dict(base, **extra)
            seen = {}

            def fake(src_, sid, span, seen=seen):
                seen["span"] = span
                return heel_bins(span)
            rsrc.heel_spectra_for_source = fake
            p, d, e = rsrc.sample_source_photons(src, 3000, np.random.default_rng(23))
            out[f"{k}_pos"], out[f"{k}_dir"], out[f"{k}_e"] = p, d, e
            centers, spectra, rel, _ = heel_bins(seen["span"])
            out[f"{k}_span"] = np.array(seen["span"])
            out[f"{k}_centers"] = centers
            out[f"{k}_rel"] = rel
            out[f"{k}_spec_e"] = np.stack([a for a, _ in spectra])
            out[f"{k}_spec_w"] = np.stack([b for _, b in spectra])
    finally:
        rsrc.heel_spectra_for_source = saved
    return out


CT_SOURCE = {"position": [0.0, -60.0, 0.0], "direction": [0.0, 1.0, 0.0],
             "field": {"shape": "rect", "size_cm": [50.0, 4.0], "sid_cm": 60.0},
             "rotation": {"isocenter": [0.0, 0.0, 0.0], "axis": "z", "scan_length_cm": 10.0},
             "spectrum": [{"energy_keV": 40.0, "weight": 1.0}, {"energy_keV": 60.0, "weight": 2.0},
                          {"energy_keV": 80.0, "weight": 1.0}],
             "ctdi_vol_mGy": 12.0}


def case_ctdi():
    from chatcarlo import ctdi as rctdi
    import json
    ctdiw, dc, dp = rctdi.ctdi_per_history_Gy(CT_SOURCE, phantom="head", n_histories=4000, seed=9)
    return {"ctdi": np.array([ctdiw, dc, dp]), "source_json": np.array(json.dumps(CT_SOURCE))}


def case_maps():
    """The CLI's output maps (__main__.py:198-209): dose per history from the
    material at each voxel centre (diagnostics.py:16-26), H*(10) per
    history, and the relative-error maps (tally.py:96-100), on a random grid
    state.  Voxel centres sit on integer coordinates, so some lie exactly on
    a box face, the sphere or a cylinder (the closed point tests)."""
    from chatcarlo.diagnostics import dose_map_Gy
    rng = np.random.default_rng(77)
    origin, shape = np.array([-16.5, -4.5, -6.5]), (33, 16, 14)
    grid = rtally.VoxelGrid(origin_cm=origin, shape=shape, voxel_size_cm=1.0, track_uncertainty=True)
    k = rng.lognormal(0.0, 2.0, shape) * (rng.random(shape) < 0.9)
    h = rng.lognormal(1.0, 1.5, shape) * (rng.random(shape) < 0.9)
    grid.kerma_keV[...] = k
    grid.h10_track_pSv_cm3[...] = h
    grid.kerma_sum2[...] = k ** 2 / 1000.0 * rng.uniform(0.5, 3.0, shape)
    grid.h10_sum2[...] = h ** 2 / 1000.0 * rng.uniform(0.5, 3.0, shape)
    grid.n_batches_hit[...] = rng.integers(0, 8, shape)
    grid.n_batches = 7
    grid.n_histories = 12345
    geometry = rgeom.Geometry(GEOMS)
    n = grid.n_histories
    out = {"kerma": k, "h10": h, "k2": grid.kerma_sum2.copy(), "h2": grid.h10_sum2.copy(),
           "nhit": grid.n_batches_hit.copy(), "nb": np.array(7), "nh": np.array(n),
           "dose": dose_map_Gy(grid, geometry) / n, "h10map": grid.h10_map_pSv() / n,
           "krel": grid.kerma_relative_error(), "hrel": grid.h10_relative_error()}
    grid.n_batches = 1                        # fewer than two batches: relative errors undefined
    out["krel_m1"] = grid.kerma_relative_error()
    out["origin"] = origin
    out["shape"] = np.array(shape)
    out["voxel_cm"] = np.array(1.0)
    names = sorted({g["material"] for g in GEOMS} | {"air"})
    out["density_names"] = np.array(names)
    out["density_values"] = np.array([rmat.density(m) for m in names])
    return out


CASES = {"geometry": case_geometry, "materials": case_materials, "samplers": case_samplers,
         "tally": case_tally, "transport": case_transport, "run": case_run, "source": case_source,
         "ctdi": case_ctdi, "maps": case_maps, "heel": case_heel}


def main(names=None):
    for name, fn in CASES.items():
        if names and name not in names:
            continue
        data = fn()
        np.savez_compressed(HERE / f"{name}.npz", **data)
        print(name, sum(v.nbytes for v in data.values() if hasattr(v, "nbytes")), "bytes")


if __name__ == "__main__":
    main(sys.argv[1:])
