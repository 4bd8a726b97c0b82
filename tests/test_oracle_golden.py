"""The CPU oracle reproduces ChatCarlo's own outputs (tests/golden/*.npz).

The fixtures were produced by running the reference modules unmodified
(tests/golden/make_golden.py); the oracle replays the same inputs and
seeds and must match exactly.  This is what makes the oracle trustworthy
as the checker of the GPU engine.
"""
import numpy as np
import pytest

import cc_oracle as O
from chatcarlo_b200 import tables as tb

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


def test_geometry_matches_reference(golden):
    g = golden("geometry")
    geo = O.OracleGeometry(GEOMS)
    np.testing.assert_array_equal(geo.bbox_min, g["bbox_min"])
    np.testing.assert_array_equal(geo.bbox_max, g["bbox_max"])
    np.testing.assert_array_equal(geo.material_at(g["o"]).astype(str), g["mat"])
    t, esc = geo.next_boundary(g["o"], g["d"])
    np.testing.assert_array_equal(t, g["t"])
    np.testing.assert_array_equal(esc, g["escape"])


def test_material_tables_match_reference(golden):
    g = golden("materials")
    e = g["e"]
    for m in MATERIALS:
        p = O.cs_parts(m, e)
        np.testing.assert_array_equal(p["photoelectric"], g[f"{m}__photo"], err_msg=m)
        np.testing.assert_array_equal(p["compton"], g[f"{m}__compt"], err_msg=m)
        np.testing.assert_array_equal(p["rayleigh"], g[f"{m}__rayl"], err_msg=m)
        np.testing.assert_array_equal(O.mu_en_rho(m, e), g[f"{m}__muen"], err_msg=m)
        assert tb.density(m) == float(g[f"{m}__density"])
    np.testing.assert_array_equal(O.h10_per_fluence(g["eh"]), g["h10"])


@pytest.mark.parametrize("z", [1, 8, 20, 26, 29, 74, 82])
def test_element_tables_match_reference(golden, z):
    g = golden("materials")
    ed, om, le, lp = tb.fluorescence_k_data(z)
    np.testing.assert_array_equal(np.concatenate([[ed, om], le, lp]), g[f"k{z}"])
    np.testing.assert_array_equal(tb.rayleigh_form_factor_table(z)[1], g[f"ff{z}"])
    np.testing.assert_array_equal(tb.rayleigh_cumulative_table(z)[1], g[f"ra{z}"])
    np.testing.assert_array_equal(tb.incoherent_sq_table(z)[1], g[f"sq{z}"])
    np.testing.assert_array_equal(tb.element_energy_grid_kev(z), g[f"grid{z}"])


def test_samplers_match_reference(golden):
    g = golden("samplers")
    n = 4000
    for m, e0 in (("water", 60.0), ("bone", 40.0), ("lead", 120.0)):
        mats = np.full(n, m, dtype=object)
        e = np.full(n, e0)
        eps, cos = O.sample_compton_bound(mats, e, np.random.default_rng(11))
        np.testing.assert_array_equal(np.stack([eps, cos]), g[f"compton_{m}"])
        z = O.sample_element(mats, e, np.random.default_rng(12), "rayl")
        np.testing.assert_array_equal(z, g[f"rayl_el_{m}"])
        np.testing.assert_array_equal(O.sample_rayleigh_cos_theta(z, e, np.random.default_rng(13)),
                                      g[f"rayl_cos_{m}"])
        emit, el = O.sample_fluorescence(mats, np.full(n, 100.0), np.random.default_rng(14))
        np.testing.assert_array_equal(np.stack([emit.astype(float), el]), g[f"fluor_{m}"])
    np.testing.assert_array_equal(np.stack(O.sample_klein_nishina(g["kn_e"], np.random.default_rng(15))), g["kn"])
    np.testing.assert_array_equal(
        O.sample_rayleigh_cos_theta_uniform(g["ru_z"], np.full(n, 30.0), np.random.default_rng(16)), g["ru"])
    np.testing.assert_array_equal(O.scatter_direction(g["sd_d"], g["sd_c"], np.random.default_rng(17)), g["sd"])
    np.testing.assert_array_equal(O.isotropic_direction(n, np.random.default_rng(18)), g["iso"])


def test_track_length_tally_matches_reference(golden):
    g = golden("tally")
    grid = O.OracleGrid([-10.0, -8.0, -6.0], (20, 16, 12), 1.0)
    target = np.zeros(grid.shape)
    O.accumulate_track_length(target, grid, g["o"], g["d"], g["L"], g["w"], np.random.default_rng(19))
    np.testing.assert_array_equal(target, g["target"])


def _tp(geoms, start, direction, e0, n, seed, grid_res=None, margin=50.0):
    geo = O.OracleGeometry(geoms, bbox_margin_cm=margin)
    pos = np.tile(np.asarray(start, dtype=float), (n, 1))
    dirv = np.tile(np.asarray(direction, dtype=float), (n, 1))
    en = np.full(n, float(e0))
    grid = None
    if grid_res is not None:
        grid = O.OracleGrid.from_bbox(geo.bbox_min, geo.bbox_max, grid_res)
    r = O.transport_photons(pos, dirv, en, geo, np.random.default_rng(seed), grid=grid)
    return pos, dirv, en, r, grid


def _check_tp(g, prefix, pos, dirv, en, r, grid):
    np.testing.assert_array_equal(pos, g[f"{prefix}_pos"])
    np.testing.assert_array_equal(dirv, g[f"{prefix}_dir"])
    np.testing.assert_array_equal(en, g[f"{prefix}_energy"])
    np.testing.assert_array_equal(r.n_scatter, g[f"{prefix}_n_scatter"])
    np.testing.assert_array_equal(r.absorbed, g[f"{prefix}_absorbed"])
    np.testing.assert_array_equal(r.escaped, g[f"{prefix}_escaped"])
    assert r.n_fluorescence == int(g[f"{prefix}_n_fluor"])
    names = sorted(r.energy_deposited)
    np.testing.assert_array_equal(np.array(names), g[f"{prefix}_dep_names"])
    np.testing.assert_array_equal(np.array([r.energy_deposited[k] for k in names]), g[f"{prefix}_dep"])
    if grid is not None:
        np.testing.assert_array_equal(grid.kerma_keV, g[f"{prefix}_kerma"])
        np.testing.assert_array_equal(grid.h10_track_pSv_cm3, g[f"{prefix}_h10"])


def test_transport_photons_matches_reference(golden):
    g = golden("transport")
    water = [{"name": "slab", "shape": "box", "material": "water", "center": [0, 0, 0],
              "size_cm": [10.0, 100.0, 100.0]}]
    _check_tp(g, "water", *_tp(water, [-15, 0, 0], [1, 0, 0], 60.0, 3000, 1))
    lead = [{"name": "slab", "shape": "box", "material": "lead", "center": [0, 0, 0],
             "size_cm": [0.5, 50.0, 50.0]}]
    _check_tp(g, "lead", *_tp(lead, [-5.25, 0, 0], [1, 0, 0], 100.0, 3000, 42, grid_res=10.0))
    d = np.array([1.0, 0.05, 0.02])
    d /= np.linalg.norm(d)
    _check_tp(g, "mixed", *_tp(GEOMS, [-55, 1, 2], d, 80.0, 2000, 7, grid_res=15.0))


def scene_small(kramers):
    e, w = kramers
    return {
        "source": {"position": [0, 0, 120], "direction": [0, 0, -1],
                   "field": {"shape": "rect", "size_cm": [20, 25], "sid_cm": 150},
                   "spectrum": [{"energy_keV": float(a), "weight": float(b)} for a, b in zip(e, w)]},
        "geometry": [
            {"name": "air", "shape": "box", "material": "air", "center": [0, 0, 30], "size_cm": [150, 150, 150]},
            {"name": "body", "shape": "box", "material": "water", "center": [0, 0, 20], "size_cm": [30, 20, 20]},
            {"name": "bone", "shape": "cylinder", "material": "bone", "axis": "y", "center": [4, 0, 20],
             "radius_cm": 1.5, "height_cm": 18},
            {"name": "pb", "shape": "box", "material": "lead", "center": [0, 0, -20], "size_cm": [30, 30, 0.05]},
        ],
        "physics": {"fluorescence": True},
    }


def test_kramers_spectrum_matches_reference(golden):
    from chatcarlo_b200.source import kramers_spectrum
    g = golden("run")
    np.testing.assert_array_equal(np.stack(kramers_spectrum(80.0, 2.5, n_bins=75)), g["kramers"])


def test_run_transport_matches_reference(golden):
    g = golden("run")
    raw = scene_small(g["kramers"])
    geo = O.OracleGeometry(raw["geometry"])
    spec = {"origin": geo.bbox_min, "shape": tuple(int(x) for x in g["shape"]), "voxel_cm": 20.0}
    agg = O.run_transport(raw, n_histories=12000, seed=5, batch_size=3000, grid_spec=spec,
                          n_workers=1, track_uncertainty=True)
    grid = agg["grid"]
    np.testing.assert_array_equal(grid.origin_cm, g["origin"])
    np.testing.assert_array_equal(grid.kerma_keV, g["kerma"])
    np.testing.assert_array_equal(grid.h10_track_pSv_cm3, g["h10"])
    np.testing.assert_array_equal(grid.kerma_sum2, g["kerma_sum2"])
    np.testing.assert_array_equal(grid.h10_sum2, g["h10_sum2"])
    np.testing.assert_array_equal(grid.n_batches_hit, g["n_hit"])
    assert grid.n_batches == int(g["n_batches"])
    n = 12000
    sc = g["scalars"]
    assert agg["n_absorbed"] / n == sc[0]
    assert agg["n_escaped"] / n == sc[1]
    assert agg["scatter_sum"] / n == sc[2]
    assert agg["n_fluorescence"] == sc[3]
    names = sorted(agg["energy_deposited"])
    np.testing.assert_array_equal(np.array(names), g["dep_names"])
    np.testing.assert_array_equal(np.array([agg["energy_deposited"][k] / 1000.0 for k in names]), g["dep"])
    mom = agg["moments"]
    from chatcarlo_b200.tally import standard_error
    sem = [float(standard_error(mom.sums[k], mom.sum2s[k], mom.n_batches, mom.n_histories)) / 1000.0
           for k in names]
    np.testing.assert_allclose(sem, g["sem"], rtol=1e-12)


def test_source_sampling_matches_reference(golden):
    g = golden("source")
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
        p, d, e = O.sample_source_photons(dict(base, **extra), 2000, np.random.default_rng(21))
        np.testing.assert_array_equal(p, g[f"{k}_pos"], err_msg=k)
        np.testing.assert_array_equal(d, g[f"{k}_dir"], err_msg=k)
        np.testing.assert_array_equal(e, g[f"{k}_e"], err_msg=k)


def test_ctdi_calibration_matches_reference(golden):
    """ctdi.py:53-100 through the oracle: CTDIw, D_center, D_periphery of the
    head phantom, 4000 histories, seed 9 -- identical to the reference."""
    import json
    g = golden("ctdi")
    src = json.loads(str(g["source_json"]))
    got = O.ctdi_per_history_Gy(src, phantom="head", n_histories=4000, seed=9)
    np.testing.assert_array_equal(np.array(got), g["ctdi"])


def test_output_maps_match_reference(golden):
    """Dose and H*(10) per history and the relative-error maps of the CLI
    (chatcarlo/__main__.py:198-209), bit for bit."""
    g = golden("maps")
    dens = dict(zip(g["density_names"].tolist(), g["density_values"].tolist()))
    for m, v in dens.items():
        assert tb.density(m) == v, m
    nh, nb, vox = int(g["nh"]), int(g["nb"]), float(g["voxel_cm"])
    dose = O.dose_map_Gy(g["kerma"], g["origin"], vox, O.OracleGeometry(GEOMS), dens.__getitem__) / nh
    np.testing.assert_array_equal(dose, g["dose"])
    np.testing.assert_array_equal(O.h10_map_pSv(g["h10"], vox) / nh, g["h10map"])
    np.testing.assert_array_equal(O.relative_error(g["kerma"], g["k2"], nb, nh), g["krel"])
    np.testing.assert_array_equal(O.relative_error(g["h10"], g["h2"], nb, nh), g["hrel"])
    np.testing.assert_array_equal(O.relative_error(g["kerma"], g["k2"], 1, nh), g["krel_m1"])
    # centres on a box face, the sphere and the cylinders are part of the case
    c = O.voxel_centers(g["origin"], tuple(g["shape"]), vox)
    assert np.any(np.abs(c[:, 0]) == 15.0)
    assert np.any(np.sum((c - np.array([5.0, -3.0, 2.0])) ** 2, axis=1) == 36.0)


def test_voxel_fixtures_are_consistent():
    """The oracle's configuration-scale voxel fixtures
    (tests/golden/make_voxel_fixtures.py): every stored voxel has a
    positive mean and a relative error under the cut, the masks and arrays
    agree, and the chunk totals add up to the run's history count."""
    from conftest import GOLDEN
    for name in ("plain", "room", "ct_slab"):
        f = np.load(GOLDEN / f"voxels_{name}.npz")
        nv = int(np.prod(f["shape"]))
        assert int(f["chunk_n"].sum()) == int(f["n_histories"])
        for tag in ("kerma", "h10"):
            mask = np.unpackbits(f[f"{tag}_mask"])[:nv].astype(bool)
            assert mask.sum() == f[f"{tag}_mean"].size == f[f"{tag}_rel"].size > 10_000
            assert np.all(f[f"{tag}_mean"] > 0)
            assert np.all(f[f"{tag}_rel"].astype(float) < float(f["rel_cut"]) + 1e-3)
            assert np.all(np.flatnonzero(mask) % int(f["keep_every"]) == 0)


HEEL_VARIANTS = {
    "rect": {"field": {"shape": "rect", "size_cm": [35, 43], "sid_cm": 100}, "anode_direction": [1.0, 0.3, 0.0]},
    "cone": {"field": {"shape": "cone", "diameter_cm": 30, "sid_cm": 100}, "anode_direction": [0.0, 1.0, 0.2]},
    "rot": {"field": {"shape": "rect", "size_cm": [50, 4], "sid_cm": 100}, "anode_direction": [1.0, 0.0, 0.0],
            "rotation": {"isocenter": [0, 0, 50], "axis": "y", "scan_length_cm": 20}},
}


def heel_bins_from_golden(g, k):
    """The fixed heel bins a golden heel case was made with."""
    spectra = tuple((a, b) for a, b in zip(g[f"{k}_spec_e"], g[f"{k}_spec_w"]))
    return g[f"{k}_centers"], spectra, g[f"{k}_rel"], g[f"{k}_rel"] * 1e6


def test_heel_effect_sampling_matches_reference(golden, monkeypatch):
    """source.py:130-149,195-207 (fluence rejection along the heel axis,
    energies from the photon's heel bin) through the oracle, with the bins
    the reference ran with: identical photons."""
    g = golden("heel")
    base = {"position": [0, -100, 50], "direction": [0, 1, 0], "heel_effect": True, "kvp": 80}
    for k, extra in HEEL_VARIANTS.items():
        bins = heel_bins_from_golden(g, k)
        monkeypatch.setattr(O, "heel_spectra_for_source", lambda src, sid, span, b=bins: b)
        p, d, e = O.sample_source_photons(dict(base, **extra), 3000, np.random.default_rng(23))
        np.testing.assert_array_equal(p, g[f"{k}_pos"], err_msg=k)
        np.testing.assert_array_equal(d, g[f"{k}_dir"], err_msg=k)
        np.testing.assert_array_equal(e, g[f"{k}_e"], err_msg=k)
