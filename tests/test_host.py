"""Host-side logic that needs no GPU: scene schema, tables handed to the
engine, statistics helpers, history sharding and the tally reduction over
ranks (world size 2 over gloo)."""
import os
import socket

import numpy as np
import pytest

import cc_oracle as O
from chatcarlo_b200 import devtables, tables as tb, workloads as W
from chatcarlo_b200.scene import validate_scene
from chatcarlo_b200.tally import ScalarMoments, VoxelGrid, relative_error, standard_error


def test_benchmark_scenes_validate():
    for raw in (W.plain_mc(), W.room()):
        sc = validate_scene(raw)
        assert sc.ok, sc.errors


@pytest.mark.parametrize("mutate,path", [
    (lambda r: r["geometry"][0].update(shape="cone"), "geometry[0].shape"),
    (lambda r: r["geometry"][1].update(material="unobtanium"), "geometry[1].material"),
    (lambda r: r["source"].update(spectrum=[{"energy_keV": 200.0, "weight": 1.0}]), "source.spectrum"),
    (lambda r: r["source"].update(kvp=80), "source"),
    (lambda r: r["geometry"][2].update(axis="w"), "geometry[2].axis"),
    (lambda r: r["source"]["field"].update(size_cm=[35.0]), "source.field.size_cm"),
    (lambda r: r["geometry"][1].update(shape="ellipsoid", semi_axes_cm=[3.0, -1.0, 2.0]), "geometry[1].semi_axes_cm"),
])
def test_scene_errors_name_the_entry(mutate, path):
    raw = W.room()
    mutate(raw)
    sc = validate_scene(raw)
    assert not sc.ok
    assert any(e.path == path for e in sc.errors), [str(e) for e in sc.errors]


def test_voxel_grid_from_bbox_matches_reference_rule():
    g = VoxelGrid.from_bbox(np.array([-250.0, -250.0, -50.0]), np.array([250.0, 250.0, 350.0]), 5.0)
    assert g.shape == (100, 100, 80)
    og = O.OracleGrid.from_bbox(np.array([-250.0, -250.0, -50.0]), np.array([250.0, 250.0, 350.0]), 5.0)
    assert og.shape == g.shape
    pts = np.array([[-250.0, -250.0, -50.0], [249.99, 0.0, 0.0], [250.0, 0.0, 0.0]])
    idx, ok = g.voxel_index(pts)
    assert ok.tolist() == [True, True, False]


def test_statistics_helpers_match_oracle_moments():
    rng = np.random.default_rng(0)
    m = O.Moments()
    batches = []
    for n_b in (100, 250, 80, 400):
        s_b = float(rng.normal(10.0, 2.0)) * n_b
        batches.append((s_b, n_b))
        m.add_batch({"x": s_b}, n_b)
    T = sum(s for s, _ in batches)
    Q = sum(s * s / n for s, n in batches)
    N = sum(n for _, n in batches)
    assert m.sums["x"] == pytest.approx(T) and m.sum2s["x"] == pytest.approx(Q)
    se = standard_error(T, Q, 4, N)
    assert se == pytest.approx(np.sqrt((Q - T * T / N) / 3 / N))
    assert relative_error(T, Q, 4, N) == pytest.approx(se / (T / N))
    assert np.isnan(relative_error(T, Q, 1, N))


@pytest.mark.parametrize("material", ["bone", "concrete", "lead", "air"])
def test_union_grid_reproduces_element_interpolation(material):
    """Per element, interpolating the union-grid table gives the element's own
    interpolation (materials.py:248-262); the mixed total differs from the sum
    of interpolated parts only at second order."""
    mt = devtables.build_material(material)
    rng = np.random.default_rng(1)
    e = np.exp(rng.uniform(0.0, np.log(150.0), 3000))
    le = np.log(e)
    idx = np.clip(np.searchsorted(mt.log_e, le), 1, len(mt.log_e) - 1)
    fr = (le - mt.log_e[idx - 1]) / (mt.log_e[idx] - mt.log_e[idx - 1])
    for i, z in enumerate(mt.zs):
        for k, kind in enumerate(("photo", "compt", "rayl")):
            y = mt.log_elem[i, k]
            got = np.exp(y[idx - 1] + fr * (y[idx] - y[idx - 1]))
            want = mt.fractions[i] * O.element_cs(int(z), e, kind)
            np.testing.assert_allclose(got, want, rtol=1e-10)
    y = mt.log_parts[:, 3]
    tot = np.exp(y[idx - 1] + fr * (y[idx] - y[idx - 1]))
    np.testing.assert_allclose(tot, O.mu_rho(material, e), rtol=2e-5)


@pytest.mark.parametrize("material", ["water", "bone", "lead", "concrete", "air"])
def test_node_tally_weights_match_reference_interpolants(material):
    """ln(mu_en/rho) and ln(h*(10)/Phi) interpolated linearly between the
    nodes vs the reference's PCHIP (materials.py:315-335) and log-log
    h*(10) interpolation (dose_coefficients.py:32-42)."""
    mt = devtables.build_material(material)
    e = np.exp(np.random.default_rng(2).uniform(0.0, np.log(150.0), 4000))
    le = np.log(e)
    idx = np.clip(np.searchsorted(mt.log_e, le), 1, len(mt.log_e) - 1)
    fr = (le - mt.log_e[idx - 1]) / (mt.log_e[idx] - mt.log_e[idx - 1])
    y = mt.log_tally
    muen = np.exp(y[idx - 1, 0] + fr * (y[idx, 0] - y[idx - 1, 0]))
    h10 = np.exp(y[idx - 1, 1] + fr * (y[idx, 1] - y[idx - 1, 1]))
    np.testing.assert_allclose(muen, O.mu_en_rho(material, e), rtol=2e-5)
    np.testing.assert_allclose(h10, O.h10_per_fluence(e), rtol=1e-12)


def test_element_tables_for_the_engine():
    el = devtables.build_element(82)
    assert el.emits and el.k_edge == pytest.approx(88.0045)
    assert el.s_over_z[0] == 0.0 and el.s_over_z[-1] == pytest.approx(1.0, rel=0.01)
    assert np.all(np.diff(el.ray_a) > 0)
    assert devtables.build_element(8).emits is False


def test_source_spec_fields():
    from chatcarlo_b200.source import SourceSpec, beam_basis
    for d in ([0, 0, 1.0], [0, 1.0, 0], [0.6, 0.0, -0.8]):
        u, v = beam_basis(np.array(d))
        m = np.stack([u, v, np.array(d)])
        np.testing.assert_allclose(m @ m.T, np.eye(3), atol=1e-12)
    spec = SourceSpec(W.room()["source"])
    assert spec.desc.n_energies == 75 and spec.desc.sid_cm == 180.0
    with pytest.raises(ValueError):
        SourceSpec(dict(W.room()["source"], heel_effect=True))      # no anode_direction


def test_cli_parser():
    from chatcarlo_b200.__main__ import build_parser
    a = build_parser().parse_args(["run", "s.yaml", "-n", "1e6", "--seed", "3", "--dose-grid",
                                   "--resolution", "2.5", "--dose-out", "d.npz"])
    assert a.n_histories == 1e6 and a.seed == 3 and a.dose_grid and a.resolution == 2.5


def test_shard_ranges_partition_the_histories():
    from chatcarlo_b200.distributed import shard_range
    for n, w in ((10, 3), (1000003, 8), (5, 8)):
        parts = [shard_range(n, r, w) for r in range(w)]
        assert sum(c for _, c in parts) == n
        firsts = [f for f, _ in parts]
        assert firsts == sorted(firsts)
        for (f, c), (g, _) in zip(parts, parts[1:]):
            assert f + c == g


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from chatcarlo_b200.distributed import reduce_result
    from chatcarlo_b200.transport import TransportResult
    g = VoxelGrid(origin_cm=np.zeros(3), shape=(4, 3, 2), voxel_size_cm=1.0, track_uncertainty=True)
    g.kerma_keV += rank + 1.0
    g.h10_track_pSv_cm3 += 10.0 * (rank + 1)
    g.kerma_sum2 += 0.5
    g.h10_sum2 += 0.25
    g.n_batches_hit += 1
    g.n_batches, g.n_histories = 3, 300
    # per-material batch moments (keV): rank 0 deposits in water and lead,
    # rank 1 in water and air, so each rank lacks a name the other has
    mom = ScalarMoments()
    for b in range(5):
        vals = {"water": 100.0 * (rank + 1) + b}
        vals["lead" if rank == 0 else "air"] = 7.0 + b
        mom.add_batch(vals, 200)
    dep = {k: v / 1000.0 for k, v in mom.sums.items()}
    res = TransportResult(n_histories=1000, energy_deposited_MeV=dep, fraction_absorbed=0.25 * (rank + 1),
                          fraction_escaped=0.5, mean_scatter_events=2.0, grid=g, n_fluorescence=7, n_batches=5,
                          moments=mom)
    reduce_result(res)
    q.put((rank, float(g.kerma_keV.sum()), float(g.h10_track_pSv_cm3[0, 0, 0]), int(g.n_batches_hit.max()),
           g.n_batches, g.n_histories, res.n_histories, res.fraction_absorbed, res.n_fluorescence,
           res.n_batches, res.energy_deposited_MeV, res.energy_deposited_sem_MeV, res.energy_deposited_rel_err))
    dist.destroy_process_group()


def _merged_reference():
    """The two ranks' batches merged the way the reference merges process
    workers (ScalarMoments.merge_from, transport.py:420-437)."""
    mom = ScalarMoments()
    for rank in range(2):
        for b in range(5):
            vals = {"water": 100.0 * (rank + 1) + b}
            vals["lead" if rank == 0 else "air"] = 7.0 + b
            mom.add_batch(vals, 200)
    return mom


def test_tally_reduction_over_two_ranks():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    want = _merged_reference()
    for rank, ksum, h0, nhit, nb, nh, n, fa, nfl, nbat, dep, sem, rel in out:
        assert ksum == pytest.approx(24 * 3.0)
        assert h0 == pytest.approx(30.0)
        assert nhit == 2 and nb == 6 and nh == 600 and n == 2000 and nfl == 14 and nbat == 10
        assert fa == pytest.approx((250 + 500) / 2000)
        assert set(dep) == {"water", "lead", "air"}
        for k in dep:
            assert dep[k] == pytest.approx(want.sums[k] / 1000.0)
            assert sem[k] == pytest.approx(want.standard_errors()[k] / 1000.0)
            assert rel[k] == pytest.approx(want.relative_errors()[k])
        assert sem["water"] > 0


def test_ellipsoid_extension_primitive():
    """The axis-aligned ellipsoid (an extension for the denoiser phantoms):
    the validator accepts it, the host packs full axis lengths, and the
    oracle's roots lie on the surface and bracket the inside."""
    from chatcarlo_b200.geometry import Geometry, contains
    g = {"name": "e", "shape": "ellipsoid", "material": "water", "center": [1.0, -2.0, 3.0],
         "semi_axes_cm": [4.0, 2.0, 7.0]}
    raw = W.plain_mc()
    raw["geometry"].append(g)
    assert validate_scene(raw).ok
    geo = Geometry(raw["geometry"])
    prim = geo.primitives({"air": 0, "water": 1})[2]
    assert prim.type == 3 and list(prim.size) == [8.0, 4.0, 14.0]
    rng = np.random.default_rng(0)
    o = rng.uniform(-12, 12, (2000, 3))
    d = rng.normal(size=(2000, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    t1, t2 = O._ellipsoid(o, d, g["center"], g["semi_axes_cm"])
    hit = ~np.isnan(t1)
    assert hit.sum() > 100
    for t in (t1, t2):
        q = (o[hit] + t[hit, None] * d[hit] - np.array(g["center"])) / np.array(g["semi_axes_cm"])
        np.testing.assert_allclose(np.sum(q * q, axis=1), 1.0, atol=1e-9)
    mid = o[hit] + 0.5 * (t1[hit] + t2[hit])[:, None] * d[hit]
    assert np.all(contains(g, mid)) and np.all(O._contains(g, mid))


def test_unet_oracle_gradients_match_finite_differences():
    """The FP64 oracle's backward pass (no BF16 rounding) against central
    differences of its own loss on an 8^3 volume."""
    import unet_oracle as UO
    from chatcarlo_b200 import denoiser as DN
    rng = np.random.default_rng(0)
    B, S = 1, 8
    xlog = rng.normal(size=(B, S, S, S))
    mat = rng.integers(0, 4, size=(B, S, S, S)).astype(np.uint8)
    dens = np.array([0.0012, 1.0, 1.85, 11.35])[mat]
    target = rng.normal(size=(B, S, S, S))
    weight = np.where(mat > 0, 1.0, 0.1)
    p = DN.init_params(1).astype(np.float64)
    ho = DN.param_layout()["head"][0]
    p[ho:ho + 17] = rng.normal(0, 0.3, 17)
    for L in DN.LAYERS:
        _, _, bo, bn = DN.param_layout()[L.name]
        p[bo:bo + bn] = 0.05
    _, g, _ = UO.loss_and_grads(p, xlog, dens, mat, target, weight, bf16_storage=False)
    lay = DN.param_layout()
    picks = [lay[n][0] + 3 for n in ("e0a", "e2", "b3", "d2a", "d0")] + [lay["d1a"][2], lay["head"][0] + 2, ho + 16]
    for i in picks:
        h = 1e-5
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (UO.loss_and_grads(pp, xlog, dens, mat, target, weight, False)[0] -
              UO.loss_and_grads(pm, xlog, dens, mat, target, weight, False)[0]) / (2 * h)
        assert abs(fd - g[i]) < 1e-5 + 1e-3 * abs(fd), (i, fd, g[i])


def test_denoiser_phantoms_validate_and_map_materials():
    from chatcarlo_b200 import phantoms as PH
    scenes, grids = PH.phantoms(4, 3, side=16, voxel_cm=1.0)
    for sc, gr in zip(scenes, grids):
        assert validate_scene(sc).ok
        mat, dens = PH.voxel_maps(sc, gr)
        assert mat.shape == (16, 16, 16) and mat.max() < 4
        assert np.any(mat == 1)                       # the water body
        np.testing.assert_allclose(dens[mat == 1], 1.0)


def test_histories_for_error_interpolates_in_log_log():
    from chatcarlo_b200.denoise_run import histories_for_error
    h = [1e5, 4e5, 1.6e6]
    e = [0.08, 0.04, 0.02]                       # exactly 1/sqrt(n)
    assert histories_for_error(h, e, 0.02) == pytest.approx(1.6e6)
    assert histories_for_error(h, e, 0.0283) == pytest.approx(8e5, rel=1e-2)
    assert histories_for_error(h, e, 0.01) is None
    assert histories_for_error(h, [0.01, 0.009, 0.008], 0.02) == 1e5


def test_shipped_denoiser_parameters_load():
    from chatcarlo_b200 import denoiser as DN
    p, meta = DN.load_params()
    assert p.shape == (DN.n_params(),) and np.all(np.isfinite(p))
    assert meta["uncertainty_channel"] is True and meta["held_out"]["time_to_2pct_s"]["speedup"] > 1
    import tempfile, os
    with tempfile.TemporaryDirectory() as d:
        DN.save_params(os.path.join(d, "p.npz"), p, meta)
        q, m2 = DN.load_params(os.path.join(d, "p.npz"))
    np.testing.assert_array_equal(p, q)


@pytest.mark.parametrize("n", [64, 65, 150, 320, 111])
def test_ct_denoiser_tiles_cover_each_voxel_once_from_inside_a_tile(n):
    """Tiled inference of the CT denoiser: the tiles cover the axis, the
    owned ranges partition it, and every owned range lies in its tile at
    least 8 voxels from an inner tile edge."""
    from chatcarlo_b200.ct_denoise import TILE, owned_bounds, tile_starts
    s = tile_starts(n)
    b = owned_bounds(s, n)
    assert s[0] == 0 and s[-1] == n - TILE and all(0 < s[i + 1] - s[i] <= 48 for i in range(len(s) - 1))
    assert b[0] == 0 and b[-1] == n and all(b[i] < b[i + 1] for i in range(len(b) - 1))
    for i, st in enumerate(s):
        assert st <= b[i] and b[i + 1] <= st + TILE
        if i > 0:
            assert b[i] - st >= 8
        if i < len(s) - 1:
            assert st + TILE - b[i + 1] >= 8


def test_ct_phantoms_are_valid_scenes():
    from chatcarlo_b200.ct_denoise import CT_MATERIALS, ct_phantom
    from chatcarlo_b200.scene import validate_scene
    rng = np.random.default_rng(3)
    for _ in range(20):
        sc = ct_phantom(rng)
        rep = validate_scene(sc)
        assert rep.ok, rep.errors
        assert all(g["material"] in CT_MATERIALS for g in sc["geometry"])
        body = sc["geometry"][0]
        for g in sc["geometry"][1:]:
            assert np.hypot(*g["center"][:2]) + g["radius_cm"] <= body["radius_cm"]
            assert abs(g["center"][2]) + g["height_cm"] / 2 <= 7.5 + 1e-9


def test_denoiser_volume_shapes():
    """The network takes cubic (S) or non-cubic (D, H, W) volumes whose
    sides are multiples of 8 (three 2x2x2 poolings)."""
    from chatcarlo_b200.denoiser import UNet3D
    assert UNet3D._side3(64) == (64, 64, 64)
    assert UNet3D._side3((320, 320, 152)) == (320, 320, 152)
    for bad in (12, (16, 30, 8), (16, 16), (0, 8, 8)):
        with pytest.raises(ValueError):
            UNet3D._side3(bad)


def test_heel_effect_without_spekpy_raises():
    """Without SpekPy's off-axis spectra the heel effect cannot be set up;
    the reference raises the same way (spectrum.py:97-99)."""
    from chatcarlo_b200.source import SourceSpec
    src = {"position": [0, -100, 50], "direction": [0, 1, 0], "heel_effect": True, "kvp": 80,
           "field": {"shape": "rect", "size_cm": [35, 43], "sid_cm": 100}, "anode_direction": [1.0, 0.3, 0.0]}
    with pytest.raises(RuntimeError):
        SourceSpec(src)


def test_heel_descriptor_from_supplied_bins(monkeypatch):
    """With bins supplied (as SpekPy would give them), the source descriptor
    carries the heel axis, span and the concatenated per-bin spectra."""
    import chatcarlo_b200.source as S
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "heel.npz"))
    spectra = tuple((a, b) for a, b in zip(g["rect_spec_e"], g["rect_spec_w"]))
    bins = (g["rect_centers"], spectra, g["rect_rel"], g["rect_rel"])
    monkeypatch.setattr(S, "heel_spectra_for_source", lambda src, sid, span, n_bins=15: bins)
    src = {"position": [0, -100, 50], "direction": [0, 1, 0], "heel_effect": True, "kvp": 80,
           "field": {"shape": "rect", "size_cm": [35, 43], "sid_cm": 100}, "anode_direction": [1.0, 0.3, 0.0]}
    spec = S.SourceSpec(src)
    h = spec.desc.heel.contents
    assert h.n_bins == 15 and h.span_cm == pytest.approx(float(g["rect_span"]))
    assert h.h_u ** 2 + h.h_v ** 2 == pytest.approx(1.0)
    assert sum(h.bin_sizes[i] for i in range(15)) == sum(len(e) for e, _ in spectra)
    with pytest.raises(ValueError):
        S.SourceSpec(dict(src, field={"shape": "parallel", "size_cm": [10, 10]}))
