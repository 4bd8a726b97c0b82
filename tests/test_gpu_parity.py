"""GPU engine vs the CPU oracle (statistical parity) and known answers.

The engine draws Philox streams, the oracle NumPy's PCG64, so results are
compared as estimates with their statistical errors: differences are
measured in units of the combined standard error (|z| < 4 per quantity, a
chi^2 per degree of freedom <= 1.2 for voxel maps).
"""
import numpy as np
import pytest

import cc_oracle as O
from chatcarlo_b200 import workloads as W
from chatcarlo_b200.geometry import Geometry

pytestmark = pytest.mark.gpu

MIXED = [
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


def _gpu_tp(engine, geoms, start, direction, e0, n, seed, fluor=True, grid=None):
    from chatcarlo_b200.transport import transport_photons
    pos, dirv, en = W.pencil_beam_arrays(n, start, direction, e0)
    r = transport_photons(pos, dirv, en, Geometry(geoms), seed=seed, fluorescence_enabled=fluor,
                          grid=grid, engine=engine)
    return pos, dirv, en, r


def _z(p1, n1, p2, n2):
    se = np.sqrt(p1 * (1 - p1) / n1 + p2 * (1 - p2) / n2)
    return (p1 - p2) / max(se, 1e-300)


@pytest.mark.parametrize("material,thick,e0", [("water", 10.0, 60.0), ("lead", 0.2, 80.0)])
def test_beer_lambert_primary_transmission(engine, material, thick, e0):
    """Uncollided fraction vs exp(-sum mu t) (tests/test_transport.py:30-51),
    including the air path to the world boundary."""
    geoms = [{"name": "slab", "shape": "box", "material": material, "center": [0, 0, 0],
              "size_cm": [thick, 100.0, 100.0]}]
    n = 1_000_000
    x0 = -thick / 2 - 10.0
    _, _, _, r = _gpu_tp(engine, geoms, [x0, 0, 0], [1, 0, 0], e0, n, seed=1)
    unc = np.mean(r.escaped & (r.n_scatter == 0))
    air_path = 10.0 + 50.0
    expect = float(np.exp(-O.linear_mu(material, e0)[0] * thick - O.linear_mu("air", e0)[0] * air_path))
    se = np.sqrt(expect * (1 - expect) / n)
    assert abs(unc - expect) < 3.0 * se, (unc, expect, se)


@pytest.mark.parametrize("fluor", [True, False])
def test_energy_conservation(engine, fluor):
    """deposited + escaped == incident (tests/test_fluorescence.py:80-97);
    photon energies are FP32 on the device, so the bound is 1e-6 relative."""
    geoms = [{"name": "slab", "shape": "box", "material": "lead", "center": [0, 0, 0],
              "size_cm": [0.5, 50.0, 50.0]}]
    n = 200_000
    _, _, en, r = _gpu_tp(engine, geoms, [-5.25, 0, 0], [1, 0, 0], 100.0, n, seed=42, fluor=fluor)
    dep = sum(r.energy_deposited.values())
    esc = float(np.sum(r.final_energy[r.escaped]))
    assert abs(dep + esc - 100.0 * n) / (100.0 * n) < 1e-6
    assert (r.n_fluorescence > 0) == fluor


def test_no_fluorescence_below_k_edge(engine):
    geoms = [{"name": "slab", "shape": "box", "material": "lead", "center": [0, 0, 0],
              "size_cm": [0.5, 50.0, 50.0]}]
    _, _, _, r = _gpu_tp(engine, geoms, [-5.25, 0, 0], [1, 0, 0], 87.0, 100_000, seed=8)
    assert r.n_fluorescence == 0


def test_transport_photons_statistics_match_oracle(engine):
    """Per-photon outcome frequencies and deposited energy per material on a
    scene with every primitive type."""
    d = np.array([1.0, 0.05, 0.02])
    d /= np.linalg.norm(d)
    start = [-55.0, 1.0, 2.0]
    ng, no = 2_000_000, 100_000
    _, _, eg, rg = _gpu_tp(engine, MIXED, start, d, 80.0, ng, seed=3)
    geo = O.OracleGeometry(MIXED)
    pos, dirv, eo = W.pencil_beam_arrays(no, start, d, 80.0)
    ro = O.transport_photons(pos, dirv, eo, geo, np.random.default_rng(4))
    for name, a, b in (("absorbed", rg.absorbed, ro.absorbed), ("escaped", rg.escaped, ro.escaped),
                       ("unscattered", rg.n_scatter == 0, ro.n_scatter == 0)):
        z = _z(a.mean(), ng, b.mean(), no)
        assert abs(z) < 4, (name, a.mean(), b.mean(), z)
    for k in (1, 2, 3):
        z = _z(np.mean(rg.n_scatter == k), ng, np.mean(ro.n_scatter == k), no)
        assert abs(z) < 4, ("n_scatter", k, z)
    # escaped spectrum: 40 bins, chi^2 of two multinomial samples
    bins = np.linspace(0, 80.0001, 41)
    hg, _ = np.histogram(eg[rg.escaped], bins)
    ho, _ = np.histogram(eo[ro.escaped], bins)
    m = (hg + ho) > 20
    pg, po = hg[m] / ng, ho[m] / no
    var = pg / ng + po / no
    chi2 = np.sum((pg - po) ** 2 / var) / m.sum()
    assert chi2 < 1.6, chi2
    # deposited energy per material (per photon), SE from the binomial-like bound
    for mat in set(ro.energy_deposited) | set(rg.energy_deposited):
        g = rg.energy_deposited.get(mat, 0.0) / ng
        o = ro.energy_deposited.get(mat, 0.0) / no
        if o == 0 and g == 0:
            continue
        rel = abs(g - o) / max(o, g)
        assert rel < max(0.05, 6.0 / np.sqrt(no * max(o, g) / 80.0)), (mat, g, o)


def _small_scene():
    from chatcarlo_b200.source import kramers_spectrum
    e, w = kramers_spectrum(80.0, 2.5, n_bins=75)
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


def _voxel_chi2(t1, q1, m1, n1, t2, q2, m2, n2, min_rel=0.25):
    from chatcarlo_b200.tally import standard_error
    mean1, mean2 = t1 / n1, t2 / n2
    s1 = standard_error(t1, q1, m1, n1)
    s2 = standard_error(t2, q2, m2, n2)
    with np.errstate(divide="ignore", invalid="ignore"):
        ok = (mean1 > 0) & (mean2 > 0) & (s1 / mean1 < min_rel) & (s2 / mean2 < min_rel)
    z = (mean1[ok] - mean2[ok]) / np.sqrt(s1[ok] ** 2 + s2[ok] ** 2)
    return float(np.mean(z ** 2)), int(ok.sum()), float(np.max(np.abs(z))) if ok.any() else 0.0


@pytest.mark.parametrize("scene_fn,grid_spec,n_gpu,n_cpu", [
    ("small", None, 8_000_000, 150_000),
])
def test_voxel_tallies_match_oracle(engine, scene_fn, grid_spec, n_gpu, n_cpu):
    """Kerma and H*(10) per voxel: GPU vs oracle within the combined batch
    uncertainty (chi^2/dof <= 1.2)."""
    from chatcarlo_b200.transport import run_transport
    raw = _small_scene()
    geo = O.OracleGeometry(raw["geometry"])
    spec = {"origin": geo.bbox_min, "shape": tuple(int(np.ceil(x / 10.0)) for x in geo.bbox_max - geo.bbox_min),
            "voxel_cm": 10.0}
    agg = O.run_transport(raw, n_histories=n_cpu, seed=11, batch_size=n_cpu // 60, grid_spec=spec,
                          n_workers=1, track_uncertainty=True)
    og = agg["grid"]
    g = W.make_grid(spec)
    res = run_transport(raw, n_histories=n_gpu, seed=12, batch_size=n_gpu // 100, dose_grid=True, grid=g,
                        engine=engine)
    for name, tg, qg, to, qo in (("kerma", g.kerma_keV, g.kerma_sum2, og.kerma_keV, og.kerma_sum2),
                                 ("h10", g.h10_track_pSv_cm3, g.h10_sum2, og.h10_track_pSv_cm3, og.h10_sum2)):
        chi2, nv, zmax = _voxel_chi2(tg, qg, g.n_batches, g.n_histories, to, qo, og.n_batches, og.n_histories)
        assert nv > 50, (name, nv)
        assert chi2 <= 1.2, (name, chi2, nv, zmax)
    # scalar outcomes
    for key, gv in (("n_absorbed", res.fraction_absorbed), ("n_escaped", res.fraction_escaped)):
        z = _z(gv, n_gpu, agg[key] / n_cpu, n_cpu)
        assert abs(z) < 4, (key, gv, agg[key] / n_cpu)
    # collision estimator per material within its batch uncertainty
    for mat, v in agg["energy_deposited"].items():
        mom = agg["moments"]
        from chatcarlo_b200.tally import standard_error
        se_o = float(standard_error(mom.sums[mat], mom.sum2s[mat], mom.n_batches, mom.n_histories))
        g_mean = res.energy_deposited_MeV.get(mat, 0.0) * 1000.0 / n_gpu
        se_g = res.energy_deposited_sem_MeV.get(mat, 0.0) * 1000.0
        z = (g_mean - v / n_cpu) / np.sqrt(se_o ** 2 + se_g ** 2)
        assert abs(z) < 4, (mat, g_mean, v / n_cpu, z)


def test_collision_and_track_length_estimators_agree(engine):
    """Total kerma in the water box vs the collision estimator
    (tests/test_tally.py:54-75: within 5 %)."""
    from chatcarlo_b200.transport import run_transport
    raw = W.plain_mc()
    g = W.make_grid(W.PLAIN_MC_GRID)
    res = run_transport(raw, n_histories=2_000_000, seed=42, dose_grid=True, grid=g, engine=engine)
    coll = res.energy_deposited_MeV["water"]
    track = g.total_kerma_MeV()
    assert abs(track - coll) / coll < 0.05, (track, coll)


def test_reproducible_and_launch_shape_independent(engine):
    """Same seed -> identical per-photon results, whatever the launch shape,
    and the same kerma up to the order of the FP64 additions.  The last run
    sums in FP32 scratch cells: a monoenergetic pencil beam is their worst
    case (equal scores round alike), so the busiest voxels may move by a few
    1e-4 relative while the median voxel stays at FP32 rounding."""
    d = np.array([1.0, 0.05, 0.02])
    d /= np.linalg.norm(d)
    out, kerma = [], []
    for block, per_sm in ((256, 0), (128, 3), (64, 1), (256, 0), (256, 0)):
        engine.set_launch(block, per_sm)
        engine.set_tally_fp32(len(out) == 4)
        g = W.make_grid({"origin": (-60.0, -50.0, -45.0), "shape": (60, 50, 45), "voxel_cm": 2.0},
                        track_uncertainty=False)
        p, dv, e, r = _gpu_tp(engine, MIXED, [-55.0, 1.0, 2.0], d, 80.0, 200_000, seed=99, grid=g)
        out.append((p, dv, e, r.n_scatter, r.absorbed, r.escaped))
        kerma.append(g.kerma_keV.copy())
    engine.set_launch(256, 0)
    engine.set_tally_fp32(False)
    # BatchResult's types as in the reference (transport.py:86-93)
    assert out[0][3].dtype == np.int64 and out[0][4].dtype == bool and out[0][5].dtype == bool
    for other, k in zip(out[1:], kerma[1:4]):
        for a, b in zip(out[0], other):
            np.testing.assert_array_equal(a, b)
        np.testing.assert_allclose(k, kerma[0], rtol=1e-9, atol=1e-12)
    for a, b in zip(out[0], out[4]):
        np.testing.assert_array_equal(a, b)
    k32, k64 = kerma[4], kerma[0]
    np.testing.assert_allclose(k32, k64, rtol=5e-3, atol=1e-6 * float(np.max(k64)))
    sel = k64 > 0
    assert float(np.median(np.abs(k32[sel] - k64[sel]) / k64[sel])) < 1e-5
    assert abs(k32.sum() - k64.sum()) / k64.sum() < 2e-4


def test_deferred_tally_scores_the_same_pieces(engine):
    """The deferred tally (segments queued, scored by a second kernel) and
    its overflow path (a 1,000-record queue: the rest scored in place) give
    the in-kernel tally's kerma and H*(10) up to the order of the FP64
    additions, through transport_photons and through run_transport with
    batch statistics."""
    from chatcarlo_b200.transport import run_transport
    d = np.array([1.0, 0.05, 0.02])
    d /= np.linalg.norm(d)
    spec = {"origin": (-60.0, -50.0, -45.0), "shape": (60, 50, 45), "voxel_cm": 2.0}
    tp, runs = [], []
    try:
        for on, cap in ((False, 0), (True, 0), (True, 1000)):
            engine.set_tally_queue(on, cap)
            g = W.make_grid(spec, track_uncertainty=False)
            _, _, _, r = _gpu_tp(engine, MIXED, [-55.0, 1.0, 2.0], d, 80.0, 200_000, seed=99, grid=g)
            tp.append((g.kerma_keV.copy(), g.h10_track_pSv_cm3.copy()))
            gr = W.make_grid(W.ROOM_GRID, track_uncertainty=True)
            res = run_transport(W.room(), n_histories=600_000, seed=4, batch_size=100_000, dose_grid=True, grid=gr,
                                engine=engine)
            runs.append((gr, res))
    finally:
        engine.set_tally_queue(False, 0)
    for k, h in tp[1:]:
        np.testing.assert_allclose(k, tp[0][0], rtol=1e-9, atol=1e-12)
        np.testing.assert_allclose(h, tp[0][1], rtol=1e-9, atol=1e-12)
    g0, r0 = runs[0]
    for g, r in runs[1:]:
        assert r.n_voxel_visits == r0.n_voxel_visits and r.n_steps == r0.n_steps
        for a in ("kerma_keV", "h10_track_pSv_cm3", "kerma_sum2", "h10_sum2"):
            np.testing.assert_allclose(getattr(g, a), getattr(g0, a), rtol=1e-9, atol=1e-12)
        np.testing.assert_array_equal(g.n_batches_hit, g0.n_batches_hit)


def test_source_sampling_matches_oracle(engine):
    """Device source sampling vs source.py distributions (rect with rotation
    and helical shift): means and spreads of positions/directions."""
    import ctypes as C
    from chatcarlo_b200 import _native as N
    from chatcarlo_b200.source import SourceSpec
    src = {"position": [0, -100, 50], "direction": [0, 1, 0],
           "field": {"shape": "rect", "size_cm": [50, 4], "sid_cm": 100},
           "rotation": {"isocenter": [0, 0, 50], "axis": "z", "scan_length_cm": 30},
           "spectrum": [{"energy_keV": 30.0, "weight": 1.0}, {"energy_keV": 60.0, "weight": 3.0},
                        {"energy_keV": 90.0, "weight": 2.0}]}
    n = 400_000
    spec = SourceSpec(src)
    h = engine.source(spec)
    pos, dirv, en = np.empty((n, 3)), np.empty((n, 3)), np.empty(n)
    N.check(engine.lib.cc_sample_source(engine.ctx, h, n, 5, 0, N.dptr(pos), N.dptr(dirv), N.dptr(en)))
    engine.lib.cc_source_destroy(h)
    po, do, eo = O.sample_source_photons(src, n, np.random.default_rng(5))
    for a, b in ((pos, po), (dirv, do)):
        np.testing.assert_allclose(a.mean(axis=0), b.mean(axis=0), atol=5 * (a.std(axis=0).max() + 1e-9) / np.sqrt(n) + 1e-6)
        np.testing.assert_allclose(a.std(axis=0), b.std(axis=0), rtol=0.01, atol=1e-3)
    for ek in (30.0, 60.0, 90.0):
        assert abs(np.mean(en == ek) - np.mean(eo == ek)) < 0.005


def test_grazing_photons_on_a_thin_sheet(engine):
    """Photons starting on the face of a 0.05 cm lead sheet at a grazing
    angle: FP32 positions cannot resolve their normal motion per step, yet
    they must enter the sheet like the FP64 oracle's photons do."""
    geoms = [{"name": "air", "shape": "box", "material": "air", "center": [0, 0, 50], "size_cm": [100, 100, 100]},
             {"name": "pb", "shape": "box", "material": "lead", "center": [0, 0, 40], "size_cm": [30, 30, 0.05]}]
    d = np.array([0.995934, -0.09004128, -0.00283073])
    d /= np.linalg.norm(d)
    start = [0.8246886, -11.880426, 40.025]
    engine.set_step_limit(2000)
    try:
        _, _, _, rg = _gpu_tp(engine, geoms, start, d, 59.0, 200_000, seed=6)
    finally:
        engine.set_step_limit(100_000)
    pos, dirv, eo = W.pencil_beam_arrays(20_000, start, d, 59.0)
    ro = O.transport_photons(pos, dirv, eo, O.OracleGeometry(geoms), np.random.default_rng(6))
    z = _z(rg.absorbed.mean(), 200_000, ro.absorbed.mean(), 20_000)
    assert abs(z) < 4, (rg.absorbed.mean(), ro.absorbed.mean())


def test_room_scene_has_no_runaway_histories(engine):
    """Regression: with seed 6 one history of the room scene used to slide
    along the lead sheet's face for 28,404 steps."""
    from chatcarlo_b200.transport import run_transport
    engine.set_step_limit(2000)
    try:
        r = run_transport(W.room(), n_histories=8_000_000, seed=6, batch_size=200_000, engine=engine)
    finally:
        engine.set_step_limit(100_000)
    assert r.n_steps / 8e6 < 10


@pytest.mark.parametrize("shape,radial", [("cylinder", -0.0129), ("cylinder", 0.0116), ("sphere", -0.004),
                                          ("sphere", 0.004)])
def test_photons_on_a_curved_surface_moving_almost_tangentially(engine, shape, radial):
    """Regression: photons reaching a cylinder's side (or a sphere) almost
    tangentially, inwards (radial < 0) or outwards, used to find the surface
    they sit on again ~7e-5 cm ahead on every step (the quadratic's rounding
    at grazing incidence) without their other coordinates changing in FP32.
    They start 5 cm before the grazing point, so they reach it by transport."""
    c = np.array([27.422334795238072, 29.138725523972028, -23.009566507349323])
    r = 18.660725241821535
    g = {"name": "p", "shape": shape, "material": "pmma", "center": list(c), "radius_cm": r}
    if shape == "cylinder":
        g.update(axis="x", height_cm=80.0)
    geoms = [{"name": "air", "shape": "box", "material": "air", "center": [0, 0, 0], "size_cm": [200, 200, 200]}, g]
    nrm = np.array([0.0, -0.553, -0.833])
    nrm /= np.linalg.norm(nrm)
    start = c + r * nrm
    tang = np.cross(nrm, [0.0, 0.0, 1.0]) if shape == "sphere" else np.array([1.0, 0.0, 0.0])
    tang /= np.linalg.norm(tang)
    d = tang + radial * nrm
    d /= np.linalg.norm(d)
    start = start - 5.0 * d
    engine.set_step_limit(2000)
    try:
        _, _, _, rg = _gpu_tp(engine, geoms, start, d, 86.0, 200_000, seed=6)
    finally:
        engine.set_step_limit(100_000)
    pos, dirv, eo = W.pencil_beam_arrays(20_000, start, d, 86.0)
    ro = O.transport_photons(pos, dirv, eo, O.OracleGeometry(geoms), np.random.default_rng(6))
    for sel_g, sel_o in ((rg.escaped & (rg.n_scatter == 0), ro.escaped & (ro.n_scatter == 0)),
                         (rg.escaped, ro.escaped)):
        pg, po = np.mean(sel_g), np.mean(sel_o)
        assert abs(_z(pg, 200_000, po, 20_000)) < 4, (pg, po)


def test_ellipsoid_transmission_and_oblique_rays(engine):
    """The ellipsoid extension primitive: uncollided transmission along its
    x axis vs exp(-sum mu t), and an oblique pencil beam vs the oracle."""
    geoms = [{"name": "e", "shape": "ellipsoid", "material": "water", "center": [0, 0, 0],
              "semi_axes_cm": [5.0, 8.0, 3.0]}]
    n = 1_000_000
    _, _, _, r = _gpu_tp(engine, geoms, [-15.0, 0, 0], [1, 0, 0], 60.0, n, seed=3)
    unc = np.mean(r.escaped & (r.n_scatter == 0))
    expect = float(np.exp(-O.linear_mu("water", 60.0)[0] * 10.0 - O.linear_mu("air", 60.0)[0] * 60.0))
    assert abs(unc - expect) < 3.0 * np.sqrt(expect * (1 - expect) / n), (unc, expect)
    d = np.array([0.8, 0.5, 0.33])
    d /= np.linalg.norm(d)
    start = np.array([1.0, 2.0, -0.5]) - 12.0 * d
    _, _, _, rg = _gpu_tp(engine, geoms, start, d, 60.0, 400_000, seed=4)
    pos, dirv, eo = W.pencil_beam_arrays(40_000, start, d, 60.0)
    ro = O.transport_photons(pos, dirv, eo, O.OracleGeometry(geoms), np.random.default_rng(4))
    for sel_g, sel_o in ((rg.escaped & (rg.n_scatter == 0), ro.escaped & (ro.n_scatter == 0)),
                         (rg.absorbed, ro.absorbed)):
        pg, po = np.mean(sel_g), np.mean(sel_o)
        assert abs(_z(pg, 400_000, po, 40_000)) < 4, (pg, po)


def test_chunked_host_transport_equals_one_device_launch(engine):
    """cc_transport_photons overlaps its copies with the transport from 2^21
    photons on (three chunks on copy streams); per photon the results equal
    one launch of cc_transport_photons_device over the same photons and
    seed, and the kerma equals it up to the order of the FP64 additions."""
    import ctypes as C
    import torch
    from chatcarlo_b200 import _native as N
    from chatcarlo_b200.transport import DeviceGrid
    n, seed = 2_500_000, 77
    d = np.array([1.0, 0.05, 0.02])
    d /= np.linalg.norm(d)
    spec = {"origin": (-60.0, -50.0, -45.0), "shape": (60, 50, 45), "voxel_cm": 2.0}
    g_host = W.make_grid(spec, track_uncertainty=False)
    p, dv, e, r = _gpu_tp(engine, MIXED, [-55.0, 1.0, 2.0], d, 80.0, n, seed=seed, grid=g_host)
    geom = Geometry(MIXED)
    ts, th = engine.tables(geom.materials(), need_muen=True)
    sh = engine.scene(geom, ts)
    g_dev = W.make_grid(spec, track_uncertainty=False)
    dg = DeviceGrid(engine, g_dev, stats=False)
    try:
        p0, d0, e0 = W.pencil_beam_arrays(n, [-55.0, 1.0, 2.0], d, 80.0)
        tp, td, te = (torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (p0, d0, e0))
        nsc = torch.zeros(n, dtype=torch.int32, device="cuda")
        ab = torch.zeros(n, dtype=torch.uint8, device="cuda")
        es = torch.zeros(n, dtype=torch.uint8, device="cuda")
        edep = np.zeros(len(ts.names))
        nfl = C.c_int64()
        ptr = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
        N.check(engine.lib.cc_transport_photons_device(engine.ctx, sh, th, dg.handle, n, ptr(tp), ptr(td), ptr(te),
                                                       seed, 0, 1, ptr(nsc), ptr(ab), ptr(es), N.dptr(edep),
                                                       C.byref(nfl)))
        torch.cuda.synchronize()
        dg.download(g_dev)
        np.testing.assert_array_equal(p, tp.cpu().numpy())
        np.testing.assert_array_equal(dv, td.cpu().numpy())
        np.testing.assert_array_equal(e, te.cpu().numpy())
        np.testing.assert_array_equal(r.n_scatter, nsc.cpu().numpy().astype(np.int64))
        np.testing.assert_array_equal(r.absorbed, ab.cpu().numpy().astype(bool))
        np.testing.assert_array_equal(r.escaped, es.cpu().numpy().astype(bool))
        assert r.n_fluorescence == nfl.value
        dep = {name: float(edep[i]) for i, name in enumerate(ts.names) if edep[i] != 0.0}
        assert set(dep) == set(r.energy_deposited)
        for k, v in dep.items():
            assert r.energy_deposited[k] == pytest.approx(v, rel=1e-9)
        np.testing.assert_allclose(g_host.kerma_keV, g_dev.kerma_keV, rtol=1e-9, atol=1e-12)
        np.testing.assert_allclose(g_host.h10_track_pSv_cm3, g_dev.h10_track_pSv_cm3, rtol=1e-9, atol=1e-12)
    finally:
        dg.close()
        engine.lib.cc_scene_destroy(sh)


def test_step_limit_ends_a_run_with_a_timeout_error(engine):
    """The per-photon step limit (the device-side guard against runaway
    histories) turns into CC_E_TIMEOUT on the host, and the context stays
    usable: with the limit reset the same photons finish."""
    from chatcarlo_b200 import _native as N
    geoms = [{"name": "slab", "shape": "box", "material": "water", "center": [0, 0, 0],
              "size_cm": [40.0, 40.0, 40.0]}]
    engine.set_step_limit(3)
    try:
        with pytest.raises(N.CCError) as ei:
            _gpu_tp(engine, geoms, [-25.0, 0, 0], [1, 0, 0], 60.0, 100_000, seed=2)
        assert ei.value.code == N.CC_E_TIMEOUT
    finally:
        engine.set_step_limit(100_000)
    _, _, _, r = _gpu_tp(engine, geoms, [-25.0, 0, 0], [1, 0, 0], 60.0, 100_000, seed=2)
    assert np.all(r.escaped | r.absorbed)


def test_energy_outside_the_tables_is_a_value_error(engine):
    """A photon above 150 keV is the reference's ValueError
    (materials.py:234-237), through transport_photons and the device
    status word; the next call runs normally."""
    geoms = [{"name": "slab", "shape": "box", "material": "water", "center": [0, 0, 0],
              "size_cm": [10.0, 10.0, 10.0]}]
    with pytest.raises(ValueError):
        _gpu_tp(engine, geoms, [-15.0, 0, 0], [1, 0, 0], 200.0, 1000, seed=3)
    _, _, _, r = _gpu_tp(engine, geoms, [-15.0, 0, 0], [1, 0, 0], 100.0, 1000, seed=3)
    assert np.all(r.escaped | r.absorbed)
