"""The engine against the reference method on the benchmark configurations,
voxel by voxel.

The oracle side is a committed fixture (tests/golden/voxels_*.npz, made by
tests/golden/make_voxel_fixtures.py): the oracle's run_transport with its
stratified track-length tally and VoxelGrid batch statistics, merged over
64 independent chunks.  The engine runs the same scene dict and grid with
its own seed; per voxel, z = (mean_engine - mean_oracle) / sqrt(se_e^2 +
se_o^2) over the voxels both runs resolve to a relative standard error
below REL_CUT.  Acceptance (the reference's own criterion for per-voxel
agreement): chi^2/dof <= 1.2; the largest |z| is reported.  Scalar outcomes
and the collision estimator are z-tested against the oracle's chunk
statistics; the collision / track-length agreement (tests/test_tally.py:
54-75) is tested as the difference of the two estimators, which the engine
must reproduce within the combined statistical error.
"""
import numpy as np
import pytest

from chatcarlo_b200 import workloads as W
from chatcarlo_b200.tally import standard_error

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

REL_CUT = 0.25
CT_SLAB_GRID = {"origin": (-16.0, -16.0, -0.5), "shape": (320, 320, 10), "voxel_cm": 0.1}
SCENES = {"plain": (W.plain_mc, W.PLAIN_MC_GRID), "room": (W.room, W.ROOM_GRID), "ct_slab": (W.ct, CT_SLAB_GRID)}


def load_fixture(name):
    f = np.load(GOLDEN / f"voxels_{name}.npz")
    shape = tuple(int(s) for s in f["shape"])
    nv = int(np.prod(shape))
    out = {"n": int(f["n_histories"]), "shape": shape, "f": f}
    for tag in ("kerma", "h10"):
        mask = np.unpackbits(f[f"{tag}_mask"])[:nv].astype(bool)
        mean = np.zeros(nv)
        se = np.full(nv, np.inf)
        mean[mask] = f[f"{tag}_mean"].astype(np.float64)
        se[mask] = mean[mask] * f[f"{tag}_rel"].astype(np.float64)
        out[tag] = (mask, mean, se)
    return out


@pytest.fixture(scope="module")
def engine():
    from chatcarlo_b200.transport import default_engine
    return default_engine()


_RUNS = {}


def engine_run(engine, name, n, batch, seed):
    """One engine run of a configuration on its grid (cached per module)."""
    from chatcarlo_b200.transport import run_transport
    key = (name, n, batch, seed)
    if key not in _RUNS:
        scene_fn, spec = SCENES[name]
        g = W.make_grid(spec)
        res = run_transport(scene_fn(), n_histories=n, seed=seed, batch_size=batch, dose_grid=True, grid=g,
                            engine=engine)
        _RUNS[key] = (g, res)
    return _RUNS[key]


def voxel_z(grid, tag, fx, report: bool = False):
    T = grid.kerma_keV if tag == "kerma" else grid.h10_track_pSv_cm3
    Q = grid.kerma_sum2 if tag == "kerma" else grid.h10_sum2
    mean_g = T.ravel() / grid.n_histories
    se_g = standard_error(T, Q, grid.n_batches, grid.n_histories).ravel()
    mask, mean_o, se_o = fx[tag]
    with np.errstate(divide="ignore", invalid="ignore"):
        ok = mask & (mean_g > 0) & (se_g / mean_g < REL_CUT) & (se_o / mean_o < REL_CUT)
    z = (mean_g[ok] - mean_o[ok]) / np.sqrt(se_g[ok] ** 2 + se_o[ok] ** 2)
    if report:
        idx = np.flatnonzero(ok)
        for j in np.argsort(-np.abs(z))[:6]:
            v = int(idx[j])
            print(f"  voxel {np.unravel_index(v, grid.shape)}: engine {mean_g[v]:.6g} +- {se_g[v]:.2g}, "
                  f"oracle {mean_o[v]:.6g} +- {se_o[v]:.2g}, z {z[j]:+.2f}")
    return z


# (configuration, engine histories, batch size, seed)
CONFIGS = [("plain", 200_000_000, 2_000_000, 101), ("room", 240_000_000, 2_400_000, 102),
           ("ct_slab", 400_000_000, 4_000_000, 103)]


@pytest.mark.parametrize("name,n,batch,seed", CONFIGS)
@pytest.mark.parametrize("tag", ["kerma", "h10"])
def test_voxel_tallies_match_the_reference_method(engine, name, n, batch, seed, tag):
    fx = load_fixture(name)
    g, _ = engine_run(engine, name, n, batch, seed)
    z = voxel_z(g, tag, fx, report=True)
    chi2 = float(np.mean(z ** 2))
    print(f"{name} {tag}: {z.size} voxels, chi2/dof {chi2:.3f}, max |z| {np.max(np.abs(z)):.2f}, "
          f"|z|>3 {np.mean(np.abs(z) > 3):.4f}, mean z {np.mean(z):+.3f}")
    assert z.size > 2000, z.size
    assert chi2 <= 1.2, chi2
    # no systematic offset: the mean z of N voxels is ~N(0, 1/sqrt(N)) (voxels
    # are nearly independent); 0.1 sigma of a voxel is far above that
    assert abs(float(np.mean(z))) < 0.1


def _chunk_stats(v, n):
    """Mean per history and its standard error from per-chunk sums."""
    per = v / n
    return float(np.sum(v) / np.sum(n)), float(per.std(ddof=1) / np.sqrt(len(per)))


@pytest.mark.parametrize("name,n,batch,seed", CONFIGS)
def test_scalar_outcomes_match_the_reference_method(engine, name, n, batch, seed):
    """Absorbed / escaped fractions, mean interactions, fluorescence
    emissions and the collision estimator per material, vs the oracle's
    chunk statistics (|z| < 4)."""
    fx = load_fixture(name)
    f = fx["f"]
    _, res = engine_run(engine, name, n, batch, seed)
    cn = f["chunk_n"].astype(float)
    for key, gv in (("n_absorbed", res.fraction_absorbed), ("n_escaped", res.fraction_escaped),
                    ("scatter_sum", res.mean_scatter_events), ("n_fluorescence", res.n_fluorescence / n)):
        mo, so = _chunk_stats(f[f"chunk_{key}"].astype(float), cn)
        if mo == 0 and gv == 0:
            continue
        z = (gv - mo) / so
        assert abs(z) < 4, (key, gv, mo, so)
    mats = [str(m) for m in f["materials"]]
    for i, m in enumerate(mats):
        mo, so = _chunk_stats(f["chunk_dep"][:, i], cn)
        if mo == 0:
            continue
        g_mean = res.energy_deposited_MeV.get(m, 0.0) * 1000.0 / n
        g_se = res.energy_deposited_sem_MeV.get(m, 0.0) * 1000.0
        z = (g_mean - mo) / np.sqrt(so ** 2 + g_se ** 2)
        assert abs(z) < 4, (m, g_mean, mo, z)


def test_collision_and_track_length_estimators_agree():
    """Plain-MC configuration: per history, the track-length kerma over the
    water box's grid minus the collision estimator in water
    (tests/test_tally.py:54-75).  The two estimate the same energy transfer
    up to the difference between mu_en and the deposit rule of the
    samplers, which the oracle measures; the engine's difference must equal
    the oracle's within 3 combined standard errors, estimated from 16
    independent engine runs and the oracle's 64 chunks."""
    from chatcarlo_b200.transport import default_engine, run_transport
    f = load_fixture("plain")["f"]
    mats = [str(m) for m in f["materials"]]
    cn = f["chunk_n"].astype(float)
    d_o = (f["chunk_kerma"] - f["chunk_dep"][:, mats.index("water")]) / cn
    eng = default_engine()
    d_g, coll = [], []
    for k in range(16):
        g = W.make_grid(W.PLAIN_MC_GRID, track_uncertainty=False)
        n = 10_000_000
        res = run_transport(W.plain_mc(), n_histories=n, seed=500 + k, batch_size=1_000_000, dose_grid=True,
                            grid=g, track_uncertainty=False, engine=eng)
        c = res.energy_deposited_MeV["water"] * 1000.0
        d_g.append((g.kerma_keV.sum() - c) / n)
        coll.append(c / n)
    d_g = np.array(d_g)
    se = np.sqrt(d_g.var(ddof=1) / len(d_g) + d_o.var(ddof=1) / len(d_o))
    z = (d_g.mean() - d_o.mean()) / se
    rel_gap = d_o.mean() / float(np.mean(coll))
    print(f"track - collision per history: engine {d_g.mean():.5f}, oracle {d_o.mean():.5f} keV "
          f"({rel_gap:+.4%} of the collision estimate), z {z:+.2f}")
    assert abs(z) < 3, (d_g.mean(), d_o.mean(), se)
    assert abs(rel_gap) < 0.05


def test_primary_transmission_through_the_water_box():
    """Plain-MC configuration: the uncollided fraction of the 60 keV pencil
    beam through 20 cm of water and 230 cm of air (the air cube and the
    background air to the world boundary) vs exp(-sum mu t) within 3 sigma
    (tests/test_transport.py:30-51)."""
    import cc_oracle as O
    from chatcarlo_b200.geometry import Geometry
    from chatcarlo_b200.transport import default_engine, transport_photons
    raw = W.plain_mc()
    n = 8_000_000
    pos, dirv, e = W.pencil_beam_arrays(n, [0.0, 0.0, -100.0], [0.0, 0.0, 1.0], 60.0)
    r = transport_photons(pos, dirv, e, Geometry(raw["geometry"]), seed=9, engine=default_engine())
    unc = float(np.mean(r.escaped & (r.n_scatter == 0)))
    expect = float(np.exp(-O.linear_mu("water", 60.0)[0] * 20.0 - O.linear_mu("air", 60.0)[0] * 230.0))
    se = np.sqrt(expect * (1 - expect) / n)
    assert abs(unc - expect) < 3 * se, (unc, expect, se)
