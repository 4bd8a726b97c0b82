"""Batched multi-scene runs: one launch over several scenes gives each scene
the same statistics as its own single-scene run, reproducibly."""
import numpy as np
import pytest

from chatcarlo_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    from chatcarlo_b200.transport import default_engine
    return default_engine()


def _chi2(a, b, n_a, n_b, min_counts=50):
    """Per-voxel comparison of two kerma maps by their totals; the variance of
    each voxel's total is estimated from its batch statistics."""
    from chatcarlo_b200.tally import standard_error
    ma, mb = a.kerma_keV / n_a, b.kerma_keV / n_b
    sa = standard_error(a.kerma_keV, a.kerma_sum2, a.n_batches, a.n_histories)
    sb = standard_error(b.kerma_keV, b.kerma_sum2, b.n_batches, b.n_histories)
    with np.errstate(divide="ignore", invalid="ignore"):
        ok = (ma > 0) & (mb > 0) & (sa / ma < 0.2) & (sb / mb < 0.2)
    z = (ma[ok] - mb[ok]) / np.sqrt(sa[ok] ** 2 + sb[ok] ** 2)
    return float(np.mean(z ** 2)) if ok.any() else 0.0, int(ok.sum())


def test_batched_matches_single_scene_runs(engine):
    from chatcarlo_b200.batched import BatchedRun
    from chatcarlo_b200.transport import run_transport
    scenes, specs, _ = W.batched_scenes(n_scenes=5, seed=7)
    counts = [400_000] * 5
    br = BatchedRun(scenes, specs, counts, slots=20, engine=engine)
    try:
        sc, out = br.run(seed=11)
        grids = br.download()
        assert out.n_histories == sum(counts)
        for i, raw in enumerate(scenes):
            single = W.make_grid(specs[i])
            res = run_transport(raw, n_histories=counts[i], seed=50 + i, batch_size=counts[i] // 20,
                                dose_grid=True, grid=single, engine=engine)
            n = counts[i]
            for k, val in ((0, res.fraction_absorbed), (1, res.fraction_escaped)):
                p = sc[i, k] / n
                se = np.sqrt(max(p * (1 - p), 1e-12) / n + max(val * (1 - val), 1e-12) / n)
                assert abs(p - val) < 5 * se + 1e-9, (i, k, p, val)
            chi2, nv = _chi2(grids[i], single, n, n)
            if nv > 30:
                assert chi2 < 1.3, (i, chi2, nv)
    finally:
        br.close()


@pytest.mark.parametrize("fp32_cells,rtol", [(False, 1e-9), (True, 1e-4)])
def test_batched_replay_is_reproducible(engine, fp32_cells, rtol):
    """Same seed -> same counts; same kerma up to the order of the FP64
    additions with the default FP64 scratch cells, and of the FP32 ones with
    FP32 cells switched on."""
    from chatcarlo_b200.batched import BatchedRun
    scenes, specs, _ = W.batched_scenes(n_scenes=8, seed=3)
    counts = [int(x) for x in np.linspace(30_000, 300_000, 8)]
    engine.set_tally_fp32(fp32_cells)
    try:
        br = BatchedRun(scenes, specs, counts, slots=1, engine=engine)
    finally:
        engine.set_tally_fp32(False)
    try:
        a, _ = br.run(seed=5)
        ka = [g.kerma_keV.copy() for g in br.download()]
        br.reset()
        b, _ = br.run(seed=5)
        kb = [g.kerma_keV.copy() for g in br.download()]
        np.testing.assert_array_equal(a, b)
        for x, y in zip(ka, kb):
            np.testing.assert_allclose(x, y, rtol=rtol, atol=rtol * float(np.max(np.abs(y))))
        br.reset()
        c, _ = br.run(seed=6)
        assert not np.array_equal(a, c)
    finally:
        br.close()


def test_autotuner_picks_and_caches_a_shape(engine, tmp_path, monkeypatch):
    from chatcarlo_b200 import batched
    monkeypatch.setattr(batched, "CACHE_PATH", tmp_path / "autotune.json")
    scenes, specs, counts = W.batched_scenes(n_scenes=6, seed=9, hist_lo=2e4, hist_hi=1e5)
    cands = [{"block": 256, "blocks_per_sm": 2, "chunk": 128}, {"block": 256, "blocks_per_sm": 4, "chunk": 256}]
    shape = batched.autotune(scenes, specs, counts, engine=engine, scale=1.0, candidates=cands)
    assert shape in cands
    assert (tmp_path / "autotune.json").exists()
    assert batched.autotune(scenes, specs, counts, engine=engine, candidates=[]) == shape
