"""Device source sampling against the oracle's restatement of source.py
(bit-identical to the reference on tests/golden/source.npz and heel.npz):
every field shape, CT rotation (continuous and n_angles), the helical
shift, and the heel effect with fixed off-axis bins standing in for SpekPy
(the bins the golden heel case was made with).  Distributions are compared
as samples of the same law: means and spreads of positions and directions,
energy frequencies, and for the heel effect the fluence profile and the
mean energy along the heel axis."""
import ctypes as C

import numpy as np
import pytest
from scipy import stats

import cc_oracle as O
from conftest import GOLDEN

pytestmark = pytest.mark.gpu

BASE = {"position": [0, -100, 50], "direction": [0, 1, 0], "spectrum": [
    {"energy_keV": 30.0, "weight": 1.0}, {"energy_keV": 60.0, "weight": 3.0}, {"energy_keV": 90.0, "weight": 2.0}]}
VARIANTS = {
    "rect": {"field": {"shape": "rect", "size_cm": [30, 40], "sid_cm": 100}},
    "cone": {"field": {"shape": "cone", "diameter_cm": 25, "sid_cm": 100}},
    "parallel": {"field": {"shape": "parallel", "size_cm": [10, 12]}},
    "rot": {"field": {"shape": "rect", "size_cm": [50, 4], "sid_cm": 100},
            "rotation": {"isocenter": [0, 0, 50], "axis": "z", "scan_length_cm": 30}},
    "rotn": {"field": {"shape": "cone", "diameter_cm": 20, "sid_cm": 100},
             "rotation": {"isocenter": [0, 0, 50], "axis": "x", "n_angles": 8}},
}
HEEL_BASE = {"position": [0, -100, 50], "direction": [0, 1, 0], "heel_effect": True, "kvp": 80}
HEEL_VARIANTS = {
    "rect": {"field": {"shape": "rect", "size_cm": [35, 43], "sid_cm": 100}, "anode_direction": [1.0, 0.3, 0.0]},
    "cone": {"field": {"shape": "cone", "diameter_cm": 30, "sid_cm": 100}, "anode_direction": [0.0, 1.0, 0.2]},
    "rot": {"field": {"shape": "rect", "size_cm": [50, 4], "sid_cm": 100}, "anode_direction": [1.0, 0.0, 0.0],
            "rotation": {"isocenter": [0, 0, 50], "axis": "y", "scan_length_cm": 20}},
}


@pytest.fixture(scope="module")
def engine():
    from chatcarlo_b200.transport import default_engine
    return default_engine()


def device_sample(engine, src, n, seed):
    from chatcarlo_b200 import _native as N
    from chatcarlo_b200.source import SourceSpec
    h = engine.source(SourceSpec(src))
    pos, dirv, en = np.empty((n, 3)), np.empty((n, 3)), np.empty(n)
    try:
        N.check(engine.lib.cc_sample_source(engine.ctx, h, n, seed, 0, N.dptr(pos), N.dptr(dirv), N.dptr(en)),
                engine.lib)
    finally:
        engine.lib.cc_source_destroy(h)
    return pos, dirv, en


def compare_geometry(pg, dg, po, do):
    n_g, n_o = len(pg), len(po)
    for a, b in ((pg, po), (dg, do)):
        se = np.sqrt(a.var(axis=0) / n_g + b.var(axis=0) / n_o) + 1e-7
        assert np.all(np.abs(a.mean(axis=0) - b.mean(axis=0)) < 5 * se), (a.mean(axis=0), b.mean(axis=0))
        np.testing.assert_allclose(a.std(axis=0), b.std(axis=0), rtol=0.02, atol=1e-4)
        for k in range(3):
            if a[:, k].std() <= 1e-6:
                continue
            ua = np.unique(np.round(a[:, k], 3))
            if len(ua) < 64:
                # a discrete coordinate (n_angles gantry positions): the FP32
                # atoms sit a rounding away from the FP64 ones, so compare
                # the atoms' frequencies instead of the ECDFs
                ka, kb = np.round(a[:, k], 3), np.round(b[:, k], 3)
                keys = np.union1d(ka, kb)
                ca = np.array([np.sum(ka == x) for x in keys], float)
                cb = np.array([np.sum(kb == x) for x in keys], float)
                assert len(keys) == len(ua), (keys, ua)
                assert stats.chi2_contingency(np.stack([ca, cb]))[1] > 1e-4
            else:
                assert stats.ks_2samp(a[:, k], b[:, k]).pvalue > 1e-4


def compare_energies(eg, eo):
    keys = np.union1d(np.round(eg, 3), np.round(eo, 3))
    cg = np.array([np.sum(np.round(eg, 3) == k) for k in keys], float)
    co = np.array([np.sum(np.round(eo, 3) == k) for k in keys], float)
    keep = (cg + co) >= 20
    assert stats.chi2_contingency(np.stack([cg[keep], co[keep]]))[1] > 1e-4


@pytest.mark.parametrize("name", list(VARIANTS))
def test_source_field_shapes_match_oracle(engine, name):
    """rect, cone, parallel, continuous rotation with helical shift, and
    n_angles rotation (source.py:67-194)."""
    src = dict(BASE, **VARIANTS[name])
    n_g, n_o = 1_000_000, 200_000
    pg, dg, eg = device_sample(engine, src, n_g, 5)
    po, do, eo = O.sample_source_photons(src, n_o, np.random.default_rng(5))
    compare_geometry(pg, dg, po, do)
    compare_energies(eg, eo)
    np.testing.assert_allclose(np.linalg.norm(dg, axis=1), 1.0, atol=1e-5)
    if name == "rotn":
        # 8 discrete gantry angles: the foci lie on 8 points
        assert len(np.unique(np.round(pg, 3), axis=0)) == 8


def _heel_bins(k):
    g = np.load(GOLDEN / "heel.npz")
    spectra = tuple((a, b) for a, b in zip(g[f"{k}_spec_e"], g[f"{k}_spec_w"]))
    return float(g[f"{k}_span"]), (g[f"{k}_centers"], spectra, g[f"{k}_rel"], g[f"{k}_rel"] * 1e6)


def _heel_coordinate(src, dirs):
    """s on the SID plane along the heel axis, from a static field's directions."""
    from chatcarlo_b200.source import beam_basis, heel_axis
    d = np.asarray(src["direction"], dtype=float)
    u, v = beam_basis(d)
    h_u, h_v = heel_axis(src, d, u, v)
    sid = src["field"]["sid_cm"]
    return sid * (dirs @ (h_u * u + h_v * v)) / (dirs @ d)


@pytest.mark.parametrize("name", list(HEEL_VARIANTS))
def test_heel_effect_matches_oracle(engine, name, monkeypatch):
    """source.py:130-149,195-207 on the device: fluence rejection along the
    heel axis and energies from each photon's heel bin."""
    import chatcarlo_b200.source as S
    span, bins = _heel_bins(name)
    monkeypatch.setattr(S, "heel_spectra_for_source", lambda src, sid, sp, n_bins=15: bins)
    monkeypatch.setattr(O, "heel_spectra_for_source", lambda src, sid, sp: bins)
    src = dict(HEEL_BASE, **HEEL_VARIANTS[name])
    n_g, n_o = 1_000_000, 200_000
    pg, dg, eg = device_sample(engine, src, n_g, 7)
    po, do, eo = O.sample_source_photons(src, n_o, np.random.default_rng(7))
    compare_geometry(pg, dg, po, do)
    compare_energies(eg, eo)
    if "rotation" in src:
        return
    sg, so = _heel_coordinate(src, dg), _heel_coordinate(src, do)
    assert np.all(np.abs(sg) <= span * (1 + 1e-4))
    assert stats.ks_2samp(sg, so).pvalue > 1e-4
    # hardening towards the anode: mean energy per heel bin
    edges = np.linspace(-span, span, 16)
    kg, ko = np.digitize(sg, edges), np.digitize(so, edges)
    means = []
    for b in range(1, 16):
        a, c = eg[kg == b], eo[ko == b]
        if len(c) < 200:
            continue
        z = (a.mean() - c.mean()) / np.sqrt(a.var() / len(a) + c.var() / len(c))
        assert abs(z) < 4.5, (b, a.mean(), c.mean())
        means.append(a.mean())
    assert means[-1] > means[0]

