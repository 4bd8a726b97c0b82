"""CTDIvol calibration (ctdi.py) on the engine against the oracle, and its
use by run_transport."""
import json
from pathlib import Path

import numpy as np
import pytest

import cc_oracle as O

pytestmark = pytest.mark.gpu

SRC = json.loads(str(np.load(Path(__file__).resolve().parent / "golden" / "ctdi.npz")["source_json"]))


def test_ctdi_per_history_matches_oracle():
    from chatcarlo_b200.ctdi import ctdi_per_history_Gy
    gpu = np.array(ctdi_per_history_Gy(SRC, phantom="head", n_histories=4_000_000, seed=3))
    ref = np.array([O.ctdi_per_history_Gy(SRC, "head", 20_000, s) for s in range(8)])
    mean, sem = ref.mean(axis=0), ref.std(axis=0, ddof=1) / np.sqrt(len(ref))
    assert np.all(np.abs(gpu - mean) < 4.0 * sem + 1e-3 * mean), (gpu, mean, sem)


def test_run_transport_reports_the_ctdi_calibration():
    from chatcarlo_b200.ctdi import ctdi_per_history_Gy
    from chatcarlo_b200.transport import run_transport
    scene = {"source": dict(SRC, ctdi_phantom="body"),
             "geometry": [{"name": "patient", "shape": "ellipsoid", "material": "water", "center": [0, 0, 0],
                           "semi_axes_cm": [15.0, 10.0, 20.0]}]}
    res = run_transport(scene, n_histories=1_000_000, seed=11, dose_grid=False)
    ctdiw, _, _ = ctdi_per_history_Gy(scene["source"], phantom="body", n_histories=200_000, seed=11)
    assert res.n_photons_real == pytest.approx(SRC["ctdi_vol_mGy"] * 1e-3 / ctdiw, rel=1e-9)
    with pytest.raises(RuntimeError):
        run_transport({"source": {k: v for k, v in SRC.items() if k != "ctdi_vol_mGy"} | {"mas": 100.0},
                       "geometry": scene["geometry"]}, n_histories=1000, seed=1)
