"""What FP32 tracking and sampling cost each tally: the same run in FP64.

The engine tracks positions, directions and distances and samples its
physics (free paths, cross-section lookups, the samplers' arithmetic) in
FP32, with fast-math intrinsics, and accumulates its tallies in FP64.
``libccb200_fp64.so`` is the same source built to do all of that in FP64,
with FP64 tables and IEEE arithmetic (same 32-bit random draws, surface
tolerance 1e-6 cm as in transport.py:155): the FP64 GPU run.
``tally_precision`` runs one scene with the same seed through both and
reports, for every tally (kerma, H*(10)), how far the FP32 result is from
the FP64 one (a history whose discrete decisions flip on a rounding
difference follows another path from there on):

* relative difference per voxel (median, 99th percentile, max) over the
  voxels the FP64 run scored;
* the difference in units of the FP64 run's own per-voxel standard error
  (batch statistics; median, 99th percentile, max) -- far below 1 means
  that FP32 tracking is invisible next to the Monte Carlo noise; the max
  comes from rarely hit voxels, where one history crossing a boundary on
  one side of a rounding decision meets an unreliable sigma;
* the relative difference of the tally's total, and of the absorbed and
  escaped fractions.

``python -m chatcarlo_b200.precision`` prints the report for the plain-MC
and room-scale configurations as one JSON line.
"""
from __future__ import annotations

import json
import sys

import numpy as np

from . import workloads as W
from .tally import standard_error
from .transport import Engine, default_engine, run_transport


def _stats(a: np.ndarray, b: np.ndarray, sq_b: np.ndarray, n_batches: int, n_hist: int) -> dict:
    sel = b != 0
    rel = np.abs(a[sel] - b[sel]) / np.abs(b[sel])
    se = standard_error(b, sq_b, n_batches, n_hist)[sel]
    with np.errstate(divide="ignore", invalid="ignore"):
        z = np.abs(a[sel] - b[sel]) / n_hist / se
    z = z[np.isfinite(z)]
    return {"voxels": int(sel.sum()),
            "rel_median": float(np.median(rel)) if rel.size else 0.0,
            "rel_p99": float(np.percentile(rel, 99)) if rel.size else 0.0,
            "rel_max": float(rel.max()) if rel.size else 0.0,
            "sigma_median": float(np.median(z)) if z.size else 0.0,
            "sigma_p99": float(np.percentile(z, 99)) if z.size else 0.0,
            "sigma_max": float(z.max()) if z.size else 0.0,
            "total_rel": float(abs(a.sum() - b.sum()) / abs(b.sum())) if b.sum() else 0.0}


def tally_precision(scene: dict, grid_spec: dict, n_histories: int, seed: int, batch_size: int = 200_000,
                    engine32: Engine | None = None, engine64: Engine | None = None) -> dict:
    e32 = engine32 or default_engine()
    e64 = engine64 or Engine(e32.device, precision="fp64")
    out = {}
    res = {}
    for name, eng in (("fp32", e32), ("fp64", e64)):
        g = W.make_grid(grid_spec, track_uncertainty=True)
        r = run_transport(scene, n_histories=n_histories, seed=seed, batch_size=batch_size, dose_grid=True,
                          grid=g, engine=eng)
        res[name] = (g, r)
    (g32, r32), (g64, r64) = res["fp32"], res["fp64"]
    out["kerma"] = _stats(g32.kerma_keV, g64.kerma_keV, g64.kerma_sum2, g64.n_batches, g64.n_histories)
    out["h10"] = _stats(g32.h10_track_pSv_cm3, g64.h10_track_pSv_cm3, g64.h10_sum2, g64.n_batches,
                        g64.n_histories)
    out["fraction_absorbed"] = {"fp32": r32.fraction_absorbed, "fp64": r64.fraction_absorbed}
    out["fraction_escaped"] = {"fp32": r32.fraction_escaped, "fp64": r64.fraction_escaped}
    out["histories"] = n_histories
    return out


def main(argv=None) -> None:
    args = sys.argv[1:] if argv is None else argv
    n = int(float(args[0])) if args else 10_000_000
    e32 = default_engine()
    e64 = Engine(e32.device, precision="fp64")
    rep = {"plain_mc": tally_precision(W.plain_mc(), W.PLAIN_MC_GRID, n, 42, engine32=e32, engine64=e64),
           "room": tally_precision(W.room(), W.ROOM_GRID, n, 42, engine32=e32, engine64=e64)}
    print(json.dumps(rep))


if __name__ == "__main__":
    main()
