"""Oracle voxel tallies of the benchmark configurations, for the GPU tests
that compare the engine with the reference method voxel by voxel.

    python tests/golden/make_voxel_fixtures.py [--workers N] [--only NAME ...]

For each workload the oracle (the NumPy restatement of chatcarlo's
run_transport with its stratified track-length tally and VoxelGrid batch
statistics, chatcarlo/transport.py:257-474, tally.py:59-175,248-293) runs
``n`` histories as ``chunks`` independent runs of ``n / chunks`` histories
(seed = (seed, chunk)), each with batch statistics over ``batch`` histories;
the chunks are merged the way the reference merges its process workers
(transport.py:416-437: totals, sums of squares and hit counts add).  Stored
per tally (kerma, H*(10)): a packed mask of the voxels whose mean is
positive and whose relative standard error is below ``REL_CUT``, their
mean per history (float32) and relative standard error (float16).  Stored
per chunk, for estimator comparisons whose variance needs whole-grid
totals: the grid's kerma and H*(10) sums, the collision-estimator sum per
material and the outcome counters.

Workloads (chatcarlo_b200/workloads.py):
* ``plain``: 60 keV pencil beam into the 30x30x20 cm water box, kerma on
  60x60x40 voxels of 0.5 cm;
* ``room``: the room-scale scene, kerma and H*(10) on 80x80x60 voxels of 5 cm;
* ``ct_slab``: the CT phantom and helical source, on the central 1 cm slab
  (320x320x10 voxels of 1 mm) of the 320x320x150 CT grid.
"""
from __future__ import annotations

import argparse
import concurrent.futures
import multiprocessing as mp
import os
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent
for p in (REPO, REPO / "oracle"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))

REL_CUT = 0.3
# voxels kept per workload: every k-th voxel of the grid in C order (a
# uniform subset that keeps the fixture small; the chi^2 needs thousands of
# voxels, not all of them)
KEEP_EVERY = {"plain": 2, "room": 4, "ct_slab": 16}

CT_SLAB_GRID = {"origin": (-16.0, -16.0, -0.5), "shape": (320, 320, 10), "voxel_cm": 0.1}


def workloads():
    from chatcarlo_b200 import workloads as W
    return {
        "plain": dict(raw=W.plain_mc(), grid=W.PLAIN_MC_GRID, n=16_000_000, chunks=64, batch=50_000, seed=42),
        "room": dict(raw=W.room(), grid=W.ROOM_GRID, n=24_000_000, chunks=64, batch=75_000, seed=7),
        "ct_slab": dict(raw=W.ct(), grid=CT_SLAB_GRID, n=40_000_000, chunks=64, batch=125_000, seed=5),
    }


def _run_chunks(raw, grid_spec, chunk_ids, n_chunk, batch, seed):
    """One worker: its chunks in order, grids summed, per-chunk totals kept."""
    import cc_oracle as O
    acc = None
    rows = []
    for c in chunk_ids:
        agg = O.run_transport(raw, n_histories=n_chunk, seed=(seed, c), batch_size=batch, grid_spec=grid_spec,
                              n_workers=1, track_uncertainty=True)
        g = agg["grid"]
        arrs = (g.kerma_keV, g.kerma_sum2, g.h10_track_pSv_cm3, g.h10_sum2, g.n_batches_hit)
        if acc is None:
            acc = [a.copy() for a in arrs] + [g.n_batches, g.n_histories]
        else:
            for a, b in zip(acc, arrs):
                a += b
            acc[5] += g.n_batches
            acc[6] += g.n_histories
        rows.append({"chunk": c, "n": n_chunk, "kerma": float(g.kerma_keV.sum()),
                     "h10": float(g.h10_track_pSv_cm3.sum()), "dep": dict(agg["energy_deposited"]),
                     "n_absorbed": agg["n_absorbed"], "n_escaped": agg["n_escaped"],
                     "scatter_sum": agg["scatter_sum"], "n_fluorescence": agg["n_fluorescence"]})
    return acc, rows


def make(name: str, spec: dict, workers: int) -> dict:
    import cc_oracle as O
    n_chunk = spec["n"] // spec["chunks"]
    ids = list(range(spec["chunks"]))
    parts = [ids[i::workers] for i in range(workers)]
    t0 = time.time()
    with concurrent.futures.ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as pool:
        futs = [pool.submit(_run_chunks, spec["raw"], spec["grid"], p, n_chunk, spec["batch"], spec["seed"])
                for p in parts if p]
        acc, rows = None, []
        for f in futs:
            a, r = f.result()
            rows += r
            if acc is None:
                acc = a
            else:
                for x, y in zip(acc[:5], a[:5]):
                    x += y
                acc[5] += a[5]
                acc[6] += a[6]
    rows.sort(key=lambda r: r["chunk"])
    T_k, Q_k, T_h, Q_h, n_hit, M, N = acc
    out = {"shape": np.array(spec["grid"]["shape"]), "origin": np.array(spec["grid"]["origin"], float),
           "voxel_cm": np.array(spec["grid"]["voxel_cm"], float), "n_histories": np.array(N),
           "n_batches": np.array(M), "seed": np.array(spec["seed"]), "rel_cut": np.array(REL_CUT)}
    for tag, T, Q in (("kerma", T_k, Q_k), ("h10", T_h, Q_h)):
        rel = O.relative_error(T, Q, M, N)
        with np.errstate(invalid="ignore"):
            sel = (T > 0) & np.isfinite(rel) & (rel < REL_CUT)
        out[f"{tag}_mask"] = np.packbits(sel.ravel())
        out[f"{tag}_mean"] = (T[sel] / N).astype(np.float32)
        out[f"{tag}_rel"] = rel[sel].astype(np.float16)
    mats = sorted({k for r in rows for k in r["dep"]})
    out["materials"] = np.array(mats)
    out["chunk_n"] = np.array([r["n"] for r in rows], dtype=np.int64)
    out["chunk_kerma"] = np.array([r["kerma"] for r in rows])
    out["chunk_h10"] = np.array([r["h10"] for r in rows])
    out["chunk_dep"] = np.array([[r["dep"].get(m, 0.0) for m in mats] for r in rows])
    for k in ("n_absorbed", "n_escaped", "scatter_sum", "n_fluorescence"):
        out[f"chunk_{k}"] = np.array([r[k] for r in rows], dtype=np.int64)
    print(f"{name}: {N} histories, {M} batches, {time.time() - t0:.0f} s; "
          f"kerma voxels kept {out['kerma_mean'].size}, "
          f"h10 voxels kept {out['h10_mean'].size}", flush=True)
    return out


def subsample(out: dict, every: int) -> dict:
    """Keep only voxels whose flat index is a multiple of ``every``."""
    nv = int(np.prod(out["shape"]))
    keep = (np.arange(nv) % every) == 0
    out = dict(out, keep_every=np.array(every))
    for tag in ("kerma", "h10"):
        sel = np.unpackbits(out[f"{tag}_mask"])[:nv].astype(bool)
        k = keep[sel]
        out[f"{tag}_mask"] = np.packbits(sel & keep)
        out[f"{tag}_mean"] = out[f"{tag}_mean"][k]
        out[f"{tag}_rel"] = out[f"{tag}_rel"][k]
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workers", type=int, default=os.cpu_count())
    ap.add_argument("--only", nargs="*")
    a = ap.parse_args()
    for name, spec in workloads().items():
        if a.only and name not in a.only:
            continue
        out = subsample(make(name, spec, a.workers), KEEP_EVERY[name])
        np.savez_compressed(HERE / f"voxels_{name}.npz", **out)


if __name__ == "__main__":
    main()
