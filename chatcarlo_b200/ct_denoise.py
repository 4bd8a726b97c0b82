"""The learned denoiser on the CT configuration: 1 mm voxels, 320 x 320 x 150,
rotating fan beam.

``python -m chatcarlo_b200.ct_denoise`` prints one JSON line:

1. training scans: random PMMA body phantoms (a z-axis cylinder of radius
   11-16 cm and length 15 cm holding 3-8 z-axis cylinders of air, water or
   bone, radius 0.4-3 cm) scanned with the CT configuration's source
   (120 kVp, 6.8 mm Al, fan 50 x 4 cm at SID 60 cm, continuous rotation,
   30 cm helical scan) on its grid, at two low history counts with batch
   statistics and at one high count as the target;
2. a network of the denoiser's architecture trained on random 64^3 crops
   of those scans, every crop normalised by its scan's kerma scale;
3. the CT configuration's own phantom (PMMA with five air holes, never
   seen in training): a high-history reference, plain runs at several
   history counts, each denoised in one pass over the whole volume (or,
   with --tiled, in 64^3 tiles, every voxel taken from the tile it lies
   deepest in);
4. the median relative voxel-kerma error inside the phantom of the plain
   and the denoised maps against the reference (its own noise removed in
   quadrature), and the time each needs to reach a 2 % median error.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import denoiser as DN
from . import phantoms as PH
from . import workloads as W
from .denoise_run import Dataset, histories_for_error, train

CT_MATERIALS = ["air", "pmma", "water", "bone"]       # one-hot order of the CT network's input
TILE = 64
STRIDE = 48
CT_PRETRAINED = __import__("pathlib").Path(__file__).resolve().parent / "data" / "denoiser_ct64.npz"


def ct_phantom(rng: np.random.Generator) -> dict:
    """A random PMMA body with z-axis inserts, scanned by the CT source."""
    r_body = float(rng.uniform(11.0, 16.0))
    geoms = [{"name": "body", "shape": "cylinder", "material": "pmma", "axis": "z", "center": [0.0, 0.0, 0.0],
              "radius_cm": r_body, "height_cm": 15.0}]
    for i in range(int(rng.integers(3, 9))):
        r = float(rng.uniform(0.4, 3.0))
        reach = r_body - r - 0.5
        ang, rad = rng.uniform(0, 2 * np.pi), reach * np.sqrt(rng.uniform(0, 1))
        h = float(rng.uniform(4.0, 15.0))
        zc = float(rng.uniform(-7.5 + h / 2, 7.5 - h / 2))
        geoms.append({"name": f"insert{i}", "shape": "cylinder", "material": str(rng.choice(["air", "water", "bone"])),
                      "axis": "z", "center": [float(rad * np.cos(ang)), float(rad * np.sin(ang)), zc],
                      "radius_cm": r, "height_cm": h})
    scene = W.ct()
    scene["geometry"] = geoms
    return scene


def scan(scene: dict, n: int, seed: int, engine, grid, batches: int = 50):
    """Kerma per history (float32) and its relative standard error (float32,
    from ``batches`` batches) of one scan on the CT grid, and the device ms."""
    from .transport import run_transport
    bs = max(1, n // batches)
    res = run_transport(scene, n_histories=n, seed=seed, batch_size=bs, dose_grid=True, grid=grid, engine=engine)
    k = (grid.kerma_keV / n).astype(np.float32)
    rel = grid.kerma_relative_error().astype(np.float32)
    return k, rel, res.device_ms


def tile_starts(n: int, t: int = TILE, stride: int = STRIDE) -> list[int]:
    """Tile origins along one axis of length n >= t: every stride, plus the
    last full tile."""
    s = list(range(0, n - t + 1, stride))
    if s[-1] != n - t:
        s.append(n - t)
    return s


def owned_bounds(starts: list[int], n: int, t: int = TILE) -> list[int]:
    """Boundaries of the ranges each tile owns: halfway between neighbouring
    tile centres, so a voxel comes from the tile it lies deepest in."""
    c = [s + t / 2 for s in starts]
    return [0] + [int(round((c[i] + c[i + 1]) / 2)) for i in range(len(c) - 1)] + [n]


def denoise_volume(model: DN.UNet3D, k: np.ndarray, rel: np.ndarray, mat: np.ndarray, dens: np.ndarray,
                   batch: int = 8, tiled: bool = False) -> tuple[np.ndarray, float]:
    """Denoised kerma of a whole volume and the device time (ms): in one pass
    over the volume (each axis padded to a multiple of 8 by repeating its
    edge), or with ``tiled`` in overlapping 64^3 tiles (each axis >= 64)."""
    import torch
    inside = mat != 0
    scale = DN.kerma_scale(k, inside)
    x = DN.to_log(k, scale)
    unc = DN.uncertainty_channel(rel)
    if not tiled:
        pad = [(0, (-n) % 8) for n in k.shape]
        xp, dp, mp, up = (np.pad(a, pad, mode="edge") for a in (x, dens, mat, unc))
        model.set_input(xp[None], dp[None], mp[None], 1, xp.shape, unc=up[None])
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        y = model.predict()
        e1.record()
        e1.synchronize()
        out = y.cpu().numpy().reshape(xp.shape)[:k.shape[0], :k.shape[1], :k.shape[2]]
        model.check_status()
        return DN.from_log(out, scale), e0.elapsed_time(e1)
    axes = [tile_starts(n) for n in k.shape]
    bounds = [owned_bounds(a, n) for a, n in zip(axes, k.shape)]
    tiles = [(i, j, l) for i in range(len(axes[0])) for j in range(len(axes[1])) for l in range(len(axes[2]))]
    out = np.empty(k.shape, dtype=np.float64)
    ms = 0.0
    for b0 in range(0, len(tiles), batch):
        part = tiles[b0:b0 + batch]
        sl = [tuple(slice(axes[a][t[a]], axes[a][t[a]] + TILE) for a in range(3)) for t in part]
        model.set_input(np.stack([x[s] for s in sl]), np.stack([dens[s] for s in sl]), np.stack([mat[s] for s in sl]),
                        len(part), TILE, unc=np.stack([unc[s] for s in sl]))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        y = model.predict()
        e1.record()
        e1.synchronize()
        ms += e0.elapsed_time(e1)
        y = y.cpu().numpy().reshape(len(part), TILE, TILE, TILE)
        for q, t in enumerate(part):
            lo = [bounds[a][t[a]] for a in range(3)]
            hi = [bounds[a][t[a] + 1] for a in range(3)]
            st = [axes[a][t[a]] for a in range(3)]
            out[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]] = y[q, lo[0] - st[0]:hi[0] - st[0], lo[1] - st[1]:hi[1] - st[1],
                                                          lo[2] - st[2]:hi[2] - st[2]]
    model.check_status()
    return DN.from_log(out, scale), ms


def denoise_ct_kerma(k: np.ndarray, rel: np.ndarray, mat: np.ndarray, density: np.ndarray,
                     model: DN.UNet3D | None = None) -> np.ndarray:
    """Denoised kerma of a CT-type volume (1 mm voxels, any shape) from a
    plain run and its batch statistics, with the CT network that ships with
    the package unless a model is given.  mat indexes CT_MATERIALS (air 0,
    pmma 1, water 2, bone 3)."""
    model = model or DN.UNet3D(params=DN.load_params(CT_PRETRAINED)[0])
    return denoise_volume(model, np.asarray(k, dtype=np.float64), rel, mat, density)[0]


def run(args) -> dict:
    from .transport import default_engine
    eng = default_engine()
    rng = np.random.default_rng(args.seed)
    t_all = time.perf_counter()
    grid = W.make_grid(W.CT_GRID, track_uncertainty=True, pinned=True)
    shape = tuple(W.CT_GRID["shape"])
    if args.load:
        model = DN.UNet3D(params=DN.load_params(args.load)[0])
        training = {"loaded": str(args.load)}
    else:
        model, training = _train(args, eng, rng, grid, shape)
    return _evaluate(args, eng, model, training, grid, t_all)


def _train(args, eng, rng, grid, shape):
    crops = {"x": [[] for _ in args.n_in], "r": [[] for _ in args.n_in], "t": [], "m": [], "d": [], "s": []}
    ms_train = 0.0
    for p in range(args.train):
        scene = ct_phantom(rng)
        mat, dens = PH.voxel_maps(scene, W.CT_GRID, CT_MATERIALS)
        lows = []
        for j, n in enumerate(args.n_in):
            k, r, ms = scan(scene, n, 100 * p + j, eng, grid)
            lows.append((k, r))
            ms_train += ms
        kt, _, ms = scan(scene, args.n_target, 100 * p + 50, eng, grid)
        ms_train += ms
        inside = mat != 0
        scales = [DN.kerma_scale(k, inside) for k, _ in lows]
        for _ in range(args.crops):
            o = [int(rng.integers(0, n - TILE + 1)) for n in shape]
            sl = tuple(slice(o[a], o[a] + TILE) for a in range(3))
            for j, (k, r) in enumerate(lows):
                crops["x"][j].append(k[sl])
                crops["r"][j].append(r[sl])
            crops["t"].append(kt[sl])
            crops["m"].append(mat[sl])
            crops["d"].append(dens[sl])
            crops["s"].append(scales)
    scale = np.array(crops["s"]).T                     # [levels, crops]
    data = Dataset([np.stack(c).astype(np.float64) for c in crops["x"]], np.stack(crops["t"]).astype(np.float64),
                   np.stack(crops["m"]), np.stack(crops["d"]), rel=[np.stack(c) for c in crops["r"]], scale=scale)
    del crops
    model = DN.UNet3D(seed=args.seed)
    losses, t_train = train(model, data, args.steps, args.batch, args.lr, seed=args.seed)
    if args.save:
        np.save(args.save, model.params_numpy())
    training = {"scans": args.train, "crops_per_scan": args.crops,
                "histories": {"input": args.n_in, "target": args.n_target}, "steps": args.steps,
                "batch": args.batch, "lr": args.lr, "seconds": t_train, "losses": losses, "mc_ms": ms_train}
    return model, training


def _evaluate(args, eng, model, training, grid, t_all):
    # the configuration's own phantom
    c5 = W.ct()
    mat, dens = PH.voxel_maps(c5, W.CT_GRID, CT_MATERIALS)
    inside = mat != 0
    k_ref, rel_ref, ms_ref = scan(c5, args.n_ref, 7, eng, grid, batches=args.ref_batches)
    sel = inside & (k_ref > 0)
    ref_noise = float(np.median(0.6745 * np.nan_to_num(rel_ref[sel], nan=0.0)))
    rate = args.n_ref / (ms_ref * 1e-3)
    levels = []
    for n in args.levels:
        k_n, rel_n, ms_n = scan(c5, n, 11 + n % 991, eng, grid)
        k_dn, ms_dn = denoise_volume(model, k_n, rel_n, mat, dens, tiled=args.tiled)
        err = lambda k: float(np.median(np.abs(k[sel] - k_ref[sel]) / k_ref[sel]))  # noqa: E731
        dn_meas = err(k_dn)
        levels.append({"histories": n, "plain_measured": err(k_n),
                       "plain_from_stats": float(np.median(0.6745 * np.nan_to_num(rel_n[sel], nan=1.0))),
                       "denoised_measured": dn_meas,
                       "denoised_corrected": float(np.sqrt(max(dn_meas ** 2 - ref_noise ** 2, 0.0))),
                       "mc_ms": ms_n, "denoise_ms": ms_dn})
    plain_c = np.median([lv["plain_from_stats"] * np.sqrt(lv["histories"]) for lv in levels])
    n_plain = (plain_c / 0.02) ** 2
    t_plain = n_plain / rate
    n_dn = histories_for_error([lv["histories"] for lv in levels], [lv["denoised_corrected"] for lv in levels], 0.02)
    t_inf = float(np.median([lv["denoise_ms"] for lv in levels])) * 1e-3
    t_dn = n_dn / rate + t_inf if n_dn is not None else None
    return {
        "workload": "CT configuration: PMMA body phantom (32 cm, 15 cm long, five 1.3 cm air holes), 120 kVp, "
                    "fan 50x4 cm, helical rotation; kerma on 320x320x150 voxels of 1 mm",
        "training": training,
        "reference": {"histories": args.n_ref, "batches": args.ref_batches, "ms": ms_ref,
                      "noise_median": ref_noise},
        "mc_histories_per_s": rate,
        "levels": levels,
        "time_to_2pct_s": {"plain_mc": t_plain, "plain_histories": n_plain, "denoised": t_dn,
                           "denoised_histories": n_dn, "inference_s": t_inf,
                           "speedup": (t_plain / t_dn) if t_dn else None},
        "wall_s": time.perf_counter() - t_all,
    }


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--train", type=int, default=10, help="training scans")
    ap.add_argument("--crops", type=int, default=16, help="64^3 crops per training scan")
    ap.add_argument("--n-in", type=int, nargs="+", default=[10_000_000, 40_000_000])
    ap.add_argument("--n-target", type=int, default=1_000_000_000)
    ap.add_argument("--n-ref", type=int, default=10_000_000_000)
    ap.add_argument("--ref-batches", type=int, default=100)
    ap.add_argument("--levels", type=int, nargs="+", default=[10_000_000, 30_000_000, 100_000_000, 300_000_000,
                                                              1_000_000_000])
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--batch", type=int, default=4)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=5)
    ap.add_argument("--save", default=None, help="write the trained parameters (.npy)")
    ap.add_argument("--tiled", action="store_true", help="denoise in 64^3 tiles instead of one pass")
    ap.add_argument("--load", default=None,
                    help="evaluate a saved network (save_params file, e.g. the shipped denoiser_ct64.npz) "
                         "instead of training one")
    ap.add_argument("--layer-times", type=int, nargs=3, metavar=("X", "Y", "Z"), default=None,
                    help="only time each convolution of the shipped CT network on a random volume of this shape "
                         "(the whole CT grid: 320 320 152)")
    args = ap.parse_args(argv)
    if args.layer_times:
        print(json.dumps(layer_times(tuple(args.layer_times))))
        return
    print(json.dumps(run(args)))


def layer_times(shape: tuple[int, int, int], repeats: int = 3) -> dict:
    """Per-convolution device time of CT-volume inference with the shipped
    network on random inputs of `shape` (every side a multiple of 8), and
    the whole prediction (forward and head) timed with CUDA events."""
    import torch
    model = DN.UNet3D(params=DN.load_params(CT_PRETRAINED)[0])
    rng = np.random.default_rng(0)
    x = rng.normal(size=(1,) + shape).astype(np.float32)
    m = rng.integers(0, len(CT_MATERIALS), size=(1,) + shape).astype(np.uint8)
    model.set_input(x, np.ones((1,) + shape, np.float32), m, 1, shape, unc=np.full((1,) + shape, 0.1, np.float32))
    layers = model.layer_times(repeats)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    for _ in range(repeats):
        ev[0].record()
        model.predict()
        ev[1].record()
    torch.cuda.synchronize()
    model.check_status()
    return {"shape": list(shape), "predict_ms": round(ev[0].elapsed_time(ev[1]), 3),
            "conv_ms": round(sum(r["ms"] for r in layers), 3), "layers": layers}


if __name__ == "__main__":
    main()
