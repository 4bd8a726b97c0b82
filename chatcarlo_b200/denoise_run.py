"""Train and score the kerma denoiser on the engine's own Monte Carlo.

``python -m chatcarlo_b200.denoise_run`` runs the whole learned-denoiser
workload on one GPU and prints one JSON line:

1. phantoms (``phantoms.py``) for training and held-out evaluation;
2. kerma maps from batched Monte Carlo launches (every phantom of a set in
   one persistent launch): a low-history input map and a high-history
   target map per training phantom, and for the held-out phantoms input
   maps at several history counts plus a reference map;
3. training of the U-Net by its own forward and backward kernels (Adam);
4. the median relative voxel-kerma error inside the phantoms (water, bone,
   lead voxels), against the reference map, of plain Monte Carlo and of the
   denoised maps, and from it the time each needs to reach a 2 % median
   error.

Plain Monte Carlo's error at n histories follows from its own batch
statistics (median |error| = 0.6745 sigma for Gaussian noise) and scales as
1/sqrt(n).  The denoised error is measured against the reference map, whose
own noise (from its batch statistics) is removed in quadrature.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import denoiser as DN
from . import phantoms as PH
from .batched import BatchedRun
from .tally import relative_error


def mc_maps(scenes, grids, n_hist: int, seed: int, engine, stats_slots: int = 1, group: int = 128):
    """Kerma per history [n, S, S, S] of every phantom (float64), the
    per-voxel relative standard error when stats_slots > 1, and the device
    time of the batched launches (ms)."""
    maps, rels, ms = [], [], 0.0
    for g0 in range(0, len(scenes), group):
        sl = slice(g0, g0 + group)
        br = BatchedRun(scenes[sl], grids[sl], [n_hist] * len(scenes[sl]), slots=stats_slots, engine=engine)
        try:
            _, out = br.run(seed + g0)
            ms += out.elapsed_ms
            for vg in br.download():
                maps.append(vg.kerma_keV / n_hist)
                if stats_slots > 1:
                    rels.append(relative_error(vg.kerma_keV, vg.kerma_sum2, vg.n_batches, vg.n_histories))
        finally:
            br.close()
    return np.stack(maps), (np.stack(rels) if rels else None), ms


def histories_for_error(hist, err, target: float):
    """Histories at which an error curve measured at ``hist`` reaches
    ``target``: log-log interpolation between the two levels around the
    crossing; None when no level reaches it.  When the first level is
    already below the target the answer is that level (no extrapolation)."""
    h = np.asarray(hist, dtype=float)
    e = np.asarray(err, dtype=float)
    order = np.argsort(h)
    h, e = h[order], e[order]
    if e[0] <= target:
        return float(h[0])
    for i in range(1, len(h)):
        if e[i] <= target:
            if e[i - 1] <= 0 or e[i] <= 0 or e[i] == e[i - 1]:
                return float(h[i])
            x = (np.log(target) - np.log(e[i - 1])) / (np.log(e[i]) - np.log(e[i - 1]))
            return float(np.exp(np.log(h[i - 1]) + x * (np.log(h[i]) - np.log(h[i - 1]))))
    return None


def inside_mask(mat: np.ndarray) -> np.ndarray:
    return mat != PH.MATERIALS.index("air")


def median_rel_error(k: np.ndarray, k_ref: np.ndarray, mask: np.ndarray) -> float:
    sel = mask & (k_ref > 0)
    return float(np.median(np.abs(k[sel] - k_ref[sel]) / k_ref[sel]))


class Dataset:
    """Normalised log maps of a set of phantoms.  ``k_in`` is one array
    [n, S, S, S] or a list of them (input maps at several history counts,
    one of which a training sample draws at random).  ``scale`` [levels, n]
    overrides the per-sample kerma scales (crops of a larger volume take
    that volume's)."""

    def __init__(self, k_in, k_tgt, mat, dens, rel=None, scale=None):
        levels = k_in if isinstance(k_in, (list, tuple)) else [k_in]
        rels = rel if isinstance(rel, (list, tuple)) else ([rel] if rel is not None else None)
        self.unc = None if rels is None else [DN.uncertainty_channel(r) for r in rels]
        self.n = levels[0].shape[0]
        self.S = levels[0].shape[1]
        self.mat = mat
        self.dens = dens
        inside = inside_mask(mat)
        self.scale = (np.asarray(scale, dtype=float).reshape(len(levels), self.n) if scale is not None else
                      np.array([[DN.kerma_scale(k[i], inside[i]) for i in range(self.n)] for k in levels]))
        self.xs = [np.stack([DN.to_log(k[i], self.scale[j, i]) for i in range(self.n)]) for j, k in enumerate(levels)]
        self.x = self.xs[0]
        self.t = None if k_tgt is None else [
            np.stack([DN.to_log(k_tgt[i], self.scale[j, i]) for i in range(self.n)]) for j in range(len(levels))]
        self.w = np.where(inside, 1.0, 0.1).astype(np.float32)

    def batch(self, idx, rng=None):
        """Arrays of a minibatch: a random input level and a random flip of
        each axis per sample when rng is given."""
        xs, ts, ds, ms, ws, us = [], [], [], [], [], []
        for i in idx:
            j = int(rng.integers(len(self.xs))) if rng is not None else 0
            arrs = [self.xs[j][i], self.t[j][i], self.dens[i], self.mat[i], self.w[i]]
            if self.unc is not None:
                arrs.append(self.unc[j][i])
            if rng is not None:
                for ax in range(3):
                    if rng.random() < 0.5:
                        arrs = [np.flip(a, axis=ax) for a in arrs]
            xs.append(arrs[0]); ts.append(arrs[1]); ds.append(arrs[2]); ms.append(arrs[3]); ws.append(arrs[4])
            if self.unc is not None:
                us.append(arrs[5])
        out = [np.ascontiguousarray(np.stack(a)) for a in (xs, ts, ds, ms, ws)]
        out.append(np.ascontiguousarray(np.stack(us)) if self.unc is not None else None)
        return out


def train(model: DN.UNet3D, data: Dataset, steps: int, batch: int, lr: float, seed: int = 0, log_every: int = 50,
          clip_ratio: float | None = None):
    """Adam with cosine learning-rate decay on random minibatches (random
    input level and axis flips); clip_ratio switches the model's adaptive
    gradient clipping (None keeps the model's setting)."""
    import torch
    rng = np.random.default_rng(seed)
    if clip_ratio is not None:
        model.clip_ratio = float(clip_ratio)
    S = data.S
    tgt = torch.empty(batch * S ** 3, dtype=torch.float32, device=model.dev)
    wgt = torch.empty_like(tgt)
    losses = []
    t0 = time.perf_counter()
    for step in range(steps):
        idx = rng.choice(data.n, size=batch, replace=data.n < batch)
        x, t, d, m, w, u = data.batch(idx, rng)
        model.set_input(x, d, m, batch, S, unc=u)
        tgt.copy_(torch.from_numpy(t.reshape(-1)))
        wgt.copy_(torch.from_numpy(w.reshape(-1)))
        model.forward()
        model.backward(tgt, wgt, 1.0 / float(w.sum()))
        # cosine decay
        cur = lr * 0.5 * (1.0 + np.cos(np.pi * step / max(steps, 1)))
        model.step(cur)
        if log_every and (step % log_every == 0 or step == steps - 1):
            losses.append((step, model.loss()))
    torch.cuda.synchronize()
    model.check_status()
    return losses, time.perf_counter() - t0


def denoise(model: DN.UNet3D, data: Dataset, batch: int = 8) -> tuple[np.ndarray, float]:
    """Denoised kerma maps of every sample and the device time (ms)."""
    import torch
    S = data.S
    out = np.empty((data.n, S, S, S))
    ms = 0.0
    for b0 in range(0, data.n, batch):
        idx = list(range(b0, min(b0 + batch, data.n)))
        bsz = len(idx)
        model.set_input(data.x[idx], data.dens[idx], data.mat[idx], bsz, S,
                        unc=data.unc[0][idx] if data.unc is not None else None)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        y = model.predict()
        e1.record()
        e1.synchronize()
        ms += e0.elapsed_time(e1)
        yl = y.cpu().numpy().reshape(bsz, S, S, S)
        for j, i in enumerate(idx):
            out[i] = DN.from_log(yl[j], data.scale[0, i])
    model.check_status()
    return out, ms


def run(args) -> dict:
    import torch
    from .transport import default_engine
    eng = default_engine()
    S = args.side
    t_all = time.perf_counter()
    tr_sc, tr_gr = PH.phantoms(args.train, args.seed, S, args.voxel_cm)
    te_sc, te_gr = PH.phantoms(args.test, args.seed + 1, S, args.voxel_cm)
    tr_maps = [PH.voxel_maps(s, g) for s, g in zip(tr_sc, tr_gr)]
    te_maps = [PH.voxel_maps(s, g) for s, g in zip(te_sc, te_gr)]
    tr_mat = np.stack([m for m, _ in tr_maps]); tr_den = np.stack([d for _, d in tr_maps])
    te_mat = np.stack([m for m, _ in te_maps]); te_den = np.stack([d for _, d in te_maps])

    k_in, r_in, ms_in = [], [], 0.0
    slots = 16 if args.uncertainty else 1
    for j, n in enumerate(args.n_in):
        k, r, ms = mc_maps(tr_sc, tr_gr, n, 1000 + 100 * j, eng, stats_slots=slots)
        k_in.append(k)
        r_in.append(r)
        ms_in += ms
    k_tg, _, ms_tg = mc_maps(tr_sc, tr_gr, args.n_target, 2000, eng)
    train_set = Dataset(k_in, k_tg, tr_mat, tr_den, rel=r_in if args.uncertainty else None)
    del k_in, k_tg, r_in
    k_ref, rel_ref, ms_ref = mc_maps(te_sc, te_gr, args.n_ref, 3000, eng, stats_slots=16)
    model = DN.UNet3D(seed=args.seed)
    losses, t_train = train(model, train_set, args.steps, args.batch, args.lr, seed=args.seed)
    if args.save:
        np.save(args.save, model.params_numpy())
    flops_step = 3.0 * DN.conv_flops(args.batch, S)

    inside = inside_mask(te_mat)
    ref_noise = float(np.median(0.6745 * np.nan_to_num(rel_ref[inside & (k_ref > 0)], nan=0.0)))
    levels = []
    for n in args.levels:
        k_n, rel_n, ms_n = mc_maps(te_sc, te_gr, n, 4000 + n % 997, eng, stats_slots=16)
        test = Dataset(k_n, None, te_mat, te_den, rel=rel_n if args.uncertainty else None)
        k_dn, ms_dn = denoise(model, test)
        plain_meas = median_rel_error(k_n, k_ref, inside)
        dn_meas = median_rel_error(k_dn, k_ref, inside)
        plain_pred = float(np.median(0.6745 * np.nan_to_num(rel_n[inside & (k_ref > 0)], nan=1.0)))
        levels.append({"histories": n, "plain_measured": plain_meas, "plain_from_stats": plain_pred,
                       "denoised_measured": dn_meas,
                       "denoised_corrected": float(np.sqrt(max(dn_meas ** 2 - ref_noise ** 2, 0.0))),
                       "mc_ms_per_phantom": ms_n / len(te_sc), "denoise_ms_per_phantom": ms_dn / len(te_sc)})
    # time to a 2 % median error per phantom, both at the batched Monte
    # Carlo's throughput on many phantoms (that of the reference run)
    rate = args.n_ref * len(te_sc) / (ms_ref * 1e-3)
    plain_c = np.median([lv["plain_from_stats"] * np.sqrt(lv["histories"]) for lv in levels])
    n_plain = (plain_c / 0.02) ** 2
    t_plain = n_plain / rate
    n_dn = histories_for_error([lv["histories"] for lv in levels], [lv["denoised_corrected"] for lv in levels], 0.02)
    t_inf = float(np.median([lv["denoise_ms_per_phantom"] for lv in levels])) * 1e-3
    t_dn = n_dn / rate + t_inf if n_dn is not None else None
    return {
        "workload": f"denoiser: {args.train} training + {args.test} held-out phantoms, {S}^3 voxels of "
                    f"{args.voxel_cm} cm, ellipsoid water/bone/lead/air, 60-120 kVp cone beam",
        "histories": {"input": args.n_in, "target": args.n_target, "reference": args.n_ref},
        "uncertainty_channel": bool(args.uncertainty),
        "mc_histories_per_s_batched": rate,
        "train": {"steps": args.steps, "batch": args.batch, "lr": args.lr, "seconds": t_train,
                  "tflops_per_s": flops_step * args.steps / t_train / 1e12, "losses": losses,
                  "params": DN.n_params()},
        "reference_noise_median": ref_noise,
        "levels": levels,
        "time_to_2pct_s": {"plain_mc": t_plain, "plain_histories": n_plain, "denoised": t_dn,
                           "denoised_histories": n_dn, "inference_s_per_phantom": t_inf,
                           "speedup": (t_plain / t_dn) if t_dn else None},
        "mc_ms": {"train_inputs": ms_in, "train_targets": ms_tg, "reference": ms_ref},
        "wall_s": time.perf_counter() - t_all,
    }


def timing(B: int, S: int, steps: int = 10, warmup: int = 3) -> dict:
    """Device time of the forward pass and of a whole training step (forward,
    backward, Adam) on B random volumes of side S, with CUDA events."""
    import torch
    rng = np.random.default_rng(0)
    xlog = rng.normal(size=(B, S, S, S)).astype(np.float32)
    mat = rng.integers(0, DN.N_MAT, size=(B, S, S, S)).astype(np.uint8)
    dens = np.array([0.0012, 1.0, 1.85, 11.35], dtype=np.float32)[mat]
    model = DN.UNet3D(seed=0)
    ho = DN.param_layout()["head"][0]
    model.p[ho:ho + DN.HEAD_CH] = 0.1
    model.set_input(xlog, dens, mat, B, S)
    tgt = torch.zeros(B * S ** 3, device=model.dev)
    wgt = torch.ones_like(tgt)
    for _ in range(warmup):
        model.forward(); model.backward(tgt, wgt, 1.0 / tgt.numel()); model.step(1e-4)
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    ev[0].record()
    for _ in range(steps):
        model.forward()
    ev[1].record()
    for _ in range(steps):
        model.forward(); model.backward(tgt, wgt, 1.0 / tgt.numel()); model.step(1e-4)
    ev[2].record()
    torch.cuda.synchronize()
    model.check_status()
    fwd = ev[0].elapsed_time(ev[1]) / steps
    step = ev[1].elapsed_time(ev[2]) / steps
    fl = DN.conv_flops(B, S)
    return {"batch": B, "side": S, "forward_ms": fwd, "train_step_ms": step,
            "forward_tflops": fl / fwd / 1e9, "train_tflops": 3 * fl / step / 1e9}


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--side", type=int, default=64)
    ap.add_argument("--voxel-cm", type=float, default=0.5)
    ap.add_argument("--train", type=int, default=256)
    ap.add_argument("--test", type=int, default=16)
    ap.add_argument("--n-in", type=int, nargs="+", default=[250_000, 1_000_000, 4_000_000])
    ap.add_argument("--n-target", type=int, default=200_000_000)
    ap.add_argument("--n-ref", type=int, default=500_000_000)
    ap.add_argument("--levels", type=int, nargs="+", default=[250_000, 500_000, 1_000_000, 2_000_000, 4_000_000])
    ap.add_argument("--steps", type=int, default=1500)
    ap.add_argument("--batch", type=int, default=4)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--save", default=None, help="write the trained parameters (.npy)")
    ap.add_argument("--no-uncertainty", dest="uncertainty", action="store_false",
                    help="do not give the network the input map's relative standard error")
    ap.add_argument("--timing", type=int, nargs=2, metavar=("B", "S"), default=None,
                    help="only time the network's kernels on B random volumes of side S")
    ap.add_argument("--timing-steps", type=int, default=10)
    args = ap.parse_args(argv)
    res = timing(*args.timing, steps=args.timing_steps) if args.timing else run(args)
    print(json.dumps(res))


if __name__ == "__main__":
    main()
