"""``python -m chatcarlo_b200 run scene.yaml ...`` -- ChatCarlo's ``run`` on the engine.

Flags and outputs follow chatcarlo/__main__.py:131-253,327-349: the same
summary lines (in English) and, with --dose-grid --dose-out, an .npz with the
keys dose_per_history_Gy, h10_per_history_pSv, kerma_keV, h10_track_pSv_cm3,
origin_cm, voxel_size_cm, shape (plus dose_Gy and h10_pSv for a CTDIvol-
calibrated source).  The dose and H*(10) maps are computed on the device.
"""
from __future__ import annotations

import argparse
import sys

import numpy as np


def cmd_run(args) -> int:
    from .scene import load_scene
    from .transport import run_transport
    scene = load_scene(args.scene)
    if not scene.ok:
        for e in scene.errors:
            print(f"[error] {e}", file=sys.stderr)
        return 1
    for w in scene.warnings:
        print(f"[warning] {w}")
    res = run_transport(scene, n_histories=int(args.n_histories), seed=args.seed,
                        batch_size=int(args.batch_size), dose_grid=args.dose_grid,
                        grid_resolution_cm=args.resolution, track_uncertainty=not args.no_uncertainty,
                        maps=args.dose_grid)
    print(f"histories: {res.n_histories:,}")
    print(f"absorbed (photoelectric) fraction: {res.fraction_absorbed:.4f}")
    print(f"escaped fraction: {res.fraction_escaped:.4f}")
    print(f"mean interactions per photon: {res.mean_scatter_events:.4f}")
    print(f"fluorescence emissions: {res.n_fluorescence:,}")
    print("absorbed energy by material [MeV, all histories]:")
    for name, e in sorted(res.energy_deposited_MeV.items(), key=lambda kv: -kv[1]):
        rel = res.energy_deposited_rel_err.get(name)
        print(f"  {name}: {e:.6g}" + (f"  (R={rel:.3g})" if rel is not None else ""))
    print(f"device time: {res.device_ms:.1f} ms ({res.n_histories / max(res.device_ms, 1e-9) * 1e3:.4g} histories/s)")
    if args.dose_grid:
        # per-history dose (density at each voxel centre) and H*(10) maps,
        # computed on the device (chatcarlo/__main__.py:200-209)
        g = res.grid
        dose = res.maps["dose_per_history_Gy"]
        h10 = res.maps["h10_per_history_pSv"]
        scale = res.n_photons_real
        print(f"dose grid: shape={g.shape}, resolution={g.voxel_size_cm}cm")
        print(f"  max absorbed dose [Gy/history]: {dose.max():.6g}")
        print(f"  total kerma: {g.total_kerma_MeV():.6g} MeV")
        print(f"  max H*(10) [pSv/history]: {h10.max():.6g}")
        if scale is not None:
            print(f"  max absorbed dose [Gy] (CTDIvol calibrated): {dose.max() * scale:.6g}")
            print(f"  max H*(10) [pSv] (CTDIvol calibrated): {h10.max() * scale:.6g}")
        if args.dose_out:
            keys = dict(dose_per_history_Gy=dose, h10_per_history_pSv=h10,
                        kerma_keV=g.kerma_keV, h10_track_pSv_cm3=g.h10_track_pSv_cm3,
                        origin_cm=g.origin_cm, voxel_size_cm=g.voxel_size_cm, shape=np.array(g.shape))
            if scale is not None:
                keys["dose_Gy"] = dose * scale
                keys["h10_pSv"] = h10 * scale
            np.savez(args.dose_out, **keys)
            print(f"wrote {args.dose_out}")
    return 0


def build_parser() -> argparse.ArgumentParser:
    ap = argparse.ArgumentParser(prog="chatcarlo_b200")
    sub = ap.add_subparsers(dest="cmd", required=True)
    p = sub.add_parser("run", help="photon transport on the GPU")
    p.add_argument("scene")
    p.add_argument("-n", "--n-histories", type=float, default=1e5)
    p.add_argument("--seed", type=int, default=None)
    p.add_argument("--dose-grid", action="store_true")
    p.add_argument("--resolution", type=float, default=5.0)
    p.add_argument("--dose-out", default=None)
    p.add_argument("--workers", type=int, default=1, help="accepted for compatibility; one GPU runs all histories")
    p.add_argument("--no-uncertainty", action="store_true")
    p.add_argument("--batch-size", type=float, default=200_000)
    p.set_defaults(func=cmd_run)
    return ap


def main(argv=None) -> int:
    args = build_parser().parse_args(argv)
    return args.func(args)


if __name__ == "__main__":
    sys.exit(main())
