"""Throughput of the room-scale plain Monte Carlo workload (histories/s).

Workload: 400x400x300 cm air room with a water torso, two bone cylinders, a
0.05 cm lead sheet and a 20 cm concrete wall; 80 kVp spectrum in 1 keV bins,
35x43 cm field at SID 180 cm; kerma and H*(10) on 5 cm voxels over the room
(80x80x60) with batch statistics (batches of 200,000 histories).  One step
is one call of the run driver over --histories-per-step histories (default
1e7, so the default 10 steps are the 1e8-history run of the
configuration).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]

Under torchrun every rank simulates its own history range (weak scaling)
and the tallies are summed with one NCCL all-reduce at the end of the
timed region.  ``--impl reference`` times the CPU restatement of ChatCarlo's
NumPy path on all host cores instead (the reference arm).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "histories/s"
BATCH = 200_000
WORKLOAD = ("room-scale plain MC: 400x400x300 cm air room, water torso 35x25x20 cm, 2 bone cylinders "
            "r1.5x20 cm, 0.05 cm lead 30x30 cm at 150 cm, 20 cm concrete wall; 80 kVp W spectrum 2.5 mm Al "
            "(Kramers model, 1 keV bins); rect field 35x43 cm at SID 180 cm; kerma + H*(10) on 5 cm voxels "
            "80x80x60 with batch statistics")
WORKLOAD_CT = ("CT dosimetry plain MC: PMMA phantom 32 cm x 15 cm with five 1.3 cm air holes, 120 kVp W "
               "spectrum 6.8 mm Al (Kramers model, 1 keV bins), fan 50x4 cm at SID 60 cm, continuous rotation "
               "with 30 cm helical scan; kerma + H*(10) on 1 mm voxels 320x320x150 with batch statistics")


def workload(name: str):
    """(scene dict, grid spec, description) of a bench workload."""
    from chatcarlo_b200 import workloads as W
    if name == "ct":
        return W.ct(), W.CT_GRID, WORKLOAD_CT
    return W.room(), W.ROOM_GRID, WORKLOAD


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic(workload: str = "room"):
    """DRAM bytes per history of the transport kernel from the committed ncu
    summary of that workload."""
    p = ROOT / "profiles" / f"transport_kernel_{workload}.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d.get("dram_bytes_per_history")
    return None


class ClockSampler:
    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return None
        rows = []
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9:
                rows.append(f)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------------------
# reference arm: the CPU oracle on all host cores
# ---------------------------------------------------------------------------

def _ref_worker(n, seed, name="room"):
    import cc_oracle as O
    from chatcarlo_b200 import workloads as W
    raw, spec, _ = workload(name)
    agg = O.run_transport(raw, n_histories=n, seed=seed, batch_size=BATCH, grid_spec=spec,
                          n_workers=1, track_uncertainty=True)
    g = agg["grid"]
    return n, g.kerma_keV, g.h10_track_pSv_cm3


def _ref_warm(name):
    _ref_worker(200, 0, name)      # builds the element tables in this process
    return os.getpid()


def run_cpu_reference(steps: int, warmup: int, per_core: int, cores: int | None = None, name: str = "room"):
    """Times the oracle's run_transport on the workload with one process per
    host core (spawned), per_core histories per process per step."""
    import concurrent.futures
    import multiprocessing as mp
    sys.path.insert(0, str(ROOT / "oracle"))
    cores = cores or os.cpu_count() or 1
    if name == "ct":
        cores = min(cores, 8)        # each process holds the 15.4M-voxel grid with its statistics (~1 GB)
    ctx = mp.get_context("spawn")
    times, total = [], 0
    with concurrent.futures.ProcessPoolExecutor(max_workers=cores, mp_context=ctx,
                                                initializer=_ref_init, initargs=(str(ROOT),)) as pool:
        list(pool.map(_ref_warm, [name] * cores))
        for s in range(warmup + steps):
            t0 = time.perf_counter()
            futs = [pool.submit(_ref_worker, per_core, 1000 * s + i, name) for i in range(cores)]
            kerma = None
            n = 0
            for f in futs:
                k, a, b = f.result()
                n += k
                kerma = a if kerma is None else kerma + a
            dt = time.perf_counter() - t0
            if s >= warmup:
                times.append(dt)
                total += n
    return total / sum(times), cores, times


def _ref_init(root):
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "oracle"))


# ---------------------------------------------------------------------------
# learned denoiser leg
# ---------------------------------------------------------------------------

def denoiser_metric(eng, n_phantoms: int, levels=(500_000, 1_000_000, 2_000_000), n_ref: int = 1_000_000_000,
                    seed: int = 1001) -> dict:
    """Time to a 2 % median voxel-kerma error per phantom: plain batched
    Monte Carlo (its error from its own batch statistics, 1/sqrt(n)) against
    batched Monte Carlo at fewer histories plus the shipped denoiser (its
    error against an n_ref-history reference, the reference's own noise
    removed in quadrature), on phantoms the network was not trained on."""
    import torch
    from chatcarlo_b200 import denoise_run as R
    from chatcarlo_b200 import denoiser as DN
    from chatcarlo_b200 import phantoms as PH
    params, meta = DN.load_params()
    model = DN.UNet3D(params=params)
    sc, gr = PH.phantoms(n_phantoms, seed, 64, 0.5)
    maps = [PH.voxel_maps(a, b) for a, b in zip(sc, gr)]
    mat = np.stack([m for m, _ in maps])
    den = np.stack([d for _, d in maps])
    inside = R.inside_mask(mat)
    k_ref, rel_ref, ms_ref = R.mc_maps(sc, gr, n_ref, seed + 1, eng, stats_slots=16)
    rate = n_ref * n_phantoms / (ms_ref * 1e-3)
    ref_noise = float(np.median(0.6745 * np.nan_to_num(rel_ref[inside & (k_ref > 0)], nan=0.0)))
    rows = []
    for n in levels:
        k_n, rel_n, _ = R.mc_maps(sc, gr, n, seed + 2 + n % 991, eng, stats_slots=16)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record()
        k_dn = DN.denoise_kerma(k_n, rel_n, mat, den, model=model)
        ev1.record()
        ev1.synchronize()
        dn = R.median_rel_error(k_dn, k_ref, inside)
        plain = float(np.median(0.6745 * np.nan_to_num(rel_n[inside & (k_ref > 0)], nan=1.0)))
        rows.append({"histories": n, "plain": plain, "plain_measured": R.median_rel_error(k_n, k_ref, inside),
                     "denoised": float(np.sqrt(max(dn * dn - ref_noise ** 2, 0.0))), "denoised_measured": dn})
    t_inf = DN_inference_s(model, n_phantoms)
    c = float(np.median([r["plain"] * np.sqrt(r["histories"]) for r in rows]))
    n_plain = (c / 0.02) ** 2
    n_dn = R.histories_for_error([r["histories"] for r in rows], [r["denoised"] for r in rows], 0.02)
    t_plain = n_plain / rate
    t_dn = n_dn / rate + t_inf if n_dn is not None else None
    return {"metric": "time to 2% median voxel-kerma error per phantom (s)", "unit": "s",
            "plain_mc": t_plain, "denoised_batched": t_dn, "speedup": (t_plain / t_dn) if t_dn else None,
            "plain_histories": n_plain, "denoised_histories": n_dn, "inference_s_per_phantom": t_inf,
            "batched_mc_histories_per_s": rate, "reference_histories": n_ref, "reference_noise": ref_noise,
            "levels": rows, "phantoms": f"{n_phantoms} held-out 64^3 ellipsoid phantoms (seed {seed})",
            "network": meta.get("trained_by")}


def ct_denoiser_metric(eng, levels=(1_000_000, 3_000_000, 10_000_000), n_ref: int = 10_000_000_000) -> dict:
    """The same measurement on the CT configuration (1 mm voxels,
    320x320x150): its own phantom, never seen by the shipped CT network,
    denoised as one whole volume in a single pass of the network, against an
    n_ref-history reference."""
    from chatcarlo_b200 import ct_denoise as CD
    from chatcarlo_b200 import denoiser as DN
    from chatcarlo_b200 import phantoms as PH
    from chatcarlo_b200 import workloads as W
    model = DN.UNet3D(params=DN.load_params(CD.CT_PRETRAINED)[0])
    grid = W.make_grid(W.CT_GRID, track_uncertainty=True, pinned=True)
    sc = W.ct()
    mat, dens = PH.voxel_maps(sc, W.CT_GRID, CD.CT_MATERIALS)
    k_ref, rel_ref, ms_ref = CD.scan(sc, n_ref, 7, eng, grid, batches=100)
    sel = (mat != 0) & (k_ref > 0)
    ref_noise = float(np.median(0.6745 * np.nan_to_num(rel_ref[sel], nan=0.0)))
    rate = n_ref / (ms_ref * 1e-3)
    rows, t_inf = [], []
    for n in levels:
        k_n, rel_n, _ = CD.scan(sc, n, 11 + n % 991, eng, grid)
        k_dn, ms_dn = CD.denoise_volume(model, k_n, rel_n, mat, dens)
        t_inf.append(ms_dn * 1e-3)
        dn = float(np.median(np.abs(k_dn[sel] - k_ref[sel]) / k_ref[sel]))
        rows.append({"histories": n, "plain": float(np.median(0.6745 * np.nan_to_num(rel_n[sel], nan=1.0))),
                     "plain_measured": float(np.median(np.abs(k_n[sel] - k_ref[sel]) / k_ref[sel])),
                     "denoised": float(np.sqrt(max(dn * dn - ref_noise ** 2, 0.0))), "denoised_measured": dn})
    from chatcarlo_b200 import denoise_run as R
    c = float(np.median([r["plain"] * np.sqrt(r["histories"]) for r in rows]))
    n_plain = (c / 0.02) ** 2
    n_dn = R.histories_for_error([r["histories"] for r in rows], [r["denoised"] for r in rows], 0.02)
    t_plain = n_plain / rate
    t_dn = n_dn / rate + float(np.median(t_inf)) if n_dn is not None else None
    return {"metric": "time to 2% median voxel-kerma error of the CT phantom (s)", "unit": "s",
            "plain_mc": t_plain, "denoised": t_dn, "speedup": (t_plain / t_dn) if t_dn else None,
            "plain_histories": n_plain, "denoised_histories": n_dn, "inference_s": float(np.median(t_inf)),
            "mc_histories_per_s": rate, "reference_histories": n_ref, "reference_noise": ref_noise,
            "levels": rows, "volume": "320x320x150 voxels of 1 mm, one pass of the network over the whole volume"}


def DN_inference_s(model, n_phantoms: int) -> float:
    """Device time per phantom of the network's forward pass at batch 8."""
    import torch
    S, B = 64, min(8, n_phantoms)
    rng = np.random.default_rng(0)
    x = rng.normal(size=(B, S, S, S)).astype(np.float32)
    m = rng.integers(0, 4, size=(B, S, S, S)).astype(np.uint8)
    d = np.ones((B, S, S, S), np.float32)
    model.set_input(x, d, m, B, S, unc=np.full((B, S, S, S), 0.1, np.float32))
    model.predict()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    for _ in range(5):
        model.predict()
    ev1.record()
    ev1.synchronize()
    return ev0.elapsed_time(ev1) / 5 / B * 1e-3


# ---------------------------------------------------------------------------
# side measurements
# ---------------------------------------------------------------------------

def fp64_reduction_ceiling(eng, n_cells: int, repeats: int = 5) -> dict:
    """Measured rate of the tally's scoring pattern with nothing else in the
    kernel (cc_measure_fp64_reductions): two FP64 reductions into one
    16-byte cell per visit, cells spread uniformly over n_cells."""
    import ctypes as C
    import torch
    from chatcarlo_b200 import _native as N
    buf = torch.zeros(2 * n_cells, dtype=torch.float64, device=f"cuda:{eng.device}")
    v = C.c_double()
    N.check(eng.lib.cc_measure_fp64_reductions(eng.device, C.c_void_p(buf.data_ptr()), n_cells, 0,
                                               eng_sm_count(eng) * 8, 256, 256, 0, 0, 0, repeats, C.byref(v)),
            eng.lib)
    del buf
    return {"visits_per_s": v.value, "reductions_per_s": 2.0 * v.value, "cells": n_cells,
            "pattern": f"uniform over {n_cells} 16-byte cells ({n_cells * 16 / 2**20:.0f} MiB)"}


def atomics_sweep(eng) -> None:
    """The FP64-reduction ceiling over the patterns a tally produces: cells
    spread over an L2-resident region (the room grid, 8 of its batch slots)
    and over one beyond L2 (a CT slot), a few hot cells (a beam's busiest
    voxels), and runs of 16 cells `stride` apart (a photon crossing a row,
    a column or a plane of voxels).  One JSON line per case."""
    import ctypes as C
    import torch
    from chatcarlo_b200 import _native as N
    sms = eng_sm_count(eng)
    for n_cells, label in ((384_000, "room grid, 6 MiB"), (8 * 384_000, "8 room slots, 47 MiB"),
                           (15_360_000, "CT grid, 234 MiB")):
        buf = torch.zeros(2 * n_cells, dtype=torch.float64, device=f"cuda:{eng.device}")
        for mode, hot, run, stride in ((0, 0, 0, 0), (1, 32, 0, 0), (1, 4096, 0, 0), (2, 0, 16, 1), (2, 0, 16, 80),
                                       (2, 0, 16, 6400)):
            v = C.c_double()
            N.check(eng.lib.cc_measure_fp64_reductions(eng.device, C.c_void_p(buf.data_ptr()), n_cells, mode,
                                                       sms * 8, 256, 256, hot, run, stride, 5, C.byref(v)), eng.lib)
            pattern = {0: "uniform", 1: f"{hot} hot cells", 2: f"runs of {run}, stride {stride}"}[mode]
            print(json.dumps({"region": label, "pattern": pattern, "reductions_per_s": 2.0 * v.value}), flush=True)
        del buf
        torch.cuda.empty_cache()


def eng_sm_count(eng) -> int:
    import torch
    return torch.cuda.get_device_properties(eng.device).multi_processor_count


def side_measurements(eng, args, flush, n_vox_per_hist: float, hist_per_s_kernel: float) -> dict:
    import ctypes as C
    import torch
    from chatcarlo_b200 import _native as N
    from chatcarlo_b200 import workloads as W
    from chatcarlo_b200.geometry import Geometry
    from chatcarlo_b200.source import SourceSpec
    from chatcarlo_b200.transport import DeviceGrid
    out = {}
    # the atomics ceiling for the headline workload: the room grid's cells
    # times the batches a launch keeps in flight (8 slots of 384,000 cells,
    # 49 MB, L2-resident like the tally's scratch)
    ceil = fp64_reduction_ceiling(eng, 8 * 384_000)
    achieved = 2.0 * n_vox_per_hist * hist_per_s_kernel
    out["atomics"] = {"ceiling_per_s": ceil["reductions_per_s"], "ceiling_pattern": ceil["pattern"],
                      "frac": achieved / ceil["reductions_per_s"]}
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    # CT dosimetry configuration (15.4M voxels of 1 mm, batch statistics)
    raw = W.ct()
    geom = Geometry(raw["geometry"])
    ts, th = eng.tables(geom.materials(), need_muen=True)
    sh = eng.scene(geom, ts)
    srch = eng.source(SourceSpec(raw["source"]))
    g = W.make_grid(W.CT_GRID, track_uncertainty=True)
    dg = DeviceGrid(eng, g, stats=True)
    edep = np.zeros(len(ts.names))
    edep2 = np.zeros(len(ts.names))
    S = int(args.histories_per_step)
    try:
        ms, outs = [], []
        for i in range(3 + 3):
            flush.zero_()
            torch.cuda.synchronize()
            o = N.RunOut()
            ev0.record()
            N.check(eng.lib.cc_run(eng.ctx, sh, th, srch, dg.handle, S, BATCH, 777, i * S, 1, N.dptr(edep),
                                   N.dptr(edep2), C.byref(o)))
            ev1.record()
            torch.cuda.synchronize()
            if i >= 3:
                ms.append(ev0.elapsed_time(ev1))
                outs.append(o)
        n = S * len(ms)
        out["ct"] = {"metric": METRIC, "value": n / (float(np.sum(ms)) / 1e3), "unit": "histories/s",
                     "workload": WORKLOAD_CT, "histories_per_step": S, "steps": len(ms), "batch_size": BATCH,
                     "transport_ms_per_step": sum(o.transport_ms for o in outs) / len(ms),
                     "segments_per_history": sum(o.n_steps for o in outs) / n,
                     "voxel_visits_per_history": sum(o.n_voxel_visits for o in outs) / n,
                     "gpu_launches_per_step": sum(o.gpu_launches for o in outs) / len(ms)}
    finally:
        dg.close()
        eng.lib.cc_source_destroy(srch)
        eng.lib.cc_scene_destroy(sh)
    # the batched configuration: 256 random scenes, log-uniform 1e5-1e7
    # histories each, 64^3 grids, one persistent launch replayed from a CUDA
    # graph (launch shape from the autotuner)
    from chatcarlo_b200.batched import BatchedRun, autotune
    scenes, specs, counts = W.batched_scenes()
    shape = autotune(scenes, specs, counts, engine=eng)
    br = BatchedRun(scenes, specs, counts, engine=eng, shape=shape)
    try:
        br.run(seed=1)
        ms = []
        for i in range(3):
            br.reset()
            flush.zero_()
            torch.cuda.synchronize()
            ms.append(br.run(seed=2 + i)[1].elapsed_ms)
    finally:
        br.close()
    total = int(sum(counts))
    out["batched"] = {"metric": METRIC, "value": total / (float(np.median(ms)) / 1e3), "unit": "histories/s",
                      "workload": "256 random scenes (1-12 primitives, 7 materials, mono 20-140 keV or 60-140 kVp "
                                  "spectra), log-uniform 1e5-1e7 histories each, 64^3 kerma grids, one launch",
                      "histories": total, "launch_ms_median": float(np.median(ms)), "replays": len(ms),
                      "shape": shape}
    return out


# ---------------------------------------------------------------------------
# engine arm
# ---------------------------------------------------------------------------

def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--histories-per-step", type=float, default=1e7)
    ap.add_argument("--e2e-histories", type=float, default=4e6)
    ap.add_argument("--cpu-histories-per-process", type=int, default=None,
                    help="CPU sample per step: histories in each of the host-core processes "
                         "(default 120,000 for room, 1,000 for ct)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-precision", action="store_true", help="skip the FP32-vs-FP64 tracking tally report")
    ap.add_argument("--precision-histories", type=float, default=1e7)
    ap.add_argument("--no-fp32-cells", action="store_true",
                    help="skip the side measurement with FP32 tally scratch cells")
    ap.add_argument("--no-denoiser", action="store_true", help="skip the denoised time-to-2 %% measurements")
    ap.add_argument("--denoiser-phantoms", type=int, default=8)
    ap.add_argument("--atomics-sweep", action="store_true",
                    help="only print the FP64-reduction ceiling for several scoring patterns (JSON lines)")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the side measurements of the CT and batched configurations and the atomics ceiling")
    ap.add_argument("--workload", choices=["room", "ct"], default="room",
                    help="room-scale (the headline configuration) or CT dosimetry")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.cpu_histories_per_process is None:
        args.cpu_histories_per_process = 1_000 if args.workload == "ct" else 120_000

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return 0
        per_core = args.cpu_histories_per_process // 2
        value, cores, times = run_cpu_reference(args.steps, args.warmup, per_core, name=args.workload)
        line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "histories/s",
                "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": 1000.0 * float(np.mean(times)), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": workload(args.workload)[2], "histories_per_step": per_core * cores,
                           "batch_size": BATCH, "l2": "n/a (CPU)"},
                "cpu_baseline": {"value": value, "unit": "histories/s", "cores": cores, "kind": "port",
                                 "sample": f"{per_core} histories per process x {cores} processes per step"},
                "e2e": {"value": value, "unit": "histories/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return 0

    import torch
    import torch.distributed as dist
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", init_method="env://",
                                timeout=__import__("datetime").timedelta(seconds=120))
    import ctypes as C
    from chatcarlo_b200 import _native as N
    from chatcarlo_b200 import workloads as W
    from chatcarlo_b200.geometry import Geometry
    from chatcarlo_b200.source import SourceSpec
    from chatcarlo_b200.transport import DeviceGrid, Engine, transport_photons

    device = local if world > 1 else 0
    torch.cuda.set_device(device)
    eng = Engine(device)
    if args.atomics_sweep:
        if rank == 0:
            atomics_sweep(eng)
        return 0
    raw, gspec, desc = workload(args.workload)
    geom = Geometry(raw["geometry"])
    ts, th = eng.tables(geom.materials(), need_muen=True)
    sh = eng.scene(geom, ts)
    spec = SourceSpec(raw["source"])
    srch = eng.source(spec)
    grid = W.make_grid(gspec, track_uncertainty=True)
    dg = DeviceGrid(eng, grid, stats=True)
    S = int(args.histories_per_step)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    edep = np.zeros(len(ts.names))
    edep2 = np.zeros(len(ts.names))
    seed = 20261203
    base = rank << 40

    def step(i):
        out = N.RunOut()
        N.check(eng.lib.cc_run(eng.ctx, sh, th, srch, dg.handle, S, BATCH, seed, base + i * S, 1,
                               N.dptr(edep), N.dptr(edep2), C.byref(out)))
        return out

    for i in range(args.warmup):
        step(i)
    N.check(eng.lib.cc_grid_reset(dg.handle))
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    step_ms, outs = [], []
    with ClockSampler(device) as clk:
        for i in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            ev0.record()
            outs.append(step(args.warmup + i))
            ev1.record()
            torch.cuda.synchronize()
            step_ms.append(ev0.elapsed_time(ev1))
        red_ms = 0.0
        if world > 1:
            # the one exchange step: sum the device-resident tally grids and
            # their batch statistics over ranks in place (totals, sums of
            # squares and hit counts are additive, as when the reference
            # merges its workers); the time covers every collective of it
            from chatcarlo_b200.distributed import allreduce_device_grid
            ev0.record()
            allreduce_device_grid(dg)
            ev1.record()
            torch.cuda.synchronize()
            red_ms = ev0.elapsed_time(ev1)
    clocks = clk.summary()
    total_ms = float(np.sum(step_ms)) + red_ms
    if world > 1:
        tt = torch.tensor([total_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        total_ms = float(tt.item())
        dist.barrier()
    hist = S * args.steps * world
    value = hist / (total_ms / 1e3)

    n_h = S * args.steps
    n_seg = sum(o.n_steps for o in outs) / n_h
    n_vox = sum(o.n_voxel_visits for o in outs) / n_h
    b_hist = 96.0 * n_seg + 32.0 * n_vox + 32.0
    tr_ms = sum(o.transport_ms for o in outs)
    tr_launch = sum(o.transport_launches for o in outs)
    launches = sum(o.gpu_launches for o in outs)
    peak, peak_kind = peaks()
    achieved = b_hist * n_h / (tr_ms / 1e3) / 1e9
    traffic_per_hist = profile_traffic(args.workload)
    hist_per_launch = n_h / max(tr_launch, 1)

    # e2e: the public run_transport call a user makes, once per step: scene,
    # source and spectrum descriptors go to the device, the five tally grids
    # (kerma, H*(10), their batch sums of squares, batches hit) come back
    e2e = None
    e2e_photons = None
    if rank == 0:
        from chatcarlo_b200.transport import run_transport
        eg = W.make_grid(gspec, track_uncertainty=True, pinned=True)
        e_ms = []
        for i in range(args.warmup + min(args.steps, 5)):
            flush.zero_()
            torch.cuda.synchronize()
            ev0.record()
            run_transport(raw, n_histories=S, seed=seed + 100 + i, batch_size=BATCH, dose_grid=True, grid=eg,
                          engine=eng, first_history=(1 << 44) + i * S)
            ev1.record()
            torch.cuda.synchronize()
            if i >= args.warmup:
                e_ms.append(ev0.elapsed_time(ev1))
        nvox = int(np.prod(grid.shape))
        h2d = (len(raw["geometry"]) * C.sizeof(N.Primitive) + C.sizeof(N.SourceDesc)
               + 2 * 8 * len(raw["source"]["spectrum"]) + 6 * 8)
        e2e = {"value": S * len(e_ms) / (float(np.sum(e_ms)) / 1e3), "unit": "histories/s",
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(nvox * (4 * 8 + 4) + C.sizeof(N.RunOut)),
               "api": "chatcarlo_b200.transport.run_transport (C ABI cc_run + cc_grid_download)"}
        # the same through transport_photons on pinned host photon arrays
        ne = int(args.e2e_histories)
        pin = lambda shape: torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy()  # noqa: E731
        p0, d0, e0 = pin((ne, 3)), pin((ne, 3)), pin((ne,))
        N.check(eng.lib.cc_sample_source(eng.ctx, srch, ne, seed + 7, 1 << 50, N.dptr(p0), N.dptr(d0), N.dptr(e0)))
        p, d, e = pin((ne, 3)), pin((ne, 3)), pin((ne,))
        egrid = W.make_grid(gspec, track_uncertainty=False)
        e_ms = []
        for i in range(args.warmup + min(args.steps, 5)):
            np.copyto(p, p0)
            np.copyto(d, d0)
            np.copyto(e, e0)
            flush.zero_()
            torch.cuda.synchronize()
            ev0.record()
            transport_photons(p, d, e, geom, seed=seed + i, grid=egrid, engine=eng)
            ev1.record()
            torch.cuda.synchronize()
            if i >= args.warmup:
                e_ms.append(ev0.elapsed_time(ev1))
        e2e_photons = {"value": ne * len(e_ms) / (float(np.sum(e_ms)) / 1e3), "unit": "histories/s",
                       "h2d_bytes_per_step": ne * (3 + 3 + 1) * 8,
                       "d2h_bytes_per_step": ne * (3 + 3 + 1) * 8 + ne * (4 + 1 + 1) + 2 * nvox * 8,
                       "api": "chatcarlo_b200.transport.transport_photons (C ABI cc_transport_photons, pinned host arrays)"}

    # precision: the same room run tracked in FP32 (the engine) and in FP64,
    # every tally's difference against its own statistical error
    precision = None
    if rank == 0 and world == 1 and not args.no_precision:
        from chatcarlo_b200.precision import tally_precision
        from chatcarlo_b200.transport import Engine as _Engine
        rep = tally_precision(raw, gspec, int(args.precision_histories), seed + 999, batch_size=BATCH,
                              engine32=eng, engine64=_Engine(eng.device, precision="fp64"))
        precision = {"reference": "the same engine tracking in FP64, same seed and random numbers",
                     "histories": rep["histories"],
                     **{t: {k: rep[t][k] for k in ("rel_median", "rel_p99", "sigma_median", "sigma_p99",
                                                   "sigma_max", "total_rel")} for t in ("kerma", "h10")}}

    # side measurement: the same steps with FP32 tally scratch cells (an
    # opt-in of the context), and what they cost each tally against the
    # default FP64 cells on the same histories (tracking identical, so the
    # difference is the FP32 summation alone)
    fp32_cells = None
    if rank == 0 and world == 1 and not args.no_fp32_cells:
        from chatcarlo_b200.precision import _stats
        n_side = min(args.steps, 5)
        eng.set_tally_fp32(True)
        try:
            N.check(eng.lib.cc_grid_reset(dg.handle))
            for i in range(args.warmup):
                step(i)
            N.check(eng.lib.cc_grid_reset(dg.handle))
            f_ms = []
            for i in range(n_side):
                flush.zero_()
                torch.cuda.synchronize()
                ev0.record()
                step(args.warmup + i)
                ev1.record()
                torch.cuda.synchronize()
                f_ms.append(ev0.elapsed_time(ev1))
            grids = []
            for on in (False, True):
                eng.set_tally_fp32(on)
                N.check(eng.lib.cc_grid_reset(dg.handle))
                step(0)
                g = W.make_grid(gspec, track_uncertainty=True)
                dg.download(g)
                grids.append(g)
        finally:
            eng.set_tally_fp32(False)
        g64, g32 = grids
        fp32_cells = {"value": S * n_side / (float(np.sum(f_ms)) / 1e3), "unit": "histories/s", "steps": n_side,
                      "vs_fp64_cells": {"histories": S,
                                        "kerma": _stats(g32.kerma_keV, g64.kerma_keV, g64.kerma_sum2,
                                                        g64.n_batches, g64.n_histories),
                                        "h10": _stats(g32.h10_track_pSv_cm3, g64.h10_track_pSv_cm3,
                                                      g64.h10_sum2, g64.n_batches, g64.n_histories)}}

    # learned denoiser: time to a 2 % median voxel-kerma error, denoised +
    # batched Monte Carlo vs plain batched Monte Carlo, on held-out phantoms
    denoise = ct_denoise = None
    if rank == 0 and world == 1 and not args.no_denoiser:
        denoise = denoiser_metric(eng, args.denoiser_phantoms)
        ct_denoise = ct_denoiser_metric(eng)

    # side measurements under the same clock record: the CT configuration's
    # plain MC and the batched configuration's one-launch run, and the
    # measured ceiling of the tally's FP64 reductions
    extras = {}
    if rank == 0 and world == 1 and not args.no_extras:
        extras = side_measurements(eng, args, flush, n_vox_per_hist=n_vox, hist_per_s_kernel=n_h / (tr_ms / 1e3))

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        per_core = args.cpu_histories_per_process
        v, cores, times = run_cpu_reference(1, 0, per_core, name=args.workload)
        cpu = {"value": v, "unit": "histories/s", "cores": cores, "kind": "port",
               "sample": f"{args.workload} workload, {per_core} histories in each of {cores} spawned processes "
                         f"({per_core * cores} histories, {times[0]:.1f} s wall incl. pool start)"}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "histories/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": desc, "histories_per_step_per_gpu": S, "batch_size": BATCH,
                           "grid": list(grid.shape), "voxel_cm": gspec["voxel_cm"], "tally_dtype": "f64",
                           "l2": "flushed between steps (256 MiB write)",
                           "parallelism": f"history shards x{world}"},
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "peak_kind": peak_kind,
                             "traffic": (traffic_per_hist * hist_per_launch) if traffic_per_hist else None,
                             "kernel": "transport_kernel<true,true>",
                             "bytes_per_history": b_hist, "segments_per_history": n_seg,
                             "voxel_visits_per_history": n_vox,
                             "avg_launch_ms": tr_ms / max(tr_launch, 1),
                             "histories_per_launch": hist_per_launch,
                             # the tally's atomic bound: two FP64 reductions (kerma, H*(10)) per voxel visit
                             "atomics": dict({"per_history": 2.0 * n_vox,
                                              "achieved_per_s": 2.0 * n_vox * n_h / (tr_ms / 1e3),
                                              "cells": "fp64"}, **extras.get("atomics", {}))},
                "cpu_baseline": cpu, "e2e": e2e, "e2e_photons": e2e_photons, "precision": precision,
                "denoiser": denoise, "denoiser_ct": ct_denoise, "tally_fp32_cells": fp32_cells,
                "ct": extras.get("ct"), "batched": extras.get("batched"),
                "clocks": clocks,
                "gpu_launches": int(launches),
                "reduce_ms": red_ms}
        print(json.dumps(line))
    dg.close()
    eng.lib.cc_source_destroy(srch)
    eng.lib.cc_scene_destroy(sh)
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
