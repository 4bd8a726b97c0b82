"""Many scenes in one launch (the batched configuration), with an autotuner.

``BatchedRun`` builds one table set over the union of the scenes' materials,
one device scene, source and grid per scene, and a cc_batch plan: the
transport of every scene in one persistent launch plus the per-scene batch
folds, captured once as a CUDA graph and replayed by ``run``.

``autotune`` times a few launch shapes (block size, blocks per SM, histories
per chunk) on a scaled-down copy of the plan and keeps the fastest in a
JSON cache keyed by the GPU and the workload, so later runs of the same
workload start from it.
"""
from __future__ import annotations

import ctypes as C
import json
import os
import time
from pathlib import Path

import numpy as np

from . import _native as N
from .geometry import Geometry
from .source import SourceSpec
from .tally import VoxelGrid
from .transport import DeviceGrid, Engine, default_engine

CACHE_PATH = Path(os.environ.get("CHATCARLO_B200_AUTOTUNE",
                                 Path.home() / ".cache" / "chatcarlo_b200" / "autotune.json"))
DEFAULT_SHAPE = {"block": 256, "blocks_per_sm": 0, "chunk": 256}


class BatchedRun:
    def __init__(self, scenes: list[dict], grid_specs: list[dict] | None, n_histories: list[int],
                 slots: int = 1, engine: Engine | None = None, shape: dict | None = None):
        self.eng = engine or default_engine()
        self.n = len(scenes)
        self.counts = [int(x) for x in n_histories]
        self.geoms = [Geometry(raw["geometry"]) for raw in scenes]
        names = ["air"]
        for g in self.geoms:
            for m in g.materials():
                if m not in names:
                    names.append(m)
        self.names = names
        self.tally = grid_specs is not None
        self.ts, self.th = self.eng.tables(names, need_muen=self.tally)
        self.scene_h = [self.eng.scene(g, self.ts) for g in self.geoms]
        self.source_h = [self.eng.source(SourceSpec(raw["source"])) for raw in scenes]
        self.grids, self.dgrids = [], []
        if self.tally:
            for spec in grid_specs:
                vg = VoxelGrid(origin_cm=np.asarray(spec["origin"], dtype=float), shape=spec["shape"],
                               voxel_size_cm=spec["voxel_cm"], track_uncertainty=slots > 1)
                self.grids.append(vg)
                self.dgrids.append(DeviceGrid(self.eng, vg, stats=slots > 1))
        self.slots = slots
        self.shape = dict(DEFAULT_SHAPE, **(shape or {}))
        self.plan = None
        self._build()

    def _build(self):
        if self.plan is not None:
            self.eng.lib.cc_batch_destroy(self.plan)
        N.check(self.eng.lib.cc_ctx_set_launch(self.eng.ctx, self.shape["block"], self.shape["blocks_per_sm"]))
        sc = (C.c_void_p * self.n)(*[h.value for h in self.scene_h])
        src = (C.c_void_p * self.n)(*[h.value for h in self.source_h])
        gr = (C.c_void_p * self.n)(*[d.handle.value for d in self.dgrids]) if self.tally else None
        cnt = (C.c_int64 * self.n)(*self.counts)
        self.plan = C.c_void_p()
        try:
            N.check(self.eng.lib.cc_batch_create(self.eng.ctx, self.th, self.n, sc, src, gr, cnt, self.slots,
                                                 int(self.shape["chunk"]), C.byref(self.plan)))
        finally:
            N.check(self.eng.lib.cc_ctx_set_launch(self.eng.ctx, 256, 0))

    def reset(self):
        for d in self.dgrids:
            d.reset()

    def run(self, seed: int, fluorescence: bool = True):
        counts = np.zeros((self.n, 4), dtype=np.int64)
        out = N.RunOut()
        N.check(self.eng.lib.cc_batch_run(self.plan, int(seed), int(bool(fluorescence)),
                                          counts.ctypes.data_as(C.POINTER(C.c_int64)), C.byref(out)))
        return counts, out

    def download(self):
        for d, g in zip(self.dgrids, self.grids):
            d.download(g)
        return self.grids

    def close(self):
        if self.plan is not None:
            self.eng.lib.cc_batch_destroy(self.plan)
            self.plan = None
        for h in self.scene_h:
            self.eng.lib.cc_scene_destroy(h)
        self.scene_h = []
        for h in self.source_h:
            self.eng.lib.cc_source_destroy(h)
        self.source_h = []
        for d in self.dgrids:
            d.close()
        self.dgrids = []


def _gpu_key(engine: Engine) -> str:
    try:
        import torch
        return torch.cuda.get_device_name(engine.device)
    except Exception:  # noqa: BLE001 - torch is optional here
        return f"device{engine.device}"


def workload_key(n_histories: list[int], slots: int, tally: bool) -> str:
    n = len(n_histories)
    tot = int(sum(n_histories))
    return f"n{n}-h{int(np.log10(max(tot, 1)) * 4)}-s{slots}-t{int(tally)}"


def autotune(scenes, grid_specs, n_histories, slots=1, engine=None, scale=0.02,
             candidates=None, use_cache=True) -> dict:
    """Fastest launch shape for this workload: times each candidate on a plan
    with the history counts scaled by `scale` (at least 20,000 per scene)."""
    eng = engine or default_engine()
    key = f"{_gpu_key(eng)}|{workload_key(n_histories, slots, grid_specs is not None)}"
    cache = {}
    if use_cache and CACHE_PATH.exists():
        try:
            cache = json.loads(CACHE_PATH.read_text())
        except (OSError, ValueError):
            cache = {}
        if key in cache:
            return cache[key]["shape"]
    if candidates is None:
        candidates = [{"block": b, "blocks_per_sm": k, "chunk": c}
                      for b, ks in ((256, (2, 3, 4)), (128, (6, 8)))
                      for k in ks for c in (128, 256, 512)]
    small = [max(20_000, int(x * scale)) for x in n_histories]
    timings = []
    for cand in candidates:
        br = BatchedRun(scenes, grid_specs, small, slots=slots, engine=eng, shape=cand)
        try:
            br.run(seed=1)                       # warm-up
            best = min(br.run(seed=2 + i)[1].elapsed_ms for i in range(2))
        finally:
            br.close()
        timings.append((best, cand))
    timings.sort(key=lambda x: x[0])
    shape = timings[0][1]
    cache[key] = {"shape": shape, "ms": timings[0][0], "tried": len(timings), "when": time.time()}
    try:
        CACHE_PATH.parent.mkdir(parents=True, exist_ok=True)
        CACHE_PATH.write_text(json.dumps(cache, indent=1))
    except OSError:
        pass
    return shape


def main(argv=None) -> None:
    """``python -m chatcarlo_b200.batched``: the batched configuration (256
    random scenes, log-uniform 1e5-1e7 histories each, 64^3 tally grids) in
    one launch, after the autotuner picked its shape; one JSON line."""
    import argparse
    from . import workloads as W
    ap = argparse.ArgumentParser(description=main.__doc__.split("\n")[0])
    ap.add_argument("--scenes", type=int, default=256)
    ap.add_argument("--seed", type=int, default=2026)
    ap.add_argument("--repeats", type=int, default=3)
    args = ap.parse_args(argv)
    eng = default_engine()
    scenes, specs, counts = W.batched_scenes(n_scenes=args.scenes, seed=args.seed)
    t0 = time.perf_counter()
    shape = autotune(scenes, specs, counts, engine=eng, use_cache=False)
    t_tune = time.perf_counter() - t0
    br = BatchedRun(scenes, specs, counts, engine=eng, shape=shape)
    try:
        br.run(seed=1)
        outs = []
        for i in range(args.repeats):
            br.reset()
            outs.append(br.run(seed=2 + i)[1])
    finally:
        br.close()
    ms = float(np.median([o.elapsed_ms for o in outs]))
    total = int(sum(counts))
    o = outs[-1]
    print(json.dumps({"workload": f"{args.scenes} random scenes, 1e5-1e7 histories each, 64^3 grids",
                      "histories": total, "launch_ms": ms, "histories_per_s": total / (ms * 1e-3),
                      "segments_per_history": o.n_steps / total, "voxel_visits_per_history": o.n_voxel_visits / total,
                      "shape": shape, "autotune_s": t_tune, "gpu_launches_per_replay": int(o.gpu_launches)}))


if __name__ == "__main__":
    main()
