"""The transport entry points, backed by the sm_100a engine.

``transport_photons`` and ``run_transport`` keep the signatures and result
types of ChatCarlo's NumPy implementation (chatcarlo/transport.py:88-95,
98-103, 236-254, 358-361).  Every photon is transported by the CUDA engine
through the C ABI of include/chatcarlo_b200.h; there is no CPU path.  The
random streams are Philox4x32-10 streams keyed by a 64-bit seed and the
history index, so results are reproducible for a given seed and
independent of the launch shape, but not bit-identical to NumPy's PCG64.
"""
from __future__ import annotations

import ctypes as C
import os
import threading
from dataclasses import dataclass, field

import numpy as np

from . import _native as N
from .devtables import TableSet, build_table_set
from .geometry import Geometry
from .source import SourceSpec
from .tally import ScalarMoments, VoxelGrid


@dataclass
class BatchResult:
    n_scatter: np.ndarray
    absorbed: np.ndarray
    escaped: np.ndarray
    final_energy: np.ndarray
    energy_deposited: dict = field(default_factory=dict)
    n_fluorescence: int = 0


@dataclass
class TransportResult:
    n_histories: int
    energy_deposited_MeV: dict
    fraction_absorbed: float
    fraction_escaped: float
    mean_scatter_events: float
    grid: VoxelGrid | None = None
    n_photons_real: float | None = None
    n_fluorescence: int = 0
    n_batches: int = 0
    energy_deposited_sem_MeV: dict = field(default_factory=dict)
    energy_deposited_rel_err: dict = field(default_factory=dict)
    # engine bookkeeping (not in the NumPy result)
    device_ms: float = 0.0
    gpu_launches: int = 0
    transport_ms: float = 0.0
    transport_launches: int = 0
    n_steps: int = 0
    n_voxel_visits: int = 0
    # output maps computed on the device when run_transport(maps=True)
    maps: dict | None = None
    # batch moments of the energy deposited per material (keV; ScalarMoments,
    # tally.py:191-245): what merging runs over ranks needs
    moments: ScalarMoments | None = None


class DeviceGrid:
    """A cc_grid with the geometry of a host VoxelGrid."""

    def __init__(self, engine: "Engine", grid: VoxelGrid, stats: bool):
        self.engine = engine
        self.shape = tuple(grid.shape)
        self.handle = C.c_void_p()
        origin = np.ascontiguousarray(grid.origin_cm, dtype=float)
        nx, ny, nz = self.shape
        self.lib = engine.lib
        N.check(self.lib.cc_grid_create(engine.ctx, N.dptr(origin), nx, ny, nz, float(grid.voxel_size_cm),
                                        N.CC_GRID_STATS if stats else 0, C.byref(self.handle)), self.lib)
        self.stats = stats
        self.voxel_cm = float(grid.voxel_size_cm)

    def maps(self, geometry: Geometry, divisor: float = 1.0, dose: bool = True, h10: bool = True,
             rel: bool = False, out: dict | None = None) -> dict:
        """Output maps on the device (cc_grid_maps): ``dose_Gy`` (kerma to dose
        with the density at each voxel centre, chatcarlo/diagnostics.py:16-26),
        ``h10_pSv`` (tally.py:130-132) and, with ``rel``, ``kerma_rel`` /
        ``h10_rel`` (tally.py:96-100), each divided by ``divisor``; equal to
        the host computation bit for bit.  ``out`` may give the arrays
        (host numpy arrays, or torch CUDA tensors to keep the maps on the
        device)."""
        from .tables import density
        names = ["dose_Gy", "h10_pSv", "kerma_rel", "h10_rel"]
        want = [dose, h10, rel, rel]
        out = dict(out or {})
        on_device = None
        ptrs = []
        for name, w in zip(names, want):
            if not w:
                ptrs.append(None)
                continue
            a = out.get(name)
            if a is None:
                a = out[name] = np.empty(self.shape)
            dev = hasattr(a, "is_cuda") and a.is_cuda
            if on_device is None:
                on_device = dev
            if dev != on_device or tuple(a.shape) != self.shape:
                raise ValueError("map outputs must all be host arrays or all device tensors of the grid's shape")
            if dev:
                ptrs.append(a.data_ptr())
            else:
                if a.dtype != np.float64 or not a.flags.c_contiguous:
                    raise ValueError("host map outputs must be C-contiguous float64 arrays")
                ptrs.append(a.ctypes.data)
        prims = geometry.primitives({m: i for i, m in enumerate(geometry.materials())})
        dens = np.array([density(g["material"]) for g in geometry.geoms], dtype=float)
        N.check(self.lib.cc_grid_maps(self.handle, prims, len(geometry.geoms), N.dptr(dens),
                                      float(density(geometry.background)), self.voxel_cm ** 3, float(divisor),
                                      int(bool(on_device)), *ptrs), self.lib)
        return {k: out[k] for k, w in zip(names, want) if w}

    def download(self, grid: VoxelGrid, accumulate: bool = False) -> None:
        """Totals (and batch statistics) into the host grid's arrays: written
        in place when they are C-contiguous arrays of this shape (by the
        device itself when they are page-locked), else copied over."""
        stats = self.stats and grid.track_uncertainty

        def target(a, dtype=np.float64):
            ok = (not accumulate and isinstance(a, np.ndarray) and a.dtype == dtype and a.shape == self.shape
                  and a.flags.c_contiguous and a.flags.writeable)
            return a if ok else np.empty(self.shape, dtype)

        k = target(grid.kerma_keV)
        h = target(grid.h10_track_pSv_cm3)
        k2 = target(grid.kerma_sum2) if stats else None
        h2 = target(grid.h10_sum2) if stats else None
        nh = target(grid.n_batches_hit, np.int32) if stats else None
        nb = C.c_int64()
        nhist = C.c_int64()
        N.check(self.lib.cc_grid_download(
            self.handle, N.dptr(k), N.dptr(h), N.dptr(k2) if k2 is not None else None,
            N.dptr(h2) if h2 is not None else None,
            nh.ctypes.data_as(C.POINTER(C.c_int32)) if nh is not None else None,
            C.byref(nb), C.byref(nhist)), self.lib)
        if accumulate:
            grid.kerma_keV += k
            grid.h10_track_pSv_cm3 += h
        else:
            if k is not grid.kerma_keV:
                grid.kerma_keV[...] = k
            if h is not grid.h10_track_pSv_cm3:
                grid.h10_track_pSv_cm3[...] = h
        if stats:
            for src, name in ((k2, "kerma_sum2"), (h2, "h10_sum2"), (nh, "n_batches_hit")):
                if src is not getattr(grid, name):
                    getattr(grid, name)[...] = src
            grid.n_batches = int(nb.value)
            grid.n_histories = int(nhist.value)

    def upload(self, grid: VoxelGrid) -> None:
        """Load a host grid's totals (and batch statistics) into this device
        grid (cc_grid_upload)."""
        f64 = lambda a: np.ascontiguousarray(a, dtype=np.float64)  # noqa: E731
        k, h = f64(grid.kerma_keV), f64(grid.h10_track_pSv_cm3)
        if self.stats:
            if not grid.track_uncertainty:
                raise ValueError("a statistics device grid needs a host grid with track_uncertainty")
            k2, h2 = f64(grid.kerma_sum2), f64(grid.h10_sum2)
            nh = np.ascontiguousarray(grid.n_batches_hit, dtype=np.int32)
            N.check(self.lib.cc_grid_upload(self.handle, N.dptr(k), N.dptr(h), N.dptr(k2), N.dptr(h2),
                                            nh.ctypes.data_as(C.POINTER(C.c_int32)), int(grid.n_batches),
                                            int(grid.n_histories)), self.lib)
        else:
            N.check(self.lib.cc_grid_upload(self.handle, N.dptr(k), N.dptr(h), None, None, None,
                                            int(grid.n_batches), int(grid.n_histories)), self.lib)

    def reset(self):
        N.check(self.lib.cc_grid_reset(self.handle), self.lib)

    def close(self):
        if self.handle:
            self.lib.cc_grid_destroy(self.handle)
            self.handle = C.c_void_p()


class Engine:
    """A device context plus cached device tables per material set."""

    def __init__(self, device: int = 0, precision: str = "fp32"):
        """precision: "fp32" (the engine) or "fp64" (the same engine tracking
        positions, directions and distances in FP64: the precision reference)."""
        if precision not in ("fp32", "fp64"):
            raise ValueError("precision must be 'fp32' or 'fp64'")
        self.precision = precision
        self.lib = N.lib(N.FP64_LIB_PATH if precision == "fp64" else None)
        self.ctx = C.c_void_p()
        N.check(self.lib.cc_ctx_create(int(device), C.byref(self.ctx)))
        self.device = device
        self._tables: dict = {}
        self._grids: dict = {}
        self._sources: dict = {}
        self._lock = threading.Lock()

    def set_launch(self, block_size: int = 256, blocks_per_sm: int = 0) -> None:
        N.check(self.lib.cc_ctx_set_launch(self.ctx, block_size, blocks_per_sm))

    def set_tally_fp32(self, on: bool = True) -> None:
        """FP32 tally scratch cells for batches of <= 1e6 histories (one
        vector reduction per voxel visit; sums depend on the order of the
        FP32 additions) instead of the default FP64 cells."""
        N.check(self.lib.cc_ctx_set_tally_fp32(self.ctx, int(bool(on))), self.lib)

    def set_tally_queue(self, on: bool = True, capacity: int = 0) -> None:
        """Deferred tally: segments queued in device memory and scored by a
        second kernel (same scores; slower on B200, off by default).
        ``capacity`` > 0 fixes the queue size in records."""
        N.check(self.lib.cc_ctx_set_tally_queue(self.ctx, int(bool(on)), int(capacity)), self.lib)

    def set_step_limit(self, max_steps: int = 100_000) -> None:
        """Transport steps a single photon may take before the run fails with CC_E_TIMEOUT."""
        N.check(self.lib.cc_ctx_set_step_limit(self.ctx, int(max_steps)))

    def tables(self, names: list[str], need_muen: bool) -> tuple[TableSet, C.c_void_p]:
        key = (tuple(names), need_muen)
        with self._lock:
            hit = self._tables.get(key)
            if hit is None:
                ts = build_table_set(list(names), need_muen=need_muen)
                h = C.c_void_p()
                N.check(self.lib.cc_tables_create(self.ctx, C.byref(ts.desc), C.byref(h)))
                hit = (ts, h)
                self._tables[key] = hit
            return hit

    def scene(self, geometry: Geometry, ts: TableSet) -> C.c_void_p:
        idx = {n: i for i, n in enumerate(ts.names)}
        prims = geometry.primitives(idx)
        lo = np.ascontiguousarray(geometry.bbox_min, dtype=float)
        hi = np.ascontiguousarray(geometry.bbox_max, dtype=float)
        h = C.c_void_p()
        N.check(self.lib.cc_scene_create(self.ctx, prims, len(geometry.geoms), idx[geometry.background],
                                         N.dptr(lo), N.dptr(hi), C.byref(h)))
        return h

    def device_grid(self, grid: VoxelGrid, stats: bool) -> DeviceGrid:
        """A zeroed device grid of this shape, reused between calls."""
        key = (tuple(grid.shape), tuple(np.asarray(grid.origin_cm, dtype=float).tolist()),
               float(grid.voxel_size_cm), bool(stats))
        dg = self._grids.get(key)
        if dg is None:
            if len(self._grids) >= 4:
                _, old = self._grids.popitem()
                old.close()
            dg = DeviceGrid(self, grid, stats)
            self._grids[key] = dg
        else:
            dg.reset()
        return dg

    def source(self, spec: SourceSpec) -> C.c_void_p:
        h = C.c_void_p()
        N.check(self.lib.cc_source_create(self.ctx, C.byref(spec.desc), C.byref(h)))
        return h

    def cached_source(self, src: dict) -> C.c_void_p:
        """Device source for a scene's source section, built once per distinct section."""
        key = repr(src)
        with self._lock:
            h = self._sources.get(key)
            if h is None:
                h = self.source(SourceSpec(src))
                if len(self._sources) >= 16:
                    _, old = self._sources.popitem()
                    self.lib.cc_source_destroy(old)
                self._sources[key] = h
            return h

    def close(self):
        for dg in self._grids.values():
            dg.close()
        self._grids.clear()
        for h in self._sources.values():
            self.lib.cc_source_destroy(h)
        self._sources.clear()
        for ts, h in self._tables.values():
            self.lib.cc_tables_destroy(h)
        self._tables.clear()
        if self.ctx:
            self.lib.cc_ctx_destroy(self.ctx)
            self.ctx = C.c_void_p()


_engines: dict = {}


def default_engine(device: int | None = None) -> Engine:
    dev = int(os.environ.get("CHATCARLO_B200_DEVICE", "0")) if device is None else device
    if dev not in _engines:
        _engines[dev] = Engine(dev)
    return _engines[dev]


def _seed_from(rng, seed):
    if seed is not None:
        return int(seed) & 0xFFFFFFFFFFFFFFFF
    if rng is not None:
        return int(rng.integers(0, 2 ** 63))
    return int.from_bytes(os.urandom(8), "little")


def transport_photons(pos: np.ndarray, dirv: np.ndarray, energy: np.ndarray, geometry: Geometry,
                      rng: np.random.Generator | None = None, grid: VoxelGrid | None = None,
                      recorder=None, tally_rng=None, fluorescence_enabled: bool = True,
                      seed: int | None = None, stream_offset: int = 0,
                      engine: Engine | None = None) -> BatchResult:
    """Transport the given photons to absorption or escape on the GPU.

    Same contract as chatcarlo/transport.py:98-233: pos/dirv/energy are
    updated in place with the final state, grid (if given) accumulates the
    track-length kerma and H*(10) tallies.  The photon streams are keyed by
    ``seed`` (or one draw of ``rng``).  ``recorder`` (trajectory capture for
    visualisation) is not supported by the engine.
    """
    if recorder is not None:
        raise NotImplementedError("trajectory recording is not part of the GPU engine")
    eng = engine or default_engine()
    n = int(pos.shape[0])
    names = geometry.materials()
    ts, th = eng.tables(names, need_muen=grid is not None)
    sh = eng.scene(geometry, ts)
    try:
        p = np.ascontiguousarray(pos, dtype=np.float64)
        d = np.ascontiguousarray(dirv, dtype=np.float64)
        e = np.ascontiguousarray(energy, dtype=np.float64)
        # the device writes every element: no zero fill; the flags land
        # directly in bool arrays (one byte, 0 or 1)
        nsc = np.empty(n, dtype=np.int64)
        absd = np.empty(n, dtype=bool)
        esc = np.empty(n, dtype=bool)
        edep = np.zeros(len(names))
        nfl = C.c_int64(0)
        dg = eng.device_grid(grid, stats=False) if grid is not None else None
        N.check(eng.lib.cc_transport_photons(
            eng.ctx, sh, th, dg.handle if dg else None, n, N.dptr(p), N.dptr(d), N.dptr(e),
            _seed_from(rng, seed), int(stream_offset), int(bool(fluorescence_enabled)),
            nsc.ctypes.data_as(C.POINTER(C.c_int64)), absd.ctypes.data_as(C.POINTER(C.c_uint8)),
            esc.ctypes.data_as(C.POINTER(C.c_uint8)), N.dptr(edep), C.byref(nfl)))
        if dg is not None:
            dg.download(grid, accumulate=True)
    finally:
        eng.lib.cc_scene_destroy(sh)
    if p is not pos:
        pos[...] = p
    if d is not dirv:
        dirv[...] = d
    if e is not energy:
        energy[...] = e
    dep = {name: float(edep[i]) for i, name in enumerate(names) if edep[i] != 0.0}
    return BatchResult(n_scatter=nsc, absorbed=absd, escaped=esc,
                       final_energy=energy, energy_deposited=dep, n_fluorescence=int(nfl.value))


def run_transport(scene, n_histories: int = 100_000, seed: int | None = None,
                  batch_size: int = 200_000, dose_grid: bool = False,
                  grid_resolution_cm: float = 5.0, n_workers: int = 1,
                  track_uncertainty: bool = True, engine: Engine | None = None,
                  first_history: int = 0, grid: VoxelGrid | None = None,
                  maps: bool = False, distributed: bool | None = None) -> TransportResult:
    """run_transport (chatcarlo/transport.py:358-474) on the GPU.

    ``n_workers`` is accepted for signature compatibility; the reference's
    process workers (transport.py:397-437) are ranks here.  The source is
    sampled on the device, histories are grouped into batches of
    ``batch_size`` for the batch statistics.  With ``maps`` and a dose grid,
    ``result.maps`` holds the per-history dose and H*(10) maps of
    chatcarlo/__main__.py:200-209 (``dose_per_history_Gy``,
    ``h10_per_history_pSv``) and, with ``track_uncertainty``, the relative
    error maps (``kerma_rel``, ``h10_rel``), all computed on the device.

    Under torchrun (a default process group of W > 1 ranks, one GPU each;
    ``distributed=None`` detects it, ``False`` turns it off) rank r runs
    histories ``shard_range(n_histories, r, W)`` of the run keyed by
    ``seed``, so the ranks together run exactly the histories of a one-GPU
    run; the device grids are summed in place by one NCCL all-reduce per
    array, the counters and per-material moments by a few small ones, and
    every rank returns the whole run's result.
    """
    raw = scene.raw if hasattr(scene, "raw") else scene
    src = raw["source"]
    if src.get("mas") is not None and src.get("ctdi_vol_mGy") is None:
        raise RuntimeError("mAs calibration needs SpekPy's fluence, which is not available "
                           "(ctdi_vol_mGy calibration is)")
    eng = engine or default_engine()
    geometry = Geometry(raw["geometry"])
    if dose_grid and grid is None:
        grid = VoxelGrid.from_bbox(geometry.bbox_min, geometry.bbox_max, grid_resolution_cm,
                                   track_uncertainty=track_uncertainty, pinned=True)
    if not dose_grid:
        grid = None
    fluorescence = raw.get("physics", {}).get("fluorescence", True)
    rank, world = 0, 1
    if distributed is not False:
        from .distributed import world_info
        rank, world = world_info()
    n_local, first_local = int(n_histories), int(first_history)
    if world > 1:
        from .distributed import shard_range
        first, n_local = shard_range(n_histories, rank, world)
        first_local += first
    names = geometry.materials()
    ts, th = eng.tables(names, need_muen=grid is not None)
    sh = eng.scene(geometry, ts)
    srch = eng.cached_source(src)
    dg = eng.device_grid(grid, stats=track_uncertainty) if grid is not None else None
    edep = np.zeros(len(names))
    edep2 = np.zeros(len(names))
    out = N.RunOut()
    out_maps = None
    try:
        N.check(eng.lib.cc_run(eng.ctx, sh, th, srch, dg.handle if dg else None, n_local,
                               int(batch_size), _seed_from(None, seed), first_local,
                               int(bool(fluorescence)), N.dptr(edep), N.dptr(edep2), C.byref(out)))
        if dg is not None:
            if world > 1:
                from .distributed import allreduce_device_grid
                allreduce_device_grid(dg)
            dg.download(grid)
            if maps:
                m = dg.maps(geometry, divisor=float(max(int(n_histories), 1)), rel=track_uncertainty)
                out_maps = {"dose_per_history_Gy": m["dose_Gy"], "h10_per_history_pSv": m["h10_pSv"]}
                if track_uncertainty:
                    out_maps["kerma_rel"] = m["kerma_rel"]
                    out_maps["h10_rel"] = m["h10_rel"]
    finally:
        eng.lib.cc_scene_destroy(sh)
    n_batches = int(out.n_batches)
    dep = {name: float(edep[i]) for i, name in enumerate(names) if edep[i] != 0.0}
    sem, rel = {}, {}
    mom = None
    if track_uncertainty:
        mom = ScalarMoments()
        mom.add_moments(dep, {name: float(edep2[i]) for i, name in enumerate(names) if edep[i] != 0.0},
                        n_batches, n_local)
        sem = {k: v / 1000.0 for k, v in mom.standard_errors().items()}
        rel = mom.relative_errors()
    # absolute calibration from CTDIvol, once, with the run's seed (transport.py:442-451)
    n_photons_real = None
    if src.get("ctdi_vol_mGy") is not None:
        from .ctdi import effective_histories_from_ctdi
        n_photons_real = effective_histories_from_ctdi(src, seed=seed, engine=eng)
    nh = max(n_local, 1)
    res = TransportResult(
        n_histories=n_local,
        energy_deposited_MeV={k: v / 1000.0 for k, v in dep.items()},
        fraction_absorbed=out.n_absorbed / nh,
        fraction_escaped=out.n_escaped / nh,
        mean_scatter_events=out.scatter_sum / nh,
        grid=grid,
        n_photons_real=n_photons_real,
        n_fluorescence=int(out.n_fluorescence),
        n_batches=n_batches if track_uncertainty else (grid.n_batches if grid is not None else 0),
        energy_deposited_sem_MeV=sem,
        energy_deposited_rel_err=rel,
        device_ms=float(out.elapsed_ms),
        gpu_launches=int(out.gpu_launches),
        transport_ms=float(out.transport_ms),
        transport_launches=int(out.transport_launches),
        n_steps=int(out.n_steps),
        n_voxel_visits=int(out.n_voxel_visits),
        maps=out_maps,
        moments=mom,
    )
    if world > 1:
        import torch
        from .distributed import reduce_result
        reduce_result(res, device=torch.device("cuda", eng.device), grid=False)
    return res
