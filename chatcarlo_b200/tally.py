"""Voxel tallies and batch statistics on the host side.

``VoxelGrid`` keeps the attribute layout of ChatCarlo's VoxelGrid
(chatcarlo/tally.py:27-132) so code that reads ``grid.kerma_keV`` and
friends works unchanged; the engine accumulates on the device and the
results land in these arrays.  The estimator helpers restate
tally.py:135-245: per-history variance from batch sums,
sigma^2 = (Q - T^2/N)/(M-1) with T = sum S_b, Q = sum S_b^2/n_b.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

MEV_TO_JOULE = 1.602176634e-13
G_TO_KG = 1e-3


def host_zeros(shape, dtype=np.float64, pinned: bool = False) -> np.ndarray:
    """Zeroed host array; page-locked (so device copies land in it directly)
    when pinned and a CUDA device is present."""
    if pinned:
        try:
            import torch
            if torch.cuda.is_available():
                tdt = {np.dtype(np.float64): torch.float64, np.dtype(np.int32): torch.int32}[np.dtype(dtype)]
                return torch.zeros(tuple(shape), dtype=tdt, pin_memory=True).numpy()
        except ImportError:
            pass
    return np.zeros(shape, dtype)


@dataclass
class VoxelGrid:
    origin_cm: np.ndarray
    shape: tuple
    voxel_size_cm: float
    track_uncertainty: bool = False
    pinned: bool = False            # page-locked arrays: the device writes results straight into them
    kerma_keV: np.ndarray = field(init=False)
    h10_track_pSv_cm3: np.ndarray = field(init=False)
    kerma_sum2: np.ndarray = field(init=False, default=None)
    h10_sum2: np.ndarray = field(init=False, default=None)
    n_batches_hit: np.ndarray = field(init=False, default=None)
    n_batches: int = field(init=False, default=0)
    n_histories: int = field(init=False, default=0)

    def __post_init__(self):
        self.origin_cm = np.asarray(self.origin_cm, dtype=float)
        self.shape = tuple(int(s) for s in self.shape)
        self.kerma_keV = host_zeros(self.shape, pinned=self.pinned)
        self.h10_track_pSv_cm3 = host_zeros(self.shape, pinned=self.pinned)
        if self.track_uncertainty:
            self.kerma_sum2 = host_zeros(self.shape, pinned=self.pinned)
            self.h10_sum2 = host_zeros(self.shape, pinned=self.pinned)
            self.n_batches_hit = host_zeros(self.shape, np.int32, pinned=self.pinned)

    @classmethod
    def from_bbox(cls, bbox_min, bbox_max, resolution_cm: float, track_uncertainty: bool = False,
                  pinned: bool = False):
        extent = np.asarray(bbox_max, dtype=float) - np.asarray(bbox_min, dtype=float)
        shape = tuple(max(1, int(np.ceil(x / resolution_cm))) for x in extent)
        return cls(origin_cm=np.asarray(bbox_min, dtype=float), shape=shape,
                   voxel_size_cm=resolution_cm, track_uncertainty=track_uncertainty, pinned=pinned)

    def kerma_relative_error(self) -> np.ndarray:
        return relative_error(self.kerma_keV, self.kerma_sum2, self.n_batches, self.n_histories)

    def h10_relative_error(self) -> np.ndarray:
        return relative_error(self.h10_track_pSv_cm3, self.h10_sum2, self.n_batches, self.n_histories)

    def voxel_index(self, points: np.ndarray):
        idx = np.floor((points - self.origin_cm) / self.voxel_size_cm).astype(int)
        valid = np.all((idx >= 0) & (idx < np.array(self.shape)), axis=1)
        return idx, valid

    def voxel_centers(self) -> np.ndarray:
        axes = [self.origin_cm[k] + (np.arange(self.shape[k]) + 0.5) * self.voxel_size_cm for k in range(3)]
        g = np.meshgrid(*axes, indexing="ij")
        return np.stack([x.ravel() for x in g], axis=1)

    def voxel_volume_cm3(self) -> float:
        return self.voxel_size_cm ** 3

    def total_kerma_MeV(self) -> float:
        return float(self.kerma_keV.sum()) / 1000.0

    def dose_map_Gy(self, density_g_cm3: np.ndarray) -> np.ndarray:
        mass_kg = density_g_cm3 * self.voxel_volume_cm3() * G_TO_KG
        energy_j = self.kerma_keV * 1e-3 * MEV_TO_JOULE
        return np.divide(energy_j, mass_kg, out=np.zeros_like(energy_j), where=mass_kg > 0)

    def h10_map_pSv(self) -> np.ndarray:
        return self.h10_track_pSv_cm3 / self.voxel_volume_cm3()


def batch_variance(T, Q, n_batches: int, n_histories: int):
    T = np.asarray(T, dtype=float)
    Q = np.asarray(Q, dtype=float)
    if n_batches < 2 or n_histories <= 0:
        return np.full_like(T, np.nan)
    return np.clip((Q - T ** 2 / n_histories) / (n_batches - 1), 0.0, None)


def standard_error(T, Q, n_batches: int, n_histories: int):
    var = batch_variance(T, Q, n_batches, n_histories)
    if n_histories <= 0:
        return np.full_like(var, np.nan)
    return np.sqrt(var / n_histories)


def relative_error(T, Q, n_batches: int, n_histories: int):
    T = np.asarray(T, dtype=float)
    sem = standard_error(T, Q, n_batches, n_histories)
    if n_histories <= 0:
        return np.full_like(T, np.nan)
    mean = T / n_histories
    with np.errstate(divide="ignore", invalid="ignore"):
        return np.where(mean != 0, sem / mean, np.nan)


def combine_moments(a: tuple, b: tuple) -> tuple:
    return tuple(x + y for x, y in zip(a, b))


@dataclass
class ScalarMoments:
    """Batch statistics of per-material scalars (tally.py:191-245)."""
    sums: dict = field(default_factory=dict)
    sum2s: dict = field(default_factory=dict)
    n_batches: int = 0
    n_histories: int = 0

    def add_batch(self, batch_values: dict, n_histories_in_batch: int) -> None:
        if n_histories_in_batch <= 0:
            return
        for name in set(self.sums) | set(batch_values):
            s_b = batch_values.get(name, 0.0)
            self.sums[name] = self.sums.get(name, 0.0) + s_b
            self.sum2s[name] = self.sum2s.get(name, 0.0) + s_b ** 2 / n_histories_in_batch
        self.n_batches += 1
        self.n_histories += n_histories_in_batch

    def add_moments(self, sums: dict, sum2s: dict, n_batches: int, n_histories: int) -> None:
        for name in set(self.sums) | set(sums):
            self.sums[name] = self.sums.get(name, 0.0) + sums.get(name, 0.0)
            self.sum2s[name] = self.sum2s.get(name, 0.0) + sum2s.get(name, 0.0)
        self.n_batches += n_batches
        self.n_histories += n_histories

    def relative_errors(self) -> dict:
        return {k: float(relative_error(self.sums[k], self.sum2s[k], self.n_batches, self.n_histories))
                for k in self.sums}

    def standard_errors(self) -> dict:
        return {k: float(standard_error(self.sums[k], self.sum2s[k], self.n_batches, self.n_histories))
                for k in self.sums}
