"""Learned kerma denoiser: a 3D U-Net trained on the engine's own Monte Carlo.

The network maps a low-history kerma map (plus density and material maps)
to an estimate of the high-history map.  It works in log space: with s the
mean input kerma per history inside the phantom,

    x   = ln(k_in / s + EPS)         (input channel 0, and the residual)
    out = x + head(U-Net(x, density, material one-hot))
    k_denoised = s * (exp(out) - EPS)

and is trained on ln(k_target / s + EPS) with a squared error weighted
towards the phantom's voxels.  Plain Monte Carlo stays the fallback and
the measure of its error: the denoised map is only ever scored against a
high-history Monte Carlo map.

Architecture: 4 levels with 16, 32, 64 and 128 channels; two 3x3x3 ReLU
convolutions per level; 2x2x2 average pooling down; nearest upsampling up,
concatenated with the skip tensor inside the convolution's gather; a 1x1x1
head.  Weights are BF16 copies of FP32 master weights; activations BF16;
every convolution accumulates in FP32 on the tensor cores.  The forward,
backward and optimizer steps are the kernels of libccunet.so; torch only
allocates device memory and provides the stream.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _unet_native as U

EPS = 0.05
IN_CH = 16
N_MAT = 4                       # air, water, bone, lead
DENSITY_SCALE = 0.25


@dataclass(frozen=True)
class Conv:
    name: str
    ca: int          # channels of the full-resolution input
    cb: int          # channels of the half-resolution input (upsampled), 0 if none
    cout: int
    level: int       # resolution level of input and output (0 = full)

    @property
    def cin(self) -> int:
        return self.ca + self.cb


LAYERS = [
    Conv("e0a", 16, 0, 16, 0), Conv("e0", 16, 0, 16, 0),
    Conv("e1a", 16, 0, 32, 1), Conv("e1", 32, 0, 32, 1),
    Conv("e2a", 32, 0, 64, 2), Conv("e2", 64, 0, 64, 2),
    Conv("b3a", 64, 0, 128, 3), Conv("b3", 128, 0, 128, 3),
    Conv("d2a", 64, 128, 64, 2), Conv("d2", 64, 0, 64, 2),
    Conv("d1a", 32, 64, 32, 1), Conv("d1", 32, 0, 32, 1),
    Conv("d0a", 16, 32, 16, 0), Conv("d0", 16, 0, 16, 0),
]
HEAD_CH = 16


def param_layout() -> dict[str, tuple[int, int, int, int]]:
    """name -> (weight offset, weight size, bias offset, bias size) in the
    flat FP32 parameter vector; the head ('head') is 16 weights + 1 bias."""
    out, off = {}, 0
    for L in LAYERS:
        nw = 27 * L.cout * L.cin
        out[L.name] = (off, nw, off + nw, L.cout)
        off += nw + L.cout
    out["head"] = (off, HEAD_CH, off + HEAD_CH, 1)
    return out


def n_params() -> int:
    lay = param_layout()
    o, n, bo, bn = lay["head"]
    return bo + bn


def init_params(seed: int = 0) -> np.ndarray:
    """He-normal convolution weights, zero biases, zero head (the untrained
    network returns its input)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(n_params(), dtype=np.float32)
    for L in LAYERS:
        o, n, _, _ = param_layout()[L.name]
        p[o:o + n] = rng.normal(0.0, np.sqrt(2.0 / (27 * L.cin)), n).astype(np.float32)
    return p


def conv_flops(B: int, S: int) -> float:
    """Multiply-adds x 2 of one forward pass over B volumes of side S."""
    return float(sum(2 * 27 * L.cin * L.cout * B * (S >> L.level) ** 3 for L in LAYERS))


class UNet3D:
    """Parameters, optimizer state and activation buffers on one device."""

    def __init__(self, params: np.ndarray | None = None, seed: int = 0, device: str = "cuda"):
        import torch
        self.torch = torch
        self.dev = torch.device(device)
        U.lib()
        p = init_params(seed) if params is None else np.asarray(params, dtype=np.float32)
        if p.size != n_params():
            raise ValueError(f"expected {n_params()} parameters, got {p.size}")
        self.lay = param_layout()
        self.p = torch.from_numpy(p.copy()).to(self.dev)
        self.g = torch.zeros_like(self.p)
        self.m = torch.zeros_like(self.p)
        self.v = torch.zeros_like(self.p)
        self.step_n = 0
        # adaptive gradient clipping: 0 = off, else the cap on the gradient
        # norm as a multiple of its running mean (ccu_adam_clipped)
        self.clip_ratio = 3.0
        self.clip_state = torch.zeros(3, dtype=torch.float64, device=self.dev)
        lib = U.lib()
        self.w = {L.name: torch.empty(lib.ccu_packed_weight_elems(L.cout, L.cin), dtype=torch.bfloat16,
                                      device=self.dev) for L in LAYERS}
        self.wt = {L.name: torch.empty(lib.ccu_packed_weight_elems(L.cin, L.cout), dtype=torch.bfloat16,
                                       device=self.dev) for L in LAYERS}
        self.acc = torch.zeros(1, dtype=torch.float32, device=self.dev)      # loss
        self.shape = None
        self.launches = 0
        self.pack()

    # -- helpers ----------------------------------------------------------
    def _stream(self):
        return self.torch.cuda.current_stream(self.dev).cuda_stream

    def _ptr(self, t, off: int = 0) -> int:
        return t.data_ptr() + off * t.element_size()

    def _call(self, fn, *args):
        U.check(fn(*args))
        self.launches += 1

    def pack(self) -> None:
        lib, st = U.lib(), self._stream()
        for L in LAYERS:
            o, _, _, _ = self.lay[L.name]
            self._call(lib.ccu_pack_weights, self._ptr(self.p, o), L.cout, L.cin, self._ptr(self.w[L.name]),
                       self._ptr(self.wt[L.name]), st)

    def params_numpy(self) -> np.ndarray:
        return self.p.detach().cpu().numpy()

    @staticmethod
    def _side3(S) -> tuple[int, int, int]:
        """(D, H, W) of a volume given as one side or three."""
        d = (int(S),) * 3 if np.isscalar(S) else tuple(int(x) for x in S)
        if len(d) != 3 or any(x <= 0 or x % 8 for x in d):
            raise ValueError("every volume side must be a positive multiple of 8 (three 2x2x2 poolings)")
        return d

    def _t(self, level: int, c: int, dtype=None):
        B, D, H, W = self.shape
        return self.torch.empty(B * (D >> level) * (H >> level) * (W >> level) * c,
                                dtype=dtype or self.torch.bfloat16, device=self.dev)

    def _alloc(self, B: int, S) -> None:
        D, H, W = self._side3(S)
        if self.shape == (B, D, H, W):
            return
        torch = self.torch
        self.shape = (B, D, H, W)
        t = self._t
        a = {"x0": t(0, IN_CH), "p0": t(1, 16), "p1": t(2, 32), "p2": t(3, 64)}
        for L in LAYERS:
            a[L.name] = t(L.level, L.cout)
        self.a = a
        self.gb = None                       # gradient buffers: allocated by the first backward pass
        n0 = B * D * H * W
        self.xlog = torch.empty(n0, dtype=torch.float32, device=self.dev)
        self.out = torch.empty(n0, dtype=torch.float32, device=self.dev)

    def _alloc_grads(self) -> None:
        if self.gb is not None:
            return
        t = self._t
        g = {}
        for L in LAYERS:
            g["dz_" + L.name] = t(L.level, L.cout)
        g.update({"g_up1": t(0, 32), "g_up2": t(1, 64), "g_up3": t(2, 128),
                  "g_p0": t(1, 16), "g_p1": t(2, 32), "g_p2": t(3, 64)})
        self.gb = g

    def _dims(self, level: int):
        B, D, H, W = self.shape
        return B, D >> level, H >> level, W >> level

    def _conv(self, L: Conv, a, b, out) -> None:
        o, _, bo, _ = self.lay[L.name]
        B, d, h, w = self._dims(L.level)
        self._call(U.lib().ccu_conv3d, self._ptr(a), L.ca, self._ptr(b) if b is not None else None, L.cb, B, d, h, w,
                   self._ptr(self.w[L.name]), self._ptr(self.p, bo), L.cout, 1, self._ptr(out), L.cout, None, None,
                   self._stream())

    # -- forward ----------------------------------------------------------
    def set_input(self, xlog: np.ndarray | None, density: np.ndarray | None, mat: np.ndarray | None,
                  B: int, S, device_xlog=None, device_density=None, device_mat=None,
                  unc: np.ndarray | None = None) -> None:
        """Input volumes [B, S, S, S], or [B, D, H, W] with S = (D, H, W)
        (host arrays, or device tensors; every side a multiple of 8); unc,
        when given, is the input map's relative standard error (see
        ``uncertainty_channel``)."""
        torch = self.torch
        self._alloc(B, S)
        n0 = int(np.prod(self.shape))
        xl = device_xlog if device_xlog is not None else torch.from_numpy(
            np.ascontiguousarray(xlog, dtype=np.float32).reshape(-1)).to(self.dev, non_blocking=True)
        de = device_density if device_density is not None else torch.from_numpy(
            np.ascontiguousarray(density, dtype=np.float32).reshape(-1) * DENSITY_SCALE).to(self.dev, non_blocking=True)
        ma = device_mat if device_mat is not None else torch.from_numpy(
            np.ascontiguousarray(mat, dtype=np.uint8).reshape(-1)).to(self.dev, non_blocking=True)
        un = None
        if unc is not None:
            un = torch.from_numpy(np.ascontiguousarray(unc, dtype=np.float32).reshape(-1)).to(self.dev,
                                                                                           non_blocking=True)
        self.xlog.copy_(xl)
        self._call(U.lib().ccu_input, self._ptr(self.xlog), self._ptr(de), self._ptr(ma), N_MAT,
                   self._ptr(un) if un is not None else None, n0, self._ptr(self.a["x0"]), self._stream())
        self._keep = (de, ma, un)

    def forward(self, last: bool = True) -> None:
        """All convolutions; `last` = False stops before the final one (d0),
        which predict() runs fused with the head."""
        a, lib, st = self.a, U.lib(), self._stream()
        L = {x.name: x for x in LAYERS}
        self._conv(L["e0a"], a["x0"], None, a["e0a"])
        self._conv(L["e0"], a["e0a"], None, a["e0"])
        B, *S0 = self._dims(0)
        self._call(lib.ccu_avgpool, self._ptr(a["e0"]), B, *S0, 16, self._ptr(a["p0"]), st)
        self._conv(L["e1a"], a["p0"], None, a["e1a"])
        self._conv(L["e1"], a["e1a"], None, a["e1"])
        _, *S1 = self._dims(1)
        self._call(lib.ccu_avgpool, self._ptr(a["e1"]), B, *S1, 32, self._ptr(a["p1"]), st)
        self._conv(L["e2a"], a["p1"], None, a["e2a"])
        self._conv(L["e2"], a["e2a"], None, a["e2"])
        _, *S2 = self._dims(2)
        self._call(lib.ccu_avgpool, self._ptr(a["e2"]), B, *S2, 64, self._ptr(a["p2"]), st)
        self._conv(L["b3a"], a["p2"], None, a["b3a"])
        self._conv(L["b3"], a["b3a"], None, a["b3"])
        self._conv(L["d2a"], a["e2"], a["b3"], a["d2a"])
        self._conv(L["d2"], a["d2a"], None, a["d2"])
        self._conv(L["d1a"], a["e1"], a["d2"], a["d1a"])
        self._conv(L["d1"], a["d1a"], None, a["d1"])
        self._conv(L["d0a"], a["e0"], a["d1"], a["d0a"])
        if last:
            self._conv(L["d0"], a["d0a"], None, a["d0"])

    def _head(self, target=None, weight=None, inv_wsum: float = 0.0, backward: bool = False) -> None:
        n0 = int(np.prod(self.shape))
        ho, _, _, _ = self.lay["head"]
        self._call(U.lib().ccu_head, self._ptr(self.a["d0"]), self._ptr(self.xlog),
                   self._ptr(target) if target is not None else None,
                   self._ptr(weight) if weight is not None else None, self._ptr(self.p, ho), inv_wsum,
                   n0, self._ptr(self.out), self._ptr(self.gb["dz_d0"]) if backward else None,
                   self._ptr(self.g, ho) if backward else None, self._ptr(self.acc) if target is not None else None,
                   self._stream())

    def predict(self) -> "torch.Tensor":
        """Forward pass and head; returns the predicted log map (device).
        The last convolution runs with the head in its epilogue
        (ccu_conv3d_head: the same values as the convolution and ccu_head,
        without storing its activations)."""
        self.forward(last=False)
        L = next(x for x in LAYERS if x.name == "d0")
        _, _, bo, _ = self.lay["d0"]
        ho, _, _, _ = self.lay["head"]
        B, d, h, w = self._dims(0)
        self._call(U.lib().ccu_conv3d_head, self._ptr(self.a["d0a"]), L.cin, B, d, h, w, self._ptr(self.w["d0"]),
                   self._ptr(self.p, bo), self._ptr(self.p, ho), self._ptr(self.xlog), self._ptr(self.out),
                   self._ptr(self.a["d0"]), 0, self._stream())
        return self.out

    # -- backward ---------------------------------------------------------
    def _layer_back(self, L: Conv, a, b, dz, out0=None, mask0=None, out1=None, slices: int | None = None) -> None:
        lib, st = U.lib(), self._stream()
        o, _, bo, _ = self.lay[L.name]
        B, d, h, w = self._dims(L.level)
        n = B * d * h * w
        if slices is None:
            slices = max(1, min(256, n // 2048))
        self._call(lib.ccu_conv3d_wgrad, self._ptr(a), L.ca, self._ptr(b) if b is not None else None, L.cb, B, d, h, w,
                   self._ptr(dz), L.cout, self._ptr(self.g, o), slices, st)
        self._call(lib.ccu_bias_grad, self._ptr(dz), n, L.cout, self._ptr(self.g, bo), st)
        if out0 is not None:
            self._call(lib.ccu_conv3d, self._ptr(dz), L.cout, None, 0, B, d, h, w, self._ptr(self.wt[L.name]), None,
                       L.cin, 0, self._ptr(out0), L.ca, self._ptr(mask0) if mask0 is not None else None,
                       self._ptr(out1) if out1 is not None else None, st)

    def backward(self, target, weight, inv_wsum: float) -> None:
        self._alloc_grads()
        a, g, lib, st = self.a, self.gb, U.lib(), self._stream()
        L = {x.name: x for x in LAYERS}
        self._call(lib.ccu_zero, self._ptr(self.g), self.g.numel() * 4, st)
        self._call(lib.ccu_zero, self._ptr(self.acc), self.acc.numel() * 4, st)
        self._head(target, weight, inv_wsum, backward=True)
        B, *S0 = self._dims(0)
        _, *S1 = self._dims(1)
        _, *S2 = self._dims(2)
        self._layer_back(L["d0"], a["d0a"], None, g["dz_d0"], g["dz_d0a"], a["d0a"])
        self._layer_back(L["d0a"], a["e0"], a["d1"], g["dz_d0a"], g["dz_e0"], a["e0"], g["g_up1"])
        self._call(lib.ccu_up_reduce, self._ptr(g["g_up1"]), self._ptr(a["d1"]), B, *S0, 32,
                   self._ptr(g["dz_d1"]), st)
        self._layer_back(L["d1"], a["d1a"], None, g["dz_d1"], g["dz_d1a"], a["d1a"])
        self._layer_back(L["d1a"], a["e1"], a["d2"], g["dz_d1a"], g["dz_e1"], a["e1"], g["g_up2"])
        self._call(lib.ccu_up_reduce, self._ptr(g["g_up2"]), self._ptr(a["d2"]), B, *S1, 64,
                   self._ptr(g["dz_d2"]), st)
        self._layer_back(L["d2"], a["d2a"], None, g["dz_d2"], g["dz_d2a"], a["d2a"])
        self._layer_back(L["d2a"], a["e2"], a["b3"], g["dz_d2a"], g["dz_e2"], a["e2"], g["g_up3"])
        self._call(lib.ccu_up_reduce, self._ptr(g["g_up3"]), self._ptr(a["b3"]), B, *S2, 128,
                   self._ptr(g["dz_b3"]), st)
        self._layer_back(L["b3"], a["b3a"], None, g["dz_b3"], g["dz_b3a"], a["b3a"])
        self._layer_back(L["b3a"], a["p2"], None, g["dz_b3a"], g["g_p2"], None)
        self._call(lib.ccu_pool_backward, self._ptr(g["g_p2"]), self._ptr(a["e2"]), B, *S2, 64,
                   self._ptr(g["dz_e2"]), st)
        self._layer_back(L["e2"], a["e2a"], None, g["dz_e2"], g["dz_e2a"], a["e2a"])
        self._layer_back(L["e2a"], a["p1"], None, g["dz_e2a"], g["g_p1"], None)
        self._call(lib.ccu_pool_backward, self._ptr(g["g_p1"]), self._ptr(a["e1"]), B, *S1, 32,
                   self._ptr(g["dz_e1"]), st)
        self._layer_back(L["e1"], a["e1a"], None, g["dz_e1"], g["dz_e1a"], a["e1a"])
        self._layer_back(L["e1a"], a["p0"], None, g["dz_e1a"], g["g_p0"], None)
        self._call(lib.ccu_pool_backward, self._ptr(g["g_p0"]), self._ptr(a["e0"]), B, *S0, 16,
                   self._ptr(g["dz_e0"]), st)
        self._layer_back(L["e0"], a["e0a"], None, g["dz_e0"], g["dz_e0a"], a["e0a"])
        self._layer_back(L["e0a"], a["x0"], None, g["dz_e0a"])
    def loss(self) -> float:
        """Loss of the last backward pass (synchronises the stream)."""
        return float(self.acc[0].item())

    def step(self, lr: float, b1: float = 0.9, b2: float = 0.999, eps: float = 1e-8, wd: float = 0.0) -> None:
        self.step_n += 1
        if self.clip_ratio > 0:
            self._call(U.lib().ccu_adam_clipped, self._ptr(self.p), self._ptr(self.g), self._ptr(self.m),
                       self._ptr(self.v), self.p.numel(), lr, b1, b2, eps, self.step_n, wd, self._ptr(self.clip_state),
                       self.clip_ratio, self._stream())
        else:
            self._call(U.lib().ccu_adam, self._ptr(self.p), self._ptr(self.g), self._ptr(self.m), self._ptr(self.v),
                       self.p.numel(), lr, b1, b2, eps, self.step_n, wd, self._stream())
        self.pack()

    def layer_times(self, repeats: int = 3) -> list[dict]:
        """Device time of each convolution of a forward pass on the current
        input (CUDA events around every layer, the last of `repeats`
        passes); FLOPs = 2 x 27 x cin x cout x voxels of the layer's level."""
        torch = self.torch
        rec = []
        conv = self._conv

        def timed(L, a, b, out):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            conv(L, a, b, out)
            e1.record()
            rec.append((L, e0, e1))

        self._conv = timed
        try:
            for _ in range(repeats):
                rec.clear()
                self.forward()
            torch.cuda.synchronize()
        finally:
            del self._conv
        self.check_status()
        out = []
        for L, e0, e1 in rec:
            B, d, h, w = self._dims(L.level)
            ms = e0.elapsed_time(e1)
            flops = 2.0 * 27 * L.cin * L.cout * B * d * h * w
            out.append({"layer": L.name, "level": L.level, "cin": L.cin, "cout": L.cout, "ms": round(ms, 4),
                        "tflops": round(flops / ms / 1e9, 1)})
        return out

    def check_status(self) -> None:
        st = U.status(reset=True)
        if st:
            raise RuntimeError(f"a tensor-core kernel reported status {st:#x} (a bounded wait ran out)")


# ---------------------------------------------------------------------------
# data normalisation
# ---------------------------------------------------------------------------

def kerma_scale(k_in: np.ndarray, inside: np.ndarray) -> float:
    sel = k_in[inside]
    s = float(sel.mean()) if sel.size else 0.0
    return s if s > 0 else float(max(k_in.mean(), 1e-30))


def to_log(k: np.ndarray, s: float) -> np.ndarray:
    return np.log(np.maximum(k, 0.0) / s + EPS).astype(np.float32)


UNC_MAX = 1.5


def uncertainty_channel(rel: np.ndarray) -> np.ndarray:
    """The relative standard error of an input map as a network channel:
    clipped to [0, UNC_MAX], voxels without an estimate (no score, or fewer
    than two batches) at UNC_MAX."""
    r = np.nan_to_num(np.asarray(rel, dtype=np.float64), nan=UNC_MAX, posinf=UNC_MAX)
    return np.clip(r, 0.0, UNC_MAX).astype(np.float32)


def from_log(x: np.ndarray, s: float) -> np.ndarray:
    return (s * (np.exp(x.astype(np.float64)) - EPS)).clip(min=0.0)


# ---------------------------------------------------------------------------
# parameter files
# ---------------------------------------------------------------------------

PRETRAINED = __import__("pathlib").Path(__file__).resolve().parent / "data" / "denoiser_unet64.npz"


def _bf16_bits(x: np.ndarray) -> np.ndarray:
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    return ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint16)


def save_params(path, params: np.ndarray, meta: dict | None = None) -> None:
    """Convolution weights as BF16 (the precision the kernels use), biases
    and head FP32, and a JSON description."""
    import json
    p = np.asarray(params, dtype=np.float32)
    lay = param_layout()
    wmask = np.zeros(p.size, dtype=bool)
    for L in LAYERS:
        o, n, _, _ = lay[L.name]
        wmask[o:o + n] = True
    np.savez_compressed(path, weights_bf16=_bf16_bits(p[wmask]), rest=p[~wmask],
                        meta=np.array(json.dumps(meta or {})), n_params=np.array(p.size))


def load_params(path=None) -> tuple[np.ndarray, dict]:
    """(flat FP32 parameters, description) from save_params; the shipped
    pretrained network by default."""
    import json
    z = np.load(path or PRETRAINED)
    n = int(z["n_params"])
    if n != n_params():
        raise ValueError(f"{path}: {n} parameters, this network has {n_params()}")
    lay = param_layout()
    wmask = np.zeros(n, dtype=bool)
    for L in LAYERS:
        o, m, _, _ = lay[L.name]
        wmask[o:o + m] = True
    p = np.empty(n, dtype=np.float32)
    p[wmask] = (z["weights_bf16"].astype(np.uint32) << 16).view(np.float32)
    p[~wmask] = z["rest"]
    return p, json.loads(str(z["meta"]))


def denoise_kerma(k_in: np.ndarray, rel: np.ndarray, mat: np.ndarray, density: np.ndarray,
                  model: "UNet3D | None" = None, batch: int = 8) -> np.ndarray:
    """Denoised kerma maps from plain Monte Carlo maps.

    k_in: [n, S, S, S] kerma (any unit, per history or total), rel: its
    per-voxel relative standard error (batch statistics), mat: material
    index (air 0, water 1, bone 2, lead 3), density [g/cm^3]; S a multiple
    of 8.  The shipped network (``PRETRAINED``) unless a model is given.
    Returns the denoised maps in the unit of k_in."""
    import torch
    model = model or UNet3D(params=load_params()[0])
    k_in = np.asarray(k_in, dtype=np.float64)
    n, S = k_in.shape[0], k_in.shape[1]
    out = np.empty_like(k_in)
    for b0 in range(0, n, batch):
        idx = list(range(b0, min(b0 + batch, n)))
        inside = [mat[i] != 0 for i in idx]
        scales = [kerma_scale(k_in[i], inside[j]) for j, i in enumerate(idx)]
        x = np.stack([to_log(k_in[i], scales[j]) for j, i in enumerate(idx)])
        model.set_input(x, density[idx], mat[idx], len(idx), S, unc=uncertainty_channel(rel[idx]))
        y = model.predict().cpu().numpy().reshape(len(idx), S, S, S)
        for j, i in enumerate(idx):
            out[i] = from_log(y[j], scales[j])
    torch.cuda.synchronize()
    model.check_status()
    return out
