"""CPU oracle of the learned denoiser (test infrastructure only).

A NumPy FP64 restatement of the 3D U-Net's forward pass, loss and backward
pass, used by the tests to check the gradients that the tensor-core
kernels of libccunet.so produce.  The reference project has no learned
part, so there is no reference file to cite; the network is the one
defined by ``chatcarlo_b200.denoiser`` (layer list and parameter layout),
and this module computes the same function independently.

With ``bf16=True`` the oracle rounds to BF16 (round to nearest even) at the
points where the device stores BF16 tensors -- input, weights, activations
and activation gradients -- so that the comparison measures the kernels'
arithmetic rather than the storage format; all sums are FP64.
"""
from __future__ import annotations

import numpy as np

from chatcarlo_b200.denoiser import DENSITY_SCALE, HEAD_CH, IN_CH, LAYERS, N_MAT, param_layout


def bf16(x: np.ndarray) -> np.ndarray:
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    f = np.ascontiguousarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def _pad(x):
    return np.pad(x, ((0, 0), (1, 1), (1, 1), (1, 1), (0, 0)))


def _taps():
    for tap in range(27):
        yield tap, tap // 9 - 1, (tap // 3) % 3 - 1, tap % 3 - 1


def _shift(xp, dz, dy, dx, s):
    """View of the padded volume at offset (dz, dy, dx) with the original size."""
    return xp[:, 1 + dz:1 + dz + s[0], 1 + dy:1 + dy + s[1], 1 + dx:1 + dx + s[2], :]


def conv3d(x, w):
    """x [B, D, H, W, Cin], w [27, Cout, Cin] -> [B, D, H, W, Cout] ("same")."""
    xp = _pad(x)
    s = x.shape[1:4]
    y = np.zeros(x.shape[:4] + (w.shape[1],))
    for tap, dz, dy, dx in _taps():
        y += _shift(xp, dz, dy, dx, s) @ w[tap].T
    return y


def conv3d_wgrad(x, dz_out):
    """dW[tap, co, ci] = sum_v dz[v, co] x[v + off(tap), ci]."""
    xp = _pad(x)
    s = x.shape[1:4]
    dw = np.zeros((27, dz_out.shape[-1], x.shape[-1]))
    g = dz_out.reshape(-1, dz_out.shape[-1])
    for tap, dz, dy, dx in _taps():
        dw[tap] = g.T @ _shift(xp, dz, dy, dx, s).reshape(-1, x.shape[-1])
    return dw


def conv3d_dgrad(dz_out, w, cin):
    """dX[u, ci] = sum_{tap, co} dz[u - off(tap), co] w[tap, co, ci]."""
    B, D, H, W, _ = dz_out.shape
    dxp = np.zeros((B, D + 2, H + 2, W + 2, cin))
    for tap, dz, dy, dx in _taps():
        dxp[:, 1 + dz:1 + dz + D, 1 + dy:1 + dy + H, 1 + dx:1 + dx + W, :] += dz_out @ w[tap]
    return dxp[:, 1:-1, 1:-1, 1:-1, :]


def up(x):
    return x.repeat(2, axis=1).repeat(2, axis=2).repeat(2, axis=3)


def pool(x):
    B, D, H, W, C = x.shape
    return x.reshape(B, D // 2, 2, H // 2, 2, W // 2, 2, C).mean(axis=(2, 4, 6))


def up_sum(g):
    B, D, H, W, C = g.shape
    return g.reshape(B, D // 2, 2, H // 2, 2, W // 2, 2, C).sum(axis=(2, 4, 6))


def make_input(xlog, density, mat, unc=None):
    """[B, S, S, S] maps -> [B, S, S, S, 16] network input (before rounding)."""
    x = np.zeros(xlog.shape + (IN_CH,))
    x[..., 0] = xlog
    x[..., 1] = density * DENSITY_SCALE
    for m in range(N_MAT):
        x[..., 2 + m] = (mat == m)
    if unc is not None:
        x[..., 15] = unc
    return x


def loss_and_grads(params, xlog, density, mat, target, weight, bf16_storage=True, tensors=None):
    """Loss and the gradient of every parameter (flat, like ``params``);
    when ``tensors`` is a dict it receives the activations ("a_<name>") and
    activation gradients ("dz_<name>", "g_<name>")."""
    r = bf16 if bf16_storage else (lambda a: np.asarray(a, dtype=np.float64))
    lay = param_layout()
    P = np.asarray(params, dtype=np.float64)
    Ls = {L.name: L for L in LAYERS}
    W = {L.name: r(P[lay[L.name][0]:lay[L.name][0] + lay[L.name][1]]).reshape(27, L.cout, L.cin) for L in LAYERS}
    Bi = {L.name: P[lay[L.name][2]:lay[L.name][2] + L.cout] for L in LAYERS}
    ho = lay["head"][0]
    hw, hb = P[ho:ho + HEAD_CH], P[ho + HEAD_CH]

    def fwd(name, a, b=None):
        x = a if b is None else np.concatenate([a, up(b)], axis=-1)
        return r(np.maximum(conv3d(x, W[name]) + Bi[name], 0.0))

    A = {"x0": r(make_input(xlog, density, mat))}
    A["e0a"] = fwd("e0a", A["x0"]); A["e0"] = fwd("e0", A["e0a"]); A["p0"] = r(pool(A["e0"]))
    A["e1a"] = fwd("e1a", A["p0"]); A["e1"] = fwd("e1", A["e1a"]); A["p1"] = r(pool(A["e1"]))
    A["e2a"] = fwd("e2a", A["p1"]); A["e2"] = fwd("e2", A["e2a"]); A["p2"] = r(pool(A["e2"]))
    A["b3a"] = fwd("b3a", A["p2"]); A["b3"] = fwd("b3", A["b3a"])
    A["d2a"] = fwd("d2a", A["e2"], A["b3"]); A["d2"] = fwd("d2", A["d2a"])
    A["d1a"] = fwd("d1a", A["e1"], A["d2"]); A["d1"] = fwd("d1", A["d1a"])
    A["d0a"] = fwd("d0a", A["e0"], A["d1"]); A["d0"] = fwd("d0", A["d0a"])
    out = xlog + A["d0"] @ hw + hb
    wsum = float(np.sum(weight))
    err = out - target
    loss = float(np.sum(weight * err * err) / wsum)
    dout = 2.0 * weight * err / wsum

    G = np.zeros_like(P)
    G[ho:ho + HEAD_CH] = np.tensordot(dout, A["d0"], axes=(list(range(dout.ndim)), list(range(dout.ndim))))
    G[ho + HEAD_CH] = dout.sum()
    dz = {"d0": r(dout[..., None] * hw * (A["d0"] > 0))}

    def back(name, a, b=None, mask=None, want=True):
        L = Ls[name]
        x = a if b is None else np.concatenate([a, up(b)], axis=-1)
        o, n, bo, bn = lay[name]
        G[o:o + n] = conv3d_wgrad(x, dz[name]).reshape(-1)
        G[bo:bo + bn] = dz[name].reshape(-1, L.cout).sum(axis=0)
        if not want:
            return None, None
        gx = conv3d_dgrad(dz[name], W[name], L.cin)
        ga = gx[..., :L.ca]
        if mask is not None:
            ga = ga * (mask > 0)
        return r(ga), (r(gx[..., L.ca:]) if L.cb else None)

    def up_back(gfull, coarse):
        return r(up_sum(gfull) * (coarse > 0))

    def pool_back(dz_x, gy, x_act):
        return r(dz_x + 0.125 * up(gy) * (x_act > 0))

    dz["d0a"], _ = back("d0", A["d0a"], mask=A["d0a"])
    dz_e0, g_up1 = back("d0a", A["e0"], A["d1"], mask=A["e0"])
    dz["d1"] = up_back(g_up1, A["d1"])
    dz["d1a"], _ = back("d1", A["d1a"], mask=A["d1a"])
    dz_e1, g_up2 = back("d1a", A["e1"], A["d2"], mask=A["e1"])
    dz["d2"] = up_back(g_up2, A["d2"])
    dz["d2a"], _ = back("d2", A["d2a"], mask=A["d2a"])
    dz_e2, g_up3 = back("d2a", A["e2"], A["b3"], mask=A["e2"])
    dz["b3"] = up_back(g_up3, A["b3"])
    dz["b3a"], _ = back("b3", A["b3a"], mask=A["b3a"])
    g_p2, _ = back("b3a", A["p2"])
    dz["e2"] = pool_back(dz_e2, g_p2, A["e2"])
    dz["e2a"], _ = back("e2", A["e2a"], mask=A["e2a"])
    g_p1, _ = back("e2a", A["p1"])
    dz["e1"] = pool_back(dz_e1, g_p1, A["e1"])
    dz["e1a"], _ = back("e1", A["e1a"], mask=A["e1a"])
    g_p0, _ = back("e1a", A["p0"])
    dz["e0"] = pool_back(dz_e0, g_p0, A["e0"])
    dz["e0a"], _ = back("e0", A["e0a"], mask=A["e0a"])
    back("e0a", A["x0"], want=False)
    if tensors is not None:
        tensors.update({"a_" + k: v for k, v in A.items()})
        tensors.update({"dz_" + k: v for k, v in dz.items()})
        tensors.update({"g_up1": g_up1, "g_up2": g_up2, "g_up3": g_up3, "g_p0": g_p0, "g_p1": g_p1, "g_p2": g_p2})
    return loss, G, out
