"""Test infrastructure: CPU oracle of ChatCarlo's photon-transport path.

A NumPy restatement of the reference algorithm (gakugaku3333/chatcarlo,
chatcarlo/*.py; citations per function) on the element data of
``chatcarlo_b200.tables``.  It consumes random numbers from a
``numpy.random.Generator`` in exactly the reference's order, so that with
the same seed it reproduces the reference's outputs bit for bit; the
golden fixtures under tests/golden (made by running the reference itself
with a stand-in for its data library) pin that.  Only the tests, the smoke
check and the CPU-baseline leg of bench.py use this module: it is the
checker, never the product path.
"""
from __future__ import annotations

import concurrent.futures
import math
from dataclasses import dataclass, field

import numpy as np
from scipy.interpolate import PchipInterpolator

from chatcarlo_b200 import physdata as pd
from chatcarlo_b200 import tables as tb

HC = tb.HC_KEV_ANGSTROM
MEC2 = tb.KN_MEC2_KEV
FLUOR_CUTOFF = tb.FLUOR_CUTOFF_KEV
AXES = {"x": 0, "y": 1, "z": 2}


# ---------------------------------------------------------------------------
# materials (chatcarlo/materials.py)
# ---------------------------------------------------------------------------

def groups(names: np.ndarray):
    """(name, mask) in sorted name order (materials.py:503-513)."""
    for name in sorted(set(names.tolist())):
        yield name, names == name


def _interp_index(z: int, e: np.ndarray):
    """materials.py:228-245."""
    if e.min() < tb.XS_GRID_MIN_KEV or e.max() > tb.XS_GRID_MAX_KEV:
        raise ValueError(f"energy {e.min():.3g}..{e.max():.3g} keV outside the cross-section tables")
    grid = tb.element_xs_tables(z)["log_e"]
    lq = np.log(e)
    idx = np.clip(np.searchsorted(grid, lq), 1, len(grid) - 1)
    x0, x1 = grid[idx - 1], grid[idx]
    return idx, (lq - x0) / (x1 - x0)


def element_cs(z: int, e, kind: str) -> np.ndarray:
    """materials.py:248-253."""
    e = np.atleast_1d(np.asarray(e, dtype=float))
    idx, frac = _interp_index(z, e)
    y = tb.element_xs_tables(z)[kind]
    return np.exp(y[idx - 1] + frac * (y[idx] - y[idx - 1]))


def element_cs_all(z: int, e) -> dict:
    """materials.py:256-262."""
    e = np.atleast_1d(np.asarray(e, dtype=float))
    idx, frac = _interp_index(z, e)
    t = tb.element_xs_tables(z)
    return {k: np.exp(t[k][idx - 1] + frac * (t[k][idx] - t[k][idx - 1])) for k in ("photo", "compt", "rayl")}


def cs_parts(material: str, e) -> dict:
    """materials.py:265-289: element tables mixed by mass fraction."""
    name, _, is_elem = tb.resolve(material)
    e = np.atleast_1d(np.asarray(e, dtype=float))
    if is_elem:
        parts = element_cs_all(pd.SYMBOL_TO_Z[name], e)
    else:
        parts = {k: np.zeros_like(e) for k in ("photo", "compt", "rayl")}
        for z, f in tb.element_composition(material):
            el = element_cs_all(z, e)
            for k in parts:
                parts[k] = parts[k] + f * el[k]
    return {"photoelectric": parts["photo"], "compton": parts["compt"], "rayleigh": parts["rayl"]}


def mu_rho(material: str, e) -> np.ndarray:
    p = cs_parts(material, e)
    return p["photoelectric"] + p["compton"] + p["rayleigh"]


def linear_mu(material: str, e) -> np.ndarray:
    return mu_rho(material, e) * tb.density(material)


_MUEN = {}


def mu_en_rho(material: str, e) -> np.ndarray:
    """materials.py:315-335: log-log PCHIP through the NIST rows."""
    key = tb.muen_key(material)
    et, _, muen = pd.load_xaamdi(key)
    e = np.atleast_1d(np.asarray(e, dtype=float))
    if e.min() < et[0] or e.max() > et[-1]:
        raise ValueError("energy outside the mu_en/rho table")
    f = _MUEN.get(key)
    if f is None:
        f = _MUEN[key] = PchipInterpolator(np.log(et), np.log(muen))
    return np.exp(f(np.log(e)))


def element_weights(material: str, e, kind: str):
    """materials.py:358-440: (Z array, normalised w_i sigma_i(E))."""
    comp = tb.element_composition(material)
    zs = np.array([z for z, _ in comp])
    fr = np.array([f for _, f in comp])
    e = np.atleast_1d(np.asarray(e, dtype=float))
    cs = np.array([element_cs(int(z), e, kind) for z in zs])
    w = fr[:, None] * cs
    tot = w.sum(axis=0, keepdims=True)
    tot = np.where(tot > 0, tot, 1.0)
    return zs, w / tot


def h10_per_fluence(e) -> np.ndarray:
    """dose_coefficients.py:32-42."""
    et, ht = tb.h10_table()
    e = np.atleast_1d(np.asarray(e, dtype=float))
    ec = np.clip(e, et[0], et[-1])
    return np.exp(np.interp(np.log(ec), np.log(et), np.log(ht)))


# ---------------------------------------------------------------------------
# geometry (chatcarlo/geometry.py)
# ---------------------------------------------------------------------------

def _box(o, d, center, size, eps=1e-12):
    """geometry.py:20-42 (slab method)."""
    n = o.shape[0]
    c = np.asarray(center, dtype=float)
    s = np.asarray(size, dtype=float)
    lo, hi = c - s / 2.0, c + s / 2.0
    t_in = np.full(n, -np.inf)
    t_out = np.full(n, np.inf)
    miss = np.zeros(n, dtype=bool)
    for k in range(3):
        dk, ok = d[:, k], o[:, k]
        par = np.abs(dk) < eps
        miss |= par & ((ok < lo[k]) | (ok > hi[k]))
        ds = np.where(par, 1.0, dk)
        ta, tb_ = (lo[k] - ok) / ds, (hi[k] - ok) / ds
        t_in = np.maximum(t_in, np.where(par, -np.inf, np.minimum(ta, tb_)))
        t_out = np.minimum(t_out, np.where(par, np.inf, np.maximum(ta, tb_)))
    hit = (~miss) & (t_in <= t_out)
    return np.where(hit, t_in, np.nan), np.where(hit, t_out, np.nan)


def _sphere(o, d, center, radius):
    """geometry.py:45-54."""
    oc = o - np.asarray(center, dtype=float)
    b = np.einsum("ij,ij->i", oc, d)
    c = np.einsum("ij,ij->i", oc, oc) - radius ** 2
    disc = b * b - c
    hit = disc >= 0
    sq = np.sqrt(np.where(hit, disc, 0.0))
    t1, t2 = -b - sq, -b + sq
    return np.where(hit, np.minimum(t1, t2), np.nan), np.where(hit, np.maximum(t1, t2), np.nan)


def _ellipsoid(o, d, center, semi):
    """Axis-aligned ellipsoid: the project's extension primitive (the
    reference has none), solved like _sphere in coordinates scaled by the
    semi-axes."""
    s = np.asarray(semi, dtype=float)
    u = (o - np.asarray(center, dtype=float)) / s
    v = d / s
    a = np.einsum("ij,ij->i", v, v)
    b = np.einsum("ij,ij->i", u, v)
    c = np.einsum("ij,ij->i", u, u) - 1.0
    disc = b * b - a * c
    hit = disc >= 0
    sq = np.sqrt(np.where(hit, disc, 0.0))
    t1, t2 = (-b - sq) / a, (-b + sq) / a
    return np.where(hit, t1, np.nan), np.where(hit, t2, np.nan)


def _cylinder(o, d, center, radius, height, axis, eps=1e-12):
    """geometry.py:57-99."""
    ai = AXES[axis]
    oi = [k for k in range(3) if k != ai]
    c = np.asarray(center, dtype=float)
    ox, oy = o[:, oi[0]] - c[oi[0]], o[:, oi[1]] - c[oi[1]]
    dx, dy = d[:, oi[0]], d[:, oi[1]]
    a = dx * dx + dy * dy
    b = ox * dx + oy * dy
    cc = ox * ox + oy * oy - radius ** 2
    small = a < eps
    disc = b * b - a * cc
    hit_r = (~small) & (disc >= 0)
    sq = np.sqrt(np.where(hit_r, disc, 0.0))
    asafe = np.where(small, 1.0, a)
    t1, t2 = (-b - sq) / asafe, (-b + sq) / asafe
    ti_r = np.where(hit_r, np.minimum(t1, t2), -np.inf)
    to_r = np.where(hit_r, np.maximum(t1, t2), np.inf)
    inside = small & (cc <= 0)
    ti_r = np.where(inside, -np.inf, ti_r)
    to_r = np.where(inside, np.inf, to_r)
    miss_r = (~hit_r) & (~inside)
    lo, hi = c[ai] - height / 2.0, c[ai] + height / 2.0
    oz, dz = o[:, ai], d[:, ai]
    par = np.abs(dz) < eps
    miss_z = par & ((oz < lo) | (oz > hi))
    dsafe = np.where(par, 1.0, dz)
    ta, tb_ = (lo - oz) / dsafe, (hi - oz) / dsafe
    ti_z = np.where(par, -np.inf, np.minimum(ta, tb_))
    to_z = np.where(par, np.inf, np.maximum(ta, tb_))
    ti = np.maximum(ti_r, ti_z)
    to = np.minimum(to_r, to_z)
    miss = miss_r | miss_z | (ti > to)
    return np.where(miss, np.nan, ti), np.where(miss, np.nan, to)


def _contains(g, p):
    """geometry.py:102-118."""
    c = np.asarray(g["center"], dtype=float)
    if g["shape"] == "box":
        s = np.asarray(g["size_cm"], dtype=float)
        return np.all((p >= c - s / 2) & (p <= c + s / 2), axis=1)
    if g["shape"] == "sphere":
        return np.sum((p - c) ** 2, axis=1) <= g["radius_cm"] ** 2
    if g["shape"] == "ellipsoid":
        return np.sum(((p - c) / np.asarray(g["semi_axes_cm"], dtype=float)) ** 2, axis=1) <= 1.0
    ai = AXES[g.get("axis", "z")]
    oi = [k for k in range(3) if k != ai]
    r2 = (p[:, oi[0]] - c[oi[0]]) ** 2 + (p[:, oi[1]] - c[oi[1]]) ** 2
    return (r2 <= g["radius_cm"] ** 2) & (np.abs(p[:, ai] - c[ai]) <= g["height_cm"] / 2)


class OracleGeometry:
    """geometry.py:121-231."""

    def __init__(self, geoms, background="air", bbox_margin_cm=50.0):
        from chatcarlo_b200.geometry import shape_bbox
        self.geoms = geoms
        self.background = background
        los, his = zip(*(shape_bbox(g) for g in geoms))
        self.bbox_min = np.min(np.stack(los), axis=0) - bbox_margin_cm
        self.bbox_max = np.max(np.stack(his), axis=0) + bbox_margin_cm

    def material_at(self, p):
        mat = np.full(p.shape[0], self.background, dtype=object)
        for g in self.geoms:
            m = _contains(g, p)
            if np.any(m):
                mat[m] = g["material"]
        return mat

    def _hit(self, g, o, d):
        if g["shape"] == "box":
            return _box(o, d, g["center"], g["size_cm"])
        if g["shape"] == "sphere":
            return _sphere(o, d, g["center"], g["radius_cm"])
        if g["shape"] == "ellipsoid":
            return _ellipsoid(o, d, g["center"], g["semi_axes_cm"])
        return _cylinder(o, d, g["center"], g["radius_cm"], g["height_cm"], g.get("axis", "z"))

    def next_boundary(self, o, d, eps=1e-6):
        t_obj = np.full(o.shape[0], np.inf)
        for g in self.geoms:
            for t in self._hit(g, o, d):
                ok = ~np.isnan(t) & (t > eps)
                t_obj = np.where(ok & (t < t_obj), t, t_obj)
        center = (self.bbox_min + self.bbox_max) / 2
        size = self.bbox_max - self.bbox_min
        _, tw = _box(o, d, center, size)
        tw = np.where(np.isnan(tw), np.inf, tw)
        return np.minimum(t_obj, tw), tw <= t_obj


# ---------------------------------------------------------------------------
# physics (chatcarlo/physics.py)
# ---------------------------------------------------------------------------

def _pick(zs, w, r):
    cum = np.cumsum(w, axis=0)
    return zs[np.clip(np.sum(r[None, :] > cum, axis=0), 0, len(zs) - 1)]


def sample_element(materials, energies, rng, kind):
    """physics.py:78-92, 138-152, 223-236 (groups in sorted order)."""
    out = np.empty(len(materials), dtype=int)
    for name, m in groups(materials):
        zs, w = element_weights(name, energies[m], kind)
        out[m] = _pick(zs, w, rng.random(int(np.sum(m))))
    return out


def _kn_trial(alpha, emin, env, rng):
    """physics.py:41-56."""
    x1 = rng.random(len(alpha))
    x2 = rng.random(len(alpha))
    eps = emin + x1 * (1.0 - emin)
    c = 1.0 - (1.0 / eps - 1.0) / alpha
    g = 1.0 / eps + eps - (1.0 - c ** 2)
    return eps, c, x2 * env <= g


def sample_klein_nishina(e, rng):
    """physics.py:59-75."""
    alpha = e / MEC2
    emin = 1.0 / (1.0 + 2.0 * alpha)
    env = 1.0 / emin + emin
    eps = np.empty(len(e))
    cos = np.empty(len(e))
    pend = np.arange(len(e))
    while len(pend):
        ep, cp, acc = _kn_trial(alpha[pend], emin[pend], env[pend], rng)
        eps[pend[acc]] = ep[acc]
        cos[pend[acc]] = cp[acc]
        pend = pend[~acc]
    return eps, cos


def sample_compton_bound(materials, e, rng):
    """physics.py:95-135."""
    z_arr = sample_element(materials, e, rng, "compt")
    alpha = e / MEC2
    emin = 1.0 / (1.0 + 2.0 * alpha)
    env = 1.0 / emin + emin
    eps = np.empty(len(e))
    cos = np.empty(len(e))
    pend = np.arange(len(e))
    while len(pend):
        ep, cp, acc_kn = _kn_trial(alpha[pend], emin[pend], env[pend], rng)
        q = e[pend] * np.sin(np.arccos(np.clip(cp, -1.0, 1.0)) / 2.0) / HC
        zp = z_arr[pend]
        soz = np.empty(len(pend))
        for z in set(zp.tolist()):
            mz = zp == z
            qg, sg = tb.incoherent_sq_table(int(z))
            soz[mz] = np.interp(q[mz], qg, sg) / z
        acc = acc_kn & (rng.random(len(pend)) <= soz)
        eps[pend[acc]] = ep[acc]
        cos[pend[acc]] = cp[acc]
        pend = pend[~acc]
    return eps, cos


def sample_fluorescence(materials, e, rng):
    """physics.py:155-212."""
    z_arr = sample_element(materials, e, rng, "photo")
    n = len(e)
    emit = np.zeros(n, dtype=bool)
    e_line = np.zeros(n)
    for z in set(z_arr.tolist()):
        mz = np.where(z_arr == z)[0]
        edge, omega, le, lp = tb.fluorescence_k_data(int(z))
        if omega <= 0 or le.size == 0 or le.max() < FLUOR_CUTOFF:
            continue
        ez = e[mz]
        above = ez > edge
        if not np.any(above):
            continue
        idx = mz[above]
        k_frac = np.array([tb.k_shell_probability(int(z), float(x)) for x in ez[above]])
        is_k = rng.random(len(idx)) < k_frac
        is_rad = rng.random(len(idx)) < omega
        cand = idx[is_k & is_rad]
        if len(cand) == 0:
            continue
        cum = np.cumsum(lp)
        li = np.clip(np.sum(rng.random(len(cand))[None, :] > cum[:, None], axis=0), 0, len(le) - 1)
        ch = le[li]
        ok = ch >= FLUOR_CUTOFF
        emit[cand[ok]] = True
        e_line[cand[ok]] = ch[ok]
    return emit, e_line


def isotropic_direction(n, rng):
    """physics.py:215-220."""
    c = rng.uniform(-1.0, 1.0, n)
    s = np.sqrt(np.clip(1.0 - c ** 2, 0.0, None))
    phi = rng.uniform(0.0, 2.0 * np.pi, n)
    return np.column_stack([s * np.cos(phi), s * np.sin(phi), c])


def sample_rayleigh_cos_theta(z_arr, e, rng):
    """physics.py:281-351 (A(x) inversion, then (1+c^2)/2 rejection)."""
    cos = np.empty(len(z_arr))
    pend = np.arange(len(z_arr))
    xmax_all = (e / HC) ** 2
    while len(pend):
        zp = z_arr[pend]
        xmax = xmax_all[pend]
        x = np.empty(len(pend))
        for z in sorted(set(zp.tolist())):
            m = zp == z
            xg, ag = tb.rayleigh_cumulative_table(int(z))
            if xmax[m].size and xmax[m].max() > xg[-1]:
                raise ValueError(f"q(E) beyond the Rayleigh table for Z={z}")
            a_cut = np.interp(xmax[m], xg, ag)
            x[m] = np.interp(rng.random(int(np.sum(m))) * a_cut, ag, xg)
        x = np.minimum(x, xmax)
        c = np.clip(1.0 - 2.0 * x / xmax, -1.0, 1.0)
        acc = rng.random(len(pend)) <= (1.0 + c ** 2) / 2.0
        cos[pend[acc]] = c[acc]
        pend = pend[~acc]
    return cos


def sample_rayleigh_cos_theta_uniform(z_arr, e, rng):
    """physics.py:239-278: uniform cos proposal against the 2 Z^2 envelope."""
    cos = np.empty(len(z_arr))
    pend = np.arange(len(z_arr))
    while len(pend):
        zp = z_arr[pend]
        ep = e[pend]
        c = rng.uniform(-1.0, 1.0, len(pend))
        q = ep * np.sin(np.arccos(c) / 2.0) / HC
        f = np.empty(len(pend))
        for z in sorted(set(zp.tolist())):
            m = zp == z
            qg, fg = tb.rayleigh_form_factor_table(int(z))
            f[m] = np.interp(q[m], qg, fg)
        acc = rng.random(len(pend)) * 2.0 * zp.astype(float) ** 2 <= (1.0 + c ** 2) * f ** 2
        cos[pend[acc]] = c[acc]
        pend = pend[~acc]
    return cos


def scatter_direction(d, cos, rng):
    """physics.py:354-367."""
    s = np.sqrt(np.clip(1.0 - cos ** 2, 0.0, None))
    phi = rng.uniform(0.0, 2.0 * np.pi, d.shape[0])
    up = np.where((np.abs(d[:, 2]) < 0.999)[:, None], np.array([0.0, 0.0, 1.0]), np.array([1.0, 0.0, 0.0]))
    u = np.cross(up, d)
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    v = np.cross(d, u)
    nd = (s * np.cos(phi))[:, None] * u + (s * np.sin(phi))[:, None] * v + cos[:, None] * d
    return nd / np.linalg.norm(nd, axis=1, keepdims=True)


# ---------------------------------------------------------------------------
# tallies (chatcarlo/tally.py)
# ---------------------------------------------------------------------------

class OracleGrid:
    """VoxelGrid with snapshot-difference batch statistics (tally.py:27-94)."""

    def __init__(self, origin, shape, voxel_cm, track_uncertainty=False):
        self.origin_cm = np.asarray(origin, dtype=float)
        self.shape = tuple(int(s) for s in shape)
        self.voxel_size_cm = float(voxel_cm)
        self.track_uncertainty = track_uncertainty
        self.kerma_keV = np.zeros(self.shape)
        self.h10_track_pSv_cm3 = np.zeros(self.shape)
        self.kerma_sum2 = np.zeros(self.shape) if track_uncertainty else None
        self.h10_sum2 = np.zeros(self.shape) if track_uncertainty else None
        self.n_batches_hit = np.zeros(self.shape, dtype=np.int32) if track_uncertainty else None
        self.n_batches = 0
        self.n_histories = 0
        self._kprev = None
        self._hprev = None

    @classmethod
    def from_bbox(cls, lo, hi, res, track_uncertainty=False):
        shape = tuple(max(1, int(np.ceil(x / res))) for x in (np.asarray(hi) - np.asarray(lo)))
        return cls(lo, shape, res, track_uncertainty)

    def end_batch(self, n_b):
        if not self.track_uncertainty or n_b <= 0:
            return
        if self._kprev is None:
            self._kprev = np.zeros(self.shape)
            self._hprev = np.zeros(self.shape)
        dk = self.kerma_keV - self._kprev
        dh = self.h10_track_pSv_cm3 - self._hprev
        self.kerma_sum2 += dk ** 2 / n_b
        self.h10_sum2 += dh ** 2 / n_b
        self.n_batches_hit += ((dk != 0) | (dh != 0)).astype(np.int32)
        np.copyto(self._kprev, self.kerma_keV)
        np.copyto(self._hprev, self.h10_track_pSv_cm3)
        self.n_batches += 1
        self.n_histories += n_b

    def voxel_index(self, p):
        idx = np.floor((p - self.origin_cm) / self.voxel_size_cm).astype(int)
        return idx, np.all((idx >= 0) & (idx < np.array(self.shape)), axis=1)


def accumulate_track_length(target, grid, o, d, length, w, rng, substep_cm=None, max_substeps=40):
    """tally.py:248-293: stratified random points per sub-step."""
    n = o.shape[0]
    if n == 0:
        return
    if substep_cm is None:
        substep_cm = grid.voxel_size_cm / 2.0
    nsub = np.clip(np.ceil(length / substep_cm).astype(int), 1, max_substeps)
    mx = int(nsub.max())
    j = np.arange(mx)
    frac = (j[None, :] + rng.random((n, mx))) / nsub[:, None]
    valid = j[None, :] < nsub[:, None]
    pts = o[:, None, :] + d[:, None, :] * (length[:, None] * frac)[:, :, None]
    sw = w * (length / nsub)
    idx, ing = grid.voxel_index(pts.reshape(-1, 3))
    keep = valid.reshape(-1) & ing
    idx = idx[keep]
    wf = np.broadcast_to(sw[:, None], (n, mx)).reshape(-1)[keep]
    if len(idx) == 0:
        return
    np.add.at(target.reshape(-1), np.ravel_multi_index((idx[:, 0], idx[:, 1], idx[:, 2]), grid.shape), wf)


def exact_track_length(target, grid, o, d, length, w):
    """Exact per-voxel overlap length (the expectation of the stratified
    estimator), computed by sorting all voxel-plane crossings of each
    segment; the engine's voxel walk scores the same quantity."""
    for i in range(o.shape[0]):
        p0 = o[i]
        di = d[i]
        L = float(length[i])
        ts = [0.0, L]
        for k in range(3):
            if abs(di[k]) < 1e-300:
                continue
            a = (p0[k] - grid.origin_cm[k]) / grid.voxel_size_cm
            b = (p0[k] + di[k] * L - grid.origin_cm[k]) / grid.voxel_size_cm
            lo, hi = sorted((a, b))
            for m in range(int(math.floor(lo)) + 1, int(math.ceil(hi))):
                ts.append((grid.origin_cm[k] + m * grid.voxel_size_cm - p0[k]) / di[k])
        ts = np.unique(np.clip(np.asarray(ts), 0.0, L))
        mids = 0.5 * (ts[1:] + ts[:-1])
        seg = ts[1:] - ts[:-1]
        pts = p0[None, :] + di[None, :] * mids[:, None]
        idx, ing = grid.voxel_index(pts)
        for (ix, iy, iz), ln, ok in zip(idx, seg, ing):
            if ok and ln > 0:
                target[ix, iy, iz] += w[i] * ln


# ---------------------------------------------------------------------------
# transport (chatcarlo/transport.py)
# ---------------------------------------------------------------------------

@dataclass
class BatchResult:
    n_scatter: np.ndarray
    absorbed: np.ndarray
    escaped: np.ndarray
    final_energy: np.ndarray
    energy_deposited: dict = field(default_factory=dict)
    n_fluorescence: int = 0


def _mu_parts(mat, e):
    """transport.py:34-56."""
    n = len(mat)
    mu = np.zeros(n)
    ph, co, ra = np.zeros(n), np.zeros(n), np.zeros(n)
    for name, m in groups(mat):
        p = cs_parts(name, e[m])
        ph[m], co[m], ra[m] = p["photoelectric"], p["compton"], p["rayleigh"]
        mu[m] = (p["photoelectric"] + p["compton"] + p["rayleigh"]) * tb.density(name)
    return mu, (ph, co, ra)


def _muen_linear(mat, e):
    """transport.py:59-64."""
    out = np.zeros(len(mat))
    for name, m in groups(mat):
        out[m] = mu_en_rho(name, e[m]) * tb.density(name)
    return out


def _deposit(acc, mat, e):
    """transport.py:67-69."""
    for name, m in groups(mat):
        acc[name] = acc.get(name, 0.0) + float(np.sum(e[m]))


def transport_photons(pos, dirv, energy, geometry, rng, grid=None, tally_rng=None,
                      fluorescence_enabled=True, exact_tally=False):
    """transport.py:98-233: the alive-mask event loop."""
    if grid is not None and tally_rng is None and not exact_tally:
        tally_rng = rng.spawn(1)[0]
    n = pos.shape[0]
    alive = np.ones(n, dtype=bool)
    tau = -np.log(rng.random(n))
    nsc = np.zeros(n, dtype=int)
    absd = np.zeros(n, dtype=bool)
    esc = np.zeros(n, dtype=bool)
    dep: dict = {}
    nfl = 0
    while np.any(alive):
        idx = np.where(alive)[0]
        o, d, e = pos[idx], dirv[idx], energy[idx]
        mat = geometry.material_at(o)
        mu, (ph, co, ra) = _mu_parts(mat, e)
        tb_, escape = geometry.next_boundary(o, d)
        mus = np.where(mu > 0, mu, 1e-30)
        tau_b = mu * tb_
        inter = tau[idx] < tau_b
        ds = np.where(inter, tau[idx] / mus, tb_)
        ends = o + d * ds[:, None]
        if grid is not None:
            wk = e * _muen_linear(mat, e)
            wh = h10_per_fluence(e)
            if exact_tally:
                exact_track_length(grid.kerma_keV, grid, o, d, ds, wk)
                exact_track_length(grid.h10_track_pSv_cm3, grid, o, d, ds, wh)
            else:
                accumulate_track_length(grid.kerma_keV, grid, o, d, ds, wk, tally_rng)
                accumulate_track_length(grid.h10_track_pSv_cm3, grid, o, d, ds, wh, tally_rng)
        pos[idx] = ends
        cross = ~inter
        gi = idx[cross]
        tau[gi] -= tau_b[cross]
        pos[gi] += dirv[gi] * 1e-6
        out = idx[cross & escape]
        alive[out] = False
        esc[out] = True
        ii = idx[inter]
        if len(ii):
            mi, ei = mat[inter], e[inter]
            r = rng.random(len(ii))
            tot = ph[inter] + co[inter] + ra[inter]
            tot = np.where(tot > 0, tot, 1.0)
            pp, pc = ph[inter] / tot, co[inter] / tot
            is_p = r < pp
            is_c = (~is_p) & (r < pp + pc)
            is_r = (~is_p) & (~is_c)
            pi = ii[is_p]
            if len(pi):
                mp, ep = mi[is_p], ei[is_p]
                if fluorescence_enabled:
                    emit, el = sample_fluorescence(mp, ep, rng)
                else:
                    emit, el = np.zeros(len(pi), dtype=bool), np.zeros(len(pi))
                _deposit(dep, mp, np.where(emit, ep - el, ep))
                nsc[pi] += 1
                alive[pi[~emit]] = False
                absd[pi[~emit]] = True
                ei_ = pi[emit]
                if len(ei_):
                    nfl += len(ei_)
                    energy[ei_] = el[emit]
                    dirv[ei_] = isotropic_direction(len(ei_), rng)
                    tau[ei_] = -np.log(rng.random(len(ei_)))
            ci = ii[is_c]
            if len(ci):
                ec = ei[is_c]
                eps, cos = sample_compton_bound(mi[is_c], ec, rng)
                en = ec * eps
                _deposit(dep, mi[is_c], ec - en)
                dirv[ci] = scatter_direction(dirv[ci], cos, rng)
                energy[ci] = en
                tau[ci] = -np.log(rng.random(len(ci)))
                nsc[ci] += 1
            ri = ii[is_r]
            if len(ri):
                zr = sample_element(mi[is_r], ei[is_r], rng, "rayl")
                cos = sample_rayleigh_cos_theta(zr, ei[is_r], rng)
                dirv[ri] = scatter_direction(dirv[ri], cos, rng)
                tau[ri] = -np.log(rng.random(len(ri)))
                nsc[ri] += 1
    return BatchResult(nsc, absd, esc, energy, dep, nfl)


# ---------------------------------------------------------------------------
# source (chatcarlo/source.py, spectrum.py)
# ---------------------------------------------------------------------------

ROT_AXES = {"x": np.array([1.0, 0.0, 0.0]), "y": np.array([0.0, 1.0, 0.0]), "z": np.array([0.0, 0.0, 1.0])}


def _rotate(v, axis, ang):
    """source.py:20-25 (Rodrigues)."""
    ca = np.cos(ang)[:, None]
    sa = np.sin(ang)[:, None]
    return v[None, :] * ca + np.cross(axis, v)[None, :] * sa + axis[None, :] * (axis @ v) * (1.0 - ca)


def sample_spectrum(src, n, rng):
    """spectrum.py:73-82 with an explicit spectrum or the Kramers fallback."""
    from chatcarlo_b200.source import spectrum_of
    e, w = spectrum_of(src)
    return e[rng.choice(len(e), size=n, p=w)]


def heel_spectra_for_source(src, sid, span_cm):
    """spectrum.py:149-153: the off-axis bins of the heel effect, which the
    reference computes with SpekPy (spectrum.py:88-129).  SpekPy is absent,
    so this raises like the reference without it; tests replace it with
    fixed bins (centres, per-bin (energies, weights), relative fluence,
    absolute fluence)."""
    raise RuntimeError("the heel effect needs SpekPy's off-axis spectra")


def heel_axis_coeffs(src, d, u, v):
    """source.py:42-57: anode direction projected on the beam's (u, v) basis."""
    a = np.asarray(src["anode_direction"], dtype=float)
    a = a - (a @ d) * d
    norm = np.linalg.norm(a)
    if norm < 1e-9:
        raise ValueError("anode_direction is parallel to the beam direction")
    a = a / norm
    return float(a @ u), float(a @ v)


def heel_span_cm(fld, h_u, h_v):
    """source.py:60-65: half-width of the field along the heel axis at the SID."""
    if fld.get("shape", "rect") == "cone":
        return fld["diameter_cm"] / 2.0
    w, h = fld["size_cm"]
    return abs(h_u) * w / 2.0 + abs(h_v) * h / 2.0


def sample_source_photons(src, n, rng):
    """source.py:67-210, the heel effect included (fluence rejection along
    the heel axis in draws of max(1.8 x missing, 1024), energies from the
    photon's heel bin, source.py:130-149,195-207)."""
    from chatcarlo_b200.source import beam_basis
    pos = np.asarray(src["position"], dtype=float)
    d = np.asarray(src["direction"], dtype=float)
    fld = src["field"]
    sid = fld.get("sid_cm")
    u, v = beam_basis(d)
    rot = src.get("rotation")
    if rot is not None:
        iso = np.asarray(rot["isocenter"], dtype=float)
        ax = ROT_AXES[rot.get("axis", "z")]
        na = rot.get("n_angles")
        if na:
            ang = 2.0 * np.pi * rng.integers(0, int(na), size=n) / int(na)
        else:
            ang = rng.uniform(0.0, 2.0 * np.pi, size=n)
        pa = iso[None, :] + _rotate(pos - iso, ax, ang)
        da, ua, va = _rotate(d, ax, ang), _rotate(u, ax, ang), _rotate(v, ax, ang)
        scan = float(rot.get("scan_length_cm") or 0.0)
        if scan > 0.0:
            pa = pa + ax[None, :] * rng.uniform(-scan / 2.0, scan / 2.0, size=n)[:, None]
        origins = pa
    else:
        pa, da, ua, va = pos, d, u, v
        origins = np.tile(pos, (n, 1))
    shape = fld.get("shape", "rect")
    heel = bool(src.get("heel_effect"))
    if heel:
        h_u, h_v = heel_axis_coeffs(src, d, u, v)
        span = heel_span_cm(fld, h_u, h_v)
        centers, spectra, rel_flu, _ = heel_spectra_for_source(src, float(sid), span)

        def accept(draw):
            kept, got = None, 0
            while got < n:
                m = max(int((n - got) * 1.8), 1024)
                s_, *payload = draw(m)
                keep = rng.random(m) < np.interp(s_, centers, rel_flu)
                cols = [s_[keep]] + [c[keep] for c in payload]
                kept = cols if kept is None else [np.concatenate([a, b]) for a, b in zip(kept, cols)]
                got = len(kept[0])
            return [c[:n] for c in kept]
    if shape == "cone":
        ch = np.cos(math.atan((fld["diameter_cm"] / 2.0) / fld["sid_cm"]))

        def draw_cone(m):
            c = rng.uniform(ch, 1.0, m)
            ph = rng.uniform(0.0, 2.0 * np.pi, m)
            s_ = sid * (np.sqrt(1.0 - c ** 2) / c) * (np.cos(ph) * h_u + np.sin(ph) * h_v) if heel else None
            return s_, c, ph

        if heel:
            s_heel, c, ph = accept(draw_cone)
        else:
            _, c, ph = draw_cone(n)
        s = np.sqrt(1.0 - c ** 2)
        dirs = c[:, None] * da + (s * np.cos(ph))[:, None] * ua + (s * np.sin(ph))[:, None] * va
    elif shape == "parallel":
        w, h = fld["size_cm"]
        su = rng.uniform(-w / 2, w / 2, n)
        sv = rng.uniform(-h / 2, h / 2, n)
        origins = origins + su[:, None] * ua + sv[:, None] * va
        dirs = np.broadcast_to(da, (n, 3)).copy()
    else:
        w, h = fld["size_cm"]

        def draw_rect(m):
            a = rng.uniform(-w / 2, w / 2, m)
            b = rng.uniform(-h / 2, h / 2, m)
            return (a * h_u + b * h_v if heel else None), a, b

        if heel:
            s_heel, su, sv = accept(draw_rect)
        else:
            _, su, sv = draw_rect(n)
        tgt = pa + da * sid + su[:, None] * ua + sv[:, None] * va
        dirs = tgt - origins
        dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    if heel:
        bin_w = 2.0 * span / len(centers)
        bins = np.clip(((s_heel + span) / bin_w).astype(int), 0, len(centers) - 1)
        nz = np.where(rel_flu > 0)[0]
        bins = np.clip(bins, nz.min(), nz.max())
        energies = np.empty(n)
        for b in np.unique(bins):
            m = bins == b
            e_b, w_b = spectra[b]
            energies[m] = e_b[rng.choice(len(e_b), size=int(m.sum()), p=w_b)]
        return origins, dirs, energies
    return origins, dirs, sample_spectrum(src, n, rng)


# ---------------------------------------------------------------------------
# run driver (chatcarlo/transport.py:257-474)
# ---------------------------------------------------------------------------

class Moments:
    """ScalarMoments (tally.py:191-245)."""

    def __init__(self):
        self.sums, self.sum2s, self.n_batches, self.n_histories = {}, {}, 0, 0

    def add_batch(self, vals, n):
        if n <= 0:
            return
        for k in set(self.sums) | set(vals):
            s = vals.get(k, 0.0)
            self.sums[k] = self.sums.get(k, 0.0) + s
            self.sum2s[k] = self.sum2s.get(k, 0.0) + s ** 2 / n
        self.n_batches += 1
        self.n_histories += n

    def merge(self, other):
        for k in set(self.sums) | set(other.sums):
            self.sums[k] = self.sums.get(k, 0.0) + other.sums.get(k, 0.0)
            self.sum2s[k] = self.sum2s.get(k, 0.0) + other.sum2s.get(k, 0.0)
        self.n_batches += other.n_batches
        self.n_histories += other.n_histories


def run_batches(src, geometry, rng, n_hist, batch_size, grid, fluorescence, track_uncertainty=False,
                exact_tally=False):
    """transport.py:257-312."""
    dep, nab, nes, ssum, nfl = {}, 0, 0, 0, 0
    mom = Moments() if track_uncertainty else None
    rem = n_hist
    while rem > 0:
        n = min(batch_size, rem)
        rem -= n
        p, d, e = sample_source_photons(src, n, rng)
        r = transport_photons(p, d, e, geometry, rng, grid=grid, fluorescence_enabled=fluorescence,
                              exact_tally=exact_tally)
        for k, v in r.energy_deposited.items():
            dep[k] = dep.get(k, 0.0) + v
        if track_uncertainty:
            mom.add_batch(r.energy_deposited, n)
        if grid is not None:
            grid.end_batch(n)
        nfl += r.n_fluorescence
        nab += int(np.sum(r.absorbed))
        nes += int(np.sum(r.escaped))
        ssum += int(np.sum(r.n_scatter))
    return {"energy_deposited": dep, "n_absorbed": nab, "n_escaped": nes, "scatter_sum": ssum,
            "n_fluorescence": nfl, "moments": mom}


def _worker(raw, n, seed_seq, batch_size, grid_spec, track_uncertainty, exact_tally):
    rng = np.random.default_rng(seed_seq)
    geom = OracleGeometry(raw["geometry"])
    grid = None
    if grid_spec is not None:
        grid = OracleGrid(grid_spec["origin"], grid_spec["shape"], grid_spec["voxel_cm"], track_uncertainty)
    fl = raw.get("physics", {}).get("fluorescence", True)
    agg = run_batches(raw["source"], geom, rng, n, batch_size, grid, fl, track_uncertainty, exact_tally)
    agg["grid"] = grid
    return agg


def run_transport(raw, n_histories=100_000, seed=None, batch_size=200_000, grid_spec=None,
                  n_workers=1, track_uncertainty=True, exact_tally=False):
    """transport.py:358-474 (serial, or SeedSequence-spawned process workers
    summed in worker order).  ``grid_spec`` = {origin, shape, voxel_cm}."""
    if n_workers <= 1:
        agg = _worker(raw, n_histories, np.random.SeedSequence(seed) if seed is not None else None,
                      batch_size, grid_spec, track_uncertainty, exact_tally)
        return agg
    counts = [n_histories // n_workers] * n_workers
    for i in range(n_histories % n_workers):
        counts[i] += 1
    seqs = np.random.SeedSequence(seed).spawn(n_workers)
    import multiprocessing as mp
    with concurrent.futures.ProcessPoolExecutor(max_workers=n_workers,
                                                mp_context=mp.get_context("spawn")) as pool:
        futs = [pool.submit(_worker, raw, counts[i], seqs[i], batch_size, grid_spec, track_uncertainty,
                            exact_tally) for i in range(n_workers) if counts[i] > 0]
        total = None
        for f in futs:
            r = f.result()
            if total is None:
                total = r
                continue
            for k, v in r["energy_deposited"].items():
                total["energy_deposited"][k] = total["energy_deposited"].get(k, 0.0) + v
            for k in ("n_absorbed", "n_escaped", "scatter_sum", "n_fluorescence"):
                total[k] += r[k]
            if track_uncertainty:
                total["moments"].merge(r["moments"])
            if r["grid"] is not None:
                g, h = total["grid"], r["grid"]
                g.kerma_keV += h.kerma_keV
                g.h10_track_pSv_cm3 += h.h10_track_pSv_cm3
                if g.track_uncertainty:
                    g.kerma_sum2 += h.kerma_sum2
                    g.h10_sum2 += h.h10_sum2
                    g.n_batches_hit += h.n_batches_hit
                    g.n_batches += h.n_batches
                    g.n_histories += h.n_histories
    return total


# ---------------------------------------------------------------------------
# CTDIvol calibration (chatcarlo/ctdi.py)
# ---------------------------------------------------------------------------

def ctdi_per_history_Gy(src, phantom="body", n_histories=200_000, seed=None):
    """ctdi.py:53-100: the PMMA CTDI phantom on the isocentre, a 1 cm grid
    with 2 cm margins, host-sampled batches of 200,000 through
    transport_photons, dose at the chamber positions."""
    from chatcarlo_b200 import tables as tb
    rot = src["rotation"]
    diameter = {"body": 32.0, "head": 16.0}[phantom]
    radius = diameter / 2.0
    g = {"name": f"ctdi_phantom_{phantom}", "shape": "cylinder", "material": "pmma",
         "axis": rot.get("axis", "z"), "radius_cm": radius, "height_cm": 15.0,
         "center": [float(x) for x in rot["isocenter"]]}
    geometry = OracleGeometry([g])
    iso = np.asarray(rot["isocenter"], dtype=float)
    ax = AXES[rot.get("axis", "z")]
    plane = [k for k in range(3) if k != ax]
    lo, hi = iso - radius - 2.0, iso + radius + 2.0
    lo[ax] = iso[ax] - 7.5 - 2.0
    hi[ax] = iso[ax] + 7.5 + 2.0
    grid = OracleGrid.from_bbox(lo, hi, 1.0)
    rng = np.random.default_rng(seed)
    remaining = n_histories
    while remaining > 0:
        n = min(200_000, remaining)
        remaining -= n
        pos, dirv, energy = sample_source_photons(src, n, rng)
        transport_photons(pos, dirv, energy, geometry, rng, grid=grid)
    axes = [grid.origin_cm[k] + (np.arange(grid.shape[k]) + 0.5) * grid.voxel_size_cm for k in range(3)]
    c = np.stack(np.meshgrid(*axes, indexing="ij"), axis=-1)
    mats = geometry.material_at(c.reshape(-1, 3))
    dens = np.array([tb.density(m) for m in mats]).reshape(grid.shape)
    mass_kg = dens * grid.voxel_size_cm ** 3 * 1e-3
    energy_j = grid.kerma_keV * 1e-3 * 1.602176634e-13
    dose = np.divide(energy_j, mass_kg, out=np.zeros_like(energy_j), where=mass_kg > 0) / n_histories
    r = np.sqrt((c[..., plane[0]] - iso[plane[0]]) ** 2 + (c[..., plane[1]] - iso[plane[1]]) ** 2)
    z_ok = np.abs(c[..., ax] - iso[ax]) <= 5.0
    d_center = float(dose[z_ok & (r < 2.0)].mean())
    d_periph = float(dose[z_ok & (r >= radius - 2.0) & (r <= radius - 1.0)].mean())
    return d_center / 3.0 + 2.0 * d_periph / 3.0, d_center, d_periph


# ---------------------------------------------------------------------------
# output maps (chatcarlo/diagnostics.py:16-26, chatcarlo/tally.py:109-175)
# ---------------------------------------------------------------------------

def voxel_centers(origin, shape, voxel_cm):
    """tally.py:109-116: voxel centres in C order, (nx*ny*nz, 3)."""
    axes = [origin[k] + (np.arange(shape[k]) + 0.5) * voxel_cm for k in range(3)]
    g = np.meshgrid(*axes, indexing="ij")
    return np.stack([x.ravel() for x in g], axis=1)


def dose_map_Gy(kerma_keV, origin, voxel_cm, geometry, density_of):
    """diagnostics.py:16-26 with tally.py:118-128: the material at each voxel
    centre gives the density that turns kerma into dose."""
    shape = kerma_keV.shape
    mat = geometry.material_at(voxel_centers(np.asarray(origin, dtype=float), shape, voxel_cm))
    rho = np.array([density_of(m) for m in mat]).reshape(shape)
    mass_kg = rho * voxel_cm ** 3 * 1e-3
    energy_j = kerma_keV * 1e-3 * 1.602176634e-13
    return np.divide(energy_j, mass_kg, out=np.zeros_like(energy_j), where=mass_kg > 0)


def h10_map_pSv(h10_track, voxel_cm):
    """tally.py:130-132."""
    return h10_track / voxel_cm ** 3


def relative_error(T, Q, n_batches, n_histories):
    """tally.py:135-175: R = SEM / (T/N) from batch sums, NaN where T = 0 or
    fewer than two batches."""
    T = np.asarray(T, dtype=float)
    Q = np.asarray(Q, dtype=float)
    if n_batches < 2 or n_histories <= 0:
        return np.full_like(T, np.nan)
    var = np.clip((Q - T ** 2 / n_histories) / (n_batches - 1), 0.0, None)
    sem = np.sqrt(var / n_histories)
    mean = T / n_histories
    with np.errstate(divide="ignore", invalid="ignore"):
        return np.where(mean != 0, sem / mean, np.nan)
