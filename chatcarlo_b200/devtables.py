"""Pack the host FP64 tables of a material set into the engine's descriptors.

For each material the element grids (materials.py:162-199) are merged into
one union energy grid.  Every element's log cross section is piecewise
linear in log E between its own nodes, and the union grid contains all of
them, so sampling it at the union nodes and interpolating linearly again
reproduces the element's own interpolation (materials.py:228-262) exactly.
The material's mass-fraction mix (materials.py:265-289) is stored as the
log of the sums per node.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np
from scipy.interpolate import PchipInterpolator

from . import _native as N
from . import physdata as pd
from . import tables as tb


def element_log_cs(z: int, log_e_query: np.ndarray) -> dict[str, np.ndarray]:
    """log sigma_kind(E) of element z by its own grid (materials.py:228-262)."""
    t = tb.element_xs_tables(z)
    grid = t["log_e"]
    idx = np.clip(np.searchsorted(grid, log_e_query), 1, len(grid) - 1)
    x0, x1 = grid[idx - 1], grid[idx]
    frac = (log_e_query - x0) / (x1 - x0)
    return {k: t[k][idx - 1] + frac * (t[k][idx] - t[k][idx - 1]) for k in ("photo", "compt", "rayl")}


@dataclass
class MaterialTables:
    name: str
    density: float
    zs: np.ndarray
    fractions: np.ndarray
    log_e: np.ndarray
    log_parts: np.ndarray           # (n, 4)
    log_elem: np.ndarray            # (n_el, 3, n)
    log_tally: np.ndarray           # (n, 2) ln(mu_en/rho), ln(h*(10)/Phi)


@dataclass
class ElementTables:
    z: int
    s_over_z: np.ndarray
    ray_x: np.ndarray
    ray_a: np.ndarray
    k_edge: float
    k_prob: float
    omega: float
    line_e: np.ndarray
    line_p: np.ndarray
    emits: bool


def _muen_rows(name: str):
    """NIST rows and PCHIP of mu_en/rho, or None without a bundled table."""
    try:
        key = tb.muen_key(name)
    except tb.UnknownMaterialError:
        return None
    e, _, muen = pd.load_xaamdi(key)
    return e, PchipInterpolator(np.log(e), np.log(muen))


def _refine_for_pchip(grid: np.ndarray, pchip, tol: float = 1e-5, rounds: int = 8) -> np.ndarray:
    """Bisect (in ln E) every interval where linear interpolation of the
    mu_en PCHIP misses its midpoint by more than tol (relative)."""
    for _ in range(rounds):
        le = np.log(grid)
        mid = 0.5 * (le[1:] + le[:-1])
        lin = 0.5 * (pchip(le[1:]) + pchip(le[:-1]))
        bad = np.abs(lin - pchip(mid)) > tol
        if not np.any(bad):
            break
        grid = np.unique(np.concatenate([grid, np.exp(mid[bad])]))
    return grid


def build_material(name: str, need_muen: bool = True) -> MaterialTables:
    comp = tb.element_composition(name)
    zs = np.array([z for z, _ in comp], dtype=np.int32)
    fr = np.array([f for _, f in comp], dtype=float)
    lo, hi = tb.XS_GRID_MIN_KEV, tb.XS_GRID_MAX_KEV
    muen = _muen_rows(name)
    if muen is None and need_muen:
        raise tb.UnknownMaterialError(
            f"no mu_en/rho table for material '{name}'; available: {sorted(tb.XAAMDI_FILES)}")
    he, hv = tb.h10_table()
    parts = [tb.element_energy_grid_kev(int(z)) for z in zs]
    parts.append(he[(he > lo) & (he < hi)])           # h*(10) rows: exact log-log interpolation
    if muen is not None:
        parts.append(muen[0][(muen[0] > lo) & (muen[0] < hi)])
    grid = np.unique(np.concatenate(parts))
    if muen is not None:
        grid = _refine_for_pchip(grid, muen[1])
    log_e = np.log(grid)
    n = len(grid)
    log_elem = np.empty((len(zs), 3, n))
    sums = np.zeros((3, n))
    for i, z in enumerate(zs):
        cs = element_log_cs(int(z), log_e)
        for k, kind in enumerate(("photo", "compt", "rayl")):
            log_elem[i, k] = np.log(fr[i]) + cs[kind]
            sums[k] += fr[i] * np.exp(cs[kind])
    log_parts = np.empty((n, 4))
    log_parts[:, :3] = np.log(sums.T)
    log_parts[:, 3] = np.log(sums.sum(axis=0))
    log_tally = np.zeros((n, 2))
    if muen is not None:
        log_tally[:, 0] = muen[1](log_e)                # materials.py:315-335
    ec = np.clip(grid, he[0], he[-1])                    # dose_coefficients.py:32-42
    log_tally[:, 1] = np.interp(np.log(ec), np.log(he), np.log(hv))
    return MaterialTables(name, tb.density(name), zs, fr, log_e, log_parts, log_elem, log_tally)


def build_element(z: int) -> ElementTables:
    q, s = tb.incoherent_sq_table(z)
    x, a = tb.rayleigh_cumulative_table(z)
    edge, omega, le, lp = tb.fluorescence_k_data(z)
    emits = bool(omega > 0 and le.size > 0 and le.max() >= tb.FLUOR_CUTOFF_KEV)
    return ElementTables(z, s / z, x, a, float(edge), float(pd.k_shell_fraction(z)) if emits else 0.0,
                         float(omega), le, lp, emits)


@dataclass
class TableSet:
    """A material set in engine order plus the ctypes descriptor keeping its buffers alive."""
    names: list
    materials: list
    elements: list
    desc: N.TableDesc = None
    _keep: list = field(default_factory=list)

    def index(self, name: str) -> int:
        return self.names.index(name)


def build_table_set(names: list[str], need_muen: bool = True) -> TableSet:
    mats = [build_material(n, need_muen) for n in names]
    zs = sorted({int(z) for m in mats for z in m.zs})
    elems = [build_element(z) for z in zs]
    ts = TableSet(list(names), mats, elems)
    keep = ts._keep

    def arr(a, dtype=np.float64):
        a = np.ascontiguousarray(a, dtype=dtype)
        keep.append(a)
        return a

    md = (N.MaterialDesc * len(mats))()
    for i, m in enumerate(mats):
        d = md[i]
        d.density = m.density
        d.n_nodes = len(m.log_e)
        d.n_elements = len(m.zs)
        d.log_e = N.dptr(arr(m.log_e))
        d.log_parts = N.dptr(arr(m.log_parts))
        d.log_elem = N.dptr(arr(m.log_elem))
        slots = arr([zs.index(int(z)) for z in m.zs], np.int32)
        d.element_slot = slots.ctypes.data_as(C.POINTER(C.c_int32))
        d.log_tally = N.dptr(arr(m.log_tally))
    ed = (N.ElementDesc * len(elems))()
    for i, e in enumerate(elems):
        d = ed[i]
        d.z = e.z
        d.n_lines = len(e.line_e)
        d.s_over_z = N.dptr(arr(e.s_over_z))
        d.ray_x = N.dptr(arr(e.ray_x))
        d.ray_a = N.dptr(arr(e.ray_a))
        d.k_edge_kev = e.k_edge
        d.k_shell_prob = e.k_prob
        d.omega_k = e.omega
        for k in range(len(e.line_e)):
            d.line_e[k] = float(e.line_e[k])
            d.line_p[k] = float(e.line_p[k])
        d.emits = int(e.emits)
    desc = N.TableDesc()
    desc.n_materials = len(mats)
    desc.n_elements = len(elems)
    desc.materials = md
    desc.elements = ed
    keep.extend([md, ed])
    ts.desc = desc
    return ts
