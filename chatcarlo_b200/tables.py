"""Host-side FP64 tables of the transport path (the table builder).

Restates the table construction of ChatCarlo's ``chatcarlo/materials.py``
and the element-data queries it makes, on top of :mod:`physdata`:

* material resolution and densities        materials.py:34-69, 499
* per-element energy grid with edge brackets materials.py:95-199
* per-element photo/Compton/Rayleigh tables  materials.py:202-262
* compound mixing by mass fraction           materials.py:265-289, 344-355
* mu_en/rho (log-log PCHIP over NIST rows)   materials.py:298-335
* Rayleigh F(Z,q) and cumulative A(x) tables materials.py:375-406
* incoherent S(Z,q) table                     materials.py:483-496
* K-shell fluorescence data                   materials.py:443-480
* H*(10)/fluence coefficients                 dose_coefficients.py:27-42

The grid algorithm and the table layouts have to be the same as the
reference's so that the same energies hit the same interpolation nodes;
the code is this project's own.
"""
from __future__ import annotations

import functools

import numpy as np
from scipy.integrate import cumulative_trapezoid

from . import physdata as pd

XS_GRID_MIN_KEV = 1.0
XS_GRID_MAX_KEV = 150.0
XS_GRID_BASE_N = 2000
EDGE_EPS_REL = 1e-5
EDGE_SCAN_N = 200
EDGE_SCAN_CAP_REL = 0.02
EDGE_SCAN_MARGIN = 0.8
EDGE_JUMP_RATIO_MIN = 1.2
NEAR_THRESHOLD_N = 30
NEAR_THRESHOLD_CAP_REL = 0.05

RAYLEIGH_Q_MAX = 20.0
RAYLEIGH_N = 2000
FLUOR_CUTOFF_KEV = 5.0
HC_KEV_ANGSTROM = pd.HC_KEV_ANGSTROM
KN_MEC2_KEV = 511.0            # the electron rest energy the samplers use (physics.py:34)

# scene.yaml short names -> data-set names (materials.py:34-47); "muscle" is
# an extension: ChatCarlo's list has no entry for it, although it ships its
# mu_en table (materials.py:27).
MATERIAL_ALIASES = {
    "water": "Water, Liquid",
    "air": "Air, Dry (near sea level)",
    "soft_tissue": "Tissue, Soft (ICRP)",
    "bone": "Bone, Cortical (ICRP)",
    "lung": "Lung (ICRP)",
    "pmma": "Polymethyl Methacralate (Lucite, Perspex)",
    "concrete": "Concrete, Portland",
    "lead": "Pb",
    "aluminum": "Al",
    "copper": "Cu",
    "iron": "Fe",
    "lead_glass": "Glass, Lead",
    "muscle": "Muscle, Skeletal (ICRP)",
}
DENSITY_OVERRIDE = {"Pb": 11.35, "Al": 2.699, "Cu": 8.96, "Fe": 7.874}
XAAMDI_FILES = {
    "water": "water", "air": "air", "soft_tissue": "soft_tissue",
    "bone": "bone", "lung": "lung", "muscle": "muscle", "adipose": "adipose",
    "pmma": "pmma", "concrete": "concrete", "lead_glass": "lead_glass",
    "aluminum": "z13_Al", "lead": "z82_Pb", "copper": "z29_Cu",
    "iron": "z26_Fe", "tungsten": "z74_W", "calcium": "z20_Ca",
}


class UnknownMaterialError(ValueError):
    pass


@functools.lru_cache(maxsize=None)
def resolve(material: str) -> tuple[str, float, bool]:
    """Material name -> (data-set name, density g/cm^3, is an element)."""
    name = MATERIAL_ALIASES.get(material.lower().strip(), material)
    if name in DENSITY_OVERRIDE:
        return name, DENSITY_OVERRIDE[name], True
    if name in pd.SYMBOL_TO_Z:
        return name, pd.ELEMENTS[pd.SYMBOL_TO_Z[name]][2], True
    if name in pd.COMPOUND_DENSITY:
        return name, pd.COMPOUND_DENSITY[name], False
    cand = [n for n in pd.COMPOUND_DENSITY if material.lower() in n.lower()][:5]
    raise UnknownMaterialError(
        f"unknown material '{material}'; candidates: {cand or sorted(MATERIAL_ALIASES)}")


def density(material: str) -> float:
    return resolve(material)[1]


@functools.lru_cache(maxsize=None)
def element_composition(material: str) -> tuple[tuple[int, float], ...]:
    name, _, is_elem = resolve(material)
    if is_elem:
        return ((pd.SYMBOL_TO_Z[name], 1.0),)
    return pd.COMPOUND_COMPOSITION[name]


# ---------------------------------------------------------------------------
# per-element energy grid and cross-section tables
# ---------------------------------------------------------------------------

@functools.lru_cache(maxsize=None)
def element_edge_energies_kev(z: int) -> tuple[float, ...]:
    edges = []
    for shell in pd.SHELL_NAMES:
        try:
            e = pd.edge_energy(z, shell)
        except ValueError:
            continue
        if e and XS_GRID_MIN_KEV < e < XS_GRID_MAX_KEV:
            edges.append(float(e))
    return tuple(sorted(set(edges)))


def _photo_scalar(z: int, e: float) -> float:
    return float(pd.cs_photo(z, np.array([float(e)]))[0])


def locate_photo_jump_kev(z: int, nominal_edge_kev: float, window_rel: float) -> float:
    """Coarse scan around the nominal edge, then bisection on the mid value."""
    scan = np.geomspace(nominal_edge_kev * (1 - window_rel),
                        nominal_edge_kev * (1 + window_rel), EDGE_SCAN_N)
    vals = pd.cs_photo(z, scan)      # elementwise, identical to point-by-point calls
    ratios = vals[1:] / np.where(vals[:-1] > 0, vals[:-1], 1e-300)
    i = int(np.argmax(ratios))
    if ratios[i] < EDGE_JUMP_RATIO_MIN:
        return nominal_edge_kev
    a, b = scan[i], scan[i + 1]
    mid_val = (vals[i] + vals[i + 1]) / 2.0
    for _ in range(50):
        m = (a + b) / 2.0
        if _photo_scalar(z, m) < mid_val:
            a = m
        else:
            b = m
    return (a + b) / 2.0


@functools.lru_cache(maxsize=None)
def element_energy_grid_kev(z: int) -> np.ndarray:
    nominal = element_edge_energies_kev(z)
    pts = [np.geomspace(XS_GRID_MIN_KEV, XS_GRID_MAX_KEV, XS_GRID_BASE_N)]
    for i, edge in enumerate(nominal):
        gaps = []
        if i > 0:
            gaps.append((edge - nominal[i - 1]) / edge)
        if i < len(nominal) - 1:
            gaps.append((nominal[i + 1] - edge) / edge)
        window = EDGE_SCAN_CAP_REL
        if gaps:
            window = min(window, min(gaps) * EDGE_SCAN_MARGIN)
        jump = locate_photo_jump_kev(z, edge, window)
        lo = max(XS_GRID_MIN_KEV, jump * (1.0 - EDGE_EPS_REL))
        hi = min(XS_GRID_MAX_KEV, jump * (1.0 + EDGE_EPS_REL))
        pts.append(np.array([lo, hi]))
        cap = min(XS_GRID_MAX_KEV, jump * (1.0 + NEAR_THRESHOLD_CAP_REL))
        if i < len(nominal) - 1:
            cap = min(cap, nominal[i + 1])
        if cap > hi:
            pts.append(np.geomspace(hi, cap, NEAR_THRESHOLD_N))
    return np.unique(np.concatenate(pts))


@functools.lru_cache(maxsize=None)
def element_xs_tables(z: int) -> dict[str, np.ndarray]:
    """log E grid and log cross sections [cm^2/g] evaluated point by point."""
    grid = element_energy_grid_kev(z)
    photo = pd.cs_photo(z, grid)
    compt = pd.cs_compton(z, grid)
    rayl = pd.cs_rayleigh(z, grid)
    return {"log_e": np.log(grid), "photo": np.log(photo), "compt": np.log(compt),
            "rayl": np.log(rayl)}


# ---------------------------------------------------------------------------
# Rayleigh / Compton angular tables, K fluorescence
# ---------------------------------------------------------------------------

@functools.lru_cache(maxsize=None)
def rayleigh_form_factor_table(z: int, q_max: float = RAYLEIGH_Q_MAX, n: int = RAYLEIGH_N):
    q = np.linspace(0.0, q_max, n)
    return q, pd.form_factor(z, q)


@functools.lru_cache(maxsize=None)
def rayleigh_cumulative_table(z: int, q_max: float = RAYLEIGH_Q_MAX, n: int = RAYLEIGH_N):
    q, f = rayleigh_form_factor_table(z, q_max, n)
    x = q ** 2
    return x, cumulative_trapezoid(f ** 2, x, initial=0.0)


@functools.lru_cache(maxsize=None)
def incoherent_sq_table(z: int, q_max: float = RAYLEIGH_Q_MAX, n: int = RAYLEIGH_N):
    q = np.concatenate([[0.0], np.linspace(1e-3, q_max, n - 1)])
    return q, np.concatenate([[0.0], pd.incoherent_function(z, q[1:])])


@functools.lru_cache(maxsize=None)
def fluorescence_k_data(z: int):
    """(K edge keV, omega_K, line energies keV, line probabilities summing to 1)."""
    edge = pd.k_edge_kev(z)
    lines = pd.k_lines(z)
    if not lines:
        return edge, 0.0, np.array([]), np.array([])
    energies = np.array([e for _, e, _ in lines])
    rates = np.array([r for _, _, r in lines])
    return edge, pd.fluorescence_yield_k(z), energies, rates / rates.sum()


def k_shell_probability(z: int, e_kev: float) -> float:
    """CS_Photo_Partial(K)/CS_Photo of the data set: 0 up to the K edge."""
    return pd.k_shell_fraction(z) if e_kev > pd.k_edge_kev(z) else 0.0


# ---------------------------------------------------------------------------
# mu_en and H*(10)
# ---------------------------------------------------------------------------

def muen_key(material: str) -> str:
    key = XAAMDI_FILES.get(material.lower().strip())
    if key is None:
        raise UnknownMaterialError(
            f"no mu_en/rho table for material '{material}'; available: {sorted(XAAMDI_FILES)}")
    return key


def h10_table():
    return pd.h10_table()
