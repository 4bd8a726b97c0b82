"""Photon interaction data for 1-150 keV, built on the host in FP64.

The NumPy path of ChatCarlo reads its element data from the third-party C
library ``xraylib`` (EPDL97-based; ``chatcarlo/materials.py:18``,
``chatcarlo/physics.py:27``; version unpinned, ``README.md:13``).  That
library is not available to this project, so this module supplies every
quantity the transport path consumes from named sources:

* total mass attenuation mu/rho and mass energy-absorption mu_en/rho:
  the NIST XAAMDI tables (Hubbell & Seltzer, public domain) under
  ``data/nist_xaamdi``; the same files ChatCarlo ships
  (``chatcarlo/data/nist_xaamdi``).  Log-log PCHIP between table rows,
  piecewise per edge-free segment so the absorption edges stay sharp.
* atomic form factor F(Z,x) and incoherent scattering function S(Z,x),
  x = sin(theta/2)/lambda [1/Angstrom]: a screened one-electron model.
  Electron configuration by the Madelung rule, effective charges by
  Slater's rules (J.C. Slater, Phys. Rev. 36, 57 (1930)), every subshell
  represented by the density of its Slater-type orbital
  r^(2n*-2) exp(-2 zeta r), zeta = Z_eff/n*, whose form factor is closed
  form; only its first lobe is kept (zero past the first node).
  F = sum N_i f_i, S = Z - sum N_i f_i^2 (Waller-Hartree without exchange
  terms).  This is exact for hydrogen and gives F(0)=Z, S(0)=0, S(inf)=Z,
  F decreasing and S increasing for every Z.
* coherent and incoherent cross sections: Thomson x F^2 and
  Klein-Nishina x S integrated over angle.
* photoelectric: NIST total minus the two scattering cross sections where
  photoabsorption is at least half of the total, and a power law in E
  fitted to that region above it.  Elements without a bundled NIST
  element table are interpolated linearly in ln Z between bundled
  neighbours at energies scaled by the ratio of K-edge energies.
* absorption-edge energies: the edge rows of the NIST tables.
* K-shell fluorescence: K-shell photoabsorption fraction from the
  photoelectric jump ratio at the K edge, P_K = 1 - 1/J; fluorescence
  yield from the fit of W. Bambynek et al., Rev. Mod. Phys. 44, 716
  (1972), (w/(1-w))^(1/4) = 0.015 + 0.0327 Z - 0.64e-6 Z^3; line energies
  as differences of edge energies (Moseley's law for K-alpha where the
  L edges lie below 1 keV); relative line rates from dipole statistical
  weights with a Kbeta/Kalpha ratio linear in Z.

Every number the GPU engine and the CPU oracle consume comes out of this
module, so both sides always share identical tables.
"""
from __future__ import annotations

import functools
import math
from pathlib import Path

import numpy as np
from scipy.interpolate import PchipInterpolator

DATA_DIR = Path(__file__).resolve().parent / "data"
XAAMDI_DIR = DATA_DIR / "nist_xaamdi"

AVOGADRO = 6.02214076e23
R_E_CM = 2.8179403262e-13          # classical electron radius
MEC2_KEV = 510.99895
HC_KEV_ANGSTROM = 12.3984193       # the hc ChatCarlo uses (physics.py:35)
BOHR_ANGSTROM = 0.529177210903
RYDBERG_KEV = 13.605693122994e-3

# Z -> (symbol, standard atomic weight [g/mol], density of the pure element
# [g/cm^3] as listed by NIST XAAMDI Table 1).
ELEMENTS: dict[int, tuple[str, float, float]] = {
    1: ("H", 1.008, 8.375e-05), 2: ("He", 4.0026, 1.663e-04),
    3: ("Li", 6.94, 0.534), 4: ("Be", 9.0122, 1.848), 5: ("B", 10.81, 2.37),
    6: ("C", 12.011, 2.0), 7: ("N", 14.007, 1.165e-03), 8: ("O", 15.999, 1.332e-03),
    9: ("F", 18.998, 1.580e-03), 10: ("Ne", 20.180, 8.385e-04),
    11: ("Na", 22.990, 0.971), 12: ("Mg", 24.305, 1.74), 13: ("Al", 26.982, 2.699),
    14: ("Si", 28.085, 2.33), 15: ("P", 30.974, 2.2), 16: ("S", 32.06, 2.0),
    17: ("Cl", 35.45, 2.995e-03), 18: ("Ar", 39.948, 1.662e-03),
    19: ("K", 39.098, 0.862), 20: ("Ca", 40.078, 1.55), 22: ("Ti", 47.867, 4.54),
    26: ("Fe", 55.845, 7.874), 29: ("Cu", 63.546, 8.96), 33: ("As", 74.922, 5.73),
    74: ("W", 183.84, 19.3), 82: ("Pb", 207.2, 11.35),
}
SYMBOL_TO_Z = {sym: z for z, (sym, _, _) in ELEMENTS.items()}

# Bundled NIST element tables.
ELEMENT_TABLE_FILES = {1: "z01_H", 6: "z06_C", 7: "z07_N", 8: "z08_O", 13: "z13_Al",
                       20: "z20_Ca", 26: "z26_Fe", 29: "z29_Cu", 74: "z74_W", 82: "z82_Pb"}

# Absorption-edge energies [keV] >= 1 keV, each one an edge row of a bundled
# NIST table (file named beside it; checked by the test suite).
EDGES_KEV: dict[int, dict[str, tuple[float, str]]] = {
    11: {"K": (1.0721, "bone")}, 12: {"K": (1.305, "bone")},
    13: {"K": (1.5596, "z13_Al")}, 14: {"K": (1.8389, "concrete")},
    15: {"K": (2.1455, "bone")}, 16: {"K": (2.472, "bone")},
    17: {"K": (2.8224, "muscle")}, 18: {"K": (3.2029, "air")},
    19: {"K": (3.6074, "muscle")}, 20: {"K": (4.0381, "z20_Ca")},
    22: {"K": (4.9664, "lead_glass")},
    26: {"K": (7.112, "z26_Fe")},
    29: {"K": (8.9789, "z29_Cu"), "L1": (1.0961, "z29_Cu")},
    33: {"K": (11.8667, "lead_glass"), "L1": (1.5265, "lead_glass"),
         "L2": (1.3586, "lead_glass"), "L3": (1.3231, "lead_glass")},
    74: {"K": (69.525, "z74_W"), "L1": (12.0998, "z74_W"), "L2": (11.544, "z74_W"),
         "L3": (10.2068, "z74_W"), "M1": (2.8196, "z74_W"), "M2": (2.5749, "z74_W"),
         "M3": (2.281, "z74_W"), "M4": (1.8716, "z74_W"), "M5": (1.8092, "z74_W")},
    82: {"K": (88.0045, "z82_Pb"), "L1": (15.8608, "z82_Pb"), "L2": (15.2, "z82_Pb"),
         "L3": (13.0352, "z82_Pb"), "M1": (3.8507, "z82_Pb"), "M2": (3.5542, "z82_Pb"),
         "M3": (3.0664, "z82_Pb"), "M4": (2.5856, "z82_Pb"), "M5": (2.484, "z82_Pb")},
}

# Shell order used by the xraylib-style shell constants (K=0, L1..L3, M1..M5, ...).
SHELL_NAMES = ["K", "L1", "L2", "L3", "M1", "M2", "M3", "M4", "M5",
               "N1", "N2", "N3", "N4", "N5", "N6", "N7", "O1", "O2", "O3", "P1"]

# Elements without a bundled element table -> the bundled pair used to
# interpolate / extrapolate the photoelectric cross section in ln Z.
PHOTO_NEIGHBOURS = {11: (13, 20), 12: (13, 20), 14: (13, 20), 15: (13, 20), 16: (13, 20),
                    17: (13, 20), 18: (13, 20), 19: (13, 20), 22: (20, 26), 33: (26, 29)}

# Compounds: ChatCarlo's scene names resolve to these NIST compound names
# (chatcarlo/materials.py:34-47); compositions (Z, mass fraction) and
# densities from the NIST ESTAR material composition data, which is what
# xraylib's NIST compound list carries.  Trace zinc (<= 1e-4 by mass) is
# left out and the remaining fractions renormalised: zinc has no edge row in
# the bundled tables.
NIST_COMPOUNDS: dict[str, tuple[float, tuple[tuple[int, float], ...]]] = {
    "Water, Liquid": (1.0, ((1, 0.111894), (8, 0.888106))),
    "Air, Dry (near sea level)": (1.20479e-03, ((6, 0.000124), (7, 0.755268),
                                                (8, 0.231781), (18, 0.012827))),
    "Tissue, Soft (ICRP)": (1.0, ((1, 0.104472), (6, 0.23219), (7, 0.02488), (8, 0.630238),
                                  (11, 0.00113), (12, 0.00013), (15, 0.00133), (16, 0.00199),
                                  (17, 0.00134), (19, 0.00199), (20, 0.00023), (26, 0.00005))),
    "Bone, Cortical (ICRP)": (1.85, ((1, 0.047234), (6, 0.14433), (7, 0.04199), (8, 0.446096),
                                     (12, 0.0022), (15, 0.10497), (16, 0.00315), (20, 0.20993))),
    "Lung (ICRP)": (1.05, ((1, 0.101278), (6, 0.10231), (7, 0.02865), (8, 0.757072),
                           (11, 0.00184), (12, 0.00073), (15, 0.0008), (16, 0.00225),
                           (17, 0.00266), (19, 0.00194), (20, 0.00009), (26, 0.00037))),
    "Muscle, Skeletal (ICRP)": (1.04, ((1, 0.100637), (6, 0.10783), (7, 0.02768),
                                       (8, 0.754773), (11, 0.00075), (12, 0.00019),
                                       (15, 0.0018), (16, 0.00241), (17, 0.00079),
                                       (19, 0.00302), (20, 0.00003), (26, 0.00004))),
    "Polymethyl Methacralate (Lucite, Perspex)": (1.19, ((1, 0.080538), (6, 0.599848),
                                                         (8, 0.319614))),
    "Concrete, Portland": (2.3, ((1, 0.01), (6, 0.001), (8, 0.529107), (11, 0.016),
                                 (12, 0.002), (13, 0.033872), (14, 0.337021), (19, 0.013),
                                 (20, 0.044), (26, 0.014))),
    "Glass, Lead": (6.22, ((8, 0.156453), (14, 0.080866), (22, 0.008092), (33, 0.002651),
                           (82, 0.751938))),
}


def _normalised(comp):
    tot = sum(f for _, f in comp)
    return tuple((z, f / tot) for z, f in comp)


COMPOUND_COMPOSITION = {k: _normalised(v[1]) for k, v in NIST_COMPOUNDS.items()}
COMPOUND_DENSITY = {k: v[0] for k, v in NIST_COMPOUNDS.items()}


# ----------------------------------------------------------------------------
# NIST XAAMDI tables
# ----------------------------------------------------------------------------

@functools.lru_cache(maxsize=None)
def load_xaamdi(key: str) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """(E_keV, mu/rho, mu_en/rho) rows of one bundled NIST table."""
    path = XAAMDI_DIR / f"{key}.csv"
    data = np.loadtxt(path, delimiter=",", comments="#")
    return data[:, 0], data[:, 1], data[:, 2]


def table_edge_rows(key: str) -> list[float]:
    """Energies at which a NIST table lists an absorption edge (a repeated
    energy within 1e-5 relative: the value below, then the value above)."""
    e, _, _ = load_xaamdi(key)
    return [float(e[i]) for i in range(len(e) - 1) if e[i + 1] / e[i] - 1.0 < 1e-5]


class _SegmentedLogPchip:
    """Log-log PCHIP through table rows, one piece per edge-free segment.

    At an edge energy the value below the edge is returned (E <= edge), the
    value above for E > edge, so the jump sits exactly at the edge row."""

    def __init__(self, e: np.ndarray, y: np.ndarray):
        breaks = [i for i in range(len(e) - 1) if e[i + 1] / e[i] - 1.0 < 1e-5]
        starts = [0] + [i + 1 for i in breaks]
        ends = [i + 1 for i in breaks] + [len(e)]
        self.edges = np.array([e[i] for i in breaks])
        self.pieces = []
        for s, t in zip(starts, ends):
            le, ly = np.log(e[s:t]), np.log(y[s:t])
            if t - s >= 2:
                self.pieces.append((le[0], le[-1], PchipInterpolator(le, ly, extrapolate=True)))
            else:
                self.pieces.append((le[0], le[-1], lambda x, v=ly[0]: np.full_like(x, v)))

    def __call__(self, e_kev) -> np.ndarray:
        e = np.atleast_1d(np.asarray(e_kev, dtype=float))
        seg = np.searchsorted(self.edges, e, side="left")  # E == edge -> lower segment
        out = np.empty_like(e)
        le = np.log(e)
        for k, (_, _, f) in enumerate(self.pieces):
            m = seg == k
            if np.any(m):
                out[m] = f(le[m])
        return np.exp(out)


@functools.lru_cache(maxsize=None)
def _total_interp(key: str) -> _SegmentedLogPchip:
    e, mu, _ = load_xaamdi(key)
    return _SegmentedLogPchip(e, mu)


# ----------------------------------------------------------------------------
# Screened one-electron model: F(Z,x), S(Z,x)
# ----------------------------------------------------------------------------

_MADELUNG = [(1, 0), (2, 0), (2, 1), (3, 0), (3, 1), (4, 0), (3, 2), (4, 1), (5, 0), (4, 2),
             (5, 1), (6, 0), (4, 3), (5, 2), (6, 1), (7, 0), (5, 3), (6, 2), (7, 1)]
_CONFIG_EXCEPTIONS = {24: {(3, 2): 5, (4, 0): 1}, 29: {(3, 2): 10, (4, 0): 1},
                      42: {(4, 2): 5, (5, 0): 1}, 47: {(4, 2): 10, (5, 0): 1},
                      78: {(5, 2): 9, (6, 0): 1}, 79: {(5, 2): 10, (6, 0): 1}}
_N_EFF = {1: 1.0, 2: 2.0, 3: 3.0, 4: 3.7, 5: 4.0, 6: 4.2, 7: 4.4}


@functools.lru_cache(maxsize=None)
def electron_configuration(z: int) -> tuple[tuple[int, int, int], ...]:
    """((n, l, occupancy), ...) by the Madelung filling order."""
    occ: dict[tuple[int, int], int] = {}
    left = z
    for n, l in _MADELUNG:
        if left <= 0:
            break
        k = min(left, 2 * (2 * l + 1))
        occ[(n, l)] = k
        left -= k
    for nl, k in _CONFIG_EXCEPTIONS.get(z, {}).items():
        occ[nl] = k
    return tuple((n, l, k) for (n, l), k in sorted(occ.items()) if k > 0)


def _slater_group(n: int, l: int) -> tuple[int, int]:
    """Slater's grouping (1s)(2s,2p)(3s,3p)(3d)(4s,4p)(4d)(4f)(5s,5p)...;
    sorting the keys (n, 0 for sp / 1 for d / 2 for f) gives Slater's order."""
    return (n, 0) if l <= 1 else (n, l - 1)


@functools.lru_cache(maxsize=None)
def shell_model(z: int) -> tuple[tuple[int, float], ...]:
    """((N_i, zeta_i [1/Angstrom]), ...) per subshell of the screened model."""
    conf = electron_configuration(z)
    groups: dict[tuple[int, int], int] = {}
    for n, l, k in conf:
        groups[_slater_group(n, l)] = groups.get(_slater_group(n, l), 0) + k
    order = sorted(groups)
    out = []
    for n, l, k in conf:
        g = _slater_group(n, l)
        gi = order.index(g)
        s = (groups[g] - 1) * (0.30 if n == 1 else 0.35)
        for gj in order[:gi]:
            cnt = groups[gj]
            if l <= 1 and gj[0] == n - 1:
                s += 0.85 * cnt
            else:
                s += 1.00 * cnt
        z_eff = max(z - s, 0.3)
        ns = _N_EFF[n]
        zeta = z_eff / ns / BOHR_ANGSTROM          # Slater orbital exponent
        out.append((k, ns, zeta))
    return tuple(out)


def _sto_form_factor(ns: float, zeta: float, k: np.ndarray) -> np.ndarray:
    """Form factor of the Slater-type density r^(2ns-2) exp(-2 zeta r):
    sin(m phi) cos^(m+1)(phi) / (m sin phi), m = 2 ns, tan(phi) = k/(2 zeta).
    Only the first lobe is kept (zero beyond the first node), which keeps
    each term non-negative and non-increasing in k."""
    m = 2.0 * ns
    phi = np.arctan(k / (2.0 * zeta))
    with np.errstate(invalid="ignore", divide="ignore"):
        f = np.sin(m * phi) * np.cos(phi) ** (m + 1.0) / (m * np.sin(phi))
    f = np.where(phi < 1e-8, 1.0, f)
    return np.where(phi < np.pi / m, f, 0.0)


def _shell_form_factors(z: int, x: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    x = np.asarray(x, dtype=float)
    k = 4.0 * np.pi * x
    f_sum = np.zeros_like(x)
    f2_sum = np.zeros_like(x)
    for n_i, ns, zeta in shell_model(z):
        f = _sto_form_factor(ns, zeta, k)
        f_sum += n_i * f
        f2_sum += n_i * f * f
    return f_sum, f2_sum


def form_factor(z: int, x) -> np.ndarray:
    """Atomic form factor F(Z, x), x = sin(theta/2)/lambda [1/Angstrom]."""
    return _shell_form_factors(z, x)[0]


def incoherent_function(z: int, x) -> np.ndarray:
    """Incoherent scattering function S(Z, x)."""
    return z - _shell_form_factors(z, x)[1]


# ----------------------------------------------------------------------------
# Cross sections [cm^2/g]
# ----------------------------------------------------------------------------

_GL_X, _GL_W = np.polynomial.legendre.leggauss(16)


def _panel_integral(fn, a: float, b: float, n_panels: int) -> float:
    edges = np.linspace(a, b, n_panels + 1)
    mid = 0.5 * (edges[1:] + edges[:-1])[:, None]
    half = 0.5 * (edges[1:] - edges[:-1])[:, None]
    pts = mid + half * _GL_X[None, :]
    return float(np.sum(fn(pts.ravel()).reshape(pts.shape) * _GL_W[None, :] * half))


@functools.lru_cache(maxsize=None)
def _scatter_atom_tables(z: int) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Coherent and incoherent cross sections per atom [cm^2] on a log grid
    covering 0.3-1000 keV (interpolated log-log in between)."""
    e_grid = np.geomspace(0.3, 1000.0, 400)
    pre = math.pi * R_E_CM ** 2
    # Gauss-Legendre panels on x in [0, x_max(E)] for all energies at once;
    # c = 1 - 2 x^2/x_max^2, dc = -4 x/x_max^2 dx
    n_panels = 48
    u_edges = np.linspace(0.0, 1.0, n_panels + 1)
    mid = 0.5 * (u_edges[1:] + u_edges[:-1])[:, None]
    half = 0.5 * (u_edges[1:] - u_edges[:-1])[:, None]
    u = (mid + half * _GL_X[None, :]).ravel()               # nodes in [0, 1]
    w = (np.broadcast_to(half, (n_panels, _GL_X.size)) * _GL_W[None, :]).ravel()
    xm = (e_grid / HC_KEV_ANGSTROM)[:, None]
    x = xm * u[None, :]
    f, f2 = _shell_form_factors(z, x)
    c = 1.0 - 2.0 * u * u
    jac = 4.0 * u                                            # (4 x / xm^2) dx = 4 u du
    coh = pre * np.sum((1.0 + c * c)[None, :] * f * f * jac[None, :] * w[None, :], axis=1)
    alpha = (e_grid / MEC2_KEV)[:, None]
    eps = 1.0 / (1.0 + alpha * (1.0 - c[None, :]))
    kn = eps * eps * (eps + 1.0 / eps - (1.0 - c * c)[None, :])
    inc = pre * np.sum(kn * (z - f2) * jac[None, :] * w[None, :], axis=1)
    return e_grid, coh, inc


def _atom_to_mass(z: int) -> float:
    return AVOGADRO / ELEMENTS[z][1]


def cs_rayleigh(z: int, e_kev) -> np.ndarray:
    e = np.atleast_1d(np.asarray(e_kev, dtype=float))
    eg, coh, _ = _scatter_atom_tables(z)
    return np.exp(np.interp(np.log(e), np.log(eg), np.log(coh))) * _atom_to_mass(z)


def cs_compton(z: int, e_kev) -> np.ndarray:
    e = np.atleast_1d(np.asarray(e_kev, dtype=float))
    eg, _, inc = _scatter_atom_tables(z)
    return np.exp(np.interp(np.log(e), np.log(eg), np.log(inc))) * _atom_to_mass(z)


_PHOTO_TRUST = 0.5


@functools.lru_cache(maxsize=None)
def _photo_tail(z: int) -> tuple[float, float, float]:
    """(E*, photo(E*), slope): above E* the photoelectric cross section of a
    bundled element is the power law photo(E*) (E/E*)^slope."""
    key = ELEMENT_TABLE_FILES[z]
    tot = _total_interp(key)
    edges = tot.edges
    lo = max(1.0, float(edges[-1]) * (1.0 + 1e-4)) if len(edges) else 1.0
    e = np.geomspace(lo, 150.0, 2000)
    raw = tot(e) - cs_rayleigh(z, e) - cs_compton(z, e)
    ok = raw >= _PHOTO_TRUST * tot(e)
    if np.all(ok):
        e_star = 150.0
    else:
        bad = np.nonzero(~ok)[0][0]
        if bad == 0:
            raise ValueError(f"Z={z}: no photoabsorption-dominated range above the last edge")
        e_star = float(e[bad - 1])
    sel = (e <= e_star) & (e >= e_star / 1.5)
    if sel.sum() < 3:
        sel = e <= e_star
    slope = float(np.polyfit(np.log(e[sel]), np.log(raw[sel]), 1)[0])
    p_star = float(tot(np.array([e_star]))[0] - cs_rayleigh(z, e_star)[0] - cs_compton(z, e_star)[0])
    return e_star, p_star, slope


def _photo_bundled(z: int, e: np.ndarray) -> np.ndarray:
    key = ELEMENT_TABLE_FILES[z]
    e_star, p_star, slope = _photo_tail(z)
    out = np.empty_like(e)
    hi = e > e_star
    lo = ~hi
    resid = _total_interp(key)(e) - cs_rayleigh(z, e) - cs_compton(z, e)
    out[lo] = resid[lo]
    if np.any(hi):
        # keep the NIST total wherever the remainder stays within a factor two
        # of the fitted power law; the power law bounds it otherwise
        tail = p_star * (e[hi] / e_star) ** slope
        out[hi] = np.clip(resid[hi], 0.5 * tail, 2.0 * tail)
    return np.maximum(out, 1e-12)


def k_edge_kev(z: int) -> float:
    """K-shell absorption edge [keV]: a NIST table edge row where the edge lies
    above 1 keV, else the screened-hydrogenic estimate Ry (Z - 1)^2 / (1 - 1/4)^-1."""
    if z in EDGES_KEV and "K" in EDGES_KEV[z]:
        return EDGES_KEV[z]["K"][0]
    # Moseley-type estimate for light elements (K edge below the table range)
    return RYDBERG_KEV * (z - 1) ** 2


def cs_photo(z: int, e_kev) -> np.ndarray:
    e = np.atleast_1d(np.asarray(e_kev, dtype=float))
    if z in ELEMENT_TABLE_FILES:
        return _photo_bundled(z, e)
    if z not in PHOTO_NEIGHBOURS:
        raise ValueError(f"no photoelectric data for Z={z}")
    za, zb = PHOTO_NEIGHBOURS[z]
    kz = k_edge_kev(z)
    vals = []
    for zn in (za, zb):
        scaled = e * k_edge_kev(zn) / kz
        lo = scaled < 1.0
        v = np.empty_like(e)
        if np.any(~lo):
            v[~lo] = _photo_bundled(zn, scaled[~lo])
        if np.any(lo):
            # log-log continuation below the 1 keV table start
            p1, p15 = _photo_bundled(zn, np.array([1.0, 1.5]))
            sl = math.log(p15 / p1) / math.log(1.5)
            v[lo] = p1 * scaled[lo] ** sl
        vals.append(np.log(v / _atom_to_mass(zn)))
    t = (math.log(z) - math.log(za)) / (math.log(zb) - math.log(za))
    return np.exp(vals[0] + t * (vals[1] - vals[0])) * _atom_to_mass(z)


def cs_total(z: int, e_kev) -> np.ndarray:
    return cs_photo(z, e_kev) + cs_compton(z, e_kev) + cs_rayleigh(z, e_kev)


def edge_energy(z: int, shell: str) -> float:
    """Absorption-edge energy [keV]; ValueError where this data set has none."""
    if shell == "K":
        return k_edge_kev(z)
    ed = EDGES_KEV.get(z, {})
    if shell in ed:
        return ed[shell][0]
    raise ValueError(f"no {shell} edge for Z={z}")


# ----------------------------------------------------------------------------
# K-shell fluorescence
# ----------------------------------------------------------------------------

K_LINES = ["KL2", "KL3", "KM2", "KM3", "KN2", "KN3", "KO", "KP"]


def fluorescence_yield_k(z: int) -> float:
    """omega_K from the Bambynek et al. (1972) fit."""
    s = 0.015 + 0.0327 * z - 0.64e-6 * z ** 3
    s4 = s ** 4
    return s4 / (1.0 + s4)


@functools.lru_cache(maxsize=None)
def k_shell_fraction(z: int) -> float:
    """Fraction of photoabsorption above the K edge that ionises the K shell,
    1 - 1/J with J the photoelectric jump ratio across the K edge."""
    ek = k_edge_kev(z)
    below = float(cs_photo(z, np.array([ek]))[0])
    above = float(cs_photo(z, np.array([ek * (1.0 + 1e-9)]))[0])
    if not above > below:
        return 0.0
    return 1.0 - below / above


def _binding_or_none(z: int, shell: str):
    ed = EDGES_KEV.get(z, {})
    return ed[shell][0] if shell in ed else None


@functools.lru_cache(maxsize=None)
def k_lines(z: int) -> tuple[tuple[str, float, float], ...]:
    """((line, energy keV, relative rate), ...) for the eight K lines; rates
    are un-normalised.  Lines with no energy above zero are dropped."""
    ek = k_edge_kev(z)
    l2, l3 = _binding_or_none(z, "L2"), _binding_or_none(z, "L3")
    m1 = _binding_or_none(z, "M1")
    m2, m3 = _binding_or_none(z, "M2"), _binding_or_none(z, "M3")
    if l3 is not None and l2 is not None:
        e_kl3, e_kl2 = ek - l3, ek - l2
    else:
        # Moseley's law for K-alpha; the L doublet is unresolved below 1 keV
        e_kl3 = e_kl2 = 0.75 * RYDBERG_KEV * (z - 1) ** 2
    if m3 is not None and m2 is not None:
        e_km3, e_km2 = ek - m3, ek - m2
    else:
        # M binding energies of these elements lie well below 1 keV
        e_km3 = e_km2 = ek - max(0.0, (ek - e_kl3) / 9.0)
    n_bind = (m1 / 4.0) if m1 is not None else 0.0
    e_kn = ek - n_bind
    # Relative rates.  Anchors: ChatCarlo's documentation records the
    # xraylib branching of lead among KL3/KL2/KM3/KM2 as 51.8/30.8/11.5/6.0 %
    # with those four lines carrying 95.05 % of all K emission
    # (docs/plan_fluorescence.md:211-212, docs/lessons_learned.md:547).
    # Below lead the ratios move linearly in Z towards the non-relativistic
    # statistical weights (1:2 inside each p doublet) reached at Z = 20.
    t = min(max((z - 20) / 62.0, 0.0), 1.0)
    a21 = 0.5 + t * (30.8 / 51.8 - 0.5)            # KL2/KL3
    b31 = 0.5 + t * (6.0 / 11.5 - 0.5)             # KM2/KM3
    kb_ka = 0.12 + t * ((11.5 + 6.0) / (51.8 + 30.8) - 0.12)
    outer = 0.0495 * min(max((z - 30) / 52.0, 0.0), 1.0)   # N, O, P shells
    ka3 = 1.0 / (1.0 + a21)
    kb3 = 1.0 / (1.0 + b31)
    main = 1.0 - outer
    alpha = main / (1.0 + kb_ka)
    beta = main - alpha
    rates = {"KL2": alpha * (1.0 - ka3), "KL3": alpha * ka3,
             "KM2": beta * (1.0 - kb3), "KM3": beta * kb3,
             "KN2": outer * 0.30, "KN3": outer * 0.60, "KO": outer * 0.09, "KP": outer * 0.01}
    energies = {"KL2": e_kl2, "KL3": e_kl3, "KM2": e_km2, "KM3": e_km3,
                "KN2": e_kn, "KN3": e_kn, "KO": ek, "KP": ek}
    out = []
    for name in K_LINES:
        r = rates[name]
        en = energies[name]
        if r > 0 and en > 0:
            out.append((name, float(en), float(r)))
    return tuple(out)


# ----------------------------------------------------------------------------
# mu_en/rho and H*(10)/fluence
# ----------------------------------------------------------------------------

@functools.lru_cache(maxsize=None)
def muen_pchip(key: str) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """(log E nodes, log mu_en nodes, PCHIP node slopes) for a NIST table:
    the Hermite form of scipy's log-log PchipInterpolator over all rows."""
    e, _, muen = load_xaamdi(key)
    p = PchipInterpolator(np.log(e), np.log(muen))
    x = np.log(e)
    y = np.log(muen)
    d = p.derivative()(x)
    return x, y, d


@functools.lru_cache(maxsize=1)
def h10_table() -> tuple[np.ndarray, np.ndarray]:
    data = np.loadtxt(DATA_DIR / "h_star_10" / "photons_icrp74.csv", delimiter=",", comments="#")
    return data[:, 0], data[:, 1]
