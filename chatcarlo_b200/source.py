"""Source description for the engine (chatcarlo/source.py, spectrum.py).

The engine samples point-focus rect/cone fields, parallel beams, CT
rotation (continuous or n_angles) and the helical shift on the device
(source.py:67-194).  The discrete spectrum is an explicit
``source.spectrum`` list or, without SpekPy, the reference's own Kramers
fallback (spectrum.py:55-62), turned into a Walker alias table by the
engine in FP64.
"""
from __future__ import annotations

import math

import numpy as np

from . import _native as N
from . import tables as tb


def beam_basis(d: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """(u, v) orthonormal to the beam axis d (source.py:28-35)."""
    if abs(d[2]) < 0.999:
        u = np.array([-d[1], d[0], 0.0])
    else:
        u = np.array([1.0, 0.0, 0.0])
    u = u / np.linalg.norm(u)
    return u, np.cross(d, u)


def linear_mu(material: str, energies_kev) -> np.ndarray:
    """mu [1/cm] from the per-element tables mixed by mass fraction."""
    from .devtables import element_log_cs
    e = np.atleast_1d(np.asarray(energies_kev, dtype=float))
    total = np.zeros_like(e)
    for z, f in tb.element_composition(material):
        cs = element_log_cs(int(z), np.log(e))
        total += f * (np.exp(cs["photo"]) + np.exp(cs["compt"]) + np.exp(cs["rayl"]))
    return total * tb.density(material)


def kramers_spectrum(kvp: float, filtration_mm_al: float, n_bins: int | None = 60):
    """Kramers' law with Al attenuation (spectrum.py:55-62); n_bins=None gives
    1 keV bins from 5 keV to kVp."""
    if n_bins is None:
        n_bins = max(1, int(round(kvp - 5.0)))
    e = np.linspace(5.0, kvp, n_bins + 1)
    e_mid = 0.5 * (e[:-1] + e[1:])
    raw = np.clip(e_mid * (kvp - e_mid), 0, None)
    atten = np.exp(-linear_mu("aluminum", e_mid) * filtration_mm_al / 10.0)
    w = raw * atten
    return e_mid, w / w.sum()


def spectrum_of(src: dict) -> tuple[np.ndarray, np.ndarray]:
    spec = src.get("spectrum")
    if spec:
        e = np.array([s["energy_keV"] for s in spec], dtype=float)
        w = np.array([s["weight"] for s in spec], dtype=float)
        return e, w / w.sum()
    return kramers_spectrum(src["kvp"], src.get("filtration_mm_al", 2.5))


class SourceSpec:
    """Host copy of a source plus the ctypes descriptor for cc_source_create."""

    def __init__(self, src: dict):
        if src.get("heel_effect"):
            raise RuntimeError("heel_effect needs SpekPy's off-axis spectra, which are not available")
        d = np.asarray(src["direction"], dtype=float)
        d = d / np.linalg.norm(d)
        u, v = beam_basis(d)
        fld = src["field"]
        shape = fld.get("shape", "rect")
        desc = N.SourceDesc()
        desc.field = {"rect": N.CC_FIELD_RECT, "cone": N.CC_FIELD_CONE,
                      "parallel": N.CC_FIELD_PARALLEL}[shape]
        for k in range(3):
            desc.position[k] = float(src["position"][k])
            desc.direction[k] = float(d[k])
            desc.u[k] = float(u[k])
            desc.v[k] = float(v[k])
        desc.sid_cm = float(fld.get("sid_cm") or 0.0)
        if shape == "cone":
            desc.cos_half_angle = math.cos(math.atan((fld["diameter_cm"] / 2.0) / fld["sid_cm"]))
        else:
            w, h = fld["size_cm"]
            desc.size_u = float(w)
            desc.size_v = float(h)
        rot = src.get("rotation")
        if rot is not None:
            desc.rotation = 1
            desc.rot_axis = {"x": 0, "y": 1, "z": 2}[rot.get("axis", "z")]
            desc.n_angles = int(rot.get("n_angles") or 0)
            for k in range(3):
                desc.isocenter[k] = float(rot["isocenter"][k])
            desc.scan_length_cm = float(rot.get("scan_length_cm") or 0.0)
        self.energies, self.weights = spectrum_of(src)
        self.energies = np.ascontiguousarray(self.energies, dtype=float)
        self.weights = np.ascontiguousarray(self.weights, dtype=float)
        desc.n_energies = len(self.energies)
        desc.energies_kev = N.dptr(self.energies)
        desc.weights = N.dptr(self.weights)
        self.desc = desc
        self.src = src
