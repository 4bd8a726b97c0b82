"""Source description for the engine (chatcarlo/source.py, spectrum.py).

The engine samples point-focus rect/cone fields, parallel beams, CT
rotation (continuous or n_angles), the helical shift and the heel effect on
the device (source.py:67-210).  The discrete spectrum is an explicit
``source.spectrum`` list or, without SpekPy, the reference's own Kramers
fallback (spectrum.py:55-62), turned into a Walker alias table by the
engine in FP64.  The heel effect's off-axis bins come from
``heel_spectra_for_source`` (SpekPy, as in spectrum.py:88-129,149-153);
the engine does the fluence rejection and the per-bin energy draw.
"""
from __future__ import annotations

import ctypes as C
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


HEEL_N_BINS = 15           # bins along the heel axis (spectrum.py:85)


def heel_spectra_for_source(src: dict, sid: float, span_cm: float, n_bins: int = HEEL_N_BINS):
    """Off-axis bins of the heel effect (spectrum.py:88-129,149-153): bin
    centres s (cm on the SID plane, s > 0 towards the anode), per-bin
    normalised spectra (energies, weights), relative and absolute fluence.
    Computed with SpekPy exactly as the reference does (one off-axis
    spectrum per bin centre at x = -s); without SpekPy it raises, like the
    reference."""
    try:
        import spekpy
    except ImportError:
        raise RuntimeError("the heel effect needs SpekPy's off-axis spectra (spekpy is not installed)") from None
    kvp, filt = float(src["kvp"]), float(src.get("filtration_mm_al", 2.5))
    angle = float(src.get("anode_angle_deg", 12.0))
    centers = (np.arange(n_bins) + 0.5) / n_bins * 2.0 * span_cm - span_cm
    spectra, flu = [], []
    for s_ in centers:
        sp = spekpy.Spek(kvp=kvp, th=angle, z=float(sid), x=-float(s_))
        sp.filter("Al", filt)
        e_mid, phi = sp.get_spectrum(edges=False)
        w = np.clip(np.asarray(phi, dtype=float), 0.0, None)
        tot = float(w.sum())
        flu.append(float(sp.get_flu()) if tot > 0 else 0.0)
        spectra.append((np.asarray(e_mid, dtype=float), w / tot if tot > 0 else w))
    flu = np.asarray(flu)
    if flu.max() <= 0:
        raise ValueError("heel effect: no bin emits (anode angle and field size)")
    return centers, tuple(spectra), flu / flu.max(), flu


def heel_axis(src: dict, d: np.ndarray, u: np.ndarray, v: np.ndarray) -> tuple[float, float]:
    """The anode direction projected on the beam's (u, v) basis (source.py:42-57)."""
    if src.get("anode_direction") is None:
        raise ValueError("source.anode_direction is required with source.heel_effect")
    a = np.asarray(src["anode_direction"], dtype=float)
    a = a - (a @ d) * d
    norm = np.linalg.norm(a)
    if norm < 1e-9:
        raise ValueError("source.anode_direction is parallel to the beam direction")
    a = a / norm
    return float(a @ u), float(a @ v)


def heel_span(fld: dict, h_u: float, h_v: float) -> float:
    """Half-width of the field along the heel axis at the SID (source.py:60-65)."""
    if fld.get("shape", "rect") == "cone":
        return fld["diameter_cm"] / 2.0
    w, h = fld["size_cm"]
    return abs(h_u) * w / 2.0 + abs(h_v) * h / 2.0


class SourceSpec:
    """Host copy of a source plus the ctypes descriptor for cc_source_create."""

    def __init__(self, src: dict):
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
        self.heel = None
        if src.get("heel_effect"):
            if shape == "parallel":
                raise ValueError("source.field.shape parallel cannot be combined with source.heel_effect")
            h_u, h_v = heel_axis(src, d, u, v)
            span = heel_span(fld, h_u, h_v)
            centers, spectra, rel, _ = heel_spectra_for_source(src, float(fld["sid_cm"]), span)
            hd = N.HeelDesc()
            hd.h_u, hd.h_v, hd.span_cm, hd.n_bins = h_u, h_v, float(span), len(centers)
            self._heel_arrays = [np.ascontiguousarray(centers, dtype=float), np.ascontiguousarray(rel, dtype=float),
                                 np.array([len(e) for e, _ in spectra], dtype=np.int32),
                                 np.ascontiguousarray(np.concatenate([e for e, _ in spectra]), dtype=float),
                                 np.ascontiguousarray(np.concatenate([w for _, w in spectra]), dtype=float)]
            c_, f_, nb_, e_, w_ = self._heel_arrays
            hd.centers, hd.rel_fluence, hd.energies_kev, hd.weights = N.dptr(c_), N.dptr(f_), N.dptr(e_), N.dptr(w_)
            hd.bin_sizes = nb_.ctypes.data_as(C.POINTER(C.c_int32))
            self.heel = hd
            # the bins' spectra replace the source spectrum; the descriptor
            # still carries a valid one (the first bin with fluence)
            first = int(np.flatnonzero(np.asarray(rel) > 0)[0])
            self.energies, self.weights = spectra[first]
        else:
            self.energies, self.weights = spectrum_of(src)
        self.energies = np.ascontiguousarray(self.energies, dtype=float)
        self.weights = np.ascontiguousarray(self.weights, dtype=float)
        desc.n_energies = len(self.energies)
        desc.energies_kev = N.dptr(self.energies)
        desc.weights = N.dptr(self.weights)
        if self.heel is not None:
            desc.heel = C.pointer(self.heel)
        self.desc = desc
        self.src = src
