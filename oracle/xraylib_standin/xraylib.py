"""Test infrastructure: a module named ``xraylib`` for importing ChatCarlo here.

ChatCarlo's NumPy transport (chatcarlo/materials.py:18, physics.py:27)
imports the third-party C library xraylib, which is absent from this
environment.  This stand-in exposes the part of xraylib's API that
ChatCarlo calls (enumerated from the reference's sources and tests) and
answers every query from ``chatcarlo_b200.physdata`` -- the same data the
GPU engine and the oracle consume.  Placing this directory first on
``sys.path`` lets the unmodified reference modules run as a generator of
golden vectors for the oracle.  Nothing in the product imports it.
"""
from __future__ import annotations

import numpy as np

from chatcarlo_b200 import physdata as _pd
from chatcarlo_b200 import tables as _tb

__version__ = "standin-chatcarlo_b200"

_SHELLS = _pd.SHELL_NAMES
for _i, _name in enumerate(_SHELLS):
    globals()[f"{_name}_SHELL"] = _i

_LINES = _pd.K_LINES
for _i, _name in enumerate(_LINES):
    globals()[f"{_name}_LINE"] = -(_i + 1)


def _z_ok(z):
    z = int(z)
    if z not in _pd.ELEMENTS:
        raise ValueError(f"Z={z} is not covered by this data set")
    return z


def _e_ok(e):
    e = float(e)
    if not e > 0.0:
        raise ValueError("energy must be positive")
    return e


def CS_Photo(z, e):
    return float(_pd.cs_photo(_z_ok(z), np.array([_e_ok(e)]))[0])


def CS_Compt(z, e):
    return float(_pd.cs_compton(_z_ok(z), np.array([_e_ok(e)]))[0])


def CS_Rayl(z, e):
    return float(_pd.cs_rayleigh(_z_ok(z), np.array([_e_ok(e)]))[0])


def CS_Total(z, e):
    return CS_Photo(z, e) + CS_Compt(z, e) + CS_Rayl(z, e)


def CS_Total_CP(name, e):
    data = GetCompoundDataNISTByName(name)
    return sum(w * CS_Total(z, e) for z, w in zip(data["Elements"], data["massFractions"]))


def CS_Photo_Partial(z, shell, e):
    z = _z_ok(z)
    e = _e_ok(e)
    if shell != globals()["K_SHELL"]:
        raise ValueError("only the K shell is tabulated")
    return _tb.k_shell_probability(z, e) * CS_Photo(z, e)


def EdgeEnergy(z, shell):
    z = _z_ok(z)
    return float(_pd.edge_energy(z, _SHELLS[int(shell)]))


def FluorYield(z, shell):
    z = _z_ok(z)
    if shell != globals()["K_SHELL"]:
        raise ValueError("only the K shell is tabulated")
    return float(_pd.fluorescence_yield_k(z))


def _line(z, line):
    z = _z_ok(z)
    name = _LINES[-int(line) - 1]
    for nm, en, rate in _pd.k_lines(z):
        if nm == name:
            return en, rate
    raise ValueError(f"line {name} not available for Z={z}")


def RadRate(z, line):
    en, rate = _line(z, line)
    total = sum(r for _, _, r in _pd.k_lines(int(z)))
    return float(rate / total)


def LineEnergy(z, line):
    return float(_line(z, line)[0])


def FF_Rayl(z, q):
    return float(_pd.form_factor(_z_ok(z), np.array([float(q)]))[0])


def SF_Compt(z, q):
    q = float(q)
    if q <= 0.0:
        raise ValueError("q must be positive")
    return float(_pd.incoherent_function(_z_ok(z), np.array([q]))[0])


def ElementDensity(z):
    return float(_pd.ELEMENTS[_z_ok(z)][2])


def SymbolToAtomicNumber(symbol):
    if symbol not in _pd.SYMBOL_TO_Z:
        raise ValueError(f"unknown element symbol {symbol!r}")
    return _pd.SYMBOL_TO_Z[symbol]


def GetCompoundDataNISTList():
    return list(_pd.COMPOUND_DENSITY)


def GetCompoundDataNISTByName(name):
    if name not in _pd.COMPOUND_DENSITY:
        raise ValueError(f"unknown NIST compound {name!r}")
    comp = _pd.COMPOUND_COMPOSITION[name]
    return {"name": name, "nElements": len(comp), "density": _pd.COMPOUND_DENSITY[name],
            "Elements": [z for z, _ in comp], "massFractions": [w for _, w in comp]}
