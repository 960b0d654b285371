"""Mechanism layer: read a kinetics mechanism file and flatten it.

The reference compiles each mechanism into C++ with CEPTR
(PelePhysics/Mechanisms/<model>/mechanism.{H,cpp}, selected at build time by
``Chemistry_Model`` in Exec/Make.PeleLMeX:110).  Here the mechanism is data:
a file in a subset of the Cantera YAML schema is parsed into the flat
``b200chem_mech_desc`` arrays of include/b200chem.h, which both the CUDA
kernels and the CPU oracle consume.

Supported subset: ideal-gas species with NASA-7 two-range thermo; reactions
of type elementary, three-body and falloff (Lindemann, Troe with or without
T2), reversible (``<=>``) or irreversible (``=>``), optional explicit reverse
rate (``reverse-rate-constant``), integer stoichiometric coefficients, at
most four distinct species per side, third-body efficiencies.  Anything else
raises ``MechanismError`` rather than being silently dropped.

All values end up in CGS-mol-K: A in (cm^3/mol)^(order-1)/s, Ea/R in K.
"""
from __future__ import annotations

import ctypes
import hashlib
import math
import re
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np
import yaml

MAX_SLOTS = 4
RXN_ELEMENTARY, RXN_THREEBODY, RXN_LINDEMANN, RXN_TROE = 0, 1, 2, 3
FLAG_REVERSIBLE, FLAG_EXPLICIT_REV, FLAG_TROE_T2 = 1, 2, 4

R_CAL = 1.98720425864083  # cal/mol/K
R_J = 8.31446261815324  # J/mol/K
R_CGS = 8.31446261815324e7  # erg/mol/K
P_ATM_CGS = 1013250.0  # dyn/cm^2

ATOMIC_WEIGHTS = {  # IUPAC standard atomic weights, g/mol
    "H": 1.00794, "C": 12.0107, "O": 15.9994, "N": 14.0067, "AR": 39.948, "Ar": 39.948,
    "HE": 4.002602, "He": 4.002602, "E": 5.48579909e-4,
}


class MechanismError(ValueError):
    pass


@dataclass
class Species:
    name: str
    composition: dict
    mw: float
    tmid: float
    nasa_lo: list
    nasa_hi: list


@dataclass
class Reaction:
    equation: str
    kind: int
    reactants: dict
    products: dict
    reversible: bool
    arr: tuple  # (A, b, Ea/R) in CGS, K
    arr_lo: tuple = (0.0, 0.0, 0.0)
    arr_rev: tuple | None = None
    troe: tuple | None = None  # (alpha, T3, T1, T2 or None)
    efficiencies: dict = field(default_factory=dict)
    default_efficiency: float = 1.0


@dataclass
class Mechanism:
    name: str
    species: list
    reactions: list
    source: str = ""

    @property
    def n_species(self) -> int:
        return len(self.species)

    @property
    def n_reactions(self) -> int:
        return len(self.reactions)

    def index(self, name: str) -> int:
        for i, s in enumerate(self.species):
            if s.name == name:
                return i
        raise KeyError(name)

    @property
    def names(self) -> list:
        return [s.name for s in self.species]

    def mw(self) -> np.ndarray:
        return np.array([s.mw for s in self.species], dtype=np.float64)

    def elements(self) -> list:
        els = []
        for s in self.species:
            for e in s.composition:
                if e not in els:
                    els.append(e)
        return els

    def element_matrix(self) -> np.ndarray:
        """[n_elements, N] atoms of each element in each species."""
        els = self.elements()
        m = np.zeros((len(els), self.n_species))
        for k, s in enumerate(self.species):
            for e, c in s.composition.items():
                m[els.index(e), k] = c
        return m

    def digest(self) -> str:
        """Stable hash of the flattened numerical content (for cache keys)."""
        f = flatten(self)
        h = hashlib.sha256()
        for key in sorted(f.arrays):
            h.update(key.encode())
            h.update(np.ascontiguousarray(f.arrays[key]).tobytes())
        return h.hexdigest()[:16]


# --------------------------------------------------------------------- parse

_UNIT_LENGTH = {"cm": 1.0, "m": 100.0, "mm": 0.1}
_UNIT_QUANTITY = {"mol": 1.0, "kmol": 1000.0, "molec": 1.0 / 6.02214076e23}
_UNIT_EA = {  # factor converting the file's unit to Ea/R in K
    "cal/mol": 1.0 / R_CAL, "kcal/mol": 1000.0 / R_CAL, "J/mol": 1.0 / R_J,
    "kJ/mol": 1000.0 / R_J, "K": 1.0, "J/kmol": 1.0 / (1000.0 * R_J),
}


def _parse_side(text: str) -> dict:
    out: dict = {}
    for tok in text.split(" + "):
        tok = tok.strip()
        if not tok:
            continue
        m = re.match(r"^(\d+(?:\.\d+)?)\s*(\S.*)$", tok)
        if m and not re.match(r"^\d", m.group(2)):
            coef, name = float(m.group(1)), m.group(2).strip()
        else:
            coef, name = 1.0, tok
        out[name] = out.get(name, 0.0) + coef
    return out


def parse_equation(eq: str):
    """Split 'A + B (+M) <=> C (+M)' into (reactants, products, reversible, third)."""
    if "<=>" in eq:
        lhs, rhs = eq.split("<=>")
        rev = True
    elif "=>" in eq:
        lhs, rhs = eq.split("=>")
        rev = False
    elif "=" in eq:
        lhs, rhs = eq.split("=")
        rev = True
    else:
        raise MechanismError(f"cannot parse equation {eq!r}")
    third = None
    for side_name in ("lhs", "rhs"):
        side = lhs if side_name == "lhs" else rhs
        m = re.search(r"\(\+\s*([^)]+)\)", side)
        if m:
            third = "falloff:" + m.group(1).strip()
            side = side[: m.start()] + side[m.end():]
        if side_name == "lhs":
            lhs = side
        else:
            rhs = side
    r = _parse_side(lhs.replace("+", " + "))
    p = _parse_side(rhs.replace("+", " + "))
    for side in (r, p):
        if "M" in side:
            if side["M"] != 1.0:
                raise MechanismError(f"bad third body in {eq!r}")
            del side["M"]
            third = third or "M"
    return r, p, rev, third


def _arrhenius(d, order: float, ulen: float, uqty: float, uea: float) -> tuple:
    if isinstance(d, dict):
        A, b, Ea = float(d["A"]), float(d.get("b", 0.0)), float(d.get("Ea", 0.0))
    else:
        A, b, Ea = (float(v) for v in d)
    # concentration unit conversion: (length^3/quantity)^(order-1)
    conv = (ulen ** 3 / uqty) ** (order - 1.0)
    return (A * conv, b, Ea * uea)


def load(path, name: str | None = None) -> Mechanism:
    """Parse a mechanism file (Cantera YAML subset) into a Mechanism."""
    path = Path(path)
    doc = yaml.safe_load(path.read_text())
    units = doc.get("units", {})  # Cantera defaults: m, kmol, J/kmol
    ulen = _UNIT_LENGTH[units.get("length", "m")]
    uqty = _UNIT_QUANTITY[units.get("quantity", "kmol")]
    uea = _UNIT_EA[units.get("activation-energy", "J/kmol")]
    phase_species = None
    if "phases" in doc and doc["phases"]:
        ph = doc["phases"][0]
        if isinstance(ph.get("species"), list) and ph["species"] and isinstance(ph["species"][0], str):
            phase_species = ph["species"]
    species = []
    sp_by_name = {}
    for s in doc["species"]:
        th = s["thermo"]
        if th.get("model", "NASA7") != "NASA7":
            raise MechanismError(f"species {s['name']}: only NASA7 thermo is supported")
        tr = [float(x) for x in th["temperature-ranges"]]
        data = th["data"]
        if len(data) == 1:
            lo = hi = [float(x) for x in data[0]]
            tmid = tr[-1]
        elif len(data) == 2 and len(tr) == 3:
            lo, hi = [float(x) for x in data[0]], [float(x) for x in data[1]]
            tmid = tr[1]
        else:
            raise MechanismError(f"species {s['name']}: 1 or 2 NASA7 ranges expected")
        comp = {str(k): float(v) for k, v in s["composition"].items()}
        mw = sum(ATOMIC_WEIGHTS[e] * c for e, c in comp.items())
        sp = Species(s["name"], comp, mw, tmid, lo, hi)
        sp_by_name[sp.name] = sp
        species.append(sp)
    if phase_species is not None:
        species = [sp_by_name[n] for n in phase_species]
    names = {s.name for s in species}
    reactions = []
    for rd in doc.get("reactions", []):
        eq = rd["equation"]
        r, p, rev, third = parse_equation(eq)
        for side in (r, p):
            for nm, c in side.items():
                if nm not in names:
                    raise MechanismError(f"{eq}: unknown species {nm}")
                if c != int(c):
                    raise MechanismError(f"{eq}: non-integer stoichiometry not supported")
            if len(side) > MAX_SLOTS:
                raise MechanismError(f"{eq}: more than {MAX_SLOTS} species on a side")
        rtype = rd.get("type", "elementary")
        order_f = sum(r.values())
        eff = {str(k): float(v) for k, v in rd.get("efficiencies", {}).items()}
        defeff = float(rd.get("default-efficiency", 1.0))
        if defeff != 1.0:
            raise MechanismError(f"{eq}: default-efficiency != 1 not supported")
        for k in eff:
            if k not in names:
                raise MechanismError(f"{eq}: efficiency for unknown species {k}")
        if rd.get("orders") or rd.get("negative-orders") or rd.get("nonreactant-orders"):
            raise MechanismError(f"{eq}: explicit reaction orders not supported")
        if rd.get("duplicate") is not None and not isinstance(rd.get("duplicate"), bool):
            raise MechanismError(f"{eq}: bad duplicate flag")
        if rtype in ("elementary", "three-body"):
            if rtype == "three-body" or third == "M":
                kind = RXN_THREEBODY
                arr = _arrhenius(rd["rate-constant"], order_f + 1, ulen, uqty, uea)
            else:
                kind = RXN_ELEMENTARY
                arr = _arrhenius(rd["rate-constant"], order_f, ulen, uqty, uea)
            rxn = Reaction(eq, kind, r, p, rev, arr, efficiencies=eff)
            if kind == RXN_ELEMENTARY and eff:
                raise MechanismError(f"{eq}: efficiencies on an elementary reaction")
        elif rtype == "falloff":
            if third is None or not third.startswith("falloff:"):
                raise MechanismError(f"{eq}: falloff needs (+M)")
            if third != "falloff:M":
                raise MechanismError(f"{eq}: specific falloff collider not supported")
            hi = _arrhenius(rd["high-P-rate-constant"], order_f, ulen, uqty, uea)
            lo = _arrhenius(rd["low-P-rate-constant"], order_f + 1, ulen, uqty, uea)
            if "Troe" in rd:
                t = rd["Troe"]
                troe = (float(t["A"]), float(t["T3"]), float(t["T1"]),
                        float(t["T2"]) if "T2" in t else None)
                kind = RXN_TROE
            elif "SRI" in rd:
                raise MechanismError(f"{eq}: SRI falloff not supported")
            else:
                troe = None
                kind = RXN_LINDEMANN
            rxn = Reaction(eq, kind, r, p, rev, hi, arr_lo=lo, troe=troe, efficiencies=eff)
        else:
            raise MechanismError(f"{eq}: reaction type {rtype!r} not supported")
        if "reverse-rate-constant" in rd:
            if kind != RXN_ELEMENTARY:
                raise MechanismError(f"{eq}: explicit reverse only for elementary reactions")
            rxn.arr_rev = _arrhenius(rd["reverse-rate-constant"], sum(p.values()), ulen, uqty, uea)
        reactions.append(rxn)
    return Mechanism(name or path.stem, species, reactions, source=str(path))


# ------------------------------------------------------------------ flatten

@dataclass
class FlatMechanism:
    n_species: int
    n_reactions: int
    n_eff: int
    arrays: dict

    def ctypes_desc(self):
        """A b200chem_mech_desc pointing into this object's arrays (keep self alive)."""
        d = MechDesc()
        d.n_species = self.n_species
        d.n_reactions = self.n_reactions
        d.n_eff = self.n_eff
        for key, ct in _DESC_FIELDS:
            arr = self.arrays[key]
            setattr(d, key, arr.ctypes.data_as(ctypes.POINTER(ct)))
        return d


class MechDesc(ctypes.Structure):
    _fields_ = [
        ("n_species", ctypes.c_int32), ("n_reactions", ctypes.c_int32), ("n_eff", ctypes.c_int32),
        ("mw", ctypes.POINTER(ctypes.c_double)), ("nasa", ctypes.POINTER(ctypes.c_double)),
        ("rtype", ctypes.POINTER(ctypes.c_int32)), ("rflags", ctypes.POINTER(ctypes.c_int32)),
        ("arr", ctypes.POINTER(ctypes.c_double)), ("arr_lo", ctypes.POINTER(ctypes.c_double)),
        ("arr_rev", ctypes.POINTER(ctypes.c_double)), ("troe", ctypes.POINTER(ctypes.c_double)),
        ("sp", ctypes.POINTER(ctypes.c_int32)), ("nu", ctypes.POINTER(ctypes.c_int32)),
        ("eff_ptr", ctypes.POINTER(ctypes.c_int32)), ("eff_sp", ctypes.POINTER(ctypes.c_int32)),
        ("eff_val", ctypes.POINTER(ctypes.c_double)),
    ]


_DESC_FIELDS = [
    ("mw", ctypes.c_double), ("nasa", ctypes.c_double), ("rtype", ctypes.c_int32),
    ("rflags", ctypes.c_int32), ("arr", ctypes.c_double), ("arr_lo", ctypes.c_double),
    ("arr_rev", ctypes.c_double), ("troe", ctypes.c_double), ("sp", ctypes.c_int32),
    ("nu", ctypes.c_int32), ("eff_ptr", ctypes.c_int32), ("eff_sp", ctypes.c_int32),
    ("eff_val", ctypes.c_double),
]


def _lnA(A: float) -> float:
    if A <= 0.0:
        raise MechanismError("pre-exponential factor must be positive")
    return math.log(A)


def flatten(mech: Mechanism) -> FlatMechanism:
    """Mechanism -> flat arrays in the b200chem_mech_desc layout."""
    N, R = mech.n_species, mech.n_reactions
    idx = {s.name: i for i, s in enumerate(mech.species)}
    mw = np.array([s.mw for s in mech.species], dtype=np.float64)
    nasa = np.zeros((N, 15))
    for k, s in enumerate(mech.species):
        nasa[k, 0] = s.tmid
        nasa[k, 1:8] = s.nasa_lo
        nasa[k, 8:15] = s.nasa_hi
    rtype = np.zeros(R, np.int32)
    rflags = np.zeros(R, np.int32)
    arr = np.zeros((R, 3))
    arr_lo = np.zeros((R, 3))
    arr_rev = np.zeros((R, 3))
    troe = np.zeros((R, 4))
    sp = -np.ones((R, 8), np.int32)
    nu = np.zeros((R, 8), np.int32)
    eff_ptr = np.zeros(R + 1, np.int32)
    eff_sp, eff_val = [], []
    for j, rx in enumerate(mech.reactions):
        rtype[j] = rx.kind
        f = FLAG_REVERSIBLE if rx.reversible else 0
        arr[j] = (_lnA(rx.arr[0]), rx.arr[1], rx.arr[2])
        if rx.kind in (RXN_LINDEMANN, RXN_TROE):
            arr_lo[j] = (_lnA(rx.arr_lo[0]), rx.arr_lo[1], rx.arr_lo[2])
        if rx.arr_rev is not None:
            f |= FLAG_EXPLICIT_REV
            arr_rev[j] = (_lnA(rx.arr_rev[0]), rx.arr_rev[1], rx.arr_rev[2])
        if rx.troe is not None:
            a, t3, t1, t2 = rx.troe
            troe[j] = (a, t3, t1, t2 if t2 is not None else 0.0)
            if t2 is not None:
                f |= FLAG_TROE_T2
        rflags[j] = f
        for s_i, (nm, c) in enumerate(rx.reactants.items()):
            sp[j, s_i], nu[j, s_i] = idx[nm], int(c)
        for s_i, (nm, c) in enumerate(rx.products.items()):
            sp[j, 4 + s_i], nu[j, 4 + s_i] = idx[nm], int(c)
        if rx.kind != RXN_ELEMENTARY:
            for nm, e in rx.efficiencies.items():
                if e != 1.0:
                    eff_sp.append(idx[nm])
                    eff_val.append(e)
        eff_ptr[j + 1] = len(eff_sp)
    arrays = dict(
        mw=mw, nasa=np.ascontiguousarray(nasa), rtype=rtype, rflags=rflags,
        arr=np.ascontiguousarray(arr), arr_lo=np.ascontiguousarray(arr_lo),
        arr_rev=np.ascontiguousarray(arr_rev), troe=np.ascontiguousarray(troe),
        sp=np.ascontiguousarray(sp), nu=np.ascontiguousarray(nu), eff_ptr=eff_ptr,
        eff_sp=np.array(eff_sp if eff_sp else [0], np.int32),
        eff_val=np.array(eff_val if eff_val else [0.0], np.float64),
    )
    return FlatMechanism(N, R, len(eff_sp), arrays)


# ------------------------------------------------------- thermo helpers (numpy)

def nasa_coeffs(mech: Mechanism, T: np.ndarray) -> np.ndarray:
    """[..., N, 7] NASA-7 coefficients selected for temperature T[...]."""
    lo = np.array([s.nasa_lo for s in mech.species])
    hi = np.array([s.nasa_hi for s in mech.species])
    tm = np.array([s.tmid for s in mech.species])
    T = np.asarray(T, dtype=np.float64)
    sel = (T[..., None] < tm)[..., None]
    return np.where(sel, lo, hi)


def cp_R(mech, T):
    a = nasa_coeffs(mech, T)
    T = np.asarray(T)[..., None]
    return a[..., 0] + T * (a[..., 1] + T * (a[..., 2] + T * (a[..., 3] + T * a[..., 4])))


def h_RT(mech, T):
    a = nasa_coeffs(mech, T)
    T = np.asarray(T)[..., None]
    return (a[..., 0] + T * (a[..., 1] / 2 + T * (a[..., 2] / 3 + T * (a[..., 3] / 4 + T * a[..., 4] / 5)))
            + a[..., 5] / T)


def s_R(mech, T):
    a = nasa_coeffs(mech, T)
    T = np.asarray(T)[..., None]
    return (a[..., 0] * np.log(T) + T * (a[..., 1] + T * (a[..., 2] / 2 + T * (a[..., 3] / 3 + T * a[..., 4] / 4)))
            + a[..., 6])


def mix_h_mass(mech, T, Y):
    """Mixture specific enthalpy, erg/g, for T[...] and Y[..., N]."""
    W = mech.mw()
    return np.sum(Y * h_RT(mech, T) * R_CGS * np.asarray(T)[..., None] / W, axis=-1)


def density(mech, T, Y, P=P_ATM_CGS):
    """Ideal-gas density, g/cm^3."""
    W = mech.mw()
    Wmix = 1.0 / np.sum(Y / W, axis=-1)
    return P * Wmix / (R_CGS * T)


def mole_to_mass(mech, X):
    W = mech.mw()
    Y = X * W
    return Y / np.sum(Y, axis=-1, keepdims=True)


def mass_to_mole(mech, Y):
    W = mech.mw()
    X = Y / W
    return X / np.sum(X, axis=-1, keepdims=True)


def builtin(name: str) -> Mechanism:
    """Load one of the mechanism files shipped in pelelmex_b200/mechanisms."""
    p = Path(__file__).resolve().parent / "mechanisms" / f"{name}.yaml"
    if not p.exists():
        raise FileNotFoundError(f"no bundled mechanism {name!r} ({p})")
    return load(p, name)
