"""Generate the synthetic mechanisms shipped with pelelmex_b200.

PeleLMeX's named mechanisms (LiDryer, drm19, dodecane_lu) live in the
PelePhysics submodule, which is empty in the reference snapshot; their
kinetics and thermo data are therefore not available.  This script writes
SYNTHETIC mechanisms instead, clearly labelled as such in their
``description`` and names (``synth_*``).  Each one keeps the species list
and ordering of the named mechanism it stands in for, taken from the
reference's flame tables:

  synth_h2_9    9 species   the H2/O2/N2 species set of LiDryer
  synth_ch4_21  21 species  Exec/RegTests/FlameSheet/drm19_pmf.dat:1
  synth_c12_53  53 species  Exec/UnitTests/DodecaneLu/dodecaneLu_pmf.dat:1

plus reaction counts of the same size (21 / 84 / 268).  No parameter of the
real mechanisms is used: every number is produced here from physical models
and a seeded random generator.

Thermo (NASA-7, two ranges split at 1000 K) is fitted to an ideal-gas
statistical-mechanics model: translation (Sackur-Tetrode), rigid rotation,
Einstein vibrational modes on a simple frequency model, electronic
degeneracy from the radical count, and a standard heat of formation: the
rounded textbook value for small (C0-C2) molecules, else textbook average
bond enthalpies on a greedy valence structure (bond additivity).  Kinetics: element-balanced reactions are enumerated among the
species (atom/group transfer A + B <=> C + D, recombination B + C (+M) <=> A,
isomerisation), written in their exothermic direction with Evans-Polanyi
barriers E = max(0, E0 + alpha * dH) and collision-bounded prefactors; the
reverse rate follows from the equilibrium constant, so every mechanism is
thermodynamically consistent.

Usage:  python pelelmex_b200/mechanisms/make_synthetic.py   (rewrites the .yaml files)
"""
from __future__ import annotations

import math
import re
from pathlib import Path

import numpy as np
import yaml

HERE = Path(__file__).resolve().parent

SPECIES_H2 = ["H2", "O2", "H2O", "H", "O", "OH", "HO2", "H2O2", "N2"]
SPECIES_CH4 = ["H2", "H", "O", "O2", "OH", "H2O", "HO2", "CH2", "CH2(S)", "CH3", "CH4", "CO", "CO2",
               "HCO", "CH2O", "CH3O", "C2H4", "C2H5", "C2H6", "N2", "AR"]
SPECIES_C12 = ["NC12H26", "H", "O", "OH", "HO2", "H2", "H2O", "H2O2", "O2", "CH2", "CH2D", "CH3", "CH4",
               "HCO", "CH2O", "CH3O", "CO", "CO2", "C2H2", "C2H3", "C2H4", "C2H5", "C2H6", "CH2CHO",
               "aC3H5", "C3H6", "nC3H7", "C2H3CHO", "C4H7", "C4H81", "pC4H9", "C5H9", "C5H10",
               "PXC5H11", "C6H12", "PXC6H13", "C7H14", "PXC7H15", "C8H16", "PXC8H17", "C9H18",
               "PXC9H19", "C10H20", "PXC10H21", "PXC12H25", "SXC12H25", "S3XC12H25", "C12H24",
               "C12H25O2", "C12OOH", "O2C12H24OOH", "OC12H23OOH", "N2"]

ELEMENTS = ["C", "H", "O", "N", "AR"]

# names whose formula cannot be read off the name itself
_FORMULA_OVERRIDE = {"C4H81": "C4H8", "CH2D": "CH2", "CH2(S)": "CH2", "C12OOH": "C12H25O2",
                     "NC12H26": "C12H26"}
_SINGLET = {"CH2(S)", "CH2D"}


def composition(name: str) -> dict:
    f = _FORMULA_OVERRIDE.get(name, name)
    f = re.sub(r"^(PX|SX|S3X|[a-z]+)", "", f)
    comp: dict = {}
    for el, cnt in re.findall(r"(AR|C|H|O|N)(\d*)", f):
        comp[el] = comp.get(el, 0) + (int(cnt) if cnt else 1)
    return comp


# ---------------------------------------------------------------- thermo model
KB, HPL, AMU, NA = 1.380649e-23, 6.62607015e-34, 1.66053906660e-27, 6.02214076e23
ATOM_HF = {"H": 218.0, "O": 249.2, "C": 716.7, "N": 472.7, "AR": 0.0}  # kJ/mol, gas atoms
BOND1 = {("H", "H"): 436, ("C", "H"): 413, ("H", "O"): 463, ("H", "N"): 391, ("C", "C"): 348,
         ("C", "O"): 358, ("O", "O"): 146, ("C", "N"): 293, ("N", "O"): 201, ("N", "N"): 163}
BONDN = {("C", "C"): {2: 614, 3: 839}, ("C", "O"): {2: 745, 3: 1072}, ("O", "O"): {2: 498},
         ("N", "N"): {2: 418, 3: 945}, ("C", "N"): {2: 615, 3: 891}, ("N", "O"): {2: 607}}
VALENCE = {"C": 4, "O": 2, "N": 3}
MASS = {"H": 1.00794, "C": 12.0107, "O": 15.9994, "N": 14.0067, "AR": 39.948}


def _key(a, b):
    return tuple(sorted((a, b)))


def structure(name: str, comp: dict):
    """Greedy valence structure -> (bonds [(a, b, order)], unpaired electrons, atoms)."""
    heavy = ["C"] * comp.get("C", 0) + ["O"] * comp.get("O", 0) + ["N"] * comp.get("N", 0)
    nH = comp.get("H", 0)
    if comp.get("AR"):
        return [], 0, ["AR"]
    if not heavy:
        if nH == 2:
            return [("H", "H", 1)], 0, ["H", "H"]
        return [], nH, ["H"] * nH
    rem = [VALENCE[a] for a in heavy]
    bonds = []  # [i, j, order] over heavy indices
    nC = comp.get("C", 0)
    for i in range(1, nC):
        bonds.append([i - 1, i, 1]); rem[i - 1] -= 1; rem[i] -= 1
    last_o = None
    for i in range(nC, len(heavy)):
        tgt = None
        cands = [c for c in range(nC) if rem[c] >= 1]
        if cands and heavy[i] == "O":
            tgt = max(cands, key=lambda c: (rem[c], -c))
        elif heavy[i] == "O" and last_o is not None and rem[last_o] >= 1:
            tgt = last_o
        elif i > 0:
            opts = [c for c in range(i) if rem[c] >= 1]
            tgt = max(opts, key=lambda c: rem[c]) if opts else None
        if tgt is not None:
            bonds.append([tgt, i, 1]); rem[tgt] -= 1; rem[i] -= 1
        if heavy[i] == "O":
            last_o = i
    hbonds = []
    for _ in range(nH):
        order = sorted(range(len(heavy)), key=lambda c: (heavy[c] != "C", heavy[c] != "N", -rem[c]))
        tgt = next((c for c in order if rem[c] >= 1), None)
        if tgt is None:
            break
        rem[tgt] -= 1
        hbonds.append(heavy[tgt])
    # multiple bonds: C-O first (carbonyl), then C-C, then the rest
    special_triple = name in ("CO",)
    prio = sorted(bonds, key=lambda b: (_key(heavy[b[0]], heavy[b[1]]) != ("C", "O"),
                                        _key(heavy[b[0]], heavy[b[1]]) != ("C", "C")))
    for b in prio:
        kk = _key(heavy[b[0]], heavy[b[1]])
        maxo = max(BONDN.get(kk, {1: 0}).keys())
        while rem[b[0]] >= 1 and (rem[b[1]] >= 1 or (special_triple and b[2] < 3)) and b[2] < maxo:
            b[2] += 1
            rem[b[0]] -= 1
            rem[b[1]] = max(rem[b[1]] - 1, 0)
    out = [(heavy[i], heavy[j], o) for i, j, o in bonds] + [(h, "H", 1) for h in hbonds]
    atoms = heavy + ["H"] * nH
    if special_triple:  # C#O: the third bond is dative, no unpaired electron left
        rem = [0] * len(rem)
    return out, sum(rem), atoms


# Rounded textbook standard heats of formation (kJ/mol, 298 K) of small gas
# molecules -- physical constants of the molecules, used where bond additivity
# is known to fail (radicals, cumulated bonds).  Larger species use additivity.
HF_TABLE = {"H": 218.0, "O": 249.2, "OH": 39.0, "H2O": -241.8, "HO2": 12.0, "H2O2": -136.1,
            "CO": -110.5, "CO2": -393.5, "CH4": -74.6, "CH3": 146.0, "CH2": 390.0, "CH2(S)": 428.0,
            "CH2D": 428.0, "HCO": 42.0, "CH2O": -108.6, "CH3O": 17.0, "C2H6": -84.0, "C2H5": 119.0,
            "C2H4": 52.5, "C2H3": 295.0, "C2H2": 228.0, "H2": 0.0, "O2": 0.0, "N2": 0.0, "AR": 0.0}


def heat_of_formation(name: str, comp: dict) -> float:
    """Standard heat of formation (kJ/mol): HF_TABLE, else bond additivity."""
    if name in HF_TABLE:
        return HF_TABLE[name]
    bonds, unpaired, atoms = structure(name, comp)
    hf = sum(ATOM_HF[a] for a in atoms)
    for a, b, o in bonds:
        k = _key(a, b)
        d = BOND1[k] if o == 1 else BONDN[k][o]
        if name == "CO2" and k == ("C", "O") and o == 2:
            d = 799.0  # cumulated C=O in CO2
        hf -= d
    if name in _SINGLET:
        hf += 40.0
    return hf


_LINEAR = {"CO2", "C2H2", "O2", "H2", "N2", "CO", "OH"}
_SIGMA = {"H2": 2, "O2": 2, "N2": 2, "CO2": 2, "H2O": 2, "CH4": 12, "CH3": 6, "CH2": 2, "C2H4": 4,
          "C2H6": 6, "C2H2": 2, "H2O2": 2}


def stat_mech(name: str, comp: dict):
    """Return functions cp_R(T), S298/R, degeneracy etc. of the model molecule."""
    bonds, unpaired, atoms = structure(name, comp)
    nat = len(atoms)
    M = sum(MASS[a] * c for a, c in comp.items())
    g_el = 3 if name in ("O2", "O") or (name in ("CH2",)) else (1 + min(unpaired, 2) if name not in _SINGLET else 1)
    linear = nat == 2 or name in _LINEAR
    if nat == 1:
        rot = 0.0
        thetas = []
    else:
        rot = 1.0 if linear else 1.5
        nmodes = 3 * nat - (5 if linear else 6)
        thetas = []
        for a, b, o in bonds:
            if "H" in (a, b):
                thetas.append(4300.0)
            else:
                thetas.append({1: 1500.0, 2: 2400.0, 3: 3100.0}[o])
        nH = comp.get("H", 0)
        while len(thetas) < nmodes:
            thetas.append(1900.0 if nH > 0 else 700.0)
            nH -= 1
            if nH < -3:
                thetas[-1] = 450.0
        thetas = thetas[:nmodes]
    # crude moment of inertia: heavy atoms on a chain 1.45 A apart, H 1.1 A off-axis
    heavy = [a for a in atoms if a != "H"] or ["H"]
    nh = len(heavy)
    pos = [(i - (nh - 1) / 2.0) * 1.45e-10 for i in range(nh)]
    Isum = sum(MASS[a] * AMU * p * p for a, p in zip(heavy, pos))
    Isum += comp.get("H", 0) * MASS["H"] * AMU * (1.1e-10) ** 2 if atoms.count("H") != nat else 0.0
    if nat == 2 and heavy == ["H"]:
        Isum = 0.5 * MASS["H"] * AMU * (0.74e-10) ** 2
    Isum = max(Isum, 1e-48)
    theta_rot = (HPL / (2 * math.pi)) ** 2 / (2 * Isum * KB)
    sigma = _SIGMA.get(name, 1)

    def cp_R(T):
        T = np.asarray(T, dtype=np.float64)
        c = 2.5 + rot + np.zeros_like(T)
        for th in thetas:
            x = th / T
            c = c + x * x * np.exp(x) / np.expm1(x) ** 2
        return c

    def s_R(T):
        T = np.asarray(T, dtype=np.float64)
        m = M * AMU
        s = np.log((2 * math.pi * m * KB * T / HPL ** 2) ** 1.5 * KB * T / 101325.0) + 2.5
        if rot == 1.0:
            s = s + np.log(T / (sigma * theta_rot)) + 1.0
        elif rot == 1.5:
            s = s + np.log(math.sqrt(math.pi) / sigma * (T / theta_rot) ** 1.5) + 1.5
        for th in thetas:
            x = th / T
            s = s + x / np.expm1(x) - np.log1p(-np.exp(-x))
        return s + math.log(g_el)

    return cp_R, s_R


def nasa7_fit(cp_R, s_R, hf_kJ: float, tlo=200.0, tmid=1000.0, thi=3500.0):
    """Two-range NASA-7 fit, continuous in cp, h and s at tmid."""
    def fit(t0, t1):
        T = np.linspace(t0, t1, 200)
        V = np.stack([T ** i for i in range(5)], axis=1)
        c, *_ = np.linalg.lstsq(V, cp_R(T), rcond=None)
        return c

    lo = fit(tlo, tmid)
    hi = fit(tmid, thi)
    # force cp continuity at tmid by shifting each constant term half-way
    dcp = sum(lo[i] * tmid ** i for i in range(5)) - sum(hi[i] * tmid ** i for i in range(5))
    lo[0] -= dcp / 2
    hi[0] += dcp / 2

    def h_noconst(a, T):
        return sum(a[i] * T ** (i + 1) / (i + 1) for i in range(5))

    def s_noconst(a, T):
        return a[0] * math.log(T) + sum(a[i] * T ** i / i for i in range(1, 5))

    T0 = 298.15
    a6_lo = hf_kJ * 1000.0 / 8.31446261815324 - h_noconst(lo, T0)
    a7_lo = float(s_R(np.array(T0))) - s_noconst(lo, T0)
    a6_hi = h_noconst(lo, tmid) + a6_lo - h_noconst(hi, tmid)
    a7_hi = s_noconst(lo, tmid) + a7_lo - s_noconst(hi, tmid)
    return [float(x) for x in list(lo) + [a6_lo, a7_lo]], [float(x) for x in list(hi) + [a6_hi, a7_hi]]


# ---------------------------------------------------------------- kinetics
def _vec(comp):
    return tuple(comp.get(e, 0) for e in ELEMENTS)


def _is_alkene(comp):
    return set(comp) == {"C", "H"} and comp["C"] >= 2 and comp["H"] == 2 * comp["C"]


def _unpaired(name, comp):
    if name in ("O2", "O", "CH2"):
        return 2
    if name in _SINGLET:
        return 0
    return min(structure(name, comp)[1], 2)


def _is_radical(name, comp):
    _, unpaired, _ = structure(name, comp)
    return unpaired > 0 or name in ("O2",)


class Thermo:
    def __init__(self, names, nasa):
        self.names = names
        self.nasa = nasa

    def h_RT(self, name, T):
        lo, hi, tm = self.nasa[name]
        a = lo if T < tm else hi
        return a[0] + a[1] * T / 2 + a[2] * T ** 2 / 3 + a[3] * T ** 3 / 4 + a[4] * T ** 4 / 5 + a[5] / T

    def dH(self, reac, prod, T=1000.0):  # kcal/mol
        s = sum(c * self.h_RT(n, T) for n, c in prod.items()) - sum(c * self.h_RT(n, T) for n, c in reac.items())
        return s * 1.98720425864083e-3 * T


def _fmt_side(side):
    parts = []
    for n, c in side.items():
        parts.append(n if c == 1 else f"{c} {n}")
    return " + ".join(parts)


def _third_body_effs(names, rng):
    table = {"H2O": (5.0, 12.0), "H2": (2.0, 2.5), "CO": (1.5, 1.9), "CO2": (2.0, 3.8),
             "AR": (0.5, 0.75), "CH4": (1.8, 2.2), "C2H6": (2.7, 3.2)}
    return {n: round(float(rng.uniform(*table[n])), 2) for n in table if n in names}


def make_mechanism(tag, species, n_reactions, seed, describe):
    rng = np.random.default_rng(seed)
    comps = {n: composition(n) for n in species}
    nasa = {}
    sp_yaml = []
    for n in species:
        c = comps[n]
        hf = heat_of_formation(n, c)
        cp_R, s_R = stat_mech(n, c)
        lo, hi = nasa7_fit(cp_R, s_R, hf)
        nasa[n] = (lo, hi, 1000.0)
        sp_yaml.append({"name": n, "composition": {k: v for k, v in c.items()},
                        "thermo": {"model": "NASA7", "temperature-ranges": [200.0, 1000.0, 3500.0],
                                   "data": [[float(f"{x:.9e}") for x in lo], [float(f"{x:.9e}") for x in hi]]},
                        "note": f"synthetic: dHf298 = {hf:.1f} kJ/mol (bond additivity)"})
    th = Thermo(species, nasa)
    inert = {n for n in species if n in ("N2", "AR")}
    reactive = [n for n in species if n not in inert]
    by_vec = {}
    for n in reactive:
        by_vec.setdefault(_vec(comps[n]), []).append(n)
    pairs = {}
    for i, a in enumerate(reactive):
        for b in reactive[i:]:
            v = tuple(x + y for x, y in zip(_vec(comps[a]), _vec(comps[b])))
            pairs.setdefault(v, []).append((a, b))
    natoms = {n: sum(comps[n].values()) for n in species}

    def transfer_size(r, p):
        (a, b), (c, d) = r, p
        best = 99
        for x, y in ((c, d), (d, c)):
            g = [abs(u - v) for u, v in zip(_vec(comps[a]), _vec(comps[x]))]
            best = min(best, sum(g))
        return best

    def h_transfer(r, p):
        """True when the smallest group moving between the pairs is one H atom."""
        (a, b), (c, d) = r, p
        hvec = _vec({"H": 1})
        for x in (c, d):
            g = [abs(u - v) for u, v in zip(_vec(comps[a]), _vec(comps[x]))]
            if tuple(g) == hvec:
                return True
        return False

    exch, recomb, isom = [], [], []
    for v, plist in pairs.items():
        for i in range(len(plist)):
            for j in range(i + 1, len(plist)):
                r, p = plist[i], plist[j]
                if set(r) & set(p):
                    continue
                t = transfer_size(r, p)
                if t > 3:
                    continue
                rad = any(_is_radical(n, comps[n]) for n in r + p)
                if not rad:
                    continue
                # keep the number of unpaired electrons (spin-count conservation)
                if sum(_unpaired(n, comps[n]) for n in r) != sum(_unpaired(n, comps[n]) for n in p):
                    continue
                exch.append((r, p, t))
        if v in by_vec:
            for A in by_vec[v]:
                for (b, c) in plist:
                    if A in (b, c):
                        continue
                    # bond formation needs a radical site on both fragments (O2, CO and
                    # alkenes accept a radical)
                    rb, rc = _is_radical(b, comps[b]), _is_radical(c, comps[c])
                    acc = {b, c} & ({"CO", "O2"} | {n for n in reactive if _is_alkene(comps[n])})
                    if (rb and rc) or ((rb or rc) and acc):
                        recomb.append(((b, c), A))
    for v, names in by_vec.items():
        for i in range(len(names)):
            for j in range(i + 1, len(names)):
                isom.append((names[i], names[j]))

    def side(lst):
        d = {}
        for n in lst:
            d[n] = d.get(n, 0) + 1
        return d

    chosen = []
    used = set()
    n_rec = max(2, int(round(0.2 * n_reactions)))
    n_iso = min(len(isom), max(0, int(round(0.03 * n_reactions)))) if len(species) > 30 else 0
    w_rec = np.array([1.0 / (1 + abs(natoms[b] - natoms[c])) for (b, c), A in recomb])
    def nrad(side_):
        return sum(1 for n in side_ if _unpaired(n, comps[n]) > 0)

    w_ex = np.array([math.exp(-1.2 * t) * (2.0 if natoms[r[0]] + natoms[r[1]] < 8 else 1.0)
                     * (0.3 if abs(nrad(r) - nrad(p)) == 2 else 1.0) for r, p, t in exch])

    def pick(cands, w, k):
        if not cands or k <= 0:
            return []
        k = min(k, len(cands))
        idx = rng.choice(len(cands), size=k, replace=False, p=w / w.sum())
        return [cands[i] for i in sorted(idx)]

    rec_sel = pick(recomb, w_rec, n_rec)
    iso_sel = pick(isom, np.ones(len(isom)), n_iso)
    ex_sel = pick(exch, w_ex, n_reactions - len(rec_sel) - len(iso_sel))
    # make sure every reactive species appears at least once
    covered = set()
    for (b, c), A in rec_sel:
        covered |= {b, c, A}
    for r, p, t in ex_sel:
        covered |= set(r) | set(p)
    for a, b in iso_sel:
        covered |= {a, b}
    for n in reactive:
        if n in covered:
            continue
        opts = [e for e in exch if n in e[0] or n in e[1]]
        ropts = [e for e in recomb if n in e[0] or n == e[1]]
        if ropts:
            add = ropts[int(rng.integers(len(ropts)))]
            rec_sel.append(add)
            covered |= {add[0][0], add[0][1], add[1]}
        elif opts:
            add = opts[int(rng.integers(len(opts)))]
            ex_sel.append(add)
            covered |= set(add[0]) | set(add[1])
    # trim back to the target count, dropping exchange reactions whose species stay covered
    while len(rec_sel) + len(ex_sel) + len(iso_sel) > n_reactions:
        cnt = {}
        for (b, c), A in rec_sel:
            for n in (b, c, A):
                cnt[n] = cnt.get(n, 0) + 1
        for r, p, t in ex_sel:
            for n in set(r) | set(p):
                cnt[n] = cnt.get(n, 0) + 1
        for a, b in iso_sel:
            for n in (a, b):
                cnt[n] = cnt.get(n, 0) + 1
        drop = next((i for i in range(len(ex_sel) - 1, -1, -1)
                     if all(cnt[n] > 1 for n in set(ex_sel[i][0]) | set(ex_sel[i][1]))), None)
        if drop is None:
            break
        ex_sel.pop(drop)

    effs = _third_body_effs(species, rng)
    rx_yaml = []
    T0 = 1000.0
    Rk = 1.98720425864083e-3  # kcal/mol/K
    for (b, c), A in rec_sel:
        reac, prod = side([b, c]), side([A])
        dh = th.dH(reac, prod)
        if dh > 0:  # write the exothermic direction first
            reac, prod = prod, reac
        big = natoms[A] >= 4
        b0 = float(rng.uniform(-1.6, -0.6))
        k0_1000 = 10 ** float(rng.uniform(15.0, 16.3))
        ent = {"equation": "", "note": "synthetic recombination/dissociation"}
        if dh <= 0:
            if big:
                binf = float(rng.uniform(-0.4, 0.4))
                kinf_1000 = 10 ** float(rng.uniform(12.8, 13.7))
                ent["equation"] = f"{_fmt_side(reac)} (+M) <=> {_fmt_side(prod)} (+M)"
                ent["type"] = "falloff"
                ent["low-P-rate-constant"] = {"A": float(f"{k0_1000 / T0 ** b0:.4e}"), "b": round(b0, 3), "Ea": 0.0}
                ent["high-P-rate-constant"] = {"A": float(f"{kinf_1000 / T0 ** binf:.4e}"), "b": round(binf, 3), "Ea": 0.0}
                if rng.uniform() < 0.8:
                    tro = {"A": round(float(rng.uniform(0.4, 0.8)), 3), "T3": round(float(rng.uniform(80, 300)), 1),
                           "T1": round(float(rng.uniform(900, 3000)), 1)}
                    if rng.uniform() < 0.5:
                        tro["T2"] = round(float(rng.uniform(4000, 8000)), 1)
                    ent["Troe"] = tro
            else:
                ent["equation"] = f"{_fmt_side(reac)} + M <=> {_fmt_side(prod)} + M"
                ent["type"] = "three-body"
                ent["rate-constant"] = {"A": float(f"{k0_1000 / T0 ** b0:.4e}"), "b": round(b0, 3), "Ea": 0.0}
        else:
            # dissociation is the exothermic direction (unstable adduct): unimolecular with barrier
            ea = float(rng.uniform(5.0, 15.0))
            ent["equation"] = f"{_fmt_side(reac)} + M <=> {_fmt_side(prod)} + M"
            ent["type"] = "three-body"
            kd = 10 ** float(rng.uniform(14.0, 15.5))
            ent["rate-constant"] = {"A": float(f"{kd:.4e}"), "b": 0.0, "Ea": round(ea * 1000, 1)}
        if effs:
            ent["efficiencies"] = {k: v for k, v in effs.items() if k not in reac and k not in prod} or None
            if ent["efficiencies"] is None:
                del ent["efficiencies"]
        rx_yaml.append(ent)
    for r, p, t in ex_sel:
        reac, prod = side(list(r)), side(list(p))
        dh = th.dH(reac, prod)
        if dh > 0:
            reac, prod = prod, reac
            dh = -dh
        bexp = float(rng.uniform(0.0, 1.6))
        logk = float(rng.uniform(11.6, 13.4))
        # intrinsic barrier by class: H-atom transfer (abstraction) is easy, other group
        # transfers are hard unless two radicals meet and a single atom moves
        nr = sum(1 for n in reac if _unpaired(n, comps[n]) > 0 and n != "O2")
        if h_transfer(r, p):
            e0 = float(rng.uniform(*{2: (0.0, 3.0), 1: (5.0, 12.0), 0: (40.0, 55.0)}[min(nr, 2)]))
        elif nr >= 2 and t == 1:
            e0 = float(rng.uniform(0.0, 3.0))
        else:
            e0 = float(rng.uniform(*{2: (25.0, 40.0), 1: (35.0, 50.0), 0: (45.0, 60.0)}[min(nr, 2)]))
        ea = max(0.0, e0 + 0.35 * dh)
        A = 10 ** logk / T0 ** bexp  # collision prefactor at 1000 K; the barrier acts on top
        rx_yaml.append({"equation": f"{_fmt_side(reac)} <=> {_fmt_side(prod)}",
                        "rate-constant": {"A": float(f"{A:.4e}"), "b": round(bexp, 3), "Ea": round(ea * 1000, 1)},
                        "note": f"synthetic exchange, dH(1000K) = {dh:.1f} kcal/mol"})
    for a, b in iso_sel:
        reac, prod = {a: 1}, {b: 1}
        dh = th.dH(reac, prod)
        if dh > 0:
            reac, prod = prod, reac
        ea = float(rng.uniform(15.0, 25.0))
        A = 10 ** float(rng.uniform(12.0, 13.5))
        rx_yaml.append({"equation": f"{_fmt_side(reac)} <=> {_fmt_side(prod)}",
                        "rate-constant": {"A": float(f"{A:.4e}"), "b": 0.0, "Ea": round(ea * 1000, 1)},
                        "note": "synthetic isomerisation"})
    doc = {
        "description": describe,
        "generator": "pelelmex_b200/mechanisms/make_synthetic.py",
        "seed": seed,
        "units": {"length": "cm", "time": "s", "quantity": "mol", "activation-energy": "cal/mol"},
        "phases": [{"name": "gas", "thermo": "ideal-gas", "elements": [e for e in ELEMENTS if any(e in comps[n] for n in species)],
                    "species": species, "kinetics": "gas", "state": {"T": 300.0, "P": "1 atm"}}],
        "species": sp_yaml,
        "reactions": rx_yaml,
    }
    return doc


def main():
    outs = [
        ("synth_h2_9", SPECIES_H2, 21, 9001,
         "SYNTHETIC H2/O2/N2 mechanism with the 9-species set of LiDryer. Not LiDryer: all thermo and "
         "rate parameters are generated by make_synthetic.py from physical models and a seeded RNG."),
        ("synth_ch4_21", SPECIES_CH4, 84, 9021,
         "SYNTHETIC CH4/air mechanism with the 21 species (and order) of drm19 "
         "(Exec/RegTests/FlameSheet/drm19_pmf.dat:1) and 84 reactions. Not drm19: all parameters are "
         "generated by make_synthetic.py."),
        ("synth_c12_53", SPECIES_C12, 268, 9053,
         "SYNTHETIC n-dodecane/air mechanism with the 53 species (and order) of dodecane_lu "
         "(Exec/UnitTests/DodecaneLu/dodecaneLu_pmf.dat:1) and 268 reactions. Not dodecane_lu: all "
         "parameters are generated by make_synthetic.py."),
    ]
    for tag, sp, nr, seed, desc in outs:
        doc = make_mechanism(tag, sp, nr, seed, desc)
        path = HERE / f"{tag}.yaml"
        path.write_text(yaml.safe_dump(doc, sort_keys=False, width=120, default_flow_style=None))
        print(f"{path.name}: {len(sp)} species, {len(doc['reactions'])} reactions")


if __name__ == "__main__":
    main()
