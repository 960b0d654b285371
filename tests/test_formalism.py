"""The rate formalism pinned by hand, one reaction kind at a time.

Each case is a single reaction written into a small mechanism file (seven
species with invented NASA-7 data): elementary irreversible and reversible,
an explicit reverse rate, three-body with efficiencies and a doubled
reactant, Lindemann falloff, Troe falloff with and without T2, and one case
in Cantera's default SI units.  Its rates of progress are computed in this
file from the published formulas, with the stoichiometry written out here
rather than parsed from the equation, and compared with the oracle's wdot
(and, on the GPU, with b200chem_inst_rr):

- k = A T^b exp(-Ea / (R T)) (modified Arrhenius, CHEMKIN-II, Kee et al.
  1989, eq. 52), A converted from the file's units to cm, mol, s;
- third body [M] = sum_k eps_k [X_k], eps_k = 1 unless listed (eq. 58);
- falloff: Pr = k0 [M] / kinf, k = kinf Pr / (1 + Pr) F, F = 1 for
  Lindemann; Troe (Gilbert, Luther & Troe 1983): Fcent = (1 - a)
  exp(-T / T3) + a exp(-T / T1) + exp(-T2 / T), c = -0.4 - 0.67 log10 Fcent,
  n = 0.75 - 1.27 log10 Fcent, f1 = (log10 Pr + c) / (n - 0.14 (log10 Pr +
  c)), log10 F = log10 Fcent / (1 + f1^2) (eqs. 73-76);
- reverse: kr = kf / Kc, Kc = exp(-dG0 / (R T)) (P_atm / (R T))^(sum nu),
  with h/RT and s/R from the NASA-7 polynomials (eqs. 19-20, 52-54).

Nothing here shares code with mechanism.flatten or the oracle beyond the
file they both read, so a misreading of the formalism on their side shows.
"""
import math

import numpy as np
import pytest
import yaml

from pelelmex_b200 import mechanism as M

RU = 8.31446261815324e7  # erg / (mol K)
R_CAL = 8.31446261815324 / 4.184  # cal / (mol K)
PATM = 1013250.0  # dyn / cm^2
AW = {"H": 1.00794, "O": 15.9994, "Ar": 39.948}  # IUPAC, g/mol

# seven species, invented two-range NASA-7 data (lo below 1000 K, hi above)
SPECIES = {
    "H": ({"H": 1}, 25470.0),
    "O": ({"O": 1}, 29230.0),
    "OH": ({"H": 1, "O": 1}, 3980.0),
    "H2": ({"H": 2}, -980.0),
    "O2": ({"O": 2}, -1060.0),
    "H2O": ({"H": 2, "O": 1}, -30020.0),
    "AR": ({"Ar": 1}, -745.0),
}
NAMES = list(SPECIES)


def _nasa(i, hi):
    atoms = sum(SPECIES[NAMES[i]][0].values())
    a1 = 2.5 + 0.45 * (atoms - 1) + (0.15 if hi else 0.0)
    a2 = (1.1e-3 if hi else 1.6e-3) * (atoms - 1) + 2e-5 * i
    a3 = -(2.0e-7 if hi else 5.0e-7) * (atoms - 1) - 1e-9 * i
    a4 = (3.0e-11 if hi else 9.0e-11) * (atoms - 1)
    a5 = -(1.5e-15 if hi else 6.0e-15) * (atoms - 1)
    a6 = SPECIES[NAMES[i]][1] + (-120.0 if hi else 0.0)
    a7 = 2.0 + 1.3 * atoms + 0.2 * i + (0.4 if hi else 0.0)
    return [a1, a2, a3, a4, a5, a6, a7]


def _species_yaml():
    return [{"name": nm, "composition": SPECIES[nm][0],
             "thermo": {"model": "NASA7", "temperature-ranges": [200.0, 1000.0, 3500.0],
                        "data": [_nasa(i, False), _nasa(i, True)]}} for i, nm in enumerate(NAMES)]


def _mech_file(tmp_path, rxn, units=None):
    doc = {"units": units or {"length": "cm", "time": "s", "quantity": "mol", "activation-energy": "cal/mol"},
           "phases": [{"name": "gas", "thermo": "ideal-gas", "elements": ["H", "O", "Ar"], "species": NAMES,
                       "kinetics": "gas"}],
           "species": _species_yaml(), "reactions": [rxn]}
    p = tmp_path / "tiny.yaml"
    p.write_text(yaml.safe_dump(doc))
    return p


def _g_RT(i, T):
    a = _nasa(i, T >= 1000.0)
    h = a[0] + a[1] * T / 2 + a[2] * T ** 2 / 3 + a[3] * T ** 3 / 4 + a[4] * T ** 4 / 5 + a[5] / T
    s = a[0] * math.log(T) + a[1] * T + a[2] * T ** 2 / 2 + a[3] * T ** 3 / 3 + a[4] * T ** 4 / 4 + a[6]
    return h - s


def _arr(d, T, conv, ea_to_K):
    return d["A"] * conv * T ** d.get("b", 0.0) * math.exp(-d.get("Ea", 0.0) * ea_to_K / T)


def _q_hand(case, T, C, si=False):
    """Net rate of progress (mol / cm^3 / s) of one case at T, C (mol / cm^3)."""
    rxn, reac, prod, kind = case["rxn"], case["reac"], case["prod"], case["kind"]
    length, qty = (100.0, 1000.0) if si else (1.0, 1.0)  # m -> cm, kmol -> mol
    ea_to_K = 1.0 / (8314.46261815324 if si else R_CAL)  # J/kmol or cal/mol over R
    order = sum(reac.values())
    conv = lambda o: (length ** 3 / qty) ** (o - 1)  # noqa: E731
    idx = {nm: i for i, nm in enumerate(NAMES)}
    M_ = sum(rxn.get("efficiencies", {}).get(nm, 1.0) * C[i] for i, nm in enumerate(NAMES))
    if kind == "elementary":
        kf = _arr(rxn["rate-constant"], T, conv(order), ea_to_K)
    elif kind == "three-body":
        kf = _arr(rxn["rate-constant"], T, conv(order + 1), ea_to_K) * M_
    else:
        kinf = _arr(rxn["high-P-rate-constant"], T, conv(order), ea_to_K)
        k0 = _arr(rxn["low-P-rate-constant"], T, conv(order + 1), ea_to_K)
        Pr = k0 * M_ / kinf
        F = 1.0
        if "Troe" in rxn:
            t = rxn["Troe"]
            Fc = (1 - t["A"]) * math.exp(-T / t["T3"]) + t["A"] * math.exp(-T / t["T1"])
            if "T2" in t:
                Fc += math.exp(-t["T2"] / T)
            lf = math.log10(Fc)
            c, n = -0.4 - 0.67 * lf, 0.75 - 1.27 * lf
            f1 = (math.log10(Pr) + c) / (n - 0.14 * (math.log10(Pr) + c))
            F = 10.0 ** (lf / (1 + f1 * f1))
        kf = kinf * Pr / (1 + Pr) * F
    fwd = kf * math.prod(C[idx[s]] ** v for s, v in reac.items())
    if "=>" in rxn["equation"] and "<=>" not in rxn["equation"]:
        return fwd
    if "reverse-rate-constant" in rxn:
        kr = _arr(rxn["reverse-rate-constant"], T, conv(sum(prod.values())), ea_to_K)
    else:
        dnu = sum(prod.values()) - sum(reac.values())
        dG = sum(v * _g_RT(idx[s], T) for s, v in prod.items()) - sum(v * _g_RT(idx[s], T) for s, v in reac.items())
        Kc = math.exp(-dG) * (PATM / (RU * T)) ** dnu
        kr = kf / Kc
    return fwd - kr * math.prod(C[idx[s]] ** v for s, v in prod.items())


CASES = {
    "elementary_irreversible": {
        "rxn": {"equation": "O + H2 => H + OH", "rate-constant": {"A": 5.08e4, "b": 2.67, "Ea": 6290.0}},
        "reac": {"O": 1, "H2": 1}, "prod": {"H": 1, "OH": 1}, "kind": "elementary"},
    "elementary_reversible": {
        "rxn": {"equation": "H + O2 <=> O + OH", "rate-constant": {"A": 3.55e15, "b": -0.41, "Ea": 16600.0}},
        "reac": {"H": 1, "O2": 1}, "prod": {"O": 1, "OH": 1}, "kind": "elementary"},
    "explicit_reverse": {
        "rxn": {"equation": "H2O + H <=> H2 + OH", "rate-constant": {"A": 4.5e8, "b": 1.6, "Ea": 18400.0},
                "reverse-rate-constant": {"A": 2.16e8, "b": 1.51, "Ea": 3430.0}},
        "reac": {"H2O": 1, "H": 1}, "prod": {"H2": 1, "OH": 1}, "kind": "elementary"},
    "three_body_efficiencies": {
        "rxn": {"equation": "2 O + M <=> O2 + M", "type": "three-body",
                "rate-constant": {"A": 1.2e17, "b": -1.0, "Ea": 0.0},
                "efficiencies": {"H2": 2.4, "H2O": 15.4, "AR": 0.83}},
        "reac": {"O": 2}, "prod": {"O2": 1}, "kind": "three-body"},
    "lindemann": {
        "rxn": {"equation": "O + H (+M) <=> OH (+M)", "type": "falloff",
                "high-P-rate-constant": {"A": 5.0e13, "b": 0.0, "Ea": 0.0},
                "low-P-rate-constant": {"A": 4.7e18, "b": -1.0, "Ea": 0.0},
                "efficiencies": {"H2O": 6.0, "AR": 0.7}},
        "reac": {"O": 1, "H": 1}, "prod": {"OH": 1}, "kind": "falloff"},
    "troe_t2": {
        "rxn": {"equation": "H + OH (+M) <=> H2O (+M)", "type": "falloff",
                "high-P-rate-constant": {"A": 2.5e13, "b": 0.23, "Ea": -110.0},
                "low-P-rate-constant": {"A": 4.0e22, "b": -2.0, "Ea": 0.0},
                "Troe": {"A": 0.5, "T3": 1.0e-30, "T1": 1.0e30, "T2": 4500.0},
                "efficiencies": {"H2": 0.73, "H2O": 3.65, "AR": 0.38}},
        "reac": {"H": 1, "OH": 1}, "prod": {"H2O": 1}, "kind": "falloff"},
    "troe_no_t2": {
        "rxn": {"equation": "H2 + O (+M) <=> H2O (+M)", "type": "falloff",
                "high-P-rate-constant": {"A": 1.1e12, "b": 0.5, "Ea": 2500.0},
                "low-P-rate-constant": {"A": 6.3e19, "b": -1.4, "Ea": 1200.0},
                "Troe": {"A": 0.62, "T3": 210.0, "T1": 2850.0},
                "efficiencies": {"H2O": 5.0}},
        "reac": {"H2": 1, "O": 1}, "prod": {"H2O": 1}, "kind": "falloff"},
}
SI_CASE = {  # the elementary reversible case in m, kmol, J/kmol
    "rxn": {"equation": "H + O2 <=> O + OH", "rate-constant": {"A": 3.55e12, "b": -0.41, "Ea": 6.94544e7}},
    "reac": {"H": 1, "O2": 1}, "prod": {"O": 1, "OH": 1}, "kind": "elementary"}
SI_UNITS = {"length": "m", "time": "s", "quantity": "kmol", "activation-energy": "J/kmol"}

TEMPS = [420.0, 880.0, 1250.0, 2100.0, 2900.0]


def _states(seed=0):
    rng = np.random.default_rng(seed)
    for T in TEMPS:
        C = PATM / (RU * T) * rng.dirichlet(np.full(len(NAMES), 0.8))
        yield T, np.maximum(C, 1e-14)


def _wdot_hand(case, T, C, si=False):
    q = _q_hand(case, T, C, si)
    w = np.zeros(len(NAMES))
    for s, v in case["reac"].items():
        w[NAMES.index(s)] -= v * q
    for s, v in case["prod"].items():
        w[NAMES.index(s)] += v * q
    return w


def _load(tmp_path, case, units=None):
    return M.load(_mech_file(tmp_path, case["rxn"], units))


@pytest.mark.parametrize("name", list(CASES) + ["si_units"])
def test_oracle_rates_match_hand_formulas(name, tmp_path, oracle_mod):
    case, units = (SI_CASE, SI_UNITS) if name == "si_units" else (CASES[name], None)
    mech = _load(tmp_path, case, units)
    assert mech.names == NAMES
    orc = oracle_mod.Oracle(M.flatten(mech))
    for T, C in _states():
        want = _wdot_hand(case, T, C, si=units is not None)
        got = orc.wdot(T, C)
        sc = np.abs(want).max()
        assert sc > 0.0
        assert np.max(np.abs(got - want)) <= 1e-11 * sc, (T, got, want)


def test_si_and_cgs_files_give_the_same_rates(tmp_path, oracle_mod):
    """The SI file's A and Ea are the CGS case's converted by hand, so both
    files describe one reaction."""
    a = M.flatten(_load(tmp_path, CASES["elementary_reversible"]))
    (tmp_path / "si").mkdir()
    b = M.flatten(_load(tmp_path / "si", SI_CASE, SI_UNITS))
    oa, ob = oracle_mod.Oracle(a), oracle_mod.Oracle(b)
    for T, C in _states(1):
        wa, wb = oa.wdot(T, C), ob.wdot(T, C)
        assert np.max(np.abs(wa - wb)) <= 1e-12 * np.abs(wa).max()


def test_all_cases_in_one_mechanism(tmp_path, oracle_mod):
    """The rates of a mechanism holding every case are the sum of the cases'."""
    doc = yaml.safe_load(_mech_file(tmp_path, CASES["lindemann"]["rxn"]).read_text())
    doc["reactions"] = [c["rxn"] for c in CASES.values()]
    p = tmp_path / "all.yaml"
    p.write_text(yaml.safe_dump(doc))
    orc = oracle_mod.Oracle(M.flatten(M.load(p)))
    for T, C in _states(2):
        want = sum(_wdot_hand(c, T, C) for c in CASES.values())
        got = orc.wdot(T, C)
        sc = max(np.abs(_wdot_hand(c, T, C)).max() for c in CASES.values())
        assert np.max(np.abs(got - want)) <= 1e-11 * sc


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
def test_gpu_rates_match_hand_formulas(name, tmp_path):
    """b200chem_inst_rr (reactionRateRhoY, MKS) on the same single-reaction
    mechanisms: T comes back from the (rho h, rho Y) solve, and the rates
    are compared with the hand formulas at that T."""
    torch = pytest.importorskip("torch")
    from pelelmex_b200.reactor import ReactorB200
    case = CASES[name]
    mech = _load(tmp_path, case)
    mw = np.array([sum(AW[e] * c for e, c in SPECIES[nm][0].items()) for nm in NAMES])
    states = list(_states(3))
    rhoY = np.stack([C * mw for _, C in states], axis=1)  # g / cm^3
    T0 = np.array([T for T, _ in states])
    hk = np.array([[(_g_RT_h(i, T)) * RU * T / mw[i] for i in range(len(NAMES))] for T in T0]).T  # erg / g
    rhoH = (rhoY * hk).sum(axis=0)
    r = ReactorB200(mech).init()
    dev = "cuda:0"
    T = torch.tensor(T0 * 0.97 + 10.0, device=dev)
    rr = r.inst_rr(torch.tensor(rhoY * 1e3, device=dev), torch.tensor(rhoH * 0.1, device=dev), T).cpu().numpy()
    Tg = T.cpu().numpy()
    r.close()
    assert np.max(np.abs(Tg - T0) / T0) < 1e-10
    for c in range(len(T0)):
        want = _wdot_hand(case, Tg[c], rhoY[:, c] / mw) * mw * 1e3  # kg / m^3 / s
        assert np.max(np.abs(rr[:, c] - want)) <= 1e-11 * np.abs(want).max(), (name, Tg[c])


def _g_RT_h(i, T):
    a = _nasa(i, T >= 1000.0)
    return a[0] + a[1] * T / 2 + a[2] * T ** 2 / 3 + a[3] * T ** 3 / 4 + a[4] * T ** 4 / 5 + a[5] / T
