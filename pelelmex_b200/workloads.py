"""Seeded synthetic chemistry workloads (CGS units, component-major layout).

Every random number comes from the counter-based Philox-4x32-10 generator
(Salmon et al., "Parallel random numbers: as easy as 1, 2, 3", SC'11) keyed
by (seed, draw) with the cell index as counter, so a field is reproducible
cell by cell on any machine and any subset of cells can be regenerated
alone (the CPU baseline times a seeded random subset of the full field).

Fields mirror the inputs of ReactorBase::react as called from
Source/PeleLMeX_Reactions.cpp:101-108 after the MKS->CGS conversion of
:69-79: rhoY [N, ncells] (g/cm^3), T [ncells] (K), rhoH [ncells]
(erg/cm^3), forcing extF_rhoY [N, ncells] and extF_rhoH [ncells].  Cells
are ordered with i (x) fastest, as in an amrex::Box.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import mechanism as mechmod

_M0, _M1 = np.uint64(0xD2511F53), np.uint64(0xCD9E8D57)
_W0, _W1 = np.uint32(0x9E3779B9), np.uint32(0xBB67AE85)
_MASK32 = np.uint64(0xFFFFFFFF)


def philox4x32(counter_lo: np.ndarray, counter_hi: int, key0: int, key1: int) -> np.ndarray:
    """Philox-4x32-10 on counters (lo, hi, 0, 0) -> [4, n] uint32 words."""
    c0 = np.asarray(counter_lo, dtype=np.uint64) & _MASK32
    c1 = (np.asarray(counter_lo, dtype=np.uint64) >> np.uint64(32)) & _MASK32
    c2 = np.full_like(c0, np.uint64(counter_hi & 0xFFFFFFFF))
    c3 = np.zeros_like(c0)
    k0 = np.uint32(key0 & 0xFFFFFFFF)
    k1 = np.uint32(key1 & 0xFFFFFFFF)
    with np.errstate(over="ignore"):
        for _ in range(10):
            p0 = _M0 * c0
            p1 = _M1 * c2
            hi0, lo0 = p0 >> np.uint64(32), p0 & _MASK32
            hi1, lo1 = p1 >> np.uint64(32), p1 & _MASK32
            c0, c1, c2, c3 = (hi1 ^ c1 ^ np.uint64(k0)), lo1, (hi0 ^ c3 ^ np.uint64(k1)), lo0
            k0 = np.uint32(k0 + _W0)
            k1 = np.uint32(k1 + _W1)
    return np.stack([c0, c1, c2, c3]).astype(np.uint32)


def uniform(seed: int, draw: int, cells: np.ndarray) -> np.ndarray:
    """U[0,1) doubles, one per cell, for stream `draw` (53 random bits each)."""
    w = philox4x32(cells, draw, seed, 0x5EED).astype(np.uint64)
    bits = (w[0] << np.uint64(21)) ^ w[1]
    return (bits & np.uint64((1 << 53) - 1)).astype(np.float64) * (1.0 / (1 << 53))


@dataclass
class Field:
    """One batch of cells to react (CGS, component-major)."""
    mech: object
    rhoY: np.ndarray
    T: np.ndarray
    rhoH: np.ndarray
    frhoY: np.ndarray
    frhoH: np.ndarray
    dt: float
    shape: tuple
    name: str

    @property
    def ncells(self) -> int:
        return self.T.shape[0]

    def subset(self, idx: np.ndarray) -> "Field":
        return Field(self.mech, self.rhoY[:, idx].copy(), self.T[idx].copy(), self.rhoH[idx].copy(),
                     self.frhoY[:, idx].copy(), self.frhoH[idx].copy(), self.dt, (len(idx),), self.name)


def _finish(mech, Y, T, dt, shape, name, P=mechmod.P_ATM_CGS):
    rho = mechmod.density(mech, T, Y, P)
    h = mechmod.mix_h_mass(mech, T, Y)
    rhoY = np.ascontiguousarray((rho[:, None] * Y).T)
    n = T.shape[0]
    return Field(mech, rhoY, T.astype(np.float64), rho * h, np.zeros((mech.n_species, n)),
                 np.zeros(n), dt, shape, name)


def _cells(shape, cells):
    n = int(np.prod(shape))
    return np.arange(n, dtype=np.int64) if cells is None else np.asarray(cells, dtype=np.int64)


def premixed_h2(mech, edge: int = 32, seed: int = 1, dt: float = 1e-6, cells=None) -> Field:
    """Stoichiometric H2/air, each Y_k x (1 + U[-0.05, 0.05]) renormalised,
    T ~ U[1000, 2000] K, P = 1 atm, no forcing (LiDryer-style 32^3 case)."""
    shape = (edge, edge, edge)
    c = _cells(shape, cells)
    names = mech.names
    X = np.zeros(mech.n_species)
    X[names.index("H2")] = 2.0
    X[names.index("O2")] = 1.0
    X[names.index("N2")] = 3.76
    Y0 = mechmod.mole_to_mass(mech, X / X.sum())
    Y = np.empty((c.size, mech.n_species))
    for k in range(mech.n_species):
        Y[:, k] = Y0[k] * (1.0 + 0.1 * (uniform(seed, 1 + k, c) - 0.5))
    Y /= Y.sum(axis=1, keepdims=True)
    T = 1000.0 + 1000.0 * uniform(seed, 0, c)
    return _finish(mech, Y, T, dt, shape, "premixed_h2")


def _ch4_air(mech, phi):
    """Unburnt CH4/air mass fractions for equivalence ratios phi[n]."""
    nm = mech.names
    X = np.zeros((phi.size, mech.n_species))
    X[:, nm.index("CH4")] = phi
    X[:, nm.index("O2")] = 2.0
    X[:, nm.index("N2")] = 7.52
    return mechmod.mole_to_mass(mech, X / X.sum(axis=1, keepdims=True))


def _ch4_products(mech, phi):
    """Complete-combustion products of CH4/air with fixed dissociation:
    5% of CO2 -> CO + 1/2 O2 and 2% of H2O -> OH + 1/2 H2 (lean), rich
    mixtures put the oxygen deficit into CO and H2."""
    nm = mech.names
    n = phi.size
    X = np.zeros((n, mech.n_species))
    o2_avail = 2.0 / phi  # per CH4
    co2 = np.ones(n)
    h2o = np.full(n, 2.0)
    co = np.zeros(n)
    h2 = np.zeros(n)
    o2 = o2_avail - 2.0
    rich = o2 < 0
    # rich: oxygen deficit (in O atoms) split equally between CO2->CO and H2O->H2
    deficit = np.where(rich, -2.0 * o2, 0.0)
    shift_c = np.minimum(deficit / 2.0, 1.0)
    co2 -= shift_c
    co += shift_c
    shift_h = np.minimum(deficit - shift_c, 2.0)
    h2o -= shift_h
    h2 += shift_h
    o2 = np.maximum(o2, 0.0)
    d1 = 0.05 * co2
    co2 -= d1; co += d1; o2 += 0.5 * d1
    d2 = 0.02 * h2o
    h2o -= d2; h2 += 0.5 * d2
    X[:, nm.index("CO2")] = co2
    X[:, nm.index("H2O")] = h2o
    X[:, nm.index("CO")] = co
    X[:, nm.index("H2")] = h2
    X[:, nm.index("O2")] = o2
    X[:, nm.index("OH")] = d2
    X[:, nm.index("N2")] = 7.52 / phi
    return mechmod.mole_to_mass(mech, X / X.sum(axis=1, keepdims=True))


def flame_ch4(mech, edge: int = 128, seed: int = 2, dt: float = 1e-6, delta: float = 8.0,
              cells=None) -> Field:
    """drm19-style 128^3 flame-like field: along x a tanh profile from unburnt
    CH4/air (T_u ~ U[300,800], phi ~ U[0.7,1.3] per (y,z) column) to burnt
    products (T_b ~ U[1500,2300]); intermediates H, O, OH, HO2, CH3, CH2O,
    HCO peak in the reaction zone; +-2% multiplicative noise on Y."""
    shape = (edge, edge, edge)
    c = _cells(shape, cells)
    i = c % edge
    col = c // edge  # (j, k) column index
    Tu = 300.0 + 500.0 * uniform(seed, 0, col)
    phi = 0.7 + 0.6 * uniform(seed, 1, col)
    Tb = 1500.0 + 800.0 * uniform(seed, 2, col)
    s = 0.5 * (1.0 + np.tanh((i - edge / 2.0) / delta))
    Yu = _ch4_air(mech, phi)
    Yb = _ch4_products(mech, phi)
    Y = (1.0 - s)[:, None] * Yu + s[:, None] * Yb
    zone = 4.0 * s * (1.0 - s)
    nm = mech.names
    peaks = {"H": 4e-4, "O": 1e-3, "OH": 3e-3, "HO2": 2e-4, "CH3": 1e-3, "CH2O": 1.5e-3, "HCO": 5e-5}
    for d, (sp, amp) in enumerate(peaks.items()):
        if sp in nm:
            Y[:, nm.index(sp)] += amp * zone * (0.5 + uniform(seed, 10 + d, col))
    for k in range(mech.n_species):
        Y[:, k] *= 1.0 + 0.04 * (uniform(seed, 100 + k, c) - 0.5)
    Y /= Y.sum(axis=1, keepdims=True)
    T = (1.0 - s) * Tu + s * Tb
    return _finish(mech, Y, T, dt, shape, "flame_ch4")


def sample_cells(n_total: int, n_sample: int, seed: int = 12345) -> np.ndarray:
    """Seeded random subset (sorted) of cell indices, for bounded CPU baselines."""
    if n_sample >= n_total:
        return np.arange(n_total, dtype=np.int64)
    u = uniform(seed, 0, np.arange(n_total, dtype=np.int64))
    return np.sort(np.argsort(u)[:n_sample]).astype(np.int64)


# --------------------------------------------------------------- dodecane
def _c12_air(mech, Z):
    """Fuel/air mixing line: n-C12H26 mass fraction Z, the rest air
    (O2 : N2 = 1 : 3.76 by moles)."""
    nm = mech.names
    Xa = np.zeros(mech.n_species)
    Xa[nm.index("O2")] = 1.0
    Xa[nm.index("N2")] = 3.76
    Ya = mechmod.mole_to_mass(mech, (Xa / Xa.sum())[None, :])[0]
    Y = (1.0 - Z)[:, None] * Ya[None, :]
    Y[:, nm.index("NC12H26")] += Z
    return Y


def _c12_phi_to_Z(mech, phi):
    """Fuel mass fraction of n-C12H26/air at equivalence ratio phi
    (stoichiometric: 18.5 O2 per C12H26)."""
    mw = mech.mw()
    nm = mech.names
    w_f = mw[nm.index("NC12H26")]
    w_air = 18.5 * (mw[nm.index("O2")] + 3.76 * mw[nm.index("N2")])
    fa = phi * w_f / w_air
    return fa / (1.0 + fa)


def _c12_products(mech, Z):
    """Complete-combustion products of the mixture at fuel mass fraction Z:
    lean -> CO2, H2O, excess O2, N2; rich -> the oxygen deficit goes to CO
    then H2, any fuel beyond that stays unburnt."""
    nm = mech.names
    mw = mech.mw()
    Y0 = _c12_air(mech, Z)
    n_f = Y0[:, nm.index("NC12H26")] / mw[nm.index("NC12H26")]
    n_o2 = Y0[:, nm.index("O2")] / mw[nm.index("O2")]
    n_n2 = Y0[:, nm.index("N2")] / mw[nm.index("N2")]
    burn = np.minimum(n_f, n_o2 / 12.5)          # fuel that at least reaches CO + H2O
    o2 = n_o2 - 12.5 * burn
    co = 12.0 * burn
    h2o = 13.0 * burn
    to_co2 = np.minimum(co, 2.0 * o2)            # remaining O2 oxidises CO
    co -= to_co2
    o2 -= 0.5 * to_co2
    X = np.zeros((Z.size, mech.n_species))
    X[:, nm.index("NC12H26")] = n_f - burn
    X[:, nm.index("CO2")] = to_co2
    X[:, nm.index("CO")] = co
    X[:, nm.index("H2O")] = h2o
    X[:, nm.index("O2")] = o2
    X[:, nm.index("N2")] = n_n2
    return mechmod.mole_to_mass(mech, X / X.sum(axis=1, keepdims=True))


def c12_boxes(mech, seed: int = 3, dt: float = 1e-6, nbox: int = 40, edges=(16, 32, 64), box_cells=None,
              only=None):
    """AMR-like dodecane box list: `nbox` cubic boxes with edges drawn from
    `edges`; the first half cold and inert (T ~ U[300, 600] K), the second
    half igniting (T ~ U[900, 1400] K); per cell phi ~ U[0.5, 2]
    (n-C12H26/air), +-2% noise on Y.  Returns [(lo, edge, Field)]; lo places
    the boxes side by side along x.  box_cells (optional) caps the cells
    generated per box (a seeded subset, for parity samples); `only`
    (optional) generates just those box indices (each box depends only on
    the seed and its index)."""
    out = []
    bidx = np.arange(nbox, dtype=np.int64)
    pick = np.minimum((uniform(seed, 0, bidx) * len(edges)).astype(np.int64), len(edges) - 1)
    x0 = 0
    for b in range(nbox):
        e = int(edges[pick[b]])
        if only is not None and b not in only:
            x0 += e
            continue
        shape = (e, e, e)
        c = _cells(shape, None)
        if box_cells is not None and box_cells < c.size:
            c = sample_cells(c.size, box_cells, seed=seed * 1000 + b)
        key = seed * 4096 + b
        cold = b < nbox // 2
        u = uniform(key, 0, c)
        T = (300.0 + 300.0 * u) if cold else (900.0 + 500.0 * u)
        phi = 0.5 + 1.5 * uniform(key, 1, c)
        Y = _c12_air(mech, _c12_phi_to_Z(mech, phi))
        for k in range(mech.n_species):
            Y[:, k] *= 1.0 + 0.04 * (uniform(key, 10 + k, c) - 0.5)
        Y /= Y.sum(axis=1, keepdims=True)
        out.append(((x0, 0, 0), e, _finish(mech, Y, T, dt, shape if box_cells is None else (c.size,),
                                           f"c12_box{b}_{'cold' if cold else 'ignite'}")))
        x0 += e
    return out


def _grf(seed: int, draw: int, cells: np.ndarray, edge: int, modes: int = 64, ell: float = 16.0):
    """Smoothed Gaussian random field on an edge^3 grid, evaluated cell by
    cell: a sum of `modes` random Fourier modes with wave vectors drawn from
    the spectrum of a Gaussian filter of width ell cells (so the field is a
    Gaussian-filtered white noise up to the mode sampling), normalised to
    zero mean and unit variance."""
    m = np.arange(modes, dtype=np.int64)
    g = []
    for d in range(3):
        u1 = np.maximum(uniform(seed, 1000 * draw + 2 * d, m), 1e-300)
        u2 = uniform(seed, 1000 * draw + 2 * d + 1, m)
        g.append(np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2) / ell)   # Box-Muller
    kx, ky, kz = g
    ph = 2.0 * np.pi * uniform(seed, 1000 * draw + 7, m)
    i = (cells % edge).astype(np.float64)
    j = ((cells // edge) % edge).astype(np.float64)
    k = (cells // (edge * edge)).astype(np.float64)
    f = np.zeros(cells.size)
    for q in range(modes):
        f += np.cos(kx[q] * i + ky[q] * j + kz[q] * k + ph[q])
    return f * np.sqrt(2.0 / modes)


def c12_flame_grf(mech, edge: int = 256, seed: int = 6, dt: float = 5e-6, cells=None) -> Field:
    """Turbulent-flame-like dodecane field: T in [300, 2400] K and mixture
    fraction Z in [0, 1] (air to n-C12H26) from two seeded smoothed Gaussian
    random fields mapped through the normal CDF; the composition blends the
    mixing line and the complete-combustion products at the local Z with
    progress (T - 300) / 2100."""
    from scipy.special import ndtr as cdf
    shape = (edge, edge, edge)
    c = _cells(shape, cells)
    T = 300.0 + 2100.0 * cdf(_grf(seed, 0, c, edge))
    Z = cdf(_grf(seed, 1, c, edge))
    prog = (T - 300.0) / 2100.0
    Y = (1.0 - prog)[:, None] * _c12_air(mech, Z) + prog[:, None] * _c12_products(mech, Z)
    Y = np.maximum(Y, 0.0)
    Y /= Y.sum(axis=1, keepdims=True)
    return _finish(mech, Y, T, dt, shape, "c12_flame_grf")
