"""Numpy restatement of the HP reactor right-hand side -- TEST INFRASTRUCTURE.

Part of the oracle: only tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg may use it, and only as the checker.  It is a second,
vectorised statement of the same mathematics as oracle/oracle.c, used to
check that file (and scipy's BDF/Radau through it) on small cases.

What it restates:
  * Chemkin-formalism production rates (what CEPTR's productionRate /
    eos.RTY2WDOT computes; reached from Source/PeleLMeX_K.H:880-885): mass
    action with Arrhenius k = A T^b exp(-Ea/RT), third-body concentration
    sum_k eff_k C_k, Lindemann/Troe falloff, reverse rates from
    Kc = exp(-sum nu g/RT) (P_atm / R T)^(sum nu).
  * The constant-pressure (HP) reaction ODE with piecewise-constant forcing
    of Docs/sphinx/manual/Model.rst:300-311, with T carried as a state:
      d(rhoY_k)/dt = W_k wdot_k + F_k
      dT/dt        = (F_H - sum_k h_k d(rhoY_k)/dt) / (rho cp)
Parity status: unpinned against the reference (its reactor is absent from
the snapshot); pinned against scipy's independent BDF/Radau integrators.
"""
from __future__ import annotations

import numpy as np

R_CGS = 8.31446261815324e7
P_ATM = 1013250.0
LN10 = np.log(10.0)


class NpKinetics:
    def __init__(self, flat):
        a = flat.arrays
        self.N = flat.n_species
        self.R = flat.n_reactions
        self.mw = a["mw"]
        self.nasa = a["nasa"]
        self.rtype = a["rtype"]
        self.rflags = a["rflags"]
        self.arr = a["arr"]
        self.arr_lo = a["arr_lo"]
        self.arr_rev = a["arr_rev"]
        self.troe = a["troe"]
        self.sp = a["sp"]
        self.nu = a["nu"]
        N, R = self.N, self.R
        # dense stoichiometry and efficiency matrices
        self.nu_f = np.zeros((R, N))
        self.nu_r = np.zeros((R, N))
        for j in range(R):
            for s in range(4):
                if self.sp[j, s] >= 0:
                    self.nu_f[j, self.sp[j, s]] += self.nu[j, s]
                if self.sp[j, 4 + s] >= 0:
                    self.nu_r[j, self.sp[j, 4 + s]] += self.nu[j, 4 + s]
        self.dnu = self.nu_r - self.nu_f
        self.eff = np.ones((R, N))
        ep = a["eff_ptr"]
        for j in range(R):
            for e in range(ep[j], ep[j + 1]):
                self.eff[j, a["eff_sp"][e]] = a["eff_val"][e]

    # thermo -----------------------------------------------------------
    def _coef(self, T):
        T = np.asarray(T, dtype=np.float64)
        lo = self.nasa[:, 1:8]
        hi = self.nasa[:, 8:15]
        sel = (T[..., None] < self.nasa[:, 0])[..., None]
        return np.where(sel, lo, hi), T[..., None]

    def cp_R(self, T):
        a, T = self._coef(T)
        return a[..., 0] + T * (a[..., 1] + T * (a[..., 2] + T * (a[..., 3] + T * a[..., 4])))

    def h_RT(self, T):
        a, T = self._coef(T)
        return (a[..., 0] + T * (a[..., 1] / 2 + T * (a[..., 2] / 3 + T * (a[..., 3] / 4 + T * a[..., 4] / 5)))
                + a[..., 5] / T)

    def s_R(self, T):
        a, T = self._coef(T)
        return (a[..., 0] * np.log(T) + T * (a[..., 1] + T * (a[..., 2] / 2 + T * (a[..., 3] / 3 + T * a[..., 4] / 4)))
                + a[..., 6])

    # kinetics -----------------------------------------------------------
    def rates_of_progress(self, T, C):
        """q_j [..., R] in mol/cm^3/s for temperature T[...] and concentrations C[..., N]."""
        T = np.asarray(T, dtype=np.float64)
        lnT = np.log(T)[..., None]
        Tc = T[..., None]
        kf = np.exp(self.arr[:, 0] + self.arr[:, 1] * lnT - self.arr[:, 2] / Tc)
        M = C @ self.eff.T
        is_tb = self.rtype == 1
        is_fo = (self.rtype == 2) | (self.rtype == 3)
        k0 = np.exp(self.arr_lo[:, 0] + self.arr_lo[:, 1] * lnT - self.arr_lo[:, 2] / Tc)
        Pr = np.where(is_fo, k0 * M / np.where(is_fo, kf, 1.0), 0.0)
        a, t3, t1, t2 = self.troe.T
        has_t2 = (self.rflags & 4) != 0
        with np.errstate(over="ignore", under="ignore", divide="ignore", invalid="ignore"):
            Fc = (1 - a) * np.exp(-Tc / np.where(t3 == 0, 1.0, t3)) + a * np.exp(-Tc / np.where(t1 == 0, 1.0, t1))
            Fc = Fc + np.where(has_t2, np.exp(-np.where(has_t2, t2, 0.0) / Tc), 0.0)
            logFc = np.log10(np.maximum(Fc, 1e-300))
            c = -0.4 - 0.67 * logFc
            n = 0.75 - 1.27 * logFc
            logPr = np.log10(np.maximum(Pr, 1e-300))
            f1 = (logPr + c) / (n - 0.14 * (logPr + c))
            F = np.where(self.rtype == 3, 10.0 ** (logFc / (1 + f1 * f1)), 1.0)
        kf = np.where(is_fo, kf * Pr / (1 + Pr) * F, kf)
        g = self.h_RT(T) - self.s_R(T)
        sdnu = self.dnu.sum(axis=1)
        lnKc = -(g @ self.dnu.T) + sdnu * np.log(P_ATM / (R_CGS * Tc))
        rev = (self.rflags & 1) != 0
        exrev = (self.rflags & 2) != 0
        kr_eq = kf * np.exp(-lnKc)
        kr_ex = np.exp(self.arr_rev[:, 0] + self.arr_rev[:, 1] * lnT - self.arr_rev[:, 2] / Tc)
        kr = np.where(exrev, kr_ex, np.where(rev, kr_eq, 0.0))
        Cn = C[..., None, :]
        pf = np.prod(np.where(self.nu_f > 0, Cn ** self.nu_f, 1.0), axis=-1)
        pr = np.prod(np.where(self.nu_r > 0, Cn ** self.nu_r, 1.0), axis=-1)
        q = kf * pf - kr * pr
        return np.where(is_tb, M * q, q)

    def wdot(self, T, C):
        """Molar production rates [..., N], mol/cm^3/s."""
        return self.rates_of_progress(T, C) @ self.dnu

    def rhs(self, y, forcing):
        """HP right-hand side for y[..., N+1] = (rhoY, T) and forcing (F_rhoY, F_rhoH)."""
        N = self.N
        rY = y[..., :N]
        T = y[..., N]
        C = rY / self.mw
        om = self.wdot(T, C)
        dY = om * self.mw + forcing[..., :N]
        cpk = self.cp_R(T) * R_CGS / self.mw
        hk = self.h_RT(T) * R_CGS * T[..., None] / self.mw
        rcp = np.sum(rY * cpk, axis=-1)
        dT = (forcing[..., N] - np.sum(hk * dY, axis=-1)) / rcp
        return np.concatenate([dY, dT[..., None]], axis=-1)

    def jac_fd(self, y, forcing, rel=1e-7):
        """Central finite-difference Jacobian of rhs, for checking the analytic one."""
        n = y.shape[-1]
        J = np.zeros(y.shape[:-1] + (n, n))
        for j in range(n):
            hj = rel * np.maximum(np.abs(y[..., j]), 1e-10 if j < n - 1 else 1.0)
            yp = y.copy(); yp[..., j] += hj
            ym = y.copy(); ym[..., j] -= hj
            J[..., :, j] = (self.rhs(yp, forcing) - self.rhs(ym, forcing)) / (2 * hj)[..., None]
        return J

    def mix_h(self, T, Y):
        """Mixture specific enthalpy erg/g."""
        return np.sum(Y * self.h_RT(T) * R_CGS * np.asarray(T)[..., None] / self.mw, axis=-1)

    def density(self, T, Y, P=P_ATM):
        return P / (R_CGS * T * np.sum(Y / self.mw, axis=-1))
