// mech_dev.cuh -- warp-cooperative evaluation of a Chemkin-formalism mechanism
// for ONE cell per warp (sm_100a).
//
// This is the device side of what a CEPTR-generated mechanism provides to the
// reference reactor (productionRate, aJacobian, species enthalpies/cp, reached
// from PeleLMeX through eos.RTY2WDOT / T2Hi, Source/PeleLMeX_K.H:611,880-885).
// The mechanism is table data in global memory in structure-of-arrays form,
// read through the read-only path; this file holds the tables and the
// per-reaction rate evaluation shared by the group (group_mech.cuh) and the
// thread-per-cell (bdf_thread.cuh) integrators.  Everything here is FP64.
#pragma once
#include <cstdint>

namespace b200 {

constexpr double kRu = 8.31446261815324e7;  // erg/mol/K
constexpr double kPatm = 1013250.0;         // dyn/cm^2
constexpr double kLn10 = 2.302585092994046;
constexpr unsigned kFull = 0xffffffffu;

// Mechanism tables in device memory (structure of arrays).
struct DevMech {
  int N, R, n;  // species, reactions, n = N + 1
  const double* mw;      // [N]
  const double* inv_mw;  // [N]
  const double* nasa;    // [15][N]: Tmid, lo a1..a7, hi a1..a7
  const int* rtype;      // [R]
  const int* rflags;     // [R]
  const double* arr;     // [3][R] lnA, b, Ea/R
  const double* arr_lo;  // [3][R]
  const double* arr_rev; // [3][R]
  const double* troe;    // [4][R] a, 1/T3, 1/T1, T2
  const int* sp;         // [8][R] slot species (-1 empty)
  const int* nu;         // [8][R] slot stoichiometric coefficient (signed: -reactant, +product)
  const double* sdnu;    // [R] sum of net stoichiometry
  const int* eff_ptr;    // [R+1]
  const int* eff_sp;     // [n_eff]
  const double* eff_m1;  // [n_eff] efficiency - 1
  const int* inc_ptr;    // [N+1] species -> (reaction, net nu) incidence
  const int* inc_rxn;    // [nnz]
  const double* inc_nu;  // [nnz]
};

// Species-indexed views used by the per-reaction evaluation (unit stride).
struct SpView {
  const double* C;    // concentrations (mol/cm^3)
  const double* gRT;  // g/RT
  const double* hRT;  // h/RT (Jacobian only)
};

// Per-lane components of one state vector, passed by value so that calls to
// the out-of-line evaluation functions keep it in registers.
template <int CPL>
struct Vec {
  double v[CPL];
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}

__device__ __forceinline__ double ipow(double x, int n) {
  double r = 1.0;
  for (int i = 0; i < n; ++i) r *= x;
  return r;
}

// NASA-7 for species k at T: cp/R, h/RT, s/R (lnT precomputed), d(cp/R)/dT.
__device__ __forceinline__ void nasa7(const DevMech& m, int k, double T, double lnT, double& cpR,
                                      double& hRT, double& sR, double& dcpR) {
  const int N = m.N;
  const double tm = __ldg(m.nasa + k);
  const int base = (T < tm) ? 1 : 8;
  const double a0 = __ldg(m.nasa + (base + 0) * N + k);
  const double a1 = __ldg(m.nasa + (base + 1) * N + k);
  const double a2 = __ldg(m.nasa + (base + 2) * N + k);
  const double a3 = __ldg(m.nasa + (base + 3) * N + k);
  const double a4 = __ldg(m.nasa + (base + 4) * N + k);
  const double a5 = __ldg(m.nasa + (base + 5) * N + k);
  const double a6 = __ldg(m.nasa + (base + 6) * N + k);
  cpR = a0 + T * (a1 + T * (a2 + T * (a3 + T * a4)));
  hRT = a0 + T * (a1 / 2 + T * (a2 / 3 + T * (a3 / 4 + T * a4 / 5))) + a5 / T;
  sR = a0 * lnT + T * (a1 + T * (a2 / 2 + T * (a3 / 3 + T * a4 / 4))) + a6;
  dcpR = a1 + T * (2 * a2 + T * (3 * a3 + T * 4 * a4));
}

// Forward-rate pieces of reaction j at T; returns kf (falloff-blended) and
// fills M (third-body concentration), and for the Jacobian dkf/dM and dln(kf)/dT.
struct RxnEval {
  double kf, kr, pf, pr, M, dkf_dM, dlnkf_dT, dkr_dT;
};

template <bool JAC>
__device__ __forceinline__ RxnEval eval_reaction(const DevMech& m, const SpView& s, int j, double T,
                                                 double lnT, double invT, double Ctot, double lnPRT) {
  const int R = m.R;
  RxnEval e;
  const double lnA = __ldg(m.arr + j), b = __ldg(m.arr + R + j), ea = __ldg(m.arr + 2 * R + j);
  double kinf = exp(lnA + b * lnT - ea * invT);
  const int type = __ldg(m.rtype + j);
  const int flags = __ldg(m.rflags + j);
  double M = 0.0;
  if (type != 0) {
    M = Ctot;
    const int e0 = __ldg(m.eff_ptr + j), e1 = __ldg(m.eff_ptr + j + 1);
    for (int q = e0; q < e1; ++q) M += __ldg(m.eff_m1 + q) * s.C[__ldg(m.eff_sp + q)];
  }
  e.M = M;
  double kf = kinf;
  double dlnkf = 0.0;
  e.dkf_dM = 0.0;
  if (JAC) dlnkf = b * invT + ea * invT * invT;
  if (type >= 2) {
    const double lnA0 = __ldg(m.arr_lo + j), b0 = __ldg(m.arr_lo + R + j), ea0 = __ldg(m.arr_lo + 2 * R + j);
    const double k0 = exp(lnA0 + b0 * lnT - ea0 * invT);
    const double Pr = k0 * M / kinf;
    double F = 1.0, D = 0.0, dlnF_T = 0.0;
    if (type == 3) {
      const double a = __ldg(m.troe + j), i3 = __ldg(m.troe + R + j), i1 = __ldg(m.troe + 2 * R + j);
      const double t2 = __ldg(m.troe + 3 * R + j);
      const double e3 = exp(-T * i3), e1 = exp(-T * i1);
      double Fc = (1.0 - a) * e3 + a * e1;
      double dFc = -(1.0 - a) * i3 * e3 - a * i1 * e1;
      if (flags & 4) {
        const double e2 = exp(-t2 * invT);
        Fc += e2;
        dFc += t2 * invT * invT * e2;
      }
      const double logFc = log10(fmax(Fc, 1e-300));
      const double c = -0.4 - 0.67 * logFc, nn = 0.75 - 1.27 * logFc;
      const double logPr = log10(fmax(Pr, 1e-300));
      const double u = logPr + c;
      const double den = nn - 0.14 * u;
      const double f1 = u / den;
      const double g = 1.0 + f1 * f1;
      const double logF = logFc / g;
      F = exp(kLn10 * logF);
      if (JAC) {
        D = (Pr <= 1e-300) ? 0.0 : -2.0 * logFc * f1 * nn / (g * g * den * den);
        const double df1 = (-0.67 * nn + 1.27 * u) / (den * den);
        const double dlogF_dlogFc = 1.0 / g - logFc * 2.0 * f1 / (g * g) * df1;
        if (Fc > 1e-300) dlnF_T = dlogF_dlogFc * dFc / Fc;
      }
    }
    kf = kinf * Pr / (1.0 + Pr) * F;
    if (JAC) {
      const double dlnk0 = b0 * invT + ea0 * invT * invT;
      const double dlnPr = dlnk0 - dlnkf;
      dlnkf = dlnkf + dlnPr / (1.0 + Pr) + D * dlnPr + dlnF_T;
      e.dkf_dM = k0 * F * (1.0 / ((1.0 + Pr) * (1.0 + Pr)) + D / (1.0 + Pr));
    }
  }
  double kr = 0.0, dkr = 0.0;
  if (flags & 2) {
    const double lr = __ldg(m.arr_rev + j), br = __ldg(m.arr_rev + R + j), er = __ldg(m.arr_rev + 2 * R + j);
    kr = exp(lr + br * lnT - er * invT);
    if (JAC) dkr = kr * (br * invT + er * invT * invT);
  } else if (flags & 1) {
    double sg = 0.0, sh = 0.0;
#pragma unroll
    for (int sl = 0; sl < 8; ++sl) {
      const int k = __ldg(m.sp + sl * R + j);
      if (k >= 0) {
        const double v = (double)__ldg(m.nu + sl * R + j);
        sg += v * s.gRT[k];
        if (JAC) sh += v * s.hRT[k];
      }
    }
    const double sd = __ldg(m.sdnu + j);
    kr = kf * exp(sg - sd * lnPRT);
    if (JAC) dkr = kr * (dlnkf - (sh * invT - sd * invT));
  }
  double pf = 1.0, pr = 1.0;
#pragma unroll
  for (int sl = 0; sl < 4; ++sl) {
    const int k = __ldg(m.sp + sl * R + j);
    if (k >= 0) pf *= ipow(s.C[k], -__ldg(m.nu + sl * R + j));
    const int k2 = __ldg(m.sp + (sl + 4) * R + j);
    if (k2 >= 0) pr *= ipow(s.C[k2], __ldg(m.nu + (sl + 4) * R + j));
  }
  e.kf = kf;
  e.kr = kr;
  e.pf = pf;
  e.pr = pr;
  e.dlnkf_dT = dlnkf;
  e.dkr_dT = dkr;
  return e;
}

}  // namespace b200
