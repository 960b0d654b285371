// mech_dev.cuh -- warp-cooperative evaluation of a Chemkin-formalism mechanism
// for ONE cell per warp (sm_100a).
//
// This is the device side of what a CEPTR-generated mechanism provides to the
// reference reactor (productionRate, aJacobian, species enthalpies/cp, reached
// from PeleLMeX through eos.RTY2WDOT / T2Hi, Source/PeleLMeX_K.H:611,880-885).
// Instead of straight-line generated code (which would serialise when lanes
// take different reactions), the mechanism is table data in global memory in
// structure-of-arrays form, read through the read-only path, and the work is
// spread over the 32 lanes of a warp:
//   * species-parallel: lane k owns species k (and lane N owns T) for thermo,
//     concentrations and the production-rate gather;
//   * reaction-parallel: lane j evaluates reactions j, j+32, ... (rates of
//     progress, stored to per-warp shared memory);
//   * column-parallel Jacobian: lane l owns column l and walks the reactions.
// Everything here is FP64.
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

// Per-warp shared-memory scratch for the mechanism evaluation.
struct MechSmem {
  double* C;    // [Npad] concentrations (mol/cm^3)
  double* gRT;  // [Npad] g/RT
  double* hRT;  // [Npad] h/RT
  double* r0;   // [Rpad] per-reaction scratch (q, or ceff)
  double* r1;   // [Rpad] kf * mult
  double* r2;   // [Rpad] kr * mult
  double* r3;   // [Rpad] dq/dT
  double* r4;   // [Rpad] q (Jacobian pass)
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
__device__ __forceinline__ RxnEval eval_reaction(const DevMech& m, const MechSmem& s, int j, double T,
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

// Thermo + concentrations for one cell. Lane k < N handles species k (and
// k + 32 when CPL = 2).  Returns per-lane cp (mass, erg/g/K) and h (erg/g)
// in the output arrays; writes C, gRT, hRT to shared memory.
template <int CPL>
__device__ __forceinline__ void species_state(const DevMech& m, const MechSmem& s, const double (&y)[CPL],
                                              double T, double lnT, double (&cpk)[CPL], double (&hk)[CPL],
                                              double (&dcpk)[CPL], int lane) {
#pragma unroll
  for (int c = 0; c < CPL; ++c) {
    const int k = lane + 32 * c;
    cpk[c] = 0.0;
    hk[c] = 0.0;
    dcpk[c] = 0.0;
    if (k < m.N) {
      double cpR, hRT, sR, dcpR;
      nasa7(m, k, T, lnT, cpR, hRT, sR, dcpR);
      const double iw = __ldg(m.inv_mw + k);
      s.C[k] = y[c] * iw;
      s.gRT[k] = hRT - sR;
      s.hRT[k] = hRT;
      cpk[c] = cpR * kRu * iw;
      hk[c] = hRT * kRu * T * iw;
      dcpk[c] = dcpR * kRu * iw;
    }
  }
}

// Temperature (component N) broadcast from its owner lane.
template <int CPL>
__device__ __forceinline__ double get_T(const double (&y)[CPL], int N) {
  const int owner = N & 31;
  const int c = N >> 5;
  double v = 0.0;
#pragma unroll
  for (int cc = 0; cc < CPL; ++cc)
    if (cc == c) v = y[cc];
  return __shfl_sync(kFull, v, owner);
}

// HP right-hand side of one cell (see the header of b200chem.h):
//   ydot_k = W_k wdot_k + F_k,  ydot_T = (F_H - sum h_k ydot_k) / (sum y_k cp_k)
template <int CPL>
__device__ __noinline__ Vec<CPL> warp_rhs_v(const DevMech* mp, const MechSmem s, const Vec<CPL> yv, const Vec<CPL> Fv,
                                           int lane) {
  const DevMech& m = *mp;
  const double(&y)[CPL] = yv.v;
  const double(&F)[CPL] = Fv.v;
  Vec<CPL> out;
  double(&ydot)[CPL] = out.v;
  const int N = m.N, R = m.R;
  const double T = get_T<CPL>(y, N);
  const double lnT = log(T), invT = 1.0 / T;
  double cpk[CPL], hk[CPL], dcpk[CPL];
  species_state<CPL>(m, s, y, T, lnT, cpk, hk, dcpk, lane);
  double csum = 0.0;
#pragma unroll
  for (int c = 0; c < CPL; ++c)
    if (lane + 32 * c < N) csum += y[c] * __ldg(m.inv_mw + lane + 32 * c);
  const double Ctot = warp_sum(csum);
  const double lnPRT = log(kPatm / (kRu * T));
  __syncwarp();
  for (int j = lane; j < R; j += 32) {
    const RxnEval e = eval_reaction<false>(m, s, j, T, lnT, invT, Ctot, lnPRT);
    double q = e.kf * e.pf - e.kr * e.pr;
    if (__ldg(m.rtype + j) == 1) q *= e.M;
    s.r0[j] = q;
  }
  __syncwarp();
  double rcp = 0.0, hs = 0.0;
#pragma unroll
  for (int c = 0; c < CPL; ++c) {
    const int k = lane + 32 * c;
    if (k < N) {
      double w = 0.0;
      const int p0 = __ldg(m.inc_ptr + k), p1 = __ldg(m.inc_ptr + k + 1);
      for (int p = p0; p < p1; ++p) w += __ldg(m.inc_nu + p) * s.r0[__ldg(m.inc_rxn + p)];
      ydot[c] = w * __ldg(m.mw + k) + F[c];
      rcp += y[c] * cpk[c];
      hs += hk[c] * ydot[c];
    }
  }
  rcp = warp_sum(rcp);
  hs = warp_sum(hs);
#pragma unroll
  for (int c = 0; c < CPL; ++c)
    if (lane + 32 * c == N) ydot[c] = (F[c] - hs) / rcp;
    else if (lane + 32 * c > N) ydot[c] = 0.0;
  __syncwarp();
  return out;
}

template <int CPL>
__device__ __forceinline__ void warp_rhs(const DevMech& m, const MechSmem& s, const double (&y)[CPL],
                                         const double (&F)[CPL], double (&ydot)[CPL], int lane) {
  Vec<CPL> a, b;
#pragma unroll
  for (int c = 0; c < CPL; ++c) {
    a.v[c] = y[c];
    b.v[c] = F[c];
  }
  const Vec<CPL> r = warp_rhs_v<CPL>(&m, s, a, b, lane);
#pragma unroll
  for (int c = 0; c < CPL; ++c) ydot[c] = r.v[c];
}

// Analytic Jacobian of the HP system into shared memory J[i*ldj + j]
// (row i = equation, column j = variable), plus ydot (same as warp_rhs).
template <int CPL>
__device__ __noinline__ Vec<CPL> warp_jac_v(const DevMech* mp, const MechSmem s, const Vec<CPL> yv, const Vec<CPL> Fv,
                                           double* J, int ldj, int lane) {
  const DevMech& m = *mp;
  const double(&y)[CPL] = yv.v;
  const double(&F)[CPL] = Fv.v;
  Vec<CPL> out;
  double(&ydot)[CPL] = out.v;
  const int N = m.N, R = m.R, n = N + 1;
  const double T = get_T<CPL>(y, N);
  const double lnT = log(T), invT = 1.0 / T;
  double cpk[CPL], hk[CPL], dcpk[CPL];
  species_state<CPL>(m, s, y, T, lnT, cpk, hk, dcpk, lane);
  double csum = 0.0;
#pragma unroll
  for (int c = 0; c < CPL; ++c)
    if (lane + 32 * c < N) csum += y[c] * __ldg(m.inv_mw + lane + 32 * c);
  const double Ctot = warp_sum(csum);
  const double lnPRT = log(kPatm / (kRu * T));
  // zero J
  for (int i = 0; i < n; ++i)
#pragma unroll
    for (int c = 0; c < CPL; ++c)
      if (lane + 32 * c < n) J[i * ldj + lane + 32 * c] = 0.0;
  __syncwarp();
  // phase 1: per-reaction scalars (lane per reaction)
  for (int j = lane; j < R; j += 32) {
    const RxnEval e = eval_reaction<true>(m, s, j, T, lnT, invT, Ctot, lnPRT);
    const int type = __ldg(m.rtype + j);
    const double mult = (type == 1) ? e.M : 1.0;
    double ceff = 0.0;
    if (type == 1) ceff = e.kf * e.pf - e.kr * e.pr;
    else if (type >= 2) ceff = e.dkf_dM * (e.pf - (e.kf > 0.0 ? e.kr / e.kf : 0.0) * e.pr);
    s.r0[j] = ceff;
    s.r1[j] = mult * e.kf;
    s.r2[j] = mult * e.kr;
    s.r3[j] = mult * (e.kf * e.dlnkf_dT * e.pf - e.dkr_dT * e.pr);
    s.r4[j] = mult * (e.kf * e.pf - e.kr * e.pr);
  }
  __syncwarp();
  // phase 2: column-parallel accumulation of d(wdot)/d(C_l) and d(wdot)/dT
  for (int j = 0; j < R; ++j) {
    const int type = __ldg(m.rtype + j);
    const double ceff = s.r0[j], kfm = s.r1[j], krm = s.r2[j], dqdT = s.r3[j];
    int spj[8], nuj[8];
#pragma unroll
    for (int sl = 0; sl < 8; ++sl) {
      spj[sl] = __ldg(m.sp + sl * R + j);
      nuj[sl] = __ldg(m.nu + sl * R + j);
    }
    const int e0 = (type != 0) ? __ldg(m.eff_ptr + j) : 0;
    const int e1 = (type != 0) ? __ldg(m.eff_ptr + j + 1) : 0;
#pragma unroll
    for (int c = 0; c < CPL; ++c) {
      const int l = lane + 32 * c;
      double d = 0.0;
      if (l < N) {
        if (type != 0) {
          double eff = 1.0;
          for (int q = e0; q < e1; ++q)
            if (__ldg(m.eff_sp + q) == l) eff += __ldg(m.eff_m1 + q);
          d = eff * ceff;
        }
#pragma unroll
        for (int sl = 0; sl < 4; ++sl) {
          if (spj[sl] == l) {
            const int v = -nuj[sl];
            double p = v * ipow(s.C[l], v - 1);
#pragma unroll
            for (int s2 = 0; s2 < 4; ++s2)
              if (s2 != sl && spj[s2] >= 0) p *= ipow(s.C[spj[s2]], -nuj[s2]);
            d += kfm * p;
          }
          if (spj[sl + 4] == l) {
            const int v = nuj[sl + 4];
            double p = v * ipow(s.C[l], v - 1);
#pragma unroll
            for (int s2 = 0; s2 < 4; ++s2)
              if (s2 != sl && spj[s2 + 4] >= 0) p *= ipow(s.C[spj[s2 + 4]], nuj[s2 + 4]);
            d -= krm * p;
          }
        }
      } else if (l == N) {
        d = dqdT;
      }
      if (l <= N && d != 0.0) {
#pragma unroll
        for (int sl = 0; sl < 8; ++sl)
          if (spj[sl] >= 0) J[spj[sl] * ldj + l] += (double)nuj[sl] * d;
      }
    }
  }
  __syncwarp();
  // species rows: scale to mass units, compute ydot
  double rcp = 0.0, hs = 0.0, drcp = 0.0, cpdot = 0.0;
#pragma unroll
  for (int c = 0; c < CPL; ++c) {
    const int k = lane + 32 * c;
    if (k < N) {
      double w = 0.0;
      const int p0 = __ldg(m.inc_ptr + k), p1 = __ldg(m.inc_ptr + k + 1);
      for (int p = p0; p < p1; ++p) w += __ldg(m.inc_nu + p) * s.r4[__ldg(m.inc_rxn + p)];
      ydot[c] = w * __ldg(m.mw + k) + F[c];
      rcp += y[c] * cpk[c];
      hs += hk[c] * ydot[c];
      drcp += y[c] * dcpk[c];
      cpdot += cpk[c] * ydot[c];
    }
  }
  rcp = warp_sum(rcp);
  hs = warp_sum(hs);
  drcp = warp_sum(drcp);
  cpdot = warp_sum(cpdot);
  double Tdot = 0.0;
#pragma unroll
  for (int c = 0; c < CPL; ++c)
    if (lane + 32 * c == N) Tdot = (F[c] - hs) / rcp;
  Tdot = warp_sum(Tdot);
#pragma unroll
  for (int c = 0; c < CPL; ++c) {
    const int l = lane + 32 * c;
    if (l == N) ydot[c] = Tdot;
    else if (l > N) ydot[c] = 0.0;
  }
  // scale species rows: J[k][l] *= W_k / W_l (l < N), J[k][N] *= W_k  (lane = column l)
  // and the T row: J[N][l] = -(sum_k h_k J[k][l] + (l<N ? Tdot cp_l : cpdot + Tdot drcp)) / rcp
  // h_k and cp_l are needed by every lane: stash mass-specific h in gRT (no longer needed).
#pragma unroll
  for (int c = 0; c < CPL; ++c)
    if (lane + 32 * c < N) s.gRT[lane + 32 * c] = hk[c];
  __syncwarp();
#pragma unroll
  for (int c = 0; c < CPL; ++c) {
    const int l = lane + 32 * c;
    if (l <= N) {
      const double inv_wl = (l < N) ? __ldg(m.inv_mw + l) : 1.0;
      double sum = 0.0;
      for (int k = 0; k < N; ++k) {
        const double v = J[k * ldj + l] * __ldg(m.mw + k) * inv_wl;
        J[k * ldj + l] = v;
        sum += s.gRT[k] * v;
      }
      J[N * ldj + l] = -(sum + ((l < N) ? Tdot * cpk[c] : cpdot + Tdot * drcp)) / rcp;
    }
  }
  __syncwarp();
  return out;
}

template <int CPL>
__device__ __forceinline__ void warp_jac(const DevMech& m, const MechSmem& s, const double (&y)[CPL],
                                         const double (&F)[CPL], double (&ydot)[CPL], double* J, int ldj, int lane) {
  Vec<CPL> a, b;
#pragma unroll
  for (int c = 0; c < CPL; ++c) {
    a.v[c] = y[c];
    b.v[c] = F[c];
  }
  const Vec<CPL> r = warp_jac_v<CPL>(&m, s, a, b, J, ldj, lane);
#pragma unroll
  for (int c = 0; c < CPL; ++c) ydot[c] = r.v[c];
}

}  // namespace b200
