// group_mech.cuh -- mechanism evaluation by a GROUP of G lanes per cell
// (G = 8, 16 or 32; 32 / G cells per warp).
//
// Within a group, lane g owns state components g, g+G, ... (CPL of them) and
// evaluates reactions g, g+G, ...; rates of progress are exchanged through
// per-group shared memory.  All shuffles and barriers use the group's lane
// mask, so the groups of one warp may follow different control paths.
// This is the device side of the reference mechanism interface
// (productionRate / aJacobian / thermo, Source/PeleLMeX_K.H:611,880-885).
#pragma once
#include "mech_dev.cuh"

namespace b200 {

template <int G>
struct Grp {
  unsigned mask;
  int gl;  // lane index within the group
  __device__ __forceinline__ explicit Grp(int lane)
      : mask(G == 32 ? 0xffffffffu : (((1u << G) - 1u) << (lane - lane % G))), gl(lane % G) {}
  __device__ __forceinline__ double sum(double v) const {
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o, G);
    return v;
  }
  __device__ __forceinline__ double maxv(double v) const {
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(mask, v, o, G));
    return v;
  }
  template <typename T>
  __device__ __forceinline__ T bcast(T v, int src) const {
    return __shfl_sync(mask, v, src, G);
  }
  template <typename T>
  __device__ __forceinline__ T up(T v, int d) const {
    return __shfl_up_sync(mask, v, d, G);
  }
  __device__ __forceinline__ bool any(bool b) const { return __any_sync(mask, b); }
  __device__ __forceinline__ void sync() const { __syncwarp(mask); }
};

// Per-group scratch: shared (C, gRT, hRT, q) and global (Jacobian pieces).
struct GrpScratch {
  double* C;    // [Npad] concentrations          (shared)
  double* gRT;  // [Npad] g/RT                    (shared)
  double* hRT;  // [Npad] h/RT, later h (erg/g)   (shared)
  double* q;    // [Rpad] rates of progress       (shared)
  double* r1;   // [Rpad] Jacobian: third-body coefficient   (global)
  double* r2;   // [Rpad] Jacobian: kf * mult                (global)
  double* r3;   // [Rpad] Jacobian: kr * mult                (global)
  double* r4;   // [Rpad] Jacobian: dq/dT                    (global)
};

template <int G, int CPL>
__device__ __forceinline__ double grp_get_T(const Grp<G>& g, const Vec<CPL>& y, int N) {
  double v = 0.0;
#pragma unroll
  for (int c = 0; c < CPL; ++c)
    if (c == N / G) v = y.v[c];
  return g.bcast(v, N % G);
}

template <int G, int CPL>
__device__ __forceinline__ void grp_species(const DevMech& m, const GrpScratch& s, const Grp<G>& g,
                                            const Vec<CPL>& y, double T, double lnT, double (&cpk)[CPL],
                                            double (&hk)[CPL], double (&dcpk)[CPL]) {
#pragma unroll
  for (int c = 0; c < CPL; ++c) {
    const int k = g.gl + G * c;
    cpk[c] = hk[c] = dcpk[c] = 0.0;
    if (k < m.N) {
      double cpR, hRT, sR, dcpR;
      nasa7(m, k, T, lnT, cpR, hRT, sR, dcpR);
      const double iw = __ldg(m.inv_mw + k);
      s.C[k] = y.v[c] * iw;
      s.gRT[k] = hRT - sR;
      s.hRT[k] = hRT;
      cpk[c] = cpR * kRu * iw;
      hk[c] = hRT * kRu * T * iw;
      dcpk[c] = dcpR * kRu * iw;
    }
  }
}

// HP right-hand side of the group's cell.  Out of line: one copy serves
// every call site (instruction-cache footprint).
template <int G, int CPL>
__device__ __noinline__ Vec<CPL> grp_rhs(const DevMech* mp, const GrpScratch s, const Vec<CPL> y, const Vec<CPL> F,
                                         int lane) {
  const DevMech& m = *mp;
  const Grp<G> g(lane);
  const int N = m.N, R = m.R;
  const double T = grp_get_T<G, CPL>(g, y, N);
  const double lnT = log(T), invT = 1.0 / T;
  double cpk[CPL], hk[CPL], dcpk[CPL];
  grp_species<G, CPL>(m, s, g, y, T, lnT, cpk, hk, dcpk);
  double csum = 0.0;
#pragma unroll
  for (int c = 0; c < CPL; ++c)
    if (g.gl + G * c < N) csum += y.v[c] * __ldg(m.inv_mw + g.gl + G * c);
  const double Ctot = g.sum(csum);
  const double lnPRT = log(kPatm / (kRu * T));
  g.sync();
  for (int j = g.gl; j < R; j += G) {
    const RxnEval e = eval_reaction<false>(m, SpView{s.C, s.gRT, s.hRT}, j, T, lnT, invT, Ctot, lnPRT);
    double q = e.kf * e.pf - e.kr * e.pr;
    if (__ldg(m.rtype + j) == 1) q *= e.M;
    s.q[j] = q;
  }
  g.sync();
  Vec<CPL> out;
  double rcp = 0.0, hs = 0.0;
#pragma unroll
  for (int c = 0; c < CPL; ++c) {
    const int k = g.gl + G * c;
    out.v[c] = 0.0;
    if (k < N) {
      double w = 0.0;
      const int p0 = __ldg(m.inc_ptr + k), p1 = __ldg(m.inc_ptr + k + 1);
      for (int p = p0; p < p1; ++p) w += __ldg(m.inc_nu + p) * s.q[__ldg(m.inc_rxn + p)];
      out.v[c] = w * __ldg(m.mw + k) + F.v[c];
      rcp += y.v[c] * cpk[c];
      hs += hk[c] * out.v[c];
    }
  }
  rcp = g.sum(rcp);
  hs = g.sum(hs);
#pragma unroll
  for (int c = 0; c < CPL; ++c)
    if (g.gl + G * c == N) out.v[c] = (F.v[c] - hs) / rcp;
  g.sync();
  return out;
}

// Analytic Jacobian of the HP system, column-major into J (J[col*ldj + row],
// global scratch: lanes read rows of a column contiguously in the solves).
// fy = f(y).  Lane g owns columns g, g+G, ...
template <int G, int CPL>
__device__ __noinline__ void grp_jac(const DevMech* mp, const GrpScratch s, const Vec<CPL> y, const Vec<CPL> fy,
                                     double* J, int ldj, int lane) {
  const DevMech& m = *mp;
  const Grp<G> g(lane);
  const int N = m.N, R = m.R, n = N + 1;
  const double T = grp_get_T<G, CPL>(g, y, N);
  const double lnT = log(T), invT = 1.0 / T;
  double cpk[CPL], hk[CPL], dcpk[CPL];
  grp_species<G, CPL>(m, s, g, y, T, lnT, cpk, hk, dcpk);
  double csum = 0.0;
#pragma unroll
  for (int c = 0; c < CPL; ++c)
    if (g.gl + G * c < N) csum += y.v[c] * __ldg(m.inv_mw + g.gl + G * c);
  const double Ctot = g.sum(csum);
  const double lnPRT = log(kPatm / (kRu * T));
#pragma unroll
  for (int c = 0; c < CPL; ++c) {
    const int l = g.gl + G * c;
    if (l < n)
      for (int i = 0; i < n; ++i) J[l * ldj + i] = 0.0;
  }
  g.sync();
  // phase 1: per-reaction scalars (lane per reaction)
  for (int j = g.gl; j < R; j += G) {
    const RxnEval e = eval_reaction<true>(m, SpView{s.C, s.gRT, s.hRT}, j, T, lnT, invT, Ctot, lnPRT);
    const int type = __ldg(m.rtype + j);
    const double mult = (type == 1) ? e.M : 1.0;
    double ceff = 0.0;
    if (type == 1) ceff = e.kf * e.pf - e.kr * e.pr;
    else if (type >= 2) ceff = e.dkf_dM * (e.pf - (e.kf > 0.0 ? e.kr / e.kf : 0.0) * e.pr);
    s.r1[j] = ceff;
    s.r2[j] = mult * e.kf;
    s.r3[j] = mult * e.kr;
    s.r4[j] = mult * (e.kf * e.dlnkf_dT * e.pf - e.dkr_dT * e.pr);
  }
  __threadfence_block();
  g.sync();
  // phase 2: column-parallel accumulation of d(wdot)/d(C_l) and d(wdot)/dT
  for (int j = 0; j < R; ++j) {
    const int type = __ldg(m.rtype + j);
    const double ceff = s.r1[j], kfm = s.r2[j], krm = s.r3[j], dqdT = s.r4[j];
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
      const int l = g.gl + G * c;
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
          if (spj[sl] >= 0) J[l * ldj + spj[sl]] += (double)nuj[sl] * d;
      }
    }
  }
  // temperature row; ydot = fy
  double rcp = 0.0, drcp = 0.0, cpdot = 0.0;
#pragma unroll
  for (int c = 0; c < CPL; ++c) {
    const int k = g.gl + G * c;
    if (k < N) {
      rcp += y.v[c] * cpk[c];
      drcp += y.v[c] * dcpk[c];
      cpdot += cpk[c] * fy.v[c];
    }
  }
  rcp = g.sum(rcp);
  drcp = g.sum(drcp);
  cpdot = g.sum(cpdot);
  double Tdot = 0.0;
#pragma unroll
  for (int c = 0; c < CPL; ++c)
    if (g.gl + G * c == N) Tdot = fy.v[c];
  Tdot = g.sum(Tdot);
#pragma unroll
  for (int c = 0; c < CPL; ++c)
    if (g.gl + G * c < N) s.hRT[g.gl + G * c] = hk[c];  // mass-specific h for the T row
  g.sync();
#pragma unroll
  for (int c = 0; c < CPL; ++c) {
    const int l = g.gl + G * c;
    if (l <= N) {
      const double inv_wl = (l < N) ? __ldg(m.inv_mw + l) : 1.0;
      double sum = 0.0;
      for (int k = 0; k < N; ++k) {
        const double v = J[l * ldj + k] * __ldg(m.mw + k) * inv_wl;
        J[l * ldj + k] = v;
        sum += s.hRT[k] * v;
      }
      J[l * ldj + N] = -(sum + ((l < N) ? Tdot * cpk[c] : cpdot + Tdot * drcp)) / rcp;
    }
  }
  __threadfence_block();
  g.sync();
}

}  // namespace b200
