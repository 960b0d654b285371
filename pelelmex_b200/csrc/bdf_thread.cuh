// bdf_thread.cuh -- one cell per THREAD: the batched BDF used for mechanisms
// with a compiled species count.
//
// Same algorithm, step for step, as the CPU oracle and the warp-per-cell
// path (CVODE's variable-order BDF in Nordsieck form with modified Newton;
// reference: PelePhysics ReactorCvode denseAJ_direct, absent from the
// snapshot).  What makes it fast on B200:
//   * every thread of a warp walks the SAME reaction table entry at the same
//     time, so mechanism reads are warp-uniform broadcasts and there is no
//     divergence in the right-hand side (the cost that dominates);
//   * the integrator is a resumable state machine.  A warp alternates
//     "RHS rounds", in which every cell that needs a right-hand side gets it
//     at the single call site, and "setup rounds", in which the cells waiting
//     for a new iteration matrix evaluate the analytic Jacobian and factor it
//     together.  Cells of very different stiffness therefore share the warp
//     without serialising each other;
//   * per-cell Jacobians (FP64) and LU factors (FP32) live in a scratch
//     buffer interleaved by thread, so that every matrix access of a warp is
//     one coalesced transaction;
//   * when a cell finishes, its thread takes the next cell from a global
//     atomic queue (warp-aggregated), so the warp stays full until the queue
//     is empty.
// Every loop is bounded; failures end with a per-cell status code.
#pragma once
#include "bdf_group.cuh"

namespace b200 {
namespace tpc {

enum Phase : int {
  kIdle = 0,       // no cell: take one from the queue
  kRhsF0,          // needs f(y0)
  kRhsHin,         // initial step-size iteration needs f(y0 + hg y0')
  kRhsNStart,      // Newton: residual at the predicted state
  kRhsNIter,       // Newton: residual at the current iterate
  kRhsRestart,     // order-1 restart after repeated error-test failures
  kSetup,          // waits for Jacobian (maybe) + LU
  kExhausted       // queue empty, thread retired
};

__device__ __forceinline__ bool needs_rhs(int ph) { return ph >= kRhsF0 && ph <= kRhsRestart; }

// Matrix element (i, j) of this thread in an interleaved scratch array.
template <typename T>
struct IMat {
  T* base;  // scratch + thread id
  long long stride;  // total threads of the launch
  int n;
  __device__ __forceinline__ T& operator()(int i, int j) const { return base[(long long)(i * n + j) * stride]; }
};

// ----------------------------------------------------------- mechanism
// Per-thread concentration / production-rate arrays in shared memory,
// element k of this thread at s[k * ss].
template <bool JAC>
__device__ __forceinline__ RxnEval tpc_eval_reaction(const DevMech& m, int j, double T, double lnT, double invT,
                                                     double Ctot, double lnPRT, const double* sC, int ss,
                                                     const double* g, const double* hR) {
  const int R = m.R;
  RxnEval e;
  const double lnA = __ldg(m.arr + j), b = __ldg(m.arr + R + j), ea = __ldg(m.arr + 2 * R + j);
  const double kinf = exp(lnA + b * lnT - ea * invT);
  const int type = __ldg(m.rtype + j);
  const int flags = __ldg(m.rflags + j);
  double M = 0.0;
  if (type != 0) {
    M = Ctot;
    const int e0 = __ldg(m.eff_ptr + j), e1 = __ldg(m.eff_ptr + j + 1);
    for (int q = e0; q < e1; ++q) M += __ldg(m.eff_m1 + q) * sC[__ldg(m.eff_sp + q) * ss];
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
      const double gg = 1.0 + f1 * f1;
      F = exp(kLn10 * (logFc / gg));
      if (JAC) {
        D = (Pr <= 1e-300) ? 0.0 : -2.0 * logFc * f1 * nn / (gg * gg * den * den);
        const double df1 = (-0.67 * nn + 1.27 * u) / (den * den);
        const double dlogF_dlogFc = 1.0 / gg - logFc * 2.0 * f1 / (gg * gg) * df1;
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
        sg += v * g[k];
        if (JAC) sh += v * hR[k];
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
    if (k >= 0) pf *= ipow(sC[k * ss], -__ldg(m.nu + sl * R + j));
    const int k2 = __ldg(m.sp + (sl + 4) * R + j);
    if (k2 >= 0) pr *= ipow(sC[k2 * ss], __ldg(m.nu + (sl + 4) * R + j));
  }
  e.kf = kf;
  e.kr = kr;
  e.pf = pf;
  e.pr = pr;
  e.dlnkf_dT = dlnkf;
  e.dkr_dT = dkr;
  return e;
}

// HP right-hand side of this thread's cell: out = f(y).
template <int NS>
__device__ __forceinline__ void tpc_rhs(const DevMech& m, const double* y, const double* F, double* out, double* sC,
                                        double* sW, int ss) {
  const double T = y[NS];
  const double lnT = log(T), invT = 1.0 / T;
  double g[NS];
  double Ctot = 0.0, rcp = 0.0;
#pragma unroll
  for (int k = 0; k < NS; ++k) {
    double cpR, hRT, sR, dcpR;
    nasa7(m, k, T, lnT, cpR, hRT, sR, dcpR);
    g[k] = hRT - sR;
    const double iw = __ldg(m.inv_mw + k);
    const double Ck = y[k] * iw;
    sC[k * ss] = Ck;
    sW[k * ss] = 0.0;
    Ctot += Ck;
    rcp += y[k] * cpR * kRu * iw;
  }
  const double lnPRT = log(kPatm / (kRu * T));
  const int R = m.R;
  for (int j = 0; j < R; ++j) {
    const RxnEval e = tpc_eval_reaction<false>(m, j, T, lnT, invT, Ctot, lnPRT, sC, ss, g, nullptr);
    double q = e.kf * e.pf - e.kr * e.pr;
    if (__ldg(m.rtype + j) == 1) q *= e.M;
#pragma unroll
    for (int sl = 0; sl < 8; ++sl) {
      const int k = __ldg(m.sp + sl * R + j);
      if (k >= 0) sW[k * ss] += (double)__ldg(m.nu + sl * R + j) * q;
    }
  }
  double hs = 0.0;
#pragma unroll
  for (int k = 0; k < NS; ++k) {
    double cpR, hRT, sR, dcpR;
    nasa7(m, k, T, lnT, cpR, hRT, sR, dcpR);
    const double yd = sW[k * ss] * __ldg(m.mw + k) + F[k];
    out[k] = yd;
    hs += hRT * kRu * T * __ldg(m.inv_mw + k) * yd;
  }
  out[NS] = (F[NS] - hs) / rcp;
}

// Analytic Jacobian of the HP system at y into J (FP64, interleaved scratch).
// fy = f(y) (the residual the Newton iteration just evaluated).
template <int NS>
__device__ __forceinline__ void tpc_jac(const DevMech& m, const double* y, const double* fy, const IMat<double>& J,
                                        double* sC, double* sW, int ss) {
  constexpr int n = NS + 1;
  const double T = y[NS];
  const double lnT = log(T), invT = 1.0 / T;
  double g[NS], hR[NS];
  double Ctot = 0.0;
#pragma unroll
  for (int k = 0; k < NS; ++k) {
    double cpR, hRT, sR, dcpR;
    nasa7(m, k, T, lnT, cpR, hRT, sR, dcpR);
    g[k] = hRT - sR;
    hR[k] = hRT;
    const double Ck = y[k] * __ldg(m.inv_mw + k);
    sC[k * ss] = Ck;
    sW[k * ss] = 0.0;  // u_k: row sums of the default-efficiency third-body terms
    Ctot += Ck;
  }
  for (int i = 0; i < n * n; ++i) J.base[(long long)i * J.stride] = 0.0;
  const double lnPRT = log(kPatm / (kRu * T));
  const int R = m.R;
  for (int j = 0; j < R; ++j) {
    const RxnEval e = tpc_eval_reaction<true>(m, j, T, lnT, invT, Ctot, lnPRT, sC, ss, g, hR);
    const int type = __ldg(m.rtype + j);
    const double mult = (type == 1) ? e.M : 1.0;
    double ceff = 0.0;
    if (type == 1) ceff = e.kf * e.pf - e.kr * e.pr;
    else if (type >= 2) ceff = e.dkf_dM * (e.pf - (e.kf > 0.0 ? e.kr / e.kf : 0.0) * e.pr);
    const double kfm = mult * e.kf, krm = mult * e.kr;
    const double dqdT = mult * (e.kf * e.dlnkf_dT * e.pf - e.dkr_dT * e.pr);
    int sp[8], nu[8];
#pragma unroll
    for (int sl = 0; sl < 8; ++sl) {
      sp[sl] = __ldg(m.sp + sl * R + j);
      nu[sl] = __ldg(m.nu + sl * R + j);
    }
    // columns touched by the mass-action terms: the reaction's own species
#pragma unroll
    for (int a = 0; a < 8; ++a) {
      if (sp[a] < 0) continue;
      const int ka = sp[a];
      const int va = (a < 4) ? -nu[a] : nu[a];
      double p = va * ipow(sC[ka * ss], va - 1);
#pragma unroll
      for (int s2 = 0; s2 < 4; ++s2) {
        const int o = (a < 4) ? s2 : s2 + 4;
        if (o != a && sp[o] >= 0) p *= ipow(sC[sp[o] * ss], (a < 4) ? -nu[o] : nu[o]);
      }
      const double d = (a < 4) ? kfm * p : -krm * p;
#pragma unroll
      for (int s = 0; s < 8; ++s)
        if (sp[s] >= 0) J(sp[s], ka) += (double)nu[s] * d;
    }
    // temperature column and third-body columns
#pragma unroll
    for (int s = 0; s < 8; ++s) {
      if (sp[s] < 0) continue;
      J(sp[s], NS) += (double)nu[s] * dqdT;
      if (type != 0) sW[sp[s] * ss] += (double)nu[s] * ceff;
    }
    if (type != 0) {
      const int e0 = __ldg(m.eff_ptr + j), e1 = __ldg(m.eff_ptr + j + 1);
      for (int q = e0; q < e1; ++q) {
        const int l = __ldg(m.eff_sp + q);
        const double d = __ldg(m.eff_m1 + q) * ceff;
#pragma unroll
        for (int s = 0; s < 8; ++s)
          if (sp[s] >= 0) J(sp[s], l) += (double)nu[s] * d;
      }
    }
  }
  // add the default-efficiency third-body part, scale to mass units
  for (int k = 0; k < NS; ++k) {
    const double uk = sW[k * ss];
    const double wk = __ldg(m.mw + k);
    for (int l = 0; l < NS; ++l) J(k, l) = (J(k, l) + uk) * wk * __ldg(m.inv_mw + l);
    J(k, NS) = J(k, NS) * wk;
  }
  // temperature row
  // (h_k in sC, cp_k in sW: the concentrations are no longer needed)
  double rcp = 0.0, drcp = 0.0, cpdot = 0.0;
#pragma unroll 1
  for (int k = 0; k < NS; ++k) {
    double cpR, hRT, sR, dcpR;
    nasa7(m, k, T, lnT, cpR, hRT, sR, dcpR);
    const double iw = __ldg(m.inv_mw + k);
    const double cp = cpR * kRu * iw;
    sC[k * ss] = hRT * kRu * T * iw;
    sW[k * ss] = cp;
    rcp += y[k] * cp;
    drcp += y[k] * dcpR * kRu * iw;
    cpdot += cp * fy[k];
  }
  const double Tdot = fy[NS];
#pragma unroll 1
  for (int l = 0; l < n; ++l) {
    double s = 0.0;
    for (int k = 0; k < NS; ++k) s += sC[k * ss] * J(k, l);
    J(NS, l) = -(s + ((l < NS) ? Tdot * sW[l * ss] : cpdot + Tdot * drcp)) / rcp;
  }
}

// LU with partial pivoting (sequential pivots like LAPACK getrf) of
// D (I - gamma J) D^-1 (FP32, D = diag(Dsc)) or I - gamma J (FP64).
template <int n, typename LUT>
__device__ __forceinline__ int tpc_lu_factor(const IMat<double>& J, const IMat<LUT>& A, int* piv, const double* Dsc,
                                             double gamma) {
#pragma unroll 1
  for (int i = 0; i < n; ++i) {
    const double di = (sizeof(LUT) == 4) ? Dsc[i] : 1.0;
#pragma unroll 2
    for (int j = 0; j < n; ++j) {
      const double mij = ((i == j) ? 1.0 : 0.0) - gamma * J(i, j);
      A(i, j) = (LUT)((sizeof(LUT) == 4) ? mij * di / Dsc[j] : mij);
    }
  }
  for (int k = 0; k < n; ++k) {
    int p = k;
    LUT amax = fabs(A(k, k));
    for (int i = k + 1; i < n; ++i) {
      const LUT v = fabs(A(i, k));
      if (v > amax) {
        amax = v;
        p = i;
      }
    }
    piv[k] = p;
    if (!(amax > (LUT)0)) return k + 1;
    if (p != k)
      for (int j = 0; j < n; ++j) {
        const LUT t = A(k, j);
        A(k, j) = A(p, j);
        A(p, j) = t;
      }
    const LUT inv = (LUT)1 / A(k, k);
    for (int i = k + 1; i < n; ++i) {
      const LUT l = A(i, k) * inv;
      A(i, k) = l;
      if (l != (LUT)0)
        for (int j = k + 1; j < n; ++j) A(i, j) -= l * A(k, j);
    }
  }
  return 0;
}

// x := D^-1 (LU)^-1 D x  (x is a local array of n doubles)
template <int n, typename LUT>
__device__ __forceinline__ void tpc_lu_apply(const IMat<LUT>& A, const int* piv, const double* Dsc, double* x) {
  LUT b[n];
#pragma unroll
  for (int i = 0; i < n; ++i) b[i] = (LUT)(x[i] * ((sizeof(LUT) == 4) ? Dsc[i] : 1.0));
  for (int k = 0; k < n; ++k) {
    const int p = piv[k];
    if (p != k) {
      const LUT t = b[k];
      b[k] = b[p];
      b[p] = t;
    }
  }
#pragma unroll 1
  for (int i = 1; i < n; ++i) {
    LUT s = b[i];
#pragma unroll 4
    for (int j = 0; j < i; ++j) s -= A(i, j) * b[j];
    b[i] = s;
  }
#pragma unroll 1
  for (int i = n - 1; i >= 0; --i) {
    LUT s = b[i];
#pragma unroll 4
    for (int j = i + 1; j < n; ++j) s -= A(i, j) * b[j];
    b[i] = s / A(i, i);
  }
#pragma unroll
  for (int i = 0; i < n; ++i) x[i] = (double)b[i] / ((sizeof(LUT) == 4) ? Dsc[i] : 1.0);
}

// Per-thread integrator state.
template <int NS, typename LUT>
struct Cell {
  static constexpr int n = NS + 1;
  double zn[kZn][n];
  double ewt[n], acor[n], ftemp[n], F[n], Dsc[n], yev[n];
  double tau[kZn + 2], tq[6], l[kZn];
  double h, hprime, hscale, eta, etamax, tn, gamma, gammap, gamrat, crate, acnrm, rl1, saved_tq5, gamma_lu;
  double dt, saved_t, delp, hg, hub, hlb, rho_h;
  int q, qprime, L, qwait, nstlp, nstlj, jcur, ncf, nef, nflag, convfail, callSetup, jbad, mnewt, attempt;
  int count1, hnewOK, nstloc, qmax, max_steps, setup_conv;
  int piv[n];
  CellCounters cnt;
};

// ---- Nordsieck / coefficient helpers (same formulas as the oracle) -------
template <int NS, typename LUT>
__device__ __forceinline__ void c_rescale(Cell<NS, LUT>& c) {
  constexpr int n = NS + 1;
  double factor = c.eta;
  for (int j = 1; j <= c.q; ++j) {
#pragma unroll
    for (int i = 0; i < n; ++i) c.zn[j][i] *= factor;
    factor *= c.eta;
  }
  c.h = c.hscale * c.eta;
  c.hscale = c.h;
}

template <int NS, typename LUT>
__device__ __forceinline__ void c_predict(Cell<NS, LUT>& c) {
  constexpr int n = NS + 1;
  c.tn += c.h;
  for (int k = 1; k <= c.q; ++k)
    for (int j = c.q; j >= k; --j)
#pragma unroll
      for (int i = 0; i < n; ++i) c.zn[j - 1][i] += c.zn[j][i];
}

template <int NS, typename LUT>
__device__ __forceinline__ void c_restore(Cell<NS, LUT>& c) {
  constexpr int n = NS + 1;
  c.tn = c.saved_t;
  for (int k = 1; k <= c.q; ++k)
    for (int j = c.q; j >= k; --j)
#pragma unroll
      for (int i = 0; i < n; ++i) c.zn[j - 1][i] -= c.zn[j][i];
}

template <int NS, typename LUT>
__device__ __forceinline__ double c_wrms(const Cell<NS, LUT>& c, const double* v) {
  constexpr int n = NS + 1;
  double s = 0.0;
#pragma unroll
  for (int i = 0; i < n; ++i) {
    const double t = v[i] * c.ewt[i];
    s += t * t;
  }
  return sqrt(s / n);
}

template <int NS, typename LUT>
__device__ __forceinline__ void c_set_bdf(Cell<NS, LUT>& c) {
  const int q = c.q;
  double xi_inv = 1.0, xistar_inv = 1.0;
  c.l[0] = c.l[1] = 1.0;
  for (int i = 2; i <= q; ++i) c.l[i] = 0.0;
  double alpha0 = -1.0, alpha0_hat = -1.0, hsum = c.h;
  if (q > 1) {
    for (int j = 2; j < q; ++j) {
      hsum += c.tau[j - 1];
      xi_inv = c.h / hsum;
      alpha0 -= 1.0 / j;
      for (int i = j; i >= 1; --i) c.l[i] += c.l[i - 1] * xi_inv;
    }
    alpha0 -= 1.0 / q;
    xistar_inv = -c.l[1] - alpha0;
    hsum += c.tau[q - 1];
    xi_inv = c.h / hsum;
    alpha0_hat = -c.l[1] - xi_inv;
    for (int i = q; i >= 1; --i) c.l[i] += c.l[i - 1] * xistar_inv;
  }
  const double A1 = 1.0 - alpha0_hat + alpha0;
  const double A2 = 1.0 + q * A1;
  c.tq[2] = fabs(A1 / (alpha0 * A2));
  c.tq[5] = fabs(A2 * xistar_inv / (c.l[q] * xi_inv));
  if (c.qwait == 1) {
    if (q > 1) {
      const double C = xistar_inv / c.l[q];
      const double A3 = alpha0 + 1.0 / q;
      const double A4 = alpha0_hat + xi_inv;
      const double Cpinv = (1.0 - A4 + A3) / A3;
      c.tq[1] = fabs(C * Cpinv);
    } else {
      c.tq[1] = 1.0;
    }
    hsum += c.tau[q];
    xi_inv = c.h / hsum;
    const double A5 = alpha0 - 1.0 / (q + 1);
    const double A6 = alpha0_hat - xi_inv;
    const double Cppinv = (1.0 - A6 + A5) / A2;
    c.tq[3] = fabs(Cppinv / (xi_inv * (q + 2) * A5));
  }
  c.tq[4] = kNLSCOEF / c.tq[2];
  c.rl1 = 1.0 / c.l[1];
  c.gamma = c.h * c.rl1;
  if (c.cnt.nst == 0) c.gammap = c.gamma;
  c.gamrat = (c.cnt.nst > 0) ? c.gamma / c.gammap : 1.0;
}

template <int NS, typename LUT>
__device__ __forceinline__ void c_increase(Cell<NS, LUT>& c) {
  constexpr int n = NS + 1;
  const int q = c.q;
  for (int i = 0; i <= c.qmax; ++i) c.l[i] = 0.0;
  double alpha1 = 1.0, prod = 1.0, xiold = 1.0, alpha0 = -1.0, hsum = c.hscale;
  c.l[2] = 1.0;
  for (int j = 1; j < q; ++j) {
    hsum += c.tau[j + 1];
    const double xi = hsum / c.hscale;
    prod *= xi;
    alpha0 -= 1.0 / (j + 1);
    alpha1 += 1.0 / xi;
    for (int i = j + 2; i >= 2; --i) c.l[i] = c.l[i] * xiold + c.l[i - 1];
    xiold = xi;
  }
  const double A1 = (-alpha0 - alpha1) / prod;
#pragma unroll
  for (int i = 0; i < n; ++i) c.zn[q + 1][i] = A1 * c.zn[c.qmax][i];
  for (int j = 2; j <= q; ++j)
#pragma unroll
    for (int i = 0; i < n; ++i) c.zn[j][i] += c.l[j] * c.zn[q + 1][i];
}

template <int NS, typename LUT>
__device__ __forceinline__ void c_decrease(Cell<NS, LUT>& c) {
  constexpr int n = NS + 1;
  const int q = c.q;
  for (int i = 0; i <= c.qmax; ++i) c.l[i] = 0.0;
  c.l[2] = 1.0;
  double hsum = 0.0;
  for (int j = 1; j <= q - 2; ++j) {
    hsum += c.tau[j];
    const double xi = hsum / c.hscale;
    for (int i = j + 2; i >= 2; --i) c.l[i] = c.l[i] * xi + c.l[i - 1];
  }
  for (int j = 2; j < q; ++j)
#pragma unroll
    for (int i = 0; i < n; ++i) c.zn[j][i] -= c.l[j] * c.zn[q][i];
}

template <int NS, typename LUT>
__device__ __forceinline__ void c_set_ewt(Cell<NS, LUT>& c, const double* atolv, double rtol) {
  constexpr int n = NS + 1;
#pragma unroll
  for (int i = 0; i < n; ++i) c.ewt[i] = 1.0 / (rtol * fabs(c.zn[0][i]) + atolv[i]);
}

template <int NS, typename LUT>
__device__ __forceinline__ void c_prepare_next(Cell<NS, LUT>& c, double dsm) {
  constexpr int n = NS + 1;
  if (c.etamax == 1.0) {
    c.qwait = c.qwait > 2 ? c.qwait : 2;
    c.qprime = c.q;
    c.hprime = c.h;
    c.eta = 1.0;
    return;
  }
  const double etaq = 1.0 / (pow(kBIAS2 * dsm, 1.0 / c.L) + kADDON);
  if (c.qwait != 0) {
    c.eta = etaq;
    c.qprime = c.q;
  } else {
    c.qwait = 2;
    double etaqm1 = 0.0, etaqp1 = 0.0;
    if (c.q > 1) {
      const double ddn = c_wrms(c, c.zn[c.q]) * c.tq[1];
      etaqm1 = 1.0 / (pow(kBIAS1 * ddn, 1.0 / c.q) + kADDON);
    }
    if (c.q != c.qmax && c.saved_tq5 != 0.0) {
      const double cquot = (c.tq[5] / c.saved_tq5) * pow(c.h / c.tau[2], (double)c.L);
      double t[n];
#pragma unroll
      for (int i = 0; i < n; ++i) t[i] = c.acor[i] - cquot * c.zn[c.qmax][i];
      const double dup = c_wrms(c, t) * c.tq[3];
      etaqp1 = 1.0 / (pow(kBIAS3 * dup, 1.0 / (c.L + 1)) + kADDON);
    }
    const double etam = fmax(etaqm1, fmax(etaq, etaqp1));
    if (etam < kTHRESH) {
      c.eta = 1.0;
      c.qprime = c.q;
    } else if (etam == etaq) {
      c.eta = etaq;
      c.qprime = c.q;
    } else if (etam == etaqm1) {
      c.eta = etaqm1;
      c.qprime = c.q - 1;
    } else {
      c.eta = etaqp1;
      c.qprime = c.q + 1;
#pragma unroll
      for (int i = 0; i < n; ++i) c.zn[c.qmax][i] = c.acor[i];
    }
  }
  if (c.eta < kTHRESH) {
    c.eta = 1.0;
    c.hprime = c.h;
  } else {
    c.eta = fmin(c.eta, c.etamax);
    c.hprime = c.h * c.eta;
  }
}

// Resume points of the state machine.
enum Label : int {
  kLAfterF0 = 0, kLAfterHin, kLStart, kLBeginStep, kLAttempt, kLNlsAttempt, kLAfterNStart, kLAfterSetup,
  kLNewtonIter, kLAfterNIter, kLNlsRecover, kLNlsFail1, kLNlsFail2, kLNlsSuccess, kLAfterRestart
};

// Advance the cell's integrator from resume point `lab` until it needs a
// right-hand side (sets c.yev and returns its phase), a setup (kSetup), or
// finishes (returns kIdle with *status set).  f is the RHS just evaluated.
template <int NS, typename LUT>
__device__ __forceinline__ int c_advance(Cell<NS, LUT>& c, int lab, const double* f, int setup_ier,
                                         const double* atolv, double rtol, const IMat<double>& J,
                                         const IMat<LUT>& A, int* status) {
  constexpr int n = NS + 1;
  for (int guard = 0; guard < 256; ++guard) {
    switch (lab) {
      case kLAfterF0: {
        bool bad = false;
#pragma unroll
        for (int i = 0; i < n; ++i) {
          c.zn[1][i] = f[i];
          bad |= !isfinite(f[i]);
        }
        if (bad) {
          *status = -4;
          return kIdle;
        }
        const double tdist = fabs(c.dt);
        const double tround = kUROUND * fabs(c.dt);
        c.hlb = 100.0 * tround;
        double hinv = 0.0;
#pragma unroll
        for (int i = 0; i < n; ++i) hinv = fmax(hinv, fabs(c.zn[1][i]) / (0.1 * fabs(c.zn[0][i]) + atolv[i]));
        c.hub = 0.1 * tdist;
        if (c.hub * hinv > 1.0) c.hub = 1.0 / hinv;
        c.hg = sqrt(c.hlb * c.hub);
        if (c.hub < c.hlb) {
          c.h = c.hg;  // initial step is the geometric mean
          lab = kLStart;
          c.count1 = -1;
          break;
        }
        c.count1 = 1;
        c.hnewOK = 0;
#pragma unroll
        for (int i = 0; i < n; ++i) c.yev[i] = c.zn[0][i] + c.hg * c.zn[1][i];
        return kRhsHin;
      }
      case kLAfterHin: {
        double t[n];
#pragma unroll
        for (int i = 0; i < n; ++i) t[i] = (f[i] - c.zn[1][i]) / c.hg;
        const double yddnrm = c_wrms(c, t);
        const double hnew = (yddnrm * c.hub * c.hub > 2.0) ? sqrt(2.0 / yddnrm) : sqrt(c.hg * c.hub);
        bool stop = false;
        if (c.hnewOK) {
          c.hg = hnew;
          stop = true;
        } else {
          const double hrat = hnew / c.hg;
          double hn = hnew;
          if (hrat > 0.5 && hrat < 2.0) c.hnewOK = 1;
          if (c.count1 > 1 && hrat > 2.0) {
            hn = c.hg;
            c.hnewOK = 1;
          }
          c.hg = hn;
          c.count1++;
          if (c.count1 > 4) stop = true;
        }
        if (!stop) {
#pragma unroll
          for (int i = 0; i < n; ++i) c.yev[i] = c.zn[0][i] + c.hg * c.zn[1][i];
          return kRhsHin;
        }
        double h0 = 0.5 * c.hg;
        if (h0 < c.hlb) h0 = c.hlb;
        if (h0 > c.hub) h0 = c.hub;
        c.h = h0;
        c.count1 = -1;
        lab = kLStart;
        break;
      }
      case kLStart: {
        const double h0 = c.h;
        c.hscale = c.hprime = h0;
#pragma unroll
        for (int i = 0; i < n; ++i) c.zn[1][i] *= h0;
        c.nstloc = 0;
        lab = kLBeginStep;
        break;
      }
      case kLBeginStep: {
        if (c.cnt.nst > 0) c_set_ewt(c, atolv, rtol);
        if (c.nstloc >= c.max_steps) {
          *status = -1;
          return kIdle;
        }
        c.saved_t = c.tn;
        c.ncf = c.nef = 0;
        c.nflag = kFirstCall;
        if (c.cnt.nst > 0 && c.hprime != c.h) {
          if (c.qprime != c.q) {
            if (c.qprime - c.q == 1) c_increase(c);
            else if (c.qprime - c.q == -1) c_decrease(c);
            c.q = c.qprime;
            c.L = c.q + 1;
            c.qwait = c.L;
          }
          c_rescale(c);
        }
        lab = kLAttempt;
        break;
      }
      case kLAttempt: {
        c_predict(c);
        c_set_bdf(c);
        c.convfail = (c.nflag == kFirstCall || c.nflag == kPrevErrFail) ? kNoFailures : kFailOther;
        c.callSetup = (c.nflag == kPrevConvFail) || (c.nflag == kPrevErrFail) || (c.cnt.nst == 0) ||
                      (c.cnt.nst >= c.nstlp + kMSBP) || (fabs(c.gamrat - 1.0) > kDGMAX_LSETUP);
        c.jbad = 0;
        c.attempt = 0;
        lab = kLNlsAttempt;
        break;
      }
      case kLNlsAttempt: {
#pragma unroll
        for (int i = 0; i < n; ++i) {
          c.acor[i] = 0.0;
          c.yev[i] = c.zn[0][i];
        }
        return kRhsNStart;
      }
      case kLAfterNStart: {
#pragma unroll
        for (int i = 0; i < n; ++i) c.ftemp[i] = f[i];
        if (c.callSetup) {
          c.setup_conv = c.jbad ? kFailBadJ : c.convfail;
          return kSetup;
        }
        c.mnewt = 0;
        c.delp = 0.0;
        lab = kLNewtonIter;
        break;
      }
      case kLAfterSetup: {
        c.callSetup = 0;
        if (setup_ier) {
          lab = kLNlsFail2;
          break;
        }
        c.mnewt = 0;
        c.delp = 0.0;
        lab = kLNewtonIter;
        break;
      }
      case kLNewtonIter: {
        c.cnt.nni++;
        double dl[n];
#pragma unroll
        for (int i = 0; i < n; ++i) dl[i] = -(c.rl1 * c.zn[1][i] + c.acor[i] - c.gamma * c.ftemp[i]);
        // solve (I - gamma_lu J) x = dl; FP32 factor + one FP64 refinement step
        double x[n];
#pragma unroll
        for (int i = 0; i < n; ++i) x[i] = dl[i];
        tpc_lu_apply<n, LUT>(A, c.piv, c.Dsc, x);
        if (sizeof(LUT) == 4) {
          double r[n];
#pragma unroll 1
          for (int i = 0; i < n; ++i) {
            double s = 0.0;
#pragma unroll 4
            for (int j = 0; j < n; ++j) s += J(i, j) * x[j];
            r[i] = dl[i] - (x[i] - c.gamma_lu * s);
          }
          tpc_lu_apply<n, LUT>(A, c.piv, c.Dsc, r);
#pragma unroll
          for (int i = 0; i < n; ++i) x[i] += r[i];
        }
        if (c.gamrat != 1.0) {
          const double sc = 2.0 / (1.0 + c.gamrat);
#pragma unroll
          for (int i = 0; i < n; ++i) x[i] *= sc;
        }
#pragma unroll
        for (int i = 0; i < n; ++i) c.acor[i] += x[i];
        const double del = c_wrms(c, x);
        if (c.mnewt > 0) c.crate = fmax(kCRDOWN * c.crate, del / c.delp);
        const double dcon = del * fmin(1.0, c.crate) / c.tq[4];
        if (dcon <= 1.0) {
          c.acnrm = (c.mnewt == 0) ? del : c_wrms(c, c.acor);
          c.jcur = 0;
          lab = kLNlsSuccess;
          break;
        }
        if ((c.mnewt >= 1 && del > kRDIV * c.delp) || !(del == del) || c.mnewt + 1 >= kMAXCOR) {
          lab = kLNlsRecover;
          break;
        }
        c.delp = del;
        c.mnewt++;
#pragma unroll
        for (int i = 0; i < n; ++i) c.yev[i] = c.zn[0][i] + c.acor[i];
        return kRhsNIter;
      }
      case kLAfterNIter: {
#pragma unroll
        for (int i = 0; i < n; ++i) c.ftemp[i] = f[i];
        lab = kLNewtonIter;
        break;
      }
      case kLNlsRecover: {
        if (!c.jcur && c.attempt < 3) {
          c.callSetup = 1;
          c.jbad = 1;
          c.attempt++;
          lab = kLNlsAttempt;
          break;
        }
        lab = kLNlsFail1;
        break;
      }
      case kLNlsFail1:
      case kLNlsFail2: {
        c.cnt.ncfn++;
        c_restore(c);
        c.ncf++;
        c.etamax = 1.0;
        if (c.ncf == kMXNCF) {
          *status = (lab == kLNlsFail2) ? -5 : -3;
          return kIdle;
        }
        c.eta = kETACF;
        c.nflag = kPrevConvFail;
        c_rescale(c);
        lab = kLAttempt;
        break;
      }
      case kLNlsSuccess: {
        const double dsm = c.acnrm * c.tq[2];
        if (dsm <= 1.0) {
          // complete the step
          c.cnt.nst++;
          for (int i = c.q; i >= 2; --i) c.tau[i] = c.tau[i - 1];
          if (c.q == 1 && c.cnt.nst > 1) c.tau[2] = c.tau[1];
          c.tau[1] = c.h;
          for (int j = 0; j <= c.q; ++j)
#pragma unroll
            for (int i = 0; i < n; ++i) c.zn[j][i] += c.l[j] * c.acor[i];
          c.qwait--;
          if (c.qwait == 1 && c.q != c.qmax) {
#pragma unroll
            for (int i = 0; i < n; ++i) c.zn[c.qmax][i] = c.acor[i];
            c.saved_tq5 = c.tq[5];
          }
          c_prepare_next(c, dsm);
          c.etamax = (c.cnt.nst <= kSMALL_NST) ? kETAMX2 : kETAMX3;
          c.nstloc++;
          if (c.tn - c.dt >= 0.0) {
            *status = 0;
            return kIdle;
          }
          lab = kLBeginStep;
          break;
        }
        c.nef++;
        c.cnt.netf++;
        c.nflag = kPrevErrFail;
        c_restore(c);
        if (c.nef == kMXNEF) {
          *status = -2;
          return kIdle;
        }
        c.etamax = 1.0;
        if (c.nef <= kMXNEF1) {
          c.eta = 1.0 / (pow(kBIAS2 * dsm, 1.0 / c.L) + kADDON);
          c.eta = fmax(kETAMIN, c.eta);
          if (c.nef >= kSMALL_NEF) c.eta = fmin(c.eta, kETAMXF);
          c_rescale(c);
          lab = kLAttempt;
          break;
        }
        if (c.q > 1) {
          c.eta = kETAMIN;
          c_decrease(c);
          c.L = c.q;
          c.q--;
          c.qwait = c.L;
          c_rescale(c);
          lab = kLAttempt;
          break;
        }
        c.eta = kETAMIN;
        c.h *= c.eta;
        c.hscale = c.h;
        c.qwait = kLONG_WAIT;
#pragma unroll
        for (int i = 0; i < n; ++i) c.yev[i] = c.zn[0][i];
        return kRhsRestart;
      }
      case kLAfterRestart: {
#pragma unroll
        for (int i = 0; i < n; ++i) c.zn[1][i] = c.h * f[i];
        lab = kLAttempt;
        break;
      }
      default:
        *status = -3;
        return kIdle;
    }
  }
  *status = -3;  // unreachable in practice: the state machine never loops this long without an RHS
  return kIdle;
}

// Start a cell: y (n) already loaded into zn[0]; sets up the counters and asks for f(y0).
template <int NS, typename LUT>
__device__ __forceinline__ int c_begin(Cell<NS, LUT>& c, const double* atolv, double rtol, double dt, int qmax,
                                       int max_steps) {
  constexpr int n = NS + 1;
  c.tn = 0.0;
  c.dt = dt;
  c.cnt = CellCounters{0, 0, 0, 0, 0, 0, 0};
  c.nstlp = c.nstlj = 0;
  c.q = c.qprime = 1;
  c.L = 2;
  c.qwait = c.L;
  c.etamax = kETAMX1;
  c.saved_tq5 = 0.0;
  c.crate = 1.0;
  c.jcur = 0;
  c.gammap = c.gamma = 1.0;
  c.gamrat = 1.0;
  c.qmax = qmax;
  c.max_steps = max_steps;
#pragma unroll
  for (int i = 0; i < kZn + 2; ++i) c.tau[i] = 0.0;
#pragma unroll
  for (int i = 0; i < 6; ++i) c.tq[i] = 0.0;
#pragma unroll
  for (int j = 1; j < kZn; ++j)
#pragma unroll
    for (int i = 0; i < n; ++i) c.zn[j][i] = 0.0;
  c_set_ewt(c, atolv, rtol);
#pragma unroll
  for (int i = 0; i < n; ++i) c.yev[i] = c.zn[0][i];
  return kRhsF0;
}

// Setup (lsetup): maybe refresh J at y = zn[0] (with f = ftemp), then factor.
template <int NS, typename LUT>
__device__ __forceinline__ int c_setup(Cell<NS, LUT>& c, const DevMech& m, const IMat<double>& J, const IMat<LUT>& A,
                                       double* sC, double* sW, int ss) {
  constexpr int n = NS + 1;
  const double dgamma = fabs(c.gamma / c.gammap - 1.0);
  const bool jbad = (c.cnt.nst == 0) || (c.cnt.nst >= c.nstlj + kMSBJ) ||
                    (c.setup_conv == kFailBadJ && dgamma < kDGMAX_JBAD) || (c.setup_conv == kFailOther);
  if (jbad) {
    tpc_jac<NS>(m, c.yev, c.ftemp, J, sC, sW, ss);
    c.cnt.nje++;
    c.nstlj = c.cnt.nst;
    c.jcur = 1;
  } else {
    c.jcur = 0;
  }
#pragma unroll
  for (int i = 0; i < n; ++i) c.Dsc[i] = c.ewt[i];
  const int ier = tpc_lu_factor<n, LUT>(J, A, c.piv, c.Dsc, c.gamma);
  c.cnt.nlu++;
  c.gamma_lu = c.gamma;
  c.gamrat = 1.0;
  c.gammap = c.gamma;
  c.crate = 1.0;
  c.nstlp = c.cnt.nst;
  return ier;
}

}  // namespace tpc
}  // namespace b200
