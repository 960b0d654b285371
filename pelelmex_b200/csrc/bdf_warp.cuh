// bdf_warp.cuh -- one cell per warp: variable-order BDF with modified Newton,
// the integrator inside ReactorBase::react (reference: PelePhysics
// ReactorCvode + SUNDIALS CVODE, denseAJ_direct; absent from the snapshot).
//
// The algorithm is CVODE's published BDF in Nordsieck form, step for step the
// same decisions as the CPU oracle (order/step selection, WRMS error test,
// Jacobian and iteration-matrix reuse, Newton convergence-rate test), so that
// both produce the same step sequence up to round-off.  B200-specific parts:
//   * state vectors live in registers, lane k holding component k (k + 32 for
//     CPL = 2); all step-control scalars are warp-uniform;
//   * the analytic Jacobian is kept in FP64 in per-warp shared memory;
//   * the Newton matrix M = I - gamma J is scaled by the error weights,
//     D M D^-1 with D = diag(ewt), so its entries are O(1) in tolerance units,
//     factored in FP32 (LU with partial pivoting, lanes over columns), and each
//     solve takes one step of FP64 iterative refinement against the FP64 J
//     (or the matrix is factored in FP64 when LUT = double).
// Every loop has a hard bound (max_steps, Newton/failure caps); failures end
// with a status code, never a trap.
#pragma once
#include "mech_dev.cuh"

namespace b200 {

constexpr int kQmaxLim = 5;
constexpr int kZn = kQmaxLim + 1;  // Nordsieck columns 0..5

// CVODE step-control constants (CVODE math chapter / cvode.c defaults)
constexpr double kETAMX1 = 10000.0, kETAMX2 = 10.0, kETAMX3 = 10.0, kETAMXF = 0.2, kETAMIN = 0.1;
constexpr double kETACF = 0.25, kADDON = 1e-6, kBIAS1 = 6.0, kBIAS2 = 6.0, kBIAS3 = 10.0;
constexpr double kTHRESH = 1.5, kCRDOWN = 0.3, kDGMAX_LSETUP = 0.3, kRDIV = 2.0, kDGMAX_JBAD = 0.2;
constexpr double kNLSCOEF = 0.1, kUROUND = 2.220446049250313e-16;
constexpr int kSMALL_NST = 10, kMXNCF = 10, kMXNEF = 7, kMXNEF1 = 3, kSMALL_NEF = 2, kLONG_WAIT = 10;
constexpr int kMAXCOR = 3, kMSBP = 20, kMSBJ = 51;

enum { kFirstCall = 0, kPrevConvFail = 1, kPrevErrFail = 2 };
enum { kNoFailures = 0, kFailBadJ = 1, kFailOther = 2 };

// a[c] for a runtime c < CPL without dynamic register indexing
template <int CPL, typename T>
__device__ __forceinline__ T pick(const T (&a)[CPL], int c) {
  T v = a[0];
#pragma unroll
  for (int cc = 1; cc < CPL; ++cc)
    if (cc == c) v = a[cc];
  return v;
}

struct CellCounters {
  int nst, nfe, nje, nlu, netf, ncfn, nni;
};

// LU with partial pivoting of the n x n matrix D (I - gamma J) D^-1 (D from
// Dsc; D = I for the FP64 variant), formed from the FP64 Jacobian J into LU.
// Lanes own columns for the row operations and rows for the pivot search.
// Returns 0, or k+1 when pivot k is zero (singular).  Out of line so that one
// copy of the code serves every call site (instruction-cache footprint).
template <typename LUT>
__device__ __noinline__ int lu_factor_f(const double* J, int ldj, LUT* LU, int ldl, int* perm, const double* Dsc,
                                        int n, double gamma, int lane) {
  for (int i = 0; i < n; ++i) {
    const double di = Dsc[i];
    for (int j = lane; j < n; j += 32) {
      const double mij = ((i == j) ? 1.0 : 0.0) - gamma * J[i * ldj + j];
      LU[i * ldl + j] = (LUT)((sizeof(LUT) == 4) ? mij * di / Dsc[j] : mij);
    }
  }
  for (int i = lane; i < n; i += 32) perm[i] = i;
  __syncwarp();
  int info = 0;
  for (int k = 0; k < n; ++k) {
    LUT best = (LUT)-1;
    int bi = k;
    for (int i = k + lane; i < n; i += 32) {
      const LUT v = fabs(LU[i * ldl + k]);
      if (v > best) {
        best = v;
        bi = i;
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const LUT ov = __shfl_xor_sync(kFull, best, o);
      const int oi = __shfl_xor_sync(kFull, bi, o);
      if (ov > best || (ov == best && oi < bi)) {
        best = ov;
        bi = oi;
      }
    }
    if (!(best > (LUT)0)) {  // zero (or NaN) pivot: singular
      info = k + 1;
      break;
    }
    if (bi != k) {
      for (int j = lane; j < n; j += 32) {
        const LUT t = LU[k * ldl + j];
        LU[k * ldl + j] = LU[bi * ldl + j];
        LU[bi * ldl + j] = t;
      }
      if (lane == 0) {
        const int t = perm[k];
        perm[k] = perm[bi];
        perm[bi] = t;
      }
    }
    __syncwarp();
    const LUT inv = (LUT)1 / LU[k * ldl + k];
    for (int i = k + 1 + lane; i < n; i += 32) LU[i * ldl + k] *= inv;
    __syncwarp();
    for (int j = k + 1 + lane; j < n; j += 32) {
      const LUT ukj = LU[k * ldl + j];
      for (int i = k + 1; i < n; ++i) LU[i * ldl + j] -= LU[i * ldl + k] * ukj;
    }
    __syncwarp();
  }
  __syncwarp();
  return info;
}

// x := (D^-1 (LU)^-1 D) x for the factorization above (x distributed over lanes).
template <int CPL, typename LUT>
__device__ __forceinline__ Vec<CPL> lu_apply(const LUT* LU, int ldl, const int* perm, const double* Dsc, int n,
                                             Vec<CPL> x, int lane) {
  LUT b[CPL];
#pragma unroll
  for (int c = 0; c < CPL; ++c) {
    const int i = lane + 32 * c;
    const int src = (i < n) ? perm[i] : 0;
    LUT v = (LUT)0;
#pragma unroll
    for (int cc = 0; cc < CPL; ++cc) {
      const int ii = lane + 32 * cc;
      const double t = __shfl_sync(kFull, x.v[cc] * ((ii < n) ? Dsc[ii] : 1.0), src & 31);
      if ((src >> 5) == cc) v = (LUT)t;
    }
    b[c] = (i < n) ? v : (LUT)0;
  }
  for (int k = 0; k < n; ++k) {
    const LUT xk = __shfl_sync(kFull, pick<CPL>(b, k >> 5), k & 31);
#pragma unroll
    for (int c = 0; c < CPL; ++c) {
      const int i = lane + 32 * c;
      if (i > k && i < n) b[c] -= LU[i * ldl + k] * xk;
    }
  }
  for (int k = n - 1; k >= 0; --k) {
    const LUT xk = __shfl_sync(kFull, pick<CPL>(b, k >> 5), k & 31) / LU[k * ldl + k];
#pragma unroll
    for (int c = 0; c < CPL; ++c) {
      const int i = lane + 32 * c;
      if (i == k) b[c] = xk;
      else if (i < k) b[c] -= LU[i * ldl + k] * xk;
    }
  }
  Vec<CPL> out;
#pragma unroll
  for (int c = 0; c < CPL; ++c) {
    const int i = lane + 32 * c;
    out.v[c] = (i < n) ? (double)b[c] / Dsc[i] : 0.0;
  }
  return out;
}

// Solve (I - gamma J) x = b with the factorization above.  FP32 factor: one
// FP64 iterative-refinement step, residual b - (I - gamma J) x from the FP64 J.
template <int CPL, typename LUT>
__device__ __noinline__ Vec<CPL> lsolve_f(const LUT* LU, int ldl, const int* perm, const double* Dsc, const double* J,
                                          int ldj, double gamma, int n, Vec<CPL> b, int lane) {
  Vec<CPL> x = lu_apply<CPL, LUT>(LU, ldl, perm, Dsc, n, b, lane);
  if (sizeof(LUT) == 8) return x;
  Vec<CPL> r;
#pragma unroll
  for (int c = 0; c < CPL; ++c) r.v[c] = 0.0;
  for (int j = 0; j < n; ++j) {
    const double xj = __shfl_sync(kFull, pick<CPL>(x.v, j >> 5), j & 31);
#pragma unroll
    for (int c = 0; c < CPL; ++c) {
      const int i = lane + 32 * c;
      if (i < n) r.v[c] += J[i * ldj + j] * xj;
    }
  }
#pragma unroll
  for (int c = 0; c < CPL; ++c) r.v[c] = (lane + 32 * c < n) ? b.v[c] - (x.v[c] - gamma * r.v[c]) : 0.0;
  r = lu_apply<CPL, LUT>(LU, ldl, perm, Dsc, n, r, lane);
#pragma unroll
  for (int c = 0; c < CPL; ++c) x.v[c] += r.v[c];
  return x;
}

template <int CPL, typename LUT>
struct WarpBdf {
  const DevMech* m;
  MechSmem ms;
  double* J;  // [n][ldj]
  int ldj;
  LUT* LU;    // [n][ldl]
  int ldl;
  int* perm;  // [n]
  int lane, n, qmax;
  double rtol;

  double zn[kZn][CPL];
  double ewt[CPL], acor[CPL], y[CPL], ftemp[CPL], F[CPL], tmp[CPL];
  double* atolv;  // [n] per-warp shared memory: absolute tolerances
  double* Dsc;    // [n] per-warp shared memory: row/column scaling of the factored matrix
  // Small warp-uniform arrays are held lane-distributed (lane i holds element i)
  // to keep them out of every lane's registers: tau[1..q+1] step history,
  // tq[1..5] error-test coefficients, l[0..q] Nordsieck corrector coefficients.
  double tau_r, tq_r, l_r;
  double h, hprime, hscale, eta, etamax, tn, gamma, gammap, gamrat, crate, acnrm, rl1, saved_tq5;
  double gamma_lu;  // gamma the current factorization was built with
  double tq2_, tq4_;  // tq[2] (error test) and tq[4] (Newton test) of the current step
  int q, qprime, L, qwait, nstlp, nstlj, jcur;
  CellCounters cnt;

  __device__ __forceinline__ bool active(int c) const { return lane + 32 * c < n; }

  __device__ __forceinline__ double wrms(const double (&v)[CPL]) const {
    double s = 0.0;
#pragma unroll
    for (int c = 0; c < CPL; ++c) {
      const double t = v[c] * ewt[c];
      s += t * t;
    }
    return sqrt(warp_sum(s) / n);
  }

  __device__ __forceinline__ void f_eval(const double (&yy)[CPL], double (&out)[CPL]) {
    warp_rhs<CPL>(*m, ms, yy, F, out, lane);
    cnt.nfe++;
  }

  __device__ __forceinline__ void set_ewt(const double (&v)[CPL]) {
#pragma unroll
    for (int c = 0; c < CPL; ++c) ewt[c] = active(c) ? 1.0 / (rtol * fabs(v[c]) + ld_atol(c)) : 0.0;
  }

  __device__ __forceinline__ void rescale() {
    double factor = eta;
#pragma unroll
    for (int j = 1; j < kZn; ++j) {
      if (j <= q) {
#pragma unroll
        for (int c = 0; c < CPL; ++c) zn[j][c] *= factor;
        factor *= eta;
      }
    }
    h = hscale * eta;
    hscale = h;
  }

  __device__ __forceinline__ void predict() {
    tn += h;
#pragma unroll
    for (int k = 1; k < kZn; ++k)
#pragma unroll
      for (int j = kZn - 1; j >= 1; --j)
        if (k <= q && j <= q && j >= k)
#pragma unroll
          for (int c = 0; c < CPL; ++c) zn[j - 1][c] += zn[j][c];
  }

  __device__ __forceinline__ void restore(double saved_t) {
    tn = saved_t;
#pragma unroll
    for (int k = 1; k < kZn; ++k)
#pragma unroll
      for (int j = kZn - 1; j >= 1; --j)
        if (k <= q && j <= q && j >= k)
#pragma unroll
          for (int c = 0; c < CPL; ++c) zn[j - 1][c] -= zn[j][c];
  }

  __device__ __forceinline__ double tau_at(int i) const { return __shfl_sync(kFull, tau_r, i); }
  __device__ __forceinline__ double l_at(int i) const { return __shfl_sync(kFull, l_r, i); }
  __device__ __forceinline__ double tq_at(int i) const { return __shfl_sync(kFull, tq_r, i); }
  __device__ __forceinline__ double ld_atol(int c) const { return active(c) ? atolv[lane + 32 * c] : 0.0; }

  __device__ __forceinline__ void set_bdf() {
    double xi_inv = 1.0, xistar_inv = 1.0;
    l_r = (lane <= 1) ? 1.0 : 0.0;
    double alpha0 = -1.0, alpha0_hat = -1.0, hsum = h;
    double l1 = 1.0;
    if (q > 1) {
      for (int j = 2; j < q; ++j) {
        hsum += tau_at(j - 1);
        xi_inv = h / hsum;
        alpha0 -= 1.0 / j;
        // l[i] += l[i-1] * xi_inv for i = j..1 (old values): one lane-parallel update
        const double up = __shfl_up_sync(kFull, l_r, 1);
        if (lane >= 1 && lane <= j) l_r += up * xi_inv;
      }
      alpha0 -= 1.0 / q;
      l1 = l_at(1);
      xistar_inv = -l1 - alpha0;
      hsum += tau_at(q - 1);
      xi_inv = h / hsum;
      alpha0_hat = -l1 - xi_inv;
      const double up = __shfl_up_sync(kFull, l_r, 1);
      if (lane >= 1 && lane <= q) l_r += up * xistar_inv;
      l1 = l_at(1);
    }
    // error-test coefficients (lane i keeps tq[i])
    const double lq = l_at(q);
    const double A1 = 1.0 - alpha0_hat + alpha0;
    const double A2 = 1.0 + q * A1;
    const double tq2 = fabs(A1 / (alpha0 * A2));
    const double tq5 = fabs(A2 * xistar_inv / (lq * xi_inv));
    if (lane == 2) tq_r = tq2;
    if (lane == 5) tq_r = tq5;
    if (qwait == 1) {
      double tq1;
      if (q > 1) {
        const double C = xistar_inv / lq;
        const double A3 = alpha0 + 1.0 / q;
        const double A4 = alpha0_hat + xi_inv;
        const double Cpinv = (1.0 - A4 + A3) / A3;
        tq1 = fabs(C * Cpinv);
      } else {
        tq1 = 1.0;
      }
      hsum += tau_at(q);
      const double xi2 = h / hsum;
      const double A5 = alpha0 - 1.0 / (q + 1);
      const double A6 = alpha0_hat - xi2;
      const double Cppinv = (1.0 - A6 + A5) / A2;
      const double tq3 = fabs(Cppinv / (xi2 * (q + 2) * A5));
      if (lane == 1) tq_r = tq1;
      if (lane == 3) tq_r = tq3;
    }
    if (lane == 4) tq_r = kNLSCOEF / tq2;
    tq2_ = tq2;
    tq4_ = kNLSCOEF / tq2;
    rl1 = 1.0 / l1;
    gamma = h * rl1;
    if (cnt.nst == 0) gammap = gamma;
    gamrat = (cnt.nst > 0) ? gamma / gammap : 1.0;
  }

  __device__ __forceinline__ void zn_get(int j, double (&out)[CPL]) const {
#pragma unroll
    for (int c = 0; c < CPL; ++c) {
      double v = 0.0;
#pragma unroll
      for (int k = 0; k < kZn; ++k)
        if (k == j) v = zn[k][c];
      out[c] = v;
    }
  }
  __device__ __forceinline__ void zn_set(int j, const double (&in)[CPL]) {
#pragma unroll
    for (int k = 0; k < kZn; ++k)
      if (k == j)
#pragma unroll
        for (int c = 0; c < CPL; ++c) zn[k][c] = in[c];
  }

  __device__ __forceinline__ void increase_order() {
    double alpha1 = 1.0, prod = 1.0, xiold = 1.0, alpha0 = -1.0, hsum = hscale;
    l_r = (lane == 2) ? 1.0 : 0.0;
    for (int j = 1; j < q; ++j) {
      hsum += tau_at(j + 1);
      const double xi = hsum / hscale;
      prod *= xi;
      alpha0 -= 1.0 / (j + 1);
      alpha1 += 1.0 / xi;
      // l[i] = l[i] * xiold + l[i-1] for i = j+2..2 (old values)
      const double up = __shfl_up_sync(kFull, l_r, 1);
      if (lane >= 2 && lane <= j + 2) l_r = l_r * xiold + up;
      xiold = xi;
    }
    const double A1 = (-alpha0 - alpha1) / prod;
    double sv[CPL];
    zn_get(qmax, sv);
#pragma unroll
    for (int c = 0; c < CPL; ++c) sv[c] *= A1;
    zn_set(q + 1, sv);
#pragma unroll
    for (int j = 2; j < kZn; ++j) {
      const double lj = l_at(j);
      if (j <= q)
#pragma unroll
        for (int c = 0; c < CPL; ++c) zn[j][c] += lj * sv[c];
    }
  }

  __device__ __forceinline__ void decrease_order() {
    l_r = (lane == 2) ? 1.0 : 0.0;
    double hsum = 0.0;
    for (int j = 1; j <= q - 2; ++j) {
      hsum += tau_at(j);
      const double xi = hsum / hscale;
      const double up = __shfl_up_sync(kFull, l_r, 1);
      if (lane >= 2 && lane <= j + 2) l_r = l_r * xi + up;
    }
    double zq[CPL];
    zn_get(q, zq);
#pragma unroll
    for (int j = 2; j < kZn; ++j) {
      const double lj = l_at(j);
      if (j < q)
#pragma unroll
        for (int c = 0; c < CPL; ++c) zn[j][c] -= lj * zq[c];
    }
  }

  // ---------------------------------------------------------- linear algebra
  // Factor D (I - gamma J) D^-1 with D = diag(ewt) (LUT = float) or I - gamma J (double).
  __device__ __forceinline__ int lu_factor() {
#pragma unroll
    for (int c = 0; c < CPL; ++c)
      if (active(c)) Dsc[lane + 32 * c] = (sizeof(LUT) == 4) ? ewt[c] : 1.0;
    __syncwarp();
    gamma_lu = gamma;
    cnt.nlu++;
    return lu_factor_f<LUT>(J, ldj, LU, ldl, perm, Dsc, n, gamma, lane);
  }

  // Solve (I - gamma_lu J) x = b in place.
  __device__ __forceinline__ void lsolve(double (&x)[CPL]) {
    Vec<CPL> b;
#pragma unroll
    for (int c = 0; c < CPL; ++c) b.v[c] = x[c];
    const Vec<CPL> r = lsolve_f<CPL, LUT>(LU, ldl, perm, Dsc, J, ldj, gamma_lu, n, b, lane);
#pragma unroll
    for (int c = 0; c < CPL; ++c) x[c] = r.v[c];
  }

  // ------------------------------------------------------------ Newton
  __device__ __forceinline__ int lsetup(int convfail) {
    const double dgamma = fabs(gamma / gammap - 1.0);
    const bool jbad = (cnt.nst == 0) || (cnt.nst >= nstlj + kMSBJ) ||
                      (convfail == kFailBadJ && dgamma < kDGMAX_JBAD) || (convfail == kFailOther);
    if (jbad) {
      warp_jac<CPL>(*m, ms, y, F, tmp, J, ldj, lane);
      cnt.nje++;
      nstlj = cnt.nst;
      jcur = 1;
    } else {
      jcur = 0;
    }
    const int ier = lu_factor();
    gamrat = 1.0;
    gammap = gamma;
    crate = 1.0;
    nstlp = cnt.nst;
    return ier;
  }

  // 0 converged, 1 recoverable failure, 2 singular matrix
  __device__ __forceinline__ int nls(int nflag) {
    const int convfail = (nflag == kFirstCall || nflag == kPrevErrFail) ? kNoFailures : kFailOther;
    bool callSetup = (nflag == kPrevConvFail) || (nflag == kPrevErrFail) || (cnt.nst == 0) ||
                     (cnt.nst >= nstlp + kMSBP) || (fabs(gamrat - 1.0) > kDGMAX_LSETUP);
    bool jbad = false;
    for (int attempt = 0; attempt < 4; ++attempt) {
#pragma unroll
      for (int c = 0; c < CPL; ++c) {
        acor[c] = 0.0;
        y[c] = zn[0][c];
      }
      f_eval(y, ftemp);
      if (callSetup) {
        const int ier = lsetup(jbad ? kFailBadJ : convfail);
        callSetup = false;
        if (ier) return 2;
      }
      double delp = 0.0;
      int ret = 1;
      for (int mm = 0; mm < kMAXCOR; ++mm) {
        cnt.nni++;
        double dl[CPL];
#pragma unroll
        for (int c = 0; c < CPL; ++c) dl[c] = -(rl1 * zn[1][c] + acor[c] - gamma * ftemp[c]);
        lsolve(dl);
        if (gamrat != 1.0) {
          const double sc = 2.0 / (1.0 + gamrat);
#pragma unroll
          for (int c = 0; c < CPL; ++c) dl[c] *= sc;
        }
#pragma unroll
        for (int c = 0; c < CPL; ++c) acor[c] += dl[c];
        const double del = wrms(dl);
        if (mm > 0) crate = fmax(kCRDOWN * crate, del / delp);
        const double dcon = del * fmin(1.0, crate) / tq4_;
        if (dcon <= 1.0) {
          acnrm = (mm == 0) ? del : wrms(acor);
          ret = 0;
          break;
        }
        if (mm >= 1 && del > kRDIV * delp) break;
        if (!(del == del)) break;  // NaN
        delp = del;
        if (mm + 1 >= kMAXCOR) break;
#pragma unroll
        for (int c = 0; c < CPL; ++c) y[c] = zn[0][c] + acor[c];
        f_eval(y, ftemp);
      }
      if (ret == 0) {
#pragma unroll
        for (int c = 0; c < CPL; ++c) y[c] = zn[0][c] + acor[c];
        jcur = 0;
        return 0;
      }
      if (!jcur) {
        callSetup = true;
        jbad = true;
        continue;
      }
      return 1;
    }
    return 1;
  }

  __device__ __forceinline__ void complete_step() {
    cnt.nst++;
    // tau[i] = tau[i-1] for i = q..2; tau[2] = tau[1] when q == 1 (after the first step); tau[1] = h
    const double up = __shfl_up_sync(kFull, tau_r, 1);
    if (lane >= 2 && lane <= q) tau_r = up;
    if (q == 1 && cnt.nst > 1 && lane == 2) tau_r = up;
    if (lane == 1) tau_r = h;
#pragma unroll
    for (int j = 0; j < kZn; ++j) {
      const double lj = l_at(j);
      if (j <= q)
#pragma unroll
        for (int c = 0; c < CPL; ++c) zn[j][c] += lj * acor[c];
    }
    qwait--;
    if (qwait == 1 && q != qmax) {
      zn_set(qmax, acor);
      saved_tq5 = tq_at(5);
    }
  }

  __device__ __forceinline__ void set_eta() {
    if (eta < kTHRESH) {
      eta = 1.0;
      hprime = h;
    } else {
      eta = fmin(eta, etamax);
      hprime = h * eta;
    }
  }

  __device__ __forceinline__ void prepare_next_step(double dsm) {
    if (etamax == 1.0) {
      qwait = qwait > 2 ? qwait : 2;
      qprime = q;
      hprime = h;
      eta = 1.0;
      return;
    }
    const double etaq = 1.0 / (pow(kBIAS2 * dsm, 1.0 / L) + kADDON);
    if (qwait != 0) {
      eta = etaq;
      qprime = q;
      set_eta();
      return;
    }
    qwait = 2;
    double etaqm1 = 0.0, etaqp1 = 0.0;
    if (q > 1) {
      double zq[CPL];
      zn_get(q, zq);
      const double ddn = wrms(zq) * tq_at(1);
      etaqm1 = 1.0 / (pow(kBIAS1 * ddn, 1.0 / q) + kADDON);
    }
    const double tq3 = tq_at(3), tq5 = tq_at(5), tau2 = tau_at(2);
    if (q != qmax && saved_tq5 != 0.0) {
      const double cquot = (tq5 / saved_tq5) * pow(h / tau2, (double)L);
      double zm[CPL];
      zn_get(qmax, zm);
#pragma unroll
      for (int c = 0; c < CPL; ++c) tmp[c] = acor[c] - cquot * zm[c];
      const double dup = wrms(tmp) * tq3;
      etaqp1 = 1.0 / (pow(kBIAS3 * dup, 1.0 / (L + 1)) + kADDON);
    }
    const double etam = fmax(etaqm1, fmax(etaq, etaqp1));
    if (etam < kTHRESH) {
      eta = 1.0;
      qprime = q;
    } else if (etam == etaq) {
      eta = etaq;
      qprime = q;
    } else if (etam == etaqm1) {
      eta = etaqm1;
      qprime = q - 1;
    } else {
      eta = etaqp1;
      qprime = q + 1;
      zn_set(qmax, acor);
    }
    set_eta();
  }

  // one internal step: 0 ok, else B200CHEM_CELL_* failure code
  __device__ __forceinline__ int step() {
    const double saved_t = tn;
    int ncf = 0, nef = 0, nflag = kFirstCall;
    double dsm = 0.0;
    if (cnt.nst > 0 && hprime != h) {
      if (qprime != q) {
        if (qprime - q == 1) increase_order();
        else if (qprime - q == -1) decrease_order();
        q = qprime;
        L = q + 1;
        qwait = L;
      }
      rescale();
    }
    for (int guard = 0; guard < 64; ++guard) {
      predict();
      set_bdf();
      const int r = nls(nflag);
      if (r != 0) {
        cnt.ncfn++;
        restore(saved_t);
        ncf++;
        etamax = 1.0;
        if (ncf == kMXNCF) return r == 2 ? -5 : -3;
        eta = kETACF;
        nflag = kPrevConvFail;
        rescale();
        continue;
      }
      dsm = acnrm * tq2_;
      if (dsm <= 1.0) {
        complete_step();
        prepare_next_step(dsm);
        etamax = (cnt.nst <= kSMALL_NST) ? kETAMX2 : kETAMX3;
        return 0;
      }
      nef++;
      cnt.netf++;
      nflag = kPrevErrFail;
      restore(saved_t);
      if (nef == kMXNEF) return -2;
      etamax = 1.0;
      if (nef <= kMXNEF1) {
        eta = 1.0 / (pow(kBIAS2 * dsm, 1.0 / L) + kADDON);
        eta = fmax(kETAMIN, eta);
        if (nef >= kSMALL_NEF) eta = fmin(eta, kETAMXF);
        rescale();
        continue;
      }
      if (q > 1) {
        eta = kETAMIN;
        decrease_order();
        L = q;
        q--;
        qwait = L;
        rescale();
        continue;
      }
      eta = kETAMIN;
      h *= eta;
      hscale = h;
      qwait = kLONG_WAIT;
      f_eval(zn[0], tmp);
#pragma unroll
      for (int c = 0; c < CPL; ++c) zn[1][c] = h * tmp[c];
    }
    return -2;
  }

  __device__ __forceinline__ double initial_h(double tout) {
    const double tdist = fabs(tout - tn);
    const double tround = kUROUND * fmax(fabs(tn), fabs(tout));
    const double hlb = 100.0 * tround;
    double hinv = 0.0;
#pragma unroll
    for (int c = 0; c < CPL; ++c)
      if (active(c)) hinv = fmax(hinv, fabs(zn[1][c]) / (0.1 * fabs(zn[0][c]) + ld_atol(c)));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) hinv = fmax(hinv, __shfl_xor_sync(kFull, hinv, o));
    double hub = 0.1 * tdist;
    if (hub * hinv > 1.0) hub = 1.0 / hinv;
    double hg = sqrt(hlb * hub);
    if (hub < hlb) return hg;
    bool hnewOK = false;
    double hnew = hg;
    for (int count1 = 1; count1 <= 4; ++count1) {
#pragma unroll
      for (int c = 0; c < CPL; ++c) y[c] = zn[0][c] + hg * zn[1][c];
      f_eval(y, tmp);
#pragma unroll
      for (int c = 0; c < CPL; ++c) tmp[c] = (tmp[c] - zn[1][c]) / hg;
      const double yddnrm = wrms(tmp);
      hnew = (yddnrm * hub * hub > 2.0) ? sqrt(2.0 / yddnrm) : sqrt(hg * hub);
      if (hnewOK) {
        hg = hnew;
        break;
      }
      const double hrat = hnew / hg;
      if (hrat > 0.5 && hrat < 2.0) hnewOK = true;
      if (count1 > 1 && hrat > 2.0) {
        hnew = hg;
        hnewOK = true;
      }
      hg = hnew;
    }
    double h0 = 0.5 * hg;
    if (h0 < hlb) h0 = hlb;
    if (h0 > hub) h0 = hub;
    return h0;
  }

  // Integrate y over [0, dt]; y in/out (per lane).  Returns B200CHEM_CELL_*.
  __device__ __forceinline__ int integrate(double (&yio)[CPL], double dt, int max_steps) {
#pragma unroll
    for (int c = 0; c < CPL; ++c) {
      zn[0][c] = active(c) ? yio[c] : 0.0;
#pragma unroll
      for (int j = 1; j < kZn; ++j) zn[j][c] = 0.0;
      acor[c] = 0.0;
    }
    tn = 0.0;
    cnt = CellCounters{0, 0, 0, 0, 0, 0, 0};
    nstlp = nstlj = 0;
    q = qprime = 1;
    L = 2;
    qwait = L;
    etamax = kETAMX1;
    saved_tq5 = 0.0;
    crate = 1.0;
    jcur = 0;
    gammap = gamma = 1.0;
    gamrat = 1.0;
    tau_r = 0.0;
    tq_r = 0.0;
    l_r = 0.0;
    tq2_ = tq4_ = 0.0;
    set_ewt(zn[0]);
    double f0[CPL];
    f_eval(zn[0], f0);
    bool bad = false;
#pragma unroll
    for (int c = 0; c < CPL; ++c) {
      zn[1][c] = f0[c];
      if (!isfinite(f0[c])) bad = true;
    }
    if (__any_sync(kFull, bad)) return -4;
    const double h0 = initial_h(dt);
    h = hscale = hprime = h0;
#pragma unroll
    for (int c = 0; c < CPL; ++c) zn[1][c] *= h0;
    int nstloc = 0;
    for (;;) {
      if (cnt.nst > 0) set_ewt(zn[0]);
      if (nstloc >= max_steps) return -1;
      const int r = step();
      if (r != 0) return r;
      nstloc++;
      if (tn - dt >= 0.0) break;
    }
    // y(dt) = sum_j zn[j] s^j, s = (dt - tn)/h, by Horner over j = q..0
    const double s = (dt - tn) / h;
#pragma unroll
    for (int c = 0; c < CPL; ++c) {
      double v = 0.0;  // columns above q contribute nothing; zn[q] + s*0 == zn[q]
#pragma unroll
      for (int j = kZn - 1; j >= 0; --j) v = (j <= q) ? zn[j][c] + s * v : 0.0;
      yio[c] = v;
    }
    return 0;
  }
};

}  // namespace b200
