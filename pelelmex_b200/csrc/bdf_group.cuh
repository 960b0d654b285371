// bdf_group.cuh -- variable-order BDF for one cell per GROUP of G lanes.
//
// The integrator inside ReactorBase::react (reference: PelePhysics
// ReactorCvode + SUNDIALS CVODE, denseAJ_direct; absent from the snapshot):
// CVODE's published BDF in Nordsieck form, making step for step the same
// decisions as the CPU oracle.  B200-specific structure:
//   * G lanes per cell (8, 16 or 32): lane g holds state components g, g+G,
//     ...; all step-control scalars are replicated in the group, small
//     coefficient arrays (tau, tq, l) are spread over lanes;
//   * the Newton iteration matrix M = I - gamma J, scaled to D M D^-1 with
//     D = diag(ewt), is inverted explicitly by Gauss-Jordan elimination with
//     partial pivoting in FP32 in shared memory (lanes over columns), so each
//     Newton solve is a lane-parallel matrix-vector product; one step of
//     iterative refinement uses the FP64 Jacobian.  LUT = double keeps the
//     whole inverse in FP64 (no refinement);
//   * the analytic FP64 Jacobian lives in a per-group global scratch slot
//     (column-major), small enough to stay resident in L2.
// Every loop is bounded; failures end with a per-cell status code.
#pragma once
#include "group_mech.cuh"

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

struct CellCounters {
  int nst, nfe, nje, nlu, netf, ncfn, nni;
};

// In-place Gauss-Jordan inverse of A = D (I - gamma J) D^-1 (FP32, D = Dsc)
// or A = I - gamma J (FP64).  J is column-major (J[col*ldj + row]); A is
// row-major in shared memory.  Returns 0, or k+1 when pivot k is zero.
template <int G, typename LUT>
__device__ __noinline__ int grp_gj_inverse(const double* J, int ldj, LUT* A, int ldl, int* ipiv, LUT* fcol,
                                           const double* Dsc, int n, double gamma, int lane) {
  const Grp<G> g(lane);
  constexpr bool kScaled = sizeof(LUT) == 4;
  for (int j = g.gl; j < n; j += G) {
    const double dj = kScaled ? Dsc[j] : 1.0;
    for (int i = 0; i < n; ++i) {
      const double mij = ((i == j) ? 1.0 : 0.0) - gamma * J[j * ldj + i];
      A[i * ldl + j] = (LUT)(kScaled ? mij * Dsc[i] / dj : mij);
    }
  }
  g.sync();
  for (int k = 0; k < n; ++k) {
    LUT best = (LUT)-1;
    int bi = k;
    for (int i = k + g.gl; i < n; i += G) {
      const LUT v = fabs(A[i * ldl + k]);
      if (v > best) {
        best = v;
        bi = i;
      }
    }
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) {
      const LUT ov = __shfl_xor_sync(g.mask, best, o, G);
      const int oi = __shfl_xor_sync(g.mask, bi, o, G);
      if (ov > best || (ov == best && oi < bi)) {
        best = ov;
        bi = oi;
      }
    }
    if (!(best > (LUT)0)) return k + 1;  // zero or NaN pivot: singular (group-uniform)
    if (g.gl == 0) ipiv[k] = bi;
    if (bi != k)
      for (int j = g.gl; j < n; j += G) {
        const LUT t = A[k * ldl + j];
        A[k * ldl + j] = A[bi * ldl + j];
        A[bi * ldl + j] = t;
      }
    g.sync();
    const LUT inv = (LUT)1 / A[k * ldl + k];
    g.sync();
    for (int j = g.gl; j < n; j += G) A[k * ldl + j] = (j == k) ? inv : A[k * ldl + j] * inv;
    for (int i = g.gl; i < n; i += G)
      if (i != k) {
        fcol[i] = A[i * ldl + k];
        A[i * ldl + k] = (LUT)0;
      }
    g.sync();
    for (int j = g.gl; j < n; j += G) {
      const LUT akj = A[k * ldl + j];
      for (int i = 0; i < n; ++i)
        if (i != k) A[i * ldl + j] -= fcol[i] * akj;
    }
    g.sync();
  }
  for (int k = n - 1; k >= 0; --k) {
    const int p = ipiv[k];
    if (p != k)
      for (int i = g.gl; i < n; i += G) {
        const LUT t = A[i * ldl + k];
        A[i * ldl + k] = A[i * ldl + p];
        A[i * ldl + p] = t;
      }
    g.sync();
  }
  return 0;
}

// x := D^-1 A D x  (A = scaled inverse; bvec is per-group shared scratch)
template <int G, int CPL, typename LUT>
__device__ __forceinline__ Vec<CPL> grp_apply_inverse(const Grp<G>& g, const LUT* A, int ldl, const double* Dsc,
                                                      double* bvec, int n, const Vec<CPL>& x) {
  constexpr bool kScaled = sizeof(LUT) == 4;
#pragma unroll
  for (int c = 0; c < CPL; ++c) {
    const int i = g.gl + G * c;
    if (i < n) bvec[i] = kScaled ? x.v[c] * Dsc[i] : x.v[c];
  }
  g.sync();
  Vec<CPL> out;
#pragma unroll
  for (int c = 0; c < CPL; ++c) {
    const int i = g.gl + G * c;
    double s = 0.0;
    if (i < n) {
      LUT acc = (LUT)0;
      for (int j = 0; j < n; ++j) acc += A[i * ldl + j] * (LUT)bvec[j];
      s = kScaled ? (double)acc / Dsc[i] : (double)acc;
    }
    out.v[c] = s;
  }
  g.sync();
  return out;
}

// Solve (I - gamma J) x = b with the inverse; FP32: one FP64 refinement step.
template <int G, int CPL, typename LUT>
__device__ __noinline__ Vec<CPL> grp_lsolve(const LUT* A, int ldl, const double* Dsc, double* bvec, const double* J,
                                            int ldj, double gamma, int n, Vec<CPL> b, int lane) {
  const Grp<G> g(lane);
  Vec<CPL> x = grp_apply_inverse<G, CPL, LUT>(g, A, ldl, Dsc, bvec, n, b);
  if (sizeof(LUT) == 8) return x;
  // r = b - (x - gamma J x); J column-major: lanes (rows) read a column contiguously
#pragma unroll
  for (int c = 0; c < CPL; ++c) {
    const int i = g.gl + G * c;
    if (i < n) bvec[i] = x.v[c];
  }
  g.sync();
  Vec<CPL> r;
#pragma unroll
  for (int c = 0; c < CPL; ++c) {
    const int i = g.gl + G * c;
    double s = 0.0;
    if (i < n)
      for (int j = 0; j < n; ++j) s += J[j * ldj + i] * bvec[j];
    r.v[c] = (i < n) ? b.v[c] - (x.v[c] - gamma * s) : 0.0;
  }
  g.sync();
  r = grp_apply_inverse<G, CPL, LUT>(g, A, ldl, Dsc, bvec, n, r);
#pragma unroll
  for (int c = 0; c < CPL; ++c) x.v[c] += r.v[c];
  return x;
}

template <int G, int CPL, typename LUT>
struct GroupBdf {
  const DevMech* m;
  GrpScratch ms;
  double* J;  // [n][ldj] global, column-major
  int ldj;
  LUT* A;     // [n][ldl] shared: the scaled inverse
  int ldl;
  int* ipiv;  // [n] shared
  LUT* fcol;  // [Npad] shared
  double* atolv;  // [Npad] shared: absolute tolerances
  double* Dsc;    // [Npad] shared: scaling of the inverted matrix
  double* bvec;   // [Npad] shared: broadcast vector of the solves
  int lane, n, qmax;
  double rtol;

  double zn[kZn][CPL];
  double ewt[CPL], acor[CPL], ftemp[CPL], F[CPL];
  // tau[1..q+1] step history, tq[1..5] error-test coefficients and l[0..q]
  // Nordsieck coefficients, held lane-distributed (group lane i keeps entry i)
  double tau_r, tq_r, l_r;
  double h, hprime, hscale, eta, etamax, tn, gamma, gammap, gamrat, crate, acnrm, rl1, saved_tq5;
  double gamma_lu, tq2_, tq4_;
  int q, qprime, L, qwait, nstlp, nstlj, jcur;
  CellCounters cnt;

  __device__ __forceinline__ Grp<G> grp() const { return Grp<G>(lane); }
  __device__ __forceinline__ int gl() const { return lane % G; }
  __device__ __forceinline__ int comp(int c) const { return (lane % G) + G * c; }
  __device__ __forceinline__ bool active(int c) const { return comp(c) < n; }

  __device__ __forceinline__ double wrms(const double (&v)[CPL]) const {
    double s = 0.0;
#pragma unroll
    for (int c = 0; c < CPL; ++c) {
      const double t = v[c] * ewt[c];
      s += t * t;
    }
    return sqrt(grp().sum(s) / n);
  }

  __device__ __forceinline__ void f_eval(const double (&yy)[CPL], double (&out)[CPL]) {
    Vec<CPL> a, b;
#pragma unroll
    for (int c = 0; c < CPL; ++c) {
      a.v[c] = yy[c];
      b.v[c] = F[c];
    }
    const Vec<CPL> r = grp_rhs<G, CPL>(m, ms, a, b, lane);
#pragma unroll
    for (int c = 0; c < CPL; ++c) out[c] = r.v[c];
    cnt.nfe++;
  }

  __device__ __forceinline__ double tau_at(int i) const { return grp().bcast(tau_r, i); }
  __device__ __forceinline__ double l_at(int i) const { return grp().bcast(l_r, i); }
  __device__ __forceinline__ double tq_at(int i) const { return grp().bcast(tq_r, i); }

  __device__ __forceinline__ void set_ewt(const double (&v)[CPL]) {
#pragma unroll
    for (int c = 0; c < CPL; ++c) ewt[c] = active(c) ? 1.0 / (rtol * fabs(v[c]) + atolv[comp(c)]) : 0.0;
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

  __device__ __forceinline__ void set_bdf() {
    const Grp<G> g = grp();
    double xi_inv = 1.0, xistar_inv = 1.0;
    l_r = (gl() <= 1) ? 1.0 : 0.0;
    double alpha0 = -1.0, alpha0_hat = -1.0, hsum = h;
    double l1 = 1.0;
    if (q > 1) {
      for (int j = 2; j < q; ++j) {
        hsum += tau_at(j - 1);
        xi_inv = h / hsum;
        alpha0 -= 1.0 / j;
        const double upv = g.up(l_r, 1);  // l[i] += l[i-1] xi_inv, i = j..1 (old values)
        if (gl() >= 1 && gl() <= j) l_r += upv * xi_inv;
      }
      alpha0 -= 1.0 / q;
      l1 = l_at(1);
      xistar_inv = -l1 - alpha0;
      hsum += tau_at(q - 1);
      xi_inv = h / hsum;
      alpha0_hat = -l1 - xi_inv;
      const double upv = g.up(l_r, 1);
      if (gl() >= 1 && gl() <= q) l_r += upv * xistar_inv;
      l1 = l_at(1);
    }
    const double lq = l_at(q);
    const double A1 = 1.0 - alpha0_hat + alpha0;
    const double A2 = 1.0 + q * A1;
    const double tq2 = fabs(A1 / (alpha0 * A2));
    const double tq5 = fabs(A2 * xistar_inv / (lq * xi_inv));
    if (gl() == 2) tq_r = tq2;
    if (gl() == 5) tq_r = tq5;
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
      if (gl() == 1) tq_r = tq1;
      if (gl() == 3) tq_r = tq3;
    }
    if (gl() == 4) tq_r = kNLSCOEF / tq2;
    tq2_ = tq2;
    tq4_ = kNLSCOEF / tq2;
    rl1 = 1.0 / l1;
    gamma = h * rl1;
    if (cnt.nst == 0) gammap = gamma;
    gamrat = (cnt.nst > 0) ? gamma / gammap : 1.0;
  }

  __device__ __forceinline__ void increase_order() {
    const Grp<G> g = grp();
    double alpha1 = 1.0, prod = 1.0, xiold = 1.0, alpha0 = -1.0, hsum = hscale;
    l_r = (gl() == 2) ? 1.0 : 0.0;
    for (int j = 1; j < q; ++j) {
      hsum += tau_at(j + 1);
      const double xi = hsum / hscale;
      prod *= xi;
      alpha0 -= 1.0 / (j + 1);
      alpha1 += 1.0 / xi;
      const double upv = g.up(l_r, 1);  // l[i] = l[i] xiold + l[i-1], i = j+2..2
      if (gl() >= 2 && gl() <= j + 2) l_r = l_r * xiold + upv;
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
    const Grp<G> g = grp();
    l_r = (gl() == 2) ? 1.0 : 0.0;
    double hsum = 0.0;
    for (int j = 1; j <= q - 2; ++j) {
      hsum += tau_at(j);
      const double xi = hsum / hscale;
      const double upv = g.up(l_r, 1);
      if (gl() >= 2 && gl() <= j + 2) l_r = l_r * xi + upv;
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

  // ------------------------------------------------------------ Newton
  __device__ __forceinline__ int lsetup(int convfail, const double (&y)[CPL]) {
    const double dgamma = fabs(gamma / gammap - 1.0);
    const bool jbad = (cnt.nst == 0) || (cnt.nst >= nstlj + kMSBJ) ||
                      (convfail == kFailBadJ && dgamma < kDGMAX_JBAD) || (convfail == kFailOther);
    if (jbad) {
      Vec<CPL> a, b;
#pragma unroll
      for (int c = 0; c < CPL; ++c) {
        a.v[c] = y[c];
        b.v[c] = ftemp[c];
      }
      grp_jac<G, CPL>(m, ms, a, b, J, ldj, lane);
      cnt.nje++;
      nstlj = cnt.nst;
      jcur = 1;
    } else {
      jcur = 0;
    }
#pragma unroll
    for (int c = 0; c < CPL; ++c)
      if (active(c)) Dsc[comp(c)] = (sizeof(LUT) == 4) ? ewt[c] : 1.0;
    grp().sync();
    const int ier = grp_gj_inverse<G, LUT>(J, ldj, A, ldl, ipiv, fcol, Dsc, n, gamma, lane);
    cnt.nlu++;
    gamma_lu = gamma;
    gamrat = 1.0;
    gammap = gamma;
    crate = 1.0;
    nstlp = cnt.nst;
    return ier;
  }

  // 0 converged, 1 recoverable failure, 2 singular matrix.  The residual is
  // evaluated at ONE call site for the first and the later iterations.
  __device__ __forceinline__ int nls(int nflag) {
    const int convfail = (nflag == kFirstCall || nflag == kPrevErrFail) ? kNoFailures : kFailOther;
    bool callSetup = (nflag == kPrevConvFail) || (nflag == kPrevErrFail) || (cnt.nst == 0) ||
                     (cnt.nst >= nstlp + kMSBP) || (fabs(gamrat - 1.0) > kDGMAX_LSETUP);
    bool jbad = false;
    int mm = 0;
    double delp = 0.0;
#pragma unroll
    for (int c = 0; c < CPL; ++c) acor[c] = 0.0;
    for (int it = 0; it < 4 * (kMAXCOR + 1); ++it) {
      double y[CPL];
#pragma unroll
      for (int c = 0; c < CPL; ++c) y[c] = zn[0][c] + acor[c];
      f_eval(y, ftemp);
      if (mm == 0 && callSetup) {
        const int ier = lsetup(jbad ? kFailBadJ : convfail, y);
        callSetup = false;
        if (ier) return 2;
      }
      cnt.nni++;
      Vec<CPL> dl;
#pragma unroll
      for (int c = 0; c < CPL; ++c) dl.v[c] = -(rl1 * zn[1][c] + acor[c] - gamma * ftemp[c]);
      dl = grp_lsolve<G, CPL, LUT>(A, ldl, Dsc, bvec, J, ldj, gamma_lu, n, dl, lane);
      if (gamrat != 1.0) {
        const double sc = 2.0 / (1.0 + gamrat);
#pragma unroll
        for (int c = 0; c < CPL; ++c) dl.v[c] *= sc;
      }
#pragma unroll
      for (int c = 0; c < CPL; ++c) acor[c] += dl.v[c];
      const double del = wrms(dl.v);
      if (mm > 0) crate = fmax(kCRDOWN * crate, del / delp);
      const double dcon = del * fmin(1.0, crate) / tq4_;
      if (dcon <= 1.0) {
        acnrm = (mm == 0) ? del : wrms(acor);
        jcur = 0;
        return 0;
      }
      const bool fail = (mm >= 1 && del > kRDIV * delp) || !(del == del) || (mm + 1 >= kMAXCOR);
      if (!fail) {
        delp = del;
        mm++;
        continue;
      }
      if (jcur) return 1;
      // stale Jacobian: start the attempt again with a fresh one
      callSetup = true;
      jbad = true;
      mm = 0;
      delp = 0.0;
#pragma unroll
      for (int c = 0; c < CPL; ++c) acor[c] = 0.0;
    }
    return 1;
  }

  __device__ __forceinline__ void complete_step() {
    const Grp<G> g = grp();
    cnt.nst++;
    const double upv = g.up(tau_r, 1);  // tau[i] = tau[i-1], i = q..2; tau[2] = tau[1] if q == 1
    if (gl() >= 2 && gl() <= q) tau_r = upv;
    if (q == 1 && cnt.nst > 1 && gl() == 2) tau_r = upv;
    if (gl() == 1) tau_r = h;
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
    } else {
      qwait = 2;
      double etaqm1 = 0.0, etaqp1 = 0.0;
      const double tq1 = tq_at(1), tq3 = tq_at(3), tq5 = tq_at(5), tau2 = tau_at(2);
      if (q > 1) {
        double zq[CPL];
        zn_get(q, zq);
        const double ddn = wrms(zq) * tq1;
        etaqm1 = 1.0 / (pow(kBIAS1 * ddn, 1.0 / q) + kADDON);
      }
      if (q != qmax && saved_tq5 != 0.0) {
        const double cquot = (tq5 / saved_tq5) * pow(h / tau2, (double)L);
        double zm[CPL], t[CPL];
        zn_get(qmax, zm);
#pragma unroll
        for (int c = 0; c < CPL; ++c) t[c] = acor[c] - cquot * zm[c];
        const double dup = wrms(t) * tq3;
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
    }
    if (eta < kTHRESH) {
      eta = 1.0;
      hprime = h;
    } else {
      eta = fmin(eta, etamax);
      hprime = h * eta;
    }
  }

  // one internal step: 0 ok, else B200CHEM_CELL_* failure code
  __device__ __forceinline__ int step() {
    const double saved_t = tn;
    int ncf = 0, nef = 0, nflag = kFirstCall;
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
      const double dsm = acnrm * tq2_;
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
      double t[CPL];
      f_eval(zn[0], t);
#pragma unroll
      for (int c = 0; c < CPL; ++c) zn[1][c] = h * t[c];
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
      if (active(c)) hinv = fmax(hinv, fabs(zn[1][c]) / (0.1 * fabs(zn[0][c]) + atolv[comp(c)]));
    hinv = grp().maxv(hinv);
    double hub = 0.1 * tdist;
    if (hub * hinv > 1.0) hub = 1.0 / hinv;
    double hg = sqrt(hlb * hub);
    if (hub < hlb) return hg;
    bool hnewOK = false;
    double hnew = hg;
    for (int count1 = 1; count1 <= 4; ++count1) {
      double y[CPL], t[CPL];
#pragma unroll
      for (int c = 0; c < CPL; ++c) y[c] = zn[0][c] + hg * zn[1][c];
      f_eval(y, t);
#pragma unroll
      for (int c = 0; c < CPL; ++c) t[c] = (t[c] - zn[1][c]) / hg;
      const double yddnrm = wrms(t);
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
    tau_r = tq_r = l_r = 0.0;
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
    if (grp().any(bad)) return -4;
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
