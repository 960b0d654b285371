// bdf_rounds.cuh -- the BDF integrator as a resumable per-cell state machine
// whose state lives in device memory, for the round-based react path.
//
// Same algorithm, step for step, as the CPU oracle and the other device
// integrators: CVODE's variable-order BDF in Nordsieck form with modified
// Newton (reference: PelePhysics ReactorCvode denseAJ_direct, absent from
// the snapshot; CVODE's published method).  The react call advances all
// cells in ROUNDS; every round gives each live cell exactly one right-hand
// side, and the cells whose Newton matrix must be rebuilt a setup:
//
//   rhs kernel    one THREAD per cell: f(y) for every cell of the list (all
//                 lanes walk the same reaction at the same time);
//   ctrl kernel   one THREAD per cell: resumes the state machine below with
//                 that f until the cell needs its next f, a setup, or is done;
//   setup kernel  one WARP per cell: analytic Jacobian (FP64) and the
//                 Gauss-Jordan inverse of D (I - gamma J) D^-1 (FP32);
//   ctrl kernel   again for the cells that were set up.
//
// Each cell ("slot") owns one contiguous record in device memory: its
// step-control scalars (RCell), its vectors (Nordsieck array, ewt, acor, ...)
// and its two matrices (FP64 Jacobian and the scaled inverse of the Newton
// matrix), both column-major.  A thread streams its own record sequentially,
// so every 32-byte sector it touches is used whole whatever the order of the
// cells in the work lists; a warp working on one cell reads a matrix column
// as one coalesced transaction.
#pragma once
#include "bdf_group.cuh"

namespace b200 {
namespace rounds {

// Resume points of the state machine (what the cell does with its next input).
enum Label : int {
  kLAfterF0 = 0,   // f(y0) evaluated
  kLAfterHin,      // f(y0 + hg y0') evaluated (initial step estimate)
  kLAfterNStart,   // f(predicted y) evaluated: maybe setup, then Newton
  kLAfterNIter,    // f(current Newton iterate) evaluated
  kLAfterRestart,  // f(y) after an order-1 restart
  kLAfterSetup,    // Newton matrix rebuilt (setup_ier holds its status)
  // internal labels
  kLStart, kLBeginStep, kLAttempt, kLNlsAttempt, kLNewtonIter, kLNlsRecover, kLNlsFail1, kLNlsFail2,
  kLNlsSuccess
};

// What the cell needs next.
// kNeedSetupJac: a setup whose Jacobian is stale (CVODE's jbad rule) and is
// recomputed first; kNeedSetup: a setup that reuses the stored Jacobian.
enum Need : int { kNeedRhs = 0, kNeedSetup = 1, kDone = 2, kNeedSetupJac = 3 };

// Step-control record of one cell (doubles first, then ints), padded to a
// multiple of 16 bytes so that it moves as 16-byte vectors.
struct alignas(16) RCell {
  double tau[kZn + 2], tq[6], l[kZn];
  double h, hprime, hscale, eta, etamax, tn, gamma, gammap, gamrat, crate, acnrm, rl1, saved_tq5, gamma_lu;
  double dt, saved_t, delp, hg, hub, hlb;
  int q, qprime, L, qwait, nstlp, nstlj, jcur, ncf, nef, nflag, convfail, callSetup, jbad, mnewt, attempt;
  int count1, hnewOK, nstloc, qmax, max_steps, setup_conv, label, setup_ier;
  CellCounters cnt;
  float refine_ratio;  // WRMS of the last FP64 refinement step over its correction (kRefineUnknown: none since
                       // the last setup)
  int pad_;
};
static_assert(sizeof(RCell) % 16 == 0, "RCell moves as 16-byte vectors");

// Byte layout of one cell record for n components and inverse type of
// lut_bytes: [RCell][vectors (kZn + 7) n doubles][J: n columns of ldj
// doubles][A: n columns of lda LUT], each part 16-byte aligned, the record
// padded to 128 bytes.
struct RLayout {
  int ldj, lda;          // column strides (elements) of J and A
  int off_vec, off_j, off_a;
  long long stride;      // bytes per record
};

__host__ __device__ inline RLayout rounds_record_layout(int n, int lut_bytes) {
  RLayout L;
  L.ldj = (n + 1) & ~1;                                  // 16-byte columns
  L.lda = (lut_bytes == 4) ? ((n + 3) & ~3) : L.ldj;     // 16-byte columns
  L.off_vec = (int)sizeof(RCell);
  L.off_j = L.off_vec + ((8 * (kZn + 7) * n + 15) & ~15);
  L.off_a = L.off_j + 8 * L.ldj * n;
  L.stride = ((long long)L.off_a + (long long)lut_bytes * L.lda * n + 127) & ~127LL;
  return L;
}

// Device-memory state of one chunk of cells.
struct RState {
  unsigned char* rec;  // [cap][L.stride]
  RLayout L;
  long long cap;       // records of the chunk
};

// Vectors of one cell (contiguous).
template <int n>
struct RVec {
  double* b;
  __device__ __forceinline__ double& zn(int j, int i) const { return b[j * n + i]; }
  __device__ __forceinline__ double& ewt(int i) const { return b[(kZn + 0) * n + i]; }
  __device__ __forceinline__ double& acor(int i) const { return b[(kZn + 1) * n + i]; }
  __device__ __forceinline__ double& ftemp(int i) const { return b[(kZn + 2) * n + i]; }
  __device__ __forceinline__ double& fv(int i) const { return b[(kZn + 3) * n + i]; }
  __device__ __forceinline__ double& F(int i) const { return b[(kZn + 4) * n + i]; }
  __device__ __forceinline__ double& dsc(int i) const { return b[(kZn + 5) * n + i]; }
  __device__ __forceinline__ double& yev(int i) const { return b[(kZn + 6) * n + i]; }
};

__device__ __forceinline__ unsigned char* rec_of(const RState& S, long long slot) {
  return S.rec + slot * S.L.stride;
}

// Field-by-field copies (no address of the local RCell is taken, so its
// fields can live in registers).
#define B200_RCELL_SCALARS(X)                                                                              \
  X(h) X(hprime) X(hscale) X(eta) X(etamax) X(tn) X(gamma) X(gammap) X(gamrat) X(crate) X(acnrm) X(rl1)    \
  X(saved_tq5) X(gamma_lu) X(dt) X(saved_t) X(delp) X(hg) X(hub) X(hlb) X(q) X(qprime) X(L) X(qwait)      \
  X(nstlp) X(nstlj) X(jcur) X(ncf) X(nef) X(nflag) X(convfail) X(callSetup) X(jbad) X(mnewt) X(attempt)    \
  X(count1) X(hnewOK) X(nstloc) X(qmax) X(max_steps) X(setup_conv) X(label) X(setup_ier) X(cnt.nst)       \
  X(cnt.nfe) X(cnt.nje) X(cnt.nlu) X(cnt.netf) X(cnt.ncfn) X(cnt.nni) X(refine_ratio)

__device__ __forceinline__ void load_cell(RCell& c, const unsigned char* rec) {
  const RCell* g = reinterpret_cast<const RCell*>(rec);
#define B200_LD(f) c.f = g->f;
  B200_RCELL_SCALARS(B200_LD)
#undef B200_LD
#pragma unroll
  for (int i = 0; i < kZn + 2; ++i) c.tau[i] = g->tau[i];
#pragma unroll
  for (int i = 0; i < 6; ++i) c.tq[i] = g->tq[i];
#pragma unroll
  for (int i = 0; i < kZn; ++i) c.l[i] = g->l[i];
}

__device__ __forceinline__ void store_cell(const RCell& c, unsigned char* rec) {
  RCell* g = reinterpret_cast<RCell*>(rec);
#define B200_ST(f) g->f = c.f;
  B200_RCELL_SCALARS(B200_ST)
#undef B200_ST
#pragma unroll
  for (int i = 0; i < kZn + 2; ++i) g->tau[i] = c.tau[i];
#pragma unroll
  for (int i = 0; i < 6; ++i) g->tq[i] = c.tq[i];
#pragma unroll
  for (int i = 0; i < kZn; ++i) g->l[i] = c.l[i];
}

// a[k] for a runtime k < N with compile-time indexing (keeps a in registers)
template <int N>
__device__ __forceinline__ double sel(const double (&a)[N], int k) {
  double r = a[0];
#pragma unroll
  for (int i = 1; i < N; ++i)
    if (i == k) r = a[i];
  return r;
}

// ------------------------------------------------------- lane groups
// The control kernel runs G lanes per cell (G = 8 or 16): lane gl of a group
// owns components gl, gl + G, ... of every vector; step-control scalars are
// computed identically by all lanes of the group.
template <int n, int G, typename F>
__device__ __forceinline__ void each(int gl, F f) {
#pragma unroll
  for (int cc = 0; cc < (n + G - 1) / G; ++cc) {
    const int i = gl + G * cc;
    if (i < n) f(i);
  }
}

template <int G>
__device__ __forceinline__ double gsum(double v, unsigned gm) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(gm, v, o, G);
  return v;
}

template <int G>
__device__ __forceinline__ double gmax(double v, unsigned gm) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(gm, v, o, G));
  return v;
}

// ---------------------------------------------------------- BDF helpers
template <int n, int G>
__device__ __forceinline__ void r_rescale(RCell& c, const RVec<n>& v, int gl) {
  double factor = c.eta;
  for (int j = 1; j <= c.q; ++j) {
    each<n, G>(gl, [&](int i) { v.zn(j, i) *= factor; });
    factor *= c.eta;
  }
  c.h = c.hscale * c.eta;
  c.hscale = c.h;
}

// Nordsieck prediction zn := zn * Pascal, column by column in registers.
template <int n, int G>
__device__ __forceinline__ void r_predict(RCell& c, const RVec<n>& v, int gl) {
  c.tn += c.h;
  const int q = c.q;
  each<n, G>(gl, [&](int i) {
    double z[kZn];
#pragma unroll
    for (int j = 0; j < kZn; ++j) z[j] = (j <= q) ? v.zn(j, i) : 0.0;
#pragma unroll
    for (int k = 1; k < kZn; ++k)
#pragma unroll
      for (int j = kZn - 1; j >= 1; --j)
        if (j >= k && j <= q) z[j - 1] += z[j];
#pragma unroll
    for (int j = 0; j < kZn - 1; ++j)
      if (j < q) v.zn(j, i) = z[j];
  });
}

template <int n, int G>
__device__ __forceinline__ void r_restore(RCell& c, const RVec<n>& v, int gl) {
  c.tn = c.saved_t;
  const int q = c.q;
  each<n, G>(gl, [&](int i) {
    double z[kZn];
#pragma unroll
    for (int j = 0; j < kZn; ++j) z[j] = (j <= q) ? v.zn(j, i) : 0.0;
#pragma unroll
    for (int k = 1; k < kZn; ++k)
#pragma unroll
      for (int j = kZn - 1; j >= 1; --j)
        if (j >= k && j <= q) z[j - 1] -= z[j];
#pragma unroll
    for (int j = 0; j < kZn - 1; ++j)
      if (j < q) v.zn(j, i) = z[j];
  });
}

// WRMS norm of a vector given element-wise by get(i) (group reduction).
template <int n, int G, typename Get>
__device__ __forceinline__ double r_wrms(const RVec<n>& v, int gl, unsigned gm, Get get) {
  double s = 0.0;
  each<n, G>(gl, [&](int i) {
    const double t = get(i) * v.ewt(i);
    s += t * t;
  });
  return sqrt(gsum<G>(s, gm) / n);
}

__device__ __forceinline__ void r_set_bdf(RCell& c) {
  const int q = c.q;
  double xi_inv = 1.0, xistar_inv = 1.0;
  c.l[0] = c.l[1] = 1.0;
#pragma unroll
  for (int i = 2; i < kZn; ++i)
    if (i <= q) c.l[i] = 0.0;
  double alpha0 = -1.0, alpha0_hat = -1.0, hsum = c.h;
  if (q > 1) {
#pragma unroll
    for (int j = 2; j < kZn; ++j) {
      if (j < q) {
        hsum += c.tau[j - 1];
        xi_inv = c.h / hsum;
        alpha0 -= 1.0 / j;
#pragma unroll
        for (int i = j; i >= 1; --i) c.l[i] += c.l[i - 1] * xi_inv;
      }
    }
    alpha0 -= 1.0 / q;
    xistar_inv = -c.l[1] - alpha0;
    hsum += sel(c.tau, q - 1);
    xi_inv = c.h / hsum;
    alpha0_hat = -c.l[1] - xi_inv;
#pragma unroll
    for (int i = kZn - 1; i >= 1; --i)
      if (i <= q) c.l[i] += c.l[i - 1] * xistar_inv;
  }
  const double lq = sel(c.l, q);
  const double A1 = 1.0 - alpha0_hat + alpha0;
  const double A2 = 1.0 + q * A1;
  c.tq[2] = fabs(A1 / (alpha0 * A2));
  c.tq[5] = fabs(A2 * xistar_inv / (lq * xi_inv));
  if (c.qwait == 1) {
    if (q > 1) {
      const double C = xistar_inv / lq;
      const double A3 = alpha0 + 1.0 / q;
      const double A4 = alpha0_hat + xi_inv;
      const double Cpinv = (1.0 - A4 + A3) / A3;
      c.tq[1] = fabs(C * Cpinv);
    } else {
      c.tq[1] = 1.0;
    }
    hsum += sel(c.tau, q);
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

template <int n, int G>
__device__ __forceinline__ void r_increase(RCell& c, const RVec<n>& v, int gl) {
  const int q = c.q;
#pragma unroll
  for (int i = 0; i < kZn; ++i)
    if (i <= c.qmax) c.l[i] = 0.0;
  double alpha1 = 1.0, prod = 1.0, xiold = 1.0, alpha0 = -1.0, hsum = c.hscale;
  c.l[2] = 1.0;
#pragma unroll
  for (int j = 1; j < kZn - 1; ++j) {
    if (j < q) {
      hsum += c.tau[j + 1];
      const double xi = hsum / c.hscale;
      prod *= xi;
      alpha0 -= 1.0 / (j + 1);
      alpha1 += 1.0 / xi;
#pragma unroll
      for (int i = j + 2; i >= 2; --i)
        if (i < kZn) c.l[i] = c.l[i] * xiold + c.l[i - 1];
      xiold = xi;
    }
  }
  const double A1 = (-alpha0 - alpha1) / prod;
  const int qm = c.qmax;
  double lj[kZn];
#pragma unroll
  for (int j = 0; j < kZn; ++j) lj[j] = c.l[j];
  each<n, G>(gl, [&](int i) {
    const double z = A1 * v.zn(qm, i);
    v.zn(q + 1, i) = z;
#pragma unroll
    for (int j = 2; j < kZn; ++j)
      if (j <= q) v.zn(j, i) += lj[j] * z;
  });
}

template <int n, int G>
__device__ __forceinline__ void r_decrease(RCell& c, const RVec<n>& v, int gl) {
  const int q = c.q;
#pragma unroll
  for (int i = 0; i < kZn; ++i)
    if (i <= c.qmax) c.l[i] = 0.0;
  c.l[2] = 1.0;
  double hsum = 0.0;
#pragma unroll
  for (int j = 1; j < kZn - 2; ++j) {
    if (j <= q - 2) {
      hsum += c.tau[j];
      const double xi = hsum / c.hscale;
#pragma unroll
      for (int i = j + 2; i >= 2; --i)
        if (i < kZn) c.l[i] = c.l[i] * xi + c.l[i - 1];
    }
  }
  double lj[kZn];
#pragma unroll
  for (int j = 0; j < kZn; ++j) lj[j] = c.l[j];
  each<n, G>(gl, [&](int i) {
    const double zq = v.zn(q, i);
#pragma unroll
    for (int j = 2; j < kZn; ++j)
      if (j < q) v.zn(j, i) -= lj[j] * zq;
  });
}

template <int n, int G>
__device__ __forceinline__ void r_set_ewt(const RVec<n>& v, const double* atolv, double rtol, int gl) {
  each<n, G>(gl, [&](int i) { v.ewt(i) = 1.0 / (rtol * fabs(v.zn(0, i)) + __ldg(atolv + i)); });
}

template <int n, int G>
__device__ __forceinline__ void r_prepare_next(RCell& c, const RVec<n>& v, double dsm, int gl, unsigned gm) {
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
      const int q = c.q;
      const double ddn = r_wrms<n, G>(v, gl, gm, [&](int i) { return v.zn(q, i); }) * c.tq[1];
      etaqm1 = 1.0 / (pow(kBIAS1 * ddn, 1.0 / c.q) + kADDON);
    }
    if (c.q != c.qmax && c.saved_tq5 != 0.0) {
      const double cquot = (c.tq[5] / c.saved_tq5) * pow(c.h / c.tau[2], (double)c.L);
      const int qm = c.qmax;
      const double dup =
          r_wrms<n, G>(v, gl, gm, [&](int i) { return v.acor(i) - cquot * v.zn(qm, i); }) * c.tq[3];
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
      const int qm = c.qmax;
      each<n, G>(gl, [&](int i) { v.zn(qm, i) = v.acor(i); });
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

// 16-byte vector loads / stores of an n-vector (n even, p 16-byte aligned).
template <int n>
__device__ __forceinline__ void vld(const double* p, double (&r)[n]) {
  static_assert(n % 2 == 0, "records hold even-length vectors");
  const double2* q = reinterpret_cast<const double2*>(p);
#pragma unroll
  for (int i = 0; i < n / 2; ++i) {
    const double2 t = q[i];
    r[2 * i] = t.x;
    r[2 * i + 1] = t.y;
  }
}

template <int n>
__device__ __forceinline__ void vst(double* p, const double (&r)[n]) {
  double2* q = reinterpret_cast<double2*>(p);
#pragma unroll
  for (int i = 0; i < n / 2; ++i) q[i] = make_double2(r[2 * i], r[2 * i + 1]);
}

// Column stride of the inverse for n components (the record layout's lda).
template <int n, typename LUT>
constexpr int inv_ld() {
  return sizeof(LUT) == 4 ? (n + 3) / 4 * 4 : (n + 1) / 2 * 2;
}

// x := D^-1 A D x for the group's cell: A is the scaled inverse
// (column-major, 16-byte columns of inv_ld<n, LUT>() elements), D = dsc;
// LUT = double: A is the plain inverse.  Lane gl holds components gl + G cc
// of x and dsc; the multiplier of column j comes from its owner lane by
// shuffle and lanes read consecutive elements of the column.
template <int n, int G, typename LUT>
__device__ __forceinline__ void g_apply_inverse(const LUT* A, const double (&dsc)[(n + G - 1) / G],
                                                double (&x)[(n + G - 1) / G], int gl, unsigned gm) {
  constexpr int CPL = (n + G - 1) / G;
  constexpr bool kScaled = sizeof(LUT) == 4;
  constexpr int LD = inv_ld<n, LUT>();
  LUT acc[CPL], bs[CPL];
#pragma unroll
  for (int cc = 0; cc < CPL; ++cc) {
    acc[cc] = (LUT)0;
    bs[cc] = (LUT)(kScaled ? x[cc] * dsc[cc] : x[cc]);
  }
#pragma unroll
  for (int j = 0; j < n; ++j) {
    const LUT bj = __shfl_sync(gm, bs[j / G], j % G, G);
    const LUT* col = A + j * LD;
#pragma unroll
    for (int cc = 0; cc < CPL; ++cc) {
      const int i = gl + G * cc;
      if (i < n) acc[cc] += col[i] * bj;
    }
  }
#pragma unroll
  for (int cc = 0; cc < CPL; ++cc) x[cc] = kScaled ? (double)acc[cc] / dsc[cc] : (double)acc[cc];
}

// One Newton correction: x = (I - gamma_lu J)^-1 dl with
// dl = -(rl1 zn[1] + acor - gamma ftemp) (FP32 inverse, then, when `refine`,
// one FP64 refinement step r = dl - (x - gamma_lu J x), x += A r, whose WRMS
// relative to x goes to *ratio; FP64 inverse: no refinement), scaled by
// 2 / (1 + gamrat) when gamma has moved since the setup; then acor += x.
// Returns the WRMS norms of x (*del) and of the new acor (*anrm).
// Internal status of a cell stopped for the FP64 retry (never reported).
constexpr int kStatusRefineStall = -100;
// refine_ratio of a cell whose current matrix has not been measured yet
constexpr float kRefineUnknown = 3.0e38f;

template <int n, int G, typename LUT>
__device__ __forceinline__ void g_newton(const RVec<n>& v, const double* J, const LUT* A, double rl1, double gamma,
                                         double gamma_lu, double gamrat, int gl, unsigned gm, double* del,
                                         double* anrm, double stall_ratio, bool* stall, bool refine,
                                         float* ratio) {
  constexpr int CPL = (n + G - 1) / G;
  double dl[CPL], x[CPL], dsc[CPL];
#pragma unroll
  for (int cc = 0; cc < CPL; ++cc) {
    const int i = gl + G * cc;
    dl[cc] = (i < n) ? -(rl1 * v.zn(1, i) + v.acor(i) - gamma * v.ftemp(i)) : 0.0;
    dsc[cc] = (i < n) ? v.dsc(i) : 1.0;
    x[cc] = dl[cc];
  }
  g_apply_inverse<n, G, LUT>(A, dsc, x, gl, gm);
  if constexpr (sizeof(LUT) == 4) {
    if (refine) {
      constexpr int LDJ = (n + 1) / 2 * 2;
      double r[CPL];
#pragma unroll
      for (int cc = 0; cc < CPL; ++cc) r[cc] = 0.0;
#pragma unroll
      for (int j = 0; j < n; ++j) {
        const double xj = __shfl_sync(gm, x[j / G], j % G, G);
        const double* col = J + j * LDJ;
#pragma unroll
        for (int cc = 0; cc < CPL; ++cc) {
          const int i = gl + G * cc;
          if (i < n) r[cc] += col[i] * xj;
        }
      }
#pragma unroll
      for (int cc = 0; cc < CPL; ++cc) r[cc] = dl[cc] - (x[cc] - gamma_lu * r[cc]);
      g_apply_inverse<n, G, LUT>(A, dsc, r, gl, gm);
      double r2 = 0.0, x2 = 0.0;
#pragma unroll
      for (int cc = 0; cc < CPL; ++cc) {
        const int i = gl + G * cc;
        if (i < n) {
          const double w = v.ewt(i);
          r2 += (r[cc] * w) * (r[cc] * w);
          x2 += (x[cc] * w) * (x[cc] * w);
        }
        x[cc] += r[cc];
      }
      // the refinement step must be small against the correction it refines
      r2 = gsum<G>(r2, gm);
      x2 = gsum<G>(x2, gm);
      *ratio = (x2 > 0.0) ? (float)fmin(sqrt(r2 / x2), 1e30) : 0.0f;
      if (stall_ratio > 0.0) *stall = !(r2 <= stall_ratio * stall_ratio * x2);
    }
  }
  const double sc = (gamrat != 1.0) ? 2.0 / (1.0 + gamrat) : 1.0;
  double s2 = 0.0, a2 = 0.0;
#pragma unroll
  for (int cc = 0; cc < CPL; ++cc) {
    const int i = gl + G * cc;
    if (i < n) {
      const double xi = x[cc] * sc;
      const double ac = v.acor(i) + xi;
      v.acor(i) = ac;
      const double w = v.ewt(i);
      s2 += (xi * w) * (xi * w);
      a2 += (ac * w) * (ac * w);
    }
  }
  *del = sqrt(gsum<G>(s2, gm) / n);
  *anrm = sqrt(gsum<G>(a2, gm) / n);
}

// Advance the cell from resume point `lab` until it needs a right-hand side
// at v.yev (returns kNeedRhs with c.label set to the label that consumes it),
// a setup (kNeedSetup, or kNeedSetupJac with a Jacobian refresh), or is
// finished (kDone, *status set).
template <int n, int G, typename LUT>
__device__ __forceinline__ int r_advance(RCell& c, const RVec<n>& v, int lab, const double* atolv, double rtol,
                                         const double* J, const LUT* A, int gl, unsigned gm, int* status,
                                         double stall_ratio = 0.0, double keep_ratio = 0.0) {
  for (int guard = 0; guard < 256; ++guard) {
    switch (lab) {
      case kLAfterF0: {
        bool bad = false;
        double hinv = 0.0;
        each<n, G>(gl, [&](int i) {
          const double f = v.fv(i);
          v.zn(1, i) = f;
          bad |= !isfinite(f);
          hinv = fmax(hinv, fabs(f) / (0.1 * fabs(v.zn(0, i)) + __ldg(atolv + i)));
        });
        hinv = gmax<G>(hinv, gm);
        bad = gmax<G>(bad ? 1.0 : 0.0, gm) > 0.0;
        if (bad) {
          *status = -4;
          return kDone;
        }
        const double tdist = fabs(c.dt);
        const double tround = kUROUND * fabs(c.dt);
        c.hlb = 100.0 * tround;
        c.hub = 0.1 * tdist;
        if (c.hub * hinv > 1.0) c.hub = 1.0 / hinv;
        c.hg = sqrt(c.hlb * c.hub);
        if (c.hub < c.hlb) {
          c.h = c.hg;  // initial step is the geometric mean
          c.count1 = -1;
          lab = kLStart;
          break;
        }
        c.count1 = 1;
        c.hnewOK = 0;
        {
          const double hg = c.hg;
          each<n, G>(gl, [&](int i) { v.yev(i) = v.zn(0, i) + hg * v.zn(1, i); });
        }
        c.label = kLAfterHin;
        return kNeedRhs;
      }
      case kLAfterHin: {
        const double hg = c.hg;
        const double yddnrm = r_wrms<n, G>(v, gl, gm, [&](int i) { return (v.fv(i) - v.zn(1, i)) / hg; });
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
          const double hg2 = c.hg;
          each<n, G>(gl, [&](int i) { v.yev(i) = v.zn(0, i) + hg2 * v.zn(1, i); });
          c.label = kLAfterHin;
          return kNeedRhs;
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
        each<n, G>(gl, [&](int i) { v.zn(1, i) *= h0; });
        c.nstloc = 0;
        lab = kLBeginStep;
        break;
      }
      case kLBeginStep: {
        if (c.cnt.nst > 0) r_set_ewt<n, G>(v, atolv, rtol, gl);
        if (c.nstloc >= c.max_steps) {
          *status = -1;
          return kDone;
        }
        c.saved_t = c.tn;
        c.ncf = c.nef = 0;
        c.nflag = kFirstCall;
        if (c.cnt.nst > 0 && c.hprime != c.h) {
          if (c.qprime != c.q) {
            if (c.qprime - c.q == 1) r_increase<n, G>(c, v, gl);
            else if (c.qprime - c.q == -1) r_decrease<n, G>(c, v, gl);
            c.q = c.qprime;
            c.L = c.q + 1;
            c.qwait = c.L;
          }
          r_rescale<n, G>(c, v, gl);
        }
        lab = kLAttempt;
        break;
      }
      case kLAttempt: {
        r_predict<n, G>(c, v, gl);
        r_set_bdf(c);
        c.convfail = (c.nflag == kFirstCall || c.nflag == kPrevErrFail) ? kNoFailures : kFailOther;
        c.callSetup = (c.nflag == kPrevConvFail) || (c.nflag == kPrevErrFail) || (c.cnt.nst == 0) ||
                      (c.cnt.nst >= c.nstlp + kMSBP) || (fabs(c.gamrat - 1.0) > kDGMAX_LSETUP);
        c.jbad = 0;
        c.attempt = 0;
        lab = kLNlsAttempt;
        break;
      }
      case kLNlsAttempt: {
        each<n, G>(gl, [&](int i) {
          v.acor(i) = 0.0;
          v.yev(i) = v.zn(0, i);
        });
        c.label = kLAfterNStart;
        return kNeedRhs;
      }
      case kLAfterNStart: {
        each<n, G>(gl, [&](int i) { v.ftemp(i) = v.fv(i); });
        if (c.callSetup) {
          c.setup_conv = c.jbad ? kFailBadJ : c.convfail;
          c.label = kLAfterSetup;
          // CVODE's jbad rule: recompute J on the first step, every msbj
          // steps, or after a convergence failure (with a stale J, or with
          // gamma little changed)
          const double dgamma = fabs(c.gamma / c.gammap - 1.0);
          const bool jbad = (c.cnt.nst == 0) || (c.cnt.nst >= c.nstlj + kMSBJ) ||
                            (c.setup_conv == kFailBadJ && dgamma < kDGMAX_JBAD) || (c.setup_conv == kFailOther);
          c.jcur = jbad ? 1 : 0;
          if (jbad) {
            c.cnt.nje++;
            c.nstlj = c.cnt.nst;
            return kNeedSetupJac;
          }
          return kNeedSetup;
        }
        c.mnewt = 0;
        c.delp = 0.0;
        lab = kLNewtonIter;
        break;
      }
      case kLAfterSetup: {
        c.callSetup = 0;
        c.refine_ratio = kRefineUnknown;
        if (c.setup_ier) {
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
        double del, anrm;
        bool stall = false;
        // the FP64 refinement runs on the first correction with a new matrix,
        // and again on every later one unless that first measurement showed
        // the FP32 solve alone accurate to keep_ratio
        const bool refine = !(keep_ratio > 0.0 && c.refine_ratio <= keep_ratio);
        float ratio = c.refine_ratio;
        g_newton<n, G, LUT>(v, J, A, c.rl1, c.gamma, c.gamma_lu, c.gamrat, gl, gm, &del, &anrm, stall_ratio,
                            &stall, refine, &ratio);
        c.refine_ratio = ratio;
        if (stall) {
          // the FP32 inverse does not resolve this iteration matrix: the cell
          // is left untouched for the pass with the FP64 LU
          *status = kStatusRefineStall;
          return kDone;
        }
        if (c.mnewt > 0) c.crate = fmax(kCRDOWN * c.crate, del / c.delp);
        const double dcon = del * fmin(1.0, c.crate) / c.tq[4];
        if (dcon <= 1.0) {
          c.acnrm = (c.mnewt == 0) ? del : anrm;
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
        each<n, G>(gl, [&](int i) { v.yev(i) = v.zn(0, i) + v.acor(i); });
        c.label = kLAfterNIter;
        return kNeedRhs;
      }
      case kLAfterNIter: {
        each<n, G>(gl, [&](int i) { v.ftemp(i) = v.fv(i); });
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
        r_restore<n, G>(c, v, gl);
        c.ncf++;
        c.etamax = 1.0;
        if (c.ncf == kMXNCF) {
          *status = (lab == kLNlsFail2) ? -5 : -3;
          return kDone;
        }
        c.eta = kETACF;
        c.nflag = kPrevConvFail;
        r_rescale<n, G>(c, v, gl);
        lab = kLAttempt;
        break;
      }
      case kLNlsSuccess: {
        const double dsm = c.acnrm * c.tq[2];
        if (dsm <= 1.0) {
          // complete the step
          c.cnt.nst++;
#pragma unroll
          for (int i = kZn + 1; i >= 2; --i)
            if (i <= c.q) c.tau[i] = c.tau[i - 1];
          if (c.q == 1 && c.cnt.nst > 1) c.tau[2] = c.tau[1];
          c.tau[1] = c.h;
          const int q = c.q;
          const bool save = (c.qwait - 1 == 1 && q != c.qmax);
          const int qm = c.qmax;
          double lj[kZn];
#pragma unroll
          for (int j = 0; j < kZn; ++j) lj[j] = c.l[j];
          each<n, G>(gl, [&](int i) {
            const double ac = v.acor(i);
#pragma unroll
            for (int j = 0; j < kZn; ++j)
              if (j <= q) v.zn(j, i) += lj[j] * ac;
            if (save) v.zn(qm, i) = ac;
          });
          c.qwait--;
          if (save) c.saved_tq5 = c.tq[5];
          r_prepare_next<n, G>(c, v, dsm, gl, gm);
          c.etamax = (c.cnt.nst <= kSMALL_NST) ? kETAMX2 : kETAMX3;
          c.nstloc++;
          if (c.tn - c.dt >= 0.0) {
            *status = 0;
            return kDone;
          }
          lab = kLBeginStep;
          break;
        }
        c.nef++;
        c.cnt.netf++;
        c.nflag = kPrevErrFail;
        r_restore<n, G>(c, v, gl);
        if (c.nef == kMXNEF) {
          *status = -2;
          return kDone;
        }
        c.etamax = 1.0;
        if (c.nef <= kMXNEF1) {
          c.eta = 1.0 / (pow(kBIAS2 * dsm, 1.0 / c.L) + kADDON);
          c.eta = fmax(kETAMIN, c.eta);
          if (c.nef >= kSMALL_NEF) c.eta = fmin(c.eta, kETAMXF);
          r_rescale<n, G>(c, v, gl);
          lab = kLAttempt;
          break;
        }
        if (c.q > 1) {
          c.eta = kETAMIN;
          r_decrease<n, G>(c, v, gl);
          c.L = c.q;
          c.q--;
          c.qwait = c.L;
          r_rescale<n, G>(c, v, gl);
          lab = kLAttempt;
          break;
        }
        c.eta = kETAMIN;
        c.h *= c.eta;
        c.hscale = c.h;
        c.qwait = kLONG_WAIT;
        each<n, G>(gl, [&](int i) { v.yev(i) = v.zn(0, i); });
        c.label = kLAfterRestart;
        return kNeedRhs;
      }
      case kLAfterRestart: {
        const double hh = c.h;
        each<n, G>(gl, [&](int i) { v.zn(1, i) = hh * v.fv(i); });
        lab = kLAttempt;
        break;
      }
      default:
        *status = -3;
        return kDone;
    }
  }
  *status = -3;  // the state machine never loops this long without an RHS
  return kDone;
}

// Start a cell whose zn[0] (state) and F (forcing) are loaded: counters and
// step-control defaults, then ask for f(y0).
template <int n>
__device__ __forceinline__ void r_begin(RCell& c, const RVec<n>& v, const double* atolv, double rtol, double dt,
                                        int qmax, int max_steps) {  // one thread per cell
  c.tn = 0.0;
  c.dt = dt;
  c.cnt = CellCounters{0, 0, 0, 0, 0, 0, 0};
  c.refine_ratio = kRefineUnknown;
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
  c.gamma_lu = 1.0;
  c.qmax = qmax;
  c.max_steps = max_steps;
  c.h = c.hprime = c.hscale = c.eta = 1.0;
  c.acnrm = c.rl1 = c.saved_t = c.delp = c.hg = c.hub = c.hlb = 0.0;
  c.ncf = c.nef = c.nflag = c.convfail = c.callSetup = c.jbad = c.mnewt = c.attempt = 0;
  c.count1 = c.hnewOK = c.nstloc = c.setup_conv = c.setup_ier = 0;
#pragma unroll
  for (int i = 0; i < kZn + 2; ++i) c.tau[i] = 0.0;
#pragma unroll
  for (int i = 0; i < 6; ++i) c.tq[i] = 0.0;
#pragma unroll
  for (int i = 0; i < kZn; ++i) c.l[i] = 0.0;
#pragma unroll 2
  for (int i = 0; i < n; ++i) {
    for (int j = 1; j < kZn; ++j) v.zn(j, i) = 0.0;
    v.acor(i) = 0.0;
    v.yev(i) = v.zn(0, i);
  }
  r_set_ewt<n, 1>(v, atolv, rtol, 0);
  c.label = kLAfterF0;
}

}  // namespace rounds
}  // namespace b200
