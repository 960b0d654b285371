// b200chem.cu -- kernels and C ABI of the B200 HP chemistry reactor.
//
// One persistent launch advances every cell of a list of boxes: each warp
// takes cells from a global atomic queue (work stealing, so cells that need
// thousands of BDF steps do not hold back cells that need a handful) and
// integrates one cell at a time with WarpBdf (bdf_warp.cuh).  The launch is
// sized to fill the GPU exactly once (SM count x resident CTAs per SM).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/b200chem.h"
#include "bdf_thread.cuh"

using namespace b200;

namespace {

thread_local std::string g_err;

int set_err(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

#define CK(x)                                                                              \
  do {                                                                                     \
    cudaError_t e_ = (x);                                                                  \
    if (e_ != cudaSuccess) return set_err(B200CHEM_ECUDA, "%s: %s", #x, cudaGetErrorString(e_)); \
  } while (0)

struct DevArr {
  double* p;
  long long js, ks, ns;
  int lo0, lo1, lo2, pad;
};
struct DevIArr {
  const int* p;
  long long js, ks;
  int lo0, lo1, lo2, pad;
};
struct DevBox {
  int lo0, lo1, lo2, nx, ny, nz;
  long long off;
  DevArr rhoY, fY, T, rhoH, fH, fc;
  DevIArr mask;
};

// stats slots in the scratch buffer (after the queue counter)
enum { kStCells = 0, kStMasked, kStFailed, kStNst, kStNfe, kStNje, kStNlu, kStNetf, kStNcfn, kStMaxNfe,
       kStMaxNst, kStCount };

struct ReactParams {
  DevMech mech;
  const DevBox* boxes;
  int nbox;
  long long total;
  double dt;
  int max_steps;
  int qmax;
  double rtol;
  const double* atol;
  unsigned long long* queue;
  long long* stats;
  int* status;
  int warp_bytes;
  int Npad, Rpad, ldj, ldl;
};

__device__ __forceinline__ double* elem(const DevArr& a, int i, int j, int k) {
  return a.p + (long long)(i - a.lo0) + (long long)(j - a.lo1) * a.js + (long long)(k - a.lo2) * a.ks;
}

template <int CPL, typename LUT>
__device__ __forceinline__ void carve(WarpBdf<CPL, LUT>& B, unsigned char* base, int n, int Npad, int Rpad, int ldj,
                                      int ldl) {
  double* d = reinterpret_cast<double*>(base);
  B.ms.C = d;
  d += Npad;
  B.ms.gRT = d;
  d += Npad;
  B.ms.hRT = d;
  d += Npad;
  B.ms.r0 = d;
  d += Rpad;
  B.ms.r1 = d;
  d += Rpad;
  B.ms.r2 = d;
  d += Rpad;
  B.ms.r3 = d;
  d += Rpad;
  B.ms.r4 = d;
  d += Rpad;
  B.atolv = d;
  d += Npad;
  B.Dsc = d;
  d += Npad;
  B.J = d;
  d += (size_t)n * ldj;
  B.LU = reinterpret_cast<LUT*>(d);
  B.perm = reinterpret_cast<int*>(B.LU + (size_t)n * ldl);
  B.ldj = ldj;
  B.ldl = ldl;
}

// Minimum resident CTAs per SM requested from the compiler (register budget):
// 1 lets the integrator keep all of its state in registers (up to 255).
#ifndef B200_REACT_MIN_CTAS
#define B200_REACT_MIN_CTAS 1
#endif

template <int CPL, typename LUT>
__global__ void __launch_bounds__(128, B200_REACT_MIN_CTAS) react_kernel(ReactParams P) {
  extern __shared__ __align__(16) unsigned char dsm[];
  __shared__ DevMech s_mech;
  __shared__ long long s_off[65];
  if (threadIdx.x == 0) s_mech = P.mech;
  const int nb_s = P.nbox <= 64 ? P.nbox : 0;
  for (int b = threadIdx.x; b <= nb_s; b += blockDim.x) s_off[b] = (b < nb_s) ? P.boxes[b].off : P.total;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int w = threadIdx.x >> 5;
  const int N = P.mech.N, n = N + 1;

  WarpBdf<CPL, LUT> B;
  B.m = &s_mech;
  B.lane = lane;
  B.n = n;
  B.qmax = P.qmax;
  B.rtol = P.rtol;
  carve<CPL, LUT>(B, dsm + (size_t)w * P.warp_bytes, n, P.Npad, P.Rpad, P.ldj, P.ldl);
  for (int k = lane; k < n; k += 32) B.atolv[k] = P.atol[k];
  __syncwarp();
  long long acc[kStCount];
#pragma unroll
  for (int i = 0; i < kStCount; ++i) acc[i] = 0;

  for (;;) {
    unsigned long long cell = 0;
    if (lane == 0) cell = atomicAdd(P.queue, 1ull);
    cell = __shfl_sync(kFull, cell, 0);
    if (cell >= (unsigned long long)P.total) break;
    // locate the box (offsets are increasing)
    int lo = 0, hi = P.nbox - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      const long long o = nb_s ? s_off[mid] : P.boxes[mid].off;
      if (o <= (long long)cell) lo = mid;
      else hi = mid - 1;
    }
    const DevBox& bx = P.boxes[lo];
    const long long loc = (long long)cell - bx.off;
    const int i = bx.lo0 + (int)(loc % bx.nx);
    const int j = bx.lo1 + (int)((loc / bx.nx) % bx.ny);
    const int k = bx.lo2 + (int)(loc / ((long long)bx.nx * bx.ny));
    int code;
    double* fcp = bx.fc.p ? elem(bx.fc, i, j, k) : nullptr;
    bool masked = false;
    if (bx.mask.p) {
      const int mv = bx.mask.p[(long long)(i - bx.mask.lo0) + (long long)(j - bx.mask.lo1) * bx.mask.js +
                               (long long)(k - bx.mask.lo2) * bx.mask.ks];
      masked = (mv == 0);
    }
    if (masked) {
      code = B200CHEM_CELL_MASKED;
      if (lane == 0) {
        if (fcp) *fcp = 0.0;
        acc[kStMasked]++;
      }
    } else {
      double* yp = elem(bx.rhoY, i, j, k);
      double* fp = elem(bx.fY, i, j, k);
      double* tp = elem(bx.T, i, j, k);
      double yv[CPL], fv[CPL];
      double rho = 0.0;
      bool bad = false;
#pragma unroll
      for (int c = 0; c < CPL; ++c) {
        const int q = lane + 32 * c;
        yv[c] = 0.0;
        fv[c] = 0.0;
        if (q < N) {
          yv[c] = yp[q * bx.rhoY.ns];
          fv[c] = fp[q * bx.fY.ns];
          rho += yv[c];
        } else if (q == N) {
          yv[c] = *tp;
          fv[c] = *elem(bx.fH, i, j, k);
          bad |= !(yv[c] > 0.0);
        }
        bad |= !isfinite(yv[c]) || !isfinite(fv[c]);
      }
      rho = warp_sum(rho);
      bad |= !(rho > 0.0);
      if (__any_sync(kFull, bad)) {
        code = B200CHEM_CELL_NONFINITE;
        B.cnt = CellCounters{0, 0, 0, 0, 0, 0, 0};
      } else {
#pragma unroll
        for (int c = 0; c < CPL; ++c) B.F[c] = fv[c];
        code = B.integrate(yv, P.dt, P.max_steps);
      }
      double fh = 0.0;
      if (lane == 0) fh = *elem(bx.fH, i, j, k);
      if (code == 0) {
#pragma unroll
        for (int c = 0; c < CPL; ++c) {
          const int q = lane + 32 * c;
          if (q < N) yp[q * bx.rhoY.ns] = yv[c];
          else if (q == N) *tp = yv[c];
        }
        if (lane == 0) {
          double* hp = elem(bx.rhoH, i, j, k);
          *hp = *hp + P.dt * fh;
        }
      }
      if (lane == 0) {
        if (fcp) *fcp = (double)B.cnt.nfe;
        acc[kStCells]++;
        if (code != 0) acc[kStFailed]++;
        acc[kStNst] += B.cnt.nst;
        acc[kStNfe] += B.cnt.nfe;
        acc[kStNje] += B.cnt.nje;
        acc[kStNlu] += B.cnt.nlu;
        acc[kStNetf] += B.cnt.netf;
        acc[kStNcfn] += B.cnt.ncfn;
        acc[kStMaxNfe] = max(acc[kStMaxNfe], (long long)B.cnt.nfe);
        acc[kStMaxNst] = max(acc[kStMaxNst], (long long)B.cnt.nst);
      }
    }
    if (lane == 0 && P.status) P.status[cell] = code;
  }
  if (lane == 0 && P.stats) {
#pragma unroll
    for (int s = 0; s < kStMaxNfe; ++s)
      if (acc[s]) atomicAdd(reinterpret_cast<unsigned long long*>(P.stats + s), (unsigned long long)acc[s]);
    atomicMax(P.stats + kStMaxNfe, acc[kStMaxNfe]);
    atomicMax(P.stats + kStMaxNst, acc[kStMaxNst]);
  }
}

// ------------------------------------------------ thread-per-cell kernel
constexpr int kTpcBlock = 128;
#ifndef B200_TPC_MIN_CTAS
#define B200_TPC_MIN_CTAS 4
#endif

struct TpcParams {
  double* J;        // [n*n][threads] FP64 Jacobians, interleaved by thread
  void* A;          // [n*n][threads] LU factors (float or double), interleaved
  long long nthr;   // threads in the launch (interleave stride)
  int setup_ratio;  // setup round when waiting * ratio >= needing an RHS
};

__device__ __forceinline__ int find_box(const ReactParams& P, const long long* s_off, int nb_s, long long cell) {
  int lo = 0, hi = P.nbox - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    const long long o = nb_s ? s_off[mid] : P.boxes[mid].off;
    if (o <= cell) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

template <int NS, typename LUT>
__global__ void __launch_bounds__(kTpcBlock, B200_TPC_MIN_CTAS) react_tpc_kernel(ReactParams P, TpcParams Q) {
  using namespace b200::tpc;
  constexpr int n = NS + 1;
  extern __shared__ __align__(16) unsigned char dsm[];
  __shared__ DevMech s_mech;
  __shared__ long long s_off[65];
  if (threadIdx.x == 0) s_mech = P.mech;
  const int nb_s = P.nbox <= 64 ? P.nbox : 0;
  for (int b = threadIdx.x; b <= nb_s; b += blockDim.x) s_off[b] = (b < nb_s) ? P.boxes[b].off : P.total;
  __syncthreads();
  const DevMech& m = s_mech;
  const int lane = threadIdx.x & 31;
  const long long gtid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double* sC = reinterpret_cast<double*>(dsm) + threadIdx.x;
  double* sW = sC + NS * kTpcBlock;
  const IMat<double> J{Q.J + gtid, Q.nthr, n};
  const IMat<LUT> A{reinterpret_cast<LUT*>(Q.A) + gtid, Q.nthr, n};
  double atolv[n];
#pragma unroll
  for (int i = 0; i < n; ++i) atolv[i] = P.atol[i];

  Cell<NS, LUT> c;
  int phase = kIdle;
  long long cell = -1;
  bool qdone = false;  // warp-uniform: the queue is exhausted
  long long acc[kStCount];
#pragma unroll
  for (int i = 0; i < kStCount; ++i) acc[i] = 0;

  for (long long round = 0;; ++round) {
    // ---- refill idle threads from the global queue (warp-aggregated atomics)
    for (;;) {
      const unsigned idle = __ballot_sync(kFull, phase == kIdle);
      if (idle == 0) break;
      if (qdone) {
        if (phase == kIdle) phase = kExhausted;
        break;
      }
      const int leader = __ffs(idle) - 1;
      const int cnt = __popc(idle);
      unsigned long long base = 0;
      if (lane == leader) base = atomicAdd(P.queue, (unsigned long long)cnt);
      base = __shfl_sync(kFull, base, leader);
      if (base + cnt >= (unsigned long long)P.total) qdone = true;
      if (phase == kIdle) {
        const unsigned long long idx = base + __popc(idle & ((1u << lane) - 1u));
        if (idx >= (unsigned long long)P.total) {
          phase = kExhausted;
        } else {
          const long long cl = (long long)idx;
          const DevBox& bx = P.boxes[find_box(P, s_off, nb_s, cl)];
          const long long loc = cl - bx.off;
          const int i = bx.lo0 + (int)(loc % bx.nx);
          const int j = bx.lo1 + (int)((loc / bx.nx) % bx.ny);
          const int k = bx.lo2 + (int)(loc / ((long long)bx.nx * bx.ny));
          bool masked = false;
          if (bx.mask.p)
            masked = bx.mask.p[(long long)(i - bx.mask.lo0) + (long long)(j - bx.mask.lo1) * bx.mask.js +
                               (long long)(k - bx.mask.lo2) * bx.mask.ks] == 0;
          int code = 0;
          if (masked) {
            if (bx.fc.p) *elem(bx.fc, i, j, k) = 0.0;
            acc[kStMasked]++;
            code = B200CHEM_CELL_MASKED;
          } else {
            const double* yp = elem(bx.rhoY, i, j, k);
            const double* fp = elem(bx.fY, i, j, k);
            double rho = 0.0;
            bool bad = false;
#pragma unroll
            for (int q = 0; q < NS; ++q) {
              c.zn[0][q] = yp[q * bx.rhoY.ns];
              c.F[q] = fp[q * bx.fY.ns];
              rho += c.zn[0][q];
              bad |= !isfinite(c.zn[0][q]) || !isfinite(c.F[q]);
            }
            c.zn[0][NS] = *elem(bx.T, i, j, k);
            c.F[NS] = *elem(bx.fH, i, j, k);
            bad |= !(c.zn[0][NS] > 0.0) || !isfinite(c.zn[0][NS]) || !isfinite(c.F[NS]) || !(rho > 0.0);
            if (bad) {
              code = B200CHEM_CELL_NONFINITE;
              if (bx.fc.p) *elem(bx.fc, i, j, k) = 0.0;
              acc[kStCells]++;
              acc[kStFailed]++;
            } else {
              cell = cl;
              phase = c_begin<NS, LUT>(c, atolv, P.rtol, P.dt, P.qmax, P.max_steps);
            }
          }
          if (phase == kIdle && P.status) P.status[cl] = code;
        }
      }
    }
    const unsigned live = __ballot_sync(kFull, phase != kExhausted);
    if (live == 0) break;
    // ---- one round: RHS for every cell that needs it, or Jacobian + LU
    const unsigned nr = __ballot_sync(kFull, needs_rhs(phase));
    const unsigned ns = __ballot_sync(kFull, phase == kSetup);
    const bool setup_round = ns != 0 && (nr == 0 || __popc(ns) * Q.setup_ratio >= __popc(nr));
    int status = 0;
    if (setup_round) {
      if (phase == kSetup) {
        const int ier = c_setup<NS, LUT>(c, m, J, A, sC, sW, kTpcBlock);
        phase = c_advance<NS, LUT>(c, kLAfterSetup, nullptr, ier, atolv, P.rtol, J, A, &status);
      }
    } else if (needs_rhs(phase)) {
      double f[n];
      tpc_rhs<NS>(m, c.yev, c.F, f, sC, sW, kTpcBlock);
      c.cnt.nfe++;
      const int lab = (phase == kRhsF0) ? kLAfterF0
                      : (phase == kRhsHin) ? kLAfterHin
                      : (phase == kRhsNStart) ? kLAfterNStart
                      : (phase == kRhsNIter) ? kLAfterNIter : kLAfterRestart;
      phase = c_advance<NS, LUT>(c, lab, f, 0, atolv, P.rtol, J, A, &status);
    }
    // ---- finished cells: write back and account
    if (phase == kIdle && cell >= 0) {
      const DevBox& bx = P.boxes[find_box(P, s_off, nb_s, cell)];
      const long long loc = cell - bx.off;
      const int i = bx.lo0 + (int)(loc % bx.nx);
      const int j = bx.lo1 + (int)((loc / bx.nx) % bx.ny);
      const int k = bx.lo2 + (int)(loc / ((long long)bx.nx * bx.ny));
      if (status == 0) {
        // y(dt) from the Nordsieck array (Horner in s = (dt - tn)/h)
        const double s = (P.dt - c.tn) / c.h;
        double* yp = elem(bx.rhoY, i, j, k);
#pragma unroll
        for (int q = 0; q < n; ++q) {
          double v = c.zn[c.q][q];
          for (int jj = c.q - 1; jj >= 0; --jj) v = c.zn[jj][q] + s * v;
          if (q < NS) yp[q * bx.rhoY.ns] = v;
          else *elem(bx.T, i, j, k) = v;
        }
        double* hp = elem(bx.rhoH, i, j, k);
        *hp = *hp + P.dt * c.F[NS];
      } else {
        acc[kStFailed]++;
      }
      if (bx.fc.p) *elem(bx.fc, i, j, k) = (double)c.cnt.nfe;
      if (P.status) P.status[cell] = status;
      acc[kStCells]++;
      acc[kStNst] += c.cnt.nst;
      acc[kStNfe] += c.cnt.nfe;
      acc[kStNje] += c.cnt.nje;
      acc[kStNlu] += c.cnt.nlu;
      acc[kStNetf] += c.cnt.netf;
      acc[kStNcfn] += c.cnt.ncfn;
      acc[kStMaxNfe] = max(acc[kStMaxNfe], (long long)c.cnt.nfe);
      acc[kStMaxNst] = max(acc[kStMaxNst], (long long)c.cnt.nst);
      cell = -1;
    }
  }
  if (P.stats) {
#pragma unroll
    for (int s = 0; s < kStMaxNfe; ++s) {
      long long v = acc[s];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
      if (lane == 0 && v) atomicAdd(reinterpret_cast<unsigned long long*>(P.stats + s), (unsigned long long)v);
    }
    long long mx = acc[kStMaxNfe], ms = acc[kStMaxNst];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      mx = max(mx, __shfl_xor_sync(kFull, mx, o));
      ms = max(ms, __shfl_xor_sync(kFull, ms, o));
    }
    if (lane == 0) {
      atomicMax(P.stats + kStMaxNfe, mx);
      atomicMax(P.stats + kStMaxNst, ms);
    }
  }
}

// ------------------------------------------------ evaluation-only kernels
struct EvalParams {
  DevMech mech;
  const double* y;
  const double* F;
  double* out;
  long long ncells;
  int warp_bytes;
  int Npad, Rpad, ldj, ldl;
  int what;  // 0 rhs, 1 jac
};

template <int CPL>
__global__ void __launch_bounds__(128) eval_kernel(EvalParams P) {
  extern __shared__ __align__(16) unsigned char dsm[];
  __shared__ DevMech s_mech;
  if (threadIdx.x == 0) s_mech = P.mech;
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int N = P.mech.N, n = N + 1;
  WarpBdf<CPL, double> B;
  carve<CPL, double>(B, dsm + (size_t)w * P.warp_bytes, n, P.Npad, P.Rpad, P.ldj, P.ldl);
  const long long wstride = (long long)gridDim.x * (blockDim.x >> 5);
  for (long long c0 = (long long)blockIdx.x * (blockDim.x >> 5) + w; c0 < P.ncells; c0 += wstride) {
    double y[CPL], F[CPL], yd[CPL];
#pragma unroll
    for (int c = 0; c < CPL; ++c) {
      const int q = lane + 32 * c;
      y[c] = (q < n) ? P.y[c0 * n + q] : 0.0;
      F[c] = (q < n) ? P.F[c0 * n + q] : 0.0;
    }
    if (P.what == 0) {
      warp_rhs<CPL>(s_mech, B.ms, y, F, yd, lane);
#pragma unroll
      for (int c = 0; c < CPL; ++c)
        if (lane + 32 * c < n) P.out[c0 * n + lane + 32 * c] = yd[c];
    } else {
      warp_jac<CPL>(s_mech, B.ms, y, F, yd, B.J, B.ldj, lane);
      for (int i = 0; i < n; ++i)
#pragma unroll
        for (int c = 0; c < CPL; ++c)
          if (lane + 32 * c < n) P.out[(c0 * n + i) * n + lane + 32 * c] = B.J[i * B.ldj + lane + 32 * c];
    }
    __syncwarp();
  }
}

// T from (h, Y) by Newton on h(T) = sum Y_k h_k(T), warp per cell (HY2T).
template <int CPL>
__device__ double warp_t_from_hy(const DevMech& m, const double (&Y)[CPL], double h, double T, int lane) {
  for (int it = 0; it < 100; ++it) {
    const double lnT = log(T);
    double hs = 0.0, cs = 0.0;
#pragma unroll
    for (int c = 0; c < CPL; ++c) {
      const int k = lane + 32 * c;
      if (k < m.N) {
        double cpR, hRT, sR, dcpR;
        nasa7(m, k, T, lnT, cpR, hRT, sR, dcpR);
        const double iw = __ldg(m.inv_mw + k);
        hs += Y[c] * hRT * kRu * T * iw;
        cs += Y[c] * cpR * kRu * iw;
      }
    }
    hs = warp_sum(hs);
    cs = warp_sum(cs);
    const double dT = (h - hs) / cs;
    T += dT;
    if (fabs(dT) <= 1e-12 * T) break;
  }
  return T;
}

struct InstParams {
  DevMech mech;
  const double* rhoY;  // MKS, component-major
  const double* rhoH;
  double* T;
  double* rhoYdot;     // MKS, component-major (may be null: T only)
  long long ncells;
  int warp_bytes;
  int Npad, Rpad, ldj, ldl;
};

template <int CPL>
__global__ void __launch_bounds__(128) inst_rr_kernel(InstParams P) {
  extern __shared__ __align__(16) unsigned char dsm[];
  __shared__ DevMech s_mech;
  if (threadIdx.x == 0) s_mech = P.mech;
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int N = P.mech.N, n = N + 1;
  WarpBdf<CPL, double> B;
  carve<CPL, double>(B, dsm + (size_t)w * P.warp_bytes, n, P.Npad, P.Rpad, P.ldj, P.ldl);
  const long long wstride = (long long)gridDim.x * (blockDim.x >> 5);
  for (long long c0 = (long long)blockIdx.x * (blockDim.x >> 5) + w; c0 < P.ncells; c0 += wstride) {
    double ry[CPL], Y[CPL];
    double rho = 0.0;
#pragma unroll
    for (int c = 0; c < CPL; ++c) {
      const int k = lane + 32 * c;
      ry[c] = (k < N) ? P.rhoY[(long long)k * P.ncells + c0] : 0.0;
      rho += ry[c];
    }
    rho = warp_sum(rho);
    const double rinv = 1.0 / rho;
#pragma unroll
    for (int c = 0; c < CPL; ++c) Y[c] = ry[c] * rinv;
    const double h = P.rhoH[c0] * rinv * 1.0e4;  // J/kg -> erg/g
    const double T = warp_t_from_hy<CPL>(s_mech, Y, h, P.T[c0], lane);
    if (lane == 0) P.T[c0] = T;
    if (P.rhoYdot) {
      double y[CPL], F[CPL], yd[CPL];
#pragma unroll
      for (int c = 0; c < CPL; ++c) {
        const int k = lane + 32 * c;
        y[c] = (k < N) ? ry[c] * 1.0e-3 : (k == N ? T : 0.0);  // kg/m^3 -> g/cm^3
        F[c] = 0.0;
      }
      warp_rhs<CPL>(s_mech, B.ms, y, F, yd, lane);
#pragma unroll
      for (int c = 0; c < CPL; ++c) {
        const int k = lane + 32 * c;
        if (k < N) P.rhoYdot[(long long)k * P.ncells + c0] = yd[c] * 1.0e3;  // g/cm^3/s -> kg/m^3/s
      }
    }
    __syncwarp();
  }
}

}  // namespace

// ------------------------------------------------------------------ handle
struct b200chem_reactor {
  int device = 0;
  int N = 0, R = 0, n = 0, cpl = 1;
  b200chem_opts opts{};
  DevMech mech{};
  void* d_mech = nullptr;
  double* d_atol = nullptr;
  std::vector<double> atol_host;
  unsigned long long* d_scratch = nullptr;  // [0] queue, [1..] stats
  DevBox* d_boxes = nullptr;
  int boxes_cap = 0;
  DevBox* h_boxes = nullptr;  // pinned staging
  cudaEvent_t stage_ev = nullptr;
  bool stage_pending = false;
  int sm_count = 0;
  int Npad = 32, Rpad = 32, ldj = 0, ldl = 0;
  int warps_per_cta = 4;
  void* d_tpc = nullptr;  // thread-per-cell scratch (Jacobians + LU factors)
  size_t tpc_bytes = 0;
};

namespace {

// warps per CTA (<= want) whose shared memory fits the opt-in per-block maximum
int fit_warps(int warp_bytes, int want) {
  int dev = 0, maxb = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&maxb, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  maxb -= 1024;  // static shared memory of the kernels
  int w = want;
  while (w > 1 && w * warp_bytes > maxb) --w;
  return w;
}

int smem_warp_bytes(const b200chem_reactor* h, bool fp64_lu) {
  size_t b = sizeof(double) * (5 * (size_t)h->Npad + 5 * (size_t)h->Rpad + (size_t)h->n * h->ldj);
  b += (fp64_lu ? sizeof(double) : sizeof(float)) * (size_t)h->n * h->ldl;
  b += sizeof(int) * (size_t)h->n;
  return (int)((b + 15) & ~(size_t)15);
}

template <typename T>
size_t push(std::vector<unsigned char>& buf, const std::vector<T>& v) {
  size_t off = (buf.size() + 255) & ~(size_t)255;
  buf.resize(off + sizeof(T) * std::max<size_t>(v.size(), 1));
  if (!v.empty()) memcpy(buf.data() + off, v.data(), sizeof(T) * v.size());
  return off;
}

template <int CPL, typename LUT>
int set_kernel_smem(int bytes) {
  CK(cudaFuncSetAttribute(react_kernel<CPL, LUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  return 0;
}

template <int CPL, typename LUT>
int launch_react(b200chem_reactor* h, const ReactParams& P, int warps, cudaStream_t st) {
  const int block = 32 * warps;
  const int smem = P.warp_bytes * warps;
  int err = set_kernel_smem<CPL, LUT>(smem);
  if (err) return err;
  int per_sm = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, react_kernel<CPL, LUT>, block, smem));
  if (per_sm < 1) return set_err(B200CHEM_ETOOBIG, "react kernel does not fit on an SM (%d B smem)", smem);
  long long need = (P.total + warps - 1) / warps;
  long long grid = std::min<long long>(need, (long long)h->sm_count * per_sm);
  if (grid < 1) grid = 1;
  react_kernel<CPL, LUT><<<(unsigned)grid, block, smem, st>>>(P);
  CK(cudaGetLastError());
  return 0;
}

bool tpc_supported(int N) { return N == 9 || N == 21; }

template <int NS, typename LUT>
int launch_tpc(b200chem_reactor* h, const ReactParams& P, cudaStream_t st) {
  const int n = NS + 1;
  const int smem = (int)(2 * sizeof(double) * NS * kTpcBlock);
  CK(cudaFuncSetAttribute(react_tpc_kernel<NS, LUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  int per_sm = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, react_tpc_kernel<NS, LUT>, kTpcBlock, smem));
  if (per_sm < 1) return set_err(B200CHEM_ETOOBIG, "thread-per-cell kernel does not fit on an SM");
  if (h->opts.ctas_per_sm > 0) per_sm = std::min(per_sm, (int)h->opts.ctas_per_sm);
  long long need = (P.total + kTpcBlock - 1) / kTpcBlock;
  long long grid = std::min<long long>(need, (long long)h->sm_count * per_sm);
  if (grid < 1) grid = 1;
  const long long nthr = grid * kTpcBlock;
  const size_t bytes = (size_t)nthr * n * n * (sizeof(double) + sizeof(LUT));
  if (bytes > h->tpc_bytes) {
    if (h->d_tpc) {
      CK(cudaStreamSynchronize(st));
      cudaFree(h->d_tpc);
      h->d_tpc = nullptr;
      h->tpc_bytes = 0;
    }
    if (cudaMalloc(&h->d_tpc, bytes) != cudaSuccess) {
      cudaGetLastError();
      return set_err(B200CHEM_ENOMEM, "cannot allocate %zu bytes of integrator scratch", bytes);
    }
    h->tpc_bytes = bytes;
  }
  TpcParams Q;
  Q.J = static_cast<double*>(h->d_tpc);
  Q.A = static_cast<void*>(static_cast<double*>(h->d_tpc) + (size_t)nthr * n * n);
  Q.nthr = nthr;
  Q.setup_ratio = h->opts.setup_ratio > 0 ? h->opts.setup_ratio : 2;
  react_tpc_kernel<NS, LUT><<<(unsigned)grid, kTpcBlock, smem, st>>>(P, Q);
  CK(cudaGetLastError());
  return 0;
}

template <typename LUT>
int launch_tpc_n(b200chem_reactor* h, const ReactParams& P, cudaStream_t st) {
  switch (h->N) {
    case 9: return launch_tpc<9, LUT>(h, P, st);
    case 21: return launch_tpc<21, LUT>(h, P, st);
    default: return set_err(B200CHEM_EINVAL, "no thread-per-cell variant for N=%d", h->N);
  }
}

int do_react(b200chem_reactor* h, const std::vector<DevBox>& boxes, long long total, double dt, cudaStream_t st,
             int32_t* cell_status, b200chem_stats* stats) {
  const int nbox = (int)boxes.size();
  if (nbox > h->boxes_cap) {
    if (h->stage_pending) CK(cudaEventSynchronize(h->stage_ev));
    h->stage_pending = false;
    if (h->d_boxes) cudaFree(h->d_boxes);
    if (h->h_boxes) cudaFreeHost(h->h_boxes);
    int cap = std::max(nbox, 64);
    CK(cudaMalloc(&h->d_boxes, sizeof(DevBox) * cap));
    CK(cudaMallocHost(&h->h_boxes, sizeof(DevBox) * cap));
    h->boxes_cap = cap;
  }
  if (h->stage_pending) CK(cudaEventSynchronize(h->stage_ev));
  memcpy(h->h_boxes, boxes.data(), sizeof(DevBox) * nbox);
  CK(cudaMemcpyAsync(h->d_boxes, h->h_boxes, sizeof(DevBox) * nbox, cudaMemcpyHostToDevice, st));
  CK(cudaEventRecord(h->stage_ev, st));
  h->stage_pending = true;
  CK(cudaMemsetAsync(h->d_scratch, 0, sizeof(unsigned long long) * (1 + kStCount), st));
  ReactParams P;
  P.mech = h->mech;
  P.boxes = h->d_boxes;
  P.nbox = nbox;
  P.total = total;
  P.dt = dt;
  P.max_steps = h->opts.max_steps;
  P.qmax = h->opts.max_order;
  P.rtol = h->opts.rtol;
  P.atol = h->d_atol;
  P.queue = h->d_scratch;
  P.stats = reinterpret_cast<long long*>(h->d_scratch + 1);
  P.status = cell_status;
  P.Npad = h->Npad;
  P.Rpad = h->Rpad;
  P.ldj = h->ldj;
  P.ldl = h->ldl;
  const bool fp64 = h->opts.lu_fp64 != 0;
  P.warp_bytes = smem_warp_bytes(h, fp64);
  const int warps = fit_warps(P.warp_bytes, h->opts.warps_per_cta > 0 ? h->opts.warps_per_cta : h->warps_per_cta);
  int err;
  const bool use_tpc = (h->opts.kernel == 1) || (h->opts.kernel == 0 && tpc_supported(h->N));
  if (h->opts.kernel == 1 && !tpc_supported(h->N))
    return set_err(B200CHEM_EINVAL, "thread-per-cell kernel requested but not compiled for N=%d", h->N);
  if (total > 0) {
    if (use_tpc) err = fp64 ? launch_tpc_n<double>(h, P, st) : launch_tpc_n<float>(h, P, st);
    else if (h->cpl == 1) err = fp64 ? launch_react<1, double>(h, P, warps, st) : launch_react<1, float>(h, P, warps, st);
    else err = fp64 ? launch_react<2, double>(h, P, warps, st) : launch_react<2, float>(h, P, warps, st);
    if (err) return err;
  }
  if (stats) {
    long long st_h[kStCount];
    CK(cudaMemcpyAsync(st_h, h->d_scratch + 1, sizeof(st_h), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    stats->n_cells = st_h[kStCells];
    stats->n_masked = st_h[kStMasked];
    stats->n_failed = st_h[kStFailed];
    stats->nst = st_h[kStNst];
    stats->nfe = st_h[kStNfe];
    stats->nje = st_h[kStNje];
    stats->nlu = st_h[kStNlu];
    stats->netf = st_h[kStNetf];
    stats->ncfn = st_h[kStNcfn];
    stats->max_nfe = (int32_t)st_h[kStMaxNfe];
    stats->max_nst = (int32_t)st_h[kStMaxNst];
    if (stats->n_failed > 0) return set_err(B200CHEM_EINTEGRATE, "%lld cell(s) failed to integrate", stats->n_failed);
  }
  return 0;
}

DevArr to_dev(const b200chem_array4& a) {
  DevArr d;
  d.p = a.p;
  d.js = a.jstride;
  d.ks = a.kstride;
  d.ns = a.nstride;
  d.lo0 = a.lo[0];
  d.lo1 = a.lo[1];
  d.lo2 = a.lo[2];
  d.pad = 0;
  return d;
}

}  // namespace

// ------------------------------------------------------------------ C ABI
extern "C" {

int b200chem_version(void) { return B200CHEM_VERSION; }
const char* b200chem_last_error(void) { return g_err.c_str(); }

b200chem_handle b200chem_create(const b200chem_mech_desc* md, const b200chem_opts* o) {
  if (!md || !o) {
    set_err(B200CHEM_EINVAL, "null mechanism or options");
    return nullptr;
  }
  const int N = md->n_species, R = md->n_reactions;
  if (N < 1 || R < 0) {
    set_err(B200CHEM_EINVAL, "bad mechanism sizes N=%d R=%d", N, R);
    return nullptr;
  }
  if (N + 1 > 64) {
    set_err(B200CHEM_ETOOBIG, "N+1 = %d components; this build supports up to 64", N + 1);
    return nullptr;
  }
  if (o->reactor_type != 2) {
    set_err(B200CHEM_EINVAL, "reactor_type %d: only 2 (HP) is supported", o->reactor_type);
    return nullptr;
  }
  if (o->max_order < 1 || o->max_order > kQmaxLim || o->max_steps < 1 || !(o->rtol > 0.0) || !(o->atol > 0.0)) {
    set_err(B200CHEM_EINVAL, "bad options (max_order 1..5, max_steps>0, rtol>0, atol>0)");
    return nullptr;
  }
  auto* h = new b200chem_reactor();
  h->N = N;
  h->R = R;
  h->n = N + 1;
  h->cpl = (N + 1 <= 32) ? 1 : 2;
  h->opts = *o;
  h->Npad = 32 * h->cpl;
  h->Rpad = std::max(32, ((R + 31) / 32) * 32);
  h->ldj = h->n | 1;
  h->ldl = h->n | 1;
  // --- flatten to structure-of-arrays
  std::vector<double> mw(N), imw(N), nasa(15 * (size_t)N), arr(3 * (size_t)R), arrlo(3 * (size_t)R),
      arrrev(3 * (size_t)R), troe(4 * (size_t)R), sdnu(R), effm1;
  std::vector<int> rtype(R), rflags(R), sp(8 * (size_t)R), nu(8 * (size_t)R), effptr(R + 1), effsp;
  for (int k = 0; k < N; ++k) {
    mw[k] = md->mw[k];
    imw[k] = 1.0 / md->mw[k];
    for (int c = 0; c < 15; ++c) nasa[(size_t)c * N + k] = md->nasa[15 * k + c];
  }
  std::vector<std::vector<std::pair<int, double>>> inc(N);
  for (int j = 0; j < R; ++j) {
    rtype[j] = md->rtype[j];
    rflags[j] = md->rflags[j];
    for (int c = 0; c < 3; ++c) {
      arr[(size_t)c * R + j] = md->arr[3 * j + c];
      arrlo[(size_t)c * R + j] = md->arr_lo[3 * j + c];
      arrrev[(size_t)c * R + j] = md->arr_rev[3 * j + c];
    }
    const double* t = md->troe + 4 * j;
    troe[j] = t[0];
    troe[(size_t)R + j] = 1.0 / t[1];
    troe[2 * (size_t)R + j] = 1.0 / t[2];
    troe[3 * (size_t)R + j] = t[3];
    double sd = 0.0;
    std::vector<double> dn(N, 0.0);
    for (int s = 0; s < 8; ++s) {
      const int k = md->sp[8 * j + s];
      const int v = md->nu[8 * j + s];
      sp[(size_t)s * R + j] = k;
      nu[(size_t)s * R + j] = (k >= 0) ? (s < 4 ? -v : v) : 0;
      if (k >= 0) {
        if (k >= N || v <= 0) {
          delete h;
          set_err(B200CHEM_EINVAL, "reaction %d: bad species slot", j);
          return nullptr;
        }
        dn[k] += (s < 4 ? -v : v);
        sd += (s < 4 ? -v : v);
      }
    }
    sdnu[j] = sd;
    for (int k = 0; k < N; ++k)
      if (dn[k] != 0.0) inc[k].push_back({j, dn[k]});
    effptr[j] = (int)effsp.size();
    for (int e = md->eff_ptr[j]; e < md->eff_ptr[j + 1]; ++e) {
      if (md->eff_sp[e] < 0 || md->eff_sp[e] >= N) {
        delete h;
        set_err(B200CHEM_EINVAL, "reaction %d: third-body species index out of range", j);
        return nullptr;
      }
      effsp.push_back(md->eff_sp[e]);
      effm1.push_back(md->eff_val[e] - 1.0);
    }
  }
  effptr[R] = (int)effsp.size();
  std::vector<int> incptr(N + 1), incrxn;
  std::vector<double> incnu;
  for (int k = 0; k < N; ++k) {
    incptr[k] = (int)incrxn.size();
    for (auto& pr : inc[k]) {
      incrxn.push_back(pr.first);
      incnu.push_back(pr.second);
    }
  }
  incptr[N] = (int)incrxn.size();
  std::vector<unsigned char> buf;
  size_t o_mw = push(buf, mw), o_imw = push(buf, imw), o_nasa = push(buf, nasa), o_rtype = push(buf, rtype),
         o_rflags = push(buf, rflags), o_arr = push(buf, arr), o_arrlo = push(buf, arrlo),
         o_arrrev = push(buf, arrrev), o_troe = push(buf, troe), o_sp = push(buf, sp), o_nu = push(buf, nu),
         o_sdnu = push(buf, sdnu), o_effptr = push(buf, effptr), o_effsp = push(buf, effsp),
         o_effm1 = push(buf, effm1), o_incptr = push(buf, incptr), o_incrxn = push(buf, incrxn),
         o_incnu = push(buf, incnu);
  auto fail = [&](cudaError_t e, const char* what) -> b200chem_handle {
    set_err(B200CHEM_ECUDA, "%s: %s", what, cudaGetErrorString(e));
    if (h->d_mech) cudaFree(h->d_mech);
    if (h->d_atol) cudaFree(h->d_atol);
    if (h->d_scratch) cudaFree(h->d_scratch);
    delete h;
    return nullptr;
  };
  cudaError_t e;
  if ((e = cudaGetDevice(&h->device)) != cudaSuccess) return fail(e, "cudaGetDevice");
  if ((e = cudaDeviceGetAttribute(&h->sm_count, cudaDevAttrMultiProcessorCount, h->device)) != cudaSuccess)
    return fail(e, "cudaDeviceGetAttribute");
  if ((e = cudaMalloc(&h->d_mech, buf.size())) != cudaSuccess) return fail(e, "cudaMalloc(mechanism)");
  if ((e = cudaMemcpy(h->d_mech, buf.data(), buf.size(), cudaMemcpyHostToDevice)) != cudaSuccess)
    return fail(e, "cudaMemcpy(mechanism)");
  auto* base = static_cast<unsigned char*>(h->d_mech);
  DevMech& m = h->mech;
  m.N = N;
  m.R = R;
  m.n = N + 1;
  m.mw = reinterpret_cast<const double*>(base + o_mw);
  m.inv_mw = reinterpret_cast<const double*>(base + o_imw);
  m.nasa = reinterpret_cast<const double*>(base + o_nasa);
  m.rtype = reinterpret_cast<const int*>(base + o_rtype);
  m.rflags = reinterpret_cast<const int*>(base + o_rflags);
  m.arr = reinterpret_cast<const double*>(base + o_arr);
  m.arr_lo = reinterpret_cast<const double*>(base + o_arrlo);
  m.arr_rev = reinterpret_cast<const double*>(base + o_arrrev);
  m.troe = reinterpret_cast<const double*>(base + o_troe);
  m.sp = reinterpret_cast<const int*>(base + o_sp);
  m.nu = reinterpret_cast<const int*>(base + o_nu);
  m.sdnu = reinterpret_cast<const double*>(base + o_sdnu);
  m.eff_ptr = reinterpret_cast<const int*>(base + o_effptr);
  m.eff_sp = reinterpret_cast<const int*>(base + o_effsp);
  m.eff_m1 = reinterpret_cast<const double*>(base + o_effm1);
  m.inc_ptr = reinterpret_cast<const int*>(base + o_incptr);
  m.inc_rxn = reinterpret_cast<const int*>(base + o_incrxn);
  m.inc_nu = reinterpret_cast<const double*>(base + o_incnu);
  h->atol_host.assign(h->n, o->atol);
  if ((e = cudaMalloc(&h->d_atol, sizeof(double) * h->n)) != cudaSuccess) return fail(e, "cudaMalloc(atol)");
  if ((e = cudaMemcpy(h->d_atol, h->atol_host.data(), sizeof(double) * h->n, cudaMemcpyHostToDevice)) != cudaSuccess)
    return fail(e, "cudaMemcpy(atol)");
  if ((e = cudaMalloc(&h->d_scratch, sizeof(unsigned long long) * (1 + kStCount))) != cudaSuccess)
    return fail(e, "cudaMalloc(scratch)");
  if ((e = cudaEventCreateWithFlags(&h->stage_ev, cudaEventDisableTiming)) != cudaSuccess)
    return fail(e, "cudaEventCreate");
  return h;
}

int b200chem_set_typvals(b200chem_handle h, const double* typ, int32_t n) {
  if (!h || !typ) return set_err(B200CHEM_EINVAL, "null argument");
  if (n != h->n) return set_err(B200CHEM_EINVAL, "typical values: got %d, need N+1 = %d", n, h->n);
  for (int i = 0; i < n; ++i) {
    if (!(typ[i] > 0.0)) return set_err(B200CHEM_EINVAL, "typical value %d is not positive", i);
    h->atol_host[i] = h->opts.atol * typ[i];
  }
  CK(cudaMemcpy(h->d_atol, h->atol_host.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
  return 0;
}

int b200chem_react(b200chem_handle h, const b200chem_box_view* views, int32_t nbox, double* dt_react,
                   double* time, void* stream, int32_t* cell_status, b200chem_stats* stats) {
  if (!h || (!views && nbox > 0) || nbox < 0 || !dt_react) return set_err(B200CHEM_EINVAL, "bad arguments");
  if (!(*dt_react > 0.0)) return set_err(B200CHEM_EINVAL, "dt_react must be positive");
  std::vector<DevBox> boxes(nbox);
  long long total = 0;
  for (int b = 0; b < nbox; ++b) {
    const b200chem_box_view& v = views[b];
    DevBox& d = boxes[b];
    d.lo0 = v.lo[0];
    d.lo1 = v.lo[1];
    d.lo2 = v.lo[2];
    d.nx = v.hi[0] - v.lo[0] + 1;
    d.ny = v.hi[1] - v.lo[1] + 1;
    d.nz = v.hi[2] - v.lo[2] + 1;
    if (d.nx < 1 || d.ny < 1 || d.nz < 1) return set_err(B200CHEM_EINVAL, "box %d is empty or inverted", b);
    if (!v.rhoY.p || !v.extF_rhoY.p || !v.T.p || !v.rhoH.p || !v.extF_rhoH.p)
      return set_err(B200CHEM_EINVAL, "box %d: null state array", b);
    d.off = total;
    total += (long long)d.nx * d.ny * d.nz;
    d.rhoY = to_dev(v.rhoY);
    d.fY = to_dev(v.extF_rhoY);
    d.T = to_dev(v.T);
    d.rhoH = to_dev(v.rhoH);
    d.fH = to_dev(v.extF_rhoH);
    d.fc = to_dev(v.fctCount);
    d.mask.p = v.mask.p;
    d.mask.js = v.mask.jstride;
    d.mask.ks = v.mask.kstride;
    d.mask.lo0 = v.mask.lo[0];
    d.mask.lo1 = v.mask.lo[1];
    d.mask.lo2 = v.mask.lo[2];
    d.mask.pad = 0;
  }
  const int err = do_react(h, boxes, total, *dt_react, static_cast<cudaStream_t>(stream), cell_status, stats);
  if (time) *time += *dt_react;
  return err;
}

int b200chem_react_flat(b200chem_handle h, double* rhoY, const double* extF_rhoY, double* T, double* rhoH,
                        const double* extF_rhoH, double* fctCount, const int32_t* mask, int64_t ncells,
                        double* dt_react, double* time, void* stream, int32_t* cell_status, b200chem_stats* stats) {
  if (!h || ncells < 0 || !dt_react) return set_err(B200CHEM_EINVAL, "bad arguments");
  if (ncells > 0 && (!rhoY || !extF_rhoY || !T || !rhoH || !extF_rhoH))
    return set_err(B200CHEM_EINVAL, "null state array");
  if (!(*dt_react > 0.0)) return set_err(B200CHEM_EINVAL, "dt_react must be positive");
  if (ncells > 0x7fffffffLL) return set_err(B200CHEM_ETOOBIG, "ncells above 2^31-1 in one flat call");
  std::vector<DevBox> boxes;
  if (ncells > 0) {
    DevBox d{};
    d.nx = (int)ncells;
    d.ny = d.nz = 1;
    d.off = 0;
    auto mk = [&](const double* p) {
      DevArr a{};
      a.p = const_cast<double*>(p);
      a.js = a.ks = ncells;
      a.ns = ncells;
      return a;
    };
    d.rhoY = mk(rhoY);
    d.fY = mk(extF_rhoY);
    d.T = mk(T);
    d.rhoH = mk(rhoH);
    d.fH = mk(extF_rhoH);
    d.fc = mk(fctCount);
    d.mask.p = mask;
    d.mask.js = d.mask.ks = ncells;
    boxes.push_back(d);
  }
  const int err = do_react(h, boxes, ncells, *dt_react, static_cast<cudaStream_t>(stream), cell_status, stats);
  if (time) *time += *dt_react;
  return err;
}

int b200chem_destroy(b200chem_handle h) {
  if (!h) return 0;
  if (h->stage_pending) cudaEventSynchronize(h->stage_ev);
  if (h->stage_ev) cudaEventDestroy(h->stage_ev);
  if (h->d_mech) cudaFree(h->d_mech);
  if (h->d_atol) cudaFree(h->d_atol);
  if (h->d_scratch) cudaFree(h->d_scratch);
  if (h->d_boxes) cudaFree(h->d_boxes);
  if (h->h_boxes) cudaFreeHost(h->h_boxes);
  if (h->d_tpc) cudaFree(h->d_tpc);
  delete h;
  return 0;
}

static int eval_launch(b200chem_handle h, const double* y, const double* F, int64_t ncells, double* out, void* stream,
                       int what) {
  if (!h || !y || !F || !out || ncells < 0) return set_err(B200CHEM_EINVAL, "bad arguments");
  if (ncells == 0) return 0;
  EvalParams P;
  P.mech = h->mech;
  P.y = y;
  P.F = F;
  P.out = out;
  P.ncells = ncells;
  P.warp_bytes = smem_warp_bytes(h, true);
  P.Npad = h->Npad;
  P.Rpad = h->Rpad;
  P.ldj = h->ldj;
  P.ldl = h->ldl;
  P.what = what;
  const int warps = fit_warps(P.warp_bytes, 4), smem = P.warp_bytes * warps;
  const long long grid = std::min<long long>((ncells + warps - 1) / warps, (long long)h->sm_count * 16);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (h->cpl == 1) {
    CK(cudaFuncSetAttribute(eval_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    eval_kernel<1><<<(unsigned)grid, 32 * warps, smem, st>>>(P);
  } else {
    CK(cudaFuncSetAttribute(eval_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    eval_kernel<2><<<(unsigned)grid, 32 * warps, smem, st>>>(P);
  }
  CK(cudaGetLastError());
  return 0;
}

int b200chem_eval_rhs(b200chem_handle h, const double* y, const double* forcing, int64_t ncells, double* ydot,
                      void* stream) {
  return eval_launch(h, y, forcing, ncells, ydot, stream, 0);
}

int b200chem_eval_jac(b200chem_handle h, const double* y, const double* forcing, int64_t ncells, double* jac,
                      void* stream) {
  return eval_launch(h, y, forcing, ncells, jac, stream, 1);
}

static int inst_launch(b200chem_handle h, const double* rhoY, const double* rhoH, double* T, double* rhoYdot,
                       int64_t ncells, void* stream) {
  if (!h || !rhoY || !rhoH || !T || ncells < 0) return set_err(B200CHEM_EINVAL, "bad arguments");
  if (ncells == 0) return 0;
  InstParams P;
  P.mech = h->mech;
  P.rhoY = rhoY;
  P.rhoH = rhoH;
  P.T = T;
  P.rhoYdot = rhoYdot;
  P.ncells = ncells;
  P.warp_bytes = smem_warp_bytes(h, true);
  P.Npad = h->Npad;
  P.Rpad = h->Rpad;
  P.ldj = h->ldj;
  P.ldl = h->ldl;
  const int warps = fit_warps(P.warp_bytes, 4), smem = P.warp_bytes * warps;
  const long long grid = std::min<long long>((ncells + warps - 1) / warps, (long long)h->sm_count * 16);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (h->cpl == 1) {
    CK(cudaFuncSetAttribute(inst_rr_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    inst_rr_kernel<1><<<(unsigned)grid, 32 * warps, smem, st>>>(P);
  } else {
    CK(cudaFuncSetAttribute(inst_rr_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    inst_rr_kernel<2><<<(unsigned)grid, 32 * warps, smem, st>>>(P);
  }
  CK(cudaGetLastError());
  return 0;
}

int b200chem_inst_rr(b200chem_handle h, const double* rhoY_mks, const double* rhoH_mks, double* T,
                     double* rhoYdot_mks, int64_t ncells, void* stream) {
  if (!rhoYdot_mks) return set_err(B200CHEM_EINVAL, "null output");
  return inst_launch(h, rhoY_mks, rhoH_mks, T, rhoYdot_mks, ncells, stream);
}

int b200chem_t_from_hy(b200chem_handle h, const double* rhoY_mks, const double* rhoH_mks, double* T, int64_t ncells,
                       void* stream) {
  return inst_launch(h, rhoY_mks, rhoH_mks, T, nullptr, ncells, stream);
}

}  // extern "C"
