// react_tpc.cu -- thread-per-cell react kernels (one cell per thread, see
// bdf_thread.cuh) for the species counts that have a compiled variant.
#include "bdf_thread.cuh"
#include "common.cuh"

namespace b200 {

// ------------------------------------------------ thread-per-cell kernel
#ifndef B200_TPC_MIN_CTAS
#define B200_TPC_MIN_CTAS 4
#endif


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


bool tpc_supported(int N) { return N == 9 || N == 21; }

template <int NS, typename LUT>
static cudaError_t tpc_occ(int* per_sm, int* smem) {
  *smem = (int)(2 * sizeof(double) * NS * kTpcBlock);
  cudaError_t e = cudaFuncSetAttribute(react_tpc_kernel<NS, LUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, *smem);
  if (e != cudaSuccess) return e;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, react_tpc_kernel<NS, LUT>, kTpcBlock, *smem);
}

cudaError_t tpc_occupancy(int N, int lut_bytes, int* per_sm, int* smem) {
  if (N == 9) return lut_bytes == 4 ? tpc_occ<9, float>(per_sm, smem) : tpc_occ<9, double>(per_sm, smem);
  if (N == 21) return lut_bytes == 4 ? tpc_occ<21, float>(per_sm, smem) : tpc_occ<21, double>(per_sm, smem);
  return cudaErrorInvalidValue;
}

cudaError_t tpc_launch(int N, int lut_bytes, const ReactParams& P, const TpcParams& Q, int grid, int smem,
                       cudaStream_t st) {
  if (N == 9) {
    if (lut_bytes == 4) react_tpc_kernel<9, float><<<grid, kTpcBlock, smem, st>>>(P, Q);
    else react_tpc_kernel<9, double><<<grid, kTpcBlock, smem, st>>>(P, Q);
  } else if (N == 21) {
    if (lut_bytes == 4) react_tpc_kernel<21, float><<<grid, kTpcBlock, smem, st>>>(P, Q);
    else react_tpc_kernel<21, double><<<grid, kTpcBlock, smem, st>>>(P, Q);
  } else {
    return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace b200
