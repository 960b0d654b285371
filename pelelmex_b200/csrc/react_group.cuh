// react_group.cuh -- the persistent react kernel of the group integrator and
// its host launch helpers (instantiated per group size in react_g*.cu).
//
// One persistent launch advances every cell of a list of boxes: each group
// of G lanes takes cells from a global atomic queue (work stealing, so cells
// that need thousands of BDF steps do not hold back cells that need a
// handful) and integrates one cell at a time.  The launch is sized to fill
// the GPU once (SM count x resident CTAs per SM).
#pragma once
#include "common.cuh"

// Minimum resident CTAs (of 128 threads) per SM requested from the compiler:
// the register budget of the group integrator (4 -> 128 registers).
#ifndef B200_REACT_MIN_CTAS
#define B200_REACT_MIN_CTAS 4
#endif

namespace b200 {

template <int G, int CPL, typename LUT>
__device__ __forceinline__ void carve_group(GroupBdf<G, CPL, LUT>& B, const GroupLayout& L, unsigned char* sbase,
                                            unsigned char* gbase) {
  double* d = reinterpret_cast<double*>(sbase);
  B.ms.C = d;
  d += L.Npad;
  B.ms.gRT = d;
  d += L.Npad;
  B.ms.hRT = d;
  d += L.Npad;
  B.atolv = d;
  d += L.Npad;
  B.Dsc = d;
  d += L.Npad;
  B.bvec = d;
  d += L.Npad;
  B.ms.q = d;
  d += L.Rpad;
  B.A = reinterpret_cast<LUT*>(d);
  B.fcol = B.A + (size_t)L.n * L.ldl;
  B.ipiv = reinterpret_cast<int*>(B.fcol + L.Npad);
  B.ldl = L.ldl;
  double* gd = reinterpret_cast<double*>(gbase);
  B.J = gd;
  gd += (size_t)L.n * L.ldj;
  B.ms.r1 = gd;
  gd += L.Rpad;
  B.ms.r2 = gd;
  gd += L.Rpad;
  B.ms.r3 = gd;
  gd += L.Rpad;
  B.ms.r4 = gd;
  B.ldj = L.ldj;
}

// Persistent launch: each group of G lanes takes cells from the global queue
// until it is empty and integrates them one after the other.
template <int G, int CPL, typename LUT>
__global__ void __launch_bounds__(128, B200_REACT_MIN_CTAS) react_group_kernel(ReactParams P, GroupParams Q) {
  extern __shared__ __align__(16) unsigned char dsm[];
  __shared__ DevMech s_mech;
  __shared__ long long s_off[65];
  if (threadIdx.x == 0) s_mech = P.mech;
  const int nb_s = P.nbox <= 64 ? P.nbox : 0;
  for (int b = threadIdx.x; b <= nb_s; b += blockDim.x) s_off[b] = (b < nb_s) ? P.boxes[b].off : P.total;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const Grp<G> g(lane);
  const int grp_in_block = threadIdx.x / G;
  const long long grp_global = (long long)blockIdx.x * (blockDim.x / G) + grp_in_block;
  const int N = P.mech.N, n = N + 1;

  GroupBdf<G, CPL, LUT> B;
  B.m = &s_mech;
  B.lane = lane;
  B.n = n;
  B.qmax = P.qmax;
  B.rtol = P.rtol;
  carve_group<G, CPL, LUT>(B, Q.L, dsm + (size_t)grp_in_block * Q.L.smem_bytes, Q.gscratch + grp_global * Q.L.gbytes);
  for (int k = g.gl; k < Q.L.Npad; k += G) B.atolv[k] = (k < n) ? P.atol[k] : 0.0;
  g.sync();
  long long acc[kStCount];
#pragma unroll
  for (int i = 0; i < kStCount; ++i) acc[i] = 0;

  for (;;) {
    unsigned long long cell = 0;
    if (g.gl == 0) cell = atomicAdd(P.queue, 1ull);
    cell = g.bcast(cell, 0);
    if (cell >= (unsigned long long)P.total) break;
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
    if (bx.mask.p)
      masked = bx.mask.p[(long long)(i - bx.mask.lo0) + (long long)(j - bx.mask.lo1) * bx.mask.js +
                         (long long)(k - bx.mask.lo2) * bx.mask.ks] == 0;
    if (masked) {
      code = B200CHEM_CELL_MASKED;
      if (g.gl == 0) {
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
        const int q = g.gl + G * c;
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
      rho = g.sum(rho);
      bad |= !(rho > 0.0);
      if (g.any(bad)) {
        code = B200CHEM_CELL_NONFINITE;
        B.cnt = CellCounters{0, 0, 0, 0, 0, 0, 0};
      } else {
#pragma unroll
        for (int c = 0; c < CPL; ++c) B.F[c] = fv[c];
        code = B.integrate(yv, P.dt, P.max_steps);
      }
      if (code == 0) {
#pragma unroll
        for (int c = 0; c < CPL; ++c) {
          const int q = g.gl + G * c;
          if (q < N) yp[q * bx.rhoY.ns] = yv[c];
          else if (q == N) *tp = yv[c];
        }
        if (g.gl == 0) {
          double* hp = elem(bx.rhoH, i, j, k);
          *hp = *hp + P.dt * (*elem(bx.fH, i, j, k));
        }
      }
      if (g.gl == 0) {
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
    if (g.gl == 0 && P.status) P.status[cell] = code;
  }
  if (g.gl == 0 && P.stats) {
#pragma unroll
    for (int s = 0; s < kStMaxNfe; ++s)
      if (acc[s]) atomicAdd(reinterpret_cast<unsigned long long*>(P.stats + s), (unsigned long long)acc[s]);
    atomicMax(P.stats + kStMaxNfe, acc[kStMaxNfe]);
    atomicMax(P.stats + kStMaxNst, acc[kStMaxNst]);
  }
}

template <int G, int CPL, typename LUT>
int group_occupancy(int smem) {
  if (cudaFuncSetAttribute(react_group_kernel<G, CPL, LUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) !=
      cudaSuccess) {
    cudaGetLastError();
    return -1;
  }
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, react_group_kernel<G, CPL, LUT>, 128, smem) !=
      cudaSuccess) {
    cudaGetLastError();
    return -1;
  }
  return per_sm;
}

template <int G, int CPL, typename LUT>
cudaError_t group_launch(const ReactParams& P, const GroupParams& Q, int grid, int smem, cudaStream_t st) {
  react_group_kernel<G, CPL, LUT><<<grid, 128, smem, st>>>(P, Q);
  return cudaGetLastError();
}

template <int G, int CPL, typename LUT>
constexpr GroupVariant make_variant() {
  return GroupVariant{G, CPL, (int)sizeof(LUT), &group_occupancy<G, CPL, LUT>, &group_launch<G, CPL, LUT>};
}

}  // namespace b200
