// advance_chem.cu -- the per-box body of PeleLM::advanceChemistry around
// react (Source/PeleLMeX_Reactions.cpp:31-175), for a list of boxes in one
// launch each:
//
//   prologue (:68-79)   rhoY_new = rhoY_old * 1e-3, extF_rhoY *= 1e-3,
//                       T_new = T_old, rhoH_new = rhoH_old * 10,
//                       extF_rhoH *= 10                        (MKS -> CGS)
//   react               (the caller runs b200chem_react between the two)
//   epilogue (:111-120, rhoY_new *= 1e3, extF_rhoY *= 1e3, rhoH_new *= 0.1,
//            :153-160)  extF_rhoH *= 0.1                       (CGS -> MKS)
//                       I_R = -(rhoY_old - rhoY_new) / dt - extF_rhoY
//
// and, before the next react, the forcing of getScalarReactForce
// (:437-475)      extF_rhoY = (rhoY_new - rhoY_old) * (1/dt) - I_R,
//                 extF_rhoH = (rhoH_new - rhoH_old) * (1/dt).
//
// The arithmetic is the reference's, operation for operation, so the MKS
// fields round the same way.  One thread per cell, grid-stride over the
// cells of all boxes; memory-bound elementwise work.
#include "common.cuh"

namespace b200 {

namespace {

template <class Box>
__device__ __forceinline__ void chem_locate(const Box* boxes, int nbox, long long cell, int* b, int* i, int* j,
                                            int* k) {
  int lo = 0, hi = nbox - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (boxes[mid].off <= cell) lo = mid;
    else hi = mid - 1;
  }
  const Box& bx = boxes[lo];
  const long long loc = cell - bx.off;
  *b = lo;
  *i = bx.lo0 + (int)(loc % bx.nx);
  *j = bx.lo1 + (int)((loc / bx.nx) % bx.ny);
  *k = bx.lo2 + (int)(loc / ((long long)bx.nx * bx.ny));
}

__global__ void chem_prologue(const ChemBoxDev* __restrict__ boxes, int nbox, long long total, int N) {
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < total;
       c += (long long)gridDim.x * blockDim.x) {
    int b, i, j, k;
    chem_locate(boxes, nbox, c, &b, &i, &j, &k);
    const ChemBoxDev& bx = boxes[b];
    for (int n = 0; n < N; ++n) {
      elem(bx.rY_n, i, j, k)[n * bx.rY_n.ns] = elem(bx.rY_o, i, j, k)[n * bx.rY_o.ns] * 1.0e-3;
      elem(bx.fY, i, j, k)[n * bx.fY.ns] *= 1.0e-3;
    }
    *elem(bx.T_n, i, j, k) = *elem(bx.T_o, i, j, k);
    *elem(bx.rH_n, i, j, k) = *elem(bx.rH_o, i, j, k) * 10.0;
    *elem(bx.fH, i, j, k) *= 10.0;
  }
}

__global__ void chem_epilogue(const ChemBoxDev* __restrict__ boxes, int nbox, long long total, int N, double dt_inv) {
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < total;
       c += (long long)gridDim.x * blockDim.x) {
    int b, i, j, k;
    chem_locate(boxes, nbox, c, &b, &i, &j, &k);
    const ChemBoxDev& bx = boxes[b];
    for (int n = 0; n < N; ++n) {
      double* yn = elem(bx.rY_n, i, j, k) + n * bx.rY_n.ns;
      double* fy = elem(bx.fY, i, j, k) + n * bx.fY.ns;
      *yn *= 1.0e3;
      *fy *= 1.0e3;
      // separately rounded multiply and subtract (no contraction into an FMA)
      if (bx.IR.p)
        elem(bx.IR, i, j, k)[n * bx.IR.ns] =
            __dsub_rn(__dmul_rn(-(elem(bx.rY_o, i, j, k)[n * bx.rY_o.ns] - *yn), dt_inv), *fy);
    }
    *elem(bx.rH_n, i, j, k) *= 0.1;
    *elem(bx.fH, i, j, k) *= 0.1;
  }
}

__global__ void react_force(const ForceBoxDev* __restrict__ boxes, int nbox, long long total, int N, double dt_inv) {
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < total;
       c += (long long)gridDim.x * blockDim.x) {
    int b, i, j, k;
    chem_locate(boxes, nbox, c, &b, &i, &j, &k);
    const ForceBoxDev& bx = boxes[b];
    const double* yo = elem(bx.rY_o, i, j, k);
    const double* yn = elem(bx.rY_n, i, j, k);
    const double* ir = elem(bx.IR, i, j, k);
    double* fy = elem(bx.fY, i, j, k);
    // separately rounded difference, product and difference (no FMA)
    for (int n = 0; n < N; ++n)
      fy[n * bx.fY.ns] =
          __dsub_rn(__dmul_rn(__dsub_rn(yn[n * bx.rY_n.ns], yo[n * bx.rY_o.ns]), dt_inv), ir[n * bx.IR.ns]);
    *elem(bx.fH, i, j, k) = __dmul_rn(__dsub_rn(*elem(bx.rH_n, i, j, k), *elem(bx.rH_o, i, j, k)), dt_inv);
  }
}

}  // namespace

cudaError_t react_force_launch(const ForceBoxDev* d_boxes, int nbox, long long total, int N, double dt_inv,
                               int sm_count, cudaStream_t st) {
  if (total <= 0) return cudaSuccess;
  const long long need = (total + 255) / 256;
  const int grid = (int)(need < 8LL * sm_count ? need : 8LL * sm_count);
  react_force<<<grid, 256, 0, st>>>(d_boxes, nbox, total, N, dt_inv);
  return cudaGetLastError();
}

cudaError_t advance_chem_launch(int phase, const ChemBoxDev* d_boxes, int nbox, long long total, int N,
                                double dt_inv, int sm_count, cudaStream_t st) {
  if (total <= 0) return cudaSuccess;
  const long long need = (total + 255) / 256;
  const int grid = (int)(need < 8LL * sm_count ? need : 8LL * sm_count);
  if (phase == 0) chem_prologue<<<grid, 256, 0, st>>>(d_boxes, nbox, total, N);
  else chem_epilogue<<<grid, 256, 0, st>>>(d_boxes, nbox, total, N, dt_inv);
  return cudaGetLastError();
}

}  // namespace b200
