// surrogate.cu -- device side of the learned surrogate of the reaction
// advance and the hybrid reactor built on it.
//
// Network (one ensemble member): N + 2 inputs (T, log10(Y_k + 1e-20) for the
// N species, log10 dt; standardised by the training-set mean and deviation,
// padded with zeros to a multiple of 16) -> 3 x 256 GELU -> N + 1 outputs
// u_j, decoded as dy_j = s_j sinh(u_j ystd_j + ymean_j) (dT in K, dY_k).
// Inputs and activations travel as two BF16 terms (hi, lo = bf16(v - hi));
// the GEMMs are the tensor-core kernels of mlp_tc.cu.
//
// Hybrid react (b200chem_react_hybrid), per chunk of cells:
//   1. features of every cell (two-term BF16);
//   2. the four GEMMs of every member (FP32 predictions);
//   3. the gate, one thread per cell (hy_gate), in this order:
//        spread   every member's dT within `spread` bars of the ensemble mean
//                 (a bar is t_rel * T1, the error allowed to the cell);
//        cap      |mean dT| within `dT_cap` bars: the members share a bias of
//                 a few percent of the change, which their spread cannot see,
//                 so agreement bounds the error only for moderate changes;
//        mass     the predicted partial densities z = rho0 (Y0 + dY) + dt F
//                 sum to the target density within tol_mass;
//        elements every element total within tol_elem of its target;
//        energy   T from (h1, Y(z)) within `gap` bars of T1 = T0 + dT, with
//                 rhoH1 = rhoH0 + dt F_H;
//        project  weighted minimum-norm correction of z onto the element
//                 totals and the energy rhoH1 = sum_k h_k(T1) z_k (weights
//                 max(|z_k|, 1e-10 rho): trace species barely move), so the
//                 accepted state conserves elements and energy exactly and
//                 its T is the one (h1, Y) gives; partial densities below
//                 -tol_mass rho reject, smaller ones are clipped;
//        residual (resid > 0) |T1 - T0 - dt/2 (f_T(y0) + f_T(y1))| within
//                 `resid` bars (two right-hand sides; the one-step implicit
//                 trapezoidal relation of the temperature);
//      accepted cells are written in place; the others are appended to a
//      list (warp-aggregated);
//   4. the listed cells are gathered into compact arrays, integrated by the
//      BDF (b200chem_react_flat), and scattered back.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "bdf_thread.cuh"
#include "common.cuh"

namespace b200 {
namespace {

// padded network widths for N species: N + 2 inputs, N + 1 outputs, rounded
// up to multiples of 16 (the tensor-core K and N granularity)
constexpr int sg_in(int N) { return (N + 2 + 15) / 16 * 16; }
constexpr int sg_out(int N) { return (N + 1 + 15) / 16 * 16; }
constexpr int kSgBlock = 64;
constexpr int kHidden = 256;
constexpr int kMaxMembers = 16;
constexpr int kMaxElem = 8;

struct FeatParams {
  const double* rhoY;  // [N][ld] (cells c0 .. c0 + ncells - 1 used)
  const double* T;
  long long ld;        // component stride of rhoY
  long long c0;        // first cell
  long long ncells, nrows;  // nrows: padded to a multiple of 128
  double log10dt;
  const float* xmean;  // [N + 2]
  const float* xstd;
  __nv_bfloat16* x;    // [nrows][terms * in]
  int terms;           // 1: bf16(x); 2: [bf16(x) | bf16(x - bf16(x))]
};

template <int NS>
__global__ void __launch_bounds__(128) sg_features(FeatParams P) {
  constexpr int kSgIn = sg_in(NS);
  for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < P.nrows;
       r += (long long)gridDim.x * blockDim.x) {
    float xv[kSgIn];
#pragma unroll
    for (int j = 0; j < kSgIn; ++j) xv[j] = 0.0f;
    if (r < P.ncells) {
      const long long c = P.c0 + r;
      double rho = 0.0;
#pragma unroll 4
      for (int k = 0; k < NS; ++k) rho += P.rhoY[(long long)k * P.ld + c];
      const double rinv = 1.0 / rho;
      xv[0] = (float)((P.T[c] - P.xmean[0]) / P.xstd[0]);
#pragma unroll
      for (int k = 0; k < NS; ++k) {
        const double Y = P.rhoY[(long long)k * P.ld + c] * rinv;
        const double f = log10(fmax(Y, 0.0) + 1e-20);
        xv[1 + k] = (float)((f - P.xmean[1 + k]) / P.xstd[1 + k]);
      }
      xv[NS + 1] = (float)((P.log10dt - P.xmean[NS + 1]) / P.xstd[NS + 1]);
    }
    __align__(16) __nv_bfloat16 row[kSgIn];
    uint4* dst = reinterpret_cast<uint4*>(P.x + r * kSgIn * P.terms);
    for (int t = 0; t < P.terms; ++t) {
#pragma unroll
      for (int j = 0; j < kSgIn; ++j) {
        row[j] = __float2bfloat16_rn(xv[j]);
        xv[j] -= __bfloat162float(row[j]);  // residual for the next term
      }
      const uint4* src = reinterpret_cast<const uint4*>(row);
#pragma unroll
      for (int q = 0; q < kSgIn * 2 / 16; ++q) dst[t * (kSgIn * 2 / 16) + q] = src[q];
    }
  }
}

template <int NS>
int launch_features(const FeatParams& P, cudaStream_t st) {
  const long long blocks = (P.nrows + 127) / 128;
  sg_features<NS><<<(unsigned)(blocks < 65535 ? blocks : 65535), 128, 0, st>>>(P);
  return cudaGetLastError() == cudaSuccess ? 0 : B200CHEM_ECUDA;
}

int features_for(int N, const FeatParams& P, cudaStream_t st) {
  switch (N) {
    case 9: return launch_features<9>(P, st);
    case 21: return launch_features<21>(P, st);
    case 53: return launch_features<53>(P, st);
    default: return B200CHEM_EINVAL;
  }
}

// ------------------------------------------------------------------ gate
enum GateReason : int {
  kAccept = 0,
  kRejSpread = 1,
  kRejCap = 2,
  kRejMass = 3,
  kRejElem = 4,
  kRejEnergy = 5,
  kRejNegative = 6,
  kRejResid = 7,
  kRejNonfinite = 8,
  kReasons = 9
};

// projection passes of the gate, and the relative residual every constraint
// of an accepted cell must meet afterwards (elements: relative to the total
// atom content; energy: relative to sum_k |h_k| z_k)
constexpr int kMinPasses = 3;
constexpr int kMaxPasses = 6;
constexpr double kConsTol = 1e-13;

struct GateParams {
  DevMech mech;
  double* rhoY;  // [N][ld] in/out
  const double* fY;
  double* T;
  double* rhoH;
  const double* fH;
  double* fct;          // may be null
  const int* mask;      // may be null
  int* status;          // may be null
  long long ld;         // component stride of the state arrays (all cells)
  long long c0, nc;     // cells c0 .. c0 + nc - 1 of this chunk
  double dt;
  const float* pred;    // [M][rows][kout] standardised outputs of every member
  long long rows;       // rows of one member's prediction block
  int members;
  const float* ymean;   // [N + 1]
  const float* ystd;
  const double* tscale; // [N + 1] asinh scales
  const double* elem;   // [ne][N] atoms of each element in each species
  int ne;
  b200chem_hybrid_opts o;
  int* rej_list;        // rejected cells (global indices)
  int* rej_count;
  unsigned long long* reasons;  // [kReasons] counts (kAccept: accepted)
};

// T from (h, Y) by Newton on sum_k Y_k h_k(T) = h, from T; false when it
// does not converge to 1e-10 relative in 50 iterations.
template <int NS>
__device__ bool t_from_h(const DevMech& m, double h, const double* z, double rho, double& T) {
  for (int it = 0; it < 50 && T > 0.0; ++it) {
    const double lnT = log(T);
    double hs = 0.0, cs = 0.0;
#pragma unroll 4
    for (int k = 0; k < NS; ++k) {
      double cpR, hRT, sR, dcpR;
      nasa7(m, k, T, lnT, cpR, hRT, sR, dcpR);
      const double w = z[k] / rho * __ldg(m.inv_mw + k) * kRu;
      hs += w * hRT * T;
      cs += w * cpR;
    }
    const double dTn = (h - hs) / cs;
    T += dTn;
    if (fabs(dTn) <= 1e-10 * T) return true;
  }
  return false;
}

template <int NS>
__global__ void __launch_bounds__(kSgBlock) hy_gate(GateParams P) {
  constexpr int n = NS + 1;
  constexpr int kout = sg_out(NS);
  extern __shared__ __align__(16) unsigned char dsm[];
  __shared__ DevMech s_mech;
  if (threadIdx.x == 0) s_mech = P.mech;
  __syncthreads();
  const DevMech& m = s_mech;
  double* sC = reinterpret_cast<double*>(dsm) + threadIdx.x;
  double* sW = sC + NS * blockDim.x;
  const int lane = threadIdx.x & 31;
  // warp-uniform trip count: every lane of a warp runs the same iterations
  for (long long base = (long long)blockIdx.x * blockDim.x; base < P.nc; base += (long long)gridDim.x * blockDim.x) {
    const long long r = base + threadIdx.x;
    const bool in = r < P.nc;
    const long long c = P.c0 + r;
    int reason = kAccept;
    const bool masked = in && P.mask && P.mask[c] == 0;
    if (in && !masked) {
      double y0[n], F[n], d[n], z[NS];
      double rho0 = 0.0;
#pragma unroll
      for (int k = 0; k < NS; ++k) {
        y0[k] = P.rhoY[(long long)k * P.ld + c];
        F[k] = P.fY[(long long)k * P.ld + c];
        rho0 += y0[k];
      }
      y0[NS] = P.T[c];
      F[NS] = P.fH[c];
      // ensemble mean of the decoded changes, and the extremes of dT
#pragma unroll
      for (int j = 0; j < n; ++j) d[j] = 0.0;
      double tmin = 1e300, tmax = -1e300;
      for (int mb = 0; mb < P.members; ++mb) {
        const float* pr = P.pred + ((long long)mb * P.rows + r) * kout;
#pragma unroll
        for (int j = 0; j < n; ++j) {
          const double u = (double)pr[j] * (double)P.ystd[j] + (double)P.ymean[j];
          const double v = P.tscale[j] * sinh(u);
          d[j] += v;
          if (j == 0) {
            tmin = fmin(tmin, v);
            tmax = fmax(tmax, v);
          }
        }
      }
      const double invM = 1.0 / P.members;
#pragma unroll
      for (int j = 0; j < n; ++j) d[j] *= invM;
      const double dT = d[0];
      const double T0 = y0[NS];
      const double T1 = T0 + dT;
      const double bar = P.o.t_rel * T1;  // the error allowed to this cell, K
      const bool fin = rho0 > 0.0 && T0 > 0.0 && isfinite(dT) && T1 > 0.0;
      if (!fin) reason = kRejNonfinite;
      if (!reason && fmax(tmax - dT, dT - tmin) > P.o.spread * bar) reason = kRejSpread;
      if (!reason && fabs(dT) > P.o.dT_cap * bar) reason = kRejCap;
      // predicted partial densities and their targets
      double rho1t = 0.0;
      if (!reason) {
#pragma unroll
        for (int k = 0; k < NS; ++k) {
          z[k] = rho0 * (y0[k] / rho0 + d[1 + k]) + P.dt * F[k];
          rho1t += y0[k] + P.dt * F[k];
          if (!isfinite(z[k])) reason = kRejNonfinite;
        }
      }
      if (!reason) {
        double zs = 0.0;
#pragma unroll
        for (int k = 0; k < NS; ++k) zs += z[k];
        if (!(fabs(zs - rho1t) <= P.o.tol_mass * rho1t)) reason = kRejMass;
      }
      // constraint rows: the elements (mol of element per gram of species),
      // then the energy at T1 (erg per gram), each scaled to unit max-norm
      const int ne = P.ne < kMaxElem ? P.ne : kMaxElem;
      double res[kMaxElem + 1], rsc[kMaxElem + 1], tgt[kMaxElem + 1];
      double hk[NS];
      const double rhoH1 = P.rhoH[c] + P.dt * F[NS];
      if (!reason) {
        double tot = 0.0, worst = 0.0;
        for (int e = 0; e < ne; ++e) {
          double ct = 0.0, cz = 0.0, mx = 0.0;
#pragma unroll
          for (int k = 0; k < NS; ++k) {
            const double a = __ldg(P.elem + e * NS + k) * __ldg(m.inv_mw + k);
            ct += a * (y0[k] + P.dt * F[k]);
            cz += a * z[k];
            mx = fmax(mx, fabs(a));
          }
          res[e] = cz - ct;
          tgt[e] = ct;
          rsc[e] = mx > 0.0 ? 1.0 / mx : 0.0;
          tot += ct;
          worst = fmax(worst, fabs(res[e]));
        }
        if (!(worst <= P.o.tol_elem * tot)) reason = kRejElem;
      }
      if (!reason) {
        // energy consistency of the raw prediction: T(h1, Y(z)) against T1
        double zc[NS];
        double zsum = 0.0;
#pragma unroll
        for (int k = 0; k < NS; ++k) {
          zc[k] = fmax(z[k], 0.0);
          zsum += zc[k];
        }
        double Th = T1;
        const bool conv = t_from_h<NS>(m, rhoH1 / zsum, zc, zsum, Th);
        if (!conv || !(fabs(Th - T1) <= P.o.gap * bar)) reason = kRejEnergy;
      }
      if (!reason) {
        // species enthalpies at T1 and the energy row
        const double lnT1 = log(T1);
        double mx = 0.0;
#pragma unroll
        for (int k = 0; k < NS; ++k) {
          double cpR, hRT, sR, dcpR;
          nasa7(m, k, T1, lnT1, cpR, hRT, sR, dcpR);
          hk[k] = hRT * kRu * T1 * __ldg(m.inv_mw + k);
          mx = fmax(mx, fabs(hk[k]));
        }
        tgt[ne] = rhoH1;
        rsc[ne] = mx > 0.0 ? 1.0 / mx : 0.0;
        // weighted minimum-norm correction z' = z - W A^T (A W A^T)^-1 (A z - b)
        // over the ne + 1 scaled rows A (zero rows are skipped), with
        // W = max(|z_k|, 1e-10 rho).  Partial densities a pass leaves
        // slightly negative are set to zero and frozen (W_k = 0) for the
        // next.  Each pass recomputes the constraint residuals, so the
        // rounding of an ill-conditioned A W A^T and the clipped amounts are
        // corrected again: at least kMinPasses passes, and more while the
        // last one clipped (a cell still clipping after kMaxPasses is
        // rejected).
        const int nr = ne + 1;
        auto row = [&](int e, int k) -> double {
          return (e < ne ? __ldg(P.elem + e * NS + k) * __ldg(m.inv_mw + k) : hk[k]) * rsc[e];
        };
        unsigned long long frozen[(NS + 63) / 64] = {};
        bool clipped = true;
        for (int pass = 0; pass < kMaxPasses && !reason && (pass < kMinPasses || clipped); ++pass) {
          clipped = false;
          double wk[NS];
#pragma unroll
          for (int k = 0; k < NS; ++k)
            wk[k] = ((frozen[k >> 6] >> (k & 63)) & 1ull) ? 0.0 : fmax(fabs(z[k]), 1e-10 * rho0);
          double G[kMaxElem + 1][kMaxElem + 1], lam[kMaxElem + 1];
          for (int e = 0; e < nr; ++e) {
            double az = 0.0;
            for (int k = 0; k < NS; ++k) az += (e < ne ? __ldg(P.elem + e * NS + k) * __ldg(m.inv_mw + k) : hk[k]) * z[k];
            res[e] = az - tgt[e];
            lam[e] = res[e] * rsc[e];
            for (int f = 0; f < nr; ++f) {
              double g = 0.0;
              for (int k = 0; k < NS; ++k) g += row(e, k) * row(f, k) * wk[k];
              G[e][f] = g;
            }
          }
          // Gauss-Jordan with partial pivoting (singular pivots: row skipped)
          for (int col = 0; col < nr; ++col) {
            int piv = col;
            for (int w = col + 1; w < nr; ++w)
              if (fabs(G[w][col]) > fabs(G[piv][col])) piv = w;
            if (!(fabs(G[piv][col]) > 1e-300)) continue;
            if (piv != col) {
              for (int w = 0; w < nr; ++w) {
                const double t = G[col][w];
                G[col][w] = G[piv][w];
                G[piv][w] = t;
              }
              const double t = lam[col];
              lam[col] = lam[piv];
              lam[piv] = t;
            }
            const double inv = 1.0 / G[col][col];
            for (int w = 0; w < nr; ++w) {
              if (w == col) continue;
              const double f = G[w][col] * inv;
              if (f == 0.0) continue;
              for (int v = col; v < nr; ++v) G[w][v] -= f * G[col][v];
              lam[w] -= f * lam[col];
            }
          }
          for (int e = 0; e < nr; ++e) lam[e] = (fabs(G[e][e]) > 1e-300) ? lam[e] / G[e][e] : 0.0;
#pragma unroll
          for (int k = 0; k < NS; ++k) {
            double corr = 0.0;
            for (int e = 0; e < nr; ++e) corr += row(e, k) * lam[e];
            z[k] -= wk[k] * corr;
          }
#pragma unroll
          for (int k = 0; k < NS; ++k) {
            if (z[k] < -P.o.tol_mass * rho1t) reason = kRejNegative;
            if (z[k] < 0.0) {
              z[k] = 0.0;
              frozen[k >> 6] |= 1ull << (k & 63);
              clipped = true;
            }
          }
        }
        if (!reason && clipped) reason = kRejNegative;
        // every constraint met to round-off, or the cell goes to the BDF:
        // the elements relative to the total atom content, the energy
        // relative to sum_k |h_k| z_k
        double tot = 0.0;
        for (int e = 0; e < ne; ++e) tot += tgt[e];
        for (int e = 0; e < nr && !reason; ++e) {
          double az = 0.0, sc = 0.0;
          for (int k = 0; k < NS; ++k) {
            const double a = e < ne ? __ldg(P.elem + e * NS + k) * __ldg(m.inv_mw + k) : hk[k];
            az += a * z[k];
            sc += fabs(a) * z[k];
          }
          if (!(fabs(az - tgt[e]) <= kConsTol * (e < ne ? tot : sc))) reason = kRejElem;
        }
      }
      if (!reason && P.o.resid > 0.0) {
        double y1[n], f0[n], f1[n];
#pragma unroll
        for (int k = 0; k < NS; ++k) y1[k] = z[k];
        y1[NS] = T1;
        tpc::tpc_rhs<NS>(m, y0, F, f0, sC, sW, blockDim.x);
        tpc::tpc_rhs<NS>(m, y1, F, f1, sC, sW, blockDim.x);
        const double rT = T1 - T0 - 0.5 * P.dt * (f0[NS] + f1[NS]);
        if (!(fabs(rT) <= P.o.resid * bar)) reason = kRejResid;
      }
      if (!reason) {
#pragma unroll
        for (int k = 0; k < NS; ++k) P.rhoY[(long long)k * P.ld + c] = z[k];
        P.T[c] = T1;
        P.rhoH[c] = rhoH1;
        if (P.fct) P.fct[c] = (P.o.resid > 0.0) ? 2.0 : 0.0;
        if (P.status) P.status[c] = B200CHEM_CELL_OK;
      }
    } else if (masked) {
      if (P.fct) P.fct[c] = 0.0;
      if (P.status) P.status[c] = B200CHEM_CELL_MASKED;
    }
    // rejected cells: warp-aggregated append to the list
    const bool rej = in && !masked && reason != kAccept;
    const unsigned bal = __ballot_sync(0xffffffffu, rej);
    if (bal) {
      int basei = 0;
      if (lane == 0) basei = atomicAdd(P.rej_count, __popc(bal));
      basei = __shfl_sync(0xffffffffu, basei, 0);
      if (rej) P.rej_list[basei + __popc(bal & ((1u << lane) - 1u))] = (int)c;
    }
    // per-reason counts, one atomic per warp and reason present
#pragma unroll
    for (int q = 0; q < kReasons; ++q) {
      const unsigned b = __ballot_sync(0xffffffffu, in && !masked && reason == q);
      if (b && lane == 0) atomicAdd(P.reasons + q, (unsigned long long)__popc(b));
    }
  }
}

template <int NS>
int launch_gate(const GateParams& P, int sm_count, cudaStream_t st) {
  const int smem = 2 * NS * kSgBlock * (int)sizeof(double);
  if (cudaFuncSetAttribute(hy_gate<NS>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess)
    return B200CHEM_ECUDA;
  const long long need = (P.nc + kSgBlock - 1) / kSgBlock;
  const long long cap = 16LL * sm_count;
  hy_gate<NS><<<(unsigned)(need < cap ? need : cap), kSgBlock, smem, st>>>(P);
  return cudaGetLastError() == cudaSuccess ? 0 : B200CHEM_ECUDA;
}

// Lane-group form of the gate (G lanes per cell, component j of the cell on
// lane j % G), used when the residual check is off: the same checks, in the
// same order and with the same arithmetic per component, with the sums over
// species as butterfly reductions inside the group (bitwise identical on
// every lane, so every decision is uniform in the group) and the small
// constraint system solved redundantly by every lane.  No per-thread arrays
// of the cell's size, so no local memory.
template <int G>
__device__ __forceinline__ double grp_sum(double v, unsigned gm) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(gm, v, o, G);
  return v;
}
template <int G>
__device__ __forceinline__ double grp_max(double v, unsigned gm) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(gm, v, o, G));
  return v;
}

// Solves G x = b in place (b -> x) for a symmetric positive semi-definite G
// given by its lower triangle, by an LDL^T factorisation without pivoting,
// fully unrolled so that G stays in registers (G is overwritten with L).  A
// column whose pivot falls to 1e-13 of its diagonal or below (a constraint
// row that vanishes, or that the others already fix) is dropped: its
// unknown is 0, as the pivoted Gauss-Jordan of hy_gate skips a zero pivot.
template <int NR>
__device__ __forceinline__ void ldl_solve(double (&Gm)[NR][NR], double (&b)[NR]) {
  double D[NR];
#pragma unroll
  for (int j = 0; j < NR; ++j) {
    double dj = Gm[j][j];
#pragma unroll
    for (int k = 0; k < j; ++k) dj -= Gm[j][k] * Gm[j][k] * D[k];
    const bool keep = dj > 1e-13 * Gm[j][j] && dj > 0.0;
    D[j] = keep ? dj : 0.0;
    const double inv = keep ? 1.0 / dj : 0.0;
#pragma unroll
    for (int i = j + 1; i < NR; ++i) {
      double v = Gm[i][j];
#pragma unroll
      for (int k = 0; k < j; ++k) v -= Gm[i][k] * Gm[j][k] * D[k];
      Gm[i][j] = v * inv;
    }
  }
#pragma unroll
  for (int j = 0; j < NR; ++j) {
#pragma unroll
    for (int k = 0; k < j; ++k) b[j] -= Gm[j][k] * b[k];
  }
#pragma unroll
  for (int j = 0; j < NR; ++j) b[j] = D[j] > 0.0 ? b[j] / D[j] : 0.0;
#pragma unroll
  for (int j = NR - 1; j >= 0; --j) {
#pragma unroll
    for (int i = j + 1; i < NR; ++i) b[j] -= Gm[i][j] * b[i];
  }
}

// Minimum resident CTAs per SM requested for the lane-group gate (bounds its
// registers per thread).
#ifndef B200_GATE_MIN_CTAS
#define B200_GATE_MIN_CTAS 3
#endif

template <int NS, int G, int NR>
__global__ void __launch_bounds__(128, B200_GATE_MIN_CTAS) hy_gate_grp(GateParams P) {
  constexpr int n = NS + 1;
  constexpr int NE = NR - 1;  // elements
  constexpr int CPL = (n + G - 1) / G;
  constexpr int kout = sg_out(NS);
  __shared__ DevMech s_mech;
  if (threadIdx.x == 0) s_mech = P.mech;
  __syncthreads();
  const DevMech& m = s_mech;
  const int lane = threadIdx.x & 31;
  const int gl = lane % G;
  const unsigned gm = (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << (lane - gl));
  const int per_block = blockDim.x / G;
  for (long long base = (long long)blockIdx.x * per_block; base < P.nc; base += (long long)gridDim.x * per_block) {
    const long long r = base + threadIdx.x / G;
    const bool in = r < P.nc;
    const long long c = P.c0 + r;
    const bool masked = in && P.mask && P.mask[c] == 0;
    int reason = kAccept;
    if (in && !masked) {
      // this lane's components: j = gl + G cc (0: T, k + 1: species k)
      double y0[CPL], F[CPL], d[CPL], z[CPL];
      double rs = 0.0;
#pragma unroll
      for (int cc = 0; cc < CPL; ++cc) {
        const int j = gl + G * cc;
        y0[cc] = F[cc] = d[cc] = z[cc] = 0.0;
        if (j >= 1 && j < n) {
          y0[cc] = P.rhoY[(long long)(j - 1) * P.ld + c];
          F[cc] = P.fY[(long long)(j - 1) * P.ld + c];
          rs += y0[cc];
        } else if (j == 0) {
          y0[cc] = P.T[c];
          F[cc] = P.fH[c];
        }
      }
      const double rho0 = grp_sum<G>(rs, gm);
      // decoded changes: ensemble mean per component, extremes of dT
      double tmin = 1e300, tmax = -1e300;
      for (int mb = 0; mb < P.members; ++mb) {
        const float* pr = P.pred + ((long long)mb * P.rows + r) * kout;
#pragma unroll
        for (int cc = 0; cc < CPL; ++cc) {
          const int j = gl + G * cc;
          if (j < n) {
            const double u = (double)pr[j] * (double)P.ystd[j] + (double)P.ymean[j];
            const double v = P.tscale[j] * sinh(u);
            d[cc] += v;
            if (j == 0) {
              tmin = fmin(tmin, v);
              tmax = fmax(tmax, v);
            }
          }
        }
      }
      const double invM = 1.0 / P.members;
#pragma unroll
      for (int cc = 0; cc < CPL; ++cc) d[cc] *= invM;
      const int src = lane - gl;  // the group's first lane holds T
      const double dT = __shfl_sync(gm, d[0], src, 32);
      const double T0 = __shfl_sync(gm, y0[0], src, 32);
      const double FH = __shfl_sync(gm, F[0], src, 32);
      tmin = __shfl_sync(gm, tmin, src, 32);
      tmax = __shfl_sync(gm, tmax, src, 32);
      const double T1 = T0 + dT;
      const double bar = P.o.t_rel * T1;
      const bool fin = rho0 > 0.0 && T0 > 0.0 && isfinite(dT) && T1 > 0.0;
      if (!fin) reason = kRejNonfinite;
      if (!reason && fmax(tmax - dT, dT - tmin) > P.o.spread * bar) reason = kRejSpread;
      if (!reason && fabs(dT) > P.o.dT_cap * bar) reason = kRejCap;
      // predicted partial densities and their target sum
      double zs = 0.0, tsum = 0.0;
      bool bad = false;
#pragma unroll
      for (int cc = 0; cc < CPL; ++cc) {
        const int j = gl + G * cc;
        if (j >= 1 && j < n) {
          z[cc] = rho0 * (y0[cc] / rho0 + d[cc]) + P.dt * F[cc];
          zs += z[cc];
          tsum += y0[cc] + P.dt * F[cc];
          bad |= !isfinite(z[cc]);
        }
      }
      const double rho1t = grp_sum<G>(tsum, gm);
      zs = grp_sum<G>(zs, gm);
      bad = grp_max<G>(bad ? 1.0 : 0.0, gm) > 0.0;
      if (!reason && bad) reason = kRejNonfinite;
      if (!reason && !(fabs(zs - rho1t) <= P.o.tol_mass * rho1t)) reason = kRejMass;
      // constraint rows on this lane's components: A[e] the element e
      // content (mol per gram of species), A[NE] the species enthalpy at T1;
      // each row scaled by rsc (unit max-norm) in the projection
      double A[NR][CPL], tgt[NR], rsc[NR];
      const double rhoH1 = P.rhoH[c] + P.dt * FH;
      double tot = 0.0;
      if (!reason) {
        double worst = 0.0;
#pragma unroll
        for (int e = 0; e < NE; ++e) {
          double ct = 0.0, cz = 0.0, mx = 0.0;
#pragma unroll
          for (int cc = 0; cc < CPL; ++cc) {
            const int j = gl + G * cc;
            double a = 0.0;
            if (j >= 1 && j < n) {
              a = __ldg(P.elem + e * NS + (j - 1)) * __ldg(m.inv_mw + (j - 1));
              ct += a * (y0[cc] + P.dt * F[cc]);
              cz += a * z[cc];
              mx = fmax(mx, fabs(a));
            }
            A[e][cc] = a;
          }
          ct = grp_sum<G>(ct, gm);
          cz = grp_sum<G>(cz, gm);
          mx = grp_max<G>(mx, gm);
          tgt[e] = ct;
          rsc[e] = mx > 0.0 ? 1.0 / mx : 0.0;
          tot += ct;
          worst = fmax(worst, fabs(cz - ct));
        }
        if (!(worst <= P.o.tol_elem * tot)) reason = kRejElem;
      }
      if (!reason) {
        // energy consistency of the raw prediction: T(h1, Y(z)) against T1
        double zsum = 0.0;
#pragma unroll
        for (int cc = 0; cc < CPL; ++cc) {
          const int j = gl + G * cc;
          if (j >= 1 && j < n) zsum += fmax(z[cc], 0.0);
        }
        zsum = grp_sum<G>(zsum, gm);
        const double h1 = rhoH1 / zsum;
        double Th = T1;
        bool conv = false;
        for (int it = 0; it < 50 && Th > 0.0 && !conv; ++it) {
          const double lnT = log(Th);
          double hs = 0.0, cs = 0.0;
#pragma unroll
          for (int cc = 0; cc < CPL; ++cc) {
            const int j = gl + G * cc;
            if (j >= 1 && j < n) {
              double cpR, hRT, sR, dcpR;
              nasa7(m, j - 1, Th, lnT, cpR, hRT, sR, dcpR);
              const double w = fmax(z[cc], 0.0) / zsum * __ldg(m.inv_mw + (j - 1)) * kRu;
              hs += w * hRT * Th;
              cs += w * cpR;
            }
          }
          hs = grp_sum<G>(hs, gm);
          cs = grp_sum<G>(cs, gm);
          const double dTn = (h1 - hs) / cs;
          Th += dTn;
          conv = fabs(dTn) <= 1e-10 * Th;
        }
        if (!conv || !(fabs(Th - T1) <= P.o.gap * bar)) reason = kRejEnergy;
      }
      if (!reason) {
        // species enthalpies at T1: the energy row
        const double lnT1 = log(T1);
        double mx = 0.0;
#pragma unroll
        for (int cc = 0; cc < CPL; ++cc) {
          const int j = gl + G * cc;
          double a = 0.0;
          if (j >= 1 && j < n) {
            double cpR, hRT, sR, dcpR;
            nasa7(m, j - 1, T1, lnT1, cpR, hRT, sR, dcpR);
            a = hRT * kRu * T1 * __ldg(m.inv_mw + (j - 1));
            mx = fmax(mx, fabs(a));
          }
          A[NE][cc] = a;
        }
        mx = grp_max<G>(mx, gm);
        tgt[NE] = rhoH1;
        rsc[NE] = mx > 0.0 ? 1.0 / mx : 0.0;
        // weighted minimum-norm correction z' = z - W A^T (A W A^T)^-1 (A z - b)
        // over the NR scaled rows, the passes of hy_gate, with the small
        // symmetric system solved by an LDL^T factorisation in registers
        unsigned frozen = 0;  // bit cc: this lane's component cc is frozen at zero
        bool clipped = true;
        for (int pass = 0; pass < kMaxPasses && !reason && (pass < kMinPasses || clipped); ++pass) {
          double w[CPL];
#pragma unroll
          for (int cc = 0; cc < CPL; ++cc) {
            const int j = gl + G * cc;
            w[cc] = (j >= 1 && j < n && !((frozen >> cc) & 1u)) ? fmax(fabs(z[cc]), 1e-10 * rho0) : 0.0;
          }
          double Gm[NR][NR], lam[NR];
#pragma unroll
          for (int e = 0; e < NR; ++e) {
            double az = 0.0;
#pragma unroll
            for (int cc = 0; cc < CPL; ++cc) az += A[e][cc] * z[cc];
            lam[e] = (grp_sum<G>(az, gm) - tgt[e]) * rsc[e];
#pragma unroll
            for (int f = 0; f <= e; ++f) {
              double g = 0.0;
#pragma unroll
              for (int cc = 0; cc < CPL; ++cc) g += A[e][cc] * A[f][cc] * w[cc];
              Gm[e][f] = grp_sum<G>(g, gm) * rsc[e] * rsc[f];
            }
          }
          ldl_solve<NR>(Gm, lam);
          bool neg = false, clip = false;
#pragma unroll
          for (int cc = 0; cc < CPL; ++cc) {
            const int j = gl + G * cc;
            if (j >= 1 && j < n && !((frozen >> cc) & 1u)) {
              double corr = 0.0;
#pragma unroll
              for (int e = 0; e < NR; ++e) corr += A[e][cc] * rsc[e] * lam[e];
              z[cc] -= w[cc] * corr;
              if (z[cc] < -P.o.tol_mass * rho1t) neg = true;
              if (z[cc] < 0.0) {
                z[cc] = 0.0;
                frozen |= 1u << cc;
                clip = true;
              }
            }
          }
          if (grp_max<G>(neg ? 1.0 : 0.0, gm) > 0.0) reason = kRejNegative;
          clipped = grp_max<G>(clip ? 1.0 : 0.0, gm) > 0.0;
        }
        if (!reason && clipped) reason = kRejNegative;
        // every constraint met to round-off, or the cell goes to the BDF
        // (the scales of hy_gate)
#pragma unroll
        for (int e = 0; e < NR; ++e) {
          double az = 0.0, sc = 0.0;
#pragma unroll
          for (int cc = 0; cc < CPL; ++cc) {
            az += A[e][cc] * z[cc];
            sc += fabs(A[e][cc]) * z[cc];
          }
          az = grp_sum<G>(az, gm);
          sc = grp_sum<G>(sc, gm);
          if (!reason && !(fabs(az - tgt[e]) <= kConsTol * (e < NE ? tot : sc))) reason = kRejElem;
        }
      }
      if (!reason) {
#pragma unroll
        for (int cc = 0; cc < CPL; ++cc) {
          const int j = gl + G * cc;
          if (j >= 1 && j < n) P.rhoY[(long long)(j - 1) * P.ld + c] = z[cc];
        }
        if (gl == 0) {
          P.T[c] = T1;
          P.rhoH[c] = rhoH1;
          if (P.fct) P.fct[c] = 0.0;
          if (P.status) P.status[c] = B200CHEM_CELL_OK;
        }
      }
    } else if (masked && gl == 0) {
      if (P.fct) P.fct[c] = 0.0;
      if (P.status) P.status[c] = B200CHEM_CELL_MASKED;
    }
    // group leaders: warp-aggregated append of the rejected cells and counts
    const bool lead = in && !masked && gl == 0;
    const bool rej = lead && reason != kAccept;
    const unsigned bal = __ballot_sync(0xffffffffu, rej);
    if (bal) {
      int basei = 0;
      if (lane == 0) basei = atomicAdd(P.rej_count, __popc(bal));
      basei = __shfl_sync(0xffffffffu, basei, 0);
      if (rej) P.rej_list[basei + __popc(bal & ((1u << lane) - 1u))] = (int)c;
    }
#pragma unroll
    for (int q = 0; q < kReasons; ++q) {
      const unsigned b = __ballot_sync(0xffffffffu, lead && reason == q);
      if (b && lane == 0) atomicAdd(P.reasons + q, (unsigned long long)__popc(b));
    }
  }
}

template <int NS, int NR>
int launch_gate_grp_nr(const GateParams& P, int sm_count, cudaStream_t st) {
  constexpr int G = NS + 1 <= 32 ? 8 : 16;
  const int per_block = 128 / G;
  const long long need = (P.nc + per_block - 1) / per_block;
  const long long cap = 32LL * sm_count;
  hy_gate_grp<NS, G, NR><<<(unsigned)(need < cap ? need : cap), 128, 0, st>>>(P);
  return cudaGetLastError() == cudaSuccess ? 0 : B200CHEM_ECUDA;
}

// One instantiation per constraint count (elements + the energy).
template <int NS>
int launch_gate_grp(const GateParams& P, int sm_count, cudaStream_t st) {
  switch ((P.ne < kMaxElem ? P.ne : kMaxElem) + 1) {
    case 1: return launch_gate_grp_nr<NS, 1>(P, sm_count, st);
    case 2: return launch_gate_grp_nr<NS, 2>(P, sm_count, st);
    case 3: return launch_gate_grp_nr<NS, 3>(P, sm_count, st);
    case 4: return launch_gate_grp_nr<NS, 4>(P, sm_count, st);
    case 5: return launch_gate_grp_nr<NS, 5>(P, sm_count, st);
    case 6: return launch_gate_grp_nr<NS, 6>(P, sm_count, st);
    case 7: return launch_gate_grp_nr<NS, 7>(P, sm_count, st);
    case 8: return launch_gate_grp_nr<NS, 8>(P, sm_count, st);
    default: return launch_gate_grp_nr<NS, 9>(P, sm_count, st);
  }
}

// The lane-group gate unless the residual check (a per-cell right-hand
// side) is on.
int gate_for(int N, const GateParams& P, int sm_count, cudaStream_t st) {
  const bool grp = !(P.o.resid > 0.0);
  switch (N) {
    case 9: return grp ? launch_gate_grp<9>(P, sm_count, st) : launch_gate<9>(P, sm_count, st);
    case 21: return grp ? launch_gate_grp<21>(P, sm_count, st) : launch_gate<21>(P, sm_count, st);
    case 53: return grp ? launch_gate_grp<53>(P, sm_count, st) : launch_gate<53>(P, sm_count, st);
    default: return B200CHEM_EINVAL;
  }
}

// ----------------------------------------------- gather / scatter / decode
struct MoveParams {
  const int* list;
  const int* count;
  int N;
  long long ld;      // component stride of the full arrays
  long long cap;     // component stride of the compact arrays
  double *rhoY, *T, *rhoH, *fct;
  const double *fY, *fH;
  int* status;
  double *cY, *cT, *cH, *cfY, *cfH, *cfct;
  int* cstatus;
};

__global__ void hy_gather(MoveParams P) {
  const int cnt = *P.count;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += (long long)gridDim.x * blockDim.x) {
    const long long c = P.list[i];
    for (int k = 0; k < P.N; ++k) {
      P.cY[k * P.cap + i] = P.rhoY[k * P.ld + c];
      P.cfY[k * P.cap + i] = P.fY[k * P.ld + c];
    }
    P.cT[i] = P.T[c];
    P.cH[i] = P.rhoH[c];
    P.cfH[i] = P.fH[c];
  }
}

__global__ void hy_scatter(MoveParams P, double fct_extra) {
  const int cnt = *P.count;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += (long long)gridDim.x * blockDim.x) {
    const long long c = P.list[i];
    for (int k = 0; k < P.N; ++k) P.rhoY[k * P.ld + c] = P.cY[k * P.cap + i];
    P.T[c] = P.cT[i];
    P.rhoH[c] = P.cH[i];
    if (P.fct) P.fct[c] = P.cfct[i] + fct_extra;
    if (P.status) P.status[c] = P.cstatus[i];
  }
}

// Ensemble mean of the decoded changes [ncells][N + 1] and the largest
// deviation of a member's dT from it [ncells].
struct DecodeParams {
  const float* pred;
  long long rows, c0, nc;
  int members, nout, kout;
  const float *ymean, *ystd;
  const double* tscale;
  double* mean;    // [ncells_total][nout], rows c0..
  double* spread;  // [ncells_total] (may be null)
};

__global__ void hy_decode(DecodeParams P) {
  for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < P.nc; r += (long long)gridDim.x * blockDim.x) {
    double tmin = 1e300, tmax = -1e300, tmean = 0.0;
    for (int j = 0; j < P.nout; ++j) {
      double s = 0.0;
      for (int mb = 0; mb < P.members; ++mb) {
        const double u = (double)P.pred[((long long)mb * P.rows + r) * P.kout + j] * (double)P.ystd[j] + P.ymean[j];
        const double v = P.tscale[j] * sinh(u);
        s += v;
        if (j == 0) {
          tmin = fmin(tmin, v);
          tmax = fmax(tmax, v);
        }
      }
      s /= P.members;
      if (j == 0) tmean = s;
      P.mean[(P.c0 + r) * P.nout + j] = s;
    }
    if (P.spread) P.spread[P.c0 + r] = fmax(tmax - tmean, tmean - tmin);
  }
}

}  // namespace
}  // namespace b200

using namespace b200;

// ------------------------------------------------------- surrogate object
struct b200chem_surrogate {
  b200chem_handle h = nullptr;
  int device = -1;
  int N = 0, nin = 0, nout = 0, kin = 0, kout = 0, members = 0, terms = 0, ne = 0;
  b200chem_hybrid_opts opts{};
  void* d_params = nullptr;  // normalisation, scales, elements, weights (one allocation)
  const float *xmean = nullptr, *xstd = nullptr, *ymean = nullptr, *ystd = nullptr;
  const double* tscale = nullptr;
  const double* elem = nullptr;
  std::vector<const void*> W;   // [members * 4] BF16 weights
  std::vector<const float*> b;  // [members * 4] FP32 biases
  void* d_scratch = nullptr;    // inference scratch (grown on demand)
  size_t scratch_bytes = 0;
  void* d_hy = nullptr;         // hybrid scratch: reject list, counters, compact state
  size_t hy_bytes = 0;
  int* h_count = nullptr;       // pinned: rejected count, GEMM error flag
  void* d_pack = nullptr;       // packed box-view state of b200chem_react_hybrid_boxes
  size_t pack_bytes = 0;
  cudaStream_t last_stream = nullptr;
};

namespace {

constexpr char kMagic[8] = {'B', '2', 'C', 'H', 'S', 'U', 'R', 'R'};
constexpr uint32_t kFileVersion = 1;
constexpr long long kChunkRows = 1LL << 20;

int sur_err(int code, const char* msg) { return handle_set_error(code, msg); }

#define SCK(x)                                                        \
  do {                                                                \
    cudaError_t e_ = (x);                                             \
    if (e_ != cudaSuccess) {                                          \
      char m_[256];                                                   \
      snprintf(m_, sizeof(m_), "%s: %s", #x, cudaGetErrorString(e_)); \
      return sur_err(B200CHEM_ECUDA, m_);                             \
    }                                                                 \
  } while (0)

size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

// Inference scratch for chunks of `rows` rows: x [rows][terms * kin] BF16,
// two activation buffers [rows][terms * 256] BF16, predictions
// [members][rows][kout] FP32, and the GEMM error flag.
struct InferBufs {
  __nv_bfloat16* x;
  __nv_bfloat16* h0;
  __nv_bfloat16* h1;
  float* pred;
  int* err;
};

size_t infer_bytes(const b200chem_surrogate* s, long long rows) {
  return align256((size_t)rows * s->terms * s->kin * 2) + 2 * align256((size_t)rows * s->terms * kHidden * 2) +
         align256((size_t)s->members * rows * s->kout * 4) + 256;
}

int ensure_infer(b200chem_surrogate* s, long long rows, cudaStream_t st, InferBufs* B) {
  const size_t need = infer_bytes(s, rows);
  if (need > s->scratch_bytes) {
    if (s->d_scratch) {
      SCK(cudaStreamSynchronize(st));
      cudaFree(s->d_scratch);
      s->d_scratch = nullptr;
      s->scratch_bytes = 0;
    }
    if (cudaMalloc(&s->d_scratch, need) != cudaSuccess) {
      cudaGetLastError();
      return sur_err(B200CHEM_ENOMEM, "cannot allocate the surrogate's inference scratch");
    }
    s->scratch_bytes = need;
  }
  unsigned char* p = static_cast<unsigned char*>(s->d_scratch);
  B->x = reinterpret_cast<__nv_bfloat16*>(p);
  p += align256((size_t)rows * s->terms * s->kin * 2);
  B->h0 = reinterpret_cast<__nv_bfloat16*>(p);
  p += align256((size_t)rows * s->terms * kHidden * 2);
  B->h1 = reinterpret_cast<__nv_bfloat16*>(p);
  p += align256((size_t)rows * s->terms * kHidden * 2);
  B->pred = reinterpret_cast<float*>(p);
  p += align256((size_t)s->members * rows * s->kout * 4);
  B->err = reinterpret_cast<int*>(p);
  return 0;
}

// Features and every member's forward pass for cells c0 .. c0 + nc - 1.
int predict_chunk(b200chem_surrogate* s, const double* rhoY, const double* T, long long ld, long long c0, long long nc,
                  double dt, const InferBufs& B, long long rows, cudaStream_t st) {
  FeatParams F{rhoY, T, ld, c0, nc, rows, log10(dt), s->xmean, s->xstd, B.x, s->terms};
  int err = features_for(s->N, F, st);
  if (err) return sur_err(err, "surrogate features: launch failed");
  handle_count_launch(s->h);
  const int split = s->terms == 2 ? (B200CHEM_GEMM_SPLIT_A | B200CHEM_GEMM_SPLIT_OUT) : 0;
  const int split_a = s->terms == 2 ? B200CHEM_GEMM_SPLIT_A : 0;
  const long long hw = (long long)s->terms * kHidden;
  for (int mb = 0; mb < s->members; ++mb) {
    const void* const* Wm = &s->W[mb * 4];
    const float* const* bm = &s->b[mb * 4];
    const __nv_bfloat16* a = B.x;
    long long lda = (long long)s->terms * s->kin;
    int K = s->kin;
    __nv_bfloat16* outs[2] = {B.h0, B.h1};
    for (int li = 0; li < 3; ++li) {
      __nv_bfloat16* o = outs[li & 1];
      if (b200chem_mlp_gemm_bf16(a, lda, Wm[li], K, (int)rows, kHidden, K, o, hw, bm[li], nullptr, 2 | split, 0,
                                 B.err, st) != 0)
        return sur_err(B200CHEM_ECUDA, "surrogate forward: hidden-layer GEMM rejected");
      handle_count_launch(s->h);
      a = o;
      lda = hw;
      K = kHidden;
    }
    float* pm = B.pred + (long long)mb * rows * s->kout;
    if (b200chem_mlp_gemm_bf16(a, lda, Wm[3], kHidden, (int)rows, s->kout, kHidden, pm, s->kout, bm[3], nullptr,
                               0 | split_a, s->nout, B.err, st) != 0)
      return sur_err(B200CHEM_ECUDA, "surrogate forward: output GEMM rejected");
    handle_count_launch(s->h);
  }
  return 0;
}

// Reads a little-endian value from the weights file.
template <class T>
T rd(const unsigned char* p) {
  T v;
  memcpy(&v, p, sizeof(T));
  return v;
}

}  // namespace

extern "C" b200chem_surrogate_handle b200chem_surrogate_load(b200chem_handle h, const void* data, size_t nbytes) {
  if (!h || !data || nbytes < 256) {
    sur_err(B200CHEM_EINVAL, "surrogate_load: bad arguments");
    return nullptr;
  }
  const unsigned char* p = static_cast<const unsigned char*>(data);
  if (memcmp(p, kMagic, 8) != 0) {
    sur_err(B200CHEM_EINVAL, "surrogate_load: not a surrogate weights file (bad magic)");
    return nullptr;
  }
  const uint32_t version = rd<uint32_t>(p + 8), hbytes = rd<uint32_t>(p + 12);
  if (version != kFileVersion || hbytes < 128 || hbytes > nbytes) {
    sur_err(B200CHEM_EINVAL, "surrogate_load: unsupported file version or header size");
    return nullptr;
  }
  if (rd<uint64_t>(p + 16) != handle_digest(h)) {
    sur_err(B200CHEM_EINVAL, "surrogate_load: the weights were trained for another mechanism (digest mismatch)");
    return nullptr;
  }
  int32_t iv[12];
  memcpy(iv, p + 24, sizeof(iv));
  const int N = iv[0], nin = iv[1], nout = iv[2], hidden = iv[3], kin = iv[4], kout = iv[5], members = iv[6],
            terms = iv[7], dtype = iv[8], min_members = iv[9], ne = iv[10];
  if (N != handle_species(h) || nin != N + 2 || nout != N + 1 || hidden != kHidden || kin != sg_in(N) ||
      kout != sg_out(N) || members < 1 || members > kMaxMembers || (terms != 1 && terms != 2) || dtype != 1 ||
      ne < 0 || ne > kMaxElem) {
    sur_err(B200CHEM_EINVAL, "surrogate_load: unsupported dimensions, member count, terms or dtype");
    return nullptr;
  }
  double dv[7];
  memcpy(dv, p + 72, sizeof(dv));
  // body: xmean, xstd [nin] f32; ymean, ystd [nout] f32; tscale [nout] f64;
  // elem [ne][N] f64; per member: W0 [256][kin] bf16, b0 [256] f32, W1, b1,
  // W2, b2 ([256][256] bf16, [256] f32), W3 [kout][256] bf16, b3 [kout] f32
  const size_t tsc_b = 8 * (size_t)nout, elem_b = 8 * (size_t)ne * N;
  const size_t wsz[4] = {(size_t)kHidden * kin * 2, (size_t)kHidden * kHidden * 2, (size_t)kHidden * kHidden * 2,
                         (size_t)kout * kHidden * 2};
  const size_t bsz[4] = {(size_t)kHidden * 4, (size_t)kHidden * 4, (size_t)kHidden * 4, (size_t)kout * 4};
  size_t member_b = 0;
  for (int li = 0; li < 4; ++li) member_b += wsz[li] + bsz[li];
  const size_t body = 4 * (2 * (size_t)nin + 2 * (size_t)nout) + tsc_b + elem_b + members * member_b;
  if (hbytes + body != nbytes) {
    sur_err(B200CHEM_EINVAL, "surrogate_load: file size does not match its header");
    return nullptr;
  }
  // device copy: every array 256-byte aligned
  std::vector<size_t> sizes = {4 * (size_t)nin, 4 * (size_t)nin, 4 * (size_t)nout, 4 * (size_t)nout, tsc_b, elem_b};
  for (int mb = 0; mb < members; ++mb)
    for (int li = 0; li < 4; ++li) {
      sizes.push_back(wsz[li]);
      sizes.push_back(bsz[li]);
    }
  size_t total = 0;
  for (size_t sz : sizes) total += align256(sz > 0 ? sz : 8);
  std::vector<unsigned char> host(total, 0);
  std::vector<size_t> offs;
  size_t src = hbytes, dst = 0;
  for (size_t sz : sizes) {
    memcpy(host.data() + dst, p + src, sz);
    offs.push_back(dst);
    src += sz;
    dst += align256(sz > 0 ? sz : 8);
  }
  auto* s = new b200chem_surrogate;
  s->h = h;
  s->device = handle_device(h);
  s->N = N;
  s->nin = nin;
  s->nout = nout;
  s->kin = kin;
  s->kout = kout;
  s->members = members;
  s->terms = terms;
  s->ne = ne;
  s->opts.t_rel = dv[0];
  s->opts.spread = dv[1];
  s->opts.dT_cap = dv[2];
  s->opts.gap = dv[3];
  s->opts.tol_elem = dv[4];
  s->opts.tol_mass = dv[5];
  s->opts.resid = dv[6];
  s->opts.min_members = min_members;
  int cur = -1;
  cudaGetDevice(&cur);
  if (cur != s->device || cudaMalloc(&s->d_params, total) != cudaSuccess ||
      cudaMemcpy(s->d_params, host.data(), total, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMallocHost(&s->h_count, 2 * sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    sur_err(B200CHEM_ECUDA, "surrogate_load: device upload failed (is the reactor's device current?)");
    if (s->d_params) cudaFree(s->d_params);
    delete s;
    return nullptr;
  }
  unsigned char* base = static_cast<unsigned char*>(s->d_params);
  s->xmean = reinterpret_cast<const float*>(base + offs[0]);
  s->xstd = reinterpret_cast<const float*>(base + offs[1]);
  s->ymean = reinterpret_cast<const float*>(base + offs[2]);
  s->ystd = reinterpret_cast<const float*>(base + offs[3]);
  s->tscale = reinterpret_cast<const double*>(base + offs[4]);
  s->elem = reinterpret_cast<const double*>(base + offs[5]);
  for (int mb = 0; mb < members; ++mb)
    for (int li = 0; li < 4; ++li) {
      s->W.push_back(base + offs[6 + (mb * 4 + li) * 2]);
      s->b.push_back(reinterpret_cast<const float*>(base + offs[6 + (mb * 4 + li) * 2 + 1]));
    }
  return s;
}

extern "C" b200chem_surrogate_handle b200chem_surrogate_load_file(b200chem_handle h, const char* path) {
  if (!h || !path) {
    sur_err(B200CHEM_EINVAL, "surrogate_load_file: bad arguments");
    return nullptr;
  }
  FILE* f = fopen(path, "rb");
  if (!f) {
    sur_err(B200CHEM_EINVAL, "surrogate_load_file: cannot open the weights file");
    return nullptr;
  }
  std::vector<unsigned char> buf;
  unsigned char tmp[1 << 16];
  size_t got;
  while ((got = fread(tmp, 1, sizeof(tmp), f)) > 0) buf.insert(buf.end(), tmp, tmp + got);
  fclose(f);
  return b200chem_surrogate_load(h, buf.data(), buf.size());
}

extern "C" int b200chem_surrogate_get_opts(b200chem_surrogate_handle s, b200chem_hybrid_opts* o) {
  if (!s || !o) return sur_err(B200CHEM_EINVAL, "surrogate_get_opts: bad arguments");
  *o = s->opts;
  return 0;
}

extern "C" int b200chem_surrogate_destroy(b200chem_surrogate_handle s) {
  if (!s) return 0;
  if (s->last_stream) cudaStreamSynchronize(s->last_stream);
  if (s->d_params) cudaFree(s->d_params);
  if (s->d_scratch) cudaFree(s->d_scratch);
  if (s->d_hy) cudaFree(s->d_hy);
  if (s->d_pack) cudaFree(s->d_pack);
  if (s->h_count) cudaFreeHost(s->h_count);
  delete s;
  return 0;
}

extern "C" int b200chem_surrogate_infer(b200chem_surrogate_handle s, const double* rhoY, const double* T,
                                        int64_t ncells, double dt, double* dy_mean, double* dT_spread, void* stream) {
  if (!s || ncells < 0 || !(dt > 0.0)) return sur_err(B200CHEM_EINVAL, "surrogate_infer: bad arguments");
  if (ncells == 0) return 0;
  if (!rhoY || !T || !dy_mean) return sur_err(B200CHEM_EINVAL, "surrogate_infer: null array");
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  s->last_stream = st;
  const long long chunk = ncells < kChunkRows ? ((ncells + 127) / 128 * 128) : kChunkRows;
  InferBufs B;
  int err = ensure_infer(s, chunk, st, &B);
  if (err) return err;
  SCK(cudaMemsetAsync(B.err, 0, sizeof(int), st));
  for (long long c0 = 0; c0 < ncells; c0 += chunk) {
    const long long nc = std::min<long long>(chunk, ncells - c0);
    const long long rows = (nc + 127) / 128 * 128;
    err = predict_chunk(s, rhoY, T, ncells, c0, nc, dt, B, rows, st);
    if (err) return err;
    DecodeParams D{B.pred, rows, c0, nc, s->members, s->nout, s->kout, s->ymean, s->ystd, s->tscale, dy_mean,
                   dT_spread};
    const long long blocks = (nc + 127) / 128;
    hy_decode<<<(unsigned)(blocks < 65535 ? blocks : 65535), 128, 0, st>>>(D);
    SCK(cudaGetLastError());
    handle_count_launch(s->h);
  }
  SCK(cudaMemcpyAsync(s->h_count + 1, B.err, sizeof(int), cudaMemcpyDeviceToHost, st));
  SCK(cudaStreamSynchronize(st));
  if (s->h_count[1]) return sur_err(B200CHEM_ECUDA, "surrogate_infer: a tensor-core completion wait timed out");
  return 0;
}

extern "C" int b200chem_react_hybrid(b200chem_handle h, b200chem_surrogate_handle s, const b200chem_hybrid_opts* opts,
                                     double* rhoY, const double* extF_rhoY, double* T, double* rhoH,
                                     const double* extF_rhoH, double* fctCount, const int32_t* mask, int64_t ncells,
                                     double* dt_react, double* time, void* stream, int32_t* cell_status,
                                     b200chem_stats* stats, b200chem_hybrid_stats* hstats) {
  if (!h || !s || s->h != h || ncells < 0 || !dt_react || !(*dt_react > 0.0))
    return sur_err(B200CHEM_EINVAL, "react_hybrid: bad arguments (the surrogate must be loaded for this reactor)");
  if (ncells > 0 && (!rhoY || !extF_rhoY || !T || !rhoH || !extF_rhoH))
    return sur_err(B200CHEM_EINVAL, "react_hybrid: null state array");
  if (ncells > 0x7fffffffLL) return sur_err(B200CHEM_ETOOBIG, "react_hybrid: ncells above 2^31-1");
  const b200chem_hybrid_opts o = opts ? *opts : s->opts;
  if (!(o.t_rel > 0.0) || o.spread < 0.0 || o.dT_cap < 0.0 || o.gap < 0.0 || o.tol_elem < 0.0 || o.tol_mass < 0.0 ||
      o.resid < 0.0)
    return sur_err(B200CHEM_EINVAL, "react_hybrid: bad acceptance options");
  if (s->members < std::max(1, (int)o.min_members))
    return sur_err(B200CHEM_EINVAL, "react_hybrid: fewer ensemble members than the options require");
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  s->last_stream = st;
  const double dt = *dt_react;
  if (stats) memset(stats, 0, sizeof(*stats));
  if (hstats) memset(hstats, 0, sizeof(*hstats));
  if (ncells == 0) {
    if (time) *time += dt;
    return 0;
  }
  const long long chunk = ncells < kChunkRows ? ((ncells + 127) / 128 * 128) : kChunkRows;
  InferBufs B;
  int err = ensure_infer(s, chunk, st, &B);
  if (err) return err;
  // hybrid scratch: reason counters and the reject count (256 B), the reject
  // list, the compact state of the rejected cells, their status
  const int N = s->N;
  const long long cap = ncells;
  const size_t list_b = align256(4 * (size_t)cap), state_b = align256(8 * (size_t)cap * (2 * N + 4));
  const size_t need = 256 + list_b + state_b + align256(4 * (size_t)cap);
  if (need > s->hy_bytes) {
    if (s->d_hy) {
      SCK(cudaStreamSynchronize(st));
      cudaFree(s->d_hy);
      s->d_hy = nullptr;
      s->hy_bytes = 0;
    }
    if (cudaMalloc(&s->d_hy, need) != cudaSuccess) {
      cudaGetLastError();
      return sur_err(B200CHEM_ENOMEM, "react_hybrid: cannot allocate the fallback scratch");
    }
    s->hy_bytes = need;
  }
  unsigned char* q = static_cast<unsigned char*>(s->d_hy);
  unsigned long long* reasons = reinterpret_cast<unsigned long long*>(q);
  int* rej_count = reinterpret_cast<int*>(q + 8 * kReasons);
  int* rej_list = reinterpret_cast<int*>(q + 256);
  double* cY = reinterpret_cast<double*>(q + 256 + list_b);
  double* cfY = cY + (size_t)N * cap;
  double* cT = cfY + (size_t)N * cap;
  double* cH = cT + cap;
  double* cfH = cH + cap;
  double* cfct = cfH + cap;
  int* cstatus = reinterpret_cast<int*>(q + 256 + list_b + state_b);
  SCK(cudaMemsetAsync(q, 0, 256, st));
  SCK(cudaMemsetAsync(B.err, 0, sizeof(int), st));
  GateParams G;
  G.mech = *handle_mech(h);
  G.rhoY = rhoY;
  G.fY = extF_rhoY;
  G.T = T;
  G.rhoH = rhoH;
  G.fH = extF_rhoH;
  G.fct = fctCount;
  G.mask = mask;
  G.status = cell_status;
  G.ld = ncells;
  G.dt = dt;
  G.pred = B.pred;
  G.members = s->members;
  G.ymean = s->ymean;
  G.ystd = s->ystd;
  G.tscale = s->tscale;
  G.elem = s->elem;
  G.ne = s->ne;
  G.o = o;
  G.rej_list = rej_list;
  G.rej_count = rej_count;
  G.reasons = reasons;
  for (long long c0 = 0; c0 < ncells; c0 += chunk) {
    const long long nc = std::min<long long>(chunk, ncells - c0);
    const long long rows = (nc + 127) / 128 * 128;
    err = predict_chunk(s, rhoY, T, ncells, c0, nc, dt, B, rows, st);
    if (err) return err;
    G.c0 = c0;
    G.nc = nc;
    G.rows = rows;
    err = gate_for(N, G, handle_sm_count(h), st);
    if (err) return sur_err(err, "react_hybrid: gate launch failed");
    handle_count_launch(h);
  }
  // the rejected count sizes the fallback call
  unsigned long long rs[kReasons];
  SCK(cudaMemcpyAsync(s->h_count, rej_count, sizeof(int), cudaMemcpyDeviceToHost, st));
  SCK(cudaMemcpyAsync(s->h_count + 1, B.err, sizeof(int), cudaMemcpyDeviceToHost, st));
  SCK(cudaMemcpyAsync(rs, reasons, sizeof(rs), cudaMemcpyDeviceToHost, st));
  SCK(cudaStreamSynchronize(st));
  if (s->h_count[1]) return sur_err(B200CHEM_ECUDA, "react_hybrid: a tensor-core completion wait timed out");
  const long long nrej = s->h_count[0];
  int rc = 0;
  if (nrej > 0) {
    MoveParams M{rej_list, rej_count, N, ncells, nrej, rhoY, T, rhoH, fctCount, extF_rhoY, extF_rhoH,
                 cell_status, cY, cT, cH, cfY, cfH, cfct, cstatus};
    const long long blocks = std::min<long long>((nrej + 255) / 256, 8LL * handle_sm_count(h));
    hy_gather<<<(unsigned)blocks, 256, 0, st>>>(M);
    SCK(cudaGetLastError());
    handle_count_launch(h);
    double dtr = dt;
    rc = b200chem_react_flat(h, cY, cfY, cT, cH, cfH, cfct, nullptr, nrej, &dtr, nullptr, stream,
                             cell_status ? cstatus : nullptr, stats);
    if (rc != 0 && rc != B200CHEM_EINTEGRATE) return rc;
    hy_scatter<<<(unsigned)blocks, 256, 0, st>>>(M, o.resid > 0.0 ? 2.0 : 0.0);
    SCK(cudaGetLastError());
    handle_count_launch(h);
  }
  long long predicted = 0;
  for (int r = 0; r < kReasons; ++r) predicted += (long long)rs[r];
  if (stats) {
    stats->n_cells += (long long)rs[kAccept];
    stats->n_masked += ncells - predicted;
    SCK(cudaStreamSynchronize(st));  // synchronous, like react_flat with stats
  }
  if (hstats) {
    hstats->predicted = predicted;
    hstats->accepted = (long long)rs[kAccept];
    hstats->rejected_spread = (long long)rs[kRejSpread];
    hstats->rejected_cap = (long long)rs[kRejCap];
    hstats->rejected_mass = (long long)rs[kRejMass];
    hstats->rejected_elements = (long long)rs[kRejElem];
    hstats->rejected_energy = (long long)rs[kRejEnergy];
    hstats->rejected_negative = (long long)rs[kRejNegative];
    hstats->rejected_residual = (long long)rs[kRejResid];
    hstats->rejected_nonfinite = (long long)rs[kRejNonfinite];
  }
  if (time) *time += dt;
  return rc;
}

extern "C" int b200chem_surrogate_features(b200chem_handle h, const double* rhoY, const double* T, int64_t ncells,
                                           int64_t nrows, double dt, const float* xmean, const float* xstd,
                                           int32_t terms, void* x_bf16, void* stream) {
  if (!h || ncells < 0 || nrows < ncells || nrows % 128 || !(dt > 0.0) || !xmean || !xstd || !x_bf16 ||
      (terms != 1 && terms != 2))
    return handle_set_error(B200CHEM_EINVAL, "surrogate_features: bad arguments");
  if (ncells > 0 && (!rhoY || !T)) return handle_set_error(B200CHEM_EINVAL, "surrogate_features: null state");
  FeatParams P{rhoY, T, ncells, 0, ncells, nrows, log10(dt), xmean, xstd, static_cast<__nv_bfloat16*>(x_bf16),
               terms};
  const int err = features_for(handle_species(h), P, static_cast<cudaStream_t>(stream));
  if (err == B200CHEM_EINVAL) return handle_set_error(err, "surrogate not compiled for this species count");
  if (err) return handle_set_error(err, "surrogate_features: launch failed");
  handle_count_launch(h);
  return 0;
}

// ------------------------------------------------ hybrid react on box views
namespace b200 {
namespace {

// One box of b200chem_react_hybrid_boxes: its Array4 views and its first
// cell in the packed (flat, component-major) order.
struct HyBox {
  int lo0, lo1, lo2, nx, ny, nz;
  long long off;
  DevArr rY, fY, T, rH, fH, fc;
  DevIArr mask;
};

__device__ __forceinline__ int hy_locate(const HyBox* boxes, int nbox, long long cell, int* i, int* j, int* k) {
  int lo = 0, hi = nbox - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (boxes[mid].off <= cell) lo = mid;
    else hi = mid - 1;
  }
  const HyBox& b = boxes[lo];
  const long long loc = cell - b.off;
  *i = b.lo0 + (int)(loc % b.nx);
  *j = b.lo1 + (int)((loc / b.nx) % b.ny);
  *k = b.lo2 + (int)(loc / ((long long)b.nx * b.ny));
  return lo;
}

// phase 0: Array4 views -> packed arrays (state, forcing, mask); phase 1:
// packed results -> Array4 views (rhoY, T, rhoH, fctCount)
__global__ void hy_pack(const HyBox* __restrict__ boxes, int nbox, long long total, int N, int phase, double* pY,
                        double* pfY, double* pT, double* pH, double* pfH, double* pfc, int* pm) {
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < total;
       c += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    const HyBox& b = boxes[hy_locate(boxes, nbox, c, &i, &j, &k)];
    if (phase == 0) {
      for (int n = 0; n < N; ++n) {
        pY[n * total + c] = elem(b.rY, i, j, k)[n * b.rY.ns];
        pfY[n * total + c] = elem(b.fY, i, j, k)[n * b.fY.ns];
      }
      pT[c] = *elem(b.T, i, j, k);
      pH[c] = *elem(b.rH, i, j, k);
      pfH[c] = *elem(b.fH, i, j, k);
      pm[c] = b.mask.p ? b.mask.p[(long long)(i - b.mask.lo0) + (long long)(j - b.mask.lo1) * b.mask.js +
                                  (long long)(k - b.mask.lo2) * b.mask.ks]
                       : 1;
    } else {
      for (int n = 0; n < N; ++n) elem(b.rY, i, j, k)[n * b.rY.ns] = pY[n * total + c];
      *elem(b.T, i, j, k) = pT[c];
      *elem(b.rH, i, j, k) = pH[c];
      if (b.fc.p) *elem(b.fc, i, j, k) = pfc[c];
    }
  }
}

DevArr view_dev(const b200chem_array4& a) {
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
}  // namespace b200

extern "C" int b200chem_react_hybrid_boxes(b200chem_handle h, b200chem_surrogate_handle s,
                                           const b200chem_hybrid_opts* opts, const b200chem_box_view* views,
                                           int32_t nbox, double* dt_react, double* time, void* stream,
                                           int32_t* cell_status, b200chem_stats* stats,
                                           b200chem_hybrid_stats* hstats) {
  if (!h || !s || (!views && nbox > 0) || nbox < 0 || !dt_react)
    return sur_err(B200CHEM_EINVAL, "react_hybrid_boxes: bad arguments");
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  std::vector<HyBox> hb(nbox);
  long long total = 0;
  for (int b = 0; b < nbox; ++b) {
    const b200chem_box_view& v = views[b];
    if (!v.rhoY.p || !v.extF_rhoY.p || !v.T.p || !v.rhoH.p || !v.extF_rhoH.p)
      return sur_err(B200CHEM_EINVAL, "react_hybrid_boxes: null state array");
    HyBox& d = hb[b];
    d.lo0 = v.lo[0];
    d.lo1 = v.lo[1];
    d.lo2 = v.lo[2];
    d.nx = v.hi[0] - v.lo[0] + 1;
    d.ny = v.hi[1] - v.lo[1] + 1;
    d.nz = v.hi[2] - v.lo[2] + 1;
    if (d.nx < 1 || d.ny < 1 || d.nz < 1) return sur_err(B200CHEM_EINVAL, "react_hybrid_boxes: empty box");
    d.off = total;
    total += (long long)d.nx * d.ny * d.nz;
    d.rY = view_dev(v.rhoY);
    d.fY = view_dev(v.extF_rhoY);
    d.T = view_dev(v.T);
    d.rH = view_dev(v.rhoH);
    d.fH = view_dev(v.extF_rhoH);
    d.fc = view_dev(v.fctCount);
    d.mask.p = v.mask.p;
    d.mask.js = v.mask.jstride;
    d.mask.ks = v.mask.kstride;
    d.mask.lo0 = v.mask.lo[0];
    d.mask.lo1 = v.mask.lo[1];
    d.mask.lo2 = v.mask.lo[2];
    d.mask.pad = 0;
  }
  if (total == 0) {
    if (stats) memset(stats, 0, sizeof(*stats));
    if (hstats) memset(hstats, 0, sizeof(*hstats));
    if (time) *time += *dt_react;
    return 0;
  }
  if (total > 0x7fffffffLL) return sur_err(B200CHEM_ETOOBIG, "react_hybrid_boxes: more than 2^31-1 cells");
  // packed arrays and the box descriptors in one allocation, owned by the
  // surrogate and reused across calls
  const int N = s->N;
  const size_t desc_b = align256(sizeof(HyBox) * (size_t)nbox);
  const size_t need = desc_b + align256(8 * (size_t)total * (2 * N + 4)) + align256(4 * (size_t)total);
  if (need > s->pack_bytes) {
    if (s->d_pack) {
      SCK(cudaStreamSynchronize(st));
      cudaFree(s->d_pack);
      s->d_pack = nullptr;
      s->pack_bytes = 0;
    }
    if (cudaMalloc(&s->d_pack, need) != cudaSuccess) {
      cudaGetLastError();
      return sur_err(B200CHEM_ENOMEM, "react_hybrid_boxes: cannot allocate the packed arrays");
    }
    s->pack_bytes = need;
  }
  unsigned char* q = static_cast<unsigned char*>(s->d_pack);
  HyBox* d_boxes = reinterpret_cast<HyBox*>(q);
  double* pY = reinterpret_cast<double*>(q + desc_b);
  double* pfY = pY + (size_t)N * total;
  double* pT = pfY + (size_t)N * total;
  double* pH = pT + total;
  double* pfH = pH + total;
  double* pfc = pfH + total;
  int* pm = reinterpret_cast<int*>(q + desc_b + align256(8 * (size_t)total * (2 * N + 4)));
  // the descriptors are copied synchronously from host memory (small)
  SCK(cudaMemcpyAsync(d_boxes, hb.data(), sizeof(HyBox) * (size_t)nbox, cudaMemcpyHostToDevice, st));
  SCK(cudaStreamSynchronize(st));
  const long long blocks = std::min<long long>((total + 255) / 256, 8LL * handle_sm_count(h));
  hy_pack<<<(unsigned)blocks, 256, 0, st>>>(d_boxes, nbox, total, N, 0, pY, pfY, pT, pH, pfH, pfc, pm);
  SCK(cudaGetLastError());
  handle_count_launch(h);
  int rc = b200chem_react_hybrid(h, s, opts, pY, pfY, pT, pH, pfH, pfc, pm, total, dt_react, time, stream,
                                 cell_status, stats, hstats);
  if (rc != 0 && rc != B200CHEM_EINTEGRATE) return rc;
  hy_pack<<<(unsigned)blocks, 256, 0, st>>>(d_boxes, nbox, total, N, 1, pY, pfY, pT, pH, pfH, pfc, pm);
  SCK(cudaGetLastError());
  handle_count_launch(h);
  return rc;
}
