// surrogate.cu -- device side of the learned surrogate of the reaction
// advance: network input features and the acceptance gate of a prediction.
//
// Network: N + 2 inputs (T, log10(Y_k + 1e-20) for the N species, log10 dt;
// each standardised by the training-set mean and deviation, padded with
// zeros to a multiple of 16 BF16 columns: 23 -> 32 for 21 species) -> 3 x 256
// GELU -> N + 1 outputs (dT, dY_k, also standardised; 22 -> 32 columns).
// The GEMMs run on the tensor cores (mlp_tc.cu).
//
// Gate, one thread per cell, in this order (any failure rejects the cell,
// which then goes to the BDF integrator):
//   0. (dT_max > 0) the predicted |dT| must not exceed dT_max: the surrogate
//      is trusted where the chemistry over dt_react is mild;
//   1. mass: the predicted partial densities z = rho0 (Y0 + dY) + dt extF_rhoY
//      must sum to the target density within tol_mass (relative);
//   2. element conservation: every element total sum_k a_ek z_k / W_k must
//      match its target within tol_elem times the total atom content; then a
//      weighted minimum-norm correction restores every element total exactly
//      (weights max(|z_k|, 1e-10 rho), so trace species barely move), and
//      partial densities below -tol_mass rho reject (smaller ones are clipped);
//   3. energy consistency: rhoH1 = rhoH0 + dt extF_rhoH; T1 from (h1, Y1) by
//      Newton from T0 + dT must agree with the predicted T0 + dT within tol_T
//      (K); the accepted temperature is T1 (t_source 0: energy conserved
//      exactly) or the predicted T0 + dT (t_source 1);
//   4. one-step implicit residual (when rtol > 0): r = y1 - y0 - dt/2 (f(y0) +
//      f(y1)) (trapezoidal rule, the second-order one-step implicit member),
//      max_i |r_i| / (rtol |y1_i| + atol s_i + rchange |y1_i - y0_i|) <= 1
//      with scales s = rho0 for species and T0 for the temperature, over all
//      components or (residual_t_only) the temperature alone.
// Accepted cells get rhoY1, T1, rhoH1 and fctCount (right-hand sides used:
// 2 with the residual check, else 0) written in place.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "bdf_thread.cuh"
#include "common.cuh"

namespace b200 {
namespace {

// padded network widths for N species: N + 2 inputs, N + 1 outputs, rounded
// up to multiples of 16 (the tensor-core K and N granularity)
constexpr int sg_in(int N) { return (N + 2 + 15) / 16 * 16; }
constexpr int sg_out(int N) { return (N + 1 + 15) / 16 * 16; }
constexpr int kSgBlock = 64;

struct FeatParams {
  const double* rhoY;  // [N][ncells]
  const double* T;
  long long ncells, nrows;  // nrows: padded to a multiple of 128
  double log10dt;
  const float* xmean;  // [N + 2]
  const float* xstd;
  __nv_bfloat16* x;    // [nrows][32]
};

template <int NS>
__global__ void __launch_bounds__(128) sg_features(FeatParams P) {
  constexpr int kSgIn = sg_in(NS);
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < P.nrows;
       c += (long long)gridDim.x * blockDim.x) {
    __align__(16) __nv_bfloat16 row[kSgIn];
#pragma unroll
    for (int j = 0; j < kSgIn; ++j) row[j] = __float2bfloat16_rn(0.0f);
    if (c < P.ncells) {
      double rho = 0.0;
#pragma unroll 4
      for (int k = 0; k < NS; ++k) rho += P.rhoY[(long long)k * P.ncells + c];
      const double rinv = 1.0 / rho;
      row[0] = __float2bfloat16_rn((float)((P.T[c] - P.xmean[0]) / P.xstd[0]));
#pragma unroll
      for (int k = 0; k < NS; ++k) {
        const double Y = P.rhoY[(long long)k * P.ncells + c] * rinv;
        const double f = log10(fmax(Y, 0.0) + 1e-20);
        row[1 + k] = __float2bfloat16_rn((float)((f - P.xmean[1 + k]) / P.xstd[1 + k]));
      }
      row[NS + 1] = __float2bfloat16_rn((float)((P.log10dt - P.xmean[NS + 1]) / P.xstd[NS + 1]));
    }
    uint4* dst = reinterpret_cast<uint4*>(P.x + c * kSgIn);
    const uint4* src = reinterpret_cast<const uint4*>(row);
#pragma unroll
    for (int q = 0; q < kSgIn * 2 / 16; ++q) dst[q] = src[q];
  }
}

struct GateParams {
  DevMech mech;
  double* rhoY;  // [N][ncells] in/out
  const double* fY;
  double* T;
  double* rhoH;
  const double* fH;
  double* fct;   // may be null
  long long ncells;
  double dt;
  const float* pred;  // [nrows][32] standardised network outputs
  const float* ymean;  // [N + 1]
  const float* ystd;
  const double* elem;  // [ne][N] atoms per species
  int ne;
  b200chem_gate_opts o;
  int* accept;   // [ncells] 1 accepted, else -(first failed check): 1 mass, 2 elements, 3 energy,
                 // 4 residual, 5 change cap
};

template <int NS>
__global__ void __launch_bounds__(kSgBlock) sg_gate(GateParams P) {
  constexpr int n = NS + 1;
  extern __shared__ __align__(16) unsigned char dsm[];
  __shared__ DevMech s_mech;
  if (threadIdx.x == 0) s_mech = P.mech;
  __syncthreads();
  const DevMech& m = s_mech;
  double* sC = reinterpret_cast<double*>(dsm) + threadIdx.x;
  double* sW = sC + NS * blockDim.x;
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < P.ncells;
       c += (long long)gridDim.x * blockDim.x) {
    double y0[n], y1[n], F[n], f0[n], f1[n];
    double rho0 = 0.0;
#pragma unroll
    for (int k = 0; k < NS; ++k) {
      y0[k] = P.rhoY[(long long)k * P.ncells + c];
      F[k] = P.fY[(long long)k * P.ncells + c];
      rho0 += y0[k];
    }
    y0[NS] = P.T[c];
    F[NS] = P.fH[c];
    const float* pr = P.pred + c * sg_out(NS);
    const double dT = (double)pr[0] * P.ystd[0] + P.ymean[0];
    bool ok = rho0 > 0.0 && y0[NS] > 0.0 && isfinite(dT);
    int stage = ok ? 0 : 1;  // first failed check (0: none)
    if (ok && P.o.dT_max > 0.0 && fabs(dT) > P.o.dT_max) {
      ok = false;
      stage = 5;
    }
    // predicted partial densities z = rho0 Y1 + dt extF_rhoY and their targets
    double rho1t = 0.0;
#pragma unroll
    for (int k = 0; k < NS; ++k) {
      const double Y = y0[k] / rho0 + ((double)pr[1 + k] * P.ystd[1 + k] + P.ymean[1 + k]);
      y1[k] = rho0 * Y + P.dt * F[k];
      rho1t += y0[k] + P.dt * F[k];
      if (!isfinite(y1[k])) ok = false;
    }
    // 1. mass, before any correction
    if (ok) {
      double zs = 0.0;
#pragma unroll
      for (int k = 0; k < NS; ++k) zs += y1[k];
      ok = fabs(zs - rho1t) <= P.o.tol_mass * rho1t;
      if (!ok) stage = 1;
    }
    // 2. elements, before any correction; then the weighted minimum-norm
    //    correction that restores every element total exactly:
    //    z' = z - D C^T (C D C^T)^-1 (C z - c), C[e][k] = a_ek / W_k,
    //    D = diag(max(|z_k|, 1e-10 rho)) (trace species barely move)
    constexpr int kMaxE = 8;
    if (ok && P.ne > 0) {
      const int ne = P.ne < kMaxE ? P.ne : kMaxE;
      double res[kMaxE], G[kMaxE][kMaxE];
      double tot = 0.0, worst = 0.0;
      for (int e = 0; e < ne; ++e) {
        double ct = 0.0, cz = 0.0;
#pragma unroll
        for (int k = 0; k < NS; ++k) {
          const double a = __ldg(P.elem + e * NS + k) * __ldg(m.inv_mw + k);
          ct += a * (y0[k] + P.dt * F[k]);
          cz += a * y1[k];
        }
        res[e] = cz - ct;
        tot += ct;
        worst = fmax(worst, fabs(res[e]));
        for (int f = 0; f < ne; ++f) {
          double g = 0.0;
#pragma unroll
          for (int k = 0; k < NS; ++k)
            g += __ldg(P.elem + e * NS + k) * __ldg(P.elem + f * NS + k) * __ldg(m.inv_mw + k) *
                 __ldg(m.inv_mw + k) * fmax(fabs(y1[k]), 1e-10 * rho0);
          G[e][f] = g;
        }
      }
      ok = worst <= P.o.tol_elem * tot;
      if (!ok) stage = 2;
      if (ok) {
        // solve G lam = res (Gauss-Jordan with partial pivoting; elements
        // absent from the mechanism give a zero row and are skipped)
        double lam[kMaxE];
        int perm[kMaxE];
        for (int e = 0; e < ne; ++e) perm[e] = e;
        for (int e = 0; e < ne; ++e) lam[e] = res[e];
        for (int col = 0; col < ne; ++col) {
          int piv = col;
          for (int r = col + 1; r < ne; ++r)
            if (fabs(G[r][col]) > fabs(G[piv][col])) piv = r;
          if (!(fabs(G[piv][col]) > 0.0)) continue;
          if (piv != col) {
            for (int q = 0; q < ne; ++q) {
              const double t = G[col][q];
              G[col][q] = G[piv][q];
              G[piv][q] = t;
            }
            const double t = lam[col];
            lam[col] = lam[piv];
            lam[piv] = t;
          }
          const double inv = 1.0 / G[col][col];
          for (int r = 0; r < ne; ++r) {
            if (r == col) continue;
            const double f = G[r][col] * inv;
            if (f == 0.0) continue;
            for (int q = col; q < ne; ++q) G[r][q] -= f * G[col][q];
            lam[r] -= f * lam[col];
          }
        }
        for (int e = 0; e < ne; ++e) lam[e] = (fabs(G[e][e]) > 0.0) ? lam[e] / G[e][e] : 0.0;
        (void)perm;
#pragma unroll
        for (int k = 0; k < NS; ++k) {
          double corr = 0.0;
          for (int e = 0; e < ne; ++e) corr += __ldg(P.elem + e * NS + k) * __ldg(m.inv_mw + k) * lam[e];
          y1[k] -= fmax(fabs(y1[k]), 1e-10 * rho0) * corr;
        }
      }
    }
    // negative partial densities: small ones are clipped, larger ones reject
    if (ok) {
#pragma unroll
      for (int k = 0; k < NS; ++k) {
        if (y1[k] < -P.o.tol_mass * rho1t) ok = false;
        y1[k] = fmax(y1[k], 0.0);
      }
      if (!ok) stage = 1;
    }
    // 3. energy: T1 from (h1, Y1) by Newton from T0 + dT must agree with T0 + dT
    double rho1 = 0.0;
#pragma unroll
    for (int k = 0; k < NS; ++k) rho1 += y1[k];
    const double rhoH1 = P.rhoH[c] + P.dt * F[NS];
    if (ok) {
      const double h1 = rhoH1 / rho1;
      double T = y0[NS] + dT;
      bool conv = false;
      for (int it = 0; it < 50 && T > 0.0; ++it) {
        const double lnT = log(T);
        double hs = 0.0, cs = 0.0;
#pragma unroll
        for (int k = 0; k < NS; ++k) {
          double cpR, hRT, sR, dcpR;
          nasa7(m, k, T, lnT, cpR, hRT, sR, dcpR);
          const double w = y1[k] / rho1 * __ldg(m.inv_mw + k) * kRu;
          hs += w * hRT * T;
          cs += w * cpR;
        }
        const double dTn = (h1 - hs) / cs;
        T += dTn;
        if (fabs(dTn) <= 1e-10 * T) {
          conv = true;
          break;
        }
      }
      ok = conv && fabs(T - (y0[NS] + dT)) <= P.o.tol_T;
      y1[NS] = P.o.t_source ? y0[NS] + dT : T;
      if (!ok) stage = 3;
    }
    // 4. one-step implicit residual (rtol <= 0 switches it off)
    if (ok && P.o.rtol > 0.0) {
      tpc::tpc_rhs<NS>(m, y0, F, f0, sC, sW, blockDim.x);
      tpc::tpc_rhs<NS>(m, y1, F, f1, sC, sW, blockDim.x);
      double worst = 0.0;
#pragma unroll
      for (int i = 0; i < n; ++i) {
        if (P.o.residual_t_only && i < NS) continue;
        const double r = y1[i] - y0[i] - 0.5 * P.dt * (f0[i] + f1[i]);
        const double sc = (i < NS) ? rho0 : y0[NS];
        worst = fmax(worst, fabs(r) / (P.o.rtol * fabs(y1[i]) + P.o.atol * sc + P.o.rchange * fabs(y1[i] - y0[i])));
      }
      ok = worst <= 1.0;
      if (!ok) stage = 4;
    }
    if (ok) {
#pragma unroll
      for (int k = 0; k < NS; ++k) P.rhoY[(long long)k * P.ncells + c] = y1[k];
      P.T[c] = y1[NS];
      P.rhoH[c] = rhoH1;
      if (P.fct) P.fct[c] = (P.o.rtol > 0.0) ? 2.0 : 0.0;
    }
    P.accept[c] = ok ? 1 : -stage;
  }
}

template <int NS>
int launch_features(const FeatParams& P, cudaStream_t st) {
  const long long blocks = (P.nrows + 127) / 128;
  sg_features<NS><<<(unsigned)(blocks < 65535 ? blocks : 65535), 128, 0, st>>>(P);
  return cudaGetLastError() == cudaSuccess ? 0 : B200CHEM_ECUDA;
}

template <int NS>
int launch_gate(const GateParams& P, cudaStream_t st) {
  const int smem = 2 * NS * kSgBlock * (int)sizeof(double);
  if (cudaFuncSetAttribute(sg_gate<NS>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess)
    return B200CHEM_ECUDA;
  const long long blocks = (P.ncells + kSgBlock - 1) / kSgBlock;
  sg_gate<NS><<<(unsigned)(blocks < 65535 ? blocks : 65535), kSgBlock, smem, st>>>(P);
  return cudaGetLastError() == cudaSuccess ? 0 : B200CHEM_ECUDA;
}

}  // namespace
}  // namespace b200

using namespace b200;

extern "C" int b200chem_surrogate_features(b200chem_handle h, const double* rhoY, const double* T, int64_t ncells,
                                           int64_t nrows, double dt, const float* xmean, const float* xstd,
                                           void* x_bf16, void* stream) {
  if (!h || ncells < 0 || nrows < ncells || nrows % 128 || !(dt > 0.0) || !xmean || !xstd || !x_bf16)
    return handle_set_error(B200CHEM_EINVAL, "surrogate_features: bad arguments");
  if (ncells > 0 && (!rhoY || !T)) return handle_set_error(B200CHEM_EINVAL, "surrogate_features: null state");
  FeatParams P{rhoY, T, ncells, nrows, log10(dt), xmean, xstd, static_cast<__nv_bfloat16*>(x_bf16)};
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  int err;
  switch (handle_species(h)) {
    case 9: err = launch_features<9>(P, st); break;
    case 21: err = launch_features<21>(P, st); break;
    case 53: err = launch_features<53>(P, st); break;
    default: return handle_set_error(B200CHEM_EINVAL, "surrogate not compiled for this species count");
  }
  if (err) return handle_set_error(err, "surrogate_features: launch failed");
  handle_count_launch(h);
  return 0;
}

extern "C" int b200chem_surrogate_gate(b200chem_handle h, double* rhoY, const double* extF_rhoY, double* T,
                                       double* rhoH, const double* extF_rhoH, double* fctCount, int64_t ncells,
                                       double dt, const float* pred, const float* ymean, const float* ystd,
                                       const double* elem, int32_t n_elements, const b200chem_gate_opts* opts,
                                       int32_t* accept, void* stream) {
  if (!h || ncells < 0 || !(dt > 0.0) || !opts || n_elements < 0 || n_elements > 16)
    return handle_set_error(B200CHEM_EINVAL, "surrogate_gate: bad arguments");
  if (ncells == 0) return 0;
  if (!rhoY || !extF_rhoY || !T || !rhoH || !extF_rhoH || !pred || !ymean || !ystd || !accept ||
      (n_elements > 0 && !elem))
    return handle_set_error(B200CHEM_EINVAL, "surrogate_gate: null array");
  GateParams P;
  P.mech = *handle_mech(h);
  P.rhoY = rhoY;
  P.fY = extF_rhoY;
  P.T = T;
  P.rhoH = rhoH;
  P.fH = extF_rhoH;
  P.fct = fctCount;
  P.ncells = ncells;
  P.dt = dt;
  P.pred = pred;
  P.ymean = ymean;
  P.ystd = ystd;
  P.elem = elem;
  P.ne = n_elements;
  P.o = *opts;
  P.accept = accept;
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  int err;
  switch (handle_species(h)) {
    case 9: err = launch_gate<9>(P, st); break;
    case 21: err = launch_gate<21>(P, st); break;
    case 53: err = launch_gate<53>(P, st); break;
    default: return handle_set_error(B200CHEM_EINVAL, "surrogate not compiled for this species count");
  }
  if (err) return handle_set_error(err, "surrogate_gate: launch failed");
  handle_count_launch(h);
  return 0;
}
