// react_rounds.cu -- round-based react path: rhs / ctrl / setup kernels over
// compacted cell lists, and their host-side launch sequence.
//
// A react call is processed in chunks of cells (as many as the state buffer
// holds).  For one chunk:
//   start                     load every cell, mask / validity checks, list A
//   repeat until A is empty:
//     rhs   (A)               f(y) for every cell of A (thread per cell)
//     ctrl  (A -> B, S)       resume each cell with its f: next f -> B,
//                             Newton-matrix setup -> S, finished -> outputs
//     setup (S)               Jacobian + inverse (warp per cell)
//     ctrl  (S -> B)          resume the set-up cells
//     swap A, B
// Lists are appended with warp-aggregated atomics, so a warp's slots stay in
// order and the interleaved state accesses stay coalesced as cells drop out.
#include <algorithm>

#include "bdf_rounds.cuh"
#include "common.cuh"
#include "gen_mechs.cuh"  // mechanism-specific right-hand sides (written by the build)

namespace b200 {
using namespace rounds;

namespace {

// (box, i, j, k) of a global cell index of the react call.
struct CellLoc {
  const DevBox* bx;
  int i, j, k;
};

__device__ __forceinline__ CellLoc locate(const ReactParams& P, long long cell) {
  int lo = 0, hi = P.nbox - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (P.boxes[mid].off <= cell) lo = mid;
    else hi = mid - 1;
  }
  CellLoc L;
  L.bx = P.boxes + lo;
  const long long loc = cell - L.bx->off;
  L.i = L.bx->lo0 + (int)(loc % L.bx->nx);
  L.j = L.bx->lo1 + (int)((loc / L.bx->nx) % L.bx->ny);
  L.k = L.bx->lo2 + (int)(loc / ((long long)L.bx->nx * L.bx->ny));
  return L;
}

// Append `val` to list/cnt for the lanes with pred (all 32 lanes call it).
__device__ __forceinline__ void warp_append(bool pred, int val, int* list, int* cnt) {
  const unsigned m = __ballot_sync(kFull, pred);
  if (m == 0) return;
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(m) - 1;
  int base = 0;
  if (lane == leader) base = atomicAdd(cnt, __popc(m));
  base = __shfl_sync(kFull, base, leader);
  if (pred) list[base + __popc(m & ((1u << lane) - 1u))] = val;
}

// Warp-aggregated statistics of the lanes with `done` (all 32 lanes call it).
__device__ __forceinline__ void warp_stats(long long* stats, bool done, bool failed, bool masked,
                                           const CellCounters& cnt) {
  if (!stats || __ballot_sync(kFull, done || masked) == 0) return;
  long long v[kStMaxNfe];
  v[kStCells] = done;
  v[kStMasked] = masked;
  v[kStFailed] = done && failed;
  v[kStNst] = done ? cnt.nst : 0;
  v[kStNfe] = done ? cnt.nfe : 0;
  v[kStNje] = done ? cnt.nje : 0;
  v[kStNlu] = done ? cnt.nlu : 0;
  v[kStNetf] = done ? cnt.netf : 0;
  v[kStNcfn] = done ? cnt.ncfn : 0;
  long long mx = done ? cnt.nfe : 0, ms = done ? cnt.nst : 0;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
    for (int s = 0; s < kStMaxNfe; ++s) v[s] += __shfl_xor_sync(kFull, v[s], o);
    mx = max(mx, __shfl_xor_sync(kFull, mx, o));
    ms = max(ms, __shfl_xor_sync(kFull, ms, o));
  }
  if ((threadIdx.x & 31) == 0) {
#pragma unroll
    for (int s = 0; s < kStMaxNfe; ++s)
      if (v[s]) atomicAdd(reinterpret_cast<unsigned long long*>(stats + s), (unsigned long long)v[s]);
    if (mx) atomicMax(stats + kStMaxNfe, mx);
    if (ms) atomicMax(stats + kStMaxNst, ms);
  }
}

// ------------------------------------------------------------ mechanism
// One reaction's rate of progress for the thread's cell; C, g/RT per thread
// in shared memory at [k * ss].  Every thread of the warp evaluates the SAME
// reaction j, so the table reads are broadcasts and the branches uniform.
__device__ __forceinline__ double r_progress(const DevMech& m, int j, double T, double lnT, double invT,
                                             double Ctot, double lnPRT, const double* sC, const double* sG,
                                             int ss) {
  const int R = m.R;
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
  double kf = kinf;
  if (type >= 2) {
    const double lnA0 = __ldg(m.arr_lo + j), b0 = __ldg(m.arr_lo + R + j), ea0 = __ldg(m.arr_lo + 2 * R + j);
    const double k0 = exp(lnA0 + b0 * lnT - ea0 * invT);
    const double Pr = k0 * M / kinf;
    double F = 1.0;
    if (type == 3) {
      const double a = __ldg(m.troe + j), i3 = __ldg(m.troe + R + j), i1 = __ldg(m.troe + 2 * R + j);
      const double t2 = __ldg(m.troe + 3 * R + j);
      double Fc = (1.0 - a) * exp(-T * i3) + a * exp(-T * i1);
      if (flags & 4) Fc += exp(-t2 * invT);
      const double logFc = log10(fmax(Fc, 1e-300));
      const double c = -0.4 - 0.67 * logFc, nn = 0.75 - 1.27 * logFc;
      const double u = log10(fmax(Pr, 1e-300)) + c;
      const double f1 = u / (nn - 0.14 * u);
      F = exp(kLn10 * (logFc / (1.0 + f1 * f1)));
    }
    kf = kinf * Pr / (1.0 + Pr) * F;
  }
  // slots 0..3 reactants (nu < 0), 4..7 products (nu > 0)
  double pf = 1.0, pr = 1.0, sg = 0.0;
#pragma unroll
  for (int sl = 0; sl < 8; ++sl) {
    const int k = __ldg(m.sp + sl * R + j);
    if (k >= 0) {
      const int nu = __ldg(m.nu + sl * R + j);
      const int na = nu < 0 ? -nu : nu;
      const double ck = sC[k * ss];
      double p = ck;
      for (int e = 1; e < na; ++e) p *= ck;
      if (sl < 4) pf *= p;
      else pr *= p;
      sg += nu * sG[k * ss];
    }
  }
  double kr = 0.0;
  if (flags & 2) {
    const double lr = __ldg(m.arr_rev + j), br = __ldg(m.arr_rev + R + j), er = __ldg(m.arr_rev + 2 * R + j);
    kr = exp(lr + br * lnT - er * invT);
  } else if (flags & 1) {
    kr = kf * exp(sg - __ldg(m.sdnu + j) * lnPRT);
  }
  double q = kf * pf - kr * pr;
  if (type == 1) q *= M;
  return q;
}

// HP right-hand side at v.yev (forcing v.F) into v.fv, thread per cell.
template <int NS>
__device__ __forceinline__ void r_rhs(const DevMech& m, const RVec<NS + 1>& v, double* sC, double* sG, double* sW,
                                      int ss) {
  const double T = v.yev(NS);
  const double lnT = log(T), invT = 1.0 / T;
  double Ctot = 0.0, rcp = 0.0;
#pragma unroll 1
  for (int k = 0; k < NS; ++k) {
    double cpR, hRT, sR, dcpR;
    nasa7(m, k, T, lnT, cpR, hRT, sR, dcpR);
    const double iw = __ldg(m.inv_mw + k);
    const double yk = v.yev(k);
    const double Ck = yk * iw;
    sC[k * ss] = Ck;
    sG[k * ss] = hRT - sR;
    sW[k * ss] = 0.0;
    Ctot += Ck;
    rcp += yk * cpR * kRu * iw;
  }
  const double lnPRT = log(kPatm / (kRu * T));
  const int R = m.R;
#pragma unroll 1
  for (int j = 0; j < R; ++j) {
    const double q = r_progress(m, j, T, lnT, invT, Ctot, lnPRT, sC, sG, ss);
#pragma unroll
    for (int sl = 0; sl < 8; ++sl) {
      const int k = __ldg(m.sp + sl * R + j);
      if (k >= 0) {
        sW[k * ss] += (double)__ldg(m.nu + sl * R + j) * q;
      }
    }
  }
  double hs = 0.0;
#pragma unroll 1
  for (int k = 0; k < NS; ++k) {
    double cpR, hRT, sR, dcpR;
    nasa7(m, k, T, lnT, cpR, hRT, sR, dcpR);
    const double yd = sW[k * ss] * __ldg(m.mw + k) + v.F(k);
    v.fv(k) = yd;
    hs += hRT * kRu * T * __ldg(m.inv_mw + k) * yd;
  }
  v.fv(NS) = (v.F(NS) - hs) / rcp;
}

// ------------------------------------------------ constant-memory table
__constant__ __align__(16) unsigned char c_mech[kConstMechBytes];

__device__ __forceinline__ const CMechHeader& cm_hdr() { return *reinterpret_cast<const CMechHeader*>(c_mech); }
__device__ __forceinline__ const double* cm_d(int off) { return reinterpret_cast<const double*>(c_mech + off); }

// NASA-7 cp/R, h/RT, g/RT of species k at T from the constant table.
__device__ __forceinline__ void cm_nasa7(const CMechHeader& H, int k, double T, double lnT, double invT,
                                        double& cpR, double& hRT, double& gRT) {
  const double* nasa = cm_d(H.off_nasa);
  const int N = H.N;
  const int base = (T < nasa[k]) ? 1 : 8;
  const double a0 = nasa[(base + 0) * N + k], a1 = nasa[(base + 1) * N + k], a2 = nasa[(base + 2) * N + k];
  const double a3 = nasa[(base + 3) * N + k], a4 = nasa[(base + 4) * N + k], a5 = nasa[(base + 5) * N + k];
  const double a6 = nasa[(base + 6) * N + k];
  cpR = a0 + T * (a1 + T * (a2 + T * (a3 + T * a4)));
  hRT = a0 + T * (a1 / 2 + T * (a2 / 3 + T * (a3 / 4 + T * a4 / 5))) + a5 * invT;
  const double sR = a0 * lnT + T * (a1 + T * (a2 / 2 + T * (a3 / 3 + T * a4 / 4))) + a6;
  gRT = hRT - sR;
}

// Rate of progress of reaction j from the constant table (same formulas as
// r_progress).
__device__ __forceinline__ double cm_progress(const CMechHeader& H, int j, double T, double lnT, double invT,
                                              double Ctot, double lnPRT, const double* sC, const double* sG,
                                              int ss) {
  const RxnC& r = reinterpret_cast<const RxnC*>(c_mech + H.off_rxn)[j];
  const int type = r.type, flags = r.flags;
  const double kinf = exp(r.lnA + r.b * lnT - r.ea * invT);
  double M = 0.0;
  if (type != 0) {
    M = Ctot;
    const short* esp = reinterpret_cast<const short*>(c_mech + H.off_effsp);
    const double* em1 = cm_d(H.off_effm1);
    for (int q = r.e0; q < r.e1; ++q) M += em1[q] * sC[esp[q] * ss];
  }
  double kf = kinf;
  if (type >= 2) {
    const double k0 = exp(r.lnA0 + r.b0 * lnT - r.ea0 * invT);
    const double Pr = k0 * M / kinf;
    double F = 1.0;
    if (type == 3) {
      double Fc = (1.0 - r.ta) * exp(-T * r.t3i) + r.ta * exp(-T * r.t1i);
      if (flags & 4) Fc += exp(-r.t2 * invT);
      const double logFc = log10(fmax(Fc, 1e-300));
      const double c = -0.4 - 0.67 * logFc, nn = 0.75 - 1.27 * logFc;
      const double u = log10(fmax(Pr, 1e-300)) + c;
      const double f1 = u / (nn - 0.14 * u);
      F = exp(kLn10 * (logFc / (1.0 + f1 * f1)));
    }
    kf = kinf * Pr / (1.0 + Pr) * F;
  }
  double pf = 1.0, pr = 1.0, sg = 0.0;
#pragma unroll
  for (int sl = 0; sl < 8; ++sl) {
    const int k = r.sp[sl];
    if (k >= 0) {
      const int nu = r.nu[sl];
      const int na = nu < 0 ? -nu : nu;
      const double ck = sC[k * ss];
      double p = ck;
      for (int e = 1; e < na; ++e) p *= ck;
      if (sl < 4) pf *= p;
      else pr *= p;
      sg += nu * sG[k * ss];
    }
  }
  double kr = 0.0;
  if (flags & 2) kr = exp(r.lr + r.br * lnT - r.er * invT);
  else if (flags & 1) kr = kf * exp(sg - r.sdnu * lnPRT);
  double q = kf * pf - kr * pr;
  if (type == 1) q *= M;
  return q;
}

// HP right-hand side from the constant table (thread per cell).
template <int NS>
__device__ __forceinline__ void cm_rhs(const RVec<NS + 1>& v, double* sC, double* sG, double* sW, int ss) {
  const CMechHeader& H = cm_hdr();
  const double* imw = cm_d(H.off_imw);
  const double* mw = cm_d(H.off_mw);
  const double T = v.yev(NS);
  const double lnT = log(T), invT = 1.0 / T;
  double Ctot = 0.0, rcp = 0.0;
#pragma unroll 1
  for (int k = 0; k < NS; ++k) {
    double cpR, hRT, gRT;
    cm_nasa7(H, k, T, lnT, invT, cpR, hRT, gRT);
    const double yk = v.yev(k);
    const double Ck = yk * imw[k];
    sC[k * ss] = Ck;
    sG[k * ss] = gRT;
    sW[k * ss] = 0.0;
    Ctot += Ck;
    rcp += yk * cpR * kRu * imw[k];
  }
  const double lnPRT = log(kPatm / (kRu * T));
  const int R = H.R;
  const RxnC* rx = reinterpret_cast<const RxnC*>(c_mech + H.off_rxn);
#pragma unroll 1
  for (int j = 0; j < R; ++j) {
    const double q = cm_progress(H, j, T, lnT, invT, Ctot, lnPRT, sC, sG, ss);
#pragma unroll
    for (int sl = 0; sl < 8; ++sl) {
      const int k = rx[j].sp[sl];
      if (k >= 0) sW[k * ss] += (double)rx[j].nu[sl] * q;
    }
  }
  double hs = 0.0;
#pragma unroll 1
  for (int k = 0; k < NS; ++k) {
    double cpR, hRT, gRT;
    cm_nasa7(H, k, T, lnT, invT, cpR, hRT, gRT);
    const double yd = sW[k * ss] * mw[k] + v.F(k);
    v.fv(k) = yd;
    hs += hRT * kRu * T * imw[k] * yd;
  }
  v.fv(NS) = (v.F(NS) - hs) / rcp;
}

}  // namespace

cudaError_t rounds_upload_const(const void* blob, int bytes, cudaStream_t st) {
  if (bytes > kConstMechBytes) return cudaErrorInvalidValue;
  return cudaMemcpyToSymbolAsync(c_mech, blob, (size_t)bytes, 0, cudaMemcpyHostToDevice, st);
}

// ---------------------------------------------------------------- kernels
template <int NS>
__global__ void __launch_bounds__(128) rk_start(RoundsParams R) {
  constexpr int n = NS + 1;
  const ReactParams& P = R.P;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long base = (long long)blockIdx.x * blockDim.x; base < R.nchunk; base += stride) {
    const long long slot = base + threadIdx.x;
    const bool live = slot < R.nchunk;
    bool go = false, done = false, masked = false;
    // the FP64 retry pass integrates only the cells the FP32 pass flagged
    const bool skip = live && P.retry_pass && P.retry[R.chunk0 + slot] == 0;
    if (live && !skip) {
      const long long cell = R.chunk0 + slot;
      const CellLoc L = locate(P, cell);
      const DevBox& bx = *L.bx;
      if (bx.mask.p)
        masked = bx.mask.p[(long long)(L.i - bx.mask.lo0) + (long long)(L.j - bx.mask.lo1) * bx.mask.js +
                           (long long)(L.k - bx.mask.lo2) * bx.mask.ks] == 0;
      int code = 0;
      if (masked) {
        code = B200CHEM_CELL_MASKED;
        if (bx.fc.p) *elem(bx.fc, L.i, L.j, L.k) = 0.0;
      } else {
        unsigned char* rec = rec_of(R.S, slot);
        const RVec<n> v{reinterpret_cast<double*>(rec + R.S.L.off_vec)};
        const double* yp = elem(bx.rhoY, L.i, L.j, L.k);
        const double* fp = elem(bx.fY, L.i, L.j, L.k);
        double rho = 0.0;
        bool bad = false;
#pragma unroll 4
        for (int q = 0; q < NS; ++q) {
          const double y = yp[q * bx.rhoY.ns], f = fp[q * bx.fY.ns];
          v.zn(0, q) = y;
          v.F(q) = f;
          rho += y;
          bad |= !isfinite(y) || !isfinite(f);
        }
        const double T = *elem(bx.T, L.i, L.j, L.k), fH = *elem(bx.fH, L.i, L.j, L.k);
        v.zn(0, NS) = T;
        v.F(NS) = fH;
        bad |= !(T > 0.0) || !isfinite(T) || !isfinite(fH) || !(rho > 0.0);
        if (bad) {
          code = B200CHEM_CELL_NONFINITE;
          if (bx.fc.p) *elem(bx.fc, L.i, L.j, L.k) = 0.0;
          done = true;
        } else {
          RCell c;
          r_begin<n>(c, v, P.atol, P.rtol, P.dt, P.qmax, P.max_steps);
          store_cell(c, rec);
          go = true;
        }
      }
      if (!go && P.status) P.status[cell] = code;
    }
    warp_append(go, (int)slot, R.list_out, R.cnt_out);
    warp_stats(P.stats, done, true, masked, CellCounters{0, 0, 0, 0, 0, 0, 0});
  }
}

// Minimum resident CTAs (of 64 threads) per SM requested for the
// right-hand-side kernel: bounds its registers per thread.
#ifndef B200_RHS_MIN_CTAS
#define B200_RHS_MIN_CTAS 6
#endif

template <int NS>
__global__ void __launch_bounds__(kRoundsRhsBlock, B200_RHS_MIN_CTAS) rk_rhs(RoundsParams R) {
  constexpr int n = NS + 1;
  extern __shared__ __align__(16) unsigned char dsm[];
  __shared__ DevMech s_mech;
  if (threadIdx.x == 0) s_mech = R.P.mech;
  __syncthreads();
  const int cnt = *R.cnt_in;
  double* sC = reinterpret_cast<double*>(dsm) + threadIdx.x;
  double* sG = sC + NS * blockDim.x;
  double* sW = sG + NS * blockDim.x;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < cnt; idx += gridDim.x * blockDim.x) {
    const int slot = R.list_in[idx];
    const RVec<n> v{reinterpret_cast<double*>(rec_of(R.S, slot) + R.S.L.off_vec)};
    if (R.gen_mech) {
      // generated code for this mechanism: every coefficient an immediate
      if constexpr (NS == 9) gen::gen_rhs_synth_h2_9(&v.yev(0), &v.F(0), &v.fv(0));
      else if constexpr (NS == 21) gen::gen_rhs_synth_ch4_21(&v.yev(0), &v.F(0), &v.fv(0));
      else if constexpr (NS == 53) gen::gen_rhs_synth_c12_53(&v.yev(0), &v.F(0), &v.fv(0));
    } else if (R.const_mech) {
      cm_rhs<NS>(v, sC, sG, sW, blockDim.x);
    } else {
      r_rhs<NS>(s_mech, v, sC, sG, sW, blockDim.x);
    }
  }
}

// Minimum resident CTAs per SM requested for the control kernel (its
// register budget: 3 -> 168 registers per thread).
#ifndef B200_CTRL_MIN_CTAS
#define B200_CTRL_MIN_CTAS 3
#endif

// Lanes per cell of the control kernel.
#ifndef B200_CTRL_LANES
#define B200_CTRL_LANES 8
#endif
constexpr int ctrl_group(int n) { return n <= 32 ? B200_CTRL_LANES : 16; }

// L2 prefetch of the control kernel: 0 none; 1 the vectors and matrices of
// each cell as it starts (they stream in while the step-control scalars are
// processed); 2 also the scalars and vectors of the cell the group takes
// next.
#ifndef B200_CTRL_PREFETCH
#define B200_CTRL_PREFETCH 1
#endif

// Bulk prefetch of [p, p + bytes) into L2 (p and bytes multiples of 16; a
// hint: no completion to wait for).
__device__ __forceinline__ void l2_prefetch(const void* p, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// One cell of the control kernel, G lanes per cell: resume the CVODE state
// machine (after_rhs: consuming the f just evaluated, counted in nfe;
// otherwise coming back from a setup), write the outputs of a finished cell,
// and append the cell to the list of its next need.  Every lane of the warp
// calls it (the appends are warp-collective); `live` marks the groups with a
// cell.
template <int NS, int G, typename LUT>
__device__ __forceinline__ void ctrl_cell(const RoundsParams& R, bool live, int slot, bool after_rhs, int gl,
                                          unsigned gm, int idx_next) {
  constexpr int n = NS + 1;
  const ReactParams& P = R.P;
  int need = kDone, status = 0;
  RCell c;
  if (live) {
    unsigned char* rec = rec_of(R.S, slot);
    if (B200_CTRL_PREFETCH >= 1 && gl == 0)
      l2_prefetch(rec + R.S.L.off_vec, (uint32_t)(R.S.L.off_j - R.S.L.off_vec));
    if (B200_CTRL_PREFETCH >= 2 && gl == 0 && idx_next >= 0)
      l2_prefetch(rec_of(R.S, R.list_in[idx_next]), (uint32_t)R.S.L.off_j);
    load_cell(c, rec);
    // the Jacobian and the inverse only when this pass starts with a Newton
    // iteration (a pass that ends in a setup would fetch them for nothing)
    if (B200_CTRL_PREFETCH >= 1 && gl == 0 &&
        (c.label == kLAfterNIter || c.label == kLAfterSetup || (c.label == kLAfterNStart && !c.callSetup)))
      l2_prefetch(rec + R.S.L.off_j, (uint32_t)(R.S.L.stride - R.S.L.off_j));
    if (after_rhs) c.cnt.nfe++;
    const RVec<n> v{reinterpret_cast<double*>(rec + R.S.L.off_vec)};
    need = r_advance<n, G, LUT>(c, v, c.label, P.atol, P.rtol, reinterpret_cast<const double*>(rec + R.S.L.off_j),
                                reinterpret_cast<const LUT*>(rec + R.S.L.off_a), gl, gm, &status,
                                sizeof(LUT) == 4 ? P.refine_stall : 0.0, sizeof(LUT) == 4 ? P.refine_keep : 0.0);
    __syncwarp(gm);
    if (gl == 0) store_cell(c, rec);
    if (need == kDone) {
      const long long cell = R.chunk0 + slot;
      const CellLoc L = locate(P, cell);
      const DevBox& bx = *L.bx;
      if (status == 0) {
        // y(dt) from the Nordsieck array (Horner in s = (dt - tn) / h)
        const double s = (P.dt - c.tn) / c.h;
        double* yp = elem(bx.rhoY, L.i, L.j, L.k);
        const int q = c.q;
        each<n, G>(gl, [&](int k) {
          double y = v.zn(q, k);
          for (int jj = q - 1; jj >= 0; --jj) y = v.zn(jj, k) + s * y;
          if (k < NS) yp[k * bx.rhoY.ns] = y;
          else *elem(bx.T, L.i, L.j, L.k) = y;
        });
        if (gl == 0) {
          double* hp = elem(bx.rhoH, L.i, L.j, L.k);
          *hp = *hp + P.dt * v.F(NS);
        }
      }
      if (gl == 0) {
        if (status == kStatusRefineStall) {
          // untouched: no outputs, no status; the FP64 pass writes them
          P.retry[cell] = 1;
          if (P.stats) atomicAdd(reinterpret_cast<unsigned long long*>(P.stats + kStStall), 1ull);
        } else {
          if (bx.fc.p) *elem(bx.fc, L.i, L.j, L.k) = (double)c.cnt.nfe;
          if (P.status) P.status[cell] = status;
        }
      }
    }
  }
  const bool lead = live && gl == 0;
  warp_append(lead && need == kNeedRhs, slot, R.list_out, R.cnt_out);
  warp_append(lead && (need == kNeedSetup || need == kNeedSetupJac), slot, R.list_setup, R.cnt_setup);
  warp_append(lead && need == kNeedSetupJac, slot, R.list_jac, R.cnt_jac);
  warp_stats(P.stats, lead && need == kDone && status != kStatusRefineStall, status != 0, false, c.cnt);
}

// Resume the cells of list_in, G lanes per cell.  after_rhs: each consumes
// the f just evaluated (counted in nfe); otherwise they come back from a
// setup.
template <int NS, typename LUT>
__global__ void __launch_bounds__(128, B200_CTRL_MIN_CTAS) rk_ctrl(RoundsParams R, int after_rhs) {
  constexpr int n = NS + 1;
  constexpr int G = ctrl_group(n);
  constexpr int GPW = 32 / G;  // cells per warp
  const int cnt = *R.cnt_in;
  const int lane = threadIdx.x & 31, gl = lane % G, gi = lane / G;
  const unsigned gm = (G == 32) ? kFull : (((1u << G) - 1u) << (gi * G));
  const int wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int base = wid * GPW; base < cnt; base += nw * GPW) {
    const int idx = base + gi;
    const bool live = idx < cnt;
    const int nxt = idx + nw * GPW;
    ctrl_cell<NS, G, LUT>(R, live, live ? R.list_in[idx] : 0, after_rhs != 0, gl, gm, nxt < cnt ? nxt : -1);
  }
}

// In-place Gauss-Jordan inverse of the scaled Newton matrix D (I - gamma J)
// D^-1 (FP32, D = diag(dsc)) or I - gamma J (FP64) with partial pivoting, one
// warp per cell, lane i holding row i in registers (n <= 32).  Rows are never
// exchanged: step k takes as pivot the unused row p_k with the largest
// |a[., k]|, and at the end the inverse is (A^-1)[k][j] = X[p_k][q_j] with
// q_j the step at which row j was the pivot; that permutation is applied
// while the result is written column-major to Ar.  Xs, prow, pinv: per-warp
// shared scratch.  Returns 0, or k+1 when no usable pivot is left at step k.
template <int n, typename LUT>
__device__ __forceinline__ int reg_gj_inverse(const double* J, int ldj, const double* dsc, double gamma, LUT* Xs,
                                              int ldl, int* prow, int* pinv, LUT* Ar, int lda, int lane) {
  static_assert(n <= 32, "one row per lane");
  constexpr bool kScaled = sizeof(LUT) == 4;
  const bool row = lane < n;
  const double di = row ? dsc[lane] : 1.0;
  const double rdi = 1.0 / di;
  LUT a[n];
#pragma unroll
  for (int j = 0; j < n; ++j) {
    const double rdj = __shfl_sync(kFull, rdi, j);
    const double mij = ((lane == j) ? 1.0 : 0.0) - gamma * (row ? J[j * ldj + lane] : 0.0);
    a[j] = row ? (LUT)(kScaled ? mij * di * rdj : mij) : (LUT)0;
  }
  // Pivot search by one warp reduction: key = the bits of |a[k]| (FP32; the
  // high word for FP64) with the low 5 bits replaced by (31 - lane), so the
  // maximum picks the largest magnitude (to 2^-18 relative in FP32, 2^-15 in
  // FP64) and, among equals, the lowest lane.
  // The pivot row goes through shared memory (two buffers, alternating per
  // step, 16-byte chunks) and every row, the pivot row included, is updated
  // by one FMA per column: a_ij -= g_i * a_pj with g_i = a_ik / a_pk off the
  // pivot row and g_p = 1 - 1 / a_pk on it (which scales the pivot row by
  // 1 / a_pk); column k is set last (1 / a_pk on the pivot row, -g_i off it).
  constexpr int kVec = 16 / (int)sizeof(LUT);      // LUTs per 16-byte chunk
  constexpr int kChunks = (n + kVec - 1) / kVec;
  constexpr int kBuf = 32;                         // LUTs per row buffer (>= kChunks * kVec)
  static_assert(kChunks * kVec <= kBuf, "row buffer");
  unsigned used = 0;
  int mystep = -1;
#pragma unroll
  for (int k = 0; k < n; ++k) {
    LUT* buf = Xs + (k & 1) * kBuf;
    unsigned key = 0u;
    if (row && !((used >> lane) & 1u)) {
      unsigned bits;
      if constexpr (sizeof(LUT) == 4) bits = __float_as_uint(fabsf((float)a[k]));
      else bits = (unsigned)__double2hiint(fabs((double)a[k]));
      key = (bits & ~31u) | (unsigned)(31 - lane);
    }
    const unsigned kmax = __reduce_max_sync(kFull, key);
    if ((kmax >> 5) == 0u) return k + 1;  // no nonzero candidate: singular (warp-uniform)
    const int p = 31 - (int)(kmax & 31u);
    used |= 1u << p;
    if (lane == p) {
      mystep = k;
#pragma unroll
      for (int c = 0; c < kChunks; ++c) {
        LUT t[kVec];
#pragma unroll
        for (int e = 0; e < kVec; ++e) t[e] = (c * kVec + e < n) ? a[c * kVec + e] : (LUT)0;
        *reinterpret_cast<uint4*>(buf + c * kVec) = *reinterpret_cast<const uint4*>(t);
      }
    }
    __syncwarp();
    LUT pr[kChunks * kVec];
#pragma unroll
    for (int c = 0; c < kChunks; ++c) *reinterpret_cast<uint4*>(pr + c * kVec) = *reinterpret_cast<const uint4*>(buf + c * kVec);
    const LUT pv = pr[k];
    if (!(fabs(pv) > (LUT)0) || isnan(pv)) return k + 1;  // zero or NaN pivot (warp-uniform)
    const LUT inv = (LUT)1 / pv;
    const LUT gi = (lane == p) ? (LUT)1 - inv : a[k] * inv;
#pragma unroll
    for (int j = 0; j < n; ++j)
      if (j != k) a[j] = fma(-gi, pr[j], a[j]);
    a[k] = (lane == p) ? inv : -gi;
  }
  if (row) {
#pragma unroll
    for (int j = 0; j < n; ++j) Xs[lane * ldl + j] = a[j];
    pinv[lane] = mystep;
    prow[mystep] = lane;
  }
  __syncwarp();
  if (lane < n) {
    const int pk = prow[lane];
    for (int j = 0; j < n; ++j) Ar[j * lda + lane] = Xs[pk * ldl + pinv[j]];
  } else if (lane < lda) {
    for (int j = 0; j < n; ++j) Ar[j * lda + lane] = (LUT)0;  // column padding
  }
  __syncwarp();
  return 0;
}

// The same inverse for 32 < n <= 64 in FP32: lane l holds rows l and l + 32
// in registers.  The pivot key carries the row index (6 bits) instead of the
// lane; the pivot row's owner writes it to shared memory and every lane
// updates both of its rows from 16-byte reads of it.
template <int n, typename LUT>
__device__ __forceinline__ int reg_gj_inverse2(const double* J, int ldj, const double* dsc, double gamma, LUT* Xs,
                                               int ldl, int* prow, int* pinv, LUT* Ar, int lda, int lane) {
  static_assert(n > 32 && n <= 64 && sizeof(LUT) == 4, "two FP32 rows per lane");
  const int r1 = lane + 32;
  const bool row1 = r1 < n;
  const double d0 = dsc[lane], d1 = row1 ? dsc[r1] : 1.0;
  const double rd0 = 1.0 / d0, rd1 = 1.0 / d1;
  LUT a0[n], a1[n];
#pragma unroll
  for (int j = 0; j < n; ++j) {
    const double rdj = (j < 32) ? __shfl_sync(kFull, rd0, j) : __shfl_sync(kFull, rd1, j - 32);
    const double m0 = ((lane == j) ? 1.0 : 0.0) - gamma * J[j * ldj + lane];
    const double m1 = row1 ? ((r1 == j) ? 1.0 : 0.0) - gamma * J[j * ldj + r1] : 0.0;
    a0[j] = (LUT)(m0 * d0 * rdj);
    a1[j] = row1 ? (LUT)(m1 * d1 * rdj) : (LUT)0;
  }
  constexpr int kChunks = (n + 3) / 4;
  constexpr int kBuf = 64;
  unsigned used0 = 0, used1 = 0;
  int step0 = -1, step1 = -1;
#pragma unroll
  for (int k = 0; k < n; ++k) {
    LUT* buf = Xs + (k & 1) * kBuf;
    unsigned key = 0u;
    if (!((used0 >> lane) & 1u)) key = (__float_as_uint(fabsf(a0[k])) & ~63u) | (unsigned)(63 - lane);
    if (row1 && !((used1 >> lane) & 1u)) {
      const unsigned k1 = (__float_as_uint(fabsf(a1[k])) & ~63u) | (unsigned)(63 - r1);
      key = key > k1 ? key : k1;
    }
    const unsigned kmax = __reduce_max_sync(kFull, key);
    if ((kmax >> 6) == 0u) return k + 1;  // no nonzero candidate: singular (warp-uniform)
    const int p = 63 - (int)(kmax & 63u);
    const int pl = p & 31;
    if (p < 32) used0 |= 1u << pl;
    else used1 |= 1u << pl;
    if (lane == pl) {
      if (p < 32) {
        step0 = k;
#pragma unroll
        for (int c = 0; c < kChunks; ++c) {
          float4 t;
          t.x = a0[4 * c];
          t.y = (4 * c + 1 < n) ? a0[4 * c + 1] : 0.f;
          t.z = (4 * c + 2 < n) ? a0[4 * c + 2] : 0.f;
          t.w = (4 * c + 3 < n) ? a0[4 * c + 3] : 0.f;
          reinterpret_cast<float4*>(buf)[c] = t;
        }
      } else {
        step1 = k;
#pragma unroll
        for (int c = 0; c < kChunks; ++c) {
          float4 t;
          t.x = a1[4 * c];
          t.y = (4 * c + 1 < n) ? a1[4 * c + 1] : 0.f;
          t.z = (4 * c + 2 < n) ? a1[4 * c + 2] : 0.f;
          t.w = (4 * c + 3 < n) ? a1[4 * c + 3] : 0.f;
          reinterpret_cast<float4*>(buf)[c] = t;
        }
      }
    }
    __syncwarp();
    const LUT pv = buf[k];
    if (!(fabsf(pv) > 0.f) || isnan(pv)) return k + 1;  // zero or NaN pivot (warp-uniform)
    const LUT inv = 1.f / pv;
    const LUT g0 = (p == lane) ? 1.f - inv : a0[k] * inv;
    const LUT g1 = (p == r1) ? 1.f - inv : a1[k] * inv;
#pragma unroll
    for (int c = 0; c < kChunks; ++c) {
      const float4 q = reinterpret_cast<const float4*>(buf)[c];
      const float qv[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int j = 4 * c + e;
        if (j < n && j != k) {
          a0[j] = fmaf(-g0, qv[e], a0[j]);
          a1[j] = fmaf(-g1, qv[e], a1[j]);
        }
      }
    }
    a0[k] = (p == lane) ? inv : -g0;
    a1[k] = (p == r1) ? inv : -g1;
  }
  __syncwarp();  // the row buffers live in Xs
#pragma unroll
  for (int j = 0; j < n; ++j) Xs[lane * ldl + j] = a0[j];
  if (row1) {
#pragma unroll
    for (int j = 0; j < n; ++j) Xs[r1 * ldl + j] = a1[j];
  }
  pinv[lane] = step0;
  prow[step0] = lane;
  if (row1) {
    pinv[r1] = step1;
    prow[step1] = r1;
  }
  __syncwarp();
  for (int h = 0; h < 2; ++h) {
    const int i = lane + 32 * h;
    if (i < n) {
      const int pk = prow[i];
      for (int j = 0; j < n; ++j) Ar[j * lda + i] = Xs[pk * ldl + pinv[j]];
    } else if (i < lda) {
      for (int j = 0; j < n; ++j) Ar[j * lda + i] = (LUT)0;  // column padding
    }
  }
  __syncwarp();
  return 0;
}

// Analytic Jacobian of one cell by one warp, lane per reaction: each lane
// evaluates its reactions (rates and their derivatives) and adds their
// contributions to a shared-memory Jacobian with atomics -- the mass-action
// columns of the reaction's own species, the temperature column, and the
// third-body terms (the default efficiency 1 of every species as a row
// vector u added to all columns at the end, the non-default ones per
// species).  Then lane l finishes column l (mass units) and its temperature
// row entry, and writes the column into the cell record (column-major, ldj).
// s: C, g/RT, h/RT [Npad]; Js: [n][n] column-major; us: [Npad] (shared).
template <int CPL>
__device__ __forceinline__ void warp_jac(const DevMech& m, const GrpScratch& s, double* Js, double* us,
                                         const Vec<CPL>& y, const Vec<CPL>& fy, double* J, int ldj, int lane) {
  const Grp<32> g(lane);
  const int N = m.N, R = m.R, n = N + 1;
  const double T = grp_get_T<32, CPL>(g, y, N);
  const double lnT = log(T), invT = 1.0 / T;
  double cpk[CPL], hk[CPL], dcpk[CPL];
  grp_species<32, CPL>(m, s, g, y, T, lnT, cpk, hk, dcpk);
  double csum = 0.0;
#pragma unroll
  for (int c = 0; c < CPL; ++c)
    if (lane + 32 * c < N) csum += y.v[c] * __ldg(m.inv_mw + lane + 32 * c);
  const double Ctot = g.sum(csum);
  const double lnPRT = log(kPatm / (kRu * T));
  for (int e = lane; e < n * n; e += 32) Js[e] = 0.0;
  for (int k = lane; k < n; k += 32) us[k] = 0.0;
  __syncwarp();
  for (int j = lane; j < R; j += 32) {
    const RxnEval e = eval_reaction<true>(m, SpView{s.C, s.gRT, s.hRT}, j, T, lnT, invT, Ctot, lnPRT);
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
    // mass-action columns: reactant slots (forward), product slots (reverse)
#pragma unroll
    for (int a = 0; a < 8; ++a) {
      if (sp[a] < 0) continue;
      const int va = (a < 4) ? -nu[a] : nu[a];
      double p = va * ipow(s.C[sp[a]], va - 1);
      const int b0 = (a < 4) ? 0 : 4;
#pragma unroll
      for (int s2 = 0; s2 < 4; ++s2) {
        const int o = b0 + s2;
        if (o != a && sp[o] >= 0) p *= ipow(s.C[sp[o]], (a < 4) ? -nu[o] : nu[o]);
      }
      const double d = (a < 4) ? kfm * p : -krm * p;
      double* col = Js + sp[a] * n;
#pragma unroll
      for (int r = 0; r < 8; ++r)
        if (sp[r] >= 0) atomicAdd(col + sp[r], (double)nu[r] * d);
    }
    // temperature column and third-body terms
    double* colT = Js + N * n;
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      if (sp[r] < 0) continue;
      atomicAdd(colT + sp[r], (double)nu[r] * dqdT);
      if (type != 0) atomicAdd(us + sp[r], (double)nu[r] * ceff);
    }
    if (type != 0) {
      const int q0 = __ldg(m.eff_ptr + j), q1 = __ldg(m.eff_ptr + j + 1);
      for (int q = q0; q < q1; ++q) {
        double* col = Js + __ldg(m.eff_sp + q) * n;
        const double d = __ldg(m.eff_m1 + q) * ceff;
#pragma unroll
        for (int r = 0; r < 8; ++r)
          if (sp[r] >= 0) atomicAdd(col + sp[r], (double)nu[r] * d);
      }
    }
  }
  // every lane is done with h/RT (read by the reaction derivatives) before it
  // is overwritten with the mass-specific enthalpy
  __syncwarp();
  // temperature-row ingredients
  double rcp = 0.0, drcp = 0.0, cpdot = 0.0, Tdot = 0.0;
#pragma unroll
  for (int c = 0; c < CPL; ++c) {
    const int k = lane + 32 * c;
    if (k < N) {
      rcp += y.v[c] * cpk[c];
      drcp += y.v[c] * dcpk[c];
      cpdot += cpk[c] * fy.v[c];
      s.hRT[k] = hk[c];  // mass-specific h for the temperature row
    } else if (k == N) {
      Tdot = fy.v[c];
    }
  }
  rcp = g.sum(rcp);
  drcp = g.sum(drcp);
  cpdot = g.sum(cpdot);
  Tdot = g.sum(Tdot);
  __syncwarp();
  // lane l finishes column l: mass units, default third-body row, T row
#pragma unroll
  for (int c = 0; c < CPL; ++c) {
    const int l = lane + 32 * c;
    if (l > N) continue;
    const double inv_wl = (l < N) ? __ldg(m.inv_mw + l) : 1.0;
    const double* src = Js + l * n;
    double* dst = J + l * ldj;
    double sum = 0.0;
    for (int k = 0; k < N; ++k) {
      const double v = (src[k] + ((l < N) ? us[k] : 0.0)) * __ldg(m.mw + k) * inv_wl;
      dst[k] = v;
      sum += s.hRT[k] * v;
    }
    dst[N] = -(sum + ((l < N) ? Tdot * cpk[c] : cpdot + Tdot * drcp)) / rcp;
  }
  __syncwarp();
}

// Jacobian refresh for the cells of the setup list whose matrix CVODE's
// jbad rule marks stale: the analytic FP64 Jacobian (column-major) into the
// cell record, one warp per cell.
// Minimum resident CTAs per SM requested for the Jacobian kernel (bounds
// its registers per thread; n > 32 keeps 2: its shared memory allows no
// more).
#ifndef B200_JAC_MIN_CTAS
#define B200_JAC_MIN_CTAS 8
#endif

template <int NS, int CPL>
__global__ void __launch_bounds__(128, CPL == 1 ? B200_JAC_MIN_CTAS : 2) rk_jac(RoundsParams R) {
  constexpr int n = NS + 1;
  extern __shared__ __align__(16) unsigned char dsm[];
  __shared__ DevMech s_mech;
  if (threadIdx.x == 0) s_mech = R.P.mech;
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const RoundsSetupLayout& SL = R.SL;
  double* d = reinterpret_cast<double*>(dsm + (size_t)w * SL.jac_smem_per_warp);
  GrpScratch ms;
  ms.C = d;
  ms.gRT = d + SL.Npad;
  ms.hRT = d + 2 * SL.Npad;
  double* us = d + 3 * SL.Npad;
  double* Js = d + 4 * SL.Npad;
  ms.q = ms.r1 = ms.r2 = ms.r3 = ms.r4 = nullptr;
  const long long gw = (long long)blockIdx.x * (blockDim.x >> 5) + w;
  const int cnt = *R.cnt_in;
  const RLayout RL = R.S.L;
  const long long nwarps = (long long)gridDim.x * (blockDim.x >> 5);
  for (long long idx = gw; idx < cnt; idx += nwarps) {
    const int slot = R.list_in[idx];
    unsigned char* rec = rec_of(R.S, slot);
    // the control kernel chose these cells by CVODE's jbad rule and already
    // counted the refresh
    const RVec<n> v{reinterpret_cast<double*>(rec + RL.off_vec)};
    Vec<CPL> y, fy;
#pragma unroll
    for (int cc = 0; cc < CPL; ++cc) {
      const int i = lane + 32 * cc;
      y.v[cc] = (i < n) ? v.yev(i) : 0.0;
      fy.v[cc] = (i < n) ? v.ftemp(i) : 0.0;
    }
    warp_jac<CPL>(s_mech, ms, Js, us, y, fy, reinterpret_cast<double*>(rec + RL.off_j), RL.ldj, lane);
    __syncwarp();
  }
}

// Minimum resident CTAs per SM requested for the inversion kernel (bounds
// its registers per thread).
#ifndef B200_GJ_MIN_CTAS
#define B200_GJ_MIN_CTAS 6
#endif

// Newton-matrix inverse of the cells of the setup list, one warp per cell:
// Gauss-Jordan inverse of D (I - gamma J) D^-1 with D = diag(ewt) (FP32) or
// of I - gamma J (FP64), written column-major into the cell record.
template <int NS, typename LUT, int CPL>
__global__ void __launch_bounds__(128, CPL == 1 ? B200_GJ_MIN_CTAS : 2) rk_gj(RoundsParams R) {
  constexpr int n = NS + 1;
  extern __shared__ __align__(16) unsigned char dsm[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const RoundsSetupLayout& SL = R.SL;
  unsigned char* sb = dsm + (size_t)w * SL.gj_smem_per_warp;
  double* Dsc = reinterpret_cast<double*>(sb);
  LUT* A = reinterpret_cast<LUT*>(Dsc + SL.Npad);
  LUT* fcol = A + (size_t)n * SL.ldl;
  int* ipiv = reinterpret_cast<int*>(fcol + SL.Npad);
  int* ipiv2 = ipiv + SL.Npad;
  const int cnt = *R.cnt_in;
  const RLayout RL = R.S.L;
  const long long gw = (long long)blockIdx.x * (blockDim.x >> 5) + w;
  const long long nwarps = (long long)gridDim.x * (blockDim.x >> 5);
  for (long long idx = gw; idx < cnt; idx += nwarps) {
    const int slot = R.list_in[idx];
    unsigned char* rec = rec_of(R.S, slot);
    RCell* cp = reinterpret_cast<RCell*>(rec);
    const RVec<n> v{reinterpret_cast<double*>(rec + RL.off_vec)};
    const double* J = reinterpret_cast<const double*>(rec + RL.off_j);
    LUT* Ar = reinterpret_cast<LUT*>(rec + RL.off_a);
    const double gamma = cp->gamma;
#pragma unroll
    for (int cc = 0; cc < CPL; ++cc) {
      const int i = lane + 32 * cc;
      if (i < n) {
        const double ds = (sizeof(LUT) == 4) ? v.ewt(i) : 1.0;
        Dsc[i] = ds;
        v.dsc(i) = ds;
      }
    }
    __syncwarp();
    int ier;
    if constexpr (CPL == 1) {
      ier = reg_gj_inverse<(CPL == 1 ? n : 1), LUT>(J, RL.ldj, Dsc, gamma, A, SL.ldl, ipiv, ipiv2, Ar, RL.lda,
                                                    lane);
    } else if constexpr (CPL == 2 && sizeof(LUT) == 4) {
      ier = reg_gj_inverse2<(CPL == 2 ? n : 33), LUT>(J, RL.ldj, Dsc, gamma, A, SL.ldl, ipiv, ipiv2, Ar, RL.lda,
                                                      lane);
    } else {
      ier = grp_gj_inverse<32, LUT>(J, RL.ldj, A, SL.ldl, ipiv, fcol, Dsc, n, gamma, lane);
      __syncwarp();
      if (ier == 0)
        for (int j = 0; j < n; ++j)
#pragma unroll
          for (int cc = 0; cc < CPL; ++cc) {
            const int i = lane + 32 * cc;
            if (i < n) Ar[j * RL.lda + i] = A[i * SL.ldl + j];
          }
    }
    __syncwarp();
    if (lane == 0) {
      cp->cnt.nlu++;
      cp->gamma_lu = gamma;
      cp->gamrat = 1.0;
      cp->gammap = gamma;
      cp->crate = 1.0;
      cp->nstlp = cp->cnt.nst;
      cp->setup_ier = ier;
    }
    __syncwarp();
  }
}

// ------------------------------------------------------------ host side
namespace {

template <int NS>
int rhs_smem(int block) { return 3 * NS * block * (int)sizeof(double); }

template <int NS, typename LUT>
cudaError_t rounds_setup_attrs(const RoundsSetupLayout& SL) {
  constexpr int n = NS + 1;
  constexpr int CPL = (n + 31) / 32;
  cudaError_t e = cudaFuncSetAttribute(rk_rhs<NS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       rhs_smem<NS>(kRoundsRhsBlock));
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(rk_jac<NS, CPL>, cudaFuncAttributeMaxDynamicSharedMemorySize, 4 * SL.jac_smem_per_warp);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(rk_gj<NS, LUT, CPL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              4 * SL.gj_smem_per_warp);
}

template <int NS, typename LUT>
cudaError_t rounds_grids(const RoundsSetupLayout& SL, int sm_count, RoundsGrids* G) {
  constexpr int n = NS + 1;
  constexpr int CPL = (n + 31) / 32;
  cudaError_t e = rounds_setup_attrs<NS, LUT>(SL);
  if (e != cudaSuccess) return e;
  int b = 0;
  // grid sized for the generated right-hand side (no shared memory); the
  // table forms run the same grid-stride loop with fewer CTAs resident
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, rk_rhs<NS>, kRoundsRhsBlock, 0)) != cudaSuccess)
    return e;
  G->rhs = std::max(1, b) * sm_count;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, rk_ctrl<NS, LUT>, 128, 0)) != cudaSuccess) return e;
  G->ctrl = std::max(1, b) * sm_count;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, rk_jac<NS, CPL>, 128, 4 * SL.jac_smem_per_warp)) !=
      cudaSuccess)
    return e;
  G->jac = std::max(1, b) * sm_count;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, rk_gj<NS, LUT, CPL>, 128, 4 * SL.gj_smem_per_warp)) !=
      cudaSuccess)
    return e;
  G->gj = std::max(1, b) * sm_count;
  G->start = 4 * sm_count;
  return cudaSuccess;
}

template <int NS, typename LUT>
cudaError_t rounds_launch_t(int what, const RoundsParams& R, const RoundsGrids& G, int after_rhs, cudaStream_t st) {
  constexpr int n = NS + 1;
  constexpr int CPL = (n + 31) / 32;
  switch (what) {
    case kRoundsStart:
      rk_start<NS><<<G.start, 128, 0, st>>>(R);
      break;
    case kRoundsRhs:
      // the generated right-hand side keeps everything in registers
      rk_rhs<NS><<<G.rhs, kRoundsRhsBlock, R.gen_mech ? 0 : rhs_smem<NS>(kRoundsRhsBlock), st>>>(R);
      break;
    case kRoundsCtrl:
      rk_ctrl<NS, LUT><<<G.ctrl, 128, 0, st>>>(R, after_rhs);
      break;
    case kRoundsJac:
      rk_jac<NS, CPL><<<G.jac, 128, 4 * R.SL.jac_smem_per_warp, st>>>(R);
      break;
    case kRoundsGj:
      rk_gj<NS, LUT, CPL><<<G.gj, 128, 4 * R.SL.gj_smem_per_warp, st>>>(R);
      break;
    default:
      return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace

bool rounds_supported(int N) { return N == 9 || N == 21 || N == 53; }

RoundsSetupLayout rounds_setup_layout(int N, int R, int lut_bytes) {
  RoundsSetupLayout L;
  const int n = N + 1;
  L.Npad = ((n + 31) / 32) * 32;
  L.Rpad = std::max(32, ((R + 31) / 32) * 32);
  L.ldl = n | 1;
  L.jac_smem_per_warp = (int)(8LL * (4 * L.Npad + (long long)n * n));
  const long long b = 8LL * L.Npad + (long long)lut_bytes * ((long long)n * L.ldl + L.Npad) + 4LL * 2 * L.Npad;
  L.gj_smem_per_warp = (int)((b + 15) & ~15LL);
  L.gbytes_per_warp = (8LL * 4LL * L.Rpad + 255) & ~255LL;
  return L;
}

long long rounds_state_bytes_per_cell(int N, int lut_bytes) {
  return rounds_record_layout(N + 1, lut_bytes).stride + 4LL * 4;  // record + four slot lists
}

RState rounds_carve(void* base, long long cap, int N, int lut_bytes) {
  RState S;
  S.rec = static_cast<unsigned char*>(base);
  S.L = rounds_record_layout(N + 1, lut_bytes);
  S.cap = cap;
  return S;
}

cudaError_t rounds_grids_for(int N, int lut_bytes, const RoundsSetupLayout& SL, int sm_count, RoundsGrids* G) {
  if (N == 9) return lut_bytes == 4 ? rounds_grids<9, float>(SL, sm_count, G) : rounds_grids<9, double>(SL, sm_count, G);
  if (N == 21)
    return lut_bytes == 4 ? rounds_grids<21, float>(SL, sm_count, G) : rounds_grids<21, double>(SL, sm_count, G);
  if (N == 53)
    return lut_bytes == 4 ? rounds_grids<53, float>(SL, sm_count, G) : rounds_grids<53, double>(SL, sm_count, G);
  return cudaErrorInvalidValue;
}

cudaError_t rounds_launch(int N, int lut_bytes, int what, const RoundsParams& R, const RoundsGrids& G, int after_rhs,
                          cudaStream_t st) {
  if (N == 9)
    return lut_bytes == 4 ? rounds_launch_t<9, float>(what, R, G, after_rhs, st)
                          : rounds_launch_t<9, double>(what, R, G, after_rhs, st);
  if (N == 21)
    return lut_bytes == 4 ? rounds_launch_t<21, float>(what, R, G, after_rhs, st)
                          : rounds_launch_t<21, double>(what, R, G, after_rhs, st);
  if (N == 53)
    return lut_bytes == 4 ? rounds_launch_t<53, float>(what, R, G, after_rhs, st)
                          : rounds_launch_t<53, double>(what, R, G, after_rhs, st);
  return cudaErrorInvalidValue;
}

}  // namespace b200

namespace b200 {
// Generated right-hand side matching a mechanism digest: 0 none, else the
// species count of the generated code.
int rounds_generated_for(unsigned long long digest) {
  if (digest == gen::kGenDigest_synth_h2_9) return 9;
  if (digest == gen::kGenDigest_synth_ch4_21) return 21;
  if (digest == gen::kGenDigest_synth_c12_53) return 53;
  return 0;
}
}  // namespace b200
