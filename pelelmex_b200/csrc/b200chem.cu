// b200chem.cu -- C ABI and host side of the B200 HP chemistry reactor, plus
// the mechanism-evaluation kernels (RHS, Jacobian, instantaneous rates,
// T from (h, Y)).  The react kernels live in react_g*.cu (group integrator)
// and react_tpc.cu (thread-per-cell integrator).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"
#include "react_group.cuh"

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

#define CK(x)                                                                                     \
  do {                                                                                            \
    cudaError_t e_ = (x);                                                                         \
    if (e_ != cudaSuccess) return set_err(B200CHEM_ECUDA, "%s: %s", #x, cudaGetErrorString(e_)); \
  } while (0)

// ------------------------------------------------ evaluation-only kernels
// One group of 32 lanes per cell (the mechanism functions of group_mech.cuh).
struct EvalParams {
  DevMech mech;
  const double* y;
  const double* F;
  double* out;
  long long ncells;
  GroupLayout L;
  unsigned char* gscratch;
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
  GroupBdf<32, CPL, double> B;
  const long long gw = (long long)blockIdx.x * (blockDim.x >> 5) + w;
  carve_group<32, CPL, double>(B, P.L, dsm + (size_t)w * P.L.smem_bytes, P.gscratch + gw * P.L.gbytes);
  const long long wstride = (long long)gridDim.x * (blockDim.x >> 5);
  for (long long c0 = gw; c0 < P.ncells; c0 += wstride) {
    Vec<CPL> y, F;
#pragma unroll
    for (int c = 0; c < CPL; ++c) {
      const int q = lane + 32 * c;
      y.v[c] = (q < n) ? P.y[c0 * n + q] : 0.0;
      F.v[c] = (q < n) ? P.F[c0 * n + q] : 0.0;
    }
    const Vec<CPL> yd = grp_rhs<32, CPL>(&s_mech, B.ms, y, F, lane);
    if (P.what == 0) {
#pragma unroll
      for (int c = 0; c < CPL; ++c)
        if (lane + 32 * c < n) P.out[c0 * n + lane + 32 * c] = yd.v[c];
    } else {
      grp_jac<32, CPL>(&s_mech, B.ms, y, yd, B.J, B.ldj, lane);
      // B.J is column-major: (row i, col l) at l*ldj + i; the output is row-major
#pragma unroll
      for (int c = 0; c < CPL; ++c) {
        const int l = lane + 32 * c;
        if (l < n)
          for (int i = 0; i < n; ++i) P.out[(c0 * n + i) * n + l] = B.J[l * B.ldj + i];
      }
    }
    __syncwarp();
  }
}

// T from (h, Y) by Newton on h(T) = sum Y_k h_k(T), warp per cell (HY2T).
template <int CPL>
__device__ double warp_t_from_hy(const DevMech& m, const double (&Y)[CPL], double h, double T, int lane) {
  const Grp<32> g(lane);
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
    hs = g.sum(hs);
    cs = g.sum(cs);
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
  GroupLayout L;
};

template <int CPL>
__global__ void __launch_bounds__(128) inst_rr_kernel(InstParams P) {
  extern __shared__ __align__(16) unsigned char dsm[];
  __shared__ DevMech s_mech;
  if (threadIdx.x == 0) s_mech = P.mech;
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int N = P.mech.N;
  GrpScratch ms;
  double* d = reinterpret_cast<double*>(dsm + (size_t)w * P.L.smem_bytes);
  ms.C = d;
  ms.gRT = d + P.L.Npad;
  ms.hRT = d + 2 * P.L.Npad;
  ms.q = d + 6 * P.L.Npad;
  ms.r1 = ms.r2 = ms.r3 = ms.r4 = nullptr;
  const long long wstride = (long long)gridDim.x * (blockDim.x >> 5);
  const Grp<32> g(lane);
  for (long long c0 = (long long)blockIdx.x * (blockDim.x >> 5) + w; c0 < P.ncells; c0 += wstride) {
    double ry[CPL], Y[CPL];
    double rho = 0.0;
#pragma unroll
    for (int c = 0; c < CPL; ++c) {
      const int k = lane + 32 * c;
      ry[c] = (k < N) ? P.rhoY[(long long)k * P.ncells + c0] : 0.0;
      rho += ry[c];
    }
    rho = g.sum(rho);
    const double rinv = 1.0 / rho;
#pragma unroll
    for (int c = 0; c < CPL; ++c) Y[c] = ry[c] * rinv;
    const double h = P.rhoH[c0] * rinv * 1.0e4;  // J/kg -> erg/g
    const double T = warp_t_from_hy<CPL>(s_mech, Y, h, P.T[c0], lane);
    if (lane == 0) P.T[c0] = T;
    if (P.rhoYdot) {
      Vec<CPL> y, F;
#pragma unroll
      for (int c = 0; c < CPL; ++c) {
        const int k = lane + 32 * c;
        y.v[c] = (k < N) ? ry[c] * 1.0e-3 : (k == N ? T : 0.0);  // kg/m^3 -> g/cm^3
        F.v[c] = 0.0;
      }
      const Vec<CPL> yd = grp_rhs<32, CPL>(&s_mech, ms, y, F, lane);
#pragma unroll
      for (int c = 0; c < CPL; ++c) {
        const int k = lane + 32 * c;
        if (k < N) P.rhoYdot[(long long)k * P.ncells + c0] = yd.v[c] * 1.0e3;  // g/cm^3/s -> kg/m^3/s
      }
    }
    __syncwarp();
  }
}

// getHGivenT (Source/PeleLMeX_K.H:598-615) and getHeatRelease
// (Source/PeleLMeX_Reactions.cpp:477-506), thread per cell: species
// enthalpies h_k(T) (CEPTR's T2Hi, erg/g) converted to J/kg, and
// HRR = -sum_k h_k I_R,k (the reference's accumulation order, one FMA per
// species).  Component-major arrays of ncells.
__global__ void thermo_hr_kernel(DevMech m, const double* __restrict__ T, const double* __restrict__ IR,
                                 double* __restrict__ Hi, double* __restrict__ HR, long long ncells) {
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < ncells;
       c += (long long)gridDim.x * blockDim.x) {
    const double t = T[c];
    const double lnT = log(t);
    double hr = 0.0;
    for (int k = 0; k < m.N; ++k) {
      double cpR, hRT, sR, dcpR;
      nasa7(m, k, t, lnT, cpR, hRT, sR, dcpR);
      const double hk = hRT * kRu * t * __ldg(m.inv_mw + k) * 0.0001;  // erg/g -> J/kg
      if (Hi) Hi[(long long)k * ncells + c] = hk;
      if (HR) hr = fma(-hk, IR[(long long)k * ncells + c], hr);
    }
    if (HR) HR[c] = hr;
  }
}

}  // namespace

// ------------------------------------------------------------------ handle
// A small host-built array (box descriptors) copied to the device on the
// caller's stream: pinned staging plus a device copy, both reused across
// calls; the staging buffer is rewritten only after the previous call's copy
// from it has completed.
struct StagedBuf {
  void* d = nullptr;
  void* h = nullptr;
  size_t bytes = 0;
  bool pending = false;
  cudaEvent_t ev = nullptr;
};

struct b200chem_reactor {
  int device = 0;
  int N = 0, R = 0, n = 0;
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
  int smem_optin = 0;
  void* d_work = nullptr;  // integrator scratch (group Jacobians, or thread-per-cell matrices)
  size_t work_bytes = 0;
  // round-based integrator
  void* d_rounds = nullptr;  // cell state of one chunk + its three slot lists
  size_t rounds_bytes = 0;
  void* d_rwarp = nullptr;   // per-warp scratch of the setup kernel
  size_t rwarp_bytes = 0;
  int* d_rcnt = nullptr;     // list counters [A, B, S]
  int* h_rcnt = nullptr;     // pinned copy of one counter
  RoundsGrids rgrid{};
  int rgrid_lut = 0;
  long long launches = 0;  // kernels launched by this handle (instrumentation)
  unsigned char* h_cmech = nullptr;  // pinned packed constant-memory table (null: too large)
  int cmech_bytes = 0;
  int gen_mech = 0;  // 1: a generated right-hand side matches the mechanism
  unsigned long long digest = 0;  // FNV-1a digest of the mechanism description
  b200chem_tuning tune{};           // launch shape of the round-based integrator
  cudaStream_t cap_stream = nullptr;  // private stream the round graph is captured on
  cudaGraphExec_t rgraph = nullptr;   // executable graph of rounds_per_check rounds
  int rgraph_rounds = 0;              // rounds in rgraph
  StagedBuf cboxes;                   // advanceChemistry box descriptors
  StagedBuf fboxes;                   // getScalarReactForce box descriptors
  int* d_retry = nullptr;             // per-cell flags of the FP64 fallback pass
  size_t retry_bytes = 0;
  int* d_zero_mask = nullptr;         // all-zero mask row of the covered (skip_react) boxes
  long long zero_mask_len = 0;
  // per-kernel profile of the round integrator (b200chem_profile_begin/end)
  struct ProfRec {
    int kind;
    int slot;  // index into h_pcnt (-1: cell count known on the host)
    long long cells;
    cudaEvent_t e0, e1;
  };
  bool prof_on = false;
  bool prof_overflow = false;
  std::vector<ProfRec> prof;
  std::vector<cudaEvent_t> ev_pool;
  size_t ev_used = 0;
  int* h_pcnt = nullptr;  // pinned list counts copied before each profiled launch
  int pcnt_used = 0;
};

namespace b200 {
// Accessors for the other translation units (surrogate kernels).
const DevMech* handle_mech(b200chem_handle h) { return &h->mech; }
int handle_species(b200chem_handle h) { return h->N; }
const double* handle_atol(b200chem_handle h) { return h->d_atol; }
int handle_device(b200chem_handle h) { return h->device; }
void handle_count_launch(b200chem_handle h) { h->launches++; }
int handle_set_error(int code, const char* msg) { return set_err(code, "%s", msg); }
unsigned long long handle_digest(b200chem_handle h) { return h->digest; }
int handle_sm_count(b200chem_handle h) { return h->sm_count; }
}  // namespace b200

namespace {

template <typename T>
size_t push(std::vector<unsigned char>& buf, const std::vector<T>& v) {
  size_t off = (buf.size() + 255) & ~(size_t)255;
  buf.resize(off + sizeof(T) * std::max<size_t>(v.size(), 1));
  if (!v.empty()) memcpy(buf.data() + off, v.data(), sizeof(T) * v.size());
  return off;
}

int ensure_work(b200chem_reactor* h, size_t bytes, cudaStream_t st) {
  if (bytes <= h->work_bytes) return 0;
  if (h->d_work) {
    CK(cudaStreamSynchronize(st));
    cudaFree(h->d_work);
    h->d_work = nullptr;
    h->work_bytes = 0;
  }
  if (cudaMalloc(&h->d_work, bytes) != cudaSuccess) {
    cudaGetLastError();
    return set_err(B200CHEM_ENOMEM, "cannot allocate %zu bytes of integrator scratch", bytes);
  }
  h->work_bytes = bytes;
  return 0;
}

// Default lanes per cell of the group integrator for n = N+1 components.
int default_group_lanes(int n) { return n <= 16 ? 8 : (n <= 32 ? 16 : 32); }

int launch_group(b200chem_reactor* h, const ReactParams& P, cudaStream_t st) {
  const int lut = h->opts.lu_fp64 ? 8 : 4;
  const int G = h->opts.group_lanes > 0 ? h->opts.group_lanes : default_group_lanes(h->n);
  if (G != 8 && G != 16 && G != 32) return set_err(B200CHEM_EINVAL, "group_lanes must be 8, 16 or 32");
  const GroupVariant* v = nullptr;
  for (int c = (h->n + G - 1) / G; c <= 8 && !v; ++c) v = find_group_variant(G, c, lut);  // next compiled CPL
  if (!v) return set_err(B200CHEM_ETOOBIG, "no group variant for G=%d and n=%d", G, h->n);
  GroupParams Q;
  Q.L = group_layout(h->N, h->R, G, lut);
  const int groups_per_cta = 128 / G;
  const int smem = Q.L.smem_bytes * groups_per_cta;
  if (smem > h->smem_optin - 2048)
    return set_err(B200CHEM_ETOOBIG, "group integrator needs %d B of shared memory per CTA", smem);
  int per_sm = v->occupancy(smem);
  if (per_sm < 1) return set_err(B200CHEM_ETOOBIG, "group kernel does not fit on an SM");
  if (h->opts.ctas_per_sm > 0) per_sm = std::min(per_sm, (int)h->opts.ctas_per_sm);
  const long long need = (P.total + groups_per_cta - 1) / groups_per_cta;
  const long long grid = std::max<long long>(1, std::min<long long>(need, (long long)h->sm_count * per_sm));
  int err = ensure_work(h, (size_t)(grid * groups_per_cta) * (size_t)Q.L.gbytes, st);
  if (err) return err;
  Q.gscratch = static_cast<unsigned char*>(h->d_work);
  CK(v->launch(P, Q, (int)grid, smem, st));
  h->launches++;
  return 0;
}

int launch_thread_per_cell(b200chem_reactor* h, const ReactParams& P, cudaStream_t st) {
  const int lut = h->opts.lu_fp64 ? 8 : 4;
  int per_sm = 0, smem = 0;
  CK(tpc_occupancy(h->N, lut, &per_sm, &smem));
  if (per_sm < 1) return set_err(B200CHEM_ETOOBIG, "thread-per-cell kernel does not fit on an SM");
  if (h->opts.ctas_per_sm > 0) per_sm = std::min(per_sm, (int)h->opts.ctas_per_sm);
  const long long need = (P.total + kTpcBlock - 1) / kTpcBlock;
  const long long grid = std::max<long long>(1, std::min<long long>(need, (long long)h->sm_count * per_sm));
  const long long nthr = grid * kTpcBlock;
  const int n = h->n;
  int err = ensure_work(h, (size_t)nthr * n * n * (sizeof(double) + lut), st);
  if (err) return err;
  TpcParams Q;
  Q.J = static_cast<double*>(h->d_work);
  Q.A = static_cast<void*>(static_cast<double*>(h->d_work) + (size_t)nthr * n * n);
  Q.nthr = nthr;
  Q.setup_ratio = h->opts.setup_ratio > 0 ? h->opts.setup_ratio : 2;
  CK(tpc_launch(h->N, lut, P, Q, (int)grid, smem, st));
  h->launches++;
  return 0;
}

// Cell-state budget of one chunk of the round-based integrator.
constexpr long long kRoundsBudgetBytes = 24LL << 30;
// Default rounds between checks of the live-cell count (one host sync each).
constexpr int kRoundsCheckEvery = 4;

int ensure_buffer(void** p, size_t* have, size_t bytes, cudaStream_t st, const char* what) {
  if (bytes <= *have) return 0;
  if (*p) {
    CK(cudaStreamSynchronize(st));
    cudaFree(*p);
    *p = nullptr;
    *have = 0;
  }
  if (cudaMalloc(p, bytes) != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return set_err(B200CHEM_ENOMEM, "cannot allocate %zu bytes of %s", bytes, what);
  }
  *have = bytes;
  return 0;
}

int tuning_valid(const b200chem_tuning& t) {
  const int32_t per_sm[4] = {t.rhs_ctas_per_sm, t.ctrl_ctas_per_sm, t.jac_ctas_per_sm, t.gj_ctas_per_sm};
  for (int32_t v : per_sm)
    if (v < 0 || v > 64) return 0;
  if (t.rounds_per_check != 0 && t.rounds_per_check != 2 && t.rounds_per_check != 4 && t.rounds_per_check != 8 &&
      t.rounds_per_check != 16)
    return 0;
  if (t.use_graph < 0 || t.use_graph > 2) return 0;
  if (t.rhs_form < 0 || t.rhs_form > 2) return 0;
  return 1;
}

int32_t& tuning_field(b200chem_tuning& t, int field) {
  switch (field) {
    case 0: return t.rhs_ctas_per_sm;
    case 1: return t.ctrl_ctas_per_sm;
    case 2: return t.jac_ctas_per_sm;
    case 3: return t.gj_ctas_per_sm;
    case 4: return t.rounds_per_check;
    case 5: return t.use_graph;
    default: return t.rhs_form;
  }
}

// Grid of one kernel: the occupancy maximum, capped by the tuned CTAs per SM.
int tuned_grid(int max_grid, int sm_count, int per_sm) {
  if (per_sm <= 0) return max_grid;
  return std::max(sm_count, std::min(max_grid, per_sm * sm_count));
}

// One round of the integrator: right-hand sides of the cells in list_in,
// step control (Newton update, error test, next prediction) appending to
// list_out and to the setup list, Jacobian and iteration-matrix inversion of
// the setup list, step control of the cells back from their setup.
constexpr int kProfCountSlots = 1 << 16;

cudaEvent_t prof_event(b200chem_reactor* h) {
  if (h->ev_used == h->ev_pool.size()) {
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
    h->ev_pool.push_back(e);
  }
  return h->ev_pool[h->ev_used++];
}

// One kernel of the round integrator; when the handle profiles, the launch is
// bracketed by two events and the count of the list it processes is copied
// to the host first (stream-ordered, so it is the count the kernel sees).
int launch_kernel(b200chem_reactor* h, int lut, int what, int prof_kind, const RoundsParams& R, const RoundsGrids& G,
                  int after_rhs, const int* cnt, long long host_cells, cudaStream_t st) {
  if (!h->prof_on || h->prof_overflow) {
    CK(rounds_launch(h->N, lut, what, R, G, after_rhs, st));
    return 0;
  }
  b200chem_reactor::ProfRec rec{prof_kind, -1, host_cells, prof_event(h), prof_event(h)};
  if (!rec.e0 || !rec.e1 || (cnt && h->pcnt_used >= kProfCountSlots)) {
    h->prof_overflow = true;
    CK(rounds_launch(h->N, lut, what, R, G, after_rhs, st));
    return 0;
  }
  if (cnt) {
    rec.slot = h->pcnt_used++;
    CK(cudaMemcpyAsync(h->h_pcnt + rec.slot, cnt, sizeof(int), cudaMemcpyDeviceToHost, st));
  }
  CK(cudaEventRecord(rec.e0, st));
  CK(rounds_launch(h->N, lut, what, R, G, after_rhs, st));
  CK(cudaEventRecord(rec.e1, st));
  h->prof.push_back(rec);
  return 0;
}

// The slot lists of one chunk: A and B (cells needing a right-hand side,
// swapped every round), S (cells needing a Newton-matrix setup) and its
// subset SJ (setups that recompute the Jacobian).
struct RoundLists {
  int* lst[2];
  int* cnt[2];
  int* setup;
  int* cnt_setup;
  int* jac;
  int* cnt_jac;
};

int enqueue_round(b200chem_reactor* h, int lut, RoundsParams R, const RoundsGrids& G, const RoundLists& Ls, int cur,
                  cudaStream_t st) {
  R.list_in = Ls.lst[cur];
  R.cnt_in = Ls.cnt[cur];
  R.list_out = Ls.lst[1 - cur];
  R.cnt_out = Ls.cnt[1 - cur];
  R.list_setup = Ls.setup;
  R.cnt_setup = Ls.cnt_setup;
  R.list_jac = Ls.jac;
  R.cnt_jac = Ls.cnt_jac;
  int err = launch_kernel(h, lut, kRoundsRhs, B200CHEM_PROF_RHS, R, G, 0, R.cnt_in, 0, st);
  if (err) return err;
  CK(cudaMemsetAsync(R.cnt_out, 0, sizeof(int), st));
  CK(cudaMemsetAsync(Ls.cnt_setup, 0, sizeof(int), st));
  CK(cudaMemsetAsync(Ls.cnt_jac, 0, sizeof(int), st));
  if ((err = launch_kernel(h, lut, kRoundsCtrl, B200CHEM_PROF_CTRL, R, G, 1, R.cnt_in, 0, st))) return err;
  R.list_in = Ls.jac;
  R.cnt_in = Ls.cnt_jac;
  if ((err = launch_kernel(h, lut, kRoundsJac, B200CHEM_PROF_JAC, R, G, 0, Ls.cnt_jac, 0, st))) return err;
  R.list_in = Ls.setup;
  R.cnt_in = Ls.cnt_setup;
  if ((err = launch_kernel(h, lut, kRoundsGj, B200CHEM_PROF_GJ, R, G, 0, Ls.cnt_setup, 0, st))) return err;
  // cells coming back from a setup always ask for a right-hand side next
  return launch_kernel(h, lut, kRoundsCtrl, B200CHEM_PROF_CTRL_SETUP, R, G, 0, Ls.cnt_setup, 0, st);
}

// Captures `rounds` rounds (an even number: the two slot lists swap roles
// every round, so the graph starts and ends on list A) into h->rgraph,
// updating the executable graph in place when only kernel parameters
// changed.
int capture_rounds(b200chem_reactor* h, int lut, const RoundsParams& R, const RoundsGrids& G, int rounds,
                   const RoundLists& Ls) {
  if (!h->cap_stream) CK(cudaStreamCreateWithFlags(&h->cap_stream, cudaStreamNonBlocking));
  CK(cudaStreamBeginCapture(h->cap_stream, cudaStreamCaptureModeThreadLocal));
  int err = 0;
  for (int r = 0; r < rounds && !err; ++r) err = enqueue_round(h, lut, R, G, Ls, r & 1, h->cap_stream);
  cudaGraph_t g = nullptr;
  const cudaError_t ce = cudaStreamEndCapture(h->cap_stream, &g);
  if (err || ce != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    return err ? err : set_err(B200CHEM_ECUDA, "graph capture of the rounds failed: %s", cudaGetErrorString(ce));
  }
  if (h->rgraph && h->rgraph_rounds == rounds) {
    cudaGraphExecUpdateResultInfo info;
    if (cudaGraphExecUpdate(h->rgraph, g, &info) != cudaSuccess) {
      cudaGetLastError();
      cudaGraphExecDestroy(h->rgraph);
      h->rgraph = nullptr;
    }
  } else if (h->rgraph) {
    cudaGraphExecDestroy(h->rgraph);
    h->rgraph = nullptr;
  }
  cudaError_t ie = cudaSuccess;
  if (!h->rgraph) ie = cudaGraphInstantiate(&h->rgraph, g, 0);
  cudaGraphDestroy(g);
  if (ie != cudaSuccess) {
    h->rgraph = nullptr;
    return set_err(B200CHEM_ECUDA, "cannot instantiate the round graph: %s", cudaGetErrorString(ie));
  }
  h->rgraph_rounds = rounds;
  return 0;
}

// Round-based integrator: rhs / ctrl / setup kernels over compacted lists,
// chunk by chunk (see react_rounds.cu).
int launch_rounds(b200chem_reactor* h, const ReactParams& P, cudaStream_t st, int force_lut = 0) {
  if (!rounds_supported(h->N))
    return set_err(B200CHEM_EINVAL, "round-based integrator not compiled for N=%d", h->N);
  const int lut = force_lut ? force_lut : (h->opts.lu_fp64 ? 8 : 4);
  const RoundsSetupLayout SL = rounds_setup_layout(h->N, h->R, lut);
  if (4 * std::max(SL.jac_smem_per_warp, SL.gj_smem_per_warp) > h->smem_optin - 2048)
    return set_err(B200CHEM_ETOOBIG, "setup kernels need %d B of shared memory per CTA",
                   4 * std::max(SL.jac_smem_per_warp, SL.gj_smem_per_warp));
  if (h->rgrid_lut != lut) {
    CK(rounds_grids_for(h->N, lut, SL, h->sm_count, &h->rgrid));
    h->rgrid_lut = lut;
  }
  const b200chem_tuning& T = h->tune;
  RoundsGrids G = h->rgrid;
  G.rhs = tuned_grid(h->rgrid.rhs, h->sm_count, T.rhs_ctas_per_sm);
  G.ctrl = tuned_grid(h->rgrid.ctrl, h->sm_count, T.ctrl_ctas_per_sm);
  G.jac = tuned_grid(h->rgrid.jac, h->sm_count, T.jac_ctas_per_sm);
  G.gj = tuned_grid(h->rgrid.gj, h->sm_count, T.gj_ctas_per_sm);
  const int per_check = T.rounds_per_check > 0 ? T.rounds_per_check : kRoundsCheckEvery;
  // a profiled call launches kernel by kernel (events between the launches)
  const bool graph = T.use_graph != 2 && !h->prof_on;
  // chunk capacity from the state budget (and the free device memory)
  size_t free_b = 0, total_b = 0;
  CK(cudaMemGetInfo(&free_b, &total_b));
  const long long per_cell = rounds_state_bytes_per_cell(h->N, lut);
  long long budget = std::min<long long>(kRoundsBudgetBytes, (long long)((free_b + h->rounds_bytes) * 0.6));
  long long cap = std::min<long long>(P.total, std::max<long long>(1024, budget / per_cell));
  cap = std::min<long long>(cap, 1LL << 30);
  const size_t state_bytes = (size_t)per_cell * cap + 16 * 256;
  int err = ensure_buffer(&h->d_rounds, &h->rounds_bytes, state_bytes, st, "round-integrator state");
  if (err) return err;
  err = ensure_buffer(&h->d_rwarp, &h->rwarp_bytes, (size_t)h->rgrid.jac * 4 * SL.gbytes_per_warp, st,
                      "setup scratch");
  if (err) return err;
  if (!h->d_rcnt) {
    CK(cudaMalloc(&h->d_rcnt, 4 * sizeof(int)));
    CK(cudaMallocHost(&h->h_rcnt, sizeof(int)));
  }
  RoundsParams R;
  R.P = P;
  R.SL = SL;
  R.S = rounds_carve(h->d_rounds, cap, h->N, lut);
  // the four slot lists follow the cell records
  const size_t rec_bytes = (size_t)R.S.L.stride * cap;
  if (rec_bytes + 16ull * cap > h->rounds_bytes)
    return set_err(B200CHEM_ECUDA, "round-integrator state layout overflows its buffer");
  int* lists = reinterpret_cast<int*>(static_cast<unsigned char*>(h->d_rounds) + rec_bytes);
  RoundLists Ls;
  Ls.lst[0] = lists;
  Ls.lst[1] = lists + cap;
  Ls.setup = lists + 2 * cap;
  Ls.jac = lists + 3 * cap;
  Ls.cnt[0] = h->d_rcnt;
  Ls.cnt[1] = h->d_rcnt + 1;
  Ls.cnt_setup = h->d_rcnt + 2;
  Ls.cnt_jac = h->d_rcnt + 3;
  R.wscratch = static_cast<unsigned char*>(h->d_rwarp);
  // right-hand-side form: generated mechanism code, the constant bank or the
  // global tables
  R.const_mech = (h->cmech_bytes > 0 && T.rhs_form <= 1) ? 1 : 0;
  R.gen_mech = (h->gen_mech && T.rhs_form == 0) ? 1 : 0;
  if (R.const_mech) CK(rounds_upload_const(h->h_cmech, h->cmech_bytes, st));
  const long long max_rounds = 64LL * std::max(1, (int)h->opts.max_steps) + 1024;
  for (long long chunk0 = 0; chunk0 < P.total; chunk0 += cap) {
    R.chunk0 = chunk0;
    R.nchunk = std::min<long long>(cap, P.total - chunk0);
    CK(cudaMemsetAsync(h->d_rcnt, 0, 4 * sizeof(int), st));
    R.list_in = nullptr;
    R.cnt_in = nullptr;
    R.list_out = Ls.lst[0];
    R.cnt_out = Ls.cnt[0];
    R.list_setup = Ls.setup;
    R.cnt_setup = Ls.cnt_setup;
    R.list_jac = Ls.jac;
    R.cnt_jac = Ls.cnt_jac;
    err = launch_kernel(h, lut, kRoundsStart, B200CHEM_PROF_START, R, G, 0, nullptr, R.nchunk, st);
    if (err) return err;
    h->launches++;
    if (graph) {
      err = capture_rounds(h, lut, R, G, per_check, Ls);
      if (err) return err;
    }
    for (long long round = 0;; round += per_check) {
      if (round >= max_rounds) return set_err(B200CHEM_EINTEGRATE, "round-based integrator did not finish");
      if (graph) {
        CK(cudaGraphLaunch(h->rgraph, st));
      } else {
        for (int r = 0; r < per_check; ++r) {
          err = enqueue_round(h, lut, R, G, Ls, r & 1, st);
          if (err) return err;
        }
      }
      h->launches += 5LL * per_check;
      // per_check is even: the live cells are back in list A
      CK(cudaMemcpyAsync(h->h_rcnt, Ls.cnt[0], sizeof(int), cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
      if (*h->h_rcnt == 0) break;
    }
  }
  return 0;
}

int do_react(b200chem_reactor* h, const std::vector<DevBox>& boxes, long long total, double dt, cudaStream_t st,
             int32_t* cell_status, b200chem_stats* stats) {
  const int nbox = (int)boxes.size();
  if (nbox > h->boxes_cap) {
    if (h->stage_pending) CK(cudaEventSynchronize(h->stage_ev));
    h->stage_pending = false;
    if (h->d_boxes) cudaFree(h->d_boxes);
    if (h->h_boxes) cudaFreeHost(h->h_boxes);
    h->d_boxes = nullptr;
    h->h_boxes = nullptr;
    h->boxes_cap = 0;
    const int cap = std::max(nbox, 64);
    CK(cudaMalloc(&h->d_boxes, sizeof(DevBox) * cap));
    CK(cudaMallocHost(&h->h_boxes, sizeof(DevBox) * cap));
    h->boxes_cap = cap;
  }
  if (h->stage_pending) CK(cudaEventSynchronize(h->stage_ev));
  if (nbox > 0) {
    memcpy(h->h_boxes, boxes.data(), sizeof(DevBox) * nbox);
    CK(cudaMemcpyAsync(h->d_boxes, h->h_boxes, sizeof(DevBox) * nbox, cudaMemcpyHostToDevice, st));
    CK(cudaEventRecord(h->stage_ev, st));
    h->stage_pending = true;
  }
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
  P.refine_stall = 0.0;
  P.refine_keep = 0.0;
  P.retry = nullptr;
  P.retry_pass = 0;
  if (h->opts.kernel == 1 && !tpc_supported(h->N))
    return set_err(B200CHEM_EINVAL, "thread-per-cell kernel requested but not compiled for N=%d", h->N);
  if (total > 0) {
    // auto: the round-based integrator where its species count is compiled,
    // else the group integrator (any species count)
    const int k = (h->opts.kernel == 0) ? (rounds_supported(h->N) ? 3 : 2) : h->opts.kernel;
    const int ppm = h->opts.refine_stall_ppm;
    const int keep = h->opts.refine_keep_ppm;
    if (k == 3 && !h->opts.lu_fp64 && keep > 0) P.refine_keep = keep * 1e-6;
    if (k == 3 && !h->opts.lu_fp64 && ppm >= 0) {
      // per-cell FP64 fallback: flags of the cells whose refined FP32 solve stalls
      P.refine_stall = (ppm == 0 ? 250000 : ppm) * 1e-6;
      int err = ensure_buffer(reinterpret_cast<void**>(&h->d_retry), &h->retry_bytes, sizeof(int) * (size_t)total,
                              st, "FP64-retry flags");
      if (err) return err;
      CK(cudaMemsetAsync(h->d_retry, 0, sizeof(int) * (size_t)total, st));
      P.retry = h->d_retry;
    }
    int err = (k == 1) ? launch_thread_per_cell(h, P, st)
              : (k == 3) ? launch_rounds(h, P, st)
                         : launch_group(h, P, st);
    if (err) return err;
    if (P.retry) {
      long long stalled = 0;
      CK(cudaMemcpyAsync(&stalled, P.stats + kStStall, sizeof(long long), cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
      if (stalled > 0) {
        // the flagged cells, from their untouched inputs, with the FP64 LU
        ReactParams Q = P;
        Q.refine_stall = 0.0;
        Q.retry_pass = 1;
        if ((err = launch_rounds(h, Q, st, 8))) return err;
      }
    }
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
    stats->n_fp64_retry = st_h[kStStall];
    if (stats->n_failed > 0) return set_err(B200CHEM_EINTEGRATE, "%lld cell(s) failed to integrate", stats->n_failed);
  }
  return 0;
}

// Copies `bytes` of host data to the device buffer of `b` on stream `st`
// (through the pinned staging buffer) and returns the device pointer.
int stage_to_device(StagedBuf& b, const void* src, size_t bytes, cudaStream_t st, void** out) {
  if (!b.ev) CK(cudaEventCreateWithFlags(&b.ev, cudaEventDisableTiming));
  if (b.pending) CK(cudaEventSynchronize(b.ev));
  b.pending = false;
  if (bytes > b.bytes) {
    if (b.d) cudaFree(b.d);
    if (b.h) cudaFreeHost(b.h);
    b.d = b.h = nullptr;
    b.bytes = 0;
    CK(cudaMalloc(&b.d, bytes));
    CK(cudaMallocHost(&b.h, bytes));
    b.bytes = bytes;
  }
  memcpy(b.h, src, bytes);
  CK(cudaMemcpyAsync(b.d, b.h, bytes, cudaMemcpyHostToDevice, st));
  CK(cudaEventRecord(b.ev, st));
  b.pending = true;
  *out = b.d;
  return 0;
}

void staged_free(StagedBuf& b) {
  if (b.pending) cudaEventSynchronize(b.ev);
  if (b.ev) cudaEventDestroy(b.ev);
  if (b.d) cudaFree(b.d);
  if (b.h) cudaFreeHost(b.h);
  b = StagedBuf{};
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

// shared memory of a 128-thread CTA of the evaluation kernels (one cell per warp)
int eval_smem(const b200chem_reactor* h, GroupLayout* L) {
  *L = group_layout(h->N, h->R, 32, 8);
  return 4 * L->smem_bytes;
}

}  // namespace

// ------------------------------------------------------------------ C ABI
extern "C" {

int b200chem_version(void) { return B200CHEM_VERSION; }
const char* b200chem_last_error(void) { return g_err.c_str(); }

// FNV-1a digest of a mechanism description over its arrays in declaration
// order, as pelelmex_b200.mechgen.mechanism_digest computes it.
static unsigned long long mech_digest(const b200chem_mech_desc* md) {
  const int N = md->n_species, R = md->n_reactions;
  unsigned long long hsh = 0xcbf29ce484222325ull;
  auto fnv = [&](const void* p, size_t bytes) {
    const unsigned char* c = static_cast<const unsigned char*>(p);
    for (size_t i = 0; i < bytes; ++i) {
      hsh ^= c[i];
      hsh *= 0x100000001b3ull;
    }
  };
  const int32_t hdr3[3] = {md->n_species, md->n_reactions, md->n_eff};
  fnv(hdr3, sizeof(hdr3));
  fnv(md->mw, sizeof(double) * N);
  fnv(md->nasa, sizeof(double) * 15 * (size_t)N);
  fnv(md->rtype, sizeof(int32_t) * R);
  fnv(md->rflags, sizeof(int32_t) * R);
  fnv(md->arr, sizeof(double) * 3 * (size_t)R);
  fnv(md->arr_lo, sizeof(double) * 3 * (size_t)R);
  fnv(md->arr_rev, sizeof(double) * 3 * (size_t)R);
  fnv(md->troe, sizeof(double) * 4 * (size_t)R);
  fnv(md->sp, sizeof(int32_t) * 8 * (size_t)R);
  fnv(md->nu, sizeof(int32_t) * 8 * (size_t)R);
  fnv(md->eff_ptr, sizeof(int32_t) * (R + 1));
  fnv(md->eff_sp, sizeof(int32_t) * (size_t)md->n_eff);
  fnv(md->eff_val, sizeof(double) * (size_t)md->n_eff);
  return hsh;
}

uint64_t b200chem_mechanism_digest(const b200chem_mech_desc* md) { return md ? mech_digest(md) : 0; }

int b200chem_generated_species(uint64_t digest) { return rounds_generated_for(digest); }

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
  h->opts = *o;
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
  // a generated right-hand side is used when the description's digest matches
  h->digest = mech_digest(md);
  h->gen_mech = (rounds_generated_for(h->digest) == N) ? 1 : 0;
  // packed constant-memory table of the round integrator's right-hand side
  std::vector<unsigned char> cblob;
  {
    auto al = [](size_t v) { return (v + 15) & ~(size_t)15; };
    CMechHeader hd{};
    hd.N = N;
    hd.R = R;
    hd.n_eff = (int)effsp.size();
    size_t off = al(sizeof(CMechHeader));
    hd.off_nasa = (int)off;
    off = al(off + sizeof(double) * nasa.size());
    hd.off_mw = (int)off;
    off = al(off + sizeof(double) * N);
    hd.off_imw = (int)off;
    off = al(off + sizeof(double) * N);
    hd.off_rxn = (int)off;
    off = al(off + sizeof(RxnC) * (size_t)R);
    hd.off_effsp = (int)off;
    off = al(off + sizeof(short) * std::max<size_t>(effsp.size(), 1));
    hd.off_effm1 = (int)off;
    off = al(off + sizeof(double) * std::max<size_t>(effm1.size(), 1));
    hd.bytes = (int)off;
    if (off <= (size_t)kConstMechBytes && N < 128) {
      cblob.assign(off, 0);
      memcpy(cblob.data(), &hd, sizeof(hd));
      memcpy(cblob.data() + hd.off_nasa, nasa.data(), sizeof(double) * nasa.size());
      memcpy(cblob.data() + hd.off_mw, mw.data(), sizeof(double) * N);
      memcpy(cblob.data() + hd.off_imw, imw.data(), sizeof(double) * N);
      RxnC* rx = reinterpret_cast<RxnC*>(cblob.data() + hd.off_rxn);
      for (int j = 0; j < R; ++j) {
        RxnC r{};
        r.lnA = arr[j];
        r.b = arr[(size_t)R + j];
        r.ea = arr[2 * (size_t)R + j];
        r.lnA0 = arrlo[j];
        r.b0 = arrlo[(size_t)R + j];
        r.ea0 = arrlo[2 * (size_t)R + j];
        r.ta = troe[j];
        r.t3i = troe[(size_t)R + j];
        r.t1i = troe[2 * (size_t)R + j];
        r.t2 = troe[3 * (size_t)R + j];
        r.sdnu = sdnu[j];
        r.lr = arrrev[j];
        r.br = arrrev[(size_t)R + j];
        r.er = arrrev[2 * (size_t)R + j];
        for (int sl = 0; sl < 8; ++sl) {
          r.sp[sl] = (signed char)sp[(size_t)sl * R + j];
          r.nu[sl] = (signed char)nu[(size_t)sl * R + j];
        }
        r.type = (short)rtype[j];
        r.flags = (short)rflags[j];
        r.e0 = (short)effptr[j];
        r.e1 = (short)effptr[j + 1];
        rx[j] = r;
      }
      short* es = reinterpret_cast<short*>(cblob.data() + hd.off_effsp);
      for (size_t q = 0; q < effsp.size(); ++q) es[q] = (short)effsp[q];
      memcpy(cblob.data() + hd.off_effm1, effm1.data(), sizeof(double) * effm1.size());
    }
  }
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
  if ((e = cudaDeviceGetAttribute(&h->smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device)) !=
      cudaSuccess)
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
  if (!cblob.empty()) {
    if ((e = cudaMallocHost(&h->h_cmech, cblob.size())) != cudaSuccess) return fail(e, "cudaMallocHost(table)");
    memcpy(h->h_cmech, cblob.data(), cblob.size());
    h->cmech_bytes = (int)cblob.size();
  }
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

int b200chem_advance_chemistry(b200chem_handle h, const b200chem_chem_box* cboxes, int32_t nbox, double dt,
                               void* stream, int32_t* cell_status, b200chem_stats* stats) {
  if (!h || (!cboxes && nbox > 0) || nbox < 0) return set_err(B200CHEM_EINVAL, "bad arguments");
  if (!(dt > 0.0)) return set_err(B200CHEM_EINVAL, "dt must be positive");
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  std::vector<ChemBoxDev> cb(nbox);
  std::vector<b200chem_box_view> views(nbox);
  long long total = 0;
  for (int b = 0; b < nbox; ++b) {
    const b200chem_chem_box& x = cboxes[b];
    if (!x.rhoY_old.p || !x.rhoH_old.p || !x.T_old.p || !x.rhoY_new.p || !x.rhoH_new.p || !x.T_new.p ||
        !x.extF_rhoY.p || !x.extF_rhoH.p)
      return set_err(B200CHEM_EINVAL, "box %d: null state array", b);
    ChemBoxDev& d = cb[b];
    d.lo0 = x.lo[0];
    d.lo1 = x.lo[1];
    d.lo2 = x.lo[2];
    d.nx = x.hi[0] - x.lo[0] + 1;
    d.ny = x.hi[1] - x.lo[1] + 1;
    d.nz = x.hi[2] - x.lo[2] + 1;
    if (d.nx < 1 || d.ny < 1 || d.nz < 1) return set_err(B200CHEM_EINVAL, "box %d is empty or inverted", b);
    d.off = total;
    total += (long long)d.nx * d.ny * d.nz;
    d.rY_o = to_dev(x.rhoY_old);
    d.rH_o = to_dev(x.rhoH_old);
    d.T_o = to_dev(x.T_old);
    d.rY_n = to_dev(x.rhoY_new);
    d.rH_n = to_dev(x.rhoH_new);
    d.T_n = to_dev(x.T_new);
    d.fY = to_dev(x.extF_rhoY);
    d.fH = to_dev(x.extF_rhoH);
    d.IR = to_dev(x.I_R);
    b200chem_box_view& v = views[b];
    memcpy(v.lo, x.lo, sizeof(v.lo));
    memcpy(v.hi, x.hi, sizeof(v.hi));
    v.rhoY = x.rhoY_new;
    v.extF_rhoY = x.extF_rhoY;
    v.T = x.T_new;
    v.rhoH = x.rhoH_new;
    v.extF_rhoH = x.extF_rhoH;
    v.fctCount = x.fctCount;
    v.mask = x.mask;
  }
  if (total == 0) return 0;
  // covered boxes (advanceChemistryBAChem's m_baChemFlag == 0) react through
  // an all-zero mask: every cell is skipped, keeps its state and gets
  // fctCount = 0 (Source/PeleLMeX_Reactions.cpp:260-289)
  long long zlen = 0;
  for (int b = 0; b < nbox; ++b)
    if (cboxes[b].skip_react) zlen = std::max<long long>(zlen, cboxes[b].hi[0] - cboxes[b].lo[0] + 1);
  if (zlen > h->zero_mask_len) {
    if (h->d_zero_mask) {
      CK(cudaStreamSynchronize(st));
      cudaFree(h->d_zero_mask);
      h->d_zero_mask = nullptr;
      h->zero_mask_len = 0;
    }
    CK(cudaMalloc(&h->d_zero_mask, sizeof(int) * (size_t)zlen));
    CK(cudaMemsetAsync(h->d_zero_mask, 0, sizeof(int) * (size_t)zlen, st));
    h->zero_mask_len = zlen;
  }
  for (int b = 0; b < nbox; ++b) {
    if (!cboxes[b].skip_react) continue;
    b200chem_iarray4& m = views[b].mask;
    m.p = h->d_zero_mask;  // element (i, j, k) -> i - lo[0]: strides 0 across j and k
    m.jstride = m.kstride = m.nstride = 0;
    for (int d = 0; d < 3; ++d) {
      m.lo[d] = cboxes[b].lo[d];
      m.hi[d] = cboxes[b].hi[d];
    }
  }
  void* d_cb = nullptr;
  int err = stage_to_device(h->cboxes, cb.data(), sizeof(ChemBoxDev) * (size_t)nbox, st, &d_cb);
  if (err) return err;
  CK(advance_chem_launch(0, static_cast<const ChemBoxDev*>(d_cb), nbox, total, h->N, 0.0, h->sm_count, st));
  h->launches++;
  double dt_react = dt, time = 0.0;
  err = b200chem_react(h, views.data(), nbox, &dt_react, &time, stream, cell_status, stats);
  if (err && err != B200CHEM_EINTEGRATE) return err;
  CK(advance_chem_launch(1, static_cast<const ChemBoxDev*>(d_cb), nbox, total, h->N, 1.0 / dt, h->sm_count, st));
  h->launches++;
  return err;
}

int b200chem_react_force(b200chem_handle h, const b200chem_force_box* fboxes, int32_t nbox, double dt,
                         void* stream) {
  if (!h || (!fboxes && nbox > 0) || nbox < 0) return set_err(B200CHEM_EINVAL, "bad arguments");
  if (!(dt > 0.0)) return set_err(B200CHEM_EINVAL, "dt must be positive");
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  std::vector<ForceBoxDev> fb(nbox);
  long long total = 0;
  for (int b = 0; b < nbox; ++b) {
    const b200chem_force_box& x = fboxes[b];
    if (!x.rhoY_old.p || !x.rhoH_old.p || !x.rhoY_new.p || !x.rhoH_new.p || !x.I_R.p || !x.extF_rhoY.p ||
        !x.extF_rhoH.p)
      return set_err(B200CHEM_EINVAL, "box %d: null array", b);
    ForceBoxDev& d = fb[b];
    d.lo0 = x.lo[0];
    d.lo1 = x.lo[1];
    d.lo2 = x.lo[2];
    d.nx = x.hi[0] - x.lo[0] + 1;
    d.ny = x.hi[1] - x.lo[1] + 1;
    d.nz = x.hi[2] - x.lo[2] + 1;
    if (d.nx < 1 || d.ny < 1 || d.nz < 1) return set_err(B200CHEM_EINVAL, "box %d is empty or inverted", b);
    d.off = total;
    total += (long long)d.nx * d.ny * d.nz;
    d.rY_o = to_dev(x.rhoY_old);
    d.rH_o = to_dev(x.rhoH_old);
    d.rY_n = to_dev(x.rhoY_new);
    d.rH_n = to_dev(x.rhoH_new);
    d.IR = to_dev(x.I_R);
    d.fY = to_dev(x.extF_rhoY);
    d.fH = to_dev(x.extF_rhoH);
  }
  if (total == 0) return 0;
  void* d_fb = nullptr;
  int err = stage_to_device(h->fboxes, fb.data(), sizeof(ForceBoxDev) * (size_t)nbox, st, &d_fb);
  if (err) return err;
  // 1/dt once on the host, as the reference's dtinv = 1.0 / m_dt
  CK(react_force_launch(static_cast<const ForceBoxDev*>(d_fb), nbox, total, h->N, 1.0 / dt, h->sm_count, st));
  h->launches++;
  return 0;
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

// ------------------------------------------------ allocation-free react
// Fixed device scratch of b200chem_react_flat_noalloc: [0, 256) the work
// queue counter and the statistics slots (must start at zero, cleared by each
// call), [256, 1024) the one box descriptor of the flat call, then the group
// integrator's per-group global scratch (Jacobian and per-reaction
// coefficients, written before they are read).
constexpr size_t kNoAllocScratchBytes = 24u << 20;  // 24 MiB
constexpr size_t kNoAllocBoxOffset = 256;
constexpr size_t kNoAllocWorkOffset = 1024;
static_assert(sizeof(unsigned long long) * (1 + kStCount) <= kNoAllocBoxOffset, "counters overflow their slot");
static_assert(sizeof(DevBox) <= kNoAllocWorkOffset - kNoAllocBoxOffset, "box descriptor overflows its slot");
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mu;
unsigned char* g_noalloc_ptr[kNoAllocMaxDevices] = {};

// Device address of the scratch on the current device, looked up once per
// device (cudaGetSymbolAddress; no allocation).
int noalloc_scratch(int device, unsigned char** out) {
  if (device < 0 || device >= kNoAllocMaxDevices) return set_err(B200CHEM_EINVAL, "device %d out of range", device);
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[device]) {
    void* p = nullptr;
    CK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_noalloc_ptr[device] = static_cast<unsigned char*>(p);
  }
  *out = g_noalloc_ptr[device];
  return 0;
}

// Stores the flat call's box descriptor into the fixed scratch.  The
// descriptor travels as a kernel argument, so no host buffer has to outlive
// the call.
__global__ void noalloc_store_box(DevBox d, DevBox* dst) { *dst = d; }

}  // namespace

extern "C" int b200chem_react_flat_noalloc(b200chem_handle h, double* rhoY, const double* extF_rhoY, double* T,
                                           double* rhoH, const double* extF_rhoH, double* fctCount,
                                           const int32_t* mask, int64_t ncells, double* dt_react, double* time,
                                           void* stream, int32_t* cell_status, b200chem_stats* stats) {
  if (!h || ncells < 0 || !dt_react) return set_err(B200CHEM_EINVAL, "bad arguments");
  if (ncells > 0 && (!rhoY || !extF_rhoY || !T || !rhoH || !extF_rhoH))
    return set_err(B200CHEM_EINVAL, "null state array");
  if (!(*dt_react > 0.0)) return set_err(B200CHEM_EINVAL, "dt_react must be positive");
  if (ncells > 0x7fffffffLL) return set_err(B200CHEM_ETOOBIG, "ncells above 2^31-1 in one flat call");
  if (h->opts.kernel != 0 && h->opts.kernel != 2)
    return set_err(B200CHEM_EINVAL, "the allocation-free react runs the group integrator only (kernel 0 or 2)");
  int dev = -1;
  CK(cudaGetDevice(&dev));
  if (dev != h->device) return set_err(B200CHEM_EINVAL, "current device %d is not the reactor's device %d", dev,
                                       h->device);
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  // integrator variant and launch shape (the group kernel of react_flat)
  const int lut = h->opts.lu_fp64 ? 8 : 4;
  const int G = h->opts.group_lanes > 0 ? h->opts.group_lanes : default_group_lanes(h->n);
  if (G != 8 && G != 16 && G != 32) return set_err(B200CHEM_EINVAL, "group_lanes must be 8, 16 or 32");
  const GroupVariant* v = nullptr;
  for (int c = (h->n + G - 1) / G; c <= 8 && !v; ++c) v = find_group_variant(G, c, lut);
  if (!v) return set_err(B200CHEM_ETOOBIG, "no group variant for G=%d and n=%d", G, h->n);
  GroupParams Q;
  Q.L = group_layout(h->N, h->R, G, lut);
  const int groups_per_cta = 128 / G;
  const int smem = Q.L.smem_bytes * groups_per_cta;
  if (smem > h->smem_optin - 2048)
    return set_err(B200CHEM_ETOOBIG, "group integrator needs %d B of shared memory per CTA", smem);
  int per_sm = v->occupancy(smem);
  if (per_sm < 1) return set_err(B200CHEM_ETOOBIG, "group kernel does not fit on an SM");
  if (h->opts.ctas_per_sm > 0) per_sm = std::min(per_sm, (int)h->opts.ctas_per_sm);
  // the grid is capped by the fixed scratch: at least one CTA per SM must fit
  const long long cta_bytes = (long long)groups_per_cta * Q.L.gbytes;
  const long long cap_ctas = (long long)(kNoAllocScratchBytes - kNoAllocWorkOffset) / cta_bytes;
  if (cap_ctas < h->sm_count)
    return set_err(B200CHEM_ETOOBIG,
                   "allocation-free react needs %lld B of scratch for one CTA per SM (%d SMs x %lld B); the fixed "
                   "scratch holds %zu B",
                   cta_bytes * h->sm_count, h->sm_count, cta_bytes, kNoAllocScratchBytes - kNoAllocWorkOffset);
  const long long rows = std::min<long long>(per_sm, cap_ctas / h->sm_count);
  const long long need = (ncells + groups_per_cta - 1) / groups_per_cta;
  const long long grid = std::max<long long>(1, std::min<long long>(need, (long long)h->sm_count * rows));
  unsigned char* base = nullptr;
  int err = noalloc_scratch(dev, &base);
  if (err) return err;
  unsigned long long* counters = reinterpret_cast<unsigned long long*>(base);
  DevBox* d_box = reinterpret_cast<DevBox*>(base + kNoAllocBoxOffset);
  // queue counter and statistics start at zero
  CK(cudaMemsetAsync(counters, 0, sizeof(unsigned long long) * (1 + kStCount), st));
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
    noalloc_store_box<<<1, 1, 0, st>>>(d, d_box);
    CK(cudaGetLastError());
    h->launches++;
    ReactParams P;
    P.mech = h->mech;
    P.boxes = d_box;
    P.nbox = 1;
    P.total = ncells;
    P.dt = *dt_react;
    P.max_steps = h->opts.max_steps;
    P.qmax = h->opts.max_order;
    P.rtol = h->opts.rtol;
    P.atol = h->d_atol;
    P.queue = counters;
    P.stats = reinterpret_cast<long long*>(counters + 1);
    P.status = cell_status;
    Q.gscratch = base + kNoAllocWorkOffset;
    CK(v->launch(P, Q, (int)grid, smem, st));
    h->launches++;
  }
  if (stats) {
    long long st_h[kStCount];
    CK(cudaMemcpyAsync(st_h, counters + 1, sizeof(st_h), cudaMemcpyDeviceToHost, st));
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
    stats->n_fp64_retry = st_h[kStStall];
    if (time) *time += *dt_react;
    if (stats->n_failed > 0) return set_err(B200CHEM_EINTEGRATE, "%lld cell(s) failed to integrate", stats->n_failed);
    return 0;
  }
  if (time) *time += *dt_react;
  return 0;
}

int64_t b200chem_kernel_launches(b200chem_handle h) { return h ? h->launches : -1; }

int b200chem_profile_begin(b200chem_handle h) {
  if (!h) return set_err(B200CHEM_EINVAL, "bad arguments");
  if (!h->h_pcnt) CK(cudaMallocHost(&h->h_pcnt, sizeof(int) * kProfCountSlots));
  h->prof.clear();
  h->ev_used = 0;
  h->pcnt_used = 0;
  h->prof_overflow = false;
  h->prof_on = true;
  return 0;
}

int b200chem_profile_end(b200chem_handle h, b200chem_kernel_profile* out) {
  if (!h || !out) return set_err(B200CHEM_EINVAL, "bad arguments");
  if (!h->prof_on) return set_err(B200CHEM_EINVAL, "profile_end without profile_begin");
  h->prof_on = false;
  memset(out, 0, sizeof(*out));
  for (const auto& r : h->prof) {
    CK(cudaEventSynchronize(r.e1));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, r.e0, r.e1));
    out->launches[r.kind] += 1;
    out->ms[r.kind] += ms;
    out->cells[r.kind] += (r.slot >= 0) ? h->h_pcnt[r.slot] : r.cells;
  }
  out->complete = h->prof_overflow ? 0 : 1;
  h->prof.clear();
  return 0;
}

int b200chem_get_tuning(b200chem_handle h, b200chem_tuning* t) {
  if (!h || !t) return set_err(B200CHEM_EINVAL, "bad arguments");
  *t = h->tune;
  return 0;
}

int b200chem_set_tuning(b200chem_handle h, const b200chem_tuning* t) {
  if (!h || !t) return set_err(B200CHEM_EINVAL, "bad arguments");
  if (!tuning_valid(*t)) return set_err(B200CHEM_EINVAL, "tuning field out of range");
  h->tune = *t;
  return 0;
}

// Tuning cache file: "B2CHTUNE", u32 version (1), u32 header bytes (128),
// u64 mechanism digest, char[64] GPU name, i32 SM count, i32 reserved, then
// the b200chem_tuning struct.  A launch shape is kept per (mechanism, GPU).
namespace {
constexpr char kTuneMagic[8] = {'B', '2', 'C', 'H', 'T', 'U', 'N', 'E'};
constexpr uint32_t kTuneVersion = 1, kTuneHeader = 128;

struct TuneHeader {
  char magic[8];
  uint32_t version, header_bytes;
  uint64_t digest;
  char gpu[64];
  int32_t sm_count, reserved;
  unsigned char pad[kTuneHeader - 8 - 8 - 8 - 64 - 8];
};
static_assert(sizeof(TuneHeader) == kTuneHeader, "tuning header layout");

int tune_header(b200chem_handle h, TuneHeader* t) {
  memset(t, 0, sizeof(*t));
  memcpy(t->magic, kTuneMagic, 8);
  t->version = kTuneVersion;
  t->header_bytes = kTuneHeader;
  t->digest = h->digest;
  cudaDeviceProp prop;
  CK(cudaGetDeviceProperties(&prop, h->device));
  strncpy(t->gpu, prop.name, sizeof(t->gpu) - 1);  // the name, cut to 63 bytes
  t->sm_count = h->sm_count;
  return 0;
}
}  // namespace

int b200chem_tuning_save(b200chem_handle h, const char* path) {
  if (!h || !path) return set_err(B200CHEM_EINVAL, "bad arguments");
  TuneHeader t;
  int err = tune_header(h, &t);
  if (err) return err;
  FILE* f = fopen(path, "wb");
  if (!f) return set_err(B200CHEM_EINVAL, "cannot write %s", path);
  const bool ok = fwrite(&t, sizeof(t), 1, f) == 1 && fwrite(&h->tune, sizeof(h->tune), 1, f) == 1;
  fclose(f);
  return ok ? 0 : set_err(B200CHEM_EINVAL, "short write to %s", path);
}

int b200chem_tuning_load(b200chem_handle h, const char* path) {
  if (!h || !path) return set_err(B200CHEM_EINVAL, "bad arguments");
  FILE* f = fopen(path, "rb");
  if (!f) return set_err(B200CHEM_EINVAL, "cannot open %s", path);
  TuneHeader t, mine;
  b200chem_tuning tu;
  const bool ok = fread(&t, sizeof(t), 1, f) == 1 && fread(&tu, sizeof(tu), 1, f) == 1;
  fclose(f);
  if (!ok || memcmp(t.magic, kTuneMagic, 8) != 0 || t.version != kTuneVersion || t.header_bytes != kTuneHeader)
    return set_err(B200CHEM_EINVAL, "%s is not a tuning file of this version", path);
  int err = tune_header(h, &mine);
  if (err) return err;
  if (t.digest != mine.digest) return set_err(B200CHEM_EINVAL, "%s was tuned for another mechanism", path);
  if (strncmp(t.gpu, mine.gpu, sizeof(t.gpu)) != 0 || t.sm_count != mine.sm_count)
    return set_err(B200CHEM_EINVAL, "%s was tuned on another GPU (%s)", path, t.gpu);
  if (!tuning_valid(tu)) return set_err(B200CHEM_EINVAL, "%s holds an invalid launch shape", path);
  h->tune = tu;
  return 0;
}

// Autotuner of the round-based integrator's launch shape.  Each trial copies
// the sample into work arrays, runs one react over them between two events
// and reads the elapsed time; coordinate descent over the tuning fields keeps
// a value when it is at least 1% faster than the best so far.
int b200chem_autotune(b200chem_handle h, const double* rhoY, const double* extF_rhoY, const double* T,
                      const double* rhoH, const double* extF_rhoH, int64_t ncells, double dt_react,
                      int32_t max_trials, void* stream, b200chem_tuning* best, double* best_ms) {
  if (!h || ncells <= 0 || !rhoY || !extF_rhoY || !T || !rhoH || !extF_rhoH)
    return set_err(B200CHEM_EINVAL, "bad arguments");
  if (!(dt_react > 0.0)) return set_err(B200CHEM_EINVAL, "dt_react must be positive");
  const int kern = (h->opts.kernel == 0) ? (rounds_supported(h->N) ? 3 : 2) : h->opts.kernel;
  if (kern != 3) return set_err(B200CHEM_EINVAL, "the autotuner tunes the round-based integrator (kernel 0 or 3)");
  if (max_trials <= 0) max_trials = 48;
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int N = h->N;
  const long long n = std::min<long long>(ncells, 1LL << 20);
  // sample arrays: inputs (compact copies) then the work copies react updates
  const size_t nb = sizeof(double) * (size_t)n;
  double* buf = nullptr;
  if (cudaMalloc(&buf, nb * (2 * (size_t)N + 6 + (size_t)N + 1)) != cudaSuccess) {
    cudaGetLastError();
    return set_err(B200CHEM_ENOMEM, "cannot allocate the autotuner sample");
  }
  double* s_rhoY = buf;
  double* s_T = s_rhoY + (size_t)N * n;
  double* s_rhoH = s_T + n;
  double* w_rhoY = s_rhoH + n;
  double* w_T = w_rhoY + (size_t)N * n;
  double* w_rhoH = w_T + n;
  double* w_fct = w_rhoH + n;
  double* s_fY = w_fct + n;
  double* s_fH = s_fY + (size_t)N * n;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int err = 0;
  auto cleanup = [&]() {
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(buf);
  };
  auto ck = [&](cudaError_t e) {
    if (e != cudaSuccess && !err) err = set_err(B200CHEM_ECUDA, "CUDA error in the autotuner: %s", cudaGetErrorString(e));
    return err;
  };
  const size_t src_pitch = sizeof(double) * (size_t)ncells;
  if (ck(cudaMemcpy2DAsync(s_rhoY, nb, rhoY, src_pitch, nb, N, cudaMemcpyDeviceToDevice, st)) ||
      ck(cudaMemcpy2DAsync(s_fY, nb, extF_rhoY, src_pitch, nb, N, cudaMemcpyDeviceToDevice, st)) ||
      ck(cudaMemcpyAsync(s_T, T, nb, cudaMemcpyDeviceToDevice, st)) ||
      ck(cudaMemcpyAsync(s_rhoH, rhoH, nb, cudaMemcpyDeviceToDevice, st)) ||
      ck(cudaMemcpyAsync(s_fH, extF_rhoH, nb, cudaMemcpyDeviceToDevice, st)) || ck(cudaEventCreate(&e0)) ||
      ck(cudaEventCreate(&e1))) {
    cleanup();
    return err;
  }
  const b200chem_tuning saved = h->tune;
  int trials = 0;
  // one timed react of the sample under tuning t; +inf when the shape fails
  auto trial = [&](const b200chem_tuning& t, double* ms) -> int {
    *ms = 1e300;
    h->tune = t;
    if (ck(cudaMemcpyAsync(w_rhoY, s_rhoY, nb * N, cudaMemcpyDeviceToDevice, st)) ||
        ck(cudaMemcpyAsync(w_T, s_T, nb, cudaMemcpyDeviceToDevice, st)) ||
        ck(cudaMemcpyAsync(w_rhoH, s_rhoH, nb, cudaMemcpyDeviceToDevice, st)) ||
        ck(cudaMemsetAsync(w_fct, 0, nb, st)) || ck(cudaEventRecord(e0, st)))
      return err;
    double dt = dt_react;
    const int rc = b200chem_react_flat(h, w_rhoY, s_fY, w_T, w_rhoH, s_fH, w_fct, nullptr, n, &dt, nullptr, st,
                                       nullptr, nullptr);
    ++trials;
    if (ck(cudaEventRecord(e1, st)) || ck(cudaEventSynchronize(e1))) return err;
    if (rc != 0) return 0;  // shape rejected: stays at +inf
    float f = 0.f;
    if (ck(cudaEventElapsedTime(&f, e0, e1))) return err;
    *ms = f;
    return 0;
  };
  b200chem_tuning cur = saved;
  double cur_ms = 1e300, m = 0;
  // warm-up (allocations, graph instantiation), then the starting point
  if (trial(cur, &m) || trial(cur, &cur_ms)) {
    h->tune = saved;
    cleanup();
    return err;
  }
  if (!(cur_ms < 1e300)) {
    h->tune = saved;
    cleanup();
    return set_err(B200CHEM_EINTEGRATE, "react of the autotuner sample failed under the starting launch shape");
  }
  const int sm = h->sm_count;
  const int max_per_sm[4] = {std::max(1, h->rgrid.rhs / sm), std::max(1, h->rgrid.ctrl / sm),
                             std::max(1, h->rgrid.jac / sm), std::max(1, h->rgrid.gj / sm)};
  for (int pass = 0; pass < 2 && !err && trials < max_trials; ++pass) {
    for (int field = 0; field < 7 && !err && trials < max_trials; ++field) {
      std::vector<int32_t> cand;
      if (field < 4) {
        cand.push_back(0);
        for (int v = 1; v < max_per_sm[field]; v *= 2) cand.push_back(v);
      } else if (field == 4) {
        cand = {2, 4, 8, 16};
      } else if (field == 5) {
        cand = {1, 2};
      } else {
        if (h->gen_mech) cand.push_back(0);
        if (h->cmech_bytes > 0) cand.push_back(1);
        cand.push_back(2);
      }
      // the value the current shape effectively uses for this field
      int32_t now = tuning_field(cur, field);
      if (field == 4 && now == 0) now = kRoundsCheckEvery;
      if (field == 5 && now == 0) now = 1;
      if (field == 6 && now == 0 && !h->gen_mech) now = h->cmech_bytes > 0 ? 1 : 2;
      if (field == 6 && now == 1 && h->cmech_bytes == 0) now = 2;
      for (int32_t v : cand) {
        if (v == now || trials >= max_trials) continue;
        b200chem_tuning t = cur;
        tuning_field(t, field) = v;
        double ms = 0;
        if (trial(t, &ms)) break;
        if (ms < 0.99 * cur_ms) {
          cur = t;
          cur_ms = ms;
          now = v;
        }
      }
    }
  }
  if (err) {
    h->tune = saved;
    cleanup();
    return err;
  }
  h->tune = cur;
  if (best) *best = cur;
  if (best_ms) *best_ms = cur_ms;
  cleanup();
  return 0;
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
  if (h->d_work) cudaFree(h->d_work);
  if (h->d_rounds) cudaFree(h->d_rounds);
  if (h->d_rwarp) cudaFree(h->d_rwarp);
  if (h->d_rcnt) cudaFree(h->d_rcnt);
  if (h->h_rcnt) cudaFreeHost(h->h_rcnt);
  if (h->h_cmech) cudaFreeHost(h->h_cmech);
  if (h->rgraph) cudaGraphExecDestroy(h->rgraph);
  staged_free(h->cboxes);
  staged_free(h->fboxes);
  if (h->d_zero_mask) cudaFree(h->d_zero_mask);
  if (h->d_retry) cudaFree(h->d_retry);
  for (cudaEvent_t e : h->ev_pool) cudaEventDestroy(e);
  if (h->h_pcnt) cudaFreeHost(h->h_pcnt);
  if (h->cap_stream) cudaStreamDestroy(h->cap_stream);
  delete h;
  return 0;
}

static int eval_launch(b200chem_handle h, const double* y, const double* F, int64_t ncells, double* out, void* stream,
                       int what) {
  if (!h || !y || !F || !out || ncells < 0) return set_err(B200CHEM_EINVAL, "bad arguments");
  if (ncells == 0) return 0;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  EvalParams P;
  P.mech = h->mech;
  P.y = y;
  P.F = F;
  P.out = out;
  P.ncells = ncells;
  P.what = what;
  const int smem = eval_smem(h, &P.L);
  const long long grid = std::min<long long>((ncells + 3) / 4, (long long)h->sm_count * 8);
  int err = ensure_work(h, (size_t)(grid * 4) * (size_t)P.L.gbytes, st);
  if (err) return err;
  P.gscratch = static_cast<unsigned char*>(h->d_work);
  if (h->n <= 32) {
    CK(cudaFuncSetAttribute(eval_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    eval_kernel<1><<<(unsigned)grid, 128, smem, st>>>(P);
  } else {
    CK(cudaFuncSetAttribute(eval_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    eval_kernel<2><<<(unsigned)grid, 128, smem, st>>>(P);
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
  const int smem = eval_smem(h, &P.L);
  const long long grid = std::min<long long>((ncells + 3) / 4, (long long)h->sm_count * 16);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (h->n <= 32) {
    CK(cudaFuncSetAttribute(inst_rr_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    inst_rr_kernel<1><<<(unsigned)grid, 128, smem, st>>>(P);
  } else {
    CK(cudaFuncSetAttribute(inst_rr_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    inst_rr_kernel<2><<<(unsigned)grid, 128, smem, st>>>(P);
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

static int thermo_launch(b200chem_handle h, const double* T, const double* IR, double* Hi, double* HR, int64_t ncells,
                         void* stream) {
  if (!h || !T || ncells < 0) return set_err(B200CHEM_EINVAL, "bad arguments");
  if (ncells == 0) return 0;
  const long long grid = std::min<long long>((ncells + 255) / 256, (long long)h->sm_count * 8);
  thermo_hr_kernel<<<(unsigned)grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(h->mech, T, IR, Hi, HR, ncells);
  CK(cudaGetLastError());
  h->launches++;
  return 0;
}

int b200chem_h_given_t(b200chem_handle h, const double* T, double* Hi_mks, int64_t ncells, void* stream) {
  if (!Hi_mks) return set_err(B200CHEM_EINVAL, "null output");
  return thermo_launch(h, T, nullptr, Hi_mks, nullptr, ncells, stream);
}

int b200chem_heat_release(b200chem_handle h, const double* T, const double* I_R_mks, double* HR_mks, int64_t ncells,
                          void* stream) {
  if (!I_R_mks || !HR_mks) return set_err(B200CHEM_EINVAL, "null array");
  return thermo_launch(h, T, I_R_mks, nullptr, HR_mks, ncells, stream);
}

}  // extern "C"

namespace b200 {
const GroupVariant* group_variants_g8(int* count);
const GroupVariant* group_variants_g16(int* count);
const GroupVariant* group_variants_g32(int* count);

const GroupVariant* find_group_variant(int G, int CPL, int lut_bytes) {
  int cnt = 0;
  const GroupVariant* v = G == 8    ? group_variants_g8(&cnt)
                          : G == 16 ? group_variants_g16(&cnt)
                          : G == 32 ? group_variants_g32(&cnt)
                                    : nullptr;
  for (int i = 0; v && i < cnt; ++i)
    if (v[i].CPL == CPL && v[i].lut_bytes == lut_bytes) return &v[i];
  return nullptr;
}
}  // namespace b200
