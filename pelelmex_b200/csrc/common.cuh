// common.cuh -- data shared by the react kernels and the host code: box
// views (amrex::Array4 mirrors), launch parameters, statistics slots, and the
// per-group memory layout of the group integrator.
#pragma once
#include <cuda_runtime.h>

#include "../../include/b200chem.h"
#include "bdf_group.cuh"
#include "bdf_rounds.cuh"

namespace b200 {

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

// One box of the advanceChemistry body (advance_chem.cu): old state,
// new state, forcing and the reaction term, MKS.
struct ChemBoxDev {
  int lo0, lo1, lo2, nx, ny, nz;
  long long off;
  DevArr rY_o, rH_o, T_o, rY_n, rH_n, T_n, fY, fH, IR;
};
// phase 0: MKS -> CGS prologue; 1: CGS -> MKS epilogue and I_R
cudaError_t advance_chem_launch(int phase, const ChemBoxDev* d_boxes, int nbox, long long total, int N,
                                double dt_inv, int sm_count, cudaStream_t st);

// One box of getScalarReactForce (advance_chem.cu), MKS.
struct ForceBoxDev {
  int lo0, lo1, lo2, nx, ny, nz;
  long long off;
  DevArr rY_o, rH_o, rY_n, rH_n, IR, fY, fH;
};
cudaError_t react_force_launch(const ForceBoxDev* d_boxes, int nbox, long long total, int N, double dt_inv,
                               int sm_count, cudaStream_t st);

// stats slots in the scratch buffer (after the queue counter)
enum { kStCells = 0, kStMasked, kStFailed, kStNst, kStNfe, kStNje, kStNlu, kStNetf, kStNcfn, kStMaxNfe,
       kStMaxNst, kStStall, kStCount };

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
  // round-based integrator, FP32 inverse: a Newton correction whose FP64
  // refinement step is larger than refine_stall times the correction itself
  // (the FP32 inverse does not resolve the iteration matrix) stops the cell
  // untouched and flags it in retry[cell] for a pass with the FP64 LU
  // (refine_stall <= 0: no check); retry_pass = 1 integrates only the
  // flagged cells
  double refine_stall = 0.0;
  // > 0: a Newton correction skips the FP64 refinement when the first
  // correction with the same matrix measured the FP32 solve accurate to this
  double refine_keep = 0.0;
  int* retry = nullptr;
  int retry_pass = 0;
};

__device__ __forceinline__ double* elem(const DevArr& a, int i, int j, int k) {
  return a.p + (long long)(i - a.lo0) + (long long)(j - a.lo1) * a.js + (long long)(k - a.lo2) * a.ks;
}


// Per-group layout.  Shared: C, gRT, hRT, atol, Dsc, bvec [Npad] (double),
// q [Rpad] (double), inverse [n][ldl] (LUT), fcol [Npad] (LUT), ipiv [n] (int).
// Global: Jacobian [n][ldj] (column-major) and r1..r4 [Rpad] (double).
struct GroupLayout {
  int Npad, Rpad, n, ldj, ldl;
  int smem_bytes;    // per group
  long long gbytes;  // per group, global scratch
};

__host__ __device__ inline GroupLayout group_layout(int N, int R, int G, int lut_bytes) {
  GroupLayout L;
  L.n = N + 1;
  L.Npad = ((L.n + G - 1) / G) * G;
  L.Rpad = ((R + 31) / 32) * 32;
  if (L.Rpad < 32) L.Rpad = 32;
  L.ldj = L.n | 1;
  L.ldl = L.n | 1;
  long long b = 8LL * (6 * L.Npad + L.Rpad);
  b += (long long)lut_bytes * ((long long)L.n * L.ldl + L.Npad);
  b += 4LL * L.Npad;
  L.smem_bytes = (int)((b + 15) & ~15LL);
  L.gbytes = 8LL * ((long long)L.n * L.ldj + 4LL * L.Rpad);
  L.gbytes = (L.gbytes + 255) & ~255LL;
  return L;
}

struct GroupParams {
  GroupLayout L;
  unsigned char* gscratch;  // [groups in launch][L.gbytes]
};

// Host-side entry points of one compiled group-kernel variant.
struct GroupVariant {
  int G, CPL, lut_bytes;
  // resident CTAs per SM for a block of 128 threads and `smem` bytes, or -1
  int (*occupancy)(int smem);
  cudaError_t (*launch)(const ReactParams& P, const GroupParams& Q, int grid, int smem, cudaStream_t st);
};

// Variants compiled in react_g*.cu; returns nullptr if (G, CPL, lut) has none.
const GroupVariant* find_group_variant(int G, int CPL, int lut_bytes);

struct TpcParams {
  double* J;        // [n*n][threads] FP64 Jacobians, interleaved by thread
  void* A;          // [n*n][threads] LU factors (float or double), interleaved
  long long nthr;   // threads in the launch (interleave stride)
  int setup_ratio;  // setup round when waiting * ratio >= needing an RHS
};

constexpr int kTpcBlock = 128;

// Thread-per-cell kernels (react_tpc.cu): species counts with a variant.
bool tpc_supported(int N);
cudaError_t tpc_occupancy(int N, int lut_bytes, int* per_sm, int* smem);
cudaError_t tpc_launch(int N, int lut_bytes, const ReactParams& P, const TpcParams& Q, int grid, int smem,
                       cudaStream_t st);

// ------------------------------------------------------ round-based path
constexpr int kRoundsRhsBlock = 64;  // threads per CTA of the rhs kernel
enum { kRoundsStart = 0, kRoundsRhs, kRoundsCtrl, kRoundsJac, kRoundsGj };

// Per-warp shared scratch of the setup kernels.  Jacobian kernel: C, g/RT,
// h/RT, third-body row [Npad] and the Jacobian [n][n] (double).
// Inverse kernel: Dsc [Npad] (double), matrix [n][ldl] and pivot column
// [Npad] (LUT), two index arrays [Npad] (int).
struct RoundsSetupLayout {
  int Npad, Rpad, ldl;
  int jac_smem_per_warp, gj_smem_per_warp;
  long long gbytes_per_warp;
};

struct RoundsParams {
  ReactParams P;
  rounds::RState S;
  RoundsSetupLayout SL;
  long long chunk0;  // first cell of the chunk (index into the react call's cells)
  long long nchunk;  // cells in the chunk
  const int* list_in;
  const int* cnt_in;
  int* list_out;     // cells that need a right-hand side next round
  int* cnt_out;
  int* list_setup;   // cells that need a Newton-matrix setup this round
  int* cnt_setup;
  int* list_jac;     // the subset of list_setup whose Jacobian is recomputed
  int* cnt_jac;
  unsigned char* wscratch;  // [setup warps][SL.gbytes_per_warp]
  int const_mech;           // 1: the packed table is in the constant bank
  int gen_mech;             // 1: the mechanism has a generated right-hand side
};

struct RoundsGrids {
  int start, rhs, ctrl, jac, gj;
};

// Handle accessors (defined with the handle in b200chem.cu).
const DevMech* handle_mech(b200chem_handle h);
int handle_species(b200chem_handle h);
const double* handle_atol(b200chem_handle h);
int handle_device(b200chem_handle h);
void handle_count_launch(b200chem_handle h);
int handle_set_error(int code, const char* msg);
unsigned long long handle_digest(b200chem_handle h);  // FNV-1a digest of the mechanism description
int handle_sm_count(b200chem_handle h);

bool rounds_supported(int N);
RoundsSetupLayout rounds_setup_layout(int N, int R, int lut_bytes);
long long rounds_state_bytes_per_cell(int N, int lut_bytes);
rounds::RState rounds_carve(void* base, long long cap, int N, int lut_bytes);
cudaError_t rounds_grids_for(int N, int lut_bytes, const RoundsSetupLayout& SL, int sm_count, RoundsGrids* G);
cudaError_t rounds_launch(int N, int lut_bytes, int what, const RoundsParams& R, const RoundsGrids& G, int after_rhs,
                          cudaStream_t st);

// ------------------------------------------- packed constant-memory table
// The round integrator's right-hand side reads the mechanism from constant
// memory (all lanes of a warp read the same reaction at the same time, which
// the constant cache serves as one broadcast): one record per reaction plus
// the species data.  Byte offsets are from the start of the blob.
struct CMechHeader {
  int N, R, n_eff, pad;
  int off_nasa, off_mw, off_imw, off_rxn, off_effsp, off_effm1, bytes, pad2;
};
struct RxnC {
  double lnA, b, ea;        // forward (high-pressure limit for falloff): ln A, b, Ea/R
  double lnA0, b0, ea0;     // low-pressure limit (falloff)
  double ta, t3i, t1i, t2;  // Troe: alpha, 1/T***, 1/T*, T**
  double sdnu;              // net stoichiometric change
  double lr, br, er;        // explicit reverse Arrhenius
  signed char sp[8];        // slots: reactants 0..3, products 4..7 (-1 empty)
  signed char nu[8];        // signed stoichiometry of each slot
  short type, flags, e0, e1;  // kind, flag bits, third-body efficiency range
};
static_assert(sizeof(RxnC) == 136, "packed reaction record");
constexpr int kConstMechBytes = 60 * 1024;

// Species count of the generated right-hand side whose mechanism digest
// matches (0: none).
int rounds_generated_for(unsigned long long digest);

// Upload a packed table to the round integrator's constant bank on `st`.
cudaError_t rounds_upload_const(const void* blob, int bytes, cudaStream_t st);

}  // namespace b200
