/*
 * b200chem.h -- C ABI of the B200 (sm_100a) constant-pressure stiff-chemistry
 * reactor.  It replaces, for one GPU, the per-cell HP reaction advance that
 * PeleLMeX drives through pele::physics::reactions::ReactorBase:
 *
 *   ReactorBase::create(name)        Source/PeleLMeX_Setup.cpp:152-153
 *   ReactorBase::init(type, ncells)  Source/PeleLMeX_Setup.cpp:146-154
 *   ReactorBase::set_typ_vals_ode(v) Source/PeleLMeX_Utils.cpp:1472
 *   ReactorBase::react(box, ...)     Source/PeleLMeX_Reactions.cpp:101-108,267-274
 *   ReactorBase::close()             Source/PeleLMeX.cpp:26
 *
 * Plain C types only: pointers, sizes, and a cudaStream_t passed as void*.
 * All state arrays are DEVICE pointers in CGS units (the caller converts from
 * MKS exactly as Source/PeleLMeX_Reactions.cpp:69-79 does).  Every entry point
 * returns 0 on success and a negative B200CHEM_E* code on failure; the text of
 * the last error of the calling thread is available from b200chem_last_error().
 */
#ifndef B200CHEM_H
#define B200CHEM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define B200CHEM_VERSION 3

/* ---------------------------------------------------------------- errors */
#define B200CHEM_OK 0
#define B200CHEM_EINVAL (-1)     /* bad argument                              */
#define B200CHEM_ECUDA (-2)      /* a CUDA runtime call failed                */
#define B200CHEM_ENOMEM (-3)     /* device allocation failed                  */
#define B200CHEM_EINTEGRATE (-4) /* at least one cell failed to integrate     */
#define B200CHEM_ETOOBIG (-5)    /* size above a compiled-in limit            */

/* ------------------------------------------------------- per-cell status */
#define B200CHEM_CELL_OK 0
#define B200CHEM_CELL_MASKED 1        /* mask == 0: left untouched, fctCount=0  */
#define B200CHEM_CELL_MAXSTEPS (-1)   /* cvode.max_substeps exceeded            */
#define B200CHEM_CELL_ERRFAIL (-2)    /* repeated error-test failures / h_min   */
#define B200CHEM_CELL_CONVFAIL (-3)   /* repeated Newton failures / h_min       */
#define B200CHEM_CELL_NONFINITE (-4)  /* NaN/Inf or non-positive rho or T input */
#define B200CHEM_CELL_SINGULAR (-5)   /* iteration matrix singular repeatedly   */

/* ------------------------------------------------------------ mechanism
 * Flat description of a gas-phase kinetics mechanism in the Chemkin formalism
 * (CGS-mol-K).  Produced from a mechanism file by pelelmex_b200.mechanism.
 * This is the data that a CEPTR-generated mechanism.cpp bakes into code
 * (productionRate, aJacobian, ckhms/ckcpms; reached from PeleLMeX through
 * eos.RTY2WDOT / eos.T2Hi / eos.HY2T, Source/PeleLMeX_K.H:611,721,880-885). */
#define B200CHEM_MAX_SLOTS 4 /* distinct species on one side of a reaction */

#define B200CHEM_RXN_ELEMENTARY 0
#define B200CHEM_RXN_THREEBODY 1
#define B200CHEM_RXN_LINDEMANN 2
#define B200CHEM_RXN_TROE 3

#define B200CHEM_RXN_REVERSIBLE 1   /* reverse rate from equilibrium constant */
#define B200CHEM_RXN_EXPLICIT_REV 2 /* reverse rate from arr_rev              */
#define B200CHEM_RXN_TROE_T2 4      /* Troe form carries the T** term         */

typedef struct b200chem_mech_desc {
  int32_t n_species;
  int32_t n_reactions;
  int32_t n_eff;          /* number of non-default third-body efficiencies */
  const double* mw;       /* [N] molecular weight, g/mol */
  const double* nasa;     /* [N][15] Tmid, low-range a1..a7, high-range a1..a7 */
  const int32_t* rtype;   /* [R] B200CHEM_RXN_* kind */
  const int32_t* rflags;  /* [R] B200CHEM_RXN_* flag bits */
  const double* arr;      /* [R][3] ln A, b, Ea/R (high-pressure limit for falloff) */
  const double* arr_lo;   /* [R][3] low-pressure limit (falloff kinds only) */
  const double* arr_rev;  /* [R][3] explicit reverse Arrhenius (flag EXPLICIT_REV) */
  const double* troe;     /* [R][4] alpha, T***, T*, T** */
  const int32_t* sp;      /* [R][8] reactant slots 0..3, product slots 4..7; -1 = empty */
  const int32_t* nu;      /* [R][8] stoichiometric coefficient of each slot (>0) */
  const int32_t* eff_ptr; /* [R+1] CSR offsets into eff_sp / eff_val */
  const int32_t* eff_sp;  /* [n_eff] species index of a non-default efficiency */
  const double* eff_val;  /* [n_eff] its efficiency (all other species: 1) */
} b200chem_mech_desc;

/* --------------------------------------------------------------- options
 * ode.rtol, ode.atol, cvode.max_order, cvode.max_substeps keep the meaning
 * given in Docs/sphinx/manual/LMeXControls.rst:301-310. */
typedef struct b200chem_opts {
  double rtol;           /* relative tolerance                                  */
  double atol;           /* absolute tolerance, or prefactor on typical values  */
  int32_t max_order;     /* BDF maximum order, 1..5                             */
  int32_t max_steps;     /* maximum internal steps per cell and call            */
  int32_t reactor_type;  /* 2 = HP (constant pressure, enthalpy forcing); only 2 */
  int32_t lu_fp64;       /* 0: FP32 LU + one FP64 refinement step (default); 1: FP64 LU */
  int32_t refine_stall_ppm; /* round-based integrator with the FP32 inverse: a
                            Newton correction whose FP64 refinement step is
                            larger (in the WRMS norm) than this many parts per
                            million of the correction (the FP32 inverse does
                            not resolve the iteration matrix) stops its cell,
                            untouched, and the cell is integrated again from
                            its input by a pass with the FP64 LU in the same
                            react call; 0 = default (250000, a quarter),
                            negative = never                                  */
  int32_t verbose;
  int32_t kernel;        /* 0: auto (round-based integrator where the species
                            count has a compiled variant, else the group
                            integrator); 1: thread-per-cell (compiled species
                            counts only); 2: group integrator (any species
                            count); 3: round-based integrator (rhs / ctrl /
                            setup kernels over compacted cell lists; compiled
                            species counts only).  The round-based integrator
                            keeps the mechanism's reaction table in a constant
                            bank shared by every handle of the process on a
                            device: react calls of handles with DIFFERENT
                            mechanisms must not overlap in time.              */
  int32_t setup_ratio;   /* thread-per-cell: a warp runs a Jacobian/LU round when
                            (cells waiting) * setup_ratio >= (cells needing an
                            RHS); 0 = default (2)                                */
  int32_t ctas_per_sm;   /* resident CTAs per SM (0 = as many as fit); fewer
                            keeps the per-cell scratch in L2                  */
  int32_t group_lanes;   /* group integrator: lanes per cell, 8, 16 or 32
                            (0 = default for the mechanism size)              */
  int32_t refine_keep_ppm; /* round-based integrator with the FP32 inverse,
                            > 0: the first Newton correction after each setup
                            is refined in FP64, which measures how accurate
                            the FP32 solve is for that matrix (WRMS of the
                            refinement step over the correction); the later
                            corrections with the same matrix skip the
                            refinement (and the Jacobian it reads) while that
                            measure is at most this many parts per million.
                            Faster (flame_ch4 128^3: 1.2x), but the unrefined
                            corrections (~5e-8 relative) flip some step
                            decisions against an FP64 solve: a few cells in
                            10^4 then differ from the dense-direct result by
                            more than 1e-8 in Y.  0 (default) or negative:
                            refine every correction                           */
  int32_t reserved;      /* 0                                                 */
} b200chem_opts;

/* ---------------------------------------------------------- Array4 views
 * Mirrors amrex::Array4<Real>: element (i,j,k,n) lives at
 *   p[(i-lo[0]) + (j-lo[1])*jstride + (k-lo[2])*kstride + n*nstride].     */
typedef struct b200chem_array4 {
  double* p;
  int64_t jstride, kstride, nstride;
  int32_t lo[3], hi[3];
} b200chem_array4;

typedef struct b200chem_iarray4 {
  const int32_t* p;
  int64_t jstride, kstride, nstride;
  int32_t lo[3], hi[3];
} b200chem_iarray4;

/* One call of react(box, rhoY, extF_rhoY, T, rhoH, extF_rhoH, fctCount, mask,
 * ...) from Source/PeleLMeX_Reactions.cpp:101-108.  lo/hi (inclusive) is the
 * box to advance; the Array4 boxes may be larger (ghost cells). */
typedef struct b200chem_box_view {
  int32_t lo[3], hi[3];
  b200chem_array4 rhoY;      /* N comps, in/out, g/cm^3                 */
  b200chem_array4 extF_rhoY; /* N comps, in, g/cm^3/s                   */
  b200chem_array4 T;         /* 1 comp,  in/out, K                       */
  b200chem_array4 rhoH;      /* 1 comp,  in/out, erg/cm^3                */
  b200chem_array4 extF_rhoH; /* 1 comp,  in, erg/cm^3/s                  */
  b200chem_array4 fctCount;  /* 1 comp,  out, RHS evaluations per cell   */
  b200chem_iarray4 mask;     /* 1 comp,  in, 0 = skip; p may be NULL     */
} b200chem_box_view;

/* Aggregate counters of one react call (sums over integrated cells). */
typedef struct b200chem_stats {
  int64_t n_cells, n_masked, n_failed;
  int64_t nst, nfe, nje, nlu, netf, ncfn;
  int32_t max_nfe, max_nst;
  int64_t n_fp64_retry; /* cells integrated again with the FP64 LU (refine_stall_ppm) */
} b200chem_stats;

typedef struct b200chem_reactor* b200chem_handle;

/* -------------------------------------------------------------- lifecycle */

/* ReactorBase::create + init (Source/PeleLMeX_Setup.cpp:146-154).  Copies the
 * mechanism to the current device.  Returns NULL on failure. */
b200chem_handle b200chem_create(const b200chem_mech_desc* mech, const b200chem_opts* opts);

/* ReactorBase::set_typ_vals_ode (Source/PeleLMeX_Utils.cpp:1472).  n must be
 * N+1 (species in CGS, then T).  Afterwards atol_k = opts.atol * typ_k;
 * before the first call atol_k = opts.atol for every component. */
int b200chem_set_typvals(b200chem_handle h, const double* typ, int32_t n);

/* ReactorBase::react (call site Source/PeleLMeX_Reactions.cpp:101-108).
 * Advances every unmasked cell of every box by *dt_react, in place, on
 * `stream` (a cudaStream_t, NULL = legacy default stream).  *time is advanced
 * by *dt_react.  cell_status (device, optional) receives one int32 per cell in
 * box order (box 0 cells with i fastest, then box 1, ...).  stats (host,
 * optional) makes the call synchronous and fills the counters.  Returns
 * B200CHEM_EINTEGRATE when stats is given and a cell failed. */
int b200chem_react(b200chem_handle h, const b200chem_box_view* boxes, int32_t nbox,
                   double* dt_react, double* time, void* stream, int32_t* cell_status,
                   b200chem_stats* stats);

/* The flat-array form of react (ReactorBase::react(rY, rYsrc, rX, rX_src, dt,
 * time, ncells, stream) in PelePhysics): component-major arrays of ncells
 * cells, i.e. rhoY[n*ncells + c].  fctCount may be NULL. */
int b200chem_react_flat(b200chem_handle h, double* rhoY, const double* extF_rhoY, double* T,
                        double* rhoH, const double* extF_rhoH, double* fctCount,
                        const int32_t* mask, int64_t ncells, double* dt_react, double* time,
                        void* stream, int32_t* cell_status, b200chem_stats* stats);

/* Allocation-free form of b200chem_react_flat: same arguments, and the
 * results of b200chem_react_flat with opts.kernel = 2 (the group integrator).
 * No reference counterpart: PelePhysics has no allocation-free react.  It
 * calls no cudaMalloc/cudaFree or other allocating routine: its scratch is a
 * fixed 24 MiB device array of the library, whose address is looked up once
 * per device (cudaGetSymbolAddress) on the first call on that device -- make
 * that first call before any stream capture.  It runs the group integrator
 * (opts.kernel 0 or 2; other values give B200CHEM_EINVAL) with the grid
 * capped to fit the fixed scratch, and
 * returns B200CHEM_ETOOBIG when one CTA per SM of the mechanism's integrator
 * scratch does not fit.  The scratch is shared by all handles on a device:
 * calls that overlap in time (other streams, other host threads) race on it
 * and must be serialised by the caller. */
int b200chem_react_flat_noalloc(b200chem_handle h, double* rhoY, const double* extF_rhoY, double* T,
                                double* rhoH, const double* extF_rhoH, double* fctCount,
                                const int32_t* mask, int64_t ncells, double* dt_react, double* time,
                                void* stream, int32_t* cell_status, b200chem_stats* stats);

/* ------------------------------------------------ advanceChemistry body
 * One box of PeleLM::advanceChemistry(lev, dt, extForcing)
 * (Source/PeleLMeX_Reactions.cpp:31-175) around react, in MKS units like
 * the caller's MultiFabs: new <- old converted to CGS (:68-79), react with
 * dt_react = dt and time = 0 (:97-108), the new state and the forcing back to
 * MKS (:111-120), and the reaction term I_R = -(rhoY_old - rhoY_new) / dt -
 * extF_rhoY (:153-160).  extF_rhoY / extF_rhoH are scaled in place and back,
 * as the reference does.  All boxes of the list go through one prologue
 * launch, one react and one epilogue launch.
 *
 * skip_react != 0 is the covered-box branch of advanceChemistryBAChem
 * (Source/PeleLMeX_Reactions.cpp:260-289, m_baChemFlag == 0): the box goes
 * through the unit conversions and gets I_R, but is not reacted; its cells
 * keep their state, get fctCount = 0 and status B200CHEM_CELL_MASKED, and
 * count as masked in the statistics.  Zero (the value of a zero-initialised
 * struct) reacts the box, as advanceChemistry does. */
typedef struct b200chem_chem_box {
  int32_t lo[3], hi[3];
  b200chem_array4 rhoY_old;  /* N comps, in,  kg/m^3                      */
  b200chem_array4 rhoH_old;  /* 1 comp,  in,  J/m^3                       */
  b200chem_array4 T_old;     /* 1 comp,  in,  K                           */
  b200chem_array4 rhoY_new;  /* N comps, out, kg/m^3                      */
  b200chem_array4 rhoH_new;  /* 1 comp,  out, J/m^3                       */
  b200chem_array4 T_new;     /* 1 comp,  out, K                           */
  b200chem_array4 extF_rhoY; /* N comps, in (scaled and restored), kg/m^3/s */
  b200chem_array4 extF_rhoH; /* 1 comp,  in (scaled and restored), J/m^3/s  */
  b200chem_array4 fctCount;  /* 1 comp,  out (p may be NULL)              */
  b200chem_iarray4 mask;     /* 1 comp,  in, 0 = skip (p may be NULL)     */
  b200chem_array4 I_R;       /* N comps, out, kg/m^3/s (p may be NULL)    */
  int32_t skip_react;        /* != 0: covered box, not reacted (BAChem)   */
  int32_t reserved;
} b200chem_chem_box;

int b200chem_advance_chemistry(b200chem_handle h, const b200chem_chem_box* boxes, int32_t nbox, double dt,
                               void* stream, int32_t* cell_status, b200chem_stats* stats);

/* ------------------------------------------------ chemistry forcing
 * PeleLM::getScalarReactForce (Source/PeleLMeX_Reactions.cpp:437-475), MKS:
 * the external forcing of the next react from the advection-diffusion
 * update of this step,
 *   extF_rhoY_k = (rhoY_new_k - rhoY_old_k) * (1/dt) - I_R_k
 *   extF_rhoH   = (rhoH_new - rhoH_old) * (1/dt)
 * with 1/dt rounded once on the host and every product and difference
 * rounded separately, as the reference writes it.  All boxes in one launch. */
typedef struct b200chem_force_box {
  int32_t lo[3], hi[3];
  b200chem_array4 rhoY_old;  /* N comps, in,  kg/m^3    (state at t^n)            */
  b200chem_array4 rhoH_old;  /* 1 comp,  in,  J/m^3                               */
  b200chem_array4 rhoY_new;  /* N comps, in,  kg/m^3    (advection-diffusion state) */
  b200chem_array4 rhoH_new;  /* 1 comp,  in,  J/m^3                               */
  b200chem_array4 I_R;       /* N comps, in,  kg/m^3/s  (last reaction term)       */
  b200chem_array4 extF_rhoY; /* N comps, out, kg/m^3/s                            */
  b200chem_array4 extF_rhoH; /* 1 comp,  out, J/m^3/s                             */
} b200chem_force_box;

int b200chem_react_force(b200chem_handle h, const b200chem_force_box* boxes, int32_t nbox, double dt, void* stream);

/* 64-bit FNV-1a digest of a mechanism description (its arrays in
 * declaration order), and the species count of the generated right-hand
 * side built into the library for that digest (0: none; react then reads
 * the mechanism from the constant bank or global tables).  Host only. */
uint64_t b200chem_mechanism_digest(const b200chem_mech_desc* md);
int b200chem_generated_species(uint64_t digest);

/* ReactorBase::close (Source/PeleLMeX.cpp:26). */
int b200chem_destroy(b200chem_handle h);

/* Number of kernels this handle has launched so far (instrumentation; no
 * reference counterpart).  -1 for a NULL handle. */
int64_t b200chem_kernel_launches(b200chem_handle h);

/* ------------------------------------------------------- launch tuning
 * Launch shape of the round-based integrator (opts.kernel 0 or 3).  No
 * reference counterpart: the reference's GPU reactors fix their launch
 * shape at compile time.  Zero fields take the defaults. */
typedef struct b200chem_tuning {
  int32_t rhs_ctas_per_sm;   /* CTAs per SM of the right-hand-side kernel (0: as many as fit) */
  int32_t ctrl_ctas_per_sm;  /* ... of the step-control / Newton kernel                      */
  int32_t jac_ctas_per_sm;   /* ... of the Jacobian kernel                                   */
  int32_t gj_ctas_per_sm;    /* ... of the iteration-matrix inversion kernel                 */
  int32_t rounds_per_check;  /* rounds between two reads of the live-cell count: 2, 4, 8
                                or 16 (0: 4)                                                 */
  int32_t use_graph;         /* 1: the rounds between two checks are replayed from one
                                captured CUDA graph; 2: launched one by one (0: 1)          */
  int32_t rhs_form;          /* 0: generated mechanism code when it matches, else the
                                constant bank, else global tables; 1: constant bank (or
                                global tables); 2: global tables                             */
  int32_t reserved;
} b200chem_tuning;

/* Current launch shape (the defaults until set). */
int b200chem_get_tuning(b200chem_handle h, b200chem_tuning* t);
/* Sets the launch shape used by later react calls; B200CHEM_EINVAL for
 * values outside the ranges above. */
int b200chem_set_tuning(b200chem_handle h, const b200chem_tuning* t);

/* Autotuner: times react on a copy of the given cells (flat layout of
 * b200chem_react_flat, at most 2^20 cells are used; the inputs are NOT
 * modified) under candidate launch shapes, by coordinate descent over the
 * fields of b200chem_tuning, keeps the fastest shape in the handle and
 * returns it in best (may be NULL).  *best_ms receives the time of one react
 * call of the sample under that shape (may be NULL).  max_trials bounds the
 * number of timed react calls (0: 48). */
int b200chem_autotune(b200chem_handle h, const double* rhoY, const double* extF_rhoY, const double* T,
                      const double* rhoH, const double* extF_rhoH, int64_t ncells, double dt_react,
                      int32_t max_trials, void* stream, b200chem_tuning* best, double* best_ms);

/* Launch-shape cache: writes the handle's tuning to `path` with a header
 * holding the mechanism digest and the GPU's name and SM count; load sets the
 * handle's tuning from such a file and fails (B200CHEM_EINVAL, the reason in
 * b200chem_last_error) when it was made for another mechanism or GPU. */
int b200chem_tuning_save(b200chem_handle h, const char* path);
int b200chem_tuning_load(b200chem_handle h, const char* path);

/* Failure detection self-test (no reference counterpart): launches one
 * thread that waits, with the bounded polling loop of the tensor-core
 * kernels, on an mbarrier nothing arrives at; after `polls` polls (1..2^22)
 * it sets *err (device int) to 1 and returns, leaving the context usable. */
int b200chem_selftest_bounded_wait(int* err, int polls, void* stream);

/* ---------------------------------------------------- kernel profile
 * Per-kernel CUDA-event timing of the round-based integrator (no reference
 * counterpart).  Between profile_begin and profile_end every react call
 * launches its kernels one by one (no graph replay), each bracketed by two
 * events, and records how many cells each launch processed. */
enum {
  B200CHEM_PROF_START = 0,       /* rk_start: load, validate, initialise   */
  B200CHEM_PROF_RHS = 1,         /* rk_rhs: right-hand sides               */
  B200CHEM_PROF_CTRL = 2,        /* rk_ctrl after the right-hand sides     */
  B200CHEM_PROF_JAC = 3,         /* rk_jac: analytic Jacobians             */
  B200CHEM_PROF_GJ = 4,          /* rk_gj: Newton-matrix inverses          */
  B200CHEM_PROF_CTRL_SETUP = 5,  /* rk_ctrl after a setup                  */
  B200CHEM_PROF_KINDS = 8
};
typedef struct b200chem_kernel_profile {
  int64_t launches[B200CHEM_PROF_KINDS];
  int64_t cells[B200CHEM_PROF_KINDS];  /* list entries processed, summed over launches */
  double ms[B200CHEM_PROF_KINDS];      /* summed event time of the launches           */
  int32_t complete;                    /* 0: more launches than the record holds      */
  int32_t reserved;
} b200chem_kernel_profile;

int b200chem_profile_begin(b200chem_handle h);
int b200chem_profile_end(b200chem_handle h, b200chem_kernel_profile* out);

const char* b200chem_last_error(void);
int b200chem_version(void);

/* ------------------------------------------------- mechanism evaluation
 * Device-side evaluations of the mechanism interface used inside react, for
 * parity tests and for callers that need them alone.  Cell-major layouts:
 * y[c*(N+1) + k] holds rhoY_k (k<N) then T; forcing likewise (extF_rhoY then
 * extF_rhoH). */

/* HP right-hand side: d(rhoY_k)/dt = W_k wdot_k + F_k and the temperature
 * equation dT/dt = (F_H - sum_k h_k d(rhoY_k)/dt) / (rho cp). */
int b200chem_eval_rhs(b200chem_handle h, const double* y, const double* forcing, int64_t ncells,
                      double* ydot, void* stream);

/* Analytic Jacobian d(ydot)/dy of the same system, jac[c*(N+1)^2 + i*(N+1) + j]. */
int b200chem_eval_jac(b200chem_handle h, const double* y, const double* forcing, int64_t ncells,
                      double* jac, void* stream);

/* reactionRateRhoY (Source/PeleLMeX_K.H:850-889) in MKS like the caller:
 * rho from sum rhoY, T from (h, Y) by Newton starting at T, then the mass
 * production rates.  Component-major arrays of ncells cells; T is updated to
 * the value consistent with rhoH. */
int b200chem_inst_rr(b200chem_handle h, const double* rhoY_mks, const double* rhoH_mks,
                     double* T, double* rhoYdot_mks, int64_t ncells, void* stream);

/* getTfromHY (Source/PeleLMeX_K.H:700-723) in MKS: T from rho, rhoY, rhoH. */
int b200chem_t_from_hy(b200chem_handle h, const double* rhoY_mks, const double* rhoH_mks,
                       double* T, int64_t ncells, void* stream);

/* getHGivenT (Source/PeleLMeX_K.H:598-615): species enthalpies h_k(T) in
 * J/kg, component-major Hi[k * ncells + c]. */
int b200chem_h_given_t(b200chem_handle h, const double* T, double* Hi_mks, int64_t ncells, void* stream);

/* getHeatRelease (Source/PeleLMeX_Reactions.cpp:477-506): heat release rate
 * HRR = -sum_k h_k(T) I_R,k in W/m^3, from T and the reaction term I_R
 * (kg/m^3/s, component-major, as b200chem_advance_chemistry writes it). */
int b200chem_heat_release(b200chem_handle h, const double* T, const double* I_R_mks, double* HR_mks,
                          int64_t ncells, void* stream);

/* ------------------------------------------------------- surrogate MLP
 * No reference counterpart: the learned part of the reactor (a small MLP
 * predicting the state change over dt_react, with residual-gated fallback to
 * the BDF integrator).  BF16 tensor-core GEMM with fused epilogue:
 *   C[M][N] = epi(A[M][K] . B[N][K]^T + bias[N])
 * A, B: device BF16, row-major, K contiguous, 16-byte aligned rows (lda, ldb
 * multiples of 8); M % 128 == 0, N % 16 == 0 (N <= 256 or N % 256 == 0),
 * K % 16 == 0.  epi: 0 C fp32; 1 C bf16; 2 C bf16 = gelu(.), aux fp32 =
 * pre-activation (aux may be NULL); 3 C bf16 = (A.B^T) * gelu'(aux).  Only
 * columns < n_valid (0 = N) of C are written.  *err (device int, optional)
 * is set to 1 if a tensor-core completion wait timed out.
 *
 * Two-term BF16 operands (flags OR-ed into epi): a value v is carried as
 * hi = bf16(v) and lo = bf16(v - hi), about 16 significant bits, and the
 * products are accumulated in FP32.  B200CHEM_GEMM_SPLIT_A: A has 2K columns,
 * [hi | lo], both multiplied by the same B (lda >= 2K; needs K <= 256, N <= 256
 * and K <= 64 or K % 64 == 0).  B200CHEM_GEMM_SPLIT_OUT (epi 1 or 2, N <= 256):
 * C is written as [hi | lo] (columns c and c + N; ldc >= 2N), and the
 * pre-activations of epi 2 go to aux with row stride N. */
#define B200CHEM_GEMM_SPLIT_OUT 0x10
#define B200CHEM_GEMM_SPLIT_A 0x20
int b200chem_mlp_gemm_bf16(const void* A, long long lda, const void* B, long long ldb, int M, int N, int K,
                           void* C, long long ldc, const float* bias, float* aux, int epi, int n_valid, int* err,
                           void* stream);

/* Fused Adam step (Kingma & Ba 2015) of one FP32 parameter tensor [rows][cols]
 * of the network, step = 1, 2, ... (bias corrections), in place on p, m, v
 * with gradient g; then writes the BF16 copies the GEMMs read: wb [rows][cols]
 * and wbt [cols][rows] (each may be NULL).  All device pointers. */
int b200chem_mlp_adam(float* p, const float* g, float* m, float* v, int rows, int cols, float lr, float beta1,
                      float beta2, float eps, int step, void* wb, void* wbt, void* stream);

/* ----------------------------------------------------- hybrid reactor
 * No reference counterpart: the surrogate-first react.  An ensemble of
 * networks predicts every cell's change over dt_react; a prediction is
 * accepted only when the acceptance rule below holds, and the accepted state
 * is corrected to conserve the element totals and the energy exactly (a
 * state the correction leaves more than 1e-13 off a constraint, relative to
 * the atom content or to sum_k |h_k rhoY_k|, is rejected and counted in
 * rejected_elements); the other cells are integrated by the BDF of
 * b200chem_react_flat.
 *
 * Weights file (b200chem_surrogate_load), little endian:
 *   header (header_bytes, >= 128):
 *     0  char[8]  "B2CHSURR"           8  u32 version (1)   12 u32 header_bytes
 *     16 u64 mechanism digest (b200chem_mechanism_digest of the description
 *        the networks were trained for; loading for another mechanism fails)
 *     24 i32[12] N, N + 2, N + 1, hidden (256), in (N + 2 padded to 16),
 *        out (N + 1 padded to 16), members (1..16), terms (1 or 2), dtype (1:
 *        BF16 weights, FP32 biases), min_members, n_elements (0..8), 0
 *     72 f64[7] the acceptance rule it was calibrated for: t_rel, spread,
 *        dT_cap, gap, tol_elem, tol_mass, resid
 *   body: xmean, xstd [N + 2] f32; ymean, ystd [N + 1] f32; s [N + 1] f64
 *   (asinh scales); elem [n_elements][N] f64 (atoms per species); then per
 *   member W0 [256][in] bf16, b0 [256] f32, W1, b1, W2, b2 ([256][256] bf16,
 *   [256] f32), W3 [out][256] bf16, b3 [out] f32.
 * A member maps x = (T, log10(Y_k + 1e-20), log10 dt), standardised, through
 * three GELU layers to u; the change is dy_j = s_j sinh(u_j ystd_j + ymean_j)
 * (dT, then dY_k). */
typedef struct b200chem_hybrid_opts {
  double t_rel;    /* relative T error allowed to an accepted cell: a "bar" is t_rel * T1 */
  double spread;   /* max |dT_member - dT_mean|, in bars                                 */
  double dT_cap;   /* max |dT_mean|, in bars                                              */
  double gap;      /* max |T(h1, Y_pred) - T1| before the energy projection, in bars      */
  double tol_elem; /* raw element-conservation error, relative to the atom content       */
  double tol_mass; /* raw mass-conservation error, relative; also the most negative
                      partial density tolerated (then clipped)                            */
  double resid;    /* > 0: |T1 - T0 - dt/2 (f_T(y0) + f_T(y1))| bound in bars (two RHS)  */
  int32_t min_members; /* fewer members in the surrogate than this: EINVAL                */
  int32_t reserved;
} b200chem_hybrid_opts;

typedef struct b200chem_hybrid_stats {
  int64_t predicted, accepted;
  int64_t rejected_spread, rejected_cap, rejected_mass, rejected_elements, rejected_energy, rejected_negative,
      rejected_residual, rejected_nonfinite;
} b200chem_hybrid_stats;

typedef struct b200chem_surrogate* b200chem_surrogate_handle;

/* Loads an ensemble (the weights file above, from memory or from a path) to
 * the reactor's device, which must be current.  NULL on failure (message in
 * b200chem_last_error).  A surrogate owns its inference and fallback scratch
 * (allocated on first use, grown as needed): calls with the same surrogate
 * must not overlap in time. */
b200chem_surrogate_handle b200chem_surrogate_load(b200chem_handle h, const void* data, size_t nbytes);
b200chem_surrogate_handle b200chem_surrogate_load_file(b200chem_handle h, const char* path);
/* The acceptance rule stored in the file. */
int b200chem_surrogate_get_opts(b200chem_surrogate_handle s, b200chem_hybrid_opts* o);
int b200chem_surrogate_destroy(b200chem_surrogate_handle s);

/* Ensemble prediction for ncells cells (component-major CGS rhoY [N][ncells],
 * T [ncells]): dy_mean [ncells][N + 1] (dT, dY_k; FP64) and, optionally,
 * dT_spread [ncells], the largest deviation of a member's dT from the mean.
 * Synchronous. */
int b200chem_surrogate_infer(b200chem_surrogate_handle s, const double* rhoY, const double* T, int64_t ncells,
                             double dt, double* dy_mean, double* dT_spread, void* stream);

/* Surrogate-first form of b200chem_react_flat (same arrays and in-place
 * semantics; mask == 0 cells untouched with fctCount 0).  opts NULL uses the
 * rule stored in the weights file.  Accepted cells get fctCount = 0 (2 with
 * the residual check) and status OK; the others carry the BDF's results.
 * Reads the rejected count back to the host once per call.  stats and hstats
 * (host, optional): BDF counters of the rejected cells (n_cells counts every
 * integrated cell) and the gate's counts. */
int b200chem_react_hybrid(b200chem_handle h, b200chem_surrogate_handle s, const b200chem_hybrid_opts* opts,
                          double* rhoY, const double* extF_rhoY, double* T, double* rhoH, const double* extF_rhoH,
                          double* fctCount, const int32_t* mask, int64_t ncells, double* dt_react, double* time,
                          void* stream, int32_t* cell_status, b200chem_stats* stats, b200chem_hybrid_stats* hstats);

/* Surrogate-first form of b200chem_react (box views with ghost cells, call
 * site Source/PeleLMeX_Reactions.cpp:101-108): the boxes' cells are packed
 * into the surrogate's flat arrays, reacted by b200chem_react_hybrid and
 * written back.  cell_status in box order as for b200chem_react. */
int b200chem_react_hybrid_boxes(b200chem_handle h, b200chem_surrogate_handle s, const b200chem_hybrid_opts* opts,
                                const b200chem_box_view* boxes, int32_t nbox, double* dt_react, double* time,
                                void* stream, int32_t* cell_status, b200chem_stats* stats,
                                b200chem_hybrid_stats* hstats);

#ifdef __cplusplus
}
#endif
#endif /* B200CHEM_H */
