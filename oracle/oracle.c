/*
 * oracle.c -- CPU FP64 restatement of the reference's dense-direct CVODE
 * reactor.  TEST INFRASTRUCTURE: only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py may load or run this code, and only as the
 * checker / the timed CPU baseline.  The product (pelelmex_b200/csrc) never
 * links it.
 *
 * What it restates (the reference's own implementation -- PelePhysics
 * ReactorCvode with cvode.solve_type = denseAJ_direct, SUNDIALS CVODE and the
 * CEPTR mechanism -- is absent from the snapshot, so this follows the
 * published methods and the call sites that remain):
 *   - the HP reaction ODE with piecewise-constant forcing,
 *       Docs/sphinx/manual/Model.rst:300-311, units/in-place semantics of
 *       Source/PeleLMeX_Reactions.cpp:69-120, T carried as a state variable:
 *       d(rhoY_k)/dt = W_k wdot_k + F_k,
 *       dT/dt = (F_H - sum_k h_k d(rhoY_k)/dt) / (sum_k rhoY_k cp_k);
 *   - Chemkin-formalism kinetics (mass action, Arrhenius, third bodies,
 *     Lindemann/Troe falloff, reverse rates from Kc of NASA-7 Gibbs
 *     energies), i.e. what productionRate / RTY2WDOT evaluate
 *     (Source/PeleLMeX_K.H:880-885), and its analytic Jacobian (aJacobian);
 *   - CVODE's variable-order (1..5) variable-step BDF in Nordsieck form with
 *     the WRMS local error test, modified Newton on M = I - gamma J with the
 *     CVODE Jacobian/setup reuse heuristics and dense LU with partial
 *     pivoting (Hindmarsh et al., ACM TOMS 31(3) 2005; CVODE math chapter).
 *     Tolerances follow Docs/sphinx/manual/LMeXControls.rst:301-310:
 *     ewt_i = 1/(rtol |y_i| + atol_i), atol_i = ode.atol * typ_i when typical
 *     values are set (Source/PeleLMeX_Utils.cpp:1445-1475).
 * Parity status: UNPINNED against the reference (no reference output exists
 * for this boundary); cross-checked against scipy's BDF and Radau
 * integrators (tests/golden) and a finite-difference Jacobian.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/b200chem.h"

#define R_CGS 8.31446261815324e7
#define P_ATM 1013250.0
#define LN10 2.302585092994046

/* ------------------------------------------------------------ mechanism */
typedef struct orc_mech {
  int N, R;
  double* mw;
  double* nasa;   /* [N][15] */
  int* rtype;
  int* rflags;
  double* arr;    /* [R][3] */
  double* arr_lo; /* [R][3] */
  double* arr_rev;
  double* troe;   /* [R][4] */
  int* sp;        /* [R][8] */
  int* nu;        /* [R][8] */
  double* eff;    /* [R][N] dense efficiencies (1 default) */
  double* dnu;    /* [R][N] net stoichiometry, products - reactants */
  double* sdnu;   /* [R] sum of net stoichiometry */
} orc_mech;

static void* xdup(const void* p, size_t n) {
  void* q = malloc(n ? n : 1);
  if (n) memcpy(q, p, n);
  return q;
}

orc_mech* orc_mech_new(const b200chem_mech_desc* d) {
  orc_mech* m = (orc_mech*)calloc(1, sizeof(orc_mech));
  int N = d->n_species, R = d->n_reactions;
  m->N = N;
  m->R = R;
  m->mw = xdup(d->mw, sizeof(double) * N);
  m->nasa = xdup(d->nasa, sizeof(double) * N * 15);
  m->rtype = xdup(d->rtype, sizeof(int) * R);
  m->rflags = xdup(d->rflags, sizeof(int) * R);
  m->arr = xdup(d->arr, sizeof(double) * R * 3);
  m->arr_lo = xdup(d->arr_lo, sizeof(double) * R * 3);
  m->arr_rev = xdup(d->arr_rev, sizeof(double) * R * 3);
  m->troe = xdup(d->troe, sizeof(double) * R * 4);
  m->sp = xdup(d->sp, sizeof(int) * R * 8);
  m->nu = xdup(d->nu, sizeof(int) * R * 8);
  m->eff = (double*)malloc(sizeof(double) * R * N);
  m->dnu = (double*)calloc((size_t)R * N, sizeof(double));
  m->sdnu = (double*)calloc(R, sizeof(double));
  for (int j = 0; j < R; ++j) {
    for (int k = 0; k < N; ++k) m->eff[j * N + k] = 1.0;
    for (int e = d->eff_ptr[j]; e < d->eff_ptr[j + 1]; ++e) m->eff[j * N + d->eff_sp[e]] = d->eff_val[e];
    for (int s = 0; s < 8; ++s) {
      int k = m->sp[j * 8 + s];
      if (k < 0) continue;
      double v = (double)m->nu[j * 8 + s] * (s < 4 ? -1.0 : 1.0);
      m->dnu[j * N + k] += v;
      m->sdnu[j] += v;
    }
  }
  return m;
}

void orc_mech_free(orc_mech* m) {
  if (!m) return;
  free(m->mw); free(m->nasa); free(m->rtype); free(m->rflags); free(m->arr); free(m->arr_lo);
  free(m->arr_rev); free(m->troe); free(m->sp); free(m->nu); free(m->eff); free(m->dnu); free(m->sdnu);
  free(m);
}

int orc_n_species(const orc_mech* m) { return m->N; }

/* NASA-7: cp/R, h/RT, s/R, and d(cp/R)/dT for species k at T */
static void nasa_eval(const orc_mech* m, int k, double T, double* cpR, double* hRT, double* sR,
                      double* dcpR) {
  const double* c = m->nasa + 15 * k;
  const double* a = (T < c[0]) ? c + 1 : c + 8;
  *cpR = a[0] + T * (a[1] + T * (a[2] + T * (a[3] + T * a[4])));
  *hRT = a[0] + T * (a[1] / 2 + T * (a[2] / 3 + T * (a[3] / 4 + T * a[4] / 5))) + a[5] / T;
  *sR = a[0] * log(T) + T * (a[1] + T * (a[2] / 2 + T * (a[3] / 3 + T * a[4] / 4))) + a[6];
  *dcpR = a[1] + T * (2 * a[2] + T * (3 * a[3] + T * 4 * a[4]));
}

/* Work arrays for one cell. */
typedef struct orc_kin_work {
  double *C, *cpR, *hRT, *gRT, *dcpR;
  double *kf, *kr, *pf, *pr, *M, *q, *Pr, *F, *dlogF_dlogPr, *logFc, *f1, *nn, *cc;
  double *dkf_dM, *dq_dT;
} orc_kin_work;

static void kin_work_alloc(orc_kin_work* w, int N, int R) {
  double* p = (double*)calloc((size_t)5 * N + (size_t)15 * R, sizeof(double));
  w->C = p; p += N; w->cpR = p; p += N; w->hRT = p; p += N; w->gRT = p; p += N; w->dcpR = p; p += N;
  w->kf = p; p += R; w->kr = p; p += R; w->pf = p; p += R; w->pr = p; p += R; w->M = p; p += R;
  w->q = p; p += R; w->Pr = p; p += R; w->F = p; p += R; w->dlogF_dlogPr = p; p += R;
  w->logFc = p; p += R; w->f1 = p; p += R; w->nn = p; p += R; w->cc = p; p += R;
  w->dkf_dM = p; p += R; w->dq_dT = p; p += R;
}

static void kin_work_free(orc_kin_work* w) { free(w->C); }

static inline double ipow(double x, int n) {
  double r = 1.0;
  for (int i = 0; i < n; ++i) r *= x;
  return r;
}

/* Rates of progress q_j and everything the Jacobian needs, at (T, C). */
static void kinetics(const orc_mech* m, double T, orc_kin_work* w, int want_jac) {
  const int N = m->N, R = m->R;
  const double lnT = log(T), invT = 1.0 / T;
  for (int k = 0; k < N; ++k) {
    double sR;
    nasa_eval(m, k, T, &w->cpR[k], &w->hRT[k], &sR, &w->dcpR[k]);
    w->gRT[k] = w->hRT[k] - sR;
  }
  double Ctot = 0.0;
  for (int k = 0; k < N; ++k) Ctot += w->C[k];
  const double lnPRT = log(P_ATM / (R_CGS * T));
  for (int j = 0; j < R; ++j) {
    const double* a = m->arr + 3 * j;
    double kf = exp(a[0] + a[1] * lnT - a[2] * invT);
    int type = m->rtype[j];
    double M = 0.0;
    if (type != B200CHEM_RXN_ELEMENTARY) {
      for (int k = 0; k < N; ++k) M += m->eff[j * N + k] * w->C[k];
    }
    w->M[j] = M;
    w->Pr[j] = 0.0;
    w->F[j] = 1.0;
    w->dlogF_dlogPr[j] = 0.0;
    w->dkf_dM[j] = 0.0;
    if (type == B200CHEM_RXN_LINDEMANN || type == B200CHEM_RXN_TROE) {
      const double* b = m->arr_lo + 3 * j;
      double k0 = exp(b[0] + b[1] * lnT - b[2] * invT);
      double Pr = k0 * M / kf;
      double F = 1.0, D = 0.0;
      if (type == B200CHEM_RXN_TROE) {
        const double* t = m->troe + 4 * j;
        double Fc = (1.0 - t[0]) * exp(-T / t[1]) + t[0] * exp(-T / t[2]);
        if (m->rflags[j] & B200CHEM_RXN_TROE_T2) Fc += exp(-t[3] * invT);
        double logFc = log10(fmax(Fc, 1e-300));
        double c = -0.4 - 0.67 * logFc, nn = 0.75 - 1.27 * logFc;
        double logPr = log10(fmax(Pr, 1e-300));
        double u = logPr + c;
        double den = nn - 0.14 * u;
        double f1 = u / den;
        double logF = logFc / (1.0 + f1 * f1);
        F = pow(10.0, logF);
        D = -2.0 * logFc * f1 * nn / ((1.0 + f1 * f1) * (1.0 + f1 * f1) * den * den);
        if (Pr <= 1e-300) D = 0.0;
        w->logFc[j] = logFc; w->f1[j] = f1; w->nn[j] = nn; w->cc[j] = c;
      }
      w->Pr[j] = Pr;
      w->F[j] = F;
      w->dlogF_dlogPr[j] = D;
      w->dkf_dM[j] = k0 * F * (1.0 / ((1.0 + Pr) * (1.0 + Pr)) + D / (1.0 + Pr));
      kf = kf * Pr / (1.0 + Pr) * F;
    }
    double kr = 0.0;
    if (m->rflags[j] & B200CHEM_RXN_EXPLICIT_REV) {
      const double* r = m->arr_rev + 3 * j;
      kr = exp(r[0] + r[1] * lnT - r[2] * invT);
    } else if (m->rflags[j] & B200CHEM_RXN_REVERSIBLE) {
      double sg = 0.0;
      for (int s = 0; s < 8; ++s) {
        int k = m->sp[j * 8 + s];
        if (k >= 0) sg += (s < 4 ? -1.0 : 1.0) * m->nu[j * 8 + s] * w->gRT[k];
      }
      double lnKc = -sg + m->sdnu[j] * lnPRT;
      kr = kf * exp(-lnKc);
    }
    double pf = 1.0, pr = 1.0;
    for (int s = 0; s < 4; ++s) {
      int k = m->sp[j * 8 + s];
      if (k >= 0) pf *= ipow(w->C[k], m->nu[j * 8 + s]);
      k = m->sp[j * 8 + 4 + s];
      if (k >= 0) pr *= ipow(w->C[k], m->nu[j * 8 + 4 + s]);
    }
    w->kf[j] = kf;
    w->kr[j] = kr;
    w->pf[j] = pf;
    w->pr[j] = pr;
    double q = kf * pf - kr * pr;
    if (type == B200CHEM_RXN_THREEBODY) q *= M;
    w->q[j] = q;
    if (want_jac) {
      /* d q / d T at fixed concentrations */
      double dlnkinf = a[1] * invT + a[2] * invT * invT;
      double dlnkf = dlnkinf;
      if (type == B200CHEM_RXN_LINDEMANN || type == B200CHEM_RXN_TROE) {
        const double* b = m->arr_lo + 3 * j;
        double dlnk0 = b[1] * invT + b[2] * invT * invT;
        double dlnPr = dlnk0 - dlnkinf;
        double Pr = w->Pr[j];
        dlnkf = dlnkinf + dlnPr / (1.0 + Pr) + w->dlogF_dlogPr[j] * dlnPr;
        if (type == B200CHEM_RXN_TROE) {
          const double* t = m->troe + 4 * j;
          double e3 = exp(-T / t[1]), e1 = exp(-T / t[2]);
          double Fc = (1.0 - t[0]) * e3 + t[0] * e1;
          double dFc = -(1.0 - t[0]) / t[1] * e3 - t[0] / t[2] * e1;
          if (m->rflags[j] & B200CHEM_RXN_TROE_T2) {
            double e2 = exp(-t[3] * invT);
            Fc += e2;
            dFc += t[3] * invT * invT * e2;
          }
          double f1 = w->f1[j], nn = w->nn[j];
          double u = (Pr > 1e-300 ? log10(Pr) : -300.0) + w->cc[j];
          double den = nn - 0.14 * u;
          double df1 = (-0.67 * nn + 1.27 * u) / (den * den);
          double g = 1.0 + f1 * f1;
          double dlogF_dlogFc = 1.0 / g - w->logFc[j] * 2.0 * f1 / (g * g) * df1;
          if (Fc > 1e-300) dlnkf += dlogF_dlogFc * dFc / Fc;
        }
      }
      double dkr_T;
      if (m->rflags[j] & B200CHEM_RXN_EXPLICIT_REV) {
        const double* r = m->arr_rev + 3 * j;
        dkr_T = kr * (r[1] * invT + r[2] * invT * invT);
      } else if (m->rflags[j] & B200CHEM_RXN_REVERSIBLE) {
        double sh = 0.0;
        for (int s = 0; s < 8; ++s) {
          int k = m->sp[j * 8 + s];
          if (k >= 0) sh += (s < 4 ? -1.0 : 1.0) * m->nu[j * 8 + s] * w->hRT[k];
        }
        double dlnKc = sh * invT - m->sdnu[j] * invT;
        dkr_T = kr * (dlnkf - dlnKc);
      } else {
        dkr_T = 0.0;
      }
      double dq = kf * dlnkf * pf - dkr_T * pr;
      if (type == B200CHEM_RXN_THREEBODY) dq *= M;
      w->dq_dT[j] = dq;
    }
  }
}

/* HP right-hand side.  y = (rhoY_0..rhoY_{N-1}, T); F = (F_rhoY, F_rhoH). */
void orc_rhs_w(const orc_mech* m, const double* y, const double* F, double* ydot, orc_kin_work* w) {
  const int N = m->N, R = m->R;
  const double T = y[N];
  for (int k = 0; k < N; ++k) w->C[k] = y[k] / m->mw[k];
  kinetics(m, T, w, 0);
  for (int k = 0; k < N; ++k) ydot[k] = 0.0;
  for (int j = 0; j < R; ++j) {
    double q = w->q[j];
    for (int s = 0; s < 8; ++s) {
      int k = m->sp[j * 8 + s];
      if (k >= 0) ydot[k] += (s < 4 ? -1.0 : 1.0) * m->nu[j * 8 + s] * q;
    }
  }
  double rcp = 0.0, hsum = 0.0;
  for (int k = 0; k < N; ++k) {
    ydot[k] = ydot[k] * m->mw[k] + F[k];
    double cpk = w->cpR[k] * R_CGS / m->mw[k];
    double hk = w->hRT[k] * R_CGS * T / m->mw[k];
    rcp += y[k] * cpk;
    hsum += hk * ydot[k];
  }
  ydot[N] = (F[N] - hsum) / rcp;
}

/* Analytic Jacobian J[i*n + j] = d ydot_i / d y_j of the HP system. */
void orc_jac_w(const orc_mech* m, const double* y, const double* F, double* J, double* ydot,
               orc_kin_work* w) {
  const int N = m->N, R = m->R, n = N + 1;
  const double T = y[N];
  for (int k = 0; k < N; ++k) w->C[k] = y[k] / m->mw[k];
  kinetics(m, T, w, 1);
  memset(J, 0, sizeof(double) * n * n);
  /* molar production-rate derivatives: dwdot_k/dC_l (stored in J[k][l]) and dwdot_k/dT */
  for (int j = 0; j < R; ++j) {
    const int type = m->rtype[j];
    /* dq/dC_l for all l */
    double base = 0.0; /* coefficient multiplying eff_l */
    if (type == B200CHEM_RXN_THREEBODY) base = w->kf[j] * w->pf[j] - w->kr[j] * w->pr[j];
    else if (type == B200CHEM_RXN_LINDEMANN || type == B200CHEM_RXN_TROE)
      base = w->dkf_dM[j] * (w->pf[j] - (w->kf[j] > 0 ? w->kr[j] / w->kf[j] : 0.0) * w->pr[j]);
    double mult = (type == B200CHEM_RXN_THREEBODY) ? w->M[j] : 1.0;
    for (int l = 0; l < N; ++l) {
      double d = 0.0;
      if (type != B200CHEM_RXN_ELEMENTARY) d += m->eff[j * N + l] * base;
      /* mass-action part */
      for (int s = 0; s < 4; ++s) {
        int k = m->sp[j * 8 + s];
        if (k == l) {
          int v = m->nu[j * 8 + s];
          double p = v * ipow(w->C[l], v - 1);
          for (int s2 = 0; s2 < 4; ++s2) {
            int k2 = m->sp[j * 8 + s2];
            if (k2 >= 0 && s2 != s) p *= ipow(w->C[k2], m->nu[j * 8 + s2]);
          }
          d += mult * w->kf[j] * p;
        }
        k = m->sp[j * 8 + 4 + s];
        if (k == l) {
          int v = m->nu[j * 8 + 4 + s];
          double p = v * ipow(w->C[l], v - 1);
          for (int s2 = 0; s2 < 4; ++s2) {
            int k2 = m->sp[j * 8 + 4 + s2];
            if (k2 >= 0 && s2 != s) p *= ipow(w->C[k2], m->nu[j * 8 + 4 + s2]);
          }
          d -= mult * w->kr[j] * p;
        }
      }
      if (d == 0.0) continue;
      for (int k = 0; k < N; ++k) {
        double v = m->dnu[j * N + k];
        if (v != 0.0) J[k * n + l] += v * d;
      }
    }
    for (int k = 0; k < N; ++k) {
      double v = m->dnu[j * N + k];
      if (v != 0.0) J[k * n + N] += v * w->dq_dT[j];
    }
  }
  /* species rows: ydot_k = W_k wdot_k + F_k, C_l = y_l / W_l */
  for (int k = 0; k < N; ++k) {
    double wdot = 0.0;
    for (int j = 0; j < R; ++j) wdot += m->dnu[j * N + k] * w->q[j];
    ydot[k] = wdot * m->mw[k] + F[k];
    for (int l = 0; l < N; ++l) J[k * n + l] *= m->mw[k] / m->mw[l];
    J[k * n + N] *= m->mw[k];
  }
  /* temperature row */
  double rcp = 0.0, hsum = 0.0, drcp = 0.0, cpdot = 0.0;
  for (int k = 0; k < N; ++k) {
    double cpk = w->cpR[k] * R_CGS / m->mw[k];
    double hk = w->hRT[k] * R_CGS * T / m->mw[k];
    rcp += y[k] * cpk;
    hsum += hk * ydot[k];
    drcp += y[k] * w->dcpR[k] * R_CGS / m->mw[k];
    cpdot += cpk * ydot[k];
  }
  double Tdot = (F[N] - hsum) / rcp;
  ydot[N] = Tdot;
  for (int l = 0; l <= N; ++l) {
    double s = 0.0;
    for (int k = 0; k < N; ++k) s += w->hRT[k] * R_CGS * T / m->mw[k] * J[k * n + l];
    if (l < N) {
      double cpl = w->cpR[l] * R_CGS / m->mw[l];
      J[N * n + l] = -(s + Tdot * cpl) / rcp;
    } else {
      J[N * n + N] = -(s + cpdot + Tdot * drcp) / rcp;
    }
  }
}

/* --------------------------------------------------------- dense LU (FP64) */
static int lu_factor(double* A, int n, int* piv) {
  for (int k = 0; k < n; ++k) {
    int p = k;
    double amax = fabs(A[k * n + k]);
    for (int i = k + 1; i < n; ++i) {
      double v = fabs(A[i * n + k]);
      if (v > amax) { amax = v; p = i; }
    }
    piv[k] = p;
    if (amax == 0.0) return k + 1;
    if (p != k)
      for (int j = 0; j < n; ++j) { double t = A[k * n + j]; A[k * n + j] = A[p * n + j]; A[p * n + j] = t; }
    double inv = 1.0 / A[k * n + k];
    for (int i = k + 1; i < n; ++i) {
      double l = A[i * n + k] * inv;
      A[i * n + k] = l;
      if (l != 0.0)
        for (int j = k + 1; j < n; ++j) A[i * n + j] -= l * A[k * n + j];
    }
  }
  return 0;
}

static void lu_solve(const double* A, int n, const int* piv, double* b) {
  for (int k = 0; k < n; ++k) {
    int p = piv[k];
    if (p != k) { double t = b[k]; b[k] = b[p]; b[p] = t; }
  }
  for (int i = 1; i < n; ++i) {
    double s = b[i];
    for (int j = 0; j < i; ++j) s -= A[i * n + j] * b[j];
    b[i] = s;
  }
  for (int i = n - 1; i >= 0; --i) {
    double s = b[i];
    for (int j = i + 1; j < n; ++j) s -= A[i * n + j] * b[j];
    b[i] = s / A[i * n + i];
  }
}

/* ----------------------------------------------------------- BDF (CVODE) */
#define QMAX_LIM 5
#define L_MAX (QMAX_LIM + 1)
#define UROUND 2.220446049250313e-16
#define ETAMX1 10000.0
#define ETAMX2 10.0
#define ETAMX3 10.0
#define ETAMXF 0.2
#define ETAMIN 0.1
#define ETACF 0.25
#define ADDON 1e-6
#define BIAS1 6.0
#define BIAS2 6.0
#define BIAS3 10.0
#define ONEPSM 1.000001
#define THRESH 1.5
#define SMALL_NST 10
#define MXNCF 10
#define MXNEF 7
#define MXNEF1 3
#define SMALL_NEF 2
#define LONG_WAIT 10
#define NLS_MAXCOR 3
#define CRDOWN 0.3
#define DGMAX_LSETUP 0.3
#define RDIV 2.0
#define MSBP 20
#define MSBJ 51
#define DGMAX_JBAD 0.2
#define NLSCOEF 0.1
#define HLB_FACTOR 100.0
#define HUB_FACTOR 0.1
#define H_BIAS 0.5

enum { FIRST_CALL, PREV_CONV_FAIL, PREV_ERR_FAIL };
enum { NO_FAILURES, FAIL_BAD_J, FAIL_OTHER };

typedef struct orc_opts {
  double rtol;
  double atol;
  int max_order;
  int max_steps;
  int lu_fp64; /* unused here: the oracle is always FP64 */
} orc_opts;

typedef struct orc_cell_stats {
  int status, nst, nfe, nje, nlu, netf, ncfn, nni;
} orc_cell_stats;

typedef struct bdf_mem {
  const orc_mech* m;
  int n, qmax;
  double* zn[L_MAX + 1];
  double *ewt, *acor, *tempv, *ftemp, *y, *atolv, *delta, *J, *Mlu;
  int* piv;
  const double* F;
  orc_kin_work kw;
  double tau[L_MAX + 2], tq[6], l[L_MAX + 1];
  double h, hprime, hscale, eta, etamax, tn, gamma, gammap, gamrat, crate, acnrm, rl1, saved_tq5;
  double rtol;
  int q, qprime, L, qwait, nst, nfe, nje, nsetups, netf, ncfn, nni, nstlp, nstlj, jcur;
  int convfail;
} bdf_mem;

static double wrms(const double* v, const double* w, int n) {
  double s = 0.0;
  for (int i = 0; i < n; ++i) { double t = v[i] * w[i]; s += t * t; }
  return sqrt(s / n);
}

static void f_eval(bdf_mem* b, const double* y, double* out) {
  orc_rhs_w(b->m, y, b->F, out, &b->kw);
  b->nfe++;
}

static void set_ewt(bdf_mem* b, const double* y) {
  for (int i = 0; i < b->n; ++i) b->ewt[i] = 1.0 / (b->rtol * fabs(y[i]) + b->atolv[i]);
}

static void bdf_rescale(bdf_mem* b) {
  double factor = b->eta;
  for (int j = 1; j <= b->q; ++j) {
    for (int i = 0; i < b->n; ++i) b->zn[j][i] *= factor;
    factor *= b->eta;
  }
  b->h = b->hscale * b->eta;
  b->hscale = b->h;
}

static void bdf_predict(bdf_mem* b) {
  b->tn += b->h;
  for (int k = 1; k <= b->q; ++k)
    for (int j = b->q; j >= k; --j)
      for (int i = 0; i < b->n; ++i) b->zn[j - 1][i] += b->zn[j][i];
}

static void bdf_restore(bdf_mem* b, double saved_t) {
  b->tn = saved_t;
  for (int k = 1; k <= b->q; ++k)
    for (int j = b->q; j >= k; --j)
      for (int i = 0; i < b->n; ++i) b->zn[j - 1][i] -= b->zn[j][i];
}

static void set_tq(bdf_mem* b, double hsum, double alpha0, double alpha0_hat, double xi_inv,
                   double xistar_inv) {
  int q = b->q;
  double A1 = 1.0 - alpha0_hat + alpha0;
  double A2 = 1.0 + q * A1;
  b->tq[2] = fabs(A1 / (alpha0 * A2));
  b->tq[5] = fabs(A2 * xistar_inv / (b->l[q] * xi_inv));
  if (b->qwait == 1) {
    if (q > 1) {
      double C = xistar_inv / b->l[q];
      double A3 = alpha0 + 1.0 / q;
      double A4 = alpha0_hat + xi_inv;
      double Cpinv = (1.0 - A4 + A3) / A3;
      b->tq[1] = fabs(C * Cpinv);
    } else {
      b->tq[1] = 1.0;
    }
    hsum += b->tau[q];
    xi_inv = b->h / hsum;
    double A5 = alpha0 - 1.0 / (q + 1);
    double A6 = alpha0_hat - xi_inv;
    double Cppinv = (1.0 - A6 + A5) / A2;
    b->tq[3] = fabs(Cppinv / (xi_inv * (q + 2) * A5));
  }
  b->tq[4] = NLSCOEF / b->tq[2];
}

static void set_bdf(bdf_mem* b) {
  int q = b->q;
  double xi_inv = 1.0, xistar_inv = 1.0;
  b->l[0] = b->l[1] = 1.0;
  for (int i = 2; i <= q; ++i) b->l[i] = 0.0;
  double alpha0 = -1.0, alpha0_hat = -1.0, hsum = b->h;
  if (q > 1) {
    for (int j = 2; j < q; ++j) {
      hsum += b->tau[j - 1];
      xi_inv = b->h / hsum;
      alpha0 -= 1.0 / j;
      for (int i = j; i >= 1; --i) b->l[i] += b->l[i - 1] * xi_inv;
    }
    alpha0 -= 1.0 / q;
    xistar_inv = -b->l[1] - alpha0;
    hsum += b->tau[q - 1];
    xi_inv = b->h / hsum;
    alpha0_hat = -b->l[1] - xi_inv;
    for (int i = q; i >= 1; --i) b->l[i] += b->l[i - 1] * xistar_inv;
  }
  set_tq(b, hsum, alpha0, alpha0_hat, xi_inv, xistar_inv);
  b->rl1 = 1.0 / b->l[1];
  b->gamma = b->h * b->rl1;
  if (b->nst == 0) b->gammap = b->gamma;
  b->gamrat = (b->nst > 0) ? b->gamma / b->gammap : 1.0;
}

static void increase_bdf(bdf_mem* b) {
  int q = b->q, n = b->n;
  for (int i = 0; i <= b->qmax; ++i) b->l[i] = 0.0;
  double alpha1 = 1.0, prod = 1.0, xiold = 1.0, alpha0 = -1.0, hsum = b->hscale;
  b->l[2] = 1.0;
  if (q > 1) {
    for (int j = 1; j < q; ++j) {
      hsum += b->tau[j + 1];
      double xi = hsum / b->hscale;
      prod *= xi;
      alpha0 -= 1.0 / (j + 1);
      alpha1 += 1.0 / xi;
      for (int i = j + 2; i >= 2; --i) b->l[i] = b->l[i] * xiold + b->l[i - 1];
      xiold = xi;
    }
  }
  double A1 = (-alpha0 - alpha1) / prod;
  int L = q + 1;
  for (int i = 0; i < n; ++i) b->zn[L][i] = A1 * b->zn[b->qmax][i];
  for (int j = 2; j <= q; ++j)
    for (int i = 0; i < n; ++i) b->zn[j][i] += b->l[j] * b->zn[L][i];
}

static void decrease_bdf(bdf_mem* b) {
  int q = b->q, n = b->n;
  for (int i = 0; i <= b->qmax; ++i) b->l[i] = 0.0;
  b->l[2] = 1.0;
  double hsum = 0.0;
  for (int j = 1; j <= q - 2; ++j) {
    hsum += b->tau[j];
    double xi = hsum / b->hscale;
    for (int i = j + 2; i >= 2; --i) b->l[i] = b->l[i] * xi + b->l[i - 1];
  }
  for (int j = 2; j < q; ++j)
    for (int i = 0; i < n; ++i) b->zn[j][i] -= b->l[j] * b->zn[q][i];
}

static void adjust_order(bdf_mem* b, int dq) {
  if (dq == 1) increase_bdf(b);
  else if (dq == -1) decrease_bdf(b);
}

/* linear-system setup: maybe refresh J, form M = I - gamma J, factor */
static int lsetup(bdf_mem* b, int convfail) {
  int n = b->n;
  double dgamma = fabs(b->gamma / b->gammap - 1.0);
  int jbad = (b->nst == 0) || (b->nst >= b->nstlj + MSBJ) ||
             (convfail == FAIL_BAD_J && dgamma < DGMAX_JBAD) || (convfail == FAIL_OTHER);
  if (jbad) {
    orc_jac_w(b->m, b->y, b->F, b->J, b->tempv, &b->kw);
    b->nje++;
    b->nstlj = b->nst;
    b->jcur = 1;
  } else {
    b->jcur = 0;
  }
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) b->Mlu[i * n + j] = (i == j ? 1.0 : 0.0) - b->gamma * b->J[i * n + j];
  int ier = lu_factor(b->Mlu, n, b->piv);
  b->nsetups++;
  b->gamrat = 1.0;
  b->gammap = b->gamma;
  b->crate = 1.0;
  b->nstlp = b->nst;
  return ier;
}

/* Newton iteration; returns 0 converged, 1 recoverable failure, 2 setup failure */
static int nls(bdf_mem* b, int nflag) {
  int n = b->n;
  int convfail = (nflag == FIRST_CALL || nflag == PREV_ERR_FAIL) ? NO_FAILURES : FAIL_OTHER;
  int callSetup = (nflag == PREV_CONV_FAIL) || (nflag == PREV_ERR_FAIL) || (b->nst == 0) ||
                  (b->nst >= b->nstlp + MSBP) || (fabs(b->gamrat - 1.0) > DGMAX_LSETUP);
  int jbad = 0;
  for (;;) {
    for (int i = 0; i < n; ++i) b->acor[i] = 0.0;
    /* residual at the predicted state */
    for (int i = 0; i < n; ++i) b->y[i] = b->zn[0][i];
    f_eval(b, b->y, b->ftemp);
    if (callSetup) {
      int ier = lsetup(b, jbad ? FAIL_BAD_J : convfail);
      callSetup = 0;
      if (ier) return 2;
    }
    double delp = 0.0, del = 0.0;
    int m = 0, ret = 1;
    for (;;) {
      b->nni++;
      for (int i = 0; i < n; ++i)
        b->delta[i] = -(b->rl1 * b->zn[1][i] + b->acor[i] - b->gamma * b->ftemp[i]);
      lu_solve(b->Mlu, n, b->piv, b->delta);
      if (b->gamrat != 1.0) {
        double s = 2.0 / (1.0 + b->gamrat);
        for (int i = 0; i < n; ++i) b->delta[i] *= s;
      }
      for (int i = 0; i < n; ++i) b->acor[i] += b->delta[i];
      del = wrms(b->delta, b->ewt, n);
      if (m > 0) b->crate = fmax(CRDOWN * b->crate, del / delp);
      double dcon = del * fmin(1.0, b->crate) / b->tq[4];
      if (dcon <= 1.0) {
        b->acnrm = (m == 0) ? del : wrms(b->acor, b->ewt, n);
        ret = 0;
        break;
      }
      if (m >= 1 && del > RDIV * delp) { ret = 1; break; }
      delp = del;
      m++;
      if (m >= NLS_MAXCOR) { ret = 1; break; }
      for (int i = 0; i < n; ++i) b->y[i] = b->zn[0][i] + b->acor[i];
      f_eval(b, b->y, b->ftemp);
    }
    if (ret == 0) {
      for (int i = 0; i < n; ++i) b->y[i] = b->zn[0][i] + b->acor[i];
      b->jcur = 0;
      return 0;
    }
    if (!b->jcur) {
      /* stale Jacobian: retry once with a fresh one */
      callSetup = 1;
      jbad = 1;
      continue;
    }
    return 1;
  }
}

static void complete_step(bdf_mem* b) {
  int n = b->n, q = b->q;
  b->nst++;
  for (int i = q; i >= 2; --i) b->tau[i] = b->tau[i - 1];
  if (q == 1 && b->nst > 1) b->tau[2] = b->tau[1];
  b->tau[1] = b->h;
  for (int j = 0; j <= q; ++j)
    for (int i = 0; i < n; ++i) b->zn[j][i] += b->l[j] * b->acor[i];
  b->qwait--;
  if (b->qwait == 1 && q != b->qmax) {
    for (int i = 0; i < n; ++i) b->zn[b->qmax][i] = b->acor[i];
    b->saved_tq5 = b->tq[5];
  }
}

static void set_eta(bdf_mem* b) {
  if (b->eta < THRESH) {
    b->eta = 1.0;
    b->hprime = b->h;
  } else {
    b->eta = fmin(b->eta, b->etamax);
    b->hprime = b->h * b->eta;
  }
}

static void prepare_next_step(bdf_mem* b, double dsm) {
  int n = b->n;
  if (b->etamax == 1.0) {
    b->qwait = b->qwait > 2 ? b->qwait : 2;
    b->qprime = b->q;
    b->hprime = b->h;
    b->eta = 1.0;
    return;
  }
  double etaq = 1.0 / (pow(BIAS2 * dsm, 1.0 / b->L) + ADDON);
  if (b->qwait != 0) {
    b->eta = etaq;
    b->qprime = b->q;
    set_eta(b);
    return;
  }
  b->qwait = 2;
  double etaqm1 = 0.0, etaqp1 = 0.0;
  if (b->q > 1) {
    double ddn = wrms(b->zn[b->q], b->ewt, n) * b->tq[1];
    etaqm1 = 1.0 / (pow(BIAS1 * ddn, 1.0 / b->q) + ADDON);
  }
  if (b->q != b->qmax && b->saved_tq5 != 0.0) {
    double cquot = (b->tq[5] / b->saved_tq5) * pow(b->h / b->tau[2], b->L);
    for (int i = 0; i < n; ++i) b->tempv[i] = b->acor[i] - cquot * b->zn[b->qmax][i];
    double dup = wrms(b->tempv, b->ewt, n) * b->tq[3];
    etaqp1 = 1.0 / (pow(BIAS3 * dup, 1.0 / (b->L + 1)) + ADDON);
  }
  double etam = fmax(etaqm1, fmax(etaq, etaqp1));
  if (etam < THRESH) {
    b->eta = 1.0;
    b->qprime = b->q;
  } else if (etam == etaq) {
    b->eta = etaq;
    b->qprime = b->q;
  } else if (etam == etaqm1) {
    b->eta = etaqm1;
    b->qprime = b->q - 1;
  } else {
    b->eta = etaqp1;
    b->qprime = b->q + 1;
    for (int i = 0; i < n; ++i) b->zn[b->qmax][i] = b->acor[i];
  }
  set_eta(b);
}

/* one internal step; returns 0 ok, else a B200CHEM_CELL_* failure code */
static int bdf_step(bdf_mem* b) {
  double saved_t = b->tn;
  int ncf = 0, nef = 0, nflag = FIRST_CALL;
  double dsm;
  if (b->nst > 0 && b->hprime != b->h) {
    /* b->eta still holds the ratio chosen by prepare_next_step */
    if (b->qprime != b->q) {
      adjust_order(b, b->qprime - b->q);
      b->q = b->qprime;
      b->L = b->q + 1;
      b->qwait = b->L;
    }
    bdf_rescale(b);
  }
  for (;;) {
    bdf_predict(b);
    set_bdf(b);
    int r = nls(b, nflag);
    if (r != 0) {
      b->ncfn++;
      bdf_restore(b, saved_t);
      ncf++;
      b->etamax = 1.0;
      if (ncf == MXNCF) return r == 2 ? B200CHEM_CELL_SINGULAR : B200CHEM_CELL_CONVFAIL;
      b->eta = ETACF;
      nflag = PREV_CONV_FAIL;
      bdf_rescale(b);
      continue;
    }
    dsm = b->acnrm * b->tq[2];
    if (dsm <= 1.0) break;
    nef++;
    b->netf++;
    nflag = PREV_ERR_FAIL;
    bdf_restore(b, saved_t);
    if (nef == MXNEF) return B200CHEM_CELL_ERRFAIL;
    b->etamax = 1.0;
    if (nef <= MXNEF1) {
      b->eta = 1.0 / (pow(BIAS2 * dsm, 1.0 / b->L) + ADDON);
      b->eta = fmax(ETAMIN, b->eta);
      if (nef >= SMALL_NEF) b->eta = fmin(b->eta, ETAMXF);
      bdf_rescale(b);
      continue;
    }
    if (b->q > 1) {
      b->eta = ETAMIN;
      adjust_order(b, -1);
      b->L = b->q;
      b->q--;
      b->qwait = b->L;
      bdf_rescale(b);
      continue;
    }
    b->eta = ETAMIN;
    b->h *= b->eta;
    b->hscale = b->h;
    b->qwait = LONG_WAIT;
    f_eval(b, b->zn[0], b->tempv);
    for (int i = 0; i < b->n; ++i) b->zn[1][i] = b->h * b->tempv[i];
  }
  complete_step(b);
  prepare_next_step(b, dsm);
  b->etamax = (b->nst <= SMALL_NST) ? ETAMX2 : ETAMX3;
  return 0;
}

static double initial_h(bdf_mem* b, double tout) {
  int n = b->n;
  double tdist = fabs(tout - b->tn);
  double tround = UROUND * fmax(fabs(b->tn), fabs(tout));
  double hlb = HLB_FACTOR * tround;
  double hub_inv = 0.0;
  for (int i = 0; i < n; ++i) {
    double t1 = HUB_FACTOR * fabs(b->zn[0][i]) + b->atolv[i];
    double r = fabs(b->zn[1][i]) / t1;
    if (r > hub_inv) hub_inv = r;
  }
  double hub = HUB_FACTOR * tdist;
  if (hub * hub_inv > 1.0) hub = 1.0 / hub_inv;
  double hg = sqrt(hlb * hub);
  if (hub < hlb) return hg;
  int hnewOK = 0;
  double hnew = hg;
  for (int count1 = 1; count1 <= 4; ++count1) {
    for (int i = 0; i < n; ++i) b->y[i] = b->zn[0][i] + hg * b->zn[1][i];
    f_eval(b, b->y, b->tempv);
    for (int i = 0; i < n; ++i) b->tempv[i] = (b->tempv[i] - b->zn[1][i]) / hg;
    double yddnrm = wrms(b->tempv, b->ewt, n);
    hnew = (yddnrm * hub * hub > 2.0) ? sqrt(2.0 / yddnrm) : sqrt(hg * hub);
    if (hnewOK) { hg = hnew; break; }
    double hrat = hnew / hg;
    if (hrat > 0.5 && hrat < 2.0) hnewOK = 1;
    if (count1 > 1 && hrat > 2.0) { hnew = hg; hnewOK = 1; }
    hg = hnew;
  }
  double h0 = H_BIAS * hg;
  if (h0 < hlb) h0 = hlb;
  if (h0 > hub) h0 = hub;
  return h0;
}

/* Integrate one cell over [0, dt]; y (n) in/out.  Returns a B200CHEM_CELL_* code. */
static int bdf_integrate(bdf_mem* b, double* y, double dt, int max_steps) {
  int n = b->n;
  for (int i = 0; i < n; ++i) b->zn[0][i] = y[i];
  b->tn = 0.0;
  b->nst = b->nfe = b->nje = b->nsetups = b->netf = b->ncfn = b->nni = 0;
  b->nstlp = b->nstlj = 0;
  b->q = b->qprime = 1;
  b->L = 2;
  b->qwait = b->L;
  b->etamax = ETAMX1;
  b->saved_tq5 = 0.0;
  b->crate = 1.0;
  b->jcur = 0;
  for (int i = 0; i <= L_MAX + 1; ++i) b->tau[i] = 0.0;
  for (int i = 0; i < 6; ++i) b->tq[i] = 0.0;
  set_ewt(b, b->zn[0]);
  f_eval(b, b->zn[0], b->zn[1]);
  for (int i = 0; i < n; ++i)
    if (!isfinite(b->zn[1][i])) return B200CHEM_CELL_NONFINITE;
  double h0 = initial_h(b, dt);
  b->h = b->hscale = b->hprime = h0;
  for (int i = 0; i < n; ++i) b->zn[1][i] *= h0;
  int nstloc = 0;
  for (;;) {
    if (b->nst > 0) set_ewt(b, b->zn[0]);
    if (nstloc >= max_steps) return B200CHEM_CELL_MAXSTEPS;
    int r = bdf_step(b);
    if (r != 0) return r;
    nstloc++;
    if (b->tn - dt >= 0.0) break;
  }
  /* interpolate to dt from the Nordsieck array */
  double s = (dt - b->tn) / b->h;
  for (int i = 0; i < n; ++i) {
    double v = b->zn[b->q][i];
    for (int j = b->q - 1; j >= 0; --j) v = b->zn[j][i] + s * v;
    y[i] = v;
  }
  return B200CHEM_CELL_OK;
}

static bdf_mem* bdf_new(const orc_mech* m, int qmax) {
  bdf_mem* b = (bdf_mem*)calloc(1, sizeof(bdf_mem));
  int n = m->N + 1;
  b->m = m;
  b->n = n;
  b->qmax = qmax;
  double* p = (double*)calloc((size_t)(L_MAX + 1) * n + 8 * (size_t)n + 2 * (size_t)n * n, sizeof(double));
  for (int j = 0; j <= L_MAX; ++j) { b->zn[j] = p; p += n; }
  b->ewt = p; p += n; b->acor = p; p += n; b->tempv = p; p += n; b->ftemp = p; p += n;
  b->y = p; p += n; b->atolv = p; p += n; b->delta = p; p += n; p += n;
  b->J = p; p += n * n; b->Mlu = p; p += n * n;
  b->piv = (int*)calloc(n, sizeof(int));
  kin_work_alloc(&b->kw, m->N, m->R);
  return b;
}

static void bdf_free(bdf_mem* b) {
  free(b->zn[0]);
  free(b->piv);
  kin_work_free(&b->kw);
  free(b);
}

/* ------------------------------------------------------------ public API */

/* Per-cell evaluation helpers for tests: y, F, out are (N+1)-vectors. */
void orc_rhs(const orc_mech* m, const double* y, const double* F, double* ydot) {
  orc_kin_work w;
  kin_work_alloc(&w, m->N, m->R);
  orc_rhs_w(m, y, F, ydot, &w);
  kin_work_free(&w);
}

void orc_jac(const orc_mech* m, const double* y, const double* F, double* J) {
  orc_kin_work w;
  kin_work_alloc(&w, m->N, m->R);
  double* yd = (double*)malloc(sizeof(double) * (m->N + 1));
  orc_jac_w(m, y, F, J, yd, &w);
  free(yd);
  kin_work_free(&w);
}

/* Molar production rates (mol/cm^3/s) at T and concentrations C. */
void orc_wdot(const orc_mech* m, double T, const double* C, double* wdot) {
  orc_kin_work w;
  kin_work_alloc(&w, m->N, m->R);
  for (int k = 0; k < m->N; ++k) w.C[k] = C[k];
  kinetics(m, T, &w, 0);
  for (int k = 0; k < m->N; ++k) {
    double s = 0.0;
    for (int j = 0; j < m->R; ++j) s += m->dnu[j * m->N + k] * w.q[j];
    wdot[k] = s;
  }
  kin_work_free(&w);
}

/* Mixture specific enthalpy h(T, Y) (erg/g) and T from (h, Y) by Newton
 * (the HY2T of the EOS, Source/PeleLMeX_K.H:700-723).  Returns iterations
 * used, or -1 if not converged. */
double orc_mix_h(const orc_mech* m, double T, const double* Y) {
  double h = 0.0;
  for (int k = 0; k < m->N; ++k) {
    double cpR, hRT, sR, d;
    nasa_eval(m, k, T, &cpR, &hRT, &sR, &d);
    h += Y[k] * hRT * R_CGS * T / m->mw[k];
  }
  return h;
}

int orc_t_from_hy(const orc_mech* m, double h, const double* Y, double* T) {
  double t = *T;
  for (int it = 0; it < 100; ++it) {
    double hm = 0.0, cp = 0.0;
    for (int k = 0; k < m->N; ++k) {
      double cpR, hRT, sR, d;
      nasa_eval(m, k, t, &cpR, &hRT, &sR, &d);
      hm += Y[k] * hRT * R_CGS * t / m->mw[k];
      cp += Y[k] * cpR * R_CGS / m->mw[k];
    }
    double dT = (h - hm) / cp;
    t += dT;
    if (fabs(dT) <= 1e-12 * t) { *T = t; return it + 1; }
  }
  *T = t;
  return -1;
}

/*
 * React a batch of cells, component-major (SoA) arrays exactly like the
 * flat form of ReactorBase::react: rhoY[k*ncells + c] etc.  atol_vec (n
 * entries) are the absolute tolerances per component.  OpenMP over cells with
 * a dynamic schedule (Source/PeleLMeX_Reactions.cpp:48-55).  Returns the
 * number of failed cells.
 */
int orc_react_batch(const orc_mech* m, const orc_opts* o, const double* atol_vec, double* rhoY,
                    const double* frhoY, double* T, double* rhoH, const double* frhoH,
                    double* fct, const int* mask, int64_t ncells, double dt, int* status,
                    int* cstats /* [ncells][7] nst,nfe,nje,nlu,netf,ncfn,nni or NULL */,
                    int nthreads) {
  const int N = m->N, n = N + 1;
  int nfail = 0;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
#pragma omp parallel reduction(+ : nfail)
  {
    bdf_mem* b = bdf_new(m, o->max_order < 1 ? 1 : (o->max_order > QMAX_LIM ? QMAX_LIM : o->max_order));
    double* y = (double*)malloc(sizeof(double) * n);
    double* F = (double*)malloc(sizeof(double) * n);
    b->rtol = o->rtol;
    for (int i = 0; i < n; ++i) b->atolv[i] = atol_vec[i];
    b->F = F;
#pragma omp for schedule(dynamic, 16)
    for (int64_t c = 0; c < ncells; ++c) {
      if (mask && mask[c] == 0) {
        if (status) status[c] = B200CHEM_CELL_MASKED;
        if (fct) fct[c] = 0.0;
        if (cstats) memset(cstats + 7 * c, 0, 7 * sizeof(int));
        continue;
      }
      double rho = 0.0;
      for (int k = 0; k < N; ++k) {
        y[k] = rhoY[(int64_t)k * ncells + c];
        F[k] = frhoY[(int64_t)k * ncells + c];
        rho += y[k];
      }
      y[N] = T[c];
      F[N] = frhoH[c];
      int st;
      int ok = rho > 0.0 && y[N] > 0.0 && isfinite(rho) && isfinite(y[N]) && isfinite(F[N]);
      for (int k = 0; k < N && ok; ++k) ok = isfinite(y[k]) && isfinite(F[k]);
      if (!ok) {
        st = B200CHEM_CELL_NONFINITE;
        b->nst = b->nfe = b->nje = b->nsetups = b->netf = b->ncfn = b->nni = 0;
      } else {
        st = bdf_integrate(b, y, dt, o->max_steps);
      }
      if (st == B200CHEM_CELL_OK) {
        for (int k = 0; k < N; ++k) rhoY[(int64_t)k * ncells + c] = y[k];
        T[c] = y[N];
        rhoH[c] = rhoH[c] + dt * F[N];
      } else {
        nfail++;
      }
      if (status) status[c] = st;
      if (fct) fct[c] = (double)b->nfe;
      if (cstats) {
        int* cs = cstats + 7 * c;
        cs[0] = b->nst; cs[1] = b->nfe; cs[2] = b->nje; cs[3] = b->nsetups;
        cs[4] = b->netf; cs[5] = b->ncfn; cs[6] = b->nni;
      }
    }
    free(y);
    free(F);
    bdf_free(b);
  }
  return nfail;
}

int orc_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
