"""Algorithmic operation counts of the HP BDF reaction advance.

The roofline figures of the reactor are quoted against these counts, not
against what a kernel happens to execute: the FP64 floating-point operations
the dense-direct BDF algorithm needs per cell (one right-hand side, one
analytic Jacobian, one LU factorisation of the (N+1)x(N+1) Newton matrix, one
pair of triangular solves), times the per-cell call counters the integrator
reports (nfe, nje, nlu, nni; the counters of CVODE's dense direct reactor,
PelePhysics Reactions/ReactorCvode.cpp, as printed by the reference at
Source/PeleLMeX_Reactions.cpp:122-141 when fctCount is requested).

Counting rules (one add, mul or compare = 1 flop; an FMA = 2; a division or
square root = 1; an exp / log / log10 / pow = 1 flop, and the number of them
is reported separately, "EXP" below):

* thermo per species: NASA-7 cp/R, h/RT, s/R, g/RT by Horner       -> 30
* concentration C_k = rhoY_k / W_k                                   -> 1
* forward rate: lnA + b lnT - Ea/(RT) then exp                       -> 4 + EXP
* third body M: Ctot + sum (eff-1) C_k                               -> 2 per entry
* falloff (Lindemann): k0 (4 + EXP), Pr, blend                       -> 8 + EXP
* Troe: Fc (3 exp + 8), logs (2 EXP), F (12 + EXP)                    -> 20 + 6 EXP
* reverse from Kc: sum nu g/RT over the slots, exp                    -> 2 per slot + 4 + EXP
* mass-action products: nu - 1 multiplies per slot                   -> sum(|nu|)
* progress rate and wdot gather                                       -> 3 + 2 per incidence
* T equation: sum Y cp, sum h ydot, divide                            -> 4 N + 2

The Jacobian adds, per reaction, the temperature derivatives (about 12
flops) and 2 flops for each (reactant slot, slot) pair, plus 2 per
efficiency entry and slot, and the T row (2 N per column).  LU is
2/3 n^3, a solve pair 2 n^2; the FP64 refinement step adds a residual
matrix-vector product (2 n^2) and a second solve pair.
"""
from __future__ import annotations

import numpy as np

EXP_FLOPS = 1


def op_counts(flat) -> dict:
    """Per-call FP64 flop counts for one cell of the flattened mechanism
    (exp/log counted as one flop each), with the number of exp/log calls of
    one right-hand side and one Jacobian in rhs_exp / jac_exp."""
    a = flat.arrays
    N, R = flat.n_species, flat.n_reactions
    n = N + 1
    rtype, rflags = a["rtype"], a["rflags"]
    sp, nu = a["sp"], a["nu"]
    eff_ptr = a["eff_ptr"]
    species = N * 31
    rx = 0
    jac_extra = 0
    nnz = 0
    n_exp = 1  # log T
    for j in range(R):
        slots = [s for s in range(8) if sp[j, s] >= 0]
        neff = int(eff_ptr[j + 1] - eff_ptr[j])
        c = 4 + EXP_FLOPS
        e = 1
        if rtype[j] != 0:
            c += 2 * neff + 1
        if rtype[j] >= 2:
            c += 8 + EXP_FLOPS
            e += 1
        if rtype[j] == 3:
            c += 20 + 6 * EXP_FLOPS
            e += 6
        if rflags[j] & 2:
            c += 4 + EXP_FLOPS
            e += 1
        elif rflags[j] & 1:
            c += 2 * len(slots) + 4 + EXP_FLOPS
            e += 1
        n_exp += e
        c += int(np.abs(nu[j, slots]).sum()) + 3
        rx += c
        nnz += len(set(int(sp[j, s]) for s in slots))
        react_slots = [s for s in slots if s < 4]
        jac_extra += 12 + 2 * len(react_slots) * len(slots)
        if rtype[j] != 0:
            jac_extra += 2 * neff * len(slots) + 2 * len(slots)
    rhs = species + rx + 2 * nnz + 4 * N + 2
    jac = rhs + jac_extra + n * 2 * N
    lu = (2 * n ** 3) // 3
    solve = 2 * n * n
    return dict(n=n, rhs=rhs, jac=jac, lu=lu, solve=solve, refine=2 * n * n + solve, rhs_exp=n_exp,
                jac_exp=n_exp)


def flops_per_cell(counts: dict, nfe: float, nje: float, nlu: float, nni: float, nst: float) -> float:
    """Algorithmic FP64 flops per cell for average per-cell counters.

    nfe counts right-hand sides (the Newton residuals and the initial-step
    estimate), nje Jacobians, nlu factorisations, nni Newton iterations (one
    refined solve each); each step adds its prediction and error test
    (about 4 (q+1) n with q = 5 at most, counted as 12 n)."""
    n = counts["n"]
    return (nfe * counts["rhs"] + nje * counts["jac"] + nlu * counts["lu"]
            + nni * (counts["solve"] + counts["refine"]) + nst * 12 * n)


def bytes_per_cell(n_species: int) -> int:
    """HBM bytes one react call must move per cell: read rhoY, extF_rhoY,
    T, rhoH, extF_rhoH and fctCount; write rhoY, T, rhoH and fctCount (FP64)."""
    return 8 * ((2 * n_species + 4) + (n_species + 3))


# ------------------------------------------------- per-kernel HBM bytes
RCELL_BYTES = 448  # step-control record of the round-based integrator


def kernel_bytes(kind: str, n_species: int, lut_bytes: int = 4) -> float:
    """Algorithmic HBM bytes ONE processed cell costs in a kernel of the
    round-based integrator (bytes the step of the algorithm must read and
    write, each once):

    * rhs: list slot, read y and the forcing (2n), write f (n)
    * ctrl / ctrl_setup (one Newton iteration): the step-control record read
      and written, read zn[1], acor, ftemp, f, ewt, scaling (6n) and write
      acor (n), read the FP64 Jacobian (n^2) for the refinement residual and
      the inverse (n^2 at lut_bytes)
    * jac (only the setups whose Jacobian is stale reach it): list slot,
      read y and f (2n), write J (n^2)
    * gj: list slot and gamma, read J (n^2) and ewt (n), write the scaling
      (n) and the inverse (n^2 at lut_bytes)
    """
    n = n_species + 1
    if kind == "rhs":
        return 4 + 8 * 3 * n
    if kind in ("ctrl", "ctrl_setup"):
        return 4 + 2 * RCELL_BYTES + 8 * 7 * n + 8 * n * n + lut_bytes * n * n
    if kind == "jac":
        return 4 + jac_refresh_bytes(n_species)
    if kind == "gj":
        return 4 + 16 + 8 * n * n + 8 * 2 * n + lut_bytes * n * n
    if kind == "start":
        return bytes_per_cell(n_species) - 8 * (n_species + 3)  # the inputs read
    raise ValueError(kind)


def jac_refresh_bytes(n_species: int) -> float:
    """HBM bytes of one analytic-Jacobian refresh: read y and f (2n), write
    J (n^2)."""
    n = n_species + 1
    return 8 * 2 * n + 8 * n * n
