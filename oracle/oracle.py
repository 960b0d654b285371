"""ctypes front-end of the CPU oracle (oracle/oracle.c) -- TEST INFRASTRUCTURE.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
import this module, and only as the checker or the timed CPU baseline; the
product path never does.  See oracle.c for what is restated and from where.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"

_i32p = ctypes.POINTER(ctypes.c_int32)
_f64p = ctypes.POINTER(ctypes.c_double)


class OrcOpts(ctypes.Structure):
    _fields_ = [("rtol", ctypes.c_double), ("atol", ctypes.c_double), ("max_order", ctypes.c_int),
                ("max_steps", ctypes.c_int), ("lu_fp64", ctypes.c_int)]


def build(force: bool = False) -> Path:
    """Compile liboracle.so with the recipe in oracle/Makefile."""
    src = HERE / "oracle.c"
    if force or not LIB.exists() or LIB.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["make", "-C", str(HERE), "-B" if force else "all"], check=True,
                       stdout=subprocess.DEVNULL)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(str(LIB))
        L.orc_mech_new.restype = ctypes.c_void_p
        L.orc_mech_new.argtypes = [ctypes.c_void_p]
        L.orc_mech_free.argtypes = [ctypes.c_void_p]
        L.orc_rhs.argtypes = [ctypes.c_void_p, _f64p, _f64p, _f64p]
        L.orc_jac.argtypes = [ctypes.c_void_p, _f64p, _f64p, _f64p]
        L.orc_wdot.argtypes = [ctypes.c_void_p, ctypes.c_double, _f64p, _f64p]
        L.orc_mix_h.restype = ctypes.c_double
        L.orc_mix_h.argtypes = [ctypes.c_void_p, ctypes.c_double, _f64p]
        L.orc_t_from_hy.restype = ctypes.c_int
        L.orc_t_from_hy.argtypes = [ctypes.c_void_p, ctypes.c_double, _f64p, _f64p]
        L.orc_react_batch.restype = ctypes.c_int
        L.orc_react_batch.argtypes = [ctypes.c_void_p, ctypes.POINTER(OrcOpts), _f64p, _f64p, _f64p, _f64p,
                                      _f64p, _f64p, _f64p, _i32p, ctypes.c_int64, ctypes.c_double, _i32p,
                                      _i32p, ctypes.c_int]
        L.orc_max_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def _p(a, t=_f64p):
    return a.ctypes.data_as(t) if a is not None else None


class Oracle:
    """One mechanism loaded into the oracle."""

    def __init__(self, flat):
        self.flat = flat
        self.N = flat.n_species
        self.n = self.N + 1
        self._desc = flat.ctypes_desc()
        self._h = lib().orc_mech_new(ctypes.byref(self._desc))

    def __del__(self):
        try:
            if self._h:
                lib().orc_mech_free(self._h)
        except Exception:
            pass

    def rhs(self, y, F):
        y = np.ascontiguousarray(y, np.float64)
        F = np.ascontiguousarray(F, np.float64)
        out = np.empty_like(y)
        for idx in np.ndindex(y.shape[:-1]):
            yi, Fi, oi = y[idx], F[idx], np.empty(self.n)
            lib().orc_rhs(self._h, _p(yi), _p(Fi), _p(oi))
            out[idx] = oi
        return out

    def jac(self, y, F):
        y = np.ascontiguousarray(y, np.float64)
        F = np.ascontiguousarray(F, np.float64)
        out = np.empty(y.shape + (self.n,))
        for idx in np.ndindex(y.shape[:-1]):
            J = np.empty((self.n, self.n))
            lib().orc_jac(self._h, _p(np.ascontiguousarray(y[idx])), _p(np.ascontiguousarray(F[idx])), _p(J))
            out[idx] = J
        return out

    def wdot(self, T, C):
        out = np.empty(self.N)
        lib().orc_wdot(self._h, float(T), _p(np.ascontiguousarray(C, np.float64)), _p(out))
        return out

    def mix_h(self, T, Y):
        return lib().orc_mix_h(self._h, float(T), _p(np.ascontiguousarray(Y, np.float64)))

    def t_from_hy(self, h, Y, T0):
        T = np.array([T0], np.float64)
        it = lib().orc_t_from_hy(self._h, float(h), _p(np.ascontiguousarray(Y, np.float64)), _p(T))
        return float(T[0]), it

    def react(self, rhoY, frhoY, T, rhoH, frhoH, dt, rtol=1e-8, atol=1e-12, typ=None, mask=None,
              max_order=5, max_steps=10000, nthreads=0):
        """React a batch of cells.  rhoY/frhoY are [N, ncells] (component-major, like
        the flat ReactorBase::react); T/rhoH/frhoH are [ncells].  Arrays are copied;
        returns a dict with the new state, status, fctCount and per-cell counters."""
        N = self.N
        rhoY = np.array(rhoY, np.float64, order="C", copy=True)
        T = np.array(T, np.float64, copy=True)
        rhoH = np.array(rhoH, np.float64, copy=True)
        frhoY = np.ascontiguousarray(frhoY, np.float64)
        frhoH = np.ascontiguousarray(frhoH, np.float64)
        nc = T.shape[0]
        assert rhoY.shape == (N, nc) and frhoY.shape == (N, nc)
        if typ is None:
            atolv = np.full(self.n, atol)
        else:
            atolv = atol * np.asarray(typ, np.float64)
        status = np.zeros(nc, np.int32)
        fct = np.zeros(nc)
        cst = np.zeros((nc, 7), np.int32)
        m = None if mask is None else np.ascontiguousarray(mask, np.int32)
        o = OrcOpts(rtol, atol, max_order, max_steps, 0)
        nfail = lib().orc_react_batch(self._h, ctypes.byref(o), _p(atolv), _p(rhoY), _p(frhoY), _p(T),
                                      _p(rhoH), _p(frhoH), _p(fct), _p(m, _i32p), nc, float(dt),
                                      _p(status, _i32p), _p(cst, _i32p), int(nthreads))
        return dict(rhoY=rhoY, T=T, rhoH=rhoH, status=status, fct=fct, nfail=nfail,
                    nst=cst[:, 0], nfe=cst[:, 1], nje=cst[:, 2], nlu=cst[:, 3], netf=cst[:, 4],
                    ncfn=cst[:, 5], nni=cst[:, 6])


def max_threads() -> int:
    return lib().orc_max_threads()
