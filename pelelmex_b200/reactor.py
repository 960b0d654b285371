"""Python mirror of pele::physics::reactions::ReactorBase for the B200 reactor.

Lifecycle and argument meaning follow the reference call sites:

    ReactorBase::create(name)            Source/PeleLMeX_Setup.cpp:152-153
    init(reactor_type=2, ncells=1)       Source/PeleLMeX_Setup.cpp:146-154
    set_eos_parm(eos_parm)               Source/PeleLMeX_Setup.cpp:155
    set_typ_vals_ode(typ[N+1])           Source/PeleLMeX_Utils.cpp:1472
    react(box, rhoY, extF_rhoY, T, rhoH, extF_rhoH, fctCount, mask,
          dt_react, time, stream)        Source/PeleLMeX_Reactions.cpp:101-108
    close()                              Source/PeleLMeX.cpp:26

Arrays are CUDA tensors in CGS units (the caller converts from MKS as
Source/PeleLMeX_Reactions.cpp:69-79 does).  A "fab" is a tensor of shape
[ncomp, nz, ny, nx] (i fastest, like amrex::Array4) covering the box
``fab_lo .. fab_lo + (nx, ny, nz) - 1``; the box to react may be smaller.
On integration failure the reference aborts the run; here ``react`` raises
ReactorError (carrying the per-cell status) unless ``raise_on_failure`` is
False.  All the arithmetic runs in libb200chem.so; nothing here computes.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from pathlib import Path

from . import _lib
from . import mechanism as mechmod

REACTOR_NAMES = {}

CELL_STATUS = {0: "ok", 1: "masked", -1: "max_steps", -2: "error_test_failures", -3: "convergence_failures",
               -4: "nonfinite_input", -5: "singular_matrix"}


class ReactorError(RuntimeError):
    def __init__(self, msg, status=None, stats=None):
        super().__init__(msg)
        self.status = status
        self.stats = stats


def register(name):
    def deco(cls):
        REACTOR_NAMES[name] = cls
        return cls
    return deco


def create(name: str, **kw):
    """ReactorBase::create: build a reactor by its registered name."""
    if name not in REACTOR_NAMES:
        raise KeyError(f"unknown reactor {name!r}; known: {sorted(REACTOR_NAMES)}")
    return REACTOR_NAMES[name](**kw)


@dataclass
class Box:
    """amrex::Box: inclusive lo/hi cell indices."""
    lo: tuple
    hi: tuple

    @property
    def shape(self):
        return tuple(h - l + 1 for l, h in zip(self.lo, self.hi))

    @property
    def numPts(self):
        s = self.shape
        return s[0] * s[1] * s[2]


def _torch():
    import torch
    return torch


def array4(t, fab_lo=(0, 0, 0)) -> _lib.Array4:
    """An Array4 view of a [ncomp, nz, ny, nx] (or [nz, ny, nx]) CUDA tensor."""
    torch = _torch()
    if t is None:
        return _lib.Array4()
    if not t.is_cuda:
        raise ValueError("react() needs CUDA tensors (device memory)")
    if t.dim() == 3:
        t = t.unsqueeze(0)
    if t.dim() != 4:
        raise ValueError("fab tensors are [ncomp, nz, ny, nx]")
    if t.stride(3) != 1:
        raise ValueError("fab tensors must be contiguous along i")
    if t.dtype not in (torch.float64, torch.int32):
        raise ValueError("fab tensors are float64 (state) or int32 (mask)")
    a = _lib.Array4()
    a.p = t.data_ptr()
    a.jstride, a.kstride, a.nstride = t.stride(2), t.stride(1), t.stride(0)
    nz, ny, nx = t.shape[1], t.shape[2], t.shape[3]
    a.lo[:] = list(fab_lo)
    a.hi[:] = [fab_lo[0] + nx - 1, fab_lo[1] + ny - 1, fab_lo[2] + nz - 1]
    return a


@register("ReactorB200")
class ReactorB200:
    """Batched HP reactor on one B200 (warp-per-cell BDF, persistent kernel)."""

    # defaults of the reference's reactor keys (Docs/sphinx/manual/LMeXControls.rst:301-310)
    KERNELS = {"auto": 0, "thread": 1, "group": 2, "rounds": 3}

    def __init__(self, mechanism=None, rtol: float = 1e-10, atol: float = 1e-10, max_order: int = 2,
                 max_steps: int = 10000, lu_fp64: bool = False, refine_stall_ppm: int = 0, kernel: str = "auto",
                 setup_ratio: int = 0, ctas_per_sm: int = 0, group_lanes: int = 0, refine_keep_ppm: int = 0):
        if mechanism is None:
            raise ValueError("a mechanism (name of a bundled file, path, or Mechanism) is required")
        if isinstance(mechanism, str) and not Path(mechanism).exists():
            mechanism = mechmod.builtin(mechanism)
        elif isinstance(mechanism, (str, Path)):
            mechanism = mechmod.load(mechanism)
        self.mech = mechanism
        self.flat = mechmod.flatten(mechanism)
        self.N = self.flat.n_species
        self.opts = _lib.Opts(rtol, atol, max_order, max_steps, 2, 1 if lu_fp64 else 0, refine_stall_ppm, 0,
                              self.KERNELS[kernel], setup_ratio, ctas_per_sm, group_lanes, refine_keep_ppm, 0)
        self._h = None
        self._typ = None

    # ----------------------------------------------------------- lifecycle
    @classmethod
    def from_inputs(cls, params: dict):
        """Build from reference-style input keys (ParmParse names)."""
        name = params.get("peleLM.chem_integrator", "ReactorB200").strip('"')
        if name != "ReactorB200":
            raise KeyError(f"peleLM.chem_integrator = {name!r} is not this reactor")
        return cls(mechanism=params["b200.mechanism"], rtol=float(params.get("ode.rtol", 1e-10)),
                   atol=float(params.get("ode.atol", 1e-10)), max_order=int(params.get("cvode.max_order", 2)),
                   max_steps=int(params.get("cvode.max_substeps", 10000)),
                   lu_fp64=bool(int(params.get("b200.lu_fp64", 0))),
                   refine_stall_ppm=int(params.get("b200.refine_stall_ppm", 0)),
                   kernel=params.get("b200.kernel", "auto"), setup_ratio=int(params.get("b200.setup_ratio", 0)),
                   ctas_per_sm=int(params.get("b200.ctas_per_sm", 0)),
                   group_lanes=int(params.get("b200.group_lanes", 0)),
                   refine_keep_ppm=int(params.get("b200.refine_keep_ppm", 0)))

    def init(self, reactor_type: int = 2, ncells: int = 1):
        if reactor_type != 2:
            raise ValueError("only reactor_type 2 (HP) is supported")
        self.opts.reactor_type = reactor_type
        L = _lib.load()
        desc = self.flat.ctypes_desc()
        h = L.b200chem_create(ctypes.byref(desc), ctypes.byref(self.opts))
        if not h:
            raise _lib.B200ChemError(-1, L.b200chem_last_error().decode())
        self._h = h
        if self._typ is not None:
            self.set_typ_vals_ode(self._typ)
        return self

    def set_eos_parm(self, eos_parm=None):
        """The EOS is the mechanism's ideal-gas thermo; nothing to set."""
        return None

    def set_typ_vals_ode(self, typ):
        typ = [float(v) for v in typ]
        if len(typ) != self.N + 1:
            raise ValueError(f"need N+1 = {self.N + 1} typical values")
        self._typ = typ
        if self._h:
            arr = (ctypes.c_double * len(typ))(*typ)
            _lib.check(_lib.load().b200chem_set_typvals(self._h, arr, len(typ)))

    def kernel_launches(self) -> int:
        """Kernels this reactor has launched so far."""
        self._need()
        return int(_lib.load().b200chem_kernel_launches(self._h))

    TUNING_FIELDS = ("rhs_ctas_per_sm", "ctrl_ctas_per_sm", "jac_ctas_per_sm", "gj_ctas_per_sm",
                     "rounds_per_check", "use_graph", "rhs_form")

    def get_tuning(self) -> dict:
        """Launch shape of the round-based integrator (b200chem_tuning)."""
        self._need()
        t = _lib.Tuning()
        _lib.check(_lib.load().b200chem_get_tuning(self._h, ctypes.byref(t)))
        return {f: int(getattr(t, f)) for f in self.TUNING_FIELDS}

    def set_tuning(self, **fields):
        """Sets fields of the launch shape (the others keep their values)."""
        self._need()
        cur = self.get_tuning()
        for k, v in fields.items():
            if k not in cur:
                raise ValueError(f"unknown tuning field {k}")
            cur[k] = int(v)
        t = _lib.Tuning(**cur)
        _lib.check(_lib.load().b200chem_set_tuning(self._h, ctypes.byref(t)))

    def autotune(self, rhoY, extF_rhoY, T, rhoH, extF_rhoH, dt_react, max_trials=0, stream=None):
        """Times react on a copy of the given flat-layout cells under candidate
        launch shapes and keeps the fastest; returns (tuning dict, ms of one
        react of the sample).  The inputs are not modified."""
        self._need()
        torch = _torch()
        nc = T.shape[0]
        for t in (rhoY, extF_rhoY, T, rhoH, extF_rhoH):
            if not (t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()):
                raise ValueError("autotune needs contiguous float64 CUDA tensors")
        best = _lib.Tuning()
        ms = ctypes.c_double(0.0)
        _lib.check(_lib.load().b200chem_autotune(
            self._h, rhoY.data_ptr(), extF_rhoY.data_ptr(), T.data_ptr(), rhoH.data_ptr(), extF_rhoH.data_ptr(), nc,
            float(dt_react), int(max_trials), _stream_ptr(stream), ctypes.byref(best), ctypes.byref(ms)))
        return {f: int(getattr(best, f)) for f in self.TUNING_FIELDS}, float(ms.value)

    def save_tuning(self, path):
        """Writes the launch shape to a cache file keyed by mechanism and GPU."""
        self._need()
        _lib.check(_lib.load().b200chem_tuning_save(self._h, str(path).encode()))

    def load_tuning(self, path) -> bool:
        """Sets the launch shape from a cache file; False (and the shape
        unchanged) when the file is missing or was made for another
        mechanism or GPU."""
        self._need()
        if not Path(path).exists():
            return False
        return _lib.load().b200chem_tuning_load(self._h, str(path).encode()) == 0

    def profile_begin(self):
        """Per-kernel event timing of the following react calls (round-based
        integrator; kernels are then launched one by one, not from a graph)."""
        self._need()
        _lib.check(_lib.load().b200chem_profile_begin(self._h))

    def profile_end(self) -> dict:
        """{kind: {"launches", "cells", "ms"}} since profile_begin, kinds
        start / rhs / ctrl / jac / gj / ctrl_setup; plus "complete"."""
        self._need()
        p = _lib.KernelProfile()
        _lib.check(_lib.load().b200chem_profile_end(self._h, ctypes.byref(p)))
        out = {k: {"launches": int(p.launches[i]), "cells": int(p.cells[i]), "ms": float(p.ms[i])}
               for i, k in enumerate(_lib.PROF_KINDS)}
        out["complete"] = bool(p.complete)
        return out

    def close(self):
        if self._h:
            _lib.load().b200chem_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _need(self):
        if not self._h:
            raise RuntimeError("reactor not initialised: call init() first")

    # --------------------------------------------------------------- react
    def react(self, box: Box, rhoY, extF_rhoY, T, rhoH, extF_rhoH, fctCount, mask, dt_react: float,
              time: float = 0.0, stream=None, fab_lo=None, status=None, stats: bool = False,
              raise_on_failure: bool = True):
        """React one box (in place).  Returns (dt_react, time[, stats])."""
        return self.react_boxes([(box, rhoY, extF_rhoY, T, rhoH, extF_rhoH, fctCount, mask, fab_lo)], dt_react,
                                time, stream, status, stats, raise_on_failure)

    def react_boxes(self, items, dt_react, time=0.0, stream=None, status=None, stats=False,
                    raise_on_failure=True):
        """React a list of boxes in ONE persistent launch.  Each item is
        (box, rhoY, extF_rhoY, T, rhoH, extF_rhoH, fctCount, mask[, fab_lo])."""
        self._need()
        views = (_lib.BoxView * max(len(items), 1))()
        for b, it in enumerate(items):
            box, rY, fY, T, rH, fH, fc, mk = it[:8]
            flo = it[8] if len(it) > 8 and it[8] is not None else box.lo
            v = views[b]
            v.lo[:] = list(box.lo)
            v.hi[:] = list(box.hi)
            v.rhoY, v.extF_rhoY, v.T = array4(rY, flo), array4(fY, flo), array4(T, flo)
            v.rhoH, v.extF_rhoH = array4(rH, flo), array4(fH, flo)
            v.fctCount, v.mask = array4(fc, flo), array4(mk, flo)
            if rY.shape[0] != self.N:
                raise ValueError(f"rhoY has {rY.shape[0]} components, mechanism has {self.N}")
        return self._call_react(lambda dtp, tp, st, sp, stp: _lib.load().b200chem_react(
            self._h, views, len(items), dtp, tp, st, sp, stp), dt_react, time, stream, status, stats,
            raise_on_failure)

    def advance_chemistry(self, items, dt, stream=None, status=None, stats=False, raise_on_failure=True,
                          skip_react=None):
        """PeleLM::advanceChemistry's box body (Source/PeleLMeX_Reactions.cpp:31-175) for a
        list of boxes, MKS fabs: each item is (box, rhoY_old, rhoH_old, T_old, rhoY_new,
        rhoH_new, T_new, extF_rhoY, extF_rhoH, fctCount, mask, I_R[, fab_lo]); fctCount,
        mask and I_R may be None.  skip_react (one flag per box, optional) marks the
        covered boxes of advanceChemistryBAChem (m_baChemFlag == 0, :260-289): converted
        and given I_R, but not reacted (fctCount = 0).  Returns stats (dict) when asked,
        else None."""
        self._need()
        boxes = (_lib.ChemBox * max(len(items), 1))()
        if skip_react is not None and len(skip_react) != len(items):
            raise ValueError("skip_react needs one flag per box")
        for b, it in enumerate(items):
            box = it[0]
            flo = it[12] if len(it) > 12 and it[12] is not None else box.lo
            x = boxes[b]
            x.lo[:] = list(box.lo)
            x.hi[:] = list(box.hi)
            names = ("rhoY_old", "rhoH_old", "T_old", "rhoY_new", "rhoH_new", "T_new", "extF_rhoY", "extF_rhoH",
                     "fctCount", "mask", "I_R")
            for name, t in zip(names, it[1:12]):
                setattr(x, name, array4(t, flo))
            x.skip_react = 1 if (skip_react is not None and skip_react[b]) else 0
            if it[1].shape[0] != self.N or it[4].shape[0] != self.N:
                raise ValueError(f"rhoY has {it[1].shape[0]} components, mechanism has {self.N}")
        st_obj = _lib.Stats()
        code = _lib.load().b200chem_advance_chemistry(
            self._h, boxes, len(items), float(dt), _stream_ptr(stream),
            status.data_ptr() if status is not None else None, ctypes.byref(st_obj) if stats else None)
        s = st_obj.as_dict() if stats else None
        if code != 0 and (code != -4 or raise_on_failure):
            raise ReactorError(f"advance_chemistry failed ({code}): {_lib.load().b200chem_last_error().decode()}",
                               status=status, stats=s)
        return s

    def react_force(self, items, dt, stream=None):
        """PeleLM::getScalarReactForce (Source/PeleLMeX_Reactions.cpp:437-475) for a list
        of boxes, MKS fabs: each item is (box, rhoY_old, rhoH_old, rhoY_new, rhoH_new, I_R,
        extF_rhoY, extF_rhoH[, fab_lo]); the two forcing fabs are written."""
        self._need()
        boxes = (_lib.ForceBox * max(len(items), 1))()
        names = ("rhoY_old", "rhoH_old", "rhoY_new", "rhoH_new", "I_R", "extF_rhoY", "extF_rhoH")
        for b, it in enumerate(items):
            box = it[0]
            flo = it[8] if len(it) > 8 and it[8] is not None else box.lo
            x = boxes[b]
            x.lo[:] = list(box.lo)
            x.hi[:] = list(box.hi)
            for name, t in zip(names, it[1:8]):
                if t is None:
                    raise ValueError(f"react_force: {name} is required")
                setattr(x, name, array4(t, flo))
            for k in (1, 3, 5, 6):
                if it[k].shape[0] != self.N:
                    raise ValueError(f"{names[k - 1]} has {it[k].shape[0]} components, mechanism has {self.N}")
        _lib.check(_lib.load().b200chem_react_force(self._h, boxes, len(items), float(dt), _stream_ptr(stream)))

    def react_flat(self, rhoY, extF_rhoY, T, rhoH, extF_rhoH, fctCount=None, mask=None, dt_react=1e-6,
                   time=0.0, stream=None, status=None, stats=False, raise_on_failure=True):
        """Flat form: rhoY/extF_rhoY are [N, ncells] CUDA tensors (component-major)."""
        self._need()
        torch = _torch()
        nc = T.shape[0]
        for t in (rhoY, extF_rhoY, T, rhoH, extF_rhoH):
            if not (t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()):
                raise ValueError("flat react needs contiguous float64 CUDA tensors")
        if rhoY.shape != (self.N, nc) or extF_rhoY.shape != (self.N, nc):
            raise ValueError("rhoY/extF_rhoY must be [N, ncells]")
        if mask is not None and not (mask.is_cuda and mask.dtype == torch.int32):
            raise ValueError("mask must be an int32 CUDA tensor")
        fp = fctCount.data_ptr() if fctCount is not None else None
        mp = mask.data_ptr() if mask is not None else None
        return self._call_react(lambda dtp, tp, st, sp, stp: _lib.load().b200chem_react_flat(
            self._h, rhoY.data_ptr(), extF_rhoY.data_ptr(), T.data_ptr(), rhoH.data_ptr(), extF_rhoH.data_ptr(),
            fp, mp, nc, dtp, tp, st, sp, stp), dt_react, time, stream, status, stats, raise_on_failure)

    def _call_react(self, fn, dt_react, time, stream, status, stats, raise_on_failure):
        st_obj = _lib.Stats()
        dtp = ctypes.c_double(dt_react)
        tp = ctypes.c_double(time)
        st = _stream_ptr(stream)
        sp = status.data_ptr() if status is not None else None
        code = fn(ctypes.byref(dtp), ctypes.byref(tp), st, sp, ctypes.byref(st_obj) if stats else None)
        s = st_obj.as_dict() if stats else None
        if code != 0:
            msg = _lib.load().b200chem_last_error().decode()
            if code == -4 and not raise_on_failure:
                return (dtp.value, tp.value, s)
            raise ReactorError(f"react failed ({code}): {msg}", status=status, stats=s)
        if stats:
            return dtp.value, tp.value, s
        return dtp.value, tp.value

    # ------------------------------------------------ mechanism evaluations
    def eval_rhs(self, y, F, stream=None):
        """HP right-hand side for cell-major [ncells, N+1] CUDA tensors."""
        self._need()
        out = _torch().empty_like(y)
        _lib.check(_lib.load().b200chem_eval_rhs(self._h, y.data_ptr(), F.data_ptr(), y.shape[0], out.data_ptr(),
                                                 _stream_ptr(stream)))
        return out

    def eval_jac(self, y, F, stream=None):
        self._need()
        n = self.N + 1
        out = _torch().empty((y.shape[0], n, n), dtype=y.dtype, device=y.device)
        _lib.check(_lib.load().b200chem_eval_jac(self._h, y.data_ptr(), F.data_ptr(), y.shape[0], out.data_ptr(),
                                                 _stream_ptr(stream)))
        return out

    def inst_rr(self, rhoY_mks, rhoH_mks, T, stream=None):
        """reactionRateRhoY (Source/PeleLMeX_K.H:850-889): returns rhoYdot [N, ncells] (MKS); T updated."""
        self._need()
        out = _torch().empty_like(rhoY_mks)
        _lib.check(_lib.load().b200chem_inst_rr(self._h, rhoY_mks.data_ptr(), rhoH_mks.data_ptr(), T.data_ptr(),
                                                out.data_ptr(), T.shape[0], _stream_ptr(stream)))
        return out

    def t_from_hy(self, rhoY_mks, rhoH_mks, T, stream=None):
        """getTfromHY (Source/PeleLMeX_K.H:700-723), T updated in place."""
        self._need()
        _lib.check(_lib.load().b200chem_t_from_hy(self._h, rhoY_mks.data_ptr(), rhoH_mks.data_ptr(), T.data_ptr(),
                                                  T.shape[0], _stream_ptr(stream)))
        return T

    def h_given_t(self, T, stream=None):
        """getHGivenT (Source/PeleLMeX_K.H:598-615): [N, ncells] species enthalpies, J/kg."""
        self._need()
        Hi = _torch().empty((self.N, T.shape[0]), dtype=T.dtype, device=T.device)
        _lib.check(_lib.load().b200chem_h_given_t(self._h, T.data_ptr(), Hi.data_ptr(), T.shape[0],
                                                  _stream_ptr(stream)))
        return Hi

    def heat_release(self, T, I_R, stream=None):
        """getHeatRelease (Source/PeleLMeX_Reactions.cpp:477-506): [ncells] HRR, W/m^3."""
        self._need()
        if I_R.shape != (self.N, T.shape[0]) or not I_R.is_contiguous():
            raise ValueError("I_R must be a contiguous [N, ncells] tensor")
        HR = _torch().empty_like(T)
        _lib.check(_lib.load().b200chem_heat_release(self._h, T.data_ptr(), I_R.data_ptr(), HR.data_ptr(), T.shape[0],
                                                     _stream_ptr(stream)))
        return HR


def _stream_ptr(stream):
    if stream is None:
        torch = _torch()
        return torch.cuda.current_stream().cuda_stream
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream
