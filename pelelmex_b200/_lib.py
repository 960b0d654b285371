"""Loader and ctypes declarations for the in-tree CUDA library libb200chem.so.

The library is the product: there is no CPU or library fallback.  If it is
missing or fails to load, every entry point raises.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libb200chem.so"

_i32p = ctypes.POINTER(ctypes.c_int32)
_f64p = ctypes.c_void_p  # device pointers are passed as integers


class Opts(ctypes.Structure):
    _fields_ = [("rtol", ctypes.c_double), ("atol", ctypes.c_double), ("max_order", ctypes.c_int32),
                ("max_steps", ctypes.c_int32), ("reactor_type", ctypes.c_int32), ("lu_fp64", ctypes.c_int32),
                ("refine_stall_ppm", ctypes.c_int32), ("verbose", ctypes.c_int32), ("kernel", ctypes.c_int32),
                ("setup_ratio", ctypes.c_int32), ("ctas_per_sm", ctypes.c_int32),
                ("group_lanes", ctypes.c_int32), ("refine_keep_ppm", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class Array4(ctypes.Structure):
    _fields_ = [("p", ctypes.c_void_p), ("jstride", ctypes.c_int64), ("kstride", ctypes.c_int64),
                ("nstride", ctypes.c_int64), ("lo", ctypes.c_int32 * 3), ("hi", ctypes.c_int32 * 3)]


class BoxView(ctypes.Structure):
    _fields_ = [("lo", ctypes.c_int32 * 3), ("hi", ctypes.c_int32 * 3), ("rhoY", Array4), ("extF_rhoY", Array4),
                ("T", Array4), ("rhoH", Array4), ("extF_rhoH", Array4), ("fctCount", Array4), ("mask", Array4)]


class ChemBox(ctypes.Structure):
    _fields_ = [("lo", ctypes.c_int32 * 3), ("hi", ctypes.c_int32 * 3), ("rhoY_old", Array4), ("rhoH_old", Array4),
                ("T_old", Array4), ("rhoY_new", Array4), ("rhoH_new", Array4), ("T_new", Array4),
                ("extF_rhoY", Array4), ("extF_rhoH", Array4), ("fctCount", Array4), ("mask", Array4),
                ("I_R", Array4), ("skip_react", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class ForceBox(ctypes.Structure):
    _fields_ = [("lo", ctypes.c_int32 * 3), ("hi", ctypes.c_int32 * 3), ("rhoY_old", Array4), ("rhoH_old", Array4),
                ("rhoY_new", Array4), ("rhoH_new", Array4), ("I_R", Array4), ("extF_rhoY", Array4),
                ("extF_rhoH", Array4)]


class Stats(ctypes.Structure):
    _fields_ = [("n_cells", ctypes.c_int64), ("n_masked", ctypes.c_int64), ("n_failed", ctypes.c_int64),
                ("nst", ctypes.c_int64), ("nfe", ctypes.c_int64), ("nje", ctypes.c_int64), ("nlu", ctypes.c_int64),
                ("netf", ctypes.c_int64), ("ncfn", ctypes.c_int64), ("max_nfe", ctypes.c_int32),
                ("max_nst", ctypes.c_int32), ("n_fp64_retry", ctypes.c_int64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class HybridOpts(ctypes.Structure):
    _fields_ = [("t_rel", ctypes.c_double), ("spread", ctypes.c_double), ("dT_cap", ctypes.c_double),
                ("gap", ctypes.c_double), ("tol_elem", ctypes.c_double), ("tol_mass", ctypes.c_double),
                ("resid", ctypes.c_double), ("min_members", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class HybridStats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int64) for n in (
        "predicted", "accepted", "rejected_spread", "rejected_cap", "rejected_mass", "rejected_elements",
        "rejected_energy", "rejected_negative", "rejected_residual", "rejected_nonfinite")]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Tuning(ctypes.Structure):
    _fields_ = [("rhs_ctas_per_sm", ctypes.c_int32), ("ctrl_ctas_per_sm", ctypes.c_int32),
                ("jac_ctas_per_sm", ctypes.c_int32), ("gj_ctas_per_sm", ctypes.c_int32),
                ("rounds_per_check", ctypes.c_int32), ("use_graph", ctypes.c_int32), ("rhs_form", ctypes.c_int32),
                ("reserved", ctypes.c_int32)]


PROF_KINDS = ("start", "rhs", "ctrl", "jac", "gj", "ctrl_setup")


class KernelProfile(ctypes.Structure):
    _fields_ = [("launches", ctypes.c_int64 * 8), ("cells", ctypes.c_int64 * 8), ("ms", ctypes.c_double * 8),
                ("complete", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class B200ChemError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"b200chem error {code}: {msg}")
        self.code = code


_lib = None


def load(path: os.PathLike | None = None):
    """Load libb200chem.so (raises if it is missing: no fallback exists)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else Path(os.environ.get("B200CHEM_LIB", LIB_PATH))
    if not p.exists():
        raise FileNotFoundError(f"{p} not built; run __graft_entry__.build() or python -m pelelmex_b200.build")
    L = ctypes.CDLL(str(p))
    from .mechanism import MechDesc
    L.b200chem_version.restype = ctypes.c_int
    L.b200chem_last_error.restype = ctypes.c_char_p
    L.b200chem_create.restype = ctypes.c_void_p
    L.b200chem_create.argtypes = [ctypes.POINTER(MechDesc), ctypes.POINTER(Opts)]
    L.b200chem_set_typvals.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_int32]
    L.b200chem_react.argtypes = [ctypes.c_void_p, ctypes.POINTER(BoxView), ctypes.c_int32,
                                 ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double), ctypes.c_void_p,
                                 ctypes.c_void_p, ctypes.POINTER(Stats)]
    L.b200chem_react_flat.argtypes = [ctypes.c_void_p, _f64p, _f64p, _f64p, _f64p, _f64p, _f64p, ctypes.c_void_p,
                                      ctypes.c_int64, ctypes.POINTER(ctypes.c_double),
                                      ctypes.POINTER(ctypes.c_double), ctypes.c_void_p, ctypes.c_void_p,
                                      ctypes.POINTER(Stats)]
    L.b200chem_destroy.argtypes = [ctypes.c_void_p]
    L.b200chem_mlp_gemm_bf16.argtypes = [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_void_p, ctypes.c_longlong,
                                         ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_longlong,
                                         ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_void_p, ctypes.c_void_p]
    L.b200chem_mlp_gemm_bf16.restype = ctypes.c_int
    L.b200chem_mlp_adam.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                    ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                    ctypes.c_float, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    L.b200chem_mlp_adam.restype = ctypes.c_int
    L.b200chem_surrogate_features.argtypes = [ctypes.c_void_p, _f64p, _f64p, ctypes.c_int64, ctypes.c_int64,
                                              ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32,
                                              ctypes.c_void_p, ctypes.c_void_p]
    L.b200chem_surrogate_features.restype = ctypes.c_int
    L.b200chem_surrogate_load.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t]
    L.b200chem_surrogate_load.restype = ctypes.c_void_p
    L.b200chem_surrogate_load_file.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
    L.b200chem_surrogate_load_file.restype = ctypes.c_void_p
    L.b200chem_surrogate_get_opts.argtypes = [ctypes.c_void_p, ctypes.POINTER(HybridOpts)]
    L.b200chem_surrogate_get_opts.restype = ctypes.c_int
    L.b200chem_surrogate_destroy.argtypes = [ctypes.c_void_p]
    L.b200chem_surrogate_destroy.restype = ctypes.c_int
    L.b200chem_surrogate_infer.argtypes = [ctypes.c_void_p, _f64p, _f64p, ctypes.c_int64, ctypes.c_double, _f64p,
                                           _f64p, ctypes.c_void_p]
    L.b200chem_surrogate_infer.restype = ctypes.c_int
    L.b200chem_react_hybrid.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(HybridOpts), _f64p, _f64p,
                                        _f64p, _f64p, _f64p, _f64p, ctypes.c_void_p, ctypes.c_int64,
                                        ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                                        ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(Stats),
                                        ctypes.POINTER(HybridStats)]
    L.b200chem_react_hybrid.restype = ctypes.c_int
    L.b200chem_kernel_launches.argtypes = [ctypes.c_void_p]
    L.b200chem_kernel_launches.restype = ctypes.c_int64
    L.b200chem_get_tuning.argtypes = [ctypes.c_void_p, ctypes.POINTER(Tuning)]
    L.b200chem_set_tuning.argtypes = [ctypes.c_void_p, ctypes.POINTER(Tuning)]
    L.b200chem_autotune.argtypes = [ctypes.c_void_p, _f64p, _f64p, _f64p, _f64p, _f64p, ctypes.c_int64,
                                    ctypes.c_double, ctypes.c_int32, ctypes.c_void_p, ctypes.POINTER(Tuning),
                                    ctypes.POINTER(ctypes.c_double)]
    L.b200chem_advance_chemistry.argtypes = [ctypes.c_void_p, ctypes.POINTER(ChemBox), ctypes.c_int32,
                                             ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    L.b200chem_advance_chemistry.restype = ctypes.c_int
    L.b200chem_react_force.argtypes = [ctypes.c_void_p, ctypes.POINTER(ForceBox), ctypes.c_int32, ctypes.c_double,
                                       ctypes.c_void_p]
    L.b200chem_react_force.restype = ctypes.c_int
    L.b200chem_mechanism_digest.argtypes = [ctypes.POINTER(MechDesc)]
    L.b200chem_mechanism_digest.restype = ctypes.c_uint64
    L.b200chem_generated_species.argtypes = [ctypes.c_uint64]
    L.b200chem_generated_species.restype = ctypes.c_int
    L.b200chem_selftest_bounded_wait.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
    L.b200chem_selftest_bounded_wait.restype = ctypes.c_int
    L.b200chem_profile_begin.argtypes = [ctypes.c_void_p]
    L.b200chem_profile_end.argtypes = [ctypes.c_void_p, ctypes.POINTER(KernelProfile)]
    L.b200chem_tuning_save.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
    L.b200chem_tuning_load.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
    for name in ("b200chem_get_tuning", "b200chem_set_tuning", "b200chem_autotune", "b200chem_profile_begin",
                 "b200chem_profile_end", "b200chem_tuning_save", "b200chem_tuning_load"):
        getattr(L, name).restype = ctypes.c_int
    for name in ("b200chem_eval_rhs", "b200chem_eval_jac"):
        f = getattr(L, name)
        f.argtypes = [ctypes.c_void_p, _f64p, _f64p, ctypes.c_int64, _f64p, ctypes.c_void_p]
    L.b200chem_inst_rr.argtypes = [ctypes.c_void_p, _f64p, _f64p, _f64p, _f64p, ctypes.c_int64, ctypes.c_void_p]
    L.b200chem_t_from_hy.argtypes = [ctypes.c_void_p, _f64p, _f64p, _f64p, ctypes.c_int64, ctypes.c_void_p]
    L.b200chem_h_given_t.argtypes = [ctypes.c_void_p, _f64p, _f64p, ctypes.c_int64, ctypes.c_void_p]
    L.b200chem_heat_release.argtypes = [ctypes.c_void_p, _f64p, _f64p, _f64p, ctypes.c_int64, ctypes.c_void_p]
    L.b200chem_h_given_t.restype = ctypes.c_int
    L.b200chem_heat_release.restype = ctypes.c_int
    for name in ("b200chem_set_typvals", "b200chem_react", "b200chem_react_flat", "b200chem_destroy",
                 "b200chem_eval_rhs", "b200chem_eval_jac", "b200chem_inst_rr", "b200chem_t_from_hy"):
        getattr(L, name).restype = ctypes.c_int
    if path is None:
        _lib = L
    return L


def check(code: int):
    if code != 0:
        raise B200ChemError(code, load().b200chem_last_error().decode())
    return code
