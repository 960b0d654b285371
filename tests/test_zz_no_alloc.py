"""Allocation-free react entry point (b200chem_react_flat_noalloc) against the
allocating one (b200chem_react_flat), both called through the C ABI.

Two chemistry steps in a row on each path from the same seeded state: the
states after each step, the per-cell status and the integrator counters must
agree (same tolerances as the oracle parity tests; the per-cell arithmetic is
the same, so they normally agree bit for bit).  A mechanism whose integrator
scratch does not fit the fixed scratch must be rejected with an error.
This file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from pelelmex_b200 import _lib, workloads as W  # noqa: E402
from pelelmex_b200 import mechanism as M  # noqa: E402
from pelelmex_b200.reactor import ReactorB200  # noqa: E402

T_RTOL = 1e-5
Y_ATOL = 1e-8
DEV = "cuda:0"
_f64p = ctypes.POINTER(ctypes.c_double)


def _fn(L, name):
    f = getattr(L, name)
    f.argtypes = [ctypes.c_void_p, _f64p, _f64p, _f64p, _f64p, _f64p, _f64p, ctypes.c_void_p, ctypes.c_int64,
                  ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double), ctypes.c_void_p,
                  ctypes.c_void_p, ctypes.POINTER(_lib.Stats)]
    f.restype = ctypes.c_int
    return f


def _p(t):
    return ctypes.cast(t.data_ptr(), _f64p)


def _steps(fn, r, f, nsteps=2):
    """nsteps react calls in a row; returns the state, status and counters after each."""
    rhoY, T, rhoH, fY, fH = (torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device=DEV)
                             for a in (f.rhoY, f.T, f.rhoH, f.frhoY, f.frhoH))
    fct = torch.zeros(f.ncells, dtype=torch.float64, device=DEV)
    status = torch.zeros(f.ncells, dtype=torch.int32, device=DEV)
    stream = torch.cuda.current_stream().cuda_stream
    out = []
    for _ in range(nsteps):
        dt = ctypes.c_double(f.dt)
        tm = ctypes.c_double(0.0)
        st = _lib.Stats()
        code = fn(r._h, _p(rhoY), _p(fY), _p(T), _p(rhoH), _p(fH), _p(fct), None, f.ncells, ctypes.byref(dt),
                  ctypes.byref(tm), stream, status.data_ptr(), ctypes.byref(st))
        assert code == 0, _lib.load().b200chem_last_error().decode()
        torch.cuda.synchronize()
        assert tm.value == pytest.approx(f.dt)
        out.append(dict(rhoY=rhoY.cpu().numpy(), T=T.cpu().numpy(), rhoH=rhoH.cpu().numpy(),
                        status=status.cpu().numpy(), stats=st.as_dict()))
    return out


@pytest.mark.parametrize("name,make", [
    ("synth_h2_9", lambda m: W.premixed_h2(m, edge=16)),
    ("synth_ch4_21", lambda m: W.flame_ch4(m, cells=W.sample_cells(128 ** 3, 4096), dt=1e-6)),
])
def test_noalloc_matches_react_flat(name, make):
    L = _lib.load()
    flat_fn, noalloc_fn = _fn(L, "b200chem_react_flat"), _fn(L, "b200chem_react_flat_noalloc")
    mech = M.builtin(name)
    f = make(mech)
    # the allocation-free entry point runs the group integrator: compare like with like
    r = ReactorB200(name, rtol=1e-8, atol=1e-12, max_order=5, kernel="group").init(2, f.ncells)
    try:
        ref = _steps(flat_fn, r, f)
        got = _steps(noalloc_fn, r, f)
    finally:
        r.close()
    for a, b in zip(ref, got):
        assert (a["status"] == 0).all() and (b["status"] == 0).all()
        np.testing.assert_allclose(b["T"], a["T"], rtol=T_RTOL, atol=0)
        Ya = a["rhoY"] / a["rhoY"].sum(axis=0)
        Yb = b["rhoY"] / b["rhoY"].sum(axis=0)
        assert np.abs(Yb - Ya).max() <= Y_ATOL
        # the counters start from zero on every call
        for k in ("n_cells", "n_failed", "nst", "nfe", "nje", "nlu"):
            assert b["stats"][k] == a["stats"][k], k
    assert got[0]["stats"]["n_cells"] == f.ncells and got[1]["stats"]["n_cells"] == f.ncells


def test_noalloc_rejects_oversized_scratch():
    # dodecane-sized mechanism on 16 lanes per cell: 8 groups x 33 KB per CTA,
    # more than the fixed scratch holds for one CTA on every SM
    L = _lib.load()
    noalloc_fn = _fn(L, "b200chem_react_flat_noalloc")
    name = "synth_c12_53"
    mech = M.builtin(name)
    N = mech.n_species
    r = ReactorB200(name, rtol=1e-8, atol=1e-12, max_order=5, group_lanes=16).init(2, 64)
    try:
        z = torch.zeros((N, 64), dtype=torch.float64, device=DEV)
        v = torch.full((64,), 1000.0, dtype=torch.float64, device=DEV)
        dt = ctypes.c_double(1e-6)
        code = noalloc_fn(r._h, _p(z), _p(z), _p(v), _p(v), _p(v), None, None, 64, ctypes.byref(dt), None,
                          torch.cuda.current_stream().cuda_stream, None, None)
        torch.cuda.synchronize()
        assert code == -5
        assert "scratch" in L.b200chem_last_error().decode()
    finally:
        r.close()


@pytest.mark.parametrize("kernel", ["thread", "rounds"])
def test_noalloc_rejects_other_integrators(kernel):
    # only the group integrator has an allocation-free form; a handle built for
    # another integrator is refused rather than silently run on the group one
    L = _lib.load()
    noalloc_fn = _fn(L, "b200chem_react_flat_noalloc")
    mech = M.builtin("synth_h2_9")
    f = W.premixed_h2(mech, edge=4)
    r = ReactorB200("synth_h2_9", rtol=1e-8, atol=1e-12, max_order=5, kernel=kernel).init(2, f.ncells)
    try:
        with pytest.raises(AssertionError, match="group integrator only"):
            _steps(noalloc_fn, r, f, nsteps=1)
    finally:
        r.close()


def test_noalloc_counts_its_launches():
    L = _lib.load()
    noalloc_fn = _fn(L, "b200chem_react_flat_noalloc")
    mech = M.builtin("synth_h2_9")
    f = W.premixed_h2(mech, edge=4)
    r = ReactorB200("synth_h2_9", rtol=1e-8, atol=1e-12, max_order=5, kernel="group").init(2, f.ncells)
    try:
        n0 = r.kernel_launches()
        _steps(noalloc_fn, r, f, nsteps=1)
        # the box-descriptor store and the integrator
        assert r.kernel_launches() - n0 == 2
    finally:
        r.close()
