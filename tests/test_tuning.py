"""Launch tuning of the round-based integrator: every launch shape
(CUDA-graph replay or stream launches, rounds between live-count checks,
CTAs per SM of each kernel, right-hand-side form) integrates the same cells
to the same result within the reactor's parity tolerances, and the
autotuner returns a valid shape without touching its inputs."""
import ctypes

import numpy as np
import pytest

from pelelmex_b200 import _lib


def test_tuning_struct_layout():
    assert ctypes.sizeof(_lib.Tuning) == 8 * 4


def test_tuning_rejects_null_handle_without_gpu():
    L = _lib.load()
    t = _lib.Tuning()
    assert L.b200chem_get_tuning(None, ctypes.byref(t)) == -1
    assert L.b200chem_set_tuning(None, ctypes.byref(t)) == -1
    assert L.b200chem_autotune(None, None, None, None, None, None, 0, 1e-6, 0, None, None, None) == -1


torch = pytest.importorskip("torch")

SHAPES = [
    dict(use_graph=2),
    dict(use_graph=1, rounds_per_check=2),
    dict(use_graph=1, rounds_per_check=16),
    dict(rhs_ctas_per_sm=1, ctrl_ctas_per_sm=1, jac_ctas_per_sm=1, gj_ctas_per_sm=1),
    dict(rhs_form=1),
    dict(rhs_form=2),
]


def _field(n, seed):
    from pelelmex_b200 import mechanism as M, workloads as W
    mech = M.builtin("synth_ch4_21")
    return W.flame_ch4(mech, cells=W.sample_cells(128 ** 3, n, seed=seed), dt=1e-5)


def _run(f, shape=None, autotune=False):
    from pelelmex_b200.reactor import ReactorB200
    dev = torch.device("cuda:0")
    r = ReactorB200("synth_ch4_21", rtol=1e-8, atol=1e-12, kernel="rounds").init(2, f.ncells)
    d = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)  # noqa: E731
    rhoY, T, rhoH, fY, fH = d(f.rhoY), d(f.T), d(f.rhoH), d(f.frhoY), d(f.frhoH)
    tuned = None
    if autotune:
        before = [x.clone() for x in (rhoY, T, rhoH)]
        tuned = r.autotune(rhoY, fY, T, rhoH, fH, f.dt, max_trials=24)
        for a, b in zip(before, (rhoY, T, rhoH)):
            assert torch.equal(a, b), "autotune modified its inputs"
    if shape:
        r.set_tuning(**shape)
    fct = torch.zeros(f.ncells, dtype=torch.float64, device=dev)
    st = torch.zeros(f.ncells, dtype=torch.int32, device=dev)
    n0 = r.kernel_launches()
    r.react_flat(rhoY, fY, T, rhoH, fH, fct, dt_react=f.dt, status=st)
    torch.cuda.synchronize()
    out = dict(rhoY=rhoY.cpu().numpy(), T=T.cpu().numpy(), fct=fct.cpu().numpy(), status=st.cpu().numpy(),
               launches=r.kernel_launches() - n0, tuning=r.get_tuning(), tuned=tuned)
    r.close()
    return out


def _same(f, a, b):
    assert (a["status"] == 0).all() and (b["status"] == 0).all()
    assert np.max(np.abs(a["T"] - b["T"]) / b["T"]) <= 1e-5
    rho = f.rhoY.sum(axis=0)
    assert (np.abs(a["rhoY"] - b["rhoY"]).max(axis=0) / rho).max() <= 1e-8
    assert abs(a["fct"].mean() - b["fct"].mean()) <= 0.02 * b["fct"].mean()


@pytest.mark.gpu
@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: ",".join(f"{k}={v}" for k, v in s.items()))
def test_launch_shapes_agree(shape):
    f = _field(4096, 5)
    ref = _run(f)
    got = _run(f, shape)
    for k, v in shape.items():
        assert got["tuning"][k] == v
    _same(f, got, ref)
    assert got["launches"] > 0


@pytest.mark.gpu
def test_set_tuning_rejects_out_of_range():
    from pelelmex_b200.reactor import ReactorB200
    r = ReactorB200("synth_ch4_21", kernel="rounds").init(2, 16)
    for bad in (dict(rounds_per_check=3), dict(use_graph=5), dict(rhs_form=7), dict(ctrl_ctas_per_sm=-1)):
        with pytest.raises(_lib.B200ChemError):
            r.set_tuning(**bad)
    r.close()


@pytest.mark.gpu
def test_autotune_valid_and_same_results():
    f = _field(16384, 9)
    ref = _run(f)
    got = _run(f, autotune=True)
    tuning, ms = got["tuned"]
    assert ms > 0.0
    assert tuning["rounds_per_check"] in (0, 2, 4, 8, 16) and tuning["use_graph"] in (0, 1, 2)
    assert got["tuning"] == tuning
    _same(f, got, ref)


@pytest.mark.gpu
def test_kernel_profile_counts_match_integrator_counters():
    from pelelmex_b200.reactor import ReactorB200
    f = _field(4096, 13)
    dev = torch.device("cuda:0")
    r = ReactorB200("synth_ch4_21", rtol=1e-8, atol=1e-12, kernel="rounds").init(2, f.ncells)
    d = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)  # noqa: E731
    rhoY, T, rhoH, fY, fH = d(f.rhoY), d(f.T), d(f.rhoH), d(f.frhoY), d(f.frhoH)
    r.profile_begin()
    _, _, st = r.react_flat(rhoY, fY, T, rhoH, fH, dt_react=f.dt, stats=True)
    p = r.profile_end()
    assert p["complete"]
    assert p["start"]["launches"] == 1 and p["start"]["cells"] == f.ncells
    rounds = p["rhs"]["launches"]
    assert rounds >= st["max_nfe"] and all(p[k]["launches"] == rounds for k in ("ctrl", "jac", "gj", "ctrl_setup"))
    # every right-hand side is consumed by one control pass; every setup by one inverse and control pass;
    # the Jacobian kernel sees only the setups whose Jacobian is recomputed
    assert p["rhs"]["cells"] == p["ctrl"]["cells"] == st["nfe"]
    assert p["gj"]["cells"] == p["ctrl_setup"]["cells"] == st["nlu"]
    assert p["jac"]["cells"] == st["nje"]
    assert all(p[k]["ms"] > 0 for k in ("start", "rhs", "ctrl", "gj"))
    # profiling changes the launch mode only, not the result
    rY2, T2, rH2 = d(f.rhoY), d(f.T), d(f.rhoH)
    r.react_flat(rY2, fY, T2, rH2, fH, dt_react=f.dt)
    torch.cuda.synchronize()
    assert torch.equal(T, T2) and torch.equal(rhoY, rY2)
    r.close()


@pytest.mark.gpu
def test_tuning_cache_round_trip_and_keys(tmp_path):
    """The launch-shape cache keeps a tuning per (mechanism, GPU): a second
    handle of the same mechanism loads it; another mechanism is refused."""
    from pelelmex_b200.reactor import ReactorB200
    a = ReactorB200("synth_ch4_21", rtol=1e-8, atol=1e-12, max_order=5).init()
    b = ReactorB200("synth_ch4_21", rtol=1e-8, atol=1e-12, max_order=5).init()
    c = ReactorB200("synth_h2_9", rtol=1e-8, atol=1e-12, max_order=5).init()
    try:
        a.set_tuning(rhs_ctas_per_sm=3, rounds_per_check=8, use_graph=2)
        path = tmp_path / "ch4.b2t"
        a.save_tuning(path)
        assert b.get_tuning() != a.get_tuning()
        assert b.load_tuning(path)
        assert b.get_tuning() == a.get_tuning()
        before = c.get_tuning()
        assert not c.load_tuning(path)
        assert c.get_tuning() == before
        assert not b.load_tuning(tmp_path / "missing.b2t")
    finally:
        for r in (a, b, c):
            r.close()
