"""Surrogate MLP: the FP64 oracle of the network against finite differences
(CPU), the tensor-core forward pass and gradients against that oracle
(GPU), training, and the hybrid (surrogate + gated BDF fallback) reactor
against the plain BDF."""
import numpy as np
import pytest

import mlp_np  # oracle/mlp_np.py (the oracle directory is on sys.path)


def _small_params(rng, dims):
    return [(rng.normal(0, 1 / np.sqrt(i), (o, i)), rng.normal(0, 0.1, o)) for o, i in dims]


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    params = _small_params(rng, [(8, 5), (8, 8), (3, 8)])
    x = rng.normal(size=(6, 5))
    t = rng.normal(size=(6, 3))
    w = np.array([2.0, 1.0, 1.0])
    L, grads = mlp_np.loss_and_grads(params, x, t, w)
    for li in range(3):
        for which in (0, 1):
            arr = params[li][which]
            for idx in [tuple(rng.integers(0, s) for s in arr.shape) for _ in range(3)]:
                fd = mlp_np.finite_difference(params, x, t, w, li, which, idx)
                an = grads[li][which][idx]
                assert abs(fd - an) <= 1e-6 * max(1.0, abs(fd))


# ----------------------------------------------------------------- GPU
torch = pytest.importorskip("torch")


def _bf(a):
    return torch.tensor(a, dtype=torch.float32).to(torch.bfloat16).float().double().numpy()


def _oracle_params(s):
    """FP64 copies of the device BF16 weights (padded shapes)."""
    return [(s.Wb[i].float().double().cpu().numpy(), s.b[i].double().cpu().numpy()) for i in range(4)]


def _net_input(x, terms):
    """Network input of a FP32 [B, kin] matrix: one BF16 term, or two (hi | lo)."""
    hi = x.to(torch.bfloat16)
    if terms == 1:
        return hi, hi.float().double().cpu().numpy()
    lo = (x - hi.float()).to(torch.bfloat16)
    return torch.cat([hi, lo], dim=1), (hi.float().double() + lo.float().double()).cpu().numpy()


@pytest.mark.gpu
@pytest.mark.parametrize("terms,tol", [(1, 3e-2), (2, 3e-3)])
def test_forward_and_gradients_match_oracle(terms, tol):
    """BF16 weights, FP32 accumulation; activations between layers in one
    BF16 term (a few percent of the output range) or two (limited by the
    hardware tanh of GELU, ~1e-3)."""
    from pelelmex_b200.surrogate import MLPSurrogate
    s = MLPSurrogate("synth_ch4_21", seed=3, terms=terms)
    B = 512
    g = torch.Generator(device="cuda:0").manual_seed(1)
    x = torch.randn((B, s.kin), device="cuda:0", generator=g)
    x[:, s.nin:] = 0
    xb, xo = _net_input(x, terms)
    target = torch.randn((B, s.nout), device="cuda:0", generator=g)
    w = torch.ones(s.nout, device="cuda:0")
    w[0] = 4.0
    y = s.forward(xb)
    torch.cuda.synchronize()
    s.check_error()
    P = _oracle_params(s)
    yo, _ = mlp_np.forward(P, xo)
    err = np.abs(y.cpu().numpy()[:, :s.nout] - yo[:, :s.nout]).max() / np.abs(yo[:, :s.nout]).max()
    assert err < tol, err
    loss, dW, db = s.loss_and_grads(xb, target, w)
    torch.cuda.synchronize()
    s.check_error()
    tpad = np.zeros((B, s.kout))
    tpad[:, :s.nout] = target.cpu().numpy()
    wpad = np.zeros(s.kout)
    wpad[:s.nout] = w.cpu().numpy()
    Lo, go = mlp_np.loss_and_grads(P, xo, tpad, wpad)
    assert abs(float(loss) - Lo) <= 2e-2 * Lo
    for li in range(4):
        gw = dW[li].double().cpu().numpy()
        gb = db[li].double().cpu().numpy()
        rel_w = np.linalg.norm(gw - go[li][0]) / np.linalg.norm(go[li][0])
        rel_b = np.linalg.norm(gb - go[li][1]) / np.linalg.norm(go[li][1])
        assert rel_w < 5e-2 and rel_b < 5e-2, (li, rel_w, rel_b)


@pytest.mark.gpu
def test_training_reduces_loss_on_a_smooth_map():
    from pelelmex_b200.surrogate import MLPSurrogate
    s = MLPSurrogate("synth_ch4_21", seed=0)
    S = 16384
    g = torch.Generator(device="cuda:0").manual_seed(2)
    x = torch.randn((S, s.kin), device="cuda:0", generator=g)
    x[:, s.nin:] = 0
    y = torch.stack([torch.sin(x[:, j % s.nin]) * torch.cos(x[:, (3 * j + 1) % s.nin]) for j in range(s.nout)], 1)
    hist = s.train(_net_input(x, s.terms)[0], y, steps=300, batch=2048, lr=2e-3, log_every=50)
    assert hist[-1][1] < 0.35 * hist[0][1], hist


def _weights():
    from pathlib import Path
    return Path(__file__).resolve().parent.parent / "pelelmex_b200" / "surrogates" / "synth_ch4_21.b2s"


def test_weights_file_header_and_round_trip():
    """The committed weights file parses on the host (no GPU): magic, version,
    mechanism digest, dimensions, the element matrix, and a byte-exact round
    trip through the Python writer."""
    import struct
    from pelelmex_b200 import mechanism as M, mechgen
    from pelelmex_b200.surrogate import Ensemble, FILE_VERSION, MAGIC, element_matrix
    data = _weights().read_bytes()
    assert data[:8] == MAGIC
    version, hbytes = struct.unpack_from("<II", data, 8)
    assert version == FILE_VERSION and hbytes == 256
    mech = M.builtin("synth_ch4_21")
    assert struct.unpack_from("<Q", data, 16)[0] == mechgen.mechanism_digest(M.flatten(mech))
    N, nin, nout, hidden, kin, kout, members, terms, dtype, min_m, ne, _ = struct.unpack_from("<12i", data, 24)
    assert (N, nin, nout, hidden, kin, kout, terms, dtype) == (21, 23, 22, 256, 32, 32, 2, 1)
    assert members >= 2 and ne == element_matrix(mech).shape[0]
    ens = Ensemble.from_bytes(data, mech, device="cpu")
    assert ens.to_bytes() == data
    assert 0 < ens.opts.spread and 0 < ens.opts.dT_cap and ens.opts.t_rel == 1e-4
    # another mechanism's digest is refused
    with pytest.raises(ValueError, match="digest"):
        Ensemble.from_bytes(data, M.builtin("synth_h2_9"), device="cpu")


def test_calibration_picks_the_rule_that_saves_most_within_the_margin():
    """The calibration's choice on a hand-made table: rules with any run over
    the margin are out, the rest ranked by BDF work saved over every field and
    time step, ties to the earlier (stricter) rule."""
    from pelelmex_b200.train_surrogate import CANDIDATES, pick_rule

    def row(rule, *runs):
        r = {"spread": rule[0], "dT_cap": rule[1], "gap": rule[2]}
        for i, (saved, err) in enumerate(runs):
            r[f"seed{i}_dt1e-06"] = {"accepted": saved, "bdf_cost_saved": saved, "max_err_bars": err}
        return r
    table = [row((0.03, 10, 1), (0.30, 0.2), (0.20, 0.3)),
             row((0.05, 10, 3), (0.45, 0.4), (0.20, 0.79)),
             row((0.08, 20, 1.5), (0.55, 0.5), (0.30, 0.81)),   # one run over the margin
             row((0.1, 10, 1), (0.40, 0.1), (0.25, 0.1))]       # saves 0.65, same as the second
    assert pick_rule(table, 0.8) == (0.05, 10, 3)
    assert pick_rule(table, 0.85) == (0.08, 20, 1.5)
    assert pick_rule(table, 0.05) is None
    assert (0.08, 20.0, 1.5) in CANDIDATES and CANDIDATES[0] == min(CANDIDATES)


def _cells(n, seed, dt):
    from pelelmex_b200 import mechanism as M, workloads as W
    mech = M.builtin("synth_ch4_21")
    return mech, W.flame_ch4(mech, cells=W.sample_cells(128 ** 3, n, seed=seed), seed=5, dt=dt)


@pytest.mark.gpu
def test_library_loader_checks_the_file():
    import ctypes
    from pelelmex_b200 import _lib
    from pelelmex_b200.reactor import ReactorB200
    L = _lib.load()
    data = _weights().read_bytes()
    r = ReactorB200("synth_ch4_21", rtol=1e-8, atol=1e-12, max_order=5).init()
    r2 = ReactorB200("synth_h2_9", rtol=1e-8, atol=1e-12, max_order=5).init()
    try:
        s = L.b200chem_surrogate_load(r._h, data, len(data))
        assert s
        o = _lib.HybridOpts()
        assert L.b200chem_surrogate_get_opts(s, ctypes.byref(o)) == 0 and o.t_rel == 1e-4
        L.b200chem_surrogate_destroy(s)
        s = L.b200chem_surrogate_load_file(r._h, str(_weights()).encode())
        assert s
        L.b200chem_surrogate_destroy(s)
        assert not L.b200chem_surrogate_load(r2._h, data, len(data))
        assert b"digest" in L.b200chem_last_error()
        bad = b"XXXXXXXX" + data[8:]
        assert not L.b200chem_surrogate_load(r._h, bad, len(bad))
        assert not L.b200chem_surrogate_load(r._h, data[:-4], len(data) - 4)
    finally:
        r.close()
        r2.close()


@pytest.mark.gpu
def test_library_inference_matches_the_python_forward():
    """b200chem_surrogate_infer (features, every member's four GEMMs, decode,
    ensemble mean and spread in the library) against the same networks run
    GEMM by GEMM from Python."""
    import ctypes
    from pelelmex_b200 import _lib
    from pelelmex_b200.reactor import ReactorB200
    from pelelmex_b200.surrogate import Ensemble, HybridReactor
    mech, f = _cells(4096, 71, 1e-6)
    r = ReactorB200(mech, rtol=1e-8, atol=1e-12, max_order=5).init()
    ens = Ensemble.load(_weights(), mech)
    h = HybridReactor(r, ens)
    rY = torch.tensor(f.rhoY, device="cuda:0")
    T = torch.tensor(f.T, device="cuda:0")
    mean = torch.empty((f.ncells, mech.n_species + 1), dtype=torch.float64, device="cuda:0")
    spread = torch.empty(f.ncells, dtype=torch.float64, device="cuda:0")
    _lib.check(_lib.load().b200chem_surrogate_infer(h._handle(), rY.data_ptr(), T.data_ptr(), f.ncells, f.dt,
                                                    mean.data_ptr(), spread.data_ptr(),
                                                    torch.cuda.current_stream().cuda_stream))
    P = ens.predict(r, rY, T, f.dt)
    ref = P.mean(0)
    assert torch.allclose(mean, ref, rtol=1e-9, atol=1e-15)
    assert torch.allclose(spread, (P[:, :, 0] - ref[:, 0]).abs().amax(0), rtol=1e-9, atol=1e-12)
    h.close()
    r.close()


@pytest.mark.gpu
@pytest.mark.parametrize("dt", [1e-6, 1e-5])
def test_hybrid_react_on_held_out_cells(dt):
    """The hybrid react (one library call) on 65,536 cells of the held-out
    flame field (seed 5, never trained on): rejected cells carry exactly the
    plain BDF result; accepted cells are within the 1e-4 relative T bar of the
    plain BDF (itself ~2e-7 from a tight solve), conserve every element and
    rhoH exactly, and have T consistent with (h, Y)."""
    from pelelmex_b200.reactor import ReactorB200
    from pelelmex_b200.surrogate import Ensemble, HybridReactor
    mech, f = _cells(65536, 5, dt)
    dev = "cuda:0"
    r = ReactorB200(mech, rtol=1e-8, atol=1e-12, max_order=5).init()
    base = [torch.tensor(a, device=dev) for a in (f.rhoY, f.T, f.rhoH, f.frhoY, f.frhoH)]
    pr = [b.clone() for b in base[:3]]
    fp = torch.zeros(f.ncells, dtype=torch.float64, device=dev)
    r.react_flat(pr[0], base[3], pr[1], pr[2], base[4], fp, dt_react=dt)
    hy = [b.clone() for b in base[:3]]
    fh = torch.full((f.ncells,), -1.0, dtype=torch.float64, device=dev)
    st = torch.full((f.ncells,), 9, dtype=torch.int32, device=dev)
    h = HybridReactor(r, Ensemble.load(_weights(), mech))
    h.react_flat(hy[0], base[3], hy[1], hy[2], base[4], fh, dt_react=dt, status=st)
    torch.cuda.synchronize()
    acc = fh == 0.0
    last = h.last
    print(f"dt {dt}: {last}")
    assert int(acc.sum()) == last["accepted"] and last["predicted"] == f.ncells
    assert last["accepted"] > 0.2 * f.ncells
    assert torch.equal(hy[1][~acc], pr[1][~acc]) and torch.equal(hy[0][:, ~acc], pr[0][:, ~acc])
    assert torch.equal(fh[~acc], fp[~acc])
    assert (st == 0).all()
    terr = (hy[1] - pr[1]).abs() / pr[1]
    assert terr.max().item() <= 1e-4
    assert torch.allclose(hy[2], pr[2], rtol=1e-14, atol=0)
    # the accepted state conserves every element exactly (the gate's projection)
    E = torch.tensor(mech.element_matrix() / mech.mw()[None, :], device=dev)
    e0, e1 = E @ base[0], E @ hy[0]
    rel = (e1 - e0).abs().amax(0) / (E.abs() @ base[0]).sum(0)
    assert rel[acc].max().item() < 1e-12
    Tc = hy[1].clone()
    r.t_from_hy(hy[0] * 1e3, hy[2] * 0.1, Tc)
    assert (((Tc - hy[1]).abs() / hy[1])[acc]).max().item() < 1e-9
    h.close()
    r.close()


@pytest.mark.gpu
def test_hybrid_fallback_and_mask_paths():
    """With a zero spread tolerance every cell falls back: the hybrid then
    equals the plain BDF bit for bit.  Masked cells are untouched with
    fctCount 0 and status MASKED."""
    from pelelmex_b200.reactor import ReactorB200
    from pelelmex_b200.surrogate import Ensemble, HybridOpts, HybridReactor
    mech, f = _cells(8192, 6, 1e-6)
    dev = "cuda:0"
    r = ReactorB200(mech, rtol=1e-8, atol=1e-12, max_order=5).init()
    base = [torch.tensor(a, device=dev) for a in (f.rhoY, f.T, f.rhoH, f.frhoY, f.frhoH)]
    mask = torch.ones(f.ncells, dtype=torch.int32, device=dev)
    mask[::7] = 0
    pr = [b.clone() for b in base[:3]]
    fp = torch.zeros(f.ncells, dtype=torch.float64, device=dev)
    r.react_flat(pr[0], base[3], pr[1], pr[2], base[4], fp, mask=mask, dt_react=f.dt)
    hy = [b.clone() for b in base[:3]]
    fh = torch.full((f.ncells,), -1.0, dtype=torch.float64, device=dev)
    st = torch.full((f.ncells,), 9, dtype=torch.int32, device=dev)
    h = HybridReactor(r, Ensemble.load(_weights(), mech), HybridOpts(spread=0.0))
    h.react_flat(hy[0], base[3], hy[1], hy[2], base[4], fh, mask=mask, dt_react=f.dt, status=st)
    torch.cuda.synchronize()
    assert h.last["accepted"] == 0 and h.last["predicted"] == int(mask.sum())
    for a, b in zip(hy, pr):
        assert torch.equal(a, b)
    assert torch.equal(fh, fp)
    m0 = mask == 0
    assert (st[m0] == 1).all() and (st[~m0] == 0).all() and (fh[m0] == 0).all()
    assert torch.equal(hy[1][m0], base[1][m0])
    h.close()
    r.close()


@pytest.mark.gpu
def test_hybrid_is_faster_than_plain_bdf_on_a_held_out_field():
    """What the trained network gains: on 524,288 held-out cells at dt 1e-6,
    one hybrid react takes less time than one plain BDF react (CUDA events,
    best of three after a warm-up each)."""
    from pelelmex_b200.reactor import ReactorB200
    from pelelmex_b200.surrogate import Ensemble, HybridReactor
    mech, f = _cells(524288, 5, 1e-6)
    dev = "cuda:0"
    r = ReactorB200(mech, rtol=1e-8, atol=1e-12, max_order=5).init()
    base = [torch.tensor(a, device=dev) for a in (f.rhoY, f.T, f.rhoH, f.frhoY, f.frhoH)]
    h = HybridReactor(r, Ensemble.load(_weights(), mech))

    def best(fn):
        ts = []
        for i in range(4):
            a = [b.clone() for b in base[:3]]
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn(a)
            e1.record()
            torch.cuda.synchronize()
            if i:
                ts.append(e0.elapsed_time(e1))
        return min(ts)
    tp = best(lambda a: r.react_flat(a[0], base[3], a[1], a[2], base[4], dt_react=f.dt))
    th = best(lambda a: h.react_flat(a[0], base[3], a[1], a[2], base[4], dt_react=f.dt, stats=False))
    print(f"plain {tp:.1f} ms, hybrid {th:.1f} ms, speedup {tp / th:.2f}x")
    assert th < tp
    h.close()
    r.close()
