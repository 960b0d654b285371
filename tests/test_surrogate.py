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


@pytest.mark.gpu
def test_hybrid_reactor_accuracy_and_gain():
    """Train a two-network ensemble on BDF-labelled cells of the flame field,
    then react held-out cells: the cells the gate rejects carry exactly the
    plain BDF result; the accepted ones stay within the error the gate's
    checks hold the surrogate to (3e-4 relative T, 3e-4 mass-weighted Y; the
    1e-4 bar of the headline is checked on the full field by the benchmark,
    which reports the plain BDF when the hybrid misses it); rhoH is exact;
    and the surrogate takes a share of the cells (what the network gains)."""
    from pelelmex_b200 import mechanism as M, workloads as W
    from pelelmex_b200.reactor import ReactorB200
    from pelelmex_b200.surrogate import HybridReactor, train_ensemble
    mech = M.builtin("synth_ch4_21")
    r = ReactorB200(mech, rtol=1e-8, atol=1e-12, max_order=5).init()
    train = W.flame_ch4(mech, cells=W.sample_cells(128 ** 3, 262144, seed=10), dt=1e-6, seed=10)
    nets = train_ensemble(r, mech, [train], members=2, steps=2500)
    test = W.flame_ch4(mech, cells=W.sample_cells(128 ** 3, 32768, seed=5), dt=1e-6, seed=5)
    dev = "cuda:0"
    base = [torch.tensor(a, device=dev) for a in (test.rhoY, test.T, test.rhoH, test.frhoY, test.frhoH)]
    pr = [b.clone() for b in base[:3]]
    r.react_flat(pr[0], base[3], pr[1], pr[2], base[4], dt_react=test.dt)
    hy = [b.clone() for b in base[:3]]
    fct = torch.zeros(test.ncells, dtype=torch.float64, device=dev)
    h = HybridReactor(r, nets)
    h.react_flat(hy[0], base[3], hy[1], hy[2], base[4], fct, dt_react=test.dt)
    torch.cuda.synchronize()
    terr = ((hy[1] - pr[1]).abs() / pr[1]).max().item()
    acc = h.last["accepted_fraction"]
    ok = h.last["accepted"]
    print(f"hybrid: accepted {acc:.3f} {h.last['rejected_by']}, max rel T err vs plain BDF {terr:.2e}")
    assert acc > 0.01 and int(ok.sum()) == round(acc * test.ncells)
    assert torch.equal(hy[1][~ok], pr[1][~ok]) and torch.equal(hy[0][:, ~ok], pr[0][:, ~ok])
    assert terr <= 3e-4
    rho = pr[0].sum(dim=0)
    assert ((hy[0] - pr[0]).abs().max(dim=0).values / rho).max().item() < 3e-4
    assert torch.allclose(hy[2], pr[2], rtol=1e-14)
    assert (fct > 0).all()
    r.close()
