"""GPU parity: the CUDA reactor (through its C ABI) against the CPU oracle.

Tolerances are the ones the reactor is specified to: final T within 1e-5
relative and Y within 1e-8 absolute of the oracle's dense-direct BDF at
rtol 1e-8 / atol 1e-12.  Mechanism evaluations (RHS, analytic Jacobian) are
FP64 on both sides and are compared at round-off level.
"""
from pathlib import Path

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from pelelmex_b200 import mechanism as M, workloads as W  # noqa: E402
from pelelmex_b200.reactor import Box, ReactorB200, ReactorError  # noqa: E402

GOLD = Path(__file__).resolve().parent / "golden"
T_RTOL = 1e-5
Y_ATOL = 1e-8
DEV = "cuda:0"


@pytest.fixture(scope="module")
def orc_cache(oracle_mod):
    cache = {}

    def get(name):
        if name not in cache:
            cache[name] = oracle_mod.Oracle(M.flatten(M.builtin(name)))
        return cache[name]
    return get


def _dev(a, dtype=torch.float64):
    return torch.tensor(np.ascontiguousarray(a), dtype=dtype, device=DEV)


def run_gpu(name, f, rtol=1e-8, atol=1e-12, max_order=5, lu_fp64=False, typ=None, mask=None, max_steps=10000,
            fY=None, fH=None, kernel="auto", group_lanes=0, refine_stall_ppm=0, refine_keep_ppm=0):
    r = ReactorB200(name, rtol=rtol, atol=atol, max_order=max_order, lu_fp64=lu_fp64,
                    max_steps=max_steps, kernel=kernel, group_lanes=group_lanes,
                    refine_stall_ppm=refine_stall_ppm, refine_keep_ppm=refine_keep_ppm).init(2, f.ncells)
    if typ is not None:
        r.set_typ_vals_ode(typ)
    rhoY, T, rhoH = _dev(f.rhoY), _dev(f.T), _dev(f.rhoH)
    fYd = _dev(f.frhoY if fY is None else fY)
    fHd = _dev(f.frhoH if fH is None else fH)
    fct = torch.zeros(f.ncells, dtype=torch.float64, device=DEV)
    st = torch.zeros(f.ncells, dtype=torch.int32, device=DEV)
    m = _dev(mask, torch.int32) if mask is not None else None
    dt, t, stats = r.react_flat(rhoY, fYd, T, rhoH, fHd, fct, m, dt_react=f.dt, status=st, stats=True,
                                raise_on_failure=False)
    torch.cuda.synchronize()
    out = dict(rhoY=rhoY.cpu().numpy(), T=T.cpu().numpy(), rhoH=rhoH.cpu().numpy(), fct=fct.cpu().numpy(),
               status=st.cpu().numpy(), stats=stats, time=t)
    r.close()
    return out


def compare(f, g, o, label):
    ok = (o["status"] == 0) & (g["status"] == 0)
    rho = f.rhoY.sum(axis=0)
    terr = np.abs(g["T"] - o["T"]) / o["T"]
    yerr = np.abs(g["rhoY"] - o["rhoY"]).max(axis=0) / rho
    print(f"{label}: cells {f.ncells} max rel T err {terr[ok].max():.2e} max abs Y err {yerr[ok].max():.2e} "
          f"gpu nfe mean {g['fct'][ok].mean():.1f} oracle nfe mean {o['fct'][ok].mean():.1f}")
    assert terr[ok].max() <= T_RTOL
    assert yerr[ok].max() <= Y_ATOL
    return terr, yerr


@pytest.mark.parametrize("name", ["synth_h2_9", "synth_ch4_21", "synth_c12_53"])
def test_rhs_and_jacobian_parity(name, orc_cache):
    orc = orc_cache(name)
    g = np.load(GOLD / f"rates_{name}.npz")
    r = ReactorB200(name).init()
    y, F = _dev(g["y"]), _dev(g["F"])
    yd = r.eval_rhs(y, F).cpu().numpy()
    J = r.eval_jac(y, F).cpu().numpy()
    yd_o = orc.rhs(g["y"], g["F"])
    J_o = orc.jac(g["y"], g["F"])
    sc = np.abs(yd_o).max(axis=1, keepdims=True)
    assert np.max(np.abs(yd - yd_o) / sc) < 1e-12
    scj = np.abs(J_o).max(axis=2, keepdims=True) + 1e-300
    assert np.max(np.abs(J - J_o) / scj) < 1e-11
    r.close()


def test_premixed_h2_32cubed(orc_cache):
    """LiDryer-shaped configuration: 32^3 cells, T in [1000, 2000] K, dt 1e-6."""
    mech = M.builtin("synth_h2_9")
    f = W.premixed_h2(mech, edge=32, dt=1e-6)
    g = run_gpu("synth_h2_9", f)
    o = orc_cache("synth_h2_9").react(f.rhoY, f.frhoY, f.T, f.rhoH, f.frhoH, f.dt, rtol=1e-8, atol=1e-12,
                                      max_order=5)
    assert (g["status"] == 0).all() and o["nfail"] == 0
    compare(f, g, o, "premixed_h2 32^3")
    assert np.allclose(g["rhoH"], o["rhoH"], rtol=1e-15, atol=0)
    assert g["stats"]["n_cells"] == f.ncells and g["stats"]["n_failed"] == 0
    assert g["time"] == pytest.approx(1e-6)


@pytest.mark.parametrize("dt", [1e-6, 1e-5])
def test_flame_ch4_sample(dt, orc_cache):
    """drm19-shaped flame field, a seeded 4096-cell sample of the 128^3 case."""
    mech = M.builtin("synth_ch4_21")
    f = W.flame_ch4(mech, cells=W.sample_cells(128 ** 3, 4096), dt=dt)
    g = run_gpu("synth_ch4_21", f)
    o = orc_cache("synth_ch4_21").react(f.rhoY, f.frhoY, f.T, f.rhoH, f.frhoH, f.dt, rtol=1e-8, atol=1e-12,
                                        max_order=5)
    assert (g["status"] == 0).all() and o["nfail"] == 0
    compare(f, g, o, f"flame_ch4 dt={dt}")


def test_dodecane_two_components_per_lane(orc_cache):
    """53 species: n = 54 components, several per lane."""
    mech = M.builtin("synth_c12_53")
    rng = np.random.default_rng(7)
    nm = mech.names
    n = 256
    X = np.zeros((n, mech.n_species))
    X[:, nm.index("NC12H26")] = rng.uniform(0.5, 2.0, n)
    X[:, nm.index("O2")] = 18.5
    X[:, nm.index("N2")] = 69.6
    X += rng.uniform(0, 1, X.shape) ** 6 * 0.5
    Y = M.mole_to_mass(mech, X / X.sum(axis=1, keepdims=True))
    T = rng.uniform(700, 1500, n)
    f = W._finish(mech, Y, T, 1e-6, (n,), "c12")
    g = run_gpu("synth_c12_53", f)
    orc = orc_cache("synth_c12_53")
    o = orc.react(f.rhoY, f.frhoY, f.T, f.rhoH, f.frhoH, f.dt, rtol=1e-8, atol=1e-12, max_order=5)
    assert (g["status"] == 0).all() and o["nfail"] == 0
    rho = f.rhoY.sum(axis=0)
    terr = np.abs(g["T"] - o["T"]) / o["T"]
    assert terr.max() <= T_RTOL
    # These cells ignite inside the step (~350 RHS evaluations each): two rtol 1e-8
    # solutions differ at the level of their own global error, so Y is compared
    # against a tight FP64 solve (rtol 1e-12): the GPU error must be of the same
    # size as the oracle's.
    tight = orc.react(f.rhoY, f.frhoY, f.T, f.rhoH, f.frhoH, f.dt, rtol=1e-12, atol=1e-20, max_order=5)
    eg = np.abs(g["rhoY"] - tight["rhoY"]).max(axis=0) / rho
    eo = np.abs(o["rhoY"] - tight["rhoY"]).max(axis=0) / rho
    print(f"dodecane-shaped: T err vs oracle {terr.max():.2e}; Y err vs rtol-1e-12 solve: gpu {eg.max():.2e} "
          f"oracle {eo.max():.2e}")
    assert eg.max() <= 3.0 * eo.max() + 1e-9


@pytest.mark.parametrize("kernel,lanes", [("thread", 0), ("group", 8), ("group", 16), ("group", 32)])
@pytest.mark.parametrize("lu_fp64", [False, True])
def test_kernels_group_sizes_and_lu_precisions(kernel, lanes, lu_fp64, orc_cache):
    """Thread-per-cell and group integrators (8/16/32 lanes per cell), FP32
    inverse + FP64 refinement and FP64 inverse."""
    mech = M.builtin("synth_ch4_21")
    f = W.flame_ch4(mech, cells=W.sample_cells(128 ** 3, 1024, seed=13), dt=1e-5)
    g = run_gpu("synth_ch4_21", f, kernel=kernel, lu_fp64=lu_fp64, group_lanes=lanes)
    o = orc_cache("synth_ch4_21").react(f.rhoY, f.frhoY, f.T, f.rhoH, f.frhoH, f.dt, rtol=1e-8, atol=1e-12,
                                        max_order=5)
    assert (g["status"] == 0).all()
    compare(f, g, o, f"{kernel} kernel G={lanes}, lu_fp64={lu_fp64}")


@pytest.mark.parametrize("lanes", [8, 16, 32])
def test_group_sizes_on_h2(lanes, orc_cache):
    """Group sizes on the 10-component system (1 or 2 components per lane)."""
    f = W.premixed_h2(M.builtin("synth_h2_9"), edge=8)
    g = run_gpu("synth_h2_9", f, group_lanes=lanes, kernel="group")
    o = orc_cache("synth_h2_9").react(f.rhoY, f.frhoY, f.T, f.rhoH, f.frhoH, f.dt, rtol=1e-8, atol=1e-12,
                                      max_order=5)
    compare(f, g, o, f"synth_h2_9 G={lanes}")


def test_fp64_lu_variant(orc_cache):
    mech = M.builtin("synth_ch4_21")
    f = W.flame_ch4(mech, cells=W.sample_cells(128 ** 3, 1024, seed=3), dt=1e-5)
    g = run_gpu("synth_ch4_21", f, lu_fp64=True)
    o = orc_cache("synth_ch4_21").react(f.rhoY, f.frhoY, f.T, f.rhoH, f.frhoH, f.dt, rtol=1e-8, atol=1e-12,
                                        max_order=5)
    compare(f, g, o, "fp64 LU")


def test_forcing_typical_values_and_order(orc_cache):
    """Non-zero forcing (SDC sources), typical-value atol, max_order 4 as in the decks."""
    mech = M.builtin("synth_ch4_21")
    f = W.flame_ch4(mech, cells=W.sample_cells(128 ** 3, 1024, seed=5), dt=1e-5)
    rng = np.random.default_rng(3)
    fY = f.rhoY * rng.normal(0, 30.0, f.rhoY.shape)
    fH = rng.normal(0, 1e9, f.ncells)
    typ = np.concatenate([np.maximum(1e-10, f.rhoY.mean(axis=1)), [1500.0]])
    g = run_gpu("synth_ch4_21", f, rtol=1e-6, atol=1e-5, max_order=4, typ=typ, fY=fY, fH=fH)
    o = orc_cache("synth_ch4_21").react(f.rhoY, fY, f.T, f.rhoH, fH, f.dt, rtol=1e-6, atol=1e-5, typ=typ,
                                        max_order=4)
    ok = (g["status"] == 0) & (o["status"] == 0)
    assert ok.all()
    rho = f.rhoY.sum(axis=0)
    terr = np.abs(g["T"] - o["T"]) / o["T"]
    # loose tolerances: both sides are rtol 1e-6 solutions of the same problem
    assert terr.max() < 1e-4
    assert (np.abs(g["rhoY"] - o["rhoY"]).max(axis=0) / rho).max() < 1e-5
    assert np.allclose(g["rhoH"], f.rhoH + f.dt * fH, rtol=1e-15)


def test_status_mask_and_bad_inputs(orc_cache):
    mech = M.builtin("synth_h2_9")
    f = W.premixed_h2(mech, edge=4)
    rY, T = f.rhoY.copy(), f.T.copy()
    rY[0, 1] = np.nan
    T[2] = -5.0
    mask = np.ones(f.ncells, np.int32)
    mask[3] = 0
    f2 = W.Field(mech, rY, T, f.rhoH.copy(), f.frhoY, f.frhoH, f.dt, f.shape, f.name)
    g = run_gpu("synth_h2_9", f2, mask=mask)
    assert list(g["status"][:4]) == [0, -4, -4, 1]
    assert g["fct"][3] == 0
    assert np.isnan(g["rhoY"][0, 1])  # failed cells are left as they were
    assert g["T"][2] == -5.0 and g["T"][3] == f.T[3]
    assert g["stats"]["n_failed"] == 2 and g["stats"]["n_masked"] == 1
    # a step cap gives max_steps, exactly as the oracle
    f3 = W.premixed_h2(mech, edge=4, dt=1e-3)
    g = run_gpu("synth_h2_9", f3, max_steps=3)
    o = orc_cache("synth_h2_9").react(f3.rhoY, f3.frhoY, f3.T, f3.rhoH, f3.frhoH, f3.dt, max_steps=3)
    assert (g["status"] == -1).any()
    assert ((g["status"] == -1) == (o["status"] == -1)).mean() > 0.9


def test_react_raises_on_failure_by_default():
    mech = M.builtin("synth_h2_9")
    f = W.premixed_h2(mech, edge=2)
    r = ReactorB200(mech, rtol=1e-8, atol=1e-12).init()
    T = _dev(f.T)
    T[0] = float("nan")
    with pytest.raises(ReactorError):
        r.react_flat(_dev(f.rhoY), _dev(f.frhoY), T, _dev(f.rhoH), _dev(f.frhoH), dt_react=f.dt, stats=True)
    r.close()


def test_box_api_with_ghost_cells_and_two_boxes():
    """Array4 views with ghost cells and a tilebox inside the fab; two boxes in one
    launch; must equal the flat form on the same cells and leave ghosts untouched."""
    mech = M.builtin("synth_ch4_21")
    N = mech.n_species
    nx, ny, nz, g = 6, 5, 4, 1
    ncell = nx * ny * nz
    f = W.flame_ch4(mech, cells=W.sample_cells(128 ** 3, 2 * ncell, seed=9), dt=1e-6)

    def fab(vals, ncomp):  # [ncomp, nz+2g, ny+2g, nx+2g] with interior = vals
        t = torch.full((ncomp, nz + 2 * g, ny + 2 * g, nx + 2 * g), 7.0, dtype=torch.float64, device=DEV)
        t[:, g:g + nz, g:g + ny, g:g + nx] = _dev(vals.reshape(ncomp, nz, ny, nx))
        return t

    r = ReactorB200(mech, rtol=1e-8, atol=1e-12, max_order=5).init()
    items, fabs = [], []
    for b in range(2):
        sl = slice(b * ncell, (b + 1) * ncell)
        lo = (10 * b, -3, 2)
        flo = (lo[0] - g, lo[1] - g, lo[2] - g)
        box = Box(lo, (lo[0] + nx - 1, lo[1] + ny - 1, lo[2] + nz - 1))
        fb = [fab(f.rhoY[:, sl], N), fab(f.frhoY[:, sl], N), fab(f.T[sl], 1), fab(f.rhoH[sl], 1),
              fab(f.frhoH[sl], 1), fab(np.zeros(ncell), 1)]
        mk = torch.ones((1, nz + 2 * g, ny + 2 * g, nx + 2 * g), dtype=torch.int32, device=DEV)
        items.append((box, *fb, mk, flo))
        fabs.append(fb)
    dt, t = r.react_boxes(items, 1e-6, 0.0)
    torch.cuda.synchronize()
    # flat reference on the same cells
    rhoY, T, rhoH = _dev(f.rhoY), _dev(f.T), _dev(f.rhoH)
    r.react_flat(rhoY, _dev(f.frhoY), T, rhoH, _dev(f.frhoH), dt_react=1e-6)
    torch.cuda.synchronize()
    for b in range(2):
        sl = slice(b * ncell, (b + 1) * ncell)
        got = fabs[b][0][:, g:g + nz, g:g + ny, g:g + nx].reshape(N, ncell)
        assert torch.equal(got, rhoY[:, sl])
        assert torch.equal(fabs[b][2][0, g:g + nz, g:g + ny, g:g + nx].reshape(ncell), T[sl])
        assert torch.equal(fabs[b][3][0, g:g + nz, g:g + ny, g:g + nx].reshape(ncell), rhoH[sl])
        ghost = fabs[b][0].clone()
        ghost[:, g:g + nz, g:g + ny, g:g + nx] = 7.0
        assert torch.all(ghost == 7.0)
        assert torch.all(fabs[b][5][0, g:g + nz, g:g + ny, g:g + nx] > 0)
    r.close()


def test_empty_call():
    r = ReactorB200("synth_h2_9").init()
    e = torch.zeros((9, 0), dtype=torch.float64, device=DEV)
    z = torch.zeros(0, dtype=torch.float64, device=DEV)
    dt, t, s = r.react_flat(e, e, z, z, z, dt_react=1e-6, stats=True)
    assert s["n_cells"] == 0 and t == pytest.approx(1e-6)
    r.close()


def test_inst_rr_and_t_from_hy(orc_cache):
    """reactionRateRhoY / getTfromHY in MKS (Source/PeleLMeX_K.H:700-723, 850-889)."""
    name = "synth_ch4_21"
    mech = M.builtin(name)
    orc = orc_cache(name)
    f = W.flame_ch4(mech, cells=W.sample_cells(128 ** 3, 512, seed=11))
    rhoY_mks = f.rhoY * 1e3
    rhoH_mks = f.rhoH * 0.1
    Tguess = f.T * 0.9 + 50.0
    r = ReactorB200(name).init()
    T = _dev(Tguess)
    rr = r.inst_rr(_dev(rhoY_mks), _dev(rhoH_mks), T).cpu().numpy()
    Tg = T.cpu().numpy()
    assert np.max(np.abs(Tg - f.T) / f.T) < 1e-10
    W_ = mech.mw()
    for c in range(0, f.ncells, 17):
        C = f.rhoY[:, c] / W_
        wd = orc.wdot(f.T[c], C) * W_ * 1e3
        sc = np.abs(wd).max()
        assert np.max(np.abs(rr[:, c] - wd)) <= 1e-9 * sc
    T2 = _dev(Tguess)
    r.t_from_hy(_dev(rhoY_mks), _dev(rhoH_mks), T2)
    assert np.max(np.abs(T2.cpu().numpy() - f.T) / f.T) < 1e-10
    r.close()


def test_h_given_t_and_heat_release():
    """getHGivenT / getHeatRelease (Source/PeleLMeX_K.H:598-615,
    Source/PeleLMeX_Reactions.cpp:477-506) against the NASA-7 restatement."""
    name = "synth_ch4_21"
    mech = M.builtin(name)
    f = W.flame_ch4(mech, cells=W.sample_cells(128 ** 3, 777, seed=12))
    rng = np.random.default_rng(6)
    IR = rng.normal(0.0, 1.0, (mech.n_species, f.ncells)) * f.rhoY * 1e3 * 1e4  # kg/m^3/s
    r = ReactorB200(name).init()
    Hi = r.h_given_t(_dev(f.T)).cpu().numpy()
    ref = (M.h_RT(mech, f.T) * M.R_CGS * f.T[:, None] / mech.mw()).T * 1e-4  # J/kg, [N, ncells]
    assert np.max(np.abs(Hi - ref) / np.maximum(np.abs(ref), 1e3)) < 1e-13
    HR = r.heat_release(_dev(f.T), _dev(IR)).cpu().numpy()
    href = -np.sum(ref * IR, axis=0)
    scale = np.sum(np.abs(ref * IR), axis=0)
    assert np.max(np.abs(HR - href) / scale) < 1e-13
    r.close()
