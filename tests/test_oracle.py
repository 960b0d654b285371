"""The CPU oracle against its golden fixtures and physical invariants."""
from pathlib import Path

import numpy as np
import pytest

from pelelmex_b200 import mechanism as M, workloads as W

GOLD = Path(__file__).resolve().parent / "golden"
NAMES = ["synth_h2_9", "synth_ch4_21", "synth_c12_53"]


@pytest.fixture(scope="module", params=NAMES)
def mo(request, oracle_mod):
    m = M.builtin(request.param)
    return m, oracle_mod.Oracle(M.flatten(m))


def test_rhs_matches_numpy_restatement(mo):
    m, orc = mo
    g = np.load(GOLD / f"rates_{m.name}.npz")
    r = orc.rhs(g["y"], g["F"])
    scale = np.abs(g["ydot"]).max(axis=1, keepdims=True)
    assert np.max(np.abs(r - g["ydot"]) / scale) < 1e-12


def test_jacobian_matches_finite_differences(mo):
    import kinetics_np
    m, orc = mo
    K = kinetics_np.NpKinetics(M.flatten(m))
    g = np.load(GOLD / f"rates_{m.name}.npz")
    for y, F in zip(g["y"][:3], g["F"][:3]):
        Ja = orc.jac(y, F)
        Jfd = K.jac_fd(y, F, rel=1e-4)
        sc = np.abs(Jfd).max(axis=1, keepdims=True) + 1e-300
        assert np.max(np.abs(Ja - Jfd) / sc) < 5e-6


def test_bdf_matches_radau_golden(mo):
    """Oracle BDF at rtol 1e-8 against scipy Radau at rtol 1e-12."""
    m, orc = mo
    g = np.load(GOLD / f"traj_{m.name}.npz")
    N = m.n_species
    y0, F, y1, dt = g["y0"], g["F"], g["y1"], float(g["dt"])
    rhoH = np.array([orc.mix_h(y[N], y[:N] / y[:N].sum()) * y[:N].sum() for y in y0])
    res = orc.react(y0[:, :N].T, F[:, :N].T, y0[:, N], rhoH, F[:, N], dt, rtol=1e-8, atol=1e-12, max_order=5)
    assert res["nfail"] == 0
    rho1 = y1[:, :N].sum(axis=1)
    terr = np.abs(res["T"] - y1[:, N]) / y1[:, N]
    yerr = np.abs(res["rhoY"].T / rho1[:, None] - y1[:, :N] / rho1[:, None])
    assert terr.max() < 2e-6, terr
    assert yerr.max() < 1e-6, yerr.max()  # global error of a rtol 1e-8 BDF vs the rtol 1e-12 solution


def test_conservation_and_enthalpy(oracle_mod):
    m = M.builtin("synth_ch4_21")
    orc = oracle_mod.Oracle(M.flatten(m))
    f = W.flame_ch4(m, cells=W.sample_cells(128 ** 3, 256), dt=1e-5)
    rng = np.random.default_rng(0)
    fY = f.rhoY * rng.normal(0, 50.0, f.rhoY.shape)
    fH = rng.normal(0, 1e9, f.ncells)
    res = orc.react(f.rhoY, fY, f.T, f.rhoH, fH, f.dt, rtol=1e-8, atol=1e-12, max_order=5)
    assert res["nfail"] == 0
    # total mass: sum rhoY changes only by the forcing
    assert np.allclose(res["rhoY"].sum(axis=0), f.rhoY.sum(axis=0) + f.dt * fY.sum(axis=0), rtol=1e-7)
    # elements are conserved by chemistry
    E = m.element_matrix() / m.mw()[None, :]
    e0 = E @ (f.rhoY + f.dt * fY)
    e1 = E @ res["rhoY"]
    assert np.max(np.abs(e1 - e0) / np.abs(e0).max(axis=0)) < 1e-7
    # rhoH advanced by the forcing, T consistent with (h, Y)
    assert np.allclose(res["rhoH"], f.rhoH + f.dt * fH, rtol=1e-14)
    rho = res["rhoY"].sum(axis=0)
    for c in range(0, f.ncells, 37):
        h = orc.mix_h(res["T"][c], res["rhoY"][:, c] / rho[c])
        assert abs(h * rho[c] - res["rhoH"][c]) <= 1e-6 * abs(res["rhoH"][c]) + 1e-6 * rho[c] * 1e9


def test_status_codes(oracle_mod):
    m = M.builtin("synth_h2_9")
    orc = oracle_mod.Oracle(M.flatten(m))
    f = W.premixed_h2(m, edge=2)
    rY = f.rhoY.copy()
    T = f.T.copy()
    rY[0, 1] = np.nan
    T[2] = -5.0
    mask = np.ones(f.ncells, np.int32)
    mask[3] = 0
    res = orc.react(rY, f.frhoY, T, f.rhoH, f.frhoH, f.dt, mask=mask)
    assert list(res["status"][:4]) == [0, -4, -4, 1]
    assert res["fct"][3] == 0
    # a step cap forces max_steps
    res = orc.react(f.rhoY, f.frhoY, f.T, f.rhoH, f.frhoH, 1e-3, max_steps=3)
    assert (res["status"] == -1).any()


def test_empty_batch(oracle_mod):
    m = M.builtin("synth_h2_9")
    orc = oracle_mod.Oracle(M.flatten(m))
    res = orc.react(np.zeros((9, 0)), np.zeros((9, 0)), np.zeros(0), np.zeros(0), np.zeros(0), 1e-6)
    assert res["nfail"] == 0 and res["T"].size == 0


def test_t_from_hy_roundtrip(oracle_mod):
    m = M.builtin("synth_c12_53")
    orc = oracle_mod.Oracle(M.flatten(m))
    rng = np.random.default_rng(1)
    for T in (350.0, 999.0, 1001.0, 2500.0):
        Y = rng.uniform(0, 1, m.n_species)
        Y /= Y.sum()
        h = orc.mix_h(T, Y)
        T2, it = orc.t_from_hy(h, Y, T * 0.8)
        assert it > 0 and abs(T2 - T) < 1e-9 * T
