"""The advanceChemistry box body (Source/PeleLMeX_Reactions.cpp:31-175):
MKS -> CGS, react, CGS -> MKS and the reaction term I_R, for several boxes
with ghost cells in one call, against the same steps composed by hand
around the flat react (bit for bit: the same operations in the same order)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from pelelmex_b200 import mechanism as M, workloads as W  # noqa: E402
from pelelmex_b200.reactor import Box, ReactorB200  # noqa: E402

DEV = "cuda:0"


def test_advance_chemistry_matches_composed_steps():
    mech = M.builtin("synth_ch4_21")
    N = mech.n_species
    nx, ny, nz, g = 5, 4, 3, 1
    nc = nx * ny * nz
    f = W.flame_ch4(mech, cells=W.sample_cells(128 ** 3, 2 * nc, seed=31), dt=1e-6)
    rng = np.random.default_rng(4)
    # MKS old state and forcing (CGS fields of the generator scaled back)
    rY_mks = f.rhoY * 1e3
    rH_mks = f.rhoH * 0.1
    fY_mks = rng.normal(0.0, 1.0, f.rhoY.shape) * rY_mks
    fH_mks = rng.normal(0.0, 1e6, f.ncells)

    def fab(vals, ncomp, fill=7.0):
        t = torch.full((ncomp, nz + 2 * g, ny + 2 * g, nx + 2 * g), fill, dtype=torch.float64, device=DEV)
        t[:, g:g + nz, g:g + ny, g:g + nx] = torch.tensor(np.ascontiguousarray(vals).reshape(ncomp, nz, ny, nx),
                                                          dtype=torch.float64, device=DEV)
        return t

    def inner(t):
        return t[:, g:g + nz, g:g + ny, g:g + nx].reshape(t.shape[0], nc)

    r = ReactorB200(mech, rtol=1e-8, atol=1e-12, max_order=5).init()
    items, fabs = [], []
    for b in range(2):
        sl = slice(b * nc, (b + 1) * nc)
        lo = (20 * b, 0, 0)
        flo = (lo[0] - g, -g, -g)
        box = Box(lo, (lo[0] + nx - 1, ny - 1, nz - 1))
        fb = dict(rY_o=fab(rY_mks[:, sl], N), rH_o=fab(rH_mks[sl], 1), T_o=fab(f.T[sl], 1),
                  rY_n=fab(np.zeros((N, nc)), N), rH_n=fab(np.zeros(nc), 1), T_n=fab(np.zeros(nc), 1),
                  fY=fab(fY_mks[:, sl], N), fH=fab(fH_mks[sl], 1), fc=fab(np.zeros(nc), 1),
                  IR=fab(np.zeros((N, nc)), N))
        mk = torch.ones((1, nz + 2 * g, ny + 2 * g, nx + 2 * g), dtype=torch.int32, device=DEV)
        items.append((box, fb["rY_o"], fb["rH_o"], fb["T_o"], fb["rY_n"], fb["rH_n"], fb["T_n"], fb["fY"], fb["fH"],
                      fb["fc"], mk, fb["IR"], flo))
        fabs.append(fb)
    fY0 = [fb["fY"].clone() for fb in fabs]
    st = r.advance_chemistry(items, f.dt, stats=True)
    torch.cuda.synchronize()
    assert st["n_cells"] == 2 * nc and st["n_failed"] == 0

    # the same steps by hand around the flat react
    d = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device=DEV)  # noqa: E731
    rYo, fYm, fHm = d(rY_mks), d(fY_mks), d(fH_mks)
    rY = rYo * 1.0e-3
    fY = fYm * 1.0e-3
    T = d(f.T).clone()
    rH = d(rH_mks) * 10.0
    fH = fHm * 10.0
    r.react_flat(rY, fY.contiguous(), T, rH, fH.contiguous(), dt_react=f.dt)
    rY *= 1.0e3
    fY *= 1.0e3
    rH *= 0.1
    fH *= 0.1
    IR = -(rYo - rY) * (1.0 / f.dt) - fY
    torch.cuda.synchronize()
    for b, fb in enumerate(fabs):
        sl = slice(b * nc, (b + 1) * nc)
        assert torch.equal(inner(fb["rY_n"]), rY[:, sl])
        assert torch.equal(inner(fb["T_n"])[0], T[sl])
        assert torch.equal(inner(fb["rH_n"])[0], rH[sl])
        assert torch.equal(inner(fb["IR"]), IR[:, sl])
        assert torch.equal(inner(fb["fY"]), fY[:, sl])
        assert torch.equal(inner(fb["fH"])[0], fH[sl])
        assert (inner(fb["fc"]) > 0).all()
        # ghost cells untouched, the old state untouched
        for key in ("rY_n", "IR", "T_n"):
            ghost = fb[key].clone()
            ghost[:, g:g + nz, g:g + ny, g:g + nx] = 7.0
            assert torch.all(ghost == 7.0)
        assert torch.equal(inner(fb["rY_o"]), rYo[:, sl])
        # the forcing round trip (x 1e-3, x 1e3) is the reference's: at most an ulp off the input
        assert torch.allclose(inner(fb["fY"]), inner(fY0[b]), rtol=4e-16, atol=0)
    r.close()


def _fab(vals, ncomp, nx, ny, nz, g, fill=7.0):
    t = torch.full((ncomp, nz + 2 * g, ny + 2 * g, nx + 2 * g), fill, dtype=torch.float64, device=DEV)
    t[:, g:g + nz, g:g + ny, g:g + nx] = torch.tensor(np.ascontiguousarray(vals).reshape(ncomp, nz, ny, nx),
                                                      dtype=torch.float64, device=DEV)
    return t


def test_covered_box_is_converted_but_not_reacted():
    """advanceChemistryBAChem (Source/PeleLMeX_Reactions.cpp:260-289): a box whose
    m_baChemFlag is 0 is not reacted (fctCount = 0) but still goes through the unit
    conversions and gets I_R; the other box of the same call is reacted."""
    mech = M.builtin("synth_ch4_21")
    N = mech.n_species
    nx, ny, nz, g = 6, 3, 2, 1
    nc = nx * ny * nz
    f = W.flame_ch4(mech, cells=W.sample_cells(128 ** 3, 2 * nc, seed=32), dt=1e-6)
    rY_mks, rH_mks = f.rhoY * 1e3, f.rhoH * 0.1
    r = ReactorB200(mech, rtol=1e-8, atol=1e-12, max_order=5).init()
    items, fabs = [], []
    for b in range(2):
        sl = slice(b * nc, (b + 1) * nc)
        lo = (0, 10 * b, 0)
        box = Box(lo, (nx - 1, lo[1] + ny - 1, nz - 1))
        flo = (-g, lo[1] - g, -g)
        fb = dict(rY_o=_fab(rY_mks[:, sl], N, nx, ny, nz, g), rH_o=_fab(rH_mks[sl], 1, nx, ny, nz, g),
                  T_o=_fab(f.T[sl], 1, nx, ny, nz, g), rY_n=_fab(np.zeros((N, nc)), N, nx, ny, nz, g),
                  rH_n=_fab(np.zeros(nc), 1, nx, ny, nz, g), T_n=_fab(np.zeros(nc), 1, nx, ny, nz, g),
                  fY=_fab(np.zeros((N, nc)), N, nx, ny, nz, g), fH=_fab(np.zeros(nc), 1, nx, ny, nz, g),
                  fc=_fab(np.full(nc, 5.0), 1, nx, ny, nz, g), IR=_fab(np.zeros((N, nc)), N, nx, ny, nz, g))
        items.append((box, fb["rY_o"], fb["rH_o"], fb["T_o"], fb["rY_n"], fb["rH_n"], fb["T_n"], fb["fY"], fb["fH"],
                      fb["fc"], None, fb["IR"], flo))
        fabs.append(fb)
    status = torch.full((2 * nc,), 9, dtype=torch.int32, device=DEV)
    st = r.advance_chemistry(items, f.dt, stats=True, status=status, skip_react=[False, True])
    torch.cuda.synchronize()
    assert st["n_masked"] == nc and st["n_failed"] == 0
    s = status.cpu().numpy()
    assert (s[:nc] == 0).all() and (s[nc:] == 1).all()

    def inner(t):
        return t[:, g:g + nz, g:g + ny, g:g + nx].reshape(t.shape[0], nc)

    a, c = fabs
    assert (inner(a["fc"]) > 0).all()
    assert torch.all(inner(c["fc"]) == 0.0)
    # the covered box: the reference's round trip x 1e-3, x 1e3 and x 10, x 0.1 of the old state
    rYo = inner(c["rY_o"])
    assert torch.equal(inner(c["rY_n"]), (rYo * 1.0e-3) * 1.0e3)
    assert torch.equal(inner(c["rH_n"]), (inner(c["rH_o"]) * 10.0) * 0.1)
    assert torch.equal(inner(c["T_n"]), inner(c["T_o"]))
    assert torch.equal(inner(c["IR"]), -(rYo - inner(c["rY_n"])) * (1.0 / f.dt) - inner(c["fY"]))
    # the reacted box moved
    assert not torch.equal(inner(a["T_n"]), inner(a["T_o"]))
    r.close()


def test_react_force_matches_reference_formula():
    """getScalarReactForce (Source/PeleLMeX_Reactions.cpp:437-475), bit for bit:
    extF_rhoY = (rhoY_new - rhoY_old) * (1/dt) - I_R, extF_rhoH = (rhoH_new - rhoH_old) * (1/dt),
    for two boxes with ghost cells in one call; ghost cells untouched."""
    mech = M.builtin("synth_ch4_21")
    N = mech.n_species
    nx, ny, nz, g = 4, 5, 3, 2
    nc = nx * ny * nz
    rng = np.random.default_rng(11)
    dt = 3.7e-7
    r = ReactorB200(mech, rtol=1e-8, atol=1e-12, max_order=5).init()
    items, fabs = [], []
    for b in range(2):
        lo = (8 * b, 0, -3)
        box = Box(lo, (lo[0] + nx - 1, ny - 1, lo[2] + nz - 1))
        flo = (lo[0] - g, -g, lo[2] - g)
        rYo = rng.uniform(0.0, 1.2, (N, nc))
        fb = dict(rY_o=_fab(rYo, N, nx, ny, nz, g), rH_o=_fab(rng.normal(0, 1e6, nc), 1, nx, ny, nz, g),
                  rY_n=_fab(rYo * (1 + rng.normal(0, 1e-3, (N, nc))), N, nx, ny, nz, g),
                  rH_n=_fab(rng.normal(0, 1e6, nc), 1, nx, ny, nz, g),
                  IR=_fab(rng.normal(0, 50.0, (N, nc)), N, nx, ny, nz, g),
                  fY=_fab(np.zeros((N, nc)), N, nx, ny, nz, g), fH=_fab(np.zeros(nc), 1, nx, ny, nz, g))
        items.append((box, fb["rY_o"], fb["rH_o"], fb["rY_n"], fb["rH_n"], fb["IR"], fb["fY"], fb["fH"], flo))
        fabs.append(fb)
    r.react_force(items, dt)
    torch.cuda.synchronize()
    dtinv = 1.0 / dt
    for fb in fabs:
        sl = (slice(None), slice(g, g + nz), slice(g, g + ny), slice(g, g + nx))
        exp_fY = (fb["rY_n"][sl] - fb["rY_o"][sl]) * dtinv - fb["IR"][sl]
        exp_fH = (fb["rH_n"][sl] - fb["rH_o"][sl]) * dtinv
        assert torch.equal(fb["fY"][sl], exp_fY)
        assert torch.equal(fb["fH"][sl], exp_fH)
        for key in ("fY", "fH"):
            ghost = fb[key].clone()
            ghost[sl] = 7.0
            assert torch.all(ghost == 7.0)
    r.close()
