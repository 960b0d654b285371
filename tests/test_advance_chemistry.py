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
