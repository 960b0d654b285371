"""Generate the golden fixtures used to pin the CPU oracle.

The reference holds no stored values for this boundary (its reactor and
mechanisms are absent from the snapshot), so the oracle is pinned against two
independent computations instead:

* rates_<mech>.npz -- right-hand side of the HP system at seeded states,
  from the numpy restatement oracle/kinetics_np.py;
* traj_<mech>.npz  -- end states of seeded cells integrated with scipy's
  Radau (an implicit Runge-Kutta method, independent of the BDF under test)
  at rtol 1e-12 / atol 1e-20, with the finite-difference Jacobian of the
  numpy right-hand side.

Run from the repository root:  python tests/golden/make_golden.py
"""
import sys
from pathlib import Path

import numpy as np
from scipy.integrate import solve_ivp

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))
from kinetics_np import NpKinetics  # noqa: E402

from pelelmex_b200 import mechanism as M  # noqa: E402

HERE = Path(__file__).resolve().parent
FUEL = {"synth_h2_9": ("H2", 0.5), "synth_ch4_21": ("CH4", 2.0), "synth_c12_53": ("NC12H26", 18.5)}


def states(mech, K, rng, n):
    N = mech.n_species
    nm = mech.names
    fuel, o2 = FUEL[mech.name]
    out = []
    for i in range(n):
        X = np.zeros(N)
        X[nm.index(fuel)] = 1.0
        X[nm.index("O2")] = o2 * rng.uniform(0.7, 1.3)
        X[nm.index("N2")] = 3.76 * o2
        X += rng.uniform(0, 1, N) ** 4 * 0.05  # some radicals and products
        X /= X.sum()
        Y = M.mole_to_mass(mech, X)
        T = rng.uniform(1100, 2200)
        rho = K.density(T, Y)
        y = np.concatenate([rho * Y, [T]])
        F = np.zeros(N + 1)
        if i % 2 == 1:  # forcing like the SDC advection/diffusion source
            F[:N] = rho * Y * rng.normal(0, 20.0, N)
            F[:N] -= F[:N].sum() * Y
            F[N] = rng.normal(0, 1e9)
        out.append((y, F))
    return out


def main():
    for name in ("synth_h2_9", "synth_ch4_21", "synth_c12_53"):
        mech = M.builtin(name)
        K = NpKinetics(M.flatten(mech))
        rng = np.random.default_rng(2024)
        st = states(mech, K, rng, 6)
        ys = np.array([s[0] for s in st])
        Fs = np.array([s[1] for s in st])
        np.savez_compressed(HERE / f"rates_{name}.npz", y=ys, F=Fs, ydot=K.rhs(ys, Fs))
        dt = 1e-5
        ends = []
        for y0, F in st[:4]:
            sol = solve_ivp(lambda t, y: K.rhs(y, F), (0.0, dt), y0, method="Radau", rtol=1e-12, atol=1e-20,
                            jac=lambda t, y: K.jac_fd(y, F, rel=1e-5))
            assert sol.status == 0
            ends.append(sol.y[:, -1])
        np.savez_compressed(HERE / f"traj_{name}.npz", y0=ys[:4], F=Fs[:4], dt=dt, y1=np.array(ends))
        print(name, "done")


if __name__ == "__main__":
    main()
