"""Train the surrogate ensemble on BDF-labelled cells of seeded flame fields.

    python -m pelelmex_b200.train_surrogate [--cells 1048576] [--steps 4000] [--out FILE]

The training fields are seeded random samples of the drm19-shaped 128^3
flame field with seeds distinct from the evaluation fields; every cell is
labelled by the plain GPU BDF at rtol 1e-8 / atol 1e-12.
"""
from __future__ import annotations

import argparse
import time


def main():
    import torch

    from . import mechanism as M, workloads as W
    from .reactor import ReactorB200
    from .surrogate import train_ensemble

    p = argparse.ArgumentParser()
    p.add_argument("--mechanism", default="synth_ch4_21")
    p.add_argument("--cells", type=int, default=1 << 20)
    p.add_argument("--steps", type=int, default=4000)
    p.add_argument("--members", type=int, default=2)
    p.add_argument("--dt", type=float, default=1e-6)
    p.add_argument("--seed", type=int, default=10)
    p.add_argument("--out", default="surrogate_ensemble.pt")
    a = p.parse_args()
    mech = M.builtin(a.mechanism)
    r = ReactorB200(mech, rtol=1e-8, atol=1e-12, max_order=5).init()
    t0 = time.time()
    f = W.flame_ch4(mech, cells=W.sample_cells(128 ** 3, a.cells, seed=a.seed), dt=a.dt, seed=a.seed)
    nets = train_ensemble(r, mech, [f], members=a.members, steps=a.steps)
    torch.save([n.state_dict() for n in nets], a.out)
    print(f"trained {len(nets)} networks on {a.cells} cells in {time.time() - t0:.1f} s -> {a.out}")


if __name__ == "__main__":
    main()
