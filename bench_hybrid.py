#!/usr/bin/env python
"""One hybrid react (b200chem_react_hybrid) on seeded cells of the flame
field, timed alone, next to the plain BDF react of the same cells.

    python bench_hybrid.py [--cells 262144] [--dt 1e-6] [--reps 3]

Loads the committed surrogate ensemble, reacts `--cells` seeded random cells
of the drm19-shaped 128^3 flame field (seed 2, the benchmark's field) with the
plain BDF and with the hybrid, `--reps` timed calls each after a warm-up call,
and prints one JSON line: ms per call (CUDA events), the gate's counts and the
largest relative T difference of the hybrid from the plain BDF.  Used for the
launch lists and ncu captures of the hybrid's kernels (features, the
two-term tcgen05 GEMMs, the gate, gather / scatter, and the BDF rounds of
the rejected cells).
"""
from __future__ import annotations

import argparse
import json
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--cells", type=int, default=262144)
    p.add_argument("--dt", type=float, default=1e-6)
    p.add_argument("--reps", type=int, default=3)
    a = p.parse_args()
    from pelelmex_b200 import mechanism as M, workloads as W
    mech = M.builtin("synth_ch4_21")
    f = W.flame_ch4(mech, cells=W.sample_cells(128 ** 3, a.cells, seed=4242), dt=a.dt)
    import torch
    from pelelmex_b200.reactor import ReactorB200
    from pelelmex_b200.surrogate import Ensemble, HybridReactor
    dev = "cuda:0"
    r = ReactorB200(mech, rtol=1e-8, atol=1e-12, max_order=5).init()
    h = HybridReactor(r, Ensemble.load(ROOT / "pelelmex_b200" / "surrogates" / "synth_ch4_21.b2s", mech))
    base = [torch.tensor(x, device=dev) for x in (f.rhoY, f.T, f.rhoH, f.frhoY, f.frhoH)]

    def timed(fn):
        ms = []
        for i in range(a.reps + 1):
            s = [b.clone() for b in base[:3]]
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn(s)
            e1.record()
            torch.cuda.synchronize()
            if i:
                ms.append(e0.elapsed_time(e1))
        return s, min(ms)

    ps, p_ms = timed(lambda s: r.react_flat(s[0], base[3], s[1], s[2], base[4], dt_react=a.dt))
    hs, h_ms = timed(lambda s: h.react_flat(s[0], base[3], s[1], s[2], base[4], dt_react=a.dt))
    err = ((hs[1] - ps[1]).abs() / ps[1]).max().item()
    print(json.dumps({"cells": f.ncells, "dt": a.dt, "plain_ms": p_ms, "hybrid_ms": h_ms, "speedup": p_ms / h_ms,
                      "gate": {k: v for k, v in h.last.items() if k != "stats"},
                      "max_rel_T_diff_vs_plain": err}), flush=True)
    h.close()
    r.close()


if __name__ == "__main__":
    main()
