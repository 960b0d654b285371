#!/usr/bin/env python
"""Forward pass of the surrogate MLP on the tensor cores, timed alone.

    python bench_mlp.py --rows 262144 --passes 10 [--terms 1|2]

Random weights of the surrogate's shape (N+2 inputs padded to 32, three
hidden layers of 256 GELU units, N+1 outputs padded to 32) and random
feature rows; each pass is the four tcgen05 GEMMs of MLPSurrogate.forward,
with inputs and activations in one BF16 term or two (hi | lo; twice the MMA
work of the network's own flops).  Prints one JSON line: ms per pass, the
network's TFLOP/s, the tensor-core TFLOP/s executed, and their fraction of
the measured BF16 peak when the peaks file is present.  Used for the
tensor-core GEMM's timing and ncu captures; it exercises no integrator code.
"""
from __future__ import annotations

import argparse
import json
from pathlib import Path


import sys

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))


def main():
    import torch
    from pelelmex_b200 import mechanism as mechmod
    from pelelmex_b200.surrogate import HIDDEN, MLPSurrogate

    p = argparse.ArgumentParser()
    p.add_argument("--rows", type=int, default=262144)
    p.add_argument("--passes", type=int, default=10)
    p.add_argument("--mechanism", default="synth_ch4_21")
    p.add_argument("--terms", type=int, default=2, choices=[1, 2])
    a = p.parse_args()
    rows = (a.rows + 127) // 128 * 128
    net = MLPSurrogate(mechmod.builtin(a.mechanism), seed=1, terms=a.terms)
    g = torch.Generator(device="cuda:0").manual_seed(2)
    x = torch.randn((rows, a.terms * net.kin), generator=g, device="cuda:0").to(torch.bfloat16)
    for _ in range(3):
        net.forward(x)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(a.passes):
        net.forward(x)
    e1.record()
    torch.cuda.synchronize()
    net.check_error()
    ms = e0.elapsed_time(e1) / a.passes
    flops = 2.0 * rows * (net.kin * HIDDEN + 2 * HIDDEN * HIDDEN + HIDDEN * net.kout)
    tf = flops / (ms * 1e-3) / 1e12
    tf_exec = a.terms * tf
    peak = None
    mp = ROOT / "MEASURED_PEAKS.json"
    if mp.exists():
        try:
            peak = json.loads(mp.read_text()).get("bf16_tflops")
        except (ValueError, OSError):
            peak = None
    print(json.dumps({"rows": rows, "terms": a.terms, "ms_per_pass": ms, "tflops": tf, "tflops_executed": tf_exec,
                      "bf16_peak_tflops": peak, "frac_executed": tf_exec / peak if peak else None,
                      "gemms_per_pass": 4}), flush=True)


if __name__ == "__main__":
    main()
