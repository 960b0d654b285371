#!/usr/bin/env python
"""Chemistry-step throughput of the B200 HP reactor (cells/s per chem step).

Workload: the drm19-shaped flame field (21 species + T, 84 reactions of the
bundled synthetic CH4/air mechanism; the drm19 mechanism file itself is not
available), 128^3 = 2,097,152 cells, dt_react = 1e-6 s, P = 1 atm, rtol 1e-8 /
atol 1e-12, max order 5 (the parity settings of the dense-direct BDF).  One
step = one react call over the whole field, state restored between steps
(inputs of 750 MB, far larger than L2).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Multi-GPU: one process per GPU (torchrun); every rank reacts its own copy of
the field (cells shard with no exchange), so scaling is weak and the value is
the cells of all ranks over the slowest rank's device time.

`--impl reference` times the CPU restatement of the dense-direct BDF (the
oracle; the reference's own CVODE reactor cannot be built here) on the host
cores, rank 0 only, over a seeded random sample of the same field.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

from pelelmex_b200 import sharding  # noqa: E402

METRIC = "cells/s per chem step (drm19 128^3) at ≤1e-4 T err: hybrid vs plain GPU BDF"
UNIT = "cells/s"
MECH = "synth_ch4_21"
RTOL, ATOL, QMAX, MAXSTEPS = 1e-8, 1e-12, 5, 10000


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--edge", type=int, default=128)
    p.add_argument("--dt", type=float, default=None,
                   help="dt_react (default 1e-6 s; 5e-6 s for the dodecane random field)")
    p.add_argument("--workload", default="flame_ch4", choices=["flame_ch4", "c12_boxes", "c12_grf"],
                   help="flame_ch4: drm19-shaped 128^3 flame field (the headline); c12_boxes: dodecane AMR-like "
                        "list of 40 boxes in one launch; c12_grf: dodecane random-field flame at --edge^3")
    p.add_argument("--cpu-seconds", type=float, default=15.0, help="bound of the CPU baseline sample")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    p.add_argument("--cells", type=int, default=0,
                   help="react only this many seeded random cells of the field (small profiling cases)")
    p.add_argument("--no-hybrid", action="store_true", help="plain BDF only (no surrogate arm)")
    p.add_argument("--no-c12", action="store_true", help="skip the dodecane box-list block of the headline line")
    p.add_argument("--no-autotune", action="store_true", help="default launch shape (no autotuner pass)")
    p.add_argument("--refine-keep-ppm", type=int, default=0,
                   help="> 0: FP32 solve accuracy (ppm) below which a Newton correction skips the FP64 refinement "
                        "(0: refine every correction, the default)")
    p.add_argument("--tune-cells", type=int, default=262144, help="cells of the autotuner's sample")
    return p.parse_args()


# DRAM bytes (read + write) of rk_ctrl per cell it processes: ncu
# dram__bytes_read.sum + dram__bytes_write.sum summed over every rk_ctrl
# launch of the kernel-profile pass of `bench.py --cells 262144`, divided by
# the cells those launches processed.
CTRL_DRAM_BYTES_PER_CELL = 10050.0


def workload_config(args):
    sub = f" ({args.cells} seeded random cells)" if args.cells else ""
    return {"workload": f"flame_ch4 {args.edge}^3{sub} drm19-shaped (synth_ch4_21: 21 species + T, 84 reactions), "
                        f"dt_react {args.dt:g} s, P 1 atm",
            "mechanism": MECH, "cells": args.cells or args.edge ** 3, "dt_react": args.dt, "rtol": RTOL, "atol": ATOL,
            "max_order": QMAX, "l2": "inputs 750 MB > L2, state restored from a device copy between steps"}


GPU_INTEGRATOR = "plain GPU BDF, round-based (FP64 state/rates, FP32 Newton inverse + FP64 refinement)"
HYBRID_INTEGRATOR = "hybrid: surrogate ensemble (tcgen05 BF16 MLPs) with gated fallback to the plain GPU BDF"
CPU_INTEGRATOR = ("CPU oracle: FP64 C restatement of the dense-direct variable-order BDF (CVODE denseAJ_direct "
                  "algorithm), OpenMP over cells")


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi clock / throttle-reason samples every 200 ms (read only)."""
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, bus_id: str | None):
        self.bus_id = bus_id
        self.rows = []
        self.proc = None
        self.thread = None

    def __enter__(self):
        cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200"]
        if self.bus_id:
            cmd += ["-i", self.bus_id]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return self
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [s.strip() for s in line.split(",")]
            if len(parts) == 7:
                self.rows.append(parts)

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.thread.join(timeout=5)

    def summary(self):
        sm = []
        mx = None
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[0]))
                mx = float(r[1])
            except ValueError:
                continue
            for nm, v in zip(names, r[3:]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# -------------------------------------------------------------- utilities
def _gen_chunk(a):
    from pelelmex_b200 import mechanism as mechmod, workloads
    edge, seed, lo, hi = a
    f = workloads.flame_ch4(mechmod.builtin(MECH), edge=edge, seed=seed, cells=np.arange(lo, hi, dtype=np.int64))
    return f.rhoY, f.T, f.rhoH


def flame_field(args, seed=2):
    """The full flame field, generated by a pool of host processes (started
    before any CUDA call; each cell depends only on its index and the seed, so
    the chunks concatenate to exactly workloads.flame_ch4's field)."""
    import multiprocessing as mp
    from types import SimpleNamespace
    n = args.edge ** 3
    chunks = 64
    step = (n + chunks - 1) // chunks
    with mp.get_context("spawn").Pool(min(32, os.cpu_count() or 1)) as pool:
        parts = pool.map(_gen_chunk, [(args.edge, seed, lo, min(n, lo + step)) for lo in range(0, n, step)])
    rhoY = np.concatenate([p[0] for p in parts], axis=1)
    T = np.concatenate([p[1] for p in parts])
    rhoH = np.concatenate([p[2] for p in parts])
    return SimpleNamespace(rhoY=rhoY, T=T, rhoH=rhoH, frhoY=np.zeros_like(rhoY), frhoH=np.zeros_like(T),
                           dt=args.dt, ncells=n)


def load_field(args):
    from pelelmex_b200 import mechanism as mechmod
    mech = mechmod.builtin(MECH)
    if args.cells:
        return mech, sample_field(mech, args, args.cells, 4242)
    return mech, flame_field(args)


def fp64_peak_tflops(torch, dev):
    """Live FP64 reference peak: cuBLAS DGEMM 8192^3, best of 5."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    for _ in range(2):
        a @ b
    best = 1e30
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        a @ b
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def fp32_peak_tflops(torch, dev):
    """Live FP32 reference peak: cuBLAS SGEMM 8192^3 without TF32, best of 5."""
    n = 8192
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    a = torch.randn(n, n, dtype=torch.float32, device=dev)
    b = torch.randn(n, n, dtype=torch.float32, device=dev)
    for _ in range(2):
        a @ b
    best = 1e30
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        a @ b
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    torch.backends.cuda.matmul.allow_tf32 = prev
    del a, b
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def sample_field(mech, args, n, seed, dt=None):
    """n seeded random cells of the full field, generated directly."""
    from pelelmex_b200 import workloads
    idx = workloads.sample_cells(args.edge ** 3, n, seed=seed)
    return workloads.flame_ch4(mech, edge=args.edge, dt=dt or args.dt, cells=idx)


def cpu_sample_run(mech, args, seconds: float, nthreads: int = 0):
    """Time the oracle on a seeded random sample sized to about `seconds`.
    Returns (cells/s, sample cells, threads, seconds taken)."""
    from oracle import oracle as orc
    from pelelmex_b200 import mechanism as mechmod
    o = orc.Oracle(mechmod.flatten(mech))
    threads = nthreads or orc.max_threads()
    total = args.edge ** 3
    n = min(total, max(256, 64 * threads))
    while True:
        sub = sample_field(mech, args, n, 777)
        t0 = time.perf_counter()
        o.react(sub.rhoY, sub.frhoY, sub.T, sub.rhoH, sub.frhoH, sub.dt, rtol=RTOL, atol=ATOL,
                max_order=QMAX, max_steps=MAXSTEPS, nthreads=threads)
        el = time.perf_counter() - t0
        if el >= 0.3 * seconds or n >= total:
            return n / el, n, threads, el
        n = min(total, int(n * min(8.0, max(1.5, 0.6 * seconds / max(el, 1e-3)))))


TIGHT = dict(rtol=1e-12, atol=1e-20)


def sample_accuracy(mech, args, dt, gpu, n=2048):
    """Errors on n seeded cells of the field at dt: the GPU results given in
    `gpu` ({name: (T [ncells], rhoY [N, ncells]) device tensors}) against the
    CPU oracle at rtol 1e-8 / atol 1e-12 and against the oracle's tight FP64
    solve (rtol 1e-12 / atol 1e-20); the oracle's own error beside them."""
    import torch
    from oracle import oracle as orc
    from pelelmex_b200 import mechanism as mechmod, workloads
    idx = workloads.sample_cells(args.edge ** 3, n, seed=2468)
    sub = workloads.flame_ch4(mech, edge=args.edge, dt=dt, cells=idx)
    o = orc.Oracle(mechmod.flatten(mech))
    kw = dict(max_order=QMAX, max_steps=100000, nthreads=orc.max_threads())
    ref = o.react(sub.rhoY, sub.frhoY, sub.T, sub.rhoH, sub.frhoH, dt, rtol=RTOL, atol=ATOL, **kw)
    tight = o.react(sub.rhoY, sub.frhoY, sub.T, sub.rhoH, sub.frhoH, dt, **TIGHT, **kw)
    rho = sub.rhoY.sum(axis=0)

    def err(T, Y, RT, RY):
        return {"max_rel_T": float(np.max(np.abs(T - RT) / RT)),
                "max_abs_Y": float(np.max(np.abs(Y - RY).max(axis=0) / rho))}
    out = {"sample_cells": int(len(idx)), "oracle_vs_oracle_tight": err(ref["T"], ref["rhoY"], tight["T"],
                                                                        tight["rhoY"]),
           "oracle_tight": "oracle BDF at rtol 1e-12 / atol 1e-20", "tolerances": f"rtol {RTOL:g} / atol {ATOL:g}"}
    it = torch.as_tensor(idx, device=next(iter(gpu.values()))[0].device)
    for name, (T, rY) in gpu.items():
        gT = T.index_select(0, it).cpu().numpy()
        gY = rY.index_select(1, it).cpu().numpy()
        out[f"{name}_vs_oracle"] = err(gT, gY, ref["T"], ref["rhoY"])
        out[f"{name}_vs_oracle_tight"] = err(gT, gY, tight["T"], tight["rhoY"])
    return out


def emit(line):
    print(json.dumps(line), flush=True)


# ------------------------------------------------------- reference arm
def run_reference(args, rank, world):
    cfg = workload_config(args)
    if rank != 0:
        return
    from oracle import oracle as orc
    from pelelmex_b200 import mechanism as mechmod
    mech = mechmod.builtin(MECH)
    total = args.edge ** 3
    o = orc.Oracle(mechmod.flatten(mech))
    threads = orc.max_threads()
    per_step = max(2.0, 150.0 / max(1, args.steps + args.warmup))
    rate, n, _, _ = cpu_sample_run(mech, args, per_step, threads)
    times = []
    for s in range(args.warmup + args.steps):
        sub = sample_field(mech, args, n, 1000 + s)
        t0 = time.perf_counter()
        o.react(sub.rhoY, sub.frhoY, sub.T, sub.rhoH, sub.frhoH, sub.dt, rtol=RTOL, atol=ATOL, max_order=QMAX,
                max_steps=MAXSTEPS, nthreads=threads)
        if s >= args.warmup:
            times.append(time.perf_counter() - t0)
    value = n * len(times) / sum(times)
    ms_full = total / value * 1e3
    sample = (f"{n} seeded random cells of the {args.edge}^3 field per step, CPU restatement of the dense-direct "
              f"BDF (OpenMP, {threads} threads), extrapolated linearly to {total} cells")
    emit({"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
          "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_full, "higher_is_better": True,
          "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfg,
          "integrator": CPU_INTEGRATOR,
          "extrapolated": {"ms_per_step": True, "sample_cells_per_step": n, "cells": total},
          "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
          "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}})


# ------------------------------------------------------------- B200 arm
SURROGATE = ROOT / "pelelmex_b200" / "surrogates" / f"{MECH}.b2s"


def time_steps(fn, restore, steps, warmup, stream, barrier):
    """warmup untimed calls, then `steps` calls each bracketed by CUDA events
    on the launching stream (state restored before every call, outside the
    events).  Returns the per-step milliseconds."""
    import torch
    for _ in range(warmup):
        restore()
        fn()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    barrier()
    torch.cuda.synchronize()
    for s in range(steps):
        restore()
        ev[s][0].record(stream)
        fn()
        ev[s][1].record(stream)
    torch.cuda.synchronize()
    barrier()
    return [a.elapsed_time(b) for a, b in ev]


def run_b200(args, rank, world, local_rank, field):
    import torch
    import torch.distributed as dist
    from pelelmex_b200 import mechanism as mechmod, perfmodel
    from pelelmex_b200.reactor import ReactorB200

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    props = torch.cuda.get_device_properties(dev)
    bus = getattr(props, "pci_bus_id", None)
    bus_id = f"{props.pci_domain_id:08x}:{bus:02x}:{props.pci_device_id:02x}.0" if bus is not None else None
    mech = mechmod.builtin(MECH)
    nc = field.ncells
    N = mech.n_species
    cfg = workload_config(args)

    r = ReactorB200(MECH, rtol=RTOL, atol=ATOL, max_order=QMAX, max_steps=MAXSTEPS,
                    refine_keep_ppm=args.refine_keep_ppm).init()
    base = {k: torch.tensor(getattr(field, k), device=dev) for k in ("rhoY", "T", "rhoH", "frhoY", "frhoH")}
    rY, T, rH = (torch.empty_like(base[k]) for k in ("rhoY", "T", "rhoH"))
    fct = torch.zeros(nc, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)

    def restore():
        rY.copy_(base["rhoY"])
        T.copy_(base["T"])
        rH.copy_(base["rhoH"])

    def barrier():
        if world > 1:
            dist.barrier()

    # launch shape: the cached one of this mechanism and GPU, else the
    # autotuner on a seeded sample of the same field distribution (untimed,
    # before the warm-up), then cached
    cache = ROOT / "pelelmex_b200" / "tuning" / f"{MECH}.b2t"
    if not args.no_autotune and r.load_tuning(cache):
        launch_tuning = dict(r.get_tuning(), source=f"cache {cache.relative_to(ROOT)}")
    elif not args.no_autotune:
        tf = sample_field(mech, args, min(args.tune_cells, nc), seed=77)
        td = {k: torch.tensor(getattr(tf, k), device=dev) for k in ("rhoY", "T", "rhoH", "frhoY", "frhoH")}
        t0 = time.perf_counter()
        tuning, tune_ms = r.autotune(td["rhoY"], td["frhoY"], td["T"], td["rhoH"], td["frhoH"], field.dt,
                                     max_trials=32)
        launch_tuning = dict(tuning, sample_cells=tf.ncells, sample_ms=round(tune_ms, 3),
                             seconds=round(time.perf_counter() - t0, 2), source="autotuned")
        del td
        if rank == 0:
            cache.parent.mkdir(exist_ok=True)
            r.save_tuning(cache)
    else:
        launch_tuning = dict(r.get_tuning(), autotuned=False)

    def plain_step(dt):
        return lambda: r.react_flat(rY, base["frhoY"], T, rH, base["frhoH"], fct, dt_react=dt)

    # integrator counters of one call (untimed)
    restore()
    counters = r.react_flat(rY, base["frhoY"], T, rH, base["frhoH"], fct, dt_react=field.dt, stats=True)[2]
    torch.cuda.synchronize()

    # headline timed region: K plain BDF steps at the configured dt
    launches0 = r.kernel_launches()
    with ClockSampler(bus_id) as clk:
        step_ms = time_steps(plain_step(field.dt), restore, args.steps, args.warmup, stream, barrier)
    launches = (r.kernel_launches() - launches0) * args.steps // (args.steps + args.warmup)
    ms = sharding.step_time_max(sum(step_ms) / len(step_ms), dev)
    value = world * nc / (ms * 1e-3)
    plain = {"value": value, "unit": UNIT, "ms_per_step": ms, "step_ms": step_ms}

    # both time steps of the drm19 config: plain BDF, hybrid, accuracy against
    # a tight FP64 solve of every cell
    from pelelmex_b200.surrogate import Ensemble, HybridReactor
    ens = Ensemble.load(SURROGATE, mech) if (SURROGATE.exists() and not args.no_hybrid) else None
    rt = ReactorB200(MECH, rtol=TIGHT["rtol"], atol=TIGHT["atol"], max_order=QMAX, max_steps=100000,
                     lu_fp64=True).init()
    blocks = {}
    other = 1e-5 if field.dt == 1e-6 else 1e-6
    k2 = max(3, args.steps // 4)
    hy_headline = None
    for dt in (field.dt, other):
        blk = {"dt_react": dt}
        if dt == field.dt:
            blk["plain_ms_per_step"] = ms
        else:
            pms = time_steps(plain_step(dt), restore, k2, 2, stream, barrier)
            blk["plain_ms_per_step"] = sharding.step_time_max(sum(pms) / len(pms), dev)
            blk["plain_steps"] = k2
        blk["plain_value"] = world * nc / (blk["plain_ms_per_step"] * 1e-3)
        # the plain result and the tight reference of every cell
        restore()
        r.react_flat(rY, base["frhoY"], T, rH, base["frhoH"], fct, dt_react=dt)
        pT, pY = T.clone(), rY.clone()
        restore()
        t0 = time.perf_counter()
        rt.react_flat(rY, base["frhoY"], T, rH, base["frhoH"], dt_react=dt)
        torch.cuda.synchronize()
        tT, tY = T.clone(), rY.clone()
        blk["tight_solve"] = {"what": "GPU BDF over every cell at rtol 1e-12 / atol 1e-20 with an FP64 Newton LU",
                              "seconds": round(time.perf_counter() - t0, 2)}
        rho = base["rhoY"].sum(dim=0)

        def errs(Tx, Yx, Tr, Yr):
            return {"max_rel_T": float(((Tx - Tr).abs() / Tr).max().item()),
                    "max_abs_Y": float(((Yx - Yr).abs().max(dim=0).values / rho).max().item())}
        blk["plain_vs_tight"] = errs(pT, pY, tT, tY)
        gpu_res = {"plain": (pT, pY), "gpu_tight": (tT, tY)}
        if ens is not None:
            h = HybridReactor(r, ens)

            def hstep(dt=dt, h=h):
                return h.react_flat(rY, base["frhoY"], T, rH, base["frhoH"], fct, dt_react=dt, stats=False)
            restore()
            h.react_flat(rY, base["frhoY"], T, rH, base["frhoH"], fct, dt_react=dt)  # gate counts
            hT, hY = T.clone(), rY.clone()
            last = dict(h.last)
            hk = args.steps if dt == field.dt else k2
            l0 = r.kernel_launches()
            hms_list = time_steps(hstep, restore, hk, 2 if dt != field.dt else args.warmup, stream, barrier)
            hl = (r.kernel_launches() - l0) * hk // (hk + (2 if dt != field.dt else args.warmup))
            hms = sharding.step_time_max(sum(hms_list) / len(hms_list), dev)
            e_t = errs(hT, hY, tT, tY)
            blk["hybrid"] = {"value": world * nc / (hms * 1e-3), "ms_per_step": hms, "steps": hk,
                             "speedup_vs_plain_gpu_bdf": blk["plain_ms_per_step"] / hms,
                             "accepted_fraction": last["accepted_fraction"],
                             "gate": {k: last[k] for k in last if k.startswith("rejected_") or k in
                                      ("predicted", "accepted")},
                             "vs_tight": e_t, "vs_plain_gpu_bdf": errs(hT, hY, pT, pY),
                             "meets_1e-4_T_bar": e_t["max_rel_T"] <= 1e-4, "gpu_launches": hl,
                             "rule": ens.opts.__dict__}
            gpu_res["hybrid"] = (hT, hY)
            if dt == field.dt:
                hy_headline = (blk["hybrid"], h)
            else:
                h.close()
        if rank == 0 and not args.no_cpu:
            blk["sample"] = sample_accuracy(mech, args, dt, gpu_res)
        blocks[f"dt_{dt:g}"] = blk
    rt.close()
    hybrid = hy_headline[0] if hy_headline else None
    # the headline is the faster of the two integrators that meets the 1e-4
    # temperature bar against the tight solve (the plain BDF does)
    use_hybrid = hybrid is not None and hybrid["meets_1e-4_T_bar"] and hybrid["value"] > value
    if use_hybrid:
        value = hybrid["value"]

    # end to end through the public API from pinned host buffers
    e2e = None
    if not args.no_e2e:
        host = {k: torch.from_numpy(np.ascontiguousarray(getattr(field, k))).pin_memory()
                for k in ("rhoY", "T", "rhoH", "frhoY", "frhoH")}
        out = {k: torch.empty_like(host[k]).pin_memory() for k in ("rhoY", "T", "rhoH")}
        fct_h = torch.empty(nc, dtype=torch.float64).pin_memory()
        dbuf = {k: torch.empty_like(base[k]) for k in host}
        h2d = sum(t.numel() * t.element_size() for t in host.values())
        d2h = sum(t.numel() * t.element_size() for t in out.values()) + fct_h.numel() * 8
        hy = hy_headline[1] if (use_hybrid and hy_headline) else None

        def e2e_step():
            for k in host:
                dbuf[k].copy_(host[k], non_blocking=True)
            if hy is not None:
                hy.react_flat(dbuf["rhoY"], dbuf["frhoY"], dbuf["T"], dbuf["rhoH"], dbuf["frhoH"], fct,
                              dt_react=field.dt, stats=False)
            else:
                r.react_flat(dbuf["rhoY"], dbuf["frhoY"], dbuf["T"], dbuf["rhoH"], dbuf["frhoH"], fct,
                             dt_react=field.dt)
            for k in out:
                out[k].copy_(dbuf[k], non_blocking=True)
            fct_h.copy_(fct, non_blocking=True)

        e2e_step()
        torch.cuda.synchronize()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            e2e_step()
        e1.record(stream)
        torch.cuda.synchronize()
        ems = e0.elapsed_time(e1) / args.steps
        ems = sharding.step_time_max(ems, dev)
        e2e = {"value": world * nc / (ems * 1e-3), "unit": UNIT, "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "ms_per_step": ems, "path": "hybrid" if hy is not None else "plain GPU BDF"}
    if hy_headline:
        hy_headline[1].close()

    # per-kernel profile: one more react of the same field with CUDA events
    # around every launch (kernel by kernel, outside the timed region)
    restore()
    torch.cuda.nvtx.range_push("kernel_profile_pass")  # the range ncu's launch lists select
    r.profile_begin()
    r.react_flat(rY, base["frhoY"], T, rH, base["frhoH"], fct, dt_react=field.dt)
    prof = r.profile_end()
    torch.cuda.nvtx.range_pop()
    kernels, tot_ms = {}, sum(v["ms"] for k, v in prof.items() if k != "complete")
    for k in ("start", "rhs", "ctrl", "jac", "gj", "ctrl_setup"):
        v = prof[k]
        b = perfmodel.kernel_bytes(k, N) * v["cells"]
        kernels[k] = dict(v, share=v["ms"] / tot_ms if tot_ms else None,
                          algorithmic_gbs=(b / (v["ms"] * 1e-3) / 1e9) if v["ms"] else None, bytes=b)
    # dominant kernel: rk_ctrl (both of its launches per round)
    c_ms = kernels["ctrl"]["ms"] + kernels["ctrl_setup"]["ms"]
    c_launch = kernels["ctrl"]["launches"] + kernels["ctrl_setup"]["launches"]
    c_cells = kernels["ctrl"]["cells"] + kernels["ctrl_setup"]["cells"]
    c_bytes = kernels["ctrl"]["bytes"] + kernels["ctrl_setup"]["bytes"]
    hbm_peak, hbm_src = None, None
    mp_ = ROOT / "MEASURED_PEAKS.json"
    if mp_.exists():
        try:
            hbm_peak = json.loads(mp_.read_text()).get("hbm_gbs")
            hbm_src = "measured (MEASURED_PEAKS.json hbm_gbs)"
        except (ValueError, OSError):
            hbm_peak = None
    if hbm_peak is None:
        hbm_peak, hbm_src = 6650.0, "fallback 6.65 TB/s"
    c_gbs = c_bytes / (c_ms * 1e-3) / 1e9
    roof = {"bound": "hbm", "achieved": c_gbs, "peak": hbm_peak, "unit": "GB/s", "frac": c_gbs / hbm_peak,
            "traffic": (CTRL_DRAM_BYTES_PER_CELL * c_cells / c_launch) if CTRL_DRAM_BYTES_PER_CELL else None,
            "kernel": "rk_ctrl (step control + FP32-inverse Newton solve with FP64 refinement), both launches "
                      "of each round",
            "peak_source": hbm_src, "launches": c_launch, "avg_launch_ms": c_ms / c_launch,
            "algorithmic_bytes_per_cell": perfmodel.kernel_bytes("ctrl", N), "cells_per_launch": c_cells / c_launch,
            "share_of_react_kernels": c_ms / tot_ms, "profile_complete": prof["complete"],
            "kernels": kernels}

    # FP64 view of the whole react call (algorithmic flops per call, exp/log
    # counted as one flop each and reported separately)
    counts = perfmodel.op_counts(r.flat)
    cn = {k: counters[k] / nc for k in ("nfe", "nje", "nlu", "nst")}
    fl_cell = perfmodel.flops_per_cell(counts, cn["nfe"], cn["nje"], cn["nlu"], cn["nfe"], cn["nst"])
    exp_cell = cn["nfe"] * counts["rhs_exp"] + cn["nje"] * counts["jac_exp"]
    achieved = fl_cell * nc / (ms * 1e-3) / 1e12
    peak = fp64_peak_tflops(torch, dev)
    n1 = N + 1
    gj_ms = kernels["gj"]["ms"]
    gj_tf = kernels["gj"]["cells"] * 2.0 * n1 ** 3 / (gj_ms * 1e-3) / 1e12 if gj_ms else None
    p32 = fp32_peak_tflops(torch, dev)
    roof["fp32_view"] = {"kernel": "rk_gj (FP32 Gauss-Jordan inverse, 2 n^3 flops per setup)", "achieved": gj_tf,
                         "peak": p32, "unit": "TFLOP/s", "frac": gj_tf / p32 if gj_tf else None,
                         "peak_source": "measured live: cuBLAS SGEMM 8192^3 without TF32, best of 5"}
    roof["fp64_view"] = {"achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                         "kernel": "one react call: rk_rhs / rk_ctrl / rk_jac / rk_gj rounds",
                         "counting": "algorithmic flops from the integrator's per-cell counters; exp/log = 1 flop",
                         "peak_source": "measured live: cuBLAS DGEMM 8192^3 best of 5 (FP64 has no entry in the "
                                        "measured-peaks file)",
                         "flops_per_cell": fl_cell, "exp_log_per_cell": exp_cell,
                         "exp_log_per_s": exp_cell * nc / (ms * 1e-3), "per_cell_counters": cn,
                         "io_bytes_per_call": perfmodel.bytes_per_cell(N) * nc}
    if hybrid is not None:
        mlp_flops = 2.0 * ((N + 2 + 15) // 16 * 16 * 256 + 2 * 256 * 256 + 256 * ((N + 1 + 15) // 16 * 16))
        hybrid["mlp_flops_per_cell_per_member"] = mlp_flops

    c12 = None
    if not args.no_c12 and not args.cells:
        c12 = c12_boxes_block(args, dev, stream, barrier, world, rank)

    cpu = None
    if world == 1 and rank == 0 and not args.no_cpu:
        rate, n, threads, el = cpu_sample_run(mech, args, args.cpu_seconds)
        cpu = {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"{n} seeded random cells of the {args.edge}^3 field, oracle restatement of the dense-direct "
                         f"BDF on {threads} host threads ({el:.1f} s), extrapolated to cells/s"}

    if rank == 0:
        path = "hybrid" if use_hybrid else "plain GPU BDF"
        emit({"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
              "warmup": args.warmup, "ms_per_step": world * nc / value * 1e3, "higher_is_better": True,
              "scaling": "weak",
              "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded flame-like field; synthetic "
              "drm19-shaped mechanism)", "config": cfg, "measured_path": path,
              "integrator": HYBRID_INTEGRATOR if use_hybrid else GPU_INTEGRATOR, "launch_tuning": launch_tuning,
              "roofline": roof, "cpu_baseline": cpu, "e2e": e2e,
              "gpu_launches": launches if path != "hybrid" else hybrid["gpu_launches"], "clocks": clk.summary(),
              "plain_gpu_bdf": plain, "hybrid": hybrid, "dt_blocks": blocks, "c12_boxes": c12,
              "counters": {k: int(v) for k, v in counters.items()}})
    r.close()


# ------------------------------------------------------ dodecane workloads
C12 = "synth_c12_53"


def _gen_c12_box(a):
    from pelelmex_b200 import mechanism as mechmod, workloads
    dt, b = a
    return workloads.c12_boxes(mechmod.builtin(C12), dt=dt, only={b})[0]


def c12_box_list(dt, nbox=40):
    """The dodecane AMR-like box list, one box per task of a pool of host
    processes (each box depends only on the seed and its index)."""
    import multiprocessing as mp
    with mp.get_context("spawn").Pool(min(nbox, os.cpu_count() or 1)) as pool:
        return pool.map(_gen_c12_box, [(dt, b) for b in range(nbox)])


def c12_boxes_block(args, dev, stream, barrier, world, rank=0):
    """The C3 workload beside the headline: the 40-box dodecane list in one
    react launch per step (2 warm-up, 3 timed steps, CUDA events), and the
    GPU result of 64 seeded cells per box against the CPU oracle (rtol 1e-8 /
    atol 1e-12) and its tight solve (rtol 1e-12 / atol 1e-20)."""
    import torch
    from oracle import oracle as orc
    from pelelmex_b200 import mechanism as mechmod, workloads
    from pelelmex_b200.reactor import Box, ReactorB200
    mech = mechmod.builtin(C12)
    N = mech.n_species
    boxes = c12_box_list(1e-6)
    r = ReactorB200(C12, rtol=RTOL, atol=ATOL, max_order=QMAX, max_steps=MAXSTEPS,
                    refine_keep_ppm=args.refine_keep_ppm).init()
    work, pristine, items = [], [], []
    for lo, e, f in boxes:
        w = {k: torch.tensor(getattr(f, k), device=dev) for k in ("rhoY", "T", "rhoH", "frhoY", "frhoH")}
        w["fct"] = torch.zeros(f.ncells, dtype=torch.float64, device=dev)
        work.append(w)
        pristine.append({k: w[k].clone() for k in ("rhoY", "T", "rhoH")})
        v = lambda t, c: t.view(c, e, e, e)  # noqa: E731
        items.append((Box(lo, (lo[0] + e - 1, e - 1, e - 1)), v(w["rhoY"], N), v(w["frhoY"], N), v(w["T"], 1),
                      v(w["rhoH"], 1), v(w["frhoH"], 1), v(w["fct"], 1), None))
    total = sum(f.ncells for _, _, f in boxes)

    def restore():
        for w, p in zip(work, pristine):
            for k in p:
                w[k].copy_(p[k])
    step_ms = time_steps(lambda: r.react_boxes(items, 1e-6), restore, 3, 2, stream, barrier)
    ms = sharding.step_time_max(sum(step_ms) / len(step_ms), dev)
    del work, pristine, items
    out = {"workload": "c12_boxes: 40 dodecane boxes (edges 16/32/64, half cold 300-600 K, half igniting "
                       "900-1400 K, phi 0.5-2), synth_c12_53, dt_react 1e-6 s, one react launch per box list",
           "cells": total, "value": world * total / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms, "steps": 3,
           "step_ms": step_ms}
    if rank != 0 or args.no_cpu:
        r.close()
        return out
    # accuracy on 64 seeded cells per box
    sub = workloads.c12_boxes(mech, dt=1e-6, box_cells=64)
    cat = lambda key, ax: np.ascontiguousarray(np.concatenate([getattr(f, key) for _, _, f in sub], axis=ax))  # noqa
    rY0, T0, rH0, fY, fH = cat("rhoY", 1), cat("T", 0), cat("rhoH", 0), cat("frhoY", 1), cat("frhoH", 0)
    g = [torch.tensor(a, device=dev) for a in (rY0, T0, rH0, fY, fH)]
    r.react_flat(g[0], g[3], g[1], g[2], g[4], dt_react=1e-6)
    gT, gY = g[1].cpu().numpy(), g[0].cpu().numpy()
    r.close()
    o = orc.Oracle(mechmod.flatten(mech))
    kw = dict(max_order=QMAX, max_steps=100000, nthreads=orc.max_threads())
    ref = o.react(rY0, fY, T0, rH0, fH, 1e-6, rtol=RTOL, atol=ATOL, **kw)
    tight = o.react(rY0, fY, T0, rH0, fH, 1e-6, **TIGHT, **kw)
    rho = rY0.sum(axis=0)

    def err(T, Y, RT, RY):
        return {"max_rel_T": float(np.max(np.abs(T - RT) / RT)),
                "max_abs_Y": float(np.max(np.abs(Y - RY).max(axis=0) / rho))}
    out["sample"] = {"cells": int(T0.size), "gpu_vs_oracle": err(gT, gY, ref["T"], ref["rhoY"]),
                     "gpu_vs_oracle_tight": err(gT, gY, tight["T"], tight["rhoY"]),
                     "oracle_vs_oracle_tight": err(ref["T"], ref["rhoY"], tight["T"], tight["rhoY"])}
    return out


def _gen_c12_chunk(a):
    from pelelmex_b200 import mechanism as mechmod, workloads
    edge, dt, cells = a
    f = workloads.c12_flame_grf(mechmod.builtin(C12), edge=edge, dt=dt, cells=cells)
    return f.rhoY, f.T, f.rhoH


def c12_grf_field(args, idx):
    """The dodecane random-field cells `idx`, generated by a pool of host
    processes for large fields (each cell depends only on its index)."""
    from pelelmex_b200 import mechanism as mechmod, workloads
    mech = mechmod.builtin(C12)
    if len(idx) <= (1 << 18):
        return workloads.c12_flame_grf(mech, edge=args.edge, dt=args.dt, cells=idx)
    import multiprocessing as mp
    parts = np.array_split(np.asarray(idx, dtype=np.int64), 256)
    with mp.get_context("spawn").Pool(min(32, os.cpu_count() or 1)) as pool:
        out = pool.map(_gen_c12_chunk, [(args.edge, args.dt, p) for p in parts])
    rhoY = np.concatenate([o[0] for o in out], axis=1)
    T = np.concatenate([o[1] for o in out])
    rhoH = np.concatenate([o[2] for o in out])
    return workloads.Field(mech, rhoY, T, rhoH, np.zeros_like(rhoY), np.zeros_like(T), args.dt, (len(idx),),
                           "c12_flame_grf")


def c12_class_accuracy(mech, flat, work, args, per_class=96):
    """GPU result against the oracle (rtol 1e-8 / atol 1e-12) and the tight
    oracle (rtol 1e-12 / atol 1e-20) on seeded samples of each cell class of
    the random-field flame: cold (T0 < 600 K), igniting (900 <= T0 < 1500 K),
    burnt (T0 >= 1800 K)."""
    from oracle import oracle as orc
    from pelelmex_b200 import mechanism as mechmod
    f = flat[0]
    T0 = f.T
    classes = {"cold": T0 < 600.0, "igniting": (T0 >= 900.0) & (T0 < 1500.0), "burnt": T0 >= 1800.0}
    o = orc.Oracle(mechmod.flatten(mech))
    rng = np.random.default_rng(20261203)
    gT_all = work[0]["T"]
    gY_all = work[0]["rhoY"]
    out = {}
    for name, m in classes.items():
        cand = np.nonzero(m)[0]
        if cand.size == 0:
            continue
        idx = np.sort(rng.choice(cand, min(per_class, cand.size), replace=False))
        sub = f.subset(idx)
        kw = dict(max_order=QMAX, max_steps=100000, nthreads=orc.max_threads())
        ref = o.react(sub.rhoY, sub.frhoY, sub.T, sub.rhoH, sub.frhoH, f.dt, rtol=RTOL, atol=ATOL, **kw)
        tight = o.react(sub.rhoY, sub.frhoY, sub.T, sub.rhoH, sub.frhoH, f.dt, rtol=1e-12, atol=1e-20, **kw)
        import torch
        it = torch.as_tensor(idx, device=gT_all.device)
        gT = gT_all.index_select(0, it).cpu().numpy()
        gY = gY_all.index_select(1, it).cpu().numpy()
        rho = sub.rhoY.sum(axis=0)

        def err(T, Y, RT, RY):
            return {"max_rel_T": float(np.max(np.abs(T - RT) / RT)),
                    "max_abs_Y": float(np.max(np.abs(Y - RY).max(axis=0) / rho))}
        out[name] = {"cells_in_class": int(cand.size), "sample": int(idx.size),
                     "gpu_vs_oracle": err(gT, gY, ref["T"], ref["rhoY"]),
                     "gpu_vs_oracle_tight": err(gT, gY, tight["T"], tight["rhoY"]),
                     "oracle_vs_oracle_tight": err(ref["T"], ref["rhoY"], tight["T"], tight["rhoY"])}
    return out


def run_dodecane(args, rank, world, local_rank):
    """The dodecane workloads (53 species + T): the AMR-like box list (all of
    this rank's boxes in one react launch, boxes dealt round-robin over the
    ranks) or the random-field flame (flat, cells split over the ranks).
    Same timing rules as the headline line; the CPU baseline is the oracle
    on a bounded seeded sample of the same cells."""
    from pelelmex_b200 import mechanism as mechmod, workloads
    mech = mechmod.builtin(C12)
    N = mech.n_species
    if args.workload == "c12_boxes":
        boxes = c12_box_list(args.dt)
        mine = sharding.shard_boxes(boxes, rank, world)
        total = sum(f.ncells for _, _, f in boxes)
        wl = (f"c12_boxes: {len(boxes)} dodecane boxes (edges 16/32/64, half cold 300-600 K, half igniting "
              f"900-1400 K, phi 0.5-2), {total} cells, one react launch per box list")
        flat = [f for _, _, f in mine]
    else:
        n_all = args.edge ** 3
        idx = sharding.shard_cells(n_all, rank, world)
        flat = [c12_grf_field(args, idx)]
        total = n_all
        wl = f"c12_grf: dodecane random-field flame {args.edge}^3 (T 300-2400 K, Z 0-1), {total} cells"
    cfg = {"workload": wl + f", synth_c12_53 (53 species + T, {mech.n_reactions} reactions), dt_react "
                            f"{args.dt:g} s, P 1 atm",
           "mechanism": C12, "cells": total, "dt_react": args.dt, "rtol": RTOL, "atol": ATOL, "max_order": QMAX,
           "integrator": "plain GPU BDF, round-based (FP64 state/rates, FP32 Newton inverse + FP64 refinement)",
           "l2": "inputs larger than L2, state restored from a device copy between steps"}
    if args.impl == "reference":
        if rank == 0:
            rate, n, threads, _ = c12_cpu_rate(mech, flat, args.cpu_seconds)
            emit({"impl": "reference", "metric": f"cells/s per chem step ({args.workload})", "value": rate,
                  "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                  "ms_per_step": total / rate * 1e3, "higher_is_better": True, "scaling": "weak",
                  "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfg,
                  "cpu_baseline": {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
                                   "sample": f"{n} seeded cells of the workload, oracle BDF, extrapolated"},
                  "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}})
        return
    import torch
    import torch.distributed as dist
    from pelelmex_b200.reactor import Box, ReactorB200
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    props = torch.cuda.get_device_properties(dev)
    bus = getattr(props, "pci_bus_id", None)
    bus_id = f"{props.pci_domain_id:08x}:{bus:02x}:{props.pci_device_id:02x}.0" if bus is not None else None
    r = ReactorB200(C12, rtol=RTOL, atol=ATOL, max_order=QMAX, max_steps=MAXSTEPS,
                    refine_keep_ppm=args.refine_keep_ppm).init()
    stream = torch.cuda.current_stream(dev)
    # device state: working arrays plus pristine copies to restore between steps
    work, pristine = [], []
    for f in flat:
        w = {k: torch.tensor(getattr(f, k), device=dev) for k in ("rhoY", "T", "rhoH", "frhoY", "frhoH")}
        w["fct"] = torch.zeros(f.ncells, dtype=torch.float64, device=dev)
        work.append(w)
        pristine.append({k: w[k].clone() for k in ("rhoY", "T", "rhoH")})
    mine_cells = sum(f.ncells for f in flat)

    def restore():
        for w, p in zip(work, pristine):
            for k in p:
                w[k].copy_(p[k])

    if args.workload == "c12_boxes":
        items = []
        for (lo, e, f), w in zip(mine, work):
            v = lambda t, c: t.view(c, e, e, e)  # noqa: E731
            items.append((Box(lo, (lo[0] + e - 1, e - 1, e - 1)), v(w["rhoY"], N), v(w["frhoY"], N), v(w["T"], 1),
                          v(w["rhoH"], 1), v(w["frhoH"], 1), v(w["fct"], 1), None))

        def step(stats=False):
            return r.react_boxes(items, args.dt, stats=stats)
    else:
        w0 = work[0]

        def step(stats=False):
            return r.react_flat(w0["rhoY"], w0["frhoY"], w0["T"], w0["rhoH"], w0["frhoH"], w0["fct"],
                                dt_react=args.dt, stats=stats)
    if not args.no_autotune:
        # seeded sample across all of this rank's cells, flat layout
        # igniting random-field cells cost ~20x a box-list cell: a smaller sample
        tune_cells = min(args.tune_cells, 16384 if args.workload == "c12_grf" else 65536)
        take = []
        for f in flat:
            k = max(1, int(round(tune_cells * f.ncells / mine_cells)))
            take.append(f.subset(workloads.sample_cells(f.ncells, min(k, f.ncells), seed=91)))
        cat = lambda key, ax: torch.tensor(np.concatenate([getattr(t, key) for t in take], axis=ax),  # noqa: E731
                                           device=dev)
        t0 = time.perf_counter()
        tuning, tune_ms = r.autotune(cat("rhoY", 1).contiguous(), cat("frhoY", 1).contiguous(), cat("T", 0),
                                     cat("rhoH", 0), cat("frhoH", 0), args.dt, max_trials=32)
        cfg["launch_tuning"] = dict(tuning, sample_ms=round(tune_ms, 3), seconds=round(time.perf_counter() - t0, 2))
    counters = None
    for wi in range(args.warmup):
        restore()
        res = step(stats=(wi == 0))
        if wi == 0:
            counters = res[2]
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    l0 = r.kernel_launches()
    with ClockSampler(bus_id) as clk:
        for s_ in range(args.steps):
            restore()
            ev[s_][0].record(stream)
            step()
            ev[s_][1].record(stream)
        torch.cuda.synchronize()
    launches = r.kernel_launches() - l0
    step_ms = [a.elapsed_time(b) for a, b in ev]
    ms = sum(step_ms) / len(step_ms)
    ms = sharding.step_time_max(ms, dev)
    counters = sharding.counters_sum(counters, dev)
    if rank != 0:
        r.close()
        return
    cpu = None
    if not args.no_cpu:
        rate, n, threads, el = c12_cpu_rate(mech, flat, args.cpu_seconds)
        cpu = {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"{n} seeded cells of the workload, oracle BDF on {threads} host threads ({el:.1f} s), "
                         f"extrapolated to cells/s"}
    accuracy = None
    if args.workload == "c12_grf" and not args.no_cpu:
        # the result of one more react of the field (untimed) against the oracle per cell class
        restore()
        step()
        torch.cuda.synchronize()
        accuracy = c12_class_accuracy(mech, flat, work, args)
    emit({"metric": f"cells/s per chem step ({args.workload})", "value": total / (ms * 1e-3), "unit": UNIT,
          "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
          "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded; synthetic "
          "dodecane-shaped mechanism)", "config": cfg, "cpu_baseline": cpu, "e2e": None, "gpu_launches": launches,
          "clocks": clk.summary(), "step_ms": step_ms, "accuracy_by_class": accuracy,
          "counters": {k: int(v) for k, v in counters.items()} if counters else None})
    r.close()


def c12_cpu_rate(mech, flat, seconds):
    """Oracle cells/s on a seeded sample drawn across the workload's fields,
    grown until the run takes about a third of `seconds`."""
    from oracle import oracle as orc
    from pelelmex_b200 import mechanism as mechmod, workloads
    o = orc.Oracle(mechmod.flatten(mech))
    threads = orc.max_threads()
    total = sum(f.ncells for f in flat)
    n = max(64, 8 * threads)
    while True:
        parts = []
        for i, f in enumerate(flat):
            k = max(1, int(round(n * f.ncells / total)))
            parts.append(f.subset(workloads.sample_cells(f.ncells, min(k, f.ncells), seed=500 + i)))
        cat = lambda key, ax: np.ascontiguousarray(np.concatenate([getattr(p, key) for p in parts], axis=ax))  # noqa
        m = sum(p.ncells for p in parts)
        t0 = time.perf_counter()
        o.react(cat("rhoY", 1), cat("frhoY", 1), cat("T", 0), cat("rhoH", 0), cat("frhoH", 0), flat[0].dt,
                rtol=RTOL, atol=ATOL, max_order=QMAX, max_steps=MAXSTEPS, nthreads=threads)
        el = time.perf_counter() - t0
        if el >= 0.3 * seconds or m >= total:
            return m / el, m, threads, el
        n = min(total, int(n * min(8.0, max(1.5, 0.6 * seconds / max(el, 1e-3)))))


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    args.warmup = max(3, args.warmup)
    if args.dt is None:
        args.dt = 5e-6 if args.workload == "c12_grf" else 1e-6
    if args.impl == "reference":
        # the CPU reference runs on rank 0 alone; the other ranks exit
        if args.workload != "flame_ch4":
            run_dodecane(args, rank, world, local_rank)
        else:
            run_reference(args, rank, world)
        return
    field = None
    if args.workload == "flame_ch4":
        # host-side field generation, before any CUDA call (process pool)
        field = load_field(args)[1]
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local_rank))
    try:
        if args.workload != "flame_ch4":
            run_dodecane(args, rank, world, local_rank)
        else:
            run_b200(args, rank, world, local_rank, field)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
