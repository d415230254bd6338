#!/usr/bin/env python
"""Benchmark of the state-vector gate-application path on B200.

Workload (default): the 30-qubit, 20-layer complex128 layered circuit - per
layer RX(theta_q) and RZ(phi_q) on every qubit then the CNOT ladder
(q, q+1), angles seeded (splitmix64, seed 1234), state |0..0> (16 GiB).
One step = one full execution of the circuit (initialisation + every group
pass = 20 layers). Metric: layers per second of the gate phase.

  value     device time (CUDA events on the launch stream) of K steps with
            the state resident in HBM; the state (16 GiB) exceeds L2, so no
            flush is needed between steps.
  e2e       the same metric through the public C ABI as a user calls it:
            per step Simulator(circuit) (plan + upload of the gate data from
            host memory) + execute(proba_state_in) with host (theta, phi)
            in and the reference's proba_state copied back to the host.
  roofline  the group-pass kernel: algorithmic bytes per launch (read and
            write of every amplitude: 2 * 16 B * 2^n) / its average launch
            time in the timed region, against MEASURED_PEAKS.json hbm_gbs.
  cpu_baseline  the reference's own CPU simulator (compiled from its
            headers into oracle/_ref) on a bounded sample: one layer of the
            same 30-qubit circuit, compiled as the reference's best CPU
            configuration (scheduling, fusion(5), grouping(12)).

``--impl reference`` times the reference's CPU implementation alone on this
workload (same metric), rank 0 only. ``--gpus N`` (torchrun) runs N
independent replicas, one per GPU (the path does not shard on one GPU).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "30q layers/s"
UNIT = "layers/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="kate_b200", choices=["kate_b200", "reference"])
    ap.add_argument("--nqubits", type=int, default=30)
    ap.add_argument("--layers", type=int, default=20)
    ap.add_argument("--seed", type=int, default=1234)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


def workload_config(args):
    return {"workload": f"layered RX/RZ/CNOT-ladder circuit, n={args.nqubits}, {args.layers} layers, complex128",
            "nqubits": args.nqubits, "layers": args.layers, "seed": args.seed,
            "gates": args.layers * (3 * args.nqubits - 1), "state_bytes": 16 << args.nqubits,
            "l2": "state larger than L2 (126 MB); no flush needed", "parallelism": "replicas"}


class Clocks:
    """Samples nvidia-smi clocks during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = os.path.join(ROOT, "gpurun_out", f"clocks_{os.getpid()}.csv")

    def __enter__(self):
        os.makedirs(os.path.dirname(self.path), exist_ok=True)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if self.proc is None or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        load = [s for s in sm if mx and s > 0.3 * mx] or sm
        return {"sm_mhz": statistics.median(load) if load else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_hbm_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        try:
            return float(json.load(open(p))["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


def committed_traffic(n):
    """Per-launch DRAM bytes of the group-pass kernel from the committed ncu
    summary (profiles/group_pass_traffic.json), scaled to 2^n amplitudes."""
    p = os.path.join(ROOT, "profiles", "group_pass_traffic.json")
    if not os.path.exists(p):
        return None
    try:
        d = json.load(open(p))
        return d["dram_bytes_per_launch"] * (2.0 ** n) / (2.0 ** d["nqubits"])
    except Exception:
        return None


def cpu_reference_sample(n, seed):
    """Times one layer of the n-qubit circuit on the reference's CPU simulator."""
    from kate_b200 import circuits
    from oracle.oracle import Ref, available_ref

    if available_ref():
        ref = Ref()
        c = ref.circuit(n, circuits.layered(n, 1, seed))
        c.schedule()
        c.fuse(5, 1e-6)
        c.group(12)
        c.compile_default(0)
        sess = c.session()
        ms = sess.run()
        sess.close()
        return {"value": 1000.0 / ms, "unit": UNIT, "cores": ref.hw_threads(), "kind": "reference",
                "sample": f"1 layer of the n={n} circuit ({3 * n - 1} gates) on the reference CPUSimulator "
                          f"(gateScheduling+gateFusion(5)+gateGrouping(12)), gate phase only",
                "ms_per_layer": ms}
    from oracle.oracle import Oracle
    o = Oracle()
    nn = min(n, 26)
    t0 = time.perf_counter()
    o.simulate(nn, circuits.layered(nn, 1, seed))
    ms = (time.perf_counter() - t0) * 1000 * (2 ** (n - nn))
    return {"value": 1000.0 / ms, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"1 layer at n={nn} on the C restatement, scaled by 2^{n - nn}", "ms_per_layer": ms}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from kate_b200 import circuits
    from oracle.oracle import Ref, available_ref
    n = args.nqubits
    if not available_ref():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libkate_ref.so was not built "
                          "(the reference headers were absent at build time)"}))
        return
    ref = Ref()
    c = ref.circuit(n, circuits.layered(n, 1, args.seed))
    c.schedule()
    c.fuse(5, 1e-6)
    c.group(12)
    c.compile_default(0)
    sess = c.session()
    for _ in range(args.warmup):
        sess.run()
    times = [sess.run() for _ in range(args.steps)]
    sess.close()
    total_ms = sum(times)
    value = args.steps * 1000.0 / total_ms
    cores = ref.hw_threads()
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c128 (f64)", "data": "synthetic",
            "impl": "reference", "config": workload_config(args),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                             "sample": f"each step = 1 layer of the n={n} circuit on the reference "
                                       f"CPUSimulator (gateScheduling+gateFusion(5)+gateGrouping(12)), "
                                       f"gate phase only, {cores} threads"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return

    import numpy as np
    import torch
    import kate_b200 as K
    from kate_b200 import circuits

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = world > 1
    if dist:
        import datetime
        import torch.distributed as tdist
        torch.cuda.set_device(local)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)

    n, L = args.nqubits, args.layers
    gates = circuits.layered(n, L, args.seed)
    circ = K.Circuit(n, gates)
    sim = K.Simulator(circ, 1, K.C128, local)
    passes = sim.passes()
    launches = sim.launches_per_run()

    stream = torch.cuda.Stream(device=dev)
    for _ in range(args.warmup):
        sim.run_async(stream.cuda_stream)
    stream.synchronize()
    if dist:
        tdist.barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            sim.run_async(stream.cuda_stream)
        ev1.record(stream)
        ev1.synchronize()
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    if dist:
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
        ms = float(t.item())
    ms_per_step = ms / args.steps
    value = world * args.steps * L / (ms / 1000.0)

    # Per-launch times of the group-pass kernel (events between launches).
    init_ms, pass_ms = sim.profile_passes()
    avg_pass_ms = (ms_per_step - init_ms) / max(1, len(passes))
    alg_bytes = 2.0 * 16.0 * (2 ** n)
    peak, peak_kind = measured_hbm_peak()
    achieved = alg_bytes / (avg_pass_ms / 1000.0) / 1e9

    # End to end through the C ABI with host buffers.
    e2e_steps = max(1, min(args.steps, 3))
    tp_in = np.zeros((n, 2))
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        s2 = K.Simulator(circ, 1, K.C128, local)
        s2.execute(K.proba_state(tp_in))
        s2.close()
    e2e_ms = (time.perf_counter() - t0) * 1000.0 / e2e_steps
    if dist:
        t = torch.tensor([e2e_ms], device=dev, dtype=torch.float64)
        tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    n_ops = sum(ng for _, ng in passes)
    h2d = n_ops * 112 + 16 * (4 ** 1) * n_ops + 2 * n * 8
    d2h = 2 * n * 8 + 16 * (1 + 2 * (12 + 4)) * (1 << 14)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        del sim
        torch.cuda.empty_cache()
        try:
            cpu = cpu_reference_sample(n, args.seed)
        except Exception as e:  # reported, not fatal
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": f"failed: {e}"}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "c128 (f64)", "data": "synthetic (seeded angles)",
                "config": workload_config(args),
                "e2e": {"value": world * L / (e2e_ms / 1000.0), "unit": UNIT, "h2d_bytes_per_step": h2d,
                        "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms},
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "traffic": committed_traffic(n),
                             "peak_source": peak_kind, "kernel": "k_pass_generic",
                             "alg_bytes_per_launch": alg_bytes, "avg_launch_ms": avg_pass_ms,
                             "profiled_pass_ms": {"min": min(pass_ms), "max": max(pass_ms),
                                                  "mean": sum(pass_ms) / len(pass_ms)}},
                "passes_per_step": len(passes), "passes_per_layer": len(passes) / L,
                "gpu_launches": launches * args.steps, "clocks": clk.summary(),
                "cpu_baseline": cpu}
        print(json.dumps(line))
    if dist:
        tdist.barrier()
        tdist.destroy_process_group()


if __name__ == "__main__":
    main()
