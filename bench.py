#!/usr/bin/env python
"""Benchmark of the state-vector gate-application path on B200.

Workload (default): the 30-qubit, 20-layer complex128 layered circuit - per
layer RX(theta_q) and RZ(phi_q) on every qubit then the CNOT ladder
(q, q+1), angles seeded (splitmix64, seed 1234), state |0..0> (16 GiB).
One step = one full execution of the circuit from |0..0> (every group pass
= 20 layers; the first pass generates |0..0> itself, so no separate
initialisation kernel runs). Metric: layers per second of the gate phase.

  value     device time (CUDA events on the launch stream) of K steps with
            the state resident in HBM; the state (16 GiB) exceeds L2, so no
            flush is needed between steps.
  e2e       the same metric through the public C ABI as a user calls it:
            per step Simulator(circuit) (plan + upload of the gate data from
            host memory) + execute(proba_state_in) with host (theta, phi)
            in and the reference's proba_state copied back to the host.
  roofline  the group-pass kernel (one pass-specialised kernel per pass):
            algorithmic bytes of the step's passes (every pass reads and
            writes every amplitude, 2 * 16 B * 2^n, except the first of a
            run from |0..0>, which generates its input and only writes) /
            their time in the timed region, against MEASURED_PEAKS.json
            hbm_gbs; per-pass rates come from CUDA events between launches.
  cpu_baseline  the reference's own CPU simulator (compiled from its
            headers into oracle/_ref) on a bounded sample: one layer of the
            same 30-qubit circuit, compiled as the reference's best CPU
            configuration (scheduling, fusion(5), grouping(12)).
  ref_gpu_baseline  the reference's own GPU path (its HIPcode headers built
            with nvcc into oracle/_ref) on the same GPU and circuit, with
            scheduling, fusion(5) and grouping(9), gate phase on the wall
            clock; its proba_state is compared with this library's.

``--impl reference`` times the reference's CPU implementation alone on this
workload (same metric), rank 0 only. ``--gpus N`` (torchrun) runs N
independent replicas, one per GPU (the path does not shard on one GPU).

Other workloads (``--workload``), one JSON line each:
  precision  32-qubit complex64 brickwork of Haar SU(4) gates, 20 layers,
             5-qubit blocks formed by the planner on the tensor cores
             (split-BF16 products, FP32 accumulation): layers/s,
             speed-up over the complex128 path on the same circuit, and the
             infidelity against complex128 at n=28.
  batch      4096 hardware-efficient-ansatz circuits (n uniform in 10..22,
             depth 2n, complex64) in one persistent CUDA-graph launch,
             autotuned: circuits/s, against one Simulator launch per circuit.
  serve      a Poisson stream of layered-circuit requests (n truncated
             geometric on 12..28, depth n, complex64, 1024 samples + <Z>)
             through the continuous-batching server under a 150 GB
             admission budget, rates swept: circuits/s and p50/p99 latency,
             against one-at-a-time plain launches.
  qulacs     the reference's own benchmark circuit (QulacsBench, 25 qubits,
             complex128): ms per execution, lower is better, against its
             published 1x MI200 time (vs_baseline), its CPU simulator and its
             GPU path on the same GPU.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "30q layers/s"


def metric_name(n):
    """The headline metric; another qubit count names its own."""
    return METRIC if n == 30 else f"{n}q layers/s"
UNIT = "layers/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="kate_b200", choices=["kate_b200", "reference"])
    ap.add_argument("--workload", default="layers", choices=["layers", "precision", "batch", "serve", "qulacs"])
    ap.add_argument("--nqubits", type=int, default=None)
    ap.add_argument("--layers", type=int, default=20)
    ap.add_argument("--circuits", type=int, default=4096, help="batch: circuits in the batch")
    ap.add_argument("--requests", type=int, default=1000, help="serve: requests per rate")
    ap.add_argument("--rates", default="1000,4000,16000", help="serve: arrival rates (requests/s)")
    ap.add_argument("--step-us", type=int, default=0, help="serve: step latency target in us (0: default)")
    ap.add_argument("--tensor-blocks", type=int, default=0, choices=[0, 1],
                    help="serve, and batch with --no-autotune: 1 runs complex64 passes of states kept in "
                         "device memory as tensor-core blocks")
    ap.add_argument("--seed", type=int, default=1234)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-ref-gpu", action="store_true", help="layers: skip the reference's own GPU path")
    ap.add_argument("--no-autotune", action="store_true", help="batch: default plan choices")
    ap.add_argument("--no-baseline", action="store_true", help="batch/serve: skip the one-at-a-time baseline")
    a = ap.parse_args()
    if a.nqubits is None:
        a.nqubits = {"precision": 32, "qulacs": 25}.get(a.workload, 30)
    return a


L2_BYTES = 126 << 20


def l2_flush_buffer(n, dev, amp_bytes=16):
    """A buffer twice the L2 size to write between timed steps when the
    state (amp_bytes * 2^n) is smaller than 128 MiB; None otherwise."""
    import torch
    if (amp_bytes << n) >= (128 << 20):
        return None
    return torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device=dev)


def l2_note(n, amp_bytes=16):
    if (amp_bytes << n) >= (128 << 20):
        return "state larger than L2 (126 MB); no flush needed"
    return "state smaller than L2: each timed step follows a 252 MB buffer write (L2 flushed), timed on its own"


def workload_config(args):
    return {"workload": f"layered RX/RZ/CNOT-ladder circuit, n={args.nqubits}, {args.layers} layers, complex128",
            "nqubits": args.nqubits, "layers": args.layers, "seed": args.seed,
            "gates": args.layers * (3 * args.nqubits - 1), "state_bytes": 16 << args.nqubits,
            "l2": l2_note(args.nqubits), "parallelism": "replicas"}


class Clocks:
    """Samples nvidia-smi clocks during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        # KATE_CLOCKS_DIR keeps the samples where the caller wants them.
        d = os.environ.get("KATE_CLOCKS_DIR") or tempfile.gettempdir()
        self.path = os.path.join(d, f"kate_clocks_{os.getpid()}_{index}.csv")

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


NOMINAL_HBM_GBS = 8000.0  # B200 HBM3e, nominal


def per_pass_gbs(alg_bytes, pass_ms, peak):
    """Each pass's HBM rate (algorithmic bytes / its event-timed duration)
    as a distribution, against the measured and the nominal peak."""
    g = sorted(alg_bytes / (ms / 1000.0) / 1e9 for ms in pass_ms if ms > 0)
    if not g:
        return None
    med = statistics.median(g)
    return {"min": g[0], "median": med, "max": g[-1], "median_frac": med / peak,
            "median_frac_of_nominal": med / NOMINAL_HBM_GBS, "passes": len(g)}


PASS_KERNEL = "kate_pass (pass-specialised register-staged group pass, NVRTC for sm_100a)"


def pass_roofline(n, npass, launches, ms_per_step, init_ms):
    """Algorithmic bytes and time of a step's group passes. Every pass reads
    and writes the 16-byte amplitudes once; when the run starts from |0..0>
    the first pass generates its input (launches == passes: no separate
    initialisation kernel) and only writes. Returns (bytes per launch on
    average, ms per launch on average, achieved GB/s)."""
    zero_start = launches == npass
    step_bytes = (2 * npass - (1 if zero_start else 0)) * 16.0 * 2 ** n
    step_ms = ms_per_step - (0.0 if zero_start else init_ms)
    return step_bytes / npass, step_ms / npass, step_bytes / (step_ms / 1000.0) / 1e9


FP64_PER_SM_CLK = 64     # FP64 instructions per SM per clock on B200 (ncu: dfma peak_sustained 64/SM)
SMEM_BYTES_PER_SM_CLK = 128  # shared-memory bytes per SM per clock (32 banks x 4 B)


def pass_bounds(n, work, pass_ms, hbm_gbs, sm_mhz, nsm):
    """Lower bound of each group pass's time from the three rates it uses:
    HBM bytes at the measured copy bandwidth, FP64 instructions and
    shared-memory bytes at B200's per-SM-clock rates times the SM clock
    sampled during the timed region. A pass is bound by the slowest; the
    sum over passes against the measured per-pass times says how close
    the kernels run to that bound."""
    if not sm_mhz or not work or any(w is None for w in work):
        return None
    amps = 2.0 ** n
    f = sm_mhz * 1e6
    tot = {"hbm": 0.0, "fp64": 0.0, "smem": 0.0}
    binding = {"hbm": 0, "fp64": 0, "smem": 0}
    bound = 0.0
    for (hb, fp, sb) in work:
        t = {"hbm": hb * amps / (hbm_gbs * 1e9) * 1e3, "fp64": fp * amps / (FP64_PER_SM_CLK * nsm * f) * 1e3,
             "smem": sb * amps / (SMEM_BYTES_PER_SM_CLK * nsm * f) * 1e3}
        for k in tot:
            tot[k] += t[k]
        k = max(t, key=t.get)
        binding[k] += 1
        bound += t[k]
    measured = float(sum(pass_ms))
    return {"unit": "ms per step", "hbm_ms": tot["hbm"], "fp64_ms": tot["fp64"], "smem_ms": tot["smem"],
            "bound_ms": bound, "measured_ms": measured, "frac": bound / measured if measured > 0 else None,
            "passes_bound_by": binding, "sm_mhz": sm_mhz,
            "rates": {"hbm_gbs": hbm_gbs, "fp64_per_sm_clk": FP64_PER_SM_CLK,
                      "smem_bytes_per_sm_clk": SMEM_BYTES_PER_SM_CLK, "sms": nsm}}


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


def max_over_ranks(ms, device=None):
    """The slowest rank's time (torch.distributed all-reduce MAX; the group
    may be NCCL on GPUs or gloo on CPU). Returns ms unchanged without a
    process group."""
    import torch
    import torch.distributed as tdist
    if not (tdist.is_available() and tdist.is_initialized()):
        return ms
    t = torch.tensor([ms], device=device, dtype=torch.float64)
    tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
    return float(t.item())


def replica_rate(units_per_rank, ms_max, world):
    """Whole-job throughput of N independent replicas: all ranks' units over
    the slowest rank's time."""
    return world * units_per_rank / (ms_max / 1000.0)


def ref_sample_layers(n, L):
    """Layers of the circuit one CPU-reference step runs: the whole circuit
    when it is small (seconds at n <= 22, e.g. the 20-qubit 10-layer
    configuration), else one layer of it (a 30-qubit layer takes about 20 s
    on 16 cores; the whole circuit would take minutes)."""
    return L if n <= 22 else 1


def cpu_reference_sample(n, seed, L=1):
    """Times the reference's CPU simulator on ref_sample_layers(n, L) layers
    of the n-qubit circuit."""
    from kate_b200 import circuits
    from oracle.oracle import Ref, available_ref

    if available_ref():
        ref = Ref()
        ls = ref_sample_layers(n, L)
        c = ref.circuit(n, circuits.layered(n, ls, seed))
        c.schedule()
        c.fuse(5, 1e-6)
        c.group(12)
        c.compile_default(0)
        sess = c.session()
        ms = sess.run()
        sess.close()
        return {"value": ls * 1000.0 / ms, "unit": UNIT, "cores": ref.hw_threads(), "kind": "reference",
                "sample": f"{ls} layer(s) of the n={n} circuit ({ls * (3 * n - 1)} gates) on the reference "
                          f"CPUSimulator (gateScheduling+gateFusion(5)+gateGrouping(12)), gate phase only",
                "ms_per_layer": ms / ls}
    from oracle.oracle import Oracle
    o = Oracle()
    nn = min(n, 26)
    t0 = time.perf_counter()
    o.simulate(nn, circuits.layered(nn, 1, seed))
    ms = (time.perf_counter() - t0) * 1000 * (2 ** (n - nn))
    return {"value": 1000.0 / ms, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"1 layer at n={nn} on the C restatement, scaled by 2^{n - nn}", "ms_per_layer": ms}


def reference_gpu_sample(n, L, seed, kate_proba=None, budget_s=90.0):
    """The reference's own GPU path on this GPU (oracle/_ref/libkate_ref_gpu.so,
    built from its HIPcode headers): the same circuit through gateScheduling,
    gateFusion(5, 1e-6), gateGrouping(9) (the largest group its kernel keeps
    inside its shared memory) and compileDefault(0). Its gate phase
    (executeCommand per group, each ending in a device synchronise) is timed
    on the wall clock: one warm-up run, then up to 3 runs within budget_s.
    Its proba_state is compared with this library's (kate_proba)."""
    import numpy as np
    from kate_b200 import circuits
    from oracle import ref_gpu

    if not ref_gpu.available():
        return {"value": None, "unavailable": "oracle/_ref/libkate_ref_gpu.so was not built"}
    c = ref_gpu.RefGpuCircuit(n, circuits.layered(n, L, seed))
    t0 = time.perf_counter()
    c.compile(fuse=5, mtm=1e-6, group=ref_gpu.MAX_GROUP_QUBITS)
    plan_s = time.perf_counter() - t0
    s = c.session()
    try:
        t0 = time.perf_counter()
        runs = [s.run()]
        while len(runs) < 4 and time.perf_counter() - t0 < budget_s / 2:
            runs.append(s.run())
        proba = s.proba_state()
    finally:
        s.close()
    timed = runs[1:] if len(runs) > 1 else runs
    ms = sum(timed) / len(timed)
    out = {"value": L / (ms / 1000.0), "unit": UNIT, "ms_per_step": ms, "runs_timed": len(timed),
           "plan": "gateScheduling + gateFusion(5, 1e-6) + gateGrouping(9) + compileDefault(0)",
           "plan_s": plan_s, "gates": c.num_gates(), "groups": c.num_groups(), "max_group": c.max_group(),
           "timing": "wall clock of the reference's instruction loop (it synchronises after every group)"}
    if kate_proba is not None:
        d = np.abs(np.asarray(kate_proba) - proba)
        d[:, 1] = np.minimum(d[:, 1], 2 * np.pi - d[:, 1])
        out["proba_state_max_abs_diff_vs_kate_b200"] = float(d.max())
    return out


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
    ls = ref_sample_layers(n, args.layers)
    c = ref.circuit(n, circuits.layered(n, ls, args.seed))
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
    value = args.steps * ls * 1000.0 / total_ms
    cores = ref.hw_threads()
    sample = (f"each step = {ls} layer(s) of the n={n} circuit (the same seeded angles; "
              f"{'the whole circuit' if ls == args.layers else 'one layer, planned on its own'}) on the "
              f"reference CPUSimulator (gateScheduling+gateFusion(5)+gateGrouping(12)), gate phase only, "
              f"{cores} threads")
    cfg = dict(workload_config(args), reference_sample=sample)
    line = {"metric": metric_name(args.nqubits), "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c128 (f64)", "data": "synthetic",
            "impl": "reference", "config": cfg,
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def main():
    args = parse()
    if args.workload != "layers":
        {"precision": run_precision, "batch": run_batch, "serve": run_serve,
         "qulacs": run_qulacs}[args.workload](args)
        return
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
    flush = l2_flush_buffer(n, dev)
    with Clocks(local) as clk:
        if flush is None:
            ev0.record(stream)
            for _ in range(args.steps):
                sim.run_async(stream.cuda_stream)
            ev1.record(stream)
            ev1.synchronize()
            ms = ev0.elapsed_time(ev1)
        else:
            # A state smaller than L2: each step timed on its own, after a
            # write of a buffer twice the L2 size (outside the events).
            ms = 0.0
            for _ in range(args.steps):
                with torch.cuda.stream(stream):
                    flush.fill_(1)
                ev0.record(stream)
                sim.run_async(stream.cuda_stream)
                ev1.record(stream)
                ev1.synchronize()
                ms += ev0.elapsed_time(ev1)
    torch.cuda.synchronize()
    del flush
    if dist:
        ms = max_over_ranks(ms, dev)
    ms_per_step = ms / args.steps
    value = replica_rate(args.steps * L, ms, world)

    # Per-launch times of the group-pass kernel (events between launches).
    init_ms, pass_ms = sim.profile_passes()
    alg_bytes, avg_pass_ms, achieved = pass_roofline(n, len(passes), launches, ms_per_step, init_ms)
    peak, peak_kind = measured_hbm_peak()
    sim_work = sim.pass_work()
    clk_summary = clk.summary()

    # End to end through the C ABI with host buffers.
    e2e_steps = max(1, min(args.steps, 3))
    tp_in = np.zeros((n, 2))
    # One untimed step first: the process's first state allocation of this
    # size is a one-time cost (later simulators reuse the released buffer).
    s2 = K.Simulator(circ, 1, K.C128, local)
    s2.execute(K.proba_state(tp_in))
    s2.close()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        s2 = K.Simulator(circ, 1, K.C128, local)
        s2.execute(K.proba_state(tp_in))
        s2.close()
    e2e_ms = (time.perf_counter() - t0) * 1000.0 / e2e_steps
    if dist:
        e2e_ms = max_over_ranks(e2e_ms, dev)
    n_ops = sum(ng for _, ng in passes)
    h2d = n_ops * 112 + 16 * (4 ** 1) * n_ops + 2 * n * 8
    # proba_state: per-CTA partial sums of the bit-sum kernel (2^g CTAs,
    # 1 + 2 (12 + r) complex sums each, g = min(n - 12, 10), r = the rest up
    # to 8), then the (theta, phi) pairs.
    g_bits = min(n - 12, 10)
    r_bits = n - 12 - g_bits
    if r_bits > 8:
        g_bits, r_bits = n - 12 - 8, 8
    d2h = 2 * n * 8 + 16 * (1 + 2 * (12 + r_bits)) * (1 << g_bits)

    ref_gpu = None
    if rank == 0 and world == 1 and not args.no_ref_gpu:
        kate_proba = sim.execute().as_array()
        try:
            ref_gpu = reference_gpu_sample(n, L, args.seed, kate_proba)
        except Exception as e:  # reported, not fatal
            ref_gpu = {"value": None, "unavailable": f"failed: {e}"}
        if ref_gpu.get("value"):
            ref_gpu["value_speedup"] = value / ref_gpu["value"]

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        del sim
        torch.cuda.empty_cache()
        try:
            cpu = cpu_reference_sample(n, args.seed, L)
        except Exception as e:  # reported, not fatal
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": f"failed: {e}"}

    if rank == 0:
        line = {"metric": metric_name(args.nqubits), "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "c128 (f64)", "data": "synthetic (seeded angles)",
                "config": workload_config(args),
                "e2e": {"value": world * L / (e2e_ms / 1000.0), "unit": UNIT, "h2d_bytes_per_step": h2d,
                        "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms},
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "traffic": committed_traffic(n),
                             "peak_source": peak_kind, "kernel": PASS_KERNEL,
                             "alg_bytes_per_launch": alg_bytes, "avg_launch_ms": avg_pass_ms,
                             "profiled_pass_ms": {"min": min(pass_ms), "max": max(pass_ms),
                                                  "mean": sum(pass_ms) / len(pass_ms)},
                             "per_pass_gbs": per_pass_gbs(2.0 * 16.0 * 2 ** n, pass_ms, peak),
                             "frac_of_nominal": achieved / NOMINAL_HBM_GBS,
                             "pass_bounds": pass_bounds(n, sim_work, pass_ms, peak, clk_summary.get("sm_mhz"),
                                                        torch.cuda.get_device_properties(dev).multi_processor_count)},
                "passes_per_step": len(passes), "passes_per_layer": len(passes) / L,
                "gpu_launches": launches * args.steps, "clocks": clk_summary,
                "cpu_baseline": cpu, "ref_gpu_baseline": ref_gpu}
        print(json.dumps(line))
    if dist:
        tdist.barrier()
        tdist.destroy_process_group()



# ---------------------------------------------------------------------------
# Other workloads
# ---------------------------------------------------------------------------

def _common(metric, unit, value, args, ms_per_step, dtype, config, **extra):
    line = {"metric": metric, "value": value, "unit": unit, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": dtype, "data": "synthetic (seeded)", "config": config}
    line.update(extra)
    return line


def _ref_seconds(n, gates, fuse=True):
    """Gate-phase seconds of one circuit on the reference's CPU simulator."""
    from oracle.oracle import Ref
    ref = Ref()
    c = ref.circuit(n, gates)
    if fuse:
        c.schedule()
        c.fuse(5, 1e-6)
        c.group(min(12, n))
    c.compile_default(0)
    sess = c.session()
    ms = sess.run()
    sess.close()
    return ms / 1000.0, ref.hw_threads()


def _reference_unavailable():
    from oracle.oracle import available_ref
    return not available_ref()


def run_precision(args):
    """Brickwork SU(4) at n qubits, complex64 on the tensor-core path."""
    import numpy as np
    import torch
    import kate_b200 as K
    from kate_b200 import circuits

    n, L = args.nqubits, args.layers
    gates = circuits.brickwork_su4(n, L, args.seed)
    cfg = {"workload": f"brickwork of Haar SU(4) gates, n={n}, {L} layers, complex64, fused by the planner's block "
                       f"selector into 5-qubit blocks on tensor cores (split-BF16 x3), two per pass; complex128 "
                       f"comparison on the same circuit (register-stage plan)", "nqubits": n, "layers": L,
           "gates": len(gates),
           "seed": args.seed,
           "state_bytes": 8 << n, "l2": "state larger than L2; no flush needed", "parallelism": "replicas"}
    if args.impl == "reference":
        if _reference_unavailable():
            print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref was not built"}))
            return
        nn = min(n, 24)
        sec, cores = _ref_seconds(nn, circuits.brickwork_su4(nn, 1, args.seed))
        v = 1.0 / (sec * 2 ** (n - nn))
        print(json.dumps(_common("layers/s", "layers/s", v, args, 1000 / v, "c128 (f64)", cfg, impl="reference",
                                 cpu_baseline={"value": v, "unit": "layers/s", "cores": cores, "kind": "reference",
                                               "sample": f"1 layer at n={nn} (complex128, the reference has no "
                                                         f"complex64), scaled by 2^{n - nn}"},
                                 e2e={"value": v, "unit": "layers/s", "h2d_bytes_per_step": 0,
                                      "d2h_bytes_per_step": 0})))
        return
    torch.cuda.set_device(0)
    circ = K.Circuit(n, gates)  # complex128 plan: register stages, each SU(4) a dense two-qubit register op
    # complex64 plan: the planner packs the gates into 5-qubit blocks itself
    # (a prior gateFusion(5) pass leaves 3-5-qubit dense gates that fit its
    # blocks less well: 29 passes against 27).
    fused = K.Circuit(n, gates)
    sim = K.Simulator(fused, 1, K.C64, 0)
    passes = sim.passes()
    stream = torch.cuda.Stream()
    for _ in range(args.warmup):
        sim.run_async(stream.cuda_stream)
    stream.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(0) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            sim.run_async(stream.cuda_stream)
        ev1.record(stream)
        ev1.synchronize()
    ms = ev0.elapsed_time(ev1) / args.steps
    init_ms, pass_ms = sim.profile_passes()
    avg_pass = sum(pass_ms) / len(pass_ms)
    alg = 2.0 * 8.0 * 2 ** n
    peak, peak_kind = measured_hbm_peak()
    launches = sim.launches_per_run()
    sim.close()
    del sim
    # End to end: plan + upload + |0> init + passes + proba_state readback,
    # after one untimed step (the first state allocation of this size is a
    # one-time cost; later simulators reuse the released buffer). Measured
    # before the complex128 and n = 28 runs below, whose states would
    # otherwise take the reused buffer's place.
    e2e_steps = 2
    for i in range(1 + e2e_steps):
        if i == 1:
            t0 = time.perf_counter()
        e = K.Simulator(fused, 1, K.C64, 0)
        e.execute()
        e.close()
    e2e_ms = (time.perf_counter() - t0) * 1000 / e2e_steps
    # The complex128 path on the same circuit.
    s128 = K.Simulator(circ, 1, K.C128, 0)
    s128.run_async(stream.cuda_stream)
    stream.synchronize()
    ev0.record(stream)
    s128.run_async(stream.cuda_stream)
    ev1.record(stream)
    ev1.synchronize()
    ms128 = ev0.elapsed_time(ev1)
    s128.close()
    del s128
    # Infidelity at n = 28 against complex128.
    nf = min(n, 28)
    cf = K.Circuit(nf, circuits.brickwork_su4(nf, L, args.seed))
    cf64 = K.Circuit(nf, circuits.brickwork_su4(nf, L, args.seed))
    a = K.Simulator(cf64, 1, K.C64, 0)
    a.execute()
    psi64 = a.state()
    a.close()
    b = K.Simulator(cf, 1, K.C128, 0)
    b.execute()
    psi128 = b.state()
    b.close()
    ov = np.vdot(psi128, psi64)
    infid = float(1.0 - abs(ov) ** 2 / (np.vdot(psi64, psi64).real * np.vdot(psi128, psi128).real))
    del psi64, psi128
    cpu = None
    if not args.no_cpu_baseline and not _reference_unavailable():
        nn = 24
        sec, cores = _ref_seconds(nn, circuits.brickwork_su4(nn, 1, args.seed))
        cpu = {"value": 1.0 / (sec * 2 ** (n - nn)), "unit": "layers/s", "cores": cores, "kind": "reference",
               "sample": f"1 layer at n={nn} on the reference CPUSimulator (complex128), scaled by 2^{n - nn}"}
    cfg.update({"c128_ms_per_step": ms128, "speedup_vs_c128": ms128 / ms, "infidelity_vs_c128": infid,
                "infidelity_nqubits": nf, "passes_per_step": len(passes), "fused_gates": fused.num_gates()})
    print(json.dumps(_common(
        f"{n}q SU(4) brickwork layers/s (complex64)", "layers/s", L * 1000.0 / ms, args, ms, "c64 (split-bf16 x3 products / f32 accumulation)",
        cfg,
        e2e={"value": L * 1000.0 / e2e_ms, "unit": "layers/s", "h2d_bytes_per_step": len(gates) * 16 * 16,
             "d2h_bytes_per_step": 2 * n * 8, "ms_per_step": e2e_ms},
        roofline={"bound": "hbm", "achieved": alg / (avg_pass / 1000) / 1e9, "peak": peak, "unit": "GB/s",
                  "frac": alg / (avg_pass / 1000) / 1e9 / peak, "traffic": None, "peak_source": peak_kind,
                  "kernel": "k_block_c64 (tcgen05 kind::f16, split-BF16 x3)", "alg_bytes_per_launch": alg,
                  "avg_launch_ms": avg_pass},
        gpu_launches=launches * args.steps, clocks=clk.summary(), cpu_baseline=cpu)))


QULACS_PUBLISHED_MS = 1035.41  # README.md:29 of the reference: QulacsBench 25q on 1x AMD MI200


def run_qulacs(args):
    """The reference's own benchmark circuit (BenchCircuits.hpp:8-42,
    QulacsBench: 41 n Hadamard and CNOT-ring gates) at n qubits, complex128,
    |0..0>; one step = one execution (initialisation + every group pass).
    Metric: wall time per execution in ms (lower is better), the figure the
    reference publishes for 25 qubits (README.md:23-31)."""
    import numpy as np
    from kate_b200 import circuits

    n = args.nqubits
    gates = circuits.qulacs_bench(n)
    cfg = {"workload": f"QulacsBench circuit (H / CNOT-ring layers), n={n}, complex128, |0..0>",
           "nqubits": n, "gates": len(gates), "state_bytes": 16 << n,
           "l2": "state larger than L2 (126 MB); no flush needed" if (16 << n) > (126 << 20)
           else "state fits L2: steps run back to back", "parallelism": "replicas"}
    metric, unit = f"QulacsBench {n}q wall time", "ms"
    published = QULACS_PUBLISHED_MS if n == 25 else None

    def line(value, ms_per_step, dtype, **extra):
        out = _common(metric, unit, value, args, ms_per_step, dtype, cfg, **extra)
        out["higher_is_better"] = False
        out["data"] = "synthetic (the benchmark's fixed gate structure, generated in code)"
        if published is not None:
            out["vs_baseline"] = value / published
            out["vs_baseline_note"] = ("value / 1035.41 ms, the reference's published 1x MI200 time "
                                       "(README.md:29); below 1 is faster")
        return out

    def cpu_run():
        """The reference's CPU simulator on the whole circuit, compiled as its
        main.cpp does (gateScheduling + gateGrouping(12) + compileDefault)."""
        from oracle.oracle import Ref
        ref = Ref()
        c = ref.circuit(n, gates)
        c.schedule()
        c.group(min(12, n))
        c.compile_default(0)
        sess = c.session()
        try:
            return sess.run(), ref.hw_threads()
        finally:
            sess.close()

    if args.impl == "reference":
        if int(os.environ.get("RANK", "0")) != 0:
            return
        if _reference_unavailable():
            print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref was not built"}))
            return
        for _ in range(args.warmup):
            cpu_run()
        runs = [cpu_run() for _ in range(args.steps)]
        ms = sum(r[0] for r in runs) / len(runs)
        cores = runs[0][1]
        print(json.dumps(line(ms, ms, "c128 (f64)", impl="reference",
                              cpu_baseline={"value": ms, "unit": unit, "cores": cores, "kind": "reference",
                                            "sample": f"each step = the whole n={n} circuit on the reference "
                                                      f"CPUSimulator (gateScheduling + gateGrouping(12)), gate "
                                                      f"phase only, {cores} threads"},
                              e2e={"value": ms, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0})))
        return

    import torch
    import kate_b200 as K

    torch.cuda.set_device(0)
    circ = K.Circuit(n, gates)
    sim = K.Simulator(circ, 1, K.C128, 0)
    passes = sim.passes()
    launches = sim.launches_per_run()
    stream = torch.cuda.Stream()
    for _ in range(args.warmup):
        sim.run_async(stream.cuda_stream)
    stream.synchronize()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(0) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            sim.run_async(stream.cuda_stream)
        ev1.record(stream)
        ev1.synchronize()
    ms = ev0.elapsed_time(ev1) / args.steps
    init_ms, pass_ms = sim.profile_passes()
    alg, avg_pass, _ = pass_roofline(n, len(passes), launches, ms, init_ms)
    peak, peak_kind = measured_hbm_peak()
    kate_proba = sim.execute().as_array()
    sim.close()
    del sim

    # End to end through the public API: Simulator(circuit) (plan + upload)
    # + execute() with the proba_state copied to the host, after one untimed
    # step (first allocation of the state).
    e2e_steps = max(1, min(args.steps, 5))
    for i in range(1 + e2e_steps):
        if i == 1:
            t0 = time.perf_counter()
        e = K.Simulator(circ, 1, K.C128, 0)
        e.execute()
        e.close()
    e2e_ms = (time.perf_counter() - t0) * 1000.0 / e2e_steps
    n_ops = sum(ng for _, ng in passes)
    h2d = n_ops * 112 + 16 * 4 * n_ops
    g_bits = min(n - 12, 10)
    r_bits = n - 12 - g_bits
    if r_bits > 8:
        g_bits, r_bits = n - 12 - 8, 8
    d2h = 2 * n * 8 + 16 * (1 + 2 * (12 + r_bits)) * (1 << g_bits)

    ref_gpu = None
    if not args.no_ref_gpu:
        try:
            from oracle import ref_gpu as RG
            if not RG.available():
                ref_gpu = {"value": None, "unavailable": "oracle/_ref/libkate_ref_gpu.so was not built"}
            else:
                rc = RG.RefGpuCircuit(n, gates)
                rc.compile(fuse=0, group=RG.MAX_GROUP_QUBITS)
                s = rc.session()
                try:
                    runs = [s.run() for _ in range(4)]
                    proba = s.proba_state()
                finally:
                    s.close()
                d = np.abs(np.asarray(kate_proba) - proba)
                d[:, 1] = np.minimum(d[:, 1], 2 * np.pi - d[:, 1])
                rms = sum(runs[1:]) / 3
                ref_gpu = {"value": rms, "unit": unit, "runs_timed": 3, "speedup": rms / ms,
                           "plan": "gateScheduling + gateGrouping(9) + compileDefault(0) (main.cpp's recipe, "
                                   "grouping capped at 9 qubits)", "groups": rc.num_groups(),
                           "timing": "wall clock of the reference's instruction loop",
                           "proba_state_max_abs_diff_vs_kate_b200": float(d.max())}
        except Exception as ex:  # reported, not fatal
            ref_gpu = {"value": None, "unavailable": f"failed: {ex}"}

    cpu = None
    if not args.no_cpu_baseline and not _reference_unavailable():
        cms, cores = cpu_run()
        cpu = {"value": cms, "unit": unit, "cores": cores, "kind": "reference",
               "sample": f"the whole n={n} circuit once on the reference CPUSimulator (gateScheduling + "
                         f"gateGrouping(12)), gate phase only"}
    cfg.update({"passes_per_step": len(passes), "ops": n_ops})
    print(json.dumps(line(
        ms, ms, "c128 (f64)",
        e2e={"value": e2e_ms, "unit": unit, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
             "ms_per_step": e2e_ms},
        roofline={"bound": "hbm", "achieved": alg / (avg_pass / 1000) / 1e9, "peak": peak, "unit": "GB/s",
                  "frac": alg / (avg_pass / 1000) / 1e9 / peak, "traffic": committed_traffic(n),
                  "peak_source": peak_kind, "kernel": PASS_KERNEL,
                  "alg_bytes_per_launch": alg, "avg_launch_ms": avg_pass,
                  "profiled_pass_ms": {"min": min(pass_ms), "max": max(pass_ms),
                                       "mean": sum(pass_ms) / len(pass_ms)},
                  "per_pass_gbs": per_pass_gbs(2.0 * 16.0 * 2 ** n, pass_ms, peak),
                  "frac_of_nominal": alg / (avg_pass / 1000) / 1e9 / NOMINAL_HBM_GBS},
        gpu_launches=launches * args.steps, clocks=clk.summary(), cpu_baseline=cpu, ref_gpu_baseline=ref_gpu)))


def _hea_batch(K, C, count, seed=2024):
    import numpy as np
    rng = np.random.default_rng(seed)
    ns = [int(x) for x in rng.integers(10, 23, count)]
    circs = []
    for i, n in enumerate(ns):
        c = K.Circuit(n)
        c.appendFlat(*C.hea_flat(n, 2 * n, seed=i))
        circs.append(c)
    return ns, circs


def run_batch(args):
    """4096 HEA circuits in one persistent CUDA-graph launch."""
    import numpy as np
    import torch
    import kate_b200 as K
    from kate_b200 import circuits as C

    N = args.circuits
    cfg = {"workload": f"{N} hardware-efficient-ansatz circuits, n uniform in 10..22 (seeded), depth 2n "
                       f"(RY, RZ on every qubit, CZ brickwork), complex64, <Z_q> outputs, one persistent "
                       f"CUDA-graph launch", "circuits": N, "seed": 2024, "parallelism": "replicas",
           "l2": "states total ~21 GB, larger than L2; no flush needed"}
    if args.impl == "reference":
        if _reference_unavailable():
            print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref was not built"}))
            return
        import numpy as np
        rng = np.random.default_rng(2024)
        ns = [int(x) for x in rng.integers(10, 23, N)]
        tot, cnt, cores = 0.0, 0, 1
        t_end = time.perf_counter() + 20.0
        for i, n in enumerate(ns):
            if time.perf_counter() > t_end and cnt >= 8:
                break
            sec, cores = _ref_seconds(n, C.hea(n, 2 * n, seed=i))
            tot += sec
            cnt += 1
        # Scale the sample's mean time by the batch's mean state size ratio.
        import statistics as st
        w_all = st.mean(2.0 ** n for n in ns)
        w_s = st.mean(2.0 ** n for n in ns[:cnt])
        v = cnt / tot * (w_s / w_all)
        print(json.dumps(_common("circuits/s", "circuits/s", v, args, 1000.0 * N / v, "c128 (f64)", cfg,
                                 impl="reference",
                                 cpu_baseline={"value": v, "unit": "circuits/s", "cores": cores, "kind": "reference",
                                               "sample": f"first {cnt} circuits of the batch on the reference "
                                                         f"CPUSimulator (complex128), rate scaled by mean 2^n"},
                                 e2e={"value": v, "unit": "circuits/s", "h2d_bytes_per_step": 0,
                                      "d2h_bytes_per_step": 0})))
        return
    torch.cuda.set_device(0)
    ns, circs = _hea_batch(K, C, N)
    t0 = time.perf_counter()
    opts = None
    if args.no_autotune and args.tensor_blocks:
        import ctypes
        opts = K._lib.BatchOptions()
        K._lib.lib().kate_batch_options_default(ctypes.byref(opts))
        for n in range(13, K._lib.KATE_BATCH_MAX_QUBITS + 1):
            opts.tune[n].blocks = 1
    b = K.Batch(circs, precision=K.C64, options=opts, autotune=not args.no_autotune)
    create_s = time.perf_counter() - t0
    tune = {n: {"fusion_k": b.options.tune[n].fusion, "max_gates": b.options.tune[n].max_gates,
                "group_m": b.options.tune[n].group_qubits, "coalesce_c": b.options.tune[n].coalesce,
                "tensor_blocks": b.options.tune[n].blocks}
            for n in sorted(set(ns))}
    info = b.info()
    b.time(max(1, args.warmup))
    with Clocks(0) as clk:
        ms = b.time(args.steps)
    value = N / (ms / 1000.0)
    # Algorithmic bytes of the launch: every pass of a resident state reads
    # and writes it once (the first pass only writes; the <Z> reduction reads
    # it once more), 8 bytes per amplitude. Circuits run in shared memory
    # move no state bytes.
    nprog, nres = b.circuit_info()
    alg = float(sum(int(p) * 16.0 * 2 ** int(r) for p, r in zip(nprog, nres) if r > 0))
    peak, peak_kind = measured_hbm_peak()
    z = b.expect_z_flat()
    # Precision: infidelity against complex128 on a seeded subsample of the
    # circuits with resident states (those of <= 12 qubits run in one CTA's
    # shared memory and keep no state), and the largest <Z> error of a
    # subsample of the small ones.
    rs = np.random.default_rng(args.seed + 7)
    res_idx = [i for i in range(N) if int(nres[i]) > 0]
    pick = sorted(rs.choice(res_idx, size=min(8, len(res_idx)), replace=False).tolist()) if res_idx else []
    infid = batch_infidelity(K, circs, pick, batch=b) if pick else None
    small = [i for i in range(N) if int(nres[i]) == 0][:16]
    zoff = np.concatenate([[0], np.cumsum(ns)])
    zerr = 0.0
    for i in small:
        s_ = K.Simulator(circs[i], 1, K.C128, 0)
        s_.execute()
        zerr = max(zerr, float(np.abs(s_.expect_z() - z[zoff[i]:zoff[i + 1]]).max()))
        s_.close()
    b.close()
    # End to end: create (plan + upload) + run + readback, through the C ABI.
    t0 = time.perf_counter()
    b2 = K.Batch(circs, precision=K.C64, options=b.options)
    b2.run()
    b2.expect_z_flat()
    create_ms = b2.create_times()
    h2d = b2.upload_bytes()
    b2.close()
    e2e_s = time.perf_counter() - t0
    # Baseline: one Simulator launch per circuit (plans and states prepared beforehand).
    M = 0 if args.no_baseline else min(256, N)
    sims = [K.Simulator(circs[i], 1, K.C64, 0) for i in range(M)]
    for s_ in sims[:4]:
        s_.run_async()
        s_.synchronize()
    t0 = time.perf_counter()
    for s_ in sims:
        s_.run_async()
        s_.expect_z()
    plain = M / (time.perf_counter() - t0) if M else None
    for s_ in sims:
        s_.close()
    cpu = None
    if not args.no_cpu_baseline and not _reference_unavailable():
        tot, cnt, cores = 0.0, 0, 1
        t_end = time.perf_counter() + 15.0
        for i, n in enumerate(ns):
            if time.perf_counter() > t_end and cnt >= 8:
                break
            sec, cores = _ref_seconds(n, C.hea(n, 2 * n, seed=i))
            tot += sec
            cnt += 1
        w_all = statistics.mean(2.0 ** n for n in ns)
        w_s = statistics.mean(2.0 ** n for n in ns[:cnt])
        cpu = {"value": cnt / tot * (w_s / w_all), "unit": "circuits/s", "cores": cores, "kind": "reference",
               "sample": f"first {cnt} circuits on the reference CPUSimulator (complex128), rate scaled by mean 2^n"}
    cfg.update({"autotuned": tune, "tasks": info["tasks"], "pass_programs": info["programs"],
                "arena_bytes": info["arena_bytes"], "ctas": info["ctas"], "create_s": create_s,
                "e2e_create_ms": create_ms, "host_cpus": os.cpu_count(),
                "baseline_one_launch_per_circuit_cps": plain,
                "speedup_vs_one_launch_per_circuit": value / plain if plain else None,
                "infidelity_vs_c128": infid,
                "small_circuits_max_abs_z_error_vs_c128": {"value": zerr, "circuits": len(small)}})
    print(json.dumps(_common(
        "circuits/s", "circuits/s", value, args, ms, "c64 (f32)", cfg,
        e2e={"value": N / e2e_s, "unit": "circuits/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": 8 * len(z),
             "ms_per_step": e2e_s * 1000, "note": "plan + upload + run + <Z> readback per step"},
        roofline={"bound": "hbm (latency-bound task queue: tensor-core block tasks and FP32 register tasks)",
                  "achieved": alg / (ms / 1000) / 1e9, "peak": peak, "unit": "GB/s",
                  "frac": alg / (ms / 1000) / 1e9 / peak, "traffic": None, "peak_source": peak_kind,
                  "kernel": "k_batch<float2> (persistent task queue; tcgen05 block tasks where autotuned)",
                  "alg_bytes_per_launch": alg,
                  "avg_launch_ms": ms},
        gpu_launches=args.steps, clocks=clk.summary(), cpu_baseline=cpu)))


def batch_infidelity(K, circs, idx, batch=None):
    """Infidelity 1 - |<psi64|psi128>|^2 of circuits `idx` (each with a
    resident state, > 12 qubits) as the complex64 batch kernel computes them
    (states read back from a batch: `batch`, or a new one of just these
    circuits) against the complex128 simulator. Returns a summary dict."""
    import numpy as np
    own = batch is None
    if own:
        batch = K.Batch([circs[i] for i in idx], precision=K.C64)
        batch.run()
    res = []
    for k, i in enumerate(idx):
        psi64 = batch.state(k if own else i)
        s = K.Simulator(circs[i], 1, K.C128, 0)
        s.execute()
        psi128 = s.state()
        s.close()
        ov = np.vdot(psi128, psi64)
        f = float(1.0 - abs(ov) ** 2 / (np.vdot(psi64, psi64).real * np.vdot(psi128, psi128).real))
        res.append({"circuit": int(i), "nqubits": int(circs[i].nqbits), "infidelity": f})
    if own:
        batch.close()
    inf = [r["infidelity"] for r in res]
    return {"max": max(inf), "mean": sum(inf) / len(inf), "circuits": res,
            "against": "complex128 simulator on the same circuits (FP64)"}


def _geometric_n(rng, lo=12, hi=28, p=0.3):
    while True:
        k = int(rng.geometric(p)) - 1
        if lo + k <= hi:
            return lo + k


def run_serve(args):
    """Poisson request stream through the continuous-batching server."""
    import threading
    import numpy as np
    import torch
    import kate_b200 as K
    from kate_b200 import circuits as C

    R = args.requests
    rates = [float(x) for x in args.rates.split(",")]
    rng = np.random.default_rng(args.seed)
    ns = [_geometric_n(rng) for _ in range(R)]
    cfg = {"workload": f"Poisson stream of {R} requests per rate, n truncated geometric (p=0.3) on 12..28, "
                       f"layered RX/RZ/CNOT-ladder circuit of depth n, complex64, 1024 samples + <Z_q> each, "
                       f"150 GB admission budget", "requests": R, "rates": rates, "seed": args.seed,
           "mean_n": float(np.mean(ns)), "max_n": int(max(ns)), "parallelism": "replicas",
           "tensor_blocks": args.tensor_blocks}
    if args.impl == "reference":
        if _reference_unavailable():
            print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref was not built"}))
            return
        tot, cnt, cores = 0.0, 0, 1
        t_end = time.perf_counter() + 20.0
        for i, n in enumerate(ns):
            if time.perf_counter() > t_end and cnt >= 8:
                break
            sec, cores = _ref_seconds(n, C.layered(n, n, seed=i))
            tot += sec
            cnt += 1
        w_all = statistics.mean(2.0 ** n * n for n in ns)
        w_s = statistics.mean(2.0 ** n * n for n in ns[:cnt])
        v = cnt / tot * (w_s / w_all)
        print(json.dumps(_common("served circuits/s", "circuits/s", v, args, 1000.0 / v, "c128 (f64)", cfg,
                                 impl="reference",
                                 cpu_baseline={"value": v, "unit": "circuits/s", "cores": cores, "kind": "reference",
                                               "sample": f"first {cnt} requests on the reference CPUSimulator "
                                                         f"(complex128, no sampling), rate scaled by mean n 2^n"},
                                 e2e={"value": v, "unit": "circuits/s", "h2d_bytes_per_step": 0,
                                      "d2h_bytes_per_step": 0})))
        return
    torch.cuda.set_device(0)
    circs = [K.Circuit(n, C.layered(n, n, seed=i)) for i, n in enumerate(ns)]
    kw = {"step_latency_us": args.step_us} if args.step_us else {}
    srv = K.Server(K.C64, 0, budget_bytes=150 * 10 ** 9, tensor_blocks=args.tensor_blocks, **kw)
    # Warm-up: a few requests of every size class present.
    for n in sorted(set(ns))[:6]:
        srv.wait(srv.submit(K.Circuit(n, C.layered(n, n, seed=999)), 1024, 1), timeout=600)
    sweep = []
    with Clocks(0) as clk:
        for rate in rates:
            gaps = rng.exponential(1.0 / rate, R)
            results = [None] * R
            ids = [None] * R
            ready = threading.Event()

            def waiter():
                ready.wait()
                for i in range(R):
                    while ids[i] is None:
                        time.sleep(0.0002)
                    results[i] = srv.wait(ids[i], timeout=3600)

            th = threading.Thread(target=waiter)
            th.start()
            t_start = time.perf_counter()
            due = t_start
            ready.set()
            for i in range(R):
                due += gaps[i]
                d = due - time.perf_counter()
                if d > 0:
                    time.sleep(d)
                ids[i] = srv.submit(circs[i], 1024, 1000 + i)
            th.join()
            t_sub = np.array([r[2][0] for r in results])
            t_done = np.array([r[2][2] for r in results])
            lat = (t_done - t_sub) * 1000.0
            span = float(t_done.max() - t_sub.min())
            sweep.append({"rate": rate, "circuits_per_s": R / span, "p50_ms": float(np.percentile(lat, 50)),
                          "p99_ms": float(np.percentile(lat, 99)), "mean_ms": float(lat.mean()),
                          "offered_s": float(gaps.sum())})
    st = srv.stats()
    srv.close()
    # Precision: the engine's kernel and plans on a seeded subsample of the
    # served circuits (more than 12 qubits), run as a batch with their
    # states read back, against complex128.
    rs = np.random.default_rng(args.seed + 7)
    cand = [i for i in range(R) if ns[i] > 12 and ns[i] <= 24]
    pick = sorted(rs.choice(cand, size=min(8, len(cand)), replace=False).tolist()) if cand else []
    infid = batch_infidelity(K, circs, pick) if pick else None
    # Baseline: one-at-a-time plain launches (a Simulator per request, run,
    # <Z>, 1024 samples), served FIFO; latencies at each rate from the
    # measured service times under the same arrival process.
    svc = []
    for i in range(R):
        t0 = time.perf_counter()
        s_ = K.Simulator(circs[i], 1, K.C64, 0)
        s_.execute()
        s_.expect_z()
        s_.sample(1024, seed=1000 + i)
        s_.close()
        svc.append(time.perf_counter() - t0)
    base = []
    rng2 = np.random.default_rng(args.seed + 1)
    for rate in rates:
        arr = np.cumsum(rng2.exponential(1.0 / rate, R))
        done, t = [], 0.0
        for a, s_ in zip(arr, svc):
            t = max(t, a) + s_
            done.append(t)
        lat = (np.array(done) - arr) * 1000
        base.append({"rate": rate, "circuits_per_s": R / (done[-1] - arr[0]),
                     "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99))})
    best = max(sweep, key=lambda x: x["circuits_per_s"])
    plain_cps = R / sum(svc)
    cfg.update({"sweep": sweep, "baseline_one_at_a_time": base, "baseline_service_cps": plain_cps,
                "speedup_vs_one_at_a_time": best["circuits_per_s"] / plain_cps, "engine_steps": st["steps"],
                "peak_resident_bytes": st["peak_resident_bytes"], "infidelity_vs_c128": infid,
                "engine_thread_s": {k[3:]: st[k] / 1e6 for k in ("us_admit", "us_build", "us_kernel", "us_collect")}})
    cpu = None
    if not args.no_cpu_baseline and not _reference_unavailable():
        tot, cnt, cores = 0.0, 0, 1
        t_end = time.perf_counter() + 15.0
        for i, n in enumerate(ns):
            if time.perf_counter() > t_end and cnt >= 8:
                break
            sec, cores = _ref_seconds(n, C.layered(n, n, seed=i))
            tot += sec
            cnt += 1
        w_all = statistics.mean(2.0 ** n * n for n in ns)
        w_s = statistics.mean(2.0 ** n * n for n in ns[:cnt])
        cpu = {"value": cnt / tot * (w_s / w_all), "unit": "circuits/s", "cores": cores, "kind": "reference",
               "sample": f"first {cnt} requests on the reference CPUSimulator (complex128, no sampling), rate "
                         f"scaled by mean n 2^n"}
    print(json.dumps(_common(
        "served circuits/s", "circuits/s", best["circuits_per_s"], args, 1000.0 / best["circuits_per_s"],
        "c64 (f32)", cfg, p50_ms=best["p50_ms"], p99_ms=best["p99_ms"],
        e2e={"value": best["circuits_per_s"], "unit": "circuits/s",
             "h2d_bytes_per_step": None, "d2h_bytes_per_step": 8 * (1024 + 28),
             "note": "the serving rate is measured end to end: submit from host circuits to results on the host"},
        gpu_launches=st["steps"], clocks=clk.summary(), cpu_baseline=cpu)))


if __name__ == "__main__":
    main()
