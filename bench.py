"""Benchmark: ICEEMDAN of an EEG-shaped channel on B200.

Workload (one step = one full decomposition): N = 244032 float64 samples at 256 Hz (unit-variance
1/f noise + alpha bursts + beta + spikes, seed 2 + rank), NR = 500 white-noise realizations
(cuRAND XORWOW, seed 1 + rank), MaxIter = 1000, 17 IMFs, Nstd = 0.2.  Every array the sift
touches (NR x N x 8 B = 976 MB) is larger than the 126 MB L2, so no flush is needed between
steps.

Metric: samples x realizations / s of the whole decomposition (noise-mode precompute + CEEMDAN
stages), aggregated over ranks; each rank decomposes its own channel (weak scaling, no
collective on the data path).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--workload differentiation measures the reverse pass instead: one step = a batch of 32 signals
(N = 8192, the two-tone chirp recipe with seeds 10-41; NR = 50, MaxIter = 100, 13 IMFs,
cuRAND seed 1), each decomposed by the taped forward and differentiated by the backward entry
(gradient of sum_k w_k |IMF_k|^2, w ~ U(0,1) seed 4), 8 signals at a time on their own CUDA
streams; the noise phase, the same for all 32 signals, is computed once per step.  Metric: samples x realizations / s of forward + reverse.

Profiling aids (not bench values): --nr, --imfs and --sift-cap shrink the workload (same N and
signal) for ncu captures; --no-cpu and --no-e2e skip the CPU sample and the e2e leg.

--impl reference times the reference algorithm's CPU rendering (the oracle, C++/OpenMP FP64)
on the host cores on a bounded sample of the same workload; it is the only place besides the
CPU-baseline leg where bench.py runs oracle/ code.
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

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N = 244032
NR = 500
MAX_ITER = 1000
NUM_IMFS = 17
NSTD = 0.2
NOISE_CAP = 2000
METRIC = "samples x realizations / s (ICEEMDAN, N=244032, NR=500, 17 IMFs, FP64)"
UNIT = "samples*realizations/s"
# Lock-step sift iterations of this workload on rank 0's inputs (sum over the 16 noise and
# 16 signal stages), a deterministic property of the inputs; used to scale the CPU sample
# when the GPU arm has not run in the same process.
WORKLOAD_ITERATIONS = 12487

# algorithmic bytes per sift iteration per realization: coefficients of N and of K (knots of
# both envelopes).  Kernel kinds follow include/ceemdan_b200.h.
BYTES_PER_N = {"extrema": 24.25, "eval": 8.25}
BYTES_PER_K = {"extrema": 12.0, "chunk_reduce": 17.0, "reduced_solve": 10.5,
               "segments": 44.5, "eval": 36.0}


def _peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _traffic_ratio(kernel):
    """DRAM bytes / algorithmic bytes of `kernel` from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", f"k_{kernel}_eeg244032.md")
    try:
        for line in open(path):
            if line.startswith("traffic_over_algorithmic:"):
                return float(line.split(":")[1])
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            if len(r) >= 9:
                for nm, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


def _cpu_sample(threads, iterations_total):
    """Oracle (CPU FP64 restatement) on a bounded sample of the workload: NR_s realizations of
    the same channel, one lock-step sift iteration in each of the 32 stages (caps of 1), so the
    per-iteration cost is averaged over the stages' knot densities.  Scaled to the whole
    decomposition by the workload's lock-step iteration total."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from __graft_entry__ import load_package
    load_package()
    from ceemdan_gpu_b200 import workloads
    nr_s = min(NR, 64)
    x = workloads.eeg_like(N, seed=2)
    w = workloads.white_noise(nr_s, N, 1)
    t0 = time.perf_counter()
    _, iters = oracle.iceemdan(x, w, NUM_IMFS, 1, NSTD, solver=1, chunk=16, threads=threads,
                               noise_sift_cap=1, return_iters=True)
    dt = time.perf_counter() - t0
    done = int(sum(iters)) * nr_s  # realization-iterations executed
    rate = done / dt
    t_full = iterations_total * NR / rate
    value = N * NR / t_full
    return value, {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                   "sample": (f"oracle (C++/OpenMP FP64, canonical solve) on {nr_s} of {NR} "
                              f"realizations, 1 sift iteration in each of the {len(iters)} "
                              f"stages ({done} realization-iterations in {dt:.2f} s), scaled "
                              f"to the workload's {iterations_total} lock-step iterations x "
                              f"{NR} realizations")}


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    vals = []
    for i in range(args.warmup + args.steps):
        v, info = _cpu_sample(threads, WORKLOAD_ITERATIONS)
        if i >= args.warmup:
            vals.append(v)
    value = statistics.median(vals)
    info["value"] = value
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": N * NR / value * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "ICEEMDAN eeg-like channel N=244032 NR=500 MaxIter=1000 "
                                   "17 IMFs Nstd=0.2 (one decomposition per step)",
                       "sample": "bounded CPU sample, see cpu_baseline"},
            "cpu_baseline": info,
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args, rank, world, local_rank):
    global NR, NUM_IMFS, MAX_ITER, NOISE_CAP
    NR, NUM_IMFS = args.nr, args.imfs
    if args.sift_cap:
        MAX_ITER = NOISE_CAP = args.sift_cap
    import torch
    import torch.distributed as dist
    from __graft_entry__ import load_package
    pkg = load_package()
    from ceemdan_gpu_b200 import multichannel, workloads

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    y_host = torch.tensor(workloads.eeg_like(N, seed=2 + rank), dtype=torch.float64)
    y = y_host.to(dev)
    seed = 1 + rank
    stream = torch.cuda.current_stream()

    def step(profile=None):
        return pkg.iceemdan(y, NR, NUM_IMFS, MAX_ITER, NSTD, seed=seed,
                            noise_sift_cap=NOISE_CAP, profile=profile, return_iters=True)

    def barrier():
        if world > 1:
            dist.barrier()

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    prof = {"ms": {}, "counters": {}}
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    iters_seen = None
    with ClockSampler(local_rank) as clk:
        barrier()
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(args.steps):
            p = {}
            _, iters_seen = step(profile=p)
            for k, v in p["ms"].items():
                prof["ms"][k] = prof["ms"].get(k, 0.0) + v
            for k, v in p["counters"].items():
                prof["counters"][k] = prof["counters"].get(k, 0) + v
        ev1.record(stream)
        torch.cuda.synchronize()
        barrier()
    ms_max = multichannel.max_over_ranks(ev0.elapsed_time(ev1), world, dev)
    ms_per_step = ms_max / args.steps
    value = world * N * NR / (ms_per_step * 1e-3)

    # e2e: host buffers through the public C-ABI call, copies inside the timed region
    e2e_value = None
    if not args.no_e2e:
        e2e_value = _e2e(pkg, multichannel, dev, stream, y_host, seed, barrier, world)

    if rank != 0:
        return 0
    return _report(args, world, prof, iters_seen, ms_per_step, value, e2e_value, clk)


def _e2e(pkg, multichannel, dev, stream, y_host, seed, barrier, world):
    import torch
    imfs_host = torch.empty((NUM_IMFS, N), dtype=torch.float64).pin_memory()
    y_pin = y_host.pin_memory()
    x_pin = torch.arange(N, dtype=torch.int32).pin_memory()
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    y_dev = y_pin.to(dev, non_blocking=True)
    x_dev = x_pin.to(dev, non_blocking=True)
    imfs_dev = pkg.iceemdan(y_dev, NR, NUM_IMFS, MAX_ITER, NSTD, seed=seed,
                            noise_sift_cap=NOISE_CAP, x=x_dev)
    imfs_host.copy_(imfs_dev, non_blocking=True)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    e2e_ms = multichannel.max_over_ranks(e0.elapsed_time(e1), world, dev)
    return world * N * NR / (e2e_ms * 1e-3)


def _report(args, world, prof, iters_seen, ms_per_step, value, e2e_value, clk):
    # roofline of the dominant kernel
    its = prof["counters"].get("iterations", 0)
    knots = prof["counters"].get("knots", 0)
    kms = prof["ms"]
    dom = max(kms, key=lambda k: kms[k])
    alg_bytes = (BYTES_PER_N.get(dom, 0.0) * N * NR * its + BYTES_PER_K.get(dom, 0.0) * knots)
    launches = its  # one launch of each sift kernel per executed iteration
    per_launch = alg_bytes / max(launches, 1)
    avg_ms = kms[dom] / max(launches, 1)
    achieved = per_launch / (avg_ms * 1e-3) / 1e9 if avg_ms > 0 else 0.0
    peak, peak_src = _peaks()
    ratio = _traffic_ratio(dom)
    roof = {"kernel": dom, "bound": "hbm", "achieved": round(achieved, 1),
            "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
            "peak_source": peak_src,
            "traffic": round(ratio * per_launch) if ratio else None,
            "algorithmic_bytes_per_launch": round(per_launch),
            "avg_launch_ms": round(avg_ms, 4),
            "kernel_ms_share": {k: round(v / sum(kms.values()), 4) for k, v in kms.items()}}
    total_iters = int(sum(iters_seen)) if iters_seen else WORKLOAD_ITERATIONS
    cpu_info = None
    if not args.no_cpu and world == 1:  # the CPU baseline is reported at N=1 only
        _, cpu_info = _cpu_sample(os.cpu_count() or 1, total_iters)

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": (f"ICEEMDAN eeg-like channel N={N} NR={NR} MaxIter={MAX_ITER} "
                                    f"{NUM_IMFS} IMFs Nstd={NSTD} (one decomposition per step, "
                                    "per rank)"),
                       "channels_per_rank": 1, "l2": "inputs larger than L2 (976 MB arrays)",
                       "noise": "cuRAND XORWOW seed 1+rank", "parallelism": f"channels x{world}",
                       "lockstep_iterations": total_iters},
            "roofline": roof, "cpu_baseline": cpu_info,
            "e2e": ({"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": N * 8 + N * 4,
                     "d2h_bytes_per_step": NUM_IMFS * N * 8} if e2e_value else None),
            "gpu_launches": int(prof["counters"].get("launches", 0)),
            "clocks": clk.summary()}
    print(json.dumps(line), flush=True)
    return 0


DIFF_SIGNALS, DIFF_N, DIFF_NR, DIFF_ITER, DIFF_IMFS = 32, 8192, 50, 100, 13
DIFF_STREAMS = 8  # signals in flight at once (one host thread and CUDA stream each)


def _differentiation_cpu_sample(ys_host):
    """The differentiation step on the host cores with the oracle (C++/OpenMP FP64), mirroring
    the GPU arm: one full decomposition of the first signal (which computes the shared noise
    phase), then every signal's taped forward from that noise phase and its vjp.  Timed: the
    full call, one shared forward and one vjp; the step is extrapolated to all signals."""
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from ceemdan_gpu_b200 import workloads
    noise = workloads.white_noise(DIFF_NR, DIFF_N, 1)
    w = np.random.default_rng(4).uniform(size=DIFF_IMFS)
    kw = dict(solver=1, noise_sift_cap=NOISE_CAP)
    t0 = time.perf_counter()
    first = oracle.Tape(ys_host[0].numpy(), noise, DIFF_IMFS, DIFF_ITER, NSTD, **kw)
    t1 = time.perf_counter()
    tp = oracle.Tape(ys_host[1].numpy(), None, DIFF_IMFS, DIFF_ITER, NSTD, noise_from=first, **kw)
    t2 = time.perf_counter()
    tp.vjp(2.0 * w[:, None] * tp.imfs)
    t3 = time.perf_counter()
    step = (t1 - t0) + DIFF_SIGNALS * (t3 - t1)
    return {"value": DIFF_SIGNALS * DIFF_N * DIFF_NR / step, "unit": UNIT,
            "cores": os.cpu_count() or 1, "kind": "port",
            "sample": (f"full decomposition of signal 1 ({t1 - t0:.2f} s), taped forward from "
                       f"the shared noise phase ({t2 - t1:.2f} s) and vjp ({t3 - t2:.2f} s) of "
                       f"signal 2, step = full + {DIFF_SIGNALS} x (forward + vjp); oracle "
                       "C++/OpenMP FP64 on all host threads")}


def run_differentiation(args, rank, world, local_rank):
    """Forward + reverse pass of the differentiation workload (see the module docstring)."""
    import numpy as np
    import torch
    from __graft_entry__ import load_package
    pkg = load_package()
    from ceemdan_gpu_b200 import multichannel, workloads

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    ys_host = [torch.tensor(workloads.two_tone_chirp(DIFF_N, seed=10 + s + DIFF_SIGNALS * rank))
               for s in range(DIFF_SIGNALS)]
    w = torch.tensor(np.random.default_rng(4).uniform(size=DIFF_IMFS), device=dev)
    stream = torch.cuda.current_stream()
    seed = 1 + rank

    def step(ys, phases=None):
        """Shared noise phase (one plain decomposition of the first signal), then taped forward
        + backward of every signal, DIFF_STREAMS signals at a time on their own streams."""
        t = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        t[0].record(stream)
        _, state = pkg.iceemdan(ys[0], DIFF_NR, DIFF_IMFS, DIFF_ITER, NSTD, seed=seed,
                                noise_sift_cap=NOISE_CAP, return_noise_state=True)
        t[1].record(stream)
        grads = multichannel.gradients_on_streams(
            pkg, ys, DIFF_NR, DIFF_IMFS, DIFF_ITER, NSTD, lambda imfs: 2.0 * w[:, None] * imfs,
            streams=DIFF_STREAMS, device=dev, seed=seed, noise_state=state,
            noise_sift_cap=NOISE_CAP)
        t[2].record(stream)
        if phases is not None:
            t[2].synchronize()
            phases["shared_noise_phase_ms"] = (phases.get("shared_noise_phase_ms", 0.0) +
                                               t[0].elapsed_time(t[1]))
            phases["forward_and_backward_ms"] = (phases.get("forward_and_backward_ms", 0.0) +
                                                 t[1].elapsed_time(t[2]))
        return grads

    ys = [y.to(dev) for y in ys_host]
    for _ in range(args.warmup):
        step(ys)
    torch.cuda.synchronize()
    launches0 = int(pkg.lib().ceemdan_kernel_launches())
    phases = {}
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(args.steps):
            step(ys, phases)
        ev1.record(stream)
        torch.cuda.synchronize()
    launches = int(pkg.lib().ceemdan_kernel_launches()) - launches0
    ms = multichannel.max_over_ranks(ev0.elapsed_time(ev1), world, dev) / args.steps
    units = DIFF_SIGNALS * DIFF_N * DIFF_NR
    value = world * units / (ms * 1e-3)

    # e2e: host signals in (pinned), gradients back to the host, inside the timed region
    pins = [y.pin_memory() for y in ys_host]
    out = torch.empty((DIFF_SIGNALS, DIFF_N), dtype=torch.float64).pin_memory()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    grads = step([p.to(dev, non_blocking=True) for p in pins])
    out.copy_(torch.stack(grads), non_blocking=True)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = multichannel.max_over_ranks(e0.elapsed_time(e1), world, dev)
    if rank != 0:
        return 0

    cpu_info = None
    if not args.no_cpu and world == 1:
        cpu_info = _differentiation_cpu_sample(ys_host)
    line = {"metric": ("samples x realizations / s (ICEEMDAN forward + reverse pass, 32 x N=8192, "
                       "NR=50, 13 IMFs, FP64)"),
            "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": (f"differentiation: {DIFF_SIGNALS} two-tone chirp signals "
                                    f"N={DIFF_N} (seeds 10-41), NR={DIFF_NR}, "
                                    f"MaxIter={DIFF_ITER}, {DIFF_IMFS} IMFs, noise cap "
                                    f"{NOISE_CAP}; taped forward + backward per signal on "
                                    f"{DIFF_STREAMS} streams, noise phase once per step"),
                       "l2": "working set below L2 (3.3 MB per realization set)",
                       "phases_ms_per_step": {k: v / args.steps for k, v in phases.items()}},
            "cpu_baseline": cpu_info,
            "e2e": {"value": world * units / (e2e_ms * 1e-3), "unit": UNIT,
                    "h2d_bytes_per_step": DIFF_SIGNALS * DIFF_N * 8,
                    "d2h_bytes_per_step": DIFF_SIGNALS * DIFF_N * 8},
            "gpu_launches": launches // max(args.steps, 1),
            "clocks": clk.summary()}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--nr", type=int, default=NR)
    ap.add_argument("--imfs", type=int, default=NUM_IMFS)
    ap.add_argument("--sift-cap", type=int, default=0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--workload", choices=["eeg", "differentiation"], default="eeg")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=180))
    try:
        if args.workload == "differentiation":
            return run_differentiation(args, rank, world, local_rank)
        return run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
