"""Benchmark: batched ICEEMDAN of ragged EEG-shaped channels on B200.

Default workload (--workload batched), the batched form the headline metric is quoted on: 64
EEG-shaped channels (unit-variance 1/f noise + alpha bursts at U(8,12) Hz + beta + spikes) of
lengths U[30000, 250000] (seed 3), NR = 100 white-noise realizations per channel (cuRAND
XORWOW, seed 1234 + channel), MaxIter = 1000, 17 IMFs, Nstd = 0.2, FP64.  The 64 channels do
not fit the B200's memory together (their noise modes alone are about 120 GB), so the batch is
dealt into 8 groups of 8 channels of nearly equal total length (about 1.05 M samples each); one
step = one group through the batched engine (ceemdan_batched_f64: every channel of the group
sifts in one device-driven loop), and consecutive steps cycle through the groups, so 8 steps
cover the batch.  Every array the sift touches (about 100 M doubles) is larger than the
126 MB L2, so no flush is needed between steps.  The line also reports the same group run
channel by channel through the plain entry point (ceemdan_plain_f64), and their ratio.

Metric: samples x realizations / s of whole decompositions (noise-mode precompute + CEEMDAN
stages), aggregated over ranks; under torchrun rank r takes groups r, r + N, ... (weak
scaling, no collective on the data path).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--workload eeg measures one plain decomposition per step instead: N = 244032 (EEG-shaped,
seed 2 + rank), NR = 500, MaxIter = 1000, 17 IMFs (cuRAND seed 1 + rank).

--workload short measures one plain decomposition of a short row per step: N = 4096 (the two-
tone chirp recipe, seed rank), NR = 50, MaxIter = 300, 12 IMFs (cuRAND seed 1 + rank); every
stage runs on chip (one cooperative launch of k_sift_small).  Its arrays fit in L2, so a
buffer larger than L2 is written between timed steps (outside the timed region: each step is
timed by its own CUDA events).

--workload large measures forward + adjoint at scale: one step = one EEG-shaped channel of
N = 244032 (seeds 100-227) with NR = 1000, 17 IMFs, through the checkpointed taped forward and
the backward entry, with the library pool's peak device memory (--nr overrides NR).

--workload differentiation measures the reverse pass: one step = a batch of 32 signals
(N = 8192, the two-tone chirp recipe with seeds 10-41; NR = 50, MaxIter = 100, 13 IMFs,
cuRAND seed 1), each decomposed by the taped forward and differentiated by the backward entry
(gradient of sum_k w_k |IMF_k|^2, w ~ U(0,1) seed 4), 8 signals at a time on their own CUDA
streams; the noise phase, the same for all 32 signals, is computed once per step.

Profiling aids (not bench values): --nr, --imfs and --sift-cap shrink the eeg and large
workloads (same N and signal) for ncu captures; --groups G cuts the batched workload into G groups; --no-cpu,
--no-e2e and --no-plain skip the CPU sample, the e2e leg and the plain comparison.

--impl reference times the reference algorithm's CPU rendering (the oracle, C++/OpenMP FP64)
on the host cores on a bounded sample of the same workload; it is the only place besides the
CPU-baseline leg where bench.py runs oracle/ code.  --impl reference-cuda times the
reference's own CUDA build (oracle/_ref) against this engine's plain decomposition at shapes
the reference runs safely (--ref-shapes NxNRxIMFsxMaxIter ...).
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
BYTES_PER_N = {"extrema": 24.25, "eval": 8.25,
               # on-chip stage kernel: global bytes per sample-iteration (mean envelope read
               # and written, upper envelope written and read back; h stays in shared memory)
               "sift_small": 32.0}
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


# batched workload (config 3): 64 ragged EEG-shaped channels, 8 groups, NR = 100
B_CHANNELS, B_GROUPS, B_NR = 64, 8, 100
B_METRIC = ("samples x realizations / s (batched ICEEMDAN, 64 ragged EEG-like channels "
            "N=30000-250000, NR=100, 17 IMFs, FP64)")
# Mean lock-step iterations per sample-realization of the whole batch (sum over channels of
# N_c * iterations_c, divided by the sum of N_c; iterations_c = the channel's lock-step
# iterations over its 32 stages), a deterministic property of the inputs measured by the GPU
# arm (which reports its own value in config): it scales the CPU sample when the GPU arm has
# not run in the same process.
B_MEAN_ITERATIONS = 7967.2
CPU_SAMPLE_N = 30720  # samples of the eeg workload's CPU sample (its channel's first 15 tiles)
# short-row workload: one channel N = 4096 (two-tone chirp), NR = 50, MaxIter = 300, 12 IMFs;
# its lock-step iterations on rank 0's inputs (measured, as WORKLOAD_ITERATIONS)
SHORT_N, SHORT_NR, SHORT_ITER, SHORT_IMFS = 4096, 50, 300, 12
SHORT_ITERATIONS = 5032


def _cpu_rate(x, threads):
    """Oracle (CPU FP64 restatement of the reference algorithm, C++/OpenMP over realizations)
    on a bounded but complete sample: one full decomposition of x with 2 x `threads`
    realizations (white noise seed 1), the workload's sift caps, stop logic and IMF count.
    Returns the rate in sample-iterations per second and a description."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from __graft_entry__ import load_package
    load_package()
    from ceemdan_gpu_b200 import workloads
    n = len(x)
    nr_s = 2 * threads
    w = workloads.white_noise(nr_s, n, 1)
    t0 = time.perf_counter()
    _, iters = oracle.iceemdan(x, w, NUM_IMFS, MAX_ITER, NSTD, solver=1, chunk=16,
                               threads=threads, noise_sift_cap=NOISE_CAP, return_iters=True)
    dt = time.perf_counter() - t0
    its = int(sum(iters))
    rate = n * nr_s * its / dt
    return rate, (f"oracle (C++/OpenMP FP64, canonical solve), one complete decomposition of "
                  f"N={n} with {nr_s} realizations on {threads} threads ({its} lock-step "
                  f"iterations, {dt:.2f} s, {rate / 1e6:.1f} M sample-iterations/s)")


_BATCH = []


def _batch_channels():
    """The 64 channels of the batched workload and their 8 groups (generated once)."""
    if not _BATCH:
        from __graft_entry__ import load_package
        load_package()
        from ceemdan_gpu_b200 import workloads
        xs = workloads.ragged_batch(B_CHANNELS)
        _BATCH.append((xs, workloads.ragged_groups([len(x) for x in xs], B_GROUPS)))
    return _BATCH[0]


def _cpu_baseline(workload, mean_iterations, whole=None):
    """CPU throughput of the workload: the oracle's sample-iteration rate on its bounded sample
    divided by the workload's mean lock-step iterations per sample-realization (`whole`: a
    short channel sampled whole)."""
    threads = max(1, min(os.cpu_count() or 1, 32))
    if whole is not None:
        x = whole
        what = "the whole channel"
    elif workload == "batched":
        xs, _ = _batch_channels()
        x = min(xs, key=len)  # the batch's shortest channel, whole
        what = "the batch's shortest channel"
    else:
        from ceemdan_gpu_b200 import workloads
        x = workloads.eeg_like(N, seed=2)[:CPU_SAMPLE_N]
        what = f"the first {CPU_SAMPLE_N} samples of the channel"
    rate, desc = _cpu_rate(x, threads)
    value = rate / mean_iterations
    return value, {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                   "sample": (f"{desc} on {what}; workload throughput = rate / "
                              f"{mean_iterations:.1f} mean lock-step iterations per "
                              "sample-realization of the workload (measured by the GPU arm)")}


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    whole = None
    if args.workload == "batched":
        metric, mean_it = B_METRIC, B_MEAN_ITERATIONS
        workload = ("batched ICEEMDAN: 64 ragged EEG-like channels N=30000-250000 (seed 3), "
                    "NR=100, MaxIter=1000, 17 IMFs, Nstd=0.2")
    elif args.workload == "short":
        global MAX_ITER, NUM_IMFS
        MAX_ITER, NUM_IMFS = SHORT_ITER, SHORT_IMFS
        metric = (f"samples x realizations / s (ICEEMDAN, N={SHORT_N}, NR={SHORT_NR}, "
                  f"{SHORT_IMFS} IMFs, FP64)")
        mean_it = float(SHORT_ITERATIONS)
        workload = (f"ICEEMDAN two-tone chirp channel N={SHORT_N} NR={SHORT_NR} "
                    f"MaxIter={SHORT_ITER} {SHORT_IMFS} IMFs Nstd={NSTD} (one decomposition "
                    "per step)")
        from __graft_entry__ import load_package
        load_package()
        from ceemdan_gpu_b200 import workloads
        whole = workloads.two_tone_chirp(SHORT_N, seed=0)
    else:
        metric, mean_it = METRIC, float(WORKLOAD_ITERATIONS)
        workload = ("ICEEMDAN eeg-like channel N=244032 NR=500 MaxIter=1000 17 IMFs Nstd=0.2 "
                    "(one decomposition per step)")
    vals, walls = [], []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        v, info = _cpu_baseline(args.workload, mean_it, whole)
        if i >= args.warmup:
            vals.append(v)
            walls.append(time.perf_counter() - t0)
    value = statistics.median(vals)
    info["value"] = value
    line = {"impl": "reference", "metric": metric, "value": value, "unit": UNIT,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            # wall time of one step = one bounded CPU sample (the workload itself would take
            # units / value seconds)
            "ms_per_step": statistics.mean(walls) * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": workload,
                       "sample": "bounded CPU sample per step, see cpu_baseline"},
            "cpu_baseline": info,
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_reference_cuda(args):
    """The reference's own CUDA build (oracle/_ref, compiled from its sources by
    oracle/build_ref.sh; iceemdanD, cuRAND seed 1234 inside) against this engine's plain
    decomposition on the same signal, both timed by wall clock around the call on one GPU, at
    shapes the reference runs safely (N a multiple of 256, NR a multiple of 32: its block
    barriers sit inside divergent code otherwise).  Prints one JSON line per shape."""
    import torch
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref
    from __graft_entry__ import load_package
    pkg = load_package()
    from ceemdan_gpu_b200 import workloads
    if not ref.available():
        print(json.dumps({"impl": "reference-cuda", "unavailable":
                          "oracle/_ref not built (needs the reference sources)"}))
        return 0
    dev = torch.device("cuda", 0)
    shapes = args.ref_shapes or ["4096x64x12x300"]
    for spec in shapes:
        n, nr, nimf, mi = (int(v) for v in spec.split("x"))
        x = workloads.eeg_like(n, seed=2) if n > 10000 else workloads.two_tone_chirp(n, seed=0)
        y = torch.tensor(x, device=dev)
        pkg.iceemdan(y, nr, 2, 2, NSTD, noise_sift_cap=2)  # warm
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        pkg.iceemdan(y, nr, nimf, mi, NSTD)
        torch.cuda.synchronize()
        ours = time.perf_counter() - t0
        t0 = time.perf_counter()
        _, own_secs = ref.iceemdan(x, nr, nimf, mi, NSTD)
        torch.cuda.synchronize()
        theirs = time.perf_counter() - t0
        print(json.dumps({"impl": "reference-cuda", "shape": {"n": n, "nr": nr, "num_imfs": nimf,
                                                               "max_iter": mi},
                          "reference_s": theirs, "reference_own_timer_s": own_secs,
                          "ours_s": ours, "ratio": theirs / ours,
                          "unit": "seconds per decomposition (wall clock, one call each)"}),
              flush=True)
    return 0


def _roofline(prof, n_bytes_units):
    """Roofline of the dominant kernel: algorithmic bytes (BYTES_PER_N per sample-realization
    iteration, BYTES_PER_K per knot) over its event-timed duration."""
    knots = prof["counters"].get("knots", 0)
    launches = max(prof["counters"].get("iterations", 0), 1)
    kms = prof["ms"]
    dom = max(kms, key=lambda k: kms[k])
    alg_bytes = BYTES_PER_N.get(dom, 0.0) * n_bytes_units + BYTES_PER_K.get(dom, 0.0) * knots
    per_launch = alg_bytes / launches
    avg_ms = kms[dom] / launches
    achieved = per_launch / (avg_ms * 1e-3) / 1e9 if avg_ms > 0 else 0.0
    peak, peak_src = _peaks()
    ratio = _traffic_ratio(dom)
    return {"kernel": dom, "bound": "hbm", "achieved": round(achieved, 1),
            "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
            "peak_source": peak_src,
            "traffic": round(ratio * per_launch) if ratio else None,
            "algorithmic_bytes_per_launch": round(per_launch),
            "avg_launch_ms": round(avg_ms, 4),
            # the on-chip kernel runs a whole stage per launch: its figures are per iteration
            "per": "iteration" if dom == "sift_small" else "launch",
            "kernel_ms_share": {k: round(v / sum(kms.values()), 4) for k, v in kms.items()}}


def _add_prof(acc, p):
    for k, v in p["ms"].items():
        acc["ms"][k] = acc["ms"].get(k, 0.0) + v
    for k, v in p["counters"].items():
        if k == "peak_bytes":
            acc["counters"][k] = max(acc["counters"].get(k, 0), v)
        else:
            acc["counters"][k] = acc["counters"].get(k, 0) + v


def run_batched(args, rank, world, local_rank):
    """The batched workload (module docstring): one group of channels per step."""
    import numpy as np
    import torch
    from __graft_entry__ import load_package
    pkg = load_package()
    from ceemdan_gpu_b200 import multichannel, workloads

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    xs, groups = _batch_channels()
    if args.groups != B_GROUPS:
        groups = workloads.ragged_groups([len(x) for x in xs], args.groups)
    mine = [g for i, g in enumerate(groups) if i % world == rank]  # this rank's groups
    ys = {c: torch.tensor(xs[c], device=dev) for g in mine for c in g}
    stream = torch.cuda.current_stream()
    seed0 = 1234

    first_stages = []  # per-stage iteration counts of the first timed channel

    def step(k, profile=None, iters=None):
        g = mine[k % len(mine)]
        out = pkg.iceemdan_batched([ys[c] for c in g], B_NR, NUM_IMFS, MAX_ITER, NSTD,
                                   seed=seed0, noise_sift_cap=NOISE_CAP,
                                   return_iters=iters is not None, profile=profile)
        if iters is not None:
            out, its = out
            iters.extend((len(xs[c]), sum(it)) for c, it in zip(g, its))
            if not first_stages:
                first_stages.append((g[0], [int(v) for v in its[0]]))
        return g, out

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    for k in range(args.warmup):
        step(k)
    torch.cuda.synchronize()

    prof = {"ms": {}, "counters": {}}
    iters = []  # (N_c, lock-step iterations of the channel) of every timed channel
    units = 0
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        barrier()
        torch.cuda.synchronize()
        ev0.record(stream)
        last = None
        for k in range(args.steps):
            p = {}
            g, last = step(args.warmup + k, profile=p, iters=iters)
            _add_prof(prof, p)
            units += sum(len(xs[c]) for c in g) * B_NR
        ev1.record(stream)
        torch.cuda.synchronize()
        barrier()
    ms_max = multichannel.max_over_ranks(ev0.elapsed_time(ev1), world, dev)
    ms_per_step = ms_max / args.steps
    units_all = multichannel.sum_over_ranks(float(units), world, dev)  # shares differ
    value = units_all / (ms_max * 1e-3)

    # check the timed output: every channel's IMFs telescope to x / std(x)
    g_last = mine[(args.warmup + args.steps - 1) % len(mine)]
    worst = 0.0
    for c, imfs in zip(g_last, last):
        x = xs[c]
        xn = x / np.sqrt(np.sum((x - x.mean()) ** 2) / (len(x) - 1))
        err = np.max(np.abs(imfs.sum(dim=0).cpu().numpy() - xn)) / np.max(np.abs(xn))
        worst = max(worst, float(err))
    if not worst <= 1e-12:
        raise AssertionError(f"timed output does not telescope to x/std(x): {worst:.3g}")

    # the same group channel by channel through the plain entry point, and the batched step
    # of that group alone
    plain = None
    if not args.no_plain:
        g0 = mine[0]
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for c in g0:
            pkg.iceemdan(ys[c], B_NR, NUM_IMFS, MAX_ITER, NSTD, seed=seed0 + c,
                         noise_sift_cap=NOISE_CAP)
        e1.record(stream)
        torch.cuda.synchronize()
        plain_ms = e0.elapsed_time(e1)
        e0.record(stream)
        step(0)
        e1.record(stream)
        torch.cuda.synchronize()
        batched_ms = e0.elapsed_time(e1)
        u0 = sum(len(xs[c]) for c in g0) * B_NR
        plain = {"group": g0, "plain_value": u0 / (plain_ms * 1e-3),
                 "batched_value": u0 / (batched_ms * 1e-3),
                 "batched_over_plain": plain_ms / batched_ms}

    # e2e: host buffers through the public C-ABI call, copies inside the timed region
    e2e = None
    if not args.no_e2e:
        g0 = mine[0]
        pins = [torch.tensor(xs[c]).pin_memory() for c in g0]
        outs = [torch.empty((NUM_IMFS, len(xs[c])), dtype=torch.float64).pin_memory()
                for c in g0]
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        dys = [p.to(dev, non_blocking=True) for p in pins]
        res = pkg.iceemdan_batched(dys, B_NR, NUM_IMFS, MAX_ITER, NSTD, seed=seed0,
                                   noise_sift_cap=NOISE_CAP)
        for o, r in zip(outs, res):
            o.copy_(r, non_blocking=True)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        e2e_ms = multichannel.max_over_ranks(e0.elapsed_time(e1), world, dev)
        u0 = multichannel.sum_over_ranks(sum(len(xs[c]) for c in g0) * B_NR, world, dev)
        e2e = {"value": u0 / (e2e_ms * 1e-3), "unit": UNIT,
               "h2d_bytes_per_step": sum(len(xs[c]) for c in g0) * 8,
               "d2h_bytes_per_step": sum(len(xs[c]) for c in g0) * NUM_IMFS * 8}
    if rank != 0:
        return 0

    sample_iters = sum(n * B_NR * it for n, it in iters)  # sample-realization iterations
    mean_it = sum(n * it for n, it in iters) / max(1, sum(n for n, _ in iters))
    roof = _roofline(prof, sample_iters)
    cpu_info = None
    if not args.no_cpu and world == 1:
        _, cpu_info = _cpu_baseline("batched", mean_it)
    line = {"metric": B_METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": (f"batched ICEEMDAN: {B_CHANNELS} ragged EEG-like channels "
                                    "N=30000-250000 (seed 3), NR=100, MaxIter=1000, 17 IMFs, "
                                    f"Nstd=0.2; {len(groups)} groups of ~{B_CHANNELS // len(groups)} "
                                    "channels, one group per step through ceemdan_batched_f64 "
                                    "(groups cycle over steps; rank r takes groups r, r+N, ...)"),
                       "l2": "inputs larger than L2 (about 100 M doubles per group)",
                       "noise": "cuRAND XORWOW seed 1234 + channel",
                       "parallelism": f"groups x{world}",
                       "mean_lockstep_iterations": round(mean_it, 1),
                       "stage_iterations_first_channel": (
                           {"channel": first_stages[0][0], "noise_then_ceemdan_stages":
                            first_stages[0][1]} if first_stages else None),
                       "telescoping_max_rel_err": worst,
                       "waves_per_step": prof["counters"].get("waves", 0) / args.steps,
                       "peak_device_bytes": prof["counters"].get("peak_bytes", 0),
                       "plain_comparison": plain},
            "roofline": roof, "cpu_baseline": cpu_info, "e2e": e2e,
            "gpu_launches": int(prof["counters"].get("launches", 0)),
            "clocks": clk.summary()}
    print(json.dumps(line), flush=True)
    return 0




def run_ours(args, rank, world, local_rank):
    global N, NR, NUM_IMFS, MAX_ITER, NOISE_CAP, METRIC
    short = args.workload == "short"
    if short:
        N, MAX_ITER = SHORT_N, SHORT_ITER
        NR = args.nr if args.nr != NR else SHORT_NR
        NUM_IMFS = args.imfs if args.imfs != NUM_IMFS else SHORT_IMFS
        METRIC = (f"samples x realizations / s (ICEEMDAN, N={N}, NR={NR}, {NUM_IMFS} IMFs, "
                  "FP64)")
    else:
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
    x_np = workloads.two_tone_chirp(N, seed=rank) if short else workloads.eeg_like(N, seed=2 + rank)
    y_host = torch.tensor(x_np, dtype=torch.float64)
    y = y_host.to(dev)
    # short rows fit in L2: a buffer larger than L2 is written between timed steps
    flush = torch.empty(64 << 20, dtype=torch.float64, device=dev) if short else None
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
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    iters_seen = None
    with ClockSampler(local_rank) as clk:
        barrier()
        torch.cuda.synchronize()
        for e0, e1 in evs:
            if flush is not None:
                flush.fill_(1.0)
            e0.record(stream)
            p = {}
            _, iters_seen = step(profile=p)
            e1.record(stream)
            for k, v in p["ms"].items():
                prof["ms"][k] = prof["ms"].get(k, 0.0) + v
            for k, v in p["counters"].items():
                prof["counters"][k] = prof["counters"].get(k, 0) + v
        torch.cuda.synchronize()
        barrier()
    ms_max = multichannel.max_over_ranks(sum(e0.elapsed_time(e1) for e0, e1 in evs), world,
                                         dev)
    ms_per_step = ms_max / args.steps
    value = world * N * NR / (ms_per_step * 1e-3)

    # e2e: host buffers through the public C-ABI call, copies inside the timed region
    e2e_value = None
    if not args.no_e2e:
        e2e_value = _e2e(pkg, multichannel, dev, stream, y_host, seed, barrier, world)

    if rank != 0:
        return 0
    return _report(args, world, prof, iters_seen, ms_per_step, value, e2e_value, clk,
                   x_np if short else None)


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


def _report(args, world, prof, iters_seen, ms_per_step, value, e2e_value, clk, short_x=None):
    # roofline of the dominant kernel
    its = prof["counters"].get("iterations", 0)
    roof = _roofline(prof, N * NR * its)
    total_iters = int(sum(iters_seen)) if iters_seen else WORKLOAD_ITERATIONS
    cpu_info = None
    if not args.no_cpu and world == 1:  # the CPU baseline is reported at N=1 only
        _, cpu_info = _cpu_baseline("eeg", float(total_iters), short_x)
    if short_x is not None:
        workload = (f"ICEEMDAN two-tone chirp channel N={N} (seed rank) NR={NR} "
                    f"MaxIter={MAX_ITER} {NUM_IMFS} IMFs Nstd={NSTD} (one decomposition per "
                    "step, per rank; every stage on chip)")
        l2 = "a 512 MB buffer written between timed steps (arrays fit in L2)"
    else:
        workload = (f"ICEEMDAN eeg-like channel N={N} NR={NR} MaxIter={MAX_ITER} "
                    f"{NUM_IMFS} IMFs Nstd={NSTD} (one decomposition per step, per rank)")
        l2 = "inputs larger than L2 (976 MB arrays)"

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": workload, "channels_per_rank": 1, "l2": l2,
                       "noise": "cuRAND XORWOW seed 1+rank", "parallelism": f"channels x{world}",
                       "lockstep_iterations": total_iters,
                       # per stage: the noise stages, then the CEEMDAN stages
                       "stage_iterations": [int(v) for v in iters_seen] if iters_seen else None},
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


LARGE_N, LARGE_NR, LARGE_CHANNELS = 244032, 1000, 128


def run_large(args, rank, world, local_rank):
    """Large forward + adjoint: channels of 244032 samples generated as the EEG workload (seeds
    100-227), NR = 1000, 17 IMFs, MaxIter 1000; one step = one channel (the wave that fits: its
    noise modes alone are 33 GB) through the checkpointed taped forward and the backward entry
    (loss sum_k w_k |IMF_k|^2, w ~ U(0,1) seed 4).  Reports samples x realizations / s of
    forward + adjoint, the forward's own time and the library pool's peak device memory.
    Rank r takes channels r, r + N, ..."""
    import numpy as np
    import torch
    from __graft_entry__ import load_package
    pkg = load_package()
    from ceemdan_gpu_b200 import multichannel, workloads
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    global NUM_IMFS, MAX_ITER, NOISE_CAP
    nr = args.nr if args.nr != NR else LARGE_NR
    NUM_IMFS = args.imfs
    if args.sift_cap:  # profiling aid (a small case of the same kernels)
        MAX_ITER = NOISE_CAP = args.sift_cap
    w = torch.tensor(np.random.default_rng(4).uniform(size=NUM_IMFS), device=dev)
    stream = torch.cuda.current_stream()

    def step(k, phases):
        ch = rank + world * (k % max(1, LARGE_CHANNELS // world))
        y = torch.tensor(workloads.eeg_like(LARGE_N, seed=100 + ch), device=dev)
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        e[0].record(stream)
        ctr = {}
        imfs, tape = pkg.iceemdan_taped(y, nr, NUM_IMFS, MAX_ITER, NSTD, seed=1 + ch,
                                        noise_sift_cap=NOISE_CAP, checkpoint=True, counters=ctr)
        for k in ("iterations", "knots"):
            phases[k] = phases.get(k, 0) + ctr.get(k, 0)
        e[1].record(stream)
        gy = tape.backward(2.0 * w[:, None] * imfs)
        e[2].record(stream)
        torch.cuda.synchronize()
        phases["forward_ms"] = phases.get("forward_ms", 0.0) + e[0].elapsed_time(e[1])
        phases["backward_ms"] = phases.get("backward_ms", 0.0) + e[1].elapsed_time(e[2])
        phases["tape_bytes"] = max(phases.get("tape_bytes", 0), tape.bytes)
        tape.free()
        return gy

    for k in range(args.warmup):
        step(k, {})
    torch.cuda.synchronize()
    pkg.memory_stats(reset_peak=True)
    phases = {}
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        torch.cuda.synchronize()
        ev0.record(stream)
        for k in range(args.steps):
            step(args.warmup + k, phases)
        ev1.record(stream)
        torch.cuda.synchronize()
    ms = multichannel.max_over_ranks(ev0.elapsed_time(ev1), world, dev) / args.steps
    mem = pkg.memory_stats()
    if rank != 0:
        return 0
    units = LARGE_N * nr
    # HBM figure of the forward: the sift kernels' algorithmic bytes (BYTES_PER_N per
    # sample-realization iteration, BYTES_PER_K per knot, summed over the kernels) over the
    # forward's device time (noise-mode precompute and stage kernels included in the time)
    alg = (sum(BYTES_PER_N.get(k, 0.0) for k in ("extrema", "eval")) * LARGE_N * nr *
           phases.get("iterations", 0) + sum(BYTES_PER_K.values()) * phases.get("knots", 0))
    fwd_s = phases.get("forward_ms", 0.0) * 1e-3
    peak, peak_src = _peaks()
    hbm = {"forward_algorithmic_bytes": round(alg),
           "forward_gbs": round(alg / fwd_s / 1e9, 1) if fwd_s > 0 else None,
           "peak_gbs": peak, "peak_source": peak_src,
           "frac": round(alg / fwd_s / 1e9 / peak, 4) if fwd_s > 0 else None}
    line = {"metric": (f"samples x realizations / s (ICEEMDAN forward + adjoint, N={LARGE_N}, "
                       f"NR={nr}, {NUM_IMFS} IMFs, FP64)"),
            "value": world * units / (ms * 1e-3), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": (f"large forward + adjoint: EEG-shaped channels N={LARGE_N} "
                                    f"(seeds 100-227), NR={nr}, MaxIter={MAX_ITER}, "
                                    f"{NUM_IMFS} IMFs, "
                                    "checkpointed taped forward + backward, one channel per "
                                    "step"),
                       "phases_ms_per_step": {k: v / args.steps for k, v in phases.items()
                                              if k.endswith("_ms")},
                       "tape_bytes": phases.get("tape_bytes", 0),
                       "peak_device_bytes": mem["peak"], "hbm": hbm,
                       "forward_lockstep_iterations": phases.get("iterations", 0) // max(
                           1, args.steps)},
            "cpu_baseline": None, "e2e": None, "clocks": clk.summary()}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference", "reference-cuda"], default="ours")
    ap.add_argument("--ref-shapes", nargs="*", default=None,
                    help="--impl reference-cuda shapes NxNRxIMFsxMaxIter")
    ap.add_argument("--nr", type=int, default=NR)
    ap.add_argument("--imfs", type=int, default=NUM_IMFS)
    ap.add_argument("--sift-cap", type=int, default=0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--groups", type=int, default=B_GROUPS)
    ap.add_argument("--workload", choices=["batched", "eeg", "short", "differentiation",
                                           "large"],
                    default="batched")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.impl == "reference-cuda":
        return run_reference_cuda(args) if rank == 0 else 0
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=180))
    try:
        if args.workload == "differentiation":
            return run_differentiation(args, rank, world, local_rank)
        if args.workload == "batched":
            return run_batched(args, rank, world, local_rank)
        if args.workload == "large":
            return run_large(args, rank, world, local_rank)
        return run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
