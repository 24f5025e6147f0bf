#!/usr/bin/env python3
"""Benchmark: cell-steps/s of the fused FP64 NEMOLite2D stepper at 4096^2.

Workload (one instance per GPU): 4096 x 4096 T-points, dx = dy = 1 km, depth
100 m plus 32 seeded Gaussian bumps (amplitude U(+-40) m, width U(20,200) km,
floor 10 m), rdt 20 s, cbfr 1.5e-4, visc 0.1 m^2/s, tidal SSH clamp at the
open boundary (amplitude 0.2 m, period 12.42 h).  One bench step = 100 model
time steps (one record interval) + the device checksums of sshn/u/v, so the
default 10 timed steps are the 1000-step run with a record every 100 steps.
The state is reset to rest after warm-up, so the timed region is steps
1..100*K from rest.  Inputs (9 x 134 MB per step) are far larger than L2.

`value`: device-timed, state resident in HBM.  `e2e`: the same metric
through the C ABI with pinned host buffers: every step uploads the state
(nemo_set_state), steps, reads the state back (nemo_retrieve) and the
checksums; two contexts alternate so that one's transfers overlap the
other's steps.  `--impl reference` times the CPU restatement of the reference
(oracle/, OpenMP over all host cores) on the same grid.

The default line also carries, measured on the same GPU after the timed
region: `ensemble` (the 256-member batched configuration, its 500-step run
from rest, graph-replayed persistent launches, with its own roofline and
clocks), `conv` (the surrogate's forward and weight-gradient convolution
kernels at 64 x 256 x 256, TFLOP/s against the measured BF16 peak) and
`cpu_baseline` (the oracle on the host cores: OpenMP over every core and
serial on one pinned core at the bench grid, and config 0 both ways).

Multi-GPU (torchrun): independent replicas, one per GPU (the stepper does not
shard); value = all ranks' cell-steps / max-over-ranks time.  The ensemble,
convolution and CPU legs run at N = 1 only.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "nemolite2d-cuda_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

N = 4096
STEPS_PER_ITER = 100
WORKLOAD = dict(jpi=N, jpj=N, dx=1000.0, dy=1000.0, dep_const=100.0, rdt=20.0, cbfr=0.00015,
                visc=0.1, amp_tide=0.2, tide_phase=0.0, nbump=32, seed=1234, bump_amp=40.0,
                bump_wmin=20e3, bump_wmax=200e3, hmin=10.0)
BYTES_PER_CELL_STEP = 72  # read sshn, un, vn, ht, hu, hv; write sshn, un, vn (FP64)
METRIC = "cell-steps/s at 4096^2 FP64 (% of HBM peak)"
CONFIG = {"workload": "plain FP64 stepper, one 4096x4096 instance per GPU, seeded 32-bump "
                      "bathymetry (seed 1234), 1000 steps from rest, checksums every 100 steps, "
                      "tidal amplitude 0.2 m (the reference's hard-coded value; 1 m diverges "
                      "in the reference scheme)",
          "grid": [N, N], "dtype": "f64",
          "l2": "inputs larger than L2 (1.2 GB touched per model step)"}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-ensemble", action="store_true",
                    help="leave out the 256-member ensemble leg of the default line")
    ap.add_argument("--no-conv", action="store_true",
                    help="leave out the convolution leg of the default line")
    ap.add_argument("--schedule", type=str, default="",
                    help="warps,occupancy,rows of the fused kernel (default: tuned)")
    ap.add_argument("--workload", choices=["grid", "ensemble", "surrogate", "hybrid", "conv", "general"],
                    default="grid",
                    help="grid: the 4096^2 line (default); ensemble: the 256-member batch")
    ap.add_argument("--hyb-steps", type=int, default=5000)
    ap.add_argument("--patch", type=int, default=4, help="surrogate patch of the hybrid")
    ap.add_argument("--train-side", type=int, default=512, help="training run side (hybrid)")
    ap.add_argument("--train-steps", type=int, default=2000, help="training run length (hybrid)")
    ap.add_argument("--train-runs", type=int, default=96, help="training runs (hybrid)")
    ap.add_argument("--rollout-runs", type=int, default=48, help="rollout fine-tuning runs (hybrid)")
    ap.add_argument("--rollout-windows", type=int, default=20, help="windows per rollout run (hybrid)")
    ap.add_argument("--noise", type=float, default=0.03,
                    help="training input noise, in units of each field's spread (hybrid)")
    ap.add_argument("--finetune-iters", type=int, default=0,
                    help="fine-tuning iterations on rollout pairs (hybrid; 0: none)")
    ap.add_argument("--batch", type=int, default=64, help="images per conv call (conv workload)")
    ap.add_argument("--train-iters", type=int, default=6000)
    ap.add_argument("--runs", type=int, default=2048,
                    help="seeded 256^2 runs of the training set (surrogate workload)")
    ap.add_argument("--nblocks", type=int, default=2, help="residual blocks of the hybrid's network")
    ap.add_argument("--k", type=int, default=10, help="model steps per surrogate call (hybrid)")
    ap.add_argument("--anchor", type=int, default=100, help="FP64 re-anchor interval (hybrid)")
    ap.add_argument("--tol", type=float, default=0.01, help="fallback tolerance (hybrid)")
    ap.add_argument("--quarantine", type=float, default=0.05, help="quarantine threshold (hybrid)")
    ap.add_argument("--correct", type=int, default=0,
                    help="1: accepted calls add the shadow step's correction (hybrid)")
    ap.add_argument("--sweep", type=str, default="",
                    help="hybrid points anchor:tol:quarantine[:correct],... run after one training")
    ap.add_argument("--repeats", type=int, default=1, help="hybrid runs per point (median reported)")
    ap.add_argument("--candidates", type=int, default=128, help="hybrid member candidates")
    ap.add_argument("--strict", action="store_true", help="time the -fmad=false library (general)")
    ap.add_argument("--members", type=int, default=256,
                    help="ensemble members (profiling of smaller cases only; the line is 256)")
    ap.add_argument("--ens-schedule", type=str, default="",
                    help="warps,occupancy,rows,order of the ensemble workload (default: autotuned)")
    ap.add_argument("--gen-schedule", type=str, default="",
                    help="ring,rows of the general grid's kernel (ring 0, 3 or 4; default 3,32)")
    ap.add_argument("--n", type=int, default=N,
                    help="grid side (profiling of smaller cases only; the bench line is 4096)")
    return ap.parse_args()


def cells():
    return WORKLOAD["jpi"] * WORKLOAD["jpj"]


def max_over_ranks(ms, dist=None, device="cuda"):
    """The largest of every rank's time (the job's time); ms itself on one rank."""
    if dist is None:
        return ms
    import torch
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(cells_per_rank, steps, world, t_max_ms):
    """Whole-job cell-steps/s: every rank's independent replica advanced
    `steps` steps, over the slowest rank's time."""
    return cells_per_rank * steps * world / (t_max_ms / 1e3)


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def load_traffic():
    """DRAM bytes per fused launch from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "fused_step_4096.txt")
    if not os.path.exists(path):
        return None
    with open(path) as fh:
        for line in fh:
            if line.startswith("dram_bytes_per_launch:"):
                return float(line.split(":", 1)[1].split()[0])
    return None


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        import tempfile
        try:
            fd, self.path = tempfile.mkstemp(prefix="nemo_clocks_%d_" % self.index, suffix=".csv")
            self.fh = os.fdopen(fd, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.fh, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.fh.close()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as fh:
            for line in fh:
                f = [x.strip() for x in line.split(",")]
                if len(f) < 9:
                    continue
                try:
                    sm.append(float(f[1]))
                    smax = float(f[2])
                except ValueError:
                    continue
                for k, n in enumerate(names):
                    if f[5 + k].lower() == "active":
                        reasons.add(n)
        try:
            os.remove(self.path)
        except OSError:
            pass
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "samples": len(sm),
                "reasons": sorted(reasons)}


def cpu_model():
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def _timed_oracle_steps(m, istp0, n):
    t0 = time.perf_counter()
    m.run(istp0, n)
    return time.perf_counter() - t0


def cpu_baselines(omp_steps=20, serial_steps=20):
    """The oracle (the CPU restatement of original/nemolite2d.f90) on the
    host cores: config 1 (the bench grid) with OpenMP over every core and
    serial on one pinned core (the reference's own benchmark mode, one
    process on one core), and config 0 (128^2, 2000 steps) both ways.
    One untimed step first; the serial runs continue the OpenMP run's state
    (the arithmetic per step does not depend on the values)."""
    from oracle import oracle
    th = host_cores()
    keep = os.sched_getaffinity(0)
    pin = max(keep)
    out = {}
    try:
        oracle.set_threads(th)
        m = oracle.Model(**WORKLOAD)
        m.run(1, 1)
        dt = _timed_oracle_steps(m, 2, omp_steps)
        out["omp"] = (cells() * omp_steps / dt, dt)
        oracle.set_threads(1)
        os.sched_setaffinity(0, {pin})
        dt = _timed_oracle_steps(m, 2 + omp_steps, serial_steps)
        out["serial"] = (cells() * serial_steps / dt, dt)
        m.close()
        c0 = dict(jpi=128, jpj=128, rdt=20.0, cbfr=0.00015, visc=0.1, amp_tide=0.2)
        m = oracle.Model(**c0)
        out["c0_serial"] = 128 * 128 * 2000 / _timed_oracle_steps(m, 1, 2000)
        m.close()
        os.sched_setaffinity(0, keep)
        oracle.set_threads(th)
        m = oracle.Model(**c0)
        out["c0_omp"] = 128 * 128 * 2000 / _timed_oracle_steps(m, 1, 2000)
        m.close()
    finally:
        os.sched_setaffinity(0, keep)
        oracle.set_threads(1)
    return {"value": out["omp"][0], "unit": "cell-steps/s", "cores": th, "kind": "port",
            "sample": "%d model steps (2..%d) of the 4096^2 bench grid, oracle port of "
                      "original/nemolite2d.f90, OpenMP %d threads" % (omp_steps, omp_steps + 1, th),
            "cpu_model": cpu_model(),
            "serial": {"value": out["serial"][0], "cores": 1, "pinned_core": pin,
                       "steps": serial_steps, "seconds": out["serial"][1],
                       "sample": "steps %d..%d of the same run on one pinned core (the "
                                 "reference's benchmark mode)" % (2 + omp_steps,
                                                                  1 + omp_steps + serial_steps)},
            "config0": {"grid": [128, 128], "steps": 2000, "serial": out["c0_serial"],
                        "openmp": out["c0_omp"], "openmp_cores": th,
                        "sample": "the whole 2000-step 128^2 run from rest, amplitude 0.2 m"}}


def run_reference(args, rank):
    """CPU restatement of original/nemolite2d.f90 (the reference's CPU path),
    OpenMP over every host core, on the bench's workload and config: `warmup`
    untimed model steps, then `steps` timed model steps (each bench step of
    this arm is one model step; the metric, cell-steps/s, is the same)."""
    if rank != 0:
        return
    from oracle import oracle
    th = host_cores()
    oracle.set_threads(th)
    m = oracle.Model(**WORKLOAD)
    istp = 1
    for _ in range(args.warmup):
        m.step(istp)
        istp += 1
    t0 = time.perf_counter()
    for _ in range(args.steps):
        m.step(istp)
        istp += 1
    dt = time.perf_counter() - t0
    v = cells() * args.steps / dt
    sample = ("%d model steps of the 4096^2 bench grid (steps %d..%d), oracle port of "
              "original/nemolite2d.f90, OpenMP %d threads" % (args.steps, args.warmup + 1,
                                                               args.warmup + args.steps, th))
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "cell-steps/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 * dt / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(CONFIG), "bench_step": "1 model time step",
            "cpu_baseline": {"value": v, "unit": "cell-steps/s", "cores": th, "kind": "port",
                             "sample": sample, "cpu_model": cpu_model()},
            "e2e": {"value": v, "unit": "cell-steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


ENS_METRIC = "ensemble cell-steps/s (256 members, 500 steps, FP64)"


def ensemble_leg(device, warmup, reps, tune_steps=3, schedule=None, nmem=256):
    """The batched configuration: 256 members of the recipe (seed 2026, sides
    log-uniform 64..1024, aspect 0.5..2, seeded 50-150 m bathymetry, random
    tidal phase), the 500-step run from rest with per-member checksums every
    100 steps, one persistent launch per step replayed from a CUDA graph,
    schedule from the autotuner; `reps` timed runs after `warmup` untimed
    ones.  Tidal amplitudes are the reference's 0.2 m scaled by U[0.5, 1.5]
    (the 1 m class diverges with a random phase; throughput does not depend
    on the amplitude)."""
    import numpy as np
    import torch
    import nemo_b200
    stream = torch.cuda.Stream()
    members = nemo_b200.generate_members(2026, nmem, 64, 1024, amp_scale=0.2)
    common = nemo_b200.default_params(dx=1000.0, dy=1000.0, rdt=20.0, cbfr=0.00015, visc=0.1,
                                      stream=stream.cuda_stream, device=device)
    e = nemo_b200.Ensemble(members, common=common)
    nmem, ncell = e.info()
    if schedule:  # a fixed schedule (profiling), else the autotuner's choice
        e.set_schedule(*schedule)
        sched = e.get_schedule()
    else:
        sched, tuned_ms = e.autotune(steps=tune_steps)
    rest = [(np.zeros((m.jpj, m.jpi)), np.zeros((m.jpj, m.jpi + 1)), np.zeros((m.jpj + 1, m.jpi)))
            for m in members]
    for w in range(warmup):
        for r in range(5):
            e.step_n(1 + 100 * r, 100)
            e.checksums()
    for k, st in enumerate(rest):
        e.set_state(k, *st)
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    clocks = ClockSampler(device)
    clocks.start()
    t0.record(stream)
    for it in range(reps):
        if it:
            for k, st in enumerate(rest):
                e.set_state(k, *st)
        for r in range(5):
            e.step_n(1 + 100 * r, 100)
            ck = e.checksums()
    t1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = t0.elapsed_time(t1)
    e.close()
    value = ncell * 500 * reps / (ms / 1e3)
    peak = load_peaks()
    return {"metric": ENS_METRIC, "value": value, "unit": "cell-steps/s", "members": nmem,
            "cells": ncell, "steps": 500, "reps": reps, "ms_per_rep": ms / reps,
            "schedule": {"warps": sched[0], "occupancy": sched[1], "rows": sched[2],
                         "order": sched[3]},
            "graph": True, "finite_members": int(np.isfinite(ck).all(axis=1).sum()),
            "roofline": {"bound": "hbm", "kernel": "k_ens_step",
                         "achieved": BYTES_PER_CELL_STEP * value / 1e9, "peak": peak[0],
                         "unit": "GB/s", "frac": BYTES_PER_CELL_STEP * value / 1e9 / peak[0],
                         "peak_source": peak[1]},
            "gpu_launches": reps * (500 + 10), "clocks": clk}


def conv_leg(device, batch=64, reps=200, warm=3):
    """The surrogate's two convolution kernels alone (64 -> 64 channels, 3x3,
    batch x 256 x 256 BF16 NHWC, FP32 accumulation): forward with the bias +
    ReLU epilogue and weight gradient with the bias gradient, `reps` timed
    launches each."""
    import torch
    import nemo_b200
    from nemo_b200 import surrogate as sm
    stream = torch.cuda.Stream()
    S = 256
    clocks = ClockSampler(device)
    clocks.start()
    rates = conv_kernel_rates(sm, nemo_b200.load(False), batch, S, S, reps, stream.cuda_stream,
                              warm=warm)
    clk = clocks.stop()
    flop = 2 * 9 * 64 * 64 * batch * S * S
    peak = load_peaks_tensor()
    out = {"batch": batch, "grid": [S, S], "flop_per_launch": flop, "launches": reps,
           "peak": peak[0], "peak_source": peak[1], "unit": "TFLOP/s", "clocks": clk,
           "gpu_launches": 2 * (reps + warm)}
    for k, name in (("fwd", "k_conv_fwd_tri"), ("wgrad", "k_conv_wgrad_strip")):
        tf = flop / rates[k] / 1e12
        out[k] = {"kernel": name, "tflops": tf, "frac": tf / peak[0], "us": rates[k] * 1e6}
    return out


def run_ensemble(args):
    """The batched configuration alone (see ensemble_leg): one bench step is
    the 500-step run of all 256 members."""
    import torch
    torch.cuda.set_device(0)
    fixed = tuple(int(x) for x in args.ens_schedule.split(",")) if args.ens_schedule else None
    leg = ensemble_leg(0, args.warmup, args.steps, schedule=fixed, nmem=args.members)
    line = {"metric": ENS_METRIC, "value": leg["value"], "unit": "cell-steps/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": leg["ms_per_rep"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": "batched ensemble: %d members, %d cells, 500 steps, checksums "
                                   "per member every 100 steps" % (leg["members"], leg["cells"]),
                       "schedule": leg["schedule"], "graph": True, "l2": "inputs larger than L2"},
            "roofline": leg["roofline"], "finite_members": leg["finite_members"],
            "gpu_launches": leg["gpu_launches"], "clocks": leg["clocks"]}
    print(json.dumps(line), flush=True)


def conv_kernel_rates(sur_mod, lib, n, h, w, reps, stream, warm=3):
    """Device time of one 3x3 conv forward (bias+ReLU epilogue) and one weight
    gradient over n x h x w pixels (64 -> 64 channels), inputs larger than L2."""
    import torch
    x = torch.randn((n, h, w, 64), device="cuda").to(torch.bfloat16)
    y = torch.empty_like(x)
    wt = (0.05 * torch.randn((9, 64, 64), device="cuda")).to(torch.bfloat16)
    b = torch.zeros(64, device="cuda")
    dw = torch.zeros((9, 64, 64), device="cuda")
    db = torch.zeros(64, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    out = {}
    for name in ("fwd", "wgrad"):
        def launch():
            if name == "fwd":
                sur_mod.conv3x3_fwd(lib, x.data_ptr(), wt.data_ptr(), n, h, w, err.data_ptr(),
                                    bias=b.data_ptr(), relu=True, out=y.data_ptr(), stream=stream)
            else:
                sur_mod.conv3x3_wgrad(lib, x.data_ptr(), y.data_ptr(), dw.data_ptr(), n, h, w,
                                      err.data_ptr(), db=db.data_ptr(), stream=stream)
        for _ in range(warm):
            launch()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        s = torch.cuda.ExternalStream(stream)
        e0.record(s)
        for _ in range(reps):
            launch()
        e1.record(s)
        torch.cuda.synchronize()
        out[name] = e0.elapsed_time(e1) / reps / 1e3
    assert int(err.item()) == 0
    return out


def run_conv(args):
    """The surrogate's two convolution kernels alone: forward (bias + ReLU
    epilogue) and weight gradient (+ bias gradient), 64 -> 64 channels, 3x3,
    batch x 256 x 256 BF16 NHWC, FP32 accumulation; `steps` timed launches
    of each after `warmup`."""
    import torch
    import nemo_b200
    from nemo_b200 import surrogate as sm
    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    B, S = args.batch, 256
    clocks = ClockSampler(0)
    clocks.start()
    rates = conv_kernel_rates(sm, nemo_b200.load(False), B, S, S, max(args.steps, 1),
                              stream.cuda_stream, warm=args.warmup)
    clk = clocks.stop()
    flop = 2 * 9 * 64 * 64 * B * S * S
    peak = load_peaks_tensor()
    tf = {k: flop / v / 1e12 for k, v in rates.items()}
    line = {"metric": "3x3 conv TFLOP/s (64->64 ch, BF16 in, FP32 accumulate, %dx256x256)" % B,
            "value": tf["fwd"], "unit": "TFLOP/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": rates["fwd"] * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "bf16", "data": "synthetic",
            "config": {"workload": "conv kernels alone", "batch": B, "grid": [S, S],
                       "l2": "%d MiB per activation tensor" % (B * S * S * 128 >> 20)},
            "roofline": {"bound": "tensor", "kernel": "k_conv_fwd_tri", "achieved": tf["fwd"],
                         "peak": peak[0], "unit": "TFLOP/s", "frac": tf["fwd"] / peak[0],
                         "peak_source": peak[1], "traffic": None},
            "wgrad": {"kernel": "k_conv_wgrad_strip", "achieved": tf["wgrad"], "frac": tf["wgrad"] / peak[0],
                      "us": rates["wgrad"] * 1e6},
            "gpu_launches": 2 * (args.steps + args.warmup), "clocks": clk}
    print(json.dumps(line), flush=True)


def run_surrogate(args):
    """Surrogate training on solver-generated data: 2048 seeded 256x256 runs
    of the batched recipe (500 steps from rest, FP32 snapshots every 10 steps,
    about 100 GiB resident in HBM, generated 256 runs at a time by the
    ensemble solver), the 8-block 64-channel residual CNN, batch 64, AdamW.
    One bench step = one training iteration (forward, loss, backward, AdamW)
    on pairs drawn from the whole set.  Also times the forward and
    weight-gradient conv kernels alone at the same batch."""
    import numpy as np
    import torch
    import nemo_b200
    from nemo_b200 import surrogate as sm
    from nemo_b200 import train as tr
    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    B, S = 64, 256
    sur = sm.Surrogate(nblocks=8, batch=B, height=S, width=S, seed=1234, stream=stream.cuda_stream,
                       device=0)
    nparams, flops_px = sur.info()
    with torch.cuda.stream(stream):
        t_gen = time.perf_counter()
        chunks, dropped = tr.generate_dataset(sur, seed=7000, nruns=args.runs, side=S, steps=500)
        torch.cuda.synchronize()
        t_gen = time.perf_counter() - t_gen
        kept = sum(c[0].shape[1] for c in chunks)
        nsnap = sum(c[0].shape[0] * c[0].shape[1] for c in chunks)
        sur.set_norm(*tr.compute_norm(chunks[0][0]))
        sampler = tr.ChunkPairSampler(chunks, seed=3)
        hp = sm.adamw(lr=1e-3, weight_decay=1e-4)
        losses = []
        for _ in range(args.warmup):
            s0, s1, t1 = sampler.batch(B)
            losses.append(sur.train_step(s0.data_ptr(), s1.data_ptr(), t1.data_ptr(), B, hp))
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        clocks = ClockSampler(0)
        clocks.start()
        e0.record(stream)
        for _ in range(args.steps):
            s0, s1, t1 = sampler.batch(B)
            losses.append(sur.train_step(s0.data_ptr(), s1.data_ptr(), t1.data_ptr(), B, hp))
        e1.record(stream)
        torch.cuda.synchronize()
        clk = clocks.stop()
        ms = e0.elapsed_time(e1) / args.steps
        del chunks, sampler
        rates = conv_kernel_rates(sm, nemo_b200.load(False), B, S, S, 20, stream.cuda_stream)
    npix = B * S * S
    conv_flop = 2 * 9 * 64 * 64 * npix
    L = 2 * 8 + 2
    # forward L convs, data gradient L-1 (none for the input), weight gradient L
    iter_flop = conv_flop * (L + (L - 1) + L)
    peak = load_peaks_tensor()
    fwd_tf = conv_flop / rates["fwd"] / 1e12
    line = {"metric": "surrogate training samples/s (8-block 64-ch BF16 residual CNN, 256^2, batch 64)",
            "value": B / (ms / 1e3), "unit": "samples/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "bf16", "data": "synthetic (solver-generated)",
            "config": {"workload": "surrogate training: %d seeded 256x256 runs, 500 steps, FP32 "
                                   "snapshots every 10 steps; batch 64; AdamW" % args.runs,
                       "params": nparams, "conv_flop_per_iter": iter_flop,
                       "runs_dropped_unbounded": dropped, "runs_kept": kept,
                       "snapshots": nsnap, "snapshot_bytes": nsnap * S * S * 16,
                       "pairs": nsnap - kept,
                       "data_generation_s": t_gen,
                       "l2": "activations 512 MiB per tensor, larger than L2"},
            "train_tflops": iter_flop / (ms / 1e3) / 1e12,
            "roofline": {"bound": "tensor", "kernel": "k_conv_fwd_tri", "achieved": fwd_tf,
                         "peak": peak[0], "unit": "TFLOP/s", "frac": fwd_tf / peak[0],
                         "peak_source": peak[1], "traffic": None,
                         "wgrad_tflops": conv_flop / rates["wgrad"] / 1e12,
                         "fwd_us": rates["fwd"] * 1e6, "wgrad_us": rates["wgrad"] * 1e6},
            "loss_first": losses[0], "loss_last": losses[-1],
            "gpu_launches": args.steps * (2 * L + L - 1 + 6), "clocks": clk}
    print(json.dumps(line), flush=True)
    sur.close()


def load_peaks_tensor():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return float(json.load(fh)["bf16_tflops"]), "measured (burst)"
    except (OSError, KeyError, ValueError):
        return 1590.0, "fallback"


def run_hybrid(args):
    """Hybrid inference versus the plain solver: 32 members at 2048x2048
    (seeded bathymetry and tides of the batched recipe), 5000 steps.  The
    surrogate runs on 4x4 patches of T-cells (a call costs 1/16 of the
    full-resolution network) and is trained first on solver runs of the same
    recipe at 512x512 (pairs of snapshots 10 steps apart every 50 steps of
    2000-step runs), then fine-tuned on pairs along trajectories it advances
    itself between solver windows; it advances 10 steps per call, and the FP64 solver
    re-anchors every 100 steps and takes the rest of the window over for each
    member whose shadow SSH error exceeds 1%.  Reports both rates and the
    hybrid's error against the plain FP64 run (which matches the FP64 oracle
    to 1e-12)."""
    import numpy as np
    import torch
    from nemo_b200 import surrogate as sm
    from nemo_b200 import train as tr
    import nemo_b200
    torch.cuda.set_device(0)
    nsteps = args.hyb_steps
    side, nm, P, ts = 2048, 32, args.patch, args.train_side
    # ---- train on solver runs of the recipe
    trainer = sm.Surrogate(nblocks=args.nblocks, batch=64, height=ts, width=ts, seed=1234, device=0, patch=P)
    t_gen = time.time()
    snaps, tides = tr.generate_runs(trainer, seed=7000, nmem=args.train_runs, side=ts,
                                    steps=args.train_steps, every=args.k, pair_stride=50)
    t_gen = time.time() - t_gen
    norm = tr.compute_norm(snaps, paired=True)
    trainer.set_norm(*norm)
    t_train = time.time()
    clean = tr.PairSampler(snaps, tides, seed=3, paired=True)
    # inputs perturbed by noise, targets the true states: the network learns to
    # advance slightly wrong states, as it meets them after its own calls
    noisy = tr.NoisySampler(clean, args.noise, tr.field_std(snaps), seed=5)
    losses = tr.train(trainer, noisy, iters=args.train_iters, batch=64, lr=1e-3)
    if args.finetune_iters > 0:
        # optional fine-tuning on the states the hybrid meets: pairs along
        # trajectories the surrogate itself advances between solver windows
        rsnaps, rtides = tr.rollout_runs(trainer, seed=9000, nmem=args.rollout_runs, side=ts,
                                         windows=args.rollout_windows)
        mix = tr.MixSampler([clean, tr.PairSampler(rsnaps, rtides, seed=4, paired=True)], [1.0, 1.0])
        losses += tr.train(trainer, mix, iters=args.finetune_iters, batch=64, lr=5e-4)
        del rsnaps, rtides, mix
    t_train = time.time() - t_train
    params = trainer.params()
    trainer.close()
    del snaps, tides, clean, noisy
    torch.cuda.empty_cache()
    # ---- members: seeded candidates screened by the FP64 solver over the run
    # (the reference scheme lets a tide that starts rising grow without bound
    # at the east-wall/open-boundary corner); the first 32 whose run stays
    # bounded (max |ssh| <= 2.5 x the tidal amplitude at mid-run and at the
    # end, the rule the training data follow) are the workload
    stream = torch.cuda.Stream()
    common = dict(tr.COMMON, stream=stream.cuda_stream, device=0)
    cands = tr.square_members(4242, args.candidates, side, 0.2)
    ok = tr.bounded_members(cands, nsteps, common, want=nm)
    members = [cands[i] for i in ok[:nm]]
    screened = min(len(cands), 64 * ((ok[nm - 1] // 64) + 1)) if len(ok) >= nm else len(cands)
    nm = len(members)
    plain = nemo_b200.Ensemble(members, **common)
    hyb = nemo_b200.Ensemble(members, **common)
    inf = sm.Surrogate(nblocks=args.nblocks, batch=nm, height=side, width=side, train=False, seed=1,
                       stream=stream.cuda_stream, device=0, patch=P)
    inf.set_params(params)
    inf.set_norm(*norm)
    cells = nm * side * side
    rest = [(np.zeros((m.jpj, m.jpi)), np.zeros((m.jpj, m.jpi + 1)), np.zeros((m.jpj + 1, m.jpi)))
            for m in members]
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]

    def timed(fn):
        torch.cuda.synchronize()
        ev[0].record(stream)
        out = fn()
        ev[1].record(stream)
        torch.cuda.synchronize()
        return ev[0].elapsed_time(ev[1]) / 1e3, out

    t_plain = []
    for r in range(args.repeats):
        if r:
            for k, st0 in enumerate(rest):
                plain.set_state(k, *st0)
        t_plain.append(timed(lambda: plain.step_n(1, nsteps))[0])
    plain.checksums()
    v_plain = cells * nsteps / statistics.median(t_plain)
    points = [(args.anchor, args.tol, args.quarantine, args.correct)]
    if args.sweep:
        points = [tuple(float(x) for x in p.split(":")) for p in args.sweep.split(",")]
        points = [p if len(p) == 4 else p + (args.correct,) for p in points]
    for anchor, tol, quar, corr in points:
        anchor, corr = int(anchor), int(corr)
        runs = []
        for r in range(args.repeats):
            for k, st0 in enumerate(rest):
                hyb.set_state(k, *st0)
            clocks = ClockSampler(0)
            clocks.start()
            t_hyb, st = timed(lambda: sm.hyb_run(inf, hyb, 0, nsteps, k=args.k, anchor=anchor, tol=tol,
                                                 quarantine=quar, correct=bool(corr)))
            clk = clocks.stop()
            err = sm.ens_compare(hyb, plain)
            finite = np.isfinite(err).all(axis=1)
            ef = err[finite] if finite.any() else np.full((1, 3), np.nan)
            runs.append({"seconds": t_hyb, "hybrid_over_plain": (cells * nsteps / t_hyb) / v_plain,
                         "stats": st, "clocks": clk,
                         "err": {"ssh_max": float(ef[:, 0].max()), "ssh_mean": float(ef[:, 0].mean()),
                                 "u_max": float(ef[:, 1].max()), "v_max": float(ef[:, 2].max()),
                                 "u_mean": float(ef[:, 1].mean()), "v_mean": float(ef[:, 2].mean()),
                                 "members_nonfinite": int((~finite).sum())}})
        med = sorted(runs, key=lambda x: x["seconds"])[len(runs) // 2]
        st = med["stats"]
        v_hyb = cells * nsteps / med["seconds"]
        line = {"metric": "hybrid vs plain ensemble cell-steps/s (32 x 2048^2, 5000 steps, <=1% SSH err)",
                "value": v_hyb, "unit": "cell-steps/s", "n_gpus": 1, "steps": args.repeats, "warmup": 0,
                "ms_per_step": med["seconds"] * 1e3, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "bf16+f64", "data": "synthetic",
                "config": {"workload": "%d members 2048x2048, %d steps, surrogate k=%d, re-anchor %d, "
                                       "tol %g relative SSH L2 vs shadow FP64 step, quarantine %g%s"
                                       % (nm, nsteps, args.k, anchor, tol, quar,
                                          ", shadow correction" if corr else ""),
                           "anchor": anchor, "tol": tol, "quarantine": quar, "k": args.k,
                           "correct": corr,
                           "candidates": len(cands), "candidates_screened": screened,
                           "screened_out": screened - len(ok),
                           "patch": P, "nblocks": args.nblocks, "train_side": ts,
                           "train_steps": args.train_steps, "train_runs": args.train_runs,
                           "fallback": "per member", "train_input_noise": args.noise,
                           "finetune_iters": args.finetune_iters,
                           "train_iters": args.train_iters, "train_s": t_train, "datagen_s": t_gen,
                           "train_runs_dropped": tr.generate_runs.dropped},
                "plain_value": v_plain, "plain_seconds": t_plain,
                "hybrid_over_plain": v_hyb / v_plain,
                "hybrid_over_plain_runs": [x["hybrid_over_plain"] for x in runs],
                "hybrid_stats": st,
                "surrogate_share": st["sur_steps"] / max(1, st["sur_steps"] + st["solver_steps"]),
                "err_vs_fp64": med["err"], "err_vs_fp64_runs": [x["err"] for x in runs],
                "loss_first": losses[0], "loss_last": losses[-1], "clocks": med["clocks"],
                "gpu_launches": st["launches"]}
        print(json.dumps(line), flush=True)


GEN_BYTES_PER_CELL_STEP = 137  # 113 read (6 state/depth + 8 metric fields, int8 mask), 24 written


def general_grid(jpi, jpj, seed=3, dx=1000.0, dy=1000.0):
    """A general grid as nemo_set_grid takes it ((jpj+2, jpi+2) arrays over
    (0:jpi+1, 0:jpj+1)): open water on parts of all four borders, 64 land
    islands, scale factors within 15% of dx, dy and latitudes 30-60 degrees
    varying smoothly per point, one smooth bathymetry of 25-75 m."""
    import numpy as np
    rng = np.random.default_rng(seed)
    shape = (jpj + 2, jpi + 2)
    pt = np.ones(shape, np.int32)
    pt[:, 0] = pt[:, jpi + 1] = pt[0, :] = pt[jpj + 1, :] = 0
    pt[0, jpi // 8: jpi // 2] = -1
    pt[jpj + 1, jpi // 3: 2 * jpi // 3] = -1
    pt[jpj // 4: jpj // 2, 0] = -1
    pt[jpj // 2: 3 * jpj // 4, jpi + 1] = -1
    for _ in range(64):
        y0, x0 = int(rng.integers(3, jpj - 40)), int(rng.integers(3, jpi - 40))
        pt[y0:y0 + int(rng.integers(1, 32)), x0:x0 + int(rng.integers(1, 32))] = 0
    jj, ji = np.mgrid[0:jpj + 2, 0:jpi + 2].astype(np.float64)
    pos = {"t": (ji, jj), "u": (ji + 0.5, jj), "v": (ji, jj + 0.5)}

    def smooth(at, amp):
        kx, ky = rng.uniform(0.5, 2.0, 2)
        p1, p2 = rng.uniform(0.0, 2.0 * np.pi, 2)
        x, y = pos[at]
        return amp * np.sin(2 * np.pi * kx * x / jpi + p1) * np.cos(2 * np.pi * ky * y / jpj + p2)

    g = {}
    for name, base, at in (("e1t", dx, "t"), ("e2t", dy, "t"), ("e1u", dx, "u"), ("e2u", dy, "u"),
                           ("e1v", dx, "v"), ("e2v", dy, "v")):
        g[name] = base * (1.0 + smooth(at, 0.15))
    g["gphiu"] = 45.0 + smooth("u", 15.0)
    g["gphiv"] = 45.0 + smooth("v", 15.0)
    kx, ky = rng.uniform(0.5, 2.0, 2)
    p1, p2 = rng.uniform(0.0, 2.0 * np.pi, 2)
    for name, at in (("ht", "t"), ("hu", "u"), ("hv", "v")):
        x, y = pos[at]
        g[name] = 50.0 + 25.0 * np.sin(2 * np.pi * kx * x / jpi + p1) * np.cos(2 * np.pi * ky * y / jpj + p2)
    return pt, g


def run_general(args):
    """The fused step on a general grid (nemo_set_grid) at 4096^2: every step
    is the general kernel plus the Flather chains; one bench step = 100 model
    steps + checksums; `steps` timed after `warmup`, from rest."""
    import numpy as np
    import torch
    import nemo_b200
    torch.cuda.set_device(0)
    n = args.n
    stream = torch.cuda.Stream()
    m = nemo_b200.Model(strict=args.strict, stream=stream.cuda_stream, device=0, jpi=n, jpj=n, rdt=10.0,
                        cbfr=0.00015, visc=0.1, amp_tide=0.3)
    pt, g = general_grid(n, n)
    names = ("e1t", "e2t", "e1u", "e2u", "e1v", "e2v", "gphiu", "gphiv", "ht", "hu", "hv")
    m.set_grid(pt, *[g[k] for k in names])
    del g
    if args.gen_schedule:
        ring, rows = (int(x) for x in args.gen_schedule.split(","))
        m.set_schedule(2, ring, rows)
    rest = (np.zeros((n, n)), np.zeros((n, n + 1)), np.zeros((n + 1, n)))
    for w in range(args.warmup):
        m.step_n(1 + 100 * w, 100)
        m.checksums()
    m.set_state(*rest)
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    clocks = ClockSampler(0)
    clocks.start()
    ev[0].record(stream)
    for k in range(args.steps):
        m.step_n(1 + 100 * k, 100)
        ck = m.checksums()
    ev[1].record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = ev[0].elapsed_time(ev[1])
    value = n * n * 100 * args.steps / (ms / 1e3)
    sch = m.get_schedule()
    peak, kind = load_peaks()
    achieved = GEN_BYTES_PER_CELL_STEP * value / 1e9
    line = {"metric": "general-grid cell-steps/s at %d^2 FP64" % n, "value": value,
            "unit": "cell-steps/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "general grid %dx%d: open water on all four borders, 64 islands, "
                                   "per-point scale factors, latitudes and depths; 100 model steps + "
                                   "checksums per bench step" % (n, n),
                       "l2": "inputs larger than L2"},
            "roofline": {"bound": "hbm", "kernel": "k_fused_general", "achieved": achieved,
                         "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_source": kind,
                         "algorithmic_bytes_per_cell_step": GEN_BYTES_PER_CELL_STEP},
            "checksums_last": [float(x) for x in ck], "build": "strict" if args.strict else "default",
            "schedule": {"warps": sch[0], "ring": sch[1], "rows": sch[2]},
            "gpu_launches": args.steps * (2 * 100 + 2), "clocks": clk}
    print(json.dumps(line), flush=True)
    m.close()


def main():
    args = parse()
    if args.workload == "ensemble":
        import numpy as np  # noqa: F401
        globals()["np"] = np
        return run_ensemble(args)
    if args.workload == "surrogate":
        return run_surrogate(args)
    if args.workload == "hybrid":
        return run_hybrid(args)
    if args.workload == "conv":
        return run_conv(args)
    if args.workload == "general":
        return run_general(args)
    if args.n != N:
        WORKLOAD["jpi"] = WORKLOAD["jpj"] = args.n
        CONFIG["grid"] = [args.n, args.n]
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank)

    import numpy as np
    import torch
    import nemo_b200

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    def barrier():
        if dist is not None:
            dist.barrier()

    stream = torch.cuda.Stream()
    m = nemo_b200.Model(strict=False, stream=stream.cuda_stream, device=local, **WORKLOAD)
    if args.schedule:
        m.set_schedule(*(int(x) for x in args.schedule.split(",")))
    jpi, jpj = m.jpi, m.jpj
    rest = (np.zeros((jpj, jpi)), np.zeros((jpj, jpi + 1)), np.zeros((jpj + 1, jpi)))

    # warm-up, then back to rest so the timed steps are 1..100*K
    for w in range(args.warmup):
        m.step_n(1 + STEPS_PER_ITER * w, STEPS_PER_ITER)
        m.checksums()
    m.set_state(*rest)
    torch.cuda.synchronize()

    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    clocks = ClockSampler(local)
    records = []
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    t_start.record(stream)
    for k in range(args.steps):
        ev[k][0].record(stream)
        m.step_n(1 + STEPS_PER_ITER * k, STEPS_PER_ITER)
        ev[k][1].record(stream)
        records.append(m.checksums())
    t_end.record(stream)
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    total_ms = t_start.elapsed_time(t_end)
    fused_ms = sum(a.elapsed_time(b) for a, b in ev)
    t_max = max_over_ranks(total_ms, dist)
    value = job_rate(cells(), STEPS_PER_ITER * args.steps, world, t_max)
    launch_s = fused_ms / 1e3 / (STEPS_PER_ITER * args.steps)
    peak, peak_kind = load_peaks()
    achieved = BYTES_PER_CELL_STEP * cells() / launch_s / 1e9
    traffic = load_traffic()

    # ---- end to end through the C ABI with pinned host buffers --------------
    # Every step uploads its state from pinned host memory (nemo_set_state),
    # runs 100 model steps, and reads the state and the checksums back
    # (nemo_retrieve, nemo_checksums).  Two contexts on their own streams
    # alternate, as a caller streaming many inputs would run them: one
    # context's transfers (blocking calls, on the copy engines) overlap the
    # other's steps.
    e2e = None
    if not args.no_e2e:
        stream2 = torch.cuda.Stream()
        m2 = nemo_b200.Model(strict=False, stream=stream2.cuda_stream, device=local, **WORKLOAD)
        m2.set_schedule(*m.get_schedule())
        ctxs = (m, m2)
        hbuf = [[torch.zeros(a.shape, dtype=torch.float64, pin_memory=True).numpy() for a in rest]
                for _ in ctxs]
        fields = (nemo_b200.SSHN, nemo_b200.UN, nemo_b200.VN)
        bi = sum(a.nbytes for a in hbuf[0])
        bo = sum(a.nbytes for a in hbuf[0]) + 3 * 8
        k_e2e = max(2, args.steps)  # the same K steps as the device-timed region
        for w in range(2):  # warm the second context's launch path
            m2.step_n(1 + STEPS_PER_ITER * w, STEPS_PER_ITER)
        barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)

        def read_back(k):
            c = ctxs[k % 2]
            for f, o in zip(fields, hbuf[k % 2]):
                c.field(f, out=o)
            c.checksums()

        for k in range(k_e2e):
            c = ctxs[k % 2]
            c.set_state(*hbuf[k % 2])
            c.step_n(1 + STEPS_PER_ITER * k, STEPS_PER_ITER)
            if k > 0:
                read_back(k - 1)
        read_back(k_e2e - 1)
        stream.wait_stream(stream2)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        e_ms = max_over_ranks(e0.elapsed_time(e1), dist)
        e2e = {"value": job_rate(cells(), STEPS_PER_ITER * k_e2e, world, e_ms),
               "unit": "cell-steps/s", "h2d_bytes_per_step": bi, "d2h_bytes_per_step": bo,
               "steps": k_e2e, "contexts": 2}
        m2.close()

    sched = m.get_schedule()
    m.close()

    # ---- the other two kernels families on the same box (one GPU only) -----
    ens = conv = None
    if world == 1 and not args.no_ensemble:
        ens = ensemble_leg(local, warmup=1, reps=1)
    if world == 1 and not args.no_conv:
        conv = conv_leg(local)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baselines()

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "cell-steps/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_max / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64", "data": "synthetic", "config": dict(CONFIG),
                "bench_step": "%d model steps + device checksums of sshn, u, v" % STEPS_PER_ITER,
                "parallelism": "replicas x%d" % world,
                "schedule": {"warps": sched[0], "occupancy": sched[1], "rows": sched[2]},
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak,
                             "unit": "GB/s", "frac": achieved / peak,
                             "peak_source": peak_kind, "traffic": traffic,
                             "kernel": "k_fused_step", "launch_us": launch_s * 1e6,
                             "algorithmic_bytes_per_launch": BYTES_PER_CELL_STEP * cells()},
                "gpu_launches": args.steps * (STEPS_PER_ITER + 2),
                "checksums_last": [float(x) for x in records[-1]],
                "clocks": clk, "e2e": e2e, "cpu_baseline": cpu,
                "ensemble": ens, "conv": conv}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
