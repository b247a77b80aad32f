#!/usr/bin/env python
"""Benchmark: one bootstrap particle-filter step (LibBi BootstrapPF::step) on
the Lorenz '96 workload, d = 40, N = 65536 FP32 particles, RK4 h = 0.01 with
N(0, 0.1^2) noise every 0.05, all 40 components observed with N(0, 1) noise
every 0.05, systematic resampling at ESS < 0.5 N.

A step is resample-if-due + fused transition/observation/reduction of all N
particles for one observation interval.  Metric: particle-steps/s.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun each rank runs an independent replica (the single filter does
not shard; replicas only) and rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = "l96_d40_n65536"
METRIC = "particle-steps/s/GPU"
UNIT = "particle-steps/s"
N_PARTICLES = 65536
DIM = 40
T_OBS = 200
DT = 0.05
ESS_REL = 0.5
SEED = 2
DATA_SEED = 102
L2_FLUSH_BYTES = 256 << 20  # > 126 MB L2
# our kernels per step with the systematic resampler: one (the step kernel,
# resampling as its prologue when due) in the one-launch form; two (the
# cooperative resample kernel, launched every step and gated on the device,
# then the fused transition) in the two-launch form
LAUNCHES_PER_STEP = {True: 1, False: 2}
# algorithmic bytes of the fused transition per particle: state read + write
# (2 * d * 4 B) and FP64 log-weight read + write (16 B); the ancestor index
# (4 B) is read only on resample steps
TRANSITION_BYTES_PER_PARTICLE = 2 * DIM * 4 + 16
# FP32 operations per particle-step of the fused transition (FMA = 2):
# RK4 5 sub-steps x 40 components x 31 + noise add 2 x 40 + observation 6 x 40
TRANSITION_FLOP_PER_PARTICLE = 5 * DIM * 31 + 2 * DIM + 6 * DIM
# DRAM bytes (read + write) of one transition launch at this workload from an
# ncu capture of the transition (dram__bytes_read.sum + dram__bytes_write.sum,
# 128-thread blocks): 10.8 MB read, nothing written back within the launch
# (the new state stays in L2)
TRANSITION_DRAM_BYTES_PER_LAUNCH = 10_814_464 + 0


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), "measured", d.get("sm_max_mhz", 1965.0)
    return 6650.0, "fallback", 1965.0


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str):
        self.gpu_id = gpu_id
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", self.gpu_id, f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                mx = float(f[1])
            except ValueError:
                continue
            for nm, v in zip(names, f[4:8]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


L2_NOTE = "flushed before every timed step (256 MiB write)"


def workload_config(world: int) -> dict:
    """The workload's `config` object, the same in both arms."""
    return {"workload": WORKLOAD, "nparticles": N_PARTICLES, "dim": DIM, "obs_interval": DT, "rk4_h": 0.01,
            "resampler": "systematic", "ess_rel": ESS_REL,
            "parallelism": f"replicas{world}" if world > 1 else "single", "l2": L2_NOTE}


def observe(xs, sigma_y):
    """Observations of a true trajectory xs (T_OBS x DIM): N(0, sigma_y^2) noise."""
    import numpy as np

    rng = np.random.default_rng(DATA_SEED)
    return (xs + sigma_y * rng.standard_normal(xs.shape)).astype(np.float32)


def synthetic_observations(model):
    """One model run (the library's own transition with its process noise,
    N = 1, no observations) from the data seed, observed with N(0, sigma_y^2)
    noise: T_OBS x DIM values in FP32, on the host."""
    import numpy as np
    from libbi_b200 import BootstrapPF

    truth = BootstrapPF(model, 1, seed=DATA_SEED)
    xs = np.zeros((T_OBS, DIM), np.float32)
    for k in range(T_OBS):
        truth.step(k * DT, (k + 1) * DT, None)
        x, _, _ = truth.state()
        xs[k] = x[:, 0].cpu().numpy()
    truth.close()
    return observe(xs, model.sigma_y)


REF_TIMED_LIB = os.path.join(ROOT, "oracle", "_ref", "libbiref_time_f32.so")


def reference_cpu_baseline(y, seconds: float = 20.0):
    """The reference's own host code, compiled from its sources with its own
    optimisation flags (-O3 -funroll-loops, real = float, OpenMP): the loop
    of Filter<BootstrapPF>::filter over its SystematicResampler,
    StaticSamplerHost, RK4IntegratorHost, StaticUpdaterHost and
    SparseStaticLogDensityHost on the hand-rendered Lorenz-96 model class
    (ref_l96_filter_timed), on all host threads, on a bounded sample of the
    workload (the first S steps of the same observations, N = 65536).  Draws
    come from pre-generated tables at the cost of a load each, so the
    reference's random number generation is not counted."""
    import ctypes

    import numpy as np
    from libbi_b200 import configs

    L = ctypes.CDLL(REF_TIMED_LIB)
    f = L.ref_l96_filter_timed
    f.restype = ctypes.c_double
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_double, ctypes.c_double,
                  ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    model = configs.L96_D40_N65536["model"]
    rng = np.random.default_rng(SEED)
    x0 = np.ascontiguousarray(model.F + model.x0_std * rng.standard_normal((N_PARTICLES, DIM)))
    yy = np.ascontiguousarray(np.asarray(y, np.float64).reshape(-1, DIM))
    nrm = rng.standard_normal(1 << 22)
    uni = rng.random(1 << 22)
    threads = os.cpu_count() or 1
    ll = ctypes.c_double()
    p = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731

    def run(S):
        return f(p(x0), N_PARTICLES, S, p(yy), DT, ESS_REL, threads, p(nrm), p(uni), int(nrm.size), ctypes.byref(ll))

    per = run(2) / 2
    S = int(max(2, min(T_OBS, seconds / max(per, 1e-6))))
    el = run(S)
    return {"value": N_PARTICLES * S / el, "unit": UNIT, "cores": threads, "kind": "reference",
            "sample": f"the reference's own host code (its resampler, integrator and updaters compiled from its "
                      f"sources with -O3 -funroll-loops, real = float) in Filter<BootstrapPF>::filter's loop, "
                      f"N={N_PARTICLES}, first {S} of {T_OBS} observation steps, {threads} OpenMP threads, "
                      f"{el:.1f} s; draws from pre-generated tables (generator cost not counted)",
            "log_likelihood": ll.value}


def cpu_baseline(y, seconds: float = 12.0):
    """The timed CPU baseline: the reference's own host code where it was
    compiled here (reference_cpu_baseline), with the oracle's port of the
    reference's CPU filter beside it; the port alone otherwise.  The
    reference runs first, on host cores that have not just run the port at
    full load."""
    if not os.path.exists(REF_TIMED_LIB):
        return port_cpu_baseline(y, seconds)
    ref = reference_cpu_baseline(y, seconds=max(seconds, 20.0))
    ref["port"] = port_cpu_baseline(y, seconds)
    return ref


def omp_threads(n: int):
    """Set the process's OpenMP thread count.  The reference's host code,
    loaded into this process for its timed leg, leaves it at one thread on
    return (its parity entry points run on one thread); the port's parallel
    loops would then run on one thread too."""
    import ctypes

    try:
        ctypes.CDLL("libgomp.so.1").omp_set_num_threads(int(n))
    except OSError:
        pass


def port_cpu_baseline(y, seconds: float = 12.0):
    """The oracle's port of the reference's CPU filter (OpenMP over particles,
    all host threads), on a bounded sample of the same workload."""
    import numpy as np
    from oracle.oracle import Oracle
    from libbi_b200 import configs
    from libbi_b200 import _native as N

    omp_threads(int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1)))
    O = Oracle()
    model = configs.L96_D40_N65536["model"]
    desc = model.desc()
    cfg = N.Config()
    cfg.nparticles = N_PARTICLES
    cfg.resampler = N.BPF_RESAMPLER_SYSTEMATIC
    cfg.ess_rel = ESS_REL
    cfg.seed = SEED
    t = time.perf_counter()
    O.filter(desc, cfg, y[:2].reshape(-1), 2, 0.0, DT)
    per = (time.perf_counter() - t) / 2
    S = int(max(2, min(T_OBS, seconds / max(per, 1e-6))))
    t = time.perf_counter()
    O.filter(desc, cfg, y[:S].reshape(-1), S, 0.0, DT)
    el = time.perf_counter() - t
    threads = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return {"value": N_PARTICLES * S / el, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"oracle port of the reference CPU filter, N={N_PARTICLES}, first {S} of {T_OBS} "
                      f"observation steps (incl. initial draw), {threads} OpenMP threads, {el:.1f} s"}


def large_n_kernels(sizes=(1 << 22, 1 << 24, 1 << 26), reps=5):
    """The memory-bound kernels at working sets beyond L2: log-weight
    reduction (ess_reduce), permuted systematic resampling and the ancestor
    gather (40 FP32 components).  Device time of the kernels from CUDA events
    (for the resampler calls, the events the resampler records around its own
    kernels).  Before every repetition L2 is flushed: 256 MiB written, then
    another 256 MiB read, so that L2 holds none of the kernel's inputs and
    no dirty lines whose write-back the timed kernel would pay for.  Achieved
    GB/s counts algorithmic bytes:
    reduce 8 B, resample 8 + 4 B (log-weight in, ancestor out), gather
    2*40*4 + 4 B per particle."""
    import torch
    from libbi_b200 import SystematicResampler, gather_rows

    hbm, _, _ = peaks()
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    flush_read = torch.ones(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    out = {"l2": "flushed before every repetition: 256 MiB written, then another 256 MiB read"}
    for n in sizes:
        g = torch.Generator(device="cuda")
        g.manual_seed(n)
        lw = torch.randn(n, dtype=torch.float64, device="cuda", generator=g) * 2.0
        a = torch.full((1,), 0.37, dtype=torch.float64, device="cuda")
        R = SystematicResampler(max_n=n)
        ld = (n + 31) // 32 * 32
        X = torch.randn((DIM, ld), dtype=torch.float32, device="cuda", generator=g)
        Y = torch.empty_like(X)
        as_ = R.ancestors(lw, a, permute=True)

        def timed(fn, kernel_only):
            # kernel_only: the resampler's own events around its kernels
            # (the call's status reset and read-back excluded); otherwise
            # events around the whole call, which enqueues one kernel
            ts = []
            for _ in range(reps):
                flush.zero_()
                flush_read.sum()
                s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                R.timing_read(reset=True)
                s0.record()
                fn()
                s1.record()
                torch.cuda.synchronize()
                ms, calls = R.timing_read(reset=True)
                ts.append(ms / calls / 1e3 if kernel_only else s0.elapsed_time(s1) / 1e3)
            return min(ts)

        R.timing(True)
        t_red = timed(lambda: R.reduce(lw), True)
        t_res = timed(lambda: R.ancestors(lw, a, permute=True), True)
        t_gat = timed(lambda: gather_rows(as_, X, Y, DIM, ld), False)
        R.timing(False)
        rows = {}
        for name, t, byt in (("ess_reduce", t_red, 8 * n), ("systematic_resample", t_res, 12 * n),
                             ("gather_rows_d40", t_gat, (2 * DIM * 4 + 4) * n)):
            gbs = byt / t / 1e9
            rows[name] = {"ms": t * 1e3, "GB/s": gbs, "frac_hbm": gbs / hbm}
        out[str(n)] = rows
        R.close()
        del lw, X, Y, as_
        torch.cuda.empty_cache()
    return out


def batched_workload(rng_seed=3, nf=256, T=100):
    """256 independent Lorenz-96 d = 40 filters: forcing F_i ~ U(6, 10),
    particle counts log-uniform in [512, 32768] rounded to 32, seeds
    1000 + i, systematic resampling for even i and multinomial for odd i,
    T = 100 observations of all 40 components every 0.05 with N(0, 1) noise."""
    import numpy as np
    from libbi_b200 import ModelL96

    rng = np.random.default_rng(rng_seed)
    Fs = rng.uniform(6.0, 10.0, nf)
    ns = np.floor(np.exp(rng.uniform(np.log(512), np.log(32768), nf))).astype(int)
    ns = np.clip((ns + 31) // 32 * 32, 512, 32768)
    models = [ModelL96(dim=DIM, F=float(F)) for F in Fs]
    res = ["systematic" if i % 2 == 0 else "multinomial" for i in range(nf)]
    seeds = [1000 + i for i in range(nf)]
    return models, [int(n) for n in ns], res, seeds, T


def batched_truth(models, T, seed0=5000):
    """Each filter's synthetic observations: one run of its own model (the
    library's transition and noise, N = 1, seed seed0 + i) observed with
    N(0, sigma_y^2) noise."""
    import numpy as np
    from libbi_b200 import BatchedBootstrapPF

    nf = len(models)
    truth = BatchedBootstrapPF(models, [1] * nf, "systematic", [seed0 + i for i in range(nf)])
    xs = np.zeros((T, nf, DIM), np.float32)
    for k in range(T):
        truth.step_device(k * DT, (k + 1) * DT, None)
        x, _, _, offs = truth.state()
        xs[k] = x[:, offs.tolist()].cpu().numpy().T
    truth.close()
    return observe(xs.reshape(T * nf, DIM), models[0].sigma_y).reshape(T, nf, DIM)


def batched_filters(runs=5):
    """The batched workload through bpf_filter_batch: device time of the
    captured init + T steps (CUDA events around the graph launch), and end to
    end (observations uploaded from host memory, log-likelihoods and
    increments read back) by the host clock.  The state (2 x 40 x sum N x 4 B,
    ~640 MB) exceeds L2, so no flush is needed between runs."""
    import numpy as np
    from libbi_b200 import BatchedBootstrapPF

    models, ns, res, seeds, T = batched_workload()
    y = batched_truth(models, T)
    b = BatchedBootstrapPF(models, ns, res, seeds, ess_rel=ESS_REL)
    rs_threads, rs_us = b.resample_threads()  # autotuned at create
    b.filter(y, 0.0, DT)  # capture the graph
    b.timing(True)
    b.timing_read(reset=True)
    walls = []
    for _ in range(runs):
        t0 = time.perf_counter()
        ll, inc, ess, st = b.filter(y, 0.0, DT)
        walls.append(time.perf_counter() - t0)
    ms, steps = b.timing_read(reset=True)
    b.close()
    total = int(np.sum(ns))
    dev_s = ms / 1e3 / runs
    hbm, how, _ = peaks()
    # algorithmic bytes per particle-step of the transition (+ resample
    # bytes on resample steps are not counted)
    bps = TRANSITION_BYTES_PER_PARTICLE * total * T / dev_s / 1e9
    return {
        "workload": "l96_d40_256filters_n512_32768_loguniform_t100",
        "autotuned_resample_threads": rs_threads,
        "resample_tuning_us": {str(k): v for k, v in rs_us.items()},
        "filters": len(ns), "total_particles": total, "T": T, "runs": runs,
        "particle_steps_per_s": total * T / dev_s,
        "ms_per_filter_run": dev_s * 1e3,
        "e2e_particle_steps_per_s": total * T / float(np.median(walls)),
        "e2e_ms_per_filter_run": float(np.median(walls)) * 1e3,
        "h2d_bytes_per_run": int(y.size * 4), "d2h_bytes_per_run": int(3 * T * len(ns) * 8),
        "degenerate_filters": int(np.sum(st != 0)),
        "gpu_launches_per_run": 1 + 2 * T,
        "roofline": {"bound": "hbm", "achieved": bps, "peak": hbm, "unit": "GB/s", "frac": bps / hbm,
                     "peak_source": how, "bytes": "336 B per particle-step (transition state + log-weight)"},
        "l2": "state larger than L2 (~640 MB), no flush",
    }


REF_TIMED_PZ_LIB = os.path.join(ROOT, "oracle", "_ref", "libbiref_time_pz.so")


def pz_c1(n=4096, T=100, runs=20):
    """The plankton configuration (C1): one PZ filter of 4096 FP64 particles,
    RK4(3) with h0 = 0.1 and tolerances 1e-3, the growth rate's log-normal
    noise redrawn each day, observations log P + N(0, 0.2^2) daily for
    T = 100 from one seeded model run (seed 1, P0, Z0 ~ LogN(ln 2, 0.2^2)),
    systematic resampling at every step (essRel = 1, strict <).  Device time
    of the filter's kernels per run (the handle's events around each step's
    kernels) and end to end through bpf_filter (host wall clock: the
    observations' upload, the initial draw, T steps, the results read
    back); beside them the reference's own host code on the same workload
    (ref_pz_filter_timed: its SystematicResampler, StaticSamplerHost,
    RK43IntegratorHost and SparseStaticLogDensityHost in
    Filter<BootstrapPF>::filter's loop, real = double, -O3 -funroll-loops,
    all host threads; draws from pre-generated tables)."""
    import ctypes

    import numpy as np
    import torch
    from libbi_b200 import BootstrapPF, ModelPZ

    model = ModelPZ()
    truth = BootstrapPF(model, 1, seed=1)
    ps = np.zeros(T)
    for k in range(T):
        truth.step(float(k), float(k + 1), None)
        x, _, _ = truth.state()
        ps[k] = float(x[0, 0].item())
    truth.close()
    y = (np.log(ps) + model.sigma_y * np.random.default_rng(1).standard_normal(T)).astype(np.float64)
    pf = BootstrapPF(model, n, resampler="systematic", ess_rel=1.0, seed=1)
    for _ in range(2):
        pf.filter(y, 0.0, 1.0)  # warm-up: the second call captures the steps as a CUDA graph
    pf.timing(True)
    pf.timing_read(reset=True)
    for _ in range(runs):
        pf.filter(y, 0.0, 1.0)
    r_ms, t_ms, steps = pf.timing_read(reset=True)
    pf.timing(False)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(runs):
        ll, _, _ = pf.filter(y, 0.0, 1.0)
    wall = (time.perf_counter() - t0) / runs
    pf.close()
    dev_ms = (r_ms + t_ms) / runs
    out = {"workload": f"pz_n{n}_t{T}_fp64_rk43_systematic_every_step", "nparticles": n, "T": T, "runs": runs,
           "particle_steps_per_s": n * T / (dev_ms * 1e-3), "ms_per_filter_run": dev_ms,
           "e2e_particle_steps_per_s": n * T / wall, "e2e_ms_per_filter_run": wall * 1e3,
           "log_likelihood": ll, "timer": "device: the handle's CUDA events around each step's kernels, summed; "
                                        "e2e: host wall clock around bpf_filter"}
    if os.path.exists(REF_TIMED_PZ_LIB):
        L = ctypes.CDLL(REF_TIMED_PZ_LIB)
        f = L.ref_pz_filter_timed
        f.restype = ctypes.c_double
        f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_double,
                      ctypes.c_double, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                      ctypes.POINTER(ctypes.c_double)]
        rng = np.random.default_rng(1)
        x0 = np.ascontiguousarray(np.exp(np.log(2.0) + 0.2 * rng.standard_normal((n, 2))))
        nrm = rng.standard_normal(1 << 20)
        uni = rng.random(1 << 20)
        threads = os.cpu_count() or 1
        rl = ctypes.c_double()
        p = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
        secs = f(p(x0), n, T, p(y), 1.0, 1.0, threads, p(nrm), p(uni), int(nrm.size), ctypes.byref(rl))
        out["cpu_reference"] = {"particle_steps_per_s": n * T / secs, "seconds": secs, "cores": threads,
                                "log_likelihood": rl.value,
                                "what": "the reference's own host code for this configuration, all T steps"}
    return out


def step_forms(y_dev, steps=300, warmup=5):
    """The headline workload in both forms of the step, one after the other
    on the same observations and seed: two launches per step (the one-launch
    resampler, then the transition as its programmatic dependent; the
    default) and one (the systematic resampling as the prologue of the step
    kernel).  CUDA events around each step, L2 flushed before each; the two
    forms compute the same log-weights bit for bit."""
    import torch
    from libbi_b200 import BootstrapPF, configs

    model = configs.L96_D40_N65536["model"]
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    out = {}
    lws = {}
    from libbi_b200 import BpfError

    for name, fused in (("two_launch", False), ("one_launch", True)):
        pf = BootstrapPF(model, N_PARTICLES, resampler="systematic", ess_rel=ESS_REL, seed=SEED)
        try:
            pf.set_step_form(fused)
        except BpfError as e:  # the GPU cannot hold every block of the step at once
            pf.close()
            out[name] = {"unavailable": str(e)}
            continue
        k = 0
        ms = []
        for i in range(warmup + steps):
            if k >= T_OBS:
                pf.init()
                k = 0
            k += 1
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            pf.step_device((k - 1) * DT, k * DT, y_dev[k - 1], sync=False)
            b.record()
            if i >= warmup:
                ms.append((a, b))
        torch.cuda.synchronize()
        t = sum(a.elapsed_time(b) for a, b in ms) / steps
        _, lw, _ = pf.state()
        lws[name] = lw.cpu().numpy().tobytes()
        pf.close()
        out[name] = {"ms_per_step": t, "particle_steps_per_s": N_PARTICLES / (t * 1e-3),
                     "launches_per_step": LAUNCHES_PER_STEP[fused]}
    if len(lws) == 2:
        out["same_log_weights_bitwise"] = lws["one_launch"] == lws["two_launch"]
    out["timer"] = f"CUDA events around each of {steps} steps after {warmup} warm-up, L2 flushed before each"
    return out


def pmmh_chains(iterations=2000, nchains=128, n_lo=1024, n_hi=8192, T=100, checks=0.01, guided=True):
    """Particle-marginal Metropolis-Hastings on the plankton model: 128
    chains over (c, e, m, q) with priors c, e ~ U(0, 1), m, q ~
    LogN(ln 0.1, 0.5^2), Gaussian random walk of 0.02 per coordinate; every
    iteration filters all chains' proposals as one batch (each chain's
    filter of N particles, N log-uniform in [1024, 8192] rounded to 32,
    systematic resampling every step) over T = 100 daily observations
    log P + N(0, 0.2^2) of one seeded model run (seed 4).  All `iterations`
    are timed (host clock around bpf_pmmh_run).  Then, on 1% of the
    iterations, one accepted proposal's log-likelihood is recomputed by an
    independent single FP64 filter with the chain's particle count, seed and
    parameters, which must reproduce the batched value."""
    import math

    import numpy as np
    from libbi_b200 import BootstrapPF, MarginalMH, ModelPZ, Prior

    model = ModelPZ()
    truth = BootstrapPF(model, 1, seed=4)
    ps = np.zeros(T)
    for k in range(T):
        truth.step(float(k), float(k + 1), None)
        x, _, _ = truth.state()
        ps[k] = float(x[0, 0].item())
    truth.close()
    rng = np.random.default_rng(4)
    y = (np.log(ps) + model.sigma_y * rng.standard_normal(T)).astype(np.float64)
    ns = np.floor(np.exp(rng.uniform(np.log(n_lo), np.log(n_hi), nchains))).astype(int)
    ns = np.clip((ns + 31) // 32 * 32, n_lo, n_hi)
    priors = [Prior(0, "uniform", 0.0, 1.0, 0.02), Prior(1, "uniform", 0.0, 1.0, 0.02),
              Prior(2, "log_normal", math.log(0.1), 0.5, 0.02), Prior(3, "log_normal", math.log(0.1), 0.5, 0.02)]
    seed = 4
    mh = MarginalMH(model, priors, y, 0.0, 1.0, nchains=nchains, nparticles=ns, resampler="systematic",
                    ess_rel=1.0, seed=seed)
    mh.run(2)  # graph capture and warm-up
    _, _, _, r0 = mh.state()
    t0 = time.perf_counter()
    out = mh.run(iterations)
    wall = time.perf_counter() - t0
    mh.close()
    acc = (out["accepted"] - 1) / (iterations + 2)
    # FP64 replays of accepted proposals (the sample after an accepted move
    # is the proposal; the filter of run r, chain c has seed seed + 1 + r C + c)
    smp, pll = out["samples"], out["proposal_loglik"]
    step = max(1, int(round(1.0 / checks)))
    errs = []
    for i0 in range(0, iterations, step):
        for i in range(max(i0, 1), min(i0 + step, iterations)):
            # chains that accepted at iteration i: their state changed
            hit = [c for c in range(nchains) if np.isfinite(pll[i, c]) and not np.array_equal(smp[i, c], smp[i - 1, c])]
            if hit:
                c = hit[0]
                th = smp[i, c]
                pf = BootstrapPF(ModelPZ(c=th[0], e=th[1], m=th[2], q=th[3]), int(ns[c]), resampler="systematic",
                                 ess_rel=1.0, seed=seed + 1 + (r0 + i) * nchains + c)
                ll, _, _ = pf.filter(y, 0.0, 1.0)
                pf.close()
                errs.append(abs(ll - pll[i, c]) / max(abs(pll[i, c]), 1.0))
                break
    errs = np.array(errs)
    particles = int(ns.sum())
    out = {
        "workload": f"pz_pmmh_{nchains}chains_n{n_lo}_{n_hi}_loguniform_t{T}",
        "chains": nchains, "nparticles_min": int(ns.min()), "nparticles_max": int(ns.max()),
        "nparticles_total": particles, "T": T, "iterations_timed": iterations,
        "seconds": wall, "iterations_per_s": iterations / wall,
        "particle_steps_per_s": particles * T * iterations / wall,
        "mean_acceptance": float(np.mean(acc)),
        "fp64_replay_checks": {"count": int(errs.size), "max_rel_err": float(errs.max()) if errs.size else None,
                               "what": "accepted proposals on 1% of the iterations, refiltered by a single FP64 "
                                       "filter with the chain's N, seed and parameters"},
        "timer": "host wall clock around bpf_pmmh_run",
    }
    if guided:
        out["guided"] = pmmh_guided(model, priors, y, ns, seed, iterations, nchains, checks)
    return out


def pmmh_guided(model, priors, y, ns, seed, iterations, nchains, checks, train_steps=1500):
    """The same chains (priors, observations, particle counts, seeds) with
    every filter guided by the learned proposal over the log-noise: the
    network (3 -> 128 -> 128 -> 2, BF16 tensor cores) trained for
    `train_steps` Adam steps on rows simulated from 65536 states of 20
    unobserved days of the model (training timed apart), then all
    `iterations` timed.  On 1% of the iterations an accepted proposal is
    refiltered by a one-filter guided batch with the chain's N, seed and
    parameters, which must reproduce the value.  The log-likelihood spread
    of 32 filters at the true parameters (N = 2048) is reported for both
    filters: the quantity a proposal is meant to cut."""
    import numpy as np
    import torch
    from libbi_b200 import BatchedBootstrapPF, BootstrapPF, LearnedProposal, MarginalMH, ModelPZ

    T = len(y)
    sim = BootstrapPF(model, 1 << 16, seed=9)
    for k in range(20):
        sim.step(float(k), float(k + 1), None)
    x, _, _ = sim.state()
    xt = x[:, :1 << 16].T.contiguous().clone()
    sim.close()
    prop = LearnedProposal(model, 1.0, max_batch=4096, seed=6)
    prop.set_states(xt)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    trace = prop.train(train_steps, 4096, 2e-3)
    train_s = time.perf_counter() - t0
    mh = MarginalMH(model, priors, y, 0.0, 1.0, nchains=nchains, nparticles=ns, resampler="systematic",
                    ess_rel=1.0, seed=seed)
    mh.set_proposal(prop)
    mh.run(2)
    _, _, _, r0 = mh.state()
    t0 = time.perf_counter()
    out = mh.run(iterations)
    wall = time.perf_counter() - t0
    mh.close()
    acc = (out["accepted"] - 1) / (iterations + 2)
    smp, pll = out["samples"], out["proposal_loglik"]
    step = max(1, int(round(1.0 / checks)))
    errs = []
    for i0 in range(0, iterations, step):
        for i in range(max(i0, 1), min(i0 + step, iterations)):
            hit = [c for c in range(nchains) if np.isfinite(pll[i, c]) and not np.array_equal(smp[i, c], smp[i - 1, c])]
            if hit:
                c = hit[0]
                th = smp[i, c]
                b = BatchedBootstrapPF([ModelPZ(c=th[0], e=th[1], m=th[2], q=th[3])], [int(ns[c])], "systematic",
                                       [seed + 1 + (r0 + i) * nchains + c], ess_rel=1.0)
                b.set_proposal(prop)
                ll, _, _, _ = b.filter(np.asarray(y, np.float64).reshape(T, 1, 1), 0.0, 1.0)
                b.close()
                errs.append(abs(ll[0] - pll[i, c]) / max(abs(pll[i, c]), 1.0))
                break
    errs = np.array(errs)
    spread = {}
    for name, p in (("bootstrap", None), ("guided", prop)):
        b = BatchedBootstrapPF([model] * 32, [2048] * 32, "systematic", list(range(900, 932)), ess_rel=1.0)
        if p is not None:
            b.set_proposal(p)
        ll, _, _, _ = b.filter(np.repeat(np.asarray(y, np.float64).reshape(T, 1, 1), 32, axis=1), 0.0, 1.0)
        b.close()
        spread[name] = float(np.std(ll, ddof=1))
    prop.close()
    particles = int(np.sum(ns))
    return {
        "train_seconds": train_s, "train_steps": train_steps,
        "train_loss_first_last": [float(trace[:10].mean()), float(trace[-50:].mean())],
        "seconds": wall, "iterations_per_s": iterations / wall,
        "particle_steps_per_s": particles * T * iterations / wall,
        "mean_acceptance": float(np.mean(acc)),
        "replay_checks": {"count": int(errs.size), "max_rel_err": float(errs.max()) if errs.size else None,
                          "what": "accepted proposals on 1% of the iterations, refiltered by a one-filter guided "
                                  "batch with the chain's N, seed and parameters"},
        "ll_sd_32_filters_n2048_true_theta": spread,
        "timer": "host wall clock around bpf_pmmh_run",
    }


def precision_check(y_host, seeds=16, n=N_PARTICLES, T=T_OBS, same_input_seeds=4):
    """The FP32 filter against the FP64 filter on the same seeds (identical
    Philox draws, so the two differ by rounding only), on the bench's
    Lorenz-96 workload.

    Along a run: per step the relative error of the FP32 filter's
    log-likelihood increment against the FP64 filter's (relative to
    max(|inc64|, 1)) and of the cumulative log-likelihood; the fraction of
    steps within 1e-4; whether the two estimators' means over the seeds agree
    within two standard errors.

    From the same input, at EVERY step of the first `same_input_seeds` FP64
    runs: the FP64 run's state and log-weights before the step are written
    into an FP32 and an FP64 probe filter (same seed, so the same draws),
    each takes that one step, and the increments are compared (relative to
    the step's own increment, max(|inc64 - lW_in|, 1)).  This is the
    arithmetic error of one step.  Every step whose along-run error exceeds
    1e-4 in those runs is then classified: "inputs diverged" when the
    same-input error at that step is within 1e-4 (the FP32 run's particles
    had already parted from the FP64 run's: a resampling integer decided by
    a rounding tie, then Lorenz-96's chaos), "arithmetic" otherwise."""
    import numpy as np
    import torch
    from dataclasses import replace
    from libbi_b200 import BootstrapPF, configs

    m32 = configs.L96_D40_N65536["model"]
    m64 = replace(m32, precision="f64")
    y32 = np.asarray(y_host[:T], np.float32)
    y64 = y32.astype(np.float64)  # the same observed values in both precisions
    inc_e, cum_e, ll32, ll64, same_e = [], [], [], [], []
    for s in range(seeds):
        seed = 20_000 + s
        pf32 = BootstrapPF(m32, n, resampler="systematic", ess_rel=ESS_REL, seed=seed)
        l32, i32, _ = pf32.filter(y32, 0.0, DT)
        pf32.close()
        ref = BootstrapPF(m64, n, resampler="systematic", ess_rel=ESS_REL, seed=seed)
        if s < same_input_seeds:
            probes = [BootstrapPF(m, n, resampler="systematic", ess_rel=ESS_REL, seed=40_000 + s)
                      for m in (m32, m64)]
            i64, errs = np.zeros(T), np.zeros(T)
            for k in range(T):
                x, lw, _ = ref.state()
                lw_in = float(torch.logsumexp(lw, 0)) - np.log(n)
                incs = []
                for pr, y in zip(probes, (y32, y64)):
                    pr.init()
                    xv, lwv, _ = pr.state()
                    xv[:, :n].copy_(x[:, :n].to(xv.dtype))
                    lwv.copy_(lw)
                    incs.append(pr.step(k * DT, (k + 1) * DT, y[k]).log_increment)
                errs[k] = abs(incs[0] - incs[1]) / max(abs(incs[1] - lw_in), 1.0)
                i64[k] = ref.step(k * DT, (k + 1) * DT, y64[k]).log_increment
            l64 = float(torch.logsumexp(ref.state()[1], 0)) - np.log(n)
            for pr in probes:
                pr.close()
            same_e.append(errs)
        else:
            l64, i64, _ = ref.filter(y64, 0.0, DT)
        ref.close()
        inc_e.append(np.abs(i32 - i64) / np.maximum(np.abs(i64), 1.0))
        c32, c64 = np.cumsum(i32), np.cumsum(i64)
        cum_e.append(np.abs(c32 - c64) / np.maximum(np.abs(c64), 1.0))
        ll32.append(l32)
        ll64.append(l64)
    inc_e, cum_e, same_e = np.array(inc_e), np.array(cum_e), np.array(same_e)
    ll32, ll64 = np.array(ll32), np.array(ll64)
    se = float(np.sqrt(ll32.var(ddof=1) / seeds + ll64.var(ddof=1) / seeds))
    within = cum_e.max(axis=0) <= 1e-4
    first_bad = int(np.argmin(within)) + 1 if not within.all() else None
    beyond = inc_e[:same_input_seeds] > 1e-4
    diverged = int(np.sum(beyond & (same_e <= 1e-4)))
    arithmetic = int(np.sum(beyond & (same_e > 1e-4)))
    return {
        "workload": f"l96_d40_n{n}_t{T}_fp32_vs_fp64_{seeds}seeds",
        "increment_rel_err": {"median": float(np.median(inc_e)), "max": float(inc_e.max()),
                              "max_first_20_steps": float(inc_e[:, :20].max())},
        "loglik_rel_err": {"median": float(np.median(cum_e)), "max": float(cum_e.max()),
                           "final_median": float(np.median(cum_e[:, -1]))},
        "steps_within_1e-4": float(within.mean()),
        "first_step_beyond_1e-4": first_bad,
        "mean_ll_fp32": float(ll32.mean()), "mean_ll_fp64": float(ll64.mean()),
        "mean_diff_in_standard_errors": float(abs(ll32.mean() - ll64.mean()) / se) if se > 0 else 0.0,
        "means_within_2_se": bool(abs(ll32.mean() - ll64.mean()) <= 2 * se),
        "same_input_every_step": {
            "seeds": same_input_seeds, "steps": T, "median_rel_err": float(np.median(same_e)),
            "max_rel_err": float(same_e.max()), "within_1e-4": bool(same_e.max() <= 1e-4)},
        "steps_beyond_1e-4_along_run": {
            "seeds": same_input_seeds, "count": int(beyond.sum()), "inputs_diverged": diverged,
            "arithmetic": arithmetic},
    }


def batched_precision(T=100):
    """The batched workload (256 Lorenz-96 filters) in FP32 against the same
    256 filters in FP64 on the same seeds and observations: per-filter
    log-likelihood relative error, per-step increment errors, and the paired
    difference of the estimates (FP32 minus FP64) in standard errors of its
    mean over the filters."""
    import numpy as np
    from dataclasses import replace
    from libbi_b200 import BatchedBootstrapPF

    models, ns, res, seeds, T = batched_workload(T=T)
    y = batched_truth(models, T)
    out = {}
    for prec in ("f32", "f64"):
        ms = [replace(m, precision=prec) for m in models]
        b = BatchedBootstrapPF(ms, ns, res, seeds, ess_rel=ESS_REL)
        yy = y if prec == "f32" else y.astype(np.float64)
        ll, inc, _, st = b.filter(yy, 0.0, DT)
        b.close()
        out[prec] = (ll, inc, st)
    (l32, i32, s32), (l64, i64, s64) = out["f32"], out["f64"]
    ok = (s32 == 0) & (s64 == 0)
    rel = np.abs(l32 - l64) / np.maximum(np.abs(l64), 1.0)
    inc_e = np.abs(i32 - i64) / np.maximum(np.abs(i64), 1.0)
    d = (l32 - l64)[ok]
    se = float(d.std(ddof=1) / np.sqrt(d.size)) if d.size > 1 else 0.0
    return {
        "workload": "l96_d40_256filters_fp32_vs_fp64_t100",
        "filters": int(ok.sum()),
        "loglik_rel_err": {"median": float(np.median(rel[ok])), "max": float(rel[ok].max())},
        "increment_rel_err": {"median": float(np.median(inc_e[:, ok])), "max": float(inc_e[:, ok].max()),
                              "steps_within_1e-4": float(np.mean(inc_e[:, ok] <= 1e-4))},
        "mean_paired_diff": float(d.mean()), "paired_diff_se": se,
        "mean_diff_in_standard_errors": float(abs(d.mean()) / se) if se > 0 else 0.0,
        "means_within_2_se": bool(abs(d.mean()) <= 2 * se),
    }


def equal_mean_time(boot, ll_target):
    """Device time per run of a bootstrap filter whose mean log-likelihood
    equals ll_target, interpolated linearly in log N between the two
    bracketing sweep points (mean LL and log time both linear in log N);
    (time, N, exact) with exact False and the nearest end point's time when
    ll_target lies outside the sweep (a bound, not a measurement)."""
    import numpy as np

    pts = sorted(boot, key=lambda b: b["n"])
    for a, b in zip(pts[:-1], pts[1:]):
        lo, hi = a["ll_mean"], b["ll_mean"]
        if lo <= ll_target <= hi and hi > lo:
            f = (ll_target - lo) / (hi - lo)
            n = float(np.exp(np.log(a["n"]) + f * (np.log(b["n"]) - np.log(a["n"]))))
            t = float(np.exp(np.log(a["ms_per_run"]) + f * (np.log(b["ms_per_run"]) - np.log(a["ms_per_run"]))))
            return t, n, True
    if ll_target < pts[0]["ll_mean"]:
        return pts[0]["ms_per_run"], float(pts[0]["n"]), False
    return pts[-1]["ms_per_run"], float(pts[-1]["n"]), False


def strip_lls(x):
    """The per-seed log-likelihoods (kept for the standard errors) left out
    of the printed line."""
    if isinstance(x, list):
        return [strip_lls(v) for v in x]
    if isinstance(x, dict):
        return {k: strip_lls(v) for k, v in x.items() if k != "_lls"}
    return x


def equal_sd_ratios(boot, guided, reps=400):
    """Batched against batched, equal deviation: the bootstrap rows
    (N_i, sd_i, t_i) give log sd = a + b log N (least squares) and a device
    time per particle (their mean of t_i / N_i); the bootstrap N that reaches
    a guided row's sd is exp((log sd_g - a) / b), its time that N times the
    per-particle time, and the ratio that time over the guided row's time.
    Standard errors by resampling the seeds (the per-seed log-likelihoods of
    every row, with replacement, `reps` times)."""
    import numpy as np

    rng = np.random.default_rng(17)
    ln_n = np.log([b["n"] for b in boot])
    per_particle = float(np.mean([b["ms_per_run"] / b["n"] for b in boot]))

    def ratios(bsd, gsd):
        slope, icpt = np.polyfit(ln_n, np.log(bsd), 1)
        out = []
        for gd, sd in zip(guided, gsd):
            if slope >= 0:
                out.append((float("nan"), float("nan")))
                continue
            n_eq = float(np.exp((np.log(sd) - icpt) / slope))
            out.append((n_eq, n_eq * per_particle / gd["ms_per_run"]))
        return slope, out

    bsd = [b["ll_sd"] for b in boot]
    gsd = [g["ll_sd"] for g in guided]
    slope, point = ratios(bsd, gsd)
    reps_r = []
    for _ in range(reps):
        rb = [np.std(rng.choice(b["_lls"], b["_lls"].size), ddof=1) for b in boot]
        rg = [np.std(rng.choice(g["_lls"], g["_lls"].size), ddof=1) for g in guided]
        reps_r.append([r for _, r in ratios(rb, rg)[1]])
    reps_r = np.array(reps_r)
    rows = []
    lo_n, hi_n = min(b["n"] for b in boot), max(b["n"] for b in boot)
    b_hi = max(boot, key=lambda b: b["n"])
    b_lo = min(boot, key=lambda b: b["n"])
    for k, gd in enumerate(guided):
        n_eq, r = point[k]
        col = reps_r[:, k]
        col = col[np.isfinite(col)]
        row = {"guided_n": gd["n"], "guided_ll_sd": gd["ll_sd"], "guided_ms_per_run": gd["ms_per_run"]}
        if np.isfinite(n_eq) and lo_n <= n_eq <= hi_n:
            row.update({"bootstrap_n_at_equal_sd": n_eq, "gpu_time_ratio_bootstrap_over_guided": r,
                        "ratio_se": float(col.std(ddof=1)) if col.size > 1 else None, "ratio_is": "interpolated"})
        elif np.isfinite(n_eq) and n_eq > hi_n:
            # the bootstrap filter at its largest N still deviates more: its
            # time there bounds the ratio from below
            row.update({"bootstrap_n_at_equal_sd": None,
                        "gpu_time_ratio_bootstrap_over_guided": b_hi["ms_per_run"] / gd["ms_per_run"],
                        "ratio_se": None,
                        "ratio_is": f"lower bound: the bootstrap filter at N = {b_hi['n']} still deviates more "
                                    f"({b_hi['ll_sd']:.4g} against {gd['ll_sd']:.4g})"})
        elif np.isfinite(n_eq):
            row.update({"bootstrap_n_at_equal_sd": None,
                        "gpu_time_ratio_bootstrap_over_guided": b_lo["ms_per_run"] / gd["ms_per_run"],
                        "ratio_se": None,
                        "ratio_is": f"upper bound: the bootstrap filter at N = {b_lo['n']} already deviates less "
                                    f"({b_lo['ll_sd']:.4g} against {gd['ll_sd']:.4g})"})
        else:
            row.update({"bootstrap_n_at_equal_sd": None, "gpu_time_ratio_bootstrap_over_guided": None,
                        "ratio_se": None, "ratio_is": "undefined: the bootstrap deviation does not fall with N"})
        rows.append(row)
    finite = [x for x in rows if x["gpu_time_ratio_bootstrap_over_guided"] is not None
              and not x["ratio_is"].startswith("upper")]
    best = max(finite or rows, key=lambda x: x["gpu_time_ratio_bootstrap_over_guided"] or -1.0)
    ratio = best["gpu_time_ratio_bootstrap_over_guided"]
    return {"bootstrap_sd_exponent_in_n": float(slope), "bootstrap_ms_per_particle": per_particle, "rows": rows,
            "best_ratio": ratio, "best_ratio_se": best["ratio_se"], "best_ratio_is": best["ratio_is"],
            "best_guided_n": best["guided_n"],
            "meets_10x": bool(ratio is not None and ratio >= 10.0 and not best["ratio_is"].startswith("upper"))}


def guided_informative(seeds=64, T=10, train_steps=1500, n_data=1 << 18, sigma_eta=0.5, sigma_y=0.1,
                       n_boot=(4096, 16384, 32768), n_guided=(256, 1024, 4096)):
    """Both arms batched on Lorenz-96 d=40 with more informative
    observations than the C4 model's (sigma_eta against sigma_y; at 0.5
    against 0.1 the transition scatters the particles far wider than the
    observation pins the state): a proposal trained for this model on 2^18
    simulated triples, T = 10 observations of one seeded run, 64 seeds per
    row, equal-deviation device time ratios with standard errors
    (equal_sd_ratios)."""
    import numpy as np
    import torch
    from dataclasses import replace
    from libbi_b200 import BatchedBootstrapPF, BootstrapPF, LearnedProposal, configs

    model = replace(configs.L96_D40_N65536["model"], sigma_eta=sigma_eta, sigma_y=sigma_y)
    sim = BootstrapPF(model, n_data, seed=5)
    for k in range(40):
        sim.step_device(k * DT, (k + 1) * DT, None, sync=False)
    x, _, _ = sim.state()
    xt = x[:, :n_data].T.contiguous().clone()
    sim.step_device(40 * DT, 41 * DT, None, sync=False)
    x, _, _ = sim.state()
    xt1 = x[:, :n_data].T.contiguous().clone()
    g = torch.Generator(device="cuda")
    g.manual_seed(5)
    yt1 = (xt1 + model.sigma_y * torch.randn(xt1.shape, generator=g, device="cuda")).contiguous()
    sim.close()
    prop = LearnedProposal(model, DT, max_batch=8192, seed=5)
    prop.set_data(xt, xt1, yt1)
    trace = prop.train(train_steps, 8192, 2e-3)
    del xt, xt1, yt1
    truth = BootstrapPF(model, 1, seed=77)
    xs = np.zeros((T, DIM), np.float32)
    for k in range(T):
        truth.step(k * DT, (k + 1) * DT, None)
        x, _, _ = truth.state()
        xs[k] = x[:, 0].cpu().numpy()
    truth.close()
    y = (xs + model.sigma_y * np.random.default_rng(78).standard_normal(xs.shape)).astype(np.float32)

    def run_batched(n, use_prop):
        b = BatchedBootstrapPF([model] * seeds, [n] * seeds, "systematic", [20_000 + s for s in range(seeds)],
                               ess_rel=ESS_REL)
        if use_prop:
            b.set_proposal(prop)
        yb = np.ascontiguousarray(np.repeat(y[:, None, :], seeds, axis=1))
        b.filter(yb, 0.0, DT)  # capture
        b.timing(True)
        b.timing_read(reset=True)
        lls, _, _, st = b.filter(yb, 0.0, DT)
        ms, _ = b.timing_read(reset=True)
        b.close()
        return {"n": n, "filters": seeds, "ll_mean": float(lls.mean()), "ll_sd": float(lls.std(ddof=1)),
                "ms_per_run": ms / seeds, "failed": int((st != 0).sum()), "_lls": lls}

    boot = [run_batched(n, False) for n in n_boot]
    guided = [run_batched(n, True) for n in n_guided]
    prop.close()
    return {"model": {"sigma_eta": model.sigma_eta, "sigma_y": model.sigma_y, "T": T},
            "train": {"triples": n_data, "steps": train_steps, "loss_first": float(trace[:10].mean()),
                      "loss_last": float(trace[-50:].mean())},
            "bootstrap": strip_lls(boot), "guided": strip_lls(guided), "equal_sd": equal_sd_ratios(boot, guided)}


def guided_vs_bootstrap(y_host, seeds=64, n_guided=(4096, 16384, 65536),
                        n_boot=(16384, 65536, 262144, 1 << 20, 1 << 22), n_ref=65536, n_data=1 << 20,
                        train_steps=3000, n_guided_batched=(1024, 4096, 16384), n_boot_batched=(16384, 32768)):
    """The learned proposal on the Lorenz-96 workload: trained on 2^20
    (x_t, x_{t+1}, y_{t+1}) triples simulated by the model (2^20 particles
    spun up for 100 intervals from the initial distribution, one more
    interval, observations with the model's observation noise), then guided
    filters at several N against bootstrap filters at several N on the
    bench's T = 200 observations over 64 seeds each: standard deviation of
    the log-likelihood estimate and device time per filter run (CUDA events
    around each step's kernels).  Monte Carlo variance falls as 1/N, so a
    guided filter with (t_g, sd_g) reaches the deviation sd_b of the
    bootstrap filter at N = n_ref in t_g * (sd_g / sd_b)^2; the bootstrap
    sweep's measured exponent of sd against N checks that premise.  Where
    the filters have lost the track (the deviation flat in N) the
    estimator's downward bias is what more particles buy; the second
    comparison is the device time at which the bootstrap sweep reaches each
    guided filter's mean log-likelihood.  The batched rows run the same
    seeds as one batch of filters (guided: the fused guided step over every
    filter's tiles), with the device time per filter; the bootstrap filters
    the guided ones are matched against need hundreds of thousands of
    particles, beyond a batch's per-filter limit, and are timed singly (at
    those sizes a single filter already fills the GPU)."""
    import numpy as np
    import torch
    from libbi_b200 import BatchedBootstrapPF, BootstrapPF, LearnedProposal, configs

    model = configs.L96_D40_N65536["model"]
    sim = BootstrapPF(model, n_data, seed=3)
    for k in range(100):
        sim.step_device(k * DT, (k + 1) * DT, None, sync=False)
    x, _, _ = sim.state()
    xt = x[:, :n_data].T.contiguous().clone()
    sim.step_device(100 * DT, 101 * DT, None, sync=False)
    x, _, _ = sim.state()
    xt1 = x[:, :n_data].T.contiguous().clone()
    g = torch.Generator(device="cuda")
    g.manual_seed(3)
    yt1 = (xt1 + model.sigma_y * torch.randn(xt1.shape, generator=g, device="cuda")).contiguous()
    sim.close()
    prop = LearnedProposal(model, DT, max_batch=8192, seed=3)
    prop.set_data(xt, xt1, yt1)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    trace = prop.train(train_steps, 8192, 2e-3)
    train_s = time.perf_counter() - t0
    del xt, xt1, yt1

    def run(n, use_prop):
        lls, ms = [], 0.0
        for s in range(seeds):
            pf = BootstrapPF(model, n, resampler="systematic", ess_rel=ESS_REL, seed=10_000 + s)
            if use_prop:
                pf.set_proposal(prop)
            pf.timing(True)
            ll, _, _ = pf.filter(y_host, 0.0, DT)
            r, t, _ = pf.timing_read(reset=True)
            ms += r + t
            lls.append(ll)
            pf.close()
        lls = np.array(lls)
        return {"n": n, "ll_mean": float(lls.mean()), "ll_sd": float(lls.std(ddof=1)), "ms_per_run": ms / seeds}

    def run_batched(n, use_prop, T=None):
        # the same seeds as the single filters, one filter per seed in one
        # batch (the same numbers, bit for bit); device time of the captured
        # run divided by the filters; T: the first T observations only
        b = BatchedBootstrapPF([model] * seeds, [n] * seeds, "systematic", [10_000 + s for s in range(seeds)],
                               ess_rel=ESS_REL)
        if use_prop:
            b.set_proposal(prop)
        yy = np.asarray(y_host if T is None else y_host[:T], np.float32)
        yb = np.ascontiguousarray(np.repeat(yy[:, None, :], seeds, axis=1))
        b.filter(yb, 0.0, DT)  # capture
        b.timing(True)
        b.timing_read(reset=True)
        lls, _, _, st = b.filter(yb, 0.0, DT)
        ms, _ = b.timing_read(reset=True)
        b.close()
        return {"n": n, "filters": seeds, "ll_mean": float(lls.mean()), "ll_sd": float(lls.std(ddof=1)),
                "ms_per_run": ms / seeds, "batch_ms": ms, "failed": int((st != 0).sum()), "_lls": lls}

    boot = [run(n, False) for n in n_boot]
    guided = [run(n, True) for n in n_guided]
    guided_b = [run_batched(n, True) for n in n_guided_batched]
    boot_b = [run_batched(n, False) for n in n_boot_batched]
    # the first 10 observations, where the filters still track (deviation
    # falling with N): the guided and bootstrap deviations at equal N
    short = {"T": 10,
             "bootstrap": [run_batched(n, False, 10) for n in (4096, 16384, 32768)],
             "guided": [run_batched(n, True, 10) for n in (1024, 4096, 16384)]}
    short["equal_sd"] = equal_sd_ratios(short["bootstrap"], short["guided"])
    prop.close()
    informative = guided_informative(seeds=seeds)
    # between the two: observations informative enough for the optimal
    # proposal to matter, not so much that the bootstrap filter degenerates
    intermediate = guided_informative(seeds=seeds, sigma_eta=0.3, sigma_y=1.0, n_boot=(1024, 4096, 16384, 32768),
                                      n_guided=(256, 1024, 4096))
    # the bootstrap filter's best measured cost per particle-step (single or
    # batched): the conservative price of a bootstrap filter of any size
    T = len(y_host)
    best_ns = min(b["ms_per_run"] * 1e6 / (b["n"] * T) for b in boot + boot_b)
    for gd in guided_b:
        t_b, n_b, exact = equal_mean_time(boot, gd["ll_mean"])
        gd["bootstrap_n_at_equal_mean_ll"] = n_b
        gd["gpu_time_ratio_bootstrap_over_guided_at_equal_mean_ll"] = t_b / gd["ms_per_run"]
        gd["gpu_time_ratio_at_equal_mean_ll_bootstrap_at_best_rate"] = n_b * T * best_ns * 1e-6 / gd["ms_per_run"]
        gd["equal_mean_ll_ratio_is"] = "interpolated" if exact else "bound: outside the bootstrap sweep"
    ref = next(b for b in boot if b["n"] == n_ref)
    for gd in guided:
        t_match = gd["ms_per_run"] * (gd["ll_sd"] / ref["ll_sd"]) ** 2 if ref["ll_sd"] > 0 else float("nan")
        gd["ms_to_bootstrap_sd"] = t_match
        gd["gpu_time_ratio_bootstrap_over_guided_at_equal_sd"] = ref["ms_per_run"] / t_match if t_match > 0 else None
    for gd in guided:
        t_b, n_b, exact = equal_mean_time(boot, gd["ll_mean"])
        gd["bootstrap_n_at_equal_mean_ll"] = n_b
        gd["gpu_time_ratio_bootstrap_over_guided_at_equal_mean_ll"] = t_b / gd["ms_per_run"]
        gd["equal_mean_ll_ratio_is"] = "interpolated" if exact else "bound: outside the bootstrap sweep"
    ln_n = np.log([b["n"] for b in boot])
    ln_sd = np.log([max(b["ll_sd"], 1e-300) for b in boot])
    slope = float(np.polyfit(ln_n, ln_sd, 1)[0]) if len(boot) > 1 else None
    best = max(guided, key=lambda gd: gd["gpu_time_ratio_bootstrap_over_guided_at_equal_sd"] or 0.0)
    # the workload's own comparison: guided N = 4096 against bootstrap
    # N = n_ref, deviation over the same seeds (standard error of a normal
    # sample's deviation: sd / sqrt(2 (seeds - 1)))
    g1 = next((gd for gd in guided if gd["n"] == 4096), None)
    gb = next((gd for gd in guided_b if gd["n"] == 4096), None)
    named = None
    if g1 is not None:
        se = lambda sd: sd / np.sqrt(2.0 * (seeds - 1))
        named = {"guided_n": 4096, "bootstrap_n": n_ref,
                 "guided_ll_sd": g1["ll_sd"], "guided_ll_sd_se": se(g1["ll_sd"]),
                 "bootstrap_ll_sd": ref["ll_sd"], "bootstrap_ll_sd_se": se(ref["ll_sd"]),
                 "sd_ratio_guided_over_bootstrap": g1["ll_sd"] / ref["ll_sd"],
                 "guided_ms_per_run_single": g1["ms_per_run"],
                 "guided_ms_per_run_batched": gb["ms_per_run"] if gb else None,
                 "bootstrap_ms_per_run": ref["ms_per_run"],
                 "gpu_time_ratio_bootstrap_over_guided_single": ref["ms_per_run"] / g1["ms_per_run"],
                 "gpu_time_ratio_bootstrap_over_guided_batched":
                     ref["ms_per_run"] / gb["ms_per_run"] if gb else None,
                 # near 0: the deviation does not fall with N, so matching
                 # it says little about the estimator (the mean
                 # log-likelihood comparisons do)
                 "bootstrap_sd_exponent_in_n": slope,
                 # equal footing (both batched, the deviation falling with N):
                 # the C4 model over its first 10 observations, and a model
                 # whose observations are informative
                 "equal_footing_batched": {
                     name: {"sigma_eta": sig[0], "sigma_y": sig[1],
                            **{k: eq[k] for k in ("best_ratio", "best_ratio_se", "best_ratio_is", "best_guided_n",
                                                  "meets_10x", "bootstrap_sd_exponent_in_n")}}
                     for name, sig, eq in (("c4_model_T10", (model.sigma_eta, model.sigma_y), short["equal_sd"]),
                                           ("intermediate_T10", (0.3, 1.0), intermediate["equal_sd"]),
                                           ("informative_T10", (0.5, 0.1), informative["equal_sd"]))}}
    best_m = max(guided, key=lambda gd: gd["gpu_time_ratio_bootstrap_over_guided_at_equal_mean_ll"])
    best_b = max(guided_b, key=lambda gd: gd["gpu_time_ratio_bootstrap_over_guided_at_equal_mean_ll"])
    return {
        "workload": f"l96_d40_t200_guided_vs_bootstrap_n{n_ref}_{seeds}seeds",
        "train": {"triples": n_data, "steps": train_steps, "batch": 8192, "seconds": train_s,
                  "loss_first": float(trace[:10].mean()), "loss_last": float(trace[-50:].mean()),
                  "loss_optimal_approx": float(40 * (np.log(model.sigma_eta * model.sigma_y /
                                                                np.sqrt(model.sigma_eta ** 2 + model.sigma_y ** 2))
                                                         + 0.5))},
        "bootstrap": boot,
        "guided": guided,
        "batched": {"guided": strip_lls(guided_b), "bootstrap": strip_lls(boot_b)},
        "short_horizon_batched": strip_lls(short),
        "informative_observations_batched": informative,
        "intermediate_observations_batched": intermediate,
        "named_comparison": named,
        "bootstrap_sd_exponent_in_n": slope,
        "best": {"equal_sd": {"guided_n": best["n"], "gpu_time_ratio_bootstrap_over_guided":
                              best["gpu_time_ratio_bootstrap_over_guided_at_equal_sd"]},
                 "equal_mean_ll": {"guided_n": best_m["n"], "gpu_time_ratio_bootstrap_over_guided":
                                   best_m["gpu_time_ratio_bootstrap_over_guided_at_equal_mean_ll"],
                                   "is": best_m["equal_mean_ll_ratio_is"]},
                 "equal_mean_ll_guided_batched": {
                     "guided_n": best_b["n"], "gpu_time_ratio_bootstrap_over_guided":
                         best_b["gpu_time_ratio_bootstrap_over_guided_at_equal_mean_ll"],
                     "gpu_time_ratio_bootstrap_at_best_rate":
                         best_b["gpu_time_ratio_at_equal_mean_ll_bootstrap_at_best_rate"],
                     "is": best_b["equal_mean_ll_ratio_is"]}},
        "bootstrap_best_ns_per_particle_step": best_ns,
        "timer": "CUDA events around each step's kernels, summed per filter run",
    }


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
    from oracle.oracle import Oracle
    from libbi_b200 import configs

    # the same true trajectory as the GPU arm (same draws, same arithmetic),
    # here from the oracle's model run, with the same observation noise
    model = configs.L96_D40_N65536["model"]
    _, xs = Oracle().simulate(model.desc(), DATA_SEED, T_OBS, 0.0, DT)
    y = observe(xs, model.sigma_y)
    # the host's caches are flushed the same way before the timed sample
    import numpy as np

    np.ones(L2_FLUSH_BYTES // 8)
    cb = cpu_baseline(y, seconds=max(5.0, 2.0 * (args.steps + args.warmup)))
    line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(args.gpus),
            "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-large-n", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--no-guided", action="store_true")
    ap.add_argument("--no-precision", action="store_true")
    ap.add_argument("--pmmh-iterations", type=int, default=2000,
                    help="PMMH iterations timed per arm (2000, the workload's; fewer for profiling)")
    ap.add_argument("--guided-seeds", type=int, default=64,
                    help="filter runs per N in the guided/bootstrap comparison (64; fewer for profiling)")
    ap.add_argument("--large-n-sizes", type=int, nargs="+", default=[1 << 22, 1 << 24, 1 << 26],
                    help="particle counts of the large-N kernel section (one small size for profiling: the "
                         "section holds about 330 B per particle on the device)")
    ap.add_argument("--headline-only", action="store_true",
                    help="the headline line alone, none of the single-GPU sections after it (for profiling)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.warmup < 3:
        args.warmup = 3
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))

    import numpy as np
    import torch

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    from libbi_b200 import BootstrapPF, build, configs

    build.build()
    model = configs.L96_D40_N65536["model"]
    y_host = synthetic_observations(model)
    y_dev = torch.as_tensor(y_host, device="cuda")
    from libbi_b200.replicas import max_over_ranks, replica_seed, whole_job_rate

    pf = BootstrapPF(model, N_PARTICLES, resampler="systematic", ess_rel=ESS_REL, seed=replica_seed(SEED, rank))
    fused = pf.step_form_fused
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    k = 0

    def next_k():
        nonlocal k
        if k >= T_OBS:
            pf.init()
            k = 0
        k += 1
        return k

    # warm-up (untimed)
    for _ in range(args.warmup):
        kk = next_k()
        pf.step_device((kk - 1) * DT, kk * DT, y_dev[kk - 1], sync=False)
    torch.cuda.synchronize()

    # timed: K steps, L2 flushed before each, CUDA events around each step
    # (and none between the step's kernels: every event recorded there adds
    # device time to the step)
    pf.timing(False)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    gpu_id = str(torch.cuda.get_device_properties(local).uuid)
    gpu_id = gpu_id if gpu_id.startswith("GPU-") else "GPU-" + gpu_id
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(gpu_id) as clk:
        wall0 = time.perf_counter()
        # an NVTX range around the timed steps, so that a profiler can select
        # exactly these launches (ncu --nvtx --nvtx-include "bench_timed_steps/")
        torch.cuda.nvtx.range_push("bench_timed_steps")
        for i in range(args.steps):
            kk = next_k()
            flush.zero_()
            starts[i].record()
            pf.step_device((kk - 1) * DT, kk * DT, y_dev[kk - 1], sync=False)
            ends[i].record()
        torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
        wall = time.perf_counter() - wall0
        # the kernel split: the same K steps again, with the handle's events
        # before the resampler, between it and the transition, and after the
        # transition (each interval includes an event's own device time)
        pf.timing(True)
        pf.timing_read(reset=True)
        for i in range(args.steps):
            kk = next_k()
            flush.zero_()
            pf.step_device((kk - 1) * DT, kk * DT, y_dev[kk - 1], sync=False)
        torch.cuda.synchronize()
        res_ms, tr_ms, nst = pf.timing_read(reset=True)
        pf.timing(False)
    if dist:
        dist.barrier()
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    total_ms = sum(step_ms)
    total_ms = max_over_ranks(total_ms, dist, "cuda")
    value = whole_job_rate(N_PARTICLES * args.steps, world, total_ms / 1e3)

    # end to end through the public API: pinned host observation copied in,
    # step statistics read back, every step
    y_pin = torch.empty((T_OBS, DIM), dtype=torch.float32).pin_memory()
    y_pin.copy_(torch.as_tensor(y_host))
    y_np = y_pin.numpy()
    e2e_s = 0.0
    resampled = 0
    for i in range(args.steps):
        kk = next_k()
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = pf.step((kk - 1) * DT, kk * DT, y_np[kk - 1])
        e2e_s += time.perf_counter() - t0
        resampled += int(r.resampled)
    e2e_s = max_over_ranks(e2e_s, dist, "cuda")
    e2e_step_api = whole_job_rate(N_PARTICLES * args.steps, world, e2e_s)

    # end to end through the call a LibBi filter client makes,
    # Filter<BootstrapPF>::filter -> bpf_filter: the T observations copied
    # from pinned host memory, the initial draw, T steps, the final term, and
    # the increments, ESS and log-likelihood read back, host wall clock
    # around each whole call (L2 flushed before each)
    e2e_runs = max(3, args.steps // 10)
    e2e_filter_s = 0.0
    # two untimed calls first: a repeated schedule runs as one CUDA graph
    # from the second call on (a sampler's steady state)
    for _ in range(2):
        pf.filter(y_np, 0.0, DT)
    for _ in range(e2e_runs):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        pf.filter(y_np, 0.0, DT)
        e2e_filter_s += time.perf_counter() - t0
    e2e_filter_s = max_over_ranks(e2e_filter_s, dist, "cuda")
    e2e = whole_job_rate(N_PARTICLES * T_OBS * e2e_runs, world, e2e_filter_s)

    hbm, how, sm_max = peaks()
    clocks = clk.summary()
    t_launch = tr_ms / max(nst, 1) / 1e3
    bytes_launch = TRANSITION_BYTES_PER_PARTICLE * N_PARTICLES
    achieved = bytes_launch / t_launch / 1e9
    f_mhz = clocks["sm_mhz"] or sm_max
    fp32_peak = 148 * 128 * 2 * f_mhz * 1e6 / 1e12
    fp32_ach = TRANSITION_FLOP_PER_PARTICLE * N_PARTICLES / t_launch / 1e12
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(world),
        "resampled_steps_end_to_end": f"{resampled} of {args.steps}",
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": DIM * 4,
                "d2h_bytes_per_step": 3 * 8, "runs": e2e_runs, "steps_per_run": T_OBS,
                "timer": "host wall clock around bpf_filter (Filter<BootstrapPF>::filter): observations "
                         "uploaded from pinned host memory, initial draw, T steps (one CUDA graph: the schedule "
                         "repeats, after two untimed calls), increments/ESS/log-likelihood read back"},
        "e2e_step_api": {"value": e2e_step_api, "unit": UNIT, "h2d_bytes_per_step": DIM * 4,
                         "d2h_bytes_per_step": 80,
                         "timer": "host wall clock around bpf_step (BootstrapPF::step), one synchronising call "
                                  "per step"},
        "gpu_launches": LAUNCHES_PER_STEP[fused] * args.steps,
        "step_form": "one launch per step (resampling as the step kernel's prologue)" if fused else
                     "two launches per step (resampler, then transition)",
        "roofline": {"kernel": "k_l96_step<float,40>" if fused else "k_l96_transition<float,40>",
                     "bound": "hbm", "achieved": achieved,
                     "peak": hbm, "unit": "GB/s", "frac": achieved / hbm, "peak_source": how,
                     "traffic": TRANSITION_DRAM_BYTES_PER_LAUNCH,
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum, one launch",
                     "algorithmic_bytes_per_launch": bytes_launch,
                     "launch_ms": t_launch * 1e3,
                     "fp32": {"achieved_tflops": fp32_ach, "peak_tflops": fp32_peak,
                              "frac": fp32_ach / fp32_peak,
                              "peak_source": "148 SM x 128 FP32 lanes x 2 x sampled SM clock"}},
        "kernel_ms_per_step": {"resample": res_ms / max(nst, 1), "transition": tr_ms / max(nst, 1),
                               "timer": "a second pass of K steps with events between the kernels" +
                                        ("; in the one-launch form 'transition' is the whole step kernel, "
                                         "resampling prologue included" if fused else "")},
        "wall_s": wall,
        "clocks": clocks,
    }
    # the sections below are single-GPU measurements: under torchrun (N > 1)
    # the line carries the replicas' headline only, so that no rank waits
    # at the final barrier while rank 0 runs them
    extras = rank == 0 and world == 1 and not args.headline_only
    if extras:
        # the resampler's tile shape for this N (bpf_create tuned it; timed
        # again here so the line shows each shape's median)
        from libbi_b200 import autotune_resampler
        from libbi_b200.filter import RESAMPLE_SHAPES, shape_name

        best, us = autotune_resampler(N_PARTICLES)
        line["autotune"] = {"systematic_resampler_n": N_PARTICLES, "shape": shape_name(RESAMPLE_SHAPES[best]),
                            "median_us": {shape_name(k): v for k, v in us.items()}}
    if extras and not args.no_large_n:
        line["kernels_large_n"] = large_n_kernels(tuple(args.large_n_sizes))
    if extras:
        line["step_forms"] = step_forms(y_dev)
        line["pz_c1"] = pz_c1()
    if extras and not args.no_batched:
        line["batched"] = batched_filters()
        line["pmmh"] = pmmh_chains(iterations=max(2, args.pmmh_iterations))
    if extras and not args.no_precision:
        line["precision"] = precision_check(y_host)
        line["precision_batched"] = batched_precision()
    if extras and not args.no_guided:
        line["guided"] = guided_vs_bootstrap(y_host, seeds=max(2, args.guided_seeds))
    if extras and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(y_host)
    pf.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
