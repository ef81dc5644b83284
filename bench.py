"""Benchmark of the B200 CIRSRADG forward model + analytic Jacobian and the
optimal-estimation retrieval built on it.

Headline workload (one step): one nadir thermal-emission spectrum of 120
layers, H2/He + CH4, C2H6, C2H2, NH3 random-overlapped (NG = 20), 2000
wavenumbers, Jacobian over NX = 124 state elements -- the full-size
single-spectrum configuration.  Beside it, each at its stated size:
  batch      4096 uneven spectra in one persistent launch (autotuned tile and
             schedule, CUDA graph)
  retrieval  1024 full-size retrievals, up to 10 Newton iterations
  serving    Poisson arrivals at 2000 req/s into the continuous-batching
             server under an HBM budget that caps the requests in flight,
             and a sub-saturation point (40 req/s for 30 s)
Inputs are the seeded synthetic workloads of radtrancode_b200/synth.py (the
reference measures on no public data set).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

`value`: spectra/s with inputs resident in HBM (CUDA events on the launching
stream around K launches; the k-tables, 384 MB of raw + ln k, exceed the
126 MB L2, so no flush is needed between steps).  `e2e`: the same metric
through the public C ABI call (rtb_cirsrtfg_wave) with host buffers, the
host->device copy of the inputs and the device->host copy of the radiance
and Jacobian inside the timed region.  Multi-GPU: one process per GPU
(torchrun), every rank runs its own spectra (independent units, no data-path
collective), weak scaling, time = max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "fwd+Jacobian spectra/s & retrievals/s at ≤1e-4 rel err; retrieval p50/p99 ms"
WORKLOAD = ("single spectrum, full size: 120 layers, H2/He + CH4/C2H6/C2H2/NH3 random overlap (NG=20), "
            "2000 wavenumbers 600-1400 cm-1, k-tables 20P x 15T x 20g, Jacobian NX=124")
PROFILE_DATA = os.path.join(ROOT, "profiles", "fwd_kernel_config2.json")


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def measured_peaks():
    """HBM GB/s and bf16 TFLOP/s of MEASURED_PEAKS.json (driver-written on
    this pool's B200s), else the pool's earlier fallback figures."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), float(p["bf16_tflops"]), "measured"
    except Exception:
        return 6650.0, 1590.0, "fallback"


def profile_data():
    """Per-launch figures of one ncu capture of the forward kernel on this
    workload (DRAM bytes, warp instructions), committed beside the summary."""
    try:
        with open(PROFILE_DATA) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def algorithmic_bytes(kt, job, in_bytes, out_bytes):
    """Bytes a launch must move at least: every distinct (P, T) corner of the
    ln k table touched by the layers' bilinear stencils, per gas and
    wavenumber (NG values of 4 B, plus the g=0 raw value the KLOG test reads),
    plus the CIA table cells touched, the packed inputs and the outputs."""
    lnp = kt.lnp.astype(np.float32)
    tk = kt.tk.astype(np.float32)
    p1 = np.clip(np.log(job.press.astype(np.float64)).astype(np.float32), lnp[0], lnp[-1])
    cp = np.clip(np.searchsorted(lnp, p1, side="right"), 1, kt.np_ - 1)
    t1 = np.clip(job.temp, tk[0], tk[-1])
    ct = np.clip(np.searchsorted(tk, t1, side="right"), 1, kt.nt - 1)
    corners = set()
    for a, b in zip(cp, ct):
        for da in (-1, 0):
            for db in (-1, 0):
                corners.add((int(a) + da, int(b) + db))
    ntabgas = int(np.sum(job.ktab >= 0))
    table = ntabgas * job.nwave * len(corners) * (kt.ng * 4 + 4)
    cia = job.nwave * 2 * 2 * 9 * 4 * len(set(int(x) for x in np.clip(job.temp // 15, 0, 24)))
    return table + cia + in_bytes + out_bytes


class ClockSampler:
    """Clock and throttle-reason samples during the timed region: NVML read
    in-process every 20 ms (the timed region lasts a fraction of a second),
    else nvidia-smi every 200 ms.  Reads only; no GPU setting is changed."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.f = None

    # clocks-event reason bits of NVML (nvml.h): sw power cap, hw slowdown,
    # sw thermal, hw thermal
    BITS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40}

    def _nvml_start(self):
        import threading

        import pynvml
        pynvml.nvmlInit()
        h = pynvml.nvmlDeviceGetHandleByIndex(self.idx)
        self.nv_max = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)
        self.nv_rows = []
        self.nv_stop = threading.Event()

        def loop():
            while not self.nv_stop.is_set():
                try:
                    sm = pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)
                    rs = pynvml.nvmlDeviceGetCurrentClocksThrottleReasons(h)
                    self.nv_rows.append((sm, rs))
                except Exception:
                    pass
                self.nv_stop.wait(0.02)

        self.nv_thread = threading.Thread(target=loop, daemon=True)
        self.nv_thread.start()

    def start(self):
        self.nv_thread = None
        try:
            self._nvml_start()
            return
        except Exception:
            self.nv_thread = None
        try:
            self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.nv_thread is not None:
            self.nv_stop.set()
            self.nv_thread.join(timeout=2)
            try:
                import pynvml
                pynvml.nvmlShutdown()
            except Exception:
                pass
            rows = list(self.nv_rows)
            if not rows:
                return None
            reasons = sorted(n for n, b in self.BITS.items() if any(r & b for _, r in rows))
            return {"sm_mhz": statistics.median(s for s, _ in rows), "sm_max_mhz": float(self.nv_max),
                    "reasons": reasons, "samples": len(rows), "source": "NVML, 20 ms"}
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.flush()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
            except (ValueError, IndexError):
                continue
            for n, v in zip(names, r[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


class BusySampler:
    """Fraction of time the GPU was running a kernel, from NVML's utilization
    counter read every 20 ms in a thread (reads only)."""

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.samples = []
        self.thread = None

    def start(self):
        import threading
        try:
            import pynvml
            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByIndex(self.idx)
        except Exception:
            return
        self.stop_ev = threading.Event()

        def loop():
            while not self.stop_ev.is_set():
                try:
                    self.samples.append(pynvml.nvmlDeviceGetUtilizationRates(h).gpu)
                except Exception:
                    pass
                self.stop_ev.wait(0.02)

        self.thread = threading.Thread(target=loop, daemon=True)
        self.thread.start()

    def stop(self):
        if self.thread is None:
            return None
        self.stop_ev.set()
        self.thread.join(timeout=2)
        if not self.samples:
            return None
        return {"mean_pct": float(np.mean(self.samples)), "samples": len(self.samples),
                "source": "NVML utilization.gpu every 20 ms"}


# ---------------------------------------------------------------- accuracy against the FP64 oracle
def _jac_errors(g, g64, nv):
    G = np.asarray(g, np.float64).reshape(nv, -1)
    R = np.asarray(g64, np.float64).reshape(nv, -1)
    scale = np.max(np.abs(R), axis=1, keepdims=True)
    colnorm = float(np.max(np.abs(G - R) / np.where(scale > 0, scale, 1.0)))
    big = (np.abs(R) >= 1e-3 * scale) & (scale > 0)
    elem = float(np.max(np.abs(G - R)[big] / np.abs(R)[big])) if big.any() else 0.0
    return colnorm, elem


def accuracy(kt, cia, pairs, nthr, what):
    """Per-result errors of device outputs against the FP64 oracle: the
    largest radiance relative error, the largest column-normalised Jacobian
    error (each state element's row scaled by its largest magnitude) and the
    element-wise relative Jacobian error over entries of at least 1e-3 of
    their row's largest magnitude, over the (job, (calcout, gradients, _))
    pairs given."""
    from oracle import pyoracle as po
    r = jc = je = 0.0
    for job, (c, g, _) in pairs:
        c64, g64, _ = po.cirsrtfg_wave(kt, cia, job, po.ORC_FP64, nthreads=nthr)
        r = max(r, float(np.max(np.abs(np.asarray(c, np.float64) - c64) / np.abs(c64))))
        a, b = _jac_errors(g, g64, job.nv)
        jc, je = max(jc, a), max(je, b)
    return {"radiance_max_rel_err": r, "jacobian_max_rel_err": jc, "jacobian_elementwise_max_rel_err": je,
            "results": len(pairs), "of": what, "vs": "FP64 oracle",
            "gates": {"radiance": 1e-4, "jacobian": 1e-3}}


# ---------------------------------------------------------------- reference arm
def reference_arm(args, rank):
    """The reference's CPU path on the host cores.  No Fortran compiler exists
    here or on the GPU host, so the reference Fortran cannot be built; the
    arm runs the oracle (the C++ restatement of the reference Fortran,
    oracle/, built -O3 -march=native on this host) on all host threads over
    the whole spectrum every step."""
    if rank != 0:
        return
    from oracle import pyoracle as po
    po.use_native()
    from radtrancode_b200 import synth
    kt, cia, job = synth.config2()
    nthr = os.cpu_count() or 1
    warm = synth.make_job(kt, synth.ABSORBERS_C2, nlayer=120, seed=1003, iw0=0, nwave=4 * nthr, vmr_perturb=0.3)
    for _ in range(args.warmup):
        po.cirsrtfg_wave(kt, cia, warm, po.ORC_MIXED, nthreads=nthr)
    times = []
    for _ in range(args.steps):
        t = time.perf_counter()
        po.cirsrtfg_wave(kt, cia, job, po.ORC_MIXED, nthreads=nthr)
        times.append(time.perf_counter() - t)
    t_step = statistics.mean(times)
    value = 1.0 / t_step
    sample = (f"the whole spectrum (2000 wavenumbers) per step, {nthr} threads on {cpu_model()}; C++ restatement "
              "of the reference Fortran, -O3 -march=native (no Fortran compiler on the host)")
    out = {
        "metric": METRIC, "value": value, "unit": "spectra/s", "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_step * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 (f64 transmissions)",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "sample": "whole spectrum per step"},
        "cpu_baseline": {"value": value, "unit": "spectra/s", "cores": nthr, "kind": "port", "sample": sample,
                         "cpu": cpu_model()},
        "e2e": {"value": value, "unit": "spectra/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "gpu_launches": 0,
    }
    print(json.dumps(out))


def cpu_baseline(kt, cia, job, nthr):
    """Rank-0 CPU baseline: the oracle port on all host threads over the whole
    spectrum (about 1.5 s)."""
    from oracle import pyoracle as po
    t = time.perf_counter()
    po.cirsrtfg_wave(kt, cia, job, po.ORC_MIXED, nthreads=nthr)
    dt = time.perf_counter() - t
    return {"value": 1.0 / dt, "unit": "spectra/s", "cores": nthr, "kind": "port", "cpu": cpu_model(),
            "sample": f"the whole spectrum (2000 wavenumbers), {nthr} threads, C++ restatement of the reference "
                      "Fortran built -O3 -march=native (no Fortran compiler on the host)"}


# ---------------------------------------------------------------- batch leg
BATCH_SPECTRA = 4096          # the batching workload: 4096 uneven spectra
BATCH_TUNE = 256              # sub-batch the autotuner times
BATCH_ACC = 8                 # spectra of the batch checked against the FP64 oracle


def batch_leg(ctx, kt, cia, nspec, nthr):
    """Uneven-spectra batch in one persistent launch: default tile and
    schedule vs the autotuned ones replayed through a CUDA graph, the batched
    C-ABI call end to end, and the accuracy of a sample of its spectra."""
    from radtrancode_b200 import synth
    jobs = synth.config3_jobs(kt, nspec, seed=1003)
    nwave = sum(j.nwave for j in jobs)
    ctx.prepare(jobs[:BATCH_TUNE])
    tune = ctx.autotune()
    t = time.perf_counter()
    ctx.prepare(jobs)
    t_prep = time.perf_counter() - t
    ctx.set_tile(0)
    ctx.set_schedule(0, 0)
    ctx.launch()
    ctx.fetch()
    ms_default = ctx.stats()["ms_kernel"]
    ctx.set_tile(tune["warps"])
    ctx.set_schedule(tune["schedule"], tune["blocks_per_sm"])
    ctx.use_graph(True)
    ms = []
    for _ in range(2):                     # capture, then a replay
        ctx.launch()
        outs = ctx.fetch()
        ms.append(ctx.stats()["ms_kernel"])
    ms_tuned = ms[-1]
    ctx.use_graph(False)
    ctx.set_tile(0)
    ctx.set_schedule(0, 0)
    pick = np.linspace(0, nspec - 1, BATCH_ACC).astype(int)
    acc = accuracy(kt, cia, [(jobs[i], outs[i]) for i in pick], nthr, f"{BATCH_ACC} spectra of the batch")
    t = time.perf_counter()
    ctx.cirsrtfg_wave_batch(jobs)
    t_e2e = time.perf_counter() - t
    st = ctx.stats()
    return {
        "workload": f"{nspec} uneven spectra: W~U[200,2000] of the 2000-bin grid, L~U[40,120], 1-4 of the four "
                    "absorbers, theta~U[0,70 deg], one persistent launch",
        "spectra": nspec, "wavenumbers": nwave,
        "value": nspec / (ms_tuned * 1e-3), "unit": "spectra/s",
        "ms_launch_tuned_graph": ms_tuned, "ms_launch_default": ms_default,
        "tuned": tune | {"schedule": ["static", "dynamic", "dynamic longest-first"][tune["schedule"]],
                         "tile": f"{tune['warps']} warps per block (one layer per warp, one g-ordinate per lane, "
                                 "one (spectrum, wavenumber) item per block)",
                         "tuned_on_spectra": BATCH_TUNE},
        "prepare_s": t_prep,
        "e2e": {"value": nspec / t_e2e, "unit": "spectra/s", "h2d_bytes": st["h2d_bytes"],
                "d2h_bytes": st["d2h_bytes"], "note": "rtb_cirsrtfg_wave_batch with host buffers, default tile"},
        "accuracy": acc,
    }


# ---------------------------------------------------------------- retrieval leg
RET_N = 1024                  # the retrieval workload: 1024 full-size retrievals
RET_FP64 = 16                 # of those, re-run with the all-FP64 Newton step
RET_ACC = 4                   # final states whose forward model is checked against the FP64 oracle
NEWTON_BATCH = 296            # retrievals per timed Newton-step launch (2 per SM)
RET_WORKLOAD = ("optimal-estimation retrievals, full size: NX=124 (120 layer T + 4 log gas scales), NY=2000, "
                "10 Newton iterations max, phlimit 0.1 %, Sa exponential correlation 1.5 scale heights "
                "3 K / 50 %, Se diagonal (1e-9)^2, y = F(x_true) + N(0, 1e-9), x_true ~ N(xa, Sa)")


def retrieval_cases(ctx, kt, n, seed0=4000):
    """Full-size retrieval cases; observations from the device forward model
    at the true states (batched launches) plus seeded noise."""
    from radtrancode_b200 import synth
    cases = [synth.make_retrieval(kt, synth.ABSORBERS_C2, nlayer=120, seed=seed0 + 17 * i, nwave=2000)
             for i in range(n)]
    outs = []
    for b in range(0, n, 256):
        outs += ctx.cirsrtfg_wave_batch([synth.job_at_state(c, c.x_true) for c in cases[b:b + 256]])
    for i, c in enumerate(cases):
        synth.observe(c, outs[i][0], seed=seed0 + 17 * i + 1)
    return cases, outs


def retrieval_leg(ctx, kt, cia, nret, bf16_peak, hbm_peak, nthr):
    """Retrievals/s and completion-time percentiles of the batched engine
    (rtb_retrieve_batch), the mixed-precision result against the all-FP64
    device solve, the forward model at the retrieved states against the FP64
    oracle, the Newton kernel against the tensor and HBM peaks, and the
    oracle's retrieval on the host cores."""
    from oracle import pyoracle as po
    from radtrancode_b200 import synth
    cases, outs = retrieval_cases(ctx, kt, nret)
    ctx.set_newton_mode(0, 1)
    t = time.perf_counter()
    res = ctx.retrieve_batch(cases, kiter=10, phlimit=0.1)
    dt = time.perf_counter() - t
    lat = np.array([r["ms"] for r in res])
    ctx.set_newton_mode(1, 0)
    try:
        res64 = ctx.retrieve_batch(cases[:RET_FP64], kiter=10, phlimit=0.1)
    finally:
        ctx.set_newton_mode(0, 1)
    dx, same = 0.0, 0
    for c, a, b in zip(cases, res, res64):
        sig = np.sqrt(np.diag(c.sa))
        dx = max(dx, float(np.max(np.abs(a["x"] - b["x"]) / sig)))
        same += int(a["iterations"] == b["iterations"] and a["converged"] == b["converged"])
    # the forward model at retrieved states, device vs FP64 oracle
    jobs = [synth.job_at_state(cases[i], res[i]["x"]) for i in range(RET_ACC)]
    acc = accuracy(kt, cia, list(zip(jobs, ctx.cirsrtfg_wave_batch(jobs))), nthr,
                   f"the forward model at {RET_ACC} retrieved states")
    # Newton-step kernel alone: NEWTON_BATCH retrievals of K at the true states
    pick = [i % nret for i in range(NEWTON_BATCH)]
    kk = np.stack([outs[i][1].reshape(124, 2000) for i in pick])
    sai = np.stack([np.linalg.inv(cases[i].sa) for i in pick])
    sei = np.stack([cases[i].sei for i in pick])
    xa = np.stack([cases[i].xa for i in pick])
    y = np.stack([cases[i].y for i in pick])
    yn = np.stack([outs[i][0] for i in pick])
    ms_newton = []
    for _ in range(4):
        ctx.newton_step_batch(kk, sei, sai, xa, xa, y, yn)
        ms_newton.append(ctx.newton_stats()["ms_kernel"])
    ms_n = statistics.median(ms_newton[1:])
    flops = NEWTON_BATCH * (2.0 * 124 * 124 * 2000 + 2.0 * 124 * 2000)
    tflops = flops / (ms_n * 1e-3) / 1e12
    kbytes = NEWTON_BATCH * 124 * 2000 * 4 * 2        # K read by the product pass and the refinement pass
    t = time.perf_counter()
    po.retrieve(kt, cia, cases[0], kiter=10, phlimit=0.1, nthreads=nthr)
    t_cpu = time.perf_counter() - t
    return {
        "workload": RET_WORKLOAD, "retrievals": nret, "value": nret / dt, "unit": "retrievals/s",
        "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
        "latency_note": "completion time from the start of the batched call (all admitted at once)",
        "iterations_mean": float(np.mean([r["iterations"] for r in res])),
        "forwards_mean": float(np.mean([r["forwards"] for r in res])),
        "converged": int(sum(r["converged"] > 0 for r in res)),
        "accuracy": acc,
        "newton": {"hessian": "K~ = Se^-1/2 K as bf16 hi + lo, hi*hi + hi*lo + lo*hi by tcgen05.mma (M=N=128, K=16) "
                              "into an FP32 accumulator in tensor memory; 1 FP64 refinement step; FP64 Cholesky",
                   "vs_fp64_solve": {"retrievals": RET_FP64, "max_dx_over_prior_sigma": dx,
                                     "same_iterations_and_stop_rule": same}},
        "newton_kernel": {"batch": NEWTON_BATCH, "ms": ms_n, "achieved_tflops": tflops, "peak_tflops": bf16_peak,
                          "frac": tflops / bf16_peak, "flops_per_retrieval": "2 NX^2 NY + 2 NX NY",
                          "k_read_gbs": kbytes / (ms_n * 1e-3) / 1e9,
                          "k_read_frac_of_hbm": kbytes / (ms_n * 1e-3) / 1e9 / hbm_peak},
        "cpu_baseline": {"value": 1.0 / t_cpu, "unit": "retrievals/s", "cores": nthr, "kind": "port",
                         "sample": f"1 retrieval of the same workload, oracle coreret restatement, {nthr} threads"},
    }


# ---------------------------------------------------------------- serving leg
SERVE_POINTS = ((2000.0, 0.5, 256 << 20), (40.0, 30.0, 16 << 30))   # (req/s, s of arrivals, HBM budget)
SERVE_PLAIN = 24              # requests run one at a time for the plain per-request form
SERVE_CHECK = 4               # served results re-run alone: bit-identical


def serving_cases(ctx, kt, n, seed=5000):
    """Requests with the uneven-batch size distribution: W~U[200,2000],
    L~U[40,120], 1-4 absorbers, theta~U[0,70 deg]; observations from the
    device forward model at the true states plus noise."""
    from radtrancode_b200 import synth
    rng = np.random.default_rng(seed)
    cases = []
    for i in range(n):
        w = int(rng.integers(200, 2001))
        iw0 = int(rng.integers(0, 2000 - w + 1))
        L = int(rng.integers(40, 121))
        na = int(rng.integers(1, 5))
        ab = [synth.ABSORBERS_C2[k] for k in sorted(rng.choice(4, size=na, replace=False))]
        cases.append(synth.make_retrieval(kt, ab, nlayer=L, seed=seed + 7 * i + 1, nwave=w, iw0=iw0,
                                          theta_deg=float(rng.uniform(0.0, 70.0))))
    outs = []
    for b in range(0, n, 512):
        outs += ctx.cirsrtfg_wave_batch([synth.job_at_state(c, c.x_true) for c in cases[b:b + 512]])
    for i, c in enumerate(cases):
        synth.observe(c, outs[i][0], seed=seed + 7 * i + 2)
    return cases


def serve_point(ctx, kt, rate, window, budget, seed):
    """Poisson arrivals into the continuous-batching server; latency from
    each request's arrival time to its completion; a few served results
    re-run alone (bit-identical expected)."""
    from radtrancode_b200 import cirsradg
    rng = np.random.default_rng(seed)
    arr = np.cumsum(rng.exponential(1.0 / rate, size=int(rate * window * 1.5) + 16))
    arr = arr[arr < window]
    n = len(arr)
    cases = serving_cases(ctx, kt, n, seed=5000 + seed)
    lat, its, rounds, peak, queued_rounds, step_s = [], [], 0, 0, 0, 0.0
    results = {}
    i, pending = 0, {}
    busy = BusySampler(ctx.device)
    busy.start()
    t0 = time.perf_counter()
    with cirsradg.Server(ctx, budget, kiter=15, phlimit=0.1, dchisq_stop=0.1) as srv:
        while i < n or pending:
            now = time.perf_counter() - t0
            while i < n and arr[i] <= now:
                pending[srv.submit(cases[i])] = (i, arr[i])
                i += 1
            if not pending:
                time.sleep(max(0.0, arr[i] - now))
                continue
            t1 = time.perf_counter()
            active, queued = srv.step()
            step_s += time.perf_counter() - t1
            rounds += 1
            peak = max(peak, active)
            queued_rounds += int(queued > 0)
            t = time.perf_counter() - t0
            for rid in list(pending):
                r = srv.poll(rid)
                if r is not None:
                    k, a = pending.pop(rid)
                    lat.append((t - a) * 1e3)
                    its.append(r["iterations"])
                    results[k] = r
    t_total = time.perf_counter() - t0
    gpu_busy = busy.stop()
    same = 0
    for k in sorted(results)[:SERVE_CHECK]:
        alone = ctx.retrieve_batch([cases[k]], kiter=15, phlimit=0.1, dchisq_stop=0.1)[0]
        same += int(np.array_equal(alone["x"], results[k]["x"]) and alone["iterations"] == results[k]["iterations"])
    lat = np.array(lat)
    return cases, {
        "offered_rate": rate, "window_s": window, "hbm_budget_bytes": budget, "requests": n,
        "value": n / t_total, "unit": "retrievals/s", "wall_s": t_total, "rounds": rounds,
        "peak_in_flight": peak, "rounds_with_requests_waiting_for_memory": queued_rounds,
        "p50_ms": float(np.percentile(lat, 50)), "p95_ms": float(np.percentile(lat, 95)),
        "p99_ms": float(np.percentile(lat, 99)), "iterations_mean": float(np.mean(its)),
        "server_step_s": step_s, "gpu_busy": gpu_busy,
        "alone_vs_mix": {"checked": min(SERVE_CHECK, len(results)), "bit_identical": same},
    }


def serving_leg(ctx, kt, cia, nthr, points=SERVE_POINTS):
    """The server at each (rate, window, budget) point, the plain per-request
    GPU form beside it, and the forward model at served states against the
    FP64 oracle."""
    from radtrancode_b200 import synth
    out = {"workload": "Poisson arrivals, sizes of the uneven batch (W~U[200,2000], L~U[40,120], 1-4 absorbers), "
                       "up to 15 Newton iterations, early exit at |delta chi2| < 0.1, continuous batching under an "
                       "HBM budget; latency from each request's arrival", "points": []}
    cases = None
    for k, (rate, window, budget) in enumerate(points):
        cs, pt = serve_point(ctx, kt, rate, window, budget, seed=77 + k)
        out["points"].append(pt)
        cases = cases or cs
    plain = []
    t = time.perf_counter()
    for c in cases[:SERVE_PLAIN]:
        t1 = time.perf_counter()
        ctx.retrieve_batch([c], kiter=15, phlimit=0.1, dchisq_stop=0.1)
        plain.append((time.perf_counter() - t1) * 1e3)
    t_plain = time.perf_counter() - t
    out["plain_per_request"] = {"requests": SERVE_PLAIN, "value": SERVE_PLAIN / t_plain, "unit": "retrievals/s",
                                "p50_ms": float(np.percentile(plain, 50)), "p99_ms": float(np.percentile(plain, 99)),
                                "note": "one request at a time, rtb_retrieve_batch of one, service time only"}
    sel = cases[:4]
    res = ctx.retrieve_batch(sel, kiter=15, phlimit=0.1, dchisq_stop=0.1)
    jobs = [synth.job_at_state(c, r["x"]) for c, r in zip(sel, res)]
    out["accuracy"] = accuracy(kt, cia, list(zip(jobs, ctx.cirsrtfg_wave_batch(jobs))), nthr,
                               "the forward model at 4 served states")
    out["value"] = out["points"][0]["value"]
    out["unit"] = "retrievals/s"
    return out


# ---------------------------------------------------------------- profiling cases
def profile_case(args):
    """Reduced cases for ncu captures (warm-up + --steps launches each):
      forward  the full-size spectrum cut to its first --profile-size wavenumbers
      newton   --profile-size full-size Newton steps (NX=124, NY=2000)
      aux      calc_phiret, the Sa inverse, calc_gain_matrix + calcnextxn on --profile-size retrievals
      layers   --profile-size calls of rtb_layerg on the full-size profile (121 levels, 6 gases, 30 deg)
      conv     --profile-size convolutions of a full-size spectrum's 126 series onto 600 square-bin
               channels (FWHM 1.2 cm-1) and 200 filter channels"""
    from radtrancode_b200 import cirsradg, synth
    n, what = args.profile_size, args.profile
    rng = np.random.default_rng(11)
    with cirsradg.Context(0) as ctx:
        if what == "forward":
            kt, cia, _ = synth.config2()
            job = synth.make_job(kt, synth.ABSORBERS_C2, nlayer=120, seed=1003, nwave=n, vmr_perturb=0.3)
            ctx.set_ktables(kt)
            ctx.set_cia(cia)
            ctx.prepare([job])
            for _ in range(args.warmup + args.steps):
                ctx.launch()
                ctx.fetch()
                print(json.dumps({"profile": what, "ms_kernel": ctx.stats()["ms_kernel"]}))
        elif what in ("newton", "aux"):
            nx, ny = 124, 2000
            _, p_lay = synth._levels(120)
            sa = synth.prior_covariance(p_lay, 4)
            sai = np.broadcast_to(np.linalg.inv(sa), (n, nx, nx))
            sei = np.full((n, ny), 1e18)
            xa = np.full((n, nx), 150.0, np.float32)
            xn = xa + rng.standard_normal((n, nx)).astype(np.float32)
            y = (rng.standard_normal((n, ny)) * 1e-8).astype(np.float32)
            yn = np.zeros((n, ny), np.float32)
            for _ in range(args.warmup + args.steps):
                if what == "newton":
                    kk = (rng.standard_normal((n, nx, ny)) * 1e-9).astype(np.float32)
                    ctx.newton_step_batch(kk, sei, sai, xa, xa, y, yn)
                    print(json.dumps({"profile": what, "ms_kernel": ctx.newton_stats()["ms_kernel"]}))
                else:
                    kk = (rng.standard_normal((nx, ny)) * 1e-9).astype(np.float32)
                    phi, _ = ctx.calc_phiret_batch(y, yn, sei, xn, xa, sai)
                    ctx.spd_inverse_batch(np.broadcast_to(sa, (n, nx, nx)))
                    dd, aa, _ = ctx.calc_gain_matrix(kk, sai[0], sei[0])
                    x = ctx.calcnextxn(xa[0], xn[0], y[0], yn[0], dd, aa)
                    print(json.dumps({"profile": what, "phi0": float(phi[0]), "x0": float(x[0])}))
        elif what == "layers":
            prof = synth.make_profile(synth.ABSORBERS_C2, npro=121, seed=1005)
            for i in range(args.warmup + n):
                t0 = time.perf_counter()
                lay = ctx.layerg(prof, nlay=120, laytyp=1, layint=1, angle=30.0)
                print(json.dumps({"profile": what, "call_ms": 1e3 * (time.perf_counter() - t0),
                                  "totam0": float(lay["totam"][0])}))
        elif what == "conv":
            kt, cia, _ = synth.config2()
            job = synth.make_job(kt, synth.ABSORBERS_C2, nlayer=120, seed=1003, nwave=2000, vmr_perturb=0.3)
            vw = job.vwave
            vc = (vw[0] + 5.0 + np.arange(600) * 1.3).astype(np.float32)
            vf = (vw[0] + 10.0 + np.arange(200) * 3.9).astype(np.float32)
            tri = np.array([-1.5, -0.5, 0.0, 0.5, 1.5], np.float32)
            fil = synth.Channels(vconv=vf, vcen=vf, nsub=np.full(200, 5, np.int32), vfil=(vf[:, None] + tri).ravel(),
                                 fil=np.tile(np.array([0.0, 0.6, 1.0, 0.6, 0.0], np.float32), 200))
            ctx.set_ktables(kt)
            ctx.set_cia(cia)
            c, g, gt = ctx.cirsrtfg_wave(job)
            series = np.vstack([c[None], gt[None], g.reshape(job.nv, job.nwave)])
            for i in range(args.warmup + n):
                t0 = time.perf_counter()
                a = ctx.cirsconv_ex(vw, series, 1.2, synth.Channels(vconv=vc))
                b = ctx.cirsconv_ex(vw, series, -1.0, fil)
                print(json.dumps({"profile": what, "call_ms": 1e3 * (time.perf_counter() - t0),
                                  "a0": float(a[0, 0]), "b0": float(b[0, 0])}))


# ---------------------------------------------------------------- main
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--batch-spectra", type=int, default=BATCH_SPECTRA, help="uneven spectra of the batch leg (0 skips)")
    ap.add_argument("--retrievals", type=int, default=RET_N, help="retrievals of the retrieval leg (0 skips)")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving leg")
    ap.add_argument("--profile", choices=["forward", "newton", "aux", "layers", "conv"], default=None,
                    help="run one reduced profiling case instead of the benchmark")
    ap.add_argument("--profile-size", type=int, default=16)
    args = ap.parse_args()
    if args.profile:
        profile_case(args)
        return
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        reference_arm(args, rank)
        return

    if rank == 0 and world == 1:
        from oracle import pyoracle as po
        po.use_native()        # the CPU baseline, built here for this host's CPU, before any GPU work
    import torch
    import torch.distributed as dist

    from radtrancode_b200 import cirsradg, synth
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    kt, cia, _ = synth.config2()
    # weak scaling: every rank its own spectrum (seeded by rank)
    job = synth.make_job(kt, synth.ABSORBERS_C2, nlayer=120, seed=1003 + 7919 * rank, nwave=2000,
                         vmr_perturb=0.3)
    ctx = cirsradg.Context(local)
    ctx.set_ktables(kt)
    ctx.set_cia(cia)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    ctx.prepare([job])
    for _ in range(args.warmup):
        ctx.launch()
    stream.synchronize()

    def barrier():
        if world > 1:
            dist.barrier()

    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        ctx.launch()
    ev1.record(stream)
    stream.synchronize()
    torch.cuda.synchronize()
    barrier()
    ms_total = ev0.elapsed_time(ev1)
    clk = clocks.stop()
    gpu_out = ctx.fetch()[0]
    st = ctx.stats()
    ms_step = ms_total / args.steps
    # e2e through the public C ABI with host buffers (wall clock per call;
    # the call itself waits for its device->host copy)
    ctx.set_stream(None)
    for _ in range(max(1, args.warmup)):
        ctx.cirsrtfg_wave(job)
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        ctx.cirsrtfg_wave(job)
    t_e2e = (time.perf_counter() - t0) / args.steps
    barrier()
    st_e2e = ctx.stats()
    if world > 1:
        tt = torch.tensor([ms_step, t_e2e], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms_step, t_e2e = float(tt[0]), float(tt[1])
    if rank == 0:
        hbm, bf16, how = measured_peaks()
        ab = algorithmic_bytes(kt, job, st_e2e["h2d_bytes"], st_e2e["d2h_bytes"])
        achieved = ab / (ms_step * 1e-3) / 1e9
        prof = profile_data()
        nthr = os.cpu_count() or 1
        elems = st["sort_passes"] * kt.ng * kt.ng
        issue = None
        if prof.get("warp_instructions_per_launch") and clk and clk.get("sm_mhz"):
            ceiling = 148 * 4 * clk["sm_mhz"] * 1e6               # warp instructions/s at 4 per SM per cycle
            got = prof["warp_instructions_per_launch"] / (ms_step * 1e-3)
            issue = {"achieved_warp_inst_per_s": got, "ceiling": ceiling, "frac": got / ceiling,
                     "warp_inst_per_sorted_pass": prof["warp_instructions_per_launch"] / max(1, st["sort_passes"]),
                     "source": "ncu warp instructions of one launch (profiles/fwd_kernel_config2.json), "
                               "ceiling 148 SMs x 4 issues x the sampled SM clock"}
        out = {
            "metric": METRIC, "value": world * 1000.0 / ms_step, "unit": "spectra/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 (f64 g-weight scans)", "data": "synthetic",
            "config": {"workload": WORKLOAD, "spectra_per_step_per_gpu": 1,
                       "l2": "inputs larger than L2: 384 MB of k-tables (raw + ln k) vs 126 MB L2, no flush",
                       "parallelism": f"dp{world} (independent spectra per rank)"},
            "e2e": {"value": world / t_e2e, "unit": "spectra/s", "h2d_bytes_per_step": st_e2e["h2d_bytes"],
                    "d2h_bytes_per_step": st_e2e["d2h_bytes"]},
            "gpu_launches": args.steps,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": achieved / hbm, "traffic": prof.get("dram_bytes_per_launch"),
                         "peak_source": ("measured (MEASURED_PEAKS.json hbm_gbs, burst)" if how == "measured" else
                                         "fallback: the pool's earlier copy measurement (MEASURED_PEAKS.json absent)"),
                         "algorithmic_bytes_per_launch": ab, "kernel": "fwd_kernel"},
            "issue_roofline": issue,
            "sorted_elements_per_s": elems / (ms_step * 1e-3),
            "overlap_passes": {"sorted": st["sort_passes"], "with_ties": st["tie_passes"],
                               "reference_heapsort": st["exact_passes"], "irregular": st["irregular_passes"],
                               "rows_already_sorted": st["block_passes"]},
            "clocks": clk,
        }
        if world == 1:
            out["cpu_baseline"] = cpu_baseline(kt, cia, job, nthr)
            out["accuracy"] = accuracy(kt, cia, [(job, gpu_out)], nthr, "the whole measured spectrum")
            if args.batch_spectra > 0:
                out["batch"] = batch_leg(ctx, kt, cia, args.batch_spectra, nthr)
            if args.retrievals > 0:
                out["retrieval"] = retrieval_leg(ctx, kt, cia, args.retrievals, bf16, hbm, nthr)
            if not args.no_serving:
                out["serving"] = serving_leg(ctx, kt, cia, nthr)
        print(json.dumps(out))
    ctx.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
