"""Benchmark of the B200 CIRSRADG forward model + analytic Jacobian.

Workload (one step): one nadir thermal-emission spectrum of 120 layers,
H2/He + CH4, C2H6, C2H2, NH3 random-overlapped (NG = 20), 2000 wavenumbers,
Jacobian over NX = 124 state elements -- the full-size single-spectrum
configuration.  Inputs are the seeded synthetic workload of
radtrancode_b200/synth.py (the reference measures on no public data set).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

`value`: spectra/s with inputs resident in HBM (CUDA events on the launching
stream around K launches; the k-tables, 384 MB of raw + log k, exceed the
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
import re
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
CPU_SAMPLE_WAVES = 1000       # bounded CPU-baseline sample (half the spectrum)
ACC_SAMPLE_WAVES = 48         # FP64-oracle accuracy sample


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def tensor_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["bf16_tflops"])
    except Exception:
        return 1590.0


def profile_traffic():
    """DRAM bytes per launch of the forward kernel from the committed ncu
    summary (profiles/fwd_kernel_config2.md, line 'dram_bytes_per_launch:')."""
    path = os.path.join(ROOT, "profiles", "fwd_kernel_config2.md")
    try:
        m = re.search(r"dram_bytes_per_launch:\s*([0-9.eE+]+)", open(path).read())
        return float(m.group(1)) if m else None
    except OSError:
        return None


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


def reference_arm(args, rank):
    """The reference's CPU path on the host cores.  No Fortran compiler exists
    here or on the GPU host, so the reference Fortran cannot be built; the
    arm runs the oracle (the C++ restatement of the reference Fortran,
    oracle/) on all host threads, each step a bounded sample of the same
    workload."""
    if rank != 0:
        return
    from oracle import pyoracle as po
    from radtrancode_b200 import synth
    kt, cia, job = synth.config2()
    sample = synth.make_job(kt, synth.ABSORBERS_C2, nlayer=120, seed=1003, iw0=0, nwave=CPU_SAMPLE_WAVES,
                            vmr_perturb=0.3)
    nthr = os.cpu_count() or 1
    for _ in range(args.warmup):
        po.cirsrtfg_wave(kt, cia, synth.make_job(kt, synth.ABSORBERS_C2, nlayer=120, seed=1003, iw0=0,
                                                 nwave=nthr, vmr_perturb=0.3), po.ORC_MIXED, nthreads=nthr)
    times = []
    for _ in range(args.steps):
        t = time.perf_counter()
        po.cirsrtfg_wave(kt, cia, sample, po.ORC_MIXED, nthreads=nthr)
        times.append(time.perf_counter() - t)
    t_step = statistics.mean(times)
    frac = CPU_SAMPLE_WAVES / job.nwave
    value = frac / t_step
    out = {
        "metric": METRIC, "value": value, "unit": "spectra/s", "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_step * 1e3 / frac,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 (f64 transmissions)",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "sample": f"{CPU_SAMPLE_WAVES} of 2000 wavenumbers per step"},
        "cpu_baseline": {"value": value, "unit": "spectra/s", "cores": nthr, "kind": "port",
                         "sample": f"{CPU_SAMPLE_WAVES} of 2000 wavenumbers per step, {nthr} threads; "
                                   "C++ restatement of the reference Fortran (no Fortran compiler on the host)"},
        "e2e": {"value": value, "unit": "spectra/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "gpu_launches": 0,
    }
    print(json.dumps(out))


def cpu_baseline_and_accuracy(kt, cia, job, gpu_out):
    """Rank-0 CPU baseline (oracle port on all host threads, bounded sample)
    and the accuracy of the measured GPU result against the FP64 oracle on a
    sample of the same spectrum."""
    from oracle import pyoracle as po
    from radtrancode_b200 import synth
    nthr = os.cpu_count() or 1
    sample = synth.make_job(kt, synth.ABSORBERS_C2, nlayer=120, seed=1003, iw0=0, nwave=CPU_SAMPLE_WAVES,
                            vmr_perturb=0.3)
    t = time.perf_counter()
    po.cirsrtfg_wave(kt, cia, sample, po.ORC_MIXED, nthreads=nthr)
    dt = time.perf_counter() - t
    base = {"value": (CPU_SAMPLE_WAVES / job.nwave) / dt, "unit": "spectra/s", "cores": nthr, "kind": "port",
            "sample": f"{CPU_SAMPLE_WAVES} of 2000 wavenumbers of the same spectrum, {nthr} threads, "
                      "C++ restatement of the reference Fortran (no Fortran compiler on the host)"}
    stride = job.nwave // ACC_SAMPLE_WAVES
    acc_rad, acc_jac = 0.0, 0.0
    c, g, _ = gpu_out
    G = g.reshape(job.nv, job.nwave)
    for iw0 in range(0, job.nwave, stride * 8):
        sj = synth.make_job(kt, synth.ABSORBERS_C2, nlayer=120, seed=1003, iw0=iw0, nwave=8, vmr_perturb=0.3)
        c64, g64, _ = po.cirsrtfg_wave(kt, cia, sj, po.ORC_FP64, nthreads=min(nthr, 8))
        acc_rad = max(acc_rad, float(np.max(np.abs(c[iw0:iw0 + 8] - c64) / np.abs(c64))))
        R = g64.reshape(job.nv, 8)
        scale = np.maximum(np.max(np.abs(G), axis=1, keepdims=True), 1e-300)
        acc_jac = max(acc_jac, float(np.max(np.abs(G[:, iw0:iw0 + 8] - R) / scale)))
    return base, {"radiance_max_rel_err": acc_rad, "jacobian_max_rel_err": acc_jac,
                  "sample_wavenumbers": len(range(0, job.nwave, stride * 8)) * 8, "vs": "FP64 oracle"}


RET_SAMPLE = 64               # full-size retrievals timed in the default run
RET_FP64_SAMPLE = 16          # of those, re-run with the all-FP64 Newton step
NEWTON_BATCH = 296            # retrievals per timed Newton-step launch (2 per SM)
RET_WORKLOAD = ("optimal-estimation retrievals, full size: NX=124 (120 layer T + 4 log gas scales), NY=2000, "
                "10 Newton iterations max, phlimit 0.1 %, Sa exponential correlation 1.5 scale heights "
                "3 K / 50 %, Se diagonal (1e-9)^2, y = F(x_true) + N(0, 1e-9), x_true ~ N(xa, Sa)")


BATCH_SPECTRA = 1024          # uneven spectra in the batched leg (the 4096 of the batching workload: --batch-spectra)
BATCH_TUNE = 256              # sub-batch the autotuner times


def batch_leg(ctx, kt, nspec):
    """Uneven-spectra batch in one persistent launch: default schedule vs
    the autotuned schedule replayed through a CUDA graph, and the batched
    C-ABI call end to end."""
    from radtrancode_b200 import synth
    jobs = synth.config3_jobs(kt, nspec, seed=1003)
    nwave = sum(j.nwave for j in jobs)
    ctx.prepare(jobs[:BATCH_TUNE])
    tune = ctx.autotune()
    t = time.perf_counter()
    ctx.prepare(jobs)
    t_prep = time.perf_counter() - t

    def timed(n):
        ms = []
        for _ in range(n):
            ctx.launch()
            ctx.fetch()
            ms.append(ctx.stats()["ms_kernel"])
        return ms[-1]
    ctx.set_schedule(0, 0)
    ms_default = timed(2)
    ctx.set_schedule(tune["schedule"], tune["blocks_per_sm"])
    ctx.use_graph(True)
    ms_tuned = timed(3)
    ctx.use_graph(False)
    ctx.set_schedule(0, 0)
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
        "tuned": {"schedule": ["static", "dynamic", "dynamic longest-first"][tune["schedule"]],
                  "blocks_per_sm": tune["blocks_per_sm"], "candidates": tune["candidates"],
                  "tuned_on_spectra": BATCH_TUNE},
        "prepare_s": t_prep,
        "e2e": {"value": nspec / t_e2e, "unit": "spectra/s", "h2d_bytes": st["h2d_bytes"],
                "d2h_bytes": st["d2h_bytes"], "note": "rtb_cirsrtfg_wave_batch with host buffers, default schedule"},
    }


SERVE_RATE = 2000.0           # offered requests/s, Poisson
SERVE_WINDOW = 0.25           # s of arrivals in the default run (the serving workload's 60 s: --serve-window 60)
SERVE_PLAIN = 24              # requests run one at a time for the plain per-request form
SERVE_BUDGET = 16 << 30       # HBM arena of the server


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
    outs = ctx.cirsrtfg_wave_batch([synth.job_at_state(c, c.x_true) for c in cases])
    for i, c in enumerate(cases):
        synth.observe(c, outs[i][0], seed=seed + 7 * i + 2)
    return cases


def serving_leg(ctx, kt, window, rate):
    """Poisson arrivals into the continuous-batching server; latency from
    each request's arrival time to its completion.  Beside it the plain
    per-request GPU form (one retrieval at a time through
    rtb_retrieve_batch)."""
    from radtrancode_b200 import cirsradg
    rng = np.random.default_rng(77)
    arr = np.cumsum(rng.exponential(1.0 / rate, size=int(rate * window * 1.5) + 16))
    arr = arr[arr < window]
    n = len(arr)
    cases = serving_cases(ctx, kt, n)
    lat, its, rounds, peak_active = [], [], 0, 0
    i, pending = 0, {}
    t0 = time.perf_counter()
    with cirsradg.Server(ctx, SERVE_BUDGET, kiter=15, phlimit=0.1, dchisq_stop=0.1) as srv:
        while i < n or pending:
            now = time.perf_counter() - t0
            while i < n and arr[i] <= now:
                pending[srv.submit(cases[i])] = arr[i]
                i += 1
            if not pending:
                time.sleep(max(0.0, arr[i] - now))
                continue
            active, _ = srv.step()
            rounds += 1
            peak_active = max(peak_active, active)
            t = time.perf_counter() - t0
            for rid in list(pending):
                r = srv.poll(rid)
                if r is not None:
                    lat.append((t - pending.pop(rid)) * 1e3)
                    its.append(r["iterations"])
    t_total = time.perf_counter() - t0
    plain = []
    t = time.perf_counter()
    for c in cases[:SERVE_PLAIN]:
        t1 = time.perf_counter()
        ctx.retrieve_batch([c], kiter=15, phlimit=0.1, dchisq_stop=0.1)
        plain.append((time.perf_counter() - t1) * 1e3)
    t_plain = time.perf_counter() - t
    lat = np.array(lat)
    return {
        "workload": f"Poisson arrivals at {rate:.0f} req/s for {window} s ({n} requests), sizes of the uneven batch, "
                    "up to 15 Newton iterations, early exit at |delta chi2| < 0.1, HBM budget "
                    f"{SERVE_BUDGET >> 30} GiB",
        "requests": n, "value": n / t_total, "unit": "retrievals/s", "wall_s": t_total, "rounds": rounds,
        "peak_in_flight": peak_active,
        "p50_ms": float(np.percentile(lat, 50)), "p95_ms": float(np.percentile(lat, 95)),
        "p99_ms": float(np.percentile(lat, 99)), "iterations_mean": float(np.mean(its)),
        "latency_note": "from the request's arrival time; the offered rate is above the service rate, so "
                        "latency includes the wait for the backlog",
        "plain_per_request": {"requests": SERVE_PLAIN, "value": SERVE_PLAIN / t_plain, "unit": "retrievals/s",
                              "p50_ms": float(np.percentile(plain, 50)), "p99_ms": float(np.percentile(plain, 99)),
                              "note": "one request at a time, rtb_retrieve_batch of one, service time only"},
    }


def retrieval_cases(ctx, kt, n, seed0=4000):
    """Full-size retrieval cases; observations from the device forward model
    at the true states (one batched launch) plus seeded noise."""
    from radtrancode_b200 import synth
    cases = [synth.make_retrieval(kt, synth.ABSORBERS_C2, nlayer=120, seed=seed0 + 17 * i, nwave=2000)
             for i in range(n)]
    outs = ctx.cirsrtfg_wave_batch([synth.job_at_state(c, c.x_true) for c in cases])
    for i, c in enumerate(cases):
        synth.observe(c, outs[i][0], seed=seed0 + 17 * i + 1)
    return cases, outs


def retrieval_leg(ctx, kt, cia, bf16_peak):
    """Retrievals/s and completion-time percentiles of the batched engine
    (rtb_retrieve_batch), the mixed-precision result against the all-FP64
    device solve, the Newton kernel against the tensor peak, and the oracle
    retrieval on the host cores."""
    from oracle import pyoracle as po
    cases, outs = retrieval_cases(ctx, kt, RET_SAMPLE)
    ctx.set_newton_mode(0, 1)
    t = time.perf_counter()
    res = ctx.retrieve_batch(cases, kiter=10, phlimit=0.1)
    dt = time.perf_counter() - t
    lat = np.array([r["ms"] for r in res])
    ctx.set_newton_mode(1, 0)
    try:
        res64 = ctx.retrieve_batch(cases[:RET_FP64_SAMPLE], kiter=10, phlimit=0.1)
    finally:
        ctx.set_newton_mode(0, 1)
    dx, same = 0.0, 0
    for c, a, b in zip(cases, res, res64):
        sig = np.sqrt(np.diag(c.sa))
        dx = max(dx, float(np.max(np.abs(a["x"] - b["x"]) / sig)))
        same += int(a["iterations"] == b["iterations"] and a["converged"] == b["converged"])
    # Newton-step kernel alone: NEWTON_BATCH retrievals of K at the true states
    pick = [i % RET_SAMPLE for i in range(NEWTON_BATCH)]
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
    # the oracle's retrieval on the host cores: one case, all threads
    nthr = os.cpu_count() or 1
    t = time.perf_counter()
    po.retrieve(kt, cia, cases[0], kiter=10, phlimit=0.1, nthreads=nthr)
    t_cpu = time.perf_counter() - t
    return {
        "workload": RET_WORKLOAD, "retrievals": RET_SAMPLE, "value": RET_SAMPLE / dt, "unit": "retrievals/s",
        "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
        "latency_note": "completion time from the start of the batched call (all admitted at once)",
        "iterations_mean": float(np.mean([r["iterations"] for r in res])),
        "forwards_mean": float(np.mean([r["forwards"] for r in res])),
        "converged": int(sum(r["converged"] > 0 for r in res)),
        "newton": {"hessian": "bf16 hi/lo split on tensor cores (mma.sync m16n8k16), FP32 accumulation, "
                              "1 FP64 refinement step; FP64 Cholesky",
                   "vs_fp64_solve": {"retrievals": RET_FP64_SAMPLE, "max_dx_over_prior_sigma": dx,
                                     "same_iterations_and_stop_rule": same}},
        "newton_kernel": {"batch": NEWTON_BATCH, "ms": ms_n, "achieved_tflops": tflops, "peak_tflops": bf16_peak,
                          "frac": tflops / bf16_peak, "flops_per_retrieval": "2 NX^2 NY + 2 NX NY"},
        "cpu_baseline": {"value": 1.0 / t_cpu, "unit": "retrievals/s", "cores": nthr, "kind": "port",
                         "sample": f"1 retrieval of the same workload, oracle coreret restatement, {nthr} threads"},
    }


def profile_case(args):
    """Reduced case for ncu captures: the same spectrum cut to its first
    `--profile-waves` wavenumbers, warm-up + `--steps` launches."""
    from radtrancode_b200 import cirsradg, synth
    kt, cia, _ = synth.config2()
    job = synth.make_job(kt, synth.ABSORBERS_C2, nlayer=120, seed=1003, nwave=args.profile_waves, vmr_perturb=0.3)
    with cirsradg.Context(0) as ctx:
        ctx.set_ktables(kt)
        ctx.set_cia(cia)
        ctx.prepare([job])
        for _ in range(args.warmup + args.steps):
            ctx.launch()
            ctx.fetch()
            print(json.dumps({"profile_waves": args.profile_waves, "ms_kernel": ctx.stats()["ms_kernel"]}))


def profile_newton(args):
    """Reduced case for ncu captures of the Newton-step kernel:
    `--profile-newton` full-size retrievals (NX=124, NY=2000) with seeded
    K of the forward model's magnitude, warm-up + `--steps` launches."""
    from radtrancode_b200 import cirsradg, synth
    n, nx, ny = args.profile_newton, 124, 2000
    rng = np.random.default_rng(11)
    p_lev, p_lay = synth._levels(120)
    sa = synth.prior_covariance(p_lay, 4)
    sai = np.broadcast_to(np.linalg.inv(sa), (n, nx, nx))
    kk = (rng.standard_normal((n, nx, ny)) * 1e-9).astype(np.float32)
    sei = np.full((n, ny), 1e18)
    xa = np.full((n, nx), 150.0, np.float32)
    y = (rng.standard_normal((n, ny)) * 1e-8).astype(np.float32)
    yn = np.zeros((n, ny), np.float32)
    with cirsradg.Context(0) as ctx:
        for _ in range(args.warmup + args.steps):
            ctx.newton_step_batch(kk, sei, sai, xa, xa, y, yn)
            print(json.dumps({"profile_newton": n, "ms_kernel": ctx.newton_stats()["ms_kernel"]}))


def profile_aux(args):
    """Reduced case for ncu captures of the small kernels of the Newton-step
    interface: `--profile-aux` retrievals (NX=124, NY=2000) through
    calc_phiret, the Sa inverse, then one calc_gain_matrix + calcnextxn."""
    from radtrancode_b200 import cirsradg, synth
    n, nx, ny = args.profile_aux, 124, 2000
    rng = np.random.default_rng(12)
    p_lev, p_lay = synth._levels(120)
    sa = synth.prior_covariance(p_lay, 4)
    sai1 = np.linalg.inv(sa)
    sai = np.broadcast_to(sai1, (n, nx, nx))
    sei = np.full((n, ny), 1e18)
    xa = np.full((n, nx), 150.0, np.float32)
    xn = xa + rng.standard_normal((n, nx)).astype(np.float32)
    y = (rng.standard_normal((n, ny)) * 1e-8).astype(np.float32)
    yn = np.zeros((n, ny), np.float32)
    kk = (rng.standard_normal((nx, ny)) * 1e-9).astype(np.float32)
    with cirsradg.Context(0) as ctx:
        for _ in range(args.warmup + args.steps):
            phi, _ = ctx.calc_phiret_batch(y, yn, sei, xn, xa, sai)
            ctx.spd_inverse_batch(np.broadcast_to(sa, (n, nx, nx)))
            dd, aa, _ = ctx.calc_gain_matrix(kk, sai1, sei[0])
            x = ctx.calcnextxn(xa[0], xn[0], y[0], yn[0], dd, aa)
            print(json.dumps({"profile_aux": n, "phi0": float(phi[0]), "x0": float(x[0])}))


def profile_layers(args):
    """Reduced case for ncu captures of the layering kernel: `--profile-layers`
    calls of rtb_layerg on a 121-level, 6-gas profile into 120 Curtis-Godson
    layers on a 30-degree path (the full-size atmosphere), after warm-up."""
    from radtrancode_b200 import cirsradg, synth
    prof = synth.make_profile(synth.ABSORBERS_C2, npro=121, seed=1005)
    with cirsradg.Context(0) as ctx:
        for i in range(args.warmup + args.profile_layers):
            t0 = time.perf_counter()
            lay = ctx.layerg(prof, nlay=120, laytyp=1, layint=1, angle=30.0)
            print(json.dumps({"profile_layers": i, "call_ms": 1e3 * (time.perf_counter() - t0),
                              "totam0": float(lay["totam"][0])}))


def profile_conv(args):
    """Reduced case for ncu captures of the convolution kernels: the
    full-size spectrum's radiance, d/dtsurf and 124 Jacobian rows (126 series
    of 2000 points) convolved `--profile-conv` times onto 600 square-bin
    channels (FWHM 1.2 cm-1) and onto 200 filter channels (FWHM < 0)."""
    from radtrancode_b200 import cirsradg, synth
    kt, cia, _ = synth.config2()
    job = synth.make_job(kt, synth.ABSORBERS_C2, nlayer=120, seed=1003, nwave=2000, vmr_perturb=0.3)
    vw = job.vwave
    vc = (vw[0] + 5.0 + np.arange(600) * 1.3).astype(np.float32)
    vf = (vw[0] + 10.0 + np.arange(200) * 3.9).astype(np.float32)
    tri = np.array([-1.5, -0.5, 0.0, 0.5, 1.5], np.float32)
    fil = synth.Channels(vconv=vf, vcen=vf, nsub=np.full(200, 5, np.int32), vfil=(vf[:, None] + tri).ravel(),
                         fil=np.tile(np.array([0.0, 0.6, 1.0, 0.6, 0.0], np.float32), 200))
    with cirsradg.Context(0) as ctx:
        ctx.set_ktables(kt)
        ctx.set_cia(cia)
        c, g, gt = ctx.cirsrtfg_wave(job)
        series = np.vstack([c[None], gt[None], g.reshape(job.nv, job.nwave)])
        for i in range(args.warmup + args.profile_conv):
            t0 = time.perf_counter()
            a = ctx.cirsconv_ex(vw, series, 1.2, synth.Channels(vconv=vc))
            b = ctx.cirsconv_ex(vw, series, -1.0, fil)
            print(json.dumps({"profile_conv": i, "call_ms": 1e3 * (time.perf_counter() - t0),
                              "a0": float(a[0, 0]), "b0": float(b[0, 0])}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--profile-waves", type=int, default=0,
                    help="profiling case: only launch the forward kernel on the first N wavenumbers of the "
                         "workload (steps launches after warmup), print the kernel time, skip e2e and baselines")
    ap.add_argument("--no-retrieval", action="store_true", help="skip the retrieval leg")
    ap.add_argument("--serve-window", type=float, default=SERVE_WINDOW,
                    help="seconds of Poisson arrivals in the serving leg (0 skips it)")
    ap.add_argument("--batch-spectra", type=int, default=BATCH_SPECTRA,
                    help="uneven spectra in the batched leg (0 skips it)")
    ap.add_argument("--profile-newton", type=int, default=0,
                    help="profiling case: only the Newton-step kernel on N full-size retrievals")
    ap.add_argument("--profile-aux", type=int, default=0,
                    help="profiling case: the small kernels of the Newton-step interface on N retrievals")
    ap.add_argument("--profile-layers", type=int, default=0,
                    help="profiling case: N calls of the layering kernel on the full-size profile")
    ap.add_argument("--profile-conv", type=int, default=0,
                    help="profiling case: N convolutions of a full-size spectrum's outputs")
    args = ap.parse_args()
    if args.profile_layers:
        profile_layers(args)
        return
    if args.profile_conv:
        profile_conv(args)
        return
    if args.profile_aux:
        profile_aux(args)
        return
    if args.profile_waves:
        profile_case(args)
        return
    if args.profile_newton:
        profile_newton(args)
        return
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        reference_arm(args, rank)
        return

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
        hbm, how = peaks()
        ab = algorithmic_bytes(kt, job, st_e2e["h2d_bytes"], st_e2e["d2h_bytes"])
        achieved = ab / (ms_step * 1e-3) / 1e9
        traffic = profile_traffic()
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
                         "frac": achieved / hbm, "traffic": traffic,
                         "peak_source": ("measured (MEASURED_PEAKS.json hbm_gbs, burst)" if how == "measured" else
                                         "fallback: the pool's earlier copy measurement (MEASURED_PEAKS.json absent)"),
                         "algorithmic_bytes_per_launch": ab, "kernel": "fwd_kernel"},
            "overlap_passes": {"sorted": st["sort_passes"], "with_ties": st["tie_passes"],
                               "reference_heapsort": st["exact_passes"], "irregular": st["irregular_passes"]},
            "clocks": clk,
        }
        if world == 1:
            base, acc = cpu_baseline_and_accuracy(kt, cia, job, gpu_out)
            out["cpu_baseline"] = base
            out["accuracy"] = acc
            if args.batch_spectra > 0:
                out["batch"] = batch_leg(ctx, kt, args.batch_spectra)
            if not args.no_retrieval:
                out["retrieval"] = retrieval_leg(ctx, kt, cia, tensor_peak())
            if args.serve_window > 0:
                out["serving"] = serving_leg(ctx, kt, args.serve_window, SERVE_RATE)
        print(json.dumps(out))
    ctx.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
