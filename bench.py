#!/usr/bin/env python
"""Benchmark of the posterior unit: posterior cells/s at 256x256x512, 5 angles.

One step = one posterior unit on one seeded synthetic case (the timed unit of
the reference: forward transforms of 3 means, 5 stacks, 6 prior covariances
and the noise correlation; the per-(kx,ky,kz) solve; inverse transforms of 3
posterior means, 5 residuals and 6 posterior covariances).
posterior cells/s = nxp*nyp*nzp / step time.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl crava_b200|reference]

Own arm: inputs resident in HBM (2.0 GB per step, larger than L2), outputs
written out of place so each step reads pristine inputs; device time with
CUDA events over K steps, max over ranks.  `e2e` runs the same unit through
crava_gpu_posterior_unit_host with pinned host buffers (copies timed).
Reference arm: the reference's own CPU code (FFTW 2.1.2 + lib_matr.c,
oracle/_ref) on the host cores: forked processes, each timing whole units
of the same workload; value = units x cells / wall time of the timed phase.
Multi-GPU (torchrun): every rank runs its own independent unit (weak
scaling, no collective on the data path).

  python bench.py --profile-unit NX,NY,NZ [--profile-precision 0|1|2]
                  [--profile-fused 0|1] [--profile-reps R] [--profile-ntheta NT]

runs the out-of-place unit R times on a seeded case and prints per-kernel
device times (CUDA events around every launch); used for ncu captures of
single kernel families on small cases.
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

METRIC = "posterior cells/s at 256x256x512x5 angles, mixed vs FP64 form; % HBM roofline"
ANGLES5 = (0.0, 10.0, 20.0, 30.0, 40.0)


FP64_NOMINAL_TFLOPS = 148 * 128 * 1.965e9 / 1e12


def solve_flops_per_inverted_bin(nt):
    """FP64 flops of the square-root form on one inverted bin (an FMA counts
    2): M built from the per-kz constants (A S rows, (A S A^T)_lm, the
    complex W_lm B + lambda E_lm), the Cholesky, four forward substitutions
    (three columns of K S and z), the columns of K S, the Gram entries of
    S - Y^H Y, the prior-mean residual, Y^H z and the posterior mean and
    residual."""
    npair = nt * (nt + 1) // 2
    build = 15 * nt + 5 * npair + 6 * npair + nt
    chol = sum(8 * j + 2 for i in range(nt) for j in range(i)) + sum(4 * i + 2 for i in range(nt))
    fwd = 8 * nt * (nt - 1) // 2 + 2 * nt
    gram = 3 * 4 * nt + (1 + 2) * 8 * nt
    return build + chol + 4 * fwd + 3 * 7 * nt + gram + 20 * nt + 3 * 8 * nt + (6 + 20 * nt)


def wb_flops_per_inverted_bin(nt):
    """FP64 flops of the Woodbury form on one inverted bin (an FMA counts
    2): the prior-mean residual d - K mu, t = T r with the per-plane
    whitening T, the weights c_i = 1 / (lambda m_i + 1), g = W^H diag(c) t,
    P = sum_i c_i H_i, the 3x3 prior Cholesky, Q = LS^T P LS, the 3x3
    complex Cholesky of I + Q, Z = R^-1 LS^T, S_post = Z^H Z, the mean
    update S_post g and the residual."""
    return 8 * nt * nt + 87 * nt + 403


def hbm_peak():
    """(GB/s, source): the measured copy bandwidth of MEASURED_PEAKS.json
    (written per pod by the driver), else the pool's earlier measurement."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            v = json.load(f).get("hbm_gbs")
        if v:
            return float(v), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except Exception:
        pass
    return 6650.0, "fallback 6650 GB/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="crava_b200", choices=["crava_b200", "reference"])
    # the plain method (FP64 per-frequency solves) is the full-size workload;
    # the other form (mixed FP32 + FP64 refinement) is timed beside it
    ap.add_argument("--precision", default="fp64", choices=["mixed", "fp64", "fp32"])
    ap.add_argument("--grid", default="256,256,512")
    ap.add_argument("--noise", type=float, default=0.10)
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64-compare", "--no-form-compare", dest="no_fp64_compare", action="store_true",
                    help="skip timing the other solve form (mixed when the headline is FP64, else FP64)")
    ap.add_argument("--no-simulation", action="store_true")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-forward", action="store_true")
    ap.add_argument("--no-state4d", action="store_true")
    ap.add_argument("--no-divide", action="store_true")
    ap.add_argument("--split-grid", action="store_true",
                    help="with several ranks, also time one grid split over them (z slabs <-> column shards)")
    ap.add_argument("--no-split-grid", action="store_true")
    ap.add_argument("--batch-sims", type=int, default=64)
    ap.add_argument("--workers", type=int, default=0, help="reference arm processes (0 = auto)")
    ap.add_argument("--profile-unit", default=None, metavar="NX,NY,NZ",
                    help="per-kernel timing of the unit on a small case (for ncu captures), then exit")
    ap.add_argument("--profile-precision", type=int, default=0, help="0 FP64, 1 mixed, 2 reference FP32")
    ap.add_argument("--profile-fused", type=int, default=0)
    ap.add_argument("--profile-reps", type=int, default=3)
    ap.add_argument("--profile-ntheta", type=int, default=5)
    ap.add_argument("--profile-lanes", type=int, default=1,
                    help="transform streams in the profile run (1: per-launch events time one kernel each)")
    ap.add_argument("--profile-xy", type=int, default=-1, help="fused x + y pass: -1 built-in, 0 off, 1 on")
    ap.add_argument("--profile-fft", default=None, metavar="NX,NY,NZ",
                    help="per-pass timing of the forward and inverse transform of one grid, then exit")
    ap.add_argument("--profile-tile-z", type=int, default=None,
                    help="z pass: -1 built-in, 1 register-resident, 2 register-resident with TMA tile loads")
    return ap.parse_args()


# ----------------------------------------------------------------- CPU reference unit
def cpu_unit_seconds(case, which="ref"):
    """One whole posterior unit of the reference's CPU path on this core:
    29 FFTW 2.1.2 transforms, each planned per call as FFTGrid does
    (src/fftgrid.cpp:1822-1825), and the per-bin loop with lib_matr.c
    (src/crava.cpp:1042-1151) -- oracle/_ref, or the restatement when the
    reference build is absent.  Returns (seconds, failed bins)."""
    from oracle import oracle as O

    t0 = time.perf_counter()
    out = O.unit_fp32(case, which)
    return time.perf_counter() - t0, out[3]


_REF_CASE = None
_REF_BARRIER = None


def _ref_worker(args):
    """One reference-arm process: `warm` untimed units, then `units` timed
    units on the case inherited from the parent (fork).  Returns the timed
    seconds and the wall-clock span of the timed phase."""
    warm, units = args
    for _ in range(warm):
        cpu_unit_seconds(_REF_CASE)
    _REF_BARRIER.wait(timeout=900)  # every process starts its timed units together
    t0 = time.time()
    per = [cpu_unit_seconds(_REF_CASE)[0] for _ in range(units)]
    return per, t0, time.time()


# ----------------------------------------------------------------- clocks
class ClockSampler:
    """SM clock, max clock and throttle reasons sampled every 20 ms through
    NVML in a thread while the timed region runs (read-only queries); falls
    back to `nvidia-smi -lms` when NVML is not importable."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = (("sw_power_cap", 0x4), ("hw_slowdown", 0x8), ("sw_thermal_slowdown", 0x20),
               ("hw_thermal_slowdown", 0x40), ("hw_power_brake_slowdown", 0x80))

    def __init__(self, device_index):
        self.dev = device_index
        self.samples = []
        self.thread = None
        self.proc = None

    def _nvml_handle(self):
        import pynvml as N
        import torch

        N.nvmlInit()
        try:
            uuid = str(torch.cuda.get_device_properties(self.dev).uuid)
            if not uuid.startswith("GPU-"):
                uuid = "GPU-" + uuid
            return N, N.nvmlDeviceGetHandleByUUID(uuid)
        except Exception:
            return N, N.nvmlDeviceGetHandleByIndex(self.dev)

    def start(self):
        import threading

        try:
            N, h = self._nvml_handle()
        except Exception:
            return self._start_smi()
        reasons_fn = getattr(N, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            N.nvmlDeviceGetCurrentClocksThrottleReasons
        mx = N.nvmlDeviceGetMaxClockInfo(h, N.NVML_CLOCK_SM)
        self.stop_flag = threading.Event()

        def sample():
            self.samples.append((N.nvmlDeviceGetClockInfo(h, N.NVML_CLOCK_SM), mx, int(reasons_fn(h))))

        sample()

        def loop():
            while not self.stop_flag.wait(0.02):
                try:
                    sample()
                except Exception:
                    break

        self.thread = threading.Thread(target=loop, daemon=True)
        self.thread.start()

    def _start_smi(self):
        import time as _t

        try:
            self.path = tempfile.mktemp(prefix="crava_clocks_", suffix=".csv")
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100", "-i", str(self.dev)], stdout=self.f, stderr=subprocess.DEVNULL)
            t0 = _t.time()
            while _t.time() - t0 < 5 and os.path.getsize(self.path) == 0:
                _t.sleep(0.05)
        except Exception:
            self.proc = None

    def stop(self):
        if self.thread is not None:
            self.stop_flag.set()
            self.thread.join(timeout=5)
            sm = [x[0] for x in self.samples]
            reasons = sorted({n for _, _, r in self.samples for n, bit in self.REASONS if r & bit})
            return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(x[1] for x in self.samples),
                    "reasons": reasons, "samples": len(sm), "source": "nvml"}
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    mx.append(float(parts[2]))
                except ValueError:
                    continue
                for n, v in zip(names, parts[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(n)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm), "source": "nvidia-smi"}


# ----------------------------------------------------------------- own arm
VINTAGES = [(128, 128, 256), (192, 160, 384), (256, 256, 512), (96, 200, 300)]


def run_batch(args, case256, dev, stream, max_over_ranks):
    """Time-lapse batch: four vintages of uneven size, 5 angles each, every
    run = posterior unit + nsim realisations per vintage, replayed as one
    CUDA graph launch (launch shapes autotuned per vintage first)."""
    import torch

    from crava_b200 import api, synth

    R = args.batch_sims
    vint, ctxs = [], []
    cells = 0
    for k, shp in enumerate(VINTAGES):
        c = case256 if (case256 is not None and shp == (256, 256, 512)) else \
            synth.make_case(*shp, ANGLES5, args.noise, seed=40 + k, wavelet_scale_range=(0.8, 1.2))
        ctx = api.Context(c, device=dev, stream=stream, precision=api.MIXED)
        d = lambda gs: [api.to_device(g, dev) for g in gs]
        src = (d(c.mu), d(c.data), d(c.cov), d([c.err_corr])[0])
        dst = (d(c.mu), d(c.data), d(c.cov), d([c.err_corr])[0])
        sims = [torch.empty_like(src[0][0]) for _ in range(3 * R)]
        vint.append(dict(ctx=ctx, src=src, dst=dst, precision=api.MIXED, nsim=R, seed=100 + k,
                         first_index=0, sims=sims))
        ctxs.append(ctx)
        cells += shp[0] * shp[1] * shp[2]

    def timed(b, runs):
        for _ in range(2):
            b.run()
        b.sync()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        n0 = api.launch_count()
        for _ in range(runs):
            b.run()
        ev1.record(stream)
        b.sync()
        torch.cuda.synchronize(dev)
        return max_over_ranks(ev0.elapsed_time(ev1) / runs), (api.launch_count() - n0) // runs

    g = api.Batch(vint, api.BATCH_AUTOTUNE, stream=stream)
    tunings = [{"cols_y_tile": t.cols_y_tile, "cols_z_tile": t.cols_z_tile, "fused": t.fused, "lanes": t.lanes}
               for t in (ctx.tuning() for ctx in ctxs)]
    ms_graph, kern = timed(g, 5)
    g.close()
    e = api.Batch(vint, api.BATCH_NO_GRAPH, stream=stream)
    ms_eager, _ = timed(e, 3)
    e.close()
    for ctx in ctxs:
        ctx.close()
    del vint
    torch.cuda.empty_cache()
    return {"workload": "vintages %s x 5 angles, mixed solve, %d realisations each, one graph launch per run"
                        % (["x".join(map(str, v)) for v in VINTAGES], R),
            "ms_per_run": ms_graph, "ms_per_run_eager": ms_eager,
            "cells_per_s": cells / (ms_graph * 1e-3),
            "realisations_per_s": len(VINTAGES) * R / (ms_graph * 1e-3),
            "kernels_per_run": kern, "tuning": tunings}


def run_prior_fill(ctx, case, dst, dev, stream, max_over_ranks):
    """The six prior covariance grids and the noise correlation grid built on
    the device (fillInParamCorr x Sigma0, fillInErrCorr) instead of uploaded:
    device time per set and the HBM rate of its 7 grid writes."""
    import numpy as np
    import torch

    from crava_b200 import api, synth

    cxy = synth.corr_xy(case.nxp, case.nyp, 25.0, 25.0, 500.0)
    circ = synth.circ_corr_t(case.nzp, case.dt, 20.0, case.low_cut)
    cov, err = dst[2], dst[3]

    def once():
        ctx.fill_prior_cov(cxy, circ, 0.0, 0.0, cov)
        ctx.fill_err_corr(cxy, 0.0, 0.0, err)

    for _ in range(3):
        once()
    torch.cuda.synchronize(dev)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    reps = 10
    ev0.record(stream)
    for _ in range(reps):
        once()
    ev1.record(stream)
    torch.cuda.synchronize(dev)
    ms = max_over_ranks(ev0.elapsed_time(ev1) / reps)
    same = all(np.array_equal(g.cpu().numpy()[..., :case.nxp], h[..., :case.nxp])
               for g, h in zip(cov, case.cov))
    gbytes = 7 * cov[0].numel() * 4
    return {"workload": "6 prior covariance grids + noise correlation, %dx%dx%d"
                        % (case.nxp, case.nyp, case.nzp),
            "ms_per_set": ms, "GB/s": gbytes / (ms * 1e-3) / 1e9,
            "equal_to_uploaded_grids": same}


def run_state4d(ctx, case, dev, stream, max_over_ranks, peak):
    """The time-lapse state (State4D split / evolve / merge and the whole
    ModelGeneral::advanceTime step) on 27 state grids of the unit's size:
    device time per kernel and its HBM rate on the algorithmic bytes
    (split reads 36 and writes 27 spectra per bin, evolve reads 28 and
    writes 27, merge reads 27 and writes 9; 8 bytes each)."""
    import numpy as np
    import torch

    from crava_b200 import api

    nxp, nyp, nzp = case.nxp, case.nyp, case.nzp
    shape = (nzp, nyp, 2 * (nxp // 2 + 1))
    bins = shape[0] * shape[1] * shape[2] // 2
    gen = torch.Generator(device=dev).manual_seed(5)
    P, Q = (0, 0, 0, 1, 1, 2), (0, 1, 2, 1, 2, 2)
    unit = (0, 3, 4, 1, 5, 2)
    rng = np.random.default_rng(5)
    G = rng.standard_normal((6, 6))
    S0 = G @ G.T / 6.0 + 0.5 * np.eye(6)
    E = np.eye(6) + 0.05 * rng.standard_normal((6, 6))
    cm = rng.standard_normal(6)
    Gc = rng.standard_normal((6, 6))
    cc = Gc @ Gc.T / 6.0 + 0.1 * np.eye(6)
    with torch.cuda.stream(stream):
        lam = torch.empty(shape, device=dev)
        ctx.fill_gen_exp_corr(nxp / 4.0, nyp / 4.0, 6.0, 0.0, 0.0, lam)
        ctx.fft_r2c(lam, api.COVARIANCE)

        def field():
            g = torch.randn(shape, device=dev, generator=gen)
            ctx.fft_r2c(g, api.PARAMETER)
            return g

        state = {"ms": [field() for _ in range(3)], "md": [field() for _ in range(3)],
                 "ss": [lam * float(S0[P[r], Q[r]]) for r in range(6)],
                 "dd": [lam * float(S0[P[r] + 3, Q[r] + 3]) for r in range(6)],
                 "sd": [lam * float(S0[l, k + 3]) for l in range(3) for k in range(3)]}
        C = S0[:3, :3] + S0[3:, 3:] + S0[3:, :3] + S0[:3, 3:]
        mu = [field() for _ in range(3)]
        cov = [None] * 6
        for r in range(6):
            cov[unit[r]] = lam * float(0.6 * C[P[r], Q[r]])
        work = torch.empty(shape, device=dev)
    torch.cuda.synchronize(dev)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)

    def timed(fn, reps=5):
        for _ in range(2):
            fn()
        torch.cuda.synchronize(dev)
        ev0.record(stream)
        for _ in range(reps):
            fn()
        ev1.record(stream)
        torch.cuda.synchronize(dev)
        return max_over_ranks(ev0.elapsed_time(ev1) / reps)

    shortcuts = ctx.state4d_split(state, mu, cov)
    res = {}
    for name, fn, nb in [("split", lambda: ctx.state4d_split(state, mu, cov), 63),
                         ("evolve", lambda: ctx.state4d_evolve(state, E, cm, cc, lam), 55),
                         ("merge", lambda: ctx.state4d_merge(state, mu, cov), 36)]:
        ms = timed(fn)
        gbs = nb * 8 * bins / (ms * 1e-3) / 1e9
        res[name] = {"ms": round(ms, 4), "bytes_per_launch": nb * 8 * bins, "GB/s": round(gbs, 1),
                     "frac_of_peak": round(gbs / peak, 4)}
    # split runs synchronously (it reads back its shortcut count); time the
    # whole step through advance_time, which also reads it back once
    step_ms = timed(lambda: ctx.advance_time(state, 1, nxp, nyp, E, cm, cc, mu, cov, work), reps=3)
    del state, mu, cov, work, lam
    return {"workload": "State4D split / evolve / merge and advanceTime, 27 state grids %dx%dx%d"
                        % (nxp, nyp, nzp),
            "kernels": res, "advance_time_ms": round(step_ms, 4), "split_shortcut_bins": shortcuts,
            "peak_GB/s": peak}


def run_divide(ctx, case, src, dev, stream, max_over_ranks, peak):
    """Crava::divideDataByScaleWavelet (non-constant thickness) on all angle
    stacks: device time per call; the HBM rate counts each stack read and
    written once (the algorithmic minimum of the per-trace filter)."""
    import numpy as np
    import torch

    nxp, nyp, nzp = case.nxp, case.nyp, case.nzp
    data = [g.clone() for g in src[1]]
    rng = np.random.default_rng(9)
    rt = rng.uniform(0.8, 1.2, (nyp, nxp))
    nz = case.nz
    dz = float(np.float32(case.lz / nz))

    def once():
        ctx.divide_data_by_scale_wavelet(data, src[2][0], rt, nxp, nyp, dz)

    # every call starts from the original stacks (copied outside the timed
    # region): the division is not idempotent
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    reps, total = 5, 0.0
    for rep in range(2 + reps):
        with torch.cuda.stream(stream):
            for d, s0 in zip(data, src[1]):
                d.copy_(s0)
        torch.cuda.synchronize(dev)
        ev0.record(stream)
        once()
        ev1.record(stream)
        torch.cuda.synchronize(dev)
        if rep >= 2:
            total += ev0.elapsed_time(ev1)
    ms = max_over_ranks(total / reps)
    nbytes = 2 * len(data) * data[0].numel() * 4
    gbs = nbytes / (ms * 1e-3) / 1e9
    del data
    return {"workload": "divideDataByScaleWavelet, %d stacks %dx%dx%d" % (case.ntheta, nxp, nyp, nzp),
            "ms_per_call": round(ms, 4), "GB/s": round(gbs, 1), "frac_of_peak": round(gbs / peak, 4),
            "passes": "per stack one pass over HBM at z lengths 128/256/512 (taper, z transform, "
                      "per-trace filter, inverse z transform, scale in one kernel); five passes otherwise"}


def run_split(case, world, rank, dist, dev, stream, max_over_ranks, prec):
    """One posterior unit with its grids split over the ranks (z slabs for
    the x and y passes, column shards for the z pass and the solve, one
    exchange each way; crava_b200.dist_grid): device time per unit, max
    over ranks, on pristine inputs every repetition."""
    import numpy as np
    import torch

    from crava_b200 import api
    from crava_b200 import dist_grid as G

    lay = G.Layout(case.nxp, case.nyp, case.nzp, world)
    G.check_layout(lay)
    z0, z1 = lay.z(rank)
    y0, y1 = lay.y(rank)
    cs = api.Context(G.shard_case(case, nzp=z1 - z0), device=dev, stream=stream, precision=prec)
    cc = api.Context(G.shard_case(case, nyp=y1 - y0), device=dev, stream=stream, precision=prec)
    ops = G.device_ops(cs, cc, prec, case.nzp)
    nt = case.ntheta
    with torch.cuda.stream(stream):
        src = [torch.from_numpy(np.ascontiguousarray(g[z0:z1])).to(dev) for g in case.grids()]
        work = [torch.empty_like(g) for g in src]
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    reps, total = 5, 0.0
    for rep in range(2 + reps):
        with torch.cuda.stream(stream):
            for w, s0 in zip(work, src):
                w.copy_(s0)
        torch.cuda.synchronize(dev)
        if dist is not None:
            dist.barrier()
        with torch.cuda.stream(stream):
            ev0.record(stream)
            G.posterior_unit_split(ops, lay, rank, dist, work[:3], work[3:3 + nt], work[3 + nt:9 + nt],
                                   work[9 + nt])
            ev1.record(stream)
        torch.cuda.synchronize(dev)
        if rep >= 2:
            total += ev0.elapsed_time(ev1)
    ms = max_over_ranks(total / reps)
    cells = case.nxp * case.nyp * case.nzp
    grid_bytes = case.mu[0].nbytes
    out_bytes = (10 + nt) * grid_bytes * (world - 1) / world
    back_bytes = (9 + nt) * grid_bytes * (world - 1) / world
    cs.close()
    cc.close()
    del src, work
    return {"workload": "one posterior unit %dx%dx%d, 5 angles, split over %d rank(s)"
                        % (case.nxp, case.nyp, case.nzp, world),
            "ranks": world, "ms_per_unit": round(ms, 4), "value": cells / (ms * 1e-3), "unit": "cells/s",
            "exchange_bytes_per_rank": out_bytes + back_bytes,
            "note": "one rank: the exchange is a local copy (the path's overhead over the one-GPU unit)"
                    if world == 1 else "strong scaling of one grid"}


def run_forward(ctx, case, src, dev, stream, max_over_ranks):
    """Synthetic seismic (Crava::computeSyntSeismic) of the three parameter
    grids for all angles: device time per call and HBM rate against the
    algorithmic (3 + ntheta) grids per call."""
    import torch

    m = src[0]
    outs = [torch.empty_like(m[0]) for _ in range(case.ntheta)]
    for _ in range(3):
        ctx.synt_seismic(*m, outs)
    torch.cuda.synchronize(dev)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    reps = 10
    ev0.record(stream)
    for _ in range(reps):
        ctx.synt_seismic(*m, outs)
    ev1.record(stream)
    torch.cuda.synchronize(dev)
    ms = max_over_ranks(ev0.elapsed_time(ev1) / reps)
    gbytes = (3 + case.ntheta) * m[0].numel() * 4
    del outs
    return {"workload": "synthetic seismic %dx%dx%d, %d angles" % (case.nxp, case.nyp, case.nzp, case.ntheta),
            "ms_per_call": ms, "cells_per_s": case.nxp * case.nyp * case.nzp / (ms * 1e-3),
            "algorithmic_GB": gbytes / 1e9, "GB/s": gbytes / (ms * 1e-3) / 1e9}


def run_adjoint(ctx, case, src, dev):
    """Log marginal likelihood + adjoint at the bench size: time of one
    evaluation (value and all gradients) and the largest relative gap to
    central finite differences (step 1e-3 relative, FP64) over the wavelet
    scales, noise variances and 8 in-band wavelet-spectrum components."""
    import numpy as np
    import torch

    from crava_b200 import api

    g = [[t.clone() for t in src[0]], [t.clone() for t in src[1]], [t.clone() for t in src[2]],
         src[3].clone()]
    for t in g[0]:
        ctx.fft_r2c(t, api.PARAMETER)
    for t in g[1]:
        ctx.fft_r2c(t, api.DATA)
    for t in g[2] + [g[3]]:
        ctx.fft_r2c(t, api.COVARIANCE)
    torch.cuda.synchronize(dev)
    nt, cn = case.ntheta, case.nzp // 2 + 1
    spec = np.fft.fft(case.wavelet.astype(np.float64), axis=-1)[:, :cn].T.copy()
    s0 = np.ones(nt)
    v0 = np.diag(case.theta_cov).copy()
    ctx.loglik_grad(*g, s0, v0, spec)  # warm-up
    t0 = time.perf_counter()
    reps = 5
    dev_ms = []
    for _ in range(reps):
        L, gs, gv, gw, nf = ctx.loglik_grad(*g, s0, v0, spec)
        dev_ms.append(ctx.stats().ms_total)  # the kernel's device time (CUDA events)
    ms = (time.perf_counter() - t0) * 1e3 / reps
    kernel_ms = statistics.median(dev_ms)

    def fd(f, x0, i, h):
        xp, xm = x0.copy(), x0.copy()
        xp[i] += h
        xm[i] -= h
        return (f(xp) - f(xm)) / (2 * h)

    # (central difference at h, Richardson extrapolation of h and h/2,
    # central difference at h/10, analytic): a plain central difference
    # carries its own O(h^2) truncation error; the extrapolation removes
    # it, and is the check reported against the 1e-4 bar
    checks = []

    def add(f, x0, i, h, g):
        d1 = fd(f, x0, i, h)
        d2 = fd(f, x0, i, h / 2)
        d10 = fd(f, x0, i, h / 10)
        checks.append((d1, (4 * d2 - d1) / 3, d10, g))

    for i in range(nt):
        add(lambda s: ctx.loglik_grad(*g, s, v0, spec)[0], s0, i, 1e-3, gs[i])
        add(lambda v: ctx.loglik_grad(*g, s0, v, spec)[0], v0, i, 1e-3 * v0[i], gv[i])
    _, _, _, _, inv = ctx.kz_tables()
    band = [k for k in range(1, cn - 1) if inv[k]]
    flat = np.stack([spec.real, spec.imag], -1).reshape(-1)
    gflat = np.stack([gw.real, gw.imag], -1).reshape(-1)
    f = lambda x: ctx.loglik_grad(*g, s0, v0, x.reshape(cn, nt, 2))[0]
    for k, l in [(band[0], 0), (band[len(band) // 3], 1), (band[len(band) // 2], 2), (band[-1], 4)]:
        for part in (0, 1):
            i = (k * nt + l) * 2 + part
            add(f, flat, i, 1e-3 * abs(spec[k, l]), gflat[i])
    r = lambda a, b: abs(a - b) / max(abs(a), abs(b), 1e-300)
    worst_rich = max(r(dr, gg) for _, dr, _, gg in checks)
    worst_h = max(r(d1, gg) for d1, _, _, gg in checks)
    worst_h10 = max(r(d10, gg) for _, _, d10, gg in checks)
    grid_bytes = g[0][0].numel() * 4
    del g
    return {"workload": "log marginal likelihood + adjoint, %dx%dx%d, %d angles (FP64)"
                        % (case.nxp, case.nyp, case.nzp, nt),
            "ms_per_eval": ms, "kernel_ms": kernel_ms, "loglik": L, "failed_bins": nf,
            # (10 + nt) resident spectra read once per evaluation, over the
            # kernel's device time
            "GB/s": round((10 + nt) * grid_bytes / (kernel_ms * 1e-3) / 1e9, 1),
            "fd_checked": len(checks),
            "fd_check": "central differences at h and h/2 (h = 1e-3 relative; |W| for spectrum components), "
                        "Richardson-extrapolated; bar 1e-4",
            "fd_max_rel_err": worst_rich,
            "fd_plain_max_rel_err": {"h": worst_h, "h/10": worst_h10}}


def run_own(args):
    import numpy as np
    import torch

    from crava_b200 import api, synth

    from crava_b200 import dist as D

    rank, world, local = D.rank_env()
    dist = D.init("nccl", timeout_s=300)
    dev = local if world > 1 else 0
    torch.cuda.set_device(dev)
    nxp, nyp, nzp = (int(x) for x in args.grid.split(","))
    nt = 5
    prec = {"mixed": api.MIXED, "fp64": api.FP64, "fp32": api.FP32}[args.precision]

    case = synth.make_case(nxp, nyp, nzp, ANGLES5, args.noise, seed=2 + rank,
                           wavelet_scale_range=(0.8, 1.2))
    stream = torch.cuda.Stream(dev)
    ctx = api.Context(case, device=dev, stream=stream, precision=prec)
    d = lambda gs: [api.to_device(g, dev) for g in gs]
    src = (d(case.mu), d(case.data), d(case.cov), d([case.err_corr])[0])
    dst = (d(case.mu), d(case.data), d(case.cov), d([case.err_corr])[0])
    torch.cuda.synchronize(dev)

    def barrier():
        D.barrier(dist)

    def max_over_ranks(x):
        return D.max_over_ranks(dist, x, device=f"cuda:{dev}")

    def timed_steps(precision, steps, profile):
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        for _ in range(args.warmup):
            ctx.posterior_unit_oop(src, dst, precision)
        ctx.set_profiling(profile)
        ctx.profile()  # reset
        barrier()
        torch.cuda.synchronize(dev)
        n0 = api.launch_count()
        with torch.cuda.stream(stream):
            ev0.record(stream)
            for _ in range(steps):
                ctx.posterior_unit_oop(src, dst, precision)
            ev1.record(stream)
        torch.cuda.synchronize(dev)
        barrier()
        launches = api.launch_count() - n0
        prof = ctx.profile()
        ctx.set_profiling(False)
        return ev0.elapsed_time(ev1) / steps, launches, prof

    clocks = ClockSampler(dev)
    clocks.start()
    ms, launches, _ = timed_steps(prec, args.steps, False)
    clk = clocks.stop()
    # per-kernel attribution: a separate pass with CUDA events around every
    # launch and the transforms on one stream (with two lanes, kernels of
    # different grids overlap and per-launch event times would include
    # each other)
    tuned = ctx.tuning()
    ctx.set_tuning(tuned.cols_y_tile, tuned.cols_z_tile, tuned.fused, 1, tuned.rows_x, tuned.kappa_refine,
                   tuned.xy_fused)
    ms_serial, _, prof = timed_steps(prec, max(10, min(args.steps, 30)), True)
    ctx.set_tuning(tuned.cols_y_tile, tuned.cols_z_tile, tuned.fused, tuned.lanes, tuned.rows_x,
                   tuned.kappa_refine, tuned.xy_fused)
    ms = max_over_ranks(ms)
    st = ctx.stats()
    cells = nxp * nyp * nzp
    value = world * cells / (ms * 1e-3)

    # the other solve form, timed the same way
    fp64_value = value if prec == api.FP64 else None
    mixed_value = value if prec == api.MIXED else None
    solve_ms = {}

    def solve_time(pr):
        return pr["posterior_solve"][1] / pr["posterior_solve"][0] if "posterior_solve" in pr else None

    tag = {api.FP64: "fp64", api.MIXED: "mixed", api.FP32: "fp32"}
    solve_ms[tag[prec]] = solve_time(prof)
    refined = None
    if not args.no_fp64_compare:
        other = api.MIXED if prec == api.FP64 else api.FP64
        ms_o, _, _ = timed_steps(other, max(10, args.steps // 4), False)
        v_o = world * cells / (max_over_ranks(ms_o) * 1e-3)
        if other == api.FP64:
            fp64_value = v_o
        else:
            mixed_value = v_o
        # the other form's solve time from the same one-stream profiling pass
        ctx.set_tuning(tuned.cols_y_tile, tuned.cols_z_tile, tuned.fused, 1, tuned.rows_x, tuned.kappa_refine,
                       tuned.xy_fused)
        _, _, prof_o = timed_steps(other, max(10, min(args.steps, 30)), True)
        ctx.set_tuning(tuned.cols_y_tile, tuned.cols_z_tile, tuned.fused, tuned.lanes, tuned.rows_x,
                       tuned.kappa_refine, tuned.xy_fused)
        solve_ms[tag[other]] = solve_time(prof_o)
    if api.MIXED in (prec,) or not args.no_fp64_compare:
        ctx.posterior_unit_oop(src, dst, api.MIXED)
        refined = ctx.stats().refined_bins

    # e2e through the host-buffer entry points (pinned host memory): every
    # step uploads its 10+nt input grids and downloads its 9+nt outputs.
    # Headline: the asynchronous entry point, two steps in flight (one
    # step's downloads overlap the next one's uploads); also the
    # synchronous entry point, one step at a time.
    host = [torch.from_numpy(g).pin_memory() for g in case.grids()]
    pristine = [g.copy() for g in case.grids()]
    split = lambda gs: (gs[:3], gs[3:3 + nt], gs[3 + nt:9 + nt], gs[9 + nt])
    outs = [[torch.empty_like(g).pin_memory() for g in host] for _ in range(2)]
    ctx.posterior_unit_host_async(split(host), split(outs[0]), prec)  # warm-up (work grids)
    ctx.host_wait()
    k_e2e = max(2, args.e2e_steps)
    barrier()
    t0 = time.perf_counter()
    for k in range(k_e2e):
        ctx.posterior_unit_host_async(split(host), split(outs[k % 2]), prec)
    ctx.host_wait()
    e2e_step = max_over_ranks((time.perf_counter() - t0) * 1e3 / k_e2e)
    assert all(np.array_equal(h.numpy(), p) for h, p in zip(host, pristine))  # inputs untouched
    hmu, hdata, hcov, herr = split(host)
    e2e_sync_ms = []
    for _ in range(2):
        for h, p in zip(host, pristine):
            h.numpy()[...] = p
        barrier()
        t0 = time.perf_counter()
        ctx.posterior_unit_host(hmu, hdata, hcov, herr, prec)
        e2e_sync_ms.append((time.perf_counter() - t0) * 1e3)
    e2e_sync = max_over_ranks(statistics.median(e2e_sync_ms))
    gbytes = case.mu[0].nbytes
    h2d = (10 + nt) * gbytes
    d2h = (9 + nt) * gbytes
    # the host link on the same bytes and buffers: a unit's uploads alone,
    # its downloads alone, and both at once on two streams (one copy per
    # grid), the time the end-to-end step cannot go below
    dev_grids = list(dst[0]) + list(dst[1]) + list(dst[2]) + [dst[3]]
    s_up, s_dn = torch.cuda.Stream(dev), torch.cuda.Stream(dev)

    def link_ms(up, down):
        best = float("inf")
        for _ in range(3):
            torch.cuda.synchronize(dev)
            t0 = time.perf_counter()
            if up:
                with torch.cuda.stream(s_up):
                    for h, d in zip(host, dev_grids):
                        d.copy_(h, non_blocking=True)
            if down:
                with torch.cuda.stream(s_dn):
                    for h, d in zip(outs[1][:9 + nt], dev_grids[:9 + nt]):
                        h.copy_(d, non_blocking=True)
            torch.cuda.synchronize(dev)
            best = min(best, (time.perf_counter() - t0) * 1e3)
        return best

    up_ms, down_ms, both_ms = link_ms(True, False), link_ms(False, True), link_ms(True, True)
    link = {"h2d_GBps": round(h2d / (up_ms * 1e-3) / 1e9, 1), "d2h_GBps": round(d2h / (down_ms * 1e-3) / 1e9, 1),
            "both_ms": round(both_ms, 2), "frac_of_link_bound": round(both_ms / e2e_step, 3),
            "how": "the unit's input grids up and output grids down, pinned buffers, one copy per grid, "
                   "two streams at once; best of 3"}
    del outs

    # simulation: realisations of the posterior (Crava::simulate) from the
    # posterior covariance spectra, 8 realisations per call
    sim = None
    if not args.no_simulation:
        covf = [g.clone() for g in dst[2]]
        for g in covf:
            ctx.fft_r2c(g, api.COVARIANCE)
        R = 8
        outs = [torch.empty_like(dst[0][0]) for _ in range(3 * R)]
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            for w in range(2):
                ctx.simulate(covf, dst[0], 11, 0, outs)
            torch.cuda.synchronize(dev)
            nsim = 3
            ev0.record(stream)
            for k in range(nsim):
                ctx.simulate(covf, dst[0], 11, R * k, outs)
            ev1.record(stream)
        torch.cuda.synchronize(dev)
        ms_call = max_over_ranks(ev0.elapsed_time(ev1) / nsim)
        # per realisation 18 grid passes: 6 covariance spectra read, 3
        # spectra written, the 3 inverse transforms' reads and writes, 3
        # mean reads (noise is drawn in registers)
        sim_gbs = 18 * gbytes / (ms_call / R * 1e-3) / 1e9
        sim = {"value": world * R / (ms_call * 1e-3), "unit": "realisations/s",
               "ms_per_realisation": ms_call / R, "batch": R,
               "grid": [nxp, nyp, nzp], "GB/s": round(sim_gbs, 1)}
        del covf, outs

    prior = run_prior_fill(ctx, case, dst, dev, stream, max_over_ranks)

    split = None
    if not args.no_split_grid and (world == 1 or args.split_grid):
        gcase = case if world == 1 else synth.make_case(nxp, nyp, nzp, ANGLES5, args.noise, seed=2,
                                                        wavelet_scale_range=(0.8, 1.2))
        split = run_split(gcase, world, rank, dist, dev, stream, max_over_ranks, prec)

    s4 = None
    if not args.no_state4d:
        torch.cuda.nvtx.range_push("state4d")  # ncu --nvtx --nvtx-include "state4d/"
        s4 = run_state4d(ctx, case, dev, stream, max_over_ranks, hbm_peak()[0])
        torch.cuda.nvtx.range_pop()
    div = None
    if not args.no_divide:
        torch.cuda.nvtx.range_push("divide")  # ncu --nvtx --nvtx-include "divide/"
        div = run_divide(ctx, case, src, dev, stream, max_over_ranks, hbm_peak()[0])
        torch.cuda.nvtx.range_pop()

    fwd = None
    if not args.no_forward:
        fwd = run_forward(ctx, case, src, dev, stream, max_over_ranks)

    adjoint = None
    if not args.no_adjoint:
        adjoint = run_adjoint(ctx, case, src, dev)

    batch = None
    if not args.no_batch:
        batch = run_batch(args, case if (nxp, nyp, nzp) == (256, 256, 512) else None, dev, stream,
                          max_over_ranks)

    roof = None
    peak, peak_source = hbm_peak()
    gbytes = case.mu[0].nbytes
    csize = (nxp // 2 + 1) * nyp * nzp
    if prof:
        name, (n, tot, bpl) = max(prof.items(), key=lambda kv: kv[1][1])
        avg_s = tot / n * 1e-3
        # algorithmic bytes per launch: the solve moves (19 + 2 nt) complex
        # values per bin (every spectrum read and written once); a
        # transform pass one read and one write of its grid
        alg = (19 + 2 * nt) * csize * 8 if name.startswith("posterior_solve") else bpl
        achieved = alg / avg_s / 1e9
        roof = {"bound": "hbm", "kernel": name,
                "measured": "profiling pass, one stream, CUDA events per launch",
                "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": None,
                "traffic_note": "DRAM bytes are not measured inside the bench (no ncu); the ncu figure "
                                "per launch is in profiles/",
                "peak_source": peak_source, "algorithmic_bytes_per_launch": alg,
                "moved_bytes_per_launch": bpl,
                "moved_frac": round(bpl / avg_s / 1e9 / peak, 4),
                "launches": n, "avg_ms": round(tot / n, 5),
                "share": round(tot / sum(v[1] for v in prof.values()), 4)}
    # the whole unit against its algorithmic bytes B_unit = 3 (19 + 2 nt) G
    b_unit = 3 * (19 + 2 * nt) * gbytes
    unit_roof = {"bound": "hbm", "algorithmic_bytes": b_unit, "ms": round(ms, 4),
                 "achieved": round(b_unit / (ms * 1e-3) / 1e9, 1), "peak": peak, "unit": "GB/s",
                 "frac": round(b_unit / (ms * 1e-3) / 1e9 / peak, 4), "peak_source": peak_source}
    # the solve stage of both forms (one-stream profiling pass): time, the
    # mixed / FP64 speed ratio, the unit's bound from it, and the FP64
    # form's arithmetic rate on the analytic flop count of an inverted bin
    n_inv_bins = int(ctx.kz_tables()[4].sum()) * (nxp // 2 + 1) * nyp
    solve_stage = {"ms": {k: (round(v, 4) if v else None) for k, v in solve_ms.items()},
                   "inverted_bins": n_inv_bins, "mixed_refined_bins": refined}
    if solve_ms.get("fp64") and solve_ms.get("mixed"):
        solve_stage["mixed_over_fp64_speed"] = round(solve_ms["fp64"] / solve_ms["mixed"], 4)
        solve_stage["unit_bound_any_solve"] = round(ms / (ms - solve_ms["fp64"]), 4)
    if solve_ms.get("fp64"):
        # the FP64 form of a context runs the Woodbury kernel unless its
        # tuning picks a square-root shape (0-5)
        woodbury = ctx.tuning().solve_shape in (-1, 6)
        fpb = wb_flops_per_inverted_bin(nt) if woodbury else solve_flops_per_inverted_bin(nt)
        fl = fpb * n_inv_bins
        tf = fl / (solve_ms["fp64"] * 1e-3) / 1e12
        solve_stage["fp64_form"] = "woodbury" if woodbury else "square-root"
        solve_stage["fp64_flops_per_inverted_bin"] = fpb
        solve_stage["fp64_tflops"] = round(tf, 2)
        solve_stage["fp64_frac_of_nominal"] = round(tf / FP64_NOMINAL_TFLOPS, 4)
        solve_stage["fp64_peak_note"] = ("nominal FP64 vector rate 148 SMs x 128 flop/clk x 1.965 GHz "
                                         "(no measured FP64 peak on this pool)")
    kernels = {k: {"launches": v[0], "ms": round(v[1], 4),
                   "GB/s": round(v[2] / (v[1] / v[0] * 1e-3) / 1e9, 1)} for k, v in prof.items()}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            from oracle import oracle as O
            which = "ref" if O.have_ref() else "orc"
            t_unit, fails = cpu_unit_seconds(case, which)
            cpu = {"value": cells / t_unit, "unit": "cells/s", "cores": 1,
                   "kind": "reference" if which == "ref" else "port",
                   "sample": f"one whole posterior unit {nxp}x{nyp}x{nzp}x{nt} on this case (29 FFTW 2.1.2 "
                             f"transforms planned per call, the per-bin loop with lib_matr.c), "
                             f"timed once: {t_unit:.1f} s",
                   "seconds_per_unit": t_unit, "chol_fail_bins": fails}
        except Exception as e:  # the baseline is reported, never required
            cpu = {"value": None, "unit": "cells/s", "cores": 1, "kind": "reference",
                   "sample": f"failed: {e}"}

    out = {
        "metric": METRIC, "value": value, "unit": "cells/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None,
        "dtype": {"mixed": "f32+f64 (f32 transforms; f32 solve, f64 refinement and Schur step)",
                  "fp64": "f32+f64 (f32 transforms; f64 per-frequency solve)",
                  "fp32": "f32"}[args.precision],
        "data": "synthetic (seeded prior realisation, Ricker wavelets, Aki-Richards, 10% noise)",
        "config": {"workload": f"posterior unit {nxp}x{nyp}x{nzp}, 5 angles",
                   "grid": [nxp, nyp, nzp], "ntheta": nt, "precision": args.precision,
                   "l2": "inputs larger than L2 (%.2f GB read per step)" % ((10 + nt) * gbytes / 1e9),
                   "parallelism": f"replicas{world}"},
        "e2e": {"value": world * cells / (e2e_step * 1e-3), "unit": "cells/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "ms_per_step": e2e_step,
                "steps": k_e2e, "pipelined": "two steps in flight (crava_gpu_posterior_unit_host_async)",
                "sync_ms_per_step": e2e_sync, "host_link": link},
        "gpu_launches": launches,
        "roofline": roof,
        "unit_roofline": unit_roof,
        "cpu_baseline": cpu,
        "clocks": clk,
        "fp64_form_value": fp64_value,
        "mixed_form_value": mixed_value,
        "mixed_over_fp64": (mixed_value / fp64_value) if (mixed_value and fp64_value) else None,
        "solve_stage": solve_stage,
        "simulation": sim,
        "batch": batch,
        "adjoint": adjoint,
        "forward_model": fwd,
        "prior_fill": prior,
        "state4d": s4,
        "divide_by_scale_wavelet": div,
        "split_grid": split,
        "profiling_pass_ms_per_step": ms_serial,
        "stages_ms": {"forward": st.ms_forward, "solve": st.ms_solve, "inverse": st.ms_inverse},
        "kernels": kernels,
        "chol_fail_bins": st.chol_fail_bins, "nonfinite_bins": st.nonfinite_bins,
    }
    if rank == 0:
        print(json.dumps(out), flush=True)
    ctx.close()
    if dist is not None:
        dist.destroy_process_group()


# ----------------------------------------------------------------- reference arm
def run_reference(args):
    """The reference's own CPU path (oracle/_ref: FFTW 2.1.2 + lib_matr.c in
    the restated loop) on the host cores.  The case is built once, then P
    processes forked from this one (no GPU is touched here) each run one
    untimed unit and ceil(K / P) timed whole units, starting their timed
    units together.  value = timed units x cells / the wall-clock span of
    the timed phase (first start to last end)."""
    global _REF_CASE, _REF_BARRIER
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    from oracle import oracle as O

    nxp, nyp, nzp = (int(x) for x in args.grid.split(","))
    nt = 5
    if not O.have_ref():
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref (the reference's FFTW 2.1.2 + lib_matr.c build) is missing"}))
        return
    import multiprocessing as mp

    from crava_b200 import synth

    _REF_CASE = synth.make_case(nxp, nyp, nzp, ANGLES5, args.noise, seed=2, wavelet_scale_range=(0.8, 1.2))
    ncpu = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    # each process holds a copy of the unit's grids while it runs
    unit_bytes = 2 * len(_REF_CASE.grids()) * _REF_CASE.mu[0].nbytes
    try:
        import psutil
        by_mem = max(1, int(psutil.virtual_memory().available * 0.7 // unit_bytes))
    except Exception:
        by_mem = ncpu
    workers = args.workers or max(1, min(ncpu, 16, by_mem))
    units = max(1, -(-args.steps // workers))
    ctxm = mp.get_context("fork")
    _REF_BARRIER = ctxm.Barrier(workers)
    t_wall0 = time.perf_counter()
    with ctxm.Pool(workers) as pool:
        res = pool.map(_ref_worker, [(min(1, args.warmup), units)] * workers, chunksize=1)
    wall_total = time.perf_counter() - t_wall0
    late = max(t0 for _, t0, _ in res) - min(t0 for _, t0, _ in res)
    span = max(t1 for _, _, t1 in res) - min(t0 for _, t0, _ in res)
    n_units = sum(len(per) for per, _, _ in res)
    cells = nxp * nyp * nzp
    value = n_units * cells / span
    per_unit = [t for per, _, _ in res for t in per]
    desc = (f"{workers} processes forked after the case was built, each one untimed and {units} timed "
            f"whole {nxp}x{nyp}x{nzp}x{nt} units (29 FFTW 2.1.2 transforms planned per call, the "
            f"per-bin loop with lib_matr.c); {n_units} units in {span:.1f} s wall, "
            f"{statistics.median(per_unit):.1f} s per unit per process (median)")
    out = {"impl": "reference", "metric": METRIC, "value": value, "unit": "cells/s", "n_gpus": world,
           "steps": args.steps, "units_timed": n_units, "warmup": args.warmup,
           "ms_per_step": span / n_units * 1e3,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
           "data": "synthetic", "config": {"workload": f"posterior unit {nxp}x{nyp}x{nzp}, 5 angles",
                                           "grid": [nxp, nyp, nzp], "ntheta": nt,
                                           "implementation": "reference CPU path (FFTW 2.1.2, lib_matr.c FP32 solve)"},
           "cpu_baseline": {"value": value, "unit": "cells/s", "cores": workers, "kind": "reference",
                            "sample": desc},
           "e2e": {"value": value, "unit": "cells/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
           "seconds_per_unit_per_process": statistics.median(per_unit),
           "start_skew_s": round(late, 3), "wall_s": round(wall_total, 1)}
    print(json.dumps(out), flush=True)


def run_profile_unit(args):
    """Per-kernel device times of the out-of-place unit on a seeded case
    (CUDA events around every launch of the context)."""
    from crava_b200 import api, synth

    nx, ny, nz = (int(v) for v in args.profile_unit.split(","))
    nt = args.profile_ntheta
    case = synth.make_case(nx, ny, nz, tuple(10.0 * i for i in range(nt)), 0.1, seed=2)
    ctx = api.Context(case)
    t = ctx.tuning()
    tz = t.cols_z_tile if args.profile_tile_z is None else args.profile_tile_z
    ctx.set_tuning(t.cols_y_tile, tz, int(bool(args.profile_fused)), args.profile_lanes, t.rows_x,
                   t.kappa_refine, args.profile_xy)
    d = lambda gs: [api.to_device(g) for g in gs]
    src = (d(case.mu), d(case.data), d(case.cov), d([case.err_corr])[0])
    dst = (d(case.mu), d(case.data), d(case.cov), d([case.err_corr])[0])
    # untimed warm-up: the first launch of every kernel loads its module
    ctx.posterior_unit_oop(src, dst, args.profile_precision)
    ctx.set_profiling(True)
    for _ in range(args.profile_reps):
        ctx.posterior_unit_oop(src, dst, args.profile_precision)
        st = ctx.stats()
        print("forward %.3f solve %.3f inverse %.3f total %.3f ms refined %d" % (
            st.ms_forward, st.ms_solve, st.ms_inverse, st.ms_total, st.refined_bins))
    for k, v in ctx.profile().items():
        per = v[1] / v[0]
        print(f"{k:18s} launches {v[0]:4d}  {per:.4f} ms/launch  {v[2] / (per * 1e-3) / 1e9:8.1f} GB/s")
    ctx.close()


def run_profile_fft(args):
    """Per-pass device times of the forward and inverse transform of one
    grid (CUDA events around every launch): one grid on the device, so a
    full-size pass can be captured with little memory held."""
    import torch

    from crava_b200 import api, synth

    nx, ny, nz = (int(v) for v in args.profile_fft.split(","))
    case = synth.make_case(nx, ny, nz, (10.0,), 0.1, seed=3)
    ctx = api.Context(case)
    t = ctx.tuning()
    tz = t.cols_z_tile if args.profile_tile_z is None else args.profile_tile_z
    ctx.set_tuning(t.cols_y_tile, tz, 0, 1, t.rows_x, t.kappa_refine, args.profile_xy)
    g = api.to_device(case.data[0])
    # untimed warm-up: the first launch of every kernel loads its module
    ctx.fft_r2c(g, api.DATA)
    ctx.fft_c2r(g, api.DATA)
    torch.cuda.synchronize()
    ctx.set_profiling(True)
    for _ in range(args.profile_reps):
        ctx.fft_r2c(g, api.DATA)
        ctx.fft_c2r(g, api.DATA)
    torch.cuda.synchronize()
    for k, v in ctx.profile().items():
        per = v[1] / v[0]
        print(f"{k:18s} launches {v[0]:4d}  {per:.4f} ms/launch  {v[2] / (per * 1e-3) / 1e9:8.1f} GB/s")
    print("tile_wait_timeouts", ctx.stats().tile_wait_timeouts)
    ctx.close()


def main():
    args = parse()
    if args.profile_fft:
        run_profile_fft(args)
    elif args.profile_unit:
        run_profile_unit(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_own(args)


if __name__ == "__main__":
    main()
