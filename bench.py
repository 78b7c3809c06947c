"""Benchmark of the FFT transform path on B200.

Headline workload (the configuration the metric is quoted on): 20,000 1D
complex f32 forward transforms whose lengths are log-uniform in [16, 65536]
(70% 13-smooth, 15% prime, 15% other composite; seed 5), values iid N(0,1),
lines stored back to back (1.27 GB in, 1.27 GB out: larger than L2, so no
flush is needed between steps).  One step = one batched launch over all
20,000 lines (b2f_batch_execute).  Reported beside it:
  - plain per-plan: the same lines, one FftPlan per length, one
    execute_checked per line (what a caller of the reference's plan API
    does), the 20,000 executions recorded once into a CUDA graph
    (FftRecorder) and replayed, so no Python runs between them;
  - e2e: the batched step through the public API with the input copied from
    pinned host memory and the output copied back inside the timed region
    (b2f_batch_execute_host: ~32 MiB chunks whose copies overlap the transforms);
  - roofline: the long-line kernel (k_long_pass: the column, row and
    Bluestein passes of every line too long for one CTA, which hold 97% of
    the points), timed alone; achieved algorithmic GB/s (16 B per complex
    point per transform, over the average of its launches of a step) against
    the measured HBM copy bandwidth, with the DRAM traffic of an ncu capture
    (profiles/) scaled to the full workload; the short-line CTA-queue kernel
    (k_batch_cta) beside it;
  - configs: every other benchmark configuration through the plain
    per-plan path, each with its relative L2 error against an FP64 FFT;
  - serving: open-loop Poisson request streams of the serving configuration
    at 1k-200k requests/s through the serving loop against the plain
    per-request path (FFTs/s, p50/p99 latency, coalescing counts);
  - cpu_baseline: the faster of scipy.fft (pocketfft, every host core; the
    stand-in for the reference's CpuFftPlan, whose rustfft backend cannot
    be built here) and the planned C port of CpuFftPlan (oracle/cpu_port.c).

python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
Under torchrun the 20,000 lines are split into one contiguous run of about
equal points per rank (strong scaling, no data-path collective); the
value is all lines over the slowest rank's time; rank 0 prints one JSON
line.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "mixed-size FFTs/s + p50/p99 latency, served vs plain per-plan, at ≤2e-6 rel L2"


def rel_l2(actual, expected) -> float:
    a = np.asarray(actual, dtype=np.complex128).reshape(-1)
    e = np.asarray(expected, dtype=np.complex128).reshape(-1)
    den = np.linalg.norm(e)
    return float(np.linalg.norm(a - e) / (den if den > 0 else 1.0))


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = os.path.join("/tmp", f"b2f_clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu),
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) < 7:
                    continue
                try:
                    sm.append(float(f[0]))
                    mx = float(f[1])
                except ValueError:
                    continue
                for name, v in zip(names, f[3:7]):
                    if v.lower() == "active":
                        reasons.add(name)
        except FileNotFoundError:
            pass
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(args):
    from wgpufft_b200.replicas import Replicas
    rep = Replicas()
    return rep


def scipy_rate(lengths, offsets, x, threads=0, reps=5):
    """scipy.fft (pocketfft, C++) over every line of the workload on the
    host cores: lines grouped by length into [count, N] arrays, the groups
    spread over a thread pool (pocketfft releases the GIL), one warm-up pass
    then the median of `reps` passes (benches/cpu_fft_bench.rs:67-84 style).
    Returns (FFTs/s, threads, seconds per pass)."""
    from concurrent.futures import ThreadPoolExecutor

    import scipy.fft as sf
    threads = threads or (os.cpu_count() or 1)
    order = np.argsort(lengths, kind="stable")
    uniq, starts = np.unique(lengths[order], return_index=True)
    ends = list(starts[1:]) + [len(order)]
    mats = [np.stack([x[offsets[j]:offsets[j] + n] for j in order[s:e]])
            for n, s, e in zip(uniq.tolist(), starts, ends)]
    cost = [m.size * np.log2(max(m.shape[1], 2)) for m in mats]
    todo = np.argsort(cost)[::-1]

    def one(i):
        sf.fft(mats[i], axis=1, workers=1)

    with ThreadPoolExecutor(threads) as ex:
        list(ex.map(one, todo))
        times = []
        for _ in range(reps):
            t0 = time.perf_counter()
            list(ex.map(one, todo))
            times.append(time.perf_counter() - t0)
    med = statistics.median(times)
    return len(lengths) / med, threads, med


def cpu_baselines(lengths, offsets, x):
    """Both CPU baselines on the host cores: scipy.fft (pocketfft; the
    stand-in for the reference's CpuFftPlan, whose rustfft backend cannot be
    built here) on every line, and the planned C port of CpuFftPlan
    (oracle/cpu_port.c) on a bounded sample.  The faster one is the baseline."""
    out = {}
    try:
        r, th, sec = scipy_rate(lengths, offsets, x)
        out["scipy"] = {"value": r, "cores": th, "seconds_per_pass": sec,
                        "sample": f"all {len(lengths)} lines"}
    except Exception as exc:
        out["scipy"] = {"error": str(exc)}
    try:
        r, ns, th, sec = cpu_sample_rate(lengths, offsets, x, seconds_target=6.0)
        out["port"] = {"value": r, "cores": th, "seconds_per_pass": sec,
                       "sample": f"{ns} lines drawn from the {len(lengths)}-line workload"}
    except Exception as exc:
        out["port"] = {"error": str(exc)}
    best = max((k for k in out if "value" in out[k]), key=lambda k: out[k]["value"], default=None)
    if best is None:
        return {"error": "no CPU baseline ran"}, out
    b = out[best]
    impl = ("scipy.fft 1.x (pocketfft C++), stand-in for CpuFftPlan (rustfft 6.4.1 "
            "unavailable: no Rust toolchain)" if best == "scipy"
            else "planned C port of CpuFftPlan (oracle/cpu_port.c)")
    return {"value": b["value"], "unit": "FFTs/s", "cores": b["cores"], "kind": "port",
            "impl": impl, "sample": b["sample"],
            "other": {k: v.get("value") for k, v in out.items() if k != best}}, out


def cpu_sample_rate(lengths, offsets, x, seconds_target=10.0, threads=0):
    """Planned CPU FFT over a bounded sample of the lines: returns
    (FFTs/s, lines in the sample, threads)."""
    from oracle import oracle as O
    rng = np.random.default_rng(11)
    idx = rng.permutation(len(lengths))
    # grow the sample until one pass takes ~seconds_target / 3
    take = 500
    while True:
        sel = np.sort(idx[:take])
        ls = lengths[sel]
        off = np.zeros(len(ls), dtype=np.int64)
        off[1:] = np.cumsum(ls[:-1])
        data = np.empty(int(ls.sum()), dtype=np.complex64)
        for j, i in enumerate(sel):
            data[off[j]:off[j] + ls[j]] = x[offsets[i]:offsets[i] + lengths[i]]
        lines = O.CpuLines(off, ls)
        lines.run(data.copy(), threads=threads)  # warm-up
        t0 = time.perf_counter()
        lines.run(data, threads=threads)
        dt = time.perf_counter() - t0
        if dt > seconds_target / 3 or take >= len(lengths):
            reps = max(1, int(seconds_target / max(dt, 1e-3)) // 2)
            times = [dt]
            for _ in range(min(reps, 4)):
                t0 = time.perf_counter()
                lines.run(data, threads=threads)
                times.append(time.perf_counter() - t0)
            med = statistics.median(times)
            nthreads = threads if threads > 0 else O.cpu_max_threads()
            lines.close()
            return len(sel) / med, len(sel), nthreads, med
        lines.close()
        take = min(len(lengths), take * 3)


def serving_measurement(local, count=300, rates=(1e3, 1e4, 5e4, 1e5, 2e5),
                        caps=(256 << 20, 8 << 20), seed=9):
    """The serving configuration: open-loop Poisson request streams (seed 9)
    of seeded C2C or R2C, forward or inverse requests (1D lengths
    log-uniform in [64, 2^22], 2D sides from {64..4096}, 3D cubes from
    {32..256}; batch 1-64; 80/10/10 f32/f64/df64), each request's batch
    reduced until it holds at most `cap` bytes of input (the stream with
    256 MiB requests, and one of small requests up to 8 MiB), with their
    buffers resident in device memory.  At every offered rate: the serving
    loop (resident plans, 120 GB admission budget, continuous batching:
    1D complex f32 requests of any length coalesced into one batched line
    launch, same-configuration requests into one plan execution, 4 streams)
    against the plain per-request path (one cached plan per configuration,
    one execute_checked per request as it arrives, on one stream).  Served
    and plain FFTs/s count the transforms over the span from the first
    arrival to the last completion; latency is arrival to completion."""
    import threading

    import torch
    import wgpufft_b200 as w
    from wgpufft_b200 import workloads as W

    out = {"requests_per_stream": count, "rates_per_s": list(rates), "buffers": "device",
           "streams": {}}
    for cap in caps:
        reqs = W.serving_requests(count, seed=seed, max_bytes=cap)

        def cfg_of(q):
            c = w.FftConfig.new_nd(q["shape"]).with_batch(q["batch"]).with_precision(q["precision"])
            return c.with_direction(w.FftDirection.Inverse if q["inverse"] else w.FftDirection.Forward)

        cfgs = [cfg_of(q) for q in reqs]
        kinds = [w.FftTransformKind(q["kind"]) for q in reqs]
        mk = {0: w.FftPlan.c2c, 1: w.FftPlan.r2c, 2: w.FftPlan.c2r}
        plans, by_key = [], {}
        for c, k in zip(cfgs, kinds):
            key = (int(k), tuple(c.shape()), c.batch(), int(c.precision()), int(c.direction()))
            if key not in by_key:
                by_key[key] = mk[int(k)](c, device=local)
            plans.append(by_key[key])
        ins, outs = [], []
        for p in plans:
            ins.append(torch.randn(p.required_input_buffer_size_bytes() // 4, device="cuda"))
            outs.append(torch.empty(p.required_output_buffer_size_bytes() // 4, device="cuda"))
        transforms = sum(q["batch"] for q in reqs)
        in_bytes = sum(t.numel() * 4 for t in ins)
        stream = torch.cuda.current_stream()
        # warm-up: every plan once; the serving loop's resident plans and line lengths
        for p, a, b in zip(plans, ins, outs):
            p.execute_checked(a, b)
        torch.cuda.synchronize()
        srv = w.FftServer(device=local, streams=4)
        # the stream twice request by request, then once as one held burst:
        # a (configuration, batch) seen twice gets its exact plan (so a
        # request that arrives alone in the timed runs finds it built), and
        # the burst's line groups register every 1D length with the line
        # kernels
        for _ in range(2):
            for c, k, a, b in zip(cfgs, kinds, ins, outs):
                srv.wait(srv.submit_device(c, k, a, b), 600.0)
        srv.hold()
        warm = [srv.submit_device(c, k, a, b) for c, k, a, b in zip(cfgs, kinds, ins, outs)]
        srv.hold(False)
        for r in warm:
            srv.wait(r, 600.0)
        # and once back to back (the saturated case): the loop's streams,
        # pool and coalesced groups reach their steady state
        warm = [srv.submit_device(c, k, a, b) for c, k, a, b in zip(cfgs, kinds, ins, outs)]
        for r in warm:
            srv.wait(r, 600.0)
        per_rate = []
        for rate in rates:
            rng = np.random.default_rng(seed + 1)
            arrivals = np.cumsum(rng.exponential(1.0 / rate, len(reqs)))
            # plain per-request path: completion events timed on the device
            evs = [torch.cuda.Event(enable_timing=True) for _ in range(len(reqs) + 1)]
            t_sub = []
            torch.cuda.synchronize()
            evs[0].record(stream)
            t0 = time.perf_counter()
            for i, (p, a, b) in enumerate(zip(plans, ins, outs)):
                while time.perf_counter() - t0 < arrivals[i]:
                    pass
                t_sub.append(time.perf_counter() - t0)
                p.execute_checked(a, b)
                evs[i + 1].record(stream)
            torch.cuda.synchronize()
            done = [evs[0].elapsed_time(e) / 1e3 for e in evs[1:]]
            lat_plain = sorted(max(d - a, d - t) for d, a, t in zip(done, arrivals, t_sub))
            span_plain = max(done) - arrivals[0]
            # served
            srv.reset_stats()
            ids = [None] * len(reqs)

            lag = [0.0]

            def feeder():
                t1 = time.perf_counter()
                for i in range(len(reqs)):
                    while time.perf_counter() - t1 < arrivals[i]:
                        pass
                    ids[i] = srv.submit_device(cfgs[i], kinds[i], ins[i], outs[i])
                lag[0] = time.perf_counter() - t1 - arrivals[-1]

            th = threading.Thread(target=feeder)
            th.start()
            th.join()
            srv.drain(600.0)
            st = srv.stats()
            for r in ids:
                srv.wait(r, 60.0)
            plain = {"ffts_per_s": transforms / span_plain, "p50_ms": lat_plain[len(lat_plain) // 2] * 1e3,
                     "p99_ms": lat_plain[int(len(lat_plain) * 0.99)] * 1e3}
            served = {"ffts_per_s": st["ffts_per_s"], "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"],
                      "groups": st["groups"], "line_groups": st["line_groups"],
                      "coalesced_requests": st["coalesced_requests"],
                      "last_submit_after_last_arrival_ms": lag[0] * 1e3}
            per_rate.append({"offered_rate_per_s": rate, "served": served,
                             "plain_per_request": plain,
                             "served_vs_plain_ffts": served["ffts_per_s"] / max(plain["ffts_per_s"], 1e-9)})
        stats = srv.stats()
        srv.close()
        out["streams"][f"max_{cap >> 20}MiB"] = {
            "transforms": transforms, "input_bytes": in_bytes, "distinct_configs": len(by_key),
            "resident_plans": stats["resident_plans"], "per_rate": per_rate,
            "served_vs_plain_at_saturation": per_rate[-1]["served_vs_plain_ffts"]}
        del plans, by_key, ins, outs
        torch.cuda.empty_cache()
    return out


def config_measurements(local, hbm_peak):
    """Every benchmark configuration through the plain per-plan path: ms per
    transform (CUDA events, inputs resident, no copies), algorithmic GB/s
    (16 B per complex point per f32 transform, 32 B for f64/df64; real
    transforms 4 N_real + 8 N_packed), fraction of the measured HBM
    bandwidth, GFLOP/s (5 N log2 N per complex line, 2.5 N log2 N per real
    one), and the relative L2 error of one execution on the configuration's
    seeded input against an FP64 FFT (scipy.fft/pocketfft in complex128) of
    the values the device saw.  The precision configuration (2^24, 8192^2)
    also reports the error on its high-dynamic-range input."""
    import math

    import scipy.fft as sf
    import torch
    import wgpufft_b200 as w
    from wgpufft_b200 import workloads as W

    F32, F64, DF64 = w.FftPrecision.F32, w.FftPrecision.F64, w.FftPrecision.Df64
    C2C, R2C, C2R = w.FftTransformKind.C2c, w.FftTransformKind.R2c, w.FftTransformKind.C2r
    workers = os.cpu_count() or 1
    # name, config, kind, forward+inverse in place, CUDA-graph timing, input seed, HDR seed
    cases = [
        ("1d_1024x512_c2c_f32", w.FftConfig.new(1024).with_batch(512), C2C, False, True, 1, None),
        ("2d_[2048,4096]_fwd+inv_in_place", w.FftConfig.new_nd([2048, 4096]), C2C, True, False,
         2, None),
        ("2d_[4096,2048]_fwd+inv_in_place", w.FftConfig.new_nd([4096, 2048]), C2C, True, False,
         2, None),
        ("3d_256^3_r2c", w.FftConfig.new_nd([256, 256, 256]), R2C, False, False, 3, None),
        ("3d_256^3_c2r", w.FftConfig.inverse_nd([256, 256, 256]), C2R, False, False, 3, None),
        ("1d_127x264208_rader", w.FftConfig.new(127).with_batch(264208), C2C, False, False, 4,
         None),
        ("1d_1009x33255", w.FftConfig.new(1009).with_batch(33255), C2C, False, False, 4, None),
        ("1d_4099x8186", w.FftConfig.new(4099).with_batch(8186), C2C, False, False, 4, None),
        ("1d_15015x2234", w.FftConfig.new(15015).with_batch(2234), C2C, False, False, 4, None),
        ("1d_2^20x32", w.FftConfig.new(1 << 20).with_batch(32), C2C, False, False, 4, None),
        ("1d_2^26", w.FftConfig.new(1 << 26), C2C, False, False, 4, None),
        ("1d_2^24", w.FftConfig.new(1 << 24), C2C, False, False, 6, 7),
        ("2d_8192x8192", w.FftConfig.new_nd([8192, 8192]), C2C, False, False, 6, 7),
        ("1d_2^20x16_f64", w.FftConfig.new(1 << 20).with_batch(16).with_precision(F64), C2C,
         False, False, 8, None),
        ("1d_2^20x16_df64", w.FftConfig.new(1 << 20).with_batch(16).with_precision(DF64), C2C,
         False, False, 8, None),
        # the precision form: 2^20 lines of 64 on the tcgen05 split-TF32 layer, beside the
        # same lines on the CUDA-core register kernel
        ("1d_64x2^20_tensor_cores", w.FftConfig.new(64).with_batch(1 << 20).with_tuning(
            w.FftTuning().with_tensor_cores(True)), C2C, False, False, 4, None),
        ("1d_64x2^20", w.FftConfig.new(64).with_batch(1 << 20), C2C, False, False, 4, None),
    ]

    def host_input(cfg, kind, seed, hdr=False):
        """Seeded input of the configuration as (device words, exact values)."""
        n_real = cfg.total_complex_len()
        if kind == R2C:
            r = np.random.default_rng(seed).uniform(-1, 1, n_real).astype(np.float32)
            return torch.from_numpy(r), r.astype(np.float64)
        if kind == C2R:
            # a Hermitian-consistent packed spectrum: the R2C of seeded reals
            r = np.random.default_rng(seed).uniform(-1, 1, n_real).reshape(cfg.shape()[::-1])
            z = sf.rfftn(r, workers=workers).astype(np.complex64).reshape(-1)
            return torch.from_numpy(z.view(np.float32)), z.astype(np.complex128)
        if hdr:
            z = W.hdr_complex(n_real, seed)
        elif seed == 1:
            z = W.uniform_complex(n_real, seed)
        else:
            z = W.normal_complex(n_real, seed)
        if cfg.precision() == F32:
            h = z.astype(np.complex64)
            return torch.from_numpy(h.view(np.float32)), h.astype(np.complex128)
        if cfg.precision() == F64:
            h = z.astype(np.complex128)
            return torch.from_numpy(h.view(np.float64)), h
        # df64 words [re_hi, re_lo, im_hi, im_lo]: exactly the f64 values split
        h = z.astype(np.complex128)
        v = h.view(np.float64)
        hi = v.astype(np.float32)
        lo = (v - hi.astype(np.float64)).astype(np.float32)
        words = np.stack([hi, lo], axis=1).reshape(-1)
        exact = (hi.astype(np.float64) + lo.astype(np.float64)).view(np.complex128)
        return torch.from_numpy(words), exact

    def host_output(t, cfg, kind):
        h = t.cpu().numpy()
        if kind == C2R:
            return h.astype(np.float64)
        if cfg.precision() == F32:
            return h.view(np.complex64).astype(np.complex128)
        if cfg.precision() == F64:
            return h.view(np.complex128)
        v = h.reshape(-1, 2).astype(np.float64)
        return (v[:, 0] + v[:, 1]).view(np.complex128)

    def reference(exact, cfg, kind):
        shape = cfg.shape()
        nd = len(shape)
        axes = tuple(range(1, nd + 1))  # numpy axes of [batch, ..., axis1, axis0]
        stored = shape if kind != C2R else [shape[0] // 2 + 1] + shape[1:]
        arr = exact.reshape([cfg.batch()] + stored[::-1])
        inv = cfg.direction() == w.FftDirection.Inverse
        norm = {0: "backward", 1: "forward", 2: "backward", 3: "ortho"}[int(cfg.normalization())]
        if int(cfg.normalization()) == 0:
            fn = sf.ifftn if inv else sf.fftn
            y = fn(arr, axes=axes, workers=workers, norm="forward" if inv else "backward")
        elif kind == R2C:
            y = sf.rfftn(arr, axes=axes, workers=workers, norm=norm)
        elif kind == C2R:
            y = sf.irfftn(arr, s=shape[::-1], axes=axes, workers=workers, norm=norm)
        else:
            y = (sf.ifftn if inv else sf.fftn)(arr, axes=axes, workers=workers, norm=norm)
        return y.reshape(-1)

    out = {}
    stream = torch.cuda.current_stream()
    for name, cfg, kind, pair, graph, seed, hdr_seed in cases:
        try:
            mk = {0: w.FftPlan.c2c, 1: w.FftPlan.r2c, 2: w.FftPlan.c2r}[int(kind)]
            plan = mk(cfg, device=local)
            inv = None
            if pair:
                inv = w.FftPlan.c2c(cfg.with_direction(w.FftDirection.Inverse), device=local)
            ib, ob = plan.required_input_buffer_size_bytes(), plan.required_output_buffer_size_bytes()
            hin, exact = host_input(cfg, kind, seed)
            a = torch.empty(max(ib, ob) // 4 + 4, device="cuda")
            a.view(torch.uint8)[:ib].copy_(hin.view(torch.uint8).cuda())
            o = torch.empty(ob // 4 + 4, device="cuda")
            # one checked execution on the seeded input: its error
            if pair:
                plan.execute_in_place(a)
                got = host_output(a[:ib // 4], cfg, kind)
            else:
                plan.execute_checked(a, o)
                got = host_output(o[:ob // 4], cfg, kind)
            torch.cuda.synchronize()
            err = rel_l2(got, reference(exact, cfg, kind))
            err_rt = None
            if pair:
                inv.execute_in_place(a)
                back = host_output(a[:ib // 4], cfg, kind)
                err_rt = rel_l2(back, exact)
            err_hdr = None
            if hdr_seed is not None:
                hh, ex_h = host_input(cfg, kind, hdr_seed, hdr=True)
                a.view(torch.uint8)[:ib].copy_(hh.view(torch.uint8).cuda())
                plan.execute_checked(a, o)
                err_hdr = rel_l2(host_output(o[:ob // 4], cfg, kind), reference(ex_h, cfg, kind))
            del got

            def step():
                if pair:
                    plan.execute_in_place(a)
                    inv.execute_in_place(a)
                else:
                    plan.execute_checked(a, o)
            reps = 20
            rec = None
            if graph:
                rec = w.FftRecorder()
                for _ in range(100):
                    plan.record(rec, a, o)
                rec.finish()
            for _ in range(3):
                step()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            if rec is not None:
                for _ in range(reps):
                    rec.submit()
            else:
                for _ in range(reps):
                    step()
            e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / reps / (100 if rec is not None else 1)
            n_tr = 2 if pair else 1
            total = cfg.total_complex_len()
            if kind == C2C:
                bpp = 16 if cfg.precision() == F32 else 32
                alg = bpp * total * n_tr
            else:
                packed = int(np.prod([cfg.shape()[0] // 2 + 1] + cfg.shape()[1:])) * cfg.batch()
                alg = 4 * total + 8 * packed
            logical = int(np.prod(cfg.shape()))
            per = (2.5 if kind != C2C else 5.0) * logical * math.log2(logical) * cfg.batch()
            gbs = alg / (ms / 1e3) / 1e9
            tol = {F32: 2e-6, F64: 1e-14, DF64: 1e-13}[cfg.precision()]
            row = {"ms": ms, "GBps_alg": gbs, "frac_hbm": gbs / hbm_peak,
                   "GFLOPs": n_tr * per / (ms / 1e3) / 1e9, "rel_l2": err, "tol": tol,
                   "stages": [s["kind"] + ":" + s["label"] for s in plan.diagnostics()["stages"]],
                   "timing": "CUDA graph of 100 executions" if rec is not None else "events"}
            if err_rt is not None:
                row["rel_l2_round_trip"] = err_rt
            if err_hdr is not None:
                row["rel_l2_hdr"] = err_hdr
            out[name] = row
            del plan, inv, a, o, rec
            torch.cuda.empty_cache()
        except Exception as exc:
            out[name] = {"error": str(exc)}
    return out


def run_reference(args, world, rank):
    """--impl reference: the reference's CPU path on the host cores, all
    threads: the faster of scipy.fft (pocketfft, the stand-in for the
    crate's CpuFftPlan, whose rustfft backend cannot be built here) over
    every line and the planned C port of CpuFftPlan over a bounded sample."""
    from wgpufft_b200 import workloads as W
    if rank != 0:
        return
    lengths = W.mixed_lengths()
    offsets = W.packed_offsets(lengths)
    x = W.normal_complex(int(lengths.sum()), 5)
    cpu, detail = cpu_baselines(lengths, offsets, x)
    rate = cpu["value"]
    sec = len(lengths) / rate  # one pass over all 20,000 lines at that rate
    out = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": "FFTs/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": sec * 1e3, "higher_is_better": True,
        "scaling": "strong",
        "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded N(0,1) complex, lengths drawn per the workload)",
        "config": {"workload": "20,000 mixed-length 1D C2C f32 forward lines, log-uniform "
                               "[16, 65536] (70% 13-smooth / 15% prime / 15% other), seed 5",
                   "lines": int(len(lengths))},
        "cpu_baseline": cpu,
        "cpu_detail": detail,
        "e2e": {"value": rate, "unit": "FFTs/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-serve", action="store_true")
    ap.add_argument("--no-configs", action="store_true")
    ap.add_argument("--no-e2e", action="store_true",
                    help="skip the host-buffer leg (launch lists of the batched step alone)")
    ap.add_argument("--lines", type=int, default=0,
                    help="use only the first K lines of the workload (profiling-sized cases)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        # the reference arm runs on rank 0's host cores alone; the other
        # ranks exit at once, with no process group to wait on
        rank = int(os.environ.get("RANK", "0"))
        if rank == 0:
            run_reference(args, int(os.environ.get("WORLD_SIZE", "1")), 0)
        return
    rep = dist_setup(args)
    world, rank, local = rep.world, rep.rank, rep.local

    def barrier(_world):
        rep.barrier()

    def max_over_ranks(_world, value):
        return rep.max(value)

    import torch
    import wgpufft_b200 as w
    from wgpufft_b200 import workloads as W

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    all_lengths = W.mixed_lengths()
    if args.lines:
        all_lengths = all_lengths[:args.lines]
    all_total = int(all_lengths.sum())
    # strong scaling: the lines are split into contiguous runs of about equal
    # points, one per rank (no data-path collective)
    from wgpufft_b200.replicas import partition_lines
    first, end = partition_lines(all_lengths, world)[rank]
    lengths = all_lengths[first:end]
    offsets = W.packed_offsets(lengths)
    total = int(lengths.sum())
    x_all = W.normal_complex(all_total, 5)
    lo = int(all_lengths[:first].sum())
    x = x_all[lo:lo + total]
    del x_all
    nbytes = total * 8
    alg_bytes = 2 * nbytes  # one read + one write of every complex point
    batch = w.FftBatch(lengths, offsets, w.FftDirection.Forward, device=local)
    diag = batch.diagnostics()
    dx = torch.from_numpy(x.view(np.float32)).to(dev)
    dy = torch.empty_like(dx)
    stream = torch.cuda.current_stream(dev)

    # ---- batched launch, data resident in HBM
    for _ in range(args.warmup):
        batch.execute(dx, dy)
    torch.cuda.synchronize()
    barrier(world)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    step_ms = []
    with ClockSampler(local) as clk:
        barrier(world)
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(args.steps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            batch.execute(dx, dy)
            e1.record(stream)
            step_ms.append((e0, e1))
        ev1.record(stream)
        torch.cuda.synchronize()
        barrier(world)
    total_ms = ev0.elapsed_time(ev1)
    per_step = [a.elapsed_time(b) for a, b in step_ms]
    total_ms = max_over_ranks(world, total_ms)
    ms_per_step = total_ms / args.steps
    value = len(all_lengths) * args.steps / (total_ms / 1e3)
    clocks = clk.summary()

    # ---- roofline of the dominant kernel: k_long_pass (parts bit 2), its
    # two or three launches of a step timed alone on the launching stream;
    # the short-line kernel k_batch_cta (parts bit 0) beside it.
    hbm_peak, peak_kind = load_peaks()
    nd = diag
    long_bytes = 16 * int(nd.get("long_elements", 0))
    long_launches = max(1, int(nd.get("long_launches", 1)))
    cta_bytes = 16 * int(nd.get("cta_elements", 0))
    rf = None

    def time_parts(parts, reps):
        for _ in range(2):
            batch.execute_parts(dx, dy, parts, sequential=True)
        torch.cuda.synchronize()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        for _ in range(reps):
            batch.execute_parts(dx, dy, parts, sequential=True)
        t1.record(stream)
        torch.cuda.synchronize()
        return t0.elapsed_time(t1) / reps

    try:
        reps = max(3, args.steps)
        long_ms = time_parts(4, reps)  # all launches of one step
        per_launch_ms = long_ms / long_launches
        per_launch_bytes = long_bytes / long_launches
        ach = per_launch_bytes / (per_launch_ms / 1e3) / 1e9
        rf = {"bound": "hbm", "kernel": "k_long_pass", "achieved": ach, "peak": hbm_peak,
              "unit": "GB/s", "frac": ach / hbm_peak, "peak_kind": peak_kind,
              "traffic": None, "algorithmic_bytes_per_launch": per_launch_bytes,
              "ms_per_launch": per_launch_ms, "launches_per_step": long_launches,
              "whole_step": {"achieved": alg_bytes / (ms_per_step / 1e3) / 1e9,
                             "frac": alg_bytes / (ms_per_step / 1e3) / 1e9 / hbm_peak}}
        if cta_bytes:
            cta_ms = time_parts(1, reps)
            rf["other_kernel"] = {"kernel": "k_batch_cta", "ms_per_launch": cta_ms,
                                  "algorithmic_bytes_per_launch": cta_bytes,
                                  "achieved": cta_bytes / (cta_ms / 1e3) / 1e9}
        traffic_file = os.path.join(ROOT, "profiles", "k_long_pass_traffic.json")
        if os.path.exists(traffic_file) and not args.lines:
            with open(traffic_file) as f:
                t = json.load(f)
            # DRAM bytes of the launches of one step captured on a subset of the
            # lines, per launch, scaled to the full workload by the algorithmic
            # bytes (the traffic grows with the points processed)
            rf["traffic"] = (t["dram_bytes_per_step"] / long_launches
                             * long_bytes / t["algorithmic_bytes"])
            rf["traffic_note"] = t.get("note")
    except Exception as exc:  # measurement must not hide the headline
        rf = {"bound": "hbm", "error": str(exc)}

    # ---- e2e: pinned host buffers, copies inside the timed region; the
    # host-buffer entry point overlaps the chunks' copies with the transforms
    e2e = None
    if not args.no_e2e:
        hx = torch.from_numpy(x.view(np.float32)).pin_memory()
        hy = torch.empty_like(hx).pin_memory()
        for _ in range(3):
            batch.execute_host(hx, hy, dx, dy)
        torch.cuda.synchronize()
        e2e_steps = max(3, min(args.steps, 10))
        barrier(world)
        c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        c0.record(stream)
        for _ in range(e2e_steps):
            batch.execute_host(hx, hy, dx, dy)
        c1.record(stream)
        torch.cuda.synchronize()
        e2e_ms = max_over_ranks(world, c0.elapsed_time(c1)) / e2e_steps
        # the PCIe bound beside it: the same bytes copied in and out
        # concurrently (two streams, no transform), one whole-buffer copy each
        s_in, s_out = torch.cuda.Stream(), torch.cuda.Stream()
        cp0, cp1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        cp0.record(stream)
        s_in.wait_event(cp0)
        s_out.wait_event(cp0)
        for _ in range(e2e_steps):
            with torch.cuda.stream(s_in):
                dx.copy_(hx, non_blocking=True)
            with torch.cuda.stream(s_out):
                hy.copy_(dy, non_blocking=True)
        stream.wait_stream(s_in)
        stream.wait_stream(s_out)
        cp1.record(stream)
        torch.cuda.synchronize()
        copy_ms = cp0.elapsed_time(cp1) / e2e_steps
        e2e = {"value": len(all_lengths) / (e2e_ms / 1e3), "unit": "FFTs/s",
               "h2d_bytes_per_step": all_total * 8, "d2h_bytes_per_step": all_total * 8,
               "ms_per_step": e2e_ms,
               "copies_alone_ms_per_step": copy_ms,
               "copies_alone_gbs_each_way": all_total * 8 / (copy_ms / 1e3) / 1e9}

    # ---- plain per-plan: one plan per length, one execute_checked per line,
    # all 20,000 executions recorded once into a CUDA graph (FftRecorder) and
    # replayed, so that no Python runs between the executions
    plain = None
    extras = world == 1  # plain, CPU, configs and serving legs: single-GPU runs only
    if extras and not args.no_plain:
        plans = {}
        for n in np.unique(lengths):
            plans[int(n)] = w.FftPlan.c2c(w.FftConfig.new(int(n)), device=local)
        base_x, base_y = dx.data_ptr(), dy.data_ptr()
        t0 = time.perf_counter()
        rec = w.FftRecorder()
        for n, o in zip(lengths.tolist(), offsets.tolist()):
            plans[n].record(rec, (base_x + 8 * o, 8 * n), (base_y + 8 * o, 8 * n))
        rec.finish()
        record_s = time.perf_counter() - t0
        for _ in range(2):
            rec.submit()
        torch.cuda.synchronize()
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        plain_steps = 3
        t0 = time.perf_counter()
        p0.record(stream)
        for _ in range(plain_steps):
            rec.submit()
        p1.record(stream)
        torch.cuda.synchronize()
        wall = (time.perf_counter() - t0) / plain_steps
        pms = p0.elapsed_time(p1) / plain_steps
        nl = sum(len(p.diagnostics()["stages"]) for p in
                 (plans[int(n)] for n in lengths.tolist()))
        plain = {"value": len(lengths) / (pms / 1e3), "unit": "FFTs/s", "ms_per_step": pms,
                 "host_wall_ms_per_step": wall * 1e3, "launches_per_step": nl,
                 "executions_per_step": len(lengths),
                 "how": "one FftPlan per distinct length; the 20,000 execute_checked calls "
                        "recorded once into a CUDA graph (FftRecorder) and replayed",
                 "record_and_instantiate_s": record_s}
        del rec, plans

    # ---- accuracy on sampled lines against an FP64 FFT (numpy's pocketfft)
    acc = None
    try:
        y = dy.cpu().numpy().view(np.complex64)
        rng = np.random.default_rng(0)
        errs = []
        for i in rng.choice(len(lengths), 64, replace=False):
            n, o = int(lengths[i]), int(offsets[i])
            errs.append(rel_l2(y[o:o + n], np.fft.fft(x[o:o + n].astype(np.complex128))))
        acc = {"max_rel_l2_sampled": max(errs), "lines": len(errs),
               "reference": "numpy.fft in complex128"}
    except Exception as exc:
        acc = {"error": str(exc)}

    cpu = None
    if extras and not args.no_cpu:
        try:
            cpu, _ = cpu_baselines(lengths, offsets, x)
        except Exception as exc:
            cpu = {"error": str(exc)}

    configs = None
    if extras and not args.no_configs:
        configs = config_measurements(local, hbm_peak)

    serving = None
    if extras and not args.no_serve:
        try:
            serving = serving_measurement(local)
        except Exception as exc:
            serving = {"error": str(exc)}

    lat = sorted(per_step)
    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": "FFTs/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded N(0,1) complex, lengths drawn per the workload)",
            "config": {"workload": "20,000 mixed-length 1D C2C f32 forward lines, lengths "
                                   "log-uniform [16, 65536] (70% 13-smooth / 15% prime / 15% "
                                   "other), batched persistent launch",
                       "lines": int(len(all_lengths)), "lines_rank0": int(len(lengths)),
                       "distinct_lengths_rank0": int(diag["distinct_lengths"]),
                       "complex_points": all_total, "bytes_in": all_total * 8,
                       "l2": "inputs (1.27 GB) larger than L2; no flush",
                       "parallelism": f"lines partitioned over {world} GPU(s), "
                                      f"no data-path collective"},
            "latency": {"p50_ms": lat[len(lat) // 2], "p99_ms": lat[min(len(lat) - 1,
                                                                        int(len(lat) * 0.99))],
                        "unit": "ms per 20,000-line batch"},
            "plain_per_plan": plain,
            "serving": serving,
            "configs": configs,
            "served_vs_plain": (value / plain["value"]) if plain else None,
            "gflops": sum(W.fft_flops(int(n)) for n in all_lengths) * args.steps
            / (total_ms / 1e3) / 1e9,
            "roofline": rf,
            "e2e": e2e,
            "cpu_baseline": cpu,
            "accuracy": acc,
            "clocks": clocks,
            "gpu_launches": args.steps * (int(diag.get("cta_launches", 1))
                                          + int(diag.get("long_launches", 0))
                                          + int(diag["cluster_tasks"] > 0)
                                          + int(diag.get("cluster16_tasks", 0) > 0)),
            "batch": diag,
        }
        print(json.dumps(out), flush=True)
    rep.close()


if __name__ == "__main__":
    main()
