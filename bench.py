#!/usr/bin/env python
"""Benchmark: proj+back voxel-ray updates/s of the 512^3 FP32 iterative reconstruction.

Workload (one GPU): the plain iterative reconstruction at 512^3 -- modified Shepp-Logan
plus 5 seeded random ellipsoids, 512 views over 360 deg, 512 x 512 detector of pitch 2,
FOD 1024, FDD 2048 (magnification 2), unit voxels; real sinogram from the Siddon projector
(RSVI geometry) plus Gaussian noise of sigma = 1% of the largest ray sum; simple gradient
descent with the quadratic (GG beta = 2) regulariser, lambda = 0.01, RSVI pair, FP32
throughout. One step = one gradient iteration = 3 operator calls (projection, VI
backprojection, projection of the gradient for the optimal step), i.e. 3 * 512^4
voxel-ray updates. Inputs (512 MiB volume, 512 MiB sinogram) are far larger than L2.

Multi-GPU (torchrun): every rank reconstructs its own job (different phantom seed) with
no data-path collective -- weak scaling; value = all ranks' updates / max-over-ranks time.

--impl reference times the reference's own CPU code for the path (the kernel sources of
RegularSamplingProjector / VIBackProjector compiled for the host through oracle/_ref, or
the oracle's restatement of them where that build is absent) on all host cores, on a
bounded sample of the same workload (a few of the 512 views of each operator call).
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
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

N, VIEWS, PITCH, FOD, MAG = 512, 512, 2.0, 1024.0, 2.0
LAMBDA = 0.01
FALLBACK_HBM_GBS = 6650.0


def workload_cfg(n=N, views=VIEWS):
    from tomogpi_b200 import ConfigCT

    return ConfigCT.cone_beam(n, views, det=n, pitch=PITCH, fod=FOD, magnification=MAG)


def sample_cfg(k: int, n=N, views=VIEWS):
    """k of the workload's views spread evenly over 360 deg: every (views / k)-th view, which
    a k-view scan reproduces exactly when views / k is a power of two (the angles
    p * 2 pi / k and (p * views / k) * 2 pi / views then round to the same doubles)."""
    stride = views // k
    if k <= 0 or views % k or stride & (stride - 1):
        raise ValueError(f"{k} views do not divide {views} by a power of two")
    return workload_cfg(n, k)


def config_dict(extra=None):
    d = {"workload": "iterative_recon_512_fp32", "volume": [N, N, N], "views": VIEWS, "detector": [N, N],
         "pitch": PITCH, "fod": FOD, "fdd": FOD * MAG, "pair": "RSVI", "regulariser": "GG beta=2 lambda=0.01",
         "data_sinogram": "Siddon(phantom) + 1% Gaussian noise", "step": "1 gradient iteration = 3 operator calls",
         "l2": "inputs larger than L2 (512 MiB volume and sinogram)"}
    if extra:
        d.update(extra)
    return d


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    try:
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def profiled_traffic(kernel: str):
    """DRAM bytes per launch from the committed ncu summary, if any (profiles/*.txt lines
    'traffic_bytes_per_launch <kernel>[:<layout>] <bytes>')."""
    for f in sorted((ROOT / "profiles").glob("*.txt")):
        for line in f.read_text().splitlines():
            parts = line.split()
            if len(parts) == 3 and parts[0] == "traffic_bytes_per_launch" and parts[1] == kernel:
                return float(parts[2])
    return None


def profiled_limits(kernel: str):
    """What binds the kernel, from the committed ncu summary of the current code (profiles/*
    lines 'limiter <kernel>[:<layout>] <unit> key=value ...'): the busiest unit and its
    utilisations, instructions per sample, and the capture it came from."""
    for f in sorted((ROOT / "profiles").glob("*")):
        for line in f.read_text().splitlines():
            parts = line.split()
            if len(parts) >= 3 and parts[0] == "limiter" and parts[1] == kernel:
                out = {"unit": parts[2], "source": f"profiles/{f.name}"}
                for kv in parts[3:]:
                    k, _, v = kv.partition("=")
                    try:
                        out[k] = float(v)
                    except ValueError:
                        out[k] = v
                return out
    return None


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.lines = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.index)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

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
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 6:
                continue
            try:
                sm.append(float(f[0]))
                mx = float(f[1])
            except ValueError:
                continue
            for nm, v in zip(names, f[2:6]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def cpu_reference_sample(k: int, reps: int = 1, warm: int = 0):
    """Times one gradient iteration's operator calls (RS projection, VI backprojection, RS
    projection) over k views of the workload spread evenly over 360 deg (sample_cfg) on the
    host cores. Returns (updates/s, kind, cores, per-rep seconds)."""
    import numpy as np

    import oracle
    from tomogpi_b200 import phantoms

    cfg = sample_cfg(k)
    vol = oracle.phantom(phantoms.config_phantom(0, N), N, N, N)
    ref = oracle.ref_lib() is not None
    kind = "reference" if ref else "port"
    proj = (lambda v: oracle.ref_project(cfg, oracle.RS, v)) if ref else (lambda v: oracle.project(cfg, oracle.RS, v))
    back = (lambda s: oracle.ref_backproject(cfg, s)) if ref else (lambda s: oracle.backproject(cfg, s))
    times = []
    for i in range(warm + reps):
        t0 = time.perf_counter()
        s = proj(vol)
        b = back(s)
        proj(b)
        dt = time.perf_counter() - t0
        if i >= warm:
            times.append(dt)
    units = 3 * N * N * N * k
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return units / (sum(times) / len(times)), kind, cores, times, units


def make_job_inputs(t, torch, n, views, mag, seed, dev, storage):
    """Phantom (seeded random ellipsoids), Siddon sinogram + 1% noise, on the GPU."""
    cfg = t.ConfigCT.cone_beam(n, views, det=n, magnification=mag)
    with t.Context(cfg, device=dev.index or 0) as ctx:
        truth = t.phantom(t.phantoms.random_ellipsoids(seed, 8, n), n, n, n, device=dev.index or 0)
        g = ctx.project("SIDDON", truth)
    gen = torch.Generator(device=dev).manual_seed(seed)
    g += torch.randn(g.shape, device=dev, generator=gen) * (0.01 * float(g.max()))
    return cfg, g.to(storage)


def batch_mix(seed, jobs):
    """The uneven job mix: N in {64,96,128,192,256}, views U[60,360], magnification U[1.5,2.5]."""
    import numpy as np

    rng = np.random.default_rng(seed)
    out = []
    for _ in range(jobs):
        n = int(rng.choice([64, 96, 128, 192, 256]))
        views = int(rng.integers(60, 361))
        mag = float(rng.uniform(1.5, 2.5))
        out.append((n, views, mag))
    return out


def run_batch_bench(t, torch, dev, jobs=64, iters=10, seed=2024):
    """Batched uneven reconstructions: `jobs` seeded jobs (batch_mix), N x N detector, BF16
    storage / FP32 accumulation with the measured sinogram kept in FP32, one persistent
    projection and backprojection launch per phase over all jobs, one iteration replayed
    from a CUDA graph; beside it the same jobs one after another with the plain FP32
    single-job solver, and the largest relative L2 difference between a job's batched
    BF16 result and its FP32 single-job result."""
    params = t.GradientParams(gradient_iteration_nb=iters, optimal_step_iteration_nb=iters + 1,
                              regularization_parameter=LAMBDA, storage="bf16", real_f32=True)
    b = t.Batch(params, device=dev.index or 0)
    units = 0
    keep = []
    layouts = {}
    for j, (n, views, mag) in enumerate(batch_mix(seed, jobs)):
        cfg, g = make_job_inputs(t, torch, n, views, mag, seed + j, dev, torch.float32)
        vol = torch.zeros(cfg.volume_shape, device=dev)
        tu = tuned(t, cfg, "bf16", dev)
        b.add(cfg, vol, g, rs_layout=tu["rs_layout"], vi_zc=tu["vi_zc"])
        layouts[n] = tu
        keep.append((cfg, vol, g))
        units += 3 * cfg.voxel_ray_updates
    b.iterate(1)  # builds the work queues and captures the graph (iteration 1)
    torch.cuda.synchronize()
    st = b.stats()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    b.iterate(iters - 1)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / (iters - 1)
    b.close()
    single_ms = 0.0
    worst = 0.0
    p32 = t.GradientParams(gradient_iteration_nb=iters, optimal_step_iteration_nb=iters + 1,
                           regularization_parameter=LAMBDA, storage="f32")
    for cfg, bvol, g in keep:
        with t.Context(cfg, device=dev.index or 0) as ctx:
            s = t.Solver(ctx, p32)
            v = torch.zeros(cfg.volume_shape, device=dev)
            g32 = g.float()
            s.iterate(v, g32, first=1, count=1)
            torch.cuda.synchronize()
            a, c = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            s.iterate(v, g32, first=2, count=iters - 1)
            c.record()
            torch.cuda.synchronize()
            single_ms += a.elapsed_time(c) / (iters - 1)
            s.close()
            worst = max(worst, float(torch.linalg.vector_norm((bvol - v).double()) / torch.linalg.vector_norm(v.double())))
    # the batch runs one persistent launch per RS layout and per VI chunking among its jobs
    # (16-bit storage reads the hybrid layout as the texture)
    rs_groups = sorted({"tex" if v["rs_layout"] == "hybrid" else v["rs_layout"] for v in layouts.values()})
    vi_groups = sorted({v["vi_zc"] for v in layouts.values()})
    return {"workload": f"{jobs} uneven jobs (N in 64..256, views 60..360, magnification 1.5..2.5), BF16 storage, "
                        f"measured sinogram in FP32, {iters} iterations, graph replay, autotuned per size",
            "jobs": jobs, "autotuned": {str(k): v for k, v in sorted(layouts.items())},
            "persistent_launches_per_phase": {"projection": len(rs_groups), "backprojection": len(vi_groups),
                                              "rs_layouts": rs_groups, "vi_slices_per_thread": [16 * z for z in vi_groups]},
            "ms_per_iteration": round(ms, 3), "value": round(units / (ms / 1e3) / 1e9, 3),
            "unit": "Gvox-ray updates/s", "work_items_per_iteration": st["work_items"], "device_bytes": st["bytes"],
            "max_rel_l2_vs_fp32_single_job": float(f"{worst:.3e}"),
            "single_job_fp32": {"ms_per_iteration_all_jobs": round(single_ms, 3),
                                "value": round(units / (single_ms / 1e3) / 1e9, 3),
                                "note": "the same jobs one after another, FP32 single-job solver"}}


def run_config1(t, torch, dev, cpu: bool):
    """Plain method, small size: 256^3 modified Shepp-Logan, unit voxels, FOD 512, FDD 1024,
    256 views over 360 deg, 256 x 256 detector of pitch 2; RSVI projection once, then VI
    backprojection of that sinogram once. Device times by CUDA events (median of 5 after a
    warm-up), the host-buffer forms by wall clock, and -- the CPU-baseline leg -- the
    reference's own kernel sources built for the host, run once each on all host cores."""
    import numpy as np

    cfg = t.ConfigCT.cone_beam(256, 256, det=256, pitch=2.0, fod=512.0, magnification=2.0)
    ell = t.phantoms.modified_shepp_logan()
    U = cfg.voxel_ray_updates
    with t.Context(cfg, device=dev.index or 0) as ctx:
        vol = t.phantom(ell, 256, 256, 256, device=dev.index or 0)
        sino = ctx.project("RS", vol)
        back = ctx.backproject("VI", sino)
        torch.cuda.synchronize()
        pm, bm = [], []
        for _ in range(5):
            a, b, c = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            a.record()
            ctx.project("RS", vol, out=sino)
            b.record()
            ctx.backproject("VI", sino, out=back)
            c.record()
            torch.cuda.synchronize()
            pm.append(a.elapsed_time(b))
            bm.append(b.elapsed_time(c))
        vh = vol.cpu().numpy()
        ctx.project_host("RS", vh)
        t0 = time.perf_counter()
        sh = ctx.project_host("RS", vh)
        ctx.backproject_host("VI", sh)
        host_ms = 1e3 * (time.perf_counter() - t0)
    proj_ms, back_ms = float(np.median(pm)), float(np.median(bm))
    out = {"workload": "256^3 modified Shepp-Logan, 256 views, 256^2 detector pitch 2, FOD 512, FDD 1024: "
                       "RSVI proj once then VI back once, FP32",
           "proj_ms": round(proj_ms, 3), "back_ms": round(back_ms, 3),
           "value": round(2 * U / ((proj_ms + back_ms) / 1e3) / 1e9, 2), "unit": "Gvox-ray updates/s",
           "e2e_host_buffers_ms": round(host_ms, 2)}
    if cpu:
        import oracle

        vc = oracle.phantom(ell, 256, 256, 256)
        ref = oracle.ref_lib() is not None
        t0 = time.perf_counter()
        sc = oracle.ref_project(cfg, oracle.RS, vc) if ref else oracle.project(cfg, oracle.RS, vc)
        t1 = time.perf_counter()
        oracle.ref_backproject(cfg, sc) if ref else oracle.backproject(cfg, sc)
        t2 = time.perf_counter()
        out["cpu_baseline"] = {"proj_s": round(t1 - t0, 3), "back_s": round(t2 - t1, 3),
                               "value": round(2 * U / (t2 - t0) / 1e9, 3), "unit": "Gvox-ray updates/s",
                               "kind": "reference" if ref else "port",
                               "cores": int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1)),
                               "sample": "the whole workload (both operators, all 256 views)"}
    return out


def run_mixed(t, torch, dev, ctx, g, iters=20):
    """Mixed precision on the 512^3 workload: BF16 and FP16 storage of the operator inputs
    and outputs (FP32 ray sums, backprojection, residual and update; FP64 geometry and
    reductions) beside the FP32 run, 20 iterations each from zero; the measured sinogram
    either rounded to the 16-bit type or kept in FP32 (real_f32). Throughput, and the
    relative L2 difference of the final iterate against (a) the FP32 solver run on the same
    16-bit-rounded sinogram (the storage error alone) and (b) the FP32 run on the FP32
    sinogram. The errors against the FP64 oracle are stated at 256^3 by the test suite
    (the oracle takes about an hour of host time per run at 512^3)."""
    U = ctx.cfg.voxel_ray_updates
    res, out = {}, {}
    layouts = {}
    runs = (("f32", "f32", False, torch.float32), ("bf16", "bf16", False, torch.bfloat16),
            ("bf16_f32data", "bf16", True, torch.float32), ("f16", "f16", False, torch.float16),
            ("f16_f32data", "f16", True, torch.float32))
    for name, storage, real_f32, tdt in runs:
        p = t.GradientParams(gradient_iteration_nb=iters, optimal_step_iteration_nb=iters + 1,
                             regularization_parameter=LAMBDA, storage=storage, real_f32=real_f32)
        layouts[storage] = tune_context(t, ctx, ctx.cfg, storage, dev)
        s = t.Solver(ctx, p)
        vol = torch.zeros(ctx.cfg.volume_shape, device=dev)
        gs = g.to(tdt)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        s.iterate(vol, gs)
        b.record()
        torch.cuda.synchronize()
        ms = a.elapsed_time(b) / iters
        s.close()
        del gs
        res[name] = vol
        out[name] = {"ms_per_iteration": round(ms, 2), "value": round(3 * U / (ms / 1e3) / 1e9, 2),
                     "measured_sinogram": "f32" if real_f32 or storage == "f32" else storage}

    def rel(a, b):
        return float(f"{float(torch.linalg.vector_norm((a - b).double()) / torch.linalg.vector_norm(b.double())):.3e}")

    for storage, tdt in (("bf16", torch.bfloat16), ("f16", torch.float16)):
        # the FP32 solver on the sinogram as stored (rounded to 16 bits): what remains is the
        # error of 16-bit operator storage alone
        p = t.GradientParams(gradient_iteration_nb=iters, optimal_step_iteration_nb=iters + 1,
                             regularization_parameter=LAMBDA, storage="f32")
        tune_context(t, ctx, ctx.cfg, "f32", dev)
        s = t.Solver(ctx, p)
        same = torch.zeros(ctx.cfg.volume_shape, device=dev)
        s.iterate(same, g.to(tdt).float())
        s.close()
        out[storage]["rel_l2_vs_fp32_same_data"] = rel(res[storage], same)
        out[storage]["rel_l2_vs_fp32_fp32_data"] = rel(res[storage], res["f32"])
        out[storage + "_f32data"]["rel_l2_vs_fp32_fp32_data"] = rel(res[storage + "_f32data"], res["f32"])
        del same
    tune_context(t, ctx, ctx.cfg, "f32", dev)
    return {"workload": "iterative_recon_512, 20 iterations each from zero, RSVI, lambda 0.01", "unit": "Gvox-ray updates/s",
            "autotuned": layouts, **out}


SERVE_SIZES = [128, 256, 512, 768, 1024]
SERVE_WEIGHTS = [0.3, 0.3, 0.2, 0.15, 0.05]


def tune_context(t, ctx, cfg, storage, dev):
    """Sets a context's RS layout and VI chunking to the autotuner's choice for the size class
    (solvers take the tuning at creation) and returns it."""
    from tomogpi_b200 import autotune

    r = autotune.tune(cfg, storage, device=dev.index or 0)
    vl = r.get("vi_layout", "padded")
    ctx.set_tuning(rs_layout=r["rs_layout"], vi_zc=r["vi_zc"], vi_layout=vl)
    return {"rs_layout": r["rs_layout"], "vi_zc": r["vi_zc"], "vi_layout": vl}


def tuned(t, cfg, storage, dev):
    """Autotuned RS layout for the size class (cached) and 16 slices per VI thread: with one
    chunking for every job, each backprojection phase of a batch is one persistent launch
    (16-bit storage reads the hybrid layout as the texture, so the projection phases are
    one launch too)."""
    from tomogpi_b200 import autotune

    r = autotune.tune(cfg, storage, device=dev.index or 0)
    return {"rs_layout": r["rs_layout"], "vi_zc": 1}


def single_job_fp32_ms(t, torch, dev, cfg, g, iters=2):
    """ms per gradient iteration of the plain FP32 single-job solver on this job (after one
    warm-up iteration): the form the served and batched forms are compared with."""
    p32 = t.GradientParams(gradient_iteration_nb=iters + 1, optimal_step_iteration_nb=iters + 2,
                           regularization_parameter=LAMBDA, storage="f32")
    with t.Context(cfg, device=dev.index or 0) as ctx:
        s = t.Solver(ctx, p32)
        v = torch.zeros(cfg.volume_shape, device=dev)
        g32 = g.to(dev, torch.float32)
        s.iterate(v, g32, first=1, count=1)
        torch.cuda.synchronize()
        a, c = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        s.iterate(v, g32, first=2, count=iters)
        c.record()
        torch.cuda.synchronize()
        s.close()
    return a.elapsed_time(c) / iters


def run_serve_bench(t, torch, dev, count=16, rate_hz=0.5, iters=20, seed=77, shared_inputs=False):
    """Served stream: `count` Poisson arrivals at `rate_hz`; N in {128,256,512,768,1024}
    (weights 0.3/0.3/0.2/0.15/0.05), views = N, N x N detector, magnification 2, seeded
    random-ellipsoid phantom, Siddon sinogram + 1% noise held on the host in FP32 (pinned),
    20 iterations, BF16 storage / FP32 accumulation, autotuned per size; admission by HBM
    footprint into size-class lanes; latency = result on the host - arrival (includes the
    sinogram upload and the volume download). Beside it: the plain FP32 single-job solver's
    rate on each distinct size (two timed iterations, scaled to 20), summed over the jobs.
    shared_inputs (long streams): one seeded phantom per size class, its sinogram shared by
    the requests of that size, and each result volume dropped once it reached the host, so
    that a stream of a hundred jobs holds a few GB of host memory, not a hundred."""
    from tomogpi_b200.serve import Request, Server, latency_percentiles, poisson_stream

    params = t.GradientParams(gradient_iteration_nb=iters, optimal_step_iteration_nb=iters + 1,
                              regularization_parameter=LAMBDA, storage="bf16", real_f32=True)
    cfgs, fp32_ms = {}, {}

    shared = {}

    def mk(rid, n, arrival):
        if shared_inputs and n in shared:
            cfg, host = shared[n]
            cfgs[rid] = cfg
            return Request(rid, cfg, host, arrival, tuning=tuned(t, cfg, "bf16", dev))
        cfg, g = make_job_inputs(t, torch, n, n, 2.0, seed + (n if shared_inputs else rid), dev, torch.float32)
        if n not in fp32_ms:
            fp32_ms[n] = single_job_fp32_ms(t, torch, dev, cfg, g)
        host = torch.empty(g.shape, dtype=torch.float32, pin_memory=True)
        host.copy_(g)
        del g
        if shared_inputs:
            shared[n] = (cfg, host)
        cfgs[rid] = cfg
        return Request(rid, cfg, host, arrival, tuning=tuned(t, cfg, "bf16", dev))

    reqs = poisson_stream(seed, count, rate_hz, SERVE_SIZES, SERVE_WEIGHTS, mk)
    torch.cuda.empty_cache()
    def drop(res):
        res.volume = None

    srv = Server(params, device=dev.index or 0, on_result=drop if shared_inputs else None)
    t0 = time.perf_counter()
    res = srv.run(reqs)
    wall = time.perf_counter() - t0
    lanes = {l.spec.name: {"iterations": l.iterations, **{k: round(v, 1) for k, v in l.batch.host_times().items()}}
             for l in srv.lanes}
    host = {k: {"total_ms": round(1e3 * v[0], 1), "worst_ms": round(1e3 * v[1], 1)} for k, v in srv.host_time.items()}
    srv.close()
    units = sum(3 * cfgs[r.rid].voxel_ray_updates * iters for r in res)
    # time during which at least one job was admitted and not yet returned (the union of the
    # jobs' [admitted, finished] spans): the server's rate while it has work, without the
    # gaps between arrivals that a sustainable offered load leaves
    spans = sorted((r.admitted, r.finished) for r in res)
    busy, cur0, cur1 = 0.0, None, None
    for a, b in spans:
        if cur1 is None or a > cur1:
            busy += 0.0 if cur1 is None else cur1 - cur0
            cur0, cur1 = a, b
        else:
            cur1 = max(cur1, b)
    busy += 0.0 if cur1 is None else cur1 - cur0
    pct = latency_percentiles(res)
    sizes = sorted({cfgs[r.rid].x_volume_pixel_nb for r in res})
    per_size = {}
    for n in sizes:
        q = latency_percentiles([r for r in res if cfgs[r.rid].x_volume_pixel_nb == n])
        per_size[str(n)] = {"jobs": q["n"], "p50_ms": round(q["p50_ms"], 1), "max_ms": round(q["max_ms"], 1),
                            "queue_p50_ms": round(q["queue_p50_ms"], 1), "service_p50_ms": round(q["service_p50_ms"], 1)}
    single_s = sum(fp32_ms[cfgs[r.rid].x_volume_pixel_nb] * iters / 1e3 for r in res)
    del res
    return {"workload": f"{count} Poisson arrivals at {rate_hz:g}/s (seed {seed}), N in {{128,256,512,768,1024}} "
                        "(0.3/0.3/0.2/0.15/0.05), views = N, N x N detector, 1% noise, 20 iterations, "
                        "BF16 storage / FP32 accumulation, measured sinogram in FP32, autotuned per size",
            "n": pct["n"], "p50_ms": round(pct["p50_ms"], 2),
            "p99_ms": None if pct["p99_ms"] is None else round(pct["p99_ms"], 2),
            "p99_note": "reported from 100 results on; below that the max and the count" if pct["p99_ms"] is None
            else "", "max_ms": round(pct["max_ms"], 2), "queue_p50_ms": round(pct["queue_p50_ms"], 2),
            "service_p50_ms": round(pct["service_p50_ms"], 2), "per_size": per_size,
            "jobs_per_s": round(count / wall, 4), "value": round(units / wall / 1e9, 3),
            "unit": "Gvox-ray updates/s (wall clock from the first arrival, arrival gaps included)",
            "busy_s": round(busy, 3), "busy_value": round(units / busy / 1e9, 3),
            "busy_jobs_per_s": round(count / busy, 4),
            "busy_note": "over the time at least one job was in the server (arrival gaps with no job excluded)",
            "makespan_s": round(wall, 3), "lane_iterations": lanes, "host_loop": host,
            "single_job_fp32": {"busy_s": round(single_s, 3), "value": round(units / single_s / 1e9, 3),
                                "jobs_per_s_if_back_to_back": round(count / single_s, 4),
                                "note": "the same jobs one after another on the FP32 single-job solver, GPU "
                                        "time only (no arrival gaps, no transfers)"}}


def run_reference(args):
    world, rank, local = dist_setup()
    if rank != 0:
        return 0
    k = args.cpu_views
    ups, kind, cores, times, units = cpu_reference_sample(k, reps=args.steps, warm=args.warmup)
    value = ups / 1e9
    sample = (f"one gradient iteration's 3 operator calls (RS proj, VI back, RS proj) over {k} of the {VIEWS} "
              f"views at 512^3, every {VIEWS // k}-th (evenly spread over 360 deg; {units:.3g} updates per step)")
    line = {"metric": "proj+back Gvox-ray updates/s", "value": value, "unit": "Gvox-ray updates/s", "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config_dict({"sample_views": f"{k} of {VIEWS}, every {VIEWS // k}-th"}),
            "cpu_baseline": {"value": value, "unit": "Gvox-ray updates/s", "cores": cores, "kind": kind,
                             "sample": sample},
            "e2e": {"value": value, "unit": "Gvox-ray updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_sharded(t, torch, dev, cfg, args, world, rank, local):
    """--shard: the same 512^3 reconstruction split over the ranks by views
    (tomogpi_b200.sharded: one dJ all-reduce and a few scalars per iteration), every rank
    building the same seeded input; device time of K iterations, max over ranks. Strong
    scaling: the total work is one job whatever the number of GPUs."""
    from tomogpi_b200.replicas import max_over_ranks
    from tomogpi_b200.sharded import ShardedSolver

    iters = max(20, args.warmup + args.steps)
    params = t.GradientParams(gradient_iteration_nb=iters, optimal_step_iteration_nb=iters + 1,
                              regularization_parameter=LAMBDA, projector="RS", backprojector="VI", storage="f32")
    with t.Context(cfg, device=local) as full:
        truth = t.phantom(t.phantoms.config_phantom(1234, N), N, N, N, device=local)
        g = full.project("SIDDON", truth)
        gen = torch.Generator(device=dev).manual_seed(4321)
        g += torch.randn(g.shape, device=dev, generator=gen) * (0.01 * float(g.max()))
        del truth
    s = ShardedSolver(cfg, params, device=local, tuning={"rs_layout": "hybrid", "vi_zc": 1})
    part = s.real_part(g)
    del g
    vol = torch.zeros(cfg.volume_shape, device=dev)
    s.iterate(vol, part, first=1, count=args.warmup)
    torch.cuda.synchronize()
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    s.iterate(vol, part, first=args.warmup + 1, count=args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1), device=dev) / args.steps
    s.close()
    return {"workload": "iterative_recon_512_fp32 split by views over all ranks", "ranks": world,
            "views_per_rank": s.count, "ms_per_iteration": round(ms, 3),
            "value": round(3 * cfg.voxel_ray_updates / (ms / 1e3) / 1e9, 2), "unit": "Gvox-ray updates/s",
            "scaling": "strong", "rs_layout": "hybrid"}


def run_ours(args):
    import numpy as np
    import torch

    import tomogpi_b200 as t
    from tomogpi_b200.replicas import max_over_ranks

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
    cfg = workload_cfg()
    U = cfg.voxel_ray_updates
    total_it = args.warmup + args.steps
    iters = max(20, total_it)
    opt_nb = 21 if total_it <= 20 else total_it + 1  # the optimal step is computed on every iteration

    # --- synthetic inputs, resident in HBM --------------------------------------------
    ctx = t.Context(cfg, device=local)
    tuned_f32 = tune_context(t, ctx, cfg, "f32", dev)  # the project's autotuner, before any timing
    truth = t.phantom(t.phantoms.config_phantom(1234 + rank, N), N, N, N, device=local)
    g = ctx.project("SIDDON", truth)
    gen = torch.Generator(device=dev).manual_seed(4321 + rank)
    g += torch.randn(g.shape, device=dev, generator=gen) * (0.01 * float(g.max()))
    del truth
    params = t.GradientParams(gradient_iteration_nb=iters, optimal_step_iteration_nb=opt_nb,
                              regularization_parameter=LAMBDA, projector="RS", backprojector="VI", storage="f32")
    solver = t.Solver(ctx, params)
    vol = torch.zeros(cfg.volume_shape, device=dev)
    stream = torch.cuda.current_stream()

    def barrier():
        if world > 1:
            import torch.distributed as dist

            dist.barrier()

    # --- warm-up ------------------------------------------------------------------------
    solver.iterate(vol, g, first=1, count=args.warmup)
    torch.cuda.synchronize()
    solver.stats(reset=True)
    solver.set_timing(True)

    # --- timed region: K gradient iterations, device-timed --------------------------------
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        for i in range(args.steps):
            solver.iterate(vol, g, first=args.warmup + 1 + i, count=1)
        e1.record(stream)
        torch.cuda.synchronize()
    barrier()
    ms = e0.elapsed_time(e1)
    st = solver.stats(reset=True)
    solver.set_timing(False)
    ms_max = max_over_ranks(ms, device=dev)
    units_per_step = 3 * U
    value = units_per_step * args.steps * world / (ms_max / 1e3) / 1e9

    # --- roofline of the dominant kernel -----------------------------------------------
    peak, peak_kind = measured_peak()
    samples = ctx.count_samples("RS")
    rays = cfg.u_detector_pixel_nb * cfg.v_detector_pixel_nb * cfg.projection_nb
    nvox = N * N * N
    proj_avg = st["proj_ms"] / max(st["proj_launches"], 1)
    back_avg = st["back_ms"] / max(st["back_launches"], 1)
    if st["proj_ms"] >= st["back_ms"]:
        kern, avg_ms, alg_bytes = "rs_project_kernel", proj_avg, 8 * 4 * samples + 4 * rays
    else:
        kern, avg_ms, alg_bytes = "vi_back_kernel", back_avg, 4 * 4 * U + 4 * nvox
    achieved = alg_bytes / (avg_ms / 1e3) / 1e9
    kkey = f"{kern}:{tuned_f32['rs_layout']}" if kern == "rs_project_kernel" else kern
    traffic = profiled_traffic(kkey)
    dram_gbs = traffic / (avg_ms / 1e3) / 1e9 if traffic else None
    limits = profiled_limits(kkey)
    binds = limits["unit"] if limits else None
    roofline = {"bound": "hbm", "kernel": kern, "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                # what binds the kernel, from the committed ncu capture of the current code:
                # a memory-side kernel (no tensor work) held by that unit, not by DRAM bandwidth
                "binds": binds,
                "binds_pct_of_peak": limits.get(f"{binds}_pct") if limits else None,
                "frac": round(achieved / peak, 4), "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"
                if peak_kind == "measured" else "fallback 6650 GB/s",
                # achieved counts every sample's texel gather (8 texels per RS sample): served by
                # L1 / L2, not by DRAM, hence above the HBM peak; DRAM moves far less
                "l1l2_gather_gbs": round(achieved, 1),
                "dram_gbs": None if dram_gbs is None else round(dram_gbs, 1),
                "dram_frac": None if dram_gbs is None else round(dram_gbs / peak, 4),
                "limiter": limits,
                "vi_limiter": profiled_limits("vi_back_tma_kernel" if tuned_f32.get("vi_layout") == "tma"
                                              else "vi_back_kernel"),
                "traffic": traffic, "alg_bytes_per_launch": alg_bytes, "avg_launch_ms": round(avg_ms, 3),
                "rs_avg_launch_ms": round(proj_avg, 3), "vi_avg_launch_ms": round(back_avg, 3),
                "rs_samples_per_launch": samples,
                # s (N^3 + P Nu Nv): every volume and sinogram value moved once
                "compulsory_bytes_per_launch": 4 * (cfg.x_volume_pixel_nb * cfg.y_volume_pixel_nb *
                                                    cfg.z_volume_pixel_nb + cfg.projection_nb *
                                                    cfg.u_detector_pixel_nb * cfg.v_detector_pixel_nb),
                "rs_gupdates_per_s": round(U / proj_avg / 1e6, 1), "vi_gupdates_per_s": round(U / back_avg / 1e6, 1)}

    # --- end to end through the host-buffer API ------------------------------------------
    vol_h = torch.zeros(cfg.volume_shape, dtype=torch.float32).pin_memory().numpy()
    g_h = g.cpu().pin_memory().numpy()
    solver2 = t.Solver(ctx, params)
    solver2.iterate_host(vol_h, g_h, first=1, count=1)  # warm the host-form buffers
    barrier()
    torch.cuda.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for i in range(args.steps):
        solver2.iterate_host(vol_h, g_h, first=2 + i, count=1)
    f1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(f0.elapsed_time(f1), device=dev)
    e2e = {"value": units_per_step * args.steps * world / (e2e_ms / 1e3) / 1e9, "unit": "Gvox-ray updates/s",
           "h2d_bytes_per_step": 4 * nvox + 4 * cfg.projection_nb * N * N, "d2h_bytes_per_step": 4 * nvox,
           "api": "tomo_solver_iterate_host (pinned host buffers)"}
    solver2.close()

    # --- CPU baseline (rank 0, one GPU) ----------------------------------------------------
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        ups, kind, cores, times, units = cpu_reference_sample(args.cpu_views, reps=1)
        cpu = {"value": ups / 1e9, "unit": "Gvox-ray updates/s", "cores": cores, "kind": kind,
               "sample": f"RS proj + VI back + RS proj over {args.cpu_views} of the {VIEWS} views at 512^3, every "
                         f"{VIEWS // args.cpu_views}-th ({units:.3g} updates, {sum(times):.1f} s)"}

    shard_line = run_sharded(t, torch, dev, cfg, args, world, rank, local) if args.shard else None

    batch_line = serve_line = small_line = mixed_line = None
    if world == 1 and not args.no_batch:
        mixed_line = run_mixed(t, torch, dev, ctx, g)
        small_line = run_config1(t, torch, dev, cpu=rank == 0 and not args.no_cpu_baseline)
        batch_line = run_batch_bench(t, torch, dev)
        serve_line = run_serve_bench(t, torch, dev, count=args.serve_jobs, rate_hz=args.serve_rate)

    if rank == 0:
        line = {"metric": "proj+back Gvox-ray updates/s", "value": round(value, 3), "unit": "Gvox-ray updates/s",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_max / args.steps, 3),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": config_dict({"parallelism": f"job replicas x{world}" if world > 1 else "single job",
                                       "autotuned": tuned_f32}),
                "e2e": e2e, "gpu_launches": st["kernel_launches"], "roofline": roofline, "cpu_baseline": cpu,
                "clocks": clk.summary(), "small_plain": small_line, "mixed": mixed_line, "batched": batch_line,
                "sharded": shard_line,
                "served": serve_line}
        print(json.dumps(line), flush=True)
    solver.close()
    ctx.close()
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return 0


def run_served_only(args):
    """--served-only: the served stream alone (one GPU), printed as its own JSON line: for
    streams long enough to state a 99th percentile (from 100 results on)."""
    import torch

    import tomogpi_b200 as t

    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    line = run_serve_bench(t, torch, dev, count=args.serve_jobs, rate_hz=args.serve_rate, shared_inputs=True)
    line["inputs"] = "one seeded phantom per size class, shared by the requests of that size"
    print(json.dumps({"served": line}), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--cpu-views", type=int, default=16,
                    help="views of the CPU sample, evenly spread (512 / views a power of two)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--shard", action="store_true",
                    help="also time one reconstruction split over the ranks by views (strong scaling)")
    ap.add_argument("--no-batch", action="store_true",
                    help="skip the small plain, mixed-precision, batched and served measurements")
    ap.add_argument("--serve-jobs", type=int, default=16, help="arrivals of the served stream")
    ap.add_argument("--served-only", action="store_true",
                    help="run only the served stream (e.g. --serve-jobs 128 for a stated p99) and print it")
    ap.add_argument("--serve-rate", type=float, default=0.1,
                    help="Poisson arrival rate of the served stream (1/s); the GPU serves about 0.1 jobs/s of this mix")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("at least 3 warm-up steps")
    if args.served_only:
        return run_served_only(args)
    return run_reference(args) if args.impl == "reference" else run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
