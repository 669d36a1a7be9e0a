"""A small, fixed operator case for profilers (ncu) and quick timing.

    python profile_case.py --n 384 --op rs --storage bf16 --layout tex

Builds an n^3 modified Shepp-Logan volume, a cone-beam geometry (n views over 360 deg unless
--views, n x n detector of pitch 2, FOD 2n, FDD 4n), runs --warmup untimed calls of the
chosen operator, then --reps timed calls, and prints the median CUDA-event time per call
with the updates/s. Operators: rs (RS projection), rs_um, siddon, vi (VI backprojection of
the projected sinogram), vi_um, iter (one gradient iteration of the single-job solver).
"""
from __future__ import annotations

import argparse
import json
import statistics

import torch

import sys
from pathlib import Path

sys.path.insert(0, str(Path(__file__).resolve().parent))

from tomogpi_b200 import ConfigCT, Context, GradientParams, Solver, phantom, phantoms  # noqa: E402


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=384)
    ap.add_argument("--views", type=int, default=0)
    ap.add_argument("--op", default="rs", choices=["rs", "rs_um", "siddon", "vi", "vi_um", "iter"])
    ap.add_argument("--storage", default="f32", choices=["f32", "bf16", "f16"])
    ap.add_argument("--layout", default="tex", choices=["tex", "hybrid", "march", "cell8", "plain"])
    ap.add_argument("--vi-zc", type=int, default=2, choices=[1, 2, 4])
    ap.add_argument("--vi-layout", default="padded", choices=["padded", "tex", "tma"])
    ap.add_argument("--warp-u", type=int, default=0, choices=[0, 8, 16, 32], help="RS rays of a warp along u")
    ap.add_argument("--tile-u", type=int, default=0, choices=[0, 16, 32, 64, 128], help="RS rays of a block along u")
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--reps", type=int, default=2)
    a = ap.parse_args(argv)
    n, views = a.n, a.views or a.n
    cfg = ConfigCT.cone_beam(n, views, det=n)
    dt = {"f32": torch.float32, "bf16": torch.bfloat16, "f16": torch.float16}[a.storage]
    with Context(cfg) as ctx:
        ctx.set_tuning(rs_layout=a.layout, vi_zc=a.vi_zc, vi_layout=a.vi_layout, rs_warp_u=a.warp_u, rs_tile_u=a.tile_u)
        vol = phantom(phantoms.config_phantom(0, n), n, n, n)
        sino = ctx.project("RS", vol)
        v_in, s_in = vol.to(dt), sino.to(dt)
        if a.op == "iter":
            s = Solver(ctx, GradientParams(gradient_iteration_nb=a.warmup + a.reps, storage=a.storage,
                                           optimal_step_iteration_nb=a.warmup + a.reps + 1))
            it = torch.zeros(cfg.volume_shape, device=vol.device)
            state = {"k": 1}

            def call():
                s.iterate(it, s_in, first=state["k"], count=1)
                state["k"] += 1
            units = 3 * cfg.voxel_ray_updates
        elif a.op in ("rs", "rs_um", "siddon"):
            kind = {"rs": "RS", "rs_um": "RS_UM", "siddon": "SIDDON"}[a.op]
            out = torch.empty(cfg.sinogram_shape, device=vol.device, dtype=dt)

            def call():
                ctx.project(kind, v_in, out=out)
            units = cfg.voxel_ray_updates
        else:
            kind = "VI" if a.op == "vi" else "VI_UM"
            out = torch.empty(cfg.volume_shape, device=vol.device, dtype=dt)

            def call():
                ctx.backproject(kind, s_in, out=out)
            units = cfg.voxel_ray_updates
        for _ in range(a.warmup):
            call()
        torch.cuda.synchronize()
        ms = []
        for _ in range(a.reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            call()
            e1.record()
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
        med = statistics.median(ms)
        print(json.dumps({"n": n, "views": views, "op": a.op, "storage": a.storage, "layout": a.layout,
                          "vi_zc": a.vi_zc, "vi_layout": a.vi_layout, "warp_u": a.warp_u or 8, "tile_u": a.tile_u or 32, "ms": round(med, 3), "gupdates_per_s": round(units / med / 1e6, 1)}))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
