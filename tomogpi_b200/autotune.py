"""Autotuner: per size class, pick the RS input layout and the VI form by timing the
candidates on the device, and cache the choice.

Candidates: RS layout in {tex, hybrid, cell8, plain}; VI slices per thread in
{16, 32, 64} (vi_zc 1, 2, 4) from the padded sinogram, or 16 slices from sinogram windows
staged in shared memory by TMA (vi_layout "tma"). The trials run the first k and 2k views of the job's own
geometry, with CUDA-event timing after a warm-up, and are extrapolated to the job's view
count. Results are cached in JSON (``$TOMOGPI_B200_TUNE_CACHE`` or
``~/.cache/tomogpi_b200/autotune.json``) keyed by the GPU name and the size class.
"""
from __future__ import annotations

import json
import os
from pathlib import Path

from .config import ConfigCT

_CACHE = Path(os.environ.get("TOMOGPI_B200_TUNE_CACHE",
                             str(Path.home() / ".cache" / "tomogpi_b200" / "autotune.json")))
_mem = None


def _load():
    global _mem
    if _mem is None:
        try:
            _mem = json.loads(_CACHE.read_text())
        except Exception:
            _mem = {}
    return _mem


def _save():
    # written to a file of this process, then renamed over the cache: processes that tune at
    # the same time (one per GPU) never leave a half-written cache behind
    try:
        _CACHE.parent.mkdir(parents=True, exist_ok=True)
        tmp = _CACHE.with_name(f"{_CACHE.name}.{os.getpid()}.tmp")
        tmp.write_text(json.dumps(_load(), indent=1, sort_keys=True))
        os.replace(tmp, _CACHE)
    except OSError:
        pass  # a read-only home only loses the cache


def size_key(cfg: ConfigCT, storage: str, gpu: str) -> str:
    return (f"v3|{gpu}|{cfg.x_volume_pixel_nb}x{cfg.y_volume_pixel_nb}x{cfg.z_volume_pixel_nb}|"
            f"{cfg.u_detector_pixel_nb}x{cfg.v_detector_pixel_nb}|{storage}")


def first_views(cfg: ConfigCT, k: int) -> ConfigCT:
    """The first k views of the scan with the same angular step: phi_p = (p + s) * step."""
    s0 = cfg.num_start_angle / cfg.den_start_angle
    s1 = cfg.num_stop_angle / cfg.den_stop_angle
    return cfg.replace(projection_nb=k, num_start_angle=s0, den_start_angle=1.0,
                       num_stop_angle=s0 + k * (s1 - s0) / cfg.projection_nb, den_stop_angle=1.0)


def pick(trials: dict) -> dict:
    """Fastest RS layout and VI form from {'rs_<layout>': ms, 'vi_zc<k>': ms, 'vi_tma': ms}:
    the TMA form when it beats every padded chunking (its chunking is 16 slices), else the
    fastest chunking; "vi_zc" is always a padded chunking (the batched kernels read the
    padded residual)."""
    rs = {k[3:]: v for k, v in trials.items() if k.startswith("rs_")}
    vi = {int(k[5:]): v for k, v in trials.items() if k.startswith("vi_zc")}
    zc = min(vi, key=vi.get)
    tma = trials.get("vi_tma")
    return {"rs_layout": min(rs, key=rs.get), "vi_zc": zc,
            "vi_layout": "tma" if tma is not None and tma < vi[zc] else "padded"}


def _time(fn, reps=3):
    import torch

    fn()
    torch.cuda.synchronize()
    best = float("inf")
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        torch.cuda.synchronize()
        best = min(best, a.elapsed_time(b))
    return best


def extrapolate(t_k: float, t_2k: float, k: int, views: int) -> float:
    """Time of a call over `views` views from trials over k and 2k views: a fixed part
    (input preparation, launch) plus a per-view part."""
    return t_k + (t_2k - t_k) * (views - k) / k


def tune(cfg: ConfigCT, storage: str = "f32", device: int = 0, trial_views: int = 64, vi_zcs=(1, 2, 4),
         force: bool = False) -> dict:
    """Returns {"rs_layout", "vi_zc", "trials", "trial_views"} for this size class. Each
    candidate runs over the first k and 2k views of the job's geometry; `trials` holds the
    times extrapolated to the job's view count (the fixed per-call cost -- e.g. filling a
    layout's input buffers -- would otherwise dominate a short trial)."""
    import torch

    from .operators import Context

    gpu = torch.cuda.get_device_name(device)
    key = size_key(cfg, storage, gpu)
    cache = _load()
    if key in cache and not force:
        return cache[key]
    P = cfg.projection_nb
    k = max(1, min(trial_views, P // 2 if P >= 2 else 1))
    tdt = {"f32": torch.float32, "bf16": torch.bfloat16, "f16": torch.float16}[storage]
    dev = torch.device("cuda", device)
    raw = {}
    # the padded layout (eight scalar loads per sample) is the slowest from 384^3 on
    big = cfg.x_volume_pixel_nb * cfg.y_volume_pixel_nb * cfg.z_volume_pixel_nb >= 384 ** 3
    layouts = ("tex", "hybrid", "cell8") if big else ("tex", "hybrid", "cell8", "plain")
    if storage == "f32":  # MARCH is an FP32 layout (16-bit storage runs it as TEX)
        layouts += ("march",)
    for views in sorted({k, min(2 * k, P)}):
        sub = first_views(cfg, views)
        with Context(sub, device=device) as ctx:
            vol = torch.rand(sub.volume_shape, device=dev).to(tdt)
            sino = torch.empty(sub.sinogram_shape, device=dev, dtype=tdt)
            for lay in layouts:
                ctx.set_tuning(rs_layout=lay)
                raw[(f"rs_{lay}", views)] = _time(lambda: ctx.project("RS", vol, out=sino), reps=2)
            res = torch.rand(sub.sinogram_shape, device=dev)
            dj = torch.empty(sub.volume_shape, device=dev)
            for zc in vi_zcs:
                ctx.set_tuning(vi_zc=zc)
                raw[(f"vi_zc{zc}", views)] = _time(lambda: ctx.backproject("VI", res, out=dj), reps=2)
            ctx.set_tuning(vi_zc=1, vi_layout="tma")
            raw[("vi_tma", views)] = _time(lambda: ctx.backproject("VI", res, out=dj), reps=2)
            ctx.set_tuning(vi_layout="padded")
            del vol, sino, res, dj
    k2 = min(2 * k, P)
    trials = {}
    for name in {n for n, _ in raw}:
        trials[name] = extrapolate(raw[(name, k)], raw[(name, k2)], k, P) if k2 > k else raw[(name, k)]
    out = dict(pick(trials), trials=trials, trial_views=[k, k2])
    cache[key] = out
    _save()
    return out
