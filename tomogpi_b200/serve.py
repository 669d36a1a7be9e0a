"""Serving: continuous batching of reconstruction jobs on one GPU.

Requests arrive over time (each: a configCT geometry and its measured sinogram). The loop
admits a waiting request as soon as its HBM footprint fits the pool (first come, first
served, with backfilling: a smaller request behind a blocked one may go first), uploads
its sinogram, adds it to the running ``Batch`` and keeps iterating. Every iteration
advances all live jobs at once (one persistent projection / backprojection launch over
all of them, replayed from a CUDA graph while the job set is unchanged); a job leaves the
batch after its last iteration, its volume is copied out and its memory returns to the
pool. Latency = completion time - arrival time.

Each job's result is bit-identical to running it alone (the batch's reductions are
deterministic per job), which ``tests/test_gpu_serve.py`` checks.
"""
from __future__ import annotations

import collections
import dataclasses
import time
from typing import Callable, Optional

import numpy as np

from .config import ConfigCT
from .operators import Batch, GradientParams


@dataclasses.dataclass
class Request:
    rid: int
    cfg: ConfigCT
    sinogram: np.ndarray           # host, [phi][v][u], any float dtype
    arrival: float                 # seconds on the server's clock
    tuning: Optional[dict] = None  # {"rs_layout": ..., "vi_zc": ...}; None = tuner / default


@dataclasses.dataclass
class Result:
    rid: int
    volume: np.ndarray
    arrival: float
    admitted: float
    finished: float
    footprint: int

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


class HBMPool:
    """Admission by device-memory footprint: a byte budget and the bytes held by live jobs."""

    def __init__(self, budget: int):
        self.budget = int(budget)
        self.used = 0

    def fits(self, nbytes: int) -> bool:
        return self.used + nbytes <= self.budget

    def take(self, nbytes: int) -> None:
        if not self.fits(nbytes):
            raise MemoryError("admission beyond the pool budget")
        self.used += nbytes

    def give(self, nbytes: int) -> None:
        self.used -= nbytes
        assert self.used >= 0


def job_footprint(cfg: ConfigCT, params: GradientParams, tuning: dict) -> int:
    """Bytes a job holds: the batch's work buffers plus its FP32 iterate and its sinogram."""
    es = {"f32": 4, "bf16": 2, "f16": 2}[params.storage]
    nvox = cfg.x_volume_pixel_nb * cfg.y_volume_pixel_nb * cfg.z_volume_pixel_nb
    nsino = cfg.projection_nb * cfg.u_detector_pixel_nb * cfg.v_detector_pixel_nb
    work = Batch.footprint(cfg, params, rs_layout=tuning.get("rs_layout", "tex"), vi_zc=tuning.get("vi_zc", 2))
    return work + 4 * nvox + es * nsino


class Server:
    """Continuous-batching reconstruction server on one device."""

    def __init__(self, params: GradientParams, device: int = 0, hbm_budget: Optional[int] = None,
                 tuner: Optional[Callable[[ConfigCT, str], dict]] = None, graph: bool = True,
                 clock: Callable[[], float] = time.perf_counter):
        import torch

        self.torch = torch
        self.params = params
        self.device = device
        self.dev = torch.device("cuda", device)
        if hbm_budget is None:
            free, _ = torch.cuda.mem_get_info(device)
            hbm_budget = int(free * 0.85)
        self.pool = HBMPool(hbm_budget)
        self.tuner = tuner
        self.batch = Batch(params, device=device, graph=graph)
        self.clock = clock
        self.t0 = clock()
        self.waiting: collections.deque = collections.deque()
        self.live = {}  # job id -> (Request, volume tensor, sinogram tensor, footprint, admitted)
        self.results: list = []
        self.iterations = 0

    def now(self) -> float:
        return self.clock() - self.t0

    def _tuning(self, cfg: ConfigCT) -> dict:
        if self.tuner is None:
            return {"rs_layout": "tex" if self.params.storage == "f32" else "cell8", "vi_zc": 2}
        t = self.tuner(cfg, self.params.storage)
        return {"rs_layout": t["rs_layout"], "vi_zc": min(int(t["vi_zc"]), 2)}  # the batch runs zc 1 or 2

    def submit(self, req: Request) -> None:
        if req.tuning is None:
            req.tuning = self._tuning(req.cfg)
        self.waiting.append(req)

    def _admit(self) -> int:
        torch = self.torch
        sdt = {"f32": torch.float32, "bf16": torch.bfloat16, "f16": torch.float16}[self.params.storage]
        now = self.now()
        admitted = 0
        kept = collections.deque()
        while self.waiting:
            req = self.waiting.popleft()
            if req.arrival > now:
                kept.append(req)
                continue
            need = job_footprint(req.cfg, self.params, req.tuning)
            if need > self.pool.budget:
                raise MemoryError(f"request {req.rid} needs {need} bytes, more than the whole pool")
            if not self.pool.fits(need):
                kept.append(req)  # backfill: later, smaller requests may still fit
                continue
            self.pool.take(need)
            g = torch.from_numpy(np.ascontiguousarray(req.sinogram)).to(self.dev, dtype=sdt)
            vol = torch.zeros(req.cfg.volume_shape, device=self.dev)
            jid = self.batch.add(req.cfg, vol, g, rs_layout=req.tuning["rs_layout"], vi_zc=req.tuning["vi_zc"])
            self.live[jid] = (req, vol, g, need, self.now())
            admitted += 1
        self.waiting = kept
        return admitted

    def _retire(self) -> int:
        done = [jid for jid in self.live if self.batch.status(jid)[0] >= self.params.gradient_iteration_nb]
        for jid in done:
            req, vol, g, need, adm = self.live.pop(jid)
            out = vol.cpu().numpy()
            self.batch.remove(jid)
            self.pool.give(need)
            self.results.append(Result(req.rid, out, req.arrival, adm, self.now(), need))
        return len(done)

    def step(self) -> bool:
        """Admit, run one iteration of every live job, retire finished ones. Returns False
        when nothing is live (the caller waits for the next arrival)."""
        self._admit()
        if not self.live:
            return False
        self.batch.iterate(1)
        self.iterations += 1
        self._retire()
        return True

    def run(self, requests, idle_sleep: float = 1e-4) -> list:
        """Serves the requests (arrival times on this server's clock) to the end."""
        for r in sorted(requests, key=lambda r: r.arrival):
            self.submit(r)
        while self.waiting or self.live:
            if not self.step():
                time.sleep(idle_sleep)
        return self.results

    def close(self):
        self.batch.close()


def latency_percentiles(results) -> dict:
    lat = np.array([r.latency for r in results]) * 1e3
    if lat.size == 0:
        return {"p50_ms": None, "p99_ms": None}
    return {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean()), "max_ms": float(lat.max())}


def poisson_stream(seed: int, count: int, rate_hz: float, sizes, weights, make_request):
    """count requests with exponential inter-arrival times (rate_hz) and sizes drawn with
    the given weights; make_request(rid, n, arrival) builds each Request."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(count):
        t += rng.exponential(1.0 / rate_hz)
        n = int(rng.choice(sizes, p=np.asarray(weights) / np.sum(weights)))
        out.append(make_request(i, n, t))
    return out
