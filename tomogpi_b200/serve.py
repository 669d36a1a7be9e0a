"""Serving: continuous batching of reconstruction jobs on one GPU.

Requests arrive over time (each: a configCT geometry and its measured sinogram). The loop
admits a waiting request as soon as its HBM footprint fits the pool (first come, first
served, with backfilling: a smaller request behind a blocked one may go first), uploads
its sinogram, adds it to a running ``Batch`` and keeps iterating. Every iteration of a
batch advances all of its live jobs at once (one persistent projection / backprojection
launch over all of them, replayed from a CUDA graph while the job set is unchanged); a job
leaves after its last iteration, its volume is copied out and its memory returns to the
pool. Latency = time the result is on the host - arrival time.

Lanes. One iteration of a batch lasts as long as its largest job's iteration (a 1024^3
job with 1024 views: seconds), so small jobs sharing a batch with it would wait that long
per iteration. Jobs are therefore split into size-class lanes (by their per-operator work
Nx*Ny*Nz*P); each lane is its own ``Batch`` on its own stream, lanes run concurrently, and
each lane is advanced as soon as its previous iteration ends. While several lanes hold
jobs, the SMs are split between them by the batches' CTA shares: the lane of the smallest
jobs may take every free slot (and its stream has the highest priority), every other lane
with jobs keeps 1/k of the persistent CTAs (k = lanes with jobs). A lane alone gets the
whole GPU. Admission into a lane happens at its iteration boundaries.

Each job's result is bit-identical to running it alone (a batch's reductions are
deterministic per job, and lanes share nothing but the SMs), which
``tests/test_gpu_serve.py`` checks.
"""
from __future__ import annotations

import collections
import concurrent.futures
import dataclasses
import math
import time
from typing import Callable, List, Optional, Sequence

import numpy as np

from .config import ConfigCT
from .operators import Batch, GradientParams


@dataclasses.dataclass
class Request:
    rid: int
    cfg: ConfigCT
    sinogram: object               # host [phi][v][u]: numpy array or CPU torch tensor (pinned: async upload)
    arrival: float                 # seconds on the server's clock
    tuning: Optional[dict] = None  # {"rs_layout": ..., "vi_zc": ...}; None = tuner / default


@dataclasses.dataclass
class Result:
    rid: int
    volume: object                 # host FP32 volume (torch tensor, pinned)
    arrival: float
    admitted: float
    finished: float
    footprint: int
    lane: str = ""

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
    work = Batch.footprint(cfg, params, rs_layout=tuning.get("rs_layout", "tex"), vi_zc=tuning.get("vi_zc", 1))
    return work + 4 * nvox + es * nsino


@dataclasses.dataclass(frozen=True)
class LaneSpec:
    name: str
    max_updates: float  # largest per-operator work Nx*Ny*Nz*P this lane takes


# N <= 256 (with up to N views), N <= 512, larger
DEFAULT_LANES = (LaneSpec("small", 256.0 ** 4), LaneSpec("medium", 512.0 ** 4), LaneSpec("large", math.inf))


def lane_index(specs: Sequence[LaneSpec], cfg: ConfigCT) -> int:
    w = float(cfg.voxel_ray_updates)
    for i, s in enumerate(specs):
        if w <= s.max_updates:
            return i
    return len(specs) - 1


def lane_shares(busy: Sequence[bool]) -> List[float]:
    """CTA share per lane: the first (smallest-job) busy lane 1.0, the other busy lanes 1/k
    (k = busy lanes), idle lanes 1.0 (their next launch starts with the whole GPU)."""
    k = sum(1 for b in busy if b)
    out = [1.0] * len(busy)
    first = True
    for i, b in enumerate(busy):
        if not b:
            continue
        if first:
            first = False
        else:
            out[i] = 1.0 / k
    return out


class _Lane:
    def __init__(self, spec: LaneSpec, batch: Batch, stream, priority: int):
        self.spec = spec
        self.batch = batch
        self.stream = stream
        self.event = None
        self.busy = False          # an iteration is in flight
        self.live = {}             # job id -> (Request, volume, sinogram, footprint, admitted, host buffer)
        self.iterations = 0
        self.share = 1.0
        batch.set_priority(priority)


class Server:
    """Continuous-batching reconstruction server on one device (size-class lanes)."""

    def __init__(self, params: GradientParams, device: int = 0, hbm_budget: Optional[int] = None,
                 tuner: Optional[Callable[[ConfigCT, str], dict]] = None, graph: bool = True,
                 clock: Callable[[], float] = time.perf_counter, lanes: Sequence[LaneSpec] = DEFAULT_LANES):
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
        self.specs = tuple(lanes)
        lo, hi = torch.cuda.Stream.priority_range() if hasattr(torch.cuda.Stream, "priority_range") else (0, -1)
        self.lanes = []
        for i, spec in enumerate(self.specs):
            pr = max(hi, min(lo, hi + i))  # smallest jobs: greatest priority
            self.lanes.append(_Lane(spec, Batch(params, device=device, graph=graph),
                                    torch.cuda.Stream(device=self.dev, priority=pr), pr))
        self.clock = clock
        self.t0 = clock()
        self.waiting: collections.deque = collections.deque()
        self.copying: list = []   # (event, Result, volume, sinogram, footprint)
        self.results: list = []
        # host time of the loop's phases, [total s, worst s]: a long worst case means a call
        # that waited for the device (the loop must never block on other lanes' kernels)
        self.host_time = {"retire": [0.0, 0.0], "admit": [0.0, 0.0], "launch": [0.0, 0.0]}
        # pinned host buffers for the results, allocated off the loop's thread while the job
        # runs (page-locking gigabytes takes long enough to delay other lanes' launches)
        self._pinner = concurrent.futures.ThreadPoolExecutor(max_workers=1)

    def _clocked(self, phase, fn, *a):
        t = time.perf_counter()
        r = fn(*a)
        d = time.perf_counter() - t
        h = self.host_time[phase]
        h[0] += d
        h[1] = max(h[1], d)
        return r

    @property
    def iterations(self) -> int:
        return sum(l.iterations for l in self.lanes)

    @property
    def live(self) -> dict:
        out = {}
        for l in self.lanes:
            out.update({(l.spec.name, j): v for j, v in l.live.items()})
        return out

    def now(self) -> float:
        return self.clock() - self.t0

    def _tuning(self, cfg: ConfigCT) -> dict:
        if self.tuner is None:
            return {"rs_layout": "tex", "vi_zc": 1}
        t = self.tuner(cfg, self.params.storage)
        return {"rs_layout": t["rs_layout"], "vi_zc": min(int(t["vi_zc"]), 2)}  # the batch runs zc 1 or 2

    def submit(self, req: Request) -> None:
        if req.tuning is None:
            req.tuning = self._tuning(req.cfg)
        self.waiting.append(req)

    def _admit(self) -> int:
        """Admits arrived requests whose footprint fits, into idle lanes only (a busy lane
        takes new jobs at its next iteration boundary)."""
        torch = self.torch
        sdt = {"f32": torch.float32, "bf16": torch.bfloat16, "f16": torch.float16}[self.params.storage]
        now = self.now()
        admitted = 0
        kept = collections.deque()
        while self.waiting:
            req = self.waiting.popleft()
            lane = self.lanes[lane_index(self.specs, req.cfg)]
            if req.arrival > now or lane.busy:
                kept.append(req)
                continue
            need = job_footprint(req.cfg, self.params, req.tuning)
            if need > self.pool.budget:
                raise MemoryError(f"request {req.rid} needs {need} bytes, more than the whole pool")
            if not self.pool.fits(need):
                kept.append(req)  # backfill: later, smaller requests may still fit
                continue
            # texture arrays parked by the lanes (for reuse by jobs of the same size) are
            # device memory too: free them, which synchronises the device, only when they
            # stand in the way
            if not self.pool.fits(need + self._parked()):
                for l in self.lanes:
                    l.batch.trim()
            self.pool.take(need)
            with torch.cuda.stream(lane.stream):
                src = req.sinogram if isinstance(req.sinogram, torch.Tensor) else \
                    torch.from_numpy(np.ascontiguousarray(req.sinogram))
                g = src.to(self.dev, dtype=sdt, non_blocking=True)
                vol = torch.zeros(req.cfg.volume_shape, device=self.dev)
            jid = lane.batch.add(req.cfg, vol, g, rs_layout=req.tuning["rs_layout"], vi_zc=req.tuning["vi_zc"])
            host = self._pinner.submit(torch.empty, req.cfg.volume_shape, dtype=torch.float32, pin_memory=True)
            lane.live[jid] = (req, vol, g, need, self.now(), host)
            admitted += 1
        self.waiting = kept
        return admitted

    def _parked(self) -> int:
        return sum(l.batch.parked_bytes() for l in self.lanes)

    def _retire(self, lane: _Lane) -> int:
        torch = self.torch
        done = [j for j in lane.live if lane.batch.status(j, stream=lane.stream)[0] >= self.params.gradient_iteration_nb]
        for jid in done:
            req, vol, g, need, adm, fut = lane.live.pop(jid)
            lane.batch.remove(jid)
            host = fut.result()
            with torch.cuda.stream(lane.stream):
                host.copy_(vol, non_blocking=True)
                ev = torch.cuda.Event()
                ev.record(lane.stream)
            self.copying.append((ev, Result(req.rid, host, req.arrival, adm, 0.0, need, lane.spec.name), vol, g, need))
        return len(done)

    def _collect(self) -> None:
        keep = []
        for ev, res, vol, g, need in self.copying:
            if ev.query():
                res.finished = self.now()
                self.pool.give(need)
                self.results.append(res)
            else:
                keep.append((ev, res, vol, g, need))
        self.copying = keep

    def _set_shares(self) -> None:
        shares = lane_shares([bool(l.live) for l in self.lanes])
        for l, s in zip(self.lanes, shares):
            if s != l.share:
                l.batch.set_share(s)
                l.share = s

    def step(self) -> bool:
        """Retires finished lanes' jobs, admits, relaunches idle lanes. Returns False when
        nothing is in flight (the caller may sleep until the next arrival)."""
        for lane in self.lanes:
            if lane.busy and lane.event.query():
                lane.busy = False
                self._clocked("retire", self._retire, lane)
        self._collect()
        self._clocked("admit", self._admit)
        self._set_shares()
        for lane in self.lanes:
            if not lane.busy and lane.live:
                self._clocked("launch", self._launch, lane)
        return any(l.busy for l in self.lanes) or bool(self.copying)

    def _launch(self, lane: _Lane) -> None:
        lane.batch.iterate(1, stream=lane.stream)
        lane.event = self.torch.cuda.Event()
        lane.event.record(lane.stream)
        lane.busy = True
        lane.iterations += 1

    def pending(self) -> bool:
        """True while requests wait, jobs are live or results are still being copied out."""
        return bool(self.waiting or self.copying or any(l.live or l.busy for l in self.lanes))

    def run(self, requests, poll: float = 2e-4) -> list:
        """Serves the requests to the end. Arrival times count from the start of this call
        (tuning of the requests happens before it)."""
        for r in sorted(requests, key=lambda r: r.arrival):
            self.submit(r)
        self.t0 = self.clock()
        while self.pending():
            self.step()
            time.sleep(poll)
        return self.results

    def close(self):
        for l in self.lanes:
            l.batch.close()
        self._pinner.shutdown(wait=True)


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
