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
import threading
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
    es = {"f32": 4, "bf16": 2, "f16": 2}[params.real_dtype()]
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
        self.inbox: list = []      # (Request, footprint) admitted, added by the lane's thread
        self.live: dict = {}       # job id -> (Request, volume, sinogram, footprint, admitted, host buffer)
        self.iterations = 0
        self.share = 1.0
        self.parked = 0            # bytes the batch keeps from removed jobs (textures, pool reserve)
        self.trim_requested = False
        self.adding = 0            # jobs taken from the inbox and not yet live
        self.thread: Optional[threading.Thread] = None
        batch.set_priority(priority)

    @property
    def holds(self) -> bool:
        return bool(self.live or self.inbox or self.adding)


class Server:
    """Continuous-batching reconstruction server on one device (size-class lanes).

    Threads: the caller's thread admits requests (HBM pool, lane choice); each lane has a
    host thread of its own that adds its admitted jobs, launches an iteration, waits for it
    (blocking only itself) and retires finished jobs. A CUDA call that waits for the device
    therefore delays only its own lane, never another lane's next launch."""

    def __init__(self, params: GradientParams, device: int = 0, hbm_budget: Optional[int] = None,
                 tuner: Optional[Callable[[ConfigCT, str], dict]] = None, graph: bool = True,
                 clock: Callable[[], float] = time.perf_counter, lanes: Sequence[LaneSpec] = DEFAULT_LANES,
                 on_result: Optional[Callable[["Result"], None]] = None):
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
        self.cv = threading.Condition()
        self.waiting: collections.deque = collections.deque()
        self.results: list = []
        self.on_result = on_result  # called (on a lane's thread) with each result as it is ready
        self.peak_live = 0
        self._stop = False
        self._error: Optional[BaseException] = None
        # host time per lane-thread phase, [total s, worst s]
        self.host_time = {"retire": [0.0, 0.0], "admit": [0.0, 0.0], "launch": [0.0, 0.0]}
        # pinned host buffers for the results, allocated while the job runs (page-locking
        # gigabytes is slow)
        self._pinner = concurrent.futures.ThreadPoolExecutor(max_workers=1)

    @property
    def iterations(self) -> int:
        return sum(l.iterations for l in self.lanes)

    @property
    def live(self) -> dict:
        out = {}
        for l in self.lanes:
            out.update({(l.spec.name, j): v for j, v in list(l.live.items())})
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
        with self.cv:
            self.waiting.append(req)

    def pending(self) -> bool:
        """True while requests wait or jobs are admitted, live or being copied out."""
        return bool(self.waiting or any(l.holds for l in self.lanes))

    # --- the caller's thread: admission -----------------------------------------------
    def _admit_locked(self) -> None:
        """Hands arrived requests whose footprint fits to their lanes (first come, first
        served with backfilling). Parked memory of the lanes counts; when it stands in the
        way the lanes are asked to trim it at their next iteration boundary."""
        now = self.now()
        kept = collections.deque()
        parked = sum(l.parked for l in self.lanes)
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
            if not self.pool.fits(need + parked):
                for l in self.lanes:
                    l.trim_requested = l.trim_requested or l.parked > 0
                kept.append(req)
                continue
            self.pool.take(need)
            self.lanes[lane_index(self.specs, req.cfg)].inbox.append((req, need))
        self.waiting = kept
        self.peak_live = max(self.peak_live, sum(len(l.live) + len(l.inbox) + l.adding for l in self.lanes))
        self.cv.notify_all()

    def _set_shares_locked(self) -> None:
        shares = lane_shares([l.holds for l in self.lanes])
        for l, s in zip(self.lanes, shares):
            if s != l.share:
                l.batch.set_share(s)
                l.share = s

    # --- lane threads ----------------------------------------------------------------------
    def _clocked(self, phase, t0):
        d = time.perf_counter() - t0
        with self.cv:
            h = self.host_time[phase]
            h[0] += d
            h[1] = max(h[1], d)

    def _add_jobs(self, lane: _Lane, new: list) -> None:
        torch = self.torch
        sdt = {"f32": torch.float32, "bf16": torch.bfloat16, "f16": torch.float16}[self.params.real_dtype()]
        for req, need in new:
            t0 = time.perf_counter()
            with torch.cuda.stream(lane.stream):
                src = req.sinogram if isinstance(req.sinogram, torch.Tensor) else \
                    torch.from_numpy(np.ascontiguousarray(req.sinogram))
                g = src.to(self.dev, dtype=sdt, non_blocking=True)
                vol = torch.zeros(req.cfg.volume_shape, device=self.dev)
            jid = lane.batch.add(req.cfg, vol, g, rs_layout=req.tuning["rs_layout"], vi_zc=req.tuning["vi_zc"])
            host = self._pinner.submit(torch.empty, req.cfg.volume_shape, dtype=torch.float32, pin_memory=True)
            with self.cv:
                lane.live[jid] = (req, vol, g, need, self.now(), host)
                lane.adding -= 1
                self._set_shares_locked()
            self._clocked("admit", t0)

    def _retire(self, lane: _Lane) -> None:
        torch = self.torch
        t0 = time.perf_counter()
        for jid in [j for j in list(lane.live) if lane.batch.status(j, stream=lane.stream)[0] >=
                    self.params.gradient_iteration_nb]:
            req, vol, g, need, adm, fut = lane.live[jid]
            lane.batch.remove(jid)
            host = fut.result()
            with torch.cuda.stream(lane.stream):
                host.copy_(vol, non_blocking=True)
                ev = torch.cuda.Event()
                ev.record(lane.stream)
            ev.synchronize()
            res = Result(req.rid, host, req.arrival, adm, self.now(), need, lane.spec.name)
            del vol, g
            if self.on_result is not None:  # e.g. hand the volume on and drop it here
                self.on_result(res)
            with self.cv:
                lane.live.pop(jid)
                self.pool.give(need)
                self.results.append(res)
                self._set_shares_locked()
                self.cv.notify_all()
        self._clocked("retire", t0)

    def _lane_loop(self, lane: _Lane) -> None:
        torch = self.torch
        try:
            torch.cuda.set_device(self.device)
            while True:
                with self.cv:
                    while not (self._stop or lane.inbox or lane.live or lane.trim_requested):
                        self.cv.wait()
                    if self._stop and (self._error is not None or not (lane.inbox or lane.live)):
                        return  # done, or another thread failed
                    new, lane.inbox = lane.inbox, []
                    trim, lane.trim_requested = lane.trim_requested, False
                    lane.adding = len(new)  # held while they are added
                if trim:
                    lane.batch.trim()
                if new:
                    self._add_jobs(lane, new)
                lane.parked = lane.batch.parked_bytes()
                if not lane.live:
                    with self.cv:
                        self.cv.notify_all()
                    continue
                t0 = time.perf_counter()
                lane.batch.iterate(1, stream=lane.stream)
                ev = torch.cuda.Event()
                ev.record(lane.stream)
                self._clocked("launch", t0)
                ev.synchronize()  # blocks this lane's thread only
                lane.iterations += 1
                self._retire(lane)
                lane.parked = lane.batch.parked_bytes()
        except BaseException as e:  # surfaced by run()
            with self.cv:
                self._error = e
                self._stop = True
                self.cv.notify_all()

    # --- driver ----------------------------------------------------------------------------
    def run(self, requests, poll: float = 0.05) -> list:
        """Serves the requests to the end. Arrival times count from the start of this call
        (tuning of the requests happens before it)."""
        for r in sorted(requests, key=lambda r: r.arrival):
            self.submit(r)
        self.t0 = self.clock()
        for l in self.lanes:
            l.thread = threading.Thread(target=self._lane_loop, args=(l,), name=f"lane-{l.spec.name}", daemon=True)
            l.thread.start()
        try:
            with self.cv:
                while True:
                    if self._error is not None:
                        raise self._error
                    self._admit_locked()
                    if not self.pending():
                        break
                    now = self.now()
                    future = [r.arrival - now for r in self.waiting if r.arrival > now]
                    self.cv.wait(timeout=max(1e-4, min([poll] + future)))
        finally:
            with self.cv:
                self._stop = True
                self.cv.notify_all()
            for l in self.lanes:
                l.thread.join()
        if self._error is not None:
            raise self._error
        return self.results

    def close(self):
        for l in self.lanes:
            l.batch.close()
        self._pinner.shutdown(wait=True)


def latency_percentiles(results, min_n_p99: int = 100) -> dict:
    """Time to reconstruction (result on the host - arrival) over the results: p50, mean and
    max, and p99 only from min_n_p99 results on (below that a "99th percentile" is an
    interpolation between the largest two or three latencies, so the max and the count are
    reported instead); plus its split into queueing (admission - arrival) and service
    (result - admission)."""
    lat = np.array([r.latency for r in results]) * 1e3
    if lat.size == 0:
        return {"n": 0, "p50_ms": None, "p99_ms": None}
    queue = np.array([r.admitted - r.arrival for r in results]) * 1e3
    service = np.array([r.finished - r.admitted for r in results]) * 1e3
    return {"n": int(lat.size), "p50_ms": float(np.percentile(lat, 50)),
            "p99_ms": float(np.percentile(lat, 99)) if lat.size >= min_n_p99 else None,
            "mean_ms": float(lat.mean()), "max_ms": float(lat.max()),
            "queue_p50_ms": float(np.percentile(queue, 50)), "queue_max_ms": float(queue.max()),
            "service_p50_ms": float(np.percentile(service, 50)), "service_max_ms": float(service.max())}


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
