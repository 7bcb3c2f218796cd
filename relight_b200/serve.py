"""Bake serving: continuous batching of lightmap bake requests on one GPU.

A request asks for one lightmap of one resident scene (BVH and gathered
photonmaps stay on the device) baked with direct light, AO and final
gather.  The server loop, once per iteration:

  1. moves requests whose arrival time has passed into the wait queue;
  2. retires requests whose last iteration the device has finished (their
     colours are in pinned host memory) and returns their HBM;
  3. admits waiting requests in arrival order while the HBM budget and the
     slot limit allow (a stream-ordered lightmap block, rasterised on the
     device);
  4. gives every active request a slice of its lumels (water-filling a
     per-iteration quantum: small requests finish in one iteration, large
     ones share the rest) and runs all slices as one batch (rl_batch_update
     + the captured graph of the batch kernels);
  5. for requests whose last slice ran, queues the colour copy and the
     lightmap's release behind the batch.

Requests that arrive while others are on the GPU join at the next
iteration, so their work overlaps on the device.  Each lumel is baked with
its request's Philox keys whatever slice or iteration it lands in, so a
result is bit-identical alone and in the mix.

The reference has no server: Relight::bake (Relight.cpp:132-163) hands one
job's lumels to worker threads and returns when they are done.
"""
from __future__ import annotations

import math
import time
from collections import deque
from dataclasses import dataclass, field, replace
from typing import Callable, Dict, List, Optional, Sequence

import numpy as np

from .batch import AO, DIRECT, INDIRECT, Batch, BakeJob, ResidentScenes


@dataclass
class Request:
    rid: int
    scene: int          # index into the resident scenes
    side: int           # lightmap width = height
    seed: int
    arrival: float      # seconds after the server starts
    t_admit: float = math.nan
    t_done: float = math.nan
    result: Optional[np.ndarray] = None  # [side*side][3] float32 colours

    @property
    def latency(self) -> float:
        return self.t_done - self.arrival


def poisson_arrivals(rate: float, n: int, seed: int) -> np.ndarray:
    """Arrival times of a Poisson stream of `rate` requests/s."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, n))


def make_requests(workload, rate: float, n: int, seed: int = 5, sides=(32, 1024)) -> List[Request]:
    """Requests drawn like the batch workload's jobs: a scene uniformly, a
    lightmap side log-uniform in `sides`; Poisson arrivals at `rate`/s."""
    rng = np.random.default_rng(seed)
    times = poisson_arrivals(rate, n, seed + 1)
    out = []
    for k in range(n):
        side = int(round(math.exp(rng.uniform(math.log(sides[0]), math.log(sides[1])))))
        out.append(Request(k, int(rng.integers(0, len(workload.scenes))), side, int(rng.integers(0, 2 ** 63)),
                           float(times[k])))
    return out


def plan_slices(remaining: Sequence[int], quantum: int, align: int = 32) -> List[int]:
    """Water-filling split of `quantum` work items over requests with
    `remaining` items: requests below the fair level get all they need, the
    rest share what is left equally (in multiples of `align`, except a
    request's final slice).  Every request with work gets at least `align`
    items (or its remainder), so each one progresses every iteration."""
    n = len(remaining)
    out = [0] * n
    order = sorted(range(n), key=lambda i: remaining[i])
    left = max(quantum, 0)
    for pos, i in enumerate(order):
        r = remaining[i]
        if r <= 0:
            continue
        fair = left // max(n - pos, 1)
        fair = max(align, (fair // align) * align)
        take = min(r, fair)
        out[i] = take
        left = max(left - take, 0)
    return out


class PinnedPool:
    """Page-locked host buffers for results, kept per power-of-two size
    class and reused, so admission never waits on a host allocation."""

    def __init__(self):
        self.free: Dict[int, list] = {}

    @staticmethod
    def _cls(nbytes: int) -> int:
        return max(1 << 16, 1 << (max(nbytes, 1) - 1).bit_length())

    def get(self, nbytes: int):
        import torch
        c = self._cls(nbytes)
        lst = self.free.setdefault(c, [])
        return lst.pop() if lst else torch.empty(c, dtype=torch.uint8, pin_memory=True)

    def put(self, buf):
        self.free.setdefault(buf.numel(), []).append(buf)

    def reserve(self, nbytes: int, count: int):
        bufs = [self.get(nbytes) for _ in range(count)]
        for b in bufs:
            self.put(b)


@dataclass
class _Active:
    req: Request
    lightmap: object
    total: int
    cursor: int = 0
    host: object = None  # pinned tensor for the colours
    fg_map: object = None  # with a denoiser: the final gather, denoised on completion


@dataclass
class ServeStats:
    requests: int
    p50_ms: float
    p99_ms: float
    mean_ms: float
    wait_p50_ms: float
    wait_p99_ms: float
    lightmaps_per_s: float
    texels_per_s: float
    iterations: int
    mean_active: float
    peak_bytes: int
    span_s: float

    def as_dict(self):
        return dict(self.__dict__)


class BakeServer:
    """Continuous-batching bake server over resident scenes.

    budget_bytes  HBM for request lightmaps (rl_map_bytes per request); the
                  resident scenes are held outside it.
    quantum       lumels per pass per iteration, summed over requests.
    """

    def __init__(self, resident: ResidentScenes, budget_bytes: int, quantum: int = 1 << 18,
                 fg_samples: int = 16, max_active: int = 256, torch_stream=None, denoiser=None, max_side: int = 1024):
        import torch
        from .device import DeviceMap
        self.rs = resident
        self.wl = resident.workload
        self.budget = int(budget_bytes)
        self.quantum = int(quantum)
        self.max_active = max_active
        self.torch_stream = torch_stream or torch.cuda.Stream()
        self.stream = self.torch_stream.cuda_stream
        self.fg = [replace(sc.settings, final_gather_samples=fg_samples) for sc in self.wl.scenes]
        self.denoiser = denoiser
        if denoiser is not None:
            denoiser.reserve(1, max_side, max_side)
        maps = 2 if denoiser is not None else 1
        self._map_bytes = lambda w, h: maps * DeviceMap.nbytes(w, h)
        self.pinned = PinnedPool()
        self.batch = Batch([])
        self.batch.capture(self.stream)

    # ------------------------------------------------------------ pieces
    def jobs_for(self, a: _Active, begin: int, end: int) -> List[BakeJob]:
        """The request's three passes over lumels [begin, end)."""
        r = a.req
        ds = self.rs.scenes[r.scene]
        kw = dict(begin=begin, end=end)
        fg_map = a.fg_map if a.fg_map is not None else a.lightmap
        return [BakeJob.direct(ds, a.lightmap, **kw),
                BakeJob.ambient_occlusion(ds, a.lightmap, self.wl.ao, seed=r.seed ^ 0xA0, **kw),
                BakeJob.indirect(ds, fg_map, self.rs.photonmaps[r.scene], self.fg[r.scene],
                                 seed=r.seed ^ 0xF6, **kw)]

    def _admit(self, r: Request, now: float) -> _Active:
        import torch
        from .device import DeviceMap
        ds = self.rs.scenes[r.scene]
        lm = DeviceMap(0, r.side, r.side, stream=self.stream, stream_ordered=True)
        for mi in range(len(ds.flat.mesh_photonmap)):
            lm.add_mesh(ds, mi, self.stream)
        fg = None
        if self.denoiser is not None:
            fg = DeviceMap(0, r.side, r.side, stream=self.stream, stream_ordered=True)
            for mi in range(len(ds.flat.mesh_photonmap)):
                fg.add_mesh(ds, mi, self.stream)
        r.t_admit = now
        host = self.pinned.get(r.side * r.side * 12)
        return _Active(r, lm, r.side * r.side, 0, host, fg)

    # -------------------------------------------------------------- loop
    def run(self, requests: Sequence[Request], clock: Optional[Callable[[], float]] = None,
            keep_results: bool = True) -> ServeStats:
        import torch
        t0 = time.perf_counter()
        clock = clock or (lambda: time.perf_counter() - t0)
        pending = deque(sorted(requests, key=lambda r: r.arrival))
        waiting: deque = deque()
        active: List[_Active] = []
        inflight: deque = deque()   # (event, [_Active finished in that iteration])
        used = peak = 0
        iters = 0
        active_sum = 0
        done: List[Request] = []

        def retire(entry):
            nonlocal used
            _ev, fin = entry
            now = clock()
            for a in fin:
                a.req.t_done = now
                if keep_results:
                    n = a.req.side * a.req.side
                    a.req.result = a.host[:12 * n].numpy().view(np.float32).reshape(n, 3).copy()
                self.pinned.put(a.host)
                used -= self._map_bytes(a.req.side, a.req.side)
                done.append(a.req)

        while pending or waiting or active or inflight:
            now = clock()
            while pending and pending[0].arrival <= now:
                waiting.append(pending.popleft())
            while inflight and inflight[0][0].query():
                retire(inflight.popleft())
            while waiting and len(active) < self.max_active:
                need = self._map_bytes(waiting[0].side, waiting[0].side)
                if need > self.budget:
                    raise ValueError(f"request {waiting[0].rid}: a {waiting[0].side}^2 lightmap exceeds the budget")
                if used + need > self.budget:
                    break
                active.append(self._admit(waiting.popleft(), now))
                used += need
                peak = max(peak, used)
            if active:
                shares = plan_slices([a.total - a.cursor for a in active], self.quantum)
                jobs, fin = [], []
                for a, q in zip(active, shares):
                    if q <= 0:
                        continue
                    jobs += self.jobs_for(a, a.cursor, a.cursor + q)
                    a.cursor += q
                    if a.cursor >= a.total:
                        fin.append(a)
                self.batch.update(jobs, self.stream)
                self.batch.replay(self.stream)
                for a in fin:
                    out = a.lightmap
                    if a.fg_map is not None:
                        # final = (direct, AO) + denoised final gather
                        self.denoiser.apply(self.rs.scenes[a.req.scene], a.fg_map,
                                            base=a.lightmap.device_arrays()["color"], stream=self.stream)
                        out = a.fg_map
                    out.download_color_async(a.host.data_ptr(), self.stream)
                    a.lightmap.close(self.stream)
                    if a.fg_map is not None:
                        a.fg_map.close(self.stream)
                ev = torch.cuda.Event()
                ev.record(self.torch_stream)
                inflight.append((ev, fin))
                iters += 1
                active_sum += len(active)
                active = [a for a in active if a.cursor < a.total]
                while len(inflight) > 2:
                    inflight[0][0].synchronize()
                    retire(inflight.popleft())
            elif inflight:
                inflight[0][0].synchronize()
                retire(inflight.popleft())
            elif pending:
                wait = pending[0].arrival - clock()
                if wait > 0:
                    time.sleep(min(wait, 0.05))
        lat = np.array([r.latency for r in done]) * 1e3
        wait_ms = np.array([r.t_admit - r.arrival for r in done]) * 1e3
        span = max(r.t_done for r in done) - min(r.arrival for r in done) if done else 0.0
        texels = sum(r.side * r.side for r in done)
        return ServeStats(len(done), float(np.percentile(lat, 50)) if len(lat) else math.nan,
                          float(np.percentile(lat, 99)) if len(lat) else math.nan,
                          float(lat.mean()) if len(lat) else math.nan,
                          float(np.percentile(wait_ms, 50)) if len(lat) else math.nan,
                          float(np.percentile(wait_ms, 99)) if len(lat) else math.nan,
                          len(done) / span if span > 0 else math.nan, texels / span if span > 0 else math.nan,
                          iters, active_sum / max(iters, 1), peak, span)

    def warm(self, sides=(32, 1024), count: int = 8):
        """Pre-allocate pinned result buffers for every size class in `sides`."""
        c = 1 << 16
        while c // 2 < sides[1] * sides[1] * 12:
            if c >= sides[0] * sides[0] * 12:
                self.pinned.reserve(c, count)
            c <<= 1

    def close(self):
        self.batch.close()


def bake_alone(resident: ResidentScenes, r: Request, fg_samples: int = 16, stream=None,
               denoiser=None) -> np.ndarray:
    """The request baked by itself through the single-job calls (the
    reference for the alone-vs-in-the-mix check); with a denoiser, the
    final gather goes to its own map, denoised onto the direct + AO map."""
    from .batch import run_per_job
    from .device import DeviceMap
    ds = resident.scenes[r.scene]
    wl = resident.workload
    lm = DeviceMap(0, r.side, r.side)
    for mi in range(len(ds.flat.mesh_photonmap)):
        lm.add_mesh(ds, mi, stream)
    fgm = lm
    if denoiser is not None:
        fgm = DeviceMap(0, r.side, r.side)
        for mi in range(len(ds.flat.mesh_photonmap)):
            fgm.add_mesh(ds, mi, stream)
    fg = replace(wl.scenes[r.scene].settings, final_gather_samples=fg_samples)
    jobs = [BakeJob.direct(ds, lm),
            BakeJob.ambient_occlusion(ds, lm, wl.ao, seed=r.seed ^ 0xA0),
            BakeJob.indirect(ds, fgm, resident.photonmaps[r.scene], fg, seed=r.seed ^ 0xF6)]
    run_per_job(jobs, stream)
    if denoiser is not None:
        denoiser.apply(ds, fgm, base=lm.device_arrays()["color"], stream=stream)
    out = fgm.download(stream, fields=("color",))["color"]
    lm.close()
    if fgm is not lm:
        fgm.close()
    return out
