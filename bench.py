"""Benchmark: Relight's photon-mapping + final-gather bake on one B200.

Workload (a "step"): the 256x256-vertex fBm terrain (amplitude 5, 2x2 tiles)
plus 2,000 boxes, 154,050 triangles, one sun + 4 point lights; one shared
1024x1024 lightmap and photonmap.  A step runs Relight::emitPhotons
(8 passes x 5 lights x 25,000 = 1,000,000 photons, up to 3 bounces, then
Photonmap::gather with radius 7) and Relight::bakeIndirectLight (256 final-
gather rays per valid lumel) — the reference's own call sequence.

  value  lightmap texels baked per second, device time, all inputs resident
         (the scene's BVH and lumels live in HBM; photonmap and lightmap
         colours are cleared at the start of each step).
  e2e    the same step through the C ABI with host buffers: lumel inputs
         uploaded from pinned memory and the baked colours read back, inside
         the timed region.
Between timed steps L2 is flushed (a 256 MiB write, outside the step's
events).  Multi-GPU (torchrun): every rank bakes its own copy of the job with
its own seed (weak scaling, no collective on the data path); the time is the
max over ranks.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# Per-ray algorithmic bytes of a final-gather ray on this scene, measured on
# the canonical binary SAH BVH by oracle/ray_bytes.py:
# 48 B ray I/O + 32 B x 43.78 box tests + 48 B x 2.80 triangle tests.
RAY_MODEL = {"n_box": 43.78, "n_tri": 2.80, "bytes_per_ray": 1583.6}
METRIC = "lightmap texels/s (photons + gather + final gather 256 spp, 1024^2)"
# --gather knn: the k-nearest-neighbour photon estimate (k = 100 deposits
# within a radius cap of 2 world units), run after the disc gather.
KNN_K, KNN_RADIUS = 100, 2.0
UNIT = "texels/s"
WORKLOAD = "terrain 256^2 verts + 2000 boxes (154,050 tris), 1M photons x3 bounces, gather r7, FG 256 spp, 1024^2"
L2_BYTES = 126 << 20
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one full-size
# k_indirect launch in one ncu capture, and the build it was captured on.
FG_DRAM_TRAFFIC = {"bytes": 85_620_000, "captured_on": "k_indirect<2> with per-triangle shading records and "
                   "three-input min/max slab tests (79.87 MB read + 5.75 MB written, 41.33 ms launch under ncu)"}


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks + throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        mhz, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            parts = [p.strip() for p in l.split(",")]
            try:
                mhz.append(float(parts[1]))
                mx = float(parts[2])
            except (ValueError, IndexError):
                continue
            for name, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(mhz) if mhz else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(mhz)}


SMALL = False


def build_workload(seed):
    from relight_b200 import scenes
    if SMALL:  # profiling case: same scene, 512^2 map, 64 spp, 2 photon passes
        return scenes.terrain_scene(seed=2, size=512, fg_samples=64, passes=2)
    return scenes.terrain_scene(seed=2)


def terrain_config(st, valid, ntris, world, knn=False, split=False):
    """The workload description both arms print (the same dict)."""
    return {"workload": WORKLOAD + (f", kNN k={KNN_K} r={KNN_RADIUS}" if knn else ""),
            "gather": "knn" if knn else "disc", "lightmap": [1024, 1024] if not SMALL else [512, 512],
            "valid_texels": valid, "photons": int(st.photon_pass_count * 125000),
            "fg_samples": st.final_gather_samples, "triangles": ntris,
            "parallelism": f"one bake split x{world}" if split else f"replicas x{world}",
            "l2": "flushed between steps (256 MiB write)"}


def gpu_arm(args, rank, world, local_rank):
    import torch
    from relight_b200 import _abi, autotune
    from relight_b200.device import Relight, _map_array

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    stream = torch.cuda.current_stream(dev)
    sh = stream.cuda_stream
    w = build_workload(rank)
    st = w.settings
    rl = Relight(stream=sh, seed=1000 + rank)
    ds = rl.device_scene(w.scene)
    torch.cuda.synchronize()
    lmap, pmap = w.lightmap._device, w.photonmap._device
    L = _abi.lib()
    flat = w.scene.flat
    lights = C.c_void_p(flat.lights.ctypes.data)
    maps = _map_array([pmap])
    sky = (C.c_float * 3)(*[float(x) for x in st.sky_color])
    amb = (C.c_float * 3)(*[float(x) for x in st.ambient_color])
    valid = lmap.valid_count()
    rays_per_step = valid * st.final_gather_samples
    launches_per_step = 3  # k_photons, k_gather, k_indirect

    ev = lambda: torch.cuda.Event(enable_timing=True)

    knn = args.gather == "knn"
    split = args.split
    if split and knn:
        raise SystemExit("--split runs the disc gather only")
    if split:
        from relight_b200 import parallel
        # photon share, all-reduce (colour + count), gather; final gather over
        # LumelBakeIterator(rank, world), all-reduce, add
        launches_per_step = 3
    records = None
    if knn:
        from relight_b200.device import PhotonRecords
        records = PhotonRecords(8 << 20)
        # k_knn_bounds, k_knn_grid, k_knn_keys, radix sort (counted as one), k_knn_scatter, k_knn_start, k_knn_query
        launches_per_step += 7

    def step(seed, fg_events=None, knn_events=None, lmap_ready=None):
        """One bake: photons, gather, final gather.  lmap_ready: an event the
        lightmap's inputs land on (uploaded on another stream); the lightmap is
        then cleared and baked only after it, while photons and the gather run."""
        _abi.check(L.rl_map_clear(pmap.handle, 1, 1, sh))
        if lmap_ready is None:
            _abi.check(L.rl_map_clear(lmap.handle, 1, 0, sh))
        if split:
            parallel.emit_photons_distributed(rl, w.scene, st, seed)
            if fg_events:
                fg_events[0].record(stream)
            parallel.bake_indirect_distributed(rl, w.scene, w.meshes[0], st, seed + 1)
            if fg_events:
                fg_events[1].record(stream)
            return
        if knn:
            _abi.check(L.rl_emit_photons_records(ds.handle, maps, 1, lights, len(flat.lights), st.photon_pass_count,
                                                 st.photon_bounce_count, st.photon_energy_threshold,
                                                 st.photon_max_distance, seed, records.handle, None, sh))
        else:
            _abi.check(L.rl_emit_photons(ds.handle, maps, 1, lights, len(flat.lights), st.photon_pass_count,
                                         st.photon_bounce_count, st.photon_energy_threshold, st.photon_max_distance,
                                         seed, None, sh))
        _abi.check(L.rl_photonmap_gather(pmap.handle, st.final_gather_radius, sh))
        if knn:
            if knn_events:
                knn_events[0].record(stream)
            records.gather_knn(pmap, 0, KNN_K, KNN_RADIUS, sh)
            if knn_events:
                knn_events[1].record(stream)
        if lmap_ready is not None:
            stream.wait_event(lmap_ready)
            _abi.check(L.rl_map_clear(lmap.handle, 1, 0, sh))
        if fg_events:
            fg_events[0].record(stream)
        _abi.check(L.rl_bake_indirect(ds.handle, lmap.handle, maps, 1, st.final_gather_samples,
                                      st.final_gather_distance, sky, amb, seed + 1, None, sh))
        if fg_events:
            fg_events[1].record(stream)

    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    for i in range(args.warmup):
        step(7 + 2 * i)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    step_ms, fg_ms, knn_ms = [], [], []
    with ClockSampler(local_rank) as clocks:
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        for i in range(args.steps):
            flush.zero_()
            e0, e1, f0, f1, k0, k1 = ev(), ev(), ev(), ev(), ev(), ev()
            e0.record(stream)
            step(1001 + 2 * i, (f0, f1), (k0, k1))
            e1.record(stream)
            torch.cuda.synchronize()
            step_ms.append(e0.elapsed_time(e1))
            fg_ms.append(f0.elapsed_time(f1))
            if knn:
                knn_ms.append(k0.elapsed_time(k1))
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
    total_ms = sum(step_ms)
    if world > 1:
        t = torch.tensor([total_ms], device=dev, dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        total_ms = float(t.item())
    ms_per_step = total_ms / args.steps
    # replicas: every rank bakes the whole job; split: the ranks share one
    jobs = 1 if split else world
    value = valid * args.steps * jobs / (total_ms / 1e3)

    # e2e: host buffers through the C ABI (lumel inputs up, baked colours down)
    host = lmap.download(sh, fields=("flags", "position", "normal"))
    phost = pmap.download(sh, fields=("flags", "position", "normal"))
    pin = {}
    for tag, src in (("l", host), ("p", phost)):
        for k, a in src.items():
            t = torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
            pin[tag + k] = t
    out_color = torch.empty((lmap.width * lmap.height, 3), dtype=torch.float32).pin_memory()
    h2d = sum(t.numel() * t.element_size() for t in pin.values())
    d2h = out_color.numel() * 4

    # the lightmap's inputs go up on a second stream while the photonmap's
    # inputs, the photons and the gather run on the first; the final gather
    # waits for them (every copy still lies between the step's two events)
    side = torch.cuda.Stream(device=dev)

    def e2e_step(seed):
        started, lmap_ready = torch.cuda.Event(), torch.cuda.Event()
        started.record(stream)
        side.wait_event(started)
        _abi.check(L.rl_map_upload(lmap.handle, C.c_void_p(pin["lflags"].data_ptr()), None,
                                   C.c_void_p(pin["lposition"].data_ptr()), C.c_void_p(pin["lnormal"].data_ptr()),
                                   None, None, None, C.c_void_p(side.cuda_stream)))
        lmap_ready.record(side)
        _abi.check(L.rl_map_upload(pmap.handle, C.c_void_p(pin["pflags"].data_ptr()), None,
                                   C.c_void_p(pin["pposition"].data_ptr()), C.c_void_p(pin["pnormal"].data_ptr()),
                                   None, None, None, sh))
        step(seed, lmap_ready=lmap_ready)
        _abi.check(L.rl_map_download(lmap.handle, None, None, None, None, C.c_void_p(out_color.data_ptr()), None,
                                     None, sh))

    e2e_step(5)
    torch.cuda.synchronize()
    e2e_ms = []
    for i in range(args.steps):
        flush.zero_()
        e0, e1 = ev(), ev()
        e0.record(stream)
        e2e_step(3001 + 2 * i)
        e1.record(stream)
        torch.cuda.synchronize()
        e2e_ms.append(e0.elapsed_time(e1))
    e2e_total = sum(e2e_ms)
    if world > 1:
        t = torch.tensor([e2e_total], device=dev, dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_total = float(t.item())
    e2e_value = valid * args.steps * jobs / (e2e_total / 1e3)

    peak, peak_kind = load_peaks()
    l2 = C.c_double()
    _abi.check(L.rl_measure_read_bandwidth(48 << 20, 50, C.byref(l2)))
    fg_avg_s = (sum(fg_ms) / len(fg_ms)) / 1e3
    # split: this rank traced 1/world of the rays (its interval also holds
    # the contribution all-reduce)
    alg_bytes = rays_per_step / (world if split else 1) * RAY_MODEL["bytes_per_ray"]
    achieved = alg_bytes / fg_avg_s / 1e9
    bvh = ds.bvh_stats()
    # node + triangle records the walk reads, plus the per-triangle shading records
    working_set = 64 * bvh["nodes"] + 48 * flat.ntris + 64 * flat.ntris
    bound = "l2" if working_set < L2_BYTES else "hbm"
    result = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
        "scaling": "strong" if split else "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded fBm terrain + boxes)",
        "config": terrain_config(st, valid, flat.ntris, world, knn, split),
        "tuning": {"bvh_width": autotune.get_width(), "fg": autotune.get("indirect"), "fg_pool": autotune.get_pool(),
                   **({"knn_cell_64ths": autotune.get_knn_cell()} if knn else {})},
        "grays_per_s": rays_per_step * args.steps * jobs / (total_ms / 1e3) / 1e9,
        "fg_ms": sum(fg_ms) / len(fg_ms),
        **({"knn_ms": sum(knn_ms) / len(knn_ms)} if knn else {}),
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "ms_per_step": e2e_total / args.steps},
        "roofline": {"kernel": "k_indirect (final gather)", "bound": bound, "achieved": achieved,
                     "peak": l2.value if bound == "l2" else peak, "unit": "GB/s",
                     "frac": achieved / (l2.value if bound == "l2" else peak),
                     "peak_source": ("L2 read bandwidth measured in this run by the library's probe "
                                     "(rl_measure_read_bandwidth: 48 MiB re-read 50 times with 16-byte loads); "
                                     "no driver-measured L2 figure exists" if bound == "l2"
                                     else f"{peak_kind} HBM copy bandwidth"),
                     "working_set_bytes": working_set, "l2_bytes": L2_BYTES,
                     "traffic": FG_DRAM_TRAFFIC["bytes"], "traffic_source": FG_DRAM_TRAFFIC["captured_on"],
                     "algorithmic_bytes_per_launch": alg_bytes, "bytes_per_ray": RAY_MODEL["bytes_per_ray"],
                     "hbm": {"peak": peak, "source": peak_kind, "frac": achieved / peak}},
        "gpu_launches": launches_per_step * args.steps,
        "clocks": clocks.summary(),
        "bvh": bvh,
    }
    return result, w


def cpu_baseline(w, budget_s=20.0, nthreads=None):
    """The reference baker (oracle/_ref/librelight_ref_fast.so, compiled
    from the reference's sources, project CPU BVH in place of Embree) timed
    on this host's cores over a bounded sample of the same step: one photon
    pass of eight (x8), the full gather, and the final gather on every k-th
    lumel via LumelBakeIterator fan-out (x k)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_bind as ob
    if not os.path.exists(ob.REF_FAST_LIB):
        return None, "reference build missing"
    nthreads = nthreads or os.cpu_count() or 1
    st = w.settings
    ref = ob.RefScene(w.scene, fast=True)
    L = ref.lib
    L.ref_set_rand(0, 1)
    t0 = time.perf_counter()
    L.ref_emit_photons(ref.h, 1, st.photon_bounce_count, st.photon_energy_threshold, st.photon_max_distance,
                       st.final_gather_radius)
    t_photons_gather = time.perf_counter() - t0
    # gather alone, to split the photon time from the gather time
    pm = ref.maps[id(w.photonmap)]
    t0 = time.perf_counter()
    L.ref_photonmap_gather(ref.h, pm, st.final_gather_radius)
    t_gather = time.perf_counter() - t0
    t_photon_pass = max(t_photons_gather - t_gather, 0.0)
    sky = np.asarray(st.sky_color, np.float32); amb = np.asarray(st.ambient_color, np.float32)
    lm = ref.lumels(w.lightmap)
    valid = int((lm.flags & 1).sum())
    npix = w.lightmap.width * w.lightmap.height
    # size the final-gather sample to the budget: probe with a sparse sample
    # first (odd strides, so samples spread over every column)
    div = 4095
    t0 = time.perf_counter()
    L.ref_bake_sampled(ref.h, 2, ref.mesh(w.meshes[0]), nthreads, div, 0, 0.8, 1.0, 1.0, st.final_gather_samples,
                       st.final_gather_distance, st.final_gather_radius, ob.ptr(sky), ob.ptr(amb))
    t_probe = time.perf_counter() - t0
    per_lumel = t_probe / max(npix / div, 1)
    target = max(budget_s - t_photons_gather, 2.0)
    div2 = int(max(17, min(4095, per_lumel * npix / target))) | 1
    t0 = time.perf_counter()
    L.ref_bake_sampled(ref.h, 2, ref.mesh(w.meshes[0]), nthreads, div2, 0, 0.8, 1.0, 1.0, st.final_gather_samples,
                       st.final_gather_distance, st.final_gather_radius, ob.ptr(sky), ob.ptr(amb))
    t_fg = (time.perf_counter() - t0) * div2
    step_s = st.photon_pass_count * t_photon_pass + t_gather + t_fg
    return {"value": valid / step_s, "unit": UNIT, "cores": nthreads, "kind": "reference",
            "sample": (f"reference C++ (Embree unavailable: project CPU BVH): 1 of {st.photon_pass_count} photon "
                       f"passes (x{st.photon_pass_count}, single-threaded as in Relight::emitPhotons), full "
                       f"gather, final gather on every {div2}th lumel over {nthreads} threads (x{div2})"),
            "est_step_s": step_s, "photon_pass_s": t_photon_pass, "gather_s": t_gather, "fg_s": t_fg}, None


def reference_arm(args, rank, world):
    """Relight itself (oracle/_ref/librelight_ref_fast.so: the reference's
    own sources, project CPU BVH in place of Embree) on this host's cores,
    through its own API: Relight::emitPhotons (single-threaded, as the
    reference is), then Relight::bakeIndirectLight over LumelBakeIterator(j,
    threads) on one std::thread per core.

      value     one full, unsampled step, timed once per run;
      steps     K sampled steps (each: 1 of 8 photon passes, the gather, and
                the final gather on every `div`-th lumel), the time of what
                ran as ms_per_step, and their extrapolation (x8 photons,
                x div final gather) beside the full step's value;
      as_is     one sampled step with the C library's global rand() (the
                reference as shipped, lock-contended across threads); the
                headline uses a per-thread rand() (fair to the reference).
    Under torchrun only rank 0 runs."""
    if rank != 0:
        return None
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_bind as ob
    if not os.path.exists(ob.REF_FAST_LIB):
        return {"impl": "reference", "unavailable": "oracle/_ref/librelight_ref_fast.so was not built"}
    w = build_workload(0)
    st = w.settings
    ref = ob.RefScene(w.scene, fast=True)
    L = ref.lib
    nthreads = os.cpu_count() or 1
    lm = ref.lumels(w.lightmap)
    valid = int((lm.flags & 1).sum())
    sky = np.asarray(st.sky_color, np.float32)
    amb = np.asarray(st.ambient_color, np.float32)
    pm = ref.maps[id(w.photonmap)]
    mesh0 = ref.mesh(w.meshes[0])

    def emit(passes):
        L.ref_emit_photons(ref.h, passes, st.photon_bounce_count, st.photon_energy_threshold, st.photon_max_distance,
                           st.final_gather_radius)

    def fg(div):
        L.ref_bake_sampled(ref.h, 2, mesh0, nthreads, div, 0, 0.8, 1.0, 1.0, st.final_gather_samples,
                           st.final_gather_distance, st.final_gather_radius, ob.ptr(sky), ob.ptr(amb))

    def sampled_step(div):
        """Returns (wall s, extrapolated full-step s)."""
        t0 = time.perf_counter()
        emit(1)  # one pass, then Photonmap::gather (Relight::emitPhotons)
        t1 = time.perf_counter()
        L.ref_photonmap_gather(ref.h, pm, st.final_gather_radius)
        t2 = time.perf_counter()
        fg(div)
        t3 = time.perf_counter()
        t_gather = t2 - t1
        t_pass = max((t1 - t0) - t_gather, 0.0)
        return t3 - t0, st.photon_pass_count * t_pass + t_gather + div * (t3 - t2)

    L.ref_set_rand(0, 1)
    # Size the final-gather sample so a sampled step is about 2-3 s.  The
    # sample is every div-th lumel; an odd div (coprime with the 1024-lumel
    # rows) spreads it over all columns instead of a few.
    npix = w.lightmap.width * w.lightmap.height
    t0 = time.perf_counter()
    fg(1023)
    per_lumel = (time.perf_counter() - t0) / (npix / 1023)
    div = int(max(9, min(4095, per_lumel * npix / 0.5))) | 1
    for _ in range(args.warmup):
        sampled_step(div)
    wall, est = [], []
    for i in range(args.steps):
        L.ref_set_rand(0, 100 + i)
        a, b = sampled_step(div)
        wall.append(a)
        est.append(b)
    # one full, unsampled step
    L.ref_set_rand(0, 7)
    t0 = time.perf_counter()
    emit(st.photon_pass_count)
    t1 = time.perf_counter()
    fg(1)
    t2 = time.perf_counter()
    full_s = t2 - t0
    value = valid / full_s
    extrapolated = valid / statistics.mean(est)
    # the reference as shipped: glibc's global rand()
    L.ref_set_rand(1, 5)
    _, est_as_is = sampled_step(div)
    L.ref_set_rand(0, 1)
    sample = (f"reference C++ (Embree unavailable: project CPU BVH), {nthreads} host threads; value from one full "
              f"unsampled step ({st.photon_pass_count} photon passes single-threaded as in Relight::emitPhotons, "
              f"gather, final gather on all {valid} valid lumels); per-thread rand()")
    return {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": statistics.mean(wall) * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded fBm terrain + boxes)",
            "config": terrain_config(st, valid, w.scene.flat.ntris, world),
            "impl": "reference", "sampled": True,
            "value_source": "one full, unsampled step timed once in this run",
            "full_step": {"s": full_s, "photons_and_gather_s": t1 - t0, "fg_s": t2 - t1},
            "sampled_steps": {"each": (f"1 of {st.photon_pass_count} photon passes, the gather, final gather on "
                                       f"every {div}th lumel"),
                              "scale": {"photon_passes": st.photon_pass_count, "fg_lumel_stride": div},
                              "ms_per_step": statistics.mean(wall) * 1e3,
                              "extrapolated_value": extrapolated,
                              "extrapolation_error": extrapolated / value - 1.0},
            "as_is_rand": {"value": valid / est_as_is, "unit": UNIT,
                           "kind": "one sampled step with glibc's global rand(), extrapolated"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": nthreads, "kind": "reference", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


BATCH_METRIC = "lightmaps/s (uneven bake jobs: direct + AO 64 spp + final gather 128 spp)"


def batch_arm(args):
    """Uneven-size batching on one GPU: scenes of log-uniform 1k-500k
    triangles, jobs with log-uniform 32^2-1024^2 lightmaps, each baked with
    direct light, AO and final gather.  BVHs and gathered photonmaps are
    resident; a step clears every job's lightmap colours and bakes all jobs,
    (a) as one captured graph of the batch kernels, (b) as the plain per-job
    loop of single-job calls.  Both arms are checked for identical bits."""
    import torch
    from relight_b200 import autotune, batch, scenes
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(dev)
    sh = stream.cuda_stream
    n_jobs, n_scenes = (64, 8) if SMALL else (512, 32)
    t0 = time.perf_counter()
    wl = scenes.batch_workload(n_jobs=n_jobs, n_scenes=n_scenes)
    t_scenes = time.perf_counter() - t0
    with torch.cuda.stream(stream):
        t0 = time.perf_counter()
        res = batch.make_resident(wl, stream=sh)
        stream.synchronize()
        t_resident = time.perf_counter() - t0
        valid = sum(m.valid_count() for m in res.lightmaps)
        t0 = time.perf_counter()
        tuned = autotune.tune_batch(res.jobs, stream, sample=8, reset=lambda: res.clear(stream=sh))
        t_tune = time.perf_counter() - t0
        b = batch.Batch(res.jobs)
        b.capture(sh)
        ev = lambda: torch.cuda.Event(enable_timing=True)
        flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

        def timed(fn, steps, warmup):
            for _ in range(warmup):
                res.clear(stream=sh)
                fn()
            stream.synchronize()
            ms = []
            for _ in range(steps):
                flush.zero_()
                res.clear(stream=sh)
                e0, e1 = ev(), ev()
                e0.record(stream)
                fn()
                e1.record(stream)
                stream.synchronize()
                ms.append(e0.elapsed_time(e1))
            return ms

        with ClockSampler(0) as clocks:
            batch_ms = timed(lambda: b.replay(sh), args.steps, args.warmup)
        sample = list(range(0, len(res.lightmaps), max(1, len(res.lightmaps) // 16)))
        got = [res.lightmaps[q].download(sh, fields=("color",))["color"] for q in sample]
        loop_ms = timed(lambda: batch.run_per_job(res.jobs, sh), max(1, args.steps // 2), 1)
        want = [res.lightmaps[q].download(sh, fields=("color",))["color"] for q in sample]
    identical = all(np.array_equal(a.view(np.uint32), c.view(np.uint32)) for a, c in zip(got, want))
    bm = statistics.mean(batch_ms)
    lm_ = statistics.mean(loop_ms)
    nl = [len(sc.scene.flat.lights) for sc in wl.scenes]
    rays = sum(res.lightmaps[q].valid_count() * (nl[wl.jobs[q].scene] + wl.ao.samples + wl.scenes[0].settings.final_gather_samples)
               for q in range(len(wl.jobs)))
    return {
        "metric": BATCH_METRIC, "value": n_jobs / (bm / 1e3), "unit": "lightmaps/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": bm, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded heightfield + boxes)",
        "config": {"workload": f"{n_jobs} jobs over {n_scenes} scenes (log-uniform 1k-500k tris), lightmaps "
                               f"log-uniform 32^2-1024^2, direct + AO 64 + FG 128 per job",
                   "jobs": n_jobs, "scenes": n_scenes, "triangles": wl.triangles, "valid_texels": valid,
                   "texels": res.texels, "l2": "flushed between steps (256 MiB write)",
                   "tuning": {"fg": autotune.get("indirect"), "ao": autotune.get("ao"),
                              "source": "autotune.tune_batch on every 8th job",
                              "fg_table_ms": {f"{k[0]}/{k[1]}": v for k, v in tuned.get("indirect", ({}, {}))[1].items()},
                              "ao_table_ms": {f"{k[0]}/{k[1]}": v for k, v in tuned.get("ao", ({}, {}))[1].items()}}},
        "texels_per_s": valid / (bm / 1e3), "grays_per_s": rays / (bm / 1e3) / 1e9,
        "per_job_loop": {"value": n_jobs / (lm_ / 1e3), "ms_per_step": lm_, "launches_per_step": len(res.jobs)},
        "batch_over_loop": lm_ / bm, "identical_to_loop": identical,
        "gpu_launches": 3 * args.steps, "clocks": clocks.summary(),
        "setup_s": {"scenes_host": t_scenes, "resident": t_resident, "tune": t_tune},
    }


DENOISE_METRIC = ("lightmaps/s at equal per-texel RMSE vs the FP64 oracle (final gather 16 spp + denoiser vs "
                  "plain)")
TRUTH_TEXELS, TRUTH_SAMPLES = 4096, 16384


def _fg_truth_part(recipe, gathered, texels, samples, seed):
    """Oracle.fg_expect (FP64, uniform hemisphere) on some texels of a
    rebuilt training scene whose photonmap holds the device's gathered
    values.  Runs in a spawned worker process."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_bind as ob
    from relight_b200 import scenes
    wl = scenes.terrain_scene(**recipe)
    orc = ob.Oracle(wl.scene.flat).bind_scene(wl.scene)
    pm = orc.maps("photonmap")[0]
    pm.gathered[:] = gathered
    lm = orc.maps()[0]
    st = wl.settings
    return orc.fg_expect(lm, [pm], texels, samples, st.final_gather_distance, st.sky_color, st.ambient_color, seed)


class FgTruth:
    """The FP64 final-gather truth for denoise.evaluate: the oracle's
    expectation over TRUTH_TEXELS seeded valid lumels at TRUTH_SAMPLES
    samples, in two independent halves whose difference estimates the
    truth's own noise variance (returned, and taken out of every RMSE).
    Spread over a process pool started with spawn."""

    def __init__(self, procs=None):
        import multiprocessing as mp
        self.procs = procs or max(1, os.cpu_count() or 1)
        self.pool = mp.get_context("spawn").Pool(self.procs)
        self.seconds = 0.0

    def __call__(self, i, wl):
        t0 = time.perf_counter()
        pmap = wl.photonmap._device.download(fields=("gathered",))["gathered"]
        flags = wl.lightmap._device.download(fields=("flags",))["flags"]
        valid = np.nonzero(flags & 1)[0]
        tex = np.sort(np.random.default_rng(1000 + i).choice(valid, min(TRUTH_TEXELS, len(valid)), replace=False))
        chunks = np.array_split(tex.astype(np.int32), self.procs)
        halves = []
        for h in range(2):
            jobs = [(wl.recipe, pmap, c, TRUTH_SAMPLES // 2, 7919 * (i + 1) + h) for c in chunks if len(c)]
            halves.append(np.concatenate(self.pool.starmap(_fg_truth_part, jobs)))
        expect = 0.5 * (halves[0] + halves[1])
        noise_var = float(np.mean((halves[0] - halves[1]) ** 2) / 4.0)
        self.seconds += time.perf_counter() - t0
        return tex, expect, noise_var

    def close(self):
        self.pool.close()
        self.pool.join()


def train_denoiser(small):
    """Bake (16, 1024) spp final-gather pairs on seeded terrain-and-boxes
    scenes, cut 64x64 patches and train the denoiser (Adam, BF16 tensor-core
    kernels).  Returns the network, its loss curve and the timings."""
    import torch
    from relight_b200 import denoise as D
    n_train = 8 if small else 24
    patches, steps = (4000, 1500) if small else (10000, 4000)
    t0 = time.perf_counter()
    pairs = D.make_pairs(D.training_scenes(n_train, seed=100), spp_lo=16, spp_hi=1024, seed=7)
    xs, ts = D.make_patches(pairs, patches, patch=64, seed=11)
    del pairs
    torch.cuda.synchronize()
    t_data = time.perf_counter() - t0
    dn = D.Denoiser(seed=1)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    losses = D.train(dn, xs, ts, steps=steps, batch=16, lr=2e-3)
    e1.record()
    torch.cuda.synchronize()
    info = {"scenes": n_train, "patches": patches, "steps": steps, "batch": 16, "lr": 2e-3, "data_s": t_data,
            "train_ms": e0.elapsed_time(e1), "loss_first50": float(losses[:50].mean()),
            "loss_last200": float(losses[-200:].mean()), "status": dn.status()}
    return dn, info


def denoise_arm(args):
    """The denoiser end to end on one GPU: train it (train_denoiser), then on
    held-out 512^2 scenes compare RMSE and device time of 16 spp + denoiser
    against plain final gathers of 16-1024 spp, all against the FP64 oracle
    (FgTruth)."""
    import torch
    from relight_b200 import denoise as D
    torch.cuda.set_device(0)
    n_eval = 2 if SMALL else 4
    truth = FgTruth()
    dn, info = train_denoiser(SMALL)
    with ClockSampler(0) as clocks:
        ev = D.evaluate(dn, D.training_scenes(n_eval, seed=900, sides=(512,)), spp_lo=16, truth=truth)
    truth.close()
    dn_ms = ev["denoised"][1]
    return {
        "metric": DENOISE_METRIC, "value": 1e3 / dn_ms, "unit": "lightmaps/s", "n_gpus": 1, "steps": n_eval,
        "warmup": 0, "ms_per_step": dn_ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "bf16 (network), f32 (baker)", "data": "synthetic (seeded heightfield + boxes)",
        "config": {"workload": f"train on {info['patches']} 64x64 patches from {info['scenes']} scenes "
                               f"(256-512^2 lightmaps), evaluate on {n_eval} held-out 512^2 lightmaps",
                   "spp_low": 16, "spp_train_target": 1024,
                   "reference": (f"FP64 oracle final-gather expectation on {TRUTH_TEXELS} seeded valid lumels per "
                                 f"scene, {TRUTH_SAMPLES} samples in two halves (their difference estimates the "
                                 f"truth's noise variance, taken out of every RMSE)")},
        "truth_s": truth.seconds,
        "plain_at_equal_rmse": {"spp": ev["equal_rmse_spp"], "extrapolated": ev["extrapolated"],
                                "ms": ev["plain_ms_at_equal_rmse"], "lightmaps_per_s": 1e3 / ev["plain_ms_at_equal_rmse"]},
        "speedup_at_equal_rmse": ev["speedup"],
        "rmse": {"denoised_16spp": ev["denoised"][0], **{f"plain_{k}spp": v[0] for k, v in ev["plain"].items()}},
        "denoised_max_err": ev["denoised_max_err"],
        "ms": {"denoised_16spp": dn_ms, **{f"plain_{k}spp": v[1] for k, v in ev["plain"].items()}},
        "train": info, "clocks": clocks.summary(),
    }


SERVE_METRIC = "bake-serving p99 latency at 100 req/s (Poisson; direct + AO 64 + FG 16 spp + denoiser per request)"


def serve_arm(args):
    """Bake serving on one GPU with the denoiser in the loop: 32 resident
    scenes (log-uniform 1k-500k triangles, BVH + gathered photonmap each),
    requests with log-uniform 32^2-1024^2 lightmaps arriving as Poisson
    streams at 20, 50 and 100 requests/s, admitted by a 16 GiB HBM budget
    and continuously batched; direct light + AO 64 + final gather 16 spp,
    the final gather denoised at completion.  Latency is arrival to colours
    in host memory on the host clock.  A closed-loop run (all requests
    queued at once) gives the saturated throughput, compared with the plain
    per-job GPU path at the final-gather sample count whose RMSE (against the
    FP64 oracle, FgTruth) equals the denoised one."""
    import torch
    from dataclasses import replace
    from relight_b200 import batch, denoise as D, scenes, serve
    from relight_b200.device import DeviceMap
    torch.cuda.set_device(0)
    n_scenes = 8 if SMALL else 32
    n_req = 40 if SMALL else 300
    t0 = time.perf_counter()
    truth = FgTruth()
    dn, info = train_denoiser(SMALL)
    ev = D.evaluate(dn, D.training_scenes(2 if SMALL else 3, seed=900, sides=(512,)), spp_lo=16, truth=truth)
    truth.close()
    t_denoiser = time.perf_counter() - t0
    # the plain path runs at the equal-RMSE sample count, capped at the largest one measured
    eq_spp = int(round(min(ev["equal_rmse_spp"], max(ev["plain"]))))
    wl = scenes.batch_workload(n_jobs=1, n_scenes=n_scenes)
    ts_ = torch.cuda.Stream()
    rs = batch.make_resident_scenes(wl, stream=ts_.cuda_stream)
    ts_.synchronize()
    budget = 16 << 30
    srv = serve.BakeServer(rs, budget_bytes=budget, quantum=1 << 18, fg_samples=16, torch_stream=ts_, denoiser=dn)
    srv.warm()
    srv.run(serve.make_requests(wl, 1000.0, max(args.warmup, 3) * 4, seed=99))  # warm-up
    rates = {}
    with ClockSampler(0) as clocks:
        for rate in (20.0, 50.0, 100.0):
            st = srv.run(serve.make_requests(wl, rate, n_req, seed=int(rate)), keep_results=False)
            rates[str(int(rate))] = st.as_dict()
        sat = srv.run(serve.make_requests(wl, 1e9, n_req, seed=7), keep_results=False).as_dict()
    srv.close()
    # the plain per-job GPU path at the equal-RMSE sample count, device time
    n_plain = 16 if SMALL else 48
    jobs, maps = [], []
    for r in serve.make_requests(wl, 1e9, n_plain, seed=7):
        ds = rs.scenes[r.scene]
        lm = DeviceMap(0, r.side, r.side)
        for mi in range(len(ds.flat.mesh_photonmap)):
            lm.add_mesh(ds, mi)
        maps.append(lm)
        fg = replace(wl.scenes[r.scene].settings, final_gather_samples=eq_spp)
        jobs += [batch.BakeJob.direct(ds, lm), batch.BakeJob.ambient_occlusion(ds, lm, wl.ao, seed=r.seed ^ 0xA0),
                 batch.BakeJob.indirect(ds, lm, rs.photonmaps[r.scene], fg, seed=r.seed ^ 0xF6)]
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    batch.run_per_job(jobs)
    e1.record()
    torch.cuda.synchronize()
    plain_lps = n_plain / (e0.elapsed_time(e1) / 1e3)
    p99 = rates["100"]["p99_ms"]
    return {
        "metric": SERVE_METRIC, "value": p99, "unit": "ms", "n_gpus": 1, "steps": n_req, "warmup": args.warmup,
        "ms_per_step": rates["100"]["mean_ms"], "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 (baker), bf16 (denoiser)", "data": "synthetic (seeded heightfield + boxes, Poisson arrivals)",
        "config": {"workload": f"{n_req} requests per rate over {n_scenes} resident scenes, lightmaps log-uniform "
                               f"32^2-1024^2, direct + AO 64 + FG 16 spp + denoiser",
                   "hbm_budget_bytes": budget, "resident_scene_bytes": rs.nbytes(), "quantum_lumels": 1 << 18,
                   "latency_clock": "host (arrival to colours in pinned host memory)"},
        "rates": rates, "saturated": sat,
        "denoiser": {"rmse_denoised_16spp": ev["denoised"][0], "max_err": ev["denoised_max_err"],
                     "equal_rmse_spp": ev["equal_rmse_spp"], "extrapolated": ev["extrapolated"],
                     "reference": f"FP64 oracle, {TRUTH_TEXELS} lumels x {TRUTH_SAMPLES} samples per scene",
                     "rmse_plain": {str(k): v[0] for k, v in ev["plain"].items()}, "train": info,
                     "setup_s": t_denoiser},
        "plain_per_job_at_equal_rmse": {"fg_spp": eq_spp, "lightmaps_per_s": plain_lps, "requests": n_plain},
        "speedup_vs_plain_at_equal_rmse": sat["lightmaps_per_s"] / plain_lps,
        "clocks": clocks.summary(),
    }


ROOM_METRIC = "lightmap texels/s (room: direct light from a point, a spot and a 16-sample area light + AO 64 spp, 256^2)"
ROOM_AO_BYTES_PER_RAY = 633.0  # room AO rays on the canonical SAH tree: 17.7 box + 0.39 triangle tests (oracle/ray_bytes.py)


def _timed_steps(stream, steps, step, flush):
    """Device time of each of `steps` calls of step(i), L2 flushed before each."""
    import torch
    ms = []
    for i in range(steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step(i)
        e1.record(stream)
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    return ms


def room_cpu_baseline(w, budget_s=15.0, nthreads=None):
    """Relight's own direct light + AO (oracle/_ref/librelight_ref_fast.so,
    project CPU BVH in place of Embree) over every k-th lumel on all host
    threads, scaled by k."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_bind as ob
    if not os.path.exists(ob.REF_FAST_LIB):
        return None
    nthreads = nthreads or os.cpu_count() or 1
    ref = ob.RefScene(w.scene, fast=True)
    L = ref.lib
    L.ref_set_rand(0, 1)
    lm = ref.lumels(w.lightmap)
    valid = int((lm.flags & 1).sum())
    npix = w.lightmap.width * w.lightmap.height
    zero = np.zeros(3, np.float32)
    ao = w.ao

    def run(div):
        t0 = time.perf_counter()
        L.ref_bake_sampled(ref.h, 0, ref.mesh(w.mesh), nthreads, div, 0, 0.8, 1.0, 1.0, 1, 1.0, 1, ob.ptr(zero), ob.ptr(zero))
        L.ref_bake_sampled(ref.h, 1, ref.mesh(w.mesh), nthreads, div, ao.samples, ao.occluded_fraction, ao.max_distance,
                           ao.exponent, 1, 1.0, 1, ob.ptr(zero), ob.ptr(zero))
        return time.perf_counter() - t0

    probe_div = 255
    per_lumel = run(probe_div) / max(npix / probe_div, 1)
    div = int(max(1, min(4095, per_lumel * npix / budget_s))) | 1
    step_s = run(div) * div
    return {"value": valid / step_s, "unit": UNIT, "cores": nthreads, "kind": "reference",
            "sample": (f"reference C++ (Embree unavailable: project CPU BVH): Relight::bakeDirectLight + "
                       f"bakeAmbientOcclusion on every {div}th lumel over {nthreads} threads (x{div})"),
            "est_step_s": step_s}


def room_arm(args):
    """The room workload on one GPU: the closed 10^3 room with 8 boxes (108
    triangles), one 256^2 lightmap, direct light from a point light, a 45
    degree spot and a 1x1 area light sampled at its 16 triangle centroids,
    then AO with 64 hemisphere rays of length 2."""
    import torch
    from relight_b200 import _abi, scenes
    from relight_b200.device import Relight
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    sh = stream.cuda_stream
    w = scenes.room_scene()
    rl = Relight(stream=sh, seed=1000)
    ds = rl.device_scene(w.scene)
    torch.cuda.synchronize()
    lmap = w.lightmap._device
    L = _abi.lib()
    f = w.scene.flat
    lights = C.c_void_p(f.lights.ctypes.data)
    lverts = C.c_void_p(f.light_vertices.ctypes.data)
    nlv = int(sum(int(l["vertex_count"]) for l in f.lights))
    shadow_per_lumel = int(sum(max(1, int(l["vertex_count"])) for l in f.lights))
    ao = w.ao
    valid = lmap.valid_count()
    ev = lambda: torch.cuda.Event(enable_timing=True)
    ao_ms = []

    def step(i, timed=False):
        _abi.check(L.rl_map_clear(lmap.handle, 1, 0, sh))
        _abi.check(L.rl_bake_direct(ds.handle, lmap.handle, lights, len(f.lights), lverts, nlv, None, sh))
        a0, a1 = ev(), ev()
        a0.record(stream)
        _abi.check(L.rl_bake_ao(ds.handle, lmap.handle, ao.samples, ao.occluded_fraction, ao.max_distance,
                                ao.exponent, 7 + 2 * i, None, sh))
        a1.record(stream)
        if timed:
            ao_ms.append((a0, a1))

    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    for i in range(args.warmup):
        step(i)
    torch.cuda.synchronize()
    # a step is under a millisecond: time enough of them for the clock sampler
    steps = max(args.steps, 1000)
    with ClockSampler(0) as clocks:
        step_ms = _timed_steps(stream, steps, lambda i: step(100 + i, True), flush)
    ao_avg_ms = sum(a.elapsed_time(b) for a, b in ao_ms) / len(ao_ms)
    total_ms = sum(step_ms)
    value = valid * steps / (total_ms / 1e3)

    host = lmap.download(sh, fields=("flags", "position", "normal"))
    pin = {k: torch.from_numpy(np.ascontiguousarray(a)).pin_memory() for k, a in host.items()}
    out_color = torch.empty((lmap.width * lmap.height, 3), dtype=torch.float32).pin_memory()
    h2d = sum(t.numel() * t.element_size() for t in pin.values())
    d2h = out_color.numel() * 4

    def e2e_step(i):
        _abi.check(L.rl_map_upload(lmap.handle, C.c_void_p(pin["flags"].data_ptr()), None,
                                   C.c_void_p(pin["position"].data_ptr()), C.c_void_p(pin["normal"].data_ptr()),
                                   None, None, None, sh))
        step(300 + i)
        _abi.check(L.rl_map_download(lmap.handle, None, None, None, None, C.c_void_p(out_color.data_ptr()), None,
                                     None, sh))

    e2e_step(0)
    torch.cuda.synchronize()
    e2e_ms = _timed_steps(stream, args.steps, lambda i: e2e_step(1 + i), flush)
    e2e_value = valid * args.steps / (sum(e2e_ms) / 1e3)

    peak, peak_kind = load_peaks()
    l1 = C.c_double()
    _abi.check(L.rl_measure_l1_read_bandwidth(64 << 10, 2000, C.byref(l1)))
    ao_rays = valid * ao.samples
    achieved = ao_rays * ROOM_AO_BYTES_PER_RAY / (ao_avg_ms / 1e3) / 1e9
    result = {
        "metric": ROOM_METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": steps,
        "warmup": args.warmup, "ms_per_step": total_ms / steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded room)",
        "config": {"workload": "room 10^3 + 8 boxes (108 tris), 256^2 lightmap, point + 45 deg spot + area "
                               "(16 samples) lights, AO 64 spp r2", "valid_texels": valid,
                   "shadow_rays_per_lumel_max": shadow_per_lumel, "ao_samples": ao.samples,
                   "l2": "flushed between steps (256 MiB write)"},
        "ao_ms": ao_avg_ms, "direct_ms": total_ms / steps - ao_avg_ms,
        "ao_grays_per_s": ao_rays / (ao_avg_ms / 1e3) / 1e9,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "ms_per_step": sum(e2e_ms) / args.steps},
        "roofline": {"kernel": "k_ao (AO 64 spp)", "bound": "l1", "achieved": achieved, "peak": l1.value,
                     "unit": "GB/s", "frac": achieved / l1.value,
                     "peak_source": ("L1 read bandwidth measured in this run by the library's probe "
                                     "(rl_measure_l1_read_bandwidth: 64 KiB per block re-read 2,000 times)"),
                     "working_set_bytes": 64 * (f.ntris - 1) + 48 * f.ntris, "traffic": None,
                     "algorithmic_bytes_per_launch": ao_rays * ROOM_AO_BYTES_PER_RAY,
                     "bytes_per_ray": ROOM_AO_BYTES_PER_RAY,
                     "hbm": {"peak": peak, "source": peak_kind, "frac": achieved / peak},
                     "note": "the 108-triangle tree stays in each SM's L1; the walk is bound by issue"},
        "gpu_launches": 3 * steps,
        "clocks": clocks.summary(),
    }
    if not args.no_cpu_baseline:
        cb = room_cpu_baseline(w)
        if cb:
            result["cpu_baseline"] = cb
    return result


RAD_METRIC = "form-factor Grays/s (16,384 patches x 512 cosine rays) + 50 Jacobi gather iterations"


def radiosity_pairwise(w, ds, n, pos, nrm, sh, threshold=0.1, reps=3):
    """Relight's own form factors (RadiosityBuilder::computeFormFactors,
    point-to-point with segment visibility, rows normalised) over the same
    patches: rl_ff_pairwise (its count call and its fill call, CSR to host)
    against the compiled reference on one host thread, and the two CSRs
    compared bit for bit.  The reference's patch list is used as input when
    it is available."""
    import torch
    from relight_b200 import _abi
    L = _abi.lib()
    out = {"patches": n, "pairs": n * (n - 1) // 2, "threshold": threshold}
    ref_csr = None
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_bind as ob
    if os.path.exists(ob.REF_FAST_LIB):
        ref = ob.RefScene(w.scene, fast=True, radiancemaps=(w.radiancemap,))
        t0 = time.perf_counter()
        rrow, rcols, rvals, rpos, rnrm = ref.radiosity(threshold)
        out["reference_s"] = time.perf_counter() - t0
        out["reference_threads"] = 1
        out["reference_patches_equal"] = bool(rpos.shape == pos.shape and np.array_equal(rpos, pos)
                                              and np.array_equal(rnrm, nrm))
        if rpos.shape[0] == n:
            pos, nrm = rpos, rnrm
            ref_csr = (rrow, rcols, rvals)
    dp = torch.from_numpy(np.ascontiguousarray(pos, np.float32)).cuda()
    dn = torch.from_numpy(np.ascontiguousarray(nrm, np.float32)).cuda()

    def run():
        cnt = C.c_int64()
        _abi.check(L.rl_ff_pairwise(ds.handle, n, C.c_void_p(dp.data_ptr()), C.c_void_p(dn.data_ptr()), threshold,
                                    None, None, None, 0, C.byref(cnt), sh))
        k = cnt.value
        row = np.zeros(n + 1, np.int64)
        cols = np.zeros(max(k, 1), np.int32)
        vals = np.zeros(max(k, 1), np.float32)
        _abi.check(L.rl_ff_pairwise(ds.handle, n, C.c_void_p(dp.data_ptr()), C.c_void_p(dn.data_ptr()), threshold,
                                    C.c_void_p(row.ctypes.data), C.c_void_p(cols.ctypes.data),
                                    C.c_void_p(vals.ctypes.data), k, C.byref(cnt), sh))
        return row, cols[:k], vals[:k]

    run()
    torch.cuda.synchronize()
    ms = []
    for _ in range(reps):
        t0 = time.perf_counter()
        csr = run()
        torch.cuda.synchronize()
        ms.append((time.perf_counter() - t0) * 1e3)
    out["gpu_ms"] = statistics.median(ms)
    out["gpu_ms_covers"] = "the count call and the fill call (each sweeps all pairs), CSR to host memory"
    out["nnz"] = int(len(csr[1]))
    out["gpu_gpairs_per_s"] = out["pairs"] / (out["gpu_ms"] / 1e3) / 1e9
    if ref_csr is not None:
        out["matches_reference"] = bool(np.array_equal(csr[0], ref_csr[0]) and np.array_equal(csr[1], ref_csr[1])
                                        and np.array_equal(csr[2].view(np.uint32), ref_csr[2].view(np.uint32)))
        out["speedup_vs_reference"] = out["reference_s"] * 1e3 / out["gpu_ms"]
    return out


def radiosity_arm(args):
    """The radiosity workload on one GPU: a 10 x 5 x 10 room whose 128^2
    radiancemap texels are 16,384 patches; form factors from 512
    cosine-distributed rays per patch (rl_ff_hemisphere), then 50 fp32 Jacobi
    iterations of B = E + rho F B (rl_radiosity_solve), checked against the
    same iterations and the converged solve in float64."""
    import torch
    import scipy.sparse as sp
    from relight_b200 import _abi, scenes
    from relight_b200.device import Relight
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    sh = stream.cuda_stream
    rays, maxd, iters = 512, 100.0, 50
    w = scenes.radiosity_room(size=128)
    rl = Relight(stream=sh, seed=1000)
    ds = rl.device_scene(w.scene)
    torch.cuda.synchronize()
    g = w.radiancemap._device.download(sh, fields=("flags", "position", "normal"))
    valid = np.nonzero(g["flags"] & 1)[0]
    n = len(valid)
    pos = np.ascontiguousarray(g["position"][valid], np.float32)
    nrm = np.ascontiguousarray(g["normal"][valid], np.float32)
    W, H = w.radiancemap.width, w.radiancemap.height
    pot = np.full(W * H, -1, np.int32)
    pot[valid] = np.arange(n, dtype=np.int32)
    mesh_map, dims, base = np.array([0], np.int32), np.array([[W, H]], np.int32), np.array([0], np.int64)
    rng = np.random.default_rng(w.albedo_seed)
    rho = rng.uniform(0.3, 0.9, (n, 3)).astype(np.float32)
    E = np.zeros((n, 3), np.float32)
    E[rng.choice(n, 16, replace=False)] = 1.0
    L = _abi.lib()
    cap = n * rays
    pin_pos = torch.from_numpy(pos).pin_memory()
    pin_nrm = torch.from_numpy(nrm).pin_memory()
    pin_E = torch.from_numpy(E).pin_memory()
    pin_rho = torch.from_numpy(rho).pin_memory()
    out_B = torch.empty((n, 3), dtype=torch.float32).pin_memory()
    dpos = torch.empty((n, 3), dtype=torch.float32, device=dev)
    dnrm = torch.empty_like(dpos)
    dE = torch.empty_like(dpos)
    drho = torch.empty_like(dpos)
    dB = torch.empty_like(dpos)
    drow = torch.empty(n + 1, dtype=torch.int64, device=dev)
    dcols = torch.empty(cap, dtype=torch.int32, device=dev)
    dvals = torch.empty(cap, dtype=torch.float32, device=dev)
    nnz = C.c_int64()
    ev = lambda: torch.cuda.Event(enable_timing=True)
    parts = {"ff": [], "solve": []}

    def upload():
        dpos.copy_(pin_pos, non_blocking=True)
        dnrm.copy_(pin_nrm, non_blocking=True)
        dE.copy_(pin_E, non_blocking=True)
        drho.copy_(pin_rho, non_blocking=True)

    def step(i, timed=False):
        """Form factors into device memory (rl_ff_hemisphere_device), then 50 iterations."""
        f0, f1, s0, s1 = ev(), ev(), ev(), ev()
        f0.record(stream)
        _abi.check(L.rl_ff_hemisphere_device(ds.handle, n, C.c_void_p(dpos.data_ptr()), C.c_void_p(dnrm.data_ptr()),
                                             rays, maxd, 11 + i, C.c_void_p(mesh_map.ctypes.data), 1,
                                             C.c_void_p(dims.ctypes.data), C.c_void_p(base.ctypes.data),
                                             C.c_void_p(pot.ctypes.data), pot.size, C.c_void_p(drow.data_ptr()),
                                             C.c_void_p(dcols.data_ptr()), C.c_void_p(dvals.data_ptr()), cap,
                                             C.byref(nnz), sh))
        f1.record(stream)
        s0.record(stream)
        _abi.check(L.rl_radiosity_solve(n, C.c_void_p(drow.data_ptr()), C.c_void_p(dcols.data_ptr()),
                                        C.c_void_p(dvals.data_ptr()), C.c_void_p(dE.data_ptr()),
                                        C.c_void_p(drho.data_ptr()), iters, C.c_void_p(dB.data_ptr()), sh))
        s1.record(stream)
        if timed:
            parts["ff"].append((f0, f1))
            parts["solve"].append((s0, s1))

    def e2e_step(i):
        """Patches, E and rho up from pinned host memory, the step, B down."""
        upload()
        step(i)
        out_B.copy_(dB, non_blocking=True)

    upload()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    for i in range(args.warmup):
        step(i)
    torch.cuda.synchronize()
    # the form-factor call waits for its per-row counts on the host, so a busy
    # host shows in its time: let the clock sampler start, and time 20 steps
    steps = max(args.steps, 20)
    with ClockSampler(0) as clocks:
        time.sleep(0.5)
        step_ms = _timed_steps(stream, steps, lambda i: step(100 + i, True), flush)
    ff_ms = sum(a.elapsed_time(b) for a, b in parts["ff"]) / steps
    solve_ms = sum(a.elapsed_time(b) for a, b in parts["solve"]) / steps
    e2e_step(0)
    torch.cuda.synchronize()
    e2e_ms = _timed_steps(stream, steps, lambda i: e2e_step(200 + i), flush)
    k = nnz.value
    # float64 checks on the last step's matrix
    F = sp.csr_matrix((dvals[:k].cpu().numpy().astype(np.float64), dcols[:k].cpu().numpy(), drow.cpu().numpy()),
                      shape=(n, n))
    E64, rho64 = E.astype(np.float64), rho.astype(np.float64)
    B64 = E64.copy()
    for _ in range(iters):
        B64 = E64 + rho64 * (F @ B64)
    Bc = B64.copy()
    conv_iters = iters
    for conv_iters in range(iters + 1, 20000):
        Bn = E64 + rho64 * (F @ Bc)
        if np.abs(Bn - Bc).max() <= 1e-13 * np.abs(Bn).max():
            Bc = Bn
            break
        Bc = Bn
    B32 = dB.cpu().numpy().astype(np.float64)
    scale = np.abs(B64).max()
    peak, peak_kind = load_peaks()
    l2 = C.c_double()
    _abi.check(L.rl_measure_read_bandwidth(48 << 20, 50, C.byref(l2)))
    jac_bytes = iters * (8.0 * k + 44.0 * n)
    # the CSR, row offsets, E, rho and both [n][4] iterates
    jac_set = 8 * k + 8 * (n + 1) + 24 * n + 32 * n
    jac_bound = "l2" if jac_set < L2_BYTES else "hbm"
    achieved = jac_bytes / (solve_ms / 1e3) / 1e9
    pairwise = radiosity_pairwise(w, ds, n, pos, nrm, sh)
    h2d = 4 * n * 12
    d2h = 12 * n
    value = n * rays / (ff_ms / 1e3) / 1e9
    e2e_value = n * rays * steps / (sum(e2e_ms) / 1e3) / 1e9
    result = {
        "metric": RAD_METRIC, "value": value, "unit": "Grays/s", "n_gpus": 1, "steps": steps,
        "warmup": args.warmup, "ms_per_step": sum(step_ms) / steps, "higher_is_better": True,
        "step_grays_per_s": n * rays * steps / (sum(step_ms) / 1e3) / 1e9,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (room of 16,384 patches, seeded albedo)",
        "config": {"workload": "radiosity room 10x5x10, 16,384 patches, 512 cosine rays per patch, 50 Jacobi "
                               "iterations over RGB", "patches": n, "rays_per_patch": rays, "nnz": k,
                   "l2": "flushed between steps (256 MiB write)"},
        "ff_ms": ff_ms, "solve_ms": solve_ms,
        "jacobi_vs_fp64_50_iters_max_rel": float(np.abs(B32 - B64).max() / scale),
        "jacobi_50_vs_converged_fp64_max_rel": float(np.abs(B64 - Bc).max() / np.abs(Bc).max()),
        "converged_after_iters": conv_iters,
        "e2e": {"value": e2e_value, "unit": "Grays/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "ms_per_step": sum(e2e_ms) / steps,
                "note": "patch positions and normals, E and rho up from pinned memory; form factors and solve; B down"},
        "roofline": {"kernel": "k_jacobi4_smem (50 iterations; the iterate staged in shared memory per block)", "bound": jac_bound, "achieved": achieved,
                     "peak": l2.value if jac_bound == "l2" else peak, "unit": "GB/s",
                     "frac": achieved / (l2.value if jac_bound == "l2" else peak),
                     "peak_source": ("L2 read bandwidth measured in this run by the library's probe "
                                     "(rl_measure_read_bandwidth: 48 MiB re-read 50 times)" if jac_bound == "l2"
                                     else f"{peak_kind} HBM copy bandwidth"),
                     "working_set_bytes": jac_set, "traffic": None,
                     "algorithmic_bytes": jac_bytes, "bytes_per_iteration": "8 B per nonzero + 44 B per row",
                     "hbm": {"peak": peak, "source": peak_kind, "frac": achieved / peak}},
        # k_ff_hemi_rays / _rle / _compact, k_pack4, k_jacobi4 per iteration, k_unpack4
        "pairwise_form_factors": pairwise,
        "gpu_launches": (5 + iters) * steps,
        "clocks": clocks.summary(),
    }
    return result


def _summary(r, keys):
    out = {k: r[k] for k in keys if k in r}
    if "roofline" in r:
        rf = r["roofline"]
        out["roofline"] = {k: rf[k] for k in ("kernel", "bound", "achieved", "peak", "unit", "frac") if k in rf}
    if "e2e" in r:
        out["e2e"] = {k: r["e2e"][k] for k in ("value", "unit") if k in r["e2e"]}
    if "clocks" in r:
        out["clocks"] = r["clocks"]
    return out


def other_workloads(args):
    """The room (direct + AO, 256^2) and radiosity (16,384 patches) workloads,
    measured after the terrain step in the same run and summarised (their
    own --workload runs print the full lines)."""
    import copy
    out = {}
    a = copy.copy(args)
    a.steps, a.warmup, a.no_cpu_baseline = 20, 3, True
    r = room_arm(a)
    out["room"] = _summary(r, ("metric", "value", "unit", "ms_per_step", "steps", "ao_ms", "direct_ms",
                               "ao_grays_per_s"))
    r = radiosity_arm(a)
    out["radiosity"] = _summary(r, ("metric", "value", "unit", "ms_per_step", "steps", "ff_ms", "solve_ms",
                                    "jacobi_vs_fp64_50_iters_max_rel"))
    pw = r.get("pairwise_form_factors", {})
    out["radiosity"]["pairwise_form_factors"] = {k: pw[k] for k in ("gpu_ms", "reference_s", "speedup_vs_reference",
                                                                    "matches_reference", "nnz") if k in pw}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the room and radiosity summaries the default terrain line carries")
    ap.add_argument("--small", action="store_true", help="512^2 / 64 spp / 2 passes case for ncu captures")
    ap.add_argument("--bvh-width", type=int, default=0, choices=[0, 2, 4, 8],
                    help="traversal tree for AO / final gather (0: the library's default)")
    ap.add_argument("--gather", default="disc", choices=["disc", "knn"],
                    help="photon estimate: Relight's disc gather (default) or the k-nearest-neighbour estimate")
    ap.add_argument("--fg-pool", type=int, default=-1, choices=[-1, 0, 1],
                    help="final gather / AO / batch kernels with per-warp lumel pools (1) or one lumel per lane (0); "
                         "-1: the library's default")
    ap.add_argument("--split", action="store_true",
                    help="one terrain bake split over the ranks (photon shares and interleaved final-gather lumels, "
                         "NCCL all-reduces; strong scaling) instead of one bake per rank")
    ap.add_argument("--knn-cell", type=int, default=0,
                    help="kNN grid cell width in 64ths of the radius (0: the library's default)")
    ap.add_argument("--workload", default="terrain",
                    choices=["terrain", "room", "radiosity", "batch", "serve", "denoise"],
                    help="terrain: the photon + final-gather bake (default); room: direct light + AO; radiosity: "
                         "hemisphere form factors + Jacobi; batch: uneven-size batching; serve: the bake-serving "
                         "loop with the denoiser; denoise: the denoiser at equal RMSE")
    args = ap.parse_args()
    global SMALL
    SMALL = args.small
    if args.bvh_width:
        from relight_b200 import autotune
        autotune.set_width(args.bvh_width)
    if args.knn_cell:
        from relight_b200 import autotune
        autotune.set_knn_cell(args.knn_cell)
    if args.fg_pool >= 0:
        from relight_b200 import autotune
        autotune.set_pool(args.fg_pool)
    if args.workload == "batch":
        print(json.dumps(batch_arm(args)), flush=True)
        return
    if args.workload == "room":
        print(json.dumps(room_arm(args)), flush=True)
        return
    if args.workload == "radiosity":
        print(json.dumps(radiosity_arm(args)), flush=True)
        return
    if args.workload == "serve":
        print(json.dumps(serve_arm(args)), flush=True)
        return
    if args.workload == "denoise":
        print(json.dumps(denoise_arm(args)), flush=True)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        out = reference_arm(args, rank, world)
        if out is not None:
            print(json.dumps(out), flush=True)
        return
    import torch
    if world > 1:
        import datetime
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                             device_id=torch.device("cuda", local_rank))
    result, w = gpu_arm(args, rank, world, local_rank)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb, err = cpu_baseline(w)
        result["cpu_baseline"] = cb if cb else {"unavailable": err}
    if rank == 0 and world == 1 and not args.split and args.gather == "disc" and not args.no_extras:
        result["other_workloads"] = other_workloads(args)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(result), flush=True)


if __name__ == "__main__":
    main()
