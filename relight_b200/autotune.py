"""Autotuner for the ray-stream kernels' launch parameters (rl_tune_set):
the warp refill threshold and the block size.  It times one kernel call per
candidate on the caller's own scene and map (device events on the given
stream) and keeps the fastest.  The parameters change only scheduling, so
every candidate produces bit-identical lightmaps; the test suite checks
that.
"""
from __future__ import annotations

import ctypes as C
import itertools

from . import _abi

REFILLS = (1, 4, 8, 12, 16, 20, 24, 28, 32)
BLOCKS = (64, 128, 256)


KERNELS = {"indirect": (_abi.TUNE_FG_REFILL, _abi.TUNE_FG_BLOCK), "ao": (_abi.TUNE_AO_REFILL, _abi.TUNE_AO_BLOCK)}


def get(kernel="indirect"):
    v = C.c_int()
    out = {}
    for name, p in zip(("refill", "block"), KERNELS[kernel]):
        _abi.check(_abi.lib().rl_tune_get(p, C.byref(v)))
        out[name] = v.value
    return out


def set(refill=None, block=None, kernel="indirect"):
    pr, pb = KERNELS[kernel]
    if refill is not None:
        _abi.check(_abi.lib().rl_tune_set(pr, int(refill)))
    if block is not None:
        _abi.check(_abi.lib().rl_tune_set(pb, int(block)))


def get_width():
    v = C.c_int()
    _abi.check(_abi.lib().rl_tune_get(_abi.TUNE_BVH_WIDTH, C.byref(v)))
    return v.value


def set_width(width):
    _abi.check(_abi.lib().rl_tune_set(_abi.TUNE_BVH_WIDTH, int(width)))


def get_speculative():
    v = C.c_int()
    _abi.check(_abi.lib().rl_tune_get(_abi.TUNE_SPECULATIVE, C.byref(v)))
    return v.value


def set_speculative(on):
    _abi.check(_abi.lib().rl_tune_set(_abi.TUNE_SPECULATIVE, int(bool(on))))


def get_pool():
    """(pool, chunk): the final gather's persistent lumel pool (0/1) and the
    lumels a warp claims at a time."""
    v = C.c_int()
    out = []
    for p in (_abi.TUNE_FG_POOL, _abi.TUNE_FG_CHUNK):
        _abi.check(_abi.lib().rl_tune_get(p, C.byref(v)))
        out.append(v.value)
    return tuple(out)


def set_pool(on=None, chunk=None):
    if on is not None:
        _abi.check(_abi.lib().rl_tune_set(_abi.TUNE_FG_POOL, int(bool(on))))
    if chunk is not None:
        _abi.check(_abi.lib().rl_tune_set(_abi.TUNE_FG_CHUNK, int(chunk)))


def get_knn_cell():
    v = C.c_int()
    _abi.check(_abi.lib().rl_tune_get(_abi.TUNE_KNN_CELL, C.byref(v)))
    return v.value


def set_knn_cell(sixty_fourths):
    """kNN grid cell width in 64ths of the search radius (8..256)."""
    _abi.check(_abi.lib().rl_tune_set(_abi.TUNE_KNN_CELL, int(sixty_fourths)))


def tune(run, kernel="indirect", refills=REFILLS, blocks=BLOCKS, widths=(2,), speculative=(0, 1), reps=2,
         stream=None):
    """`run()` enqueues one call of `kernel` ("indirect" or "ao") on `stream`
    (a torch stream, None = the current one).  Returns (best, table), table
    mapping (refill, block, width, speculative) -> milliseconds; the best
    setting is left applied.  Width and speculation are shared by both kernels."""
    import torch
    st = stream or torch.cuda.current_stream()
    table = {}
    for width, spec, refill, block in itertools.product(widths, speculative, refills, blocks):
        if width == 4 and spec:
            continue
        set_width(width)
        set_speculative(spec)
        set(refill, block, kernel)
        run()
        ms = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            run()
            e1.record(st)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
        table[(refill, block, width, spec)] = min(ms)
    best = min(table, key=table.get)
    set(best[0], best[1], kernel)
    set_width(best[2])
    set_speculative(best[3])
    return {"refill": best[0], "block": best[1], "width": best[2], "speculative": best[3], "ms": table[best]}, table


def tune_batch(jobs, stream=None, refills=(16, 24, 32), blocks=(64, 128), sample=8, reps=2, reset=None):
    """Tune the batch kernels' refill threshold (rays in flight per warp)
    and block size, per pass kind, on every `sample`-th job of `jobs` (a
    list of batch.BakeJob).  Each candidate builds a batch (the launch shape
    is fixed when a batch is made) and times one launch per rep; `reset()`
    (optional) restores the lightmaps between launches.  The best setting
    per kind is left applied, so batches made afterwards use it.  Returns
    {kind: (best, table)}."""
    import torch
    from . import batch as B
    st = stream or torch.cuda.current_stream()
    out = {}
    for kind, name in ((B.AO, "ao"), (B.INDIRECT, "indirect")):
        sub = [j for j in jobs if j.kind == kind][::max(sample, 1)]
        if not sub:
            continue
        table = {}
        for refill, block in itertools.product(refills, blocks):
            set(refill, block, name)
            b = B.Batch(sub)
            ms = []
            for _ in range(reps + 1):
                if reset:
                    reset()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(st)
                b.launch(st.cuda_stream)
                e1.record(st)
                e1.synchronize()
                ms.append(e0.elapsed_time(e1))
            b.close()
            table[(refill, block)] = min(ms[1:])
        best = min(table, key=table.get)
        set(best[0], best[1], name)
        out[name] = ({"refill": best[0], "block": best[1], "ms": table[best]}, table)
    return out
