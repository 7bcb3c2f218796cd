"""One bake split across GPUs (one process per GPU, torch.distributed).

Each pass shards its units with no exchange until the step that needs one:

  photons       rank r traces the contiguous share [first, first + count) of
                the reference's global photon sequence (pass-major, then light,
                then photon, as Photons::emit loops, baker/Photons.cpp:50-92)
                into its own replica of every photonmap; one all-reduce (sum)
                of the colour and count accumulators then gives every rank the
                unsplit accumulators, and each rank gathers
                (Photonmap::gather) its replica locally.
  final gather  rank r bakes the lumels first = r, step = world
                (LumelBakeIterator(r, world), baker/Baker.cpp:176-185) into a
                zeroed colour buffer; one all-reduce (sum) assembles the
                contributions (each lumel has exactly one non-zero term, so the
                sum is exact) and every rank adds them to its base colours:
                bit-identical to one GPU.
  radiosity     rank r steps its block of rows of B' = E + rho .* (F B); one
                all-gather of B per iteration.

The sharded_* functions take the collective and the compute as arguments;
the *_distributed functions take an engine object (the CUDA Relight, or an
oracle adapter in the tests), so the same code drives the CUDA library
under NCCL and the CPU oracle under gloo.
"""
from __future__ import annotations

from typing import Callable, Sequence


def photon_share(total: int, rank: int, world: int):
    """Contiguous block of the photon sequence owned by `rank`."""
    base, extra = divmod(total, world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def row_block(n: int, rank: int, world: int):
    first, count = photon_share(n, rank, world)
    return first, first + count


def sharded_photons(emit_range: Callable[[int, int], None], accumulators: Sequence, total: int, rank: int,
                    world: int, all_reduce_sum: Callable) -> None:
    """Trace this rank's photon share, then sum the photonmap accumulators
    (colour float sums, integer counts) over ranks in place."""
    first, count = photon_share(total, rank, world)
    emit_range(first, count)
    for acc in accumulators:
        all_reduce_sum(acc)


def sharded_final_gather(bake_subset: Callable[[int, int], None], contribution, base, rank: int, world: int,
                         all_reduce_sum: Callable, add_inplace: Callable) -> None:
    """`bake_subset(first, step)` bakes the lumels first, first+step, ... into
    `contribution` (zeroed beforehand); after the all-reduce every rank holds
    all contributions and adds them to `base`."""
    bake_subset(rank, world)
    all_reduce_sum(contribution)
    add_inplace(base, contribution)


def sharded_jacobi(step_rows: Callable[[int, int, object, object], None], B, B_next_local, iters: int, n: int,
                   rank: int, world: int, all_gather_rows: Callable) -> None:
    """`step_rows(r0, r1, B, out)` writes rows [r0, r1) of one Jacobi step
    into `out`; `all_gather_rows(out, B)` assembles every rank's rows into B."""
    r0, r1 = row_block(n, rank, world)
    for _ in range(iters):
        step_rows(r0, r1, B, B_next_local)
        all_gather_rows(B_next_local, B)


# ------------------------------------------------------------- CUDA engine

class _CudaArray:
    """A torch-visible view of a device pointer owned by an rl_map."""

    def __init__(self, ptr: int, shape, typestr: str):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 3, "strides": None}


def map_tensor(dev_map, field: str):
    """Zero-copy torch tensor over one lumel array of a DeviceMap."""
    import torch
    ptrs = dev_map.device_arrays()
    n = dev_map.width * dev_map.height
    if field in ("flags", "photons"):
        return torch.as_tensor(_CudaArray(ptrs[field], (n,), "<i4"), device="cuda")
    return torch.as_tensor(_CudaArray(ptrs[field], (n, 3), "<f4"), device="cuda")


def _group_info(group):
    import torch.distributed as dist
    return dist.get_rank(group), dist.get_world_size(group)


def _all_reduce_sum(group):
    import torch.distributed as dist
    return lambda t: dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)


class _on_stream:
    """Run the collectives on the engine's stream (torch's current stream
    when it has none), so they order with its kernels."""

    def __init__(self, engine):
        self.s = engine.torch_stream() if hasattr(engine, "torch_stream") else None

    def __enter__(self):
        if self.s is not None:
            import torch
            self.ctx = torch.cuda.stream(self.s)
            self.ctx.__enter__()
        return self

    def __exit__(self, *a):
        if self.s is not None:
            self.ctx.__exit__(*a)


# An engine provides: photon_total, emit_photon_range, photon_accumulators,
# gather_photons, color_tensor, bake_indirect_light (Relight's signature,
# with iterator and seed), radiosity_step and, for CUDA, torch_stream.
# relight_b200.device.Relight is the CUDA engine (NCCL); the tests drive the
# same functions with the oracle under gloo.

def emit_photons_distributed(engine, scene, settings, seed: int, group=None) -> None:
    """Relight::emitPhotons for one bake split over the ranks of `group`:
    every rank traces its share of the photon sequence, the photonmap
    accumulators are summed over ranks, and every rank gathers its (now
    complete) photonmaps."""
    rank, world = _group_info(group)
    total = engine.photon_total(scene, settings)
    with _on_stream(engine):
        sharded_photons(lambda first, count: engine.emit_photon_range(scene, settings, seed, first, count),
                        engine.photon_accumulators(scene), total, rank, world, _all_reduce_sum(group))
    engine.gather_photons(scene, settings)


def bake_indirect_distributed(engine, scene, mesh, settings, seed: int, group=None) -> None:
    """Relight::bakeIndirectLight over the whole lightmap of `mesh`, split
    over the ranks of `group`: rank r bakes LumelBakeIterator(r, world) into
    zeroed colours, the contributions are summed over ranks (one non-zero
    term per lumel, so exactly), and every rank adds its base colours.
    Every lumel gets base + contribution, the single-GPU bake's own float
    addition: the same bits on every rank as one GPU baking alone."""
    from .device import LumelBakeIterator
    rank, world = _group_info(group)
    color = engine.color_tensor(mesh.lightmap)
    with _on_stream(engine):
        base = color.clone()
        color.zero_()
    sharded_final_gather(
        lambda first, step: engine.bake_indirect_light(scene, mesh, None, settings, LumelBakeIterator(first, step),
                                                       seed=seed),
        color, base, rank, world, lambda t: _run_on(engine, _all_reduce_sum(group), t),
        lambda b, c: _run_on(engine, lambda t: t.add_(b), c))


def _run_on(engine, fn, t):
    with _on_stream(engine):
        return fn(t)


def radiosity_solve_distributed(engine, n: int, row, cols, vals, E, rho, iters: int, B_out, group=None) -> None:
    """The 50-iteration Jacobi solve with rows sharded over the ranks of
    `group`: each iteration, rank r steps its block of rows
    (engine.radiosity_step) and one all-gather assembles B on every rank.
    Tensors are [n][3] (colours) on the engine's device; B_out receives B."""
    import torch
    import torch.distributed as dist
    rank, world = _group_info(group)
    r0, r1 = row_block(n, rank, world)
    blocks = [row_block(n, q, world) for q in range(world)]
    rows = max(b - a for a, b in blocks)
    with _on_stream(engine):
        B = E.clone()
        Bn = torch.empty_like(E)
        local = torch.zeros((rows, 3), dtype=E.dtype, device=E.device)
        gathered = torch.empty((world * rows, 3), dtype=E.dtype, device=E.device)
    for _ in range(iters):
        engine.radiosity_step(r0, r1, row, cols, vals, E, rho, B, Bn)
        with _on_stream(engine):
            local[:r1 - r0].copy_(Bn[r0:r1])
            dist.all_gather(list(gathered.view(world, rows, 3).unbind(0)), local, group=group)
            for q, (a, b) in enumerate(blocks):
                B[a:b].copy_(gathered[q * rows:q * rows + (b - a)])
    with _on_stream(engine):
        B_out.copy_(B)
