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

The functions take the collective and the compute as arguments, so the same
code drives the CUDA library under NCCL and the CPU oracle under gloo.
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


def emit_photons_distributed(relight, scene, settings, seed: int, group=None) -> None:
    """Relight::emitPhotons for one bake split over the ranks of `group`
    (NCCL): every rank ends with the full, gathered photonmaps."""
    import ctypes as C

    import torch.distributed as dist

    from . import _abi
    from .device import _map_array

    rank, world = dist.get_rank(group), dist.get_world_size(group)
    ds = relight.device_scene(scene)
    f = scene.flat
    maps = [m._device for m in f.photonmaps]
    lights = C.c_void_p(f.lights.ctypes.data)
    total = C.c_int64()
    _abi.check(_abi.lib().rl_photon_count(lights, len(f.lights), settings.photon_pass_count, C.byref(total)))
    L = _abi.lib()

    def emit_range(first, count):
        _abi.check(L.rl_emit_photons_range(ds.handle, _map_array(maps), len(maps), lights, len(f.lights),
                                           settings.photon_pass_count, settings.photon_bounce_count,
                                           settings.photon_energy_threshold, settings.photon_max_distance, seed,
                                           first, count, None, relight.stream))

    accs = [map_tensor(m, "color") for m in maps] + [map_tensor(m, "photons") for m in maps]
    sharded_photons(emit_range, accs, total.value, rank, world,
                    lambda t: dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group))
    for m in maps:
        _abi.check(L.rl_photonmap_gather(m.handle, settings.final_gather_radius, relight.stream))
