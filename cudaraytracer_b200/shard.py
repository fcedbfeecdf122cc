"""Multi-GPU rendering of one frame by sample ranges.

Every path's PCG32 stream is keyed by (seed, pixel, sample), so disjoint
sample ranges of the same frame are independent: each rank renders its own
range on its own GPU, and the one exchange is a sum-reduce of the float
accumulators (direct, indirect and optionally sum of squares, float4 per
pixel) onto the destination rank, over NCCL on NVLink. The sum over ranks is
the frame a single GPU renders with all samples, up to the order of the float
additions. The reference renders on one GPU only (Src/Core/renderer.cuh:
1106-1307); this module is the process-per-GPU extension of that loop.

One process per GPU, launched by torchrun; the process group is the
caller's (`torch.distributed.init_process_group("nccl")`).
"""
from __future__ import annotations

from typing import Callable


def sample_range(spp: int, rank: int, world: int, first_sample: int = 0) -> tuple[int, int]:
    """Contiguous share [first, first + count) of samples [first_sample,
    first_sample + spp) for `rank` of `world`; the first spp % world ranks
    take one extra sample, so the shares tile the range exactly."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world of {world}")
    if spp < 0:
        raise ValueError("spp must be >= 0")
    base, extra = divmod(spp, world)
    count = base + (1 if rank < extra else 0)
    first = first_sample + rank * base + min(rank, extra)
    return first, count


def reduce_sample_shards(render_fn: Callable[[int, int], tuple], spp: int, first_sample: int = 0, dst: int = 0,
                         group=None, all_ranks: bool = False):
    """Runs render_fn(first, count) for this rank's share of the samples,
    returning accumulator tensors (direct, indirect[, sumsq]), then sums them
    over the group onto rank `dst` (every rank when all_ranks). Every rank
    calls this with the same spp, first_sample and dst, in the same order.
    Returns the summed tensors on dst (and on every rank when all_ranks);
    on other ranks the returned tensors hold undefined partial data after
    the reduce, as a collective reduce leaves them."""
    import torch.distributed as dist

    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    first, count = sample_range(spp, rank, world, first_sample)
    acc = tuple(t for t in render_fn(first, count) if t is not None)
    for t in acc:
        if all_ranks:
            dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        else:
            dist.reduce(t, dst=dist.get_global_rank(group, dst) if group is not None else dst,
                        op=dist.ReduceOp.SUM, group=group)
    return acc


def render_sharded(scene, spp: int, first_sample: int = 0, with_sumsq: bool = False, dst: int = 0, group=None,
                   all_ranks: bool = False):
    """Renders samples [first_sample, first_sample + spp) of `scene`'s
    current camera over all ranks of `group` (one GPU each, the scene loaded
    on every rank) and sums the accumulators onto `dst`. Returns CUDA float32
    tensors (H, W, 4): direct, indirect[, sumsq], rows bottom-up."""
    import torch

    rp = scene.render_params()
    dev = torch.device("cuda", scene.ctx.device)
    shape = (rp["height"], rp["width"], 4)

    def render(first, count):
        d = torch.zeros(shape, device=dev)
        i = torch.zeros(shape, device=dev)
        q = torch.zeros(shape, device=dev) if with_sumsq else None
        if count:
            scene.render_device(d, i, count, first_sample=first, sumsq=q)
        return d, i, q

    return reduce_sample_shards(render, spp, first_sample, dst, group, all_ranks)
