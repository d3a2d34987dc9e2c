"""One image over N GPUs by sample index (one process per GPU, torch.distributed).

Physical and guided renders depend only on (pixel, sample index, seed), so N
ranks that render disjoint, contiguous slices of the sample indices and sum
their FP64 accumulations (rgb sum, sample count per pixel) produce the render
of all samples, up to the order of the FP64 additions. The one exchange is an
all-reduce (sum) of W * H * 4 doubles: over NCCL between B200s (NVLink /
NVSwitch; 32 MB for a 1024^2 image), over gloo in the CPU tests. The
accumulation is reduced in place in the library's device buffer; nothing else
crosses between ranks. In the guided mode every rank trains its own guide on
its own samples (no gradient exchange), which keeps each rank's estimate
unbiased and the sum a valid render.

Scene replication is the caller's: each rank uploads the same scene to its
own context.
"""
from __future__ import annotations


def sample_slice(spp: int, rank: int, world: int) -> tuple[int, int]:
    """(first sample index, count) of `rank` among `world` ranks: contiguous
    slices covering 0 .. spp - 1, the remainder spread over the first ranks."""
    if world < 1 or not 0 <= rank < world or spp < 0:
        raise ValueError("need world >= 1, 0 <= rank < world, spp >= 0")
    base, extra = divmod(spp, world)
    return rank * base + min(rank, extra), base + (1 if rank < extra else 0)


class _DeviceArray:
    """__cuda_array_interface__ over a device pointer, for a zero-copy torch view."""

    def __init__(self, ptr: int, shape, typestr: str):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 3, "strides": None}


def accumulation_f64(ctx, width: int, height: int):
    """torch float64 [H, W, 4] view (no copy) of the context's device FP64
    accumulation: rgb sum and sample count per pixel."""
    import torch

    return torch.as_tensor(_DeviceArray(ctx.render_buffer_f64(), (height, width, 4), "<f8"), device="cuda")


def allreduce_accumulation(acc, group=None):
    """Sums the ranks' accumulations in place (the one collective of a sharded render)."""
    import torch.distributed as dist

    dist.all_reduce(acc, op=dist.ReduceOp.SUM, group=group)
    return acc


def resolve(acc):
    """Mean radiance per pixel (sum / count) of a reduced accumulation."""
    return acc[..., :3] / acc[..., 3:4].clamp_min(1.0)


def render_sharded(ctx, inverse_view, inverse_projection, width: int, height: int, spp: int, group=None, **kw):
    """This rank's slice of a physical (or guided, guided=True) render of `spp`
    samples per pixel, then the all-reduce. Returns the reduced FP64
    accumulation as a torch tensor on this rank's GPU (a view of the library's
    buffer when this rank rendered samples). Every rank must call it with the
    same arguments."""
    import torch
    import torch.distributed as dist

    rank, world = dist.get_rank(group), dist.get_world_size(group)
    first, count = sample_slice(spp, rank, world)
    if count:
        ctx.begin_samples(first)
        ctx.render_physical(inverse_view, inverse_projection, width, height, spp=count, fp64=True, **kw)
        ctx.sync()  # the library's stream is done before torch's stream reduces the buffer
        acc = accumulation_f64(ctx, width, height)
    else:
        acc = torch.zeros((height, width, 4), dtype=torch.float64, device="cuda")
    allreduce_accumulation(acc, group)
    # the next render on this context writes the same buffer from the library's stream
    torch.cuda.current_stream().synchronize()
    return acc
