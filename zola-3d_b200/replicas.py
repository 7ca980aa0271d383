"""Replica plumbing for several GPUs, one process per GPU.

Frames and ROIs are independent, so N GPUs run N independent replicas of the
whole detect -> fit path.  Each rank takes a contiguous share of the frames
(or ROIs), runs it on its own GPU, and rank 0 concatenates the result rows in
rank order, which is frame order; localization ids are renumbered over the
whole stack as one process would number them.  The only collectives are host
bookkeeping: barriers around timed regions, the maximum of the per-rank device
times, and the gather of result rows.  Nothing crosses NVLink on the data
path.

Works with any torch.distributed backend (NCCL on GPUs, gloo on CPU); with no
process group, or a group of one, every function is the single-process case.
"""
import numpy as np


def _dist():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        return dist
    return None


def contiguous_share(n, rank, world):
    """[start, stop) of `rank`'s contiguous share of n items; the first n % world ranks take one extra."""
    if world < 1 or not 0 <= rank < world or n < 0:
        raise ValueError("need world >= 1, 0 <= rank < world, n >= 0")
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def max_over_ranks(value, device=None):
    """Maximum of a per-rank float (a device time) over all ranks."""
    dist = _dist()
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier():
    dist = _dist()
    if dist is not None:
        dist.barrier()


def gather_rows(rows, dst=0):
    """Concatenate every rank's structured result rows on rank `dst` in rank
    order; other ranks get None.  An `id` field is renumbered 0..n-1."""
    dist = _dist()
    if dist is None:
        return rows
    parts = [None] * dist.get_world_size() if dist.get_rank() == dst else None
    dist.gather_object(np.asarray(rows), parts, dst=dst)
    if dist.get_rank() != dst:
        return None
    out = np.concatenate(parts)
    if out.dtype.names and "id" in out.dtype.names:
        out["id"] = np.arange(len(out), dtype=out["id"].dtype)
    return out


def localize_frames_replicated(localize, frames, rank, world, **kw):
    """Run `localize(frames_share, frame0=start, **kw)` (e.g. the package's
    localize_frames bound to this rank's context and PSFs) on this rank's
    contiguous share of the stack and gather the rows on rank 0."""
    start, stop = contiguous_share(len(frames), rank, world)
    rows = localize(frames[start:stop], frame0=start, **kw)
    return gather_rows(rows)
