"""Replicas across GPUs: one process per GPU, each running the whole path on
its own block of columns.

Columns are independent (src/pyPamtraLib.f90:119-133), so there is no
exchange step on the data path; the reference farms (column, frequency)
chunks to CPU worker processes for the same reason
(python/pyPamtra/core.py:1570-1676, runParallelPamtra).  What crosses ranks
is host-side only: the device time of a step, reduced to the maximum over
ranks, and the results of each block, gathered to rank 0.  Any
``torch.distributed`` process group works (NCCL on GPUs, gloo on CPU).
"""

import numpy as np


def column_block(ncol, world, rank):
    """Contiguous block of the ``ncol`` columns owned by ``rank`` of
    ``world``: block sizes differ by at most one, lower ranks take the
    larger ones."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank %d outside a world of %d" % (rank, world))
    base, extra = divmod(int(ncol), world)
    start = rank * base + min(rank, extra)
    return slice(start, start + base + (1 if rank < extra else 0))


def slice_columns(cols, sl):
    """The packed columns (pamtra_b200.packing.profile_columns, optionally
    with full spectra) of block ``sl``: every per-column array is cut along
    its first axis, the scalar sizes are kept, ``ncol`` follows the block."""
    ncol = int(cols["ncol"])
    out = dict()
    for k, v in cols.items():
        if isinstance(v, np.ndarray) and v.ndim >= 1 and v.shape[0] == ncol:
            out[k] = np.ascontiguousarray(v[sl])
        else:
            out[k] = v
    out["ncol"] = len(range(ncol)[sl])
    return out


def max_over_ranks(value, group=None):
    """Maximum of a per-rank scalar (the time of a step) over all ranks;
    ``value`` itself without an initialised process group."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def gather_blocks(block, group=None):
    """Concatenate every rank's result block (first axis = its columns, in
    rank order) on rank 0; other ranks get None.  Host-side, after the
    device work of the step has finished."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return np.asarray(block)
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    parts = [None] * world if rank == 0 else None
    dist.gather_object(np.asarray(block), parts, dst=0, group=group)
    return np.concatenate(parts, axis=0) if rank == 0 else None
