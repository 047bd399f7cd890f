"""How a multi-GPU job splits the sysmat: one process per GPU, disjoint parts,
no collective on the data path.

Every (crystal, voxel) entry is independent (the reference computes each in
its own thread, PESysMatGen.cu:375-764), so ranks take disjoint z-slabs of the
image (and, for the C ABI's callers, disjoint crystal row ranges) and write
disjoint parts of the output.  The only collective is the timing scalar,
reduced with MAX so the job is as slow as its slowest rank.
"""
from typing import List, Tuple


def slab_of(step: int, rank: int, world: int, n_slabs: int) -> int:
    """The z-slab rank `rank` computes at bench step `step`: within a step the
    ranks take consecutive slabs, and steps walk through the image."""
    if not (0 <= rank < world) or n_slabs <= 0:
        raise ValueError("rank %d of %d, %d slabs" % (rank, world, n_slabs))
    return (step * world + rank) % n_slabs


def row_range(n_rows: int, rank: int, world: int) -> Tuple[int, int]:
    """Crystal rows [r0, r1) of rank `rank` when a whole matrix is split by
    rows: contiguous, sizes differing by at most one."""
    if not (0 <= rank < world):
        raise ValueError("rank %d of %d" % (rank, world))
    base, extra = divmod(n_rows, world)
    r0 = rank * base + min(rank, extra)
    return r0, r0 + base + (1 if rank < extra else 0)


def max_over_ranks(values: List[float], device=None) -> List[float]:
    """Element-wise maximum over the ranks of the default process group (the
    identity without one).  Every rank must call it with the same length."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return [float(v) for v in values]
    t = torch.tensor(values, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]
