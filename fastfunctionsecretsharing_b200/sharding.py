"""Element sharding across ranks (one process per GPU).

Every FSS element is independent (src/kernel/parallel_execute.h:96-106 of the reference), so
a batch splits into contiguous element ranges with no data-path collective; outputs stay
sharded. The only cross-rank traffic is timing: the max of per-rank durations.
"""

from __future__ import annotations


def shard_range(n: int, rank: int, world: int) -> tuple[int, int]:
    """[begin, end) of the contiguous slice of n elements owned by `rank`."""
    if world <= 0 or not (0 <= rank < world):
        raise ValueError("rank must be in [0, world)")
    base, rem = divmod(n, world)
    begin = rank * base + min(rank, rem)
    return begin, begin + base + (1 if rank < rem else 0)


def key_slice_offsets(n_elems: int, regions: list[int], begin: int, end: int) -> list[tuple[int, int]]:
    """Byte ranges of a key whose layout is a sequence of element-major regions (per-element
    strides `regions`) that belong to elements [begin, end): one (offset, length) per region.
    A rank copies these ranges to build its local key buffer."""
    out, off = [], 0
    for stride in regions:
        out.append((off + begin * stride, (end - begin) * stride))
        off += n_elems * stride
    return out


def max_over_ranks(value: float, world: int) -> float:
    """Max of a per-rank float over the default process group (identity when world == 1)."""
    if world <= 1:
        return value
    import torch
    import torch.distributed as dist

    backend = dist.get_backend()
    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
