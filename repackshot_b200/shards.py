"""How a render is split over ranks (one process per GPU). Every (pixel, sample index) of a frame
is independent: its random numbers depend only on (seed, x, y, sample index)
(engine/crates/rt-core/src/sampler.rs:17-26). So a multi-GPU render is a set of replicas with no
data-path collective: each rank renders either its own range of sample indices of the whole frame,
or its own band of rows at every sample; films combine at the end (a sum, or a gather of rows).

A band of rows keeps each pixel's samples on one rank, added in index order, so gathered bands
equal a one-process film bit for bit. Sample ranges keep per-GPU work fixed as ranks are added
(the benchmark's weak scaling); their films sum to the film of all samples up to float rounding.
"""
from __future__ import annotations


def sample_range(rank: int, world: int, spp_per_rank: int) -> tuple[int, int]:
    """(first sample index, count) of a rank's replica of the frame."""
    if not (0 <= rank < world) or spp_per_rank < 1:
        raise ValueError(f"rank {rank} of {world}, {spp_per_rank} spp per rank")
    return rank * spp_per_rank, spp_per_rank


def row_band(rank: int, world: int, height: int) -> tuple[int, int]:
    """(first row, row count) of a rank's band: rows split as evenly as whole rows allow, the
    first ``height % world`` ranks one row taller. A rank may get no rows when world > height."""
    if not (0 <= rank < world) or height < 0:
        raise ValueError(f"rank {rank} of {world}, height {height}")
    base, extra = divmod(height, world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def max_over_ranks(value: float, dist=None) -> float:
    """The largest of every rank's value (the job's time is its slowest rank's). ``dist`` is an
    initialised torch.distributed module, or None for one process."""
    if dist is None or not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
