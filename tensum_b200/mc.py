"""Monte Carlo sample driver and moment reduction over groups.

The reference runs N_MC_GROUPS processor groups, each over a contiguous block
of the sorted sample list (src/parameter.cc:826-845), accumulates online
statistics per group with increment_moments at every output time
(src/fv.cc:595-694, called from FiniteVolume::solve, src/fv.cc:2230-2380) and
merges the groups into group 0 with reduce_moments (src/reduce_moments.cc:
14-221).  Here a group is one GPU (one process, one ``gpu.Solver``); the merge
gathers every group's device block with one collective and applies the same
per-group update in the same (ascending group) order into group 0, as
reduce_moments does.
"""
from __future__ import annotations

from typing import Callable, Iterable, Sequence

import numpy as np


def group_range(n_samples: int, n_groups: int, group: int) -> tuple[int, int]:
    """Indices [start, end] (inclusive) of the sample list handled by `group`
    (src/parameter.cc:831-842: the first n_samples % n_groups groups take one
    extra sample)."""
    if n_samples < n_groups:
        raise ValueError("fewer samples than Monte Carlo groups (src/parameter.cc:208-209)")
    overflow = n_samples % n_groups
    normal = n_samples // n_groups
    if group < overflow:
        start = group * (normal + 1)
        end = start + normal
    else:
        start = group * normal + overflow
        end = start + normal - 1
    return start, end


def run_group(solver, initial_states: Iterable[np.ndarray], n_instances: int, extras: int = 0,
              max_steps_per_instance: int = 1 << 40) -> int:
    """Advance each sample of one group from its initial state through every
    output time, incrementing the group moments as FiniteVolume::solve does
    (instance 0 at the initial state, then each output time when reached).
    Unsteady runs only.  Returns the number of samples in the group."""
    solver.moments_init(n_instances, extras)
    k = 0
    for ic in initial_states:
        k += 1
        solver.set_state(ic)
        solver.moments_increment(0, k)
        for t in range(1, n_instances):
            info = solver.advance(t, max_steps_per_instance)
            if info[4] <= t:
                raise RuntimeError(f"sample {k}: the run ended before output time {t} was reached")
            solver.moments_increment(t, k)
    return k


def reduce_groups(local_block, n_local: int, merge: Callable[[int, int, int, object], None], dist=None,
                  n_instances: int = 1) -> int:
    """Merge every group's moments into group 0 (rank 0), in ascending group order.

    local_block(t) returns this rank's group block of instance t as a tensor
    (three [nvar][n_vertex] arrays; a CUDA tensor under NCCL, a CPU tensor
    under gloo).  merge(t, n_self, n_other, block) applies reduce_moments'
    per-group update of `block` into this rank's moments.  Without a process
    group (or with one rank) nothing is exchanged.  Returns the total sample
    count.

    The collective is one all_gather of the sample counts and one per output
    instance of the blocks; every rank takes the same collective steps in the
    same order, and rank 0 alone merges (groups 1, 2, ... in turn, each with
    the running count, src/reduce_moments.cc:30-38)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return n_local
    import torch
    world = dist.get_world_size()
    rank = dist.get_rank()
    probe = local_block(0)
    counts_t = torch.tensor([n_local], dtype=torch.int64, device=probe.device)
    gathered_counts = [torch.zeros_like(counts_t) for _ in range(world)]
    dist.all_gather(gathered_counts, counts_t)
    counts = [int(c.item()) for c in gathered_counts]
    for t in range(n_instances):
        blk = local_block(t).contiguous()
        parts = [torch.empty_like(blk) for _ in range(world)]
        dist.all_gather(parts, blk)
        if rank == 0:
            n_acc = counts[0]
            for g in range(1, world):
                merge(t, n_acc, counts[g], parts[g])
                n_acc += counts[g]
    return sum(counts)


def sample_shard(samples: Sequence[int], rank: int, world: int) -> list[int]:
    """The samples of one group (one rank) in the reference's contiguous split."""
    s, e = group_range(len(samples), world, rank)
    return list(samples[s:e + 1])
