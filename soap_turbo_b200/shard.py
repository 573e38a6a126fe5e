"""Site sharding for one process per GPU.

Every site (environment) is independent given its CSR row, and W, S and the
compression map are small replicated constants, so N GPUs split a batch into
contiguous, pair-balanced site ranges and need no collective on the data path.
The only collective is the max-over-ranks of the step time.
"""
from __future__ import annotations

import copy

import numpy as np


def site_shards(n_neigh, world_size: int):
    """Contiguous site ranges [(lo, hi), ...], one per rank, balanced by pairs."""
    n_neigh = np.asarray(n_neigh, dtype=np.int64)
    off = np.concatenate([[0], np.cumsum(n_neigh)])
    total = off[-1]
    cuts = [0]
    for r in range(1, world_size):
        cuts.append(int(np.searchsorted(off, total * r / world_size, side="left")))
    cuts.append(len(n_neigh))
    cuts = np.maximum.accumulate(np.asarray(cuts))
    return [(int(cuts[r]), int(cuts[r + 1])) for r in range(world_size)]


def slice_sites(nl, lo: int, hi: int):
    """The neighbour list of sites [lo, hi) as a batch of its own."""
    off = np.concatenate([[0], np.cumsum(nl.n_neigh)])
    p0, p1 = int(off[lo]), int(off[hi])
    out = copy.copy(nl)
    out.n_sites = hi - lo
    out.n_neigh = nl.n_neigh[lo:hi]
    out.rjs, out.thetas, out.phis = nl.rjs[p0:p1], nl.thetas[p0:p1], nl.phis[p0:p1]
    out.mask = nl.mask[:, p0:p1]
    out.species = nl.species[lo:hi]
    out.species_multiplicity = nl.species_multiplicity[lo:hi]
    out.site_atom = nl.site_atom[lo:hi]
    out.neigh_atom = nl.neigh_atom[p0:p1]
    out.disp = nl.disp[p0:p1]
    return out


def max_over_ranks(value: float, device=None) -> float:
    """The largest value over all ranks (step times are reported this way)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
