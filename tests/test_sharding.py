"""Multi-rank host logic on CPU (gloo, world size 2): pair-balanced site
shards cover the batch exactly once, sharded results equal the unsharded
ones (sites are independent), and step times reduce as a max over ranks."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

import oracle as O
from soap_turbo_b200 import shard
from soap_turbo_b200 import synthetic as syn


def test_site_shards_cover_and_balance():
    w = syn.config(2, seed=2, scale=0.25)
    for ws in (1, 2, 3, 8):
        parts = shard.site_shards(w.nl.n_neigh, ws)
        assert parts[0][0] == 0 and parts[-1][1] == w.nl.n_sites
        for (a, b), (c, d) in zip(parts, parts[1:]):
            assert b == c and a <= b
        pairs = [int(w.nl.n_neigh[a:b].sum()) for a, b in parts]
        assert max(pairs) - min(pairs) <= 2 * int(w.nl.n_neigh.max())


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    w = syn.config(2, seed=4, scale=0.1)
    W, S = O.basis_matrices(w.hyper)
    lo, hi = shard.site_shards(w.nl.n_neigh, world)[rank]
    part = shard.slice_sites(w.nl, lo, hi)
    soap = O.get_soap(w.hyper, part, W, S, do_derivatives=False).soap
    gathered = [None] * world
    dist.all_gather_object(gathered, (lo, hi, soap))
    t = shard.max_over_ranks(float(rank + 1))
    if rank == 0:
        out.put((gathered, t))
    dist.barrier()
    dist.destroy_process_group()


def test_gloo_sharded_descriptor_equals_unsharded():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    gathered, t = q.get(timeout=240)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert t == 2.0
    w = syn.config(2, seed=4, scale=0.1)
    W, S = O.basis_matrices(w.hyper)
    full = O.get_soap(w.hyper, w.nl, W, S, do_derivatives=False).soap
    got = np.concatenate([g[2] for g in sorted(gathered, key=lambda g: g[0])])
    np.testing.assert_array_equal(got, full)
