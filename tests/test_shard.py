"""Sector sharding of one curve over ranks: assignment, and the merge of the
grand-canonical accumulators over a gloo process group (CPU, world size 2),
checked against one accumulation over all blocks by the oracle."""
import os
import socket
import sys
from math import comb

import numpy as np
import torch.multiprocessing as tmp

from ftlm_extended_hubbard_development_b200 import shard

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "oracle"))
import pyoracle as po  # noqa: E402

BETAS = [0.7, 4.0]
MU = np.linspace(-2.0, 6.0, 17)


def _blocks(seed=5, nblocks=24):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(nblocks):
        p = int(rng.integers(0, 9))
        ev = np.sort(rng.normal(size=30) * 2 + 0.6 * p * p - 1.5 * p)
        w = rng.random(30) + 0.05
        out.append((ev, w, float(rng.integers(1, 50)), p))
    return out


def _accumulate(blocks):
    nb, nm = len(BETAS), len(MU)
    emin = np.full((nb, nm), np.inf)
    z, n, n2 = np.zeros((nb, nm)), np.zeros((nb, nm)), np.zeros((nb, nm))
    for ib, beta in enumerate(BETAS):
        st = (emin[ib], z[ib], n[ib], n2[ib])
        for ev, w, pref, p in blocks:
            po.thermo_accumulate(ev, w, pref, p, beta, MU, st)
    return emin, z, n, n2


def test_sector_owners_cover_and_balance():
    for sites, world in ((8, 2), (16, 8), (18, 3), (4, 5)):
        own = shard.sector_owners(sites, world)
        assert sorted(own) == [(a, b) for a in range(sites + 1) for b in range(sites + 1)]
        load = [0] * world
        for (a, b), r in own.items():
            load[r] += comb(sites, a) * comb(sites, b)
        biggest = comb(sites, sites // 2) ** 2
        assert max(load) - min(load) <= biggest
    assert shard.sector_owners(8, 1) == {s: 0 for s in shard.sector_owners(8, 1)}


def _worker(rank, world, port, q):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        blocks = _blocks()
        mine = [b for i, b in enumerate(blocks) if i % world == rank]
        emin, z, n, n2 = _accumulate(mine)
        mn, sm = shard.torch_collectives()
        g = shard.merge_accumulators(emin, z, n, n2, BETAS, mn, sm)
        q.put((rank, [np.asarray(a) for a in g]))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_merge_over_gloo_equals_single_accumulation():
    world = 2
    ctx = tmp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    ref = shard.finalize(BETAS, 8, *_accumulate(_blocks()))
    for r in range(world):
        res = shard.finalize(BETAS, 8, *got[r])
        for k in ("n", "charge_correlation", "log_partition"):
            assert np.allclose(res[k], ref[k], rtol=1e-12, atol=1e-12), k


def test_merge_handles_ranks_without_blocks():
    """A rank that owns no sector (emin = +inf, sums 0) changes nothing."""
    parts = [_accumulate(_blocks(seed=9, nblocks=6)), _accumulate([])]
    mn = lambda a: np.minimum(parts[0][0], parts[1][0])  # noqa: E731
    rescaled = [shard.merge_accumulators(*p, BETAS, mn, lambda a: a)[1:] for p in parts]
    total = [rescaled[0][i] + rescaled[1][i] for i in range(3)]
    res = shard.finalize(BETAS, 8, mn(None), *total)
    ref = shard.finalize(BETAS, 8, *parts[0])
    assert np.isfinite(res["n"]).all()
    assert np.allclose(res["n"], ref["n"], rtol=1e-14, atol=0)
