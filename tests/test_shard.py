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


def test_block_dims_host_match_reference_goldens(golden):
    """Character counting on the host gives the reference's block
    dimensions (main.cpp:745-766) for every sector of the golden lattices."""
    n = 0
    for case, nu, nd in golden.sector_keys():
        c = golden.cases[case]
        want = golden.sec(case, nu, nd, "block_dim")
        assert shard.block_dims_host(c["lx"], c["ly"], nu, nd) == list(want), (case, nu, nd)
        n += 1
    assert n > 100


def test_block_owners_cover_and_balance():
    for lx, ly, world in ((4, 2, 2), (3, 3, 3), (4, 4, 8), (2, 2, 5)):
        m = shard.Model(lx=lx, ly=ly, tp=0.2)
        opts = shard.RunOpts(samples=32, lanczos_steps=80, exact_block_threshold=256)
        own = shard.block_owners(m, world, opts)
        want = {(a, b, k % lx, k // lx) for a in range(m.sites + 1) for b in range(m.sites + 1)
                for k, d in enumerate(shard.block_dims_host(lx, ly, a, b)) if d > 0}
        assert set(own) == want and set(own.values()) <= set(range(world))
        load = [0.0] * world
        big = 0.0
        for (a, b, mx, my), r in own.items():
            d = shard.block_dims_host(lx, ly, a, b)[my * lx + mx]
            h = sum((4 + 4) * p * (m.sites - p) / max(m.sites - 1, 1) for p in (a, b))
            c = shard.block_cost(d, d <= 256, 32, 80, h)
            load[r] += c
            big = max(big, c)
        assert max(load) - min(load) <= big  # LPT bound
    m = shard.Model(lx=4, ly=2)
    assert set(shard.block_owners(m, 1).values()) == {0}


def test_config5_sector_splits_over_two_ranks():
    """The 6x3 (9,9) sector is 18 k-blocks of ~1.313e8 rows: two ranks take
    9 each (one sector no longer lands on one rank)."""
    m = shard.Model(lx=6, ly=3, tp=0.2, phix=0.25, phiy=0.5, u=8.0, v=1.5)
    opts = shard.RunOpts(samples=16, lanczos_steps=100)
    own = shard.block_owners(m, 2, opts, sectors=[(9, 9)])
    assert len(own) == 18
    per = [sum(1 for r in own.values() if r == k) for k in range(2)]
    assert per == [9, 9]


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


def _plan_worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        m = shard.Model(lx=6, ly=3, tp=0.2, phix=0.25, phiy=0.5, u=8.0, v=1.5)
        own = shard.block_owners(m, world, shard.RunOpts(samples=16, lanczos_steps=100), sectors=[(9, 9)])
        mine = sorted(k for k, r in own.items() if r == rank)
        t = torch.zeros(18, dtype=torch.int64)
        for (_, _, mx, my) in mine:
            t[my * 6 + mx] = rank + 1
        dist.all_reduce(t)  # every block claimed by exactly one rank
        q.put((rank, t.tolist(), len(mine)))
    finally:
        dist.destroy_process_group()


def test_config5_plan_agrees_across_gloo_ranks():
    world = 2
    ctx = tmp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_plan_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = dict((r, (t, n)) for r, t, n in (q.get(timeout=120) for _ in range(world)))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(world):
        t, n = got[r]
        assert n == 9 and sorted(t) == [1] * 9 + [2] * 9


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
