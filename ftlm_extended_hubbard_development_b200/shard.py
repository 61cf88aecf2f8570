"""One n(mu) curve over several GPUs: sectors sharded over ranks.

The (N_up, N_down) sectors of a curve are independent; each rank runs its
share on its own GPU (one process per GPU, torch.distributed for the
plumbing) and keeps the grand-canonical accumulators (emin, z, <N>z,
<N^2>z)[beta][mu] of its blocks on the device. The only exchange is at the
end: the minimum of emin over ranks (MIN all-reduce), each rank's sums
rescaled to that minimum by exp(-beta (emin_r - emin)), and one SUM
all-reduce of the three sums, 3 * nbeta * nmu doubles, which is the
reference's rescale rule (main.cpp:1172-1219) applied once per rank instead
of once per block.

Sectors are assigned largest first to the least-loaded rank, with the
sector's full dimension C(n, N_up) C(n, N_down) as its cost, so the ranks
finish together; a rank runs its sectors in the reference's block order.
"""
from __future__ import annotations

import heapq
from math import comb

import numpy as np

from .engine import Engine, Model, RunOpts


def sector_owners(sites: int, world: int):
    """{(n_up, n_down): rank}: longest-processing-time assignment by full
    sector dimension (ties broken by the reference's sector order)."""
    sectors = [(nu, nd) for nu in range(sites + 1) for nd in range(sites + 1)]
    order = sorted(sectors, key=lambda s: (-comb(sites, s[0]) * comb(sites, s[1]), s))
    heap = [(0, r) for r in range(world)]
    owner = {}
    for s in order:
        load, r = heapq.heappop(heap)
        owner[s] = r
        heapq.heappush(heap, (load + comb(sites, s[0]) * comb(sites, s[1]), r))
    return owner


def merge_accumulators(emin, z, ns, n2, betas, allreduce_min, allreduce_sum):
    """Combine per-rank accumulators ([nbeta][nmu] arrays) given the two
    collectives; returns the global (emin, z, ns, n2)."""
    emin = np.asarray(emin, np.float64)
    g = allreduce_min(emin.copy())
    b = np.asarray(betas, np.float64).reshape(-1, 1)
    with np.errstate(invalid="ignore", over="ignore"):
        scale = np.where(np.isfinite(emin), np.exp(-b * (emin - g)), 0.0)
    sums = np.stack([np.asarray(z) * scale, np.asarray(ns) * scale, np.asarray(n2) * scale])
    sums = allreduce_sum(sums)
    return g, sums[0], sums[1], sums[2]


def torch_collectives(device=None):
    """MIN / SUM all-reduce of numpy arrays over the default process group
    (NCCL on GPU tensors, or gloo on CPU tensors)."""
    import torch
    import torch.distributed as dist

    def run(a, op):
        t = torch.from_numpy(np.ascontiguousarray(a, np.float64))
        if device is not None:
            t = t.to(device)
        dist.all_reduce(t, op=op)
        return t.cpu().numpy()

    return (lambda a: run(a, dist.ReduceOp.MIN)), (lambda a: run(a, dist.ReduceOp.SUM))


def finalize(betas, sites, emin, z, ns, n2):
    """Observables from accumulators (main.cpp:1770-1788)."""
    b = np.asarray(betas, np.float64).reshape(-1, 1)
    mean = ns / z
    chi = np.maximum(0.0, (n2 / z - mean * mean) / sites)
    return {"n": mean / sites, "charge_correlation": chi, "compressibility": b * chi, "partition_like": z,
            "log_partition": np.log(z) - b * emin}


def shard_accumulators(model: Model, betas, mu, opts: RunOpts | None = None, ed: bool = False, rank: int = 0,
                       world: int = 1):
    """(emin, z, ns, n2) of this rank's sectors, run on device opts.device."""
    opts = opts or RunOpts()
    owner = sector_owners(model.sites, world)
    eng = Engine(model, opts)
    try:
        eng.thermo_configure(betas, mu)
        for nu in range(model.sites + 1):
            for nd in range(model.sites + 1):
                if owner[(nu, nd)] != rank:
                    continue
                info = eng.sector_prepare(nu, nd)
                blocks = [(k % model.lx, k // model.lx) for k, d in enumerate(info.block_dims) if d > 0]
                exact = [b for b in blocks
                         if ed or info.block_dims[b[1] * model.lx + b[0]] <= opts.exact_block_threshold]
                eng.blocks_exact_batched(exact)
                eng.blocks_ftlm_batched([b for b in blocks if b not in exact])
                for b in blocks:
                    eng.thermo_accumulate_block(*b)
        return eng.thermo_read()
    finally:
        eng.close()


def run_curve_sharded(model: Model, betas, mu, opts: RunOpts | None = None, ed: bool = False, rank: int = 0,
                      world: int = 1, collectives=None):
    """This rank's share of the curve, merged over the process group; every
    rank returns the same finalised observables."""
    emin, z, ns, n2 = shard_accumulators(model, betas, mu, opts, ed, rank, world)
    if world > 1:
        mn, sm = collectives or torch_collectives()
        emin, z, ns, n2 = merge_accumulators(emin, z, ns, n2, betas, mn, sm)
    return finalize(betas, model.sites, emin, z, ns, n2)
