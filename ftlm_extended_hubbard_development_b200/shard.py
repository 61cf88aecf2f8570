"""One n(mu) curve over several GPUs: momentum blocks sharded over ranks.

The (N_up, N_down, k) blocks of a curve are independent; each rank runs its
share on its own GPU (one process per GPU, torch.distributed for the
plumbing) and keeps the grand-canonical accumulators (emin, z, <N>z,
<N^2>z)[beta][mu] of its blocks on the device. The only exchange is at the
end: the minimum of emin over ranks (MIN all-reduce), each rank's sums
rescaled to that minimum by exp(-beta (emin_r - emin)), and one SUM
all-reduce of the three sums, 3 * nbeta * nmu doubles, which is the
reference's rescale rule (main.cpp:1172-1219) applied once per rank instead
of once per block.

Blocks are assigned longest-processing-time first to the least-loaded rank
(ties in the reference's block order, main.cpp:1519-1534), with cost
D*R*L*h (FTLM: R random vectors x L Lanczos steps of an H*V over h hops per
row) or D^3 (dense exact diagonalisation), so one sector's k-blocks spread
over ranks and the ranks finish together. A rank prepares only the sectors
it owns blocks of and runs its blocks in the reference's order. Block
dimensions come from character counting on the host (block_dims_host), so
every rank computes the same plan without a GPU or a collective.
"""
from __future__ import annotations

import cmath
import heapq
from itertools import combinations
from math import comb

import numpy as np

from .engine import Engine, Model, RunOpts


def _translate(bits: int, dx: int, dy: int, lx: int, ly: int):
    """Translation of a spin word by (dx, dy) with the parity of reordering
    its creation operators into ascending site order (main.cpp:579-613):
    rows rotate by dx, costing w*(n-w) transpositions per row with w of its n
    particles wrapping; then the word rotates by dy rows, costing w*(n-w)."""
    n = lx * ly
    par = 0
    if dx:
        out = 0
        for y in range(ly):
            row = (bits >> (y * lx)) & ((1 << lx) - 1)
            ny = bin(row).count("1")
            wrap = bin(row >> (lx - dx)).count("1")
            par += wrap * (ny - wrap)
            row = ((row << dx) | (row >> (lx - dx))) & ((1 << lx) - 1)
            out |= row << (y * lx)
        bits = out
    if dy:
        sh = dy * lx
        top = bits >> (n - sh)
        w = bin(top).count("1")
        par += w * (bin(bits).count("1") - w)
        bits = ((bits << sh) | top) & ((1 << n) - 1)
    return bits, par & 1


def _fixed_trace(lx: int, ly: int, n_part: int, dx: int, dy: int) -> int:
    """Trace of the translation T_(dx,dy) on the n_part-particle space of one
    spin: sum over words it maps onto themselves of its sign."""
    n = lx * ly
    if dx == 0 and dy == 0:
        return comb(n, n_part)
    # a fixed word is a union of cycles of the site permutation
    perm = [((s % lx + dx) % lx) + ((s // lx + dy) % ly) * lx for s in range(n)]
    seen, cycles = set(), []
    for s in range(n):
        if s not in seen:
            cyc, t = [], s
            while t not in seen:
                seen.add(t)
                cyc.append(t)
                t = perm[t]
            cycles.append(cyc)
    clen = len(cycles[0])
    if n_part % clen:
        return 0
    tr = 0
    for pick in combinations(range(len(cycles)), n_part // clen):
        word = 0
        for c in pick:
            for t in cycles[c]:
                word |= 1 << t
        img, par = _translate(word, dx, dy, lx, ly)
        assert img == word
        tr += -1 if par else 1
    return tr


def block_dims_host(lx: int, ly: int, n_up: int, n_dn: int):
    """Dimension of every momentum block k = my*lx + mx of sector
    (n_up, n_dn): the multiplicity of the character e^{ik.s} in the signed
    translation representation, (1/N) sum_s e^{-ik.s} tr_up(T_s) tr_dn(T_s)
    (a translation acts on both spin words, its sign is the product). Equals
    the number of orbits the reference finds active (main.cpp:745-766)."""
    n = lx * ly
    tr = {}
    for dy in range(ly):
        for dx in range(lx):
            tr[(dx, dy)] = _fixed_trace(lx, ly, n_up, dx, dy) * _fixed_trace(lx, ly, n_dn, dx, dy)
    dims = []
    for my in range(ly):
        for mx in range(lx):
            acc = 0j
            for (dx, dy), t in tr.items():
                if t:
                    acc += t * cmath.exp(-2j * cmath.pi * (mx * dx / lx + my * dy / ly))
            d = acc.real / n
            dims.append(int(round(d)))
    return dims


def block_cost(dim: int, exact: bool, samples: int, steps: int, hops_per_row: float) -> float:
    """Work of one block in complex multiply-adds: dense Householder
    tridiagonalisation (~(4/3) D^3) for exact blocks, R x min(L, D) H*V
    sweeps of D rows x (h + 1) terms for FTLM blocks."""
    if exact:
        return 4.0 / 3.0 * float(dim) ** 3
    return float(dim) * samples * min(steps, dim) * (hops_per_row + 1.0)


def block_owners(model: Model, world: int, opts: RunOpts | None = None, ed: bool = False, sectors=None,
                 dims=None):
    """{(n_up, n_down, mx, my): rank} over the non-empty blocks of the given
    sectors (default: all): longest-processing-time assignment by block_cost,
    ties in the reference's block order. dims maps a sector to its block
    dimensions (default: block_dims_host)."""
    opts = opts or RunOpts()
    sites = model.sites
    secs = sectors if sectors is not None else [(a, b) for a in range(sites + 1) for b in range(sites + 1)]
    ndir = 4 + (4 if model.tp != 0.0 else 0)
    blocks = []
    for order, (nu, nd) in enumerate(secs):
        dd = dims[(nu, nd)] if dims is not None else block_dims_host(model.lx, model.ly, nu, nd)
        # mean open hops per row: each particle tries ndir neighbours, free with probability (N - n)/(N - 1)
        h = sum(ndir * p * (sites - p) / max(sites - 1, 1) for p in (nu, nd))
        for my in range(model.ly):
            for mx in range(model.lx):
                d = dd[my * model.lx + mx]
                if d <= 0:
                    continue
                exact = ed or d <= opts.exact_block_threshold
                c = block_cost(d, exact, opts.samples, opts.lanczos_steps, h)
                blocks.append((-c, order, my, mx, nu, nd))
    blocks.sort()
    heap = [(0.0, r) for r in range(world)]
    owner = {}
    for negc, _, my, mx, nu, nd in blocks:
        load, r = heapq.heappop(heap)
        owner[(nu, nd, mx, my)] = r
        heapq.heappush(heap, (load - negc, r))
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
                       world: int = 1, owners=None):
    """(emin, z, ns, n2) of this rank's blocks, run on device opts.device."""
    opts = opts or RunOpts()
    owner = owners if owners is not None else block_owners(model, world, opts, ed)
    mine = {}
    for (nu, nd, mx, my), r in owner.items():
        if r == rank:
            mine.setdefault((nu, nd), set()).add((mx, my))
    eng = Engine(model, opts)
    try:
        eng.thermo_configure(betas, mu)
        eng.spectra_defer(True)  # as run_curve: the small blocks of all sectors solved together
        for nu in range(model.sites + 1):
            for nd in range(model.sites + 1):
                if (nu, nd) not in mine:
                    continue
                info = eng.sector_prepare(nu, nd)
                blocks = [(k % model.lx, k // model.lx) for k, d in enumerate(info.block_dims)
                          if d > 0 and (k % model.lx, k // model.lx) in mine[(nu, nd)]]
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
