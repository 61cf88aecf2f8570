"""Learned twist surrogate: per-block low-lying spectra as a function of twist.

Small FP32 MLPs (engine.Mlp, trained on the GPU by the library's own forward /
backward / Adam kernels) map a block's twist and quantum numbers
(phi_x, phi_y, N_up, N_down, k_x, k_y) to the block's `levels` lowest energy
levels and their trace weights. The training data are the spectra the GPU
engine itself produces on a uniform grid of twists. From the predicted levels
the surrogate proposes the n(mu) curve at any twist, e.g. on a dense grid for
the twist average. Plain FTLM (or ED) at held-out twists is its judge: when
the surrogate's n(mu) there is off by more than the threshold, the twist
average falls back to the engine's own twists.

Per block and twist the spectrum is split in two:
  * low part - the lowest `levels` levels: for an exactly diagonalised block
    its lowest eigenvalues one by one (weight 1 each); for an FTLM block the
    Ritz values merged across random vectors where they agree to `tol`, each
    with its summed trace weight (prefactor * FTLM weights). These are the
    network's targets, masked where the block has fewer levels;
  * tail - everything above, kept only as its partition sum per beta,
    log sum_i w_i exp(-beta e_i).
A proposal at twist phi takes the low part from the network and the tail of
the training twist nearest to phi; the tail's Boltzmann weight is small, so
truncating the spectrum costs little.

Inputs. A block's spectrum has period L in its own twist (the per-bond phase
is 2 pi phi / L) but not period 1: the gauge change that removes one flux
quantum moves the block to momentum k + N. The twist enters as sin/cos of the
per-bond phase and of its second harmonic; the quantum numbers enter one-hot,
which lets one network keep the blocks apart.

Targets and loss. The network predicts the deviation from the per-(block,
level) mean over the training twists, in units of the global spread of those
deviations. Each target is weighted by its importance for n(mu): the largest
Boltzmann probability the level reaches on the (beta, mu) grid, plus 1e-3, so
the network's capacity goes to the levels that set the curve.

Training: Adam, mini-batches of 512 (block, twist) rows, learning rate stepped
down over six stages; an ensemble of `members` networks (different seeds)
whose mean is the prediction.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass, replace

import numpy as np

from .engine import Engine, Mlp, Model, RunOpts
from .twist import combine_rows, curve_rows, uniform_grid

LEVELS = 16
HARMONICS = 2
MEMBERS = 3
# learning-rate factors of the six training stages (a stepped cosine decay)
LR_STAGES = (1.0, 0.8, 0.55, 0.3, 0.12, 0.03)


def n_features(model: Model) -> int:
    return 4 * HARMONICS + 2 * (model.sites + 1) + model.lx + model.ly


def block_features(phix, phiy, nup, ndn, mx, my, lx, ly):
    """Network input of one block at one twist: sin/cos of the per-bond twist
    phase and its harmonics, then one-hot N_up, N_down, k_x, k_y."""
    t = 2.0 * math.pi
    n = lx * ly
    f = []
    for h in range(1, HARMONICS + 1):
        f += [math.sin(h * t * phix / lx), math.cos(h * t * phix / lx), math.sin(h * t * phiy / ly),
              math.cos(h * t * phiy / ly)]
    oh = [0.0] * (2 * (n + 1) + lx + ly)
    oh[nup] = 1.0
    oh[n + 1 + ndn] = 1.0
    oh[2 * (n + 1) + mx] = 1.0
    oh[2 * (n + 1) + lx + my] = 1.0
    return f + oh


def reduce_spectrum(ev, w, pref, exact, levels=LEVELS, tol=1e-6):
    """Lowest `levels` levels (energy, trace weight, present mask) of a block
    and the remaining (energies, trace weights) as the tail. Exact blocks keep
    every eigenvalue as its own level (weight 1); FTLM Ritz values that agree
    to `tol` (relative) are merged and their weights summed."""
    ev = np.asarray(ev, np.float64)
    o = np.argsort(ev, kind="stable")
    e = ev[o]
    ww = np.ones_like(e) if exact or w is None else pref * np.asarray(w, np.float64)[o]
    E = np.zeros(levels)
    W = np.zeros(levels)
    M = np.zeros(levels)
    k = -1
    cut = len(e)
    for i in range(len(e)):
        if not exact and k >= 0 and abs(e[i] - E[k]) <= tol * max(1.0, abs(E[k])):
            W[k] += ww[i]
            continue
        if k + 1 >= levels:
            cut = i
            break
        k += 1
        E[k], W[k], M[k] = e[i], ww[i], 1.0
    return E, W, M, e[cut:], ww[cut:]


def tail_log_partition(e, w, betas):
    """log sum_i w_i exp(-beta e_i) per beta (-inf for an empty tail)."""
    out = np.full(len(betas), -np.inf)
    keep = w > 0
    e, w = e[keep], w[keep]
    if len(e):
        for ib, b in enumerate(betas):
            a = np.log(w) - b * e
            top = a.max()
            out[ib] = top + math.log(np.exp(a - top).sum())
    return out


@dataclass
class TwistData:
    """Engine output at one twist: per block (nup, ndn, mx, my, particles,
    E[levels], W[levels], M[levels], tail_logz[nbeta], exact) and the
    engine's own n(mu) curve (dict of [nbeta][nmu] arrays)."""
    phix: float
    phiy: float
    blocks: list
    curve: dict


def collect(model: Model, phix, phiy, betas, mu, opts: RunOpts, ed=False, levels=LEVELS) -> TwistData:
    """Every block's spectrum and the n(mu) curve at one twist, in the
    reference's (N_up, N_down, k) block order."""
    eng = Engine(replace(model, phix=float(phix), phiy=float(phiy)), opts)
    blocks = []
    try:
        eng.thermo_configure(betas, mu)
        n = model.sites
        for nu in range(n + 1):
            for nd in range(n + 1):
                info = eng.sector_prepare(nu, nd)
                ks = [(k % model.lx, k // model.lx) for k, d in enumerate(info.block_dims) if d > 0]
                exact = [b for b in ks
                         if ed or info.block_dims[b[1] * model.lx + b[0]] <= opts.exact_block_threshold]
                eng.blocks_exact_batched(exact)
                eng.blocks_ftlm_batched([b for b in ks if b not in exact])
                for b in ks:
                    is_exact = b in exact
                    ev, w, pref = eng.block_spectrum(b[0], b[1], exact=is_exact)
                    E, W, M, te, tw = reduce_spectrum(ev, w, pref, is_exact, levels)
                    blocks.append((nu, nd, b[0], b[1], nu + nd, E, W, M, tail_log_partition(te, tw, betas),
                                   is_exact))
                    eng.thermo_accumulate_block(*b)
        emin, z, ns, n2 = eng.thermo_read()
    finally:
        eng.close()
    bb = np.asarray(betas, np.float64).reshape(-1, 1)
    mean = ns / z
    chi = np.maximum(0.0, (n2 / z - mean * mean) / model.sites)
    curve = {"n": mean / model.sites, "charge_correlation": chi, "compressibility": bb * chi,
             "partition_like": z, "log_partition": np.log(z) - bb * emin}
    return TwistData(float(phix), float(phiy), blocks, curve)


def _shift(blocks, mu):
    shift = np.full(len(mu), np.inf)
    for b in blocks:
        if b[7].any():
            shift = np.minimum(shift, b[5][b[7] > 0].min() - mu * b[4])
    return shift


def _block_z(b, beta, mu, shift, ib):
    sel = b[7] > 0
    zz = (b[6][sel, None] * np.exp(-beta * (b[5][sel, None] - mu[None, :] * b[4] - shift[None, :]))).sum(0)
    if np.isfinite(b[8][ib]):
        zz = zz + np.exp(b[8][ib] + beta * (mu * b[4] + shift))
    return zz


def curve_from_blocks(blocks, sites, betas, mu):
    """n(mu) observables from per-block levels plus tail partition sums; the
    shifted log-sum-exp of the reference (main.cpp:1172-1219, 1770-1788)
    with one shift per mu, the lowest level of any block minus mu * N."""
    mu = np.asarray(mu, np.float64)
    shift = _shift(blocks, mu)
    out = {k: np.zeros((len(betas), len(mu))) for k in
           ("n", "charge_correlation", "compressibility", "partition_like", "log_partition")}
    for ib, beta in enumerate(betas):
        z = np.zeros(len(mu))
        n1 = np.zeros(len(mu))
        n2 = np.zeros(len(mu))
        for b in blocks:
            zz = _block_z(b, beta, mu, shift, ib)
            z += zz
            n1 += b[4] * zz
            n2 += b[4] * b[4] * zz
        mean = n1 / z
        chi = np.maximum(0.0, (n2 / z - mean * mean) / sites)
        out["n"][ib] = mean / sites
        out["charge_correlation"][ib] = chi
        out["compressibility"][ib] = beta * chi
        out["partition_like"][ib] = z
        out["log_partition"][ib] = np.log(z) - beta * shift
    return out


def level_importance(blocks, betas, mu):
    """Largest Boltzmann probability each level reaches on the (beta, mu)
    grid: [nblocks][levels]."""
    mu = np.asarray(mu, np.float64)
    shift = _shift(blocks, mu)
    imp = np.zeros((len(blocks), len(blocks[0][5])))
    for ib, beta in enumerate(betas):
        z = sum(_block_z(b, beta, mu, shift, ib) for b in blocks)
        for i, b in enumerate(blocks):
            p = b[6][:, None] * np.exp(-beta * (b[5][:, None] - mu[None, :] * b[4] - shift[None, :])) / z[None, :]
            imp[i] = np.maximum(imp[i], np.where(b[7] > 0, p.max(1), 0.0))
    return imp


def _dist2(a, b, wrap):
    d = [abs(x - y) for x, y in zip(a, b)]
    if wrap:
        d = [min(x, 1.0 - x) for x in d]
    return d[0] ** 2 + d[1] ** 2


class TwistSurrogate:
    """Ensemble of MLPs over (twist, block quantum numbers) -> lowest levels
    and weights of every block."""

    def __init__(self, model: Model, levels=LEVELS, width=128, depth=3, members=MEMBERS, seed=1234, device=0):
        self.model = model
        self.levels = levels
        self.nets = [Mlp(n_features(model), width, depth, 2 * levels, seed=seed + 7919 * i, device=device)
                     for i in range(members)]
        self.keys = None
        self.train_data = None

    def close(self):
        for n in self.nets:
            n.close()

    def features(self, phix, phiy):
        lx, ly = self.model.lx, self.model.ly
        return np.array([block_features(phix, phiy, k[0], k[1], k[2], k[3], lx, ly) for k in self.keys],
                        np.float32)

    def fit(self, data, betas, mu, epochs=600, batch=512, lr=1e-3, seed=7):
        """Train on the TwistData of the training twists; returns the loss
        history of the first member (one value per epoch)."""
        self.train_data = data
        self.keys = [b[:5] for b in data[0].blocks]
        self.exact = np.array([b[9] for b in data[0].blocks], bool)
        L = self.levels
        E = np.array([[b[5] for b in td.blocks] for td in data])
        W = np.array([[b[6] for b in td.blocks] for td in data])
        M = np.array([[b[7] for b in td.blocks] for td in data])
        imp = np.array([level_importance(td.blocks, betas, mu) for td in data])
        cnt = np.maximum(M.sum(0), 1.0)
        self.mask = (M.sum(0) > 0).astype(np.float64)  # a level present at any training twist
        self.e0 = (E * M).sum(0) / cnt
        self.w0 = (W * M).sum(0) / cnt
        rE = (E - self.e0) * M
        rW = (W - self.w0) * M
        fw = M * (~self.exact)[None, :, None]  # weights are learned for FTLM levels only
        self.se = max(float(np.sqrt((rE ** 2).sum() / max(M.sum(), 1.0))), 1e-6)
        self.sw = max(float(np.sqrt((rW ** 2 * fw).sum() / max(fw.sum(), 1.0))), 1e-6)
        X = np.concatenate([self.features(td.phix, td.phiy) for td in data])
        T = np.concatenate([rE / self.se, rW / self.sw], 2).reshape(-1, 2 * L).astype(np.float32)
        wgt = M * (1e-3 + imp)
        Mk = np.concatenate([wgt, wgt * (~self.exact)[None, :, None]], 2).reshape(-1, 2 * L).astype(np.float32)
        per = max(epochs // len(LR_STAGES), 1)
        hist = []
        for i, net in enumerate(self.nets):
            h = [net.train(X, T, Mk, per, batch, lr * f, seed + 31 * i + s) for s, f in enumerate(LR_STAGES)]
            if i == 0:
                hist = np.concatenate(h)
        return hist

    def nearest(self, phix, phiy, wrap=False):
        return min(self.train_data, key=lambda t: _dist2((t.phix, t.phiy), (phix, phiy), wrap))

    def predict_blocks(self, phix, phiy):
        """Blocks at a twist: predicted low levels, nearest training tail."""
        x = self.features(phix, phiy)
        y = sum(n.forward(x).astype(np.float64) for n in self.nets) / len(self.nets)
        L = self.levels
        E = self.e0 + y[:, :L] * self.se
        W = np.where(self.exact[:, None], 1.0, np.maximum(self.w0 + y[:, L:] * self.sw, 0.0))
        near = self.nearest(phix, phiy)
        return [(*k, E[i], W[i], self.mask[i], near.blocks[i][8], self.exact[i]) for i, k in enumerate(self.keys)]

    def curve(self, phix, phiy, betas, mu):
        return curve_from_blocks(self.predict_blocks(phix, phiy), self.model.sites, betas, mu)


def save_twist_data(path, data):
    """TwistData list to a compressed .npz: per twist the block quantum
    numbers, levels (energies FP64; weights, masks FP32), tail log-partitions
    and exact flags as arrays, and the engine curve."""
    arrs = {"n": np.array([len(data)])}
    for i, d in enumerate(data):
        b = d.blocks
        arrs[f"{i}/tw"] = np.array([d.phix, d.phiy])
        arrs[f"{i}/q"] = np.array([x[:5] for x in b], np.int16).reshape(-1, 5)
        arrs[f"{i}/E"] = np.array([x[5] for x in b], np.float64)
        arrs[f"{i}/W"] = np.array([x[6] for x in b], np.float64)
        arrs[f"{i}/M"] = np.array([x[7] for x in b], np.float32)
        arrs[f"{i}/T"] = np.array([x[8] for x in b], np.float64)
        arrs[f"{i}/X"] = np.array([x[9] for x in b], np.bool_)
        for k, v in d.curve.items():
            arrs[f"{i}/c/{k}"] = np.asarray(v)
    tmp = path + ".tmp.npz"
    np.savez_compressed(tmp, **arrs)
    import os
    os.replace(tmp, path)


def load_twist_data(path):
    z = np.load(path)
    out = []
    for i in range(int(z["n"][0])):
        q, E, W, M, T, X = (z[f"{i}/{k}"] for k in ("q", "E", "W", "M", "T", "X"))
        blocks = [(int(q[j, 0]), int(q[j, 1]), int(q[j, 2]), int(q[j, 3]), int(q[j, 4]), E[j], W[j],
                   M[j].astype(np.float64), T[j], bool(X[j])) for j in range(len(q))]
        curve = {k.split("/")[-1]: z[k] for k in z.files if k.startswith(f"{i}/c/")}
        tw = z[f"{i}/tw"]
        out.append(TwistData(float(tw[0]), float(tw[1]), blocks, curve))
    return out


def heldout_twists(count=8, seed=2024):
    """Held-out judge twists in [0, 1)^2 from a Philox generator of fixed seed."""
    g = np.random.Generator(np.random.Philox(seed))
    return [tuple(map(float, t)) for t in g.random((count, 2))]


def collect_grid(model: Model, betas, mu, opts: RunOpts, grid, ed=False, levels=LEVELS, train=None,
                 save_train=None, log=None):
    """Training spectra at the grid x grid twists in `uniform_grid` order.
    `train` holds spectra already collected at the first twists of that
    order (from `load_twist_data`); collection continues after them and,
    with `save_train`, rewrites the file after every twist, so a job cut
    off by a time limit loses at most one twist and the next job resumes."""
    pts = uniform_grid(grid)
    train = list(train or [])
    if len(train) > len(pts):
        raise ValueError(f"{len(train)} training twists given for a {grid}x{grid} grid")
    for td, (px, py) in zip(train, pts):
        if abs(td.phix - px) > 1e-12 or abs(td.phiy - py) > 1e-12:
            raise ValueError(f"training twist ({td.phix}, {td.phiy}) is not grid twist ({px}, {py})")
    t0 = time.perf_counter()
    for px, py in pts[len(train):]:
        train.append(collect(model, px, py, betas, mu, opts, ed, levels))
        if log:
            log(f"training twist {len(train)}/{len(pts)} ({px:.4f}, {py:.4f}) at {time.perf_counter() - t0:.1f} s")
        if save_train:
            save_twist_data(save_train, train)
    return train


def surrogate_twist_average(model: Model, betas, mu, opts: RunOpts, grid=6, heldout=8, dense=24,
                            threshold=0.01, ed=False, epochs=600, seed=2024, levels=LEVELS, members=MEMBERS,
                            device=0, log=None, judge_opts: RunOpts | None = None, train=None,
                            save_train=None):
    """Train on a grid x grid twist set, judge at `heldout` Philox twists with
    the engine, and average n(mu) over the surrogate's dense x dense grid when
    every judge passes (max |dn| <= threshold); otherwise average the
    engine's own curves at the training and held-out twists (fallback).

    Two budgets: the training spectra are computed with `opts` (the network's
    targets are each block's lowest levels, which converge from a few random
    vectors) and the judges with `judge_opts` (default: the same), the full
    FTLM budget the surrogate is held to."""
    opts = replace(opts, device=device)
    judge_opts = replace(judge_opts or opts, device=device)
    t0 = time.perf_counter()
    # training spectra given (a run can stop after collecting them) are the
    # first twists of the grid; the rest are collected here
    train = collect_grid(model, betas, mu, opts, grid, ed, levels, train, save_train, log)
    t1 = time.perf_counter()
    if log:
        log(f"training the surrogate on {len(train)} twists")
    sur = TwistSurrogate(model, levels=levels, members=members, device=device)
    hist = sur.fit(train, betas, mu, epochs=epochs)
    t2 = time.perf_counter()
    judges = []
    t_judge = t_pred = 0.0
    for px, py in heldout_twists(heldout, seed):
        ta = time.perf_counter()
        td = collect(model, px, py, betas, mu, judge_opts, ed, levels)
        tb = time.perf_counter()
        pred = sur.curve(px, py, betas, mu)
        t_judge += tb - ta
        t_pred += time.perf_counter() - tb
        near = sur.nearest(px, py, wrap=True)  # the curve without the network
        judges.append({"twist": (px, py), "curve": td.curve,
                       "err_surrogate": float(np.abs(pred["n"] - td.curve["n"]).max()),
                       "err_nearest_twist": float(np.abs(near.curve["n"] - td.curve["n"]).max())})
        if log:
            log(f"judge twist ({px:.4f}, {py:.4f}): engine {tb - ta:.1f} s, max|dn| surrogate "
                f"{judges[-1]['err_surrogate']:.5f}, nearest training twist {judges[-1]['err_nearest_twist']:.5f}")
    accepted = all(j["err_surrogate"] <= threshold for j in judges)
    rows = []
    if accepted:
        for px, py in uniform_grid(dense):
            rows += curve_rows(sur.curve(px, py, betas, mu), betas, mu)
        source = f"surrogate {dense}x{dense} grid"
    else:
        for td in train:
            rows += curve_rows(td.curve, betas, mu)
        for j in judges:
            rows += curve_rows(j["curve"], betas, mu)
        source = "engine twists (fallback)"
    grid_rows = []
    for td in train:
        grid_rows += curve_rows(td.curve, betas, mu)
    timing = {"engine_s_per_twist": (t1 - t0 + t_judge) / max(len(train) + len(judges), 1),
              "engine_s_per_training_twist": (t1 - t0) / max(len(train), 1),
              "engine_s_per_judge_twist": t_judge / max(len(judges), 1),
              "training_s": t2 - t1, "surrogate_s_per_twist": t_pred / max(len(judges), 1)}
    return {"average": combine_rows(rows, "observable-average"), "source": source, "accepted": accepted,
            "judges": judges, "loss_history": hist, "training_grid_average": combine_rows(grid_rows),
            "surrogate": sur, "train": train, "timing": timing}


def main(argv=None):
    """Command line: the surrogate twist average of one model, with a JSON
    summary (judges' errors, the nearest-twist baseline, timings) on stdout
    and the averaged curve as CSV (twist.py's columns)."""
    import argparse
    import json
    import sys

    from .engine import PREC_FP64, PREC_MIXED, START_PHILOX_PHASE, START_REF_GAUSSIAN, linspace
    from .twist import write_rows

    ap = argparse.ArgumentParser(description="Twist average of n(mu) with the learned surrogate")
    ap.add_argument("--lx", type=int, default=4)
    ap.add_argument("--ly", type=int, default=4)
    ap.add_argument("--tx", type=float, default=1.0)
    ap.add_argument("--ty", type=float, default=1.0)
    ap.add_argument("--tp", type=float, default=-0.25)
    ap.add_argument("--u", type=float, default=7.0)
    ap.add_argument("--v", type=float, default=1.0)
    ap.add_argument("--beta-list", default="5")
    ap.add_argument("--mu-min", type=float, default=-3.0)
    ap.add_argument("--mu-max", type=float, default=4.0)
    ap.add_argument("--mu-points", type=int, default=141)
    ap.add_argument("--samples", type=int, default=128, help="random vectors of the training spectra")
    ap.add_argument("--lanczos-steps", type=int, default=80, help="Lanczos steps of the training spectra")
    ap.add_argument("--judge-samples", type=int, default=0, help="random vectors of the judges (default --samples)")
    ap.add_argument("--judge-steps", type=int, default=0, help="Lanczos steps of the judges (default --lanczos-steps)")
    ap.add_argument("--exact-block-threshold", type=int, default=256)
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="mixed")
    ap.add_argument("--start-vector", choices=["ref-gaussian", "philox-phase"], default="philox-phase")
    ap.add_argument("--ed", action="store_true", help="diagonalise every block exactly")
    ap.add_argument("--grid", type=int, default=6)
    ap.add_argument("--heldout", type=int, default=8)
    ap.add_argument("--dense", type=int, default=24)
    ap.add_argument("--threshold", type=float, default=0.01)
    ap.add_argument("--epochs", type=int, default=600)
    ap.add_argument("--members", type=int, default=MEMBERS)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--output", help="CSV of the twist-averaged curve")
    ap.add_argument("--save-train", help="write the training spectra here as they are collected")
    ap.add_argument("--load-train", help="training spectra from an earlier --save-train, the first twists of the grid "
                    "(collection continues after them)")
    ap.add_argument("--collect-only", action="store_true", help="stop after collecting the training spectra")
    a = ap.parse_args(argv)
    model = Model(lx=a.lx, ly=a.ly, tx=a.tx, ty=a.ty, tp=a.tp, u=a.u, v=a.v)
    betas = [float(b) for b in a.beta_list.split(",")]
    mu = linspace(a.mu_min, a.mu_max, a.mu_points)
    opts = RunOpts(samples=a.samples, lanczos_steps=a.lanczos_steps, exact_block_threshold=a.exact_block_threshold,
                   precision=PREC_MIXED if a.precision == "mixed" else PREC_FP64,
                   start_vector=START_PHILOX_PHASE if a.start_vector == "philox-phase" else START_REF_GAUSSIAN)
    jopts = replace(opts, samples=a.judge_samples or a.samples, lanczos_steps=a.judge_steps or a.lanczos_steps)
    log = lambda m: print(m, file=sys.stderr, flush=True)  # noqa: E731
    train = load_twist_data(a.load_train) if a.load_train else None
    if a.collect_only:
        t0 = time.perf_counter()
        have = len(train or [])
        train = collect_grid(model, betas, mu, replace(opts, device=a.device), a.grid, a.ed, train=train,
                             save_train=a.save_train, log=log)
        new = len(train) - have
        print(json.dumps({"collected": len(train), "new": new, "seconds": time.perf_counter() - t0,
                          "s_per_twist": (time.perf_counter() - t0) / max(new, 1)}))
        return 0
    res = surrogate_twist_average(model, betas, mu, opts, grid=a.grid, heldout=a.heldout, dense=a.dense,
                                  threshold=a.threshold, ed=a.ed, epochs=a.epochs, members=a.members,
                                  device=a.device, log=log, judge_opts=jopts, train=train,
                                  save_train=a.save_train)
    es = np.array([j["err_surrogate"] for j in res["judges"]])
    en = np.array([j["err_nearest_twist"] for j in res["judges"]])
    g = np.array([r["n"] for r in res["training_grid_average"]])
    avg = np.array([r["n"] for r in res["average"]])
    print(json.dumps({"model": model.__dict__, "betas": betas, "mu": [a.mu_min, a.mu_max, a.mu_points],
                      "samples": a.samples, "lanczos_steps": a.lanczos_steps,
                      "judge_samples": jopts.samples, "judge_steps": jopts.lanczos_steps, "ed": a.ed, "grid": a.grid,
                      "heldout": a.heldout, "threshold": a.threshold, "accepted": res["accepted"],
                      "source": res["source"], "judge_max_dn_surrogate": es.round(6).tolist(),
                      "judge_max_dn_nearest_twist": en.round(6).tolist(),
                      "loss_first_last": [float(res["loss_history"][0]), float(res["loss_history"][-1])],
                      "max_dn_average_vs_training_grid_average": float(np.abs(avg - g).max()),
                      **res["timing"]}))
    if a.output:
        write_rows(a.output, res["average"])
    res["surrogate"].close()
    return 0


if __name__ == "__main__":
    import sys
    sys.exit(main())
