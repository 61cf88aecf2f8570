#!/usr/bin/env python3
"""Benchmark of the B200 FTLM engine: H*v HBM GB/s on the 4x4 U=7 production block.

Workload (one step): the largest momentum block of the batched 4x4 production
curve (lx=ly=4, tx=ty=1, t'=0, U=7, V=0; sector N_up=N_down=8, k=(0,0),
dim ~1.04e7): FTLM with 128 random vectors x 80 Lanczos steps run as one
multi-vector sweep per step, mixed precision (FP32 complex vectors and H*V,
FP64 dot products / norms / alpha-beta / tridiagonal), Philox uniform-phase
start vectors; the Ritz values and weights of all 128 samples are produced on
the device. With --gpus N each rank runs its own k-block of the same sector
(weak scaling); there is no data-path collective.

Metric: H*v HBM GB/s = algorithmic H*V bytes / time, with bytes per H*V
launch D*[nvec*s*(1+h_nz) + nvec*s + m] (s = 8 B per FP32 complex, h_nz =
nonzero-amplitude hops per row, m = 8 B per row). `value` divides by the
whole step (Lanczos updates, reductions, tridiagonal solve included);
`roofline.achieved` divides by the H*V kernel's own CUDA-event time.

With --workload 6x3 the block is the large bandwidth-bound one instead: 6x3
torus (18 sites), t'=0.2, U=8, V=1.5, twist (0.25, 0.5), sector
N_up=N_down=9, k=(0,0), dim ~1.31e8, 16 vectors x 100 steps, mixed precision.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference] [--workload 4x4|6x3]
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "H*v HBM GB/s; sec per n(mu) curve, mixed vs FP64 GPU at |dn|<=1e-4"
# Block workloads (one bench step = the FTLM of one momentum block):
#  4x4: the largest block of the batched 4x4 production curve (the metric's
#       workload); 6x3: the large bandwidth-bound block, 6x3 half filling.
# `ref` is the bounded CPU sample of the reference's own apply_hamiltonian:
# the same couplings on the largest sector of the lattice that the reference
# builds within seconds.
WORKLOADS = {
    "4x4": dict(model=dict(lx=4, ly=4, tx=1.0, ty=1.0, tp=0.0, phix=1.0, phiy=1.0, u=7.0, v=0.0),
                sector=(8, 8), samples=128, steps=80, betas=[2.857142857142857, 12.5], mu=(-3.0, 4.0, 281),
                name="4x4 U=7 t'=0", ref_sector=(4, 4)),
    "6x3": dict(model=dict(lx=6, ly=3, tx=1.0, ty=1.0, tp=0.2, phix=0.25, phiy=0.5, u=8.0, v=1.5),
                sector=(9, 9), samples=16, steps=100, betas=[10.0], mu=(-4.0, 8.0, 121),
                name="6x3 U=8 V=1.5 t'=0.2 twist (0.25,0.5)", ref_sector=(3, 4)),
}
WL = "4x4"
MODEL = WORKLOADS[WL]["model"]
SECTOR = WORKLOADS[WL]["sector"]
SAMPLES, STEPS = WORKLOADS[WL]["samples"], WORKLOADS[WL]["steps"]
FALLBACK_HBM = 6650.0


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def hbm_peak():
    p = os.path.join(HERE, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def ncu_traffic(args, split):
    """DRAM bytes per H*V application of the bench block, from the committed
    ncu captures (profiles/traffic.json; each entry names its capture and how
    it scales to the bench block); None for any other workload."""
    if SECTOR != WORKLOADS[WL]["sector"] or STEPS <= 0 or args.precision != "mixed" or args.batch != 0:
        return None
    key = ("split_" if split else "fly_") + {"4x4": "4x4_sector88_nv128_mixed", "6x3": "6x3_sector99_nv16_mixed"}[WL]
    try:
        with open(os.path.join(HERE, "profiles", "traffic.json")) as f:
            return float(json.load(f)[key]["dram_bytes_per_launch"])
    except (OSError, KeyError, ValueError):
        return None


def cpu_baseline(threads: int, sweeps: int = 2, skip: int = 0):
    """The reference's own apply_hamiltonian (oracle/_ref/ref_bench, compiled
    from the reference sources) on a bounded sample: same lattice and
    couplings, the largest sector it builds in seconds (4x4: (4,4), ~15 s;
    6x3: (3,4), ~15 s), 16 vectors per sweep; the first `skip` sweeps are
    warm-up."""
    exe = os.path.join(HERE, "oracle", "_ref", "ref_bench")
    if not os.path.exists(exe):
        return None
    w = WORKLOADS[WL]
    m = w["model"]
    nu, nd = w["ref_sector"]
    flags = []
    for k in ("lx", "ly", "tx", "ty", "tp", "phix", "phiy", "u", "v"):
        flags += ["--" + k, repr(m[k]) if isinstance(m[k], float) else str(m[k])]
    args = [exe, "hv", str(nu), str(nd), "0", "0", "16", str(sweeps + skip), "--"] + flags + [
        "--threads", str(threads), "--max-sector-dim", "100000000"]
    r = subprocess.run(args, capture_output=True, text=True, env={**os.environ, "OPENBLAS_NUM_THREADS": "1"})
    if r.returncode != 0:
        return None
    j = json.loads(r.stdout.strip().splitlines()[-1])
    D, nz, nv = j["dim"], j["nnz_nonzero"], j["nvec"]
    per = j["sweep_seconds"][skip:]
    bytes_per_sweep = D * nv * 16 * 2 + nz * nv * 16 + D * 8
    gbs = bytes_per_sweep * len(per) / sum(per) / 1e9
    return {"value": gbs, "unit": "GB/s", "cores": j["threads"], "kind": "reference",
            "per_sweep_gbs": [bytes_per_sweep / s / 1e9 for s in per],
            "dim": D, "vectors": nv, "nonzero_hops": nz,
            "hop_vector_products_per_s": nz * nv * len(per) / sum(per),
            "sample": (f"reference apply_hamiltonian (FP64 CSR SpMV, OpenMP over vectors) on {w['name']} "
                       f"sector ({nu},{nd}) k=(0,0), dim {D}, {nv} vectors x {len(per)} timed sweeps "
                       f"({sum(per):.3f} s); the GPU block's sector {w['sector']} is beyond the reference "
                       f"on this host (4x4 (8,8): ~15 min and ~30 GB to build; 6x3 (9,9): its 32-bit "
                       f"CSR overflows and it needs ~300 GB)")}


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    base = cpu_baseline(threads, sweeps=max(args.steps, 1), skip=args.warmup)
    if base is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ref_bench not built (make -C oracle ref)"}))
        return
    v = base["value"]
    line = {"metric": METRIC, "value": v, "unit": "GB/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "c128", "data": "synthetic (model-defined Hilbert space, Gaussian vectors)",
            "impl": "reference",
            "config": {"workload": (f"{WORKLOADS[WL]['name']} H*V of the reference's apply_hamiltonian "
                                    f"(FP64 CSR SpMV, OpenMP over vectors, {base['cores']} host threads) on "
                                    f"sector {WORKLOADS[WL]['ref_sector']} k=(0,0), dim {base['dim']}, "
                                    f"{base['vectors']} vectors per sweep: the largest block of this lattice "
                                    f"the reference builds within a bench step (the GPU arm's sector "
                                    f"{WORKLOADS[WL]['sector']} is beyond it on this host)"),
                       "lattice": WL, "sector": list(WORKLOADS[WL]["ref_sector"]), "k": [0, 0], "dim": base["dim"],
                       "vectors_per_sweep": base["vectors"], "precision": "fp64", "threads": base["cores"]},
            "rate": {"hop_vector_products_per_s": base["hop_vector_products_per_s"],
                     "note": "nonzero off-diagonal hops x vectors per second: precision-neutral"},
            "cpu_baseline": {**base, "value": v},
            "e2e": {"value": v, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def run_ours(args):
    import numpy as np
    import torch
    import ftlm_extended_hubbard_development_b200 as pkg

    ws, rank, local = dist_env()
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl" if torch.cuda.is_available() else "gloo",
                                timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)
    model = pkg.Model(**MODEL)
    prec = pkg.engine.PREC_MIXED if args.precision == "mixed" else pkg.engine.PREC_FP64
    opts = pkg.RunOpts(samples=SAMPLES, lanczos_steps=STEPS, exact_block_threshold=256,
                       precision=prec, start_vector=pkg.engine.START_PHILOX_PHASE,
                       batch_vectors=args.batch, device=local)
    eng = pkg.Engine(model, opts)
    info = eng.sector_prepare(*SECTOR)
    k = rank % len(info.block_dims)
    mx, my = k % model.lx, k // model.lx
    dim = info.block_dims[k]

    def barrier():
        if ws > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        eng.spectra_reset()
        eng.block_spectrum(mx, my, fetch=False)
    eng.profile(True)
    eng.profile_reset()
    barrier()
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            eng.spectra_reset()
            eng.block_spectrum(mx, my, fetch=False)
        barrier()
    prof = eng.profile()
    dev_s = prof["block_ms"] / 1e3
    t = torch.tensor([dev_s], dtype=torch.float64, device="cuda")
    b = torch.tensor([prof["hv_bytes"]], dtype=torch.float64, device="cuda")
    if ws > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        torch.distributed.all_reduce(b, op=torch.distributed.ReduceOp.SUM)
    dev_s_max, bytes_all = float(t.item()), float(b.item())
    value = bytes_all / dev_s_max / 1e9
    split = prof["hv_source"] == 2
    peak, peak_kind = hbm_peak()
    launches = max(prof["hv_launches"], 1)
    hv_s = prof["hv_ms"] / 1e3
    # Roofline bytes of the dominant kernel. The on-the-fly kernel gathers every
    # hop's row from HBM: the gather model D*[nv*s*(1+h_nz) + nv*s + 8]. The
    # split-spin sweeps gather only inside the L2-resident segment of the row
    # being processed, so their HBM bytes are the compulsory D*(2*nv*s + 8) per
    # sweep, two sweeps (both row orders) per H*V; the gather model over their
    # time is reported beside it as the L2-served rate.
    model_bytes = prof["hv_bytes"] / launches
    roof_bytes = (2.0 * prof["hv_min_bytes"] if split else prof["hv_bytes"]) / launches
    achieved = roof_bytes / (hv_s / launches) / 1e9
    bytes_per_launch = roof_bytes

    # e2e through the C ABI: tables from the model, spectrum and thermodynamic
    # sums read back to host buffers every step
    mu = pkg.linspace(*WORKLOADS[WL]["mu"])
    betas = np.array(WORKLOADS[WL]["betas"])
    eng.profile_reset()
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        eng.thermo_configure(betas, mu)
        eng.sector_prepare(*SECTOR)
        ev, w, pref = eng.block_spectrum(mx, my)
        eng.thermo_accumulate_block(mx, my)
        eng.thermo_read()
    barrier()
    e2e_s = time.perf_counter() - t0
    pe = eng.profile()
    e2e_t = torch.tensor([e2e_s], dtype=torch.float64, device="cuda")
    if ws > 1:
        torch.distributed.all_reduce(e2e_t, op=torch.distributed.ReduceOp.MAX)
    e2e_val = bytes_all / float(e2e_t.item()) / 1e9

    if rank == 0:
        base = cpu_baseline(os.cpu_count() or 1) if (ws == 1 and not args.no_cpu_baseline) else None
        line = {
            "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dev_s_max * 1e3 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "c64 vectors, f64 reductions" if prec == pkg.engine.PREC_MIXED else "c128",
            "data": "synthetic (model-defined Hilbert space; Philox uniform-phase start vectors)",
            "config": {"workload": (f"{WORKLOADS[WL]['name']} FTLM block, sector {SECTOR} k=({mx},{my}) "
                                    f"dim {dim}: {SAMPLES} vectors x {STEPS} Lanczos steps per step, "
                                    f"{args.precision}"),
                       "lattice": WL, "model": MODEL, "sector": list(SECTOR), "k": [mx, my], "dim": dim,
                       "samples": SAMPLES, "lanczos_steps": STEPS, "precision": args.precision,
                       "batch_vectors": args.batch or min(SAMPLES, 128),
                       "l2": "inputs larger than L2 (vector arrays of dim x vectors x 8 B each)",
                       "parallelism": f"weak: one k-block per rank x{ws}"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "kernel": (["k_hv (on-the-fly multi-vector H*V)", "k_hv_list (cached hop list)",
                                     "k_hv_stn x2 (split-spin segment sweeps on the class stencils, both "
                                     "row orders; k_hv_stn_rows at <= 4 chunks per row)"]
                                    [prof["hv_source"]] if prof["hv_source"] in (0, 1, 2) else "unknown"),
                         "kernel_variant": prof["hv_variant"],
                         "bytes_per_launch": bytes_per_launch,
                         "bytes_model": ("compulsory: 2 sweeps x D*(2*nv*s + 8)" if split else
                                         "gather model: D*[nv*s*(1+h_nz) + nv*s + 8]"),
                         "gather_model_bytes_per_launch": model_bytes,
                         "gather_model_gbs": model_bytes / (hv_s / launches) / 1e9,
                         "gather_model_frac": model_bytes / (hv_s / launches) / 1e9 / peak,
                         "traffic": ncu_traffic(args, split),
                         **({"l2_gather_gbs": prof["hv_hops"] * (8 if prec == pkg.engine.PREC_MIXED else 16)
                                             / hv_s / 1e9,
                             "note": ("split-spin sweeps: every gather is an L2 hit inside the segment being "
                                      "processed, so HBM carries only the compulsory bytes (ncu: 1.006x); the "
                                      "sweeps are bound by L2 gather latency and instruction issue (ncu on the "
                                      "4x4 (5,5) block: 61% issue, 50% of L2 throughput), "
                                      "profiles/k_hv_stn_4x4_sector55_nv128_mixed_full.md")} if split else {})},
            "rate": {"hop_vector_products_per_s": prof["hv_hops"] / dev_s,
                     "hv_kernel_hop_vector_products_per_s": prof["hv_hops"] / hv_s,
                     "note": "nonzero off-diagonal hops x vectors per second: precision-neutral"},
            "e2e": {"value": e2e_val, "unit": "GB/s",
                    "h2d_bytes_per_step": pe["h2d_bytes"] / args.steps,
                    "d2h_bytes_per_step": pe["d2h_bytes"] / args.steps},
            "gpu_launches": prof["kernel_launches"],
            "clocks": clk.summary(),
        }
        if base:
            line["cpu_baseline"] = base
        print(json.dumps(line))
    eng.close()
    if ws > 1:
        torch.distributed.destroy_process_group()


# n(mu) curve workloads (--curve): model, betas, mu grid, samples x steps
CURVES = {
    "config2": dict(model=dict(lx=4, ly=2, tx=1.0, ty=1.0, tp=0.0, phix=1.0, phiy=1.0, u=8.0, v=0.0),
                    betas=[20.0], mu=(-5.0, 15.0, 81), samples=32, steps=120, threshold=256,
                    name="4x2 U=8 beta=20, 32 vectors x 120 steps, mu [-5,15] x 81"),
    "config3": dict(model=dict(lx=4, ly=4, tx=1.0, ty=1.0, tp=0.0, phix=1.0, phiy=1.0, u=7.0, v=0.0),
                    betas=[2.857142857142857, 12.5], mu=(-3.0, 4.0, 281), samples=128, steps=80, threshold=256,
                    name="4x4 U=7 beta {2.857, 12.5}, 128 vectors x 80 steps, mu [-3,4] x 281"),
}
# The two GPU paths the curve metric compares. "plain": FP64 vectors, one
# random vector per sweep, every block on the sweep kernels with on-the-fly
# H*V; "batched": FP32 vectors with FP64 sums, all vectors of a block in one
# sweep, small blocks in one persistent launch, hop list where it pays.
PATHS = {
    "mixed_batched": dict(precision="mixed", batch=0, defer=True,
                          env={"FTLM_SMALL_BLOCKS": "1", "FTLM_HV_MODE": "auto"}),
    "fp64_batched": dict(precision="fp64", batch=0, defer=True,
                         env={"FTLM_SMALL_BLOCKS": "1", "FTLM_HV_MODE": "auto"}),
    "fp64_plain": dict(precision="fp64", batch=1, defer=False,
                       env={"FTLM_SMALL_BLOCKS": "0", "FTLM_HV_MODE": "fly"}),
}


def time_curve(pkg, cfg, path, sectors=None, samples=None, per_sector=None, per_sector_tables=None):
    """Wall time of one n(mu) curve through the C ABI (block order of the
    reference), or of the listed sectors only; returns (seconds, observables).
    per_sector (a dict) receives each sector's wall time (every engine call
    of a sector returns after its device work; so the batched paths solve
    their small blocks sector by sector there, not pooled over the curve);
    per_sector_tables receives the part of it spent in sector_prepare."""
    import numpy as np
    p = PATHS[path]
    os.environ.update(p["env"])
    model = pkg.Model(**cfg["model"])
    prec = pkg.engine.PREC_MIXED if p["precision"] == "mixed" else pkg.engine.PREC_FP64
    opts = pkg.RunOpts(samples=samples or cfg["samples"], lanczos_steps=cfg["steps"],
                       exact_block_threshold=cfg["threshold"], precision=prec,
                       start_vector=pkg.engine.START_PHILOX_PHASE, batch_vectors=p["batch"])
    mu = pkg.linspace(*cfg["mu"])
    eng = pkg.Engine(model, opts)
    try:
        t0 = time.perf_counter()
        eng.thermo_configure(cfg["betas"], mu)
        # batched paths: the small blocks of all sectors in one dense-solver and one Ritz launch
        eng.spectra_defer(p["defer"] and per_sector is None)
        n = model.sites
        for nu in range(n + 1):
            for nd in range(n + 1):
                if sectors is not None and (nu, nd) not in sectors:
                    continue
                ts = time.perf_counter()
                info = eng.sector_prepare(nu, nd)
                if per_sector_tables is not None:
                    per_sector_tables[(nu, nd)] = time.perf_counter() - ts
                blocks = [(k % model.lx, k // model.lx) for k, d in enumerate(info.block_dims) if d > 0]
                exact = [b for b in blocks if info.block_dims[b[1] * model.lx + b[0]] <= cfg["threshold"]]
                eng.blocks_exact_batched(exact)
                eng.blocks_ftlm_batched([b for b in blocks if b not in exact])
                for b in blocks:
                    eng.thermo_accumulate_block(*b)
                if per_sector is not None:
                    per_sector[(nu, nd)] = time.perf_counter() - ts
        emin, z, ns, n2 = eng.thermo_read()
        secs = time.perf_counter() - t0
    finally:
        eng.close()
    b = np.asarray(cfg["betas"], np.float64).reshape(-1, 1)
    return secs, {"n": ns / z / n, "log_partition": np.log(z) - b * emin}


def run_curve_reference(args):
    """--curve config2 --impl reference: the reference's own executable
    (compiled from its sources into oracle/_ref) on the config-2 curve with
    all host threads, wall time per curve. Config 3 is out of its reach
    (the (8,8) sector alone needs ~15 min and ~30 GB to build on the CPU)."""
    cfg = CURVES[args.curve]
    exe = os.path.join(HERE, "oracle", "_ref", "ftlm_n_vs_mu")
    if args.curve != "config2" or not os.path.exists(exe):
        why = "config3 exceeds the reference's CPU memory/time" if args.curve != "config2" else \
              "oracle/_ref/ftlm_n_vs_mu not built (make -C oracle ref)"
        print(json.dumps({"impl": "reference", "unavailable": why}))
        return
    m = cfg["model"]
    threads = os.cpu_count() or 1
    cmd = [exe, "--lx", str(m["lx"]), "--ly", str(m["ly"]), "--tx", repr(m["tx"]), "--ty", repr(m["ty"]),
           "--tp", repr(m["tp"]), "--u", repr(m["u"]), "--v", repr(m["v"]), "--beta", repr(cfg["betas"][0]),
           "--mu-min", repr(cfg["mu"][0]), "--mu-max", repr(cfg["mu"][1]), "--mu-count", str(cfg["mu"][2]),
           "--samples", str(cfg["samples"]), "--lanczos-steps", str(cfg["steps"]),
           "--exact-block-threshold", str(cfg["threshold"]), "--threads", str(threads)]
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        t0 = time.perf_counter()
        r = subprocess.run(cmd + ["--output", os.path.join(d, "n.csv")], capture_output=True, text=True)
        secs = time.perf_counter() - t0
    if r.returncode != 0:
        print(json.dumps({"impl": "reference", "unavailable": "reference run failed: " + r.stderr[-200:]}))
        return
    print(json.dumps({"metric": "sec per n(mu) curve", "value": secs, "unit": "s", "n_gpus": 0, "steps": 1,
                      "warmup": 0, "higher_is_better": False, "impl": "reference",
                      "config": {"workload": cfg["name"]},
                      "cpu_baseline": {"value": secs, "unit": "s", "cores": threads, "kind": "reference",
                                       "sample": "whole config-2 curve, reference ftlm_n_vs_mu (OpenMP)"},
                      "e2e": {"value": secs, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))


def run_curve_phases(args, pkg, cfg, reps=2):
    """--curve ... --phases: the mixed batched curve `reps` times in one
    process with the engine's profile counters on (CUDA events around each
    engine call, so slightly slower than the timed curve): host seconds per
    call kind and the device milliseconds of each phase, one JSON line per
    repetition; the first repetition pays the process's one-time costs."""
    p = PATHS["mixed_batched"]
    os.environ.update(p["env"])
    model = pkg.Model(**cfg["model"])
    opts = pkg.RunOpts(samples=cfg["samples"], lanczos_steps=cfg["steps"], exact_block_threshold=cfg["threshold"],
                       precision=pkg.engine.PREC_MIXED, start_vector=pkg.engine.START_PHILOX_PHASE, batch_vectors=0)
    mu = pkg.linspace(*cfg["mu"])
    keys = ("sector_ms", "dense_ms", "eig_ms", "block_ms", "small_ms", "thermo_ms", "kernel_launches")
    for rep in range(reps):
        split = dict.fromkeys(("sector_prepare", "exact", "ftlm", "thermo", "flush_and_read"), 0.0)
        with pkg.Engine(model, opts) as eng:
            eng.profile(True)
            eng.profile_reset()
            t0 = time.perf_counter()
            eng.thermo_configure(cfg["betas"], mu)
            eng.spectra_defer(True)
            for nu in range(model.sites + 1):
                for nd in range(model.sites + 1):
                    ta = time.perf_counter()
                    info = eng.sector_prepare(nu, nd)
                    tb = time.perf_counter()
                    blocks = [(k % model.lx, k // model.lx) for k, d in enumerate(info.block_dims) if d > 0]
                    exact = [b for b in blocks if info.block_dims[b[1] * model.lx + b[0]] <= cfg["threshold"]]
                    eng.blocks_exact_batched(exact)
                    tc = time.perf_counter()
                    eng.blocks_ftlm_batched([b for b in blocks if b not in exact])
                    td = time.perf_counter()
                    for b in blocks:
                        eng.thermo_accumulate_block(*b)
                    te = time.perf_counter()
                    split["sector_prepare"] += tb - ta
                    split["exact"] += tc - tb
                    split["ftlm"] += td - tc
                    split["thermo"] += te - td
            tf = time.perf_counter()
            eng.thermo_read()  # solves the pooled blocks, then the queued sums
            split["flush_and_read"] = time.perf_counter() - tf
            total = time.perf_counter() - t0
            prof = eng.profile()
        print(json.dumps({"rep": rep, "workload": cfg["name"], "total_s": total, "host_split_s": split,
                          "profile": {k: prof[k] for k in keys}}))


def run_curve_per_sector(args, pkg, cfg):
    """Seconds per n(mu) curve with every sector measured: the mixed batched
    curve at its full vector count, the FP64 plain path over every sector at
    --plain-samples vectors (one sweep per vector, so its time is that many
    vectors' worth; scaled to the full count per sector), and |dn|,
    |d log Z| of mixed against FP64 batched over the whole curve with the
    same --dn-samples Philox start vectors on both. Per-sector table to
    --table (JSON). A sector's plain time is scaled as tables + (rest) x
    vectors / --plain-samples: the sector tables are built once whatever the
    vector count. --mixed-seconds S takes the mixed curve's time from an
    earlier whole-curve run instead of measuring it (no per-sector mixed
    column then); --dn-samples -1 skips the |dn| curves."""
    import numpy as np
    S = cfg["samples"]
    ps = args.plain_samples or 1
    ds = args.dn_samples or 8
    t_mix, t_plain, t_tab = {}, {}, {}
    with ClockSampler(0) as clk:
        if args.mixed_seconds > 0:
            tm = args.mixed_seconds
        else:
            tm, _ = time_curve(pkg, cfg, "mixed_batched", per_sector=t_mix)
        tp, _ = time_curve(pkg, cfg, "fp64_plain", samples=ps, per_sector=t_plain, per_sector_tables=t_tab)
        if ds > 0:
            _, cm = time_curve(pkg, cfg, "mixed_batched", samples=ds)
            _, cb = time_curve(pkg, cfg, "fp64_batched", samples=ds)
    rows = []
    plain_total = 0.0
    for sec in sorted(t_plain):
        scaled = t_tab[sec] + (t_plain[sec] - t_tab[sec]) * S / ps
        plain_total += scaled
        rows.append({"sector": list(sec), "mixed_batched_s": t_mix.get(sec), "fp64_plain_s_measured": t_plain[sec],
                     "fp64_plain_tables_s": t_tab[sec], "fp64_plain_s_scaled": scaled})
    line = {"metric": "sec per n(mu) curve", "value": tm, "unit": "s", "n_gpus": 1, "steps": 1, "warmup": 0,
            "higher_is_better": False, "scaling": "none", "vs_baseline": None,
            "dtype": "c64 vectors, f64 reductions", "data": "synthetic (model-defined; Philox start vectors)",
            "config": {"workload": cfg["name"], **{k: v for k, v in cfg.items() if k != "name"}},
            "curve": {"mixed_batched_s": tm,
                      "mixed_batched_kind": ("given (--mixed-seconds, an earlier whole-curve run)"
                                             if args.mixed_seconds > 0 else "measured"),
                      "fp64_plain_s": plain_total,
                      "fp64_plain_kind": (f"measured on every sector at {ps} of {S} vectors; per sector tables + "
                                          f"rest x {S}/{ps}"),
                      "fp64_plain_s_at_measured_vectors": tp,
                      "speedup_mixed_batched_vs_fp64_plain": plain_total / tm},
            "clocks": clk.summary()}
    if ds > 0:
        line["curve"].update({
            "dn_max_mixed_vs_fp64": float(np.abs(cm["n"] - cb["n"]).max()),
            "dlogz_max_mixed_vs_fp64": float(np.abs(cm["log_partition"] - cb["log_partition"]).max()),
            "dn_scope": f"whole curve, mixed vs FP64 batched, both with the same {ds} Philox vectors"})
    if args.table:
        with open(args.table, "w") as f:
            json.dump({"line": line, "sectors": rows}, f, indent=1)
    print(json.dumps(line))


def run_curve_mode(args):
    """--curve: seconds per n(mu) curve of the mixed batched path and of the
    FP64 plain path, and |dn|, |d log Z| of mixed against FP64 with the same
    Philox start vectors. With --plain-sectors the FP64 runs cover only those
    sectors (the plain one with --plain-samples vectors; its time scales with
    the vector count since each vector is its own sweep), the mixed curve is
    still measured whole, and the FP64 curve times are extrapolated by the
    FP64/mixed time ratios measured on exactly that work; |dn| is then the
    difference of the grand-canonical sums over those sectors."""
    import numpy as np
    import ftlm_extended_hubbard_development_b200 as pkg
    cfg = CURVES[args.curve]
    S = cfg["samples"]
    if args.phases:
        run_curve_phases(args, pkg, cfg)
        return
    if args.per_sector:
        run_curve_per_sector(args, pkg, cfg)
        return
    with ClockSampler(0) as clk:
        t_mixed, c_mixed = time_curve(pkg, cfg, "mixed_batched")
        if args.plain_sectors:
            secs = [tuple(int(v) for v in x.split(",")) for x in args.plain_sectors.split(";")]
            ns = args.plain_samples or S
            tm, cm = time_curve(pkg, cfg, "mixed_batched", secs)
            tb, cb = time_curve(pkg, cfg, "fp64_batched", secs)
            tp, _ = time_curve(pkg, cfg, "fp64_plain", secs, ns)
            tp_all = tp * S / ns
            res = {"fp64_batched_s": t_mixed * tb / tm, "fp64_plain_s": t_mixed * tp_all / tm,
                   "fp64_kind": "extrapolated",
                   "fp64_basis": {"sectors": secs, "mixed_batched_s": tm, "fp64_batched_s": tb,
                                  "fp64_plain_s": tp, "fp64_plain_samples": ns,
                                  "fp64_plain_s_scaled_to_all_samples": tp_all},
                   "dn_scope": "grand-canonical sums over the listed sectors"}
        else:
            tb, cb = time_curve(pkg, cfg, "fp64_batched")
            tp, cp = time_curve(pkg, cfg, "fp64_plain")
            cm = c_mixed
            res = {"fp64_batched_s": tb, "fp64_plain_s": tp, "fp64_kind": "measured", "dn_scope": "whole curve",
                   "dn_max_plain_vs_batched_fp64": float(np.abs(cp["n"] - cb["n"]).max())}
    res["dn_max_mixed_vs_fp64"] = float(np.abs(cm["n"] - cb["n"]).max())
    res["dlogz_max_mixed_vs_fp64"] = float(np.abs(cm["log_partition"] - cb["log_partition"]).max())
    res["speedup_mixed_batched_vs_fp64_plain"] = res["fp64_plain_s"] / t_mixed
    line = {"metric": "sec per n(mu) curve", "value": t_mixed, "unit": "s", "n_gpus": 1, "steps": 1, "warmup": 0,
            "higher_is_better": False, "scaling": "none", "vs_baseline": None,
            "dtype": "c64 vectors, f64 reductions", "data": "synthetic (model-defined; Philox start vectors)",
            "config": {"workload": cfg["name"], **{k: v for k, v in cfg.items() if k != "name"}},
            "curve": {"mixed_batched_s": t_mixed, **res}, "clocks": clk.summary()}
    print(json.dumps(line))


def main():
    global SECTOR, STEPS, WL, MODEL, SAMPLES
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", choices=["mixed", "fp64"], default="mixed")
    ap.add_argument("--batch", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="4x4",
                    help="4x4: 4x4 U=7 (8,8) block, 128 x 80 (default); 6x3: 6x3 (9,9) block, 16 x 100")
    ap.add_argument("--sector", default="", help="N_up,N_down of another sector of the lattice (profiling cases)")
    ap.add_argument("--lanczos-steps", type=int, default=0)
    ap.add_argument("--curve", choices=sorted(CURVES), help="time whole n(mu) curves instead")
    ap.add_argument("--plain-sectors", default="", help="'nu,nd;nu,nd': run the FP64 plain path on these only")
    ap.add_argument("--plain-samples", type=int, default=0)
    ap.add_argument("--per-sector", action="store_true",
                    help="--curve: measure every sector (plain path at --plain-samples vectors)")
    ap.add_argument("--dn-samples", type=int, default=0,
                    help="--per-sector: vectors of the |dn| curves (default 8; -1 skips them)")
    ap.add_argument("--mixed-seconds", type=float, default=0.0,
                    help="--per-sector: the mixed curve's seconds from an earlier whole-curve run (skips it)")
    ap.add_argument("--phases", action="store_true",
                    help="--curve: per-phase breakdown of the mixed batched curve (profile counters on)")
    ap.add_argument("--table", default="", help="--per-sector: write the per-sector table here (JSON)")
    args = ap.parse_args()
    if args.curve:
        if args.impl == "reference":
            run_curve_reference(args)
        else:
            run_curve_mode(args)
        return
    WL = args.workload
    w = WORKLOADS[WL]
    MODEL, SAMPLES = w["model"], w["samples"]
    SECTOR = tuple(int(x) for x in args.sector.split(",")) if args.sector else w["sector"]
    STEPS = args.lanczos_steps or w["steps"]
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
