#!/usr/bin/env python3
"""Regenerate the golden fixtures in tests/golden/ from the reference itself.

Runs only where the reference checkout is present: it needs the binaries that
`make -C oracle ref` compiles from the reference's own sources into
oracle/_ref/ (ref_probe, ftlm_n_vs_mu, ftlm_ed_n_vs_mu). The fixtures it
writes are what the tests read on machines without the reference:

  sectors.npz   basis, relations and CSR of every momentum block, per case/sector
  lanczos.npz   start vectors, alpha/beta, Ritz values and weights per block
  exact.npz     exact block eigenvalues (reference zheev path)
  cases.json    the model flags of every case and the CLI runs below
  csv/*.csv     reference CLI outputs (FTLM, multi-beta, ED), plus one
                checkpoint + .meta pair written by the reference

Usage: python tests/golden/make_golden.py [--skip-slow]
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REF = os.path.join(REPO, "oracle", "_ref")

# Model cases: lattice plus Hamiltonian flags.
CASES = {
    "c1x1": dict(lx=1, ly=1, tp=0.0, phix=1.0, phiy=1.0, u=4.0, v=1.0),
    "c1x4": dict(lx=1, ly=4, tp=0.2, phix=0.25, phiy=0.5, u=4.0, v=1.0),
    "c4x1": dict(lx=4, ly=1, tp=0.0, phix=0.3, phiy=0.7, u=8.0, v=1.5),
    "c2x2": dict(lx=2, ly=2, tp=0.2, phix=1.0, phiy=1.0, u=4.0, v=1.0),
    "c3x2": dict(lx=3, ly=2, tp=0.2, phix=0.25, phiy=0.5, u=8.0, v=1.5),
    "c2x3": dict(lx=2, ly=3, tp=-0.25, phix=0.3, phiy=0.7, u=7.0, v=1.0),
    "c4x2": dict(lx=4, ly=2, tp=0.0, phix=1.0, phiy=1.0, u=8.0, v=0.0),
    "c4x2t": dict(lx=4, ly=2, tp=0.2, phix=0.25, phiy=0.5, u=8.0, v=1.5),
    "c3x3": dict(lx=3, ly=3, tp=-0.25, phix=0.3, phiy=0.7, u=7.0, v=1.0),
    "c4x3": dict(lx=4, ly=3, tp=0.2, phix=0.25, phiy=0.5, u=8.0, v=1.5),
    "c4x4": dict(lx=4, ly=4, tp=-0.25, phix=0.3, phiy=0.7, u=7.0, v=1.0),
    "c6x3": dict(lx=6, ly=3, tp=0.2, phix=0.25, phiy=0.5, u=8.0, v=1.5),
}

# (case, sectors) dumped with relations and all k-block CSRs.
SECTOR_DUMPS = [
    ("c1x1", "all"),
    ("c1x4", "all"),
    ("c4x1", "all"),
    ("c2x2", "all"),
    ("c3x2", "all"),
    ("c2x3", [(1, 2), (3, 3), (2, 4), (6, 0)]),
    ("c4x2", [(4, 4), (3, 5), (2, 2), (0, 8), (8, 8)]),
    ("c4x2t", [(4, 4), (1, 6)]),
    ("c3x3", [(4, 5), (1, 2), (0, 9), (9, 9)]),
    ("c4x3", [(1, 2), (1, 1)]),
    ("c4x4", [(2, 2), (1, 1), (4, 0), (16, 16)]),
    ("c6x3", [(1, 2), (3, 0)]),
]

# (case, nup, ndn, mx, my, samples, steps)
LANCZOS_DUMPS = [
    ("c3x2", 3, 3, 0, 0, 3, 20),
    ("c3x2", 2, 3, 1, 1, 2, 12),
    ("c4x2", 4, 4, 0, 0, 4, 70),
    ("c4x2t", 4, 3, 1, 1, 3, 50),
    ("c3x3", 4, 5, 1, 2, 2, 60),
    ("c2x2", 2, 2, 0, 0, 5, 40),
    ("c4x3", 2, 3, 2, 1, 2, 40),
]

EXACT_DUMPS = [
    ("c3x2", 3, 3, 0, 0),
    ("c3x2", 2, 3, 1, 1),
    ("c4x2", 4, 4, 0, 0),
    ("c4x2t", 4, 3, 1, 1),
    ("c3x3", 4, 5, 1, 2),
    ("c2x2", 2, 2, 0, 0),
    ("c2x2", 1, 1, 1, 0),
]

CONFIG1 = ["--lx", "2", "--ly", "2", "--tx", "1.0", "--ty", "1.0", "--tp", "0.2", "--phix", "1.0",
           "--phiy", "1.0", "--u", "4.0", "--v", "1.0", "--beta", "1.5", "--samples", "5",
           "--lanczos-steps", "40", "--mu-min", "-2", "--mu-max", "6", "--mu-count", "33"]
CONFIG2 = ["--lx", "4", "--ly", "2", "--tx", "1", "--ty", "1", "--tp", "0", "--u", "8", "--v", "0",
           "--beta", "20", "--mu-min", "-5", "--mu-max", "15", "--mu-count", "81"]

# name -> (executable, args, slow)
CLI_RUNS = {
    "config1": ("ftlm_n_vs_mu", CONFIG1, False),
    "config1_t0": ("ftlm_n_vs_mu", CONFIG1 + ["--exact-block-threshold", "0"], False),
    "config1_multibeta": ("ftlm_n_vs_mu", CONFIG1 + ["--beta-list", "1.5,0.5,4",
                                                      "--exact-block-threshold", "0"], False),
    "config1_ed": ("ftlm_ed_n_vs_mu", CONFIG1, False),
    "c3x2_t0": ("ftlm_n_vs_mu", ["--lx", "3", "--ly", "2", "--tp", "0.2", "--phix", "0.25",
                                 "--phiy", "0.5", "--u", "8", "--v", "1.5", "--beta", "3",
                                 "--samples", "4", "--lanczos-steps", "30",
                                 "--exact-block-threshold", "0", "--mu-min", "-3",
                                 "--mu-max", "9", "--mu-count", "25"], False),
    "c3x2_ed": ("ftlm_ed_n_vs_mu", ["--lx", "3", "--ly", "2", "--tp", "0.2", "--phix", "0.25",
                                    "--phiy", "0.5", "--u", "8", "--v", "1.5", "--beta", "3",
                                    "--mu-min", "-3", "--mu-max", "9", "--mu-count", "25"], False),
    "config2_ed": ("ftlm_ed_n_vs_mu", CONFIG2, False),
    "config2": ("ftlm_n_vs_mu", CONFIG2 + ["--samples", "32", "--lanczos-steps", "120",
                                           "--threads", str(os.cpu_count() or 8)], True),
}


# Per-block trace and selected-block debug outputs (main.cpp:1583-1663,
# 1233-1267): name -> (args, selected block (nup, ndown, mx, my)).
TRACE_RUNS = {
    "config1_t0": (CONFIG1 + ["--exact-block-threshold", "0"], (2, 2, 0, 0)),
    # 3x2 with t', V and twists; the reference's trace mode ends in SIGSEGV on
    # 4x2 lattices in this build (its ftlm_n_vs_mu with OpenMP + OpenBLAS
    # 0.3.15), while 2x2 and 3x2 run to completion.
    "c3x2_t0": (CLI_RUNS["c3x2_t0"][1], (3, 2, 1, 1)),
}


def write_trace_goldens(csvdir, tmp):
    """Reference trace and debug CSVs of TRACE_RUNS into csv/<name>_trace.csv
    and csv/<name>_debug.csv (plus the run's stdout)."""
    for name, (cli, (nu, nd, mx, my)) in TRACE_RUNS.items():
        tr = os.path.join(csvdir, name + "_trace.csv")
        dbg = os.path.join(csvdir, name + "_debug.csv")
        r = run([os.path.join(REF, "ftlm_n_vs_mu")] + cli + [
            "--output", os.path.join(tmp, name + ".csv"), "--trace-partition-csv", tr,
            "--debug-block-nup", str(nu), "--debug-block-ndown", str(nd), "--debug-block-mx", str(mx),
            "--debug-block-my", str(my), "--debug-block-csv", dbg])
        with open(os.path.join(csvdir, name + "_trace.stdout"), "w") as f:
            f.write(r.stdout)
    return {k: {"exe": "ftlm_n_vs_mu", "args": v[0], "block": list(v[1])} for k, v in TRACE_RUNS.items()}


def run(cmd, **kw):
    r = subprocess.run(cmd, capture_output=True, text=True, **kw)
    if r.returncode != 0:
        raise SystemExit(f"failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return r


def flags(case):
    c = CASES[case]
    out = []
    for k in ("lx", "ly", "tp", "phix", "phiy", "u", "v"):
        out += [f"--{k}", repr(c[k])]
    return out


def load_dir(d):
    return {f[:-4]: np.load(os.path.join(d, f)) for f in os.listdir(d) if f.endswith(".npy")}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--skip-slow", action="store_true")
    ap.add_argument("--only-trace", action="store_true",
                    help="write only the trace/debug fixtures and their cases.json entry")
    args = ap.parse_args()
    for b in ("ref_probe", "ftlm_n_vs_mu", "ftlm_ed_n_vs_mu"):
        if not os.path.exists(os.path.join(REF, b)):
            raise SystemExit("reference binaries missing: run `make -C oracle ref` first")
    tmp = tempfile.mkdtemp()
    if args.only_trace:
        try:
            path = os.path.join(HERE, "cases.json")
            with open(path) as f:
                meta = json.load(f)
            meta["trace_runs"] = write_trace_goldens(os.path.join(HERE, "csv"), tmp)
            with open(path, "w") as f:
                json.dump(meta, f, indent=1)
        finally:
            shutil.rmtree(tmp, ignore_errors=True)
        return
    try:
        sectors = {}
        for case, which in SECTOR_DUMPS:
            n = CASES[case]["lx"] * CASES[case]["ly"]
            secs = [(a, b) for a in range(n + 1) for b in range(n + 1)] if which == "all" else which
            for nu, nd in secs:
                d = os.path.join(tmp, f"s_{case}_{nu}_{nd}")
                run([os.path.join(REF, "ref_probe"), "sector", d, str(nu), str(nd), "--"]
                    + flags(case))
                for k, v in load_dir(d).items():
                    sectors[f"{case}/{nu}_{nd}/{k}"] = v
        np.savez_compressed(os.path.join(HERE, "sectors.npz"), **sectors)

        lanczos = {}
        for case, nu, nd, mx, my, smp, stp in LANCZOS_DUMPS:
            d = os.path.join(tmp, f"l_{case}_{nu}_{nd}_{mx}_{my}")
            run([os.path.join(REF, "ref_probe"), "lanczos", d, str(nu), str(nd), str(mx), str(my),
                 "--"] + flags(case) + ["--samples", str(smp), "--lanczos-steps", str(stp)])
            for k, v in load_dir(d).items():
                lanczos[f"{case}/{nu}_{nd}_{mx}_{my}/{k}"] = v
        np.savez_compressed(os.path.join(HERE, "lanczos.npz"), **lanczos)

        exact = {}
        for case, nu, nd, mx, my in EXACT_DUMPS:
            d = os.path.join(tmp, f"e_{case}_{nu}_{nd}_{mx}_{my}")
            run([os.path.join(REF, "ref_probe"), "exact", d, str(nu), str(nd), str(mx), str(my),
                 "--"] + flags(case))
            exact[f"{case}/{nu}_{nd}_{mx}_{my}/exact"] = np.load(os.path.join(d, "exact.npy"))
        np.savez_compressed(os.path.join(HERE, "exact.npz"), **exact)

        csvdir = os.path.join(HERE, "csv")
        os.makedirs(csvdir, exist_ok=True)
        timings = {}
        for name, (exe, cli, slow) in CLI_RUNS.items():
            if slow and args.skip_slow and os.path.exists(os.path.join(csvdir, name + ".csv")):
                continue
            t0 = time.time()
            r = run([os.path.join(REF, exe)] + cli + ["--output", os.path.join(csvdir, name + ".csv")])
            timings[name] = time.time() - t0
            with open(os.path.join(csvdir, name + ".stdout"), "w") as f:
                f.write(r.stdout)
        # One checkpoint written by the reference (FTLM + exact blocks).
        ck = os.path.join(csvdir, "config1_ckpt.ftlmcp")
        for p in (ck, ck + ".meta"):
            if os.path.exists(p):
                os.remove(p)
        run([os.path.join(REF, "ftlm_n_vs_mu")] + CONFIG1 + ["--exact-block-threshold", "4",
            "--checkpoint", ck, "--output", os.path.join(tmp, "ck.csv")])
        shutil.copy(os.path.join(tmp, "ck.csv"), os.path.join(csvdir, "config1_ckpt.csv"))

        trace_runs = write_trace_goldens(csvdir, tmp)
        meta = {"cases": CASES,
                "cli_runs": {k: {"exe": v[0], "args": v[1]} for k, v in CLI_RUNS.items()},
                "trace_runs": trace_runs,
                "checkpoint_run": {"exe": "ftlm_n_vs_mu",
                                   "args": CONFIG1 + ["--exact-block-threshold", "4"]},
                "lanczos_dumps": LANCZOS_DUMPS, "exact_dumps": EXACT_DUMPS,
                "sector_dumps": [[c, w] for c, w in SECTOR_DUMPS],
                "reference_wall_seconds": timings}
        old = os.path.join(HERE, "cases.json")
        if os.path.exists(old):
            prev = json.load(open(old)).get("reference_wall_seconds", {})
            for k, v in prev.items():
                meta["reference_wall_seconds"].setdefault(k, v)
        with open(old, "w") as f:
            json.dump(meta, f, indent=1)
    finally:
        shutil.rmtree(tmp)


if __name__ == "__main__":
    sys.exit(main())
