"""Twist grids and twist averaging.

* `curve_at_twist` / `run_twist_grid`: n(mu) curves of the engine at a list of
  homogeneous twists (phi_x, phi_y), one GPU context per twist.
* `combine_rows` / `main`: the two combination modes of the reference's
  scripts/average_twist_outputs.py (lines 37-115) on CSV rows with the same
  columns, so this module is a drop-in for that script:
    observable-average  plain mean of n, charge_correlation and
                        compressibility; log-mean-exp of log_partition
    partition-sum       twists weighted by exp(log Z_t - logsumexp log Z),
                        <N> and <N^2> recombined with --sites
  Output columns: beta, mu, n, charge_correlation, compressibility,
  twist_count, mode, log_partition (rows sorted by (beta, mu)).

    python -m ftlm_extended_hubbard_development_b200.twist twist_*.csv \
        --mode partition-sum --sites 16 --output avg.csv
"""
from __future__ import annotations

import argparse
import csv
import math
import sys
from collections import defaultdict
from dataclasses import replace

import numpy as np

from .engine import Model, RunOpts, run_curve


def _logsumexp(values):
    top = max(values)
    return top + math.log(sum(math.exp(v - top) for v in values))


def read_rows(paths, single_beta=None):
    """Rows of n(mu) CSVs (reference columns); files without a beta column
    need single_beta (average_twist_outputs.py:13-34)."""
    for path in paths:
        with open(path, newline="") as f:
            reader = csv.DictReader(f)
            has_beta = "beta" in (reader.fieldnames or [])
            if not has_beta and single_beta is None:
                raise SystemExit(f"{path} has no beta column; pass --single-beta for legacy single-beta files")
            for row in reader:
                lp = row.get("log_partition")
                yield {
                    "path": path,
                    "beta": float(row["beta"]) if has_beta else float(single_beta),
                    "mu": float(row["mu"]),
                    "n": float(row["n"]),
                    "charge_correlation": float(row["charge_correlation"]),
                    "compressibility": float(row["compressibility"]),
                    "log_partition": float(lp) if lp not in (None, "") else None,
                }


def combine_rows(rows, mode="observable-average", sites=None):
    """Group by (beta, mu) and combine the twists of each group."""
    if mode == "partition-sum" and (sites is None or sites <= 0):
        raise SystemExit("--sites is required and must be positive for --mode partition-sum")
    groups = defaultdict(list)
    for r in rows:
        groups[(r["beta"], r["mu"])].append(r)
    out = []
    for (beta, mu), g in sorted(groups.items()):
        if mode == "observable-average":
            k = len(g)
            n = sum(r["n"] for r in g) / k
            chi = sum(r["charge_correlation"] for r in g) / k
            kappa = sum(r["compressibility"] for r in g) / k
            logs = [r["log_partition"] for r in g if r["log_partition"] is not None]
            logz = _logsumexp(logs) - math.log(len(logs)) if logs else ""
        elif mode == "partition-sum":
            if any(r["log_partition"] is None for r in g):
                raise SystemExit("partition-sum mode requires log_partition in every input row")
            lz = [r["log_partition"] for r in g]
            total = _logsumexp(lz)
            n1 = n2 = 0.0
            for r in g:
                w = math.exp(r["log_partition"] - total)
                p = r["n"] * sites
                n1 += w * p
                n2 += w * (r["charge_correlation"] * sites + p * p)
            n = n1 / sites
            chi = max(0.0, (n2 - n1 * n1) / sites)
            kappa = beta * chi
            logz = total
        else:
            raise SystemExit(f"unknown mode {mode}")
        out.append({"beta": beta, "mu": mu, "n": n, "charge_correlation": chi, "compressibility": kappa,
                    "twist_count": len(g), "mode": mode, "log_partition": logz})
    return out


FIELDS = ["beta", "mu", "n", "charge_correlation", "compressibility", "twist_count", "mode", "log_partition"]


def write_rows(path, out_rows):
    with open(path, "w", newline="") as f:
        w = csv.DictWriter(f, fieldnames=FIELDS)
        w.writeheader()
        for r in out_rows:
            w.writerow(r)


def curve_rows(curve, betas, mu):
    """Engine curve (dict of [nbeta][nmu] arrays) as CSV-like rows."""
    rows = []
    for ib, b in enumerate(betas):
        for im, m in enumerate(mu):
            rows.append({"beta": float(b), "mu": float(m), "n": float(curve["n"][ib][im]),
                         "charge_correlation": float(curve["charge_correlation"][ib][im]),
                         "compressibility": float(curve["compressibility"][ib][im]),
                         "log_partition": float(curve["log_partition"][ib][im])})
    return rows


def curve_at_twist(model: Model, phix: float, phiy: float, betas, mu, opts: RunOpts | None = None,
                   ed: bool = False):
    return run_curve(replace(model, phix=float(phix), phiy=float(phiy)), betas, mu, opts, ed=ed)


def twist_owners(n_twists: int, world: int):
    """Rank of each twist: the curves at different twists cost the same, so
    longest-processing-time assignment is a deal in list order."""
    return [i % world for i in range(n_twists)]


def run_twist_grid(model: Model, twists, betas, mu, opts: RunOpts | None = None, ed: bool = False,
                   rank: int = 0, world: int = 1):
    """Engine n(mu) curves at this rank's twists (all of them with one rank):
    list of (phix, phiy, curve). Ranks share nothing while running; gather
    the lists (e.g. torch.distributed.all_gather_object) to combine them."""
    own = twist_owners(len(twists), world)
    return [(px, py, curve_at_twist(model, px, py, betas, mu, opts, ed))
            for i, (px, py) in enumerate(twists) if own[i] == rank]


def uniform_grid(n: int):
    """n x n twists i/n, j/n in [0, 1)^2."""
    return [(i / n, j / n) for i in range(n) for j in range(n)]


def main(argv=None):
    ap = argparse.ArgumentParser(description="Average or partition-sum FTLM n(mu) CSV files over twists.")
    ap.add_argument("inputs", nargs="+")
    ap.add_argument("--output", required=True)
    ap.add_argument("--mode", choices=["observable-average", "partition-sum"], default="observable-average")
    ap.add_argument("--sites", type=int)
    ap.add_argument("--single-beta", type=float)
    a = ap.parse_args(argv)
    if a.mode == "partition-sum" and (a.sites is None or a.sites <= 0):
        raise SystemExit("--sites is required and must be positive for --mode partition-sum")
    write_rows(a.output, combine_rows(read_rows(a.inputs, a.single_beta), a.mode, a.sites))
    return 0


if __name__ == "__main__":
    sys.exit(main())
