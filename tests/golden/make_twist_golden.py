"""Golden fixtures for the twist-averaging module.

Writes seeded synthetic twist-resolved n(mu) CSVs (reference column layout)
under tests/golden/twist/, runs the reference's scripts/average_twist_outputs.py
on them in both modes (and on a legacy file without a beta column with
--single-beta), and stores its outputs beside the inputs. Run from the
repository root with the reference checkout available:

    python tests/golden/make_twist_golden.py /root/reference
"""
import csv
import math
import os
import subprocess
import sys

import numpy as np

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "twist")
SITES = 8


def write_inputs(rng):
    paths = []
    betas = [2.5, 20.0]
    mus = np.linspace(-2.0, 6.0, 9)
    for t in range(3):
        path = os.path.join(HERE, f"twist_{t}.csv")
        with open(path, "w", newline="") as f:
            w = csv.writer(f)
            w.writerow(["beta", "mu", "n", "charge_correlation", "compressibility", "log_partition"])
            for b in betas:
                for mu in mus:
                    n = 1.0 / (1.0 + math.exp(-(mu - 2.0 + 0.3 * rng.standard_normal()))) * 2.0
                    chi = abs(0.2 * rng.standard_normal())
                    lz = b * mu * n * SITES / 4 + rng.standard_normal()
                    w.writerow([repr(float(v)) for v in (b, mu, n, chi, b * chi, lz)])
        paths.append(path)
    legacy = os.path.join(HERE, "legacy_single_beta.csv")
    with open(legacy, "w", newline="") as f:
        w = csv.writer(f)
        w.writerow(["mu", "n", "charge_correlation", "compressibility"])
        for mu in mus:
            chi = abs(0.1 * rng.standard_normal())
            w.writerow([repr(float(v)) for v in (mu, rng.random() * 2, chi, 4.0 * chi)])
    return paths, legacy


def main(ref_root):
    os.makedirs(HERE, exist_ok=True)
    rng = np.random.default_rng(20240611)
    paths, legacy = write_inputs(rng)
    script = os.path.join(ref_root, "scripts", "average_twist_outputs.py")
    runs = {
        "avg_observable.csv": paths + ["--mode", "observable-average"],
        "avg_partition.csv": paths + ["--mode", "partition-sum", "--sites", str(SITES)],
        "avg_legacy.csv": [legacy, paths[0], "--single-beta", "2.5"],
    }
    for out, args in runs.items():
        subprocess.run([sys.executable, script, *args, "--output", os.path.join(HERE, out)], check=True)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
