import json
import os
import subprocess
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(REPO, "tests", "golden")
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running")


def _ensure_oracle_built():
    so = os.path.join(REPO, "oracle", "libftlm_oracle.so")
    if not os.path.exists(so):
        subprocess.run(["make", "-C", os.path.join(REPO, "oracle")], check=True,
                       capture_output=True)


_ensure_oracle_built()


class Golden:
    def __init__(self):
        self.sectors = np.load(os.path.join(GOLDEN, "sectors.npz"))
        self.lanczos = np.load(os.path.join(GOLDEN, "lanczos.npz"))
        self.exact = np.load(os.path.join(GOLDEN, "exact.npz"))
        with open(os.path.join(GOLDEN, "cases.json")) as f:
            self.meta = json.load(f)
        self.cases = self.meta["cases"]

    def model(self, case):
        import pyoracle
        c = self.cases[case]
        return pyoracle.Model(lx=c["lx"], ly=c["ly"], tp=c["tp"], phix=c["phix"],
                              phiy=c["phiy"], u=c["u"], v=c["v"])

    def sector_keys(self):
        """(case, nup, ndn) triples present in sectors.npz."""
        out = set()
        for k in self.sectors.files:
            case, sec, _ = k.split("/")
            nu, nd = sec.split("_")
            out.add((case, int(nu), int(nd)))
        return sorted(out)

    def sec(self, case, nu, nd, name):
        return self.sectors[f"{case}/{nu}_{nd}/{name}"]

    def has(self, case, nu, nd, name):
        return f"{case}/{nu}_{nd}/{name}" in self.sectors.files

    def lz(self, case, nu, nd, mx, my, name):
        return self.lanczos[f"{case}/{nu}_{nd}_{mx}_{my}/{name}"]


@pytest.fixture(scope="session")
def golden():
    return Golden()


def read_csv(path):
    with open(path) as f:
        header = f.readline().strip().split(",")
        rows = [list(map(float, line.strip().split(","))) for line in f if line.strip()]
    return header, np.array(rows)
