"""Sector sharding on the GPU: one rank reproduces run_curve exactly, and two
ranks' shares (run one after the other on the one GPU, merged on the host)
equal the single-rank curve."""
import numpy as np
import pytest

from ftlm_extended_hubbard_development_b200 import shard
from ftlm_extended_hubbard_development_b200.engine import Model, RunOpts, linspace, run_curve

pytestmark = pytest.mark.gpu

MODEL = Model(lx=4, ly=2, tx=1.0, ty=1.0, tp=0.0, u=8.0, v=0.0)
BETAS = [20.0, 2.0]
MU = linspace(-5.0, 15.0, 81)
OPTS = RunOpts(samples=8, lanczos_steps=60)


def test_one_rank_is_run_curve():
    a = run_curve(MODEL, BETAS, MU, OPTS)
    b = shard.run_curve_sharded(MODEL, BETAS, MU, OPTS, rank=0, world=1)
    for k in ("n", "charge_correlation", "log_partition"):
        assert np.array_equal(a[k], b[k])


@pytest.mark.parametrize("world", [2, 3])
def test_shares_merge_to_the_whole_curve(world):
    parts = [shard.shard_accumulators(MODEL, BETAS, MU, OPTS, rank=r, world=world) for r in range(world)]
    gmin = np.minimum.reduce([p[0] for p in parts])
    rescaled = [shard.merge_accumulators(*p, BETAS, lambda a: gmin, lambda a: a)[1:] for p in parts]
    total = [sum(r[i] for r in rescaled) for i in range(3)]
    got = shard.finalize(BETAS, MODEL.sites, gmin, *total)
    ref = run_curve(MODEL, BETAS, MU, OPTS)
    assert np.abs(got["n"] - ref["n"]).max() < 1e-12
    assert np.abs(got["log_partition"] - ref["log_partition"]).max() < 1e-10
