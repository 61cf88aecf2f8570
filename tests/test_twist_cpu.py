"""Twist averaging (CPU): the module's CLI against outputs of the reference's
scripts/average_twist_outputs.py on the same inputs (tests/golden/twist,
made by tests/golden/make_twist_golden.py), and the surrogate's host-side
spectral bookkeeping."""
import csv
import math
import os

import numpy as np
import pytest

from ftlm_extended_hubbard_development_b200 import twist
from ftlm_extended_hubbard_development_b200.surrogate import (block_features, curve_from_blocks,
                                                              heldout_twists, reduce_spectrum,
                                                              tail_log_partition)

G = os.path.join(os.path.dirname(__file__), "golden", "twist")
INPUTS = [os.path.join(G, f"twist_{t}.csv") for t in range(3)]


def _read(path):
    with open(path, newline="") as f:
        return list(csv.DictReader(f))


@pytest.mark.parametrize("golden,args", [
    ("avg_observable.csv", INPUTS + ["--mode", "observable-average"]),
    ("avg_partition.csv", INPUTS + ["--mode", "partition-sum", "--sites", "8"]),
    ("avg_legacy.csv", [os.path.join(G, "legacy_single_beta.csv"), INPUTS[0], "--single-beta", "2.5"]),
])
def test_cli_matches_reference_script(tmp_path, golden, args):
    out = tmp_path / "out.csv"
    assert twist.main(args + ["--output", str(out)]) == 0
    got, want = _read(out), _read(os.path.join(G, golden))
    assert list(got[0].keys()) == list(want[0].keys())
    assert len(got) == len(want)
    for g, w in zip(got, want):
        assert g == w  # same float text: same arithmetic in the same order


def test_cli_errors(tmp_path):
    with pytest.raises(SystemExit, match="--sites is required"):
        twist.main(INPUTS + ["--mode", "partition-sum", "--output", str(tmp_path / "o.csv")])
    with pytest.raises(SystemExit, match="no beta column"):
        twist.main([os.path.join(G, "legacy_single_beta.csv"), "--output", str(tmp_path / "o.csv")])
    rows = list(twist.read_rows([os.path.join(G, "legacy_single_beta.csv")], 1.0))
    with pytest.raises(SystemExit, match="requires log_partition"):
        twist.combine_rows(rows, "partition-sum", 8)


def test_uniform_grid_and_heldout():
    g = twist.uniform_grid(6)
    assert len(g) == 36 and g[0] == (0.0, 0.0) and g[-1] == (5 / 6, 5 / 6)
    h = heldout_twists(8, 2024)
    assert len(h) == 8 and all(0.0 <= a < 1.0 and 0.0 <= b < 1.0 for a, b in h)
    assert h == heldout_twists(8, 2024)
    assert not set(h) & set(g)


def test_reduce_spectrum_merges_levels_and_splits_tail():
    ev = np.array([0.5, -1.0, -1.0 + 1e-9, 2.0, 0.5, 3.0, 4.0])
    w = np.array([0.1, 0.2, 0.3, 0.4, 0.5, 0.6, 0.7])
    E, W, M, te, tw = reduce_spectrum(ev, w, 2.0, False, levels=3)  # FTLM: Ritz values merged
    assert np.allclose(E, [-1.0, 0.5, 2.0])
    assert np.allclose(W, [1.0, 1.2, 0.8])
    assert M.tolist() == [1, 1, 1]
    assert np.allclose(te, [3.0, 4.0]) and np.allclose(tw, [1.2, 1.4])
    E, W, M, te, tw = reduce_spectrum(np.array([2.0, 1.0, 1.0]), None, 1.0, True, levels=4)  # exact: one by one
    assert M.tolist() == [1, 1, 1, 0] and W.tolist() == [1, 1, 1, 0] and E.tolist()[:3] == [1, 1, 2]
    assert len(te) == 0


def test_curve_from_blocks_equals_direct_sums():
    """Low levels + tail partition sums give the same grand-canonical curve
    as the full spectra, whatever the split."""
    rng = np.random.default_rng(3)
    sites, betas, mu = 4, [0.7, 5.0], np.linspace(-2, 6, 17)
    full, split = [], []
    for p in range(0, 9):
        e = np.sort(rng.normal(size=12) * 2 + 0.8 * p * p / 4 - 0.5 * p)
        w = rng.random(12) + 0.1
        full.append((p, e, w))
        E, W, M, te, tw = reduce_spectrum(e, w, 1.0, False, levels=4)
        split.append((0, 0, 0, 0, p, E, W, M, tail_log_partition(te, tw, betas)))
    got = curve_from_blocks(split, sites, betas, mu)
    for ib, b in enumerate(betas):
        lz = np.array([math.log(sum((w * np.exp(-b * (e - m * p))).sum() for p, e, w in full)) for m in mu])
        n = np.array([sum((p * w * np.exp(-b * (e - m * p))).sum() for p, e, w in full) for m in mu])
        n = n / np.exp(lz) / sites
        assert np.allclose(got["log_partition"][ib], lz, rtol=1e-12, atol=1e-9)
        assert np.allclose(got["n"][ib], n, rtol=1e-10, atol=1e-12)


def test_block_features_periodicity():
    """Per-bond twist phases: period lx in phi_x, ly in phi_y, not 1."""
    from ftlm_extended_hubbard_development_b200.surrogate import n_features
    from ftlm_extended_hubbard_development_b200.engine import Model
    a = block_features(0.25, 0.5, 3, 4, 1, 0, 4, 2)
    assert len(a) == n_features(Model(lx=4, ly=2)) == 32
    assert np.allclose(a, block_features(4.25, 2.5, 3, 4, 1, 0, 4, 2))
    assert not np.allclose(a, block_features(1.25, 0.5, 3, 4, 1, 0, 4, 2))
    assert sum(a[8:]) == 4.0 and a[8 + 3] == 1 and a[8 + 9 + 4] == 1 and a[8 + 18 + 1] == 1 and a[8 + 22] == 1


def test_level_importance_is_a_boltzmann_probability():
    """The loss weight of a level is the largest probability it reaches on
    the (beta, mu) grid: in [0, 1], 1 for a level that alone dominates at some
    mu, and tails count in the normalisation."""
    from ftlm_extended_hubbard_development_b200.surrogate import level_importance
    betas, mu = [2.0, 8.0], np.linspace(-3.0, 3.0, 61)
    blocks = []
    for p, e0 in ((0, 0.0), (1, -1.0), (2, 0.5)):
        E = np.array([e0, e0 + 0.3, e0 + 2.0, 0.0])
        W = np.array([1.0, 2.0, 1.0, 0.0])
        M = np.array([1.0, 1.0, 1.0, 0.0])
        blocks.append((0, 0, 0, 0, p, E, W, M, tail_log_partition(np.array([e0 + 3.0]), np.array([5.0]), betas)))
    imp = level_importance(blocks, betas, mu)
    assert imp.shape == (3, 4) and (imp >= 0).all() and (imp <= 1 + 1e-12).all()
    assert imp[:, 3].max() == 0.0            # absent levels carry no weight
    # deep inside a block's mu window at beta = 8 its ground level has
    # probability 1 / (1 + 2 e^{-2.4} + e^{-16} + 5 e^{-24}) (own excited
    # levels and tail; the other blocks are negligible there)
    p0 = 1.0 / (1.0 + 2.0 * math.exp(-2.4) + math.exp(-16.0) + 5.0 * math.exp(-24.0))
    assert np.allclose(imp[:, 0], p0, rtol=2e-3)
    assert (imp[:, 2] < imp[:, 0]).all()     # higher levels matter less
