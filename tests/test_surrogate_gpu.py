"""Twist-surrogate MLP on the GPU: forward, gradient and Adam of the library's
own kernels against the float64 CPU oracle (oracle/mlp_oracle.py), training,
and what the trained surrogate gains over the method without it."""
import os
import sys
import time
from dataclasses import replace

import numpy as np
import pytest

from ftlm_extended_hubbard_development_b200.engine import FtlmError, Mlp, Model, RunOpts, run_curve
from ftlm_extended_hubbard_development_b200 import surrogate as S

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "oracle"))
import mlp_oracle as mo  # noqa: E402

pytestmark = pytest.mark.gpu


def _data(rng, n, n_in, n_out):
    x = rng.uniform(-1, 1, size=(n, n_in)).astype(np.float32)
    t = rng.normal(size=(n, n_out)).astype(np.float32)
    m = (rng.random((n, n_out)) > 0.25).astype(np.float32)
    return x, t, m


def test_mlp_forward_and_gradient_match_oracle():
    rng = np.random.default_rng(11)
    net = Mlp(10, 48, 3, 12, seed=5)
    shapes = mo.layer_shapes(10, 48, 3, 12)
    assert net.num_params == mo.num_params(10, 48, 3, 12)
    p0 = net.get_params()
    for (i, o), (W, b) in zip(shapes, mo.unpack(p0, shapes)):  # Glorot-uniform, zero biases
        assert np.abs(W).max() <= np.sqrt(6.0 / (i + o)) and not b.any()
    p = (rng.normal(size=net.num_params) * 0.3).astype(np.float32)
    net.set_params(p)
    assert np.array_equal(net.get_params(), p)
    x, t, m = _data(rng, 333, 10, 12)  # ragged against the 32-wide tiles
    y = net.forward(x)
    yo = mo.forward(p, shapes, x)[-1]
    assert np.abs(y - yo).max() <= 1e-5 * max(1.0, np.abs(yo).max())
    loss, g = net.loss_grad(x, t, m)
    lo, go = mo.loss_grad(p, shapes, x, t, m)
    assert abs(loss - lo) <= 1e-5 * lo
    assert np.linalg.norm(g - go) <= 2e-5 * np.linalg.norm(go)
    assert np.abs(g - go).max() <= 1e-5 * np.abs(go).max()
    net.close()


def test_mlp_adam_matches_oracle():
    """Full-batch epochs: the shuffle only reorders rows inside the batch."""
    rng = np.random.default_rng(12)
    net = Mlp(6, 32, 2, 5, seed=9)
    shapes = mo.layer_shapes(6, 32, 2, 5)
    p0 = net.get_params().astype(np.float64)
    x, t, m = _data(rng, 200, 6, 5)
    epochs, lr = 6, 1e-3
    hist = net.train(x, t, m, epochs, 200, lr, seed=3)
    po = mo.adam_steps(p0, shapes, [(x, t, m)] * epochs, lr)
    p = net.get_params().astype(np.float64)
    d = np.abs(p - po)
    # a gradient entry within float32 rounding of zero may take the other
    # sign in Adam's first steps; every other entry follows the oracle
    assert np.mean(d <= 2e-6) >= 0.995, d.max()
    # history entry e is the loss of the batch before epoch e's step
    assert abs(hist[0] - mo.loss_grad(p0, shapes, x, t, m)[0]) <= 1e-5 * hist[0]
    pl = mo.adam_steps(p0, shapes, [(x, t, m)] * (epochs - 1), lr)
    assert abs(hist[-1] - mo.loss_grad(pl, shapes, x, t, m)[0]) <= 1e-4 * hist[-1]
    net.close()


def test_mlp_training_reduces_loss_and_is_deterministic():
    rng = np.random.default_rng(13)
    x = rng.uniform(-1, 1, size=(4096, 4)).astype(np.float32)
    t = np.stack([np.sin(3 * x[:, 0]) * np.cos(2 * x[:, 1]), x[:, 2] * x[:, 3] - 0.3 * x[:, 0]], 1)
    t = t.astype(np.float32)
    m = np.ones_like(t)
    a, b = Mlp(4, 64, 3, 2, seed=21), Mlp(4, 64, 3, 2, seed=21)
    ha = a.train(x, t, m, 60, 256, 3e-3, seed=4)
    hb = b.train(x, t, m, 60, 256, 3e-3, seed=4)
    assert np.array_equal(ha, hb) and np.array_equal(a.get_params(), b.get_params())
    assert ha[-1] < 0.05 * ha[0]
    # the loss of the trained net on its data agrees with the history's scale
    lo, _ = a.loss_grad(x, t, m)
    assert lo < 2 * ha[-1] + 1e-4
    a.close()
    b.close()


def test_mlp_argument_errors():
    with pytest.raises(FtlmError):
        Mlp(0, 8, 1, 1)
    net = Mlp(3, 8, 1, 2)
    with pytest.raises(FtlmError, match="parameter count"):
        net.set_params(np.zeros(3, np.float32))
    with pytest.raises(FtlmError, match="empty mask"):
        net.loss_grad(np.zeros((4, 3)), np.zeros((4, 2)), np.zeros((4, 2)))
    net.close()


# The twist-surrogate Hamiltonian (t' = -0.25, U = 7, V = 1, beta = 5,
# n(mu) over 141 points in [-3, 4]) on a 4x2 lattice, where every block is
# diagonalised exactly so that the judges carry no FTLM noise.
SUR_MODEL = Model(lx=4, ly=2, tx=1.0, ty=1.0, tp=-0.25, u=7.0, v=1.0)
SUR_BETAS = [5.0]
SUR_MU = np.linspace(-3.0, 4.0, 141)


def test_collect_curve_is_the_engine_curve():
    opts = RunOpts(exact_block_threshold=256)
    td = S.collect(SUR_MODEL, 0.3, 0.7, SUR_BETAS, SUR_MU, opts, ed=True)
    ref = run_curve(replace(SUR_MODEL, phix=0.3, phiy=0.7), SUR_BETAS, SUR_MU, opts, ed=True)
    for k in ("n", "log_partition"):
        assert np.allclose(td.curve[k], ref[k], rtol=1e-13, atol=1e-13)
    # low levels + tail partition sums reproduce the same curve
    split = S.curve_from_blocks(td.blocks, SUR_MODEL.sites, SUR_BETAS, SUR_MU)
    assert np.abs(split["n"] - ref["n"]).max() < 1e-10
    assert np.abs(split["log_partition"] - ref["log_partition"]).max() < 1e-9


def test_surrogate_gain_over_nearest_training_twist():
    """What the trained network gains: at twists it has not seen, its n(mu)
    is closer to plain ED than the method without it, which reuses the curve
    of the nearest training twist."""
    t0 = time.time()
    res = S.surrogate_twist_average(SUR_MODEL, SUR_BETAS, SUR_MU, RunOpts(), grid=6, heldout=8, dense=24,
                                    threshold=0.02, ed=True, epochs=600)
    sur = res["surrogate"]
    es = [j["err_surrogate"] for j in res["judges"]]
    en = [j["err_nearest_twist"] for j in res["judges"]]
    for px, py in S.heldout_twists(12, seed=77):  # further unseen twists
        td = S.collect(SUR_MODEL, px, py, SUR_BETAS, SUR_MU, RunOpts(), ed=True)
        es.append(float(np.abs(sur.curve(px, py, SUR_BETAS, SUR_MU)["n"] - td.curve["n"]).max()))
        en.append(float(np.abs(sur.nearest(px, py, wrap=True).curve["n"] - td.curve["n"]).max()))
    es, en = np.array(es), np.array(en)
    h = res["loss_history"]
    print(f"\nsurrogate workflow {time.time() - t0:.1f} s; loss {h[0]:.3e} -> {h[-1]:.3e}; "
          f"unseen-twist max|dn|: surrogate mean {es.mean():.4f} max {es.max():.4f}, nearest training twist "
          f"mean {en.mean():.4f} max {en.max():.4f}, surrogate better at {np.mean(es < en):.2f}; "
          f"source: {res['source']}")
    assert h[-1] < 0.2 * h[0]
    # measured on a B200: mean 0.0183 vs 0.0227, better at 16 of 20 twists
    assert es.mean() < 0.9 * en.mean()
    assert np.mean(es < en) >= 0.65
    sur.close()


def test_surrogate_falls_back_when_judges_fail():
    m = Model(lx=2, ly=2, tx=1.0, ty=1.0, tp=0.2, u=4.0, v=1.0)
    res = S.surrogate_twist_average(m, [1.5], np.linspace(-2, 6, 33), RunOpts(), grid=3, heldout=2, dense=4,
                                    threshold=-1.0, ed=True, epochs=20)
    assert not res["accepted"] and res["source"].startswith("engine twists")
    assert res["average"][0]["twist_count"] == 9 + 2
    res["surrogate"].close()
