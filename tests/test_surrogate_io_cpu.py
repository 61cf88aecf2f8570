"""Training spectra of the twist surrogate survive a save/load round trip
(a long run can collect them in one job and train in the next)."""
import numpy as np
import pytest

from ftlm_extended_hubbard_development_b200 import surrogate as S


def test_twist_data_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    data = []
    for i in range(3):
        blocks = [(4, 4, k, 1, 8, rng.normal(size=16), rng.random(16), np.arange(16.0), rng.normal(size=2), bool(k % 2))
                  for k in range(4)]
        curve = {"n": rng.random((1, 5)), "log_partition": rng.normal(size=(1, 5))}
        data.append(S.TwistData(i / 3, 0.5, blocks, curve))
    p = str(tmp_path / "train.npz")
    S.save_twist_data(p, data)
    back = S.load_twist_data(p)
    assert len(back) == 3
    for a, b in zip(data, back):
        assert (a.phix, a.phiy) == (b.phix, b.phiy)
        assert np.array_equal(a.curve["n"], b.curve["n"])
        for ba, bb in zip(a.blocks, b.blocks):
            for x, y in zip(ba, bb):
                assert np.array_equal(np.asarray(x), np.asarray(y))


def test_collection_resumes_after_the_saved_twists(tmp_path, monkeypatch):
    """A collection cut off after k twists resumes at twist k + 1 of the grid,
    and training spectra that are not the grid's first twists are refused."""
    calls = []

    def fake_collect(model, px, py, betas, mu, opts, ed=False, levels=16):
        calls.append((px, py))
        return S.TwistData(px, py, [], {"n": np.full((1, 2), px + py)})

    monkeypatch.setattr(S, "collect", fake_collect)
    p = str(tmp_path / "train.npz")
    first = S.collect_grid(None, [5.0], np.zeros(2), None, 2, train=None, save_train=p)
    assert calls == [(0.0, 0.0), (0.0, 0.5), (0.5, 0.0), (0.5, 0.5)]
    calls.clear()
    part = S.load_twist_data(p)[:2]
    full = S.collect_grid(None, [5.0], np.zeros(2), None, 2, train=part, save_train=p)
    assert calls == [(0.5, 0.0), (0.5, 0.5)]
    assert [(t.phix, t.phiy) for t in full] == [(t.phix, t.phiy) for t in first]
    assert len(S.load_twist_data(p)) == 4
    with pytest.raises(ValueError):
        S.collect_grid(None, [5.0], np.zeros(2), None, 3, train=part)
