"""Small FTLM blocks in one persistent launch (ftlm_blocks_ftlm_batched)
against the per-block sweep path of ftlm_block_spectrum, and against the
oracle's Lanczos from the reference start vectors."""
import os
import sys

import numpy as np
import pytest

from ftlm_extended_hubbard_development_b200.engine import (PREC_FP64, PREC_MIXED, START_PHILOX_PHASE as START_PHILOX,
                                                           START_REF_GAUSSIAN, Engine, Model, RunOpts)

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "oracle"))
import pyoracle as po  # noqa: E402

pytestmark = pytest.mark.gpu

MODEL = Model(lx=4, ly=2, tx=1.0, ty=1.0, tp=-0.25, phix=0.3, phiy=0.1, u=7.0, v=1.0)


def _spectra(eng, blocks, batched):
    if batched:
        eng.blocks_ftlm_batched(blocks)
    out = {}
    for b in blocks:
        ev, w, pref = eng.block_spectrum(b[0], b[1], exact=False)
        out[b] = (ev, w, pref)
    return out


def _z(ev, w, pref, beta, e0):
    return pref * float((w * np.exp(-beta * (ev - e0))).sum())


@pytest.mark.parametrize("precision,start", [(PREC_FP64, START_REF_GAUSSIAN), (PREC_FP64, START_PHILOX),
                                             (PREC_MIXED, START_PHILOX)])
def test_batched_small_blocks_match_sweep_path(precision, start):
    opts = RunOpts(samples=12, lanczos_steps=60, precision=precision, start_vector=start)
    tol = 1e-10 if precision == PREC_FP64 else 2e-5
    with Engine(MODEL, opts) as a, Engine(MODEL, opts) as b:
        for nu, nd in ((4, 4), (3, 4), (2, 5)):
            info = a.sector_prepare(nu, nd)
            b.sector_prepare(nu, nd)
            blocks = [(k % 4, k // 4) for k, d in enumerate(info.block_dims) if d > 0]
            a.profile(True)
            a.profile_reset()
            sa = _spectra(a, blocks, True)
            prof = a.profile()
            assert prof["small_tasks"] == 12 * len(blocks)
            sb = _spectra(b, blocks, False)
            for blk in blocks:
                (ea, wa, pa), (eb, wb, pb) = sa[blk], sb[blk]
                assert len(ea) == len(eb) and pa == pb
                e0 = min(ea.min(), eb.min())
                # per random vector: the lowest Ritz value (converged)
                K = len(ea) // 12
                assert np.abs(ea.reshape(12, K)[:, 0] - eb.reshape(12, K)[:, 0]).max() <= tol * max(1, abs(e0))
                for beta in (0.5, 5.0):
                    za, zb = _z(ea, wa, pa, beta, e0), _z(eb, wb, pb, beta, e0)
                    assert abs(za - zb) <= 10 * tol * zb


def test_batched_small_block_lanczos_matches_oracle():
    """Reference start vectors: the first Ritz values and weights of each
    vector equal the oracle's Lanczos + Jacobi on the oracle's CSR."""
    R, K = 4, 30
    opts = RunOpts(samples=R, lanczos_steps=K, precision=PREC_FP64, start_vector=START_REF_GAUSSIAN, seed=99)
    om = po.Model(lx=4, ly=2, tx=1.0, ty=1.0, tp=-0.25, phix=0.3, phiy=0.1, u=7.0, v=1.0)
    with Engine(MODEL, opts) as eng:
        info = eng.sector_prepare(3, 3)
        blocks = [(k % 4, k // 4) for k, d in enumerate(info.block_dims) if d > 0]
        eng.blocks_ftlm_batched(blocks)
        for mx, my in blocks[:3]:
            ev, w, pref = eng.block_spectrum(mx, my, exact=False)
            csr = po.block_csr(om, 3, 3, mx, my)
            bseed = po.block_seed(99, 3, 3, mx, my)
            for r in range(R):
                a, b = po.lanczos(csr, po.start_vector(bseed, r, csr.dim), K)
                e, z = po.tridiag_jacobi(a, b)
                assert np.abs(ev[r * K:r * K + 3] - e[:3]).max() < 1e-10
                assert np.abs(w[r * K:r * K + 3] - z[:3] / R).max() < 1e-10
