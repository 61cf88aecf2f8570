"""Exact blocks pooled across sectors (ftlm_exact_defer / ftlm_exact_flush):
the dense solver diagonalises the pooled matrices of a whole curve in one
launch instead of one launch per sector.

* a pooled block's eigenvalues equal the sector-by-sector solve bit for bit
  (one CTA per matrix, whatever else shares the launch);
* the grand-canonical sums equal the immediate path's to rounding (only the
  accumulation order changes), on an FTLM + exact curve and an all-exact one;
* the curve's exact blocks take one dense-solver launch: the launch count
  drops by the number of sectors with exact blocks, minus one;
* implicit flushes: ftlm_block_spectrum of a pooled block, ftlm_thermo_read,
  ftlm_exact_defer(0), and a thermo reconfiguration (queued sums go to the
  accumulators they were queued for, which the reset then clears).
"""
import numpy as np
import pytest

from ftlm_extended_hubbard_development_b200.engine import Engine, Model, RunOpts, linspace

pytestmark = pytest.mark.gpu

MODEL = Model(lx=4, ly=2, tx=1.0, ty=1.0, tp=-0.25, phix=0.3, phiy=0.1, u=7.0, v=1.0)
BETAS = [20.0, 2.0]
MU = linspace(-5.0, 15.0, 61)
OPTS = RunOpts(samples=8, lanczos_steps=60)


def _blocks(info, lx):
    return [(k % lx, k // lx) for k, d in enumerate(info.block_dims) if d > 0]


def _curve(eng, defer, ed=False):
    eng.thermo_configure(BETAS, MU)
    eng.exact_defer(defer)
    sectors_with_exact = 0
    for nu in range(MODEL.sites + 1):
        for nd in range(MODEL.sites + 1):
            info = eng.sector_prepare(nu, nd)
            blocks = _blocks(info, MODEL.lx)
            exact = [b for b in blocks if ed or info.block_dims[b[1] * MODEL.lx + b[0]] <= OPTS.exact_block_threshold]
            sectors_with_exact += bool(exact)
            eng.blocks_exact_batched(exact)
            eng.blocks_ftlm_batched([b for b in blocks if b not in exact])
            for b in blocks:
                eng.thermo_accumulate_block(*b)
    out = eng.thermo_read()
    eng.exact_defer(False)
    return out, sectors_with_exact


def _close(a, b):
    emin_a, z_a, n_a, n2_a = a
    emin_b, z_b, n_b, n2_b = b
    assert np.array_equal(emin_a, emin_b)  # minima do not depend on order
    for x, y in ((z_a, z_b), (n_a, n_b), (n2_a, n2_b)):
        assert np.abs(x - y).max() <= 1e-13 * np.abs(y).max()


@pytest.mark.parametrize("ed", [False, True])
def test_pooled_curve_equals_sector_by_sector(ed):
    with Engine(MODEL, OPTS) as a, Engine(MODEL, OPTS) as b:
        a.profile(True)
        b.profile(True)
        ref, nsec = _curve(a, False, ed)
        got, _ = _curve(b, True, ed)
        la, lb = a.profile()["kernel_launches"], b.profile()["kernel_launches"]
    _close(got, ref)
    assert nsec > 10
    assert la - lb == nsec - 1, (la, lb, nsec)


def test_pooled_spectra_bit_identical_and_flushes():
    with Engine(MODEL, OPTS) as a, Engine(MODEL, OPTS) as b:
        a.thermo_configure(BETAS, MU)
        b.thermo_configure(BETAS, MU)
        b.exact_defer(True)
        for nu, nd in ((2, 1), (3, 3), (4, 2)):
            ia = a.sector_prepare(nu, nd)
            ib = b.sector_prepare(nu, nd)
            blocks = _blocks(ia, MODEL.lx)
            assert ia.block_dims == ib.block_dims
            a.blocks_exact_batched(blocks)
            b.blocks_exact_batched(blocks)
            for blk in blocks:
                a.thermo_accumulate_block(*blk)
                b.thermo_accumulate_block(*blk)
        # the last sector's blocks are still pooled: reading one solves the pool
        for blk in blocks:
            ea, _, pa = a.block_spectrum(*blk, exact=True)
            eb, _, pb = b.block_spectrum(*blk, exact=True)
            assert pa == pb == 1.0
            assert np.array_equal(ea, eb)
        _close(b.thermo_read(), a.thermo_read())
        # reconfiguring flushes the queued sums into the old accumulators, then resets them
        info = b.sector_prepare(3, 2)
        blocks = _blocks(info, MODEL.lx)
        b.blocks_exact_batched(blocks)
        for blk in blocks:
            b.thermo_accumulate_block(*blk)
        b.thermo_configure(BETAS, MU)
        emin, z, _, _ = b.thermo_read()
        assert np.all(np.isinf(emin)) and np.all(z == 0.0)
        b.exact_defer(False)
