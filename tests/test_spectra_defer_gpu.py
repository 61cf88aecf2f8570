"""Block spectra pooled across sectors (ftlm_spectra_defer / ftlm_spectra_flush):
the dense solver diagonalises the exact blocks of a whole curve in one launch
and the Ritz stage of its small FTLM blocks runs in one more, instead of one
of each per sector.

* a pooled block's spectrum equals the sector-by-sector one bit for bit
  (one CTA per matrix, one per 32 vectors of a block, whatever else shares
  the launch), for exact and for FTLM blocks;
* the grand-canonical sums equal the immediate path's to rounding (only the
  accumulation order changes), on an FTLM + exact curve and an all-exact one;
* the launch count drops by the per-sector launches the pool replaces: one
  dense-solver launch per sector with exact blocks and two Ritz-stage
  launches per sector with small FTLM blocks, less the pool's own;
* implicit flushes: ftlm_block_spectrum of a pooled block, ftlm_thermo_read,
  ftlm_spectra_defer(0), and a thermo reconfiguration (queued sums go to the
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
    eng.spectra_defer(defer)
    n_exact = n_small = 0  # sectors with exact / small FTLM blocks
    for nu in range(MODEL.sites + 1):
        for nd in range(MODEL.sites + 1):
            info = eng.sector_prepare(nu, nd)
            blocks = _blocks(info, MODEL.lx)
            exact = [b for b in blocks if ed or info.block_dims[b[1] * MODEL.lx + b[0]] <= OPTS.exact_block_threshold]
            ftlm = [b for b in blocks if b not in exact]
            n_exact += bool(exact)
            n_small += bool(ftlm)  # every block of a 4x2 lattice is small (<= 4096 rows)
            eng.blocks_exact_batched(exact)
            eng.blocks_ftlm_batched(ftlm)
            for b in blocks:
                eng.thermo_accumulate_block(*b)
    out = eng.thermo_read()
    eng.spectra_defer(False)
    return out, n_exact, n_small


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
        ref, n_exact, n_small = _curve(a, False, ed)
        got, _, _ = _curve(b, True, ed)
        la, lb = a.profile()["kernel_launches"], b.profile()["kernel_launches"]
    _close(got, ref)
    assert n_exact > 10 and (ed or n_small > 5)  # 4x2 at threshold 256: 72 and 9 sectors
    assert la - lb == max(n_exact - 1, 0) + 2 * max(n_small - 1, 0), (la, lb, n_exact, n_small)


def test_pooled_spectra_bit_identical_and_flushes():
    opts = RunOpts(samples=8, lanczos_steps=60, exact_block_threshold=240)
    # (2, 1): exact blocks; (3, 3): small FTLM blocks; (4, 2): both (dims 236 and 248)
    sectors = ((2, 1), (3, 3), (4, 2))
    with Engine(MODEL, opts) as a, Engine(MODEL, opts) as b:
        a.thermo_configure(BETAS, MU)
        b.thermo_configure(BETAS, MU)
        b.spectra_defer(True)
        for nu, nd in sectors:
            ia = a.sector_prepare(nu, nd)
            ib = b.sector_prepare(nu, nd)
            assert ia.block_dims == ib.block_dims
            blocks = _blocks(ia, MODEL.lx)
            exact = [k for k in blocks if ia.block_dims[k[1] * MODEL.lx + k[0]] <= 240]
            ftlm = [k for k in blocks if k not in exact]
            for eng in (a, b):
                eng.blocks_exact_batched(exact)
                eng.blocks_ftlm_batched(ftlm)
                for blk in blocks:
                    eng.thermo_accumulate_block(*blk)
        assert exact and ftlm
        # the last sector's blocks are still pooled: reading one solves the pool
        for blk in blocks:
            is_exact = blk in exact
            ea, wa, pa = a.block_spectrum(*blk, exact=is_exact)
            eb, wb, pb = b.block_spectrum(*blk, exact=is_exact)
            assert pa == pb
            assert np.array_equal(ea, eb)
            if not is_exact:
                assert np.array_equal(wa, wb)
        _close(b.thermo_read(), a.thermo_read())
        # reconfiguring flushes the queued sums into the old accumulators, then resets them
        info = b.sector_prepare(3, 3)
        blocks = _blocks(info, MODEL.lx)
        b.blocks_exact_batched(blocks[:2])
        b.blocks_ftlm_batched(blocks[2:])
        for blk in blocks:
            b.thermo_accumulate_block(*blk)
        b.thermo_configure(BETAS, MU)
        emin, z, _, _ = b.thermo_read()
        assert np.all(np.isinf(emin)) and np.all(z == 0.0)
        b.spectra_defer(False)
