"""Every H*V kernel instantiation the engine launches, through the C ABI,
against the oracle CSR (apply_hamiltonian, main.cpp:833-845) on blocks large
enough (>= 2^15 rows) that the autotuner itself runs.

* on-the-fly kernel `k_hv`, all five (gather unroll, CTAs per SM) variants
  and the autotuner's own choice: bit-identical to each other, and equal to
  the oracle CSR within 1e-13 (FP64) / 2e-6 (FP32 vectors) of max |H x|;
* cached hop list `k_hv_list` (all variants) and the narrow-sweep row kernel
  `k_hv_rows`: the same bars;
* split-spin segment sweeps (both row orders, the spin-flip gather/scatter;
  sector (3,4) has a separate flipped sector (4,3), sector (3,3) is its own),
  with the class stencils (`k_hv_stn`, mode "split") and with on-the-fly
  lookups (`k_hv_seg`, mode "splitfly"): the same bars against the oracle,
  bit-identical across variants although each variant runs its own grid and
  rows are taken from a shared counter in whatever order the warps get them;
* Lanczos alpha/beta identical across variants and equal to the oracle's
  Lanczos from the same start vectors (1e-10 FP64 before the horizon).

Blocks: 4x4 t'=-0.25 V=1 twisted (0.3, 0.7), sector (3,4), k=(1,0), dim 63,700
(up to 56 hops per row, so rows take a second 32-hop round); 6x3 t'=0.2
U=8 V=1.5 twisted (0.25, 0.5), sector (3,3), k=(1,0), dim 36,990 (has hops
to inactive orbits).
"""
import numpy as np
import pytest

import pyoracle as O

import ftlm_extended_hubbard_development_b200 as pkg
from ftlm_extended_hubbard_development_b200 import engine as E

pytestmark = pytest.mark.gpu

BLOCKS = [("c4x4", 3, 4, 1, 0), ("c6x3", 3, 3, 1, 0)]
VARIANTS = [None, 0, 1, 2, 3, 4]  # None: the autotuner (FTLM_HV_RETUNE=1 forces a fresh run)


def model_of(golden, case):
    c = golden.cases[case]
    return pkg.Model(lx=c["lx"], ly=c["ly"], tp=c["tp"], phix=c["phix"], phiy=c["phiy"], u=c["u"], v=c["v"])


@pytest.fixture(scope="module")
def csrs(golden):
    out = {}
    for case, nu, nd, mx, my in BLOCKS:
        m = model_of(golden, case)
        out[(case, nu, nd, mx, my)] = O.block_csr(O.Model(**m.__dict__), nu, nd, mx, my)
    return out


def set_variant(monkeypatch, var):
    if var is None:
        monkeypatch.delenv("FTLM_HV_VARIANT", raising=False)
        monkeypatch.setenv("FTLM_HV_RETUNE", "1")
    else:
        monkeypatch.setenv("FTLM_HV_VARIANT", str(var))
        monkeypatch.delenv("FTLM_HV_RETUNE", raising=False)


def test_blocks_exercise_the_tuner_and_long_rows(csrs):
    for key, csr in csrs.items():
        assert csr.dim >= 1 << 15, key
        per_row = np.add.reduceat(csr.val != 0, csr.row_ptr[:-1])
        assert per_row.max() > 32, key


CASES = [("fly", E.PREC_FP64, 16), ("fly", E.PREC_MIXED, 128), ("fly", E.PREC_FP64, 128),
         ("fly", E.PREC_MIXED, 8), ("list", E.PREC_FP64, 16), ("list", E.PREC_MIXED, 32),
         ("list", E.PREC_MIXED, 2), ("list", E.PREC_FP64, 1), ("split", E.PREC_FP64, 16),
         ("split", E.PREC_MIXED, 128), ("split", E.PREC_FP64, 128), ("split", E.PREC_MIXED, 16),
         ("split", E.PREC_MIXED, 2), ("split", E.PREC_FP64, 1), ("split", E.PREC_MIXED, 4),
         ("split", E.PREC_MIXED, 8), ("split", E.PREC_FP64, 4), ("splitfly", E.PREC_FP64, 16),
         ("splitfly", E.PREC_MIXED, 128), ("splitfly", E.PREC_MIXED, 2)]


def set_mode(monkeypatch, mode):
    monkeypatch.setenv("FTLM_HV_MODE", "split" if mode == "splitfly" else mode)
    if mode == "splitfly":
        monkeypatch.setenv("FTLM_SPLIT_OP", "fly")
    else:
        monkeypatch.delenv("FTLM_SPLIT_OP", raising=False)


@pytest.mark.parametrize("mode,prec,nvec", CASES)
def test_hv_variants_bit_identical_and_match_oracle(golden, csrs, monkeypatch, mode, prec, nvec):
    set_mode(monkeypatch, mode)
    rng = np.random.default_rng(11)
    tol = 1e-13 if prec == E.PREC_FP64 else 2e-6
    row_bytes = nvec * (8 if prec == E.PREC_MIXED else 16)
    # the 8-lanes-per-row kernels have no variants to tune
    rows_kernel = (mode == "list" and row_bytes == 16) or (mode == "split" and max(row_bytes, 16) <= 64)
    for (case, nu, nd, mx, my), csr in csrs.items():
        m = model_of(golden, case)
        x = rng.standard_normal((csr.dim, nvec)) + 1j * rng.standard_normal((csr.dim, nvec))
        if prec == E.PREC_MIXED:
            x = x.astype(np.complex64).astype(np.complex128)
        want = np.stack([csr.apply(x[:, v]) for v in range(nvec)], 1)
        scale = np.abs(want).max()
        got = {}
        for var in VARIANTS:
            set_variant(monkeypatch, var)
            with pkg.Engine(m, pkg.RunOpts(precision=prec)) as eng:
                eng.sector_prepare(nu, nd)
                eng.profile(True)
                eng.profile_reset()
                got[var] = eng.block_apply(mx, my, x)
                prof = eng.profile()
            assert prof["hv_source"] == {"fly": 0, "list": 1, "split": 2, "splitfly": 2}[mode]
            if var is None and not rows_kernel:
                assert prof["tune_runs"] == 1, (case, mode, nvec)  # the tuner measured this block
            assert 0 <= prof["hv_variant"] < 5
            err = np.abs(got[var] - want).max()
            assert err <= tol * scale, (case, mode, prec, nvec, var, err / scale)
        for var in VARIANTS[1:]:
            assert np.array_equal(got[var], got[VARIANTS[0]]), (case, mode, nvec, var)


@pytest.mark.parametrize("prec,nvec,tol", [(E.PREC_FP64, 16, 1e-14), (E.PREC_MIXED, 32, 1e-6)])
def test_hop_list_agrees_with_on_the_fly_on_large_block(golden, csrs, monkeypatch, prec, nvec, tol):
    """The list holds only hops to active targets; the on-the-fly kernel
    queues every hop and zeroes the inactive ones, so where a block has
    inactive targets the two assign hops to lane groups differently and agree
    to rounding (bit-identical where every target is active:
    test_gpu_parity.py::test_cached_hop_list_equals_on_the_fly)."""
    monkeypatch.setenv("FTLM_HV_ROWS", "0")
    monkeypatch.setenv("FTLM_HV_VARIANT", "4")
    rng = np.random.default_rng(5)
    for (case, nu, nd, mx, my), csr in csrs.items():
        m = model_of(golden, case)
        x = rng.standard_normal((csr.dim, nvec)) + 1j * rng.standard_normal((csr.dim, nvec))
        out = {}
        for mode in ("fly", "list"):
            monkeypatch.setenv("FTLM_HV_MODE", mode)
            with pkg.Engine(m, pkg.RunOpts(precision=prec)) as eng:
                eng.sector_prepare(nu, nd)
                out[mode] = eng.block_apply(mx, my, x)
        assert np.abs(out["fly"] - out["list"]).max() <= tol * np.abs(out["fly"]).max(), case


@pytest.mark.parametrize("mode,prec,batch", [("fly", E.PREC_FP64, 16), ("fly", E.PREC_MIXED, 128),
                                             ("list", E.PREC_FP64, 8), ("split", E.PREC_FP64, 16),
                                             ("split", E.PREC_MIXED, 128), ("splitfly", E.PREC_FP64, 16)])
def test_lanczos_variants_identical_and_match_oracle(golden, csrs, monkeypatch, mode, prec, batch):
    """Alpha/beta of every variant bit-identical; against the oracle's
    Lanczos (main.cpp:1027-1060) from the same start vectors: 1e-10 relative
    (FP64) / 1e-5 (FP32 vectors) over the first 12 steps, well before the
    reproducibility horizon of these blocks."""
    set_mode(monkeypatch, mode)
    case, nu, nd, mx, my = BLOCKS[0]
    csr = csrs[BLOCKS[0]]
    m = model_of(golden, case)
    steps = 12
    seed = O.block_seed(12345, nu, nd, mx, my)
    starts = np.stack([O.start_vector(seed, s, csr.dim) for s in range(batch)])
    ref_a = np.zeros((batch, steps))
    ref_b = np.zeros((batch, steps))
    for s in range(batch):
        a, b = O.lanczos(csr, starts[s], steps)
        ref_a[s, :len(a)] = a
        ref_b[s, :len(b)] = b
    res = {}
    for var in VARIANTS:
        set_variant(monkeypatch, var)
        opts = pkg.RunOpts(samples=batch, lanczos_steps=steps, exact_block_threshold=0, precision=prec,
                           batch_vectors=batch)
        with pkg.Engine(m, opts) as eng:
            eng.sector_prepare(nu, nd)
            res[var] = eng.block_lanczos(mx, my, start=starts)
    a0, b0, s0 = res[VARIANTS[0]][:3]
    for var in VARIANTS[1:]:
        a, b, s = res[var][:3]
        assert np.array_equal(a, a0) and np.array_equal(b, b0) and np.array_equal(s, s0), var
    tol = 1e-10 if prec == E.PREC_FP64 else 1e-5
    assert np.all(s0 == steps)
    assert np.all(np.abs(a0 - ref_a) <= tol * np.maximum(1.0, np.abs(ref_a)))
    rb = ref_b[:, :steps - 1]
    assert np.all(np.abs(b0[:, :steps - 1] - rb) <= tol * np.maximum(1.0, np.abs(rb)))


@pytest.mark.parametrize("prec,batch,tol", [(E.PREC_FP64, 16, 1e-12), (E.PREC_MIXED, 64, 2e-5)])
def test_split_lanczos_agrees_with_on_the_fly(golden, monkeypatch, prec, batch, tol):
    """The split sweeps sum a row's up- and down-spin hops in two passes, so
    alpha/beta agree with the single-pass kernel to rounding, on both
    blocks (one with a separate flipped sector)."""
    for case, nu, nd, mx, my in BLOCKS:
        m = model_of(golden, case)
        opts = pkg.RunOpts(samples=batch, lanczos_steps=20, exact_block_threshold=0, precision=prec,
                           batch_vectors=batch, start_vector=E.START_PHILOX_PHASE)
        out = {}
        for mode in ("fly", "split", "splitfly"):
            set_mode(monkeypatch, mode)
            with pkg.Engine(m, opts) as eng:
                eng.sector_prepare(nu, nd)
                out[mode] = eng.block_lanczos(mx, my)
        af, bf, sf = out["fly"][:3]
        for mode in ("split", "splitfly"):
            as_, bs, ss = out[mode][:3]
            assert np.array_equal(sf, ss)
            n = 10  # well before the reproducibility horizon
            assert np.abs(as_[:, :n] - af[:, :n]).max() <= tol * np.abs(af[:, :n]).max(), (case, mode)
            assert np.abs(bs[:, :n] - bf[:, :n]).max() <= tol * np.abs(bf[:, :n]).max(), (case, mode)
