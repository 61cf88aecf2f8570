"""Pin the restated C oracle against golden vectors dumped from the reference.

The oracle is the checker for every GPU parity test, so it is itself checked
here, on the CPU, against the reference's own outputs (tests/golden/):
integer/index objects bit-exact, floating-point objects to rounding.
"""
import math
import os

import numpy as np
import pytest

import pyoracle as O
from conftest import GOLDEN, read_csv


def test_seed_mixer_matches_reference_block_seeds(golden):
    for key in golden.lanczos.files:
        if key.endswith("/lanczos_meta"):
            case, blk, _ = key.split("/")
            nu, nd, mx, my = map(int, blk.split("_"))
            want = int(golden.lanczos[key][2]) & (2**64 - 1)
            assert O.block_seed(12345, nu, nd, mx, my) == want


def test_sector_basis_and_relations_bit_exact(golden):
    checked = 0
    for case, nu, nd in golden.sector_keys():
        m = golden.model(case)
        up, dn, deg, diag = O.sector_parents(m, nu, nd)
        assert np.array_equal(up, golden.sec(case, nu, nd, "parent_up")), (case, nu, nd)
        assert np.array_equal(dn, golden.sec(case, nu, nd, "parent_down"))
        assert np.array_equal(deg, golden.sec(case, nu, nd, "parent_deg"))
        assert np.array_equal(diag, golden.sec(case, nu, nd, "parent_diag"))
        par, sh, sg = O.sector_relations(m, nu, nd)
        assert np.array_equal(par, golden.sec(case, nu, nd, "rel_parent"))
        assert np.array_equal(sh, golden.sec(case, nu, nd, "rel_shift"))
        assert np.array_equal(sg, golden.sec(case, nu, nd, "rel_sign"))
        checked += 1
    assert checked > 150


def test_block_csr_matches_reference(golden):
    for case, nu, nd in golden.sector_keys():
        m = golden.model(case)
        dims = golden.sec(case, nu, nd, "block_dim")
        i = 0
        for my in range(m.ly):
            for mx in range(m.lx):
                c = O.block_csr(m, nu, nd, mx, my)
                t = f"_k{mx}_{my}"
                assert c.dim == dims[i]
                i += 1
                if c.dim == 0:
                    continue
                assert np.array_equal(c.row_ptr, golden.sec(case, nu, nd, "row_ptr" + t))
                assert np.array_equal(c.col, golden.sec(case, nu, nd, "col" + t))
                ref = golden.sec(case, nu, nd, "val" + t).view(np.complex128)
                assert np.max(np.abs(c.val - ref), initial=0.0) <= 1e-14
                assert np.array_equal(c.diag, golden.sec(case, nu, nd, "diag" + t))


def test_start_vectors_alpha_beta_and_spectra(golden):
    for case, nu, nd, mx, my, samples, steps in golden.meta["lanczos_dumps"]:
        m = golden.model(case)
        c = O.block_csr(m, nu, nd, mx, my)
        seed = O.block_seed(12345, nu, nd, mx, my)
        kdim = min(steps, c.dim)
        starts = golden.lz(case, nu, nd, mx, my, "start").view(np.complex128).reshape(samples, -1)
        A = golden.lz(case, nu, nd, mx, my, "alpha").reshape(samples, kdim)
        B = golden.lz(case, nu, nd, mx, my, "beta").reshape(samples, kdim)
        nsteps = golden.lz(case, nu, nd, mx, my, "steps")
        ritz = golden.lz(case, nu, nd, mx, my, "ritz")
        wts = golden.lz(case, nu, nd, mx, my, "weights")
        off = 0
        for s in range(samples):
            sv = O.start_vector(seed, s, c.dim)
            assert np.array_equal(sv, starts[s])
            a, b = O.lanczos(c, sv, kdim)
            assert len(a) == nsteps[s]
            assert np.array_equal(a, A[s, : len(a)])
            assert np.array_equal(b, B[s, : len(b)])
            ev, w = O.tridiag_jacobi(a, b)
            n = len(a)
            assert np.array_equal(ev, ritz[off: off + n])
            assert np.allclose(w / samples, wts[off: off + n], rtol=0, atol=1e-15)
            off += n


def test_exact_eigenvalues_match_reference(golden):
    for case, nu, nd, mx, my in golden.meta["exact_dumps"]:
        m = golden.model(case)
        ev = O.block_exact(O.block_csr(m, nu, nd, mx, my))
        ref = golden.exact[f"{case}/{nu}_{nd}_{mx}_{my}/exact"]
        assert np.allclose(ev, ref, rtol=0, atol=1e-12 * max(1.0, np.abs(ref).max()))


def _cli_to_run(args):
    """Parse the reference flags used by the golden CLI runs."""
    kv = {}
    it = iter(args)
    for a in it:
        kv[a[2:]] = next(it)
    m = O.Model(lx=int(kv.get("lx", 2)), ly=int(kv.get("ly", 2)), tx=float(kv.get("tx", 1)),
                ty=float(kv.get("ty", 1)), tp=float(kv.get("tp", 0)),
                phix=float(kv.get("phix", 1)), phiy=float(kv.get("phiy", 1)),
                u=float(kv.get("u", 8)), v=float(kv.get("v", 0)))
    betas = [float(x) for x in kv["beta-list"].split(",")] if "beta-list" in kv else \
        [float(kv.get("beta", 2.0))]
    mu = O.linspace(float(kv.get("mu-min", -4)), float(kv.get("mu-max", 10)),
                    int(kv.get("mu-count", 61)))
    opts = dict(samples=int(kv.get("samples", 5)), steps=int(kv.get("lanczos-steps", 80)),
                threshold=int(kv.get("exact-block-threshold", 256)), seed=int(kv.get("seed", 12345)))
    return m, betas, mu, opts


@pytest.mark.parametrize("name", ["config1", "config1_t0", "config1_multibeta", "config1_ed",
                                  "c3x2_t0", "c3x2_ed", "config2_ed"])
def test_oracle_curve_matches_reference_csv(golden, name):
    run = golden.meta["cli_runs"][name]
    m, betas, mu, opts = _cli_to_run(run["args"])
    ed = run["exe"] == "ftlm_ed_n_vs_mu"
    if ed:
        betas = betas[:1]
    res = O.run_curve(m, betas, mu, ed=ed, **opts)
    header, ref = read_csv(os.path.join(GOLDEN, "csv", name + ".csv"))
    cols = ["n", "charge_correlation", "compressibility", "partition_like", "log_partition"]
    for ib in range(len(betas)):
        rows = ref[ib * len(mu):(ib + 1) * len(mu)]
        mucol = header.index("mu")
        assert np.allclose(rows[:, mucol], mu, rtol=0, atol=1e-14)
        for c in cols:
            got = res[c][ib]
            want = rows[:, header.index(c)]
            tol = 1e-10 * np.maximum(1.0, np.abs(want))
            assert np.all(np.abs(got - want) <= tol), (name, c)


def test_translate_sign_is_a_group_action():
    """T_a T_b = T_{a+b} with multiplicative signs, on a 4x3 torus."""
    lx, ly = 4, 3
    rng = np.random.default_rng(1)
    for _ in range(200):
        bits = int(rng.integers(0, 2**12))
        for a in range(lx * ly):
            for b in (1, 5, 7):
                ax, ay, bx, by = a % lx, a // lx, b % lx, b // lx
                t1, s1 = O.translate_spin(bits, bx, by, lx, ly)
                t2, s2 = O.translate_spin(t1, ax, ay, lx, ly)
                t3, s3 = O.translate_spin(bits, (ax + bx) % lx, (ay + by) % ly, lx, ly)
                assert t2 == t3 and s1 * s2 == s3
