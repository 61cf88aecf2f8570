"""GPU parity: the CUDA engine, called through the C ABI, against the oracle
and the reference's golden vectors.

Tolerances (FP64 GPU vs reference CPU):
  * basis, relations, block dimensions, CSR structure: bit-exact
  * CSR values, H*V:                     <= 1e-13 relative (FP64), 2e-6 (mixed)
  * Lanczos alpha/beta:                  <= 1e-10 relative before the
                                          reproducibility horizon
  * per-block Z(beta, mu), CSV n, chi:   <= 1e-10 (relative for Z)
  * exact eigenvalues:                   <= 1e-12 * max(1, |E|max)
"""
import math
import os
import subprocess

import numpy as np
import pytest

import pyoracle as O
from conftest import GOLDEN, read_csv

import ftlm_extended_hubbard_development_b200 as pkg
from ftlm_extended_hubbard_development_b200 import engine as E

pytestmark = pytest.mark.gpu
BIN = E.BIN_DIR


def model_of(golden, case):
    c = golden.cases[case]
    return pkg.Model(lx=c["lx"], ly=c["ly"], tp=c["tp"], phix=c["phix"], phiy=c["phiy"], u=c["u"], v=c["v"])


def omodel(m):
    return O.Model(**m.__dict__)


@pytest.fixture(scope="module")
def sectors_by_case(golden):
    out = {}
    for case, nu, nd in golden.sector_keys():
        out.setdefault(case, []).append((nu, nd))
    return out


def test_loaded_device_code_is_sm100():
    """The runtime loaded this library's SASS for compute capability 10.0,
    compiled from the sm_100 virtual architecture."""
    import ctypes as C
    lib = pkg.load_library()
    bv, pv = C.c_int32(0), C.c_int32(-1)
    assert lib.ftlm_device_code_version(0, C.byref(bv), C.byref(pv)) == 0
    assert bv.value == 100 and pv.value == 100, (bv.value, pv.value)


def test_sector_basis_relations_and_csr_bit_exact(golden, sectors_by_case):
    checked_blocks = 0
    for case, secs in sectors_by_case.items():
        m = model_of(golden, case)
        with pkg.Engine(m, pkg.RunOpts()) as eng:
            for nu, nd in secs:
                info = eng.sector_prepare(nu, nd)
                assert info.full_dim == int(golden.sec(case, nu, nd, "sector_meta")[0])
                assert info.parents == int(golden.sec(case, nu, nd, "sector_meta")[1])
                up, dn, deg, diag = eng.debug_sector_parents()
                assert np.array_equal(up, golden.sec(case, nu, nd, "parent_up")), (case, nu, nd)
                assert np.array_equal(dn, golden.sec(case, nu, nd, "parent_down"))
                assert np.array_equal(deg, golden.sec(case, nu, nd, "parent_deg"))
                assert np.array_equal(diag, golden.sec(case, nu, nd, "parent_diag"))
                par, sh, sg = eng.debug_sector_relations(info.full_dim)
                assert np.array_equal(par, golden.sec(case, nu, nd, "rel_parent"))
                assert np.array_equal(sh, golden.sec(case, nu, nd, "rel_shift"))
                assert np.array_equal(sg, golden.sec(case, nu, nd, "rel_sign"))
                assert np.array_equal(np.array(info.block_dims, np.int64), golden.sec(case, nu, nd, "block_dim"))
                for my in range(m.ly):
                    for mx in range(m.lx):
                        if info.block_dims[my * m.lx + mx] == 0:
                            continue
                        t = f"_k{mx}_{my}"
                        d, rp, col, val = eng.debug_block_csr(mx, my)
                        assert np.array_equal(rp, golden.sec(case, nu, nd, "row_ptr" + t))
                        assert np.array_equal(col, golden.sec(case, nu, nd, "col" + t))
                        ref = golden.sec(case, nu, nd, "val" + t).view(np.complex128)
                        assert np.abs(val - ref).max(initial=0.0) <= 1e-13
                        assert np.array_equal(d, golden.sec(case, nu, nd, "diag" + t))
                        checked_blocks += 1
    assert checked_blocks > 500


HV_CASES = [("c3x2", 2, 2), ("c3x3", 4, 5), ("c4x2t", 4, 4), ("c4x4", 2, 2), ("c4x4", 4, 0),
            ("c2x3", 3, 3), ("c6x3", 1, 2), ("c4x1", 2, 1), ("c1x4", 1, 2)]


@pytest.mark.parametrize("prec", [E.PREC_FP64, E.PREC_MIXED])
def test_block_apply_matches_oracle_csr(golden, prec):
    rng = np.random.default_rng(7)
    for case, nu, nd in HV_CASES:
        m = model_of(golden, case)
        with pkg.Engine(m, pkg.RunOpts(precision=prec)) as eng:
            info = eng.sector_prepare(nu, nd)
            for k, dim in enumerate(info.block_dims):
                if dim == 0:
                    continue
                mx, my = k % m.lx, k // m.lx
                csr = O.block_csr(omodel(m), nu, nd, mx, my)
                for nvec in (1, 3, 16, 128):
                    x = rng.standard_normal((dim, nvec)) + 1j * rng.standard_normal((dim, nvec))
                    if prec == E.PREC_MIXED:
                        x = x.astype(np.complex64).astype(np.complex128)
                    y = eng.block_apply(mx, my, x)
                    want = np.stack([csr.apply(x[:, v]) for v in range(nvec)], 1)
                    scale = np.abs(want).max() + 1e-30
                    tol = 1e-13 if prec == E.PREC_FP64 else 2e-6
                    assert np.abs(y - want).max() <= tol * scale, (case, nu, nd, mx, my, nvec)


def twin_horizon(csr, start, ref_alpha, tol=1e-11):
    """First step at which a perturbed-start twin run of the oracle departs
    from the reference alphas: the reproducibility horizon of this block.
    The 1e-13 start perturbation stands for the rounding differences of a
    different summation order (loss of orthogonality amplifies any of them
    exponentially once it sets in)."""
    rng = np.random.default_rng(3)
    pert = start * (1.0 + 1e-13 * rng.standard_normal(start.shape))
    pert /= np.linalg.norm(pert)
    a, _ = O.lanczos(csr, pert, len(ref_alpha))
    n = min(len(a), len(ref_alpha))
    bad = np.nonzero(np.abs(a[:n] - ref_alpha[:n]) > tol * np.maximum(1.0, np.abs(ref_alpha[:n])))[0]
    return int(bad[0]) if len(bad) else n


@pytest.mark.parametrize("batch", [0, 1])
def test_lanczos_alpha_beta_before_horizon_and_block_z(golden, batch):
    for case, nu, nd, mx, my, samples, steps in golden.meta["lanczos_dumps"]:
        m = model_of(golden, case)
        csr = O.block_csr(omodel(m), nu, nd, mx, my)
        kdim = min(steps, csr.dim)
        starts = golden.lz(case, nu, nd, mx, my, "start").view(np.complex128).reshape(samples, -1)
        A = golden.lz(case, nu, nd, mx, my, "alpha").reshape(samples, kdim)
        B = golden.lz(case, nu, nd, mx, my, "beta").reshape(samples, kdim)
        nsteps = golden.lz(case, nu, nd, mx, my, "steps")
        opts = pkg.RunOpts(samples=samples, lanczos_steps=steps, exact_block_threshold=0, batch_vectors=batch)
        with pkg.Engine(m, opts) as eng:
            eng.sector_prepare(nu, nd)
            a, b, s = eng.block_lanczos(mx, my, start=starts)
            for r in range(samples):
                n = min(s[r], nsteps[r])
                if s[r] != nsteps[r]:
                    # A breakdown decision (beta < 1e-12) may flip only when the
                    # reference's beta there is rounding noise: Lanczos ran to the
                    # full dimension of a tiny block.
                    assert n == kdim - 1 and B[r, n - 1] < 1e-9, (case, r, s[r], nsteps[r])
                h = min(twin_horizon(csr, starts[r], A[r, :n]), n)
                assert h >= min(10, n)
                ra, rb = A[r, :h], B[r, : max(h - 1, 0)]
                assert np.all(np.abs(a[r, :h] - ra) <= 1e-10 * np.maximum(1.0, np.abs(ra))), (case, r, h)
                assert np.all(np.abs(b[r, : len(rb)] - rb) <= 1e-10 * np.maximum(1.0, np.abs(rb)))
            # whole-block spectra: Z(beta, mu) against the reference's run_ftlm_block
            ev, w, pref = eng.block_spectrum(mx, my, exact=False)
        ritz = golden.lz(case, nu, nd, mx, my, "ritz")
        wts = golden.lz(case, nu, nd, mx, my, "weights")
        assert pref == csr.dim and abs(len(ev) - len(ritz)) <= samples
        N = nu + nd
        for beta in (1.0, 5.0, 20.0):
            for mu in (-2.0, 1.0, 4.0):
                def z(e, ww):
                    sh = e - mu * N
                    return np.sum(pref * ww * np.exp(-beta * (sh - sh.min())))
                zr, zg = z(ritz, wts), z(ev, w)
                assert abs(zg - zr) <= 1e-10 * zr, (case, beta, mu)


def test_profile_counters_and_byte_model(golden):
    """The instrumented path (CUDA-event timing, nonzero-hop count of the
    byte model) on a block whose CSR is known."""
    m = model_of(golden, "c4x2t")
    opts = pkg.RunOpts(samples=4, lanczos_steps=30, precision=E.PREC_MIXED, start_vector=E.START_PHILOX_PHASE)
    with pkg.Engine(m, opts) as eng:
        info = eng.sector_prepare(4, 4)
        eng.profile(True)
        eng.profile_reset()
        eng.block_spectrum(0, 0, fetch=False)
        p = eng.profile()
    D = info.block_dims[0]
    csr = O.block_csr(omodel(m), 4, 4, 0, 0)
    nz = int(np.count_nonzero(csr.val))
    K = min(30, D)
    assert p["hv_launches"] == K and p["hv_ms"] > 0 and p["block_ms"] >= p["hv_ms"]
    want = K * (D * 4 * 8 * 2 + nz * 4 * 8 + D * 8)
    assert abs(p["hv_bytes"] - want) <= 1e-9 * want
    assert p["kernel_launches"] >= 4 * K


@pytest.mark.parametrize("prec,batch", [(E.PREC_FP64, 1), (E.PREC_MIXED, 16), (E.PREC_FP64, 4)])
def test_cached_hop_list_equals_on_the_fly(golden, monkeypatch, prec, batch):
    """The cached hop list resolves the same hops in the same order with the
    same coefficient arithmetic as the on-the-fly kernel: identical results."""
    m = model_of(golden, "c4x4")
    opts = pkg.RunOpts(samples=4, lanczos_steps=30, precision=prec, batch_vectors=batch,
                       start_vector=E.START_PHILOX_PHASE)
    monkeypatch.setenv("FTLM_HV_ROWS", "0")  # the warp-per-row list kernel (same sum order)
    out = {}
    for mode in ("fly", "list"):
        monkeypatch.setenv("FTLM_HV_MODE", mode)
        with pkg.Engine(m, opts) as eng:
            eng.sector_prepare(2, 3)
            out[mode] = eng.block_lanczos(1, 2)
    for a, b in zip(out["fly"], out["list"]):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("prec,batch,tol", [(E.PREC_FP64, 1, 1e-12), (E.PREC_MIXED, 2, 2e-5)])
def test_narrow_sweep_row_kernel(golden, monkeypatch, prec, batch, tol):
    """Sweeps of one 16-byte chunk per row on the hop list run 8 lanes per
    row: same alpha/beta as the on-the-fly kernel up to rounding (another sum
    order), deterministic from run to run."""
    m = model_of(golden, "c4x4")
    opts = pkg.RunOpts(samples=4, lanczos_steps=30, precision=prec, batch_vectors=batch,
                       start_vector=E.START_PHILOX_PHASE)
    out = {}
    for key, mode in (("fly", "fly"), ("rows", "list"), ("rows2", "list")):
        monkeypatch.setenv("FTLM_HV_MODE", mode)
        with pkg.Engine(m, opts) as eng:
            eng.sector_prepare(2, 3)
            out[key] = eng.block_lanczos(1, 2)
    for a, b in zip(out["rows"], out["rows2"]):
        assert np.array_equal(a, b)
    (af, bf, sf), (ar, br, sr) = out["fly"][:3], out["rows"][:3]
    assert np.array_equal(sf, sr)
    n = 10  # well before the reproducibility horizon
    assert np.abs(ar[:, :n] - af[:, :n]).max() <= tol * np.abs(af[:, :n]).max()
    assert np.abs(br[:, :n] - bf[:, :n]).max() <= tol * np.abs(bf[:, :n]).max()


def test_exact_eigenvalues_match_reference(golden):
    for case, nu, nd, mx, my in golden.meta["exact_dumps"]:
        m = model_of(golden, case)
        ref = golden.exact[f"{case}/{nu}_{nd}_{mx}_{my}/exact"]
        with pkg.Engine(m, pkg.RunOpts()) as eng:
            eng.sector_prepare(nu, nd)
            ev, _, pref = eng.block_spectrum(mx, my, exact=True)
        assert pref == 1.0
        assert np.abs(ev - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max()), case


def test_batched_exact_equals_single(golden):
    m = model_of(golden, "c3x3")
    with pkg.Engine(m, pkg.RunOpts()) as eng:
        info = eng.sector_prepare(4, 5)
        blocks = [(k % 3, k // 3) for k, d in enumerate(info.block_dims) if d > 0]
        eng.blocks_exact_batched(blocks)
        got = {b: eng.block_spectrum(*b, exact=True)[0] for b in blocks}
    for b in blocks:
        ref = O.block_exact(O.block_csr(omodel(m), 4, 5, *b))
        assert np.abs(got[b] - ref).max() <= 1e-11


def run_cli(exe, args, out, extra=()):
    r = subprocess.run([os.path.join(BIN, exe)] + list(args) + ["--output", str(out)] + list(extra),
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return r


def compare_csv(got_path, ref_path, tol=1e-10):
    h1, a = read_csv(got_path)
    h2, b = read_csv(ref_path)
    assert h1 == h2 and a.shape == b.shape
    for c in ("mu", "n", "charge_correlation", "compressibility"):
        i = h1.index(c)
        assert np.abs(a[:, i] - b[:, i]).max() <= tol, c
    i = h1.index("log_partition")
    assert np.all(np.abs(a[:, i] - b[:, i]) <= tol * np.maximum(1.0, np.abs(b[:, i])))
    if "beta" in h1:
        assert np.array_equal(a[:, 0], b[:, 0])


@pytest.mark.parametrize("name", ["config1", "config1_t0", "config1_multibeta", "config1_ed", "c3x2_t0",
                                  "c3x2_ed", "config2_ed"])
def test_cli_csv_matches_reference(golden, tmp_path, name):
    run = golden.meta["cli_runs"][name]
    out = tmp_path / "out.csv"
    r = run_cli(run["exe"], run["args"], out)
    compare_csv(out, os.path.join(GOLDEN, "csv", name + ".csv"))
    # stdout: sector lines identical to the reference's
    ref_lines = [ln for ln in open(os.path.join(GOLDEN, "csv", name + ".stdout")) if "sector Nup" in ln]
    got_lines = [ln + "\n" for ln in r.stdout.splitlines() if "sector Nup" in ln]
    assert got_lines == ref_lines


def test_config2_ftlm_curve_matches_reference(golden, tmp_path):
    """4x2, 32 samples x 120 steps: far past the reproducibility horizon,
    yet the thermodynamics agree with the reference (main.cpp path)."""
    run = golden.meta["cli_runs"]["config2"]
    out = tmp_path / "c2.csv"
    run_cli(run["exe"], run["args"], out)
    compare_csv(out, os.path.join(GOLDEN, "csv", "config2.csv"), tol=1e-8)


def parse_checkpoint(blob: bytes):
    """Records of a .ftlmcp file (main.cpp:1297-1398 byte layout)."""
    import struct
    assert blob[:8] == b"FTLMCP1\n"
    pos, recs = 8, []
    while pos + 8 <= len(blob) and blob[pos:pos + 8] == b"BLKREC1\n":
        pos += 8
        head = struct.calcsize("<5iQdBQQ")
        if pos + head > len(blob):
            break
        nu, nd, mx, my, part, dim, pref, exact, ne, nw = struct.unpack_from("<5iQdBQQ", blob, pos)
        pos += head
        if pos + 8 * (ne + nw) > len(blob):
            break
        ev = np.frombuffer(blob, np.float64, ne, pos)
        w = np.frombuffer(blob, np.float64, nw, pos + 8 * ne)
        pos += 8 * (ne + nw)
        recs.append(dict(key=(nu, nd, mx, my), particles=part, dim=dim, pref=pref, exact=exact, ev=ev, w=w))
    return recs


def test_checkpoint_resume_and_cross_engine(golden, tmp_path):
    run = golden.meta["checkpoint_run"]
    ck = tmp_path / "run.ftlmcp"
    out1 = tmp_path / "a.csv"
    run_cli(run["exe"], run["args"], out1, ["--checkpoint", str(ck)])
    # .meta identical to the reference's; records in the same order and layout
    assert (tmp_path / "run.ftlmcp.meta").read_bytes() == \
        open(os.path.join(GOLDEN, "csv", "config1_ckpt.ftlmcp.meta"), "rb").read()
    ours, ref = ck.read_bytes(), open(os.path.join(GOLDEN, "csv", "config1_ckpt.ftlmcp"), "rb").read()
    ro, rr = parse_checkpoint(ours), parse_checkpoint(ref)
    assert [r["key"] for r in ro] == [r["key"] for r in rr]
    for a, b in zip(ro, rr):
        assert (a["particles"], a["dim"], a["pref"], a["exact"]) == (b["particles"], b["dim"], b["pref"], b["exact"])
        if a["exact"]:
            assert np.abs(a["ev"] - b["ev"]).max() <= 1e-12 * max(1.0, np.abs(b["ev"]).max())
        else:  # whole-dimension Lanczos on tiny blocks: counts may differ by noise-level breakdowns
            assert abs(len(a["ev"]) - len(b["ev"])) <= 5 and abs(a["w"].sum() - b["w"].sum()) <= 1e-12
    compare_csv(out1, os.path.join(GOLDEN, "csv", "config1_ckpt.csv"))
    # resume from our own checkpoint: byte-identical CSV
    out2 = tmp_path / "b.csv"
    r = run_cli(run["exe"], run["args"], out2, ["--checkpoint", str(ck)])
    assert "loaded_blocks=" in r.stdout
    assert out1.read_bytes() == out2.read_bytes()
    # resume from the reference's checkpoint
    ck2 = tmp_path / "ref.ftlmcp"
    ck2.write_bytes(ref)
    (tmp_path / "ref.ftlmcp.meta").write_bytes(open(os.path.join(GOLDEN, "csv", "config1_ckpt.ftlmcp.meta"), "rb").read())
    out3 = tmp_path / "c.csv"
    run_cli(run["exe"], run["args"], out3, ["--checkpoint", str(ck2)])
    compare_csv(out3, os.path.join(GOLDEN, "csv", "config1_ckpt.csv"))
    # truncated checkpoint: the partial record is ignored, the rest recomputed
    ck3 = tmp_path / "trunc.ftlmcp"
    ck3.write_bytes(ours[: len(ours) // 2 + 3])
    (tmp_path / "trunc.ftlmcp.meta").write_bytes((tmp_path / "run.ftlmcp.meta").read_bytes())
    out4 = tmp_path / "d.csv"
    run_cli(run["exe"], run["args"], out4, ["--checkpoint", str(ck3)])
    compare_csv(out4, os.path.join(GOLDEN, "csv", "config1_ckpt.csv"))


def test_mixed_precision_config2_against_fp64(tmp_path):
    args = ["--lx", "4", "--ly", "2", "--u", "8", "--beta", "20", "--mu-min", "-5", "--mu-max", "15",
            "--mu-count", "81", "--samples", "32", "--lanczos-steps", "120"]
    f64, mix = tmp_path / "f.csv", tmp_path / "m.csv"
    run_cli("ftlm_n_vs_mu", args, f64)
    run_cli("ftlm_n_vs_mu", args, mix, ["--precision", "mixed"])
    h, a = read_csv(f64)
    _, b = read_csv(mix)
    assert np.abs(a[:, h.index("n")] - b[:, h.index("n")]).max() <= 1e-4


def test_philox_start_vectors_estimate_ed(golden, tmp_path):
    run = golden.meta["cli_runs"]["config2_ed"]
    args = run["args"] + ["--samples", "32", "--lanczos-steps", "120", "--start-vector", "philox-phase",
                          "--precision", "mixed"]
    out = tmp_path / "p.csv"
    run_cli("ftlm_n_vs_mu", args, out)
    h, a = read_csv(out)
    _, b = read_csv(os.path.join(GOLDEN, "csv", "config2_ed.csv"))
    assert np.abs(a[:, h.index("n")] - b[:, h.index("n")]).max() <= 0.02


def _read_rows(path):
    with open(path) as f:
        header = f.readline().strip().split(",")
        rows = [line.strip().split(",") for line in f if line.strip()]
    return header, rows


@pytest.mark.parametrize("name", ["config1_t0", "c3x2_t0"])
def test_trace_and_debug_outputs_match_reference(golden, tmp_path, name):
    """--trace-partition-csv (main.cpp:1583-1607) and --debug-block-csv
    (main.cpp:1233-1267) against the reference's own files: same header, same
    rows in the same block order, same method column, every numeric column
    within 1e-8 relative (1e-10 absolute); the stdout debug header line
    identical."""
    run = golden.meta["trace_runs"][name]
    nu, nd, mx, my = run["block"]
    tr, dbg, out = tmp_path / "trace.csv", tmp_path / "dbg.csv", tmp_path / "o.csv"
    r = run_cli("ftlm_n_vs_mu", run["args"], out, ["--trace-partition-csv", str(tr), "--debug-block-nup", str(nu),
                                                  "--debug-block-ndown", str(nd), "--debug-block-mx", str(mx),
                                                  "--debug-block-my", str(my), "--debug-block-csv", str(dbg)])
    ref_out = open(os.path.join(GOLDEN, "csv", name + "_trace.stdout")).read().splitlines()
    want = [ln for ln in ref_out if ln.startswith("Selected block debug")]
    got = [ln for ln in r.stdout.splitlines() if ln.startswith("Selected block debug")]
    assert len(want) == 1 and len(got) == 1
    # the weight sum is printed by FTLM blocks; compare the rest of the line text
    assert got[0].split(" sum_sample_weights=")[0] == want[0].split(" sum_sample_weights=")[0]
    for mine, ref in ((tr, name + "_trace.csv"), (dbg, name + "_debug.csv")):
        h1, a = _read_rows(mine)
        h2, b = _read_rows(os.path.join(GOLDEN, "csv", ref))
        assert h1 == h2 and len(a) == len(b) and len(a) > 0, ref
        for ra, rb in zip(a, b):
            assert len(ra) == len(rb)
            for col, x, y in zip(h1, ra, rb):
                if col == "method":
                    assert x == y
                    continue
                fx, fy = float(x), float(y)
                assert abs(fx - fy) <= 1e-10 + 1e-8 * abs(fy), (ref, col, ra[:4], x, y)
