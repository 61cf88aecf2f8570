"""CPU-side checks of the C ABI library and the drop-in CLIs (no GPU needed)."""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import REPO

import ftlm_extended_hubbard_development_b200 as pkg
from ftlm_extended_hubbard_development_b200 import engine as E

HEADER = os.path.join(REPO, "include", "ftlm_gpu.h")
BIN = os.path.join(REPO, "ftlm_extended_hubbard_development_b200", "bin")


def header_functions():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"^(?:int|void)\s+(ftlm_\w+)\s*\(", src, re.M)))


def test_library_exports_every_declared_symbol():
    names = header_functions()
    assert len(names) >= 19
    out = subprocess.run(["nm", "-D", "--defined-only", E.LIB_PATH], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r"\sT\s(ftlm_\w+)$", out, re.M))
    assert set(names) <= exported, set(names) - exported
    assert set(names) == set(E.EXPORTS)


def test_library_loads_and_reports_abi_version():
    lib = pkg.load_library()
    assert lib.ftlm_abi_version() == 2


def test_build_targets_sm100a_only():
    """Every CUDA object of the library is compiled for sm_100a SASS with no
    PTX fallback (the loaded code object is checked on a GPU in
    test_gpu_parity.py::test_loaded_device_code_is_sm100)."""
    mk = open(os.path.join(E.PKG, "Makefile")).read()
    assert "ARCH      ?= -gencode arch=compute_100a,code=sm_100a" in mk
    assert "compute_100a,code=compute" not in mk


@pytest.mark.skipif(os.path.exists("/dev/nvidia0"), reason="a GPU is present")
def test_no_cpu_fallback_without_gpu():
    with pytest.raises(E.FtlmError) as ei:
        E.Engine(E.Model(lx=2, ly=2))
    assert ei.value.code == E.ERR_CUDA


def test_ctx_create_validates_like_parse_args():
    lib = pkg.load_library()
    import ctypes as C
    h = C.c_void_p()
    bad = [E._Model(0, 2, 1, 1, 0, 1, 1, 8, 0), E._Model(8, 8, 1, 1, 0, 1, 1, 8, 0)]
    for m in bad:
        o = E._Opts(5, 80, 256, 12345, 0, 0, 0, 0)
        assert lib.ftlm_ctx_create(C.byref(m), C.byref(o), C.byref(h)) == E.ERR_ARG
    m = E._Model(2, 2, 1, 1, 0, 1, 1, 8, 0)
    for o in (E._Opts(0, 80, 256, 1, 0, 0, 0, 0), E._Opts(5, 0, 256, 1, 0, 0, 0, 0),
              E._Opts(5, 80, 256, 1, 7, 0, 0, 0), E._Opts(5, 80, 256, 1, 0, 0, 999, 0)):
        assert lib.ftlm_ctx_create(C.byref(m), C.byref(o), C.byref(h)) == E.ERR_ARG


@pytest.mark.parametrize("args,msg", [
    (["--lx", "0"], "Lattice dimensions must be positive."),
    (["--lx", "8", "--ly", "8"], "This implementation supports at most 63 sites."),
    (["--beta", "-1"], "All beta values must be positive."),
    (["--beta-list", "1,,2"], "Empty entry in comma-separated value list: 1,,2"),
    (["--samples", "0"], "--samples and --lanczos-steps must be positive."),
    (["--threads", "-2"], "--threads must be non-negative."),
    (["--mu-count", "1"], "--mu-count must be at least 2."),
    (["--debug-block-nup", "1"], "Selected-block debug requires"),
    (["--lx", "2x"], "Failed to parse value: 2x"),
    (["--lx"], "Missing value for --lx"),
    (["--frobnicate"], "Unknown argument: --frobnicate"),
    (["--precision", "fp16"], "--precision must be fp64 or mixed."),
])
def test_cli_validation_messages(args, msg):
    for exe in ("ftlm_n_vs_mu", "ftlm_ed_n_vs_mu"):
        r = subprocess.run([os.path.join(BIN, exe)] + args, capture_output=True, text=True)
        assert r.returncode == 1
        assert r.stderr.startswith("Error: " + msg), r.stderr


def test_cli_checkpoint_with_trace_is_rejected(tmp_path):
    r = subprocess.run([os.path.join(BIN, "ftlm_n_vs_mu"), "--checkpoint", str(tmp_path / "c"),
                        "--trace-partition-csv", str(tmp_path / "t.csv")], capture_output=True, text=True)
    assert r.returncode == 1
    assert "--checkpoint is not currently compatible with trace/debug block output." in r.stderr


def test_cli_meta_mismatch_exits_1(tmp_path):
    ck = tmp_path / "run.ftlmcp"
    (tmp_path / "run.ftlmcp.meta").write_text("lx=9\n")
    r = subprocess.run([os.path.join(BIN, "ftlm_n_vs_mu"), "--checkpoint", str(ck)], capture_output=True,
                       text=True)
    assert r.returncode == 1
    assert "Checkpoint metadata does not match current run" in r.stderr


def test_cli_help_lists_reference_flags():
    r = subprocess.run([os.path.join(BIN, "ftlm_n_vs_mu"), "--help"], capture_output=True, text=True)
    assert r.returncode == 0
    for flag in ("--lx", "--ly", "--tx", "--ty", "--tp", "--phix", "--phiy", "--u", "--v", "--beta",
                 "--beta-list", "--mu-min", "--mu-max", "--mu-count", "--samples", "--lanczos-steps",
                 "--threads", "--exact-block-threshold", "--seed", "--max-sector-dim", "--checkpoint",
                 "--trace-partition-csv", "--debug-block-nup", "--debug-block-ndown", "--debug-block-mx",
                 "--debug-block-my", "--debug-block-csv", "--output", "--help"):
        assert flag in r.stdout


def test_linspace_matches_reference_grid():
    mu = pkg.linspace(-3.0, 4.0, 281)
    assert mu[0] == -3.0 and len(mu) == 281
    step = 7.0 / 280.0
    assert all(mu[i] == -3.0 + step * i for i in range(281))


def philox4x32_10(ctr, key):
    """Philox4x32-10 (Salmon et al., SC'11) restated in Python for the known-answer test."""
    c = list(ctr)
    k0, k1 = key
    M = 0xFFFFFFFF
    for _ in range(10):
        p0 = 0xD2511F53 * c[0]
        p1 = 0xCD9E8D57 * c[2]
        c = [((p1 >> 32) ^ c[1] ^ k0) & M, p1 & M, ((p0 >> 32) ^ c[3] ^ k1) & M, p0 & M]
        k0 = (k0 + 0x9E3779B9) & M
        k1 = (k1 + 0xBB67AE85) & M
    return c


def test_philox_known_answers():
    # Random123 known-answer vectors for Philox4x32-10
    assert philox4x32_10([0, 0, 0, 0], [0, 0]) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert philox4x32_10([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2) == \
        [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
