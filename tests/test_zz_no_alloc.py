"""ftlm_ritz_noalloc: the allocation-free Ritz stage, through the C ABI.

For callers that cannot allocate device memory when they need Ritz values
(a framework whose caching allocator already holds the device pool, or a
latency-critical loop that cannot pay for cudaMalloc/cudaFree). The test is
such a caller: it owns its device buffers (torch tensors) and hands them to
the entry point, which must reproduce what the existing entry point
ftlm_block_spectrum returns for the same Lanczos run, on two calls in a row.
The file name makes pytest collect it last.
"""
import ctypes as C

import numpy as np
import pytest

import ftlm_extended_hubbard_development_b200 as pkg
from ftlm_extended_hubbard_development_b200 import engine as E

pytestmark = pytest.mark.gpu

TOL = 1e-12  # same FP64 QL on the same coefficients


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def test_noalloc_ritz_matches_block_spectrum_twice():
    import torch

    model = pkg.Model(lx=4, ly=2, tp=0.2, phix=0.25, phiy=0.5, u=8.0, v=1.5)
    R, L = 6, 50
    opts = pkg.RunOpts(samples=R, lanczos_steps=L, exact_block_threshold=0,
                       start_vector=E.START_PHILOX_PHASE)
    with pkg.Engine(model, opts) as eng:
        eng.sector_prepare(4, 3)
        alpha, beta, steps = eng.block_lanczos(1, 1)
        ev_ref, w_ref, _ = eng.block_spectrum(1, 1, exact=False)  # same run, existing entry point
    lib = E.load_library()
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    a = torch.tensor(alpha, dtype=torch.float64, device=dev).contiguous()
    b = torch.tensor(beta, dtype=torch.float64, device=dev).contiguous()
    s = torch.tensor(steps, dtype=torch.int32, device=dev).contiguous()
    err = C.create_string_buffer(256)
    for call in range(2):
        ev = torch.full((R * L,), float("nan"), dtype=torch.float64, device=dev)
        w = torch.full((R * L,), float("nan"), dtype=torch.float64, device=dev)
        cnt = torch.zeros(1, dtype=torch.int64, device=dev)
        stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        st = lib.ftlm_ritz_noalloc(_ptr(a), _ptr(b), _ptr(s), R, L, 1.0 / R, _ptr(ev), _ptr(w), _ptr(cnt),
                                   stream, err, 256)
        assert st == E.OK, err.value
        torch.cuda.synchronize()
        n = int(cnt.item())
        assert n == len(ev_ref) == int(steps.sum()), call
        got_ev, got_w = ev[:n].cpu().numpy(), w[:n].cpu().numpy()
        assert np.abs(got_ev - ev_ref).max() <= TOL * max(1.0, np.abs(ev_ref).max()), call
        assert np.abs(got_w - w_ref).max() <= TOL, call


def test_noalloc_rejects_sizes_beyond_its_work_space():
    lib = E.load_library()
    err = C.create_string_buffer(256)
    fake = C.c_void_p(1)  # never dereferenced: the size check comes first
    st = lib.ftlm_ritz_noalloc(fake, fake, fake, 128, 1024, 1.0, fake, fake, None, None, err, 256)
    assert st == E.ERR_CAPACITY
    assert b"exceeds the fixed work space" in err.value
