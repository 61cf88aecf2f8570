"""ctypes view of the restated C oracle (oracle/ftlm_oracle.c).

TEST INFRASTRUCTURE: imported only by tests/, the smoke check and bench.py's
CPU-baseline / reference legs. It is the checker, never the product path.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libftlm_oracle.so")
REF_DIR = os.path.join(HERE, "_ref")


class FoModel(C.Structure):
    _fields_ = [("lx", C.c_int), ("ly", C.c_int), ("tx", C.c_double), ("ty", C.c_double),
                ("tp", C.c_double), ("phix", C.c_double), ("phiy", C.c_double),
                ("u", C.c_double), ("v", C.c_double)]


@dataclass
class Model:
    lx: int = 2
    ly: int = 2
    tx: float = 1.0
    ty: float = 1.0
    tp: float = 0.0
    phix: float = 1.0
    phiy: float = 1.0
    u: float = 8.0
    v: float = 0.0

    def c(self) -> FoModel:
        return FoModel(self.lx, self.ly, self.tx, self.ty, self.tp, self.phix, self.phiy,
                       self.u, self.v)

    def flags(self) -> list[str]:
        return ["--lx", str(self.lx), "--ly", str(self.ly), "--tx", repr(self.tx),
                "--ty", repr(self.ty), "--tp", repr(self.tp), "--phix", repr(self.phix),
                "--phiy", repr(self.phiy), "--u", repr(self.u), "--v", repr(self.v)]


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"oracle library missing: {LIB_PATH} (run make -C oracle)")
        L = C.CDLL(LIB_PATH)
        P = C.POINTER
        L.fo_mix_u64.restype = C.c_uint64
        L.fo_mix_u64.argtypes = [C.c_uint64]
        L.fo_block_seed.restype = C.c_uint64
        L.fo_block_seed.argtypes = [C.c_uint64, C.c_int, C.c_int, C.c_int, C.c_int]
        L.fo_translate_spin.restype = C.c_uint64
        L.fo_translate_spin.argtypes = [C.c_uint64, C.c_int, C.c_int, C.c_int, C.c_int, P(C.c_int)]
        L.fo_sector_parents.restype = C.c_int64
        L.fo_sector_parents.argtypes = [P(FoModel), C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                        C.c_void_p, C.c_void_p, C.c_int64]
        L.fo_sector_relations.argtypes = [P(FoModel), C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                          C.c_void_p]
        L.fo_block_csr.argtypes = [P(FoModel), C.c_int, C.c_int, C.c_int, C.c_int,
                                   P(C.c_int64), P(C.c_int64), C.c_void_p, C.c_void_p,
                                   C.c_void_p, C.c_void_p]
        L.fo_csr_apply.argtypes = [C.c_int64] + [C.c_void_p] * 6
        L.fo_start_vector.argtypes = [C.c_uint64, C.c_int, C.c_int64, C.c_void_p]
        L.fo_lanczos.restype = C.c_int
        L.fo_lanczos.argtypes = [C.c_int64] + [C.c_void_p] * 5 + [C.c_int, C.c_void_p, C.c_void_p]
        L.fo_tridiag_jacobi.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.fo_block_exact.restype = C.c_int
        L.fo_block_exact.argtypes = [C.c_int64] + [C.c_void_p] * 5
        L.fo_thermo_accumulate.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.c_double, C.c_int,
                                           C.c_double, C.c_int] + [C.c_void_p] * 5
        L.fo_run_curve.restype = C.c_int
        L.fo_run_curve.argtypes = [P(FoModel), C.c_int, C.c_int, C.c_uint64, C.c_uint64,
                                   C.c_uint64, C.c_int, C.c_int, C.c_void_p, C.c_int] + \
            [C.c_void_p] * 5
        _lib = L
    return _lib


def _p(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


def mix_u64(v: int) -> int:
    return lib().fo_mix_u64(v)


def block_seed(seed: int, nup: int, ndn: int, mx: int, my: int) -> int:
    return lib().fo_block_seed(seed, nup, ndn, mx, my)


def translate_spin(bits: int, dx: int, dy: int, lx: int, ly: int) -> tuple[int, int]:
    s = C.c_int(0)
    out = lib().fo_translate_spin(bits, dx, dy, lx, ly, C.byref(s))
    return out, s.value


def sector_parents(m: Model, nup: int, ndn: int):
    mc = m.c()
    n = lib().fo_sector_parents(C.byref(mc), nup, ndn, None, None, None, None, 0)
    up = np.zeros(n, np.uint64)
    dn = np.zeros(n, np.uint64)
    deg = np.zeros(n, np.int32)
    diag = np.zeros(n, np.float64)
    lib().fo_sector_parents(C.byref(mc), nup, ndn, _p(up), _p(dn), _p(deg), _p(diag), n)
    return up, dn, deg, diag


def sector_relations(m: Model, nup: int, ndn: int):
    from math import comb
    n = m.lx * m.ly
    full = comb(n, nup) * comb(n, ndn)
    par = np.zeros(full, np.int32)
    sh = np.zeros(full, np.int32)
    sg = np.zeros(full, np.int32)
    mc = m.c()
    lib().fo_sector_relations(C.byref(mc), nup, ndn, _p(par), _p(sh), _p(sg))
    return par, sh, sg


@dataclass
class Csr:
    dim: int
    diag: np.ndarray
    row_ptr: np.ndarray
    col: np.ndarray
    val: np.ndarray  # complex128

    def apply(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, np.complex128)
        out = np.zeros(self.dim, np.complex128)
        v = np.ascontiguousarray(self.val.view(np.float64))
        lib().fo_csr_apply(self.dim, _p(self.diag), _p(self.row_ptr), _p(self.col), _p(v),
                           _p(x), _p(out))
        return out

    def dense(self) -> np.ndarray:
        a = np.zeros((self.dim, self.dim), np.complex128)
        for i in range(self.dim):
            a[i, i] += self.diag[i]
            for e in range(self.row_ptr[i], self.row_ptr[i + 1]):
                a[i, self.col[e]] += self.val[e]
        return a


def block_csr(m: Model, nup: int, ndn: int, mx: int, my: int) -> Csr:
    mc = m.c()
    dim = C.c_int64(0)
    nnz = C.c_int64(0)
    lib().fo_block_csr(C.byref(mc), nup, ndn, mx, my, C.byref(dim), C.byref(nnz),
                       None, None, None, None)
    d = dim.value
    diag = np.zeros(d, np.float64)
    rp = np.zeros(d + 1, np.int32)
    col = np.zeros(max(nnz.value, 1), np.int32)
    val = np.zeros(2 * max(nnz.value, 1), np.float64)
    lib().fo_block_csr(C.byref(mc), nup, ndn, mx, my, C.byref(dim), C.byref(nnz),
                       _p(diag), _p(rp), _p(col), _p(val))
    n = nnz.value
    return Csr(d, diag, rp, col[:n].copy(), val[: 2 * n].view(np.complex128).copy())


def start_vector(bseed: int, sample: int, dim: int) -> np.ndarray:
    out = np.zeros(2 * dim, np.float64)
    lib().fo_start_vector(bseed, sample, dim, _p(out))
    return out.view(np.complex128)


def lanczos(csr: Csr, start: np.ndarray, kmax: int):
    a = np.zeros(kmax, np.float64)
    b = np.zeros(kmax, np.float64)
    s = np.ascontiguousarray(start, np.complex128)
    v = np.ascontiguousarray(csr.val.view(np.float64))
    n = lib().fo_lanczos(csr.dim, _p(csr.diag), _p(csr.row_ptr), _p(csr.col), _p(v), _p(s),
                         kmax, _p(a), _p(b))
    return a[:n].copy(), b[: max(n - 1, 0)].copy()


def tridiag_jacobi(alpha: np.ndarray, beta: np.ndarray):
    n = len(alpha)
    a = np.ascontiguousarray(alpha, np.float64)
    b = np.zeros(max(n, 1), np.float64)
    b[: len(beta)] = beta
    ev = np.zeros(n, np.float64)
    w = np.zeros(n, np.float64)
    lib().fo_tridiag_jacobi(n, _p(a), _p(b), _p(ev), _p(w))
    return ev, w


def block_exact(csr: Csr) -> np.ndarray:
    ev = np.zeros(max(csr.dim, 1), np.float64)
    v = np.ascontiguousarray(csr.val.view(np.float64)) if len(csr.val) else np.zeros(2)
    info = lib().fo_block_exact(csr.dim, _p(csr.diag), _p(csr.row_ptr), _p(csr.col), _p(v), _p(ev))
    if info != 0:
        raise RuntimeError(f"zheev info={info}")
    return ev[: csr.dim].copy()


def thermo_accumulate(evals, weights, pref, particles, beta, mu, state):
    emin, z, n, n2 = state
    e = np.ascontiguousarray(evals, np.float64)
    w = None if weights is None else np.ascontiguousarray(weights, np.float64)
    muv = np.ascontiguousarray(mu, np.float64)
    lib().fo_thermo_accumulate(len(e), _p(e), None if w is None else _p(w), pref, particles, beta,
                               len(muv), _p(muv), _p(emin), _p(z), _p(n), _p(n2))


def linspace(lo: float, hi: float, count: int) -> np.ndarray:
    """mu grid exactly as main.cpp:1400-1407 (start + step * i)."""
    step = (hi - lo) / float(count - 1)
    return np.array([lo + step * float(i) for i in range(count)], np.float64)


def run_curve(m: Model, betas, mu, *, samples=5, steps=80, threshold=256, seed=12345,
              max_sector_dim=2000000, ed=False):
    """Oracle n(mu) curve; returns dict of arrays [nbeta][nmu] with the
    finalised observables of main.cpp:1770-1788."""
    betas = np.ascontiguousarray(betas, np.float64)
    mu = np.ascontiguousarray(mu, np.float64)
    nb, nm = len(betas), len(mu)
    emin = np.full(nb * nm, np.inf)
    z = np.zeros(nb * nm)
    ns = np.zeros(nb * nm)
    n2 = np.zeros(nb * nm)
    mc = m.c()
    rc = lib().fo_run_curve(C.byref(mc), samples, steps, threshold, seed, max_sector_dim,
                            1 if ed else 0, nb, _p(betas), nm, _p(mu), _p(emin), _p(z), _p(ns),
                            _p(n2))
    if rc != 0:
        raise RuntimeError("sector exceeds max_sector_dim")
    return finalize(m.lx * m.ly, betas, emin.reshape(nb, nm), z.reshape(nb, nm),
                    ns.reshape(nb, nm), n2.reshape(nb, nm))


def finalize(sites, betas, emin, z, ns, n2):
    betas = np.asarray(betas, np.float64).reshape(-1, 1)
    mean = ns / z
    mean2 = n2 / z
    chi = np.maximum(0.0, (mean2 - mean * mean) / sites)
    return {"n": mean / sites, "charge_correlation": chi, "compressibility": betas * chi,
            "partition_like": z, "log_partition": np.log(z) - betas * emin}
