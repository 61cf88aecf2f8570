"""Python view of libftlm_gpu (include/ftlm_gpu.h) through ctypes.

The engine is the compiled CUDA library; this module only marshals host
buffers. There is no CPU fallback: if the shared library is missing or no
CUDA device is usable, the calls raise.

The per-block seam mirrors the reference program's chain
(PeizhiMai/FTLM_extended_Hubbard_development src/main.cpp:1519-1720):
sector_prepare (build_sector_basis) -> block_spectrum (run_ftlm_block /
diagonalize_block_exact) -> thermo_accumulate_block (accumulate_block_thermo).
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "lib", "libftlm_gpu.so")
BIN_DIR = os.path.join(PKG, "bin")

OK, ERR_ARG, ERR_STATE, ERR_CUDA, ERR_CAPACITY, ERR_NUMERIC, ERR_INTERNAL = range(7)
PREC_FP64, PREC_MIXED = 0, 1
START_REF_GAUSSIAN, START_PHILOX_PHASE = 0, 1


class FtlmError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class _Model(C.Structure):
    _fields_ = [("lx", C.c_int32), ("ly", C.c_int32), ("tx", C.c_double), ("ty", C.c_double),
                ("tp", C.c_double), ("phix", C.c_double), ("phiy", C.c_double),
                ("u", C.c_double), ("v", C.c_double)]


class _Opts(C.Structure):
    _fields_ = [("samples", C.c_int32), ("lanczos_steps", C.c_int32),
                ("exact_block_threshold", C.c_uint64), ("seed", C.c_uint64),
                ("precision", C.c_int32), ("start_vector", C.c_int32),
                ("batch_vectors", C.c_int32), ("device", C.c_int32)]


class _SectorInfo(C.Structure):
    _fields_ = [("full_dim", C.c_uint64), ("parents", C.c_uint64), ("n_k", C.c_int32),
                ("block_dim", C.c_uint64 * 64)]


class _Profile(C.Structure):
    _fields_ = [("hv_ms", C.c_double), ("hv_launches", C.c_int64), ("hv_bytes", C.c_double),
                ("update_ms", C.c_double), ("update_launches", C.c_int64),
                ("eig_ms", C.c_double), ("dense_ms", C.c_double), ("thermo_ms", C.c_double),
                ("sector_ms", C.c_double), ("block_ms", C.c_double),
                ("kernel_launches", C.c_int64), ("h2d_bytes", C.c_int64), ("d2h_bytes", C.c_int64),
                ("hv_variant", C.c_int32), ("tune_runs", C.c_int32), ("small_ms", C.c_double),
                ("small_tasks", C.c_int64), ("hv_hops", C.c_double), ("hv_min_bytes", C.c_double),
                ("hv_source", C.c_int32), ("pad0", C.c_int32)]


EXPORTS = [
    "ftlm_abi_version", "ftlm_device_code_version", "ftlm_ctx_create", "ftlm_ctx_destroy", "ftlm_last_error",
    "ftlm_sector_prepare", "ftlm_block_spectrum", "ftlm_spectra_reset", "ftlm_blocks_exact_batched",
    "ftlm_spectra_defer", "ftlm_spectra_flush", "ftlm_blocks_ftlm_batched",
    "ftlm_thermo_configure", "ftlm_thermo_accumulate_block", "ftlm_thermo_accumulate_host",
    "ftlm_thermo_read", "ftlm_block_apply", "ftlm_block_lanczos",
    "ftlm_debug_sector_parents", "ftlm_debug_sector_relations", "ftlm_debug_block_csr",
    "ftlm_profile_enable", "ftlm_profile_read", "ftlm_profile_reset", "ftlm_ritz_noalloc",
    "ftlm_mlp_create", "ftlm_mlp_destroy", "ftlm_mlp_last_error", "ftlm_mlp_num_params",
    "ftlm_mlp_get_params", "ftlm_mlp_set_params", "ftlm_mlp_forward", "ftlm_mlp_loss_grad",
    "ftlm_mlp_train",
]

_lib = None


def load_library(path: str = LIB_PATH) -> C.CDLL:
    """Load libftlm_gpu.so and declare its prototypes (raises if absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FtlmError(ERR_CUDA, f"libftlm_gpu.so not built at {path}; run __graft_entry__.build()")
    L = C.CDLL(path)
    P, vp, i32, u64, sz, d = C.POINTER, C.c_void_p, C.c_int32, C.c_uint64, C.c_size_t, C.c_double
    sig = {
        "ftlm_abi_version": ([], C.c_int),
        "ftlm_device_code_version": ([i32, C.POINTER(C.c_int32), C.POINTER(C.c_int32)], C.c_int),
        "ftlm_ctx_create": ([P(_Model), P(_Opts), P(vp)], C.c_int),
        "ftlm_ctx_destroy": ([vp], None),
        "ftlm_last_error": ([vp, C.c_char_p, sz], C.c_int),
        "ftlm_sector_prepare": ([vp, i32, i32, P(_SectorInfo)], C.c_int),
        "ftlm_block_spectrum": ([vp, i32, i32, i32, vp, vp, sz, P(sz), P(d)], C.c_int),
        "ftlm_spectra_reset": ([vp], C.c_int),
        "ftlm_blocks_exact_batched": ([vp, vp, vp, i32], C.c_int),
        "ftlm_spectra_defer": ([vp, i32], C.c_int),
        "ftlm_spectra_flush": ([vp], C.c_int),
        "ftlm_blocks_ftlm_batched": ([vp, vp, vp, i32], C.c_int),
        "ftlm_thermo_configure": ([vp, i32, vp, i32, vp], C.c_int),
        "ftlm_thermo_accumulate_block": ([vp, i32, i32], C.c_int),
        "ftlm_thermo_accumulate_host": ([vp, vp, vp, sz, d, i32], C.c_int),
        "ftlm_thermo_read": ([vp, vp, vp, vp, vp], C.c_int),
        "ftlm_block_apply": ([vp, i32, i32, i32, vp, vp], C.c_int),
        "ftlm_block_lanczos": ([vp, i32, i32, vp, vp, vp, vp], C.c_int),
        "ftlm_debug_sector_parents": ([vp, vp, vp, vp, vp, sz, P(sz)], C.c_int),
        "ftlm_debug_sector_relations": ([vp, vp, vp, vp, sz], C.c_int),
        "ftlm_debug_block_csr": ([vp, i32, i32, vp, vp, vp, vp, sz, sz, P(sz), P(sz)], C.c_int),
        "ftlm_profile_enable": ([vp, i32], C.c_int),
        "ftlm_profile_read": ([vp, P(_Profile)], C.c_int),
        "ftlm_profile_reset": ([vp], C.c_int),
        "ftlm_ritz_noalloc": ([vp, vp, vp, i32, i32, d, vp, vp, vp, vp, C.c_char_p, sz], C.c_int),
        "ftlm_mlp_create": ([i32, i32, i32, i32, u64, i32, P(vp)], C.c_int),
        "ftlm_mlp_destroy": ([vp], None),
        "ftlm_mlp_last_error": ([vp, C.c_char_p, sz], C.c_int),
        "ftlm_mlp_num_params": ([vp, P(C.c_int64)], C.c_int),
        "ftlm_mlp_get_params": ([vp, vp, C.c_int64], C.c_int),
        "ftlm_mlp_set_params": ([vp, vp, C.c_int64], C.c_int),
        "ftlm_mlp_forward": ([vp, vp, C.c_int64, vp], C.c_int),
        "ftlm_mlp_loss_grad": ([vp, vp, vp, vp, C.c_int64, P(C.c_float), vp], C.c_int),
        "ftlm_mlp_train": ([vp, vp, vp, vp, C.c_int64, i32, i32, C.c_float, u64, vp], C.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def _p(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


@dataclass
class Model:
    """Hamiltonian fields of the reference's Params (main.cpp:32-41)."""
    lx: int = 2
    ly: int = 2
    tx: float = 1.0
    ty: float = 1.0
    tp: float = 0.0
    phix: float = 1.0
    phiy: float = 1.0
    u: float = 8.0
    v: float = 0.0

    @property
    def sites(self) -> int:
        return self.lx * self.ly


@dataclass
class RunOpts:
    samples: int = 5
    lanczos_steps: int = 80
    exact_block_threshold: int = 256
    seed: int = 12345
    precision: int = PREC_FP64
    start_vector: int = START_REF_GAUSSIAN
    batch_vectors: int = 0
    device: int = 0


@dataclass
class SectorInfo:
    full_dim: int
    parents: int
    block_dims: list = field(default_factory=list)  # index k = my*lx + mx


class Engine:
    """One GPU context (ftlm_ctx)."""

    def __init__(self, model: Model, opts: RunOpts | None = None):
        self.model = model
        self.opts = opts or RunOpts()
        self.lib = load_library()
        m = _Model(model.lx, model.ly, model.tx, model.ty, model.tp, model.phix, model.phiy,
                   model.u, model.v)
        o = _Opts(self.opts.samples, self.opts.lanczos_steps, self.opts.exact_block_threshold,
                  self.opts.seed, self.opts.precision, self.opts.start_vector,
                  self.opts.batch_vectors, self.opts.device)
        h = C.c_void_p()
        st = self.lib.ftlm_ctx_create(C.byref(m), C.byref(o), C.byref(h))
        if st != OK:
            raise FtlmError(st, "ftlm_ctx_create failed (no usable CUDA device or bad parameters)")
        self.h = h
        self.sector = None

    def close(self):
        if getattr(self, "h", None):
            self.lib.ftlm_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, st: int):
        if st != OK:
            buf = C.create_string_buffer(512)
            self.lib.ftlm_last_error(self.h, buf, 512)
            raise FtlmError(st, buf.value.decode())

    # ---- sector / block
    def sector_prepare(self, n_up: int, n_down: int) -> SectorInfo:
        info = _SectorInfo()
        self._check(self.lib.ftlm_sector_prepare(self.h, n_up, n_down, C.byref(info)))
        self.sector = (n_up, n_down)
        return SectorInfo(info.full_dim, info.parents, [info.block_dim[i] for i in range(info.n_k)])

    def block_spectrum(self, mx: int, my: int, exact: bool = False, fetch: bool = True):
        cnt = C.c_size_t(0)
        pref = C.c_double(0.0)
        self._check(self.lib.ftlm_block_spectrum(self.h, mx, my, int(exact), None, None, 0,
                                                 C.byref(cnt), C.byref(pref)))
        if not fetch:
            return cnt.value, pref.value
        ev = np.zeros(cnt.value, np.float64)
        w = None if exact else np.zeros(cnt.value, np.float64)
        self._check(self.lib.ftlm_block_spectrum(self.h, mx, my, int(exact), _p(ev), _p(w), cnt.value,
                                                 C.byref(cnt), C.byref(pref)))
        return ev, w, pref.value

    def spectra_reset(self):
        self._check(self.lib.ftlm_spectra_reset(self.h))

    def blocks_exact_batched(self, blocks):
        mx = np.array([b[0] for b in blocks], np.int32)
        my = np.array([b[1] for b in blocks], np.int32)
        self._check(self.lib.ftlm_blocks_exact_batched(self.h, _p(mx), _p(my), len(blocks)))

    def spectra_defer(self, on: bool = True):
        """Pool the exact blocks' matrices and the small FTLM blocks' Lanczos
        coefficients across sectors and solve them together
        (ftlm_spectra_defer); off flushes the pool."""
        self._check(self.lib.ftlm_spectra_defer(self.h, int(bool(on))))

    def spectra_flush(self):
        self._check(self.lib.ftlm_spectra_flush(self.h))

    def blocks_ftlm_batched(self, blocks):
        """FTLM spectra of several blocks; the small ones in one persistent launch."""
        mx = np.array([b[0] for b in blocks], np.int32)
        my = np.array([b[1] for b in blocks], np.int32)
        self._check(self.lib.ftlm_blocks_ftlm_batched(self.h, _p(mx), _p(my), len(blocks)))

    # ---- thermodynamics
    def thermo_configure(self, betas, mu):
        self._betas = np.ascontiguousarray(betas, np.float64)
        self._mu = np.ascontiguousarray(mu, np.float64)
        self._check(self.lib.ftlm_thermo_configure(self.h, len(self._betas), _p(self._betas),
                                                   len(self._mu), _p(self._mu)))

    def thermo_accumulate_block(self, mx: int, my: int):
        self._check(self.lib.ftlm_thermo_accumulate_block(self.h, mx, my))

    def thermo_accumulate_host(self, evals, weights, prefactor, particles):
        e = np.ascontiguousarray(evals, np.float64)
        w = None if weights is None else np.ascontiguousarray(weights, np.float64)
        self._check(self.lib.ftlm_thermo_accumulate_host(self.h, _p(e), _p(w), len(e), prefactor,
                                                         particles))

    def thermo_read(self):
        nb, nm = len(self._betas), len(self._mu)
        arrs = [np.zeros(nb * nm) for _ in range(4)]
        self._check(self.lib.ftlm_thermo_read(self.h, *[_p(a) for a in arrs]))
        return [a.reshape(nb, nm) for a in arrs]

    # ---- operators
    def block_apply(self, mx: int, my: int, x: np.ndarray) -> np.ndarray:
        """H*X for X[dim, nvec] (complex128) on block (mx, my) of the prepared sector."""
        x = np.ascontiguousarray(x, np.complex128)
        if x.ndim == 1:
            x = x[:, None]
        out = np.zeros_like(x)
        self._check(self.lib.ftlm_block_apply(self.h, mx, my, x.shape[1], _p(x), _p(out)))
        return out

    def block_lanczos(self, mx: int, my: int, start: np.ndarray | None = None):
        R, L = self.opts.samples, self.opts.lanczos_steps
        a = np.zeros(R * L)
        b = np.zeros(R * L)
        s = np.zeros(R, np.int32)
        st = None if start is None else np.ascontiguousarray(start, np.complex128)
        self._check(self.lib.ftlm_block_lanczos(self.h, mx, my, _p(st), _p(a), _p(b), _p(s)))
        return a.reshape(R, L), b.reshape(R, L), s

    # ---- parity views
    def debug_sector_parents(self):
        cnt = C.c_size_t(0)
        self._check(self.lib.ftlm_debug_sector_parents(self.h, None, None, None, None, 0, C.byref(cnt)))
        n = cnt.value
        up = np.zeros(n, np.uint64)
        dn = np.zeros(n, np.uint64)
        deg = np.zeros(n, np.int32)
        diag = np.zeros(n, np.float64)
        self._check(self.lib.ftlm_debug_sector_parents(self.h, _p(up), _p(dn), _p(deg), _p(diag), n,
                                                       C.byref(cnt)))
        return up, dn, deg, diag

    def debug_sector_relations(self, full_dim: int):
        par = np.zeros(full_dim, np.int32)
        sh = np.zeros(full_dim, np.int32)
        sg = np.zeros(full_dim, np.int32)
        self._check(self.lib.ftlm_debug_sector_relations(self.h, _p(par), _p(sh), _p(sg), full_dim))
        return par, sh, sg

    def debug_block_csr(self, mx: int, my: int):
        dim = C.c_size_t(0)
        nnz = C.c_size_t(0)
        self._check(self.lib.ftlm_debug_block_csr(self.h, mx, my, None, None, None, None, 0, 0,
                                                  C.byref(dim), C.byref(nnz)))
        D, Z = dim.value, nnz.value
        diag = np.zeros(max(D, 1))
        rp = np.zeros(D + 1, np.int32)
        col = np.zeros(max(Z, 1), np.int32)
        val = np.zeros(2 * max(Z, 1))
        self._check(self.lib.ftlm_debug_block_csr(self.h, mx, my, _p(diag), _p(rp), _p(col), _p(val),
                                                  D, Z, C.byref(dim), C.byref(nnz)))
        return diag[:D], rp, col[:Z], val[: 2 * Z].view(np.complex128)

    # ---- instrumentation
    def profile(self, enable: bool | None = None) -> dict:
        if enable is not None:
            self._check(self.lib.ftlm_profile_enable(self.h, int(enable)))
        p = _Profile()
        self._check(self.lib.ftlm_profile_read(self.h, C.byref(p)))
        return {k: getattr(p, k) for k, _ in _Profile._fields_}

    def profile_reset(self):
        self._check(self.lib.ftlm_profile_reset(self.h))


def linspace(lo: float, hi: float, count: int) -> np.ndarray:
    """The reference's mu grid (main.cpp:1400-1407)."""
    step = (hi - lo) / float(count - 1)
    return np.array([lo + step * float(i) for i in range(count)], np.float64)


def run_curve(model: Model, betas, mu, opts: RunOpts | None = None, ed: bool = False,
              engine: Engine | None = None):
    """Whole n(mu) curve through the C ABI in the reference's block order
    (main.cpp:1519-1788). Returns the finalised observables [nbeta][nmu]."""
    opts = opts or RunOpts()
    own = engine is None
    eng = engine or Engine(model, opts)
    try:
        eng.thermo_configure(betas, mu)
        eng.spectra_defer(True)  # the small blocks of all sectors in one dense-solver and one Ritz launch
        n = model.sites
        for nu in range(n + 1):
            for nd in range(n + 1):
                info = eng.sector_prepare(nu, nd)
                blocks = [(k % model.lx, k // model.lx) for k, d in enumerate(info.block_dims) if d > 0]
                exact = [b for b in blocks
                         if ed or info.block_dims[b[1] * model.lx + b[0]] <= opts.exact_block_threshold]
                eng.blocks_exact_batched(exact)
                eng.blocks_ftlm_batched([b for b in blocks if b not in exact])
                for b in blocks:
                    eng.thermo_accumulate_block(*b)
        emin, z, ns, n2 = eng.thermo_read()
        eng.spectra_defer(False)
    finally:
        if own:
            eng.close()
    b = np.asarray(betas, np.float64).reshape(-1, 1)
    mean = ns / z
    chi = np.maximum(0.0, (n2 / z - mean * mean) / n)
    return {"n": mean / n, "charge_correlation": chi, "compressibility": b * chi,
            "partition_like": z, "log_partition": np.log(z) - b * emin}


class Mlp:
    """The twist-surrogate network (ftlm_mlp): FP32 MLP trained on the GPU by
    the library's own forward/backward/Adam kernels."""

    def __init__(self, n_in: int, width: int, depth: int, n_out: int, seed: int = 1234,
                 device: int = 0):
        self.lib = load_library()
        h = C.c_void_p()
        st = self.lib.ftlm_mlp_create(n_in, width, depth, n_out, seed, device, C.byref(h))
        if st != OK:
            raise FtlmError(st, "ftlm_mlp_create failed")
        self.h = h
        self.n_in, self.width, self.depth, self.n_out = n_in, width, depth, n_out

    def close(self):
        if getattr(self, "h", None):
            self.lib.ftlm_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int):
        if st != OK:
            buf = C.create_string_buffer(512)
            self.lib.ftlm_mlp_last_error(self.h, buf, 512)
            raise FtlmError(st, buf.value.decode())

    @property
    def num_params(self) -> int:
        n = C.c_int64(0)
        self._check(self.lib.ftlm_mlp_num_params(self.h, C.byref(n)))
        return n.value

    def get_params(self) -> np.ndarray:
        p = np.zeros(self.num_params, np.float32)
        self._check(self.lib.ftlm_mlp_get_params(self.h, _p(p), len(p)))
        return p

    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, np.float32)
        self._check(self.lib.ftlm_mlp_set_params(self.h, _p(p), len(p)))

    def forward(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, np.float32)
        y = np.zeros((x.shape[0], self.n_out), np.float32)
        self._check(self.lib.ftlm_mlp_forward(self.h, _p(x), x.shape[0], _p(y)))
        return y

    def loss_grad(self, x, t, mask):
        x = np.ascontiguousarray(x, np.float32)
        t = np.ascontiguousarray(t, np.float32)
        m = np.ascontiguousarray(mask, np.float32)
        loss = C.c_float(0.0)
        g = np.zeros(self.num_params, np.float32)
        self._check(self.lib.ftlm_mlp_loss_grad(self.h, _p(x), _p(t), _p(m), x.shape[0], C.byref(loss), _p(g)))
        return loss.value, g

    def train(self, x, t, mask, epochs: int, batch: int, lr: float, seed: int = 7) -> np.ndarray:
        x = np.ascontiguousarray(x, np.float32)
        t = np.ascontiguousarray(t, np.float32)
        m = np.ascontiguousarray(mask, np.float32)
        hist = np.zeros(epochs, np.float32)
        self._check(self.lib.ftlm_mlp_train(self.h, _p(x), _p(t), _p(m), x.shape[0], epochs, batch, lr,
                                            seed, _p(hist)))
        return hist
