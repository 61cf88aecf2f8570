// C ABI of libftlm_gpu (declared in include/ftlm_gpu.h).
//
// Every entry point validates its arguments, runs on the context's device
// and stream, converts C++ exceptions into status codes and stores the
// message for ftlm_last_error. No exception crosses the ABI.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "ftlm_internal.h"

struct ftlm_ctx {
  ftlm::Ctx c;
};

namespace ftlm {

// Never launched: its attributes tell which code object the runtime loaded.
__global__ void k_code_probe() {}

namespace {

const double kPi = 3.141592653589793238462643383279502884;

void setup_geometry(Ctx& c) {
  Geom& g = c.geom;
  std::memset(&g, 0, sizeof g);
  const ftlm_model& m = c.model;
  g.lx = m.lx;
  g.ly = m.ly;
  g.n = m.lx * m.ly;
  const int ox[8] = {1, -1, 0, 0, 1, -1, 1, -1};
  const int oy[8] = {0, 0, 1, -1, 1, 1, -1, -1};
  const double t[8] = {m.tx, m.tx, m.ty, m.ty, m.tp, m.tp, m.tp, m.tp};
  // twist angles of twist_phase_for_dir (main.cpp:544-577)
  const double thx = 2.0 * kPi * m.phix / static_cast<double>(m.lx);
  const double thy = 2.0 * kPi * m.phiy / static_cast<double>(m.ly);
  const double ang[8] = {thx, -thx, thy, -thy, thx + thy, -thx + thy, thx - thy, -thx - thy};
  g.ndir = 0;
  for (int d = 0; d < 8; ++d) {
    g.dox[d] = static_cast<int8_t>(ox[d]);
    g.doy[d] = static_cast<int8_t>(oy[d]);
    const double pre = -t[d];
    g.amp_re[d] = pre * std::cos(ang[d]);
    g.amp_im[d] = pre * std::sin(ang[d]);
    if (t[d] != 0.0) g.dirs[g.ndir++] = static_cast<int8_t>(d);
  }
  g.U = m.u;
  g.V = m.v;
  g.v_mode = m.v == 0.0 ? 0 : (g.n == 1 ? 2 : 1);
  g.full = g.n >= 64 ? ~0ULL : ((1ULL << g.n) - 1ULL);
  g.rowmask = (1ULL << g.lx) - 1ULL;
  for (int dx = 0; dx < g.lx; ++dx) {
    uint64_t k = 0;
    for (int y = 0; y < g.ly; ++y) k |= ((1ULL << (g.lx - dx)) - 1ULL) << (y * g.lx);
    g.xkeep[dx] = k;
  }
  for (int y = 0; y < g.ly; ++y)
    for (int x = 0; x < g.lx; ++x)
      for (int d = 0; d < 8; ++d) {
        const int nx = ((x + ox[d]) % g.lx + g.lx) % g.lx;
        const int ny = ((y + oy[d]) % g.ly + g.ly) % g.ly;
        g.nb[y * g.lx + x][d] = static_cast<int8_t>(ny * g.lx + nx);
      }
  for (int d = 0; d <= 64; ++d) g.sqrt_deg[d] = std::sqrt(static_cast<double>(d));
}

void setup_binom(Ctx& c) {
  std::vector<uint64_t> b(65 * 65, 0);
  std::vector<uint32_t> b32(65 * 65, 0);
  for (int n = 0; n <= 64; ++n) {
    b[n * 65] = 1;
    for (int k = 1; k <= n; ++k) b[n * 65 + k] = b[(n - 1) * 65 + k - 1] + (k <= n - 1 ? b[(n - 1) * 65 + k] : 0);
  }
  for (int i = 0; i < 65 * 65; ++i) b32[i] = static_cast<uint32_t>(b[i]);
  c.binom.ensure(sizeof(uint64_t) * b.size());
  c.binom32.ensure(sizeof(uint32_t) * b32.size());
  FTLM_CUDA(cudaMemcpy(c.binom.p, b.data(), sizeof(uint64_t) * b.size(), cudaMemcpyHostToDevice));
  FTLM_CUDA(cudaMemcpy(c.binom32.p, b32.data(), sizeof(uint32_t) * b32.size(), cudaMemcpyHostToDevice));
}

template <typename F>
int guarded(ftlm_ctx* ctx, F&& f) {
  if (!ctx) return FTLM_ERR_ARG;
  try {
    FTLM_CUDA(cudaSetDevice(ctx->c.device));
    f(ctx->c);
    return FTLM_OK;
  } catch (const Error& e) {
    ctx->c.last_error = e.what();
    return e.code;
  } catch (const std::bad_alloc&) {
    ctx->c.last_error = "host allocation failed";
    return FTLM_ERR_INTERNAL;
  } catch (const std::exception& e) {
    ctx->c.last_error = e.what();
    return FTLM_ERR_INTERNAL;
  }
}

void need_sector(Ctx& c) {
  if (c.sec.n_up < 0) throw Error(FTLM_ERR_STATE, "no sector prepared");
}

void check_k(Ctx& c, int mx, int my) {
  if (mx < 0 || my < 0 || mx >= c.geom.lx || my >= c.geom.ly) throw Error(FTLM_ERR_ARG, "momentum index out of range");
}

}  // namespace
}  // namespace ftlm

using ftlm::Ctx;
using ftlm::Error;

extern "C" {

int ftlm_abi_version(void) { return FTLM_ABI_VERSION; }

int ftlm_device_code_version(int32_t device, int32_t* binary_version, int32_t* ptx_version) {
  if (!binary_version || !ptx_version) return FTLM_ERR_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    cudaGetLastError();
    return FTLM_ERR_CUDA;
  }
  int prev = 0;
  cudaGetDevice(&prev);
  cudaFuncAttributes a{};
  const cudaError_t e = cudaSetDevice(device) == cudaSuccess
                            ? cudaFuncGetAttributes(&a, reinterpret_cast<const void*>(ftlm::k_code_probe))
                            : cudaErrorInvalidDevice;
  cudaSetDevice(prev);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return FTLM_ERR_CUDA;
  }
  *binary_version = a.binaryVersion;
  *ptx_version = a.ptxVersion;
  return FTLM_OK;
}

int ftlm_ctx_create(const ftlm_model* model, const ftlm_run_opts* opts, ftlm_ctx** out) {
  if (!model || !opts || !out) return FTLM_ERR_ARG;
  *out = nullptr;
  // parse_args validation (main.cpp:332-353)
  if (model->lx <= 0 || model->ly <= 0) return FTLM_ERR_ARG;
  if (model->lx * model->ly > 63) return FTLM_ERR_ARG;
  if (opts->samples <= 0 || opts->lanczos_steps <= 0) return FTLM_ERR_ARG;
  if (opts->precision != FTLM_PREC_FP64 && opts->precision != FTLM_PREC_MIXED) return FTLM_ERR_ARG;
  if (opts->start_vector != FTLM_START_REF_GAUSSIAN && opts->start_vector != FTLM_START_PHILOX_PHASE) return FTLM_ERR_ARG;
  if (opts->batch_vectors < 0 || opts->batch_vectors > 128) return FTLM_ERR_ARG;
  ftlm_ctx* ctx = new (std::nothrow) ftlm_ctx();
  if (!ctx) return FTLM_ERR_INTERNAL;
  Ctx& c = ctx->c;
  c.model = *model;
  c.opts = *opts;
  c.device = opts->device;
  c.wide = model->lx * model->ly > 32;
  if (const char* hv = std::getenv("FTLM_HV_VARIANT")) c.hv_forced = std::atoi(hv);
  if (const char* rt = std::getenv("FTLM_HV_RETUNE")) c.hv_retune = std::string(rt) == "1";
  if (const char* sr = std::getenv("FTLM_SEG_ROWS")) c.seg_dynamic = std::string(sr) != "stride";
  if (const char* so = std::getenv("FTLM_SPLIT_OP")) c.split_stencil = std::string(so) != "fly";
  if (const char* sr2 = std::getenv("FTLM_STN_ROWS")) c.stn_rows = std::string(sr2) != "0";
  if (const char* hm = std::getenv("FTLM_HV_MODE")) {
    const std::string m(hm);
    c.hv_mode = m == "list" ? ftlm::kSrcList : m == "fly" ? ftlm::kSrcFly : m == "split" ? ftlm::kSrcSplit : -1;
  }
  if (const char* sb = std::getenv("FTLM_SMALL_BLOCKS")) c.small_blocks = std::string(sb) != "0";
  if (const char* hr = std::getenv("FTLM_HV_ROWS")) c.hv_rows = std::string(hr) != "0";
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0 || c.device < 0 || c.device >= ndev) {
    cudaGetLastError();
    delete ctx;
    return FTLM_ERR_CUDA;
  }
  try {
    FTLM_CUDA(cudaSetDevice(c.device));
    FTLM_CUDA(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
    FTLM_CUDA(cudaDeviceGetAttribute(&c.sm_count, cudaDevAttrMultiProcessorCount, c.device));
    ftlm::setup_geometry(c);
    ftlm::setup_binom(c);
  } catch (const Error&) {
    delete ctx;
    return FTLM_ERR_CUDA;
  }
  *out = ctx;
  return FTLM_OK;
}

void ftlm_ctx_destroy(ftlm_ctx* ctx) {
  if (!ctx) return;
  Ctx& c = ctx->c;
  cudaSetDevice(c.device);
  if (c.stream) cudaStreamSynchronize(c.stream);
  ftlm::DBuf* bufs[] = {&c.binom, &c.binom32, &c.sec.ups, &c.sec.dns, &c.sec.up_info, &c.sec.ur_bits,
                        &c.sec.ur_class, &c.sec.ur_poff, &c.sec.d_star, &c.sec.d_hs, &c.sec.d_stab,
                        &c.sec.d_chi, &c.sec.d_cidx, &c.sec.canon, &c.sec.tmp_a, &c.sec.tmp_b, &c.sec.tmp_c,
                        &c.sec.tmp_d, &c.sec.tmp_e, &c.blk.act, &c.blk.act_list, &c.blk.aoff, &c.blk.dtab,
                        &c.blk.row_meta, &c.blk.row_dn, &c.vec_a, &c.vec_b, &c.vec_h, &c.partial,
                        &c.lz_alpha, &c.lz_beta, &c.lz_scale, &c.lz_state, &c.host_start, &c.ritz_tmp, &c.ritz_out, &c.ritz_meta,
                        &c.sb_rp, &c.sb_col, &c.sb_val, &c.sb_diag, &c.sb_meta, &c.sb_steps,
                        &c.scan_tmp, &c.dense_arena, &c.dense_meta, &c.dense_out, &c.spectra, &c.th_beta,
                        &c.th_mu, &c.th_state, &c.hl_ptr, &c.hl_ent, &c.flip_map, &c.vec_xd, &c.vec_yd, &c.seg_counter, &c.stn_crb, &c.stn_rp, &c.stn_rp32, &c.stn_ent, &c.stn_cnt,
                        &c.defer_arena, &c.defer_ev, &c.defer_work, &c.defer_ab, &c.defer_st};
  for (auto* b : bufs) b->release();
  if (c.flipped) {
    ftlm::Ctx& f = *c.flipped;
    ftlm::DBuf* fb[] = {&f.sec.ups, &f.sec.dns, &f.sec.up_info, &f.sec.ur_bits, &f.sec.ur_class, &f.sec.ur_poff,
                        &f.sec.d_star, &f.sec.d_hs, &f.sec.d_stab, &f.sec.d_chi, &f.sec.d_cidx, &f.sec.canon,
                        &f.sec.tmp_a, &f.sec.tmp_b, &f.sec.tmp_c, &f.sec.tmp_d, &f.sec.tmp_e, &f.blk.act,
                        &f.blk.act_list, &f.blk.aoff, &f.blk.dtab, &f.blk.row_meta, &f.blk.row_dn, &f.scan_tmp,
                        &f.stn_crb, &f.stn_rp, &f.stn_rp32, &f.stn_ent, &f.stn_cnt};
    for (auto* b : fb) b->release();  // binom tables are the owner's
    c.flipped.reset();
  }
  if (c.stream) cudaStreamDestroy(c.stream);
  delete ctx;
}

int ftlm_last_error(const ftlm_ctx* ctx, char* buf, size_t len) {
  if (!buf || len == 0) return FTLM_ERR_ARG;
  const std::string msg = ctx ? ctx->c.last_error : std::string("null context");
  const size_t n = std::min(len - 1, msg.size());
  std::memcpy(buf, msg.data(), n);
  buf[n] = '\0';
  return FTLM_OK;
}

int ftlm_sector_prepare(ftlm_ctx* ctx, int32_t n_up, int32_t n_down, ftlm_sector_info* out) {
  return ftlm::guarded(ctx, [&](Ctx& c) {
    const int n = c.geom.n;
    if (n_up < 0 || n_down < 0 || n_up > n || n_down > n) throw Error(FTLM_ERR_ARG, "particle numbers out of range");
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (c.timing) {
      FTLM_CUDA(cudaEventCreate(&e0));
      FTLM_CUDA(cudaEventCreate(&e1));
      FTLM_CUDA(cudaEventRecord(e0, c.stream));
    }
    ftlm::spectra_reset(c);
    ftlm::sector_prepare(c, n_up, n_down);
    ftlm_sector_info info{};
    info.full_dim = static_cast<uint64_t>(c.sec.full_dim);
    info.parents = static_cast<uint64_t>(c.sec.parents);
    info.n_k = n;
    // block dimensions by character counting on the host (no GPU round
    // trips); block_prepare checks each against its own row count
    c.block_dims = ftlm::block_dims_by_characters(c, n_up, n_down);
    for (int k = 0; k < n; ++k) info.block_dim[k] = static_cast<uint64_t>(c.block_dims[k]);
    if (c.timing) {
      FTLM_CUDA(cudaEventRecord(e1, c.stream));
      FTLM_CUDA(cudaEventSynchronize(e1));
      float ms = 0.f;
      FTLM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      c.prof.sector_ms += ms;
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
    }
    if (out) *out = info;
  });
}

int ftlm_spectra_reset(ftlm_ctx* ctx) {
  return ftlm::guarded(ctx, [&](Ctx& c) { ftlm::spectra_reset(c); });
}

int ftlm_blocks_exact_batched(ftlm_ctx* ctx, const int32_t* mx, const int32_t* my, int32_t nblocks) {
  return ftlm::guarded(ctx, [&](Ctx& c) {
    ftlm::need_sector(c);
    if (nblocks < 0 || (nblocks > 0 && (!mx || !my))) throw Error(FTLM_ERR_ARG, "bad block list");
    std::vector<std::pair<int, int>> list;
    for (int i = 0; i < nblocks; ++i) {
      ftlm::check_k(c, mx[i], my[i]);
      list.emplace_back(mx[i], my[i]);
    }
    if (c.spectra_defer) ftlm::queue_exact_blocks(c, list);
    else ftlm::run_exact_blocks(c, list);
  });
}

int ftlm_spectra_defer(ftlm_ctx* ctx, int32_t on) {
  return ftlm::guarded(ctx, [&](Ctx& c) {
    if (!on) ftlm::flush_deferred(c);
    c.spectra_defer = on != 0;
  });
}

int ftlm_spectra_flush(ftlm_ctx* ctx) {
  return ftlm::guarded(ctx, [&](Ctx& c) { ftlm::flush_deferred(c); });
}

int ftlm_blocks_ftlm_batched(ftlm_ctx* ctx, const int32_t* mx, const int32_t* my, int32_t nblocks) {
  return ftlm::guarded(ctx, [&](Ctx& c) {
    ftlm::need_sector(c);
    if (nblocks < 0 || (nblocks > 0 && (!mx || !my))) throw Error(FTLM_ERR_ARG, "bad block list");
    static_assert(FTLM_SMALL_BLOCK_MAX == ftlm::kSmallMaxDim, "small-block limit");
    std::vector<std::pair<int, int>> small, large;
    for (int i = 0; i < nblocks; ++i) {
      ftlm::check_k(c, mx[i], my[i]);
      const int64_t d = c.block_dims[my[i] * c.geom.lx + mx[i]];
      if (d <= 0) continue;
      (c.small_blocks && d <= ftlm::kSmallMaxDim ? small : large).emplace_back(mx[i], my[i]);
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (c.timing) {
      FTLM_CUDA(cudaEventCreate(&e0));
      FTLM_CUDA(cudaEventCreate(&e1));
      FTLM_CUDA(cudaEventRecord(e0, c.stream));
    }
    ftlm::run_small_ftlm_blocks(c, small);
    for (const auto& b : large) {
      ftlm::Spectrum s;
      ftlm::run_ftlm_block(c, c.sec.n_up, c.sec.n_dn, b.first, b.second, s, nullptr, nullptr, nullptr, nullptr);
      c.spec[b] = s;
    }
    if (c.timing) {
      FTLM_CUDA(cudaEventRecord(e1, c.stream));
      FTLM_CUDA(cudaEventSynchronize(e1));
      float ms = 0.f;
      FTLM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      c.prof.block_ms += ms;
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
    }
  });
}

int ftlm_block_spectrum(ftlm_ctx* ctx, int32_t mx, int32_t my, int32_t exact, double* evals, double* weights,
                        size_t cap, size_t* count, double* trace_prefactor) {
  return ftlm::guarded(ctx, [&](Ctx& c) {
    ftlm::need_sector(c);
    ftlm::check_k(c, mx, my);
    const auto key = std::make_pair(static_cast<int>(mx), static_cast<int>(my));
    auto it = c.spec.find(key);
    const bool have = it != c.spec.end() && it->second.exact == (exact != 0);
    if (have && (it->second.pending >= 0 || it->second.pending_ritz >= 0)) {  // pooled: solve the pool now
      ftlm::flush_deferred(c);
      it = c.spec.find(key);
    }
    if (!have) {
      cudaEvent_t e0 = nullptr, e1 = nullptr;
      if (c.timing) {
        FTLM_CUDA(cudaEventCreate(&e0));
        FTLM_CUDA(cudaEventCreate(&e1));
        FTLM_CUDA(cudaEventRecord(e0, c.stream));
      }
      if (exact) {
        ftlm::run_exact_blocks(c, {key});
      } else {
        ftlm::Spectrum s;
        ftlm::run_ftlm_block(c, c.sec.n_up, c.sec.n_dn, mx, my, s, nullptr, nullptr, nullptr, nullptr);
        c.spec[key] = s;
      }
      if (c.timing) {
        FTLM_CUDA(cudaEventRecord(e1, c.stream));
        FTLM_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        FTLM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        c.prof.block_ms += ms;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
      }
      it = c.spec.find(key);
      if (it == c.spec.end()) {  // empty block
        if (count) *count = 0;
        if (trace_prefactor) *trace_prefactor = exact ? 1.0 : 0.0;
        return;
      }
    }
    const ftlm::Spectrum& s = it->second;
    if (count) *count = static_cast<size_t>(s.count);
    if (trace_prefactor) *trace_prefactor = s.prefactor;
    if (evals) {
      if (cap < static_cast<size_t>(s.count)) throw Error(FTLM_ERR_CAPACITY, "spectrum buffer too small");
      FTLM_CUDA(cudaMemcpyAsync(evals, c.spectra.as<double>() + s.ev_off, sizeof(double) * s.count,
                                cudaMemcpyDeviceToHost, c.stream));
      c.prof.d2h_bytes += static_cast<int64_t>(sizeof(double)) * s.count;
      if (weights && s.w_off >= 0) {
        FTLM_CUDA(cudaMemcpyAsync(weights, c.spectra.as<double>() + s.w_off, sizeof(double) * s.count,
                                  cudaMemcpyDeviceToHost, c.stream));
        c.prof.d2h_bytes += static_cast<int64_t>(sizeof(double)) * s.count;
      }
      FTLM_CUDA(cudaStreamSynchronize(c.stream));
    }
  });
}

int ftlm_thermo_configure(ftlm_ctx* ctx, int32_t nbeta, const double* betas, int32_t nmu, const double* mu) {
  return ftlm::guarded(ctx, [&](Ctx& c) {
    if (nbeta <= 0 || nmu <= 0 || !betas || !mu) throw Error(FTLM_ERR_ARG, "bad beta/mu grid");
    for (int i = 0; i < nbeta; ++i)
      if (!(betas[i] > 0.0)) throw Error(FTLM_ERR_ARG, "All beta values must be positive.");
    ftlm::flush_deferred(c);  // queued accumulations belong to the previous grid
    ftlm::thermo_configure(c, nbeta, betas, nmu, mu);
  });
}

int ftlm_thermo_accumulate_block(ftlm_ctx* ctx, int32_t mx, int32_t my) {
  return ftlm::guarded(ctx, [&](Ctx& c) {
    ftlm::need_sector(c);
    ftlm::check_k(c, mx, my);
    auto it = c.spec.find({mx, my});
    if (it == c.spec.end()) throw Error(FTLM_ERR_STATE, "block spectrum not computed");
    if (it->second.pending >= 0 || it->second.pending_ritz >= 0) {  // accumulated when the pool is solved
      if (c.nbeta <= 0 || c.nmu <= 0) throw Error(FTLM_ERR_STATE, "thermo accumulators not configured");
      const bool ritz = it->second.pending_ritz >= 0;
      c.defer_acc.push_back({ritz, ritz ? it->second.pending_ritz : it->second.pending});
      return;
    }
    ftlm::thermo_accumulate(c, it->second);
  });
}

int ftlm_thermo_accumulate_host(ftlm_ctx* ctx, const double* evals, const double* weights, size_t count,
                                double trace_prefactor, int32_t particles) {
  return ftlm::guarded(ctx, [&](Ctx& c) {
    if (count > 0 && !evals) throw Error(FTLM_ERR_ARG, "null spectrum");
    ftlm::thermo_accumulate_host(c, evals, weights, static_cast<int64_t>(count), trace_prefactor, particles);
  });
}

int ftlm_thermo_read(ftlm_ctx* ctx, double* emin, double* z, double* n, double* n2) {
  return ftlm::guarded(ctx, [&](Ctx& c) {
    if (!emin || !z || !n || !n2) throw Error(FTLM_ERR_ARG, "null output");
    if (c.nbeta <= 0) throw Error(FTLM_ERR_STATE, "thermo accumulators not configured");
    ftlm::flush_deferred(c);
    ftlm::thermo_read(c, emin, z, n, n2);
  });
}

int ftlm_block_apply(ftlm_ctx* ctx, int32_t mx, int32_t my, int32_t nvec, const double* in, double* out) {
  return ftlm::guarded(ctx, [&](Ctx& c) {
    ftlm::need_sector(c);
    ftlm::check_k(c, mx, my);
    if (!in || !out) throw Error(FTLM_ERR_ARG, "null vector");
    const bool fp32 = c.opts.precision == FTLM_PREC_MIXED;
    int NV = 1;
    while (NV < nvec) NV <<= 1;
    if (fp32 && NV < 2) NV = 2;
    if (nvec <= 0 || NV > 128) throw Error(FTLM_ERR_ARG, "nvec must be in 1..128");
    ftlm::block_prepare(c, mx, my);
    const int64_t D = c.blk.dim;
    if (D == 0) return;
    const size_t esize = fp32 ? 8 : 16;
    const size_t bytes = static_cast<size_t>(D) * NV * esize;
    c.vec_a.ensure(bytes);
    c.vec_h.ensure(bytes);
    // pack host [dim][nvec] FP64 complex into [dim][NV] of the working precision
    std::vector<char> h(bytes, 0);
    for (int64_t i = 0; i < D; ++i)
      for (int v = 0; v < nvec; ++v) {
        const double re = in[2 * (i * nvec + v)], im = in[2 * (i * nvec + v) + 1];
        if (fp32) {
          float* p = reinterpret_cast<float*>(h.data()) + 2 * (i * NV + v);
          p[0] = static_cast<float>(re);
          p[1] = static_cast<float>(im);
        } else {
          double* p = reinterpret_cast<double*>(h.data()) + 2 * (i * NV + v);
          p[0] = re;
          p[1] = im;
        }
      }
    FTLM_CUDA(cudaMemcpyAsync(c.vec_a.p, h.data(), bytes, cudaMemcpyHostToDevice, c.stream));
    c.prof.h2d_bytes += static_cast<int64_t>(bytes);
    ftlm::HvSourceGuard guard{c};
    c.prof.hv_source = ftlm::hv_select_source(c, NV, fp32);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (c.timing) {
      FTLM_CUDA(cudaEventCreate(&e0));
      FTLM_CUDA(cudaEventCreate(&e1));
      FTLM_CUDA(cudaEventRecord(e0, c.stream));
    }
    if (c.split_active) {
      ftlm::flip_scatter(c, c.vec_a.p, c.vec_xd.p, NV, fp32);
      ftlm::hv_apply_split(c, c.vec_a.p, c.vec_xd.p, c.vec_h.p, c.vec_yd.p, NV, fp32, nullptr, nullptr);
      ftlm::flip_gather_add(c, c.vec_h.p, c.vec_yd.p, NV, fp32);
    } else {
      ftlm::hv_apply(c, c.vec_a.p, c.vec_h.p, NV, fp32, nullptr, nullptr, 0);
    }
    if (c.timing) {
      FTLM_CUDA(cudaEventRecord(e1, c.stream));
    }
    FTLM_CUDA(cudaMemcpyAsync(h.data(), c.vec_h.p, bytes, cudaMemcpyDeviceToHost, c.stream));
    FTLM_CUDA(cudaStreamSynchronize(c.stream));
    c.prof.d2h_bytes += static_cast<int64_t>(bytes);
    if (c.timing) {
      float ms = 0.f;
      FTLM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      c.prof.hv_ms += ms;
      c.prof.hv_launches += 1;
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      const double s = fp32 ? 8.0 : 16.0;
      const double nzh = static_cast<double>(ftlm::block_nonzero_hops(c));
      c.prof.hv_bytes += static_cast<double>(D) * nvec * s * 2.0 + nzh * nvec * s + static_cast<double>(D) * 8.0;
      c.prof.hv_hops += nzh * nvec;
      c.prof.hv_min_bytes += static_cast<double>(D) * (2.0 * nvec * s + 8.0);
    }
    for (int64_t i = 0; i < D; ++i)
      for (int v = 0; v < nvec; ++v) {
        if (fp32) {
          const float* p = reinterpret_cast<const float*>(h.data()) + 2 * (i * NV + v);
          out[2 * (i * nvec + v)] = p[0];
          out[2 * (i * nvec + v) + 1] = p[1];
        } else {
          const double* p = reinterpret_cast<const double*>(h.data()) + 2 * (i * NV + v);
          out[2 * (i * nvec + v)] = p[0];
          out[2 * (i * nvec + v) + 1] = p[1];
        }
      }
  });
}

int ftlm_block_lanczos(ftlm_ctx* ctx, int32_t mx, int32_t my, const double* start, double* alpha, double* beta,
                       int32_t* steps) {
  return ftlm::guarded(ctx, [&](Ctx& c) {
    ftlm::need_sector(c);
    ftlm::check_k(c, mx, my);
    if (!alpha || !beta || !steps) throw Error(FTLM_ERR_ARG, "null output");
    std::vector<double> a, b;
    std::vector<int32_t> s;
    ftlm::Spectrum sp;
    ftlm::run_ftlm_block(c, c.sec.n_up, c.sec.n_dn, mx, my, sp, start, &a, &b, &s);
    c.spec[{mx, my}] = sp;
    std::memcpy(alpha, a.data(), sizeof(double) * a.size());
    std::memcpy(beta, b.data(), sizeof(double) * b.size());
    std::memcpy(steps, s.data(), sizeof(int32_t) * s.size());
  });
}

int ftlm_debug_sector_parents(ftlm_ctx* ctx, uint64_t* up, uint64_t* down, int32_t* deg, double* diag, size_t cap,
                              size_t* count) {
  return ftlm::guarded(ctx, [&](Ctx& c) {
    ftlm::need_sector(c);
    const size_t P = static_cast<size_t>(c.sec.parents);
    if (count) *count = P;
    if (!up) return;
    if (!down || !deg || !diag) throw Error(FTLM_ERR_ARG, "null output");
    if (cap < P) throw Error(FTLM_ERR_CAPACITY, "parent buffer too small");
    ftlm::debug_parents(c, up, down, deg, diag);
  });
}

int ftlm_debug_sector_relations(ftlm_ctx* ctx, int32_t* parent, int32_t* shift, int32_t* sign, size_t cap) {
  return ftlm::guarded(ctx, [&](Ctx& c) {
    ftlm::need_sector(c);
    if (!parent || !shift || !sign) throw Error(FTLM_ERR_ARG, "null output");
    if (cap < static_cast<size_t>(c.sec.full_dim)) throw Error(FTLM_ERR_CAPACITY, "relation buffer too small");
    ftlm::debug_relations(c, parent, shift, sign);
  });
}

int ftlm_debug_block_csr(ftlm_ctx* ctx, int32_t mx, int32_t my, double* diag, int32_t* row_ptr, int32_t* col,
                         double* val, size_t dim_cap, size_t nnz_cap, size_t* dim, size_t* nnz) {
  return ftlm::guarded(ctx, [&](Ctx& c) {
    ftlm::need_sector(c);
    ftlm::check_k(c, mx, my);
    ftlm::block_prepare(c, mx, my);
    std::vector<int32_t> rp, cl;
    std::vector<double> vl, dg;
    if (c.blk.dim > 0) ftlm::block_csr(c, rp, cl, vl, dg);
    else rp.assign(1, 0);
    if (dim) *dim = static_cast<size_t>(c.blk.dim);
    if (nnz) *nnz = cl.size();
    if (!row_ptr) return;
    if (dim_cap < static_cast<size_t>(c.blk.dim) || nnz_cap < cl.size())
      throw Error(FTLM_ERR_CAPACITY, "CSR buffers too small");
    std::memcpy(row_ptr, rp.data(), sizeof(int32_t) * rp.size());
    if (!cl.empty()) {
      std::memcpy(col, cl.data(), sizeof(int32_t) * cl.size());
      std::memcpy(val, vl.data(), sizeof(double) * vl.size());
    }
    if (!dg.empty()) std::memcpy(diag, dg.data(), sizeof(double) * dg.size());
  });
}

int ftlm_profile_enable(ftlm_ctx* ctx, int32_t on) {
  return ftlm::guarded(ctx, [&](Ctx& c) { c.timing = on != 0; });
}

int ftlm_profile_read(ftlm_ctx* ctx, ftlm_profile* out) {
  return ftlm::guarded(ctx, [&](Ctx& c) {
    if (!out) throw Error(FTLM_ERR_ARG, "null output");
    const ftlm::Profile& p = c.prof;
    out->hv_ms = p.hv_ms;
    out->hv_launches = p.hv_launches;
    out->hv_bytes = p.hv_bytes;
    out->update_ms = p.update_ms;
    out->update_launches = p.update_launches;
    out->eig_ms = p.eig_ms;
    out->dense_ms = p.dense_ms;
    out->thermo_ms = p.thermo_ms;
    out->sector_ms = p.sector_ms;
    out->block_ms = p.block_ms;
    out->kernel_launches = p.kernel_launches;
    out->h2d_bytes = p.h2d_bytes;
    out->d2h_bytes = p.d2h_bytes;
    out->hv_variant = p.hv_variant;
    out->tune_runs = p.tune_runs;
    out->small_ms = p.small_ms;
    out->small_tasks = p.small_tasks;
    out->hv_hops = p.hv_hops;
    out->hv_min_bytes = p.hv_min_bytes;
    out->hv_source = p.hv_source;
    out->pad0 = 0;
  });
}

int ftlm_profile_reset(ftlm_ctx* ctx) {
  return ftlm::guarded(ctx, [&](Ctx& c) { c.prof = ftlm::Profile{}; });
}

}  // extern "C"
