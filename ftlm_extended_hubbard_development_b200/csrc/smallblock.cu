// Small FTLM blocks in one persistent launch (run_ftlm_block,
// main.cpp:996-1113, for every block of a sector up to kSmallMaxDim rows).
//
// A block of a few thousand rows gives one H*V far too little work to fill
// the GPU, so stepping it with the sweep kernels spends its time in launch
// latency (four launches per Lanczos step). Here one CTA runs the whole
// Lanczos recurrence of one (block, random vector) pair: the three working
// vectors live in shared memory, the block's CSR (reference entry order) is
// read from L2, where all CTAs of the block share it, and alpha/beta go to
// the same [K][ld] layout the sweep path writes, so the Ritz stage
// (k_tridiag) and everything after it are shared. Tasks are ordered largest
// block first and taken in a grid-stride loop by a grid sized to the SMs.
//
// Arithmetic is the reference's: w = H v; alpha = Re<v, w>;
// w -= alpha v + beta_prev v_prev; beta = |w|; stop at beta < 1e-12 or the
// last step; v_next = w / beta. Sums are FP64 in a fixed order
// (deterministic). In mixed precision the vectors are stored as FP32 complex
// (each element rounded once per step) and every sum stays FP64.
#include <algorithm>
#include <cmath>
#include <numeric>

#include "ftlm_internal.h"

namespace ftlm {

namespace {

constexpr int kSmallThreads = 256;
constexpr int kRowLanes = 8;  // lanes sharing one CSR row
constexpr int kWarps = kSmallThreads / 32;

struct SmallBlockDesc {
  int64_t rp_off;     // row pointers (int32) at rp[rp_off .. rp_off+dim]
  int64_t nz_off;     // CSR entries start at col/val[nz_off]
  int64_t diag_off;   // diagonal at diag[diag_off ..)
  int64_t ab_off;     // alpha/beta [K][ld] at ab[ab_off ..)
  int64_t start_off;  // reference start vectors [R][dim] complex at start[start_off ..), -1: Philox
  int64_t steps_off;  // steps[steps_off + r]
  uint64_t seed;      // block seed (Philox key)
  int32_t dim, K, ld, pad;
};

template <typename T>
struct CT;
template <>
struct CT<double> {
  using C = double2;
  __device__ static C make(double re, double im) { return make_double2(re, im); }
};
template <>
struct CT<float> {
  using C = float2;
  __device__ static C make(double re, double im) {
    return make_float2(static_cast<float>(re), static_cast<float>(im));
  }
};

// Fixed-order CTA sum of one double per thread; every thread gets the result.
__device__ __forceinline__ double cta_sum(double v, double* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int warp = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) red[warp] = v;
  __syncthreads();
  double s = 0.0;
#pragma unroll
  for (int i = 0; i < kWarps; ++i) s += red[i];
  __syncthreads();  // red is reused by the next sum
  return s;
}

template <typename T>
__global__ void __launch_bounds__(kSmallThreads) k_lanczos_small(
    int ntasks, const int2* __restrict__ tasks, const SmallBlockDesc* __restrict__ blocks,
    const int32_t* __restrict__ rp_all, const int32_t* __restrict__ col_all, const double2* __restrict__ val_all,
    const double* __restrict__ diag_all, const double2* __restrict__ start_all, double* __restrict__ alpha_all,
    double* __restrict__ beta_all, int32_t* __restrict__ steps_all, int cap) {
  using C = typename CT<T>::C;
  extern __shared__ __align__(16) unsigned char small_smem[];
  C* b0 = reinterpret_cast<C*>(small_smem);
  __shared__ double red[kWarps];
  const int tid = threadIdx.x;
  const int lane8 = tid & (kRowLanes - 1);
  const int group = tid / kRowLanes;
  constexpr int kGroups = kSmallThreads / kRowLanes;
  for (int t = blockIdx.x; t < ntasks; t += gridDim.x) {
    const int2 task = tasks[t];
    const SmallBlockDesc B = blocks[task.x];
    const int r = task.y;
    const int D = B.dim;
    const int32_t* rp = rp_all + B.rp_off;
    const int32_t* col = col_all + B.nz_off;
    const double2* val = val_all + B.nz_off;
    const double* diag = diag_all + B.diag_off;
    C* v = b0;
    C* vp = b0 + cap;
    C* w = b0 + 2 * cap;
    const double amp = 1.0 / sqrt(static_cast<double>(D));
    for (int i = tid; i < D; i += kSmallThreads) {
      double re, im;
      if (B.start_off >= 0) {
        const double2 z = start_all[B.start_off + static_cast<int64_t>(r) * D + i];
        re = z.x;
        im = z.y;
      } else {
        philox_phase(i, r, B.seed, amp, re, im);
      }
      v[i] = CT<T>::make(re, im);
      vp[i] = CT<T>::make(0.0, 0.0);
    }
    __syncthreads();
    double beta_prev = 0.0;
    int steps = B.K;
    for (int j = 0; j < B.K; ++j) {
      // w = H v; partial Re<v, w>
      double ap = 0.0;
      // the row loop is warp-uniform (the shuffles below need all 32 lanes):
      // each warp takes 4 consecutive rows per pass, one per 8-lane group
      for (int i0 = (tid >> 5) * (32 / kRowLanes); i0 < D; i0 += kGroups) {
        const int i = i0 + group % (32 / kRowLanes);
        double ar = 0.0, ai = 0.0;
        const int e0 = i < D ? rp[i] + lane8 : 0;
        const int e1 = i < D ? rp[i + 1] : 0;
        for (int e = e0; e < e1; e += kRowLanes) {
          const double2 h = val[e];
          const C x = v[col[e]];
          ar += h.x * static_cast<double>(x.x) - h.y * static_cast<double>(x.y);
          ai += h.x * static_cast<double>(x.y) + h.y * static_cast<double>(x.x);
        }
#pragma unroll
        for (int o = kRowLanes / 2; o > 0; o >>= 1) {
          ar += __shfl_xor_sync(0xffffffffu, ar, o);
          ai += __shfl_xor_sync(0xffffffffu, ai, o);
        }
        if (lane8 == 0 && i < D) {
          const C xi = v[i];
          ar += diag[i] * static_cast<double>(xi.x);
          ai += diag[i] * static_cast<double>(xi.y);
          const C wi = CT<T>::make(ar, ai);
          w[i] = wi;
          ap += static_cast<double>(xi.x) * static_cast<double>(wi.x) +
                static_cast<double>(xi.y) * static_cast<double>(wi.y);
        }
      }
      const double alpha = cta_sum(ap, red);  // also orders the writes of w before the update
      // w -= alpha v + beta_prev vp; partial |w|^2
      double np = 0.0;
      for (int i = tid; i < D; i += kSmallThreads) {
        const C hi = w[i], xi = v[i], pi = vp[i];
        const C ri = CT<T>::make(static_cast<double>(hi.x) - alpha * static_cast<double>(xi.x) -
                                     beta_prev * static_cast<double>(pi.x),
                                 static_cast<double>(hi.y) - alpha * static_cast<double>(xi.y) -
                                     beta_prev * static_cast<double>(pi.y));
        w[i] = ri;
        np += static_cast<double>(ri.x) * static_cast<double>(ri.x) +
              static_cast<double>(ri.y) * static_cast<double>(ri.y);
      }
      const double beta = sqrt(cta_sum(np, red));
      if (tid == 0) alpha_all[B.ab_off + static_cast<int64_t>(j) * B.ld + r] = alpha;
      if (beta < 1e-12 || j + 1 == B.K) {  // uniform: every thread holds the same beta
        steps = j + 1;
        break;
      }
      if (tid == 0) beta_all[B.ab_off + static_cast<int64_t>(j) * B.ld + r] = beta;
      const double inv = 1.0 / beta;
      for (int i = tid; i < D; i += kSmallThreads) {
        const C ri = w[i];
        w[i] = CT<T>::make(static_cast<double>(ri.x) * inv, static_cast<double>(ri.y) * inv);
      }
      __syncthreads();
      C* tmp = vp;  // rotate: v_prev <- v, v <- w, w <- old v_prev
      vp = v;
      v = w;
      w = tmp;
      beta_prev = beta;
    }
    if (tid == 0) steps_all[B.steps_off + r] = steps;
    __syncthreads();  // the next task overwrites the vectors
  }
}

}  // namespace

void run_small_ftlm_blocks(Ctx& c, const std::vector<std::pair<int, int>>& blocks) {
  if (blocks.empty()) return;
  const bool fp32 = c.opts.precision == FTLM_PREC_MIXED;
  const int R = c.opts.samples;
  struct Item {
    int mx, my;
    int64_t dim;
    int K;
    SmallBlockDesc d;
  };
  std::vector<Item> items;
  int64_t rp_tot = 0, nz_tot = 0, dg_tot = 0, ab_tot = 0, st_tot = 0;
  int ld = 1;  // alpha/beta row stride, as the sweep path uses for one sweep of R vectors
  while (ld < std::max(R, fp32 ? 2 : 1)) ld <<= 1;
  for (const auto& b : blocks) {
    const int64_t D = c.block_dims.at(static_cast<size_t>(b.second * c.geom.lx + b.first));
    if (D <= 0) continue;
    if (D > kSmallMaxDim) throw Error(FTLM_ERR_ARG, "block too large for the small-block FTLM launch");
    Item it{b.first, b.second, D, static_cast<int>(std::min<int64_t>(c.opts.lanczos_steps, D)), {}};
    items.push_back(it);
  }
  if (items.empty()) return;
  // CSR of every block into one arena (built block by block)
  DBuf rp, cl, vl, dg;
  std::vector<int64_t> nnz(items.size());
  for (size_t i = 0; i < items.size(); ++i) {
    Item& it = items[i];
    it.d.rp_off = rp_tot;
    it.d.diag_off = dg_tot;
    it.d.ab_off = ab_tot;
    it.d.steps_off = st_tot;
    rp_tot += it.dim + 1;
    dg_tot += it.dim;
    ab_tot += static_cast<int64_t>(it.K) * ld;
    st_tot += R;
  }
  for (size_t i = 0; i < items.size(); ++i) {
    block_prepare(c, items[i].mx, items[i].my);
    nnz[i] = block_csr_device(c, rp, cl, vl, dg);
    items[i].d.nz_off = nz_tot;
    nz_tot += std::max<int64_t>(nnz[i], 1);
    // copy into the arenas right away (the per-block buffers are rebuilt next)
    c.sb_rp.ensure_keep(sizeof(int32_t) * rp_tot, c.stream);
    c.sb_col.ensure_keep(sizeof(int32_t) * nz_tot, c.stream);
    c.sb_val.ensure_keep(sizeof(double2) * nz_tot, c.stream);
    c.sb_diag.ensure_keep(sizeof(double) * dg_tot, c.stream);
    const Item& it = items[i];
    FTLM_CUDA(cudaMemcpyAsync(c.sb_rp.as<int32_t>() + it.d.rp_off, rp.p, sizeof(int32_t) * (it.dim + 1),
                              cudaMemcpyDeviceToDevice, c.stream));
    if (nnz[i] > 0) {
      FTLM_CUDA(cudaMemcpyAsync(c.sb_col.as<int32_t>() + it.d.nz_off, cl.p, sizeof(int32_t) * nnz[i],
                                cudaMemcpyDeviceToDevice, c.stream));
      FTLM_CUDA(cudaMemcpyAsync(c.sb_val.as<double2>() + it.d.nz_off, vl.p, sizeof(double2) * nnz[i],
                                cudaMemcpyDeviceToDevice, c.stream));
    }
    FTLM_CUDA(cudaMemcpyAsync(c.sb_diag.as<double>() + it.d.diag_off, dg.p, sizeof(double) * it.dim,
                              cudaMemcpyDeviceToDevice, c.stream));
    FTLM_CUDA(cudaStreamSynchronize(c.stream));  // rp/cl/vl/dg are rebuilt for the next block
  }
  rp.release();
  cl.release();
  vl.release();
  dg.release();
  // start vectors: reference Gaussian ones from the host, Philox on the device
  const bool ref_start = c.opts.start_vector == FTLM_START_REF_GAUSSIAN;
  std::vector<double> hstart;
  int64_t start_tot = 0;
  for (Item& it : items) {
    it.d.seed = block_seed(c.opts.seed, c.sec.n_up, c.sec.n_dn, it.mx, it.my);
    it.d.dim = static_cast<int32_t>(it.dim);
    it.d.K = it.K;
    it.d.ld = ld;
    it.d.pad = 0;
    it.d.start_off = ref_start ? start_tot : -1;
    if (ref_start) start_tot += static_cast<int64_t>(R) * it.dim;
  }
  if (ref_start) {
    hstart.resize(2 * static_cast<size_t>(start_tot));
    for (const Item& it : items)
      reference_start_vectors(it.d.seed, 0, R, it.dim, hstart.data() + 2 * it.d.start_off);
    c.host_start.ensure(sizeof(double) * hstart.size());
    FTLM_CUDA(cudaMemcpyAsync(c.host_start.p, hstart.data(), sizeof(double) * hstart.size(), cudaMemcpyHostToDevice,
                              c.stream));
    c.prof.h2d_bytes += static_cast<int64_t>(sizeof(double) * hstart.size());
  }
  // tasks, largest block first
  std::vector<int> order(items.size());
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return items[a].dim > items[b].dim; });
  std::vector<int2> tasks;
  tasks.reserve(items.size() * R);
  int64_t dmax = 0;
  for (int b : order) {
    dmax = std::max(dmax, items[b].dim);
    for (int r = 0; r < R; ++r) tasks.push_back(make_int2(b, r));
  }
  std::vector<SmallBlockDesc> desc(items.size());
  for (size_t i = 0; i < items.size(); ++i) desc[i] = items[i].d;
  c.sb_meta.ensure(sizeof(int2) * tasks.size() + sizeof(SmallBlockDesc) * desc.size() + 64);
  int2* d_tasks = c.sb_meta.as<int2>();
  SmallBlockDesc* d_desc = reinterpret_cast<SmallBlockDesc*>(
      (reinterpret_cast<uintptr_t>(d_tasks + tasks.size()) + 15) & ~static_cast<uintptr_t>(15));
  FTLM_CUDA(cudaMemcpyAsync(d_tasks, tasks.data(), sizeof(int2) * tasks.size(), cudaMemcpyHostToDevice, c.stream));
  FTLM_CUDA(cudaMemcpyAsync(d_desc, desc.data(), sizeof(SmallBlockDesc) * desc.size(), cudaMemcpyHostToDevice,
                            c.stream));
  c.lz_alpha.ensure(sizeof(double) * ab_tot);
  c.lz_beta.ensure(sizeof(double) * ab_tot);
  FTLM_CUDA(cudaMemsetAsync(c.lz_alpha.p, 0, sizeof(double) * ab_tot, c.stream));
  FTLM_CUDA(cudaMemsetAsync(c.lz_beta.p, 0, sizeof(double) * ab_tot, c.stream));
  c.sb_steps.ensure(sizeof(int32_t) * st_tot);
  // one persistent launch
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (c.timing) {
    FTLM_CUDA(cudaEventCreate(&e0));
    FTLM_CUDA(cudaEventCreate(&e1));
    FTLM_CUDA(cudaEventRecord(e0, c.stream));
  }
  const int cap = static_cast<int>(dmax);
  const size_t smem = static_cast<size_t>(3) * cap * (fp32 ? sizeof(float2) : sizeof(double2));
  int per_sm = 1;
  if (fp32) {
    FTLM_CUDA(cudaFuncSetAttribute(k_lanczos_small<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(std::max<size_t>(smem, 1))));
    FTLM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_lanczos_small<float>, kSmallThreads, smem));
  } else {
    FTLM_CUDA(cudaFuncSetAttribute(k_lanczos_small<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(std::max<size_t>(smem, 1))));
    FTLM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_lanczos_small<double>, kSmallThreads, smem));
  }
  if (per_sm < 1) throw Error(FTLM_ERR_CAPACITY, "small-block Lanczos does not fit on an SM");
  const int grid = static_cast<int>(std::min<int64_t>(static_cast<int64_t>(tasks.size()),
                                                      static_cast<int64_t>(c.sm_count) * per_sm));
  const double2* start = ref_start ? c.host_start.as<double2>() : nullptr;
  if (fp32)
    k_lanczos_small<float><<<grid, kSmallThreads, smem, c.stream>>>(
        static_cast<int>(tasks.size()), d_tasks, d_desc, c.sb_rp.as<int32_t>(), c.sb_col.as<int32_t>(),
        c.sb_val.as<double2>(), c.sb_diag.as<double>(), start, c.lz_alpha.as<double>(), c.lz_beta.as<double>(),
        c.sb_steps.as<int32_t>(), cap);
  else
    k_lanczos_small<double><<<grid, kSmallThreads, smem, c.stream>>>(
        static_cast<int>(tasks.size()), d_tasks, d_desc, c.sb_rp.as<int32_t>(), c.sb_col.as<int32_t>(),
        c.sb_val.as<double2>(), c.sb_diag.as<double>(), start, c.lz_alpha.as<double>(), c.lz_beta.as<double>(),
        c.sb_steps.as<int32_t>(), cap);
  FTLM_LAUNCH_CHECK();
  c.prof.kernel_launches += 1;
  if (c.timing) {
    FTLM_CUDA(cudaEventRecord(e1, c.stream));
    FTLM_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    FTLM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    c.prof.small_ms += ms;
    c.prof.small_tasks += static_cast<int64_t>(tasks.size());
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  }
  if (c.spectra_defer) {
    // Lanczos coefficients into the pool; the Ritz stage runs for every
    // pooled block of every sector in one launch when the pool is flushed
    const int64_t add = static_cast<int64_t>(sizeof(double)) * 2 * ab_tot + static_cast<int64_t>(sizeof(int32_t)) * st_tot;
    if (defer_pool_bytes(c) > 0 && defer_pool_bytes(c) + add > kDeferPoolBytes) flush_deferred(c);
    const int64_t ab0 = c.defer_ab_used, st0 = c.defer_st_used;
    c.defer_ab.ensure_keep(sizeof(double) * (ab0 + 2 * ab_tot), c.stream);
    c.defer_st.ensure_keep(sizeof(int32_t) * (st0 + st_tot), c.stream);
    FTLM_CUDA(cudaMemcpyAsync(c.defer_ab.as<double>() + ab0, c.lz_alpha.p, sizeof(double) * ab_tot,
                              cudaMemcpyDeviceToDevice, c.stream));
    FTLM_CUDA(cudaMemcpyAsync(c.defer_ab.as<double>() + ab0 + ab_tot, c.lz_beta.p, sizeof(double) * ab_tot,
                              cudaMemcpyDeviceToDevice, c.stream));
    FTLM_CUDA(cudaMemcpyAsync(c.defer_st.as<int32_t>() + st0, c.sb_steps.p, sizeof(int32_t) * st_tot,
                              cudaMemcpyDeviceToDevice, c.stream));
    c.defer_ab_used = ab0 + 2 * ab_tot;
    c.defer_st_used = st0 + st_tot;
    for (const Item& it : items) {
      Spectrum s;
      s.exact = false;
      s.prefactor = static_cast<double>(it.dim);
      s.particles = c.sec.n_up + c.sec.n_dn;
      s.dim = it.dim;
      s.pending_ritz = static_cast<int>(c.defer_ritz.size());
      c.spec[{it.mx, it.my}] = s;
      c.defer_ritz.push_back(DeferRitz{c.sec.n_up, c.sec.n_dn, it.mx, it.my, R, ld, it.K, ab0 + it.d.ab_off,
                                       ab0 + ab_tot + it.d.ab_off, st0 + it.d.steps_off, it.dim, c.sec_gen});
    }
    return;
  }
  // Ritz values and weights per block, then compaction into the spectra arena
  std::vector<Spectrum> spec(items.size());
  std::vector<RitzJob> jobs;
  for (size_t i = 0; i < items.size(); ++i) {
    const Item& it = items[i];
    jobs.push_back(RitzJob{R, R, ld, it.K, c.lz_alpha.as<double>() + it.d.ab_off,
                           c.lz_beta.as<double>() + it.d.ab_off, c.sb_steps.as<int32_t>() + it.d.steps_off,
                           &spec[i]});
  }
  ritz_stage_many(c, jobs);
  for (size_t i = 0; i < items.size(); ++i) {
    spec[i].prefactor = static_cast<double>(items[i].dim);
    spec[i].particles = c.sec.n_up + c.sec.n_dn;
    spec[i].dim = items[i].dim;
    c.spec[{items[i].mx, items[i].my}] = spec[i];
  }
}

}  // namespace ftlm
