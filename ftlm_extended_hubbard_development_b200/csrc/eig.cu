// Exact block spectra on the GPU (diagonalize_block_exact, main.cpp:847-911).
//
// Every block of the list is assembled as a dense column-major Hermitian
// matrix straight from its hop enumeration (the CSR's entries, summed in
// the CSR's order, with no CSR stored and no host synchronisation between
// blocks), symmetrised as (M + M^H)/2 like the
// reference, then all matrices are diagonalised by ONE batched launch:
// one CTA per matrix (largest first) reduces it to real symmetric
// tridiagonal form with complex Householder reflections (trailing
// rank-2 updates, coalesced along columns) and finds every eigenvalue
// independently by Sturm-sequence bisection, one thread per eigenvalue,
// which yields them sorted ascending. Eigenvalues only (jobz = 'N').
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <numeric>

#include "ftlm_internal.h"

namespace ftlm {

namespace {

constexpr int kEigThreads = 256;
constexpr int kMaxDense = 7000;  // two complex work vectors in shared memory: 2*7000*16 B <= 227 KB

// (M + M^H)/2 with a real diagonal (main.cpp:875-886); upper triangle
// holds the average, the lower triangle its conjugate.
__global__ void k_dense_herm(int64_t n, double2* __restrict__ A) {
  for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < n * n;
       t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t i = t % n, j = t / n;
    if (i > j) continue;
    if (i == j) {
      A[i + i * n].y = 0.0;
      continue;
    }
    const double2 a = A[i + j * n], b = A[j + i * n];
    const double re = 0.5 * (a.x + b.x), im = 0.5 * (a.y - b.y);
    A[i + j * n] = make_double2(re, im);
    A[j + i * n] = make_double2(re, -im);
  }
}

__device__ double block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double s = 0.0;
  for (int w = 0; w < kEigThreads / 32; ++w) s += red[w];
  __syncthreads();
  return s;
}

__device__ double block_minmax(double v, double* red, bool is_max) {
  for (int o = 16; o > 0; o >>= 1) {
    const double t = __shfl_xor_sync(0xffffffffu, v, o);
    v = is_max ? fmax(v, t) : fmin(v, t);
  }
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double s = red[0];
  for (int w = 1; w < kEigThreads / 32; ++w) s = is_max ? fmax(s, red[w]) : fmin(s, red[w]);
  __syncthreads();
  return s;
}

// Number of eigenvalues of the tridiagonal (d, e2 = e^2) below x.
__device__ int sturm_count(int n, const double* d, const double* e2, double x, double pivmin) {
  double q = d[0] - x;
  if (fabs(q) < pivmin) q = -pivmin;
  int cnt = q < 0.0;
  for (int i = 1; i < n; ++i) {
    q = d[i] - x - e2[i - 1] / q;
    if (fabs(q) < pivmin) q = -pivmin;
    cnt += q < 0.0;
  }
  return cnt;
}

// One CTA per matrix. work: per matrix 2*n doubles (d, e2) at woff.
__global__ void __launch_bounds__(kEigThreads) k_dense_eig(int nmat, const int32_t* __restrict__ order,
                                                          const int32_t* __restrict__ dims,
                                                          const int64_t* __restrict__ aoff, double2* __restrict__ arena,
                                                          const int64_t* __restrict__ eoff, double* __restrict__ evout,
                                                          double* __restrict__ work, const int64_t* __restrict__ woff) {
  extern __shared__ double2 sh[];
  __shared__ double red[kEigThreads / 32];
  for (int task = blockIdx.x; task < nmat; task += gridDim.x) {
    const int mi = order[task];
    const int n = dims[mi];
    double2* A = arena + aoff[mi];
    double* d = work + woff[mi];
    double* e2 = d + n;
    double2* v = sh;
    double2* w = sh + n;
    const int tid = threadIdx.x;
    for (int k = 0; k + 2 < n; ++k) {
      const int m = n - k - 1;
      const int64_t base = (k + 1) + static_cast<int64_t>(k) * n;  // A[k+1][k]
      double s2 = 0.0;
      for (int i = tid; i < m; i += kEigThreads) {
        const double2 x = A[base + i];
        s2 += x.x * x.x + x.y * x.y;
      }
      const double alpha = sqrt(block_sum(s2, red));
      if (tid == 0) d[k] = A[k + static_cast<int64_t>(k) * n].x;
      if (alpha == 0.0) {
        if (tid == 0) e2[k] = 0.0;
        __syncthreads();
        continue;
      }
      const double2 x0 = A[base];
      const double ax0 = hypot(x0.x, x0.y);
      const double phr = ax0 > 0.0 ? x0.x / ax0 : 1.0;
      const double phi = ax0 > 0.0 ? x0.y / ax0 : 0.0;
      for (int i = tid; i < m; i += kEigThreads) {
        double2 x = A[base + i];
        if (i == 0) {
          x.x += phr * alpha;
          x.y += phi * alpha;
        }
        v[i] = x;
      }
      const double tau = 1.0 / (alpha * (alpha + ax0));  // 2 / |v|^2
      __syncthreads();
      // p = tau * B v, B = A[k+1.., k+1..] (thread per row, columns in order)
      const int64_t b0 = (k + 1) + static_cast<int64_t>(k + 1) * n;
      double kr = 0.0;
      for (int i = tid; i < m; i += kEigThreads) {
        double pr = 0.0, pi = 0.0;
        for (int j = 0; j < m; ++j) {
          const double2 b = A[b0 + i + static_cast<int64_t>(j) * n];
          const double2 vj = v[j];
          pr += b.x * vj.x - b.y * vj.y;
          pi += b.x * vj.y + b.y * vj.x;
        }
        pr *= tau;
        pi *= tau;
        w[i] = make_double2(pr, pi);
        kr += v[i].x * pr + v[i].y * pi;  // Re(conj(v_i) p_i)
      }
      const double K = 0.5 * tau * block_sum(kr, red);
      for (int i = tid; i < m; i += kEigThreads) {
        w[i].x -= K * v[i].x;
        w[i].y -= K * v[i].y;
      }
      __syncthreads();
      // B -= v w^H + w v^H
      for (int j = 0; j < m; ++j) {
        const double2 vj = v[j], wj = w[j];
        for (int i = tid; i < m; i += kEigThreads) {
          const double2 vi = v[i], wi = w[i];
          double2& b = A[b0 + i + static_cast<int64_t>(j) * n];
          b.x -= (vi.x * wj.x + vi.y * wj.y) + (wi.x * vj.x + wi.y * vj.y);
          b.y -= (vi.y * wj.x - vi.x * wj.y) + (wi.y * vj.x - wi.x * vj.y);
        }
      }
      if (tid == 0) e2[k] = alpha * alpha;
      __syncthreads();
    }
    if (tid == 0) {
      if (n >= 2) {
        d[n - 2] = A[(n - 2) + static_cast<int64_t>(n - 2) * n].x;
        const double2 t = A[(n - 1) + static_cast<int64_t>(n - 2) * n];
        e2[n - 2] = t.x * t.x + t.y * t.y;
      }
      d[n - 1] = A[(n - 1) + static_cast<int64_t>(n - 1) * n].x;
      e2[n - 1] = 0.0;
    }
    __syncthreads();
    // Gershgorin interval and bisection
    double lo = DBL_MAX, hi = -DBL_MAX, emax = 0.0;
    for (int i = tid; i < n; i += kEigThreads) {
      const double el = i > 0 ? sqrt(e2[i - 1]) : 0.0;
      const double er = i + 1 < n ? sqrt(e2[i]) : 0.0;
      lo = fmin(lo, d[i] - el - er);
      hi = fmax(hi, d[i] + el + er);
      emax = fmax(emax, e2[i]);
    }
    lo = block_minmax(lo, red, false);
    hi = block_minmax(hi, red, true);
    emax = block_minmax(emax, red, true);
    const double pivmin = DBL_MIN * fmax(1.0, emax);
    const double span = fmax(fabs(lo), fabs(hi));
    lo -= 4.0 * DBL_EPSILON * span + pivmin;
    hi += 4.0 * DBL_EPSILON * span + pivmin;
    double* ev = evout + eoff[mi];
    for (int j = tid; j < n; j += kEigThreads) {
      double a = lo, b = hi;
      for (int it = 0; it < 128; ++it) {
        const double mid = 0.5 * (a + b);
        if (mid <= a || mid >= b) break;
        if (b - a <= 2.0 * DBL_EPSILON * fmax(fabs(a), fabs(b))) break;
        if (sturm_count(n, d, e2, mid, pivmin) > j) b = mid;
        else a = mid;
      }
      ev[j] = 0.5 * (a + b);
    }
    __syncthreads();
  }
}

struct DenseItem {
  int mx, my;
  int64_t n, aoff, woff;
};

// Dimensions of the listed blocks (empty ones dropped); aoff/woff relative.
std::vector<DenseItem> dense_items(Ctx& c, const std::vector<std::pair<int, int>>& blocks, int64_t& asz,
                                   int64_t& wsz) {
  std::vector<DenseItem> items;
  asz = wsz = 0;
  for (const auto& b : blocks) {
    const int64_t n = c.block_dims.at(static_cast<size_t>(b.second * c.geom.lx + b.first));
    if (n <= 0) continue;
    if (n > kMaxDense) throw Error(FTLM_ERR_CAPACITY, "block too large for the dense exact solver: " + std::to_string(n));
    items.push_back({b.first, b.second, n, asz, wsz});
    asz += n * n;
    wsz += 2 * n;
  }
  return items;
}

// Dense Hermitian matrix of every item at arena + aoff (zeroed by the caller).
void dense_fill(Ctx& c, const std::vector<DenseItem>& items, double2* arena, int64_t abase) {
  for (const DenseItem& it : items) {
    // the block's rows are built in stream order; the fill reads them before
    // the next block_prepare overwrites them
    block_prepare(c, it.mx, it.my);
    double2* A = arena + abase + it.aoff;
    block_dense_device(c, A);
    const int g2 = static_cast<int>(std::min<int64_t>((it.n * it.n + 255) / 256, 4096));
    k_dense_herm<<<g2, 256, 0, c.stream>>>(it.n, A);
    FTLM_LAUNCH_CHECK();
    c.prof.kernel_launches += 1;
  }
}

// One k_dense_eig launch over matrices (dims, aoff into arena) writing the
// eigenvalues at evout + eoff; largest matrix first, one CTA per matrix.
void dense_solve(Ctx& c, const std::vector<int32_t>& dims, const std::vector<int64_t>& aoff,
                 const std::vector<int64_t>& eoff, double2* arena, double* evout, double* work) {
  const size_t nb = dims.size();
  if (nb == 0) return;
  std::vector<int32_t> order(nb);
  std::vector<int64_t> woff(nb);
  int64_t nmax = 0, wtot = 0;
  for (size_t i = 0; i < nb; ++i) {
    woff[i] = wtot;
    wtot += 2 * static_cast<int64_t>(dims[i]);
    nmax = std::max<int64_t>(nmax, dims[i]);
  }
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return dims[a] > dims[b]; });
  const size_t i32bytes = ((sizeof(int32_t) * 2 * nb + 7) / 8) * 8;  // int64 arrays stay 8-byte aligned
  c.dense_meta.ensure(i32bytes + sizeof(int64_t) * 3 * nb);
  int32_t* d_order = c.dense_meta.as<int32_t>();
  int32_t* d_dims = d_order + nb;
  int64_t* d_aoff = reinterpret_cast<int64_t*>(c.dense_meta.as<char>() + i32bytes);
  int64_t* d_eoff = d_aoff + nb;
  int64_t* d_woff = d_eoff + nb;
  FTLM_CUDA(cudaMemcpyAsync(d_order, order.data(), sizeof(int32_t) * nb, cudaMemcpyHostToDevice, c.stream));
  FTLM_CUDA(cudaMemcpyAsync(d_dims, dims.data(), sizeof(int32_t) * nb, cudaMemcpyHostToDevice, c.stream));
  FTLM_CUDA(cudaMemcpyAsync(d_aoff, aoff.data(), sizeof(int64_t) * nb, cudaMemcpyHostToDevice, c.stream));
  FTLM_CUDA(cudaMemcpyAsync(d_eoff, eoff.data(), sizeof(int64_t) * nb, cudaMemcpyHostToDevice, c.stream));
  FTLM_CUDA(cudaMemcpyAsync(d_woff, woff.data(), sizeof(int64_t) * nb, cudaMemcpyHostToDevice, c.stream));
  c.prof.h2d_bytes += static_cast<int64_t>(nb) * 32;
  const size_t smem = sizeof(double2) * 2 * static_cast<size_t>(nmax);
  if (smem > 48 * 1024)
    FTLM_CUDA(cudaFuncSetAttribute(k_dense_eig, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
  const int grid = static_cast<int>(std::min<size_t>(nb, static_cast<size_t>(c.sm_count) * 4));
  k_dense_eig<<<grid, kEigThreads, smem, c.stream>>>(static_cast<int>(nb), d_order, d_dims, d_aoff, arena, d_eoff,
                                                     evout, work, d_woff);
  FTLM_LAUNCH_CHECK();
  c.prof.kernel_launches += 1;
}

struct EventTimer {
  Ctx& c;
  double& acc;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  EventTimer(Ctx& c_, double& acc_) : c(c_), acc(acc_) {
    if (!c.timing) return;
    FTLM_CUDA(cudaEventCreate(&e0));
    FTLM_CUDA(cudaEventCreate(&e1));
    FTLM_CUDA(cudaEventRecord(e0, c.stream));
  }
  void stop() {
    if (!e0) return;
    FTLM_CUDA(cudaEventRecord(e1, c.stream));
    FTLM_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    FTLM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    acc += ms;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    e0 = e1 = nullptr;
  }
  ~EventTimer() {
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
  }
};

Spectrum exact_spectrum(const Ctx& c, int64_t n, int64_t ev_off) {
  Spectrum s;
  s.ev_off = ev_off;
  s.w_off = -1;
  s.count = n;
  s.exact = true;
  s.prefactor = 1.0;
  s.particles = c.sec.n_up + c.sec.n_dn;
  s.dim = n;
  return s;
}

}  // namespace

void run_exact_blocks(Ctx& c, const std::vector<std::pair<int, int>>& blocks) {
  int64_t asz = 0, wsz = 0;
  const std::vector<DenseItem> items = dense_items(c, blocks, asz, wsz);
  if (items.empty()) return;
  c.dense_arena.ensure(sizeof(double2) * asz);
  c.dense_out.ensure(sizeof(double) * wsz);
  FTLM_CUDA(cudaMemsetAsync(c.dense_arena.p, 0, sizeof(double2) * asz, c.stream));
  std::vector<int32_t> dims;
  std::vector<int64_t> aoff, eoff;
  for (const DenseItem& it : items) {
    dims.push_back(static_cast<int32_t>(it.n));
    aoff.push_back(it.aoff);
    eoff.push_back(spectra_alloc(c, it.n));
  }
  {
    EventTimer t(c, c.prof.dense_ms);
    dense_fill(c, items, c.dense_arena.as<double2>(), 0);
    t.stop();
  }
  {
    EventTimer t(c, c.prof.eig_ms);
    dense_solve(c, dims, aoff, eoff, c.dense_arena.as<double2>(), c.spectra.as<double>(), c.dense_out.as<double>());
    t.stop();
  }
  FTLM_CUDA(cudaStreamSynchronize(c.stream));
  for (size_t i = 0; i < items.size(); ++i) c.spec[{items[i].mx, items[i].my}] = exact_spectrum(c, items[i].n, eoff[i]);
}

void queue_exact_blocks(Ctx& c, const std::vector<std::pair<int, int>>& blocks) {
  int64_t asz = 0, wsz = 0;
  std::vector<DenseItem> items = dense_items(c, blocks, asz, wsz);
  if (items.empty()) return;
  if (defer_pool_bytes(c) > 0 && defer_pool_bytes(c) + static_cast<int64_t>(sizeof(double2)) * asz > kDeferPoolBytes)
    flush_deferred(c);
  const int64_t base = c.defer_asz;
  c.defer_arena.ensure_keep(sizeof(double2) * (base + asz), c.stream);
  FTLM_CUDA(cudaMemsetAsync(c.defer_arena.as<double2>() + base, 0, sizeof(double2) * asz, c.stream));
  {
    EventTimer t(c, c.prof.dense_ms);
    dense_fill(c, items, c.defer_arena.as<double2>(), base);
    t.stop();
  }
  c.defer_asz = base + asz;
  for (const DenseItem& it : items) {
    Spectrum s = exact_spectrum(c, it.n, -1);
    s.pending = static_cast<int>(c.defer_items.size());
    c.spec[{it.mx, it.my}] = s;
    c.defer_items.push_back({c.sec.n_up, c.sec.n_dn, it.mx, it.my, it.n, base + it.aoff, c.sec_gen});
  }
}

int64_t defer_pool_bytes(const Ctx& c) {
  return static_cast<int64_t>(sizeof(double2)) * c.defer_asz + static_cast<int64_t>(sizeof(double)) * c.defer_ab_used +
         static_cast<int64_t>(sizeof(int32_t)) * c.defer_st_used;
}

void flush_deferred(Ctx& c) {
  const size_t nb = c.defer_items.size();
  const size_t nr = c.defer_ritz.size();
  if (nb == 0 && nr == 0) {
    c.defer_acc.clear();
    return;
  }
  // exact blocks: one dense-solver launch
  std::vector<int64_t> eoff(nb);
  if (nb > 0) {
    std::vector<int32_t> dims(nb);
    std::vector<int64_t> aoff(nb);
    int64_t etot = 0;
    for (size_t i = 0; i < nb; ++i) {
      dims[i] = static_cast<int32_t>(c.defer_items[i].n);
      aoff[i] = c.defer_items[i].aoff;
      eoff[i] = etot;
      etot += c.defer_items[i].n;
    }
    c.defer_ev.ensure(sizeof(double) * etot);
    c.defer_work.ensure(sizeof(double) * 2 * etot);
    EventTimer t(c, c.prof.eig_ms);
    dense_solve(c, dims, aoff, eoff, c.defer_arena.as<double2>(), c.defer_ev.as<double>(), c.defer_work.as<double>());
    t.stop();
  }
  // small FTLM blocks: one Ritz-stage launch; the spectra land in this
  // sector's arena (those of earlier sectors are dropped with it later)
  std::vector<Spectrum> rs(nr);
  if (nr > 0) {
    std::vector<RitzJob> jobs;
    jobs.reserve(nr);
    for (size_t i = 0; i < nr; ++i) {
      const DeferRitz& d = c.defer_ritz[i];
      jobs.push_back(RitzJob{d.R, d.R, d.ld, d.K, c.defer_ab.as<double>() + d.alpha_off,
                             c.defer_ab.as<double>() + d.beta_off, c.defer_st.as<int32_t>() + d.steps_off, &rs[i]});
    }
    ritz_stage_many(c, jobs);
    for (size_t i = 0; i < nr; ++i) {
      rs[i].prefactor = static_cast<double>(c.defer_ritz[i].dim);
      rs[i].particles = c.defer_ritz[i].n_up + c.defer_ritz[i].n_dn;
      rs[i].dim = c.defer_ritz[i].dim;
    }
  }
  for (const DeferAcc& a : c.defer_acc) {
    const size_t i = static_cast<size_t>(a.idx);
    if (a.ritz) {
      thermo_accumulate(c, rs[i]);
    } else {
      const DeferItem& d = c.defer_items[i];
      thermo_accumulate_dev(c, c.defer_ev.as<double>() + eoff[i], nullptr, d.n, 1.0, d.n_up + d.n_dn);
    }
  }
  // pending spectra of the current sector become ordinary ones
  for (size_t i = 0; i < nb; ++i) {
    const DeferItem& d = c.defer_items[i];
    if (d.sec_gen != c.sec_gen) continue;
    auto it = c.spec.find({d.mx, d.my});
    if (it == c.spec.end() || it->second.pending != static_cast<int>(i)) continue;
    const int64_t off = spectra_alloc(c, d.n);
    FTLM_CUDA(cudaMemcpyAsync(c.spectra.as<double>() + off, c.defer_ev.as<double>() + eoff[i], sizeof(double) * d.n,
                              cudaMemcpyDeviceToDevice, c.stream));
    it->second.ev_off = off;
    it->second.pending = -1;
  }
  for (size_t i = 0; i < nr; ++i) {
    const DeferRitz& d = c.defer_ritz[i];
    if (d.sec_gen != c.sec_gen) continue;
    auto it = c.spec.find({d.mx, d.my});
    if (it == c.spec.end() || it->second.pending_ritz != static_cast<int>(i)) continue;
    it->second = rs[i];
  }
  c.defer_items.clear();
  c.defer_ritz.clear();
  c.defer_acc.clear();
  c.defer_asz = 0;
  c.defer_ab_used = 0;
  c.defer_st_used = 0;
}

}  // namespace ftlm
