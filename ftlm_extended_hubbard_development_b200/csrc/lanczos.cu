// FTLM block: multi-vector Lanczos on the GPU (run_ftlm_block,
// main.cpp:996-1113).
//
// All random vectors of a sweep advance together: one H*V launch per step
// serves nv vectors. Per step
//   hv        y = s_j H w_j (on the fly), partial Re<s_j w_j, y>
//   alpha     alpha_j = sum of partials (fixed order, FP64)
//   update    w_{j+1} = y - alpha_j s_j w_j - beta_{j-1} s_{j-1} w_{j-1},
//             partial |w_{j+1}|^2 (FP64)
//   beta      beta_j = sqrt(sum); s_{j+1} = 1/beta_j, or stop the vector
//             at beta_j < 1e-12 / the last step (main.cpp:1044-1048)
// Vectors stay unnormalised (q_j = s_j w_j) so no separate scaling pass is
// needed. No re-orthogonalisation, as in the reference. The tridiagonal
// matrices are then solved in one batched launch by implicit QL with
// shifts, tracking only the first row of the eigenvector matrix
// (Golub-Welsch), which gives the Ritz values and the FTLM weights v1^2/R.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <atomic>
#include <random>
#include <thread>

#include "ftlm_internal.h"
#include "hv_common.cuh"
#include "ql.cuh"

namespace ftlm {

namespace {

constexpr int kUpdThreads = 256;

template <typename T>
struct VT;
template <>
struct VT<float> {
  using V = float4;
  static constexpr int VPL = 2;
};
template <>
struct VT<double> {
  using V = double2;
  static constexpr int VPL = 1;
};

// Lanczos state block (doubles), NV entries each.
enum { S_CUR = 0, S_PREV = 1, S_BPREV = 2, S_CA = 3, S_CB = 4, S_DONE = 5, S_STEPS = 6, S_NFIELD = 7 };

__global__ void k_state_init(double* st, int NV, int nva) {
  const int v = threadIdx.x;
  if (v >= NV) return;
  st[S_CUR * NV + v] = v < nva ? 1.0 : 0.0;
  st[S_PREV * NV + v] = 0.0;
  st[S_BPREV * NV + v] = 0.0;
  st[S_CA * NV + v] = 0.0;
  st[S_CB * NV + v] = 0.0;
  st[S_DONE * NV + v] = v < nva ? 0.0 : 1.0;
  st[S_STEPS * NV + v] = v < nva ? 0.0 : 1.0;
}

// alpha_j = Re<q_j, H q_j>: exact sum of the H*V kernels' fixed-point
// partials, so it does not depend on their grid or row scheduling.
__global__ void k_alpha_fin(int NV, int ncta, const fx128* __restrict__ partial, double* __restrict__ st,
                            double* __restrict__ alpha_j) {
  const int v = threadIdx.x;
  if (v >= NV) return;
  fx128 t = 0;
  for (int b = 0; b < ncta; ++b) t += partial[static_cast<int64_t>(b) * NV + v];
  const double s = fx_to_double(t);
  alpha_j[v] = s;
  st[S_CA * NV + v] = s * st[S_CUR * NV + v];
  st[S_CB * NV + v] = st[S_BPREV * NV + v] * st[S_PREV * NV + v];
}

__global__ void k_beta_fin(int NV, int ncta, const double* __restrict__ partial, double* __restrict__ st,
                           double* __restrict__ beta_j, int j, int kdim) {
  const int v = threadIdx.x;
  if (v >= NV) return;
  if (st[S_DONE * NV + v] != 0.0) {
    st[S_CUR * NV + v] = 0.0;
    st[S_PREV * NV + v] = 0.0;
    st[S_BPREV * NV + v] = 0.0;
    return;
  }
  double s = 0.0;
  for (int b = 0; b < ncta; ++b) s += partial[static_cast<int64_t>(b) * NV + v];
  const double bet = sqrt(s);
  if (bet < 1e-12 || j + 1 == kdim) {
    st[S_STEPS * NV + v] = static_cast<double>(j + 1);
    st[S_DONE * NV + v] = 1.0;
    st[S_CUR * NV + v] = 0.0;
    st[S_PREV * NV + v] = 0.0;
    st[S_BPREV * NV + v] = 0.0;
    return;
  }
  beta_j[v] = bet;
  st[S_PREV * NV + v] = st[S_CUR * NV + v];
  st[S_CUR * NV + v] = 1.0 / bet;
  st[S_BPREV * NV + v] = bet;
}

// w_prev <- y - ca*w_cur - cb*w_prev, per-vector |.|^2 partials.
// FLIP (split-spin H*V): y is completed by the flipped-order output,
// y[q] + f_q y_D[p(q)], and the new vector is also written in the flipped
// order, x_D[p(q)] = conj(f_q) w[q].
template <typename T, bool FLIP>
__global__ void __launch_bounds__(kUpdThreads) k_update(int64_t nchunks, int NV, const typename VT<T>::V* __restrict__ y,
                                                        const typename VT<T>::V* __restrict__ wc,
                                                        typename VT<T>::V* __restrict__ wp,
                                                        const double* __restrict__ st, double* __restrict__ partial,
                                                        const typename VT<T>::V* __restrict__ yd,
                                                        typename VT<T>::V* __restrict__ xd,
                                                        const uint64_t* __restrict__ fmap,
                                                        const __grid_constant__ FlipPhase ph) {
  using V = typename VT<T>::V;
  constexpr int VPL = VT<T>::VPL;
  const int CPR = NV / VPL;
  __shared__ double red[kUpdThreads * 2];
  const int tid = threadIdx.x;
  const int cv = tid % CPR;  // stride is a multiple of CPR, so fixed per thread
  double ca[VPL], cb[VPL], acc[VPL];
#pragma unroll
  for (int e = 0; e < VPL; ++e) {
    ca[e] = st[S_CA * NV + cv * VPL + e];
    cb[e] = st[S_CB * NV + cv * VPL + e];
    acc[e] = 0.0;
  }
  const int64_t stride = static_cast<int64_t>(gridDim.x) * kUpdThreads;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * kUpdThreads + tid; i < nchunks; i += stride) {
    const V h = y[i], x = wc[i], p = wp[i];
    int64_t fi_idx = 0;
    double fr = 1.0, fim = 0.0;
    if constexpr (FLIP) {
      const int64_t row = i / CPR;
      int64_t pr;
      flip_coef(__ldg(fmap + row), ph, pr, fr, fim);
      fi_idx = pr * CPR + (i - row * CPR);
    }
    V r;
    if constexpr (VPL == 2) {
      double h0 = h.x, h1 = h.y, h2 = h.z, h3 = h.w;
      if constexpr (FLIP) {
        const V d = yd[fi_idx];
        h0 += fr * d.x - fim * d.y;
        h1 += fr * d.y + fim * d.x;
        h2 += fr * d.z - fim * d.w;
        h3 += fr * d.w + fim * d.z;
      }
      const double r0 = h0 - ca[0] * x.x - cb[0] * p.x;
      const double r1 = h1 - ca[0] * x.y - cb[0] * p.y;
      const double r2 = h2 - ca[1] * x.z - cb[1] * p.z;
      const double r3 = h3 - ca[1] * x.w - cb[1] * p.w;
      r = make_float4(static_cast<float>(r0), static_cast<float>(r1), static_cast<float>(r2), static_cast<float>(r3));
      acc[0] += static_cast<double>(r.x) * r.x + static_cast<double>(r.y) * r.y;
      acc[1] += static_cast<double>(r.z) * r.z + static_cast<double>(r.w) * r.w;
    } else {
      double h0 = h.x, h1 = h.y;
      if constexpr (FLIP) {
        const V d = yd[fi_idx];
        h0 += fr * d.x - fim * d.y;
        h1 += fr * d.y + fim * d.x;
      }
      r.x = h0 - ca[0] * x.x - cb[0] * p.x;
      r.y = h1 - ca[0] * x.y - cb[0] * p.y;
      acc[0] += r.x * r.x + r.y * r.y;
    }
    wp[i] = r;
    if constexpr (FLIP) xd[fi_idx] = cmul_conj<T>(fr, fim, r);
  }
#pragma unroll
  for (int e = 0; e < VPL; ++e) red[tid * VPL + e] = acc[e];
  __syncthreads();
  for (int v = tid; v < NV; v += kUpdThreads) {
    const int c = v / VPL, e = v % VPL;
    double s = 0.0;
    for (int t = c; t < kUpdThreads; t += CPR) s += red[t * VPL + e];
    partial[static_cast<int64_t>(blockIdx.x) * NV + v] = s;
  }
}

// Start vectors, production mode: uniform phase, |q_i|^2 = 1/dim.
// Philox4x32-10 keyed by the block seed, counter (row, sample).
template <typename T>
__global__ void k_start_philox(int64_t dim, int NV, int nva, int sample0, uint64_t seed, typename VT<T>::V* __restrict__ out) {
  using V = typename VT<T>::V;
  constexpr int VPL = VT<T>::VPL;
  const int CPR = NV / VPL;
  const double amp = 1.0 / sqrt(static_cast<double>(dim));
  const int64_t n = dim * CPR;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t row = i / CPR;
    const int c = static_cast<int>(i % CPR);
    double re[VPL], im[VPL];
#pragma unroll
    for (int e = 0; e < VPL; ++e) {
      const int v = c * VPL + e;
      re[e] = 0.0;
      im[e] = 0.0;
      if (v < nva) philox_phase(row, sample0 + v, seed, amp, re[e], im[e]);
    }
    V o;
    if constexpr (VPL == 2) {
      o = make_float4(static_cast<float>(re[0]), static_cast<float>(im[0]), static_cast<float>(re[1]),
                      static_cast<float>(im[1]));
    } else {
      o = make_double2(re[0], im[0]);
    }
    out[i] = o;
  }
}

// Start vectors given per sample ([nva][dim] complex FP64) into [dim][NV].
template <typename T>
__global__ void k_start_gather(int64_t dim, int NV, int nva, const double2* __restrict__ src,
                               typename VT<T>::V* __restrict__ out) {
  using V = typename VT<T>::V;
  constexpr int VPL = VT<T>::VPL;
  const int CPR = NV / VPL;
  const int64_t n = dim * CPR;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t row = i / CPR;
    const int c = static_cast<int>(i % CPR);
    double2 z[VPL];
#pragma unroll
    for (int e = 0; e < VPL; ++e) {
      const int v = c * VPL + e;
      z[e] = v < nva ? src[static_cast<int64_t>(v) * dim + row] : make_double2(0.0, 0.0);
    }
    V o;
    if constexpr (VPL == 2) {
      o = make_float4(static_cast<float>(z[0].x), static_cast<float>(z[0].y), static_cast<float>(z[1].x),
                      static_cast<float>(z[1].y));
    } else {
      o = z[0];
    }
    out[i] = o;
  }
}

// Strided view of one vector's work array (shared memory: stride 32, one
// column per thread; global memory: stride 1, one row per thread).
struct Col {
  double* p;
  int st;
  __device__ __forceinline__ double& operator[](int i) const { return p[i * st]; }
};

// Implicit QL with shifts on every Lanczos tridiagonal (one thread per
// random vector; k_tridiag_many serves all vectors of several blocks in one
// launch, 32 vectors per CTA), tracking
// the first row z of the eigenvector matrix; then an ascending sort.
// alpha/beta are [sweep][K][ld] (vector r = sweep r/nvmax, lane r%nvmax),
// steps[r] the alphas taken. Outputs eigenvalues and z^2 * inv_r into [R][K]
// rows. With smem != 0 the three work columns of the warp's 32 vectors live
// in shared memory ([3][K][32]), otherwise in global memory.
__device__ void tridiag_vector(int r, int t, int nvmax, int ld, int K, const double* __restrict__ alpha,
                               const double* __restrict__ beta, const int32_t* __restrict__ steps,
                               double* __restrict__ dout, double* __restrict__ zout, double* __restrict__ escr,
                               double inv_r, int* __restrict__ status, double* sm, int smem) {
  const int n = steps[r];
  const int64_t base = (static_cast<int64_t>(r / nvmax) * K) * ld + r % nvmax;
  Col d, z, e;
  if (smem) {
    d = {sm + t, 32};
    z = {sm + 32 * K + t, 32};
    e = {sm + 64 * K + t, 32};
  } else {
    d = {dout + static_cast<int64_t>(r) * K, 1};
    z = {zout + static_cast<int64_t>(r) * K, 1};
    e = {escr + static_cast<int64_t>(r) * K, 1};
  }
  for (int i = 0; i < n; ++i) {
    d[i] = alpha[base + static_cast<int64_t>(i) * ld];
    e[i] = i + 1 < n ? beta[base + static_cast<int64_t>(i) * ld] : 0.0;
    z[i] = i == 0 ? 1.0 : 0.0;
  }
  if (!ql_first_row(n, d, z, e)) atomicExch(status, 1);
  double* dr = dout + static_cast<int64_t>(r) * K;
  double* zr = zout + static_cast<int64_t>(r) * K;
  for (int i = 0; i < n; ++i) {
    const double zi = z[i];
    dr[i] = d[i];
    zr[i] = zi * zi * inv_r;
  }
}

// Several blocks' Ritz stages in one launch: CTA b belongs to the job j with
// cta0[j] <= b < cta0[j+1] and serves that job's vectors 32(b-cta0[j]) ...
struct RitzJobDev {
  int R, nvmax, ld, K, cta0, pad;
  const double* alpha;
  const double* beta;
  const int32_t* steps;
  double *dout, *zout, *escr, *ev_out, *w_out;
  int64_t* total;
  int* status;
};

__global__ void k_tridiag_many(int njobs, const RitzJobDev* __restrict__ jobs, int smem) {
  extern __shared__ double sm[];
  int j = 0;
  while (j + 1 < njobs && jobs[j + 1].cta0 <= static_cast<int>(blockIdx.x)) ++j;
  const RitzJobDev J = jobs[j];
  const int r = (blockIdx.x - J.cta0) * blockDim.x + threadIdx.x;
  if (r >= J.R) return;
  tridiag_vector(r, threadIdx.x, J.nvmax, J.ld, J.K, J.alpha, J.beta, J.steps, J.dout, J.zout, J.escr, 1.0 / J.R,
                 J.status, sm, smem);
}

// Concatenate the per-vector spectra sample by sample (main.cpp:1097-1110).
// Dynamic shared memory: R+1 offsets.
__device__ void compact_block(int R, int K, const int32_t* __restrict__ steps, const double* __restrict__ d,
                              const double* __restrict__ w, double* __restrict__ ev_out, double* __restrict__ w_out,
                              int64_t* __restrict__ total, int* off) {
  if (threadIdx.x == 0) {
    int o = 0;
    for (int v = 0; v < R; ++v) {
      off[v] = o;
      o += steps[v];
    }
    off[R] = o;
    *total = o;
  }
  __syncthreads();
  for (int v = 0; v < R; ++v) {
    const int n = off[v + 1] - off[v];
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      ev_out[off[v] + i] = d[static_cast<int64_t>(v) * K + i];
      w_out[off[v] + i] = w[static_cast<int64_t>(v) * K + i];
    }
  }
}

// One CTA per job.
__global__ void k_compact_many(const RitzJobDev* __restrict__ jobs) {
  extern __shared__ int off[];
  const RitzJobDev J = jobs[blockIdx.x];
  compact_block(J.R, J.K, J.steps, J.dout, J.zout, J.ev_out, J.w_out, J.total, off);
}

// Steps of the nva vectors of one sweep, into the block's [R] array.
__global__ void k_collect_steps(const double* __restrict__ st, int NV, int nva, int32_t* __restrict__ out) {
  const int v = threadIdx.x;
  if (v < nva) out[v] = static_cast<int32_t>(st[S_STEPS * NV + v]);
}

// Algorithmic-byte model count: nonzero-amplitude hops with active
// targets per block (the h_nz of the H*V roofline).
int next_pow2(int x) {
  int p = 1;
  while (p < x) p <<= 1;
  return p;
}

uint64_t mix_u64(uint64_t value) {  // main.cpp:514-519
  value += 0x9e3779b97f4a7c15ULL;
  value = (value ^ (value >> 30U)) * 0xbf58476d1ce4e5b9ULL;
  value = (value ^ (value >> 27U)) * 0x94d049bb133111ebULL;
  return value ^ (value >> 31U);
}

}  // namespace

uint64_t block_seed(uint64_t seed, int n_up, int n_dn, int mx, int my) {  // main.cpp:521-533
  uint64_t s = mix_u64(seed);
  s ^= mix_u64(static_cast<uint64_t>(n_up + 1));
  s ^= mix_u64(static_cast<uint64_t>(n_dn + 17));
  s ^= mix_u64(static_cast<uint64_t>(mx + 257));
  s ^= mix_u64(static_cast<uint64_t>(my + 65537));
  return mix_u64(s);
}

// Reference start vectors (main.cpp:1015-1025): libstdc++ mt19937_64 and
// normal_distribution; g++ evaluates Complex(normal(rng), normal(rng))
// right to left, so each element is (second draw, first draw).
void reference_start_vectors(uint64_t bseed, int sample0, int nva, int64_t dim, double* out) {
  auto work = [&](int v) {
    std::mt19937_64 rng(mix_u64(bseed ^ static_cast<uint64_t>(sample0 + v)));
    std::normal_distribution<double> normal(0.0, 1.0);
    double* q = out + 2 * static_cast<int64_t>(v) * dim;
    double n2 = 0.0;
    for (int64_t i = 0; i < dim; ++i) {
      const double first = normal(rng);
      const double second = normal(rng);
      q[2 * i] = second;
      q[2 * i + 1] = first;
      n2 += second * second + first * first;
    }
    const double nrm = std::sqrt(n2);
    for (int64_t i = 0; i < 2 * dim; ++i) q[i] /= nrm;
  };
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  if (nva == 1 || dim < 4096 || hw == 1) {
    for (int v = 0; v < nva; ++v) work(v);
    return;
  }
  std::vector<std::thread> th;
  std::atomic<int> next{0};
  for (unsigned t = 0; t < std::min<unsigned>(hw, static_cast<unsigned>(nva)); ++t)
    th.emplace_back([&] {
      for (int v = next++; v < nva; v = next++) work(v);
    });
  for (auto& t : th) t.join();
}

int64_t spectra_alloc(Ctx& c, int64_t count) {
  const int64_t need = c.spectra_used + count;
  if (static_cast<size_t>(need) * sizeof(double) > c.spectra.cap) {
    DBuf n;
    n.ensure(sizeof(double) * std::max<int64_t>(need * 2, 1 << 16));
    if (c.spectra_used > 0)
      FTLM_CUDA(cudaMemcpyAsync(n.p, c.spectra.p, sizeof(double) * c.spectra_used, cudaMemcpyDeviceToDevice, c.stream));
    FTLM_CUDA(cudaStreamSynchronize(c.stream));
    c.spectra.release();
    c.spectra = n;
  }
  const int64_t off = c.spectra_used;
  c.spectra_used = need;
  return off;
}

void spectra_reset(Ctx& c) {
  c.spectra_used = 0;
  c.spec.clear();
}

void ritz_stage_many(Ctx& c, std::vector<RitzJob>& jobs) {
  if (jobs.empty()) return;
  // spectra slots first: spectra_alloc may move the arena
  const size_t nj = jobs.size();
  std::vector<int64_t> off(nj), scr(nj);
  int64_t scr_tot = 0;
  for (size_t i = 0; i < nj; ++i) {
    off[i] = spectra_alloc(c, 2 * static_cast<int64_t>(jobs[i].R) * jobs[i].K);
    scr[i] = scr_tot;
    scr_tot += 3 * static_cast<int64_t>(jobs[i].R) * jobs[i].K;
  }
  c.ritz_out.ensure(sizeof(double) * scr_tot + sizeof(int64_t) * 2 * nj + 64);
  double* scratch = c.ritz_out.as<double>();
  int64_t* totals = reinterpret_cast<int64_t*>(scratch + scr_tot);  // [nj] counts, then [nj] status words
  int* status = reinterpret_cast<int*>(totals + nj);
  FTLM_CUDA(cudaMemsetAsync(status, 0, sizeof(int) * nj, c.stream));
  cudaEvent_t ee0 = nullptr, ee1 = nullptr;
  if (c.timing) {
    FTLM_CUDA(cudaEventCreate(&ee0));
    FTLM_CUDA(cudaEventCreate(&ee1));
    FTLM_CUDA(cudaEventRecord(ee0, c.stream));
  }
  std::vector<RitzJobDev> dj(nj);
  int ctas = 0, kmax = 1, rmax = 1;
  for (size_t i = 0; i < nj; ++i) {
    const RitzJob& jb = jobs[i];
    const size_t rk = static_cast<size_t>(jb.R) * jb.K;
    RitzJobDev& d = dj[i];
    d.R = jb.R;
    d.nvmax = jb.nvmax;
    d.ld = jb.ld;
    d.K = jb.K;
    d.cta0 = ctas;
    d.pad = 0;
    d.alpha = jb.alpha;
    d.beta = jb.beta;
    d.steps = jb.steps;
    d.dout = scratch + scr[i];
    d.zout = d.dout + rk;
    d.escr = d.zout + rk;
    d.ev_out = c.spectra.as<double>() + off[i];
    d.w_out = d.ev_out + rk;
    d.total = totals + i;
    d.status = status + i;
    ctas += (jb.R + 31) / 32;
    kmax = std::max(kmax, jb.K);
    rmax = std::max(rmax, jb.R);
  }
  c.ritz_meta.ensure(sizeof(RitzJobDev) * nj);
  FTLM_CUDA(cudaMemcpyAsync(c.ritz_meta.p, dj.data(), sizeof(RitzJobDev) * nj, cudaMemcpyHostToDevice, c.stream));
  const size_t tsmem = sizeof(double) * 3 * 32 * static_cast<size_t>(kmax);
  const int use_smem = tsmem <= 200 * 1024;
  if (use_smem && tsmem > 48 * 1024)
    FTLM_CUDA(cudaFuncSetAttribute(k_tridiag_many, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(tsmem)));
  k_tridiag_many<<<ctas, 32, use_smem ? tsmem : 0, c.stream>>>(static_cast<int>(nj), c.ritz_meta.as<RitzJobDev>(),
                                                              use_smem);
  k_compact_many<<<static_cast<int>(nj), 256, sizeof(int) * (rmax + 1), c.stream>>>(c.ritz_meta.as<RitzJobDev>());
  FTLM_LAUNCH_CHECK();
  c.prof.kernel_launches += 2;
  if (c.timing) FTLM_CUDA(cudaEventRecord(ee1, c.stream));
  std::vector<int64_t> cnt(nj);
  std::vector<int> hstatus(nj);
  FTLM_CUDA(cudaMemcpyAsync(cnt.data(), totals, sizeof(int64_t) * nj, cudaMemcpyDeviceToHost, c.stream));
  FTLM_CUDA(cudaMemcpyAsync(hstatus.data(), status, sizeof(int) * nj, cudaMemcpyDeviceToHost, c.stream));
  FTLM_CUDA(cudaStreamSynchronize(c.stream));
  if (c.timing) {
    float ms = 0.f;
    FTLM_CUDA(cudaEventElapsedTime(&ms, ee0, ee1));
    c.prof.eig_ms += ms;
    cudaEventDestroy(ee0);
    cudaEventDestroy(ee1);
  }
  for (size_t i = 0; i < nj; ++i) {
    if (hstatus[i]) throw Error(FTLM_ERR_NUMERIC, "tridiagonal QL did not converge");
    Spectrum& out = *jobs[i].out;
    out.ev_off = off[i];
    out.w_off = off[i] + static_cast<int64_t>(jobs[i].R) * jobs[i].K;
    out.count = cnt[i];
    out.exact = false;
  }
}

void ritz_stage(Ctx& c, int R, int nvmax, int ld, int K, const double* alpha, const double* beta,
                const int32_t* steps, Spectrum& out) {
  std::vector<RitzJob> jobs{RitzJob{R, nvmax, ld, K, alpha, beta, steps, &out}};
  ritz_stage_many(c, jobs);
}

void run_ftlm_block(Ctx& c, int n_up, int n_dn, int mx, int my, Spectrum& out, const double* host_start,
                    std::vector<double>* alpha_out, std::vector<double>* beta_out, std::vector<int32_t>* steps_out) {
  block_prepare(c, mx, my);
  const int64_t D = c.blk.dim;
  if (D <= 0) throw Error(FTLM_ERR_ARG, "empty block");
  const int R = c.opts.samples;
  const int K = static_cast<int>(std::min<int64_t>(c.opts.lanczos_steps, D));
  const bool fp32 = c.opts.precision == FTLM_PREC_MIXED;
  int nvmax = c.opts.batch_vectors > 0 ? c.opts.batch_vectors : std::min(R, 128);
  nvmax = std::min(nvmax, 128);
  if (c.opts.batch_vectors <= 0) {
    // Vectors per sweep: the widest sweep whose arrays fit on the device with
    // 2 GiB to spare (wider sweeps cost less per vector at every width
    // measured); a large block counts the split sweeps' five arrays.
    size_t free_b = 0, total_b = 0;
    FTLM_CUDA(cudaMemGetInfo(&free_b, &total_b));
    const size_t have = c.vec_a.cap + c.vec_b.cap + c.vec_h.cap + c.vec_xd.cap + c.vec_yd.cap;
    const size_t arrays = D >= kSplitMinDim ? 5 : 3;
    while (nvmax > 1) {
      const size_t nv = static_cast<size_t>(next_pow2(std::max(nvmax, fp32 ? 2 : 1)));
      if (arrays * static_cast<size_t>(D) * nv * (fp32 ? 8 : 16) + (size_t(2) << 30) <= free_b + have) break;
      nvmax = std::max(1, nvmax / 2);
    }
  }
  const uint64_t bseed = block_seed(c.opts.seed, n_up, n_dn, mx, my);
  if (alpha_out) {
    alpha_out->assign(static_cast<size_t>(R) * c.opts.lanczos_steps, 0.0);
    beta_out->assign(static_cast<size_t>(R) * c.opts.lanczos_steps, 0.0);
    steps_out->assign(R, 0);
  }
  const int esize = fp32 ? 8 : 16;
  const int nsweep = (R + nvmax - 1) / nvmax;
  const int ld = next_pow2(std::max(nvmax, fp32 ? 2 : 1));  // alpha/beta row stride
  c.lz_alpha.ensure(sizeof(double) * static_cast<size_t>(nsweep) * K * ld);
  c.lz_beta.ensure(sizeof(double) * static_cast<size_t>(nsweep) * K * ld);
  FTLM_CUDA(cudaMemsetAsync(c.lz_beta.p, 0, sizeof(double) * static_cast<size_t>(nsweep) * K * ld, c.stream));
  c.ritz_tmp.ensure(sizeof(int32_t) * (R + 8));
  int32_t* steps_all = c.ritz_tmp.as<int32_t>();
  std::vector<double> hstart;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> evs;
  double hv_bytes = 0.0, hv_hops = 0.0, hv_min_bytes = 0.0;
  // Operator source: the cached hop list pays one lookup pass per block and
  // then streams 8 B per hop (few vectors share each lookup); large blocks
  // run the split-spin segment sweeps; the rest the on-the-fly kernel.
  HvSourceGuard guard{c};
  const int src = hv_select_source(c, next_pow2(std::max(std::min(nvmax, R), fp32 ? 2 : 1)), fp32);
  c.prof.hv_source = src;
  const bool split = src == kSrcSplit;
  const double nzh = c.timing ? static_cast<double>(src == kSrcList ? c.hl_nnz : block_nonzero_hops(c)) : 0.0;
  const FlipPhase fph = flip_phase(c);
  const uint64_t* fmap = split ? c.flip_map.as<uint64_t>() : nullptr;
  for (int s0 = 0; s0 < R; s0 += nvmax) {
    const int nva = std::min(nvmax, R - s0);
    const int NV = next_pow2(std::max(nva, fp32 ? 2 : 1));
    const size_t bytes = static_cast<size_t>(D) * NV * esize;
    c.vec_a.ensure(bytes);
    c.vec_b.ensure(bytes);
    c.vec_h.ensure(bytes);
    const int CPR = fp32 ? NV / 2 : NV;
    const int64_t nchunks = D * CPR;
    const int sgrid = static_cast<int>(std::min<int64_t>((nchunks + 255) / 256, static_cast<int64_t>(c.sm_count) * 16));
    // start vectors into vec_a
    if (host_start || c.opts.start_vector == FTLM_START_REF_GAUSSIAN) {
      const double* src = nullptr;
      if (host_start) {
        src = host_start + 2 * static_cast<int64_t>(s0) * D;
      } else {
        hstart.resize(2 * static_cast<size_t>(nva) * D);
        reference_start_vectors(bseed, s0, nva, D, hstart.data());
        src = hstart.data();
      }
      c.host_start.ensure(sizeof(double) * 2 * static_cast<size_t>(nva) * D);
      FTLM_CUDA(cudaMemcpyAsync(c.host_start.p, src, sizeof(double) * 2 * static_cast<size_t>(nva) * D,
                                cudaMemcpyHostToDevice, c.stream));
      c.prof.h2d_bytes += sizeof(double) * 2 * static_cast<int64_t>(nva) * D;
      if (fp32)
        k_start_gather<float><<<sgrid, 256, 0, c.stream>>>(D, NV, nva, c.host_start.as<double2>(), c.vec_a.as<float4>());
      else
        k_start_gather<double><<<sgrid, 256, 0, c.stream>>>(D, NV, nva, c.host_start.as<double2>(), c.vec_a.as<double2>());
    } else {
      if (fp32)
        k_start_philox<float><<<sgrid, 256, 0, c.stream>>>(D, NV, nva, s0, bseed, c.vec_a.as<float4>());
      else
        k_start_philox<double><<<sgrid, 256, 0, c.stream>>>(D, NV, nva, s0, bseed, c.vec_a.as<double2>());
    }
    FTLM_LAUNCH_CHECK();
    FTLM_CUDA(cudaMemsetAsync(c.vec_b.p, 0, bytes, c.stream));
    if (split) flip_scatter(c, c.vec_a.p, c.vec_xd.p, NV, fp32);
    const int hgrid = split ? hv_split_max_grid(c) : hv_grid(c, NV, fp32);
    const int ugrid = std::max(1, std::min<int>(static_cast<int>((nchunks + kUpdThreads - 1) / kUpdThreads),
                                                c.sm_count * 8));
    c.partial.ensure(std::max(sizeof(fx128) * hgrid, sizeof(double) * ugrid) * NV);
    c.lz_state.ensure(sizeof(double) * S_NFIELD * NV);
    double* st = c.lz_state.as<double>();
    double* alpha = c.lz_alpha.as<double>() + static_cast<int64_t>(s0 / nvmax) * K * ld;
    double* beta = c.lz_beta.as<double>() + static_cast<int64_t>(s0 / nvmax) * K * ld;
    k_state_init<<<1, 128, 0, c.stream>>>(st, NV, nva);
    void* cur = c.vec_a.p;
    void* prev = c.vec_b.p;
    for (int j = 0; j < K; ++j) {
      cudaEvent_t e0 = nullptr, e1 = nullptr;
      if (c.timing) {
        FTLM_CUDA(cudaEventCreate(&e0));
        FTLM_CUDA(cudaEventCreate(&e1));
        FTLM_CUDA(cudaEventRecord(e0, c.stream));
      }
      int ncta = hgrid;
      if (split)
        ncta = hv_apply_split(c, cur, c.vec_xd.p, c.vec_h.p, c.vec_yd.p, NV, fp32, st + S_CUR * NV,
                              c.partial.as<fx128>());
      else
        hv_apply(c, cur, c.vec_h.p, NV, fp32, st + S_CUR * NV, c.partial.as<fx128>(), hgrid);
      if (c.timing) {
        FTLM_CUDA(cudaEventRecord(e1, c.stream));
        evs.emplace_back(e0, e1);
      }
      k_alpha_fin<<<1, 128, 0, c.stream>>>(NV, ncta, c.partial.as<fx128>(), st, alpha + static_cast<int64_t>(j) * ld);
      if (fp32) {
        using V = float4;
        if (split)
          k_update<float, true><<<ugrid, kUpdThreads, 0, c.stream>>>(
              nchunks, NV, c.vec_h.as<V>(), static_cast<const V*>(cur), static_cast<V*>(prev), st,
              c.partial.as<double>(), c.vec_yd.as<V>(), c.vec_xd.as<V>(), fmap, fph);
        else
          k_update<float, false><<<ugrid, kUpdThreads, 0, c.stream>>>(
              nchunks, NV, c.vec_h.as<V>(), static_cast<const V*>(cur), static_cast<V*>(prev), st,
              c.partial.as<double>(), nullptr, nullptr, nullptr, fph);
      } else {
        using V = double2;
        if (split)
          k_update<double, true><<<ugrid, kUpdThreads, 0, c.stream>>>(
              nchunks, NV, c.vec_h.as<V>(), static_cast<const V*>(cur), static_cast<V*>(prev), st,
              c.partial.as<double>(), c.vec_yd.as<V>(), c.vec_xd.as<V>(), fmap, fph);
        else
          k_update<double, false><<<ugrid, kUpdThreads, 0, c.stream>>>(
              nchunks, NV, c.vec_h.as<V>(), static_cast<const V*>(cur), static_cast<V*>(prev), st,
              c.partial.as<double>(), nullptr, nullptr, nullptr, fph);
      }
      k_beta_fin<<<1, 128, 0, c.stream>>>(NV, ugrid, c.partial.as<double>(), st, beta + static_cast<int64_t>(j) * ld, j, K);
      FTLM_LAUNCH_CHECK();
      c.prof.kernel_launches += 3;
      std::swap(cur, prev);
    }
    k_collect_steps<<<1, 128, 0, c.stream>>>(st, NV, nva, steps_all + s0);
    FTLM_LAUNCH_CHECK();
    c.prof.kernel_launches += 1;
    if (c.timing) {
      // algorithmic bytes per H*V launch: D*[nv*s*(1 + h_nz) + nv*s + m],
      // h_nz*D = nonzero-amplitude hops to active targets, m = 8 B per row
      const double s = fp32 ? 8.0 : 16.0;
      hv_bytes += (static_cast<double>(D) * nva * s * 2.0 + nzh * nva * s + static_cast<double>(D) * 8.0) * K;
      hv_hops += nzh * nva * K;
      hv_min_bytes += static_cast<double>(D) * (2.0 * nva * s + 8.0) * K;
    }
    c.last_kdim = K;
    c.last_nv = NV;
  }
  // Ritz values and weights of all sweeps in one batched launch
  ritz_stage(c, R, nvmax, ld, K, c.lz_alpha.as<double>(), c.lz_beta.as<double>(), steps_all, out);
  if (alpha_out) {
    std::vector<double> a(static_cast<size_t>(nsweep) * K * ld), b(a.size());
    std::vector<int32_t> sv(R);
    FTLM_CUDA(cudaMemcpyAsync(a.data(), c.lz_alpha.p, sizeof(double) * a.size(), cudaMemcpyDeviceToHost, c.stream));
    FTLM_CUDA(cudaMemcpyAsync(b.data(), c.lz_beta.p, sizeof(double) * b.size(), cudaMemcpyDeviceToHost, c.stream));
    FTLM_CUDA(cudaMemcpyAsync(sv.data(), steps_all, sizeof(int32_t) * R, cudaMemcpyDeviceToHost, c.stream));
    FTLM_CUDA(cudaStreamSynchronize(c.stream));
    const int L = c.opts.lanczos_steps;
    for (int r = 0; r < R; ++r) {
      const int n = sv[r];
      const size_t base = (static_cast<size_t>(r / nvmax) * K) * ld + r % nvmax;
      (*steps_out)[r] = n;
      for (int j = 0; j < n; ++j) (*alpha_out)[static_cast<size_t>(r) * L + j] = a[base + static_cast<size_t>(j) * ld];
      for (int j = 0; j + 1 < n; ++j) (*beta_out)[static_cast<size_t>(r) * L + j] = b[base + static_cast<size_t>(j) * ld];
    }
  }
  if (c.timing) {
    for (auto& pr : evs) {
      float ms = 0.f;
      FTLM_CUDA(cudaEventElapsedTime(&ms, pr.first, pr.second));
      c.prof.hv_ms += ms;
      c.prof.hv_launches += 1;
      cudaEventDestroy(pr.first);
      cudaEventDestroy(pr.second);
    }
    c.prof.hv_bytes += hv_bytes;
    c.prof.hv_hops += hv_hops;
    c.prof.hv_min_bytes += hv_min_bytes;
  }
  out.prefactor = static_cast<double>(D);
  out.particles = n_up + n_dn;
  out.dim = D;
}

}  // namespace ftlm
