// Grand-canonical accumulation on the GPU (accumulate_block_thermo,
// main.cpp:1172-1219; accumulate_exact_block, ed_main.cpp:7-45).
//
// State per (beta, mu): the running minimum shifted energy emin and the
// sums z, <N>z, <N^2>z scaled by exp(beta*emin). One warp owns one
// (beta, mu) pair: it finds the block minimum, rescales the running sums
// when the minimum drops (exactly the reference's rule), then sums the
// block's Boltzmann weights across its lanes with a fixed butterfly order.
#include <algorithm>
#include <cmath>
#include <limits>
#include <vector>

#include "ftlm_internal.h"

namespace ftlm {

namespace {

__global__ void k_thermo(const double* __restrict__ ev, const double* __restrict__ w, int64_t count, double pref,
                         int particles, int nbeta, const double* __restrict__ betas, int nmu,
                         const double* __restrict__ mus, double* __restrict__ state) {
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (gw >= nbeta * nmu || count <= 0) return;
  const int ib = gw / nmu, im = gw % nmu;
  const int64_t plane = static_cast<int64_t>(nbeta) * nmu;
  double* emin = state + gw;
  double* z = state + plane + gw;
  double* ns = state + 2 * plane + gw;
  double* n2 = state + 3 * plane + gw;
  double lo = INFINITY;
  for (int64_t j = lane; j < count; j += 32) lo = fmin(lo, ev[j]);
  for (int o = 16; o > 0; o >>= 1) lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
  const double N = static_cast<double>(particles);
  const double beta = betas[ib];
  const double mun = mus[im] * N;
  // min_j (E_j - mu N) == (min_j E_j) - mu N: rounding is monotone
  const double bmin = lo - mun;
  if (!isfinite(bmin)) return;
  double E = *emin, Z = *z, NS = *ns, N2 = *n2;
  if (!isfinite(E)) {
    E = bmin;
  } else if (bmin < E) {
    const double scale = exp(-beta * (E - bmin));
    Z *= scale;
    NS *= scale;
    N2 *= scale;
    E = bmin;
  }
  double zs = 0.0, nsum = 0.0, n2sum = 0.0;
  for (int64_t j = lane; j < count; j += 32) {
    const double sh = ev[j] - mun - E;
    const double wt = pref * (w ? w[j] : 1.0) * exp(-beta * sh);
    zs += wt;
    nsum += N * wt;
    n2sum += N * N * wt;
  }
  for (int o = 16; o > 0; o >>= 1) {
    zs += __shfl_xor_sync(0xffffffffu, zs, o);
    nsum += __shfl_xor_sync(0xffffffffu, nsum, o);
    n2sum += __shfl_xor_sync(0xffffffffu, n2sum, o);
  }
  if (lane == 0) {
    *emin = E;
    *z = Z + zs;
    *ns = NS + nsum;
    *n2 = N2 + n2sum;
  }
}

__global__ void k_thermo_reset(double* state, int64_t plane) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < 4 * plane;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    state[i] = i < plane ? INFINITY : 0.0;
}

void launch(Ctx& c, const double* ev, const double* w, int64_t count, double pref, int particles) {
  if (c.nbeta <= 0 || c.nmu <= 0) throw Error(FTLM_ERR_STATE, "thermo accumulators not configured");
  const int warps = c.nbeta * c.nmu;
  const int threads = 256;
  const int grid = (warps * 32 + threads - 1) / threads;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (c.timing) {
    FTLM_CUDA(cudaEventCreate(&e0));
    FTLM_CUDA(cudaEventCreate(&e1));
    FTLM_CUDA(cudaEventRecord(e0, c.stream));
  }
  k_thermo<<<grid, threads, 0, c.stream>>>(ev, w, count, pref, particles, c.nbeta, c.th_beta.as<double>(), c.nmu,
                                           c.th_mu.as<double>(), c.th_state.as<double>());
  FTLM_LAUNCH_CHECK();
  c.prof.kernel_launches += 1;
  if (c.timing) {
    FTLM_CUDA(cudaEventRecord(e1, c.stream));
    FTLM_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    FTLM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    c.prof.thermo_ms += ms;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  }
}

}  // namespace

void thermo_configure(Ctx& c, int nbeta, const double* beta, int nmu, const double* mu) {
  c.nbeta = nbeta;
  c.nmu = nmu;
  c.th_beta.ensure(sizeof(double) * nbeta);
  c.th_mu.ensure(sizeof(double) * nmu);
  const int64_t plane = static_cast<int64_t>(nbeta) * nmu;
  c.th_state.ensure(sizeof(double) * 4 * plane);
  FTLM_CUDA(cudaMemcpyAsync(c.th_beta.p, beta, sizeof(double) * nbeta, cudaMemcpyHostToDevice, c.stream));
  FTLM_CUDA(cudaMemcpyAsync(c.th_mu.p, mu, sizeof(double) * nmu, cudaMemcpyHostToDevice, c.stream));
  k_thermo_reset<<<static_cast<int>(std::min<int64_t>((4 * plane + 255) / 256, 1024)), 256, 0, c.stream>>>(
      c.th_state.as<double>(), plane);
  FTLM_LAUNCH_CHECK();
  FTLM_CUDA(cudaStreamSynchronize(c.stream));
}

void thermo_accumulate(Ctx& c, const Spectrum& s) {
  const double* base = c.spectra.as<double>();
  launch(c, base + s.ev_off, s.w_off >= 0 ? base + s.w_off : nullptr, s.count, s.prefactor, s.particles);
}

void thermo_accumulate_dev(Ctx& c, const double* ev, const double* w, int64_t count, double pref, int particles) {
  launch(c, ev, w, count, pref, particles);
}

void thermo_accumulate_host(Ctx& c, const double* ev, const double* w, int64_t count, double pref, int particles) {
  if (count <= 0) return;
  DBuf& tmp = c.host_start;
  tmp.ensure(sizeof(double) * 2 * count);
  FTLM_CUDA(cudaMemcpyAsync(tmp.p, ev, sizeof(double) * count, cudaMemcpyHostToDevice, c.stream));
  if (w) FTLM_CUDA(cudaMemcpyAsync(tmp.as<double>() + count, w, sizeof(double) * count, cudaMemcpyHostToDevice, c.stream));
  c.prof.h2d_bytes += static_cast<int64_t>(sizeof(double)) * count * (w ? 2 : 1);
  launch(c, tmp.as<double>(), w ? tmp.as<double>() + count : nullptr, count, pref, particles);
  FTLM_CUDA(cudaStreamSynchronize(c.stream));
}

void thermo_read(Ctx& c, double* emin, double* z, double* n, double* n2) {
  const int64_t plane = static_cast<int64_t>(c.nbeta) * c.nmu;
  double* st = c.th_state.as<double>();
  FTLM_CUDA(cudaMemcpyAsync(emin, st, sizeof(double) * plane, cudaMemcpyDeviceToHost, c.stream));
  FTLM_CUDA(cudaMemcpyAsync(z, st + plane, sizeof(double) * plane, cudaMemcpyDeviceToHost, c.stream));
  FTLM_CUDA(cudaMemcpyAsync(n, st + 2 * plane, sizeof(double) * plane, cudaMemcpyDeviceToHost, c.stream));
  FTLM_CUDA(cudaMemcpyAsync(n2, st + 3 * plane, sizeof(double) * plane, cudaMemcpyDeviceToHost, c.stream));
  FTLM_CUDA(cudaStreamSynchronize(c.stream));
  c.prof.d2h_bytes += static_cast<int64_t>(sizeof(double)) * 4 * plane;
}

}  // namespace ftlm
