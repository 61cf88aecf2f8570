// Twist-surrogate MLP: FP32 forward, backward and Adam kernels on the GPU.
//
// Network: x[n_in] -> depth hidden layers of `width` units with tanh -> linear
// y[n_out]. Parameters are one flat FP32 buffer, per layer W[out][in] then
// b[out]. Loss: masked mean squared error, sum(mask*(y-t)^2)/sum(mask).
// Every product is a tiled GEMM with a fixed summation order (no atomics),
// so training is deterministic for a given seed. The sizes are small
// (widths of 128, a few thousand samples per batch); FP32 CUDA-core tiles are
// exact to the requested precision and take milliseconds per epoch.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "ftlm_internal.h"

struct ftlm_mlp {
  int device = 0;
  int n_in = 0, width = 0, depth = 0, n_out = 0;
  cudaStream_t stream = nullptr;
  std::vector<int> fan_in, fan_out;   // per layer
  std::vector<int64_t> w_off, b_off;  // offsets into the flat parameter buffer
  int64_t n_params = 0;
  ftlm::DBuf params, grads, adam_m, adam_v;
  ftlm::DBuf act;      // activations of the current batch, per layer [n][fan_out]
  ftlm::DBuf dact;     // gradients w.r.t. activations
  ftlm::DBuf data_x, data_t, data_m, batch_idx, batch_x, batch_t, batch_m, red, io;
  ftlm::DBuf perm, history;  // training order of one epoch; per-epoch loss sums
  int64_t data_n = 0;
  int64_t batch_cap = 0;
  int64_t adam_t = 0;
  std::string last_error;
};

namespace ftlm {
namespace {

constexpr int kTile = 32;

// C[m][n] = sum_k A(m,k) B(k,n), A(m,k) = A[m*as + k*ak], B(k,n) = B[k*bs + n*bn].
// mode 0: store; 1: + bias[n], tanh; 2: + bias[n]; 3: multiply by (1 - aux[m][n]^2).
__global__ void k_gemm(int M, int N, int K, const float* __restrict__ A, int64_t as, int64_t ak,
                       const float* __restrict__ B, int64_t bs, int64_t bn, float* __restrict__ C,
                       const float* __restrict__ bias, const float* __restrict__ aux, int mode) {
  __shared__ float As[kTile][kTile + 1];
  __shared__ float Bs[kTile][kTile + 1];
  const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
  const int m0 = blockIdx.y * kTile, n0 = blockIdx.x * kTile;
  float acc[4] = {0.f, 0.f, 0.f, 0.f};
  for (int k0 = 0; k0 < K; k0 += kTile) {
    for (int r = ty; r < kTile; r += 8) {
      const int m = m0 + r, k = k0 + tx;
      As[r][tx] = (m < M && k < K) ? A[m * as + k * ak] : 0.f;
      const int kk = k0 + r, n = n0 + tx;
      Bs[r][tx] = (kk < K && n < N) ? B[kk * bs + n * bn] : 0.f;
    }
    __syncthreads();
#pragma unroll 8
    for (int k = 0; k < kTile; ++k) {
      const float b = Bs[k][tx];
#pragma unroll
      for (int i = 0; i < 4; ++i) acc[i] = fmaf(As[ty + 8 * i][k], b, acc[i]);
    }
    __syncthreads();
  }
  const int n = n0 + tx;
  if (n >= N) return;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int m = m0 + ty + 8 * i;
    if (m >= M) continue;
    float v = acc[i];
    if (mode == 1) v = tanhf(v + bias[n]);
    else if (mode == 2) v = v + bias[n];
    else if (mode == 3) {
      const float h = aux[static_cast<int64_t>(m) * N + n];
      v = v * (1.f - h * h);
    }
    C[static_cast<int64_t>(m) * N + n] = v;
  }
}

// Column sums db[n] = sum_m dz[m][n] (fixed order).
__global__ void k_colsum(int M, int N, const float* __restrict__ dz, float* __restrict__ db) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  float s = 0.f;
  for (int m = 0; m < M; ++m) s += dz[static_cast<int64_t>(m) * N + n];
  db[n] = s;
}

// Output gradient of the masked MSE and per-row loss partials.
__global__ void k_mse(int M, int N, const float* __restrict__ y, const float* __restrict__ t,
                      const float* __restrict__ mask, float inv_count, float* __restrict__ dy,
                      float* __restrict__ row_loss) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= M) return;
  float l = 0.f;
  for (int n = 0; n < N; ++n) {
    const int64_t i = static_cast<int64_t>(m) * N + n;
    const float d = y[i] - t[i];
    dy[i] = 2.f * mask[i] * d * inv_count;
    l += mask[i] * d * d;
  }
  row_loss[m] = l;
}

// out = sum(v) * scale, or out += sum(v) * scale when accumulating.
__global__ void k_sum(int M, const float* __restrict__ v, float* __restrict__ out, float scale, int accumulate) {
  __shared__ double s[256];
  double a = 0.0;
  for (int i = threadIdx.x; i < M; i += 256) a += v[i];
  s[threadIdx.x] = a;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) s[threadIdx.x] += s[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = static_cast<float>(s[0] * scale) + (accumulate ? *out : 0.f);
}

__global__ void k_gather_rows(int M, int W, const int32_t* __restrict__ idx, const float* __restrict__ src,
                              float* __restrict__ dst) {
  const int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  if (t >= static_cast<int64_t>(M) * W) return;
  const int m = static_cast<int>(t / W), w = static_cast<int>(t % W);
  dst[t] = src[static_cast<int64_t>(idx[m]) * W + w];
}

__global__ void k_adam(int64_t n, float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2) {
  const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

void gemm(ftlm_mlp* net, int M, int N, int K, const float* A, int64_t as, int64_t ak, const float* B, int64_t bs,
          int64_t bn, float* Cc, const float* bias, const float* aux, int mode) {
  dim3 grid((N + kTile - 1) / kTile, (M + kTile - 1) / kTile);
  k_gemm<<<grid, dim3(32, 8), 0, net->stream>>>(M, N, K, A, as, ak, B, bs, bn, Cc, bias, aux, mode);
  FTLM_LAUNCH_CHECK();
}

int64_t act_offset(const ftlm_mlp* net, int layer, int64_t n) {
  int64_t o = 0;
  for (int l = 0; l < layer; ++l) o += n * net->fan_out[l];
  return o;
}

void ensure_batch(ftlm_mlp* net, int64_t n) {
  if (n <= net->batch_cap) return;
  int64_t per_row = 0;
  for (int f : net->fan_out) per_row += f;
  net->act.ensure(sizeof(float) * n * per_row);
  net->dact.ensure(sizeof(float) * n * per_row);
  net->batch_x.ensure(sizeof(float) * n * net->n_in);
  net->batch_t.ensure(sizeof(float) * n * net->n_out);
  net->batch_m.ensure(sizeof(float) * n * net->n_out);
  net->batch_idx.ensure(sizeof(int32_t) * n);
  net->red.ensure(sizeof(float) * (n + 8));
  net->batch_cap = n;
}

// Forward of n rows of x (device): activations in net->act; returns output.
float* forward(ftlm_mlp* net, const float* x, int64_t n) {
  ensure_batch(net, n);
  const int L = static_cast<int>(net->fan_in.size());
  const float* in = x;
  float* p = net->params.as<float>();
  for (int l = 0; l < L; ++l) {
    float* out = net->act.as<float>() + act_offset(net, l, n);
    const int fi = net->fan_in[l], fo = net->fan_out[l];
    // out[n][fo] = in[n][fi] * W^T, W[fo][fi]
    gemm(net, static_cast<int>(n), fo, fi, in, fi, 1, p + net->w_off[l], 1, fi, out, p + net->b_off[l], nullptr,
         l + 1 < L ? 1 : 2);
    in = out;
  }
  return net->act.as<float>() + act_offset(net, L - 1, n);
}

// Backward from dy = dL/dy (in net->dact, last layer) into net->grads.
void backward(ftlm_mlp* net, const float* x, int64_t n) {
  const int L = static_cast<int>(net->fan_in.size());
  float* p = net->params.as<float>();
  float* g = net->grads.as<float>();
  for (int l = L - 1; l >= 0; --l) {
    const int fi = net->fan_in[l], fo = net->fan_out[l];
    const float* dz = net->dact.as<float>() + act_offset(net, l, n);  // dL/d(pre-activation) of layer l
    const float* xin = l == 0 ? x : net->act.as<float>() + act_offset(net, l - 1, n);
    // dW[fo][fi] = dz^T xin
    gemm(net, fo, fi, static_cast<int>(n), dz, 1, fo, xin, fi, 1, g + net->w_off[l], nullptr, nullptr, 0);
    k_colsum<<<(fo + 127) / 128, 128, 0, net->stream>>>(static_cast<int>(n), fo, dz, g + net->b_off[l]);
    FTLM_LAUNCH_CHECK();
    if (l > 0) {
      // dz_prev[n][fi] = (dz W) * (1 - h_prev^2)
      float* dprev = net->dact.as<float>() + act_offset(net, l - 1, n);
      gemm(net, static_cast<int>(n), fi, fo, dz, fo, 1, p + net->w_off[l], fi, 1, dprev, nullptr,
           net->act.as<float>() + act_offset(net, l - 1, n), 3);
    }
  }
}

// Loss and gradient on n rows already on the device. The loss (sum over the
// mask / count) is written to `loss_slot` on the device, or added to it when
// `accumulate` is set; nothing waits for the host.
void loss_grad(ftlm_mlp* net, const float* x, const float* t, const float* mask, int64_t n, float count,
               float* loss_slot, int accumulate) {
  float* y = forward(net, x, n);
  const int L = static_cast<int>(net->fan_in.size());
  float* dy = net->dact.as<float>() + act_offset(net, L - 1, n);
  k_mse<<<static_cast<int>((n + 127) / 128), 128, 0, net->stream>>>(static_cast<int>(n), net->n_out, y, t, mask,
                                                                    1.f / count, dy, net->red.as<float>());
  k_sum<<<1, 256, 0, net->stream>>>(static_cast<int>(n), net->red.as<float>(), loss_slot, 1.f / count, accumulate);
  FTLM_LAUNCH_CHECK();
  backward(net, x, n);
}

template <typename F>
int guarded(ftlm_mlp* net, F&& f) {
  if (!net) return FTLM_ERR_ARG;
  try {
    FTLM_CUDA(cudaSetDevice(net->device));
    f(net);
    return FTLM_OK;
  } catch (const Error& e) {
    net->last_error = e.what();
    return e.code;
  } catch (const std::exception& e) {
    net->last_error = e.what();
    return FTLM_ERR_INTERNAL;
  }
}

}  // namespace
}  // namespace ftlm

using ftlm::Error;

extern "C" {

int ftlm_mlp_create(int32_t n_in, int32_t width, int32_t depth, int32_t n_out, uint64_t seed, int32_t device,
                    ftlm_mlp** out) {
  if (!out || n_in <= 0 || width <= 0 || depth <= 0 || n_out <= 0 || depth > 16) return FTLM_ERR_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    cudaGetLastError();
    return FTLM_ERR_CUDA;
  }
  ftlm_mlp* net = new (std::nothrow) ftlm_mlp();
  if (!net) return FTLM_ERR_INTERNAL;
  net->device = device;
  net->n_in = n_in;
  net->width = width;
  net->depth = depth;
  net->n_out = n_out;
  for (int l = 0; l <= depth; ++l) {
    net->fan_in.push_back(l == 0 ? n_in : width);
    net->fan_out.push_back(l == depth ? n_out : width);
  }
  int64_t off = 0;
  for (size_t l = 0; l < net->fan_in.size(); ++l) {
    net->w_off.push_back(off);
    off += static_cast<int64_t>(net->fan_in[l]) * net->fan_out[l];
    net->b_off.push_back(off);
    off += net->fan_out[l];
  }
  net->n_params = off;
  // Glorot-uniform weights, zero biases, from a seeded generator
  std::vector<float> h(static_cast<size_t>(off), 0.f);
  std::mt19937_64 rng(seed);
  for (size_t l = 0; l < net->fan_in.size(); ++l) {
    const double a = std::sqrt(6.0 / (net->fan_in[l] + net->fan_out[l]));
    std::uniform_real_distribution<double> u(-a, a);
    for (int64_t i = 0; i < static_cast<int64_t>(net->fan_in[l]) * net->fan_out[l]; ++i)
      h[static_cast<size_t>(net->w_off[l] + i)] = static_cast<float>(u(rng));
  }
  try {
    FTLM_CUDA(cudaSetDevice(device));
    FTLM_CUDA(cudaStreamCreateWithFlags(&net->stream, cudaStreamNonBlocking));
    net->params.ensure(sizeof(float) * off);
    net->grads.ensure(sizeof(float) * off);
    net->adam_m.ensure(sizeof(float) * off);
    net->adam_v.ensure(sizeof(float) * off);
    FTLM_CUDA(cudaMemcpy(net->params.p, h.data(), sizeof(float) * off, cudaMemcpyHostToDevice));
    FTLM_CUDA(cudaMemset(net->adam_m.p, 0, sizeof(float) * off));
    FTLM_CUDA(cudaMemset(net->adam_v.p, 0, sizeof(float) * off));
  } catch (const Error&) {
    delete net;
    return FTLM_ERR_CUDA;
  }
  *out = net;
  return FTLM_OK;
}

void ftlm_mlp_destroy(ftlm_mlp* net) {
  if (!net) return;
  cudaSetDevice(net->device);
  if (net->stream) cudaStreamSynchronize(net->stream);
  ftlm::DBuf* b[] = {&net->params, &net->grads, &net->adam_m, &net->adam_v, &net->act, &net->dact,
                     &net->data_x, &net->data_t, &net->data_m, &net->batch_idx, &net->batch_x,
                     &net->batch_t, &net->batch_m, &net->red, &net->io, &net->perm, &net->history};
  for (auto* x : b) x->release();
  if (net->stream) cudaStreamDestroy(net->stream);
  delete net;
}

int ftlm_mlp_last_error(const ftlm_mlp* net, char* buf, size_t len) {
  if (!buf || len == 0) return FTLM_ERR_ARG;
  const std::string msg = net ? net->last_error : std::string("null network");
  const size_t n = std::min(len - 1, msg.size());
  std::memcpy(buf, msg.data(), n);
  buf[n] = '\0';
  return FTLM_OK;
}

int ftlm_mlp_num_params(const ftlm_mlp* net, int64_t* count) {
  if (!net || !count) return FTLM_ERR_ARG;
  *count = net->n_params;
  return FTLM_OK;
}

int ftlm_mlp_get_params(ftlm_mlp* net, float* host, int64_t count) {
  return ftlm::guarded(net, [&](ftlm_mlp* m) {
    if (!host || count != m->n_params) throw Error(FTLM_ERR_ARG, "parameter count mismatch");
    FTLM_CUDA(cudaMemcpy(host, m->params.p, sizeof(float) * count, cudaMemcpyDeviceToHost));
  });
}

int ftlm_mlp_set_params(ftlm_mlp* net, const float* host, int64_t count) {
  return ftlm::guarded(net, [&](ftlm_mlp* m) {
    if (!host || count != m->n_params) throw Error(FTLM_ERR_ARG, "parameter count mismatch");
    FTLM_CUDA(cudaMemcpy(m->params.p, host, sizeof(float) * count, cudaMemcpyHostToDevice));
  });
}

int ftlm_mlp_forward(ftlm_mlp* net, const float* x, int64_t n, float* y) {
  return ftlm::guarded(net, [&](ftlm_mlp* m) {
    if (!x || !y || n <= 0) throw Error(FTLM_ERR_ARG, "bad forward arguments");
    m->io.ensure(sizeof(float) * n * m->n_in);
    FTLM_CUDA(cudaMemcpyAsync(m->io.p, x, sizeof(float) * n * m->n_in, cudaMemcpyHostToDevice, m->stream));
    const float* out = ftlm::forward(m, m->io.as<float>(), n);
    FTLM_CUDA(cudaMemcpyAsync(y, out, sizeof(float) * n * m->n_out, cudaMemcpyDeviceToHost, m->stream));
    FTLM_CUDA(cudaStreamSynchronize(m->stream));
  });
}

int ftlm_mlp_loss_grad(ftlm_mlp* net, const float* x, const float* t, const float* mask, int64_t n, float* loss,
                       float* grad) {
  return ftlm::guarded(net, [&](ftlm_mlp* m) {
    if (!x || !t || !mask || !loss || n <= 0) throw Error(FTLM_ERR_ARG, "bad loss_grad arguments");
    ftlm::ensure_batch(m, n);
    FTLM_CUDA(cudaMemcpyAsync(m->batch_x.p, x, sizeof(float) * n * m->n_in, cudaMemcpyHostToDevice, m->stream));
    FTLM_CUDA(cudaMemcpyAsync(m->batch_t.p, t, sizeof(float) * n * m->n_out, cudaMemcpyHostToDevice, m->stream));
    FTLM_CUDA(cudaMemcpyAsync(m->batch_m.p, mask, sizeof(float) * n * m->n_out, cudaMemcpyHostToDevice, m->stream));
    double cnt = 0.0;
    for (int64_t i = 0; i < n * m->n_out; ++i) cnt += mask[i];
    if (cnt <= 0.0) throw Error(FTLM_ERR_ARG, "empty mask");
    float* slot = m->red.as<float>() + n;
    ftlm::loss_grad(m, m->batch_x.as<float>(), m->batch_t.as<float>(), m->batch_m.as<float>(), n,
                    static_cast<float>(cnt), slot, 0);
    FTLM_CUDA(cudaMemcpyAsync(loss, slot, sizeof(float), cudaMemcpyDeviceToHost, m->stream));
    FTLM_CUDA(cudaStreamSynchronize(m->stream));
    if (grad)
      FTLM_CUDA(cudaMemcpy(grad, m->grads.p, sizeof(float) * m->n_params, cudaMemcpyDeviceToHost));
  });
}

int ftlm_mlp_train(ftlm_mlp* net, const float* x, const float* t, const float* mask, int64_t n, int32_t epochs,
                   int32_t batch, float lr, uint64_t seed, float* loss_history) {
  return ftlm::guarded(net, [&](ftlm_mlp* m) {
    if (!x || !t || !mask || n <= 0 || epochs <= 0 || batch <= 0) throw Error(FTLM_ERR_ARG, "bad train arguments");
    m->data_x.ensure(sizeof(float) * n * m->n_in);
    m->data_t.ensure(sizeof(float) * n * m->n_out);
    m->data_m.ensure(sizeof(float) * n * m->n_out);
    FTLM_CUDA(cudaMemcpyAsync(m->data_x.p, x, sizeof(float) * n * m->n_in, cudaMemcpyHostToDevice, m->stream));
    FTLM_CUDA(cudaMemcpyAsync(m->data_t.p, t, sizeof(float) * n * m->n_out, cudaMemcpyHostToDevice, m->stream));
    FTLM_CUDA(cudaMemcpyAsync(m->data_m.p, mask, sizeof(float) * n * m->n_out, cudaMemcpyHostToDevice, m->stream));
    const int64_t B = std::min<int64_t>(batch, n);
    ftlm::ensure_batch(m, B);
    m->perm.ensure(sizeof(int32_t) * n);
    m->history.ensure(sizeof(float) * epochs);
    FTLM_CUDA(cudaMemsetAsync(m->history.p, 0, sizeof(float) * epochs, m->stream));
    // Pinned staging of one epoch's order: the copy is asynchronous, so the
    // host shuffles the next epoch only after the previous copy has landed.
    int32_t* perm_h = nullptr;
    FTLM_CUDA(cudaMallocHost(&perm_h, sizeof(int32_t) * n));
    std::vector<int32_t> perm(static_cast<size_t>(n));
    for (int64_t i = 0; i < n; ++i) perm[static_cast<size_t>(i)] = static_cast<int32_t>(i);
    std::mt19937_64 rng(seed);
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    std::vector<int> batches(static_cast<size_t>(epochs), 0);
    try {
      for (int e = 0; e < epochs; ++e) {
        std::shuffle(perm.begin(), perm.end(), rng);
        FTLM_CUDA(cudaStreamSynchronize(m->stream));  // the previous epoch's order is no longer read
        std::memcpy(perm_h, perm.data(), sizeof(int32_t) * n);
        FTLM_CUDA(cudaMemcpyAsync(m->perm.p, perm_h, sizeof(int32_t) * n, cudaMemcpyHostToDevice, m->stream));
        float* slot = m->history.as<float>() + e;
        for (int64_t s = 0; s + B <= n; s += B) {  // full batches only
          double cnt = 0.0;
          for (int64_t i = 0; i < B; ++i)
            for (int o = 0; o < m->n_out; ++o)
              cnt += mask[static_cast<int64_t>(perm[static_cast<size_t>(s + i)]) * m->n_out + o];
          if (cnt <= 0.0) continue;
          const int32_t* idx = m->perm.as<int32_t>() + s;
          const int th = 256;
          ftlm::k_gather_rows<<<static_cast<int>((B * m->n_in + th - 1) / th), th, 0, m->stream>>>(
              static_cast<int>(B), m->n_in, idx, m->data_x.as<float>(), m->batch_x.as<float>());
          ftlm::k_gather_rows<<<static_cast<int>((B * m->n_out + th - 1) / th), th, 0, m->stream>>>(
              static_cast<int>(B), m->n_out, idx, m->data_t.as<float>(), m->batch_t.as<float>());
          ftlm::k_gather_rows<<<static_cast<int>((B * m->n_out + th - 1) / th), th, 0, m->stream>>>(
              static_cast<int>(B), m->n_out, idx, m->data_m.as<float>(), m->batch_m.as<float>());
          FTLM_LAUNCH_CHECK();
          ftlm::loss_grad(m, m->batch_x.as<float>(), m->batch_t.as<float>(), m->batch_m.as<float>(), B,
                          static_cast<float>(cnt), slot, 1);
          ++batches[static_cast<size_t>(e)];
          ++m->adam_t;
          const float c1 = 1.f - std::pow(b1, static_cast<float>(m->adam_t));
          const float c2 = 1.f - std::pow(b2, static_cast<float>(m->adam_t));
          ftlm::k_adam<<<static_cast<int>((m->n_params + 255) / 256), 256, 0, m->stream>>>(
              m->n_params, m->params.as<float>(), m->grads.as<float>(), m->adam_m.as<float>(),
              m->adam_v.as<float>(), lr, b1, b2, eps, c1, c2);
          FTLM_LAUNCH_CHECK();
        }
      }
      FTLM_CUDA(cudaStreamSynchronize(m->stream));
    } catch (...) {
      cudaFreeHost(perm_h);
      throw;
    }
    cudaFreeHost(perm_h);
    if (loss_history) {
      std::vector<float> h(static_cast<size_t>(epochs));
      FTLM_CUDA(cudaMemcpy(h.data(), m->history.p, sizeof(float) * epochs, cudaMemcpyDeviceToHost));
      for (int e = 0; e < epochs; ++e)
        loss_history[e] = batches[static_cast<size_t>(e)] ? h[static_cast<size_t>(e)] / batches[static_cast<size_t>(e)]
                                                          : 0.f;
    }
  });
}

}  // extern "C"
