// Allocation-free Ritz-value stage (ftlm_ritz_noalloc, include/ftlm_gpu.h).
//
// Some callers cannot allocate device memory when they need this stage: a
// host framework whose caching allocator has already reserved the whole
// device memory pool (a side cudaMalloc fails or fragments that pool), and a
// latency-critical loop that must not pay for cudaMalloc / cudaFree (cudaFree
// synchronises the whole device). For them this entry point turns Lanczos
// coefficients that the caller already holds on the device into Ritz values
// and FTLM weights without any allocation: its only work space is the
// file-scope device array below, of a fixed size, which every GPU that loads
// the library holds until the process exits. The first call on a device
// looks up that array's device address (cudaGetSymbolAddress); make that
// first call before any stream capture. The address is kept per device and
// CUDA context, so a call after a device reset looks it up again (that call
// is then a first call again).
//
// The computation is the same as the engine's own Ritz stage: implicit QL
// with shifts on each tridiagonal, tracking the first row of the eigenvector
// matrix, an ascending sort, weights v1^2 * inv_samples, spectra concatenated
// sample by sample.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/ftlm_gpu.h"
#include "ql.cuh"

namespace {

constexpr int kMaxNvec = 128;

// Work space shared by every call on a device: d, z, e rows of the QL for up
// to FTLM_NOALLOC_MAX_ENTRIES (vector, step) pairs, plus the status word.
// A call overwrites what the previous call left; calls that overlap on the
// GPU race on it.
__device__ __align__(256) double g_noalloc_scratch[3 * FTLM_NOALLOC_MAX_ENTRIES + 32];

// Device address of g_noalloc_scratch per device ordinal, set up on the first
// call on that device (host code cannot use the symbol itself as an address),
// together with the CUDA context it belongs to: after a device reset the
// runtime creates a new context with the module loaded again, and the
// address is looked up again there.
std::mutex g_mu;
double* g_scratch_addr[64] = {nullptr};
CUcontext g_scratch_ctx[64] = {nullptr};

typedef CUresult (*CtxGetCurrentFn)(CUcontext*);

// cuCtxGetCurrent through the runtime's driver entry-point table (no link
// against the driver library); null when it cannot be resolved.
CtxGetCurrentFn ctx_get_current() {
  static const CtxGetCurrentFn fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return static_cast<CtxGetCurrentFn>(nullptr);
    return reinterpret_cast<CtxGetCurrentFn>(p);
  }();
  return fn;
}

void set_err(char* buf, size_t len, const char* msg) {
  if (buf && len) {
    std::strncpy(buf, msg, len - 1);
    buf[len - 1] = '\0';
  }
}

__global__ void k_ritz_noalloc(const double* __restrict__ alpha, const double* __restrict__ beta,
                               const int32_t* __restrict__ steps, int nvec, int ld, double inv_r,
                               double* __restrict__ ev_out, double* __restrict__ w_out, int64_t* __restrict__ count,
                               double* __restrict__ scratch) {
  __shared__ int off[kMaxNvec + 1];
  __shared__ int failed;
  const int v = threadIdx.x;
  if (v == 0) failed = 0;
  __syncthreads();
  if (v < nvec) {
    int n = steps[v];
    n = n < 0 ? 0 : (n > ld ? ld : n);
    double* d = scratch + static_cast<int64_t>(v) * ld;
    double* z = scratch + static_cast<int64_t>(nvec) * ld + static_cast<int64_t>(v) * ld;
    double* e = scratch + 2 * static_cast<int64_t>(nvec) * ld + static_cast<int64_t>(v) * ld;
    for (int i = 0; i < n; ++i) {
      d[i] = alpha[static_cast<int64_t>(v) * ld + i];
      e[i] = i + 1 < n ? beta[static_cast<int64_t>(v) * ld + i] : 0.0;
      z[i] = i == 0 ? 1.0 : 0.0;
    }
    if (!ftlm::ql_first_row(n, d, z, e)) atomicExch(&failed, 1);
  }
  __syncthreads();
  if (v == 0) {
    int o = 0;
    for (int t = 0; t < nvec; ++t) {
      off[t] = o;
      const int n = steps[t];
      o += n < 0 ? 0 : (n > ld ? ld : n);
    }
    off[nvec] = o;
    if (count) *count = failed ? -1 : o;
  }
  __syncthreads();
  if (v < nvec) {
    const int n = off[v + 1] - off[v];
    const double* d = scratch + static_cast<int64_t>(v) * ld;
    const double* z = scratch + static_cast<int64_t>(nvec) * ld + static_cast<int64_t>(v) * ld;
    for (int i = 0; i < n; ++i) {
      ev_out[off[v] + i] = d[i];
      w_out[off[v] + i] = z[i] * z[i] * inv_r;
    }
  }
}

}  // namespace

extern "C" int ftlm_ritz_noalloc(const double* alpha, const double* beta, const int32_t* steps, int32_t nvec,
                                 int32_t ld, double inv_samples, double* evals, double* weights, int64_t* count,
                                 void* stream, char* errbuf, size_t errlen) {
  if (!alpha || !beta || !steps || !evals || !weights) {
    set_err(errbuf, errlen, "ftlm_ritz_noalloc: null device pointer");
    return FTLM_ERR_ARG;
  }
  if (nvec <= 0 || ld <= 0) {
    set_err(errbuf, errlen, "ftlm_ritz_noalloc: nvec and ld must be positive");
    return FTLM_ERR_ARG;
  }
  if (nvec > kMaxNvec || static_cast<int64_t>(nvec) * ld > FTLM_NOALLOC_MAX_ENTRIES) {
    char msg[200];
    std::snprintf(msg, sizeof msg,
                  "ftlm_ritz_noalloc: nvec*ld = %lld exceeds the fixed work space of %d entries "
                  "(nvec <= %d); use ftlm_block_spectrum for larger problems",
                  static_cast<long long>(nvec) * ld, FTLM_NOALLOC_MAX_ENTRIES, kMaxNvec);
    set_err(errbuf, errlen, msg);
    return FTLM_ERR_CAPACITY;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    set_err(errbuf, errlen, "ftlm_ritz_noalloc: no current CUDA device");
    return FTLM_ERR_CUDA;
  }
  double* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_mu);
    CUcontext cur = nullptr;
    const CtxGetCurrentFn get = ctx_get_current();
    if (get) get(&cur);
    if (!get || cur != g_scratch_ctx[dev]) g_scratch_addr[dev] = nullptr;  // new context: look it up again
    g_scratch_ctx[dev] = cur;
    if (!g_scratch_addr[dev]) {
      // first call on this device: resolve the array's device address
      void* p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess || !p) {
        set_err(errbuf, errlen, "ftlm_ritz_noalloc: cudaGetSymbolAddress of the work space failed");
        return FTLM_ERR_CUDA;
      }
      g_scratch_addr[dev] = static_cast<double*>(p);
    }
    scratch = g_scratch_addr[dev];
  }
  k_ritz_noalloc<<<1, kMaxNvec, 0, static_cast<cudaStream_t>(stream)>>>(alpha, beta, steps, nvec, ld, inv_samples,
                                                                       evals, weights, count, scratch);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_err(errbuf, errlen, cudaGetErrorString(e));
    return FTLM_ERR_CUDA;
  }
  return FTLM_OK;
}
