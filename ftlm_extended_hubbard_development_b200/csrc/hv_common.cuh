// Device building blocks shared by the H*V kernels (hv.cu, split.cu) and
// the Lanczos update: 16-byte vector chunks, streaming loads, complex FMAs,
// the hop-target resolver over the factorised orbit tables, the gather loop,
// the spin-flip coefficients and the fixed-point flush of the Lanczos dot
// products.
#pragma once

#include "ftlm_internal.h"

namespace ftlm {
namespace {

// Resolve a hop target (tu, td) to its block column, translation shift,
// sign parity and orbit stabiliser size. Returns false when the target's
// orbit is inactive in this block (main.cpp:790-793).
template <typename W, typename R>
__device__ __forceinline__ bool resolve(W tu, W td, bool up_hop, uint32_t ur_src, const BlockView<W>& v,
                                        const Geom& g, const R* binom, int64_t& col, int& shift, int& sgn,
                                        int& deg) {
  uint32_t ur = ur_src;
  int g0 = 0;
  int s = 0;
  W dd = td;
  if (up_hop) {
    const uint64_t info = __ldg(v.up_info + rank_of<W, R>(tu, binom));
    ur = static_cast<uint32_t>(info);
    g0 = static_cast<int>((info >> 32) & 0xFF);
    s = static_cast<int>((info >> 40) & 1);
    if (g0) {
      int p;
      const int ng = shift_neg(g0, g);
      dd = translate(td, shift_dx(ng, g), shift_dy(ng, g), g, &p);
      s ^= p;
    }
  }
  const int cls = __ldg(v.ur_class + ur);
  const int64_t rd = static_cast<int64_t>(rank_of<W, R>(dd, binom));
  int64_t a = rd;
  int h = 0;
  deg = 1;
  if (cls != 0) {
    const uint64_t e = __ldg(v.dtab + static_cast<int64_t>(cls - 1) * v.c_dn + rd);
    a = static_cast<int32_t>(static_cast<uint32_t>(e));
    if (a < 0) return false;
    h = static_cast<int>((e >> 32) & 0xFF);
    s ^= static_cast<int>((e >> 40) & 1);
    deg = static_cast<int>((e >> 48) & 0xFF);
  }
  shift = h ? shift_add(g0, h, g) : g0;
  sgn = s;
  col = __ldg(v.aoff + ur) + a;
  return true;
}

template <typename T>
struct CT;  // 16-byte chunk type and complex-per-chunk count
template <>
struct CT<float> {
  using V = float4;
  static constexpr int VPL = 2;
};
template <>
struct CT<double> {
  using V = double2;
  static constexpr int VPL = 1;
};

template <typename W>
struct HvParams {
  Geom g;
  BlockView<W> v;
};

constexpr int kHvThreads = 256;
constexpr int kHvWarps = kHvThreads / 32;
// hop codes per warp: 8 directions * (N_up + N_down) <= 16 * bits per word
template <typename W>
constexpr int queue_len() { return 16 * static_cast<int>(sizeof(W)) * 8; }

// k-th (0-based) set bit of x.
template <typename W>
__device__ __forceinline__ int kth_bit(W x, int k) {
  int pos = 0;
#pragma unroll
  for (int w = sizeof(W) * 4; w >= 1; w >>= 1) {
    const W lowmask = static_cast<W>((static_cast<W>(1) << w) - 1);
    const int c = popc(static_cast<W>(x & lowmask));
    if (k >= c) {
      k -= c;
      x >>= w;
      pos += w;
    }
  }
  return pos;
}

// Gathered vector rows stream through without allocating in L1, so the small
// orbit tables of the target lookups (up_info, class tables, offsets) stay
// L1-resident; L2 still caches the rows.
__device__ __forceinline__ float4 ld_stream(const float4* p) {
  float4 r;
  asm("ld.global.nc.L1::no_allocate.v4.f32 {%0, %1, %2, %3}, [%4];"
      : "=f"(r.x), "=f"(r.y), "=f"(r.z), "=f"(r.w)
      : "l"(p));
  return r;
}
__device__ __forceinline__ double2 ld_stream(const double2* p) {
  double2 r;
  asm("ld.global.nc.L1::no_allocate.v2.f64 {%0, %1}, [%2];" : "=d"(r.x), "=d"(r.y) : "l"(p));
  return r;
}

template <typename T>
__device__ __forceinline__ void cfma(typename CT<T>::V& acc, T cr, T ci, const typename CT<T>::V& x);

template <>
__device__ __forceinline__ void cfma<float>(float4& acc, float cr, float ci, const float4& x) {
  acc.x = fmaf(cr, x.x, fmaf(-ci, x.y, acc.x));
  acc.y = fmaf(cr, x.y, fmaf(ci, x.x, acc.y));
  acc.z = fmaf(cr, x.z, fmaf(-ci, x.w, acc.z));
  acc.w = fmaf(cr, x.w, fmaf(ci, x.z, acc.w));
}
template <>
__device__ __forceinline__ void cfma<double>(double2& acc, double cr, double ci, const double2& x) {
  acc.x = fma(cr, x.x, fma(-ci, x.y, acc.x));
  acc.y = fma(cr, x.y, fma(ci, x.x, acc.y));
}

__device__ __forceinline__ float4 shfl_xor_v(float4 a, int m) {
  a.x = __shfl_xor_sync(0xffffffffu, a.x, m);
  a.y = __shfl_xor_sync(0xffffffffu, a.y, m);
  a.z = __shfl_xor_sync(0xffffffffu, a.z, m);
  a.w = __shfl_xor_sync(0xffffffffu, a.w, m);
  return a;
}
__device__ __forceinline__ double2 shfl_xor_v(double2 a, int m) {
  a.x = __shfl_xor_sync(0xffffffffu, a.x, m);
  a.y = __shfl_xor_sync(0xffffffffu, a.y, m);
  return a;
}
__device__ __forceinline__ void vzero(float4& a) { a = make_float4(0.f, 0.f, 0.f, 0.f); }
__device__ __forceinline__ void vzero(double2& a) { a = make_double2(0.0, 0.0); }
__device__ __forceinline__ void vadd(float4& a, const float4& b) {
  a.x += b.x; a.y += b.y; a.z += b.z; a.w += b.w;
}
__device__ __forceinline__ void vadd(double2& a, const double2& b) {
  a.x += b.x; a.y += b.y;
}

// y = s_v * (diag * x + acc) per complex element; dot[e] = Re(conj(s_v x) y)
// of element e.
__device__ __forceinline__ float4 finish_row(const float4& x, const float4& acc, double diag, const double* s,
                                             double* dot) {
  const float df = static_cast<float>(diag);
  float4 y;
  y.x = fmaf(df, x.x, acc.x);
  y.y = fmaf(df, x.y, acc.y);
  y.z = fmaf(df, x.z, acc.z);
  y.w = fmaf(df, x.w, acc.w);
  y.x = static_cast<float>(s[0] * y.x);
  y.y = static_cast<float>(s[0] * y.y);
  y.z = static_cast<float>(s[1] * y.z);
  y.w = static_cast<float>(s[1] * y.w);
  dot[0] = s[0] * (static_cast<double>(x.x) * y.x + static_cast<double>(x.y) * y.y);
  dot[1] = s[1] * (static_cast<double>(x.z) * y.z + static_cast<double>(x.w) * y.w);
  return y;
}
__device__ __forceinline__ double2 finish_row(const double2& x, const double2& acc, double diag, const double* s,
                                              double* dot) {
  double2 y;
  y.x = s[0] * fma(diag, x.x, acc.x);
  y.y = s[0] * fma(diag, x.y, acc.y);
  dot[0] = s[0] * (x.x * y.x + x.y * y.y);
  return y;
}

// Flip map entry -> flipped row p and coefficient f = sign * e^{i k.shift}.
__device__ __forceinline__ void flip_coef(uint64_t f, const FlipPhase& ph, int64_t& p, double& fr, double& fi) {
  p = static_cast<int64_t>(static_cast<uint32_t>(f));
  const int shift = static_cast<int>((f >> 32) & 63);
  const bool neg = (f >> 38) & 1;
  fr = neg ? -ph.re[shift] : ph.re[shift];
  fi = neg ? -ph.im[shift] : ph.im[shift];
}

// conj(f) * x and y + f * x per complex element of a chunk, FP64 arithmetic.
template <typename T>
__device__ __forceinline__ typename CT<T>::V cmul_conj(double fr, double fi, const typename CT<T>::V& x);
template <>
__device__ __forceinline__ float4 cmul_conj<float>(double fr, double fi, const float4& x) {
  return make_float4(static_cast<float>(fr * x.x + fi * x.y), static_cast<float>(fr * x.y - fi * x.x),
                     static_cast<float>(fr * x.z + fi * x.w), static_cast<float>(fr * x.w - fi * x.z));
}
template <>
__device__ __forceinline__ double2 cmul_conj<double>(double fr, double fi, const double2& x) {
  return make_double2(fr * x.x + fi * x.y, fr * x.y - fi * x.x);
}
template <typename T>
__device__ __forceinline__ typename CT<T>::V cadd_mul(const typename CT<T>::V& y, double fr, double fi,
                                                      const typename CT<T>::V& x);
template <>
__device__ __forceinline__ float4 cadd_mul<float>(const float4& y, double fr, double fi, const float4& x) {
  return make_float4(static_cast<float>(y.x + (fr * x.x - fi * x.y)), static_cast<float>(y.y + (fr * x.y + fi * x.x)),
                     static_cast<float>(y.z + (fr * x.z - fi * x.w)), static_cast<float>(y.w + (fr * x.w + fi * x.z)));
}
template <>
__device__ __forceinline__ double2 cadd_mul<double>(const double2& y, double fr, double fi, const double2& x) {
  return make_double2(y.x + (fr * x.x - fi * x.y), y.y + (fr * x.y + fi * x.x));
}

// Sum of the warps' fixed-point dot accumulators of this CTA into
// partial[cta][NV] (nothing when partial is null). All threads must call it.
template <int NV, int NW>
__device__ __forceinline__ void flush_dot(fx128 (&s_acc)[NW][NV], fx128* __restrict__ partial) {
  if (!partial) return;
  __syncthreads();
  for (int vv = threadIdx.x; vv < NV; vv += blockDim.x) {
    fx128 t = 0;
#pragma unroll
    for (int w = 0; w < NW; ++w) t += s_acc[w][vv];
    partial[static_cast<int64_t>(blockIdx.x) * NV + vv] = t;
  }
}

// Gathers of one batch of nb <= 32 hops, whose (column, coefficient) lane
// q holds for hop q: groups of G lanes take hops grp, grp+HPAR, ..., U hops
// per group per iteration with all their loads issued before any FMA
// (U*LPL 16-byte gathers in flight per lane). Summation order per lane is
// the hop order, independent of U.
template <typename T, int NV, int U>
__device__ __forceinline__ void gather_batch(const typename CT<T>::V* __restrict__ in, int64_t col, T cr, T ci,
                                             int nb,
                                             typename CT<T>::V (&acc)[(NV / CT<T>::VPL < 32 ? 1 : NV / CT<T>::VPL / 32)]) {
  using V = typename CT<T>::V;
  constexpr int CPR = NV / CT<T>::VPL;
  constexpr int G = CPR < 32 ? CPR : 32;
  constexpr int LPL = CPR / G;
  constexpr int HPAR = 32 / G;
  const int lane = threadIdx.x & 31;
  const int grp = lane / G;
  const int sub = lane % G;
  for (int j = 0; j < nb; j += HPAR * U) {
    int64_t c[U];
    T r[U], i[U];
    V x[U][LPL];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int q = j + u * HPAR + grp;
      c[u] = __shfl_sync(0xffffffffu, col, q & 31);
      r[u] = __shfl_sync(0xffffffffu, cr, q & 31);
      i[u] = __shfl_sync(0xffffffffu, ci, q & 31);
      if (q >= nb) c[u] = -1;
    }
#pragma unroll
    for (int u = 0; u < U; ++u)
#pragma unroll
      for (int l = 0; l < LPL; ++l) {
        if (c[u] >= 0) x[u][l] = ld_stream(in + c[u] * CPR + l * G + sub);
        else vzero(x[u][l]);
      }
#pragma unroll
    for (int u = 0; u < U; ++u)
#pragma unroll
      for (int l = 0; l < LPL; ++l) cfma<T>(acc[l], r[u], i[u], x[u][l]);
  }
}

}  // namespace
}  // namespace ftlm
