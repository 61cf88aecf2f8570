// Momentum-block Hamiltonian on the GPU.
//
// Two forms of H of block (mx, my):
//  * block_csr_device: explicit CSR in the reference's entry order
//    (build_momentum_block, main.cpp:779-804), for parity checks and the
//    dense exact path;
//  * k_hv: on-the-fly multi-vector H*V (apply_hamiltonian, main.cpp:833-845,
//    applied to nv vectors at once). No matrix is stored. Each warp owns a
//    row: its lanes enumerate the row's hops into a shared-memory queue,
//    resolve one hop target each (rank -> orbit table -> column, sign, phase),
//    then broadcast (column, coefficient) by warp shuffle while groups of
//    lanes gather the target rows of all nv vectors with 16-byte loads.
//    Vector layout is [dim][nv] so one gathered row is nv*sizeof(complex)
//    contiguous bytes.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>

#include "ftlm_internal.h"
#include "hv_common.cuh"

namespace ftlm {

namespace {

int grid_for(int64_t n, int threads) {
  return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>((n + threads - 1) / threads, 1 << 20)));
}

template <typename W>
struct CsrParams {
  Geom g;
  BlockView<W> v;
};

// One thread per row, hops in reference order: up spin first, occupied
// source sites ascending, directions 0..7, zero-amplitude hops included.
// fill 0: count entries; 1: write the CSR; 2: count nonzero-amplitude hops;
// 3: add the row straight into a dense column-major matrix (val as double2
// A[row + col*dim], zeroed by the caller): diagonal first, then the entries
// in CSR order, which is the sum order of building it from the CSR.
template <typename W>
__global__ void k_csr(const __grid_constant__ CsrParams<W> P, const uint64_t* __restrict__ binom, int fill,
                      int32_t* __restrict__ counts, const int64_t* __restrict__ row_ptr, int32_t* __restrict__ col,
                      double* __restrict__ val, double* __restrict__ diag) {
  const Geom& g = P.g;
  const BlockView<W>& v = P.v;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < v.dim;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const uint32_t meta = v.row_meta[i];
    const uint32_t ur = meta & 0x3FFFFFFu;
    const int deg_s = static_cast<int>(meta >> 26) + 1;
    const W u = v.ur_bits[ur];
    const W d = v.row_dn[i];
    int64_t pos = fill == 1 ? row_ptr[i] : 0;  // row_ptr exists only in the fill pass
    if (fill == 3) {
      double2* a = reinterpret_cast<double2*>(val) + (i + i * v.dim);
      a->x = __dadd_rn(a->x, diag_energy(u, d, g));
    }
    int cnt = 0;
    for (int spin = 0; spin < 2; ++spin) {
      const W bits = spin ? d : u;
      for (W m = bits; m; m &= m - 1) {
        const int from = ctz(m);
        for (int dir = 0; dir < 8; ++dir) {
          const int to = g.nb[from][dir];
          if ((bits >> to) & 1) continue;
          if (fill == 2 && g.amp_re[dir] == 0.0 && g.amp_im[dir] == 0.0) continue;
          const W moved = bits ^ (static_cast<W>(1) << from) ^ (static_cast<W>(1) << to);
          int64_t c;
          int shift, sgn, deg_t;
          if (!resolve<W, uint64_t>(spin ? u : moved, spin ? moved : d, spin == 0, ur, v, g, binom, c, shift,
                                    sgn, deg_t))
            continue;
          if (fill == 1 || fill == 3) {
            const int p = jw_parity(bits, from, to) ^ sgn;
            // ((amp * sign) * phase) * ratio, the operation order of main.cpp:794-797
            const double ar = p ? -g.amp_re[dir] : g.amp_re[dir];
            const double ai = p ? -g.amp_im[dir] : g.amp_im[dir];
            const double pr = v.phase_re[shift], pi = v.phase_im[shift];
            const double re = __dsub_rn(__dmul_rn(ar, pr), __dmul_rn(ai, pi));
            const double im = __dadd_rn(__dmul_rn(ar, pi), __dmul_rn(ai, pr));
            const double ratio = __ddiv_rn(g.sqrt_deg[deg_t], g.sqrt_deg[deg_s]);
            if (fill == 1) {
              col[pos] = static_cast<int32_t>(c);
              val[2 * pos] = __dmul_rn(re, ratio);
              val[2 * pos + 1] = __dmul_rn(im, ratio);
              ++pos;
            } else {
              double2* a = reinterpret_cast<double2*>(val) + (i + c * v.dim);
              a->x = __dadd_rn(a->x, __dmul_rn(re, ratio));
              a->y = __dadd_rn(a->y, __dmul_rn(im, ratio));
            }
          }
          ++cnt;
        }
      }
    }
    if (fill == 1) diag[i] = diag_energy(u, d, g);
    else if (fill != 3) counts[i] = cnt;
  }
}

__global__ void k_i64_to_i32(const int64_t* __restrict__ in, int32_t* __restrict__ out, int64_t n) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    out[i] = static_cast<int32_t>(in[i]);
}

// ------------------------------------------------------------ H*V kernel

// H*V over all rows of the block. in/out: [dim][NV] complex T as 16-byte
// chunks. scale[v] multiplies the result of vector v (Lanczos vectors are
// stored unnormalised). partial[block][NV] receives Re<s*in, out> sums
// (deterministic order), or nothing when partial == nullptr.
// U: hops gathered per lane group per iteration (loads in flight);
// MINB: CTAs per SM the register budget is sized for.
template <typename W, typename R, typename T, int NV, int U, int MINB>
__global__ void __launch_bounds__(kHvThreads, MINB) k_hv(const __grid_constant__ HvParams<W> P,
                                                   const typename CT<T>::V* __restrict__ in,
                                                   typename CT<T>::V* __restrict__ out,
                                                   const double* __restrict__ scale, fx128* __restrict__ partial,
                                                   const R* __restrict__ gbinom) {
  using V = typename CT<T>::V;
  constexpr int VPL = CT<T>::VPL;
  constexpr int CPR = NV / VPL;                 // 16-byte chunks per row
  constexpr int G = CPR < 32 ? CPR : 32;        // lanes per gathered row
  constexpr int LPL = CPR / G;                  // chunks per lane
  constexpr bool kSmemBinom = sizeof(W) == 4;   // 64-bit words read C(n,k) from global/L1
  constexpr int kQ = queue_len<W>();

  __shared__ R s_binom[kSmemBinom ? 32 * 65 : 1];
  __shared__ int8_t s_nb[64][8];
  __shared__ double s_ph[2][64];
  __shared__ double s_amp[2][8];
  __shared__ double s_sq[65];
  __shared__ uint16_t s_q[kHvWarps][kQ];
  __shared__ fx128 s_acc[kHvWarps][NV];

  const Geom& g = P.g;
  const BlockView<W>& v = P.v;
  const int tid = threadIdx.x;
  if (kSmemBinom)
    for (int i = tid; i < 32 * 65; i += kHvThreads) s_binom[i] = gbinom[i];
  const R* binom = kSmemBinom ? s_binom : gbinom;
  for (int i = tid; i < 64 * 8; i += kHvThreads) s_nb[i / 8][i % 8] = g.nb[i / 8][i % 8];
  for (int i = tid; i < 64; i += kHvThreads) {
    s_ph[0][i] = v.phase_re[i];
    s_ph[1][i] = v.phase_im[i];
  }
  if (tid < 8) {
    s_amp[0][tid] = g.amp_re[tid];
    s_amp[1][tid] = g.amp_im[tid];
  }
  if (tid < 65) s_sq[tid] = g.sqrt_deg[tid];
  for (int i = tid; i < kHvWarps * NV; i += kHvThreads) s_acc[i / NV][i % NV] = 0;
  __syncthreads();

  const int lane = tid & 31;
  const int wid = tid >> 5;
  const int grp = lane / G;
  const int sub = lane % G;
  uint16_t* queue = s_q[wid];

  double sc[LPL][VPL];
#pragma unroll
  for (int l = 0; l < LPL; ++l)
#pragma unroll
    for (int e = 0; e < VPL; ++e) sc[l][e] = scale ? scale[(l * G + sub) * VPL + e] : 1.0;

  const int nsite = v.n_up + v.n_dn;
  const int64_t nwarps = static_cast<int64_t>(gridDim.x) * kHvWarps;
  for (int64_t row = static_cast<int64_t>(blockIdx.x) * kHvWarps + wid; row < v.dim; row += nwarps) {
    const uint32_t meta = __ldg(v.row_meta + row);
    const uint32_t ur = meta & 0x3FFFFFFu;
    const int deg_s = static_cast<int>(meta >> 26) + 1;
    const W u = __ldg(v.ur_bits + ur);
    const W d = __ldg(v.row_dn + row);
    const double inv_s = 1.0 / s_sq[deg_s];

    // 1) hop queue: lane k handles the k-th occupied (spin, site) pair
    int total = 0;
    for (int k0 = 0; k0 < nsite; k0 += 32) {
      const int k = k0 + lane;
      uint32_t dm = 0;
      int spin = 0, from = 0;
      if (k < nsite) {
        spin = k >= v.n_up;
        const W bits = spin ? d : u;
        from = kth_bit(bits, spin ? k - v.n_up : k);
        for (int j = 0; j < g.ndir; ++j) {
          const int to = s_nb[from][g.dirs[j]];
          if (!((bits >> to) & 1)) dm |= 1u << j;
        }
      }
      const int cnt = __popc(dm);
      int incl = cnt;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
      }
      int pos = total + incl - cnt;
      for (uint32_t m = dm; m; m &= m - 1) {
        const int j = __ffs(m) - 1;
        queue[pos++] = static_cast<uint16_t>((spin << 9) | (from << 3) | g.dirs[j]);
      }
      total += __shfl_sync(0xffffffffu, incl, 31);
    }
    __syncwarp();

    // 2) resolve 32 hops at a time, gather their rows
    V acc[LPL];
#pragma unroll
    for (int l = 0; l < LPL; ++l) vzero(acc[l]);
    for (int b = 0; b < total; b += 32) {
      const int q = b + lane;
      int64_t col = -1;
      T cr = 0, ci = 0;
      if (q < total) {
        const int code = queue[q];
        const int spin = code >> 9, from = (code >> 3) & 63, dir = code & 7;
        const int to = s_nb[from][dir];
        const W bits = spin ? d : u;
        const W moved = bits ^ (static_cast<W>(1) << from) ^ (static_cast<W>(1) << to);
        int shift, sgn, deg_t;
        if (resolve<W, R>(spin ? u : moved, spin ? moved : d, spin == 0, ur, v, g, binom, col, shift, sgn, deg_t)) {
          const int p = jw_parity(bits, from, to) ^ sgn;
          const double ar = p ? -s_amp[0][dir] : s_amp[0][dir];
          const double ai = p ? -s_amp[1][dir] : s_amp[1][dir];
          const double pr = s_ph[0][shift], pi = s_ph[1][shift];
          const double ratio = s_sq[deg_t] * inv_s;
          cr = static_cast<T>((ar * pr - ai * pi) * ratio);
          ci = static_cast<T>((ar * pi + ai * pr) * ratio);
        }
      }
      gather_batch<T, NV, U>(in, col, cr, ci, min(32, total - b), acc);
    }
    __syncwarp();
    // 3) fold the HPAR partial sums
#pragma unroll
    for (int o = G; o < 32; o <<= 1)
#pragma unroll
      for (int l = 0; l < LPL; ++l) vadd(acc[l], shfl_xor_v(acc[l], o));
    // 4) own-row diagonal term, scale, store, Lanczos dot
    if (grp == 0) {
      const double diag = diag_energy(u, d, g);
#pragma unroll
      for (int l = 0; l < LPL; ++l) {
        const V x = ld_stream(in + row * CPR + l * G + sub);
        double dt[VPL];
        out[row * CPR + l * G + sub] = finish_row(x, acc[l], diag, sc[l], dt);
        if (partial) {
#pragma unroll
          for (int e = 0; e < VPL; ++e) s_acc[wid][(l * G + sub) * VPL + e] += fx_of(dt[e]);
        }
      }
    }
  }
  flush_dot<NV>(s_acc, partial);
}

// ------------------------------------------------------- cached hop list
//
// The alternative to recomputing every target lookup at every Lanczos step:
// resolve the block's hops once into packed 8-byte entries
//   col(32) | dir(3)<<32 | sign parity(1)<<35 | shift(6)<<36 | deg_t(7)<<42
// (nonzero-amplitude hops to active targets, rows contiguous, int64 row
// pointers) and stream them. The coefficient is rebuilt from the direction
// amplitude, momentum phase and orbit sizes with a few FLOPs. Entries are in
// the on-the-fly kernel's hop order (spin, source site, direction), so both
// sources give identical sums.

__device__ __forceinline__ uint64_t pack_hop(uint32_t col, int dir, int par, int shift, int deg) {
  return static_cast<uint64_t>(col) | (static_cast<uint64_t>(dir) << 32) | (static_cast<uint64_t>(par) << 35) |
         (static_cast<uint64_t>(shift) << 36) | (static_cast<uint64_t>(deg) << 42);
}

template <typename W>
__global__ void k_hoplist(const __grid_constant__ CsrParams<W> P, const uint64_t* __restrict__ binom,
                          const int64_t* __restrict__ row_ptr, uint64_t* __restrict__ hops) {
  const Geom& g = P.g;
  const BlockView<W>& v = P.v;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < v.dim;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const uint32_t ur = v.row_meta[i] & 0x3FFFFFFu;
    const W u = v.ur_bits[ur];
    const W d = v.row_dn[i];
    int64_t pos = row_ptr[i];
    for (int spin = 0; spin < 2; ++spin) {
      const W bits = spin ? d : u;
      for (W m = bits; m; m &= m - 1) {
        const int from = ctz(m);
        for (int dir = 0; dir < 8; ++dir) {  // same filter as the nonzero-hop count pass
          const int to = g.nb[from][dir];
          if ((bits >> to) & 1) continue;
          if (g.amp_re[dir] == 0.0 && g.amp_im[dir] == 0.0) continue;
          const W moved = bits ^ (static_cast<W>(1) << from) ^ (static_cast<W>(1) << to);
          int64_t c;
          int shift, sgn, deg_t;
          if (!resolve<W, uint64_t>(spin ? u : moved, spin ? moved : d, spin == 0, ur, v, g, binom, c, shift, sgn,
                                    deg_t))
            continue;
          hops[pos++] = pack_hop(static_cast<uint32_t>(c), dir, jw_parity(bits, from, to) ^ sgn, shift, deg_t);
        }
      }
    }
  }
}

__device__ __forceinline__ uint64_t ld_stream_u64(const uint64_t* p) {
  uint64_t r;
  asm("ld.global.nc.L1::no_allocate.u64 %0, [%1];" : "=l"(r) : "l"(p));
  return r;
}

// H*V from the cached hop list (same contract as k_hv).
template <typename W, typename T, int NV, int U, int MINB>
__global__ void __launch_bounds__(kHvThreads, MINB) k_hv_list(const __grid_constant__ HvParams<W> P,
                                                              const int64_t* __restrict__ hptr,
                                                              const uint64_t* __restrict__ hops,
                                                              const typename CT<T>::V* __restrict__ in,
                                                              typename CT<T>::V* __restrict__ out,
                                                              const double* __restrict__ scale,
                                                              fx128* __restrict__ partial) {
  using V = typename CT<T>::V;
  constexpr int VPL = CT<T>::VPL;
  constexpr int CPR = NV / VPL;
  constexpr int G = CPR < 32 ? CPR : 32;
  constexpr int LPL = CPR / G;
  __shared__ double s_ph[2][64];
  __shared__ double s_amp[2][8];
  __shared__ double s_sq[65];
  __shared__ fx128 s_acc[kHvWarps][NV];
  const Geom& g = P.g;
  const BlockView<W>& v = P.v;
  const int tid = threadIdx.x;
  for (int i = tid; i < 64; i += kHvThreads) {
    s_ph[0][i] = v.phase_re[i];
    s_ph[1][i] = v.phase_im[i];
  }
  if (tid < 8) {
    s_amp[0][tid] = g.amp_re[tid];
    s_amp[1][tid] = g.amp_im[tid];
  }
  if (tid < 65) s_sq[tid] = g.sqrt_deg[tid];
  for (int i = tid; i < kHvWarps * NV; i += kHvThreads) s_acc[i / NV][i % NV] = 0;
  __syncthreads();
  const int lane = tid & 31;
  const int wid = tid >> 5;
  const int grp = lane / G;
  const int sub = lane % G;
  double sc[LPL][VPL];
#pragma unroll
  for (int l = 0; l < LPL; ++l)
#pragma unroll
    for (int e = 0; e < VPL; ++e) sc[l][e] = scale ? scale[(l * G + sub) * VPL + e] : 1.0;
  const int64_t nwarps = static_cast<int64_t>(gridDim.x) * kHvWarps;
  for (int64_t row = static_cast<int64_t>(blockIdx.x) * kHvWarps + wid; row < v.dim; row += nwarps) {
    const uint32_t meta = __ldg(v.row_meta + row);
    const double inv_s = 1.0 / s_sq[static_cast<int>(meta >> 26) + 1];
    const int64_t h0 = __ldg(hptr + row), h1 = __ldg(hptr + row + 1);
    V acc[LPL];
#pragma unroll
    for (int l = 0; l < LPL; ++l) vzero(acc[l]);
    for (int64_t b = h0; b < h1; b += 32) {
      const int64_t q = b + lane;
      int64_t col = -1;
      T cr = 0, ci = 0;
      if (q < h1) {
        const uint64_t e = ld_stream_u64(hops + q);
        col = static_cast<int64_t>(static_cast<uint32_t>(e));
        const int dir = static_cast<int>((e >> 32) & 7);
        const int p = static_cast<int>((e >> 35) & 1);
        const int shift = static_cast<int>((e >> 36) & 63);
        const int deg_t = static_cast<int>((e >> 42) & 127);
        const double ar = p ? -s_amp[0][dir] : s_amp[0][dir];
        const double ai = p ? -s_amp[1][dir] : s_amp[1][dir];
        const double pr = s_ph[0][shift], pi = s_ph[1][shift];
        const double ratio = s_sq[deg_t] * inv_s;
        cr = static_cast<T>((ar * pr - ai * pi) * ratio);
        ci = static_cast<T>((ar * pi + ai * pr) * ratio);
      }
      gather_batch<T, NV, U>(in, col, cr, ci, static_cast<int>(min(static_cast<int64_t>(32), h1 - b)), acc);
    }
#pragma unroll
    for (int o = G; o < 32; o <<= 1)
#pragma unroll
      for (int l = 0; l < LPL; ++l) vadd(acc[l], shfl_xor_v(acc[l], o));
    if (grp == 0) {
      const W u = __ldg(v.ur_bits + (meta & 0x3FFFFFFu));
      const W d = __ldg(v.row_dn + row);
      const double diag = diag_energy(u, d, g);
#pragma unroll
      for (int l = 0; l < LPL; ++l) {
        const V x = ld_stream(in + row * CPR + l * G + sub);
        double dt[VPL];
        out[row * CPR + l * G + sub] = finish_row(x, acc[l], diag, sc[l], dt);
        if (partial) {
#pragma unroll
          for (int e = 0; e < VPL; ++e) s_acc[wid][(l * G + sub) * VPL + e] += fx_of(dt[e]);
        }
      }
    }
  }
  flush_dot<NV>(s_acc, partial);
}

// H*V from the cached hop list for sweeps whose row is one 16-byte chunk
// (2 FP32 or 1 FP64 complex vectors). There a warp per row leaves most of
// the hop chain's latency exposed (a row's range, then its entries, then its
// gathers, two 32-lane rounds for a 34-hop row), so here 8 lanes share a row
// and a warp works on 4 rows at once; each lane takes every 8th hop of its
// row with kRowU entries and gathers in flight, then the 8 partial sums are
// folded by shuffles. The sum order differs from k_hv / k_hv_list (lane
// partials over every 8th hop instead of every 32nd) but is fixed, so the
// results are deterministic; the grid, and hence the order of the per-CTA
// dot-product partials, is the other kernels'.
constexpr int kRowLanes = 8;
constexpr int kRowU = 4;

template <typename W, typename T, int NV>
__global__ void __launch_bounds__(kHvThreads, 4) k_hv_rows(const __grid_constant__ HvParams<W> P,
                                                           const int64_t* __restrict__ hptr,
                                                           const uint64_t* __restrict__ hops,
                                                           const typename CT<T>::V* __restrict__ in,
                                                           typename CT<T>::V* __restrict__ out,
                                                           const double* __restrict__ scale,
                                                           fx128* __restrict__ partial) {
  using V = typename CT<T>::V;
  constexpr int VPL = CT<T>::VPL;
  static_assert(NV == VPL, "one 16-byte chunk per row");
  constexpr int kRowsPerWarp = 32 / kRowLanes;
  __shared__ double s_ph[2][64];
  __shared__ double s_amp[2][8];
  __shared__ double s_sq[65];
  __shared__ fx128 s_acc[kHvWarps * kRowsPerWarp][NV];
  const Geom& g = P.g;
  const BlockView<W>& v = P.v;
  const int tid = threadIdx.x;
  for (int i = tid; i < 64; i += kHvThreads) {
    s_ph[0][i] = v.phase_re[i];
    s_ph[1][i] = v.phase_im[i];
  }
  if (tid < 8) {
    s_amp[0][tid] = g.amp_re[tid];
    s_amp[1][tid] = g.amp_im[tid];
  }
  if (tid < 65) s_sq[tid] = g.sqrt_deg[tid];
  for (int i = tid; i < kHvWarps * kRowsPerWarp * NV; i += kHvThreads) s_acc[i / NV][i % NV] = 0;
  __syncthreads();
  const int lane = tid & 31;
  const int wid = tid >> 5;
  const int grp = lane / kRowLanes;
  const int sub = lane % kRowLanes;
  double sc[VPL];
#pragma unroll
  for (int e = 0; e < VPL; ++e) sc[e] = scale ? scale[e] : 1.0;
  const int64_t nwarps = static_cast<int64_t>(gridDim.x) * kHvWarps;
  // warp-uniform loop over groups of 4 rows (the shuffles need all lanes)
  for (int64_t rb = (static_cast<int64_t>(blockIdx.x) * kHvWarps + wid) * kRowsPerWarp; rb < v.dim;
       rb += nwarps * kRowsPerWarp) {
    const int64_t row = rb + grp;
    const bool ok = row < v.dim;
    uint32_t meta = 0;
    int64_t h0 = 0, h1 = 0;
    if (ok) {
      meta = __ldg(v.row_meta + row);
      h0 = __ldg(hptr + row);
      h1 = __ldg(hptr + row + 1);
    }
    const double inv_s = 1.0 / s_sq[static_cast<int>(meta >> 26) + 1];
    V acc;
    vzero(acc);
    for (int64_t q0 = h0 + sub; q0 < h1; q0 += kRowLanes * kRowU) {
      uint64_t e[kRowU];
#pragma unroll
      for (int u = 0; u < kRowU; ++u) {
        const int64_t q = q0 + u * kRowLanes;
        e[u] = q < h1 ? ld_stream_u64(hops + q) : ~0ULL;
      }
      V x[kRowU];
      T cr[kRowU], ci[kRowU];
#pragma unroll
      for (int u = 0; u < kRowU; ++u) {
        cr[u] = 0;
        ci[u] = 0;
        vzero(x[u]);
        if (e[u] != ~0ULL) {
          const int64_t col = static_cast<int64_t>(static_cast<uint32_t>(e[u]));
          const int dir = static_cast<int>((e[u] >> 32) & 7);
          const int p = static_cast<int>((e[u] >> 35) & 1);
          const int shift = static_cast<int>((e[u] >> 36) & 63);
          const int deg_t = static_cast<int>((e[u] >> 42) & 127);
          const double ar = p ? -s_amp[0][dir] : s_amp[0][dir];
          const double ai = p ? -s_amp[1][dir] : s_amp[1][dir];
          const double pr = s_ph[0][shift], pi = s_ph[1][shift];
          const double ratio = s_sq[deg_t] * inv_s;
          cr[u] = static_cast<T>((ar * pr - ai * pi) * ratio);
          ci[u] = static_cast<T>((ar * pi + ai * pr) * ratio);
          x[u] = ld_stream(in + col);
        }
      }
#pragma unroll
      for (int u = 0; u < kRowU; ++u) cfma<T>(acc, cr[u], ci[u], x[u]);
    }
#pragma unroll
    for (int o = kRowLanes / 2; o > 0; o >>= 1) vadd(acc, shfl_xor_v(acc, o));
    if (sub == 0 && ok) {
      const W uw = __ldg(v.ur_bits + (meta & 0x3FFFFFFu));
      const W dw = __ldg(v.row_dn + row);
      const double diag = diag_energy(uw, dw, g);
      const V xr = ld_stream(in + row);
      double dt[VPL];
      out[row] = finish_row(xr, acc, diag, sc, dt);
      if (partial) {
#pragma unroll
        for (int e = 0; e < VPL; ++e) s_acc[wid * kRowsPerWarp + grp][e] += fx_of(dt[e]);
      }
    }
  }
  flush_dot<NV>(s_acc, partial);
}

template <typename W, typename R, typename T, int NV, int U, int MINB>
void launch_hv_t(Ctx& c, const void* in, void* out, const double* scale, fx128* partial, int grid) {
  HvParams<W> P;
  P.g = c.geom;
  if constexpr (sizeof(W) == 4) P.v = view32(c);
  else P.v = view64(c);
  using V = typename CT<T>::V;
  if (c.hl_active) {
    if constexpr (NV == CT<T>::VPL) {
      if (c.hv_rows) {
        k_hv_rows<W, T, NV><<<grid, kHvThreads, 0, c.stream>>>(P, c.hl_ptr.as<int64_t>(), c.hl_ent.as<uint64_t>(),
                                                               static_cast<const V*>(in), static_cast<V*>(out),
                                                               scale, partial);
        return;
      }
    }
    k_hv_list<W, T, NV, U, MINB><<<grid, kHvThreads, 0, c.stream>>>(P, c.hl_ptr.as<int64_t>(), c.hl_ent.as<uint64_t>(),
                                                                    static_cast<const V*>(in), static_cast<V*>(out),
                                                                    scale, partial);
    return;
  }
  const R* gb = sizeof(R) == 4 ? reinterpret_cast<const R*>(c.binom32.p) : reinterpret_cast<const R*>(c.binom.p);
  k_hv<W, R, T, NV, U, MINB><<<grid, kHvThreads, 0, c.stream>>>(P, static_cast<const V*>(in), static_cast<V*>(out),
                                                                scale, partial, gb);
}

// Kernel variants the autotuner chooses from, (gather unroll U, CTAs/SM):
// 0 (1,4), 1 (2,4), 2 (4,3), 3 (4,2), 4 (8,2).
constexpr int kNumVariants = 5;

template <typename W, typename R, typename T, int NV>
void launch_hv_var(Ctx& c, int var, const void* in, void* out, const double* scale, fx128* partial, int grid) {
  switch (var) {
    case 0: launch_hv_t<W, R, T, NV, 1, 4>(c, in, out, scale, partial, grid); return;
    case 1: launch_hv_t<W, R, T, NV, 2, 4>(c, in, out, scale, partial, grid); return;
    case 2: launch_hv_t<W, R, T, NV, 4, 3>(c, in, out, scale, partial, grid); return;
    case 3: launch_hv_t<W, R, T, NV, 4, 2>(c, in, out, scale, partial, grid); return;
    case 4: launch_hv_t<W, R, T, NV, 8, 2>(c, in, out, scale, partial, grid); return;
    default: break;
  }
  throw Error(FTLM_ERR_ARG, "bad H*V kernel variant");
}

template <typename W, typename R, typename T>
void launch_hv_nv(Ctx& c, int var, const void* in, void* out, int nv, const double* scale, fx128* partial,
                  int grid) {
  switch (nv) {
    case 1:
      if constexpr (sizeof(T) == 8) { launch_hv_var<W, R, T, 1>(c, var, in, out, scale, partial, grid); return; }
      break;
    case 2: launch_hv_var<W, R, T, 2>(c, var, in, out, scale, partial, grid); return;
    case 4: launch_hv_var<W, R, T, 4>(c, var, in, out, scale, partial, grid); return;
    case 8: launch_hv_var<W, R, T, 8>(c, var, in, out, scale, partial, grid); return;
    case 16: launch_hv_var<W, R, T, 16>(c, var, in, out, scale, partial, grid); return;
    case 32: launch_hv_var<W, R, T, 32>(c, var, in, out, scale, partial, grid); return;
    case 64: launch_hv_var<W, R, T, 64>(c, var, in, out, scale, partial, grid); return;
    case 128: launch_hv_var<W, R, T, 128>(c, var, in, out, scale, partial, grid); return;
    default: break;
  }
  throw Error(FTLM_ERR_ARG, "unsupported vectors per sweep: " + std::to_string(nv));
}

void launch_any(Ctx& c, int var, const void* in, void* out, int nv, bool fp32, const double* scale,
                fx128* partial, int grid) {
  if (c.wide) {
    if (fp32) launch_hv_nv<uint64_t, uint64_t, float>(c, var, in, out, nv, scale, partial, grid);
    else launch_hv_nv<uint64_t, uint64_t, double>(c, var, in, out, nv, scale, partial, grid);
  } else {
    if (fp32) launch_hv_nv<uint32_t, uint32_t, float>(c, var, in, out, nv, scale, partial, grid);
    else launch_hv_nv<uint32_t, uint32_t, double>(c, var, in, out, nv, scale, partial, grid);
  }
}

// Autotuner: the first time an H*V of a given (word size, precision, vectors
// per sweep, block-size class) runs on a block big enough to measure, every
// variant is timed on that block (output to the caller's scratch, no state
// touched) and the fastest is kept for the process (FTLM_HV_RETUNE=1: once per
// context instead). Results do not depend on the variant (same per-row sum
// order; the dot-product partials are exact fixed-point sums).
std::mutex g_tune_mu;
std::map<uint64_t, int> g_tuned;

}  // namespace

bool hv_tuned_lookup(Ctx& c, uint64_t key, int& var) {
  auto lt = c.tuned_local.find(key);
  if (lt != c.tuned_local.end()) {
    var = lt->second;
    return true;
  }
  if (c.hv_retune) return false;
  std::lock_guard<std::mutex> lock(g_tune_mu);
  auto it = g_tuned.find(key);
  if (it == g_tuned.end()) return false;
  var = it->second;
  return true;
}

void hv_tuned_store(Ctx& c, uint64_t key, int var) {
  c.tuned_local[key] = var;
  std::lock_guard<std::mutex> lock(g_tune_mu);
  g_tuned[key] = var;
}

int hv_size_class(int64_t dim) {
  int k = 0;
  while (dim >= 16 && k < 40) {
    dim >>= 2;
    ++k;
  }
  return k;
}

namespace {

template <typename W>
int64_t block_csr_device_t(Ctx& c, DBuf& row_ptr, DBuf& col, DBuf& val, DBuf& diag) {
  const int64_t D = c.blk.dim;
  if (D > 0x7fffffffLL) throw Error(FTLM_ERR_CAPACITY, "block CSR keeps 32-bit columns: block above 2^31 rows");
  CsrParams<W> P;
  P.g = c.geom;
  if constexpr (sizeof(W) == 4) P.v = view32(c);
  else P.v = view64(c);
  DBuf& cnt = c.sec.tmp_a;
  cnt.ensure(sizeof(int32_t) * std::max<int64_t>(D, 1));
  DBuf& rp64 = c.sec.tmp_d;
  rp64.ensure(sizeof(int64_t) * (D + 1));
  k_csr<W><<<grid_for(D, 128), 128, 0, c.stream>>>(P, c.binom.as<uint64_t>(), 0, cnt.as<int32_t>(), nullptr, nullptr,
                                                    nullptr, nullptr);
  FTLM_LAUNCH_CHECK();
  const int64_t nnz = scan_excl_i32_to_i64(c, cnt.as<int32_t>(), rp64.as<int64_t>(), D);
  FTLM_CUDA(cudaMemcpyAsync(rp64.as<int64_t>() + D, &nnz, sizeof(int64_t), cudaMemcpyHostToDevice, c.stream));
  if (nnz > 0x7fffffffLL) throw Error(FTLM_ERR_CAPACITY, "block CSR exceeds 2^31 entries");
  row_ptr.ensure(sizeof(int32_t) * (D + 1));
  col.ensure(sizeof(int32_t) * std::max<int64_t>(nnz, 1));
  val.ensure(sizeof(double) * 2 * std::max<int64_t>(nnz, 1));
  diag.ensure(sizeof(double) * std::max<int64_t>(D, 1));
  k_csr<W><<<grid_for(D, 128), 128, 0, c.stream>>>(P, c.binom.as<uint64_t>(), 1, nullptr, rp64.as<int64_t>(),
                                                    col.as<int32_t>(), val.as<double>(), diag.as<double>());
  k_i64_to_i32<<<grid_for(D + 1, 256), 256, 0, c.stream>>>(rp64.as<int64_t>(), row_ptr.as<int32_t>(), D + 1);
  FTLM_LAUNCH_CHECK();
  FTLM_CUDA(cudaStreamSynchronize(c.stream));
  c.prof.kernel_launches += 3;
  return nnz;
}

template <typename W>
void block_dense_device_t(Ctx& c, double2* A) {
  CsrParams<W> P;
  P.g = c.geom;
  if constexpr (sizeof(W) == 4) P.v = view32(c);
  else P.v = view64(c);
  k_csr<W><<<grid_for(c.blk.dim, 128), 128, 0, c.stream>>>(P, c.binom.as<uint64_t>(), 3, nullptr, nullptr, nullptr,
                                                            reinterpret_cast<double*>(A), nullptr);
  FTLM_LAUNCH_CHECK();
  c.prof.kernel_launches += 1;
}

template <typename W>
int64_t block_nonzero_hops_t(Ctx& c) {
  const int64_t D = c.blk.dim;
  if (D <= 0) return 0;
  CsrParams<W> P;
  P.g = c.geom;
  if constexpr (sizeof(W) == 4) P.v = view32(c);
  else P.v = view64(c);
  DBuf& cnt = c.sec.tmp_a;
  cnt.ensure(sizeof(int32_t) * D);
  DBuf& rp64 = c.sec.tmp_d;
  rp64.ensure(sizeof(int64_t) * (D + 1));
  k_csr<W><<<grid_for(D, 128), 128, 0, c.stream>>>(P, c.binom.as<uint64_t>(), 2, cnt.as<int32_t>(), nullptr, nullptr,
                                                    nullptr, nullptr);
  FTLM_LAUNCH_CHECK();
  return scan_excl_i32_to_i64(c, cnt.as<int32_t>(), rp64.as<int64_t>(), D);
}

template <typename W>
bool hoplist_build_t(Ctx& c) {
  const int64_t D = c.blk.dim;
  if (D <= 0) return false;
  if (D > 0xFFFFFFFFLL) return false;  // entries keep 32-bit columns
  CsrParams<W> P;
  P.g = c.geom;
  if constexpr (sizeof(W) == 4) P.v = view32(c);
  else P.v = view64(c);
  DBuf& cnt = c.sec.tmp_a;
  cnt.ensure(sizeof(int32_t) * D);
  k_csr<W><<<grid_for(D, 128), 128, 0, c.stream>>>(P, c.binom.as<uint64_t>(), 2, cnt.as<int32_t>(), nullptr, nullptr,
                                                    nullptr, nullptr);
  FTLM_LAUNCH_CHECK();
  c.hl_ptr.ensure(sizeof(int64_t) * (D + 1));
  const int64_t nnz = scan_excl_i32_to_i64(c, cnt.as<int32_t>(), c.hl_ptr.as<int64_t>(), D);
  FTLM_CUDA(cudaMemcpyAsync(c.hl_ptr.as<int64_t>() + D, &nnz, sizeof(int64_t), cudaMemcpyHostToDevice, c.stream));
  size_t free_b = 0, total_b = 0;
  FTLM_CUDA(cudaMemGetInfo(&free_b, &total_b));
  const size_t need = sizeof(uint64_t) * static_cast<size_t>(std::max<int64_t>(nnz, 1));
  if (need > c.hl_ent.cap && need + (size_t(2) << 30) > free_b + c.hl_ent.cap) return false;  // keep 2 GiB headroom
  c.hl_ent.ensure(need);
  k_hoplist<W><<<grid_for(D, 128), 128, 0, c.stream>>>(P, c.binom.as<uint64_t>(), c.hl_ptr.as<int64_t>(),
                                                        c.hl_ent.as<uint64_t>());
  FTLM_LAUNCH_CHECK();
  FTLM_CUDA(cudaStreamSynchronize(c.stream));
  c.prof.kernel_launches += 5;
  c.hl_nnz = nnz;
  return true;
}

}  // namespace

bool hoplist_build(Ctx& c) {
  if (c.wide) return hoplist_build_t<uint64_t>(c);
  return hoplist_build_t<uint32_t>(c);
}

int64_t block_nonzero_hops(Ctx& c) {
  if (c.wide) return block_nonzero_hops_t<uint64_t>(c);
  return block_nonzero_hops_t<uint32_t>(c);
}

int64_t block_csr_device(Ctx& c, DBuf& row_ptr, DBuf& col, DBuf& val, DBuf& diag) {
  if (c.wide) return block_csr_device_t<uint64_t>(c, row_ptr, col, val, diag);
  return block_csr_device_t<uint32_t>(c, row_ptr, col, val, diag);
}

void block_dense_device(Ctx& c, double2* A) {
  if (c.wide) block_dense_device_t<uint64_t>(c, A);
  else block_dense_device_t<uint32_t>(c, A);
}

void block_csr(Ctx& c, std::vector<int32_t>& row_ptr, std::vector<int32_t>& col, std::vector<double>& val,
               std::vector<double>& diag) {
  DBuf rp, cl, vl, dg;
  const int64_t D = c.blk.dim;
  const int64_t nnz = block_csr_device(c, rp, cl, vl, dg);
  row_ptr.resize(D + 1);
  col.resize(nnz);
  val.resize(2 * nnz);
  diag.resize(D);
  FTLM_CUDA(cudaMemcpy(row_ptr.data(), rp.p, sizeof(int32_t) * (D + 1), cudaMemcpyDeviceToHost));
  if (nnz) {
    FTLM_CUDA(cudaMemcpy(col.data(), cl.p, sizeof(int32_t) * nnz, cudaMemcpyDeviceToHost));
    FTLM_CUDA(cudaMemcpy(val.data(), vl.p, sizeof(double) * 2 * nnz, cudaMemcpyDeviceToHost));
  }
  if (D) FTLM_CUDA(cudaMemcpy(diag.data(), dg.p, sizeof(double) * D, cudaMemcpyDeviceToHost));
  rp.release();
  cl.release();
  vl.release();
  dg.release();
}

// Grid of the H*V kernel: one warp per row for small blocks, else four CTAs
// per SM (rows round-robin over warps). Independent of the kernel variant, so
// the order of the per-CTA dot-product partials is too.
int hv_grid(Ctx& c, int nv, bool fp32) {
  (void)nv;
  (void)fp32;
  const int64_t by_rows = (c.blk.dim + kHvWarps - 1) / kHvWarps;
  const int64_t cap = static_cast<int64_t>(c.sm_count) * 4;
  return static_cast<int>(std::max<int64_t>(1, std::min(by_rows, cap)));
}

int hv_variant(Ctx& c, const void* in, void* out, int nv, bool fp32, int grid) {
  if (c.hv_forced >= 0 && c.hv_forced < kNumVariants) return c.hv_forced;
  if (c.hl_active && c.hv_rows && nv == (fp32 ? 2 : 1)) return 0;  // k_hv_rows has no variants
  const uint64_t key = static_cast<uint64_t>((c.wide ? 1 : 0) | (c.hl_active ? 2 : 0)) |
                       (static_cast<uint64_t>(fp32 ? 1 : 0) << 4) | (static_cast<uint64_t>(nv) << 8) |
                       (static_cast<uint64_t>(hv_size_class(c.blk.dim)) << 20) |
                       (static_cast<uint64_t>(c.device) << 32);
  int known = -1;
  if (hv_tuned_lookup(c, key, known)) return known;
  if (c.blk.dim < (1 << 15)) return 1;  // too small to measure; launch overhead dominates
  cudaEvent_t e0, e1;
  FTLM_CUDA(cudaEventCreate(&e0));
  FTLM_CUDA(cudaEventCreate(&e1));
  // best of 3 single-launch timings per variant, variants interleaved so a
  // clock or power transient does not favour one of them
  float best_ms[kNumVariants];
  for (int v = 0; v < kNumVariants; ++v) {
    best_ms[v] = 1e30f;
    launch_any(c, v, in, out, nv, fp32, nullptr, nullptr, grid);  // warm
  }
  for (int rep = 0; rep < 3; ++rep)
    for (int v = 0; v < kNumVariants; ++v) {
      FTLM_CUDA(cudaEventRecord(e0, c.stream));
      launch_any(c, v, in, out, nv, fp32, nullptr, nullptr, grid);
      FTLM_CUDA(cudaEventRecord(e1, c.stream));
      FTLM_LAUNCH_CHECK();
      FTLM_CUDA(cudaEventSynchronize(e1));
      float ms = 0.f;
      FTLM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      best_ms[v] = std::min(best_ms[v], ms);
    }
  int best = 0;
  for (int v = 1; v < kNumVariants; ++v)
    if (best_ms[v] < best_ms[best]) best = v;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  c.prof.tune_runs += 1;
  c.prof.kernel_launches += 4 * kNumVariants;
  hv_tuned_store(c, key, best);
  return best;
}

int hv_select_source(Ctx& c, int nv, bool fp32) {
  c.hl_active = false;
  c.split_active = false;
  const int64_t D = c.blk.dim;
  int mode = c.hv_mode;
  if (mode < 0) {
    // measured on a 4x4 (8,8) block (FP32): split-spin sweeps fastest from 4
    // vectors up (4.6 vs 7.8 ms per H*V at 4, 35 vs 56 at 128; 243 vs 282 ms at
    // 16 on 6x3 (9,9)), the hop list's row kernel at one chunk per row
    const bool one_chunk = nv == (fp32 ? 2 : 1);
    if (D >= kSplitMinDim && !one_chunk) mode = kSrcSplit;
    else if (D >= (1 << 14) && nv <= (fp32 ? 32 : 16)) mode = kSrcList;
    else mode = kSrcFly;
  }
  if (mode == kSrcList && !hoplist_build(c)) mode = c.hv_mode < 0 && D >= kSplitMinDim ? kSrcSplit : kSrcFly;
  if (mode == kSrcSplit && !split_prepare(c, nv, fp32)) mode = kSrcFly;
  c.hl_active = mode == kSrcList;
  c.split_active = mode == kSrcSplit;
  return mode;
}

void hv_apply(Ctx& c, const void* in, void* out, int nv, bool fp32, const double* scale, fx128* partial,
              int grid) {
  if (grid == 0) grid = hv_grid(c, nv, fp32);
  const int var = hv_variant(c, in, out, nv, fp32, grid);
  c.prof.hv_variant = var;
  launch_any(c, var, in, out, nv, fp32, scale, partial, grid);
  FTLM_LAUNCH_CHECK();
  c.prof.kernel_launches += 1;
}

}  // namespace ftlm
