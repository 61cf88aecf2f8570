// Split-spin H*V: the momentum-block Hamiltonian applied as two
// segment-local sweeps.
//
// Rows of a block are orbit representatives in the reference's parent order
// (main.cpp:643-675): (up representative ur, canonical down word), so the
// rows sharing an ur form one contiguous segment of at most C(N, N_down)
// rows. A down-spin hop keeps ur, so its target lies in the source row's own
// segment (13 MB of a 128-vector FP32 sweep on the 4x4 half-filled sector:
// L2-resident while the CTAs walk the rows in order). An up-spin hop lands in
// another segment and, on a large block, misses L2. The spin flip S
// (u, d) -> (d, u) maps the block onto the same momentum block of sector
// (N_down, N_up) and turns up-spin hops into down-spin hops there, so with
// the reference's matrix convention (M[src][tgt] = coefficient of |tgt,k> in
// H|src,k>, main.cpp:779-804)
//
//   M x = (diag + M_dn) x + S^T M'_dn conj(S) x,
//
// where M'_dn holds the down-spin hops of sector (N_down, N_up) and S is a
// permutation with one unit phase per row: row q of this block (state
// (u, d)) has the flipped state (d, u) = sign * T_shift(rep) of flipped row
// p(q), f_q = sign * e^{i k.shift}, and
//
//   x_D[p(q)] = conj(f_q) x[q],     (M_up x)[q] = f_q (M'_dn x_D)[p(q)].
//
// Both sweeps gather only inside the current segment. The Lanczos update
// writes w_{j+1} in both row orders, so no permutation pass runs per step.
// Alpha = Re<x, M x> = Re<x, y_U> + Re<x_D, y_D> (S is unitary). For
// N_up == N_down the flipped sector is the sector itself and its tables are
// shared.
#include <algorithm>
#include <cstring>

#include "ftlm_internal.h"
#include "hv_common.cuh"

namespace ftlm {

namespace {

constexpr int kSegGrab = 2;  // rows a warp takes from the shared row counter at a time
constexpr int kStnGrab = 4;  // the same for the stencil sweeps

int grid_rows(int64_t n, int threads) {
  return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>((n + threads - 1) / threads, 1 << 20)));
}

// Output rows are written once and read once by the Lanczos update: evict
// them first so the segment being gathered keeps its place in L2.
__device__ __forceinline__ void st_stream(float4* p, const float4& v) { __stcs(p, v); }
__device__ __forceinline__ void st_stream(double2* p, const double2& v) { __stcs(p, v); }

// Down-spin hops of every row of the block P.v (+ the diagonal term when
// with_diag): y = s * ((diag) x + M_dn x), per-CTA fixed-point partials of
// Re<s x, y>. One warp per row: lanes queue the row's down-spin hops, resolve
// one target each inside the segment (rank of the moved word -> class table
// of ur -> active index + segment offset), then groups of G lanes gather the
// target rows of all NV vectors. Hop order within a row: occupied source
// sites ascending, directions ascending (the reference's hop order).
template <typename W, typename R, typename T, int NV, int U, int MINB>
__global__ void __launch_bounds__(kHvThreads, MINB) k_hv_seg(const __grid_constant__ HvParams<W> P,
                                                           const typename CT<T>::V* __restrict__ in,
                                                           typename CT<T>::V* __restrict__ out,
                                                           const double* __restrict__ scale,
                                                           fx128* __restrict__ partial, const R* __restrict__ gbinom,
                                                           int with_diag, unsigned long long* __restrict__ next_row) {
  using V = typename CT<T>::V;
  constexpr int VPL = CT<T>::VPL;
  constexpr int CPR = NV / VPL;
  constexpr int G = CPR < 32 ? CPR : 32;
  constexpr int LPL = CPR / G;
  constexpr bool kSmemBinom = sizeof(W) == 4;
  constexpr int kQ = 8 * static_cast<int>(sizeof(W)) * 8;  // 8 directions x occupied sites of one spin

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

  // Rows in order: from a shared counter (next_row, zeroed before the
  // launch), kSegGrab rows per grab, so all warps stay within a few thousand
  // consecutive rows and the segment they gather from stays in L2; or
  // grid-stride when next_row is null. The order does not change any result:
  // rows are independent and the dot partials are exact integer sums.
  const int64_t nwarps = static_cast<int64_t>(gridDim.x) * kHvWarps;
  int64_t grab = 0, grab_end = 0;
  int64_t row = static_cast<int64_t>(blockIdx.x) * kHvWarps + wid;
  // lane 0 keeps the next grab in flight while the current rows are processed
  unsigned long long pend = 0;
  if (next_row && lane == 0) pend = atomicAdd(next_row, static_cast<unsigned long long>(kSegGrab));
  while (true) {
    if (next_row) {
      if (grab >= grab_end) {
        grab = static_cast<int64_t>(__shfl_sync(0xffffffffu, pend, 0));
        grab_end = min(grab + kSegGrab, v.dim);
        if (lane == 0 && grab < v.dim) pend = atomicAdd(next_row, static_cast<unsigned long long>(kSegGrab));
      }
      row = grab++;
    }
    if (row >= v.dim) break;
    const uint32_t meta = __ldg(v.row_meta + row);
    const uint32_t ur = meta & 0x3FFFFFFu;
    const int deg_s = static_cast<int>(meta >> 26) + 1;
    const W d = __ldg(v.row_dn + row);
    const int cls = __ldg(v.ur_class + ur);
    const int64_t seg = __ldg(v.aoff + ur);
    const uint64_t* dt = v.dtab + static_cast<int64_t>(cls > 0 ? cls - 1 : 0) * v.c_dn;
    const double inv_s = 1.0 / s_sq[deg_s];

    // 1) hop queue: lane k takes the k-th occupied site of the down word
    int total = 0;
    for (int k0 = 0; k0 < v.n_dn; k0 += 32) {
      const int k = k0 + lane;
      uint32_t dm = 0;
      int from = 0;
      if (k < v.n_dn) {
        from = kth_bit(d, k);
        for (int j = 0; j < g.ndir; ++j) {
          const int to = s_nb[from][g.dirs[j]];
          if (!((d >> to) & 1)) dm |= 1u << j;
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
        queue[pos++] = static_cast<uint16_t>((from << 3) | g.dirs[j]);
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
        const int from = code >> 3, dir = code & 7;
        const int to = s_nb[from][dir];
        const W moved = d ^ (static_cast<W>(1) << from) ^ (static_cast<W>(1) << to);
        const int64_t rd = static_cast<int64_t>(rank_of<W, R>(moved, binom));
        int64_t a = rd;
        int h = 0, s = 0, deg_t = 1;
        if (cls != 0) {
          const uint64_t e = __ldg(dt + rd);
          a = static_cast<int32_t>(static_cast<uint32_t>(e));
          h = static_cast<int>((e >> 32) & 0xFF);
          s = static_cast<int>((e >> 40) & 1);
          deg_t = static_cast<int>((e >> 48) & 0xFF);
        }
        if (a >= 0) {
          col = seg + a;
          const int p = jw_parity(d, from, to) ^ s;
          const double ar = p ? -s_amp[0][dir] : s_amp[0][dir];
          const double ai = p ? -s_amp[1][dir] : s_amp[1][dir];
          const double pr = s_ph[0][h], pi = s_ph[1][h];
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
    // 4) own-row term, scale, store, Lanczos dot
    if (grp == 0) {
      const double diag = with_diag ? diag_energy(__ldg(v.ur_bits + ur), d, g) : 0.0;
#pragma unroll
      for (int l = 0; l < LPL; ++l) {
        const V x = ld_stream(in + row * CPR + l * G + sub);
        double dt2[VPL];
        st_stream(out + row * CPR + l * G + sub, finish_row(x, acc[l], diag, sc[l], dt2));
        if (partial) {
#pragma unroll
          for (int e = 0; e < VPL; ++e) s_acc[wid][(l * G + sub) * VPL + e] += fx_of(dt2[e]);
        }
      }
    }
    if (!next_row) row += nwarps;
  }
  flush_dot<NV>(s_acc, partial);
}

// ---------------------------------------------------------------- stencils
//
// Class stencils: within one segment (fixed up representative ur) the
// down-spin operator depends only on the stabiliser class of ur, not on ur
// itself. Class 0 (trivial stabiliser) has every down word as a row in rank
// order; class c > 0 has its active canonical down words (act_list). So the
// down-spin hops of a whole block are one small CSR per class ("stencil"),
// rows = class rows, entries = the hop's target index inside the segment
// (16 bits) | dir << 16 | parity << 19 | shift << 20 | (deg - 1) << 26, in the
// on-the-fly kernel's hop order (source site ascending, direction ascending;
// hops to inactive orbits left out). The stencils of a 4x4 half-filled block
// take about 1 MB and stay in L1/L2, so a sweep reads per row only its row
// metadata and the gathered rows; the per-row rank and class-table lookups
// of k_hv_seg are gone. Needs C(N, N_down) <= 65536 (18 sites at half filling).

constexpr int64_t kStencilMaxRows = 65536;

template <typename W>
__global__ void k_stencil(int fill, const __grid_constant__ Geom g, int nclass, const int64_t* __restrict__ crb,
                          int64_t c_dn, const uint32_t* __restrict__ act_list, const uint64_t* __restrict__ dtab,
                          const W* __restrict__ dns, const uint64_t* __restrict__ binom, int64_t rows,
                          int32_t* __restrict__ counts, const int64_t* __restrict__ rp, uint32_t* __restrict__ ent) {
  for (int64_t r = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; r < rows;
       r += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int lo = 0, hi = nclass - 1;  // class c with crb[c] <= r < crb[c+1]
    while (lo < hi) {
      const int mid = (lo + hi + 1) / 2;
      if (crb[mid] <= r) lo = mid;
      else hi = mid - 1;
    }
    const int c = lo;
    const int64_t a = r - crb[c];
    const int64_t j = c == 0 ? a : static_cast<int64_t>(act_list[static_cast<int64_t>(c - 1) * c_dn + a]);
    const W d = dns[j];
    int64_t pos = fill ? rp[r] : 0;
    int cnt = 0;
    for (W m = d; m; m &= m - 1) {
      const int from = ctz(m);
      for (int dir = 0; dir < 8; ++dir) {
        if (g.amp_re[dir] == 0.0 && g.amp_im[dir] == 0.0) continue;
        const int to = g.nb[from][dir];
        if ((d >> to) & 1) continue;
        const W moved = d ^ (static_cast<W>(1) << from) ^ (static_cast<W>(1) << to);
        const int64_t rd = static_cast<int64_t>(rank_of<W, uint64_t>(moved, binom));
        int64_t at = rd;
        int h = 0, sg = 0, deg = 1;
        if (c != 0) {
          const uint64_t e = dtab[static_cast<int64_t>(c - 1) * c_dn + rd];
          at = static_cast<int32_t>(static_cast<uint32_t>(e));
          if (at < 0) continue;
          h = static_cast<int>((e >> 32) & 0xFF);
          sg = static_cast<int>((e >> 40) & 1);
          deg = static_cast<int>((e >> 48) & 0xFF);
        }
        if (fill)
          ent[pos++] = static_cast<uint32_t>(at) | (static_cast<uint32_t>(dir) << 16) |
                       (static_cast<uint32_t>(jw_parity(d, from, to) ^ sg) << 19) | (static_cast<uint32_t>(h) << 20) |
                       (static_cast<uint32_t>(deg - 1) << 26);
        ++cnt;
      }
    }
    if (!fill) counts[r] = cnt;
  }
}

// The segment sweep (same contract as k_hv_seg) with the class stencils as
// the operator source.
template <typename W, typename T, int NV, int U, int MINB>
__global__ void __launch_bounds__(kHvThreads, MINB) k_hv_stn(const __grid_constant__ HvParams<W> P,
                                                           const int64_t* __restrict__ crb,
                                                           const int32_t* __restrict__ srp,
                                                           const uint32_t* __restrict__ sent,
                                                           const typename CT<T>::V* __restrict__ in,
                                                           typename CT<T>::V* __restrict__ out,
                                                           const double* __restrict__ scale,
                                                           fx128* __restrict__ partial, int with_diag,
                                                           unsigned long long* __restrict__ next_row) {
  using V = typename CT<T>::V;
  constexpr int VPL = CT<T>::VPL;
  constexpr int CPR = NV / VPL;
  constexpr int G = CPR < 32 ? CPR : 32;
  constexpr int LPL = CPR / G;
  __shared__ double s_ph[2][64];
  __shared__ double s_amp[2][8];
  __shared__ double s_sq[65];
  __shared__ double s_sc[NV];  // vector scales, read at the end of a row (keeps registers for gathers)
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
  for (int i = tid; i < NV; i += kHvThreads) s_sc[i] = scale ? scale[i] : 1.0;
  for (int i = tid; i < kHvWarps * NV; i += kHvThreads) s_acc[i / NV][i % NV] = 0;
  __syncthreads();
  const int lane = tid & 31;
  const int wid = tid >> 5;
  const int grp = lane / G;
  const int sub = lane % G;
  const int64_t nwarps = static_cast<int64_t>(gridDim.x) * kHvWarps;
  int64_t grab = 0, grab_end = 0;
  int64_t row = static_cast<int64_t>(blockIdx.x) * kHvWarps + wid;
  // lane 0 keeps the next grab in flight while the current rows are processed
  unsigned long long pend = 0;
  if (next_row && lane == 0) pend = atomicAdd(next_row, static_cast<unsigned long long>(kStnGrab));
  // Re<s x, y> of the rows of one grab (kStnGrab consecutive rows starting at
  // a multiple of kStnGrab, always in row order) summed in FP64, then added
  // to the exact fixed-point accumulator once per grab: deterministic.
  double gdot[LPL][VPL];
#pragma unroll
  for (int l = 0; l < LPL; ++l)
#pragma unroll
    for (int e = 0; e < VPL; ++e) gdot[l][e] = 0.0;
  while (true) {
    if (next_row) {
      if (grab >= grab_end) {
        grab = static_cast<int64_t>(__shfl_sync(0xffffffffu, pend, 0));
        grab_end = min(grab + kStnGrab, v.dim);
        if (lane == 0 && grab < v.dim) pend = atomicAdd(next_row, static_cast<unsigned long long>(kStnGrab));
      }
      row = grab++;
    }
    if (row >= v.dim) break;
    const uint32_t meta = __ldg(v.row_meta + row);
    const uint32_t ur = meta & 0x3FFFFFFu;
    const double inv_s = 1.0 / s_sq[static_cast<int>(meta >> 26) + 1];
    const int64_t seg = __ldg(v.aoff + ur);
    const int64_t cr = __ldg(crb + __ldg(v.ur_class + ur)) + (row - seg);
    const int h0 = __ldg(srp + cr), h1 = __ldg(srp + cr + 1);
    V acc[LPL];
#pragma unroll
    for (int l = 0; l < LPL; ++l) vzero(acc[l]);
    for (int b = h0; b < h1; b += 32) {
      const int q = b + lane;
      int64_t col = -1;
      T cr_ = 0, ci = 0;
      if (q < h1) {
        const uint32_t e = __ldg(sent + q);
        col = seg + static_cast<int64_t>(e & 0xFFFFu);
        const int dir = static_cast<int>((e >> 16) & 7);
        const int p = static_cast<int>((e >> 19) & 1);
        const int shift = static_cast<int>((e >> 20) & 63);
        const int deg_t = static_cast<int>((e >> 26) & 63) + 1;
        const double ar = p ? -s_amp[0][dir] : s_amp[0][dir];
        const double ai = p ? -s_amp[1][dir] : s_amp[1][dir];
        const double pr = s_ph[0][shift], pi = s_ph[1][shift];
        const double ratio = s_sq[deg_t] * inv_s;
        cr_ = static_cast<T>((ar * pr - ai * pi) * ratio);
        ci = static_cast<T>((ar * pi + ai * pr) * ratio);
      }
      gather_batch<T, NV, U>(in, col, cr_, ci, min(32, h1 - b), acc);
    }
#pragma unroll
    for (int o = G; o < 32; o <<= 1)
#pragma unroll
      for (int l = 0; l < LPL; ++l) vadd(acc[l], shfl_xor_v(acc[l], o));
    if (grp == 0) {
      const double diag = with_diag ? diag_energy(__ldg(v.ur_bits + ur), __ldg(v.row_dn + row), g) : 0.0;
#pragma unroll
      for (int l = 0; l < LPL; ++l) {
        const V x = ld_stream(in + row * CPR + l * G + sub);
        double sc[VPL], dt2[VPL];
#pragma unroll
        for (int e = 0; e < VPL; ++e) sc[e] = s_sc[(l * G + sub) * VPL + e];
        st_stream(out + row * CPR + l * G + sub, finish_row(x, acc[l], diag, sc, dt2));
#pragma unroll
        for (int e = 0; e < VPL; ++e) gdot[l][e] += dt2[e];
      }
      if (partial && (!next_row || grab >= grab_end)) {  // end of a grab (every row when grid-stride)
#pragma unroll
        for (int l = 0; l < LPL; ++l)
#pragma unroll
          for (int e = 0; e < VPL; ++e) {
            s_acc[wid][(l * G + sub) * VPL + e] += fx_of(gdot[l][e]);
            gdot[l][e] = 0.0;
          }
      }
    }
    if (!next_row) row += nwarps;
  }
  flush_dot<NV>(s_acc, partial);
}

// Narrow sweeps (rows of at most 4 chunks: <= 8 FP32 / 4 FP64 vectors) on the
// class stencils: one warp per row leaves the row's dependent loads (meta ->
// class, offset -> stencil row -> entries -> gathers) exposed, so 8 lanes
// share a row and a warp works on 4 rows, each lane taking every 8th hop of
// its row with kStnChunks 16-byte gathers in flight (kStnChunks / CPR hops);
// shuffles fold the row. Same contract as k_hv_stn; rows are taken 4 at a
// time from the shared counter.
constexpr int kStnLanes = 8;
constexpr int kStnChunks = 4;

template <typename W, typename T, int NV>
__global__ void __launch_bounds__(kHvThreads, 4) k_hv_stn_rows(const __grid_constant__ HvParams<W> P,
                                                               const int64_t* __restrict__ crb,
                                                               const int32_t* __restrict__ srp,
                                                               const uint32_t* __restrict__ sent,
                                                               const typename CT<T>::V* __restrict__ in,
                                                               typename CT<T>::V* __restrict__ out,
                                                               const double* __restrict__ scale,
                                                               fx128* __restrict__ partial, int with_diag,
                                                               unsigned long long* __restrict__ next_row) {
  using V = typename CT<T>::V;
  constexpr int VPL = CT<T>::VPL;
  constexpr int CPR = NV / VPL;
  static_assert(CPR >= 1 && CPR <= 4, "narrow sweeps only");
  constexpr int kStnU = kStnChunks / CPR;  // hops in flight per lane
  constexpr int kRows = 32 / kStnLanes;  // rows per warp
  __shared__ double s_ph[2][64];
  __shared__ double s_amp[2][8];
  __shared__ double s_sq[65];
  __shared__ fx128 s_acc[kHvWarps * kRows][NV];
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
  for (int i = tid; i < kHvWarps * kRows * NV; i += kHvThreads) s_acc[i / NV][i % NV] = 0;
  __syncthreads();
  const int lane = tid & 31;
  const int wid = tid >> 5;
  const int grp = lane / kStnLanes;
  const int sub = lane % kStnLanes;
  double sc[CPR][VPL];
#pragma unroll
  for (int l = 0; l < CPR; ++l)
#pragma unroll
    for (int e = 0; e < VPL; ++e) sc[l][e] = scale ? scale[l * VPL + e] : 1.0;
  const int64_t nwarps = static_cast<int64_t>(gridDim.x) * kHvWarps;
  int64_t rb = (static_cast<int64_t>(blockIdx.x) * kHvWarps + wid) * kRows;
  unsigned long long pend = 0;  // lane 0: the next grab, in flight while this one is processed
  if (next_row && lane == 0) pend = atomicAdd(next_row, static_cast<unsigned long long>(kRows));
  while (true) {
    if (next_row) {
      rb = static_cast<int64_t>(__shfl_sync(0xffffffffu, pend, 0));
      if (lane == 0 && rb < v.dim) pend = atomicAdd(next_row, static_cast<unsigned long long>(kRows));
    }
    if (rb >= v.dim) break;  // warp-uniform
    const int64_t row = rb + grp;
    const bool ok = row < v.dim;
    uint32_t meta = 0;
    int64_t seg = 0;
    int h0 = 0, h1 = 0;
    if (ok) {
      meta = __ldg(v.row_meta + row);
      const uint32_t ur = meta & 0x3FFFFFFu;
      seg = __ldg(v.aoff + ur);
      const int64_t cr = __ldg(crb + __ldg(v.ur_class + ur)) + (row - seg);
      h0 = __ldg(srp + cr);
      h1 = __ldg(srp + cr + 1);
    }
    const double inv_s = 1.0 / s_sq[static_cast<int>(meta >> 26) + 1];
    V acc[CPR];
#pragma unroll
    for (int l = 0; l < CPR; ++l) vzero(acc[l]);
    for (int q0 = h0 + sub; q0 < h1; q0 += kStnLanes * kStnU) {
      uint32_t e[kStnU];
#pragma unroll
      for (int u = 0; u < kStnU; ++u) {
        const int q = q0 + u * kStnLanes;
        e[u] = q < h1 ? __ldg(sent + q) : 0xFFFFFFFFu;
      }
      V x[kStnU][CPR];
      T cr_[kStnU], ci[kStnU];
#pragma unroll
      for (int u = 0; u < kStnU; ++u) {
        cr_[u] = 0;
        ci[u] = 0;
#pragma unroll
        for (int l = 0; l < CPR; ++l) vzero(x[u][l]);
        if (e[u] != 0xFFFFFFFFu) {
          const int64_t col = seg + static_cast<int64_t>(e[u] & 0xFFFFu);
          const int dir = static_cast<int>((e[u] >> 16) & 7);
          const int p = static_cast<int>((e[u] >> 19) & 1);
          const int shift = static_cast<int>((e[u] >> 20) & 63);
          const int deg_t = static_cast<int>((e[u] >> 26) & 63) + 1;
          const double ar = p ? -s_amp[0][dir] : s_amp[0][dir];
          const double ai = p ? -s_amp[1][dir] : s_amp[1][dir];
          const double pr = s_ph[0][shift], pi = s_ph[1][shift];
          const double ratio = s_sq[deg_t] * inv_s;
          cr_[u] = static_cast<T>((ar * pr - ai * pi) * ratio);
          ci[u] = static_cast<T>((ar * pi + ai * pr) * ratio);
#pragma unroll
          for (int l = 0; l < CPR; ++l) x[u][l] = ld_stream(in + col * CPR + l);
        }
      }
#pragma unroll
      for (int u = 0; u < kStnU; ++u)
#pragma unroll
        for (int l = 0; l < CPR; ++l) cfma<T>(acc[l], cr_[u], ci[u], x[u][l]);
    }
#pragma unroll
    for (int o = kStnLanes / 2; o > 0; o >>= 1)
#pragma unroll
      for (int l = 0; l < CPR; ++l) vadd(acc[l], shfl_xor_v(acc[l], o));
    if (sub == 0 && ok) {
      const uint32_t ur = meta & 0x3FFFFFFu;
      const double diag = with_diag ? diag_energy(__ldg(v.ur_bits + ur), __ldg(v.row_dn + row), g) : 0.0;
#pragma unroll
      for (int l = 0; l < CPR; ++l) {
        const V xr = ld_stream(in + row * CPR + l);
        double dt2[VPL];
        st_stream(out + row * CPR + l, finish_row(xr, acc[l], diag, sc[l], dt2));
        if (partial) {
#pragma unroll
          for (int e2 = 0; e2 < VPL; ++e2) s_acc[wid * kRows + grp][l * VPL + e2] += fx_of(dt2[e2]);
        }
      }
    }
    if (!next_row) rb += nwarps * kRows;
  }
  flush_dot<NV>(s_acc, partial);
}

// Flip map of every row q of block Pu: the flipped state (d, u) resolved in
// the tables vd of sector (N_down, N_up): row p | shift << 32 | sign << 38.
template <typename W>
__global__ void k_flip_map(const __grid_constant__ HvParams<W> Pu, const __grid_constant__ BlockView<W> vd,
                           const uint64_t* __restrict__ binom, uint64_t* __restrict__ fmap, int* __restrict__ bad) {
  const BlockView<W>& v = Pu.v;
  for (int64_t q = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; q < v.dim;
       q += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const uint32_t ur = v.row_meta[q] & 0x3FFFFFFu;
    const W u = v.ur_bits[ur];
    const W d = v.row_dn[q];
    int64_t col;
    int shift, sgn, deg;
    if (!resolve<W, uint64_t>(d, u, true, 0, vd, Pu.g, binom, col, shift, sgn, deg) || col < 0 || col >= vd.dim) {
      atomicAdd(bad, 1);
      fmap[q] = 0;
      continue;
    }
    fmap[q] = static_cast<uint64_t>(col) | (static_cast<uint64_t>(shift) << 32) | (static_cast<uint64_t>(sgn) << 38);
  }
}

// x_D[p(q)] = conj(f_q) x[q] for every 16-byte chunk.
template <typename T>
__global__ void k_flip_scatter(int64_t dim, int CPR, const typename CT<T>::V* __restrict__ x,
                               typename CT<T>::V* __restrict__ xd, const uint64_t* __restrict__ fmap,
                               const __grid_constant__ FlipPhase ph) {
  const int64_t n = dim * CPR;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t row = i / CPR;
    int64_t p;
    double fr, fi;
    flip_coef(__ldg(fmap + row), ph, p, fr, fi);
    xd[p * CPR + (i - row * CPR)] = cmul_conj<T>(fr, fi, x[i]);
  }
}

// y[q] += f_q y_D[p(q)] for every 16-byte chunk (FP64 arithmetic).
template <typename T>
__global__ void k_flip_gather_add(int64_t dim, int CPR, typename CT<T>::V* __restrict__ y,
                                  const typename CT<T>::V* __restrict__ yd, const uint64_t* __restrict__ fmap,
                                  const __grid_constant__ FlipPhase ph) {
  const int64_t n = dim * CPR;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t row = i / CPR;
    int64_t p;
    double fr, fi;
    flip_coef(__ldg(fmap + row), ph, p, fr, fi);
    y[i] = cadd_mul<T>(y[i], fr, fi, yd[p * CPR + (i - row * CPR)]);
  }
}

template <typename W, typename R, typename T, int NV, int U, int MINB>
void launch_seg_t(Ctx& c, Ctx& t, const void* in, void* out, const double* scale, fx128* partial, int grid,
                  bool with_diag, unsigned long long* next_row) {
  HvParams<W> P;
  P.g = c.geom;
  if constexpr (sizeof(W) == 4) P.v = view32(t);
  else P.v = view64(t);
  using V = typename CT<T>::V;
  if (c.split_stencil && t.stn_ok) {
    if constexpr (NV / CT<T>::VPL <= 4) {
      if (c.stn_rows) {  // narrow rows: 8 lanes per row (no variants: the same kernel for every U, MINB)
        k_hv_stn_rows<W, T, NV><<<static_cast<int>(std::min<int64_t>(
                                      (t.blk.dim + 4 * kHvWarps - 1) / (4 * kHvWarps), int64_t(c.sm_count) * 4)),
                                  kHvThreads, 0, c.stream>>>(
            P, t.stn_crb.as<int64_t>(), t.stn_rp32.as<int32_t>(), t.stn_ent.as<uint32_t>(), static_cast<const V*>(in),
            static_cast<V*>(out), scale, partial, with_diag ? 1 : 0, next_row);
        return;
      }
    }
    k_hv_stn<W, T, NV, U, MINB><<<grid, kHvThreads, 0, c.stream>>>(
        P, t.stn_crb.as<int64_t>(), t.stn_rp32.as<int32_t>(), t.stn_ent.as<uint32_t>(), static_cast<const V*>(in),
        static_cast<V*>(out), scale, partial, with_diag ? 1 : 0, next_row);
    return;
  }
  const R* gb = sizeof(R) == 4 ? reinterpret_cast<const R*>(c.binom32.p) : reinterpret_cast<const R*>(c.binom.p);
  k_hv_seg<W, R, T, NV, U, MINB><<<grid, kHvThreads, 0, c.stream>>>(P, static_cast<const V*>(in), static_cast<V*>(out),
                                                                    scale, partial, gb, with_diag ? 1 : 0, next_row);
}

// Variants (gather unroll U, CTAs per SM), as for k_hv; each runs one wave
// of sm_count x CTAs-per-SM CTAs (the grid does not change the results: the
// dot partials are exact fixed-point sums).
constexpr int kSegVariants = 5;
constexpr int kSegMinB[kSegVariants] = {4, 4, 3, 2, 2};

template <typename W, typename R, typename T, int NV>
void launch_seg_var(Ctx& c, Ctx& t, int var, const void* in, void* out, const double* scale, fx128* partial,
                    int grid, bool with_diag, unsigned long long* nr) {
  switch (var) {
    case 0: launch_seg_t<W, R, T, NV, 1, 4>(c, t, in, out, scale, partial, grid, with_diag, nr); return;
    case 1: launch_seg_t<W, R, T, NV, 2, 4>(c, t, in, out, scale, partial, grid, with_diag, nr); return;
    case 2: launch_seg_t<W, R, T, NV, 4, 3>(c, t, in, out, scale, partial, grid, with_diag, nr); return;
    case 3: launch_seg_t<W, R, T, NV, 4, 2>(c, t, in, out, scale, partial, grid, with_diag, nr); return;
    case 4: launch_seg_t<W, R, T, NV, 8, 2>(c, t, in, out, scale, partial, grid, with_diag, nr); return;
    default: break;
  }
  throw Error(FTLM_ERR_ARG, "bad H*V kernel variant");
}

template <typename W, typename R, typename T>
void launch_seg_nv(Ctx& c, Ctx& t, int var, const void* in, void* out, int nv, const double* scale, fx128* partial,
                   int grid, bool with_diag, unsigned long long* nr) {
  switch (nv) {
    case 1:
      if constexpr (sizeof(T) == 8) {
        launch_seg_var<W, R, T, 1>(c, t, var, in, out, scale, partial, grid, with_diag, nr);
        return;
      }
      break;
    case 2: launch_seg_var<W, R, T, 2>(c, t, var, in, out, scale, partial, grid, with_diag, nr); return;
    case 4: launch_seg_var<W, R, T, 4>(c, t, var, in, out, scale, partial, grid, with_diag, nr); return;
    case 8: launch_seg_var<W, R, T, 8>(c, t, var, in, out, scale, partial, grid, with_diag, nr); return;
    case 16: launch_seg_var<W, R, T, 16>(c, t, var, in, out, scale, partial, grid, with_diag, nr); return;
    case 32: launch_seg_var<W, R, T, 32>(c, t, var, in, out, scale, partial, grid, with_diag, nr); return;
    case 64: launch_seg_var<W, R, T, 64>(c, t, var, in, out, scale, partial, grid, with_diag, nr); return;
    case 128: launch_seg_var<W, R, T, 128>(c, t, var, in, out, scale, partial, grid, with_diag, nr); return;
    default: break;
  }
  throw Error(FTLM_ERR_ARG, "unsupported vectors per sweep: " + std::to_string(nv));
}

// next_row: c.seg_sched's counter for this sweep (zeroed here, on the
// stream) or null for grid-stride rows.
void launch_seg(Ctx& c, Ctx& t, int var, const void* in, void* out, int nv, bool fp32, const double* scale,
                fx128* partial, int grid, bool with_diag, int counter_slot) {
  unsigned long long* nr = nullptr;
  if (c.seg_dynamic) {
    c.seg_counter.ensure(sizeof(unsigned long long) * 4);
    nr = c.seg_counter.as<unsigned long long>() + counter_slot;
    FTLM_CUDA(cudaMemsetAsync(nr, 0, sizeof(unsigned long long), c.stream));
  }
  if (c.wide) {
    if (fp32) launch_seg_nv<uint64_t, uint64_t, float>(c, t, var, in, out, nv, scale, partial, grid, with_diag, nr);
    else launch_seg_nv<uint64_t, uint64_t, double>(c, t, var, in, out, nv, scale, partial, grid, with_diag, nr);
  } else {
    if (fp32) launch_seg_nv<uint32_t, uint32_t, float>(c, t, var, in, out, nv, scale, partial, grid, with_diag, nr);
    else launch_seg_nv<uint32_t, uint32_t, double>(c, t, var, in, out, nv, scale, partial, grid, with_diag, nr);
  }
  FTLM_LAUNCH_CHECK();
}

int seg_grid(const Ctx& c, int var) {
  const int64_t by_rows = (c.blk.dim + kHvWarps - 1) / kHvWarps;
  const int64_t cap = static_cast<int64_t>(c.sm_count) * kSegMinB[var];
  return static_cast<int>(std::max<int64_t>(1, std::min(by_rows, cap)));
}

// The flipped tables: the context itself when N_up == N_down, else a
// companion context holding sector (N_down, N_up) of the same model.
Ctx& flipped_tables(Ctx& c) {
  if (c.sec.n_up == c.sec.n_dn) return c;
  if (!c.flipped) {
    c.flipped.reset(new Ctx());
    Ctx& f = *c.flipped;
    f.model = c.model;
    f.opts = c.opts;
    f.geom = c.geom;
    f.wide = c.wide;
    f.device = c.device;
    f.sm_count = c.sm_count;
    f.stream = c.stream;
    f.binom = c.binom;  // shared, owned by c
    f.binom32 = c.binom32;
  }
  Ctx& f = *c.flipped;
  if (f.sec.n_up != c.sec.n_dn || f.sec.n_dn != c.sec.n_up) {
    sector_prepare(f, c.sec.n_dn, c.sec.n_up);
    c.prof.kernel_launches += f.prof.kernel_launches;
    f.prof.kernel_launches = 0;
  }
  block_prepare(f, c.blk.mx, c.blk.my);
  if (f.blk.dim != c.blk.dim) throw Error(FTLM_ERR_INTERNAL, "spin-flipped block has another dimension");
  return f;
}

__global__ void k_rp_narrow(const int64_t* __restrict__ in, int32_t* __restrict__ out, int64_t n) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    out[i] = static_cast<int32_t>(in[i]);
}

// Class stencils of the prepared block of tables t (its own sector and
// block); false when a class has more than kStencilMaxRows rows.
template <typename W>
bool stencil_build_t(Ctx& c, Ctx& t) {
  const SectorTables& S = t.sec;
  const BlockTables& B = t.blk;
  if (S.c_dn > kStencilMaxRows) return false;
  std::vector<int64_t> crb(S.nclass + 1, 0);
  for (int k = 0; k < S.nclass; ++k) crb[k + 1] = crb[k] + (k == 0 ? S.c_dn : B.cls_nact[k]);
  const int64_t rows = crb[S.nclass];
  t.stn_crb.ensure(sizeof(int64_t) * (S.nclass + 1));
  FTLM_CUDA(cudaMemcpyAsync(t.stn_crb.p, crb.data(), sizeof(int64_t) * crb.size(), cudaMemcpyHostToDevice, c.stream));
  t.stn_cnt.ensure(sizeof(int32_t) * std::max<int64_t>(rows, 1));
  t.stn_rp.ensure(sizeof(int64_t) * (rows + 1));  // int64 scan, narrowed to int32 below
  const int grid = grid_rows(rows, 128);
  k_stencil<W><<<grid, 128, 0, c.stream>>>(0, c.geom, S.nclass, t.stn_crb.as<int64_t>(), S.c_dn,
                                           B.act_list.as<uint32_t>(), B.dtab.as<uint64_t>(), S.dns.as<W>(),
                                           c.binom.as<uint64_t>(), rows, t.stn_cnt.as<int32_t>(), nullptr, nullptr);
  FTLM_LAUNCH_CHECK();
  const int64_t total = scan_excl_i32_to_i64(c, t.stn_cnt.as<int32_t>(), t.stn_rp.as<int64_t>(), rows);
  if (total > 0x7fffffffLL) return false;  // the sweeps keep 32-bit entry offsets
  FTLM_CUDA(cudaMemcpyAsync(t.stn_rp.as<int64_t>() + rows, &total, sizeof(int64_t), cudaMemcpyHostToDevice,
                            c.stream));
  t.stn_ent.ensure(sizeof(uint32_t) * std::max<int64_t>(total, 1));
  k_stencil<W><<<grid, 128, 0, c.stream>>>(1, c.geom, S.nclass, t.stn_crb.as<int64_t>(), S.c_dn,
                                           B.act_list.as<uint32_t>(), B.dtab.as<uint64_t>(), S.dns.as<W>(),
                                           c.binom.as<uint64_t>(), rows, nullptr, t.stn_rp.as<int64_t>(),
                                           t.stn_ent.as<uint32_t>());
  // row offsets as int32 for the sweeps (fewer registers per row)
  t.stn_rp32.ensure(sizeof(int32_t) * (rows + 1));
  k_rp_narrow<<<grid_rows(rows + 1, 256), 256, 0, c.stream>>>(t.stn_rp.as<int64_t>(), t.stn_rp32.as<int32_t>(),
                                                             rows + 1);
  FTLM_LAUNCH_CHECK();
  FTLM_CUDA(cudaStreamSynchronize(c.stream));
  c.prof.kernel_launches += 6;
  return true;
}

// Stencils of tables t for its prepared block, built once per (sector
// generation, block).
void stencil_prepare(Ctx& c, Ctx& t) {
  const int64_t key[3] = {t.sec_gen, t.blk.mx, t.blk.my};
  if (std::memcmp(key, t.stn_for, sizeof key) == 0) return;
  t.stn_ok = c.wide ? stencil_build_t<uint64_t>(c, t) : stencil_build_t<uint32_t>(c, t);
  std::memcpy(t.stn_for, key, sizeof key);
}

template <typename W>
void flip_map_build_t(Ctx& c, Ctx& f) {
  HvParams<W> P;
  P.g = c.geom;
  BlockView<W> vd;
  if constexpr (sizeof(W) == 4) {
    P.v = view32(c);
    vd = view32(f);
  } else {
    P.v = view64(c);
    vd = view64(f);
  }
  const int64_t D = c.blk.dim;
  c.flip_map.ensure(sizeof(uint64_t) * std::max<int64_t>(D, 1) + 64);
  int* bad = reinterpret_cast<int*>(c.flip_map.as<uint64_t>() + D);
  FTLM_CUDA(cudaMemsetAsync(bad, 0, sizeof(int), c.stream));
  k_flip_map<W><<<grid_rows(D, 128), 128, 0, c.stream>>>(P, vd, c.binom.as<uint64_t>(), c.flip_map.as<uint64_t>(), bad);
  FTLM_LAUNCH_CHECK();
  int hbad = 0;
  FTLM_CUDA(cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
  FTLM_CUDA(cudaStreamSynchronize(c.stream));
  c.prof.kernel_launches += 1;
  if (hbad) throw Error(FTLM_ERR_INTERNAL, "spin flip: " + std::to_string(hbad) + " rows without an image");
}

}  // namespace

FlipPhase flip_phase(const Ctx& c) {
  FlipPhase ph;
  std::memcpy(ph.re, c.blk.phase_re, sizeof ph.re);
  std::memcpy(ph.im, c.blk.phase_im, sizeof ph.im);
  return ph;
}

bool split_prepare(Ctx& c, int nv, bool fp32) {
  const int64_t D = c.blk.dim;
  if (D <= 0) return false;
  if (D > 0x7fffffffLL) return false;  // the flip map keeps 32-bit rows
  // memory: two extra vector arrays (flipped x and y) and the 8-byte map
  const size_t esize = fp32 ? 8 : 16;
  const size_t vec = static_cast<size_t>(D) * nv * esize;
  const size_t need = 2 * vec + sizeof(uint64_t) * D;
  const size_t have = c.vec_xd.cap + c.vec_yd.cap + c.flip_map.cap;
  size_t free_b = 0, total_b = 0;
  FTLM_CUDA(cudaMemGetInfo(&free_b, &total_b));
  if (need > have && need + (size_t(2) << 30) > free_b + have) return false;  // keep 2 GiB headroom
  const int key[4] = {c.sec.n_up, c.sec.n_dn, c.blk.mx, c.blk.my};
  Ctx& f = flipped_tables(c);
  if (std::memcmp(key, c.flip_for, sizeof key) != 0 || c.flip_gen != c.sec_gen) {
    if (c.wide) flip_map_build_t<uint64_t>(c, f);
    else flip_map_build_t<uint32_t>(c, f);
    std::memcpy(c.flip_for, key, sizeof key);
    c.flip_gen = c.sec_gen;
  }
  if (c.split_stencil) {
    stencil_prepare(c, c);
    if (&f != &c) stencil_prepare(c, f);
  }
  c.vec_xd.ensure(vec);
  c.vec_yd.ensure(vec);
  return true;
}

int seg_variant(Ctx& c, const void* in, void* out, int nv, bool fp32) {
  if (c.hv_forced >= 0 && c.hv_forced < kSegVariants) return c.hv_forced;
  if (c.split_stencil && c.stn_ok && c.stn_rows && (fp32 ? nv / 2 : nv) <= 4) return 0;  // k_hv_stn_rows: no variants
  const uint64_t key = static_cast<uint64_t>((c.wide ? 1 : 0) | 4 | (c.split_stencil && c.stn_ok ? 8 : 0)) |
                       (static_cast<uint64_t>(fp32 ? 1 : 0) << 4) |
                       (static_cast<uint64_t>(nv) << 8) |
                       (static_cast<uint64_t>(hv_size_class(c.blk.dim)) << 20) |
                       (static_cast<uint64_t>(c.device) << 32);
  int best = -1;
  if (hv_tuned_lookup(c, key, best)) return best;
  if (c.blk.dim < (1 << 15)) return 1;  // too small to measure
  cudaEvent_t e0, e1;
  FTLM_CUDA(cudaEventCreate(&e0));
  FTLM_CUDA(cudaEventCreate(&e1));
  // best of 3 single-launch timings per variant, variants interleaved
  float best_ms[kSegVariants];
  for (int v = 0; v < kSegVariants; ++v) {
    best_ms[v] = 1e30f;
    launch_seg(c, c, v, in, out, nv, fp32, nullptr, nullptr, seg_grid(c, v), true, 0);  // warm
  }
  for (int rep = 0; rep < 3; ++rep)
    for (int v = 0; v < kSegVariants; ++v) {
      FTLM_CUDA(cudaEventRecord(e0, c.stream));
      launch_seg(c, c, v, in, out, nv, fp32, nullptr, nullptr, seg_grid(c, v), true, 0);
      FTLM_CUDA(cudaEventRecord(e1, c.stream));
      FTLM_CUDA(cudaEventSynchronize(e1));
      float ms = 0.f;
      FTLM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      best_ms[v] = std::min(best_ms[v], ms);
    }
  best = 0;
  for (int v = 1; v < kSegVariants; ++v)
    if (best_ms[v] < best_ms[best]) best = v;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  c.prof.tune_runs += 1;
  c.prof.kernel_launches += 4 * kSegVariants;
  hv_tuned_store(c, key, best);
  return best;
}

int hv_apply_split(Ctx& c, const void* in, const void* in_d, void* out, void* out_d, int nv, bool fp32,
                   const double* scale, fx128* partial) {
  Ctx& f = flipped_tables(c);
  const int var = seg_variant(c, in, out, nv, fp32);
  c.prof.hv_variant = var;
  const int grid = seg_grid(c, var);
  // flipped sweep first: its partials follow this block's in the array
  launch_seg(c, f, var, in_d, out_d, nv, fp32, scale, partial ? partial + static_cast<int64_t>(grid) * nv : nullptr,
             grid, false, 1);
  launch_seg(c, c, var, in, out, nv, fp32, scale, partial, grid, true, 0);
  c.prof.kernel_launches += 2;
  return 2 * grid;
}

int hv_split_max_grid(const Ctx& c) { return 2 * c.sm_count * 4; }

void flip_scatter(Ctx& c, const void* x, void* xd, int nv, bool fp32) {
  const int64_t D = c.blk.dim;
  const int CPR = fp32 ? nv / 2 : nv;
  const int grid = grid_rows(D * CPR, 256);
  if (fp32)
    k_flip_scatter<float><<<grid, 256, 0, c.stream>>>(D, CPR, static_cast<const float4*>(x), static_cast<float4*>(xd),
                                                      c.flip_map.as<uint64_t>(), flip_phase(c));
  else
    k_flip_scatter<double><<<grid, 256, 0, c.stream>>>(D, CPR, static_cast<const double2*>(x),
                                                       static_cast<double2*>(xd), c.flip_map.as<uint64_t>(),
                                                       flip_phase(c));
  FTLM_LAUNCH_CHECK();
  c.prof.kernel_launches += 1;
}

void flip_gather_add(Ctx& c, void* y, const void* yd, int nv, bool fp32) {
  const int64_t D = c.blk.dim;
  const int CPR = fp32 ? nv / 2 : nv;
  const int grid = grid_rows(D * CPR, 256);
  if (fp32)
    k_flip_gather_add<float><<<grid, 256, 0, c.stream>>>(D, CPR, static_cast<float4*>(y), static_cast<const float4*>(yd),
                                                         c.flip_map.as<uint64_t>(), flip_phase(c));
  else
    k_flip_gather_add<double><<<grid, 256, 0, c.stream>>>(D, CPR, static_cast<double2*>(y),
                                                          static_cast<const double2*>(yd), c.flip_map.as<uint64_t>(),
                                                          flip_phase(c));
  FTLM_LAUNCH_CHECK();
  c.prof.kernel_launches += 1;
}

}  // namespace ftlm
