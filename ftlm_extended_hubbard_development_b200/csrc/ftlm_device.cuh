// Device primitives of the B200 FTLM engine: lattice geometry, translations
// with their fermionic reorder signs, combinadic ranks, Philox counters.
//
// Conventions follow the reference program (PeizhiMai/FTLM_extended_Hubbard_
// development, src/main.cpp):
//   * site s = y*lx + x, bit s of a spin word (main.cpp:436)
//   * hop directions 0:+x 1:-x 2:+y 3:-y 4:+x+y 5:-x+y 6:+x-y 7:-x-y
//     (main.cpp:440-449)
//   * translation index s = dy*lx + dx (main.cpp:632-638)
//   * a translation's sign is the parity of reordering the translated
//     creation operators into ascending site order (main.cpp:579-613)
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace ftlm {

constexpr int kMaxSites = 63;

// Geometry and Hamiltonian constants shared by every kernel (passed by value).
struct Geom {
  int lx, ly, n;
  int ndir;            // number of hop directions with non-zero amplitude
  int8_t dirs[8];      // those directions
  int8_t dox[8], doy[8];  // (dx, dy) offset of each direction
  int v_mode;          // 0: V == 0; 1: V over the +x/+y bond set; 2: 1x1 self bond
  double U, V;
  double amp_re[8], amp_im[8];  // -t_dir * exp(i theta_dir), main.cpp:686-689
  uint64_t full;        // mask of the n site bits
  uint64_t rowmask;     // bits 0..lx-1
  uint64_t xkeep[64];   // xkeep[dx]: sites with x < lx - dx (stay in row under +dx)
  int8_t nb[64][8];     // neighbour of site s in direction d, main.cpp:437-449
  double sqrt_deg[65];  // sqrt(d) for orbit stabiliser sizes d = 0..64
};

__device__ __forceinline__ int popc(uint32_t x) { return __popc(x); }
__device__ __forceinline__ int popc(uint64_t x) { return __popcll(x); }
__device__ __forceinline__ int ctz(uint32_t x) { return __ffs(x) - 1; }
__device__ __forceinline__ int ctz(uint64_t x) { return __ffsll(static_cast<long long>(x)) - 1; }

// Translate a spin word by (dx, dy), 0 <= dx < lx, 0 <= dy < ly.
// Rows rotate by dx, then the whole word rotates by dy*lx. The reorder
// sign factorises: an x-rotation of a row with n_y particles, w_y of which
// wrap, costs w_y*(n_y-w_y) transpositions; a y-rotation with w wrapped out
// of N costs w*(N-w). Returns the translated word; *parity = sign bit.
template <typename W>
__device__ __forceinline__ W translate(W b, int dx, int dy, const Geom& g, int* parity) {
  int par = 0;
  const int lx = g.lx;
  if (dx) {
    const W keep = static_cast<W>(g.xkeep[dx]);
    const W rm = static_cast<W>(g.rowmask);
    for (int y = 0; y < g.ly; ++y) {
      const W row = (b >> (y * lx)) & rm;
      const int ny = popc(row);
      const int wy = popc(static_cast<W>(row >> (lx - dx)));
      par += wy * (ny - wy);
    }
    b = static_cast<W>((b & keep) << dx) | static_cast<W>((b & ~keep) >> (lx - dx));
  }
  if (dy) {
    const int sh = dy * lx;
    const W top = b >> (g.n - sh);
    const int w = popc(top);
    par += w * (popc(b) - w);
    b = static_cast<W>((b << sh) | top) & static_cast<W>(g.full);
  }
  *parity = par & 1;
  return b;
}

// Translation without the sign (occupation masks only).
template <typename W>
__device__ __forceinline__ W translate_bits(W b, int dx, int dy, const Geom& g) {
  const int lx = g.lx;
  if (dx) {
    const W keep = static_cast<W>(g.xkeep[dx]);
    b = static_cast<W>((b & keep) << dx) | static_cast<W>((b & ~keep) >> (lx - dx));
  }
  if (dy) {
    const int sh = dy * lx;
    b = static_cast<W>((b << sh) | (b >> (g.n - sh))) & static_cast<W>(g.full);
  }
  return b;
}

__device__ __forceinline__ int shift_dx(int s, const Geom& g) { return s % g.lx; }
__device__ __forceinline__ int shift_dy(int s, const Geom& g) { return s / g.lx; }
// Group law of translations: (a + b) and (-a), as shift indices.
__device__ __forceinline__ int shift_add(int a, int b, const Geom& g) {
  const int x = (a % g.lx + b % g.lx) % g.lx;
  const int y = (a / g.lx + b / g.lx) % g.ly;
  return y * g.lx + x;
}
__device__ __forceinline__ int shift_neg(int a, const Geom& g) {
  const int x = (g.lx - a % g.lx) % g.lx;
  const int y = (g.ly - a / g.lx) % g.ly;
  return y * g.lx + x;
}

// Jordan-Wigner parity of a hop from -> to: occupied sites strictly between
// them in site order (main.cpp:503-512).
template <typename W>
__device__ __forceinline__ int jw_parity(W bits, int from, int to) {
  const int lo = from < to ? from : to;
  const int hi = from < to ? to : from;
  if (hi - lo <= 1) return 0;
  const W mask = static_cast<W>((static_cast<W>(1) << (hi - lo - 1)) - 1) << (lo + 1);
  return popc(static_cast<W>(bits & mask)) & 1;
}

// Diagonal energy U*#doublons + V*sum_{bonds} n_i n_j (main.cpp:486-501).
// The reference bond set is the sorted, de-duplicated union of the +x and
// +y bonds; the only coincidences occur on the 1x1 lattice, so for every
// larger lattice the V term is four popcounts per bond direction.
template <typename W>
__device__ __forceinline__ double diag_energy(W up, W dn, const Geom& g) {
  const int doub = popc(static_cast<W>(up & dn));
  int nn = 0;
  if (g.v_mode == 1) {
    // bit s of R*(b) holds b at the +x / +y neighbour of s
    const W rxu = translate_bits(up, g.lx - 1 == 0 ? 0 : g.lx - 1, 0, g);
    const W rxd = translate_bits(dn, g.lx - 1 == 0 ? 0 : g.lx - 1, 0, g);
    const W ryu = translate_bits(up, 0, g.ly - 1 == 0 ? 0 : g.ly - 1, g);
    const W ryd = translate_bits(dn, 0, g.ly - 1 == 0 ? 0 : g.ly - 1, g);
    nn = popc(static_cast<W>(up & rxu)) + popc(static_cast<W>(up & rxd)) +
         popc(static_cast<W>(dn & rxu)) + popc(static_cast<W>(dn & rxd)) +
         popc(static_cast<W>(up & ryu)) + popc(static_cast<W>(up & ryd)) +
         popc(static_cast<W>(dn & ryu)) + popc(static_cast<W>(dn & ryd));
  } else if (g.v_mode == 2) {
    const int n0 = static_cast<int>(up & 1) + static_cast<int>(dn & 1);
    nn = n0 * n0;
  }
  return __dadd_rn(__dmul_rn(g.U, static_cast<double>(doub)),
                   __dmul_rn(g.V, static_cast<double>(nn)));
}

// Combinadic rank: rank(x) = sum_j C(p_j, j+1) over the set bits p_0 < p_1 <
// ... of x. For words of fixed popcount this is the position of x in
// ascending integer order (the order of the reference's Gosper sweep,
// main.cpp:462-484). binom is a [65][65] table, binom[n*65+k] = C(n,k).
template <typename W, typename R>
__device__ __forceinline__ R rank_of(W x, const R* binom) {
  R r = 0;
  int j = 1;
  while (x) {
    const int p = ctz(x);
    r += binom[p * 65 + j];
    ++j;
    x &= x - 1;
  }
  return r;
}

template <typename W>
__device__ W unrank(uint64_t r, int k, int n, const uint64_t* binom) {
  W x = 0;
  int hi = n;  // bits below hi remain
  for (int j = k; j >= 1; --j) {
    int p = j - 1;
    while (p + 1 < hi && binom[(p + 1) * 65 + j] <= r) ++p;
    x |= static_cast<W>(1) << p;
    r -= binom[p * 65 + j];
    hi = p;
  }
  return x;
}

// Exact fixed-point accumulation of FP64 terms (the Lanczos dot products):
// v -> round(v * 2^64) as a 128-bit two's-complement integer. Integer sums
// are associative, so a sum of converted terms does not depend on the order
// or grouping of its terms (grid size, row scheduling, kernel variant).
// Terms and sums must stay below 2^62 in magnitude; resolution 2^-64.
typedef unsigned __int128 fx128;

__device__ __forceinline__ fx128 fx_of(double v) {
  const double h = floor(v);
  const double l = v - h;  // exact, 0 <= l < 1
  const unsigned long long hi = static_cast<unsigned long long>(static_cast<long long>(h));
  return (static_cast<fx128>(hi) << 64) + static_cast<fx128>(__double2ull_rn(l * 18446744073709551616.0));
}

__device__ __forceinline__ double fx_to_double(fx128 a) {
  const long long hi = static_cast<long long>(static_cast<unsigned long long>(a >> 64));
  const unsigned long long lo = static_cast<unsigned long long>(a);
  return static_cast<double>(hi) + static_cast<double>(lo) * 5.42101086242752217003726400434970855712890625e-20;
}

// Philox4x32-10 counter-based generator (Salmon, Moraes, Dror, Shaw, SC'11).
struct P4 {
  uint32_t x[4];
};

__device__ __host__ __forceinline__ P4 philox4x32_10(P4 c, uint32_t k0, uint32_t k1) {
  for (int r = 0; r < 10; ++r) {
    const uint64_t p0 = static_cast<uint64_t>(0xD2511F53u) * c.x[0];
    const uint64_t p1 = static_cast<uint64_t>(0xCD9E8D57u) * c.x[2];
    const uint32_t hi0 = static_cast<uint32_t>(p0 >> 32), lo0 = static_cast<uint32_t>(p0);
    const uint32_t hi1 = static_cast<uint32_t>(p1 >> 32), lo1 = static_cast<uint32_t>(p1);
    P4 n;
    n.x[0] = hi1 ^ c.x[1] ^ k0;
    n.x[1] = lo1;
    n.x[2] = hi0 ^ c.x[3] ^ k1;
    n.x[3] = lo0;
    c = n;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return c;
}

// Production start-vector element: unit-modulus phase exp(2 pi i u) * amp,
// u uniform in [0, 1) from Philox keyed by the block seed with counter
// (row, sample).
__device__ __forceinline__ void philox_phase(int64_t row, int sample, uint64_t seed, double amp, double& re,
                                             double& im) {
  P4 ctr;
  ctr.x[0] = static_cast<uint32_t>(row);
  ctr.x[1] = static_cast<uint32_t>(static_cast<uint64_t>(row) >> 32);
  ctr.x[2] = static_cast<uint32_t>(sample);
  ctr.x[3] = 0x46544C4Du;
  const P4 r = philox4x32_10(ctr, static_cast<uint32_t>(seed), static_cast<uint32_t>(seed >> 32));
  const uint64_t bits53 = (static_cast<uint64_t>(r.x[0]) << 21) ^ (r.x[1] >> 11);
  const double u = static_cast<double>(bits53 & ((1ULL << 53) - 1)) * (1.0 / 9007199254740992.0);
  double sn, cs;
  sincospi(2.0 * u, &sn, &cs);
  re = amp * cs;
  im = amp * sn;
}

// Packed lookup entries.
//  up_info: ur(32) | g0(8)<<32 | sign(1)<<40   (T_g0 maps the up
//           representative onto this up word with that sign)
//  dtab:    act(int32, -1 inactive) | h(8)<<32 | sign(1)<<40 | deg(8)<<48
__device__ __host__ __forceinline__ uint64_t pack_up(uint32_t ur, int g0, int sgn) {
  return static_cast<uint64_t>(ur) | (static_cast<uint64_t>(g0) << 32) |
         (static_cast<uint64_t>(sgn & 1) << 40);
}
__device__ __host__ __forceinline__ uint64_t pack_dtab(int32_t act, int h, int sgn, int deg) {
  return static_cast<uint64_t>(static_cast<uint32_t>(act)) | (static_cast<uint64_t>(h) << 32) |
         (static_cast<uint64_t>(sgn & 1) << 40) | (static_cast<uint64_t>(deg) << 48);
}

}  // namespace ftlm
