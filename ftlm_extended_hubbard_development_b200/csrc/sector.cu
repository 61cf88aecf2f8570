// Sector and momentum-block tables, built on the GPU.
//
// Replaces build_sector_basis (main.cpp:622-721) and the orbit/activity part
// of build_momentum_block (main.cpp:723-777). Instead of a hash map over all
// full-sector states, the orbit structure is factorised: up words are
// canonicalised under the full translation group, down words under the
// stabiliser of their up representative. Every table is at most
// C(N, N_up) or C(N, N_down) long, so nothing proportional to the full
// sector dimension is stored; the only block-sized arrays are the row list
// (4 + sizeof(W) bytes per row).
#include <algorithm>
#include <cmath>
#include <cstring>

#include "ftlm_internal.h"

namespace ftlm {

namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

__global__ void k_scan_tiles(const int32_t* __restrict__ in, int64_t n, int64_t* __restrict__ tile_sums) {
  __shared__ int64_t red[kScanThreads];
  const int64_t base = static_cast<int64_t>(blockIdx.x) * kScanTile;
  int64_t s = 0;
  for (int i = 0; i < kScanItems; ++i) {
    const int64_t idx = base + static_cast<int64_t>(threadIdx.x) * kScanItems + i;
    if (idx < n) s += in[idx];
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = kScanThreads / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) tile_sums[blockIdx.x] = red[0];
}

// Exclusive scan of the tile sums by one CTA (sequential chunks of 256).
__global__ void k_scan_tile_offsets(int64_t* __restrict__ sums, int64_t ntiles, int64_t* __restrict__ total) {
  __shared__ int64_t buf[kScanThreads];
  __shared__ int64_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int64_t b = 0; b < ntiles; b += kScanThreads) {
    const int64_t i = b + threadIdx.x;
    const int64_t v = i < ntiles ? sums[i] : 0;
    buf[threadIdx.x] = v;
    __syncthreads();
    for (int o = 1; o < kScanThreads; o <<= 1) {
      const int64_t t = threadIdx.x >= o ? buf[threadIdx.x - o] : 0;
      __syncthreads();
      buf[threadIdx.x] += t;
      __syncthreads();
    }
    if (i < ntiles) sums[i] = carry + buf[threadIdx.x] - v;
    __syncthreads();
    if (threadIdx.x == kScanThreads - 1) carry += buf[kScanThreads - 1];
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = carry;
}

__global__ void k_scan_apply(const int32_t* __restrict__ in, int64_t n, const int64_t* __restrict__ offs,
                             int64_t* __restrict__ out) {
  __shared__ int64_t buf[kScanThreads];
  const int64_t base = static_cast<int64_t>(blockIdx.x) * kScanTile;
  int64_t loc[kScanItems];
  int64_t s = 0;
  for (int i = 0; i < kScanItems; ++i) {
    const int64_t idx = base + static_cast<int64_t>(threadIdx.x) * kScanItems + i;
    loc[i] = s;
    if (idx < n) s += in[idx];
  }
  buf[threadIdx.x] = s;
  __syncthreads();
  for (int o = 1; o < kScanThreads; o <<= 1) {
    const int64_t t = threadIdx.x >= o ? buf[threadIdx.x - o] : 0;
    __syncthreads();
    buf[threadIdx.x] += t;
    __syncthreads();
  }
  const int64_t pre = offs[blockIdx.x] + buf[threadIdx.x] - s;
  for (int i = 0; i < kScanItems; ++i) {
    const int64_t idx = base + static_cast<int64_t>(threadIdx.x) * kScanItems + i;
    if (idx < n) out[idx] = pre + loc[i];
  }
}

int blocks_for(int64_t n, int threads) {
  return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>((n + threads - 1) / threads, 1 << 20)));
}

// ---------------------------------------------------------------- sector

template <typename W>
__global__ void k_enum(int64_t count, int k, int n, const uint64_t* __restrict__ binom, W* __restrict__ out) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < count;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    out[i] = unrank<W>(static_cast<uint64_t>(i), k, n, binom);
}

// Up-orbit analysis: the up representative is the minimum of the up word's
// translation orbit; g0 = -s* for the first s* reaching it.
template <typename W>
__global__ void k_up_orbit(const W* __restrict__ ups, int64_t c_up, const __grid_constant__ Geom g,
                           const uint64_t* __restrict__ binom, int32_t* __restrict__ flag,
                           uint32_t* __restrict__ minrank, uint8_t* __restrict__ g0s,
                           uint8_t* __restrict__ sgns, uint64_t* __restrict__ stab,
                           uint64_t* __restrict__ sig) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < c_up;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const W u = ups[i];
    W best = u;
    int sbest = 0;
    uint64_t st = 1, sg = 0;
    for (int s = 1; s < g.n; ++s) {
      int par;
      const W t = translate(u, shift_dx(s, g), shift_dy(s, g), g, &par);
      if (t < best) {
        best = t;
        sbest = s;
      }
      if (t == u) {
        st |= 1ULL << s;
        if (par) sg |= 1ULL << s;
      }
    }
    const int g0 = shift_neg(sbest, g);
    int par0 = 0;
    translate(best, shift_dx(g0, g), shift_dy(g0, g), g, &par0);
    flag[i] = best == u ? 1 : 0;
    minrank[i] = static_cast<uint32_t>(rank_of<W, uint64_t>(best, binom));
    g0s[i] = static_cast<uint8_t>(g0);
    sgns[i] = static_cast<uint8_t>(par0);
    stab[i] = st;
    sig[i] = sg;
  }
}

template <typename W>
__global__ void k_up_finalize(const W* __restrict__ ups, int64_t c_up, const int32_t* __restrict__ flag,
                              const uint32_t* __restrict__ minrank, const uint8_t* __restrict__ g0s,
                              const uint8_t* __restrict__ sgns, const int64_t* __restrict__ urpos,
                              const uint64_t* __restrict__ stab_in, const uint64_t* __restrict__ sig_in,
                              uint64_t* __restrict__ up_info, W* __restrict__ ur_bits,
                              uint64_t* __restrict__ ur_stab, uint64_t* __restrict__ ur_sig) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < c_up;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const uint32_t ur = static_cast<uint32_t>(urpos[minrank[i]]);
    up_info[i] = pack_up(ur, g0s[i], sgns[i]);
    if (flag[i]) {
      ur_bits[ur] = ups[i];
      ur_stab[ur] = stab_in[i];
      ur_sig[ur] = sig_in[i];
    }
  }
}

struct ClassDesc {
  uint64_t stab[64];
  uint64_t sig[64];
};

// Down words under the stabiliser H of a class: canonical image d* (minimum
// over H), an h with T_h d* = d and its sign, and for canonical words the
// stabiliser in H plus the sign character of the full representative.
template <typename W>
__global__ void k_dn_class(const W* __restrict__ dns, int64_t c_dn, int ncls, const __grid_constant__ Geom g,
                           const uint64_t* __restrict__ cls_stab, const uint64_t* __restrict__ cls_sig,
                           const uint64_t* __restrict__ binom, uint32_t* __restrict__ d_star,
                           uint16_t* __restrict__ d_hs, int32_t* __restrict__ canon,
                           uint64_t* __restrict__ d_stab, uint64_t* __restrict__ d_chi) {
  const int64_t total = c_dn * ncls;
  for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int c = static_cast<int>(t / c_dn) + 1;
    const int64_t j = t % c_dn;
    const uint64_t H = cls_stab[c];
    const uint64_t S = cls_sig[c];
    const W d = dns[j];
    W best = d;
    int hbest = 0;
    uint64_t st = 1, ds = 0;
    for (uint64_t m = H & ~1ULL; m; m &= m - 1) {
      const int s = __ffsll(static_cast<long long>(m)) - 1;
      int par;
      const W x = translate(d, shift_dx(s, g), shift_dy(s, g), g, &par);
      if (x < best) {
        best = x;
        hbest = s;
      }
      if (x == d) {
        st |= 1ULL << s;
        if (par) ds |= 1ULL << s;
      }
    }
    const int h = shift_neg(hbest, g);
    int ph = 0;
    translate(best, shift_dx(h, g), shift_dy(h, g), g, &ph);
    const int sigma_h = static_cast<int>((S >> h) & 1ULL);
    d_star[t] = static_cast<uint32_t>(rank_of<W, uint64_t>(best, binom));
    d_hs[t] = static_cast<uint16_t>(h | ((ph ^ sigma_h) << 8));
    const bool is_canon = best == d;
    canon[t] = is_canon ? 1 : 0;
    d_stab[t] = is_canon ? st : 0;
    d_chi[t] = is_canon ? ((ds ^ S) & st) : 0;
  }
}

__global__ void k_narrow(const int64_t* __restrict__ in, int32_t* __restrict__ out, int64_t n) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    out[i] = static_cast<int32_t>(in[i]);
}

__global__ void k_class_counts(const uint16_t* __restrict__ ur_class, int64_t nur,
                               const int64_t* __restrict__ cls_count, int32_t* __restrict__ out) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < nur;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    out[i] = static_cast<int32_t>(cls_count[ur_class[i]]);
}

// ------------------------------------------------------------------ block

// Stabiliser character test of a canonical word for momentum (mx, my):
// active iff sign(s) * exp(2 pi i (mx dx/lx + my dy/ly)) == 1 on the whole
// stabiliser (exact integer form of the dnf > 1e-12 test, main.cpp:748-768:
// the orbit sum of a group character is |stab| or exactly zero).
__device__ __forceinline__ bool char_trivial(uint64_t stab, uint64_t chi, int mx, int my, const Geom& g) {
  const int L = g.lx * g.ly;
  for (uint64_t m = stab & ~1ULL; m; m &= m - 1) {
    const int s = __ffsll(static_cast<long long>(m)) - 1;
    const int q = (mx * shift_dx(s, g) * g.ly + my * shift_dy(s, g) * g.lx) % L;
    const bool neg = (chi >> s) & 1ULL;
    if (!neg && q != 0) return false;
    if (neg && 2 * q != L) return false;
  }
  return true;
}

__global__ void k_dn_active(int64_t total, const int32_t* __restrict__ canon, const uint64_t* __restrict__ d_stab,
                            const uint64_t* __restrict__ d_chi, int mx, int my, const __grid_constant__ Geom g,
                            int32_t* __restrict__ flag) {
  for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<int64_t>(gridDim.x) * blockDim.x)
    flag[t] = (canon[t] && char_trivial(d_stab[t], d_chi[t], mx, my, g)) ? 1 : 0;
}

// act[t] = active index or -1; act_list[c][a] = rank of the a-th active word.
__global__ void k_act_finalize(int64_t total, int64_t c_dn, const int32_t* __restrict__ flag,
                               const int64_t* __restrict__ pos, const int64_t* __restrict__ cls_base,
                               int32_t* __restrict__ act, uint32_t* __restrict__ act_list) {
  for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t c = t / c_dn;
    if (flag[t]) {
      const int64_t a = pos[t] - cls_base[c];
      act[t] = static_cast<int32_t>(a);
      act_list[c * c_dn + a] = static_cast<uint32_t>(t % c_dn);
    } else {
      act[t] = -1;
    }
  }
}

__global__ void k_dtab(int64_t total, int64_t c_dn, const uint32_t* __restrict__ d_star,
                       const uint16_t* __restrict__ d_hs, const int32_t* __restrict__ act,
                       const uint64_t* __restrict__ d_stab, uint64_t* __restrict__ dtab) {
  for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t base = (t / c_dn) * c_dn;
    const int64_t s = base + d_star[t];
    const uint16_t hs = d_hs[t];
    dtab[t] = pack_dtab(act[s], hs & 0xFF, hs >> 8, __popcll(d_stab[s]));
  }
}

template <typename W>
__global__ void k_rows(int64_t nur, int64_t c_dn, const uint16_t* __restrict__ ur_class,
                       const int64_t* __restrict__ aoff, const uint32_t* __restrict__ act_list,
                       const uint64_t* __restrict__ d_stab, const W* __restrict__ dns,
                       uint32_t* __restrict__ row_meta, W* __restrict__ row_dn) {
  for (int64_t ur = blockIdx.x; ur < nur; ur += gridDim.x) {
    const int c = ur_class[ur];
    const int64_t r0 = aoff[ur], cnt = aoff[ur + 1] - r0;
    for (int64_t t = threadIdx.x; t < cnt; t += blockDim.x) {
      int64_t j;
      int deg;
      if (c == 0) {
        j = t;
        deg = 1;
      } else {
        const int64_t base = static_cast<int64_t>(c - 1) * c_dn;
        j = act_list[base + t];
        deg = __popcll(d_stab[base + j]);
      }
      row_meta[r0 + t] = static_cast<uint32_t>(ur) | (static_cast<uint32_t>(deg - 1) << 26);
      row_dn[r0 + t] = dns[j];
    }
  }
}

// ------------------------------------------------------------------ debug

template <typename W>
__global__ void k_debug_parents(int64_t nur, int64_t c_dn, const __grid_constant__ Geom g,
                                const W* __restrict__ ur_bits, const uint16_t* __restrict__ ur_class,
                                const int64_t* __restrict__ poff, const int32_t* __restrict__ canon,
                                const int32_t* __restrict__ cidx, const uint64_t* __restrict__ d_stab,
                                const W* __restrict__ dns, uint64_t* __restrict__ up, uint64_t* __restrict__ dn,
                                int32_t* __restrict__ deg, double* __restrict__ diag) {
  for (int64_t ur = blockIdx.x; ur < nur; ur += gridDim.x) {
    const int c = ur_class[ur];
    for (int64_t j = threadIdx.x; j < c_dn; j += blockDim.x) {
      int64_t p;
      int dg;
      if (c == 0) {
        p = poff[ur] + j;
        dg = 1;
      } else {
        const int64_t t = static_cast<int64_t>(c - 1) * c_dn + j;
        if (!canon[t]) continue;
        p = poff[ur] + cidx[t];
        dg = __popcll(d_stab[t]);
      }
      up[p] = ur_bits[ur];
      dn[p] = dns[j];
      deg[p] = dg;
      diag[p] = diag_energy(ur_bits[ur], dns[j], g);
    }
  }
}

// Reference relation of every state: brute-force lexicographic minimum over
// all translations, then the first translation carrying it onto the state.
template <typename W>
__global__ void k_debug_relations(int64_t c_up, int64_t c_dn, const __grid_constant__ Geom g,
                                  const W* __restrict__ ups, const W* __restrict__ dns,
                                  const uint64_t* __restrict__ binom, const uint64_t* __restrict__ up_info,
                                  const uint16_t* __restrict__ ur_class, const int64_t* __restrict__ poff,
                                  const int32_t* __restrict__ cidx, int32_t* __restrict__ parent,
                                  int32_t* __restrict__ shift, int32_t* __restrict__ sign) {
  const int64_t total = c_up * c_dn;
  for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const W u = ups[t / c_dn], d = dns[t % c_dn];
    W bu = u, bd = d;
    for (int s = 1; s < g.n; ++s) {
      int p1, p2;
      const W tu = translate(u, shift_dx(s, g), shift_dy(s, g), g, &p1);
      const W td = translate(d, shift_dx(s, g), shift_dy(s, g), g, &p2);
      if (tu < bu || (tu == bu && td < bd)) {
        bu = tu;
        bd = td;
      }
    }
    int sh = 0, sg = 0;
    if (!(bu == u && bd == d)) {
      for (int s = 1; s < g.n; ++s) {
        int p1, p2;
        const W tu = translate(bu, shift_dx(s, g), shift_dy(s, g), g, &p1);
        const W td = translate(bd, shift_dx(s, g), shift_dy(s, g), g, &p2);
        if (tu == u && td == d) {
          sh = s;
          sg = p1 ^ p2;
          break;
        }
      }
    }
    const uint64_t info = up_info[rank_of<W, uint64_t>(bu, binom)];
    const uint32_t ur = static_cast<uint32_t>(info);
    const int c = ur_class[ur];
    const int64_t rd = static_cast<int64_t>(rank_of<W, uint64_t>(bd, binom));
    const int64_t ci = c == 0 ? rd : cidx[static_cast<int64_t>(c - 1) * c_dn + rd];
    parent[t] = static_cast<int32_t>(poff[ur] + ci);
    shift[t] = sh;
    sign[t] = sg ? -1 : 1;
  }
}

template <typename W>
W* wptr(const DBuf& b) { return b.as<W>(); }

template <typename W>
void sector_prepare_t(Ctx& c, int n_up, int n_dn) {
  SectorTables& S = c.sec;
  const Geom& g = c.geom;
  const int n = g.n;
  cudaStream_t st = c.stream;
  const uint64_t* binom = c.binom.as<uint64_t>();
  auto C = [](int a, int b) -> int64_t {  // exact: r * (a-b+i) is divisible by i
    if (b < 0 || b > a) return 0;
    unsigned __int128 r = 1;
    for (int i = 1; i <= b; ++i) r = r * static_cast<unsigned>(a - b + i) / static_cast<unsigned>(i);
    return static_cast<int64_t>(r);
  };
  S.n_up = n_up;
  S.n_dn = n_dn;
  S.c_up = C(n, n_up);
  S.c_dn = C(n, n_dn);
  S.full_dim = S.c_up * S.c_dn;
  S.ups.ensure(sizeof(W) * S.c_up);
  S.dns.ensure(sizeof(W) * S.c_dn);
  k_enum<W><<<blocks_for(S.c_up, 256), 256, 0, st>>>(S.c_up, n_up, n, binom, S.ups.as<W>());
  k_enum<W><<<blocks_for(S.c_dn, 256), 256, 0, st>>>(S.c_dn, n_dn, n, binom, S.dns.as<W>());
  FTLM_LAUNCH_CHECK();

  // up orbits
  S.tmp_a.ensure(sizeof(int32_t) * S.c_up);                    // flag
  S.tmp_b.ensure((sizeof(uint32_t) + 2) * S.c_up + 16);         // minrank | g0 | sgn
  S.tmp_c.ensure(sizeof(uint64_t) * 2 * S.c_up);                // stab | sig
  S.tmp_d.ensure(sizeof(int64_t) * (S.c_up + 1));               // urpos
  int32_t* flag = S.tmp_a.as<int32_t>();
  uint32_t* minrank = S.tmp_b.as<uint32_t>();
  uint8_t* g0s = reinterpret_cast<uint8_t*>(minrank + S.c_up);
  uint8_t* sgns = g0s + S.c_up;
  uint64_t* stab = S.tmp_c.as<uint64_t>();
  uint64_t* sig = stab + S.c_up;
  k_up_orbit<W><<<blocks_for(S.c_up, 128), 128, 0, st>>>(S.ups.as<W>(), S.c_up, g, binom, flag, minrank,
                                                          g0s, sgns, stab, sig);
  FTLM_LAUNCH_CHECK();
  S.nur = scan_excl_i32_to_i64(c, flag, S.tmp_d.as<int64_t>(), S.c_up);
  // rows pack the up-representative index into 26 bits (row_meta)
  if (S.nur > (int64_t(1) << 26))
    throw Error(FTLM_ERR_CAPACITY, "sector has more than 2^26 up representatives");
  S.up_info.ensure(sizeof(uint64_t) * S.c_up);
  S.ur_bits.ensure(sizeof(W) * S.nur);
  S.tmp_e.ensure(sizeof(uint64_t) * 2 * S.nur);
  uint64_t* ur_stab = S.tmp_e.as<uint64_t>();
  uint64_t* ur_sig = ur_stab + S.nur;
  k_up_finalize<W><<<blocks_for(S.c_up, 256), 256, 0, st>>>(S.ups.as<W>(), S.c_up, flag, minrank, g0s, sgns,
                                                             S.tmp_d.as<int64_t>(), stab, sig,
                                                             S.up_info.as<uint64_t>(), S.ur_bits.as<W>(),
                                                             ur_stab, ur_sig);
  FTLM_LAUNCH_CHECK();

  // classes (host: the list of up representatives is short)
  std::vector<uint64_t> h_st(2 * S.nur);
  FTLM_CUDA(cudaMemcpyAsync(h_st.data(), ur_stab, sizeof(uint64_t) * 2 * S.nur, cudaMemcpyDeviceToHost, st));
  FTLM_CUDA(cudaStreamSynchronize(st));
  S.cls_stab.assign(1, 1ULL);
  S.cls_sig.assign(1, 0ULL);
  std::map<std::pair<uint64_t, uint64_t>, int> cmap;
  cmap[{1ULL, 0ULL}] = 0;
  S.h_ur_class.resize(S.nur);
  for (int64_t i = 0; i < S.nur; ++i) {
    const auto key = std::make_pair(h_st[i], h_st[S.nur + i]);
    auto it = cmap.find(key);
    int cls;
    if (it == cmap.end()) {
      cls = static_cast<int>(S.cls_stab.size());
      if (cls > 65535) throw Error(FTLM_ERR_INTERNAL, "too many stabiliser classes");
      cmap[key] = cls;
      S.cls_stab.push_back(key.first);
      S.cls_sig.push_back(key.second);
    } else {
      cls = it->second;
    }
    S.h_ur_class[i] = static_cast<uint16_t>(cls);
  }
  S.nclass = static_cast<int>(S.cls_stab.size());
  S.ur_class.ensure(sizeof(uint16_t) * S.nur);
  FTLM_CUDA(cudaMemcpyAsync(S.ur_class.p, S.h_ur_class.data(), sizeof(uint16_t) * S.nur,
                            cudaMemcpyHostToDevice, st));
  c.prof.h2d_bytes += sizeof(uint16_t) * S.nur;

  // per-class down tables
  const int ncls = S.nclass - 1;
  const int64_t tot = static_cast<int64_t>(ncls) * S.c_dn;
  S.cls_ncanon.assign(S.nclass, 0);
  S.cls_ncanon[0] = S.c_dn;
  S.d_star.ensure(sizeof(uint32_t) * std::max<int64_t>(tot, 1));
  S.d_hs.ensure(sizeof(uint16_t) * std::max<int64_t>(tot, 1));
  S.d_stab.ensure(sizeof(uint64_t) * std::max<int64_t>(tot, 1));
  S.d_chi.ensure(sizeof(uint64_t) * std::max<int64_t>(tot, 1));
  S.d_cidx.ensure(sizeof(int32_t) * std::max<int64_t>(tot, 1));
  S.tmp_a.ensure(sizeof(int32_t) * std::max<int64_t>({tot, S.nur, 1}));
  S.tmp_d.ensure(sizeof(int64_t) * (std::max<int64_t>({tot, S.nur, 1}) + 1));
  std::vector<uint64_t> cs(S.cls_stab), cg(S.cls_sig);
  DBuf& cdesc = S.tmp_b;
  cdesc.ensure(sizeof(uint64_t) * 2 * S.nclass);
  FTLM_CUDA(cudaMemcpyAsync(cdesc.p, cs.data(), sizeof(uint64_t) * S.nclass, cudaMemcpyHostToDevice, st));
  FTLM_CUDA(cudaMemcpyAsync(cdesc.as<uint64_t>() + S.nclass, cg.data(), sizeof(uint64_t) * S.nclass,
                            cudaMemcpyHostToDevice, st));
  int32_t* canon = S.tmp_a.as<int32_t>();
  if (ncls > 0) {
    k_dn_class<W><<<blocks_for(tot, 128), 128, 0, st>>>(S.dns.as<W>(), S.c_dn, ncls, g, cdesc.as<uint64_t>(),
                                                        cdesc.as<uint64_t>() + S.nclass, binom,
                                                        S.d_star.as<uint32_t>(), S.d_hs.as<uint16_t>(), canon,
                                                        S.d_stab.as<uint64_t>(), S.d_chi.as<uint64_t>());
    FTLM_LAUNCH_CHECK();
    for (int cl = 1; cl < S.nclass; ++cl) {
      const int64_t base = static_cast<int64_t>(cl - 1) * S.c_dn;
      S.cls_ncanon[cl] = scan_excl_i32_to_i64(c, canon + base, S.tmp_d.as<int64_t>() + base, S.c_dn);
    }
    k_narrow<<<blocks_for(tot, 256), 256, 0, st>>>(S.tmp_d.as<int64_t>(), S.d_cidx.as<int32_t>(), tot);
    FTLM_LAUNCH_CHECK();
  }
  // keep the canonical flags for block builds and the debug views
  S.canon.ensure(sizeof(int32_t) * std::max<int64_t>(tot, 1));
  if (tot > 0)
    FTLM_CUDA(cudaMemcpyAsync(S.canon.p, canon, sizeof(int32_t) * tot, cudaMemcpyDeviceToDevice, st));

  // parent offsets
  std::vector<int64_t> h_cnt(S.nclass);
  for (int cl = 0; cl < S.nclass; ++cl) h_cnt[cl] = S.cls_ncanon[cl];
  DBuf& ccount = S.tmp_e;  // reuse: ur_stab/sig no longer needed
  ccount.ensure(sizeof(int64_t) * S.nclass + sizeof(uint64_t) * 2 * S.nur);
  int64_t* d_cnt = ccount.as<int64_t>();
  FTLM_CUDA(cudaMemcpyAsync(d_cnt, h_cnt.data(), sizeof(int64_t) * S.nclass, cudaMemcpyHostToDevice, st));
  int32_t* per_ur = S.tmp_a.as<int32_t>();
  k_class_counts<<<blocks_for(S.nur, 256), 256, 0, st>>>(S.ur_class.as<uint16_t>(), S.nur, d_cnt, per_ur);
  FTLM_LAUNCH_CHECK();
  S.ur_poff.ensure(sizeof(int64_t) * (S.nur + 1));
  S.parents = scan_excl_i32_to_i64(c, per_ur, S.ur_poff.as<int64_t>(), S.nur);
  FTLM_CUDA(cudaMemcpyAsync(S.ur_poff.as<int64_t>() + S.nur, &S.parents, sizeof(int64_t), cudaMemcpyHostToDevice, st));
  FTLM_CUDA(cudaStreamSynchronize(st));
  c.blk.mx = c.blk.my = -1;
  ++c.sec_gen;
}

template <typename W>
void block_prepare_t(Ctx& c, int mx, int my, bool rows) {
  SectorTables& S = c.sec;
  BlockTables& B = c.blk;
  const Geom& g = c.geom;
  cudaStream_t st = c.stream;
  const int ncls = S.nclass - 1;
  const int64_t tot = static_cast<int64_t>(ncls) * S.c_dn;
  B.cls_nact.assign(S.nclass, 0);
  B.cls_nact[0] = S.c_dn;
  const int32_t* canon = S.canon.as<int32_t>();
  B.act.ensure(sizeof(int32_t) * std::max<int64_t>(tot, 1));
  B.act_list.ensure(sizeof(uint32_t) * std::max<int64_t>(tot, 1));
  B.dtab.ensure(sizeof(uint64_t) * std::max<int64_t>(tot, 1));
  if (ncls > 0) {
    int32_t* flag = S.tmp_a.as<int32_t>();
    S.tmp_d.ensure(sizeof(int64_t) * (std::max<int64_t>({tot, S.nur, 1}) + 1));
    k_dn_active<<<blocks_for(tot, 256), 256, 0, st>>>(tot, canon, S.d_stab.as<uint64_t>(), S.d_chi.as<uint64_t>(),
                                                      mx, my, g, flag);
    FTLM_LAUNCH_CHECK();
    const int64_t all = scan_excl_i32_to_i64(c, flag, S.tmp_d.as<int64_t>(), tot);
    (void)all;
    // class bases within the global scan
    std::vector<int64_t> base(ncls + 1);
    for (int cl = 0; cl <= ncls; ++cl) {
      const int64_t idx = static_cast<int64_t>(cl) * S.c_dn;
      int64_t v = 0;
      if (idx < tot) {
        FTLM_CUDA(cudaMemcpyAsync(&v, S.tmp_d.as<int64_t>() + idx, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
      } else {
        v = all;
      }
      base[cl] = v;
    }
    FTLM_CUDA(cudaStreamSynchronize(st));
    base[ncls] = all;
    for (int cl = 1; cl < S.nclass; ++cl) B.cls_nact[cl] = base[cl] - base[cl - 1];
    DBuf& bb = S.tmp_e;
    bb.ensure(sizeof(int64_t) * (ncls + 1) + sizeof(int64_t) * S.nclass);
    FTLM_CUDA(cudaMemcpyAsync(bb.p, base.data(), sizeof(int64_t) * (ncls + 1), cudaMemcpyHostToDevice, st));
    k_act_finalize<<<blocks_for(tot, 256), 256, 0, st>>>(tot, S.c_dn, flag, S.tmp_d.as<int64_t>(),
                                                         bb.as<int64_t>(), B.act.as<int32_t>(),
                                                         B.act_list.as<uint32_t>());
    k_dtab<<<blocks_for(tot, 256), 256, 0, st>>>(tot, S.c_dn, S.d_star.as<uint32_t>(), S.d_hs.as<uint16_t>(),
                                                 B.act.as<int32_t>(), S.d_stab.as<uint64_t>(),
                                                 B.dtab.as<uint64_t>());
    FTLM_LAUNCH_CHECK();
  }
  // active row offsets per up representative
  DBuf& cc = S.tmp_e;
  cc.ensure(sizeof(int64_t) * (ncls + 1) + sizeof(int64_t) * S.nclass);
  int64_t* d_nact = cc.as<int64_t>() + (ncls + 1);
  FTLM_CUDA(cudaMemcpyAsync(d_nact, B.cls_nact.data(), sizeof(int64_t) * S.nclass, cudaMemcpyHostToDevice, st));
  int32_t* per_ur = S.tmp_a.as<int32_t>();
  k_class_counts<<<blocks_for(S.nur, 256), 256, 0, st>>>(S.ur_class.as<uint16_t>(), S.nur, d_nact, per_ur);
  FTLM_LAUNCH_CHECK();
  B.aoff.ensure(sizeof(int64_t) * (S.nur + 1));
  B.dim = scan_excl_i32_to_i64(c, per_ur, B.aoff.as<int64_t>(), S.nur);
  FTLM_CUDA(cudaMemcpyAsync(B.aoff.as<int64_t>() + S.nur, &B.dim, sizeof(int64_t), cudaMemcpyHostToDevice, st));
  // momentum phases, computed exactly as main.cpp:736-743
  const double kPi = 3.141592653589793238462643383279502884;
  for (int s = 0; s < g.n; ++s) {
    const int dx = s % g.lx, dy = s / g.lx;
    const double arg = 2.0 * kPi *
                       (static_cast<double>(mx * dx) / static_cast<double>(g.lx) +
                        static_cast<double>(my * dy) / static_cast<double>(g.ly));
    B.phase_re[s] = std::cos(arg);
    B.phase_im[s] = std::sin(arg);
  }
  B.mx = mx;
  B.my = my;
  if (rows && B.dim > 0) {
    B.row_meta.ensure(sizeof(uint32_t) * B.dim);
    B.row_dn.ensure(sizeof(W) * B.dim);
    const int grid = static_cast<int>(std::min<int64_t>(S.nur, 65535));
    k_rows<W><<<grid, 256, 0, st>>>(S.nur, S.c_dn, S.ur_class.as<uint16_t>(), B.aoff.as<int64_t>(),
                                    B.act_list.as<uint32_t>(), S.d_stab.as<uint64_t>(), S.dns.as<W>(),
                                    B.row_meta.as<uint32_t>(), B.row_dn.as<W>());
    FTLM_LAUNCH_CHECK();
  }
  FTLM_CUDA(cudaStreamSynchronize(st));
}

}  // namespace

int64_t scan_excl_i32_to_i64(Ctx& c, const int32_t* flags, int64_t* out, int64_t n) {
  if (n <= 0) return 0;
  const int64_t ntiles = (n + kScanTile - 1) / kScanTile;
  DBuf& tiles = c.scan_tmp;
  tiles.ensure(sizeof(int64_t) * (ntiles + 1));
  int64_t* ts = tiles.as<int64_t>();
  k_scan_tiles<<<static_cast<unsigned>(ntiles), kScanThreads, 0, c.stream>>>(flags, n, ts);
  k_scan_tile_offsets<<<1, kScanThreads, 0, c.stream>>>(ts, ntiles, ts + ntiles);
  k_scan_apply<<<static_cast<unsigned>(ntiles), kScanThreads, 0, c.stream>>>(flags, n, ts, out);
  FTLM_LAUNCH_CHECK();
  int64_t total = 0;
  FTLM_CUDA(cudaMemcpyAsync(&total, ts + ntiles, sizeof(int64_t), cudaMemcpyDeviceToHost, c.stream));
  FTLM_CUDA(cudaStreamSynchronize(c.stream));
  c.prof.kernel_launches += 3;
  return total;
}

void sector_prepare(Ctx& c, int n_up, int n_dn) {
  if (c.wide) sector_prepare_t<uint64_t>(c, n_up, n_dn);
  else sector_prepare_t<uint32_t>(c, n_up, n_dn);
}

void block_prepare(Ctx& c, int mx, int my) {
  if (c.blk.mx == mx && c.blk.my == my) return;
  if (c.wide) block_prepare_t<uint64_t>(c, mx, my, true);
  else block_prepare_t<uint32_t>(c, mx, my, true);
  const size_t k = static_cast<size_t>(my * c.geom.lx + mx);
  if (k < c.block_dims.size() && c.block_dims[k] != c.blk.dim)
    throw Error(FTLM_ERR_INTERNAL, "block dimension from the orbit tables differs from the character count");
}

namespace {

// Translation of a spin word on the host, with the parity of reordering its
// creation operators (the factorised count of the device translate()).
uint64_t host_translate(uint64_t b, int dx, int dy, const Geom& g, int* parity) {
  int par = 0;
  const int lx = g.lx;
  if (dx) {
    uint64_t out = 0;
    const uint64_t rm = g.rowmask;
    for (int y = 0; y < g.ly; ++y) {
      uint64_t row = (b >> (y * lx)) & rm;
      const int ny = __builtin_popcountll(row);
      const int wy = __builtin_popcountll(row >> (lx - dx));
      par += wy * (ny - wy);
      row = ((row << dx) | (row >> (lx - dx))) & rm;
      out |= row << (y * lx);
    }
    b = out;
  }
  if (dy) {
    const int sh = dy * lx;
    const uint64_t top = b >> (g.n - sh);
    const int w = __builtin_popcountll(top);
    par += w * (__builtin_popcountll(b) - w);
    b = ((b << sh) | top) & g.full;
  }
  *parity = par & 1;
  return b;
}

// Trace of T_(dx,dy) on the n-particle words of one spin: the sum over the
// words it fixes (unions of its site cycles) of its sign.
int64_t fixed_trace(const Geom& g, int n, int dx, int dy) {
  if (dx == 0 && dy == 0) {
    unsigned __int128 r = 1;
    for (int i = 1; i <= n; ++i) r = r * static_cast<unsigned>(g.n - n + i) / static_cast<unsigned>(i);
    return static_cast<int64_t>(r);
  }
  std::vector<uint64_t> cyc;
  uint64_t seen = 0;
  int clen = 0;
  for (int s0 = 0; s0 < g.n; ++s0) {
    if ((seen >> s0) & 1) continue;
    uint64_t m = 0;
    int len = 0;
    for (int t = s0; !((seen >> t) & 1);) {
      seen |= 1ULL << t;
      m |= 1ULL << t;
      ++len;
      t = ((t % g.lx + dx) % g.lx) + ((t / g.lx + dy) % g.ly) * g.lx;
    }
    cyc.push_back(m);
    clen = len;  // every cycle of a translation has the same length
  }
  if (n % clen) return 0;
  const int k = n / clen, nc = static_cast<int>(cyc.size());
  int64_t tr = 0;
  std::vector<int> pick(k);
  for (int i = 0; i < k; ++i) pick[i] = i;
  while (true) {
    uint64_t w = 0;
    for (int i = 0; i < k; ++i) w |= cyc[pick[i]];
    int par = 0;
    host_translate(w, dx, dy, g, &par);
    tr += par ? -1 : 1;
    int i = k - 1;
    while (i >= 0 && pick[i] == nc - k + i) --i;
    if (i < 0) break;
    ++pick[i];
    for (int j = i + 1; j < k; ++j) pick[j] = pick[j - 1] + 1;
  }
  return tr;
}

}  // namespace

std::vector<int64_t> block_dims_by_characters(Ctx& c, int n_up, int n_dn) {
  const Geom& g = c.geom;
  std::vector<int64_t> tr(g.n);
  for (int s = 0; s < g.n; ++s)
    tr[s] = fixed_trace(g, n_up, s % g.lx, s / g.lx) * fixed_trace(g, n_dn, s % g.lx, s / g.lx);
  const double kPi = 3.141592653589793238462643383279502884;
  std::vector<int64_t> dims(g.n);
  for (int my = 0; my < g.ly; ++my)
    for (int mx = 0; mx < g.lx; ++mx) {
      double re = 0.0;
      for (int s = 0; s < g.n; ++s)
        if (tr[s])
          re += static_cast<double>(tr[s]) *
                std::cos(2.0 * kPi * (static_cast<double>(mx * (s % g.lx)) / g.lx +
                                      static_cast<double>(my * (s / g.lx)) / g.ly));
      dims[my * g.lx + mx] = static_cast<int64_t>(std::llround(re / g.n));
    }
  return dims;
}

template <typename W>
BlockView<W> make_view(Ctx& c) {
  BlockView<W> v{};
  v.up_info = c.sec.up_info.as<uint64_t>();
  v.ur_bits = c.sec.ur_bits.as<W>();
  v.ur_class = c.sec.ur_class.as<uint16_t>();
  v.aoff = c.blk.aoff.as<int64_t>();
  v.dtab = c.blk.dtab.as<uint64_t>();
  v.row_meta = c.blk.row_meta.as<uint32_t>();
  v.row_dn = c.blk.row_dn.as<W>();
  v.c_dn = c.sec.c_dn;
  v.dim = c.blk.dim;
  v.n_up = c.sec.n_up;
  v.n_dn = c.sec.n_dn;
  std::memcpy(v.phase_re, c.blk.phase_re, sizeof v.phase_re);
  std::memcpy(v.phase_im, c.blk.phase_im, sizeof v.phase_im);
  return v;
}

BlockView<uint32_t> view32(Ctx& c) { return make_view<uint32_t>(c); }
BlockView<uint64_t> view64(Ctx& c) { return make_view<uint64_t>(c); }

template <typename W>
void debug_parents_t(Ctx& c, uint64_t* up, uint64_t* dn, int32_t* deg, double* diag) {
  SectorTables& S = c.sec;
  const int64_t P = S.parents;
  DBuf out;
  out.ensure((sizeof(uint64_t) * 2 + sizeof(int32_t) + sizeof(double)) * std::max<int64_t>(P, 1));
  uint64_t* d_up = out.as<uint64_t>();
  uint64_t* d_dn = d_up + P;
  double* d_diag = reinterpret_cast<double*>(d_dn + P);
  int32_t* d_deg = reinterpret_cast<int32_t*>(d_diag + P);
  const int grid = static_cast<int>(std::min<int64_t>(std::max<int64_t>(S.nur, 1), 65535));
  k_debug_parents<W><<<grid, 256, 0, c.stream>>>(S.nur, S.c_dn, c.geom, S.ur_bits.as<W>(), S.ur_class.as<uint16_t>(),
                                                 S.ur_poff.as<int64_t>(), S.canon.as<int32_t>(), S.d_cidx.as<int32_t>(),
                                                 S.d_stab.as<uint64_t>(), S.dns.as<W>(), d_up, d_dn, d_deg, d_diag);
  FTLM_LAUNCH_CHECK();
  FTLM_CUDA(cudaMemcpyAsync(up, d_up, sizeof(uint64_t) * P, cudaMemcpyDeviceToHost, c.stream));
  FTLM_CUDA(cudaMemcpyAsync(dn, d_dn, sizeof(uint64_t) * P, cudaMemcpyDeviceToHost, c.stream));
  FTLM_CUDA(cudaMemcpyAsync(deg, d_deg, sizeof(int32_t) * P, cudaMemcpyDeviceToHost, c.stream));
  FTLM_CUDA(cudaMemcpyAsync(diag, d_diag, sizeof(double) * P, cudaMemcpyDeviceToHost, c.stream));
  FTLM_CUDA(cudaStreamSynchronize(c.stream));
  out.release();
}

void debug_parents(Ctx& c, uint64_t* up, uint64_t* dn, int32_t* deg, double* diag) {
  if (c.wide) debug_parents_t<uint64_t>(c, up, dn, deg, diag);
  else debug_parents_t<uint32_t>(c, up, dn, deg, diag);
}

template <typename W>
void debug_relations_t(Ctx& c, int32_t* parent, int32_t* shift, int32_t* sign) {
  SectorTables& S = c.sec;
  const int64_t F = S.full_dim;
  DBuf out;
  out.ensure(sizeof(int32_t) * 3 * std::max<int64_t>(F, 1));
  int32_t* dp = out.as<int32_t>();
  k_debug_relations<W><<<blocks_for(F, 128), 128, 0, c.stream>>>(S.c_up, S.c_dn, c.geom, S.ups.as<W>(), S.dns.as<W>(),
                                                                  c.binom.as<uint64_t>(), S.up_info.as<uint64_t>(),
                                                                  S.ur_class.as<uint16_t>(), S.ur_poff.as<int64_t>(),
                                                                  S.d_cidx.as<int32_t>(), dp, dp + F, dp + 2 * F);
  FTLM_LAUNCH_CHECK();
  FTLM_CUDA(cudaMemcpyAsync(parent, dp, sizeof(int32_t) * F, cudaMemcpyDeviceToHost, c.stream));
  FTLM_CUDA(cudaMemcpyAsync(shift, dp + F, sizeof(int32_t) * F, cudaMemcpyDeviceToHost, c.stream));
  FTLM_CUDA(cudaMemcpyAsync(sign, dp + 2 * F, sizeof(int32_t) * F, cudaMemcpyDeviceToHost, c.stream));
  FTLM_CUDA(cudaStreamSynchronize(c.stream));
  out.release();
}

void debug_relations(Ctx& c, int32_t* parent, int32_t* shift, int32_t* sign) {
  if (c.wide) debug_relations_t<uint64_t>(c, parent, shift, sign);
  else debug_relations_t<uint32_t>(c, parent, shift, sign);
}

}  // namespace ftlm
