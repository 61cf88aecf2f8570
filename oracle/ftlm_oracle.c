/* Oracle: CPU restatement of the reference FTLM hot path (TEST INFRASTRUCTURE).
 *
 * Checker only: loaded by tests/, by the smoke check and by bench.py's
 * cpu_baseline/reference legs; never by the product path. Each function
 * restates the reference algorithm (PeizhiMai/FTLM_extended_Hubbard_development
 * src/main.cpp, src/ed_main.cpp) at the cited lines, written independently:
 * the orbit bookkeeping uses canonicalisation plus binary search instead of
 * the reference's hash map, while the floating-point expressions keep the
 * reference's operation order so that results agree to rounding.
 *
 * Pinned against golden vectors dumped from the reference compiled in this
 * container (tests/golden/, generated by tests/golden/make_golden.py).
 */
#include "ftlm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

static const double kPi = 3.141592653589793238462643383279502884;

/* ------------------------------------------------------------------ seeds */

uint64_t fo_mix_u64(uint64_t v) { /* main.cpp:514-519 */
  v += 0x9e3779b97f4a7c15ULL;
  v = (v ^ (v >> 30)) * 0xbf58476d1ce4e5b9ULL;
  v = (v ^ (v >> 27)) * 0x94d049bb133111ebULL;
  return v ^ (v >> 31);
}

uint64_t fo_block_seed(uint64_t seed, int n_up, int n_down, int mx, int my) { /* main.cpp:521-533 */
  uint64_t s = fo_mix_u64(seed);
  s ^= fo_mix_u64((uint64_t)(n_up + 1));
  s ^= fo_mix_u64((uint64_t)(n_down + 17));
  s ^= fo_mix_u64((uint64_t)(mx + 257));
  s ^= fo_mix_u64((uint64_t)(my + 65537));
  return fo_mix_u64(s);
}

/* ------------------------------------------------------------ lattice */

typedef struct lat {
  int lx, ly, n;
  int nb[64][8];      /* neighbour per direction, main.cpp:437-449 */
  int bonds[128][2];  /* sorted unique (+x, +y) bonds, main.cpp:450-458 */
  int nbonds;
} lat;

static int bond_cmp(const void* a, const void* b) {
  const int* x = (const int*)a;
  const int* y = (const int*)b;
  if (x[0] != y[0]) return x[0] < y[0] ? -1 : 1;
  if (x[1] != y[1]) return x[1] < y[1] ? -1 : 1;
  return 0;
}

static void lat_build(lat* L, int lx, int ly) { /* main.cpp:429-460 */
  L->lx = lx;
  L->ly = ly;
  L->n = lx * ly;
  int raw[128][2];
  int nraw = 0;
  for (int y = 0; y < ly; ++y) {
    for (int x = 0; x < lx; ++x) {
      const int s = y * lx + x;
      const int xp = (x + 1) % lx, xm = (x - 1 + lx) % lx;
      const int yp = (y + 1) % ly, ym = (y - 1 + ly) % ly;
      const int d[8] = {y * lx + xp,  y * lx + xm,  yp * lx + x,  ym * lx + x,
                        yp * lx + xp, yp * lx + xm, ym * lx + xp, ym * lx + xm};
      memcpy(L->nb[s], d, sizeof d);
      raw[nraw][0] = s;
      raw[nraw][1] = y * lx + xp;
      ++nraw;
      raw[nraw][0] = s;
      raw[nraw][1] = yp * lx + x;
      ++nraw;
    }
  }
  qsort(raw, (size_t)nraw, sizeof raw[0], bond_cmp);
  L->nbonds = 0;
  for (int i = 0; i < nraw; ++i) {
    if (L->nbonds > 0 && bond_cmp(raw[i], L->bonds[L->nbonds - 1]) == 0) continue;
    L->bonds[L->nbonds][0] = raw[i][0];
    L->bonds[L->nbonds][1] = raw[i][1];
    ++L->nbonds;
  }
}

static double diag_energy(const lat* L, uint64_t up, uint64_t dn, double u, double v) {
  /* main.cpp:486-501 */
  const int doublons = __builtin_popcountll(up & dn);
  int nn = 0;
  for (int b = 0; b < L->nbonds; ++b) {
    const int i = L->bonds[b][0], j = L->bonds[b][1];
    const int ni = (int)((up >> i) & 1ULL) + (int)((dn >> i) & 1ULL);
    const int nj = (int)((up >> j) & 1ULL) + (int)((dn >> j) & 1ULL);
    nn += ni * nj;
  }
  return u * (double)doublons + v * (double)nn;
}

static double jw_sign(uint64_t bits, int from, int to) { /* main.cpp:503-512 */
  const int lo = from < to ? from : to;
  const int hi = from < to ? to : from;
  if (hi - lo <= 1) return 1.0;
  const uint64_t mask = ((1ULL << (uint64_t)(hi - lo - 1)) - 1ULL) << (lo + 1);
  return (__builtin_popcountll(bits & mask) & 1) ? -1.0 : 1.0;
}

uint64_t fo_translate_spin(uint64_t bits, int dx, int dy, int lx, int ly, int* sign) {
  /* main.cpp:579-613: move every occupied site, then the sign is the parity
   * of the inversions of the moved list taken in ascending source order. */
  int moved[64];
  int k = 0;
  const int n = lx * ly;
  for (int s = 0; s < n; ++s) {
    if (!((bits >> s) & 1ULL)) continue;
    moved[k++] = ((s / lx + dy) % ly) * lx + (s % lx + dx) % lx;
  }
  int inv = 0;
  uint64_t out = 0;
  for (int i = 0; i < k; ++i) {
    for (int j = i + 1; j < k; ++j) inv += moved[i] > moved[j];
    out |= 1ULL << moved[i];
  }
  *sign = (inv & 1) ? -1 : 1;
  return out;
}

/* --------------------------------------------------------------- basis */

typedef struct st {
  uint64_t up, dn;
} st;

static int st_lt(st a, st b) { return a.up < b.up || (a.up == b.up && a.dn < b.dn); }
static int st_eq(st a, st b) { return a.up == b.up && a.dn == b.dn; }

static st translate_state(const lat* L, st a, int s, int* sign) { /* main.cpp:615-620 */
  int su, sd;
  st r;
  r.up = fo_translate_spin(a.up, s % L->lx, s / L->lx, L->lx, L->ly, &su);
  r.dn = fo_translate_spin(a.dn, s % L->lx, s / L->lx, L->lx, L->ly, &sd);
  *sign = su * sd;
  return r;
}

/* The representative is the first orbit member met in the reference's
 * (up ascending, down ascending) sweep, i.e. the lexicographic minimum. */
static st canonical(const lat* L, st a) {
  st best = a;
  for (int s = 1; s < L->n; ++s) {
    int sg;
    const st t = translate_state(L, a, s, &sg);
    if (st_lt(t, best)) best = t;
  }
  return best;
}

static int64_t n_choose_k(int n, int k) {
  if (k < 0 || k > n) return 0;
  int64_t r = 1;
  for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
  return r;
}

static uint64_t* combinations(int n, int k, int64_t* count) { /* main.cpp:462-484 */
  *count = n_choose_k(n, k);
  uint64_t* out = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)(*count ? *count : 1));
  if (k == 0) {
    out[0] = 0;
    return out;
  }
  uint64_t x = (1ULL << k) - 1ULL;
  for (int64_t i = 0; i < *count; ++i) {
    out[i] = x;
    const uint64_t low = x & (~x + 1ULL);
    const uint64_t ripple = x + low;
    x = (((ripple ^ x) >> 2) / low) | ripple;
  }
  return out;
}

typedef struct sector {
  lat L;
  fo_model m;
  int n_up, n_dn;
  int64_t full_dim, np;
  st* rep;       /* parents in reference order */
  int32_t* deg;
  double* diag;
} sector;

static void sector_free(sector* S) {
  free(S->rep);
  free(S->deg);
  free(S->diag);
}

static void sector_build(sector* S, const fo_model* m, int n_up, int n_dn) { /* main.cpp:622-675 */
  memset(S, 0, sizeof *S);
  S->m = *m;
  lat_build(&S->L, m->lx, m->ly);
  S->n_up = n_up;
  S->n_dn = n_dn;
  int64_t cu, cd;
  uint64_t* ups = combinations(S->L.n, n_up, &cu);
  uint64_t* dns = combinations(S->L.n, n_dn, &cd);
  S->full_dim = cu * cd;
  S->rep = (st*)malloc(sizeof(st) * (size_t)(S->full_dim ? S->full_dim : 1));
  S->np = 0;
  for (int64_t i = 0; i < cu; ++i) {
    for (int64_t j = 0; j < cd; ++j) {
      const st a = {ups[i], dns[j]};
      if (st_eq(canonical(&S->L, a), a)) S->rep[S->np++] = a;
    }
  }
  S->deg = (int32_t*)malloc(sizeof(int32_t) * (size_t)(S->np ? S->np : 1));
  S->diag = (double*)malloc(sizeof(double) * (size_t)(S->np ? S->np : 1));
  for (int64_t p = 0; p < S->np; ++p) {
    int d = 0;
    for (int s = 0; s < S->L.n; ++s) {
      int sg;
      d += st_eq(translate_state(&S->L, S->rep[p], s, &sg), S->rep[p]);
    }
    S->deg[p] = d;
    S->diag[p] = diag_energy(&S->L, S->rep[p].up, S->rep[p].dn, m->u, m->v);
  }
  free(ups);
  free(dns);
}

static int64_t find_parent(const sector* S, st r) {
  int64_t lo = 0, hi = S->np - 1;
  while (lo <= hi) {
    const int64_t mid = (lo + hi) / 2;
    if (st_eq(S->rep[mid], r)) return mid;
    if (st_lt(S->rep[mid], r)) lo = mid + 1;
    else hi = mid - 1;
  }
  return -1;
}

/* Relation of a state: its parent, the first shift (order dy*lx+dx) that
 * carries the representative onto it and that translation's sign. */
static void relation(const sector* S, st t, int64_t* parent, int* shift, int* sign) {
  const st r = canonical(&S->L, t);
  *parent = find_parent(S, r);
  *shift = 0;
  *sign = 1;
  if (st_eq(r, t)) return;
  for (int s = 1; s < S->L.n; ++s) {
    int sg;
    if (st_eq(translate_state(&S->L, r, s, &sg), t)) {
      *shift = s;
      *sign = sg;
      return;
    }
  }
}

int64_t fo_sector_parents(const fo_model* m, int n_up, int n_down, uint64_t* up, uint64_t* down,
                          int32_t* deg, double* diag, int64_t cap) {
  sector S;
  sector_build(&S, m, n_up, n_down);
  const int64_t np = S.np;
  if (up) {
    if (cap < np) {
      sector_free(&S);
      return -1;
    }
    for (int64_t p = 0; p < np; ++p) {
      up[p] = S.rep[p].up;
      down[p] = S.rep[p].dn;
      deg[p] = S.deg[p];
      diag[p] = S.diag[p];
    }
  }
  sector_free(&S);
  return np;
}

int fo_sector_relations(const fo_model* m, int n_up, int n_down, int32_t* parent, int32_t* shift,
                        int32_t* sign) {
  sector S;
  sector_build(&S, m, n_up, n_down);
  int64_t cu, cd;
  uint64_t* ups = combinations(S.L.n, n_up, &cu);
  uint64_t* dns = combinations(S.L.n, n_down, &cd);
  for (int64_t i = 0; i < cu; ++i) {
    for (int64_t j = 0; j < cd; ++j) {
      int64_t p;
      int sh, sg;
      const st t = {ups[i], dns[j]};
      relation(&S, t, &p, &sh, &sg);
      parent[i * cd + j] = (int32_t)p;
      shift[i * cd + j] = sh;
      sign[i * cd + j] = sg;
    }
  }
  free(ups);
  free(dns);
  sector_free(&S);
  return 0;
}

/* -------------------------------------------------------- momentum block */

typedef struct cplx {
  double re, im;
} cplx;

static cplx cmul(cplx a, cplx b) {
  cplx r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
  return r;
}

static cplx twist(const fo_model* m, int dir) { /* main.cpp:544-577 */
  const double thx = 2.0 * kPi * m->phix / (double)m->lx;
  const double thy = 2.0 * kPi * m->phiy / (double)m->ly;
  const double ang[8] = {thx, -thx, thy, -thy, thx + thy, -thx + thy, thx - thy, -thx - thy};
  cplx r = {cos(ang[dir]), sin(ang[dir])};
  return r;
}

int fo_block_csr(const fo_model* m, int n_up, int n_down, int mx, int my, int64_t* dim_out,
                 int64_t* nnz_out, double* diag, int32_t* row_ptr, int32_t* col, double* val) {
  /* main.cpp:723-805 with the hop list of main.cpp:677-718 */
  sector S;
  sector_build(&S, m, n_up, n_down);
  const lat* L = &S.L;
  cplx* phase = (cplx*)malloc(sizeof(cplx) * (size_t)L->n);
  for (int s = 0; s < L->n; ++s) {
    const int dx = s % L->lx, dy = s / L->lx;
    const double arg =
        2.0 * kPi * ((double)(mx * dx) / (double)L->lx + (double)(my * dy) / (double)L->ly);
    phase[s].re = cos(arg);
    phase[s].im = sin(arg);
  }
  double* dnf = (double*)malloc(sizeof(double) * (size_t)(S.np ? S.np : 1));
  int64_t* act = (int64_t*)malloc(sizeof(int64_t) * (size_t)(S.np ? S.np : 1));
  int64_t dim = 0;
  for (int64_t p = 0; p < S.np; ++p) {
    cplx sum = {0.0, 0.0};
    for (int s = 0; s < L->n; ++s) {
      int sg;
      if (st_eq(translate_state(L, S.rep[p], s, &sg), S.rep[p])) {
        sum.re += (double)sg * phase[s].re;
        sum.im += (double)sg * phase[s].im;
      }
    }
    dnf[p] = hypot(sum.re, sum.im) / sqrt((double)S.deg[p]);
    act[p] = dnf[p] > 1e-12 ? dim++ : -1;
  }
  const double hop_t[8] = {m->tx, m->tx, m->ty, m->ty, m->tp, m->tp, m->tp, m->tp};
  int64_t nnz = 0;
  if (row_ptr) row_ptr[0] = 0;
  for (int64_t p = 0; p < S.np; ++p) {
    if (act[p] < 0) continue;
    if (diag) diag[act[p]] = S.diag[p];
    for (int spin = 0; spin < 2; ++spin) {
      const uint64_t bits = spin == 0 ? S.rep[p].up : S.rep[p].dn;
      for (int from = 0; from < L->n; ++from) {
        if (!((bits >> from) & 1ULL)) continue;
        for (int dir = 0; dir < 8; ++dir) {
          const int to = L->nb[from][dir];
          if ((bits >> to) & 1ULL) continue;
          const double pref = -hop_t[dir] * jw_sign(bits, from, to);
          const cplx tw = twist(m, dir);
          const cplx amp = {pref * tw.re, pref * tw.im};
          const uint64_t moved = bits ^ (1ULL << from) ^ (1ULL << to);
          st t = S.rep[p];
          if (spin == 0) t.up = moved;
          else t.dn = moved;
          int64_t tp;
          int sh, sg;
          relation(&S, t, &tp, &sh, &sg);
          if (act[tp] < 0) continue;
          if (col) {
            const cplx a1 = {amp.re * (double)sg, amp.im * (double)sg};
            const cplx a2 = cmul(a1, phase[sh]);
            const double ratio = dnf[tp] / dnf[p];
            col[nnz] = (int32_t)act[tp];
            val[2 * nnz] = a2.re * ratio;
            val[2 * nnz + 1] = a2.im * ratio;
          }
          ++nnz;
        }
      }
    }
    if (row_ptr) row_ptr[act[p] + 1] = (int32_t)nnz;
  }
  *dim_out = dim;
  *nnz_out = nnz;
  free(phase);
  free(dnf);
  free(act);
  sector_free(&S);
  return 0;
}

void fo_csr_apply(int64_t dim, const double* diag, const int32_t* row_ptr, const int32_t* col,
                  const double* val, const double* in, double* out) { /* main.cpp:833-845 */
  for (int64_t i = 0; i < dim; ++i) {
    double re = 0.0 + diag[i] * in[2 * i];
    double im = 0.0 + diag[i] * in[2 * i + 1];
    for (int32_t e = row_ptr[i]; e < row_ptr[i + 1]; ++e) {
      const double vr = val[2 * e], vi = val[2 * e + 1];
      const double xr = in[2 * col[e]], xi = in[2 * col[e] + 1];
      re += vr * xr - vi * xi;
      im += vr * xi + vi * xr;
    }
    out[2 * i] = re;
    out[2 * i + 1] = im;
  }
}

/* ------------------------------------------------------- start vectors */

/* mt19937_64 (Matsumoto & Nishimura; the std::mt19937_64 parameter set). */
typedef struct mt64 {
  uint64_t x[312];
  int i;
} mt64;

static void mt64_seed(mt64* g, uint64_t s) {
  g->x[0] = s;
  for (int i = 1; i < 312; ++i)
    g->x[i] = 6364136223846793005ULL * (g->x[i - 1] ^ (g->x[i - 1] >> 62)) + (uint64_t)i;
  g->i = 312;
}

static uint64_t mt64_next(mt64* g) {
  if (g->i >= 312) {
    for (int k = 0; k < 312; ++k) {
      const uint64_t y = (g->x[k] & 0xFFFFFFFF80000000ULL) | (g->x[(k + 1) % 312] & 0x7FFFFFFFULL);
      uint64_t v = y >> 1;
      if (y & 1ULL) v ^= 0xB5026F5AA96619E9ULL;
      g->x[k] = g->x[(k + 156) % 312] ^ v;
    }
    g->i = 0;
  }
  uint64_t z = g->x[g->i++];
  z ^= (z >> 29) & 0x5555555555555555ULL;
  z ^= (z << 17) & 0x71D67FFFEDA60000ULL;
  z ^= (z << 37) & 0xFFF7EEE000000000ULL;
  z ^= z >> 43;
  return z;
}

/* Uniform [0,1) double from one 64-bit draw, as libstdc++'s
 * generate_canonical<double, 53> does for a 64-bit engine. */
static double unit_draw(mt64* g) {
  const double r = (double)mt64_next(g) / 18446744073709551616.0;
  return r >= 1.0 ? nextafter(1.0, 0.0) : r;
}

/* Marsaglia polar method with one cached value (libstdc++ normal_distribution). */
typedef struct polar {
  double saved;
  int have;
} polar;

static double polar_next(polar* p, mt64* g) {
  if (p->have) {
    p->have = 0;
    return p->saved;
  }
  double x, y, r2;
  do {
    x = 2.0 * unit_draw(g) - 1.0;
    y = 2.0 * unit_draw(g) - 1.0;
    r2 = x * x + y * y;
  } while (r2 > 1.0 || r2 == 0.0);
  const double mult = sqrt(-2.0 * log(r2) / r2);
  p->saved = x * mult;
  p->have = 1;
  return y * mult;
}

void fo_start_vector(uint64_t block_seed, int sample, int64_t dim, double* out) {
  /* main.cpp:1015-1025; the second draw of each pair is the real part. */
  mt64 g;
  polar p = {0.0, 0};
  mt64_seed(&g, fo_mix_u64(block_seed ^ (uint64_t)sample));
  double norm2 = 0.0;
  for (int64_t i = 0; i < dim; ++i) {
    const double first = polar_next(&p, &g);
    const double second = polar_next(&p, &g);
    out[2 * i] = second;
    out[2 * i + 1] = first;
    norm2 += second * second + first * first;
  }
  const double nrm = sqrt(norm2);
  for (int64_t i = 0; i < 2 * dim; ++i) out[i] /= nrm;
}

/* ------------------------------------------------------------- Lanczos */

int fo_lanczos(int64_t dim, const double* diag, const int32_t* row_ptr, const int32_t* col,
               const double* val, const double* start, int kmax, double* alpha, double* beta) {
  /* main.cpp:1033-1057: no reorthogonalisation, stop at b < 1e-12 or kmax. */
  double* q = (double*)malloc(sizeof(double) * 2 * (size_t)dim);
  double* qp = (double*)calloc(2 * (size_t)dim, sizeof(double));
  double* hq = (double*)malloc(sizeof(double) * 2 * (size_t)dim);
  memcpy(q, start, sizeof(double) * 2 * (size_t)dim);
  double bprev = 0.0;
  int taken = 0;
  for (int j = 0; j < kmax; ++j) {
    fo_csr_apply(dim, diag, row_ptr, col, val, q, hq);
    double a = 0.0;
    for (int64_t i = 0; i < dim; ++i) a += q[2 * i] * hq[2 * i] + q[2 * i + 1] * hq[2 * i + 1];
    double n2 = 0.0;
    for (int64_t i = 0; i < 2 * dim; ++i) {
      hq[i] = hq[i] - a * q[i] - bprev * qp[i];
    }
    for (int64_t i = 0; i < dim; ++i) n2 += hq[2 * i] * hq[2 * i] + hq[2 * i + 1] * hq[2 * i + 1];
    alpha[j] = a;
    const double b = sqrt(n2);
    ++taken;
    if (b < 1e-12 || j + 1 == kmax) break;
    beta[j] = b;
    double* t = qp;
    qp = q;
    q = hq;
    hq = t;
    for (int64_t i = 0; i < 2 * dim; ++i) q[i] /= b;
    bprev = b;
  }
  free(q);
  free(qp);
  free(hq);
  return taken;
}

void fo_tridiag_jacobi(int n, const double* alpha, const double* beta, double* evals,
                       double* v1sq) {
  /* main.cpp:913-994 (classical Jacobi, largest pivot, tol 1e-12, at most
   * 50 n^2 rotations) followed by the ascending sort of main.cpp:1076-1094. */
  if (n <= 0) return;
  if (n == 1) {
    evals[0] = alpha[0];
    v1sq[0] = 1.0;
    return;
  }
  double* a = (double*)calloc((size_t)n * (size_t)n, sizeof(double));
  double* v = (double*)calloc((size_t)n * (size_t)n, sizeof(double));
#define A(i, j) a[(size_t)(i) * (size_t)n + (size_t)(j)]
#define V(i, j) v[(size_t)(i) * (size_t)n + (size_t)(j)]
  for (int i = 0; i < n; ++i) {
    A(i, i) = alpha[i];
    V(i, i) = 1.0;
    if (i + 1 < n) {
      A(i, i + 1) = beta[i];
      A(i + 1, i) = beta[i];
    }
  }
  for (long it = 0; it < 50L * n * n; ++it) {
    int p = 0, q = 1;
    double best = 0.0;
    for (int i = 0; i < n; ++i)
      for (int j = i + 1; j < n; ++j)
        if (fabs(A(i, j)) > best) {
          best = fabs(A(i, j));
          p = i;
          q = j;
        }
    if (best < 1e-12) break;
    const double app = A(p, p), aqq = A(q, q), apq = A(p, q);
    const double tau = (aqq - app) / (2.0 * apq);
    const double t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
    const double c = 1.0 / sqrt(1.0 + t * t);
    const double s = t * c;
    for (int k = 0; k < n; ++k) {
      if (k == p || k == q) continue;
      const double kp = A(k, p), kq = A(k, q);
      A(k, p) = c * kp - s * kq;
      A(p, k) = A(k, p);
      A(k, q) = s * kp + c * kq;
      A(q, k) = A(k, q);
    }
    A(p, p) = c * c * app - 2.0 * s * c * apq + s * s * aqq;
    A(q, q) = s * s * app + 2.0 * s * c * apq + c * c * aqq;
    A(p, q) = 0.0;
    A(q, p) = 0.0;
    for (int k = 0; k < n; ++k) {
      const double kp = V(k, p), kq = V(k, q);
      V(k, p) = c * kp - s * kq;
      V(k, q) = s * kp + c * kq;
    }
  }
  /* insertion sort of indices by eigenvalue (stable) */
  int* ord = (int*)malloc(sizeof(int) * (size_t)n);
  for (int i = 0; i < n; ++i) ord[i] = i;
  for (int i = 1; i < n; ++i) {
    const int k = ord[i];
    int j = i - 1;
    while (j >= 0 && A(ord[j], ord[j]) > A(k, k)) {
      ord[j + 1] = ord[j];
      --j;
    }
    ord[j + 1] = k;
  }
  for (int i = 0; i < n; ++i) {
    evals[i] = A(ord[i], ord[i]);
    v1sq[i] = V(0, ord[i]) * V(0, ord[i]);
  }
#undef A
#undef V
  free(ord);
  free(a);
  free(v);
}

/* ---------------------------------------------------------- exact block */

extern void zheev_(char* jobz, char* uplo, int* n, double* a, int* lda, double* w, double* work,
                   int* lwork, double* rwork, int* info);

int fo_block_exact(int64_t dim, const double* diag, const int32_t* row_ptr, const int32_t* col,
                   const double* val, double* evals) { /* main.cpp:847-911 */
  int n = (int)dim;
  if (n == 0) return 0;
  if (n == 1) {
    double e = diag[0];
    for (int32_t k = row_ptr[0]; k < row_ptr[1]; ++k)
      if (col[k] == 0) e += val[2 * k];
    evals[0] = e;
    return 0;
  }
  double* a = (double*)calloc(2 * (size_t)n * (size_t)n, sizeof(double));
#define RE(i, j) a[2 * ((size_t)(i) + (size_t)(j) * (size_t)n)]
#define IM(i, j) a[2 * ((size_t)(i) + (size_t)(j) * (size_t)n) + 1]
  for (int i = 0; i < n; ++i) {
    RE(i, i) = diag[i];
    for (int32_t k = row_ptr[i]; k < row_ptr[i + 1]; ++k) {
      RE(i, col[k]) += val[2 * k];
      IM(i, col[k]) += val[2 * k + 1];
    }
  }
  for (int j = 0; j < n; ++j) {
    IM(j, j) = 0.0;
    for (int i = 0; i < j; ++i) {
      const double re = 0.5 * (RE(i, j) + RE(j, i));
      const double im = 0.5 * (IM(i, j) - IM(j, i));
      RE(i, j) = re;
      IM(i, j) = im;
      RE(j, i) = re;
      IM(j, i) = -im;
    }
  }
#undef RE
#undef IM
  char jobz = 'N', uplo = 'U';
  int lda = n, lwork = -1, info = 0;
  double query[2] = {0.0, 0.0};
  double* rwork = (double*)calloc((size_t)(3 * n > 1 ? 3 * n - 2 : 1), sizeof(double));
  zheev_(&jobz, &uplo, &n, a, &lda, evals, query, &lwork, rwork, &info);
  if (info == 0) {
    lwork = (int)query[0] > 1 ? (int)query[0] : 1;
    double* work = (double*)calloc(2 * (size_t)lwork, sizeof(double));
    zheev_(&jobz, &uplo, &n, a, &lda, evals, work, &lwork, rwork, &info);
    free(work);
  }
  free(rwork);
  free(a);
  return info;
}

/* --------------------------------------------------------------- thermo */

void fo_thermo_accumulate(int64_t n, const double* evals, const double* weights, double prefactor,
                          int particles, double beta, int nmu, const double* mu, double* emin,
                          double* z, double* nsum, double* n2sum) { /* main.cpp:1172-1219 */
  const double pc = (double)particles;
  for (int k = 0; k < nmu; ++k) {
    double bmin = INFINITY;
    for (int64_t i = 0; i < n; ++i) {
      const double sh = evals[i] - mu[k] * pc;
      if (sh < bmin) bmin = sh;
    }
    if (!isfinite(bmin)) continue;
    if (!isfinite(emin[k])) {
      emin[k] = bmin;
    } else if (bmin < emin[k]) {
      const double scale = exp(-beta * (emin[k] - bmin));
      z[k] *= scale;
      nsum[k] *= scale;
      n2sum[k] *= scale;
      emin[k] = bmin;
    }
    for (int64_t i = 0; i < n; ++i) {
      const double sh = evals[i] - mu[k] * pc - emin[k];
      const double w = prefactor * (weights ? weights[i] : 1.0) * exp(-beta * sh);
      z[k] += w;
      nsum[k] += pc * w;
      n2sum[k] += pc * pc * w;
    }
  }
}

/* ---------------------------------------------------------------- curve */

int fo_run_curve(const fo_model* m, int samples, int steps, uint64_t threshold, uint64_t seed,
                 uint64_t max_sector_dim, int ed, int nbeta, const double* betas, int nmu,
                 const double* mu, double* emin, double* z, double* nsum, double* n2sum) {
  const int nsites = m->lx * m->ly;
  for (int nu = 0; nu <= nsites; ++nu) {
    for (int nd = 0; nd <= nsites; ++nd) {
      const int64_t full = n_choose_k(nsites, nu) * n_choose_k(nsites, nd);
      if (full == 0) continue;
      if ((uint64_t)full > max_sector_dim) return -1;
      for (int my = 0; my < m->ly; ++my) {
        for (int mx = 0; mx < m->lx; ++mx) {
          int64_t dim, nnz;
          fo_block_csr(m, nu, nd, mx, my, &dim, &nnz, NULL, NULL, NULL, NULL);
          if (dim == 0) continue;
          double* diag = (double*)malloc(sizeof(double) * (size_t)dim);
          int32_t* rp = (int32_t*)malloc(sizeof(int32_t) * (size_t)(dim + 1));
          int32_t* col = (int32_t*)malloc(sizeof(int32_t) * (size_t)(nnz ? nnz : 1));
          double* val = (double*)malloc(sizeof(double) * 2 * (size_t)(nnz ? nnz : 1));
          fo_block_csr(m, nu, nd, mx, my, &dim, &nnz, diag, rp, col, val);
          const int exact = ed || (uint64_t)dim <= threshold;
          double* ev;
          double* w = NULL;
          int64_t count;
          double pref;
          if (exact) {
            ev = (double*)malloc(sizeof(double) * (size_t)dim);
            fo_block_exact(dim, diag, rp, col, val, ev);
            count = dim;
            pref = 1.0;
          } else {
            const int kdim = steps < dim ? steps : (int)dim;
            ev = (double*)malloc(sizeof(double) * (size_t)samples * (size_t)kdim);
            w = (double*)malloc(sizeof(double) * (size_t)samples * (size_t)kdim);
            int* taken = (int*)malloc(sizeof(int) * (size_t)samples);
            const uint64_t bseed = fo_block_seed(seed, nu, nd, mx, my);
#pragma omp parallel for schedule(static)
            for (int s = 0; s < samples; ++s) {
              double* start = (double*)malloc(sizeof(double) * 2 * (size_t)dim);
              double* al = (double*)calloc((size_t)kdim, sizeof(double));
              double* be = (double*)calloc((size_t)kdim, sizeof(double));
              fo_start_vector(bseed, s, dim, start);
              taken[s] = fo_lanczos(dim, diag, rp, col, val, start, kdim, al, be);
              fo_tridiag_jacobi(taken[s], al, be, ev + (size_t)s * kdim, w + (size_t)s * kdim);
              for (int j = 0; j < taken[s]; ++j) w[(size_t)s * kdim + j] /= (double)samples;
              free(start);
              free(al);
              free(be);
            }
            /* concatenate samples in order (main.cpp:1097-1110) */
            count = 0;
            for (int s = 0; s < samples; ++s) {
              for (int j = 0; j < taken[s]; ++j) {
                ev[count] = ev[(size_t)s * kdim + j];
                w[count] = w[(size_t)s * kdim + j];
                ++count;
              }
            }
            free(taken);
            pref = (double)dim;
          }
          for (int b = 0; b < nbeta; ++b) {
            fo_thermo_accumulate(count, ev, w, pref, nu + nd, betas[b], nmu, mu, emin + b * nmu,
                                 z + b * nmu, nsum + b * nmu, n2sum + b * nmu);
          }
          free(ev);
          free(w);
          free(diag);
          free(rp);
          free(col);
          free(val);
        }
      }
    }
  }
  return 0;
}
