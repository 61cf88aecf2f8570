// Internal host-side structures of the B200 FTLM engine (not part of the ABI).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/ftlm_gpu.h"
#include "ftlm_device.cuh"

namespace ftlm {

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define FTLM_CUDA(call)                                                                  \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess)                                                               \
      throw ::ftlm::Error(FTLM_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

#define FTLM_LAUNCH_CHECK() FTLM_CUDA(cudaGetLastError())

// Grow-only device buffer owned by a context.
struct DBuf {
  void* p = nullptr;
  size_t cap = 0;
  void ensure(size_t bytes) {
    if (bytes <= cap) return;
    if (p) FTLM_CUDA(cudaFree(p));
    p = nullptr;
    cap = 0;
    if (bytes == 0) return;
    FTLM_CUDA(cudaMalloc(&p, bytes));
    cap = bytes;
  }
  // Grows (by at least half) keeping the first `cap` bytes; stream-ordered copy.
  void ensure_keep(size_t bytes, cudaStream_t stream) {
    if (bytes <= cap) return;
    const size_t want = std::max(bytes, cap + cap / 2);
    void* q = nullptr;
    FTLM_CUDA(cudaMalloc(&q, want));
    if (p) {
      FTLM_CUDA(cudaMemcpyAsync(q, p, cap, cudaMemcpyDeviceToDevice, stream));
      FTLM_CUDA(cudaStreamSynchronize(stream));
      FTLM_CUDA(cudaFree(p));
    }
    p = q;
    cap = want;
  }
  template <typename T>
  T* as() const { return static_cast<T*>(p); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
  }
};

// Translation-orbit tables of one (N_up, N_down) sector.
//
// Representatives are the lexicographic minima of (up, down) orbits
// (main.cpp:643-675 keeps the first member met in an (up, down) ascending
// sweep). Hence the representative's up word is the minimum of its up
// orbit ("up representative" ur), and its down word is minimal among the
// images of the down word under the stabiliser H of ur. Up representatives
// with equal (H, sign character of H on the up word) form a class; each
// non-trivial class owns a table over all down words. Parents are ordered
// by (ur, canonical down), which is the reference's parent order.
struct SectorTables {
  int n_up = -1, n_dn = -1;
  int64_t c_up = 0, c_dn = 0, full_dim = 0, parents = 0;
  int64_t nur = 0;      // number of up representatives
  int nclass = 0;       // classes; class 0 is the trivial stabiliser
  std::vector<uint64_t> cls_stab, cls_sig;   // per class: H mask, sign mask
  std::vector<int64_t> cls_ncanon;           // canonical downs per class
  std::vector<uint16_t> h_ur_class;          // host copy of ur -> class
  DBuf ups, dns;         // W[c_up], W[c_dn] bit words in ascending order
  DBuf up_info;          // uint64[c_up]
  DBuf ur_bits;          // W[nur]
  DBuf ur_class;         // uint16[nur]
  DBuf ur_poff;          // int64[nur+1] parent offsets
  // per non-trivial class c (index c-1), over all down ranks
  DBuf d_star;           // uint32[(nclass-1)*c_dn] rank of the canonical image
  DBuf d_hs;             // uint16[(nclass-1)*c_dn] h | sign<<8 (T_h d* = d)
  DBuf d_stab, d_chi;    // uint64[(nclass-1)*c_dn] for canonical words
  DBuf d_cidx;           // int32[(nclass-1)*c_dn] canonical index (scan)
  DBuf canon;            // int32[(nclass-1)*c_dn] 1 for canonical words
  DBuf tmp_a, tmp_b, tmp_c, tmp_d, tmp_e;  // build scratch
};

// Tables of one momentum block (mx, my) of the prepared sector.
struct BlockTables {
  int mx = -1, my = -1;
  int64_t dim = 0;
  std::vector<int64_t> cls_nact;  // active canonical downs per class
  DBuf act;       // int32[(nclass-1)*c_dn] active index of canonical words (-1)
  DBuf act_list;  // uint32[(nclass-1)*c_dn] ranks of active canonical words
  DBuf aoff;      // int64[nur+1] active row offsets
  DBuf dtab;      // uint64[(nclass-1)*c_dn] packed lookup entries
  DBuf row_meta;  // uint32[dim]: ur | (deg-1)<<26
  DBuf row_dn;    // W[dim]
  double phase_re[64], phase_im[64];
};

// Everything the H*V / CSR kernels need about one block.
template <typename W>
struct BlockView {
  const uint64_t* up_info;
  const W* ur_bits;
  const uint16_t* ur_class;
  const int64_t* aoff;
  const uint64_t* dtab;
  const uint32_t* row_meta;
  const W* row_dn;
  int64_t c_dn;
  int64_t dim;
  int n_up, n_dn;
  double phase_re[64], phase_im[64];
};

// Device-resident spectrum of one block.
struct Spectrum {
  int64_t ev_off = 0;  // eigenvalues at spectra[ev_off .. ev_off+count)
  int64_t w_off = -1;  // weights at spectra[w_off ..), -1 for exact blocks
  int64_t count = 0;   // number of eigenvalues
  bool exact = false;
  double prefactor = 1.0;
  int particles = 0;
  int64_t dim = 0;
  int pending = -1;       // exact block queued for a deferred solve: index into Ctx::defer_items
  int pending_ritz = -1;  // small FTLM block whose Ritz stage is deferred: index into Ctx::defer_ritz
};

// An exact block whose dense matrix waits in the deferred pool.
struct DeferItem {
  int n_up, n_dn, mx, my;
  int64_t n, aoff;   // dimension, offset (complex entries) of its matrix in defer_arena
  int64_t sec_gen;   // sector generation it was assembled in
};

// A small FTLM block whose Lanczos coefficients wait in the deferred pool.
struct DeferRitz {
  int n_up, n_dn, mx, my;
  int R, ld, K;
  int64_t alpha_off, beta_off;  // doubles into defer_ab ([K][ld] each)
  int64_t steps_off;            // int32 into defer_st ([R])
  int64_t dim, sec_gen;
};

// A queued accumulation: an exact (ritz = false) or FTLM block of the pool.
struct DeferAcc {
  bool ritz;
  int idx;
};

struct Profile {
  double hv_ms = 0.0;       // summed CUDA-event time of H*V launches
  int64_t hv_launches = 0;
  double hv_bytes = 0.0;    // algorithmic bytes of those launches
  double update_ms = 0.0;
  int64_t update_launches = 0;
  double eig_ms = 0.0;
  double dense_ms = 0.0;
  double thermo_ms = 0.0;
  double sector_ms = 0.0;
  double block_ms = 0.0;
  int64_t kernel_launches = 0;
  int64_t h2d_bytes = 0, d2h_bytes = 0;
  int hv_variant = -1;  // H*V kernel variant of the last launch
  int tune_runs = 0;    // autotuner measurements made by this context
  double small_ms = 0.0;     // device time of small-block Lanczos launches
  int64_t small_tasks = 0;   // (block, random vector) pairs they ran
  double hv_hops = 0.0;      // nonzero hop x vector products of the timed H*V launches
  double hv_min_bytes = 0.0; // their compulsory bytes D * (2 nv s + 8) per launch
  int hv_source = -1;        // operator source of the last sweep (kSrcFly / kSrcList / kSrcSplit)
};

// Momentum phases e^{i k.s} of a block, by translation index s.
struct FlipPhase {
  double re[64], im[64];
};

// Largest block dimension the small-block Lanczos launch takes (three FP64
// complex vectors of this length fill 192 KB of shared memory).
constexpr int64_t kSmallMaxDim = 4096;

struct Ctx {
  ftlm_model model{};
  ftlm_run_opts opts{};
  Geom geom{};
  bool wide = false;  // 64-bit spin words (more than 32 sites)
  int hv_forced = -1; // H*V kernel variant forced by FTLM_HV_VARIANT (-1: autotune)
  bool hv_retune = false;  // FTLM_HV_RETUNE=1: tune once per context, ignoring the process-wide choices
  std::map<uint64_t, int> tuned_local;  // variants chosen by this context's tuner runs
  int hv_mode = -1;   // H*V operator source: -1 auto, 0 on-the-fly lookups, 1 cached hop list,
                      // 2 split-spin segment sweeps (FTLM_HV_MODE=fly|list|split)
  bool hl_active = false;  // H*V kernels read the cached hop list of the prepared block
  bool split_active = false;  // H*V runs as the two segment sweeps of split.cu
  std::unique_ptr<Ctx> flipped;  // tables of sector (N_down, N_up) when N_up != N_down
  DBuf flip_map;      // uint64 per row: flipped row | shift << 32 | sign << 38 (+ an error word)
  int flip_for[4] = {-1, -1, -1, -1};  // (n_up, n_dn, mx, my) the flip map belongs to
  int64_t flip_gen = -1, sec_gen = 0;  // sector generation of the flip map / of the tables
  DBuf vec_xd, vec_yd;  // Lanczos vector and H*V output in the spin-flipped row order
  bool seg_dynamic = true;  // segment sweeps take rows from a shared counter (FTLM_SEG_ROWS=stride: grid-stride)
  DBuf seg_counter;         // the row counters of the two sweeps
  bool split_stencil = true;  // segment sweeps read the class stencils (FTLM_SPLIT_OP=fly: on-the-fly lookups)
  bool stn_rows = true;       // narrow stencil sweeps run 8 lanes per row (FTLM_STN_ROWS=0: warp per row)
  // class stencils of this context's prepared block (split.cu)
  bool stn_ok = false;
  int64_t stn_for[3] = {-1, -1, -1};  // (sector generation, mx, my) they belong to
  DBuf stn_crb, stn_rp, stn_rp32, stn_ent, stn_cnt;
  bool hv_rows = true;  // narrow sweeps on the hop list: 8 lanes per row (FTLM_HV_ROWS=0: warp per row)
  bool small_blocks = true;  // batched FTLM runs blocks <= kSmallMaxDim in one launch (FTLM_SMALL_BLOCKS=0: off)
  int64_t hl_nnz = 0;
  DBuf hl_ptr, hl_ent;     // hop list: int64 row pointers, packed uint64 entries
  int device = 0;
  int sm_count = 148;
  cudaStream_t stream = nullptr;
  std::string last_error;
  DBuf binom;         // uint64 [65*65]
  DBuf binom32;       // uint32 [65*65]
  SectorTables sec;
  std::vector<int64_t> block_dims;  // dimension of every k-block of the prepared sector (k = my*lx + mx)
  BlockTables blk;
  // Lanczos work space
  DBuf vec_a, vec_b, vec_h, partial, lz_alpha, lz_beta, lz_scale, lz_state, host_start;
  DBuf ritz_tmp, ritz_out, ritz_meta, scan_tmp;
  // exact batch
  DBuf dense_arena, dense_meta, dense_out;
  // deferred block spectra (ftlm_spectra_defer): dense matrices of exact
  // blocks and Lanczos coefficients of small FTLM blocks of any number of
  // sectors, solved together by flush_deferred, then the queued accumulations
  bool spectra_defer = false;
  DBuf defer_arena, defer_ev, defer_work;
  int64_t defer_asz = 0;
  std::vector<DeferItem> defer_items;
  DBuf defer_ab, defer_st;
  int64_t defer_ab_used = 0, defer_st_used = 0;
  std::vector<DeferRitz> defer_ritz;
  std::vector<DeferAcc> defer_acc;
  // small-block FTLM batch: CSR arenas, task list, per-vector step counts
  DBuf sb_rp, sb_col, sb_val, sb_diag, sb_meta, sb_steps;
  // spectra of the current sector's blocks (device arena)
  DBuf spectra;
  int64_t spectra_used = 0;
  std::map<std::pair<int, int>, Spectrum> spec;
  // thermo
  int nbeta = 0, nmu = 0;
  DBuf th_beta, th_mu, th_state;  // state: [4][nbeta][nmu] emin, z, n, n2
  // instrumentation
  bool timing = false;
  Profile prof;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // last Lanczos run (debug readback)
  int last_kdim = 0, last_nv = 0;
};

// ---- launchers implemented in the .cu files
void sector_prepare(Ctx& c, int n_up, int n_dn);
void block_prepare(Ctx& c, int mx, int my);
// Dimensions of every block k = my*lx + mx of sector (n_up, n_dn) on the host,
// by character counting: (1/N) sum_s e^{-ik.s} tr_up(T_s) tr_dn(T_s).
std::vector<int64_t> block_dims_by_characters(Ctx& c, int n_up, int n_dn);
void debug_parents(Ctx& c, uint64_t* up, uint64_t* dn, int32_t* deg, double* diag);
void debug_relations(Ctx& c, int32_t* parent, int32_t* shift, int32_t* sign);
void block_csr(Ctx& c, std::vector<int32_t>& row_ptr, std::vector<int32_t>& col,
               std::vector<double>& val, std::vector<double>& diag);
// Device CSR of the prepared block (reference entry order); returns nnz.
int64_t block_csr_device(Ctx& c, DBuf& row_ptr, DBuf& col, DBuf& val, DBuf& diag);
// Dense column-major matrix of the prepared block added into A (zeroed by the
// caller), entries summed in the CSR's order; no host synchronisation.
void block_dense_device(Ctx& c, double2* A);
// H*V of the prepared block on device arrays [dim][nv] complex (FP64 or FP32).
// partial_dev[grid][nv] receives each CTA's fixed-point sum of Re<s x, y>.
void hv_apply(Ctx& c, const void* in, void* out, int nv, bool fp32, const double* scale_dev,
              fx128* partial_dev, int nblocks_hint);
int hv_grid(Ctx& c, int nv, bool fp32);
// Chooses the operator source of sweeps of nv vectors over the prepared
// block (FTLM_HV_MODE or the automatic rule): on-the-fly lookups, the cached
// hop list (few vectors per sweep), or the split-spin segment sweeps (large
// blocks); builds what it needs and sets c.hl_active / c.split_active. The
// guard clears them again.
enum { kSrcFly = 0, kSrcList = 1, kSrcSplit = 2 };
constexpr int64_t kSplitMinDim = int64_t(1) << 15;
int hv_select_source(Ctx& c, int nv, bool fp32);
struct HvSourceGuard {
  Ctx& c;
  ~HvSourceGuard() {
    c.hl_active = false;
    c.split_active = false;
  }
};
// Autotuner cache (hv.cu): variant chosen for a key by this context or the process.
int hv_size_class(int64_t dim);
bool hv_tuned_lookup(Ctx& c, uint64_t key, int& var);
void hv_tuned_store(Ctx& c, uint64_t key, int var);

// ---- split-spin H*V (split.cu)
// Prepares the spin-flipped tables and the flip map of the prepared block and
// the two flipped-order arrays for sweeps of nv vectors; false when they do
// not fit in device memory.
bool split_prepare(Ctx& c, int nv, bool fp32);
// y = M x for x given in both row orders: out (this block's order, diagonal
// included) and out_d (flipped order) such that M x = out + S^T out_d.
// partial receives 2 x grid rows of fixed-point Re<s x, y> sums; returns
// that row count.
int hv_apply_split(Ctx& c, const void* in, const void* in_d, void* out, void* out_d, int nv, bool fp32,
                   const double* scale, fx128* partial);
int hv_split_max_grid(const Ctx& c);
// x_D[p(q)] = conj(f_q) x[q];  y[q] += f_q y_D[p(q)].
void flip_scatter(Ctx& c, const void* x, void* xd, int nv, bool fp32);
void flip_gather_add(Ctx& c, void* y, const void* yd, int nv, bool fp32);
FlipPhase flip_phase(const Ctx& c);
BlockView<uint32_t> view32(Ctx& c);
BlockView<uint64_t> view64(Ctx& c);

// Lanczos over the prepared block; results stored as a Spectrum.
void run_ftlm_block(Ctx& c, int n_up, int n_dn, int mx, int my, Spectrum& out,
                    const double* host_start /* [R][dim] complex or null */,
                    std::vector<double>* alpha_out, std::vector<double>* beta_out,
                    std::vector<int32_t>* steps_out);
// FTLM spectra of several small blocks (dim <= kSmallMaxDim) of the prepared
// sector in one persistent launch; stored like run_ftlm_block's.
void run_small_ftlm_blocks(Ctx& c, const std::vector<std::pair<int, int>>& blocks);
// Ritz values and weights of R Lanczos runs (alpha/beta [sweep][K][ld],
// nvmax vectors per sweep, steps[R] on the device) into the spectra arena.
void ritz_stage(Ctx& c, int R, int nvmax, int ld, int K, const double* alpha, const double* beta,
                const int32_t* steps, Spectrum& out);
// The same for several blocks with one host synchronisation.
struct RitzJob {
  int R, nvmax, ld, K;
  const double* alpha;
  const double* beta;
  const int32_t* steps;
  Spectrum* out;
};
void ritz_stage_many(Ctx& c, std::vector<RitzJob>& jobs);
// Exact spectra of several blocks of the prepared sector (one batched launch).
void run_exact_blocks(Ctx& c, const std::vector<std::pair<int, int>>& blocks);
// Deferred form: assembles the blocks' matrices into the pool (flushing it
// first when they would push it past kDeferPoolBytes) and registers them as
// pending spectra of the current sector.
void queue_exact_blocks(Ctx& c, const std::vector<std::pair<int, int>>& blocks);
// Diagonalises every pooled matrix in one launch, runs the Ritz stage of
// every pooled FTLM block in one more, then the queued accumulations in
// queue order, and turns the current sector's pending spectra into ordinary
// ones; empties the pool.
void flush_deferred(Ctx& c);
// Bytes held by the pool (matrices and Lanczos coefficients).
int64_t defer_pool_bytes(const Ctx& c);
constexpr int64_t kDeferPoolBytes = int64_t(4) << 30;
// Thermo
void thermo_configure(Ctx& c, int nbeta, const double* beta, int nmu, const double* mu);
void thermo_accumulate(Ctx& c, const Spectrum& s);
void thermo_accumulate_host(Ctx& c, const double* ev, const double* w, int64_t count, double pref, int particles);
// Accumulates a spectrum already on the device (w null: unit weights).
void thermo_accumulate_dev(Ctx& c, const double* ev, const double* w, int64_t count, double pref, int particles);
void thermo_read(Ctx& c, double* emin, double* z, double* n, double* n2);

// Seeds and reference start vectors (main.cpp:514-533, 1015-1025)
uint64_t block_seed(uint64_t seed, int n_up, int n_dn, int mx, int my);
void reference_start_vectors(uint64_t bseed, int sample0, int nva, int64_t dim, double* out);
// Nonzero-amplitude hops with active targets in the prepared block (the
// h_nz * dim of the H*V byte model).
int64_t block_nonzero_hops(Ctx& c);
// Builds the cached hop list of the prepared block; false when it does not fit in memory.
bool hoplist_build(Ctx& c);

// Spectra arena
int64_t spectra_alloc(Ctx& c, int64_t count);  // returns offset (doubles) of 2*count slots
void spectra_reset(Ctx& c);

// Scan helpers (exclusive, in place on device, returns total)
int64_t scan_excl_i32_to_i64(Ctx& c, const int32_t* flags, int64_t* out, int64_t n);

}  // namespace ftlm
