/* libftlm_gpu: C ABI of the B200 FTLM engine.
 *
 * Drop-in seam for the hot path of PeizhiMai/FTLM_extended_Hubbard_development
 * (src/main.cpp). The reference runs, per (N_up, N_down) sector and per
 * momentum block (mx, my), the chain
 *   build_sector_basis -> build_momentum_block -> {run_ftlm_block |
 *   diagonalize_block_exact} -> accumulate_block_thermo
 * (main.cpp:1519-1720). Each entry point below replaces one link of that
 * chain; its comment cites the reference interface it stands in for.
 *
 * Conventions
 *  - Every function returns an int status: FTLM_OK (0) or an FTLM_ERR_*
 *    code. ftlm_last_error() returns the message of the last failure.
 *  - Plain pointers and sizes only. Host buffers are owned by the caller;
 *    device memory is owned by the context.
 *  - Complex arrays are interleaved (re, im) doubles.
 *  - One host thread per context; a context owns one CUDA stream.
 *  - There is no CPU fallback: without a usable CUDA device
 *    ftlm_ctx_create fails with FTLM_ERR_CUDA.
 */
#ifndef FTLM_GPU_H
#define FTLM_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FTLM_ABI_VERSION 2

enum {
  FTLM_OK = 0,
  FTLM_ERR_ARG = 1,       /* invalid argument */
  FTLM_ERR_STATE = 2,     /* call out of order (e.g. no sector prepared) */
  FTLM_ERR_CUDA = 3,      /* CUDA runtime error / no device */
  FTLM_ERR_CAPACITY = 4,  /* caller buffer too small (count reports the need) */
  FTLM_ERR_NUMERIC = 5,   /* eigen-solver did not converge */
  FTLM_ERR_INTERNAL = 6
};

enum { FTLM_PREC_FP64 = 0, FTLM_PREC_MIXED = 1 };
enum { FTLM_START_REF_GAUSSIAN = 0, FTLM_START_PHILOX_PHASE = 1 };

/* Model parameters: the Hamiltonian fields of Params (main.cpp:32-41). */
typedef struct ftlm_model {
  int32_t lx, ly;
  double tx, ty, tp;  /* x, y and diagonal hoppings */
  double phix, phiy;  /* twists in units of 2*pi */
  double u, v;        /* on-site and nearest-neighbour interactions */
} ftlm_model;

/* Run options: the sampling fields of Params (main.cpp:47-51) plus the
 * engine's own knobs. */
typedef struct ftlm_run_opts {
  int32_t samples;                /* --samples: random vectors per block */
  int32_t lanczos_steps;          /* --lanczos-steps */
  uint64_t exact_block_threshold; /* --exact-block-threshold */
  uint64_t seed;                  /* --seed */
  int32_t precision;              /* FTLM_PREC_FP64 | FTLM_PREC_MIXED */
  int32_t start_vector;           /* FTLM_START_REF_GAUSSIAN | FTLM_START_PHILOX_PHASE */
  int32_t batch_vectors;          /* vectors per H*V sweep; 0 = min(samples, 128), halved until the sweep's arrays fit in device memory */
  int32_t device;                 /* CUDA device ordinal */
} ftlm_run_opts;

typedef struct ftlm_sector_info {
  uint64_t full_dim;       /* C(N, N_up) * C(N, N_down) (SectorBasis::full_dim) */
  uint64_t parents;        /* number of orbit representatives */
  int32_t n_k;             /* lx * ly momentum blocks */
  uint64_t block_dim[64];  /* dimension of block k = my*lx + mx */
} ftlm_sector_info;

typedef struct ftlm_profile {
  double hv_ms;            /* CUDA-event time of all H*V launches (when timing is on) */
  int64_t hv_launches;
  double hv_bytes;         /* algorithmic bytes of those launches */
  double update_ms;        /* Lanczos vector-update launches */
  int64_t update_launches;
  double eig_ms, dense_ms, thermo_ms, sector_ms, block_ms;
  int64_t kernel_launches; /* kernels of this library launched since the last reset */
  int64_t h2d_bytes, d2h_bytes;
  int32_t hv_variant;      /* H*V kernel variant used last (autotuned unless FTLM_HV_VARIANT is set) */
  int32_t tune_runs;       /* autotuner measurements made */
  double small_ms;         /* small-block Lanczos launches (ftlm_blocks_ftlm_batched) */
  int64_t small_tasks;     /* (block, random vector) pairs they ran */
  double hv_hops;          /* nonzero off-diagonal hop x vector products of the timed H*V launches */
  double hv_min_bytes;     /* their compulsory bytes: per launch D * (2 * nv * s + 8) */
  int32_t hv_source;       /* operator source of the last sweep: 0 on the fly, 1 hop list, 2 split-spin */
  int32_t pad0;
} ftlm_profile;

typedef struct ftlm_ctx ftlm_ctx;

/* Context: lattice + couplings + sampling options (replaces Params and the
 * build_lattice call, main.cpp:1461-1462). Validation follows
 * parse_args (main.cpp:332-366): positive lattice, at most 63 sites,
 * positive samples and steps. */
int ftlm_ctx_create(const ftlm_model* model, const ftlm_run_opts* opts, ftlm_ctx** out);
void ftlm_ctx_destroy(ftlm_ctx* ctx);
/* Copies the last error message into buf (always NUL-terminated). */
int ftlm_last_error(const ftlm_ctx* ctx, char* buf, size_t len);
int ftlm_abi_version(void);
/* Architecture of this library's device code as the CUDA runtime loaded it on
 * `device` (cudaFuncGetAttributes of one of its kernels): binary_version is
 * major*10+minor of the SASS (100 for sm_100a), ptx_version that of the
 * virtual architecture it was compiled from. No counterpart in the reference
 * (build check). */
int ftlm_device_code_version(int32_t device, int32_t* binary_version, int32_t* ptx_version);

/* Builds the translation-orbit tables of sector (n_up, n_down) on the GPU
 * and reports the dimension of every momentum block.
 * Replaces build_sector_basis (main.cpp:622-721) and the block dimensions
 * of build_momentum_block (main.cpp:723-777). */
int ftlm_sector_prepare(ftlm_ctx* ctx, int32_t n_up, int32_t n_down, ftlm_sector_info* out);

/* Spectrum of block (mx, my) of the prepared sector.
 * exact = 0: FTLM (main.cpp:996-1113); evals/weights receive samples*K
 *   Ritz values and weights v1^2/R, sample by sample, each sample sorted
 *   ascending; *trace_prefactor = dim.
 * exact = 1: eigenvalues ascending (main.cpp:847-911); weights untouched;
 *   *trace_prefactor = 1. A spectrum computed by
 *   ftlm_blocks_exact_batched is returned from the device cache.
 * evals == NULL queries *count only (the spectrum is still computed and
 * kept on the device for ftlm_thermo_accumulate_block). */
int ftlm_block_spectrum(ftlm_ctx* ctx, int32_t mx, int32_t my, int32_t exact, double* evals,
                        double* weights, size_t cap, size_t* count, double* trace_prefactor);

/* Drops the device-cached spectra of the prepared sector, so the next
 * ftlm_block_spectrum recomputes (the reference recomputes every block it
 * visits, main.cpp:1569-1581; the cache is this engine's own). */
int ftlm_spectra_reset(ftlm_ctx* ctx);

/* Exact spectra of several blocks of the prepared sector in one batched
 * launch of the dense Hermitian eigen-solver; the results stay on the
 * device (diagonalize_block_exact, main.cpp:847-911, for a list of blocks). */
int ftlm_blocks_exact_batched(ftlm_ctx* ctx, const int32_t* mx, const int32_t* my,
                              int32_t nblocks);

/* Deferred block spectra across sectors (the reference solves each block as
 * its sector loop reaches it, main.cpp:1519-1534 with 847-911 and 996-1113).
 * With on != 0, ftlm_blocks_exact_batched only assembles the exact blocks'
 * dense matrices into a device pool, ftlm_blocks_ftlm_batched keeps the
 * Lanczos coefficients of its small blocks (<= FTLM_SMALL_BLOCK_MAX rows)
 * there instead of running their Ritz stage, and
 * ftlm_thermo_accumulate_block of a pooled block is queued.
 * ftlm_spectra_flush diagonalises every pooled matrix, of any number of
 * sectors, in ONE launch of the dense solver and runs the Ritz stage of every
 * pooled FTLM block in ONE more, then runs the queued accumulations in the
 * order they were queued. A sector's blocks alone keep few SMs busy; a
 * curve's keep all of them. The pool is flushed implicitly by
 * ftlm_thermo_read, ftlm_thermo_configure (before the reset),
 * ftlm_block_spectrum of a pooled block, ftlm_spectra_defer(ctx, 0), and
 * before a batch that would take the pool past 4 GiB. Pooled spectra are
 * bit-identical to the immediate ones; the accumulation order changes, so
 * the sums differ from the immediate path by rounding only. A Ritz stage
 * that fails to converge is reported by the call that flushes. Off by
 * default; large FTLM blocks are not pooled. */
int ftlm_spectra_defer(ftlm_ctx* ctx, int32_t on);
int ftlm_spectra_flush(ftlm_ctx* ctx);

/* FTLM spectra of several blocks of the prepared sector (run_ftlm_block,
 * main.cpp:996-1113, for a list of blocks). Blocks of at most
 * FTLM_SMALL_BLOCK_MAX rows run in one persistent launch, one CTA per
 * (block, random vector) with the vectors in shared memory; larger blocks
 * run one after another on the sweep path. Results stay on the device, as
 * ftlm_block_spectrum(exact = 0) would leave them, and are what that call
 * then returns. */
#define FTLM_SMALL_BLOCK_MAX 4096
int ftlm_blocks_ftlm_batched(ftlm_ctx* ctx, const int32_t* mx, const int32_t* my,
                             int32_t nblocks);

/* Grand-canonical accumulators over a beta list and mu grid (the
 * emin/z/n/n2 vectors of main.cpp:1500-1504 and 1748-1752). Resets them. */
int ftlm_thermo_configure(ftlm_ctx* ctx, int32_t nbeta, const double* betas, int32_t nmu,
                          const double* mu);
/* Adds the device-resident spectrum of block (mx, my) of the prepared
 * sector (accumulate_block_thermo, main.cpp:1172-1219). */
int ftlm_thermo_accumulate_block(ftlm_ctx* ctx, int32_t mx, int32_t my);
/* Adds a host spectrum, e.g. a checkpointed block (main.cpp:1549-1566).
 * weights == NULL for exact blocks. */
int ftlm_thermo_accumulate_host(ftlm_ctx* ctx, const double* evals, const double* weights,
                                size_t count, double trace_prefactor, int32_t particles);
/* Reads the accumulators, each [nbeta][nmu]. */
int ftlm_thermo_read(ftlm_ctx* ctx, double* emin, double* z, double* n, double* n2);

/* H*V on block (mx, my) of the prepared sector with host buffers
 * in/out[dim][nvec] (complex). The matrix elements are generated on the fly
 * on the GPU (apply_hamiltonian, main.cpp:833-845, applied to nvec vectors). */
int ftlm_block_apply(ftlm_ctx* ctx, int32_t mx, int32_t my, int32_t nvec, const double* in,
                     double* out);

/* Plain Lanczos coefficients of block (mx, my) from caller start vectors
 * start[samples][dim] (complex), or from the context's start-vector mode
 * when start == NULL. alpha/beta are [samples][lanczos_steps], steps
 * [samples] (the recurrence of run_ftlm_block, main.cpp:1033-1057). */
int ftlm_block_lanczos(ftlm_ctx* ctx, int32_t mx, int32_t my, const double* start,
                       double* alpha, double* beta, int32_t* steps);

/* Parity views of the GPU tables.
 * Parents (representative up/down words, degeneracy, diagonal energy) in
 * reference order (SectorBasis::parents, main.cpp:622-675). */
int ftlm_debug_sector_parents(ftlm_ctx* ctx, uint64_t* up, uint64_t* down, int32_t* deg,
                              double* diag, size_t cap, size_t* count);
/* Relation of every state of the sector, in (up-rank, down-rank) order:
 * parent, first translation onto it, its sign (main.cpp:640-675). */
int ftlm_debug_sector_relations(ftlm_ctx* ctx, int32_t* parent, int32_t* shift, int32_t* sign,
                                size_t cap);
/* CSR of block (mx, my) in the reference's entry order (MomentumBlock,
 * main.cpp:113-122, 779-804). val holds 2*nnz doubles. */
int ftlm_debug_block_csr(ftlm_ctx* ctx, int32_t mx, int32_t my, double* diag, int32_t* row_ptr,
                         int32_t* col, double* val, size_t dim_cap, size_t nnz_cap,
                         size_t* dim, size_t* nnz);

/* Allocation-free Ritz stage. No counterpart in the reference: it exists for
 * callers that cannot allocate device memory when they need the Ritz values,
 * e.g. a host framework whose caching allocator already holds the device's
 * memory pool, or a latency-critical loop that cannot afford cudaMalloc /
 * cudaFree (cudaFree synchronises the device). It computes what
 * ftlm_block_spectrum returns for an FTLM block from Lanczos coefficients the
 * caller holds on the device, without allocating anything.
 *  - alpha, beta: device arrays [nvec][ld] (the layout ftlm_block_lanczos
 *    returns on the host); steps: device [nvec], the alphas taken per vector.
 *  - evals, weights: device outputs of at least nvec*ld doubles; each vector's
 *    Ritz values ascending with weights v1^2 * inv_samples, concatenated vector
 *    by vector. count (device, may be NULL) receives the total, or -1 when a
 *    QL iteration failed to converge.
 *  - Runs on `stream` (a cudaStream_t; NULL = default stream) of the current
 *    device. Work space: a fixed device array of 3*FTLM_NOALLOC_MAX_ENTRIES
 *    doubles (1.5 MiB) that every device loading the library keeps until the
 *    process exits; nvec > 128 or nvec*ld > FTLM_NOALLOC_MAX_ENTRIES is
 *    rejected with FTLM_ERR_CAPACITY. All calls share that array: calls that
 *    overlap on the GPU race. The first call on a device looks up the array's
 *    address; make it before any stream capture. The address is kept per
 *    device and CUDA context: after a device reset the next call is a first
 *    call again.
 *  - errbuf (may be NULL) receives a message on failure. */
#define FTLM_NOALLOC_MAX_ENTRIES 65536
int ftlm_ritz_noalloc(const double* alpha, const double* beta, const int32_t* steps, int32_t nvec, int32_t ld,
                      double inv_samples, double* evals, double* weights, int64_t* count, void* stream,
                      char* errbuf, size_t errlen);

/* Twist-surrogate network (no counterpart in the reference: the learned part
 * of the engine). An FP32 MLP, x[n_in] -> `depth` hidden tanh layers of
 * `width` -> linear y[n_out], trained on the GPU by this library's own
 * forward / backward / Adam kernels on a masked mean-squared error. Host
 * arrays are row-major [n][n_in] / [n][n_out]. Parameters are one flat FP32
 * vector, per layer W[out][in] then b[out]. */
typedef struct ftlm_mlp ftlm_mlp;
int ftlm_mlp_create(int32_t n_in, int32_t width, int32_t depth, int32_t n_out, uint64_t seed, int32_t device,
                    ftlm_mlp** out);
void ftlm_mlp_destroy(ftlm_mlp* net);
int ftlm_mlp_last_error(const ftlm_mlp* net, char* buf, size_t len);
int ftlm_mlp_num_params(const ftlm_mlp* net, int64_t* count);
int ftlm_mlp_get_params(ftlm_mlp* net, float* host, int64_t count);
int ftlm_mlp_set_params(ftlm_mlp* net, const float* host, int64_t count);
/* Inference: y = f(x) for n rows. */
int ftlm_mlp_forward(ftlm_mlp* net, const float* x, int64_t n, float* y);
/* Loss sum(mask*(f(x)-t)^2)/sum(mask) and, if grad != NULL, its gradient
 * w.r.t. the flat parameter vector (one forward + backward pass). */
int ftlm_mlp_loss_grad(ftlm_mlp* net, const float* x, const float* t, const float* mask, int64_t n, float* loss,
                       float* grad);
/* Adam training: `epochs` shuffled passes of full mini-batches of `batch`
 * rows (seeded shuffle); loss_history[epochs] (may be NULL) gets the mean
 * batch loss of each epoch. */
int ftlm_mlp_train(ftlm_mlp* net, const float* x, const float* t, const float* mask, int64_t n, int32_t epochs,
                   int32_t batch, float lr, uint64_t seed, float* loss_history);

/* Instrumentation: per-kernel CUDA-event timing (adds a sync per timed
 * launch), and the counters accumulated since the last reset. */
int ftlm_profile_enable(ftlm_ctx* ctx, int32_t on);
int ftlm_profile_read(ftlm_ctx* ctx, ftlm_profile* out);
int ftlm_profile_reset(ftlm_ctx* ctx);

#ifdef __cplusplus
}
#endif
#endif /* FTLM_GPU_H */
