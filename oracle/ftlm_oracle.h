/* Oracle: CPU restatement of the reference FTLM hot path (TEST INFRASTRUCTURE).
 *
 * This library is the checker for the CUDA engine. Only tests/, the smoke
 * check in __graft_entry__.py and the cpu_baseline / reference legs of
 * bench.py may load it. The product path never calls it.
 *
 * Every function restates one piece of the reference program
 * (PeizhiMai/FTLM_extended_Hubbard_development, src/main.cpp and
 * src/ed_main.cpp); the citation is given beside each declaration. The
 * restatement is pinned against golden vectors dumped from the reference
 * compiled in this container (oracle/ref_probe.cpp, tests/golden/).
 *
 * Complex numbers are interleaved (re, im) double pairs.
 */
#ifndef FTLM_ORACLE_H
#define FTLM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fo_model {
  int lx, ly;
  double tx, ty, tp, phix, phiy, u, v;
} fo_model;

/* splitmix-style mixer and per-block seed (main.cpp:514-533). */
uint64_t fo_mix_u64(uint64_t v);
uint64_t fo_block_seed(uint64_t seed, int n_up, int n_down, int mx, int my);

/* Translation of one spin species by (dx, dy) with its fermionic reorder
 * sign (main.cpp:579-613). Returns the translated bits; *sign = +-1. */
uint64_t fo_translate_spin(uint64_t bits, int dx, int dy, int lx, int ly, int* sign);

/* Sector basis (main.cpp:622-721): parents in reference order. Returns the
 * parent count, or -1 when cap is too small. Arrays may be NULL to query. */
int64_t fo_sector_parents(const fo_model* m, int n_up, int n_down, uint64_t* up,
                          uint64_t* down, int32_t* deg, double* diag, int64_t cap);

/* Relation (parent, first shift, sign) of every state of the sector, in
 * (up-rank, down-rank) order (main.cpp:640-675). Arrays hold full_dim. */
int fo_sector_relations(const fo_model* m, int n_up, int n_down, int32_t* parent,
                        int32_t* shift, int32_t* sign);

/* Momentum block as CSR (main.cpp:723-805). Query with NULL arrays to get
 * *dim and *nnz; then call again with arrays of that size. val holds 2*nnz. */
int fo_block_csr(const fo_model* m, int n_up, int n_down, int mx, int my, int64_t* dim,
                 int64_t* nnz, double* diag, int32_t* row_ptr, int32_t* col, double* val);

/* CSR H*v (main.cpp:833-845). */
void fo_csr_apply(int64_t dim, const double* diag, const int32_t* row_ptr, const int32_t* col,
                  const double* val, const double* in, double* out);

/* Reference start vector of one sample (main.cpp:1015-1025): mt19937_64
 * seeded with mix(block_seed ^ sample), libstdc++ polar normals, element i =
 * (draw 2i+1, draw 2i), normalised. out holds 2*dim doubles. */
void fo_start_vector(uint64_t block_seed, int sample, int64_t dim, double* out);

/* Plain Lanczos recurrence from a given start vector (main.cpp:1033-1057).
 * alpha/beta hold kmax entries; returns the number of alphas taken. */
int fo_lanczos(int64_t dim, const double* diag, const int32_t* row_ptr, const int32_t* col,
               const double* val, const double* start, int kmax, double* alpha, double* beta);

/* Classical Jacobi on the Lanczos tridiagonal, eigenvalues sorted ascending
 * with squared first eigenvector components (main.cpp:913-994, 1059-1094). */
void fo_tridiag_jacobi(int n, const double* alpha, const double* beta, double* evals,
                       double* v1sq);

/* Exact eigenvalues of a block via dense Hermitian zheev (main.cpp:847-911). */
int fo_block_exact(int64_t dim, const double* diag, const int32_t* row_ptr, const int32_t* col,
                   const double* val, double* evals);

/* Shifted log-sum-exp accumulation of one block (main.cpp:1172-1219).
 * weights may be NULL (exact blocks). */
void fo_thermo_accumulate(int64_t n, const double* evals, const double* weights,
                          double prefactor, int particles, double beta, int nmu,
                          const double* mu, double* emin, double* z, double* nsum,
                          double* n2sum);

/* Whole n(mu) curve over all (N_up, N_down, k) blocks in reference order.
 * ed != 0 diagonalises every block exactly (ed_main.cpp:74-106); otherwise
 * blocks with dim <= threshold are exact and the rest use FTLM with
 * reference start vectors (main.cpp:1519-1720). Accumulators are
 * [nbeta][nmu]; emin must be +inf and z/nsum/n2sum zero on entry.
 * Returns 0, or -1 when a sector exceeds max_sector_dim. */
int fo_run_curve(const fo_model* m, int samples, int steps, uint64_t threshold, uint64_t seed,
                 uint64_t max_sector_dim, int ed, int nbeta, const double* betas, int nmu,
                 const double* mu, double* emin, double* z, double* nsum, double* n2sum);

#ifdef __cplusplus
}
#endif
#endif
