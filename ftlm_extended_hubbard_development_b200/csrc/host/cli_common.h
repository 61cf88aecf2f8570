// Host side of the drop-in executables ftlm_n_vs_mu / ftlm_ed_n_vs_mu.
//
// Mirrors the reference program's user-facing contract
// (PeizhiMai/FTLM_extended_Hubbard_development src/main.cpp, ed_main.cpp):
// the same flags and defaults (main.cpp:32-61, 257-368), the same error
// messages and exit codes (main.cpp:177-179, 1835-1838), the same
// (N_up, N_down, my, mx) block order (main.cpp:1519-1534), the same CSV
// columns and number formatting (main.cpp:1409-1455), the same checkpoint
// and .meta byte formats (main.cpp:370-412, 1269-1398) and the same trace /
// debug CSVs (main.cpp:1233-1267, 1505-1663). The numerical work goes to the
// GPU through the C ABI of libftlm_gpu (include/ftlm_gpu.h).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "ftlm_gpu.h"

namespace ftlm_cli {

struct Params {  // main.cpp:32-61 plus the engine's additive flags
  int lx = 2;
  int ly = 2;
  double tx = 1.0;
  double ty = 1.0;
  double tp = 0.0;
  double phix = 1.0;
  double phiy = 1.0;
  double u = 8.0;
  double v = 0.0;
  double beta = 2.0;
  std::vector<double> beta_values;
  double mu_min = -4.0;
  double mu_max = 10.0;
  int mu_count = 61;
  int samples = 5;
  int lanczos_steps = 80;
  int threads = 0;
  std::size_t exact_block_threshold = 256;
  std::uint64_t seed = 12345;
  std::size_t max_sector_dim = 2000000;
  std::string output = "n_vs_mu.csv";
  std::string checkpoint;
  std::string trace_partition_csv;
  std::string debug_block_csv;
  int debug_block_nup = -1;
  int debug_block_ndown = -1;
  int debug_block_mx = -1;
  int debug_block_my = -1;
  // engine flags (new, additive)
  int precision = FTLM_PREC_FP64;
  int start_vector = FTLM_START_REF_GAUSSIAN;
  int batch_vectors = 0;
  int device = 0;
  std::string profile_json;
};

[[noreturn]] void die(const std::string& message);
Params parse_args(int argc, char** argv);
void print_help(const char* argv0);

std::vector<double> linspace(double start, double stop, int count);

struct Spectrum {  // StoredSpectrum, main.cpp:138-145
  std::vector<double> eigenvalues;
  std::vector<double> sample_weights;
  double trace_prefactor = 1.0;
  std::size_t basis_dim = 0;
  int particles = 0;
  bool exact = false;
};

struct BlockKey {
  int n_up, n_down, mx, my;
  bool operator<(const BlockKey& o) const;
};

// checkpoint + .meta (main.cpp:370-412, 1279-1398)
std::string checkpoint_metadata_text(const Params& p);
void validate_or_write_checkpoint_metadata(const Params& p);
void ensure_checkpoint_header(const std::string& path);
std::vector<std::pair<BlockKey, Spectrum>> read_checkpoint(const std::string& path);
void append_checkpoint_record(const std::string& path, const BlockKey& key, const Spectrum& s);

// CSV writers (main.cpp:1409-1455)
void write_results(const std::string& path, const std::vector<double>& mu, const std::vector<double>& n,
                   const std::vector<double>& chi, const std::vector<double>& kappa,
                   const std::vector<double>& z, const std::vector<double>& logz);
void write_multi_beta_results(const std::string& path, const std::vector<double>& betas,
                              const std::vector<double>& mu, const std::vector<std::vector<double>>& n,
                              const std::vector<std::vector<double>>& chi,
                              const std::vector<std::vector<double>>& kappa,
                              const std::vector<std::vector<double>>& z,
                              const std::vector<std::vector<double>>& logz);

// RAII view of one engine context; errors become die().
class Engine {
 public:
  Engine(const Params& p);
  ~Engine();
  Engine(const Engine&) = delete;
  Engine& operator=(const Engine&) = delete;
  ftlm_ctx* ctx() const { return ctx_; }
  void check(int status, const char* what) const;

 private:
  ftlm_ctx* ctx_ = nullptr;
};

int run_ftlm_main(int argc, char** argv);
int run_ed_main(int argc, char** argv);

}  // namespace ftlm_cli
