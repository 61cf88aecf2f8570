// Host side of the drop-in executables (see cli_common.h).
#include "cli_common.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <limits>
#include <map>
#include <numeric>
#include <sstream>
#include <stdexcept>
#include <thread>

namespace ftlm_cli {

[[noreturn]] void die(const std::string& message) { throw std::runtime_error(message); }

namespace {

template <typename T>
T parse_value(const std::string& text) {  // main.cpp:193-202
  std::istringstream in(text);
  T value{};
  in >> value;
  if (!in || !in.eof()) die("Failed to parse value: " + text);
  return value;
}

std::vector<double> parse_double_list(const std::string& text) {  // main.cpp:204-218
  std::vector<double> values;
  std::istringstream in(text);
  std::string item;
  while (std::getline(in, item, ',')) {
    if (item.empty()) die("Empty entry in comma-separated value list: " + text);
    values.push_back(parse_value<double>(item));
  }
  if (values.empty()) die("Expected at least one value in comma-separated list: " + text);
  return values;
}

uint64_t n_choose_k(int n, int k) {
  if (k < 0 || k > n) return 0;
  unsigned __int128 r = 1;
  for (int i = 1; i <= k; ++i) r = r * static_cast<unsigned>(n - k + i) / static_cast<unsigned>(i);
  return static_cast<uint64_t>(r);
}

template <typename T>
void write_binary(std::ostream& out, const T& v) {
  out.write(reinterpret_cast<const char*>(&v), sizeof(T));
}
template <typename T>
bool read_binary(std::istream& in, T& v) {
  return static_cast<bool>(in.read(reinterpret_cast<char*>(&v), sizeof(T)));
}

const char kMagic[8] = {'F', 'T', 'L', 'M', 'C', 'P', '1', '\n'};
const char kRecord[8] = {'B', 'L', 'K', 'R', 'E', 'C', '1', '\n'};

// Per-block Boltzmann sums at one mu, shifted by the block minimum
// (raw_block_thermo_from_ftlm / _from_exact, main.cpp:1115-1170).
struct BlockThermo {
  double z = 0.0;
  double n_total = 0.0;
  double n2_total = 0.0;
  double min_shifted_energy = std::numeric_limits<double>::infinity();
};

BlockThermo raw_thermo(const std::vector<double>& ev, const std::vector<double>* w, double pref, int particles,
                       double beta, double mu) {
  BlockThermo t;
  for (double e : ev) t.min_shifted_energy = std::min(t.min_shifted_energy, e - mu * static_cast<double>(particles));
  if (!std::isfinite(t.min_shifted_energy)) return t;
  for (std::size_t i = 0; i < ev.size(); ++i) {
    const double shifted = ev[i] - mu * static_cast<double>(particles) - t.min_shifted_energy;
    const double weight = w ? pref * (*w)[i] * std::exp(-beta * shifted) : std::exp(-beta * shifted);
    const double pc = static_cast<double>(particles);
    t.z += weight;
    t.n_total += pc * weight;
    t.n2_total += pc * pc * weight;
  }
  return t;
}

void write_selected_block_debug(const std::string& path, int n_up, int n_down, int mx, int my,
                                const Spectrum& ftlm, const std::vector<double>& exact, double beta,
                                const std::vector<double>& mu_values) {  // main.cpp:1233-1267
  std::ofstream out(path);
  if (!out) die("Failed to open selected block debug file: " + path);
  out << "nup,ndown,mx,my,basis_dim,mu,z_ftlm,z_ed,z_ratio,"
      << "n_ftlm_total,n_ed_total,n_diff,n2_ftlm_total,n2_ed_total,n2_diff,"
      << "min_ftlm,min_ed,sum_sample_weights\n";
  out << std::setprecision(15);
  const double sw = std::accumulate(ftlm.sample_weights.begin(), ftlm.sample_weights.end(), 0.0);
  for (double mu : mu_values) {
    const BlockThermo f = raw_thermo(ftlm.eigenvalues, &ftlm.sample_weights, static_cast<double>(ftlm.basis_dim),
                                     ftlm.particles, beta, mu);
    const BlockThermo e = raw_thermo(exact, nullptr, 1.0, ftlm.particles, beta, mu);
    const double ratio = (e.z > 0.0) ? (f.z / e.z) : 0.0;
    out << n_up << "," << n_down << "," << mx << "," << my << "," << ftlm.basis_dim << "," << mu << "," << f.z << ","
        << e.z << "," << ratio << "," << f.n_total << "," << e.n_total << "," << (f.n_total - e.n_total) << ","
        << f.n2_total << "," << e.n2_total << "," << (f.n2_total - e.n2_total) << "," << f.min_shifted_energy << ","
        << e.min_shifted_energy << "," << sw << "\n";
  }
}

struct Observables {
  std::vector<std::vector<double>> n, chi, kappa, z, logz;
};

// main.cpp:1770-1788 / 1805-1823
Observables finalize(Engine& eng, const std::vector<double>& betas, std::size_t nmu, int sites) {
  const std::size_t nb = betas.size();
  std::vector<double> emin(nb * nmu), z(nb * nmu), ns(nb * nmu), n2(nb * nmu);
  eng.check(ftlm_thermo_read(eng.ctx(), emin.data(), z.data(), ns.data(), n2.data()), "thermo_read");
  Observables o;
  o.n.assign(nb, std::vector<double>(nmu));
  o.chi = o.kappa = o.z = o.logz = o.n;
  for (std::size_t b = 0; b < nb; ++b) {
    for (std::size_t i = 0; i < nmu; ++i) {
      const std::size_t k = b * nmu + i;
      o.z[b][i] = z[k];
      o.logz[b][i] = std::log(z[k]) - betas[b] * emin[k];
      const double s = static_cast<double>(sites);
      const double mean = ns[k] / z[k];
      const double mean2 = n2[k] / z[k];
      const double cc = (mean2 - mean * mean) / s;
      o.n[b][i] = mean / s;
      o.chi[b][i] = std::max(0.0, cc);
      o.kappa[b][i] = betas[b] * o.chi[b][i];
    }
  }
  return o;
}

void write_profile(const Params& p, Engine& eng, double wall_s) {
  if (p.profile_json.empty()) return;
  ftlm_profile pr{};
  eng.check(ftlm_profile_read(eng.ctx(), &pr), "profile_read");
  std::ofstream out(p.profile_json);
  if (!out) die("Failed to open profile JSON: " + p.profile_json);
  out << std::setprecision(10) << "{\"wall_s\": " << wall_s << ", \"sector_ms\": " << pr.sector_ms
      << ", \"block_ms\": " << pr.block_ms << ", \"hv_ms\": " << pr.hv_ms << ", \"hv_launches\": " << pr.hv_launches
      << ", \"hv_bytes\": " << pr.hv_bytes
      << ", \"hv_gbs\": " << (pr.hv_ms > 0 ? pr.hv_bytes / (pr.hv_ms * 1e6) : 0.0) << ", \"eig_ms\": " << pr.eig_ms
      << ", \"dense_ms\": " << pr.dense_ms << ", \"thermo_ms\": " << pr.thermo_ms
      << ", \"kernel_launches\": " << pr.kernel_launches << ", \"h2d_bytes\": " << pr.h2d_bytes
      << ", \"d2h_bytes\": " << pr.d2h_bytes << "}\n";
}

void fetch(Engine& eng, int mx, int my, int exact, Spectrum& s) {
  size_t count = 0;
  double pref = 0.0;
  eng.check(ftlm_block_spectrum(eng.ctx(), mx, my, exact, nullptr, nullptr, 0, &count, &pref), "block_spectrum");
  s.eigenvalues.assign(count, 0.0);
  s.sample_weights.assign(exact ? 0 : count, 0.0);
  eng.check(ftlm_block_spectrum(eng.ctx(), mx, my, exact, s.eigenvalues.data(),
                                exact ? nullptr : s.sample_weights.data(), count, &count, &pref),
            "block_spectrum");
  s.trace_prefactor = pref;
  s.exact = exact != 0;
}

}  // namespace

bool BlockKey::operator<(const BlockKey& o) const {
  if (n_up != o.n_up) return n_up < o.n_up;
  if (n_down != o.n_down) return n_down < o.n_down;
  if (mx != o.mx) return mx < o.mx;
  return my < o.my;
}

void print_help(const char* argv0) {  // main.cpp:220-255 plus the engine flags
  std::cout << "Usage: " << argv0 << " [options]\n"
            << "  --lx N                lattice size in x\n"
            << "  --ly N                lattice size in y\n"
            << "  --tx X                hopping along x bonds\n"
            << "  --ty Y                hopping along y bonds\n"
            << "  --tp X                second-neighbor diagonal hopping\n"
            << "  --phix X              homogeneous x twist in units of 2*pi\n"
            << "  --phiy Y              homogeneous y twist in units of 2*pi\n"
            << "  --u U                 onsite interaction\n"
            << "  --v V                 nearest-neighbor interaction\n"
            << "  --beta B              inverse temperature\n"
            << "  --beta-list LIST      comma-separated inverse temperatures\n"
            << "  --mu-min X            minimum chemical potential\n"
            << "  --mu-max X            maximum chemical potential\n"
            << "  --mu-count N          number of mu points\n"
            << "  --samples N           FTLM random vectors per k block\n"
            << "  --lanczos-steps N     Lanczos steps per random vector\n"
            << "  --threads N           host threads for reference start vectors (0 uses all cores)\n"
            << "  --exact-block-threshold N\n"
            << "                        use exact diagonalization for k blocks with dimension <= N\n"
            << "  --seed N              random seed\n"
            << "  --max-sector-dim N    abort if a full sector exceeds this size\n"
            << "  --checkpoint PATH     append/resume compact per-block spectra\n"
            << "  --trace-partition-csv PATH\n"
            << "                        write per-block FTLM vs ED thermodynamic traces\n"
            << "  --debug-block-nup N   selected block debug Nup\n"
            << "  --debug-block-ndown N selected block debug Ndown\n"
            << "  --debug-block-mx N    selected block debug mx\n"
            << "  --debug-block-my N    selected block debug my\n"
            << "  --debug-block-csv PATH\n"
            << "                        write selected-block FTLM vs ED comparison\n"
            << "  --output PATH         CSV output path\n"
            << "  --precision P         fp64 (default) or mixed (FP32 vectors, FP64 reductions)\n"
            << "  --start-vector S      ref-gaussian (default, reference start vectors) or philox-phase\n"
            << "  --batch-vectors N     random vectors per H*V sweep (0 = min(samples,128))\n"
            << "  --device N            CUDA device ordinal\n"
            << "  --profile-json PATH   write per-phase GPU timings\n"
            << "  --help                show this message\n";
}

Params parse_args(int argc, char** argv) {  // main.cpp:257-368
  Params p;
  for (int i = 1; i < argc; ++i) {
    const std::string arg = argv[i];
    auto next = [&](const std::string& name) {
      if (i + 1 >= argc) die("Missing value for " + name);
      return std::string(argv[++i]);
    };
    if (arg == "--help") {
      print_help(argv[0]);
      std::exit(0);
    } else if (arg == "--lx") {
      p.lx = parse_value<int>(next(arg));
    } else if (arg == "--ly") {
      p.ly = parse_value<int>(next(arg));
    } else if (arg == "--tx") {
      p.tx = parse_value<double>(next(arg));
    } else if (arg == "--ty") {
      p.ty = parse_value<double>(next(arg));
    } else if (arg == "--tp") {
      p.tp = parse_value<double>(next(arg));
    } else if (arg == "--phix") {
      p.phix = parse_value<double>(next(arg));
    } else if (arg == "--phiy") {
      p.phiy = parse_value<double>(next(arg));
    } else if (arg == "--u") {
      p.u = parse_value<double>(next(arg));
    } else if (arg == "--v") {
      p.v = parse_value<double>(next(arg));
    } else if (arg == "--beta") {
      p.beta = parse_value<double>(next(arg));
    } else if (arg == "--beta-list") {
      p.beta_values = parse_double_list(next(arg));
    } else if (arg == "--mu-min") {
      p.mu_min = parse_value<double>(next(arg));
    } else if (arg == "--mu-max") {
      p.mu_max = parse_value<double>(next(arg));
    } else if (arg == "--mu-count") {
      p.mu_count = parse_value<int>(next(arg));
    } else if (arg == "--samples") {
      p.samples = parse_value<int>(next(arg));
    } else if (arg == "--lanczos-steps") {
      p.lanczos_steps = parse_value<int>(next(arg));
    } else if (arg == "--threads") {
      p.threads = parse_value<int>(next(arg));
    } else if (arg == "--exact-block-threshold") {
      p.exact_block_threshold = parse_value<std::size_t>(next(arg));
    } else if (arg == "--seed") {
      p.seed = parse_value<std::uint64_t>(next(arg));
    } else if (arg == "--max-sector-dim") {
      p.max_sector_dim = parse_value<std::size_t>(next(arg));
    } else if (arg == "--checkpoint") {
      p.checkpoint = next(arg);
    } else if (arg == "--trace-partition-csv") {
      p.trace_partition_csv = next(arg);
    } else if (arg == "--debug-block-nup") {
      p.debug_block_nup = parse_value<int>(next(arg));
    } else if (arg == "--debug-block-ndown") {
      p.debug_block_ndown = parse_value<int>(next(arg));
    } else if (arg == "--debug-block-mx") {
      p.debug_block_mx = parse_value<int>(next(arg));
    } else if (arg == "--debug-block-my") {
      p.debug_block_my = parse_value<int>(next(arg));
    } else if (arg == "--debug-block-csv") {
      p.debug_block_csv = next(arg);
    } else if (arg == "--output") {
      p.output = next(arg);
    } else if (arg == "--precision") {
      const std::string v = next(arg);
      if (v == "fp64") p.precision = FTLM_PREC_FP64;
      else if (v == "mixed") p.precision = FTLM_PREC_MIXED;
      else die("--precision must be fp64 or mixed.");
    } else if (arg == "--start-vector") {
      const std::string v = next(arg);
      if (v == "ref-gaussian") p.start_vector = FTLM_START_REF_GAUSSIAN;
      else if (v == "philox-phase") p.start_vector = FTLM_START_PHILOX_PHASE;
      else die("--start-vector must be ref-gaussian or philox-phase.");
    } else if (arg == "--batch-vectors") {
      p.batch_vectors = parse_value<int>(next(arg));
    } else if (arg == "--device") {
      p.device = parse_value<int>(next(arg));
    } else if (arg == "--profile-json") {
      p.profile_json = next(arg);
    } else {
      die("Unknown argument: " + arg);
    }
  }
  if (p.lx <= 0 || p.ly <= 0) die("Lattice dimensions must be positive.");
  if (p.lx * p.ly > 63) die("This implementation supports at most 63 sites.");
  if (p.beta_values.empty()) p.beta_values.push_back(p.beta);
  else p.beta = p.beta_values.front();
  for (double b : p.beta_values)
    if (b <= 0.0) die("All beta values must be positive.");
  if (p.samples <= 0 || p.lanczos_steps <= 0) die("--samples and --lanczos-steps must be positive.");
  if (p.threads < 0) die("--threads must be non-negative.");
  if (p.mu_count < 2) die("--mu-count must be at least 2.");
  const bool partial = (p.debug_block_nup >= 0) || (p.debug_block_ndown >= 0) || (p.debug_block_mx >= 0) ||
                       (p.debug_block_my >= 0) || !p.debug_block_csv.empty();
  const bool full = (p.debug_block_nup >= 0) && (p.debug_block_ndown >= 0) && (p.debug_block_mx >= 0) &&
                    (p.debug_block_my >= 0);
  if (partial && !full)
    die("Selected-block debug requires --debug-block-nup/--debug-block-ndown/--debug-block-mx/--debug-block-my "
        "together.");
  if (p.batch_vectors < 0 || p.batch_vectors > 128) die("--batch-vectors must be in 0..128.");
  if (p.device < 0) die("--device must be non-negative.");
  return p;
}

std::vector<double> linspace(double start, double stop, int count) {  // main.cpp:1400-1407
  std::vector<double> values(static_cast<std::size_t>(count));
  const double step = (stop - start) / static_cast<double>(count - 1);
  for (int i = 0; i < count; ++i) values[static_cast<std::size_t>(i)] = start + step * static_cast<double>(i);
  return values;
}

std::string checkpoint_metadata_text(const Params& params) {  // main.cpp:370-387
  std::ostringstream out;
  out << std::setprecision(17) << "lx=" << params.lx << "\n"
      << "ly=" << params.ly << "\n"
      << "tx=" << params.tx << "\n"
      << "ty=" << params.ty << "\n"
      << "tp=" << params.tp << "\n"
      << "phix=" << params.phix << "\n"
      << "phiy=" << params.phiy << "\n"
      << "u=" << params.u << "\n"
      << "v=" << params.v << "\n"
      << "samples=" << params.samples << "\n"
      << "lanczos_steps=" << params.lanczos_steps << "\n"
      << "exact_block_threshold=" << params.exact_block_threshold << "\n"
      << "seed=" << params.seed << "\n";
  return out.str();
}

void validate_or_write_checkpoint_metadata(const Params& params) {  // main.cpp:389-412
  if (params.checkpoint.empty()) return;
  const std::string path = params.checkpoint + ".meta";
  const std::string expected = checkpoint_metadata_text(params);
  {
    std::ifstream in(path);
    if (in) {
      const std::string existing((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
      if (existing != expected) die("Checkpoint metadata does not match current run: " + path);
      return;
    }
  }
  std::ofstream out(path);
  if (!out) die("Failed to write checkpoint metadata: " + path);
  out << expected;
}

void ensure_checkpoint_header(const std::string& path) {  // main.cpp:1279-1295
  if (path.empty()) return;
  {
    std::ifstream in(path, std::ios::binary);
    if (in && in.peek() != std::ifstream::traits_type::eof()) return;
  }
  std::ofstream out(path, std::ios::binary);
  if (!out) die("Failed to create checkpoint file: " + path);
  out.write(kMagic, sizeof(kMagic));
}

std::vector<std::pair<BlockKey, Spectrum>> read_checkpoint(const std::string& path) {  // main.cpp:1297-1361
  std::vector<std::pair<BlockKey, Spectrum>> out;
  if (path.empty()) return out;
  std::ifstream in(path, std::ios::binary);
  if (!in) return out;
  char magic[8] = {};
  if (!in.read(magic, sizeof(magic))) return out;
  if (std::memcmp(magic, kMagic, sizeof(magic)) != 0) die("Checkpoint has an unrecognized format: " + path);
  while (true) {
    char rec[8] = {};
    if (!in.read(rec, sizeof(rec))) break;
    if (std::memcmp(rec, kRecord, sizeof(rec)) != 0) break;
    BlockKey key{};
    Spectrum s;
    std::uint8_t exact = 0;
    std::uint64_t dim = 0, ne = 0, nw = 0;
    if (!read_binary(in, key.n_up) || !read_binary(in, key.n_down) || !read_binary(in, key.mx) ||
        !read_binary(in, key.my) || !read_binary(in, s.particles) || !read_binary(in, dim) ||
        !read_binary(in, s.trace_prefactor) || !read_binary(in, exact) || !read_binary(in, ne) ||
        !read_binary(in, nw))
      break;
    if (ne > 100000000ULL || nw > 100000000ULL) die("Checkpoint record is implausibly large: " + path);
    s.basis_dim = static_cast<std::size_t>(dim);
    s.exact = exact != 0;
    s.eigenvalues.resize(ne);
    s.sample_weights.resize(nw);
    if (!in.read(reinterpret_cast<char*>(s.eigenvalues.data()), static_cast<std::streamsize>(sizeof(double) * ne)) ||
        !in.read(reinterpret_cast<char*>(s.sample_weights.data()), static_cast<std::streamsize>(sizeof(double) * nw)))
      break;
    out.emplace_back(key, std::move(s));
  }
  return out;
}

void append_checkpoint_record(const std::string& path, const BlockKey& key, const Spectrum& s) {  // main.cpp:1363-1398
  if (path.empty()) return;
  ensure_checkpoint_header(path);
  std::ofstream out(path, std::ios::binary | std::ios::app);
  if (!out) die("Failed to append checkpoint file: " + path);
  out.write(kRecord, sizeof(kRecord));
  write_binary(out, key.n_up);
  write_binary(out, key.n_down);
  write_binary(out, key.mx);
  write_binary(out, key.my);
  write_binary(out, s.particles);
  const std::uint64_t dim = static_cast<std::uint64_t>(s.basis_dim);
  write_binary(out, dim);
  write_binary(out, s.trace_prefactor);
  const std::uint8_t exact = s.exact ? 1 : 0;
  write_binary(out, exact);
  const std::uint64_t ne = s.eigenvalues.size(), nw = s.sample_weights.size();
  write_binary(out, ne);
  write_binary(out, nw);
  out.write(reinterpret_cast<const char*>(s.eigenvalues.data()), static_cast<std::streamsize>(sizeof(double) * ne));
  out.write(reinterpret_cast<const char*>(s.sample_weights.data()), static_cast<std::streamsize>(sizeof(double) * nw));
  out.flush();
}

void write_results(const std::string& path, const std::vector<double>& mu, const std::vector<double>& n,
                   const std::vector<double>& chi, const std::vector<double>& kappa, const std::vector<double>& z,
                   const std::vector<double>& logz) {  // main.cpp:1409-1428
  std::ofstream out(path);
  if (!out) die("Failed to open output file: " + path);
  out << "mu,n,charge_correlation,compressibility,partition_like,log_partition\n";
  out << std::setprecision(15);
  for (std::size_t i = 0; i < mu.size(); ++i)
    out << mu[i] << "," << n[i] << "," << chi[i] << "," << kappa[i] << "," << z[i] << "," << logz[i] << "\n";
}

void write_multi_beta_results(const std::string& path, const std::vector<double>& betas,
                              const std::vector<double>& mu, const std::vector<std::vector<double>>& n,
                              const std::vector<std::vector<double>>& chi,
                              const std::vector<std::vector<double>>& kappa,
                              const std::vector<std::vector<double>>& z,
                              const std::vector<std::vector<double>>& logz) {  // main.cpp:1430-1455
  std::ofstream out(path);
  if (!out) die("Failed to open output file: " + path);
  out << "beta,mu,n,charge_correlation,compressibility,partition_like,log_partition\n";
  out << std::setprecision(15);
  for (std::size_t b = 0; b < betas.size(); ++b)
    for (std::size_t i = 0; i < mu.size(); ++i)
      out << betas[b] << "," << mu[i] << "," << n[b][i] << "," << chi[b][i] << "," << kappa[b][i] << "," << z[b][i]
          << "," << logz[b][i] << "\n";
}

Engine::Engine(const Params& p) {
  ftlm_model m{};
  m.lx = p.lx;
  m.ly = p.ly;
  m.tx = p.tx;
  m.ty = p.ty;
  m.tp = p.tp;
  m.phix = p.phix;
  m.phiy = p.phiy;
  m.u = p.u;
  m.v = p.v;
  ftlm_run_opts o{};
  o.samples = p.samples;
  o.lanczos_steps = p.lanczos_steps;
  o.exact_block_threshold = p.exact_block_threshold;
  o.seed = p.seed;
  o.precision = p.precision;
  o.start_vector = p.start_vector;
  o.batch_vectors = p.batch_vectors;
  o.device = p.device;
  const int st = ftlm_ctx_create(&m, &o, &ctx_);
  if (st != FTLM_OK) {
    if (st == FTLM_ERR_CUDA) die("No usable CUDA device for the GPU engine (device " + std::to_string(p.device) + ").");
    die("Engine rejected the parameters (status " + std::to_string(st) + ").");
  }
  if (!p.profile_json.empty()) check(ftlm_profile_enable(ctx_, 1), "profile_enable");
}

Engine::~Engine() { ftlm_ctx_destroy(ctx_); }

void Engine::check(int status, const char* what) const {
  if (status == FTLM_OK) return;
  char buf[512];
  ftlm_last_error(ctx_, buf, sizeof buf);
  die(std::string("GPU engine ") + what + " failed: " + buf);
}

int run_ftlm_main(int argc, char** argv) {  // main.cpp:1459-1839
  try {
    const auto t0 = std::chrono::steady_clock::now();
    const Params params = parse_args(argc, argv);
    const int sites = params.lx * params.ly;
    const bool multi_beta = params.beta_values.size() > 1;
    const std::vector<double> mu_values = linspace(params.mu_min, params.mu_max, params.mu_count);
    const bool trace_blocks = !params.trace_partition_csv.empty();
    const bool debug_selected_block = params.debug_block_nup >= 0 && params.debug_block_ndown >= 0 &&
                                      params.debug_block_mx >= 0 && params.debug_block_my >= 0;
    if (!params.checkpoint.empty() && (trace_blocks || debug_selected_block))
      die("--checkpoint is not currently compatible with trace/debug block output.");
    validate_or_write_checkpoint_metadata(params);
    ensure_checkpoint_header(params.checkpoint);
    std::map<BlockKey, Spectrum> ckpt;
    for (auto& kv : read_checkpoint(params.checkpoint)) ckpt[kv.first] = std::move(kv.second);

    std::cout << "Reference used: "
              << "reference_ftlm_hub_cond/fltm_hub_cond/hubTri2Dcond_omp.f"
              << " and cond_spect_omp.f\n";
    std::cout << "Running FTLM with translation-symmetry k blocks on a " << params.lx << "x" << params.ly
              << " rectangular lattice (" << sites << " sites)\n";
    std::cout << "beta=";
    for (std::size_t i = 0; i < params.beta_values.size(); ++i) {
      if (i > 0) std::cout << ",";
      std::cout << params.beta_values[i];
    }
    const int threads =
        params.threads > 0 ? params.threads : static_cast<int>(std::max(1u, std::thread::hardware_concurrency()));
    std::cout << " U=" << params.u << " V=" << params.v << " tx=" << params.tx << " ty=" << params.ty
              << " tp=" << params.tp << " phix=" << params.phix << " phiy=" << params.phiy << " threads=" << threads
              << " exact_block_threshold=" << params.exact_block_threshold << "\n";
    if (!params.checkpoint.empty())
      std::cout << "checkpoint=" << params.checkpoint << " loaded_blocks=" << ckpt.size() << "\n";

    Engine eng(params);
    eng.check(ftlm_thermo_configure(eng.ctx(), static_cast<int>(params.beta_values.size()), params.beta_values.data(),
                                    static_cast<int>(mu_values.size()), mu_values.data()),
              "thermo_configure");
    std::ofstream trace_out;
    if (trace_blocks) {
      trace_out.open(params.trace_partition_csv);
      if (!trace_out) die("Failed to open trace CSV: " + params.trace_partition_csv);
      trace_out << "nup,ndown,mx,my,particles,basis_dim,mu,"
                << "method,z_used,z_ed,z_ratio,n_used_total,n_ed_total,n_total_diff,"
                << "n2_used_total,n2_ed_total,n2_total_diff,"
                << "min_ftlm,min_ed,sum_sample_weights\n";
      trace_out << std::setprecision(15);
    }
    bool wrote_debug = false;

    for (int n_up = 0; n_up <= sites; ++n_up) {
      for (int n_down = 0; n_down <= sites; ++n_down) {
        const uint64_t full_dim = n_choose_k(sites, n_up) * n_choose_k(sites, n_down);
        if (full_dim == 0) continue;
        if (full_dim > params.max_sector_dim) {
          std::ostringstream msg;
          msg << "Sector (Nup=" << n_up << ", Ndown=" << n_down << ") has full dimension " << full_dim
              << ", which exceeds --max-sector-dim=" << params.max_sector_dim;
          die(msg.str());
        }
        ftlm_sector_info info{};
        eng.check(ftlm_sector_prepare(eng.ctx(), n_up, n_down, &info), "sector_prepare");
        const int particles = n_up + n_down;
        auto matches = [&](int mx, int my) {
          return debug_selected_block && n_up == params.debug_block_nup && n_down == params.debug_block_ndown &&
                 mx == params.debug_block_mx && my == params.debug_block_my;
        };
        // every exact spectrum this sector needs, in one batched launch
        std::vector<int32_t> ex_mx, ex_my;
        for (int my = 0; my < params.ly; ++my)
          for (int mx = 0; mx < params.lx; ++mx) {
            const uint64_t dim = info.block_dim[my * params.lx + mx];
            if (dim == 0 || ckpt.count(BlockKey{n_up, n_down, mx, my})) continue;
            const bool use_exact = dim <= params.exact_block_threshold;
            if (use_exact || trace_blocks || matches(mx, my)) {
              ex_mx.push_back(mx);
              ex_my.push_back(my);
            }
          }
        eng.check(ftlm_blocks_exact_batched(eng.ctx(), ex_mx.data(), ex_my.data(), static_cast<int>(ex_mx.size())),
                  "blocks_exact_batched");
        // and every FTLM spectrum of blocks without exact/trace/debug output;
        // with a checkpoint only the small ones, so that a large block is
        // still written to the checkpoint as soon as it is done
        std::vector<int32_t> ft_mx, ft_my;
        for (int my = 0; my < params.ly; ++my)
          for (int mx = 0; mx < params.lx; ++mx) {
            const uint64_t dim = info.block_dim[my * params.lx + mx];
            if (dim == 0 || dim <= params.exact_block_threshold || ckpt.count(BlockKey{n_up, n_down, mx, my}) ||
                trace_blocks || matches(mx, my) || (!params.checkpoint.empty() && dim > FTLM_SMALL_BLOCK_MAX))
              continue;
            ft_mx.push_back(mx);
            ft_my.push_back(my);
          }
        eng.check(ftlm_blocks_ftlm_batched(eng.ctx(), ft_mx.data(), ft_my.data(), static_cast<int>(ft_mx.size())),
                  "blocks_ftlm_batched");
        std::size_t active_sum = 0;
        for (int my = 0; my < params.ly; ++my) {
          for (int mx = 0; mx < params.lx; ++mx) {
            const std::size_t dim = static_cast<std::size_t>(info.block_dim[my * params.lx + mx]);
            active_sum += dim;
            if (dim == 0) continue;
            const BlockKey key{n_up, n_down, mx, my};
            auto hit = ckpt.find(key);
            if (hit != ckpt.end()) {  // main.cpp:1541-1567
              const Spectrum& s = hit->second;
              if (s.basis_dim != dim || s.particles != particles)
                die("Checkpoint block metadata does not match current run.");
              eng.check(ftlm_thermo_accumulate_host(eng.ctx(), s.eigenvalues.data(),
                                                    s.sample_weights.empty() ? nullptr : s.sample_weights.data(),
                                                    s.eigenvalues.size(), s.trace_prefactor, s.particles),
                        "thermo_accumulate_host");
              continue;
            }
            const bool use_exact = dim <= params.exact_block_threshold;
            const bool need_exact = use_exact || trace_blocks || matches(mx, my);
            const bool want_host = trace_blocks || matches(mx, my) || !params.checkpoint.empty();
            Spectrum exact_s, ftlm_s;
            exact_s.basis_dim = ftlm_s.basis_dim = dim;
            exact_s.particles = ftlm_s.particles = particles;
            if (need_exact && want_host) fetch(eng, mx, my, 1, exact_s);
            if (!use_exact) {
              if (want_host) {
                fetch(eng, mx, my, 0, ftlm_s);
              } else {
                size_t cnt = 0;
                eng.check(ftlm_block_spectrum(eng.ctx(), mx, my, 0, nullptr, nullptr, 0, &cnt, nullptr),
                          "block_spectrum");
              }
            }
            if (trace_blocks) {  // main.cpp:1583-1608
              const double sw = use_exact ? 1.0
                                          : std::accumulate(ftlm_s.sample_weights.begin(),
                                                            ftlm_s.sample_weights.end(), 0.0);
              for (double mu : mu_values) {
                const BlockThermo used = use_exact
                    ? raw_thermo(exact_s.eigenvalues, nullptr, 1.0, particles, params.beta, mu)
                    : raw_thermo(ftlm_s.eigenvalues, &ftlm_s.sample_weights, static_cast<double>(dim), particles,
                                 params.beta, mu);
                const BlockThermo ex = raw_thermo(exact_s.eigenvalues, nullptr, 1.0, particles, params.beta, mu);
                const double ratio = (ex.z > 0.0) ? (used.z / ex.z) : 0.0;
                trace_out << n_up << "," << n_down << "," << mx << "," << my << "," << particles << "," << dim << ","
                          << mu << "," << (use_exact ? "exact" : "ftlm") << "," << used.z << "," << ex.z << ","
                          << ratio << "," << used.n_total << "," << ex.n_total << ","
                          << (used.n_total - ex.n_total) << "," << used.n2_total << "," << ex.n2_total << ","
                          << (used.n2_total - ex.n2_total) << "," << used.min_shifted_energy << ","
                          << ex.min_shifted_energy << "," << sw << "\n";
              }
            }
            if (matches(mx, my)) {  // main.cpp:1610-1663
              const double sw = use_exact ? 1.0
                                          : std::accumulate(ftlm_s.sample_weights.begin(),
                                                            ftlm_s.sample_weights.end(), 0.0);
              std::cout << "Selected block debug Nup=" << n_up << " Ndown=" << n_down << " mx=" << mx << " my=" << my
                        << " basis_dim=" << dim << " method=" << (use_exact ? "exact" : "ftlm")
                        << " sum_sample_weights=" << sw << "\n";
              for (double mu : mu_values) {
                const BlockThermo used = use_exact
                    ? raw_thermo(exact_s.eigenvalues, nullptr, 1.0, particles, params.beta, mu)
                    : raw_thermo(ftlm_s.eigenvalues, &ftlm_s.sample_weights, static_cast<double>(dim), particles,
                                 params.beta, mu);
                const BlockThermo ex = raw_thermo(exact_s.eigenvalues, nullptr, 1.0, particles, params.beta, mu);
                const double ratio = (ex.z > 0.0) ? (used.z / ex.z) : 0.0;
                std::cout << "  debug mu=" << std::setw(12) << mu << " z_used=" << std::setw(14) << used.z
                          << " z_ed=" << std::setw(14) << ex.z << " ratio=" << std::setw(14) << ratio
                          << " n_diff=" << std::setw(14) << (used.n_total - ex.n_total) << "\n";
              }
              if (!params.debug_block_csv.empty()) {
                Spectrum f = use_exact ? Spectrum{} : ftlm_s;
                f.basis_dim = dim;
                f.particles = particles;
                write_selected_block_debug(params.debug_block_csv, n_up, n_down, mx, my, f, exact_s.eigenvalues,
                                           params.beta, mu_values);
                wrote_debug = true;
              }
            }
            if (!params.checkpoint.empty()) {  // main.cpp:1665-1678
              Spectrum st = use_exact ? exact_s : ftlm_s;
              st.exact = use_exact;
              st.trace_prefactor = use_exact ? 1.0 : static_cast<double>(dim);
              if (use_exact) st.sample_weights.clear();
              append_checkpoint_record(params.checkpoint, key, st);
            }
            eng.check(ftlm_thermo_accumulate_block(eng.ctx(), mx, my), "thermo_accumulate_block");
          }
        }
        std::cout << "  sector Nup=" << n_up << " Ndown=" << n_down << " full_dim=" << info.full_dim
                  << " parents=" << info.parents << " active_k_dim_sum=" << active_sum << "\n";
      }
    }
    if (debug_selected_block && !params.debug_block_csv.empty() && !wrote_debug)
      die("Selected block debug target was not found among active FTLM blocks.");

    const Observables o = finalize(eng, params.beta_values, mu_values.size(), sites);
    for (std::size_t b = 0; b < params.beta_values.size(); ++b)
      for (std::size_t i = 0; i < mu_values.size(); ++i)
        std::cout << "beta=" << std::setw(12) << params.beta_values[b] << "  mu=" << std::setw(12) << mu_values[i]
                  << "  n=" << std::setw(12) << o.n[b][i] << "  kappa=" << std::setw(12) << o.kappa[b][i] << "\n";
    if (multi_beta)
      write_multi_beta_results(params.output, params.beta_values, mu_values, o.n, o.chi, o.kappa, o.z, o.logz);
    else
      write_results(params.output, mu_values, o.n[0], o.chi[0], o.kappa[0], o.z[0], o.logz[0]);
    std::cout << "Wrote " << params.output << "\n";
    write_profile(params, eng,
                  std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count());
    return 0;
  } catch (const std::exception& ex) {
    std::cerr << "Error: " << ex.what() << "\n";
    return 1;
  }
}

int run_ed_main(int argc, char** argv) {  // ed_main.cpp:49-146
  try {
    const auto t0 = std::chrono::steady_clock::now();
    const Params params = parse_args(argc, argv);
    const int sites = params.lx * params.ly;
    const std::vector<double> mu_values = linspace(params.mu_min, params.mu_max, params.mu_count);
    std::cout << "Exact diagonalization using the FTLM sector and k-block builder\n";
    std::cout << "Running ED on a " << params.lx << "x" << params.ly << " rectangular lattice (" << sites
              << " sites)\n";
    std::cout << "beta=" << params.beta << " U=" << params.u << " V=" << params.v << " tx=" << params.tx
              << " ty=" << params.ty << " tp=" << params.tp << " phix=" << params.phix << " phiy=" << params.phiy
              << "\n";
    Engine eng(params);
    const std::vector<double> betas = {params.beta};
    eng.check(ftlm_thermo_configure(eng.ctx(), 1, betas.data(), static_cast<int>(mu_values.size()), mu_values.data()),
              "thermo_configure");
    for (int n_up = 0; n_up <= sites; ++n_up) {
      for (int n_down = 0; n_down <= sites; ++n_down) {
        const uint64_t full_dim = n_choose_k(sites, n_up) * n_choose_k(sites, n_down);
        if (full_dim == 0) continue;
        if (full_dim > params.max_sector_dim) {
          std::ostringstream msg;
          msg << "Sector (Nup=" << n_up << ", Ndown=" << n_down << ") has full dimension " << full_dim
              << ", which exceeds --max-sector-dim=" << params.max_sector_dim;
          die(msg.str());
        }
        ftlm_sector_info info{};
        eng.check(ftlm_sector_prepare(eng.ctx(), n_up, n_down, &info), "sector_prepare");
        std::vector<int32_t> ex_mx, ex_my;
        std::size_t active_sum = 0;
        for (int my = 0; my < params.ly; ++my)
          for (int mx = 0; mx < params.lx; ++mx) {
            const uint64_t dim = info.block_dim[my * params.lx + mx];
            active_sum += dim;
            if (dim == 0) continue;
            ex_mx.push_back(mx);
            ex_my.push_back(my);
          }
        eng.check(ftlm_blocks_exact_batched(eng.ctx(), ex_mx.data(), ex_my.data(), static_cast<int>(ex_mx.size())),
                  "blocks_exact_batched");
        for (std::size_t i = 0; i < ex_mx.size(); ++i)
          eng.check(ftlm_thermo_accumulate_block(eng.ctx(), ex_mx[i], ex_my[i]), "thermo_accumulate_block");
        std::cout << "  sector Nup=" << n_up << " Ndown=" << n_down << " full_dim=" << info.full_dim
                  << " parents=" << info.parents << " active_k_dim_sum=" << active_sum << "\n";
      }
    }
    const Observables o = finalize(eng, betas, mu_values.size(), sites);
    for (std::size_t i = 0; i < mu_values.size(); ++i)
      std::cout << "mu=" << std::setw(12) << mu_values[i] << "  n=" << std::setw(12) << o.n[0][i]
                << "  kappa=" << std::setw(12) << o.kappa[0][i] << "\n";
    write_results(params.output, mu_values, o.n[0], o.chi[0], o.kappa[0], o.z[0], o.logz[0]);
    std::cout << "Wrote " << params.output << "\n";
    write_profile(params, eng, std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count());
    return 0;
  } catch (const std::exception& ex) {
    std::cerr << "Error: " << ex.what() << "\n";
    return 1;
  }
}

}  // namespace ftlm_cli
