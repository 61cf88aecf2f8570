// Reference CPU timing harness (TEST / BASELINE INFRASTRUCTURE ONLY).
//
// Compiles the reference's own src/main.cpp (included by path, never copied)
// and times its hot path on one momentum block, for the CPU baseline beside
// the GPU engine:
//   ref_bench hv    NUP NDOWN MX MY NVEC SWEEPS -- <reference flags>
//       apply_hamiltonian (main.cpp:833-845) on NVEC vectors, parallel over
//       vectors with OpenMP exactly as run_ftlm_block parallelises over
//       samples (main.cpp:1011-1013); SWEEPS timed sweeps.
//   ref_bench block NUP NDOWN MX MY -- <reference flags>
//       run_ftlm_block (main.cpp:996-1113) on the block, timed once.
// Prints one JSON line with the block size, the CSR entry counts and the
// wall seconds of the timed region. Sector/block construction is setup and
// is reported separately.
#define main ftlm_reference_main
#include "main.cpp"
#undef main

#include <chrono>
#include <cstdio>

int main(int argc, char** argv) {
  try {
    if (argc < 6) {
      std::cerr << "usage: ref_bench hv|block NUP NDOWN MX MY [NVEC SWEEPS] -- flags\n";
      return 2;
    }
    const std::string mode = argv[1];
    int sep = 2;
    while (sep < argc && std::string(argv[sep]) != "--") ++sep;
    std::vector<long> nums;
    for (int i = 2; i < sep; ++i) nums.push_back(std::atol(argv[i]));
    std::vector<char*> fwd = {argv[0]};
    for (int i = sep + 1; i < argc; ++i) fwd.push_back(argv[i]);
    const Params params = parse_args(static_cast<int>(fwd.size()), fwd.data());
    const int n_up = static_cast<int>(nums.at(0)), n_down = static_cast<int>(nums.at(1));
    const int mx = static_cast<int>(nums.at(2)), my = static_cast<int>(nums.at(3));
    using clk = std::chrono::steady_clock;
    const auto t0 = clk::now();
    const Lattice lattice = build_lattice(params.lx, params.ly);
    const SectorBasis sector = build_sector_basis(lattice, n_up, n_down, params);
    const MomentumBlock block = build_momentum_block(sector, lattice, mx, my);
    const double setup = std::chrono::duration<double>(clk::now() - t0).count();
    std::size_t nnz_nonzero = 0;
    for (const Complex& v : block.values) nnz_nonzero += (v != Complex(0.0, 0.0));
    const int threads = requested_omp_threads(params);
    double seconds = 0.0;
    long nvec = 0, sweeps = 0;
    std::vector<double> sweep_s;
    if (mode == "hv") {
      nvec = nums.at(4);
      sweeps = nums.at(5);
      std::vector<std::vector<Complex>> in(static_cast<std::size_t>(nvec)), out(static_cast<std::size_t>(nvec));
      for (long v = 0; v < nvec; ++v) {
        std::mt19937_64 rng(static_cast<std::uint64_t>(v) + 1);
        std::normal_distribution<double> nd(0.0, 1.0);
        in[v].resize(block.basis_dim);
        out[v].assign(block.basis_dim, 0.0);
        for (Complex& z : in[v]) z = Complex(nd(rng), nd(rng));
      }
      const auto t1 = clk::now();
      for (long s = 0; s < sweeps; ++s) {
        const auto ts = clk::now();
#if defined(_OPENMP)
#pragma omp parallel for schedule(static) num_threads(threads)
#endif
        for (long v = 0; v < nvec; ++v) apply_hamiltonian(block, in[v], out[v]);
        sweep_s.push_back(std::chrono::duration<double>(clk::now() - ts).count());
      }
      seconds = std::chrono::duration<double>(clk::now() - t1).count();
    } else if (mode == "block") {
      const auto t1 = clk::now();
      const LanczosSpectrum spec = run_ftlm_block(block, params, make_block_seed(params, n_up, n_down, mx, my));
      seconds = std::chrono::duration<double>(clk::now() - t1).count();
      nvec = params.samples;
      sweeps = static_cast<long>(spec.eigenvalues.size());
    } else {
      std::cerr << "bad mode\n";
      return 2;
    }
    std::string per = "[";
    for (std::size_t i = 0; i < sweep_s.size(); ++i) per += (i ? ", " : "") + std::to_string(sweep_s[i]);
    per += "]";
    std::printf(
        "{\"mode\": \"%s\", \"dim\": %zu, \"nnz\": %zu, \"nnz_nonzero\": %zu, \"full_dim\": %zu, "
        "\"threads\": %d, \"nvec\": %ld, \"sweeps\": %ld, \"setup_s\": %.6f, \"seconds\": %.6f, "
        "\"sweep_seconds\": %s}\n",
        mode.c_str(), block.basis_dim, block.col_idx.size(), nnz_nonzero, sector.full_dim, threads, nvec, sweeps,
        setup, seconds, per.c_str());
    return 0;
  } catch (const std::exception& ex) {
    std::cerr << "Error: " << ex.what() << "\n";
    return 1;
  }
}
