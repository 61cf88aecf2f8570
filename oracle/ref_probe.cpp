// Reference probe: test infrastructure only.
//
// Compiles the reference's own src/main.cpp (included by path from the
// reference checkout, never copied) with its `main` renamed, and dumps the
// internal objects of the FTLM hot path as .npy files so that the restated
// oracle (oracle/ftlm_oracle.c) and the CUDA engine can be pinned against
// the reference's exact basis, relations, CSR blocks, Lanczos coefficients,
// FTLM spectra and exact eigenvalues.
//
// Usage:
//   ref_probe sector  OUTDIR NUP NDOWN            -- <reference flags>
//   ref_probe lanczos OUTDIR NUP NDOWN MX MY      -- <reference flags>
//   ref_probe exact   OUTDIR NUP NDOWN MX MY      -- <reference flags>
//
// The reference flags are parsed by the reference's own parse_args
// (src/main.cpp:257-368).
#define main ftlm_reference_main
#include "main.cpp"
#undef main

#include <cstdio>
#include <sys/stat.h>

namespace probe {

// Minimal .npy (format 1.0) writer for 1-D arrays.
template <typename T>
const char* npy_descr();
template <> const char* npy_descr<double>() { return "<f8"; }
template <> const char* npy_descr<std::int32_t>() { return "<i4"; }
template <> const char* npy_descr<std::int64_t>() { return "<i8"; }
template <> const char* npy_descr<std::uint64_t>() { return "<u8"; }

template <typename T>
void write_npy(const std::string& path, const T* data, std::size_t n) {
  std::string header = std::string("{'descr': '") + npy_descr<T>() +
                       "', 'fortran_order': False, 'shape': (" + std::to_string(n) + ",), }";
  std::size_t total = 10 + header.size() + 1;
  std::size_t pad = (64 - total % 64) % 64;
  header.append(pad, ' ');
  header.push_back('\n');
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) throw std::runtime_error("cannot write " + path);
  const unsigned char magic[8] = {0x93, 'N', 'U', 'M', 'P', 'Y', 1, 0};
  std::fwrite(magic, 1, 8, f);
  const std::uint16_t hlen = static_cast<std::uint16_t>(header.size());
  std::fwrite(&hlen, 2, 1, f);
  std::fwrite(header.data(), 1, header.size(), f);
  if (n) std::fwrite(data, sizeof(T), n, f);
  std::fclose(f);
}

template <typename T>
void write_vec(const std::string& dir, const std::string& name, const std::vector<T>& v) {
  write_npy(dir + "/" + name + ".npy", v.data(), v.size());
}

void write_complex(const std::string& dir, const std::string& name, const std::vector<Complex>& v) {
  std::vector<double> flat;
  flat.reserve(2 * v.size());
  for (const Complex& c : v) {
    flat.push_back(c.real());
    flat.push_back(c.imag());
  }
  write_vec(dir, name, flat);
}

// Sector dump: parents, relations for every state in (up-rank, down-rank)
// order, and the CSR of every momentum block.
void dump_sector(const std::string& dir, const Params& params, int n_up, int n_down) {
  const Lattice lattice = build_lattice(params.lx, params.ly);
  const SectorBasis sector = build_sector_basis(lattice, n_up, n_down, params);
  std::vector<std::uint64_t> p_up, p_dn;
  std::vector<std::int32_t> p_deg;
  std::vector<double> p_diag;
  std::vector<std::int64_t> hop_count;
  for (const ParentData& p : sector.parents) {
    p_up.push_back(p.representative.up);
    p_dn.push_back(p.representative.down);
    p_deg.push_back(p.degeneracy);
    p_diag.push_back(p.diagonal);
    hop_count.push_back(static_cast<std::int64_t>(p.hops.size()));
  }
  write_vec(dir, "parent_up", p_up);
  write_vec(dir, "parent_down", p_dn);
  write_vec(dir, "parent_deg", p_deg);
  write_vec(dir, "parent_diag", p_diag);
  write_vec(dir, "parent_hops", hop_count);

  // Relations (parent, shift, sign) of every state. The reference keeps them
  // in a local map inside build_sector_basis (main.cpp:640-675); they are
  // recovered here through the public pieces: the first translation of each
  // representative that produces the state.
  const auto ups = generate_combinations(lattice.sites, n_up);
  const auto dns = generate_combinations(lattice.sites, n_down);
  std::unordered_map<StateKey, std::int32_t, StateKeyHash> rep_index;
  for (std::size_t i = 0; i < sector.parents.size(); ++i) {
    rep_index[sector.parents[i].representative] = static_cast<std::int32_t>(i);
  }
  std::unordered_map<StateKey, std::array<std::int32_t, 3>, StateKeyHash> rel;
  for (std::size_t i = 0; i < sector.parents.size(); ++i) {
    const StateKey r = sector.parents[i].representative;
    rel[r] = {static_cast<std::int32_t>(i), 0, 1};
    for (int dy = 0; dy < lattice.ly; ++dy) {
      for (int dx = 0; dx < lattice.lx; ++dx) {
        int sign = 1;
        const StateKey t = translate_state(r, dx, dy, lattice.lx, lattice.ly, sign);
        if (!(t == r) && rel.find(t) == rel.end()) {
          rel[t] = {static_cast<std::int32_t>(i), dy * lattice.lx + dx, sign};
        }
      }
    }
  }
  std::vector<std::int32_t> r_parent, r_shift, r_sign;
  for (auto u : ups) {
    for (auto d : dns) {
      const auto& e = rel.at(StateKey{u, d});
      r_parent.push_back(e[0]);
      r_shift.push_back(e[1]);
      r_sign.push_back(e[2]);
    }
  }
  write_vec(dir, "rel_parent", r_parent);
  write_vec(dir, "rel_shift", r_shift);
  write_vec(dir, "rel_sign", r_sign);

  // Momentum blocks in the reference's loop order (my outer, mx inner).
  std::vector<std::int64_t> dims, nnzs;
  for (int my = 0; my < lattice.ly; ++my) {
    for (int mx = 0; mx < lattice.lx; ++mx) {
      const MomentumBlock b = build_momentum_block(sector, lattice, mx, my);
      dims.push_back(static_cast<std::int64_t>(b.basis_dim));
      nnzs.push_back(static_cast<std::int64_t>(b.col_idx.size()));
      const std::string tag = "_k" + std::to_string(mx) + "_" + std::to_string(my);
      write_vec(dir, "diag" + tag, b.diagonal);
      std::vector<std::int32_t> rp(b.row_ptr.begin(), b.row_ptr.end());
      std::vector<std::int32_t> ci(b.col_idx.begin(), b.col_idx.end());
      write_vec(dir, "row_ptr" + tag, rp);
      write_vec(dir, "col" + tag, ci);
      write_complex(dir, "val" + tag, b.values);
    }
  }
  write_vec(dir, "block_dim", dims);
  write_vec(dir, "block_nnz", nnzs);
  std::vector<std::int64_t> meta = {static_cast<std::int64_t>(sector.full_dim),
                                    static_cast<std::int64_t>(sector.parents.size())};
  write_vec(dir, "sector_meta", meta);
}

// Lanczos dump: the start vectors, per-sample alpha/beta and the spectrum
// returned by the reference's run_ftlm_block (main.cpp:996-1113). The
// alpha/beta recurrence is re-driven here through the reference's own
// apply_hamiltonian / dot / complex_norm2 so the coefficients can be
// recorded; the spectrum comes from the untouched reference function.
void dump_lanczos(const std::string& dir, const Params& params, int n_up, int n_down, int mx, int my) {
  const Lattice lattice = build_lattice(params.lx, params.ly);
  const SectorBasis sector = build_sector_basis(lattice, n_up, n_down, params);
  const MomentumBlock block = build_momentum_block(sector, lattice, mx, my);
  const std::uint64_t seed = make_block_seed(params, n_up, n_down, mx, my);
  const std::size_t dim = block.basis_dim;
  const int kdim = std::min<int>(params.lanczos_steps, static_cast<int>(dim));

  std::vector<Complex> starts;
  std::vector<double> alphas, betas;
  std::vector<std::int32_t> steps;
  for (int s = 0; s < params.samples; ++s) {
    std::mt19937_64 rng(mix_u64(seed ^ static_cast<std::uint64_t>(s)));
    std::normal_distribution<double> normal(0.0, 1.0);
    std::vector<Complex> q(dim), qp(dim, 0.0), w(dim), hq(dim);
    for (Complex& v : q) v = Complex(normal(rng), normal(rng));
    normalize(q);
    starts.insert(starts.end(), q.begin(), q.end());
    double bprev = 0.0;
    int taken = 0;
    std::vector<double> a_s(static_cast<std::size_t>(kdim), 0.0), b_s(static_cast<std::size_t>(kdim), 0.0);
    for (int j = 0; j < kdim; ++j) {
      apply_hamiltonian(block, q, hq);
      const double a = dot(q, hq).real();
      for (std::size_t i = 0; i < dim; ++i) w[i] = hq[i] - a * q[i] - bprev * qp[i];
      a_s[static_cast<std::size_t>(j)] = a;
      const double b = std::sqrt(complex_norm2(w));
      ++taken;
      if (b < 1e-12 || j + 1 == kdim) break;
      b_s[static_cast<std::size_t>(j)] = b;
      qp.swap(q);
      q.swap(w);
      for (Complex& v : q) v /= b;
      bprev = b;
    }
    alphas.insert(alphas.end(), a_s.begin(), a_s.end());
    betas.insert(betas.end(), b_s.begin(), b_s.end());
    steps.push_back(taken);
  }
  write_complex(dir, "start", starts);
  write_vec(dir, "alpha", alphas);
  write_vec(dir, "beta", betas);
  write_vec(dir, "steps", steps);

  const LanczosSpectrum spec = run_ftlm_block(block, params, seed);
  write_vec(dir, "ritz", spec.eigenvalues);
  write_vec(dir, "weights", spec.sample_weights);
  std::vector<std::int64_t> meta = {static_cast<std::int64_t>(dim), kdim,
                                    static_cast<std::int64_t>(seed)};
  write_vec(dir, "lanczos_meta", meta);
}

void dump_exact(const std::string& dir, const Params& params, int n_up, int n_down, int mx, int my) {
  const Lattice lattice = build_lattice(params.lx, params.ly);
  const SectorBasis sector = build_sector_basis(lattice, n_up, n_down, params);
  const MomentumBlock block = build_momentum_block(sector, lattice, mx, my);
  write_vec(dir, "exact", diagonalize_block_exact(block));
}

}  // namespace probe

int main(int argc, char** argv) {
  try {
    if (argc < 5) {
      std::cerr << "usage: ref_probe MODE OUTDIR NUP NDOWN [MX MY] -- flags\n";
      return 2;
    }
    const std::string mode = argv[1];
    const std::string dir = argv[2];
    mkdir(dir.c_str(), 0755);
    int sep = 3;
    while (sep < argc && std::string(argv[sep]) != "--") ++sep;
    std::vector<int> nums;
    for (int i = 3; i < sep; ++i) nums.push_back(std::atoi(argv[i]));
    std::vector<char*> fwd = {argv[0]};
    for (int i = sep + 1; i < argc; ++i) fwd.push_back(argv[i]);
    const Params params = parse_args(static_cast<int>(fwd.size()), fwd.data());
    if (mode == "sector" && nums.size() == 2) {
      probe::dump_sector(dir, params, nums[0], nums[1]);
    } else if (mode == "lanczos" && nums.size() == 4) {
      probe::dump_lanczos(dir, params, nums[0], nums[1], nums[2], nums[3]);
    } else if (mode == "exact" && nums.size() == 4) {
      probe::dump_exact(dir, params, nums[0], nums[1], nums[2], nums[3]);
    } else {
      std::cerr << "bad mode/arguments\n";
      return 2;
    }
    return 0;
  } catch (const std::exception& ex) {
    std::cerr << "Error: " << ex.what() << "\n";
    return 1;
  }
}
