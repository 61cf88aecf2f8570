// Drop-in replacement for the reference's ftlm_ed_n_vs_mu executable
// (src/ed_main.cpp:49-146): every (N_up, N_down, k) block is diagonalised
// exactly by the GPU's batched dense eigen-solver.
#include "cli_common.h"

int main(int argc, char** argv) { return ftlm_cli::run_ed_main(argc, argv); }
