// Drop-in replacement for the reference's ftlm_n_vs_mu executable
// (src/main.cpp:1459-1839): same flags, CSV and checkpoint formats; the
// hot path runs on the GPU through libftlm_gpu.
#include "cli_common.h"

int main(int argc, char** argv) { return ftlm_cli::run_ftlm_main(argc, argv); }
