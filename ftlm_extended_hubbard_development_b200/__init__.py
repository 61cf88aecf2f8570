"""B200-native FTLM engine for the extended Hubbard model (drop-in for the
ftlm_n_vs_mu / ftlm_ed_n_vs_mu executables). The compute path is the CUDA
library lib/libftlm_gpu.so; see engine.py for its Python view."""
from .engine import (BIN_DIR, LIB_PATH, Engine, FtlmError, Model, RunOpts, linspace,  # noqa: F401
                     load_library, run_curve)
