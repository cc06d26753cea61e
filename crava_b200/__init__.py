"""crava_b200 -- B200 (sm_100a) Fourier-domain Bayesian AVO inversion hot path.

The computation lives in the in-tree CUDA library lib/libcrava_gpu.so behind
the C ABI of include/crava_gpu.h; api.py binds it for Python callers and
synth.py builds seeded synthetic cases in the reference's grid layout.
"""
from .api import (COVARIANCE, DATA, FP32, FP64, MIXED, PARAMETER, Context, Crava,  # noqa: F401
                  CravaGpuError, FFTGrid, complex_view, launch_count, load_library, to_device)
