"""crava_b200 -- B200 (sm_100a) Fourier-domain Bayesian AVO inversion hot path.

The computation lives in the in-tree CUDA library lib/libcrava_gpu.so behind
the C ABI of include/crava_gpu.h; api.py binds it for Python callers,
synth.py builds seeded synthetic cases in the reference's grid layout,
dist.py holds the rank plumbing of independent units over several GPUs and
dist_grid.py splits one grid over several GPUs; loglik.py wraps the
log-likelihood adjoint for torch.autograd.
"""
from .api import (COVARIANCE, DATA, FP32, FP64, MIXED, PARAMETER, Context, Crava,  # noqa: F401
                  CravaGpuError, FFTGrid, complex_view, launch_count, load_library, to_device)
