"""astro_transit_gpu_b200 -- B200-native Box Least Squares transit search.

Drop-in for the BLS hot path of ubunbun18/Astro_Transit_GPU
(``BoxLeastSquaresGPU(t, y, dy).power(periods, durations, method=...)``),
computed by hand-written sm_100a kernels behind a C ABI
(``include/astrotransit_b200.h``).  There is no CPU fallback: without a CUDA
device and the built library every compute entry point raises.
"""
from .api import BLSResult, BoxLeastSquaresGPU, Candidate, power_batch
from .gpu_bls import get_top_k_candidates, run_gpu_bls
from .v42_parity import run_vbls_exact_parity

__version__ = "0.1.0"
__all__ = [
    "BoxLeastSquaresGPU", "BLSResult", "Candidate", "power_batch", "run_gpu_bls",
    "get_top_k_candidates", "run_vbls_exact_parity",
]
