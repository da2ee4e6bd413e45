"""ironav_b200 — IronAV's H.264 P-picture inter-analysis stage on NVIDIA B200 (sm_100a).

The stage (half-sample planes, P_Skip test, motion search, partition decision) runs as CUDA kernels
behind the C ABI of include/ironav_inter.h; `inter.InterStage` is its Python binding and
`synth.Sequence` generates the seeded synthetic inputs of the benchmark configurations.
"""
from .inter import (MBRESULT_DTYPE, MBSTATE_DTYPE, RESULT_INTER, RESULT_SKIP, InterStage, IronavError,
                    cuda_library, default_bands, load_library, reference_slices)

__all__ = [
    "InterStage", "IronavError", "MBSTATE_DTYPE", "MBRESULT_DTYPE", "RESULT_INTER", "RESULT_SKIP",
    "cuda_library", "load_library", "default_bands", "reference_slices",
]
