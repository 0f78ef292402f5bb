"""B200-native Harvest F0 estimator.

A drop-in for the reference package's API (``harvest``, ``cuda_available``,
``clear_cache``) backed by hand-written sm_100a CUDA kernels behind the C ABI
of ``include/harvest_b200.h``, plus a ragged batched path.
"""
from .api import (clear_cache, cuda_available, harvest, harvest_batch, harvest_batch_pcm16,
                  harvest_many, output_length, profile)

__version__ = "0.1.0"
__all__ = ["harvest", "harvest_batch", "harvest_batch_pcm16", "harvest_many", "cuda_available",
           "clear_cache", "output_length", "profile", "__version__"]
