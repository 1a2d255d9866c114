"""B200-native HIT-Leiden incremental update path.

The compute path is libhl.so (hand-written sm_100a CUDA kernels behind the C
ABI in include/hl.h); this package is its Python host-side mirror of the
reference crate's API.  Importing it fails loudly if the library is missing.
"""
from ._lib import HitLeidenError, BatchStats  # noqa: F401  (loads libhl.so)
from .api import (GraphInput, PartitionResult, PartitionState, RunConfig, RunMode,  # noqa: F401
                  RunOutcome, Server, apply_batches, canonicalize_community_ids,
                  compute_modularity, hit_leiden, run)

__all__ = ["GraphInput", "PartitionResult", "PartitionState", "RunConfig", "RunMode", "RunOutcome",
           "HitLeidenError", "BatchStats", "canonicalize_community_ids", "compute_modularity",
           "hit_leiden", "run", "apply_batches", "Server"]
