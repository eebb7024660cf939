"""B200-native batched banded seed extension and mate-rescue Smith-Waterman.

A drop-in for FerrousAlign's batch-extension call (execute_batch_simd_scoring), the
region merge that consumes its results (merge_scores_to_regions) and its mate-rescue
ksw_align2 calls, computed by hand-written sm_100a CUDA kernels behind the C ABI in
include/ferrous_b200.h.
"""
from ._native import Context, NativeError, default_context, load  # noqa: F401
from .batch_extension import (BandedPairWiseSW, BatchedExtensionJob, BatchExtensionResult,  # noqa: F401
                              ExtensionDirection, ExtensionJobBatch, bwa_fill_scmat,
                              execute_batch_simd_scoring, extend_batch, make_policy)
from .mate_rescue import (MATE_RESCUE_SCORING_MATRIX, Kswr, MateRescueJob, MateRescueResult,  # noqa: F401
                          execute_mate_rescue_batch_with_engine, make_mate_params, mate_sw_batch,
                          mate_sw_batch_packed,
                          mate_xtra)
from .region import chain_seed_table, merge_scores_to_regions, region_opts  # noqa: F401
from .hostbuf import HostBuffers  # noqa: F401
from .collect import (CollectBuffers, CollectedJobs, collect_extension_jobs, collect_extension_jobs_packed,  # noqa: F401
                      collect_opts, pack_reference)
from .cigar import CigarBatch, infer_band_width, scalar_banded_swa_batch  # noqa: F401
from .pair_batch import pair_batch  # noqa: F401
from .packed import PackedSeq, extend_batch_learned_packed, extend_batch_packed, pack, unpack  # noqa: F401

__version__ = "0.1.0"
