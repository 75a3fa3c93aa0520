"""B200 (sm_100a) implementation of CURC's pseudogenome compression path.

The compute path is libcurc_b200.so (CUDA kernels behind the C-ABI in
include/curc_b200.h); this package is a thin host-side binding used by the
tests and the benchmark.
"""
from ._native import (Context, CurcError, LIB_PATH, Learner, archive_info, decompress_file,  # noqa: F401
                      fastq_blocks, general_mismatch_bytes, kernel_launches, learn_param_count, lib,
                      plain_mismatch_bytes)

RECORD_DTYPE = None


def _record_dtype():
    import numpy as np
    return np.dtype([("read_id", "<u4"), ("is_n", "u1"), ("strand", "u1"), ("pad", "<u2"), ("pos", "<u8")])


def record_dtype():
    """Layout of a pseudogenome record (compress.cu:68-77 AlignmentRecord)."""
    global RECORD_DTYPE
    if RECORD_DTYPE is None:
        RECORD_DTYPE = _record_dtype()
    return RECORD_DTYPE
