"""snapmrf_b200: B200-native (sm_100a) MRF dictionary generation and
template matching behind the C ABI of libsnapmrf.so (include/snapmrf.h)."""
from .api import (  # noqa: F401
    DICT_ALL_B1_BLOCKS, DICT_IMAG_ROWS, DICT_NORMALIZE, DICT_NORMALIZE_OPERAND, DICT_REFERENCE_ORDER, DICT_SEPARATE_RELAX, ECHO_TYPES, MATCH_ASSUME_UNIFORM_B1, MATCH_IMAG_ATOMS,
    MATCH_IMAG_ROWS, MATCH_UPLOAD_EARLY, START_IMAG_ATOMS, START_IMAG_ROWS, refine_start, scratch_allocations, selftest_bounded_wait,
    NMAPS, NOALLOC_MAX_B1_BLOCKS, NOALLOC_MAX_VOXELS, NPARAMS, PREC_BF16, PREC_FP16, PREC_FP32, PREC_FP8, SnapMRFError, MRF_dict,
    MRF_match, MRF_match_noalloc, compute_natoms, csv_dim,
    csv_read, crb_gradient, device_error, epg_adjoint, epg_jvp, grid_params, refine_gn, kernel_launches, lib, packed_pitch, linspace, logspace, normalize, parse_length, parse_params,
    parse_range, ra_read, ra_write, trans_params, Compressed, SVD_IMAG_ATOMS, SVD_MAX_SUBSPACE, svd_compress,
)
