"""The reference's CSV-driven test cases for the batched LU chain, restated as data.

Sources (hicann/ops-blas):
  GETRF: test/getrf_batched/sgetrf_batched/arch35/sgetrf_batched_test.csv:2-33
  GETRS: test/getrs_batched/arch35/getrs_batched_test.csv:2-48
  GETRI: test/getri_batched/sgetri_batched/arch35/sgetri_batched_test.csv:2-48
Matrix types are the generators of test/frame/fill.h:587-740 (oracle/case_inputs.cpp).
"""
from __future__ import annotations

from collections import namedtuple

GetrfCase = namedtuple("GetrfCase", "name n lda batch pivot mtype status seed")
GetrsCase = namedtuple("GetrsCase", "name trans n nrhs lda ldb batch pivot mtype status info_null seed")
GetriCase = namedtuple("GetriCase", "name n lda ldc batch pivot mtype status seed")

S, IV, HN, IE = "SUCCESS", "INVALID_VALUE", "HANDLE_IS_NULLPTR", "INVALID_ENUM"
RN = "RANDOM_NONSINGULAR"

GETRF = [
    GetrfCase("TC_L0_01", 64, 64, 4, True, RN, S, 42),
    GetrfCase("TC_L0_02", 64, 64, 4, False, RN, S, 42),
    GetrfCase("TC_L0_03", 1, 1, 1, True, RN, S, 42),
    GetrfCase("TC_L0_04", 0, 1, 4, True, RN, S, 0),
    GetrfCase("TC_L0_05", 32, 32, 0, True, RN, S, 0),
    GetrfCase("TC_L0_06", 32, 32, 4, True, "SINGULAR_ZERO_COL", S, 42),
    GetrfCase("TC_L0_07", 32, 32, 16, True, RN, S, 42),
    GetrfCase("TC_L0_08", 32, 48, 4, True, RN, S, 42),
    GetrfCase("TC_L0_09", 128, 128, 4, True, RN, S, 42),
    GetrfCase("TC_L0_10", 2, 2, 4, True, RN, S, 42),
    GetrfCase("TC_L1_01", 256, 256, 2, True, RN, S, 42),
    GetrfCase("TC_L1_02", 257, 257, 2, True, RN, S, 42),
    GetrfCase("TC_L1_03", 512, 512, 1, True, RN, S, 42),
    GetrfCase("TC_L1_04", 32, 32, 1, True, RN, S, 42),
    GetrfCase("TC_L1_05", 16, 16, 64, True, RN, S, 99),
    GetrfCase("TC_L1_06", 32, 32, 4, True, "MIXED", S, 42),
    GetrfCase("TC_L1_07", 32, 32, 4, True, "IDENTITY", S, 42),
    GetrfCase("TC_L1_08", 64, 64, 4, True, "DIAGONALLY_DOMINANT", S, 42),
    GetrfCase("TC_L1_09", 4, 4, 4, True, "ILL_CONDITIONED", S, 42),
    GetrfCase("TC_L1_10", 64, 64, 4, False, "DIAGONALLY_DOMINANT", S, 42),
    GetrfCase("TC_L1_11", 16, 128, 4, True, RN, S, 42),
    GetrfCase("TC_L1_12", 1, 1, 4, True, RN, S, 42),
    GetrfCase("TC_L1_13", 32, 32, 4, True, "SINGULAR_DEPENDENT_ROW", S, 42),
    GetrfCase("TC_L1_14", 1, 1, 1, False, RN, S, 42),
    GetrfCase("TC_L1_15", 3, 3, 4, True, RN, S, 42),
]
# Error rows (TC_L1_E01..E07): (name, n, lda, batch, null_aarray, null_info, null_handle, status)
GETRF_ERRORS = [
    ("TC_L1_E01", -1, 1, 4, False, False, False, IV),
    ("TC_L1_E02", 32, 32, -1, False, False, False, IV),
    ("TC_L1_E03", 5, 3, 4, False, False, False, IV),
    ("TC_L1_E04", 0, 0, 4, False, False, False, IV),
    ("TC_L1_E05", 32, 32, 4, True, False, False, IV),
    ("TC_L1_E06", 32, 32, 4, False, True, False, IV),
    ("TC_L1_E07", 32, 32, 4, False, False, True, HN),
]

GETRS = [
    GetrsCase("TC_L0_01", "N", 64, 4, 64, 64, 4, True, RN, S, False, 42),
    GetrsCase("TC_L0_02", "T", 64, 4, 64, 64, 4, True, RN, S, False, 42),
    GetrsCase("TC_L0_03", "C", 64, 4, 64, 64, 4, True, RN, S, False, 42),
    GetrsCase("TC_L0_04", "N", 64, 4, 64, 64, 4, False, RN, S, False, 42),
    GetrsCase("TC_L0_05", "N", 1, 1, 1, 1, 1, True, RN, S, False, 42),
    GetrsCase("TC_L0_06", "N", 2, 2, 2, 2, 4, True, RN, S, False, 42),
    GetrsCase("TC_L0_07", "N", 0, 4, 1, 1, 4, True, RN, S, False, 0),
    GetrsCase("TC_L0_08", "N", 32, 0, 32, 32, 4, True, RN, S, False, 0),
    GetrsCase("TC_L0_09", "N", 32, 4, 32, 32, 0, True, RN, S, False, 0),
    GetrsCase("TC_L0_10", "N", 32, 4, 32, 32, 16, True, RN, S, False, 42),
    GetrsCase("TC_L0_11", "N", 32, 4, 48, 32, 4, True, RN, S, False, 42),
    GetrsCase("TC_L0_12", "N", 128, 8, 128, 128, 4, True, RN, S, False, 42),
    GetrsCase("TC_L0_13", "N", 1024, 4, 1024, 1024, 2, True, RN, S, False, 42),
    GetrsCase("TC_L0_14", "N", 2048, 2, 2048, 2048, 1, True, RN, S, False, 42),
    GetrsCase("TC_L1_01", "N", 4, 4, 4, 4, 4, True, RN, S, False, 42),
    GetrsCase("TC_L1_02", "N", 8, 4, 8, 8, 4, True, RN, S, False, 42),
    GetrsCase("TC_L1_03", "N", 16, 4, 16, 16, 4, True, RN, S, False, 42),
    GetrsCase("TC_L1_04", "N", 32, 4, 32, 32, 4, True, RN, S, False, 42),
    GetrsCase("TC_L1_05", "N", 256, 4, 256, 256, 2, True, RN, S, False, 42),
    GetrsCase("TC_L1_06", "N", 512, 4, 512, 512, 1, True, RN, S, False, 42),
    GetrsCase("TC_L1_07", "N", 4096, 1, 4096, 4096, 1, True, RN, S, False, 42),
    GetrsCase("TC_L1_08", "N", 257, 4, 257, 257, 2, True, RN, S, False, 42),
    GetrsCase("TC_L1_09", "N", 32, 1, 32, 32, 4, True, RN, S, False, 42),
    GetrsCase("TC_L1_10", "N", 32, 2, 32, 32, 4, True, RN, S, False, 42),
    GetrsCase("TC_L1_11", "N", 32, 8, 32, 32, 4, True, RN, S, False, 42),
    GetrsCase("TC_L1_12", "N", 32, 16, 32, 32, 4, True, RN, S, False, 42),
    GetrsCase("TC_L1_13", "N", 32, 4, 32, 32, 1, True, RN, S, False, 42),
    GetrsCase("TC_L1_14", "N", 16, 4, 16, 16, 8, True, RN, S, False, 42),
    GetrsCase("TC_L1_15", "N", 16, 4, 16, 16, 32, True, RN, S, False, 42),
    GetrsCase("TC_L1_16", "N", 1024, 4, 1024, 1024, 8, True, RN, S, False, 42),
    GetrsCase("TC_L1_17", "T", 128, 4, 128, 128, 4, True, RN, S, False, 42),
    GetrsCase("TC_L1_18", "T", 1024, 4, 1024, 1024, 2, True, RN, S, False, 42),
    GetrsCase("TC_L1_19", "C", 128, 4, 128, 128, 4, True, RN, S, False, 42),
    GetrsCase("TC_L1_20", "T", 64, 4, 64, 64, 4, False, RN, S, False, 42),
    GetrsCase("TC_L1_21", "N", 1, 1, 1, 1, 4, True, RN, S, False, 42),
    GetrsCase("TC_L1_22", "N", 3, 3, 3, 3, 4, True, RN, S, False, 42),
    GetrsCase("TC_L1_23", "N", 32, 4, 32, 48, 4, True, RN, S, False, 42),
    GetrsCase("TC_L1_24", "N", 16, 4, 128, 128, 4, True, RN, S, False, 42),
    GetrsCase("TC_L1_25", "N", 16, 4, 128, 16, 4, True, RN, S, False, 42),
    GetrsCase("TC_L1_26", "N", 0, 4, 1, 1, 0, True, RN, S, False, 0),
    GetrsCase("TC_L1_27", "N", 32, 4, 32, 32, 4, True, "IDENTITY", S, False, 42),
    GetrsCase("TC_L1_28", "N", 64, 4, 64, 64, 4, True, "DIAGONALLY_DOMINANT", S, False, 42),
    GetrsCase("TC_L1_29", "N", 4, 4, 4, 4, 4, True, "ILL_CONDITIONED", S, False, 42),
    GetrsCase("TC_L1_30", "N", 8, 2, 8, 8, 2, True, "DIAGONAL", S, False, 42),
    GetrsCase("TC_L1_31", "N", 8, 2, 8, 8, 2, True, "UPPER_TRIANGULAR", S, False, 42),
    GetrsCase("TC_L1_32", "N", 8, 2, 8, 8, 2, True, "LOWER_TRIANGULAR", S, False, 42),
    GetrsCase("TC_L1_33", "N", 32, 4, 32, 32, 4, True, "SINGULAR_ZERO_COL", S, False, 42),
    GetrsCase("TC_L1_34", "N", 32, 4, 32, 32, 4, True, "SINGULAR_DEPENDENT_ROW", S, False, 42),
    GetrsCase("TC_L1_35", "N", 32, 4, 32, 32, 4, True, "MIXED", S, False, 42),
    GetrsCase("TC_L1_36", "N", 64, 4, 64, 64, 4, False, "DIAGONALLY_DOMINANT", S, False, 42),
    GetrsCase("TC_L1_37", "T", 64, 4, 64, 64, 4, True, "DIAGONALLY_DOMINANT", S, False, 42),
    GetrsCase("TC_L1_38", "N", 1, 1, 1, 1, 1, False, RN, S, False, 42),
    GetrsCase("TC_L1_39", "N", 32, 4, 32, 32, 4, True, RN, S, False, 42),
    GetrsCase("TC_L1_41", "N", 32, 4, 32, 32, 4, True, RN, S, True, 42),
    GetrsCase("TC_L1_42", "C", 64, 4, 64, 64, 4, False, RN, S, False, 42),
]
# Error rows: (name, trans, n, nrhs, lda, ldb, batch, null_a, null_b, null_handle, status, expected_info)
# Expected info follows the validation order of sgetrs_batched_host.cpp:49-95, restated by the
# reference test's GetExpectedErrorInfoValue (getrs_batched_test.cpp:72-94).
GETRS_ERRORS = [
    ("TC_L0_E01", "N", 32, 4, 32, 32, 4, False, False, True, HN, None),
    ("TC_L0_E02", "N", -1, 4, 1, 1, 4, False, False, False, IV, -3),
    ("TC_L0_E03", "N", 32, -1, 32, 32, 4, False, False, False, IV, -4),
    ("TC_L0_E04", "N", 32, 4, 32, 32, -1, False, False, False, IV, -11),
    ("TC_L1_E01", "N", 5, 4, 3, 5, 4, False, False, False, IV, -6),
    ("TC_L1_E02", "N", 5, 4, 5, 3, 4, False, False, False, IV, -9),
    ("TC_L1_E03", "N", 0, 4, 0, 1, 4, False, False, False, IV, -6),
    ("TC_L1_E04", "N", 32, 4, 32, 32, 4, True, False, False, IV, -5),
    ("TC_L1_E05", "N", 32, 4, 32, 32, 4, False, True, False, IV, -8),
    ("TC_L1_E06", "INVALID", 32, 4, 32, 32, 4, False, False, False, IE, -2),
    ("TC_L1_E07", "N", 32, 257, 32, 32, 4, False, False, False, IV, -4),
    ("TC_L1_40", "N", 5, 4, 3, 5, 4, False, False, False, IV, -6),
]

GETRI = [
    GetriCase("TC_L0_01", 64, 64, 64, 4, True, RN, S, 42),
    GetriCase("TC_L0_02", 64, 64, 64, 4, False, RN, S, 42),
    GetriCase("TC_L0_03", 1, 1, 1, 1, True, RN, S, 42),
    GetriCase("TC_L0_04", 0, 1, 1, 4, True, RN, S, 0),
    GetriCase("TC_L0_05", 32, 32, 32, 0, True, RN, S, 0),
    GetriCase("TC_L0_06", 32, 32, 32, 4, True, "SINGULAR_ZERO_COL", S, 42),
    GetriCase("TC_L0_07", 32, 32, 32, 16, True, RN, S, 42),
    GetriCase("TC_L0_08", 32, 48, 32, 4, True, RN, S, 42),
    GetriCase("TC_L0_09", 128, 128, 128, 4, True, RN, S, 42),
    GetriCase("TC_L0_10", 2, 2, 2, 4, True, RN, S, 42),
    GetriCase("TC_L0_11", 1024, 1024, 1024, 2, True, RN, S, 42),
    GetriCase("TC_L0_12", 2048, 2048, 2048, 1, True, RN, S, 42),
    GetriCase("TC_L1_01", 256, 256, 256, 2, True, RN, S, 42),
    GetriCase("TC_L1_02", 257, 257, 257, 2, True, RN, S, 42),
    GetriCase("TC_L1_03", 512, 512, 512, 1, True, RN, S, 42),
    GetriCase("TC_L1_04", 32, 32, 32, 1, True, RN, S, 42),
    GetriCase("TC_L1_05", 16, 16, 16, 64, True, RN, S, 42),
    GetriCase("TC_L1_06", 8, 8, 8, 128, True, RN, S, 42),
    GetriCase("TC_L1_07", 32, 32, 32, 4, True, "MIXED", S, 42),
    GetriCase("TC_L1_08", 32, 32, 32, 4, True, "IDENTITY", S, 42),
    GetriCase("TC_L1_09", 64, 64, 64, 4, True, "DIAGONALLY_DOMINANT", S, 42),
    GetriCase("TC_L1_10", 4, 4, 4, 4, True, "ILL_CONDITIONED", S, 42),
    GetriCase("TC_L1_11", 64, 64, 64, 4, False, "DIAGONALLY_DOMINANT", S, 42),
    GetriCase("TC_L1_12", 16, 128, 16, 4, True, RN, S, 42),
    GetriCase("TC_L1_13", 32, 32, 48, 4, True, RN, S, 42),
    GetriCase("TC_L1_14", 1, 1, 1, 4, True, RN, S, 42),
    GetriCase("TC_L1_15", 32, 32, 32, 4, True, "SINGULAR_DEPENDENT_ROW", S, 42),
    GetriCase("TC_L1_16", 1, 1, 1, 1, False, RN, S, 42),
    GetriCase("TC_L1_17", 3, 3, 3, 4, True, RN, S, 42),
    GetriCase("TC_L1_18", 4, 4, 4, 4, True, RN, S, 42),
    GetriCase("TC_L1_19", 8, 8, 8, 4, True, RN, S, 42),
    GetriCase("TC_L1_20", 16, 16, 16, 4, True, RN, S, 42),
    GetriCase("TC_L1_21", 16, 16, 16, 32, True, RN, S, 42),
    GetriCase("TC_L1_22", 1024, 1024, 1024, 8, True, RN, S, 42),
    GetriCase("TC_L1_23", 8, 8, 8, 2, True, "DIAGONAL", S, 42),
    GetriCase("TC_L1_24", 8, 8, 8, 2, True, "UPPER_TRIANGULAR", S, 42),
    GetriCase("TC_L1_25", 8, 8, 8, 2, True, "LOWER_TRIANGULAR", S, 42),
    GetriCase("TC_L1_26", 0, 1, 1, 0, True, RN, S, 0),
    GetriCase("TC_L1_27", 16, 128, 128, 4, True, RN, S, 42),
]
# Error rows: (name, n, lda, ldc, batch, null_a, null_c, null_info, null_handle, status)
GETRI_ERRORS = [
    ("TC_L0_E02", -1, 1, 1, 4, False, False, False, False, IV),
    ("TC_L0_E03", 32, 32, 32, -1, False, False, False, False, IV),
    ("TC_L1_E01", 5, 3, 5, 4, False, False, False, False, IV),
    ("TC_L1_E02", 5, 5, 3, 4, False, False, False, False, IV),
    ("TC_L1_E03", 0, 0, 1, 4, False, False, False, False, IV),
    ("TC_L1_E04", 32, 32, 32, 4, True, False, False, False, IV),
    ("TC_L1_E05", 32, 32, 32, 4, False, True, False, False, IV),
    ("TC_L1_E06", 32, 32, 32, 4, False, False, True, False, IV),
]

# aclblasSmatinvBatched success rows of test/matinv_batched/arch35/matinv_batched_test.csv with
# work to do: (name, n, lda, lda_inv, batch, matrix_type); every row uses random_seed 42.
MATINV_CASES = [
    ("TC_L0_01", 4, 4, 4, 1, "RANDOM_NONSINGULAR"),
    ("TC_L0_02", 8, 8, 8, 2, "RANDOM_NONSINGULAR"),
    ("TC_L0_03", 16, 16, 16, 4, "RANDOM_NONSINGULAR"),
    ("TC_L0_04", 32, 32, 32, 8, "RANDOM_NONSINGULAR"),
    ("TC_L0_05", 1, 1, 1, 1, "RANDOM_NONSINGULAR"),
    ("TC_L0_06", 2, 2, 2, 1, "RANDOM_NONSINGULAR"),
    ("TC_L0_07", 4, 4, 4, 2, "RANDOM_NONSINGULAR"),
    ("TC_L0_08", 8, 8, 8, 4, "RANDOM_NONSINGULAR"),
    ("TC_L0_09", 16, 16, 16, 8, "RANDOM_NONSINGULAR"),
    ("TC_L0_10", 32, 32, 32, 1, "RANDOM_NONSINGULAR"),
    ("TC_L0_11", 1, 1, 1, 8, "RANDOM_NONSINGULAR"),
    ("TC_L0_12", 4, 4, 4, 2, "IDENTITY"),
    ("TC_L0_16", 3, 3, 3, 4, "RANDOM_NONSINGULAR"),
    ("TC_L0_17", 8, 8, 8, 2, "SINGULAR_ZERO_COL"),
    ("TC_L0_18", 5, 5, 5, 2, "RANDOM_NONSINGULAR"),
    ("TC_L0_19", 20, 20, 20, 4, "RANDOM_NONSINGULAR"),
    ("TC_L1_01", 8, 8, 8, 64, "RANDOM_NONSINGULAR"),
    ("TC_L1_02", 8, 8, 8, 128, "RANDOM_NONSINGULAR"),
    ("TC_L1_03", 4, 4, 4, 256, "RANDOM_NONSINGULAR"),
    ("TC_L1_04", 4, 4, 4, 512, "RANDOM_NONSINGULAR"),
    ("TC_L1_05", 4, 4, 4, 1024, "RANDOM_NONSINGULAR"),
    ("TC_L1_06", 32, 32, 32, 64, "RANDOM_NONSINGULAR"),
    ("TC_L1_07", 32, 32, 32, 256, "RANDOM_NONSINGULAR"),
    ("TC_L1_08", 32, 32, 32, 512, "RANDOM_NONSINGULAR"),
    ("TC_L1_09", 32, 32, 32, 1024, "RANDOM_NONSINGULAR"),
    ("TC_L1_10", 16, 16, 16, 512, "RANDOM_NONSINGULAR"),
    ("TC_L1_11", 1, 1, 1, 1024, "RANDOM_NONSINGULAR"),
    ("TC_L1_12", 16, 16, 16, 4, "SINGULAR_ZERO_COL"),
    ("TC_L1_13", 8, 8, 8, 4, "SINGULAR_ZERO_COL"),
    ("TC_L1_14", 16, 16, 16, 4, "SINGULAR_DEPENDENT_ROW"),
    ("TC_L1_15", 16, 16, 16, 4, "MIXED"),
    ("TC_L1_16", 8, 8, 8, 4, "MIXED"),
    ("TC_L1_17", 7, 7, 7, 2, "RANDOM_NONSINGULAR"),
    ("TC_L1_18", 12, 12, 12, 8, "RANDOM_NONSINGULAR"),
    ("TC_L1_19", 24, 24, 24, 4, "RANDOM_NONSINGULAR"),
    ("TC_L1_20", 8, 16, 8, 4, "RANDOM_NONSINGULAR"),
    ("TC_L1_21", 8, 8, 16, 4, "RANDOM_NONSINGULAR"),
    ("TC_L1_22", 16, 32, 32, 4, "RANDOM_NONSINGULAR"),
    ("TC_L1_23", 4, 32, 4, 2, "RANDOM_NONSINGULAR"),
    ("TC_L1_24", 4, 32, 32, 4, "RANDOM_NONSINGULAR"),
    ("TC_L1_25", 16, 16, 16, 2, "IDENTITY"),
    ("TC_L1_26", 8, 8, 8, 2, "DIAGONAL"),
    ("TC_L1_27", 16, 16, 16, 4, "DIAGONALLY_DOMINANT"),
    ("TC_L1_28", 8, 8, 8, 2, "UPPER_TRIANGULAR"),
    ("TC_L1_29", 8, 8, 8, 2, "LOWER_TRIANGULAR"),
    ("TC_L1_OBS_01", 4, 4, 4, 2, "ILL_CONDITIONED"),
]
MATINV_SEED = 42

# aclblasSmatinvBatched rows of test/matinv_batched/arch35/matinv_batched_test.csv that expect an
# error or the empty-operation success: (name, n, lda, lda_inv, batch, null_a, null_ainv,
# null_info, status)
MATINV_ARG_ROWS = [
    ("TC_L0_13", 0, 1, 1, 4, False, False, False, S),
    ("TC_L0_14", 32, 32, 32, 0, False, False, False, S),
    ("TC_L0_15", 0, 1, 1, 0, False, False, False, S),
    ("TC_L0_E02", -1, 1, 1, 4, False, False, False, IV),
    ("TC_L0_E03", 33, 33, 33, 4, False, False, False, IV),
    ("TC_L0_E04", 16, 16, 16, -1, False, False, False, IV),
    ("TC_L1_E01", 16, 8, 16, 4, False, False, False, IV),
    ("TC_L1_E02", 16, 16, 8, 4, False, False, False, IV),
    ("TC_L1_E03", 16, 16, 16, 4, True, False, False, IV),
    ("TC_L1_E04", 16, 16, 16, 4, False, True, False, IV),
    ("TC_L1_E05", 16, 16, 16, 4, False, False, True, IV),
    ("TC_L1_E06", -100, 1, 1, 4, False, False, False, IV),
    ("TC_L1_E07", 64, 64, 64, 4, False, False, False, IV),
    ("TC_L1_E08", 0, 0, 1, 4, False, False, False, IV),
    ("TC_L1_E09", 16, 16, 16, 4, True, True, True, IV),
    ("TC_L1_E10", 0, 1, 0, 4, False, False, False, IV),
]


def work(case) -> int:
    """Rough n^3 * batch size, to keep the slowest CPU-side checks optional."""
    return max(case.n, 0) ** 3 * max(case.batch, 0)

# GemmBatchedEx error rows (test/gemm_batched_ex/arch35/gemm_batched_ex_test.csv, expect != SUCCESS):
# (name, transA, transB, m, n, k, Atype, Btype, Ctype, lda, ldb, ldc, batch, compute, algo,
#  alpha_null, beta_null, a_null, b_null, c_null, null_handle, status)
GEMM_ERRORS = [
    ("L0_24", "N", "N", 128, 128, 128, "F16", "F16", "F16", 128, 128, 128, 4, "16F", 0, 0, 0, 0, 0, 0, 1, HN),
    ("L0_25", "N", "N", -1, 128, 128, "F16", "F16", "F16", 1, 128, 1, 4, "16F", 0, 0, 0, 0, 0, 0, 0, IV),
    ("L0_26", "N", "N", 128, 128, 128, "F16", "F16", "F16", 128, 128, 128, 4, "16F", 0, 1, 0, 0, 0, 0, 0, IV),
    ("L0_27", "N", "N", 128, 128, 128, "F16", "F16", "F16", 128, 128, 128, 4, "16F", 0, 0, 1, 0, 0, 0, 0, IV),
    ("L0_28", "N", "N", 128, 128, 128, "F16", "F16", "F16", 128, 128, 128, -1, "16F", 0, 0, 0, 0, 0, 0, 0, IV),
    ("L0_29", "N", "N", 128, 128, 128, "F16", "F16", "F16", 128, 128, 128, 4, "16F", 0, 0, 0, 1, 0, 0, 0, IV),
    ("L0_30", "N", "N", 128, 128, 128, "F16", "F16", "F16", 128, 128, 128, 4, "16F", 0, 0, 0, 0, 1, 0, 0, IV),
    ("L0_31", "N", "N", 128, 128, 128, "F16", "F16", "F16", 128, 128, 128, 4, "16F", 0, 0, 0, 0, 0, 1, 0, IV),
    ("L0_32", "N", "N", 128, 128, 128, "F16", "F16", "F16", 64, 128, 128, 4, "16F", 0, 0, 0, 0, 0, 0, 0, IV),
    ("L0_33", "N", "N", 128, 128, 128, "F16", "F16", "F16", 128, 64, 128, 4, "16F", 0, 0, 0, 0, 0, 0, 0, IV),
    ("L0_34", "N", "N", 128, 128, 128, "F16", "F16", "F16", 128, 128, 64, 4, "16F", 0, 0, 0, 0, 0, 0, 0, IV),
    ("L0_35", "T", "N", 128, 128, 128, "F16", "F16", "F16", 64, 128, 128, 4, "16F", 0, 0, 0, 0, 0, 0, 0, IV),
    ("L0_36", "N", "N", 128, 128, 128, "F32", "F32", "F32", 128, 128, 128, 4, "32F", 0, 0, 0, 0, 0, 0, 0, "NOT_SUPPORTED"),
    ("L0_37", "N", "N", 128, 128, 128, "E4M3", "E4M3", "F16", 128, 128, 128, 4, "16F", 0, 0, 0, 0, 0, 0, 0,
     "NOT_SUPPORTED"),
    ("L1_36", "N", "N", 128, -1, 128, "F16", "F16", "F16", 128, 128, 128, 4, "16F", 0, 0, 0, 0, 0, 0, 0, IV),
    ("L1_37", "N", "N", 128, 128, -1, "F16", "F16", "F16", 128, 128, 128, 4, "16F", 0, 0, 0, 0, 0, 0, 0, IV),
    ("L1_38", "INVALID", "N", 128, 128, 128, "F16", "F16", "F16", 128, 128, 128, 4, "16F", 0, 0, 0, 0, 0, 0, 0, IV),
    ("L1_39", "N", "INVALID", 128, 128, 128, "F16", "F16", "F16", 128, 128, 128, 4, "16F", 0, 0, 0, 0, 0, 0, 0, IV),
    ("L1_40", "N", "N", 128, 128, 128, "F16", "F16", "F16", 128, 128, 128, 4, "16F", 0, 0, 0, 0, 0, 1, 0, IV),
    ("L1_41", "N", "N", 128, 128, 128, "F16", "F32", "F16", 128, 128, 128, 4, "32F", 0, 0, 0, 0, 0, 0, 0,
     "NOT_SUPPORTED"),
    ("L1_42", "N", "N", 128, 128, 128, "F16", "F16", "F16", 128, 128, 128, 4, "16F", 1, 0, 0, 0, 0, 0, 0,
     "NOT_SUPPORTED"),
]

# aclblasSgemmBatched rows of test/gemm_batched/sgemm_batched/arch35/sgemm_batched_test.csv.
# Success rows: name transA transB m n k alpha beta lda ldb ldc batch c_fill (0 = the default
# leading dimension; c_fill Z = zeros, R = N(0,1); A and B are N(0,1) in every row).
_SGEMM_OK = """
L0_012 N N 0 128 128 1 0 0 0 0 4 Z
L0_013 N N 128 0 128 1 0 0 0 0 4 Z
L0_014 N N 128 128 0 1 0 0 0 0 4 Z
L0_015 N N 128 128 128 1 0 0 0 0 0 Z
G1_Msweep_001 N N 1 64 64 1.0 0.0 0 0 0 1 Z
G1_Msweep_002 N N 3 64 64 1.0 0.0 0 0 0 1 Z
G1_Msweep_003 N N 13 64 64 1.0 0.0 0 0 0 1 Z
G1_Msweep_004 N N 32 64 64 1.0 0.0 0 0 0 1 Z
G1_Msweep_005 N N 55 64 64 1.0 0.0 0 0 0 1 Z
G1_Msweep_006 N N 64 64 64 1.0 0.0 0 0 0 1 Z
G1_Msweep_007 N N 128 64 64 1.0 0.0 0 0 0 1 Z
G1_Msweep_008 N N 234 64 64 1.0 0.0 0 0 0 1 Z
G1_Msweep_009 N N 256 64 64 1.0 0.0 0 0 0 1 Z
G1_Msweep_010 N N 591 64 64 1.0 0.0 0 0 0 1 Z
G1_Msweep_011 N N 512 64 64 1.0 0.0 0 0 0 1 Z
G1_Nsweep_012 N N 64 1 64 1.0 0.0 0 0 0 1 Z
G1_Nsweep_013 N N 64 3 64 1.0 0.0 0 0 0 1 Z
G1_Nsweep_014 N N 64 13 64 1.0 0.0 0 0 0 1 Z
G1_Nsweep_015 N N 64 32 64 1.0 0.0 0 0 0 1 Z
G1_Nsweep_016 N N 64 55 64 1.0 0.0 0 0 0 1 Z
G1_Nsweep_017 N N 64 128 64 1.0 0.0 0 0 0 1 Z
G1_Nsweep_018 N N 64 234 64 1.0 0.0 0 0 0 1 Z
G1_Nsweep_019 N N 64 256 64 1.0 0.0 0 0 0 1 Z
G1_Nsweep_020 N N 64 591 64 1.0 0.0 0 0 0 1 Z
G1_Nsweep_021 N N 64 512 64 1.0 0.0 0 0 0 1 Z
G1_Ksweep_022 N N 64 64 1 1.0 0.0 0 0 0 1 Z
G1_Ksweep_023 N N 64 64 3 1.0 0.0 0 0 0 1 Z
G1_Ksweep_024 N N 64 64 13 1.0 0.0 0 0 0 1 Z
G1_Ksweep_025 N N 64 64 32 1.0 0.0 0 0 0 1 Z
G1_Ksweep_026 N N 64 64 55 1.0 0.0 0 0 0 1 Z
G1_Ksweep_027 N N 64 64 128 1.0 0.0 0 0 0 1 Z
G1_Ksweep_028 N N 64 64 234 1.0 0.0 0 0 0 1 Z
G1_Ksweep_029 N N 64 64 256 1.0 0.0 0 0 0 1 Z
G1_Ksweep_030 N N 64 64 591 1.0 0.0 0 0 0 1 Z
G1_Ksweep_031 N N 64 64 512 1.0 0.0 0 0 0 1 Z
G2_Mixed_032 N N 1 3 13 1.0 0.0 0 0 0 1 Z
G2_Mixed_033 N N 32 55 64 1.0 0.0 0 0 0 1 Z
G2_Mixed_034 N N 128 234 256 1.0 0.0 0 0 0 1 Z
G2_Mixed_035 N N 591 512 128 1.0 0.0 0 0 0 1 Z
G2_Mixed_036 N N 256 13 55 1.0 0.0 0 0 0 1 Z
G2_Mixed_037 N N 512 234 3 1.0 0.0 0 0 0 1 Z
G2_Mixed_038 N N 55 256 591 1.0 0.0 0 0 0 1 Z
G2_Mixed_039 N N 234 128 1 1.0 0.0 0 0 0 1 Z
G2_Mixed_040 N N 13 591 32 1.0 0.0 0 0 0 1 Z
G2_Mixed_041 N N 3 512 234 1.0 0.0 0 0 0 1 Z
G3_Trans_042 N N 64 64 64 1.5 0.3 0 0 0 1 R
G3_Trans_043 N T 64 64 64 1.5 0.3 0 0 0 1 R
G3_Trans_044 N C 64 64 64 1.5 0.3 0 0 0 1 R
G3_Trans_045 T N 64 64 64 1.5 0.3 0 0 0 1 R
G3_Trans_046 T T 64 64 64 1.5 0.3 0 0 0 1 R
G3_Trans_047 T C 64 64 64 1.5 0.3 0 0 0 1 R
G3_Trans_048 C N 64 64 64 1.5 0.3 0 0 0 1 R
G3_Trans_049 C T 64 64 64 1.5 0.3 0 0 0 1 R
G3_Trans_050 C C 64 64 64 1.5 0.3 0 0 0 1 R
G4_Alpha_051 N N 64 64 64 0.0 0.0 0 0 0 1 Z
G4_Alpha_052 N N 64 64 64 0.3 0.0 0 0 0 1 Z
G4_Alpha_053 N N 64 64 64 0.5 0.0 0 0 0 1 Z
G4_Alpha_054 N N 64 64 64 0.7 0.0 0 0 0 1 Z
G4_Alpha_055 N N 64 64 64 1.0 0.0 0 0 0 1 Z
G4_Alpha_056 N N 64 64 64 1.2 0.0 0 0 0 1 Z
G4_Alpha_057 N N 64 64 64 1.7 0.0 0 0 0 1 Z
G4_Alpha_058 N N 64 64 64 2.0 0.0 0 0 0 1 Z
G4_Alpha_059 N N 64 64 64 2.3 0.0 0 0 0 1 Z
G5_Beta_060 N N 64 64 64 1.0 0.0 0 0 0 1 Z
G5_Beta_061 N N 64 64 64 1.0 0.3 0 0 0 1 R
G5_Beta_062 N N 64 64 64 1.0 0.5 0 0 0 1 R
G5_Beta_063 N N 64 64 64 1.0 0.7 0 0 0 1 R
G5_Beta_064 N N 64 64 64 1.0 1.0 0 0 0 1 R
G5_Beta_065 N N 64 64 64 1.0 1.2 0 0 0 1 R
G5_Beta_066 N N 64 64 64 1.0 1.7 0 0 0 1 R
G5_Beta_067 N N 64 64 64 1.0 2.0 0 0 0 1 R
G5_Beta_068 N N 64 64 64 1.0 2.3 0 0 0 1 R
G6_AB_069 N N 64 64 64 0.0 0.3 0 0 0 1 R
G6_AB_070 N N 64 64 64 0.3 1.7 0 0 0 1 R
G6_AB_071 N N 64 64 64 0.5 0.5 0 0 0 1 R
G6_AB_072 N N 64 64 64 0.7 2.0 0 0 0 1 R
G6_AB_073 N N 64 64 64 1.0 0.0 0 0 0 1 Z
G6_AB_074 N N 64 64 64 1.2 1.2 0 0 0 1 R
G6_AB_075 N N 64 64 64 1.7 0.3 0 0 0 1 R
G6_AB_076 N N 64 64 64 2.0 0.5 0 0 0 1 R
G6_AB_077 N N 64 64 64 2.3 1.0 0 0 0 1 R
G6_AB_078 N N 64 64 64 0.0 0.0 0 0 0 1 Z
G7_Batch_079 N N 64 64 64 1.5 0.3 0 0 0 1 R
G7_Batch_080 N N 64 64 64 1.5 0.3 0 0 0 2 R
G7_Batch_081 N N 64 64 64 1.5 0.3 0 0 0 3 R
G7_Batch_082 N N 64 64 64 1.5 0.3 0 0 0 4 R
G7_Batch_083 N N 64 64 64 1.5 0.3 0 0 0 8 R
G8_Edge_084 N N 1 1 1 1.0 0.0 0 0 0 1 Z
G8_Edge_085 N N 3 3 3 1.0 0.0 0 0 0 1 Z
G8_Edge_086 N N 13 13 13 1.0 0.0 0 0 0 1 Z
G8_Edge_087 N N 1 128 128 1.0 0.0 0 0 0 1 Z
G8_Edge_088 N N 128 1 128 1.0 0.0 0 0 0 1 Z
G8_Edge_089 N N 128 128 1 1.0 0.0 0 0 0 1 Z
G8_Stress_090 T T 128 256 13 2.0 1.0 0 0 0 1 R
G8_Stress_091 N T 256 128 55 1.7 0.7 0 0 0 1 R
G8_Stress_092 N N 234 591 32 0.5 0.3 0 0 0 1 R
G8_Stress_093 N N 512 512 64 1.0 0.0 0 0 0 1 Z
G8_Stress_094 N N 512 512 512 1.0 0.0 0 0 0 1 Z
G8_Stress_095 N N 512 512 512 1.5 0.3 0 0 0 1 R
G8_Stress_096 N N 591 591 591 1.0 0.0 0 0 0 1 Z
G8_Stress_097 N N 256 512 256 1.2 0.5 0 0 0 3 R
G8_Stress_098 T N 128 128 128 0.7 1.7 0 0 0 3 R
G8_Stress_099 N T 1 512 591 2.3 0.0 0 0 0 1 Z
G9_NonAligned_100 N N 17 19 23 1.0 0.0 0 0 0 1 Z
G9_NonAligned_101 N T 17 19 23 1.0 0.0 0 0 0 1 Z
G9_NonAligned_102 T N 17 19 23 1.0 0.0 0 0 0 1 Z
G9_NonAligned_103 T T 17 19 23 1.0 0.0 0 0 0 1 Z
G9_NonAligned_104 N N 33 47 29 1.0 0.0 0 0 0 1 Z
G9_NonAligned_105 N T 33 47 29 1.0 0.0 0 0 0 1 Z
G9_NonAligned_106 T N 33 47 29 1.0 0.0 0 0 0 1 Z
G9_NonAligned_107 T T 33 47 29 1.0 0.0 0 0 0 1 Z
G9_NonAligned_108 N N 55 13 7 1.0 0.0 0 0 0 1 Z
G9_NonAligned_109 N T 55 13 7 1.0 0.0 0 0 0 1 Z
G9_NonAligned_110 T N 55 13 7 1.0 0.0 0 0 0 1 Z
G9_NonAligned_111 T T 55 13 7 1.0 0.0 0 0 0 1 Z
G9_NonAligned_112 N N 13 55 23 1.0 0.0 0 0 0 1 Z
G9_NonAligned_113 N T 13 55 23 1.0 0.0 0 0 0 1 Z
G9_NonAligned_114 T N 13 55 23 1.0 0.0 0 0 0 1 Z
G9_NonAligned_115 T T 13 55 23 1.0 0.0 0 0 0 1 Z
G10_LdLarge_116 N N 128 128 128 1.0 0.0 0 0 0 4 Z
G10_LdLarge_117 N N 128 128 128 1.0 0.0 256 128 128 4 Z
G10_LdLarge_118 N N 128 128 128 1.0 0.0 128 256 128 4 Z
G10_LdLarge_119 N N 128 128 128 1.0 0.0 128 128 256 4 Z
G11_K0_beta0_120 N N 128 128 0 1.0 0.0 0 0 0 4 Z
G11_K0_beta1_121 N N 128 128 0 1.0 1.0 0 0 0 4 R
G11_K0_beta0p5_122 N N 128 128 0 1.0 0.5 0 0 0 4 R
G11_A0_beta1_123 N N 128 128 128 0.0 1.0 0 0 0 4 R
G11_A0_beta0_124 N N 128 128 128 0.0 0.0 0 0 0 4 Z
DIAG_M1_PP_NN N N 1 128 128 1.5 0.3 0 0 0 1 R
DIAG_M1_PP_NN_b0 N N 1 128 128 2.0 0.0 0 0 0 1 Z
DIAG_N1_PP_NN N N 128 1 128 1.5 0.3 0 0 0 1 R
DIAG_M1_PP_NT N T 1 128 128 2.3 0.0 0 0 0 1 Z
DIAG_M1_PP_TN T N 1 128 128 1.5 0.3 0 0 0 1 R
DIAG_M3_PP_NN N N 3 128 128 1.5 0.3 0 0 0 1 R
DIAG_M7_PP_NN N N 7 128 128 1.5 0.3 0 0 0 1 R
DIAG_M8_PP_NN N N 8 128 128 1.5 0.3 0 0 0 1 R
DIAG_M9_PP_NN N N 9 128 128 1.5 0.3 0 0 0 1 R
G12_LargeBatch_155 N N 64 64 64 1.5 0.3 0 0 0 16 R
G12_LargeBatch_156 N N 64 64 64 1.0 0.0 0 0 0 32 Z
G12_LargeBatch_157 T T 32 32 32 1.7 0.7 0 0 0 64 R
"""
# Error rows: name transA transB m n k lda ldb ldc batch nulls(alpha beta A B C) null_handle status
_SGEMM_ERR = """
L0_016 N N 128 128 128 0 0 0 4 00000 1 HN
L0_017 N N -1 128 128 0 0 0 4 00000 0 IV
L0_018 N N 128 128 128 0 0 0 4 10000 0 IV
L0_019 N N 128 128 128 0 0 0 4 01000 0 IV
L0_020 N N 128 128 128 0 0 0 -1 00000 0 IV
L0_021 N N 128 128 128 0 0 0 4 00100 0 IV
L0_022 N N 128 128 128 0 0 0 4 00010 0 IV
L0_023 N N 128 128 128 0 0 0 4 00001 0 IV
L0_024 N N 128 128 128 64 128 128 4 00000 0 IV
L0_025 N N 128 128 128 128 64 128 4 00000 0 IV
L0_026 N N 128 128 128 128 128 64 4 00000 0 IV
L0_027 T N 128 128 128 64 128 128 4 00000 0 IV
L0_028 N N 128 -1 128 0 0 0 4 00000 0 IV
L0_029 N N 128 128 -1 0 0 0 4 00000 0 IV
L0_030 INVALID N 128 128 128 0 0 0 4 00000 0 IV
L0_031 N INVALID 128 128 128 0 0 0 4 00000 0 IV
"""


def _sgemm_ld(v, default):
    return int(v) if int(v) > 0 else max(1, default)


def _sgemm_rows():
    out = []
    for line in _SGEMM_OK.split("\n"):
        if not line.strip():
            continue
        name, ta, tb, m, n, k, alpha, beta, lda, ldb, ldc, batch, cfill = line.split()
        m, n, k = int(m), int(n), int(k)
        out.append((name, ta, tb, m, n, k, float(alpha), float(beta), _sgemm_ld(lda, k if ta != "N" else m),
                    _sgemm_ld(ldb, n if tb != "N" else k), _sgemm_ld(ldc, m), int(batch), cfill))
    return out


def _sgemm_errors():
    out = []
    for line in _SGEMM_ERR.split("\n"):
        if not line.strip():
            continue
        name, ta, tb, m, n, k, lda, ldb, ldc, batch, nulls, hn, status = line.split()
        m, n, k = int(m), int(n), int(k)
        out.append((name, ta, tb, m, n, k, _sgemm_ld(lda, k if ta == "T" else m), _sgemm_ld(ldb, n if tb == "T" else k),
                    _sgemm_ld(ldc, m), int(batch), [c == "1" for c in nulls], hn == "1", {"IV": IV, "HN": HN}[status]))
    return out


SGEMM_CASES = _sgemm_rows()
SGEMM_ERRORS = _sgemm_errors()


# aclblasSgeqrfBatched rows of test/geqrf_batched/sgeqrf_batched/arch35/sgeqrf_batched_test.csv:
# (name, m, n, lda, batch, a_fill, a_array_null, tau_array_null, status); the verification
# multiplier of MERE_MARE (threshold 0.000122) is 10 except where GEQRF_MARE_MULTIPLIER says.
GEQRF_MARE_MULTIPLIER = {"TC_L0_005": 15.0, "TC_L1_031": 1000.0, "TC_L1_032": 10000.0}
GEQRF_ROWS = [
    ("TC_L0_001", 4, 4, 4, 1, "RANDOM_NORM_2", False, False, S),
    ("TC_L0_002", 8, 8, 8, 4, "RANDOM_NORM_2", False, False, S),
    ("TC_L0_003", 16, 4, 16, 2, "RANDOM_NORM_2", False, False, S),
    ("TC_L0_004", 4, 16, 4, 2, "RANDOM_NORM_2", False, False, S),
    ("TC_L0_005", 32, 32, 32, 4, "RANDOM_NORM_2", False, False, S),
    ("TC_L0_006", 0, 8, 1, 2, "RANDOM_NORM_2", False, False, S),
    ("TC_L0_007", 8, 0, 8, 2, "RANDOM_NORM_2", False, False, S),
    ("TC_L0_008", 8, 8, 8, 0, "RANDOM_NORM_2", False, False, S),
    ("TC_L0_009", 1, 1, 1, 1, "RANDOM_NORM_2", False, False, S),
    ("TC_L0_011", -1, 8, 1, 2, "RANDOM_NORM_2", False, False, IV),
    ("TC_L0_012", 8, -1, 8, 2, "RANDOM_NORM_2", False, False, IV),
    ("TC_L0_013", 8, 8, 4, 2, "RANDOM_NORM_2", False, False, IV),
    ("TC_L0_014", 8, 8, 8, -1, "RANDOM_NORM_2", False, False, IV),
    ("TC_L1_002", 64, 16, 64, 4, "RANDOM_NORM_2", False, False, S),
    ("TC_L1_003", 16, 64, 16, 4, "RANDOM_NORM_2", False, False, S),
    ("TC_L1_006", 8, 8, 16, 2, "RANDOM_NORM_2", False, False, S),
    ("TC_L1_007", 16, 16, 32, 2, "RANDOM_NORM_2", False, False, S),
    ("TC_L1_008", 4, 4, 4, 32, "RANDOM_NORM_2", False, False, S),
    ("TC_L1_009", 8, 8, 8, 64, "RANDOM_NORM_2", False, False, S),
    ("TC_L1_011", 0, 0, 1, 2, "RANDOM_NORM_2", False, False, S),
    ("TC_L1_012", 1, 8, 1, 2, "RANDOM_NORM_2", False, False, S),
    ("TC_L1_013", 8, 1, 8, 2, "RANDOM_NORM_2", False, False, S),
    ("TC_L1_014", 2, 2, 2, 1, "RANDOM_NORM_2", False, False, S),
    ("TC_L1_015", 3, 3, 3, 1, "RANDOM_NORM_2", False, False, S),
    ("TC_L1_016", 1, 1, 1, 4, "RANDOM_NORM_2", False, False, S),
    ("TC_L1_017", 8, 8, 8, 2, "VALUE_DIAG_1", False, False, S),
    ("TC_L1_018", 8, 8, 8, 2, "VALUE_NORM_0", False, False, S),
    ("TC_L1_019", 8, 8, 8, 2, "RANDOM_DIAG", False, False, S),
    ("TC_L1_020", 8, 8, 8, 2, "RANDOM_UPPER", False, False, S),
    ("TC_L1_021", 8, 8, 8, 2, "RANDOM_LOWER", False, False, S),
    ("TC_L1_022", 8, 8, 8, 2, "RANDOM_NORM_1E6", False, False, S),
    ("TC_L1_023", 8, 8, 8, 2, "RANDOM_NORM_1EN6", False, False, S),
    ("TC_L1_024", 8, 8, 8, 2, "RANDOM_ILLCOND", False, False, S),
    ("TC_L1_025", 8, 8, 8, 2, "RANDOM_NORM_2", True, False, IV),
    ("TC_L1_026", 8, 8, 8, 2, "RANDOM_NORM_2", False, True, IV),
    ("TC_L1_027", 0, 8, 0, 2, "RANDOM_NORM_2", False, False, IV),
    ("TC_L1_028", -2, 8, 1, 2, "RANDOM_NORM_2", False, False, IV),
    ("TC_L1_029", 8, -2, 8, 2, "RANDOM_NORM_2", False, False, IV),
    ("TC_L1_030", 8, 8, 8, -2, "RANDOM_NORM_2", False, False, IV),
    ("TC_L1_031", 66, 66, 66, 2, "RANDOM_NORM_2", False, False, S),
    ("TC_L1_032", 512, 512, 512, 2, "RANDOM_NORM_2", False, False, S),
]


def geqrf_matrices(m, n, lda, fill, seed, batch):
    """Inputs of the geqrf rows, shape (batch, n, lda) column-major, padding rows set to 99.
    The fills follow the CSV's names (N(0,1) scaled as named, identity, zeros, random diagonal /
    triangular, and a graded ill-conditioned matrix); the values are this suite's own draw."""
    import numpy as np

    rng = np.random.default_rng(seed)
    a = np.full((batch, max(1, n), lda), 99.0, np.float32)
    if m == 0 or n == 0 or batch == 0:
        return a
    g = rng.standard_normal((batch, m, n))  # [batch, row, column]
    if fill == "VALUE_DIAG_1":
        g = np.broadcast_to(np.eye(m, n), g.shape).copy()
    elif fill == "VALUE_NORM_0":
        g = np.zeros_like(g)
    elif fill == "RANDOM_DIAG":
        g = g * np.eye(m, n)
    elif fill == "RANDOM_UPPER":
        g = np.triu(g)
    elif fill == "RANDOM_LOWER":
        g = np.tril(g)
    elif fill == "RANDOM_NORM_1E6":
        g = g * 1e6
    elif fill == "RANDOM_NORM_1EN6":
        g = g * 1e-6
    elif fill == "RANDOM_ILLCOND":
        g = g * np.logspace(0, -6, n)[None, None, :]
    a[:, :n, :m] = np.swapaxes(g, 1, 2).astype(np.float32)
    return a

# aclblasSgelsBatched rows of test/gels_batched/sgels_batched/arch35/sgels_batched_test.csv:
# name trans m n nrhs lda ldc batch c_fill null(A/C/I/H/-) status description (trans X = invalid)
_GELS = """
TC_L0_01 N 8 4 1 8 8 1 RANDOM - S overdetermined_small_transN
TC_L0_02 N 4 8 1 4 8 1 RANDOM - S underdetermined_small_transN
TC_L0_03 N 8 8 1 8 8 1 RANDOM - S square_transN
TC_L0_04 T 8 4 1 8 8 1 RANDOM - S overdetermined_small_transT
TC_L0_05 T 4 8 1 4 8 1 RANDOM - S underdetermined_small_transT
TC_L0_06 N 32 16 1 32 32 1 RANDOM - S overdetermined_medium_transN
TC_L0_07 N 16 8 4 16 16 1 RANDOM - S multi_rhs_overdetermined
TC_L0_08 N 8 4 1 8 8 4 RANDOM - S multi_batch_overdetermined
TC_L0_09 N 16 8 3 16 16 4 RANDOM - S multi_batch_multi_rhs
TC_L0_10 N 1 1 1 1 1 1 RANDOM - S minimal_1x1
TC_L0_11 N 1 8 1 1 8 1 RANDOM - S single_row_underdetermined
TC_L0_12 N 8 1 1 8 8 1 RANDOM - S single_column_overdetermined
TC_L0_13 N 0 8 1 1 8 1 RANDOM - S m_zero_fast_return
TC_L0_14 N 8 0 1 8 8 1 RANDOM - S n_zero_fast_return
TC_L0_15 N 8 4 0 8 8 1 RANDOM - S nrhs_zero_fast_return
TC_L0_16 N 8 4 1 8 8 0 RANDOM - S batch_zero_fast_return
TC_L0_17 T 8 8 1 8 8 1 RANDOM - S square_transT
TC_L0_18 N 16 32 1 16 32 1 RANDOM - S underdetermined_medium
TC_L0_19 N 8 16 2 8 16 3 RANDOM - S multi_batch_underdetermined
TC_L0_20 N 8 8 1 8 8 1 RANDOM - S identity_matrix
TC_L1_01 N 128 64 1 128 128 1 RANDOM - S large_overdetermined
TC_L1_02 N 64 128 1 64 128 1 RANDOM - S large_underdetermined
TC_L1_03 N 128 128 1 128 128 1 RANDOM - S large_square
TC_L1_04 N 256 4 1 256 256 1 RANDOM - S extreme_aspect_m_gt_n
TC_L1_05 N 4 256 1 4 256 1 RANDOM - S extreme_aspect_n_gt_m
TC_L1_06 N 8 4 1 16 8 1 RANDOM - S noncompact_lda
TC_L1_07 N 8 4 1 8 16 1 RANDOM - S noncompact_ldc
TC_L1_08 N 8 4 1 16 16 1 RANDOM - S noncompact_lda_ldc
TC_L1_09 N 31 17 1 31 31 1 RANDOM - S prime_dimensions
TC_L1_10 N 127 97 1 127 127 1 RANDOM - S prime_dimensions_large
TC_L1_11 N 8 4 1 8 8 1 RANDOM - S rank_deficient
TC_L1_12 N 8 4 1 8 8 1 ZEROS - S rhs_zeros
TC_L1_13 N 16 8 1 16 16 1 RANDOM - S known_solution
TC_L1_14 N 8 4 1 8 8 16 RANDOM - S large_batch
TC_L1_15 N 4 8 1 4 8 16 RANDOM - S large_batch_underdetermined
TC_L1_16 T 128 64 1 128 128 1 RANDOM - S transT_large_overdetermined
TC_L1_17 T 64 128 1 64 128 1 RANDOM - S transT_large_underdetermined
TC_L1_18 T 32 16 4 32 32 1 RANDOM - S transT_multi_rhs
TC_L1_19 T 16 8 1 16 16 4 RANDOM - S transT_multi_batch
TC_L1_20 T 16 8 3 16 16 4 RANDOM - S transT_multi_rhs_batch
TC_L1_21 N 16 8 2 32 32 4 RANDOM - S noncompact_multi_batch_rhs
TC_L1_22 N 256 2 1 256 256 1 RANDOM - S extreme_aspect_m_gt_n_large
TC_L1_23 N 2 256 1 2 256 1 RANDOM - S extreme_aspect_n_gt_m_large
TC_L1_24 N 2 2 1 2 2 1 RANDOM - S small_2x2_square
TC_L1_25 N 64 32 1 64 64 1 RANDOM - S medium_single_batch
TC_L1_26 N 8 4 1 8 8 1 RANDOM H HN handle_nullptr
TC_L1_27 N -1 4 1 1 4 1 RANDOM - IV m_negative
TC_L1_28 N 8 -1 1 8 8 1 RANDOM - IV n_negative
TC_L1_29 N 8 4 -1 8 8 1 RANDOM - IV nrhs_negative
TC_L1_30 N 8 4 1 8 8 -1 RANDOM - IV batch_negative
TC_L1_31 N 8 4 1 4 8 1 RANDOM - IV lda_lt_max1m
TC_L1_32 N 0 4 1 0 4 1 RANDOM - IV lda_lt_1_m0
TC_L1_33 N 8 16 1 8 8 1 RANDOM - IV ldc_lt_max1mn
TC_L1_34 X 8 4 1 8 8 1 RANDOM - IE trans_invalid
TC_L1_35 N 8 4 1 8 8 1 RANDOM A IV aarray_nullptr
TC_L1_36 N 8 4 1 8 8 1 RANDOM C IV carray_nullptr
TC_L1_37 N 8 4 1 8 8 1 RANDOM I IV devinfo_nullptr
"""


def _gels_rows():
    st = {"S": S, "IV": IV, "HN": HN, "IE": IE}
    out = []
    for line in _GELS.split("\n"):
        if not line.strip():
            continue
        name, t, m, n, nrhs, lda, ldc, batch, cfill, null, status, desc = line.split()
        out.append((name, t, int(m), int(n), int(nrhs), int(lda), int(ldc), int(batch), cfill, null, st[status], desc))
    return out


GELS_ROWS = _gels_rows()


def gels_inputs(row, seed):
    """A (batch, n, lda) and C (batch, nrhs, ldc) of a gels row, column-major, padding 99 / 77.
    A is N(0,1) except the identity and rank-deficient (a repeated column) rows; C holds the
    right-hand sides in its first m (trans N) or n (trans T) rows: N(0,1), zeros, or A x for a
    known x."""
    import numpy as np

    name, t, m, n, nrhs, lda, ldc, batch, cfill, null, status, desc = row
    rng = np.random.default_rng(seed)
    rows_b = m if t == "N" else n
    a = np.full((batch, max(1, n), lda), 99.0, np.float32)
    c = np.full((batch, max(1, nrhs), ldc), 77.0, np.float32)
    g = rng.standard_normal((batch, m, n))
    if desc == "identity_matrix":
        g = np.broadcast_to(np.eye(m, n), g.shape).copy()
    if desc == "rank_deficient" and n > 1:
        g[:, :, n - 1] = g[:, :, 0]
    a[:, :n, :m] = np.swapaxes(g, 1, 2)
    rhs = rng.standard_normal((batch, rows_b, nrhs))
    if cfill == "ZEROS":
        rhs[:] = 0.0
    if desc == "known_solution":
        op = g if t == "N" else np.swapaxes(g, 1, 2)
        rhs = op @ rng.standard_normal((batch, op.shape[2], nrhs))
    c[:, :nrhs, :rows_b] = np.swapaxes(rhs, 1, 2)
    return a, c


# aclblasCgemmBatched rows of test/gemm_batched/cgemm_batched/arch35/cgemm_batched_test.csv
# (duplicated rows once). Success rows: name transA transB m n k alpha(re;im) beta(re;im) lda ldb
# ldc batch c_fill (R random, Z zero); 0 for a leading dimension means the CSV's default
# (cgemm_batched_param.h:83-88: the stored rows of op's operand, ldc = m, at least 1).
_CGEMM_OK = """
L0_001 N N 0 128 128 1.0;0.0 0.0;0.0 0 0 128 4 Z
L0_002 N N 128 0 128 1.0;0.0 0.0;0.0 0 0 128 4 Z
L0_003 N N 128 128 0 1.0;0.0 0.0;0.0 0 0 128 4 Z
L0_004 N N 128 128 128 1.0;0.0 0.0;0.0 0 0 128 0 Z
G1_Msweep_021 N N 1 64 64 1.0;0.0 0.0;0.0 0 0 64 1 Z
G1_Msweep_022 N N 3 64 64 1.0;0.0 0.0;0.0 0 0 64 1 Z
G1_Msweep_023 N N 13 64 64 1.0;0.0 0.0;0.0 0 0 64 1 Z
G1_Msweep_024 N N 32 64 64 1.0;0.0 0.0;0.0 0 0 64 1 Z
G1_Msweep_025 N N 55 64 64 1.0;0.0 0.0;0.0 0 0 64 1 Z
G1_Msweep_026 N N 64 64 64 1.0;0.0 0.0;0.0 0 0 64 1 Z
G1_Msweep_027 N N 128 64 64 1.0;0.0 0.0;0.0 0 0 0 1 Z
G1_Msweep_028 N N 234 64 64 1.0;0.0 0.0;0.0 0 0 0 1 Z
G1_Msweep_029 N N 256 64 64 1.0;0.0 0.0;0.0 0 0 0 1 Z
G1_Msweep_030 N N 128 64 64 1.0;0.5 0.0;0.0 0 0 0 1 Z
G1_Msweep_031 N N 591 64 64 1.0;0.0 0.0;0.0 0 0 0 1 Z
G1_Msweep_032 N N 512 64 64 1.0;0.0 0.0;0.0 0 0 0 1 Z
G1_Nsweep_033 N N 64 1 64 1.0;0.0 0.0;0.0 0 0 64 1 Z
G1_Nsweep_034 N N 64 3 64 1.0;0.0 0.0;0.0 0 0 64 1 Z
G1_Nsweep_035 N N 64 13 64 1.0;0.0 0.0;0.0 0 0 64 1 Z
G1_Nsweep_036 N N 64 32 64 1.0;0.0 0.0;0.0 0 0 64 1 Z
G1_Nsweep_037 N N 64 55 64 1.0;0.0 0.0;0.0 0 0 64 1 Z
G1_Nsweep_038 N N 64 128 64 1.0;0.0 0.0;0.0 0 0 64 1 Z
G1_Nsweep_039 N N 64 234 64 1.0;0.0 0.0;0.0 0 0 64 1 Z
G1_Nsweep_040 N N 64 256 64 1.0;0.0 0.0;0.0 0 0 64 1 Z
G1_Nsweep_041 N N 64 591 64 1.0;0.0 0.0;0.0 0 0 64 1 Z
G1_Nsweep_042 N N 64 512 64 1.0;0.0 0.0;0.0 0 0 64 1 Z
G1_Ksweep_043 N N 64 64 1 1.0;0.0 0.0;0.0 0 0 64 1 Z
G1_Ksweep_044 N N 64 64 3 1.0;0.0 0.0;0.0 0 0 64 1 Z
G1_Ksweep_045 N N 64 64 13 1.0;0.0 0.0;0.0 0 0 64 1 Z
G1_Ksweep_046 N N 64 64 32 1.0;0.0 0.0;0.0 0 0 64 1 Z
G1_Ksweep_047 N N 64 64 55 1.0;0.0 0.0;0.0 0 0 64 1 Z
G1_Ksweep_048 N N 64 64 128 1.0;0.0 0.0;0.0 0 0 64 1 Z
G1_Ksweep_049 N N 64 64 234 1.0;0.0 0.0;0.0 0 0 64 1 Z
G1_Ksweep_050 N N 64 64 256 1.0;0.0 0.0;0.0 0 0 64 1 Z
G1_Ksweep_051 N N 64 64 591 1.0;0.0 0.0;0.0 0 0 64 1 Z
G1_Ksweep_052 N N 64 64 512 1.0;0.0 0.0;0.0 0 0 64 1 Z
G2_Mixed_053 N N 1 3 13 1.0;0.0 0.0;0.0 0 0 13 1 Z
G2_Mixed_054 N N 32 55 64 1.0;0.0 0.0;0.0 0 0 64 1 Z
G2_Mixed_055 N N 128 234 256 1.0;0.0 0.0;0.0 0 0 256 1 Z
G2_Mixed_056 N N 64 64 64 1.0;0.5 0.0;0.0 0 0 64 1 Z
G2_Mixed_057 N N 64 64 64 0.5;0.3 0.0;0.0 0 0 64 1 Z
G2_Mixed_058 N N 591 512 128 1.0;0.0 0.0;0.0 0 0 0 1 Z
G2_Mixed_059 N N 256 13 55 1.0;0.0 0.0;0.0 0 0 0 1 Z
G2_Mixed_060 N N 512 234 3 1.0;0.0 0.0;0.0 0 0 0 1 Z
G2_Mixed_061 N N 55 256 591 1.0;0.0 0.0;0.0 0 0 0 1 Z
G2_Mixed_062 N N 234 128 1 1.0;0.0 0.0;0.0 0 0 0 1 Z
G2_Mixed_063 N N 13 591 32 1.0;0.0 0.0;0.0 0 0 0 1 Z
G2_Mixed_064 N N 3 512 234 1.0;0.0 0.0;0.0 0 0 0 1 Z
G3_Trans_065 N N 64 64 64 1.5;0.3 0.3;0.0 0 0 64 1 R
G3_Trans_066 N T 64 64 64 1.5;0.3 0.3;0.0 0 0 64 1 R
G3_Trans_067 N C 64 64 64 1.5;0.3 0.3;0.0 0 0 64 1 R
G3_Trans_068 T N 64 64 64 1.5;0.3 0.3;0.0 0 0 64 1 R
G3_Trans_069 T T 64 64 64 1.5;0.3 0.3;0.0 0 0 64 1 R
G3_Trans_070 T C 64 64 64 1.5;0.3 0.3;0.0 0 0 64 1 R
G3_Trans_071 C N 64 64 64 1.5;0.3 0.3;0.0 0 0 64 1 R
G3_Trans_072 C T 64 64 64 1.5;0.3 0.3;0.0 0 0 64 1 R
G3_Trans_073 C C 64 64 64 1.5;0.3 0.3;0.0 0 0 64 1 R
G4_Alpha_074 N N 64 64 64 0.0;0.0 0.0;0.0 0 0 64 1 Z
G4_Alpha_075 N N 64 64 64 0.3;0.0 0.0;0.0 0 0 64 1 Z
G4_Alpha_076 N N 64 64 64 0.5;0.0 0.0;0.0 0 0 64 1 Z
G4_Alpha_077 N N 64 64 64 1.0;0.0 0.0;0.0 0 0 64 1 Z
G4_Alpha_078 N N 64 64 64 1.0;0.5 0.0;0.0 0 0 64 1 Z
G4_Alpha_079 N N 64 64 64 2.0;0.0 0.0;0.0 0 0 64 1 Z
G4_Alpha_080 N N 64 64 64 2.3;0.0 0.0;0.0 0 0 64 1 Z
G4_Alpha_081 N N 64 64 64 0.0;2.0 0.0;0.0 0 0 64 1 Z
G4_Alpha_082 N N 64 64 64 1.5;0.7 0.0;0.0 0 0 64 1 Z
G5_Beta_083 N N 64 64 64 1.0;0.0 0.0;0.0 0 0 64 1 Z
G5_Beta_084 N N 64 64 64 1.0;0.0 0.3;0.0 0 0 64 1 R
G5_Beta_085 N N 64 64 64 1.0;0.0 0.5;0.0 0 0 64 1 R
G5_Beta_086 N N 64 64 64 1.0;0.0 0.7;0.0 0 0 64 1 R
G5_Beta_087 N N 64 64 64 1.0;0.0 1.0;0.0 0 0 64 1 R
G5_Beta_088 N N 64 64 64 1.0;0.0 1.2;0.0 0 0 64 1 R
G5_Beta_089 N N 64 64 64 1.0;0.0 1.7;0.0 0 0 64 1 R
G5_Beta_090 N N 64 64 64 1.0;0.0 2.0;0.0 0 0 64 1 R
G5_Beta_091 N N 64 64 64 1.0;0.0 2.3;0.0 0 0 64 1 R
G6_AB_092 N N 64 64 64 0.0;0.0 0.3;0.0 0 0 64 1 R
G6_AB_093 N N 64 64 64 0.3;0.5 1.7;0.2 0 0 64 1 R
G6_AB_094 N N 64 64 64 0.5;0.3 0.5;0.7 0 0 64 1 R
G6_AB_095 N N 64 64 64 0.7;0.2 2.0;0.5 0 0 64 1 R
G6_AB_096 N N 64 64 64 1.0;0.0 0.0;0.0 0 0 64 1 Z
G6_AB_097 N N 64 64 64 1.2;0.3 1.2;0.4 0 0 64 1 R
G6_AB_098 N N 64 64 64 1.7;0.5 0.3;0.6 0 0 64 1 R
G6_AB_099 N N 64 64 64 2.0;0.7 0.5;0.3 0 0 64 1 R
G6_AB_100 N N 64 64 64 2.3;0.1 1.0;0.9 0 0 64 1 R
G6_AB_101 N N 64 64 64 0.0;0.0 0.0;0.0 0 0 64 1 Z
G7_Batch_102 N N 64 64 64 1.5;0.3 0.3;0.0 0 0 64 1 R
G7_Batch_103 N N 64 64 64 1.5;0.3 0.3;0.0 0 0 64 2 R
G7_Batch_104 N N 64 64 64 1.5;0.3 0.3;0.0 0 0 64 3 R
G7_Batch_105 N N 64 64 64 1.5;0.3 0.3;0.0 0 0 64 4 R
G7_Batch_106 N N 64 64 64 1.5;0.3 0.3;0.0 0 0 64 8 R
G8_Edge_107 N N 1 1 1 1.0;0.0 0.0;0.0 0 0 1 1 Z
G8_Edge_108 N N 3 3 3 1.0;0.0 0.0;0.0 0 0 3 1 Z
G8_Edge_109 N N 13 13 13 1.0;0.0 0.0;0.0 0 0 13 1 Z
G8_Edge_110 N N 1 128 128 1.0;0.0 0.0;0.0 0 0 128 1 Z
G8_Edge_111 N N 128 1 128 1.0;0.0 0.0;0.0 0 0 128 1 Z
G8_Edge_112 N N 128 128 1 1.0;0.0 0.0;0.0 0 0 128 1 Z
G8_Stress_113 T T 128 256 13 2.0;1.0 1.0;0.5 0 0 256 1 R
G8_Stress_114 N T 256 128 55 1.7;0.7 0.7;0.3 0 0 0 1 R
G8_Stress_115 N N 234 591 32 0.5;0.3 0.3;0.1 0 0 591 1 R
G8_Stress_116 N N 128 128 128 1.0;0.0 0.0;0.0 0 0 128 1 Z
G8_Stress_117 N N 128 128 128 1.5;0.3 0.3;0.0 0 0 128 1 Z
G8_Stress_118 N N 256 256 128 1.0;0.5 0.5;0.2 0 0 256 1 R
G8_Stress_119 N N 256 256 256 1.0;0.0 0.0;0.0 0 0 256 1 Z
G8_Stress_120 N N 256 256 256 1.5;0.3 0.3;0.1 0 0 256 3 R
G8_Stress_121 T N 128 128 128 0.7;1.7 1.7;0.3 0 0 128 3 R
G8_Stress_122 N T 1 128 128 2.3;0.0 0.0;0.0 0 0 128 1 Z
G8_Stress_123 N N 512 512 64 1.0;0.0 0.0;0.0 0 0 0 1 Z
G8_Stress_124 N N 512 512 512 1.0;0.0 0.0;0.0 0 0 0 1 Z
G8_Stress_125 N N 512 512 512 1.5;0.3 0.3;0.0 0 0 0 1 R
G8_Stress_126 N N 591 591 591 1.0;0.0 0.0;0.0 0 0 0 1 Z
G9_NonAligned_127 N N 17 19 23 1.0;0.0 0.0;0.0 0 0 0 1 Z
G9_NonAligned_128 N T 17 19 23 1.0;0.0 0.0;0.0 0 0 0 1 Z
G9_NonAligned_129 T N 17 19 23 1.0;0.0 0.0;0.0 0 0 0 1 Z
G9_NonAligned_130 T T 17 19 23 1.0;0.0 0.0;0.0 0 0 0 1 Z
G9_NonAligned_131 N N 33 47 29 1.0;0.0 0.0;0.0 0 0 0 1 Z
G9_NonAligned_132 N T 33 47 29 1.0;0.0 0.0;0.0 0 0 0 1 Z
G9_NonAligned_133 T N 33 47 29 1.0;0.0 0.0;0.0 0 0 0 1 Z
G9_NonAligned_134 T T 33 47 29 1.0;0.0 0.0;0.0 0 0 0 1 Z
G9_NonAligned_135 N N 55 13 7 1.0;0.0 0.0;0.0 0 0 0 1 Z
G9_NonAligned_136 N T 55 13 7 1.0;0.0 0.0;0.0 0 0 0 1 Z
G9_NonAligned_137 T N 55 13 7 1.0;0.0 0.0;0.0 0 0 0 1 Z
G9_NonAligned_138 T T 55 13 7 1.0;0.0 0.0;0.0 0 0 0 1 Z
G9_NonAligned_139 N N 13 55 23 1.0;0.0 0.0;0.0 0 0 0 1 Z
G9_NonAligned_140 N T 13 55 23 1.0;0.0 0.0;0.0 0 0 0 1 Z
G9_NonAligned_141 T N 13 55 23 1.0;0.0 0.0;0.0 0 0 0 1 Z
G9_NonAligned_142 T T 13 55 23 1.0;0.0 0.0;0.0 0 0 0 1 Z
G10_LdLarge_143 N N 128 128 128 1.0;0.0 0.0;0.0 0 0 128 4 Z
G10_LdLarge_144 N N 128 128 128 1.0;0.0 0.0;0.0 256 128 128 4 Z
G10_LdLarge_145 N N 128 128 128 1.0;0.0 0.0;0.0 128 256 128 4 Z
G10_LdLarge_146 N N 128 128 128 1.0;0.0 0.0;0.0 128 128 256 4 Z
G11_K0_beta0_147 N N 128 128 0 1.0;0.0 0.0;0.0 0 0 128 4 Z
G11_K0_beta1_148 N N 128 128 0 1.0;0.0 1.0;0.0 0 0 128 4 R
G11_K0_beta0p5_149 N N 128 128 0 1.0;0.0 0.5;0.0 0 0 128 4 R
G11_A0_beta1_150 N N 128 128 128 0.0;0.0 1.0;0.0 0 0 128 4 R
G11_A0_beta0_151 N N 128 128 128 0.0;0.0 0.0;0.0 0 0 128 4 Z
G11_A0_betacplx_152 N N 128 128 128 0.0;0.0 0.5;0.3 0 0 128 4 R
DIAG_M1_PP_NN N N 1 128 128 1.5;0.3 0.3;0.0 0 0 128 1 R
DIAG_M1_PP_NN_b0 N N 1 128 128 2.0;0.0 0.0;0.0 0 0 128 1 Z
DIAG_N1_PP_NN N N 128 1 128 1.5;0.3 0.3;0.0 0 0 128 1 R
DIAG_M1_PP_NT N T 1 128 128 2.3;0.0 0.0;0.0 0 0 128 1 Z
DIAG_M1_PP_TN T N 1 128 128 1.5;0.3 0.3;0.0 0 0 128 1 R
DIAG_M3_PP_NN N N 3 128 128 1.5;0.3 0.3;0.0 0 0 128 1 R
DIAG_M7_PP_NN N N 7 128 128 1.5;0.3 0.3;0.0 0 0 128 1 R
DIAG_M8_PP_NN N N 8 128 128 1.5;0.3 0.3;0.0 0 0 128 1 R
DIAG_M9_PP_NN N N 9 128 128 1.5;0.3 0.3;0.0 0 0 128 1 R
G12_LargeBatch_153 N N 64 64 64 1.5;0.3 0.3;0.0 0 0 64 16 R
G12_LargeBatch_154 N N 64 64 64 1.0;0.0 0.0;0.0 0 0 64 32 Z
G12_LargeBatch_155 T T 32 32 32 1.7;0.7 0.7;0.3 0 0 32 16 R
G12_LargeBatch_156 T T 32 32 32 1.7;0.7 0.7;0.3 0 0 32 64 R
"""
# Error rows: name transA transB m n k lda ldb ldc batch nulls(alpha beta A B C) null_handle status
_CGEMM_ERR = """
L0_005 N N 128 128 128 0 0 128 4 00000 1 HN
L0_006 N N -1 128 128 0 0 128 4 00000 0 IV
L0_007 N N 128 128 128 0 0 128 4 10000 0 IV
L0_008 N N 128 128 128 0 0 128 4 01000 0 IV
L0_009 N N 128 128 128 0 0 128 -1 00000 0 IV
L0_010 N N 128 128 128 0 0 128 4 00100 0 IV
L0_011 N N 128 128 128 0 0 128 4 00010 0 IV
L0_012 N N 128 128 128 0 0 128 4 00001 0 IV
L0_013 N N 128 128 128 64 128 128 4 00000 0 IV
L0_014 N N 128 128 128 128 64 128 4 00000 0 IV
L0_015 N N 128 128 128 128 128 64 4 00000 0 IV
L0_016 T N 128 128 128 64 128 128 4 00000 0 IV
L0_017 N N 128 -1 128 0 0 128 4 00000 0 IV
L0_018 N N 128 128 -1 0 0 128 4 00000 0 IV
L0_019 INVALID N 128 128 128 0 0 128 4 00000 0 IV
L0_020 N INVALID 128 128 128 0 0 128 4 00000 0 IV
"""


def _cplx(v):
    re, im = v.split(";")
    return complex(float(re), float(im))


def _cgemm_rows():
    out = []
    for line in _CGEMM_OK.split("\n"):
        if not line.strip():
            continue
        name, ta, tb, m, n, k, alpha, beta, lda, ldb, ldc, batch, cfill = line.split()
        m, n, k = int(m), int(n), int(k)
        out.append((name, ta, tb, m, n, k, _cplx(alpha), _cplx(beta), _sgemm_ld(lda, m if ta == "N" else k),
                    _sgemm_ld(ldb, k if tb == "N" else n), _sgemm_ld(ldc, m), int(batch), cfill))
    return out


def _cgemm_errors():
    out = []
    for line in _CGEMM_ERR.split("\n"):
        if not line.strip():
            continue
        name, ta, tb, m, n, k, lda, ldb, ldc, batch, nulls, hn, status = line.split()
        m, n, k = int(m), int(n), int(k)
        out.append((name, ta, tb, m, n, k, _sgemm_ld(lda, m if ta == "N" else k),
                    _sgemm_ld(ldb, k if tb == "N" else n), _sgemm_ld(ldc, m), int(batch),
                    [c == "1" for c in nulls], hn == "1", {"IV": IV, "HN": HN}[status]))
    return out


CGEMM_CASES = _cgemm_rows()
CGEMM_ERRORS = _cgemm_errors()
