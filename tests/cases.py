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
