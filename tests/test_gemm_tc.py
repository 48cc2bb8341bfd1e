"""The tcgen05 GEMM (TMA-fed, TMEM accumulator) against float64 products of
the same BF16 operands: FP32 accumulation over Kd terms stays within
gamma_Kd = Kd * 2^-24 of sum |a_k b_k|, so the test allows 2 * Kd * 2^-24
relative to that sum (plus a tiny absolute term for all-zero rows)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SHAPES = [(1, 8, 64), (5, 256, 64), (128, 256, 640), (300, 300, 128), (257, 1024, 4608),
          (129, 4096, 512)]


def bf16_bits(x):
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    return (((u + 0x7FFF + ((u >> 16) & 1)) >> 16) & 0xFFFF).astype(np.uint16)


def bits_to_f64(b):
    return (b.astype(np.uint32) << 16).view(np.float32).astype(np.float64)


@pytest.mark.parametrize("M,N,Kd", SHAPES)
def test_gemm_matches_float64(M, N, Kd):
    from erq_b200._lib import check, load_library

    rng = np.random.default_rng(M * 7 + N * 3 + Kd)
    A = bf16_bits(rng.standard_normal((M, Kd)).astype(np.float32))
    B = bf16_bits(rng.standard_normal((N, Kd)).astype(np.float32))
    C = np.empty((M, N), np.float32)
    check(load_library().erq_debug_gemm_bf16(A.ctypes.data, B.ctypes.data, M, N, Kd,
                                             C.ctypes.data, 0))
    a, b = bits_to_f64(A), bits_to_f64(B)
    ref = a @ b.T
    bound = 2 * Kd * 2.0 ** -24 * (np.abs(a) @ np.abs(b).T) + 1e-30
    err = np.abs(C.astype(np.float64) - ref)
    assert (err <= bound).all(), float((err / bound).max())


def test_gemm_wait_limit_reports_timeout_and_recovers():
    """Every mbarrier wait of the GEMM is bounded.  With a limit of one poll
    the pipeline waits run out before the TMA copies land: the GEMM must
    return ERQ_ERR_TIMEOUT (its CTAs drain their copies and MMAs, free their
    tensor memory and exit), and the next GEMM with the default limit must
    succeed with correct results on the same device."""
    from erq_b200._lib import ERQ_ERR_TIMEOUT, check, load_library

    lib = load_library()
    M, N, Kd = 512, 1024, 1536
    rng = np.random.default_rng(5)
    A = bf16_bits(rng.standard_normal((M, Kd)).astype(np.float32))
    B = bf16_bits(rng.standard_normal((N, Kd)).astype(np.float32))
    C = np.empty((M, N), np.float32)
    check(lib.erq_debug_set_gemm_wait_limit(1))
    try:
        st = lib.erq_debug_gemm_bf16(A.ctypes.data, B.ctypes.data, M, N, Kd, C.ctypes.data, 0)
    finally:
        check(lib.erq_debug_set_gemm_wait_limit(0))
    assert st == ERQ_ERR_TIMEOUT, (st, lib.erq_last_error())
    assert b"limit" in lib.erq_last_error()
    check(lib.erq_debug_gemm_bf16(A.ctypes.data, B.ctypes.data, M, N, Kd, C.ctypes.data, 0))
    a, b = bits_to_f64(A), bits_to_f64(B)
    bound = 2 * Kd * 2.0 ** -24 * (np.abs(a) @ np.abs(b).T) + 1e-30
    assert (np.abs(C.astype(np.float64) - a @ b.T) <= bound).all()
