"""Index arithmetic of k_mf_post's block staging (ho-cxx_b200/csrc/krylov.cu), replayed on
the CPU for every K, both block storages (FP32 T, and the BF16 copy of HO2D_SMOOTHER_BF16)
and many mesh sizes, before and independently of any GPU run.

Per CTA b: elements el0 = b EPB .. el1 = min(el0 + EPB, N); the blocks' bytes
[b0, b1) = [el0, el1) K^4 s are staged as the 16-byte-aligned superset [a0, a1) with
cp.async 16-byte pieces into a shared buffer of EPB K^4 s + 32 bytes (staging only when that
is at most 32 KB); element le then reads K^4 values at (b0 - a0) + le K^4 s. The device
array holds N K^4 values plus 8 zero values of padding. Checked: every piece lies inside
the allocation and the shared buffer, pieces are 16-byte aligned, and every element's block
lies inside the staged bytes at an offset aligned for its type.
"""

import pytest


def shape(K):
    K2 = K * K
    epb = 32 if 256 // K2 > 32 else max(256 // K2, 1)
    threads = ((epb * K2 + 31) // 32) * 32
    return epb, threads


@pytest.mark.parametrize("K", range(1, 9))
@pytest.mark.parametrize("size", [4, 2])  # FP32 blocks, BF16 blocks
def test_block_staging_stays_in_bounds(K, size):
    epb, threads = shape(K)
    K4 = K ** 4
    k_bytes = epb * K4 * size + 32
    staged = k_bytes <= 32768
    sizes = list(range(1, 3 * epb + 2)) + [14625, 4096, 262144, 131072 + 3]
    for N in sizes:
        alloc = (N * K4 + 8) * size
        for b in range((N + epb - 1) // epb):
            el0, el1 = b * epb, min(b * epb + epb, N)
            if not staged:
                assert el1 * K4 * size <= alloc
                continue
            b0, b1 = el0 * K4 * size, el1 * K4 * size
            a0, a1 = b0 & ~15, (b1 + 15) & ~15
            nbytes = a1 - a0
            assert a0 % 16 == 0 and nbytes % 16 == 0
            assert nbytes <= k_bytes, (N, b)      # fits the shared buffer
            assert a1 <= alloc, (N, b)            # never past the padded allocation
            assert nbytes < 2 ** 32
            # every piece o in [0, nbytes) step 16: in the buffer and in the allocation
            assert a0 + nbytes <= alloc
            for le in range(el1 - el0):
                off = (b0 - a0) + le * K4 * size
                assert off % size == 0
                assert off + K4 * size <= nbytes, (N, b, le)
    # the threads of a CTA cover its elements' points
    assert threads >= epb * K * K


def test_bf16_stages_where_fp32_cannot():
    """At K = 6 and 7 the FP32 blocks of a CTA exceed 32 KB and are read from global memory;
    the BF16 blocks fit and are staged."""
    for K, fp32, bf16 in ((5, True, True), (6, False, True), (7, False, True), (8, False, False)):
        epb, _ = shape(K)
        assert (epb * K ** 4 * 4 + 32 <= 32768) == fp32, K
        assert (epb * K ** 4 * 2 + 32 <= 32768) == bf16, K
