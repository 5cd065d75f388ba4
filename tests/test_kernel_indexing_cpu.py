"""Index arithmetic of the row-parallel smoothing kernel's block staging
(k_mf_post, ho-cxx_b200/csrc/krylov.cu), replayed on the CPU for every K, every block
storage (FP64, FP32, BF16) and many mesh sizes, before and independently of any GPU run.

Rows<K>: EPW = 32 // K elements per warp, 4 warps per CTA. Each element's K^4 block is
stored at a stride padded to 16 bytes (padded_count). Warp w of CTA b owns elements
wel0 = (4 b + w) EPW .. + wn, wn = min(EPW, N - wel0); when a warp's span
(EPW x stride x size) is at most 26 KB, one bulk copy moves wn x stride x size bytes from
wel0 x stride x size into the warp's slice [w SPAN, (w + 1) SPAN) of the dynamic shared
memory, and element lw reads its K^4 values at lw x stride x size. Checked: source,
destination and size are 16-byte multiples (the bulk copy's rule), the copy stays inside
the device allocation and the warp's shared slice, every element's block lies inside what
was copied, and every vector load of a block slice is aligned for its width.
"""

import pytest

WARPS = 4


def padded_count(n, elem_bytes):
    """device.cuh: n values rounded up to whole 16-byte pieces."""
    return (n * elem_bytes + 15) // 16 * 16 // elem_bytes


def post_layout(K, size):
    epw = 32 // K
    k4 = K ** 4
    stride = padded_count(k4, size)
    span = epw * stride * size
    staged = span <= 26 * 1024
    return epw, stride, span, staged


def slice_alignment(K, size):
    """load_slice's vector width: the alignment K x size bytes guarantees (<= 16)."""
    b = K * size
    for al in (16, 8, 4):
        if b % al == 0:
            return al
    return size


@pytest.mark.parametrize("K", range(1, 9))
@pytest.mark.parametrize("size", [8, 4, 2])  # FP64, FP32 blocks, BF16 blocks
def test_block_staging_stays_in_bounds(K, size):
    epw, stride, span, staged = post_layout(K, size)
    k4, k2 = K ** 4, K * K
    assert stride >= k4 and (stride * size) % 16 == 0
    sizes = list(range(1, 3 * WARPS * epw + 2)) + [14625, 4096, 262144, 131072 + 3]
    for N in sizes:
        alloc = (N * stride + 1) * size  # padded_rows: one spare value
        ctas = (N + WARPS * epw - 1) // (WARPS * epw)
        for b in range(ctas):
            for w in range(WARPS):
                wel0 = (b * WARPS + w) * epw
                wn = min(epw, N - wel0)
                if wn <= 0:
                    continue
                if not staged:
                    assert (wel0 + wn) * stride * size <= alloc
                    continue
                src, nbytes, dst = wel0 * stride * size, wn * stride * size, w * span
                assert src % 16 == 0 and nbytes % 16 == 0 and dst % 16 == 0
                assert src + nbytes <= alloc, (N, b, w)
                assert nbytes <= span and dst + nbytes <= WARPS * span
                for lw in range(wn):
                    off = lw * stride * size
                    assert off % 16 == 0 and off + k4 * size <= nbytes
    # every slice a thread reads (row t of slice r) is aligned for its vector width
    al = slice_alignment(K, size)
    for r in range(k2):
        for t in range(K):
            assert ((r * k2 + t * K) * size) % al == 0
    # the dynamic shared memory of the staged kernels leaves room for two CTAs per SM
    if staged:
        assert WARPS * span <= 104 * 1024


@pytest.mark.parametrize("K", range(1, 9))
def test_kronecker_factor_staging_stays_in_bounds(K):
    """The Kronecker-sum smoother stages each warp's factor sets (4K^2 + 2K FP32 values per
    element, stride padded to 16 bytes) the same way: always within the 26 KB per warp."""
    epw = 32 // K
    stride = padded_count(4 * K * K + 2 * K, 4)
    elem = stride * 4
    span = epw * elem
    assert elem % 16 == 0 and span <= 26 * 1024
    for N in list(range(1, 3 * WARPS * epw + 2)) + [4096, 131072 + 3]:
        alloc = (N * stride + 1) * 4
        for b in range((N + WARPS * epw - 1) // (WARPS * epw)):
            for w in range(WARPS):
                wel0 = (b * WARPS + w) * epw
                wn = min(epw, N - wel0)
                if wn <= 0:
                    continue
                src, nbytes = wel0 * elem, wn * elem
                assert src % 16 == 0 and nbytes % 16 == 0 and src + nbytes <= alloc
                for lw in range(wn):
                    assert lw * elem + (4 * K * K + 2 * K) * 4 <= nbytes


def test_staging_choice():
    """Which storages are staged by bulk copies: all of K <= 5, FP32 and BF16 at K = 6, BF16
    at K = 7; FP64 from K = 5 on and everything at K = 8 read from global memory."""
    expect = {(5, 8): False, (5, 4): True, (5, 2): True, (6, 8): False, (6, 4): True, (6, 2): True,
              (7, 8): False, (7, 4): False, (7, 2): True, (8, 4): False, (8, 2): False, (4, 8): True}
    for (K, size), st in expect.items():
        assert post_layout(K, size)[3] == st, (K, size)
