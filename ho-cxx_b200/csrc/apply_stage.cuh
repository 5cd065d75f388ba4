// apply_stage.cuh -- the FP32 operator's element data staged in shared memory by bulk
// copies (cp.async.bulk through the Tensor Memory Accelerator), one warp tile ahead.
//
// A warp's tile is EPW consecutive elements, so each input array is one contiguous span:
// the operand and the three metric coefficients (K^2 values per element), the second
// vector of the kernel's dot products (K^2), the six face arrays ([N][K][4]: face
// coefficients fa, fb, nfa, nfb and the incoming traces) and the face codes (4 ints).
// Lane 0 of the warp issues the twelve copies for its next tile into the warp's slice of
// the dynamic shared memory, on one mbarrier whose phase counts the tiles; the lanes read
// their rows from there, then the warp releases the slice for the next copy. The copies
// are plain (no cluster multicast) and read this GPU's own memory.
//
// Alignment: a copy moves whole 16-byte pieces between 16-byte aligned addresses. The
// face arrays and the codes are 16K and 16 bytes per element, so their spans are aligned.
// A K^2 span starts at element wel0 * K^2 * 4 bytes, which is 16-byte aligned only for even
// K; its copy starts at the 16-byte boundary below and ends at the one above, and the
// readers skip the first (address % 16) / 4 values. The end can lie up to 12 bytes past
// the array, which every device buffer leaves allocated (DeviceBuffer::alloc pads by 16).
#pragma once

#include <cstdint>

#include "bulk_copy.cuh"
#include "rows.cuh"

namespace ho2d {

template <int K>
struct ApplyStage {
    using R = Rows<K>;
    static constexpr int EPW = R::EPW, K2 = K * K;
    // floats of one K^2 span's slot: the warp's values plus the alignment slack on both
    // sides (at most 3 + 3 values), rounded up to a 16-byte multiple
    static constexpr int VEC = ((EPW * K2 + 6 + 3) / 4) * 4;
    static constexpr int FACE = EPW * K * 4;  // floats of one face array's span
    static constexpr int WARP_FLOATS = 5 * VEC + 6 * FACE + EPW * 4;
    static constexpr int WARP_BYTES = WARP_FLOATS * 4;
    static constexpr int CTA_BYTES = R::WARPS * WARP_BYTES;
    static_assert(VEC % 4 == 0 && FACE % 4 == 0, "slots must start on 16-byte boundaries");
    // slot offsets in floats
    static constexpr int X = 0, G11 = VEC, G12 = 2 * VEC, G22 = 3 * VEC, SEC = 4 * VEC;
    static constexpr int FA = 5 * VEC, FB = FA + FACE, NFA = FB + FACE, NFB = NFA + FACE, TV = NFB + FACE,
                         TG = TV + FACE, CODE = TG + FACE;
};

// The first element of a warp's tile.
template <int K>
__device__ __forceinline__ int stage_first(int tile, int warp) {
    return (tile * Rows<K>::WARPS + warp) * Rows<K>::EPW;
}

// Values to skip at the start of a K^2 slot: the span's start is a rounded-down copy.
__device__ __forceinline__ int stage_skip(const float* span) {
    return (int)((reinterpret_cast<uintptr_t>(span) & 15u) >> 2);
}

// Issues the copies of the tile whose first element is wel0 (wn elements) into slice `st`,
// completing on bar. Lane 0 only.
template <int K>
__device__ __forceinline__ void stage_issue(float* st, uint64_t* bar, const PoisGeom<float>& g, const float* x,
                                            const float* tvin, const float* tgin, const float* sec, int wel0,
                                            int wn) {
    using S = ApplyStage<K>;
    const float* vec[5] = {x + (size_t)wel0 * S::K2, g.G11 + (size_t)wel0 * S::K2, g.G12 + (size_t)wel0 * S::K2,
                           g.G22 + (size_t)wel0 * S::K2, sec + (size_t)wel0 * S::K2};
    const float* face[6] = {g.fa, g.fb, g.nfa, g.nfb, tvin, tgin};
    unsigned total = 0;
    uintptr_t lo[5];
    unsigned nb[5];
#pragma unroll
    for (int a = 0; a < 5; ++a) {
        const uintptr_t s = reinterpret_cast<uintptr_t>(vec[a]);
        const uintptr_t e = s + (size_t)wn * S::K2 * 4;
        lo[a] = s & ~(uintptr_t)15;
        nb[a] = (unsigned)(((e + 15) & ~(uintptr_t)15) - lo[a]);
        total += nb[a];
    }
    const unsigned fbytes = (unsigned)(wn * K * 16);
    total += 6 * fbytes + (unsigned)(wn * 16);
    mbar_arrive_expect(bar, total);
    const int vslot[5] = {S::X, S::G11, S::G12, S::G22, S::SEC};
#pragma unroll
    for (int a = 0; a < 5; ++a) bulk_load(st + vslot[a], reinterpret_cast<const void*>(lo[a]), nb[a], bar);
#pragma unroll
    for (int f = 0; f < 6; ++f)
        bulk_load(st + S::FA + f * S::FACE, face[f] + (size_t)wel0 * K * 4, fbytes, bar);
    bulk_load(st + S::CODE, g.code + (size_t)wel0 * 4, (unsigned)(wn * 16), bar);
}

// This thread's operator inputs and its row of the second vector from the staged tile
// (the spans' starts give the slack to skip). Inactive threads get zeros.
template <int K>
__device__ __forceinline__ void stage_read(const float* st, const PoisGeom<float>& g, const float* x,
                                           const float* sec, int wel0, const RowIdx<K>& ix, ApplyIn<K, float>& in,
                                           float (&sr)[K]) {
    using S = ApplyStage<K>;
    if (!ix.active) {
#pragma unroll
        for (int i = 0; i < K; ++i) in.xr[i] = in.xc[i] = in.g11[i] = in.g12r[i] = in.g22[i] = in.g12c[i] = sr[i] = 0.f;
#pragma unroll
        for (int f = 0; f < 4; ++f) {
            in.fa[f] = in.fb[f] = in.nfa[f] = in.nfb[f] = in.ntv[f] = in.ntg[f] = 0.f;
            in.code[f] = -1;
        }
        return;
    }
    const size_t w2 = (size_t)wel0 * S::K2;
    const int e = ix.lw * S::K2, t = ix.t;
    const float* xs = st + S::X + stage_skip(x + w2) + e;
    const float* g1 = st + S::G11 + stage_skip(g.G11 + w2) + e;
    const float* g2 = st + S::G12 + stage_skip(g.G12 + w2) + e;
    const float* g3 = st + S::G22 + stage_skip(g.G22 + w2) + e;
    const float* ss = st + S::SEC + stage_skip(sec + w2) + e;
#pragma unroll
    for (int i = 0; i < K; ++i) {
        in.xr[i] = xs[t * K + i];
        in.xc[i] = xs[t + i * K];
        in.g11[i] = g1[t * K + i];
        in.g12r[i] = g2[t * K + i];
        in.g22[i] = g3[t + i * K];
        in.g12c[i] = g2[t + i * K];
        sr[i] = ss[t * K + i];
    }
    const int q = (ix.lw * K + t) * 4;
    auto f4 = [&](int slot, float (&v)[4]) {
        const float4 a = *reinterpret_cast<const float4*>(st + slot + q);
        v[0] = a.x;
        v[1] = a.y;
        v[2] = a.z;
        v[3] = a.w;
    };
    f4(S::FA, in.fa);
    f4(S::FB, in.fb);
    f4(S::NFA, in.nfa);
    f4(S::NFB, in.nfb);
    f4(S::TV, in.ntv);
    f4(S::TG, in.ntg);
    const int4 c = *reinterpret_cast<const int4*>(st + S::CODE + ix.lw * 4);
    in.code[0] = c.x;
    in.code[1] = c.y;
    in.code[2] = c.z;
    in.code[3] = c.w;
}

// Orders this warp's reads of its slice before the copy engine's next writes into it.
__device__ __forceinline__ void stage_release() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

}  // namespace ho2d
