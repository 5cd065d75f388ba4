// rows.cuh -- row-parallel element kernels: K threads per element, thread t holding row t
// (and, where needed, column t) of the element's K x K block, several elements per warp.
//
// Every tensor-product contraction of the FR operator is then a loop over compile-time
// indices into the 1-D basis tables, which live in the kernel's parameter (constant) bank,
// so the basis value is an instruction operand instead of a load; an element's threads
// are lanes of one warp, so the transposes between the xi (row) and eta (column) passes
// and the exchange of a face's common values go through a few words of shared memory with
// __syncwarp, never a CTA-wide barrier. Face point k of each of the four faces belongs to
// thread k: W/E traces come from row k, S/N traces from column k.
#pragma once

#include "device.cuh"
#include "fr_launch.hpp"

namespace ho2d {

template <int K>
struct Rows {
    static constexpr int K2 = K * K, NF = 4 * K;
    static constexpr int EPW = 32 / K;      // elements per warp
    static constexpr int LANES = EPW * K;   // lanes with an element row (the rest idle)
    static constexpr int WARPS = 4;         // warps per CTA
    static constexpr int THREADS = 32 * WARPS;
    static constexpr int EPC = EPW * WARPS;  // elements per CTA
};

// This thread's element and row.
template <int K>
struct RowIdx {
    int lane, warp, lw, t, el;
    bool active;
    __device__ __forceinline__ RowIdx(int N, int tile) {
        using R = Rows<K>;
        lane = threadIdx.x & 31;
        warp = threadIdx.x >> 5;
        lw = lane / K;
        t = lane - lw * K;
        el = (tile * R::WARPS + warp) * R::EPW + lw;
        active = lane < R::LANES && el < N;
        if (lw >= R::EPW) lw = 0;  // idle lanes address element slot 0 (and write nothing)
    }
};

// Non-binding prefetch of one address's line into L2 (PTX prefetch.global.L2).
__device__ __forceinline__ void prefetch_l2(const void* p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

// The lines an operator tile will read for this thread's row (operand row, the three metric
// rows, the face point's coefficients and incoming traces, and the row of the dot product's
// second vector), prefetched into L2 one tile ahead so that the tile's loads do not wait on
// DRAM.
template <int K, typename T>
__device__ __forceinline__ void prefetch_apply_rows(const PoisGeom<T>& g, const T* x, const T* tvin, const T* tgin,
                                                    const T* second, int tile) {
    const RowIdx<K> ix(g.N, tile);
    if (!ix.active) return;
    const size_t r = (size_t)ix.el * K * K + ix.t * K, q4 = ((size_t)ix.el * K + ix.t) * 4;
    prefetch_l2(x + r);
    prefetch_l2(g.G11 + r);
    prefetch_l2(g.G12 + r);
    prefetch_l2(g.G22 + r);
    prefetch_l2(second + r);
    prefetch_l2(g.fa + q4);
    prefetch_l2(g.fb + q4);
    prefetch_l2(g.nfa + q4);
    prefetch_l2(g.nfb + q4);
    prefetch_l2(tvin + q4);
    prefetch_l2(tgin + q4);
}

// Per-warp shared scratch of the operator: the common values of the four faces, the
// Neumann right-hand sides and two K x K transpose buffers for each element of the warp.
template <int K, typename T>
struct RowScratch {
    T com[Rows<K>::EPW][4][K];
    T nr[Rows<K>::EPW][4][K];
    T tr[2][Rows<K>::EPW][K][K];
};

// K consecutive values; 8- or 16-byte loads when the row is aligned for them.
template <int K, typename T>
__device__ __forceinline__ void load_row(const T* __restrict__ p, T (&v)[K]) {
    if constexpr (sizeof(T) == 4 && K % 4 == 0) {
#pragma unroll
        for (int i = 0; i < K; i += 4) {
            const float4 q = __ldg(reinterpret_cast<const float4*>(p + i));
            v[i] = q.x;
            v[i + 1] = q.y;
            v[i + 2] = q.z;
            v[i + 3] = q.w;
        }
    } else if constexpr (sizeof(T) == 4 && K % 2 == 0) {
#pragma unroll
        for (int i = 0; i < K; i += 2) {
            const float2 q = __ldg(reinterpret_cast<const float2*>(p + i));
            v[i] = q.x;
            v[i + 1] = q.y;
        }
    } else if constexpr (sizeof(T) == 8 && K % 2 == 0) {
#pragma unroll
        for (int i = 0; i < K; i += 2) {
            const double2 q = __ldg(reinterpret_cast<const double2*>(p + i));
            v[i] = q.x;
            v[i + 1] = q.y;
        }
    } else {
#pragma unroll
        for (int i = 0; i < K; ++i) v[i] = __ldg(p + i);
    }
}

template <int K, typename T>
__device__ __forceinline__ void store_row(T* __restrict__ p, const T (&v)[K]) {
    if constexpr (sizeof(T) == 4 && K % 4 == 0) {
#pragma unroll
        for (int i = 0; i < K; i += 4) *reinterpret_cast<float4*>(p + i) = make_float4(v[i], v[i + 1], v[i + 2], v[i + 3]);
    } else if constexpr (sizeof(T) == 4 && K % 2 == 0) {
#pragma unroll
        for (int i = 0; i < K; i += 2) *reinterpret_cast<float2*>(p + i) = make_float2(v[i], v[i + 1]);
    } else if constexpr (sizeof(T) == 8 && K % 2 == 0) {
#pragma unroll
        for (int i = 0; i < K; i += 2) *reinterpret_cast<double2*>(p + i) = make_double2(v[i], v[i + 1]);
    } else {
#pragma unroll
        for (int i = 0; i < K; ++i) p[i] = v[i];
    }
}

// The four faces' values of one face point ([N][K][4] layout), one 16-byte (float) or two
// 16-byte (double) loads.
template <typename T>
__device__ __forceinline__ void load4(const T* __restrict__ p, T (&v)[4]) {
    if constexpr (sizeof(T) == 4) {
        const float4 q = __ldg(reinterpret_cast<const float4*>(p));
        v[0] = q.x;
        v[1] = q.y;
        v[2] = q.z;
        v[3] = q.w;
    } else {
        const double2 a = __ldg(reinterpret_cast<const double2*>(p));
        const double2 c = __ldg(reinterpret_cast<const double2*>(p) + 1);
        v[0] = a.x;
        v[1] = a.y;
        v[2] = c.x;
        v[3] = c.y;
    }
}

__device__ __forceinline__ void load4i(const int* __restrict__ p, int (&v)[4]) {
    const int4 q = __ldg(reinterpret_cast<const int4*>(p));
    v[0] = q.x;
    v[1] = q.y;
    v[2] = q.z;
    v[3] = q.w;
}

// Stride-K column of an element block.
template <int K, typename T>
__device__ __forceinline__ void load_col(const T* __restrict__ p, T (&v)[K]) {
#pragma unroll
    for (int j = 0; j < K; ++j) v[j] = __ldg(p + j * K);
}

// Face value and normal derivative at the -1 (lr = 0) or +1 (lr = 1) end of a line of
// K values (a row for the W/E faces, a column for the S/N faces).
template <int K, typename T, int LR>
__device__ __forceinline__ void line_trace(const DevBases<T>& b, const T (&f)[K], T& val, T& der) {
    T v = T(0), g = T(0);
#pragma unroll
    for (int m = 0; m < K; ++m) {
        v += f[m] * b.sbb[m * 2 + LR];
        g += f[m] * b.sbgb[m * 2 + LR];
    }
    val = v;
    der = g;
}

// The four face traces (value, normal derivative) of face point k = t, from row t and
// column t of the element block: index f = ijp (0 W, 1 E, 2 S, 3 N).
template <int K, typename T>
__device__ __forceinline__ void row_traces(const DevBases<T>& b, const T (&xr)[K], const T (&xc)[K], T (&tv)[4],
                                           T (&tg)[4]) {
    line_trace<K, T, 0>(b, xr, tv[0], tg[0]);
    line_trace<K, T, 1>(b, xr, tv[1], tg[1]);
    line_trace<K, T, 0>(b, xc, tv[2], tg[2]);
    line_trace<K, T, 1>(b, xc, tv[3], tg[3]);
}

// Writes this thread's column of an element block held as rows: every thread of the
// element stores its row into buf, then reads column t. Warp-collective (all 32 lanes).
template <int K, typename T>
__device__ __forceinline__ void rows_to_col(T (&buf)[K][K], const T (&row)[K], T (&col)[K], int t, bool active) {
    if (active) {
#pragma unroll
        for (int i = 0; i < K; ++i) buf[t][i] = row[i];
    }
    __syncwarp();
    if (active) {
#pragma unroll
        for (int j = 0; j < K; ++j) col[j] = buf[j][t];
    }
}

// Columns to rows: thread t stores column t, then reads row t. Warp-collective.
template <int K, typename T>
__device__ __forceinline__ void col_to_row(T (&buf)[K][K], const T (&col)[K], T (&row)[K], int t, bool active) {
    if (active) {
#pragma unroll
        for (int j = 0; j < K; ++j) buf[j][t] = col[j];
    }
    __syncwarp();
    if (active) {
#pragma unroll
        for (int i = 0; i < K; ++i) row[i] = buf[t][i];
    }
}

// Sum of one value over the K threads of each element, in the fixed order t = 0..K-1,
// returned to every thread of the element. Warp-collective.
template <int K, typename T>
__device__ __forceinline__ T element_total(T v, int lw) {
    T s = T(0);
#pragma unroll
    for (int m = 0; m < K; ++m) s += __shfl_sync(0xffffffffu, v, lw * K + m);
    return s;
}

// What one thread of the operator reads for its row t of element `el`: rows and columns
// of the operand and the metric coefficients, face point t of the four faces' coefficients
// and incoming traces, and the element's face codes.
template <int K, typename T>
struct ApplyIn {
    T xr[K], xc[K], g11[K], g12r[K], g22[K], g12c[K];
    T fa[4], fb[4], nfa[4], nfb[4], ntv[4], ntg[4];
    int code[4];
};

// The operator's inputs from global memory (zeros for an inactive thread).
template <int K, typename T>
__device__ __forceinline__ void row_apply_load(const PoisGeom<T>& g, const T* __restrict__ x,
                                               const T* __restrict__ tvin, const T* __restrict__ tgin,
                                               const RowIdx<K>& ix, ApplyIn<K, T>& in) {
    constexpr int K2 = K * K;
    const int t = ix.t, el = ix.el;
    if (ix.active) {
        const size_t e2 = (size_t)el * K2;
        load_row<K, T>(x + e2 + t * K, in.xr);
        load_col<K, T>(x + e2 + t, in.xc);
        load_row<K, T>(g.G11 + e2 + t * K, in.g11);
        load_row<K, T>(g.G12 + e2 + t * K, in.g12r);
        load_col<K, T>(g.G22 + e2 + t, in.g22);
        load_col<K, T>(g.G12 + e2 + t, in.g12c);
        const size_t q4 = ((size_t)el * K + t) * 4;  // face point t of the 4 faces ([N][K][4])
        load4<T>(g.fa + q4, in.fa);
        load4<T>(g.fb + q4, in.fb);
        load4<T>(g.nfa + q4, in.nfa);
        load4<T>(g.nfb + q4, in.nfb);
        load4<T>(tvin + q4, in.ntv);
        load4<T>(tgin + q4, in.ntg);
        load4i(g.code + el * 4, in.code);
    } else {
#pragma unroll
        for (int i = 0; i < K; ++i) in.xr[i] = in.xc[i] = in.g11[i] = in.g12r[i] = in.g22[i] = in.g12c[i] = T(0);
#pragma unroll
        for (int f = 0; f < 4; ++f) {
            in.fa[f] = in.fb[f] = in.nfa[f] = in.nfb[f] = in.ntv[f] = in.ntg[f] = T(0);
            in.code[f] = -1;
        }
    }
}

// y = A x, rows: the homogeneous-boundary Poisson operator (the method-2 FR Laplacian
// that the reference assembles in form_Laplace_operator_matrix, src/HO_2D.cpp:1533-1804)
// of element `el`, row t, from the element's own rows of x, its metric coefficients, its
// face coefficients and the incoming face traces of x that its neighbours' producers
// wrote (in, read by row_apply_load or from a staged copy). Warp-collective: every lane
// of the warp calls it.
template <int K, typename T>
__device__ __forceinline__ void row_apply_core(const MfOp<T>& op, const ApplyIn<K, T>& in, RowScratch<K, T>& sm,
                                               const RowIdx<K>& ix, T (&y)[K]) {
    const PoisGeom<T>& g = op.g;
    const DevBases<T>& b = op.b;
    const int t = ix.t, lw = ix.lw;
    const bool act = ix.active;
    const T(&xr)[K] = in.xr;
    const T(&xc)[K] = in.xc;
    const T(&g11)[K] = in.g11;
    const T(&g12r)[K] = in.g12r;
    const T(&g22)[K] = in.g22;
    const T(&g12c)[K] = in.g12c;
    const T(&fa)[4] = in.fa;
    const T(&fb)[4] = in.fb;
    const T(&nfa)[4] = in.nfa;
    const T(&nfb)[4] = in.nfb;
    const T(&ntv)[4] = in.ntv;
    const T(&ntg)[4] = in.ntg;
    const int(&code)[4] = in.code;
    T Dc[K], Dr[K];  // column t and column K-1-t of D (thread-dependent basis entries)
#pragma unroll
    for (int m = 0; m < K; ++m) {
        Dc[m] = b.D[m * K + t];
        Dr[m] = b.D[m * K + (K - 1 - t)];
    }
    // own traces; common values on interior (average) and Dirichlet (zero) faces
    T tv[4], tg[4], com[4];
    row_traces<K, T>(b, xr, xc, tv, tg);
#pragma unroll
    for (int f = 0; f < 4; ++f) com[f] = code[f] >= 0 ? T(0.5) * (tv[f] + ntv[f]) : T(0);
    // homogeneous Neumann faces: com = Minv r, r_m = -fa_m (tg_m - tv_m g'(+-1)), the K x K
    // common-value system of src/HO_2D.cpp:2899-2924 inverted once at setup
    bool neu = false;
#pragma unroll
    for (int f = 0; f < 4; ++f) neu |= act && code[f] <= -2;
    if (__any_sync(0xffffffffu, neu)) {
        if (act) {
#pragma unroll
            for (int f = 0; f < 4; ++f) sm.nr[lw][f][t] = -fa[f] * (tg[f] - tv[f] * b.gp[f & 1]);
        }
        __syncwarp();
        if (act) {
#pragma unroll
            for (int f = 0; f < 4; ++f) {
                if (code[f] > -2) continue;
                const T* mi = g.minv + ((size_t)(-2 - code[f]) * K + t) * K;
                T acc = T(0);
#pragma unroll
                for (int m = 0; m < K; ++m) acc += __ldg(mi + m) * sm.nr[lw][f][m];
                com[f] = acc;
            }
        }
    }
    if (act) {
#pragma unroll
        for (int f = 0; f < 4; ++f) sm.com[lw][f][t] = com[f];
    }
    // contravariant gradient (src/HO_2D.cpp:2775-2792): d/dxi along row t, d/deta along
    // column t, each with the Radau corrections of its own face points
    T dx[K], de[K];
#pragma unroll
    for (int i = 0; i < K; ++i) {
        T s = T(0);
#pragma unroll
        for (int d = 0; d < K; ++d) s += xr[d] * b.D[d * K + i];
        s += (com[0] - tv[0]) * b.gR[i * 2 + 0];
        s += (com[1] - tv[1]) * b.gR[i * 2 + 1];
        dx[i] = s;
    }
#pragma unroll
    for (int j = 0; j < K; ++j) {
        T s = T(0);
#pragma unroll
        for (int d = 0; d < K; ++d) s += xc[d] * b.D[d * K + j];
        s += (com[2] - tv[2]) * b.gR[j * 2 + 0];
        s += (com[3] - tv[3]) * b.gR[j * 2 + 1];
        de[j] = s;
    }
    // a = dx g11 + de g12 along row t; b = de g22 + dx g12 down column t
    T der[K], dxc[K];
    col_to_row<K, T>(sm.tr[0][lw], de, der, t, act);  // (the barrier also publishes sm.com)
    rows_to_col<K, T>(sm.tr[1][lw], dx, dxc, t, act);
    T a[K], bb[K];
#pragma unroll
    for (int i = 0; i < K; ++i) {
        a[i] = dx[i] * g11[i] + der[i] * g12r[i];
        bb[i] = de[i] * g22[i] + dxc[i] * g12c[i];
    }
    // common normal fluxes at face point t of each face, then the jumps against the
    // interior flux extrapolated to it
    T cg[4];
#pragma unroll
    for (int f = 0; f < 4; ++f) {
        T cm[K];
#pragma unroll
        for (int m = 0; m < K; ++m) cm[m] = sm.com[lw][f][m];
        T cross = T(0);
#pragma unroll
        for (int m = 0; m < K; ++m) cross += cm[m] * Dc[m];
        const T dv = tg[f] + (com[f] - tv[f]) * b.gp[f & 1];
        const T fl = dv * fa[f] - cross * fb[f];
        T c;
        if (code[f] <= -2) {
            c = T(0);
        } else if (code[f] < 0) {
            c = fl;
        } else {
            const int nijp = code[f] & 3, rev = code[f] >> 2;
            T crn = cross;
            if (rev) {
                crn = T(0);
#pragma unroll
                for (int m = 0; m < K; ++m) crn += cm[K - 1 - m] * Dr[m];
            }
            const T gpn = (nijp & 1) ? b.gp[1] : b.gp[0];
            const T dvn = ntg[f] + (com[f] - ntv[f]) * gpn;
            const T fln = dvn * nfa[f] - crn * nfb[f];
            c = T(0.5) * (fl + T(2 * ((f + nijp) % 2) - 1) * fln);
        }
        // flux jump: W/E against row t of a, S/N against column t of b
        if (f < 2) {
#pragma unroll
            for (int d = 0; d < K; ++d) c -= a[d] * b.sbb[d * 2 + (f & 1)];
        } else {
#pragma unroll
            for (int d = 0; d < K; ++d) c -= bb[d] * b.sbb[d * 2 + (f & 1)];
        }
        cg[f] = c;
    }
    // divergence: xi part along row t, eta part down column t (moved to rows)
    T yc[K], ycr[K];
#pragma unroll
    for (int j = 0; j < K; ++j) {
        T s = T(0);
#pragma unroll
        for (int d = 0; d < K; ++d) s += bb[d] * b.D[d * K + j];
        s += cg[2] * b.gR[j * 2 + 0] + cg[3] * b.gR[j * 2 + 1];
        yc[j] = s;
    }
    // tr[0] is free again: every lane read its rows of de before the barrier in the dx
    // transpose above
    col_to_row<K, T>(sm.tr[0][lw], yc, ycr, t, act);
#pragma unroll
    for (int i = 0; i < K; ++i) {
        T s = T(0);
#pragma unroll
        for (int d = 0; d < K; ++d) s += a[d] * b.D[d * K + i];
        s += cg[0] * b.gR[i * 2 + 0] + cg[1] * b.gR[i * 2 + 1];
        y[i] = s + ycr[i];
    }
    __syncwarp();  // the scratch may be rewritten by the caller's next use
}

// y = A x with the inputs read from global memory (row_apply_load, row_apply_core).
template <int K, typename T>
__device__ __forceinline__ void row_apply(const MfOp<T>& op, const T* __restrict__ x, const T* __restrict__ tvin,
                                          const T* __restrict__ tgin, RowScratch<K, T>& sm, const RowIdx<K>& ix,
                                          T (&y)[K]) {
    ApplyIn<K, T> in;
    row_apply_load<K, T>(op.g, x, tvin, tgin, ix, in);
    row_apply_core<K, T>(op, in, sm, ix, y);
}

// Face traces of an element block held as rows (row t in `row`), scattered to the
// neighbours' incoming slots dst[f] (-1: none). Warp-collective.
template <int K, typename T>
__device__ __forceinline__ void row_emit_traces(const DevBases<T>& b, T (&buf)[K][K], const T (&row)[K],
                                                const int (&dst)[4], T* __restrict__ tv, T* __restrict__ tg, int t,
                                                bool active) {
    T col[K];
    rows_to_col<K, T>(buf, row, col, t, active);
    if (!active) return;
    T v[4], d[4];
    row_traces<K, T>(b, row, col, v, d);
#pragma unroll
    for (int f = 0; f < 4; ++f) {
        if (dst[f] < 0) continue;
        tv[dst[f]] = v[f];
        tg[dst[f]] = d[f];
    }
}

}  // namespace ho2d
