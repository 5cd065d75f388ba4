// coarse.cu -- the coarse part of the two-level Poisson preconditioner (sm_100a).
//
// Level 0 of the coarse space holds one value per element (P0); its smoothed-aggregation
// hierarchy is built on the host (host_amg.cpp) down to a level of at most kDenseMax
// rows, whose inverse is precomputed. One V(1,1) cycle with SPAI-0 smoothing is linear
// in f, so every other level's cycle is stored as three fixed row-padded operators,
//   f_next = M f,   u = S f + Q u_next,
// and a cycle is a chain of matrix-vector products with no intermediate residual or
// correction vectors:
//   downs    f_{l+1} = M_l f_l              l = 0 .. d-1   (k_coarse_rows)
//   coarsest u_d = A_d^{-1} f_d                             (k_dense_gemv)
//   ups      u_l = S_l f_l + Q_l u_{l+1}    l = d-1 .. 1   (k_coarse_rows)
// The cycle ends with level 0's own up step u0 = S0 f0 + Q0 u1, one value per element,
// which the fine smoothing kernel (krylov.cu, k_mf_post) reads for each element and its
// four face neighbours.
//
// Every kernel spans all SMs and sums in a fixed order (fixed lane-to-entry assignment
// and xor-shuffle trees), so results are bitwise reproducible.
#include <type_traits>

#include "device.cuh"
#include "fr_launch.hpp"

namespace ho2d {

namespace {

constexpr int kRowBatch = 2;  // rows a lane group works on at once
constexpr int kChunks = 4;    // row chunks of G entries loaded before any is used

// acc[r] += A_row[r] . x over the row chunks of one lane. All kRowBatch x kChunks loads
// of a step are issued before the first gather, so a lane keeps that many L2 requests in
// flight instead of waiting once per chunk.
template <typename T, typename X>
__device__ __forceinline__ void ell_accumulate(const DevEll<T>& A, const X& x, const int (&row)[kRowBatch],
                                               const bool (&ok)[kRowBatch], int G, int sub, T (&acc)[kRowBatch]) {
    const int w = A.w;
    const int nch = (w + G - 1) / G;
    for (int c0 = 0; c0 < nch; c0 += kChunks) {
        T v[kRowBatch][kChunks];
        int j[kRowBatch][kChunks];
#pragma unroll
        for (int r = 0; r < kRowBatch; ++r)
#pragma unroll
            for (int u = 0; u < kChunks; ++u) {
                const int k = (c0 + u) * G + sub;
                const bool in = ok[r] && k < w;
                const size_t e = in ? (size_t)row[r] * w + k : 0;
                v[r][u] = in ? A.val[e] : T(0);
                j[r][u] = in ? A.col[e] : 0;
            }
#pragma unroll
        for (int r = 0; r < kRowBatch; ++r)
#pragma unroll
            for (int u = 0; u < kChunks; ++u) acc[r] += v[r][u] * x[j[r][u]];
    }
}

// grid-wide down (f_next = M f) or up (u = S f + Q u_next): G lanes per row, the group's
// lanes combine their partial sums with an xor-shuffle tree. XA is a plain vector, or
// (the level-0 restriction) the right-hand side formed from the element sums.
template <typename T, typename XA>
__global__ void __launch_bounds__(256) k_coarse_rows(DevEll<T> A, XA xa, DevEll<T> B, const T* __restrict__ xb,
                                                      int has_b, T* __restrict__ y, const KrylovScalars* sc) {
    const bool skip = sc->done;  // read early: the round trip overlaps the loads
    const int G = A.g;
    const int gid = blockIdx.x * blockDim.x + threadIdx.x;
    const int group = gid / G, sub = gid % G, ngroups = (int)(gridDim.x * blockDim.x) / G;
    const int iters = (A.n + ngroups - 1) / ngroups;
    for (int it = 0; it < iters; it += kRowBatch) {
        T acc[kRowBatch];
        int row[kRowBatch];
        bool ok[kRowBatch];
#pragma unroll
        for (int r = 0; r < kRowBatch; ++r) {
            acc[r] = T(0);
            row[r] = group + (it + r) * ngroups;
            ok[r] = it + r < iters && row[r] < A.n;
        }
        ell_accumulate<T>(A, xa, row, ok, G, sub, acc);
        if (has_b) ell_accumulate<T>(B, xb, row, ok, G, sub, acc);
#pragma unroll
        for (int r = 0; r < kRowBatch; ++r) {
            T a = acc[r];
            for (int off = G >> 1; off > 0; off >>= 1) a += __shfl_xor_sync(0xffffffffu, a, off);
            if (sub == 0 && ok[r] && !skip) y[row[r]] = a;
        }
    }
}

// 16-byte vector of T
template <typename T>
struct Vec16;
template <>
struct Vec16<float> {
    using type = float4;
    static constexpr int N = 4;
    __device__ static float dot(const float4& a, const float4& b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
    // zero the components at and past `keep` (the tail of a vector that ends inside a piece)
    __device__ static void keep_first(float4& v, int keep) {
        if (keep < 4) v.w = 0.f;
        if (keep < 3) v.z = 0.f;
        if (keep < 2) v.y = 0.f;
    }
};
template <>
struct Vec16<double> {
    using type = double2;
    static constexpr int N = 2;
    __device__ static double dot(const double2& a, const double2& b) { return a.x * b.x + a.y * b.y; }
    __device__ static void keep_first(double2& v, int keep) {
        if (keep < 2) v.y = 0.0;
    }
};

constexpr int kGemvWarps = 8;  // rows (one warp each) per CTA
constexpr int kGemvUnroll = 8;

// u = W f for the dense coarsest inverse W (rows padded to w, a multiple of 4 entries):
// one warp per row, lanes stream the row in 16-byte pieces with kGemvUnroll loads in
// flight; f is read in the same pieces (its buffer is zero-padded past n).
template <typename T>
__global__ void __launch_bounds__(32 * kGemvWarps) k_dense_gemv(DevEll<T> W, const T* __restrict__ f,
                                                                 T* __restrict__ u, const KrylovScalars* sc) {
    using V = Vec16<T>;
    using VT = typename V::type;
    const bool skip = sc->done;
    const int lane = threadIdx.x & 31;
    const int row = blockIdx.x * kGemvWarps + (threadIdx.x >> 5);
    if (row >= W.n) return;
    const int nvec = (W.n + V::N - 1) / V::N;
    const int tail = W.n - (nvec - 1) * V::N;  // entries of the last piece inside the vector
    const VT* wr = reinterpret_cast<const VT*>(W.val + (size_t)row * W.w);
    const VT* fv = reinterpret_cast<const VT*>(f);
    T acc = T(0);
    for (int c0 = lane; c0 < nvec; c0 += 32 * kGemvUnroll) {
        VT a[kGemvUnroll], b[kGemvUnroll];
#pragma unroll
        for (int q = 0; q < kGemvUnroll; ++q) {
            const int c = c0 + 32 * q;
            if (c < nvec) {
                a[q] = __ldg(wr + c);
                b[q] = __ldg(fv + c);
                // the padding of f is zero when written in this precision, but a buffer
                // shared by both precisions may hold the other one's bytes there
                if (c == nvec - 1) V::keep_first(b[q], tail);
            }
        }
#pragma unroll
        for (int q = 0; q < kGemvUnroll; ++q)
            if (c0 + 32 * q < nvec) acc += V::dot(a[q], b[q]);
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
    if (lane == 0 && !skip) u[row] = acc;
}

// u = W f for the dense coarsest inverse stored as BF16 (FP32 preconditioner): one warp per
// row, lanes stream the row in 16-byte pieces of 8 values with kGemvUnroll loads in flight;
// f is read as two float4 per piece (its buffer is zero-padded past n to a multiple of 8).
__global__ void __launch_bounds__(32 * kGemvWarps) k_dense_gemv16(DevEll<float> W, const float* __restrict__ f,
                                                                   float* __restrict__ u, const KrylovScalars* sc) {
    const bool skip = sc->done;
    const int lane = threadIdx.x & 31;
    const int row = blockIdx.x * kGemvWarps + (threadIdx.x >> 5);
    if (row >= W.n) return;
    const int nvec = (W.n + 7) / 8;
    const int tail = W.n - (nvec - 1) * 8;  // values of the last piece inside the vector
    const uint4* wr = reinterpret_cast<const uint4*>(W.val16 + (size_t)row * W.w);
    const float4* fv = reinterpret_cast<const float4*>(f);
    float acc = 0.f;
    for (int c0 = lane; c0 < nvec; c0 += 32 * kGemvUnroll) {
        uint4 a[kGemvUnroll];
        float4 b0[kGemvUnroll], b1[kGemvUnroll];
#pragma unroll
        for (int q = 0; q < kGemvUnroll; ++q) {
            const int c = c0 + 32 * q;
            if (c < nvec) {
                a[q] = __ldg(wr + c);
                b0[q] = __ldg(fv + 2 * c);
                b1[q] = __ldg(fv + 2 * c + 1);
                if (c == nvec - 1) {  // a buffer shared by both precisions may hold other bytes there
                    Vec16<float>::keep_first(b0[q], tail);
                    Vec16<float>::keep_first(b1[q], tail - 4);
                }
            }
        }
#pragma unroll
        for (int q = 0; q < kGemvUnroll; ++q) {
            if (c0 + 32 * q >= nvec) continue;
            const unsigned w4[4] = {a[q].x, a[q].y, a[q].z, a[q].w};
            const float fx[8] = {b0[q].x, b0[q].y, b0[q].z, b0[q].w, b1[q].x, b1[q].y, b1[q].z, b1[q].w};
#pragma unroll
            for (int h = 0; h < 4; ++h) {
                acc += __uint_as_float(w4[h] << 16) * fx[2 * h];
                acc += __uint_as_float(w4[h] & 0xffff0000u) * fx[2 * h + 1];
            }
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
    if (lane == 0 && !skip) u[row] = acc;
}

template <typename T>
void dense_gemv(const DevEll<T>& W, const T* f, T* u, const KrylovScalars* sc, cudaStream_t s) {
    const unsigned gd = (unsigned)((W.n + kGemvWarps - 1) / kGemvWarps);
    if constexpr (std::is_same<T, float>::value) {
        if (W.val16) {
            k_dense_gemv16<<<gd, 32 * kGemvWarps, 0, s>>>(W, f, u, sc);
            return;
        }
    }
    k_dense_gemv<T><<<gd, 32 * kGemvWarps, 0, s>>>(W, f, u, sc);
}

// u0 of element c into every block slot that reads it (Precond::u0dst)
template <typename T>
__device__ __forceinline__ void scatter_u0(const int* __restrict__ u0dst, T* __restrict__ ue5, int c, T a) {
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        const int d = u0dst[c * 5 + k];
        if (d >= 0) ue5[d] = a;
    }
}

// u0 = W f0 when the P0 level itself is the dense one (small meshes): f0 is formed from
// the element sums as it is read, one warp per row, scalar loads
template <typename T>
__global__ void __launch_bounds__(32 * kGemvWarps) k_dense_gemv_f0(DevEll<T> W, BicgVectors<T> v,
                                                                    const int* __restrict__ u0dst,
                                                                    T* __restrict__ ue5, const KrylovScalars* sc,
                                                                    int mode) {
    const bool skip = sc->done;
    const F0<T> f = f0_of(v, sc, mode);
    const int lane = threadIdx.x & 31;
    const int row = blockIdx.x * kGemvWarps + (threadIdx.x >> 5);
    if (row >= W.n) return;
    const T* wr = W.val + (size_t)row * W.w;
    T acc = T(0);
    for (int k = lane; k < W.n; k += 32) acc += __ldg(wr + k) * f[k];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
    if (lane == 0 && !skip) scatter_u0(u0dst, ue5, row, acc);
}

// level-0 restriction with the right-hand side formed from the element sums
template <typename T>
__global__ void __launch_bounds__(256) k_coarse_rows_f0(DevEll<T> M, BicgVectors<T> v, T* __restrict__ y,
                                                         const KrylovScalars* sc, int mode);

template <typename T>
unsigned rows_grid(const DevEll<T>& A) {
    const long long lanes = (long long)A.n * A.g;
    const long long per_block = 256;
    long long blocks = (lanes + per_block * kRowBatch - 1) / (per_block * kRowBatch);
    return (unsigned)(blocks < 1 ? 1 : blocks);
}

template <typename T>
__global__ void __launch_bounds__(256) k_coarse_rows_f0(DevEll<T> M, BicgVectors<T> v, T* __restrict__ y,
                                                         const KrylovScalars* sc, int mode) {
    // the same row loop as k_coarse_rows, gathering f0 = a + cb b + cc c
    const bool skip = sc->done;
    const F0<T> xa = f0_of(v, sc, mode);
    const int G = M.g;
    const int gid = blockIdx.x * blockDim.x + threadIdx.x;
    const int group = gid / G, sub = gid % G, ngroups = (int)(gridDim.x * blockDim.x) / G;
    const int iters = (M.n + ngroups - 1) / ngroups;
    for (int it = 0; it < iters; it += kRowBatch) {
        T acc[kRowBatch];
        int row[kRowBatch];
        bool ok[kRowBatch];
#pragma unroll
        for (int r = 0; r < kRowBatch; ++r) {
            acc[r] = T(0);
            row[r] = group + (it + r) * ngroups;
            ok[r] = it + r < iters && row[r] < M.n;
        }
        ell_accumulate<T>(M, xa, row, ok, G, sub, acc);
#pragma unroll
        for (int r = 0; r < kRowBatch; ++r) {
            T a = acc[r];
            for (int off = G >> 1; off > 0; off >>= 1) a += __shfl_xor_sync(0xffffffffu, a, off);
            if (sub == 0 && ok[r] && !skip) y[row[r]] = a;
        }
    }
}

// level-0 up step u0 = S0 f0 + Q0 u1 with the right-hand side formed from the element sums;
// each row's value goes to the block slots that read it (scatter_u0)
template <typename T>
__global__ void __launch_bounds__(256) k_coarse_up0(DevEll<T> S, DevEll<T> Q, BicgVectors<T> v,
                                                     const T* __restrict__ u1, const int* __restrict__ u0dst,
                                                     T* __restrict__ ue5, const KrylovScalars* sc, int mode) {
    const bool skip = sc->done;
    const F0<T> xa = f0_of(v, sc, mode);
    const int G = S.g;
    const int gid = blockIdx.x * blockDim.x + threadIdx.x;
    const int group = gid / G, sub = gid % G, ngroups = (int)(gridDim.x * blockDim.x) / G;
    const int iters = (S.n + ngroups - 1) / ngroups;
    for (int it = 0; it < iters; it += kRowBatch) {
        T acc[kRowBatch];
        int row[kRowBatch];
        bool ok[kRowBatch];
#pragma unroll
        for (int r = 0; r < kRowBatch; ++r) {
            acc[r] = T(0);
            row[r] = group + (it + r) * ngroups;
            ok[r] = it + r < iters && row[r] < S.n;
        }
        ell_accumulate<T>(S, xa, row, ok, G, sub, acc);
        ell_accumulate<T>(Q, u1, row, ok, G, sub, acc);
#pragma unroll
        for (int r = 0; r < kRowBatch; ++r) {
            T a = acc[r];
            for (int off = G >> 1; off > 0; off >>= 1) a += __shfl_xor_sync(0xffffffffu, a, off);
            if (sub == 0 && ok[r] && !skip) scatter_u0(u0dst, ue5, row[r], a);
        }
    }
}

}  // namespace

template <typename T>
cudaError_t coarse_cycle(const Precond<T>& pc, const BicgVectors<T>& v, const KrylovScalars* sc, int mode,
                         cudaStream_t s) {
    const int d = pc.nlev - 1;
    const unsigned gd = (unsigned)((pc.dense.n + kGemvWarps - 1) / kGemvWarps);
    if (d == 0) {
        k_dense_gemv_f0<T><<<gd, 32 * kGemvWarps, 0, s>>>(pc.dense, v, pc.u0dst, pc.ue5, sc, mode);
        return cudaGetLastError();
    }
    k_coarse_rows_f0<T><<<rows_grid(pc.lev[0].M), 256, 0, s>>>(pc.lev[0].M, v, pc.lev[1].f, sc, mode);
    for (int l = 1; l < d; ++l) {
        const CoarseLevel<T>& L = pc.lev[l];
        k_coarse_rows<T, const T*><<<rows_grid(L.M), 256, 0, s>>>(L.M, L.f, DevEll<T>(), nullptr, 0,
                                                                   pc.lev[l + 1].f, sc);
    }
    dense_gemv<T>(pc.dense, pc.lev[d].f, pc.lev[d].u, sc, s);
    for (int l = d - 1; l >= 1; --l) {
        const CoarseLevel<T>& L = pc.lev[l];
        k_coarse_rows<T, const T*><<<rows_grid(L.S), 256, 0, s>>>(L.S, L.f, L.Q, pc.lev[l + 1].u, 1, L.u, sc);
    }
    const CoarseLevel<T>& L0 = pc.lev[0];
    k_coarse_up0<T><<<rows_grid(L0.S), 256, 0, s>>>(L0.S, L0.Q, v, pc.lev[1].u, pc.u0dst, pc.ue5, sc, mode);
    return cudaGetLastError();
}

// The whole cycle on a plain level-0 right-hand side f0 (N entries, zero-padded to a
// multiple of 4): u0 = cycle(f0) in pc.lev[0].u, level 0's own up step included. Used by
// the transposed solve of the adjoint, whose preconditioner forms f0 in its own kernel.
template <typename T>
cudaError_t coarse_cycle_vec(const Precond<T>& pc, const T* f0, const KrylovScalars* sc, cudaStream_t s) {
    const int d = pc.nlev - 1;
    if (d < 0) return cudaSuccess;
    const unsigned gd = (unsigned)((pc.dense.n + kGemvWarps - 1) / kGemvWarps);
    if (d == 0) {
        dense_gemv<T>(pc.dense, f0, pc.lev[0].u, sc, s);
        return cudaGetLastError();
    }
    k_coarse_rows<T, const T*><<<rows_grid(pc.lev[0].M), 256, 0, s>>>(pc.lev[0].M, f0, DevEll<T>(), nullptr, 0,
                                                                       pc.lev[1].f, sc);
    for (int l = 1; l < d; ++l) {
        const CoarseLevel<T>& L = pc.lev[l];
        k_coarse_rows<T, const T*><<<rows_grid(L.M), 256, 0, s>>>(L.M, L.f, DevEll<T>(), nullptr, 0,
                                                                   pc.lev[l + 1].f, sc);
    }
    dense_gemv<T>(pc.dense, pc.lev[d].f, pc.lev[d].u, sc, s);
    for (int l = d - 1; l >= 1; --l) {
        const CoarseLevel<T>& L = pc.lev[l];
        k_coarse_rows<T, const T*><<<rows_grid(L.S), 256, 0, s>>>(L.S, L.f, L.Q, pc.lev[l + 1].u, 1, L.u, sc);
    }
    const CoarseLevel<T>& L0 = pc.lev[0];
    k_coarse_rows<T, const T*><<<rows_grid(L0.S), 256, 0, s>>>(L0.S, f0, L0.Q, pc.lev[1].u, 1, L0.u, sc);
    return cudaGetLastError();
}

template <typename T>
int coarse_vec_launches(const Precond<T>& pc) {
    if (pc.nlev <= 0) return 0;
    const int d = pc.nlev - 1;
    return d == 0 ? 1 : 2 * d + 1;
}

template <typename T>
int coarse_launches(const Precond<T>& pc) {
    if (pc.nlev <= 0) return 0;
    const int d = pc.nlev - 1;
    return d == 0 ? 1 : d + 1 + (d - 1) + 1;
}

// Algorithmic bytes of one coarse cycle as coarse_cycle launches it: every row-padded
// operator's values and column indices, the dense inverse, each level's right-hand side
// read and result written; the level-0 right-hand side is formed from three element-sum
// vectors.
template <typename T>
int coarse_cycle_bytes(const Precond<T>& pc) {
    if (pc.nlev <= 0) return 0;
    const int d = pc.nlev - 1;
    auto ell = [](const DevEll<T>& A) { return (double)A.n * A.w * (sizeof(T) + (A.col ? 4 : 0)); };
    const double dsz = pc.dense.val16 ? 2.0 : (double)sizeof(T);
    double b = (double)pc.dense.n * pc.dense.w * dsz + 2.0 * pc.dense.n * sizeof(T);
    if (d == 0) return (int)(b + 3.0 * pc.dense.n * sizeof(T));
    b += ell(pc.lev[0].M) + 3.0 * pc.lev[0].n * sizeof(T) + pc.lev[1].n * sizeof(T);
    for (int l = 1; l < d; ++l) b += ell(pc.lev[l].M) + (double)(pc.lev[l].n + pc.lev[l + 1].n) * sizeof(T);
    for (int l = d - 1; l >= 1; --l)
        b += ell(pc.lev[l].S) + ell(pc.lev[l].Q) + (double)(2 * pc.lev[l].n + pc.lev[l + 1].n) * sizeof(T);
    b += ell(pc.lev[0].S) + ell(pc.lev[0].Q) + (double)(4 * pc.lev[0].n + pc.lev[1].n) * sizeof(T);
    return (int)b;
}

template <typename T>
CoarseOut<T> coarse_out(const Precond<T>& pc) {
    CoarseOut<T> c;
    c.ue5 = pc.ue5;
    return c;
}

#define HO2D_INSTANTIATE_COARSE(T)                                                                   \
    template cudaError_t coarse_cycle<T>(const Precond<T>&, const BicgVectors<T>&, const KrylovScalars*, int,  \
                                         cudaStream_t);                                                      \
    template int coarse_launches<T>(const Precond<T>&);                                              \
    template cudaError_t coarse_cycle_vec<T>(const Precond<T>&, const T*, const KrylovScalars*, cudaStream_t); \
    template int coarse_vec_launches<T>(const Precond<T>&);                                          \
    template CoarseOut<T> coarse_out<T>(const Precond<T>&);                                          \
    template int coarse_cycle_bytes<T>(const Precond<T>&);

HO2D_INSTANTIATE_COARSE(double)
HO2D_INSTANTIATE_COARSE(float)

}  // namespace ho2d
