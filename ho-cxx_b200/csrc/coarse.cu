// coarse.cu -- the coarse part of the two-level Poisson preconditioner (sm_100a).
//
// Level 0 of the coarse space holds one value per element (P0); its smoothed-aggregation
// hierarchy is built on the host (host_amg.cpp). One V(1,1) cycle with SPAI-0 smoothing
// is linear in f, so every level's cycle is stored as three fixed row-padded operators,
//   f_next = M f,   u = S f + Q u_next,
// and the coarsest level as its dense inverse. A cycle is then a chain of sparse
// matrix-vector products with no intermediate residual or correction vectors.
//
// The levels below `top` are small: they run inside ONE thread-block cluster (8 or 16
// CTAs of 1024 threads). Every CTA keeps a full copy of each small level's f and u in its
// own shared memory; each row's result is stored into all copies through distributed
// shared memory, and the hardware cluster barrier separates the phases. The whole
// small-level cycle is therefore one launch with no global-memory round trips and no
// software grid barrier. Levels above `top` (large meshes only) run as grid-wide kernels.
// Level 0's own up step is not launched here: the fine smoothing kernel evaluates
// u0 = S0 f0 + Q0 u1 for the five elements each element needs (krylov.cu, k_mf_post).
//
// All sums are taken in a fixed order (fixed lane-to-entry assignment and xor-shuffle
// trees), so results are bitwise reproducible.
#include <cooperative_groups.h>

#include "device.cuh"
#include "fr_launch.hpp"

namespace cg = cooperative_groups;

namespace ho2d {

namespace {

constexpr int kClusterThreads = 1024;
constexpr int kRowBatch = 2;  // rows a lane group works on at once
constexpr int kChunks = 4;    // row chunks of G entries loaded before any is used

// acc[r] += A_row[r] . x over the row chunks of one lane. All kRowBatch x kChunks loads
// of a step are issued before the first gather, so a lane keeps that many L2 requests in
// flight instead of waiting once per chunk.
template <typename T>
__device__ __forceinline__ void ell_accumulate(const DevEll<T>& A, const T* x, const int (&row)[kRowBatch],
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
                j[r][u] = in ? (A.col ? A.col[e] : k) : 0;
            }
#pragma unroll
        for (int r = 0; r < kRowBatch; ++r)
#pragma unroll
            for (int u = 0; u < kChunks; ++u) acc[r] += v[r][u] * x[j[r][u]];
    }
}

// y_i = A_i . xa (+ B_i . xb) for the rows this thread's lane group owns; all G lanes of a
// group hold the row sum after the shuffle tree. `gid`/`nthreads` enumerate the threads
// of the whole cluster (or grid); `store(i, value, sub)` is called by every lane of the
// group for each valid row.
template <typename T, typename Store>
__device__ __forceinline__ void ell_rows(const DevEll<T>& A, const T* xa, const DevEll<T>* B, const T* xb, int G,
                                         int gid, int nthreads, Store store) {
    const int n = A.n;
    const int group = gid / G, sub = gid % G, ngroups = nthreads / G;
    const int iters = (n + ngroups - 1) / ngroups;
    for (int it = 0; it < iters; it += kRowBatch) {
        T acc[kRowBatch];
        int row[kRowBatch];
        bool ok[kRowBatch];
#pragma unroll
        for (int r = 0; r < kRowBatch; ++r) {
            acc[r] = T(0);
            row[r] = group + (it + r) * ngroups;
            ok[r] = it + r < iters && row[r] < n;
        }
        ell_accumulate<T>(A, xa, row, ok, G, sub, acc);
        if (B) ell_accumulate<T>(*B, xb, row, ok, G, sub, acc);
#pragma unroll
        for (int r = 0; r < kRowBatch; ++r) {
            T a = acc[r];
            for (int off = G >> 1; off > 0; off >>= 1) a += __shfl_xor_sync(0xffffffffu, a, off);
            if (ok[r]) store(row[r], a, sub);
        }
    }
}

// The small levels' cycle in one cluster: downs from f_top (global) into shared copies,
// the dense solve, and ups back to level o, whose u is written to global memory. The
// level table is a __grid_constant__ parameter, so indexing it by level reads the
// parameter bank instead of making a per-thread copy. A row's value is stored into every
// CTA's copy by the lanes of its group (lane r stores rank r, r + G, ...).
template <typename T>
__global__ void __launch_bounds__(kClusterThreads, 1) k_coarse_cluster(const __grid_constant__ Precond<T> pc,
                                                                          const KrylovScalars* sc, int mode) {
    // sc is not written while this kernel runs, so every CTA of the cluster sees the same
    // flag; it is read first and tested only before the global result is written, so its
    // round trip overlaps the first phase's loads
    const bool skip = pc_skip(sc, mode);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* sm = reinterpret_cast<T*>(smem_raw);
    cg::cluster_group cl = cg::this_cluster();
    const int C = (int)cl.num_blocks();
    const int gid = (int)cl.block_rank() * kClusterThreads + (int)threadIdx.x;
    const int nthreads = C * kClusterThreads;
    const int top = pc.top, d = pc.nlev - 1, o = top + 1 < d ? top + 1 : d;
    // every CTA must be running before any CTA stores into its shared memory
    cl.sync();
    auto to_global = [skip](T* y) {
        return [=](int i, T a, int sub) {
            if (sub == 0 && !skip) y[i] = a;
        };
    };
    for (int l = top; l < d; ++l) {  // downs
        const CoarseLevel<T>& L = pc.lev[l];
        const T* x = l == top ? L.f : sm + L.sf;
        const int G = L.M.g;
        auto st = [&](int i, T a, int sub) {
            for (int r = sub; r < C; r += G) cl.map_shared_rank(sm, r)[pc.lev[l + 1].sf + i] = a;
        };
        ell_rows<T>(L.M, x, nullptr, nullptr, G, gid, nthreads, st);
        cl.sync();
    }
    {  // coarsest level
        const CoarseLevel<T>& L = pc.lev[d];
        const T* x = d == top ? L.f : sm + L.sf;
        const int G = pc.dense.g;
        if (d == o) {
            ell_rows<T>(pc.dense, x, nullptr, nullptr, G, gid, nthreads, to_global(L.u));
            return;
        }
        auto st = [&](int i, T a, int sub) {
            for (int r = sub; r < C; r += G) cl.map_shared_rank(sm, r)[L.su + i] = a;
        };
        ell_rows<T>(pc.dense, x, nullptr, nullptr, G, gid, nthreads, st);
        cl.sync();
    }
    for (int l = d - 1; l >= o; --l) {  // ups
        const CoarseLevel<T>& L = pc.lev[l];
        const T* un = sm + pc.lev[l + 1].su;
        const int G = L.S.g;
        if (l == o) {
            ell_rows<T>(L.S, sm + L.sf, &L.Q, un, G, gid, nthreads, to_global(L.u));
        } else {
            auto st = [&](int i, T a, int sub) {
                for (int r = sub; r < C; r += G) cl.map_shared_rank(sm, r)[L.su + i] = a;
            };
            ell_rows<T>(L.S, sm + L.sf, &L.Q, un, G, gid, nthreads, st);
            cl.sync();
        }
    }
}

// grid-wide down (f_next = M f) or up (u = S f + Q u_next) of a large level
template <typename T>
__global__ void k_coarse_rows(DevEll<T> A, const T* __restrict__ xa, DevEll<T> B, const T* __restrict__ xb,
                              int has_b, T* __restrict__ y, const KrylovScalars* sc, int mode) {
    if (pc_skip(sc, mode)) return;
    const int gid = blockIdx.x * blockDim.x + threadIdx.x;
    ell_rows<T>(A, xa, has_b ? &B : nullptr, xb, A.g, gid, gridDim.x * blockDim.x, [=](int i, T a, int sub) {
        if (sub == 0) y[i] = a;
    });
}

template <typename T>
unsigned rows_grid(const DevEll<T>& A) {
    const long long lanes = (long long)A.n * A.g;
    const long long per_block = 256;
    long long blocks = (lanes + per_block * kRowBatch - 1) / (per_block * kRowBatch);
    return (unsigned)(blocks < 1 ? 1 : blocks);
}

template <typename T>
cudaError_t launch_cluster(const Precond<T>& pc, const KrylovScalars* sc, int mode, cudaStream_t s) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)pc.cluster, 1, 1);
    cfg.blockDim = dim3(kClusterThreads, 1, 1);
    cfg.dynamicSmemBytes = (size_t)pc.smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)pc.cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k_coarse_cluster<T>, pc, sc, mode);
}

}  // namespace

template <typename T>
cudaError_t coarse_prepare(Precond<T>& pc) {
    if (pc.nlev <= 0) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(k_coarse_cluster<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, pc.smem);
    if (e != cudaSuccess) return e;
    // 16 CTAs (non-portable size) when the device can co-schedule them, else the portable 8
    pc.cluster = 8;
    if (cudaFuncSetAttribute(k_coarse_cluster<T>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) ==
        cudaSuccess) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(16, 1, 1);
        cfg.blockDim = dim3(kClusterThreads, 1, 1);
        cfg.dynamicSmemBytes = (size_t)pc.smem;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = 16;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        int nclusters = 0;
        if (cudaOccupancyMaxActiveClusters(&nclusters, k_coarse_cluster<T>, &cfg) == cudaSuccess && nclusters >= 1)
            pc.cluster = 16;
    }
    cudaGetLastError();  // a refused non-portable query leaves no sticky error
    return cudaSuccess;
}

template <typename T>
cudaError_t coarse_cycle(const Precond<T>& pc, const KrylovScalars* sc, int mode, cudaStream_t s) {
    const int d = pc.nlev - 1, top = pc.top, o = top + 1 < d ? top + 1 : d;
    for (int l = 0; l < top; ++l) {
        const CoarseLevel<T>& L = pc.lev[l];
        k_coarse_rows<T><<<rows_grid(L.M), 256, 0, s>>>(L.M, L.f, DevEll<T>(), nullptr, 0, pc.lev[l + 1].f, sc,
                                                         mode);
    }
    cudaError_t e = launch_cluster<T>(pc, sc, mode, s);
    if (e != cudaSuccess) return e;
    for (int l = o - 1; l >= 1; --l) {
        const CoarseLevel<T>& L = pc.lev[l];
        k_coarse_rows<T><<<rows_grid(L.S), 256, 0, s>>>(L.S, L.f, L.Q, pc.lev[l + 1].u, 1, L.u, sc, mode);
    }
    return cudaGetLastError();
}

template <typename T>
int coarse_launches(const Precond<T>& pc) {
    if (pc.nlev <= 0) return 0;
    const int d = pc.nlev - 1, o = pc.top + 1 < d ? pc.top + 1 : d;
    return pc.top + 1 + (o > 1 ? o - 1 : 0);
}

template <typename T>
CoarseOut<T> coarse_out(const Precond<T>& pc) {
    CoarseOut<T> c;
    if (pc.nlev == 1) {
        c.u0 = pc.lev[0].u;
    } else {
        c.S = pc.lev[0].S;
        c.Q = pc.lev[0].Q;
        c.f0 = pc.lev[0].f;
        c.u1 = pc.lev[1].u;
    }
    return c;
}

#define HO2D_INSTANTIATE_COARSE(T)                                                             \
    template cudaError_t coarse_prepare<T>(Precond<T>&);                                       \
    template cudaError_t coarse_cycle<T>(const Precond<T>&, const KrylovScalars*, int, cudaStream_t); \
    template int coarse_launches<T>(const Precond<T>&);                                        \
    template CoarseOut<T> coarse_out<T>(const Precond<T>&);

HO2D_INSTANTIATE_COARSE(double)
HO2D_INSTANTIATE_COARSE(float)

}  // namespace ho2d
