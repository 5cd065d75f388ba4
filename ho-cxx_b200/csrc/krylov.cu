// krylov.cu -- matrix-free FR Poisson operator and preconditioned BiCGSTAB (sm_100a).
//
// Operator. The reference assembles the FR Laplacian into a CSR matrix with up to
// 5 K^4 entries per element (src/HO_2D.cpp:1533-1804, 3011-3062) and hands it to AMGCL.
// That matrix is exactly the method-2 FR Laplacian of calc_RHS_diffusion applied with
// homogeneous Poisson boundary values, so here A x is evaluated matrix-free from face
// traces (row_apply in rows.cuh): per DOF it reads x, 3 metric coefficients and a share
// of the face data instead of 5 K^2 matrix entries. Every kernel that produces
// a vector the operator is applied to next also writes that vector's face traces, so
// one operator application is one launch.
//
// Solver. Right-preconditioned BiCGSTAB (van der Vorst 1992) replacing AMGCL's BiCGSTAB
// (src/HO_2D.hpp:53-54, src/HO_2D.cpp:1960). Preconditioner, two-level V(0,1):
//   coarse:  e = P A1^{-1} P^T f, P = element-wise constants, A1 = P^T A P, A1^{-1}
//            approximated by one smoothed-aggregation V-cycle (host_amg.cpp);
//   smooth:  z = e + w D^{-1} (f - A e), D = the K^2 x K^2 diagonal blocks of A; A e is
//            cheap because e is element-wise constant (A e = sum_s rowsum_s e_s).
// With HO2D_PRECOND=bj the preconditioner is z = D^{-1} f (block-Jacobi).
// Scalars stay on the device; every vector update fuses the dot products the next step
// needs, reduced deterministically (per-CTA partials summed in a fixed order by the last
// CTA to finish); a `done` flag turns the rest of an enqueued batch into no-ops, so the
// host only polls for convergence every few iterations.
#include <type_traits>

#include "device.cuh"
#include "fr_device.cuh"
#include "fr_launch.hpp"
#include "kron_apply.cuh"
#include "rows.cuh"
#include "apply_stage.cuh"
#include "bulk_copy.cuh"

namespace ho2d {

namespace {

// Deterministic grid-wide sum of NV values per thread, in two levels so no CTA reads more
// than a few hundred partials: every CTA stores its sums; the last CTA to finish within
// each group of kReduceGroup consecutive CTAs adds the group's sums (fixed order) and
// stores the group total; the last group to finish adds the group totals (fixed order)
// and gets `out`, returning true in that CTA only. Counters: counter[0] for the groups,
// counter[1 + g] for group g; every one is back to zero when the kernel ends. partials
// holds NV x (gridDim.x + the number of groups) doubles. Collective (all threads).
constexpr int kReduceGroup = 64;

template <int NV>
__device__ __forceinline__ bool grid_reduce(const double (&v)[NV], double* partials, unsigned* counter,
                                            double (&out)[NV]) {
    __shared__ double red[NV][32];
    __shared__ double fin[NV];
    __shared__ bool s_last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int G = (int)gridDim.x, ng = (G + kReduceGroup - 1) / kReduceGroup;
    const int grp = (int)blockIdx.x / kReduceGroup;
    const int g0 = grp * kReduceGroup, gs = min(kReduceGroup, G - g0);
    double* gpart = partials + (size_t)NV * G;
#pragma unroll
    for (int j = 0; j < NV; ++j) {
        double x = v[j];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) x += __shfl_xor_sync(0xffffffffu, x, off);
        if (lane == 0) red[j][warp] = x;
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int j = 0; j < NV; ++j) {
            double x = lane < nw ? red[j][lane] : 0.0;
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) x += __shfl_xor_sync(0xffffffffu, x, off);
            if (lane == 0) partials[j * G + blockIdx.x] = x;
        }
        __threadfence();
    }
    __syncthreads();
    if (threadIdx.x == 0) s_last = (atomicAdd(&counter[1 + grp], 1u) == (unsigned)gs - 1);
    __syncthreads();
    if (!s_last) return false;
    // the group's total: warp 0 adds its <= 64 CTA sums (lanes l and l + 32, then a tree)
    __threadfence();
    if (warp == 0) {
#pragma unroll
        for (int j = 0; j < NV; ++j) {
            double x = lane < gs ? __ldcg(&partials[j * G + g0 + lane]) : 0.0;
            if (lane + 32 < gs) x += __ldcg(&partials[j * G + g0 + lane + 32]);
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) x += __shfl_xor_sync(0xffffffffu, x, off);
            if (lane == 0) gpart[j * ng + grp] = x;
        }
        if (lane == 0) counter[1 + grp] = 0u;
        __threadfence();
    }
    __syncthreads();
    if (threadIdx.x == 0) s_last = (atomicAdd(&counter[0], 1u) == (unsigned)ng - 1);
    __syncthreads();
    if (!s_last) return false;
    __threadfence();
#pragma unroll
    for (int j = 0; j < NV; ++j) {
        double x = 0.0;
#pragma unroll 4
        for (int i = threadIdx.x; i < ng; i += blockDim.x) x += __ldcg(&gpart[j * ng + i]);
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) x += __shfl_xor_sync(0xffffffffu, x, off);
        if (lane == 0) red[j][warp] = x;
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int j = 0; j < NV; ++j) {
            double x = lane < nw ? red[j][lane] : 0.0;
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) x += __shfl_xor_sync(0xffffffffu, x, off);
            if (lane == 0) fin[j] = x;
        }
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < NV; ++j) out[j] = fin[j];
    if (threadIdx.x == 0) counter[0] = 0u;
    return true;
}

}  // namespace

// ---------------------------------------------------------------- fine-level kernels
// The operator kernels run row-parallel (rows.cuh): K threads per element, Rows<K>::EPC
// elements per CTA.
template <int K>
static __host__ __device__ constexpr unsigned rgrid_of(int N) {
    return (unsigned)((N + Rows<K>::EPC - 1) / Rows<K>::EPC);
}

// CTAs of one full wave of each reducing row kernel (resident CTAs per SM x SMs), per K and
// precision ([K][0] FP64, [K][1] FP32): those kernels loop over element tiles, so one wave
// covers any mesh and each CTA reduces once. Set by krylov_configure.
struct WaveSizes {
    unsigned init = 0, v = 0, t = 0, xr = 0, res = 0, v_st = 0, t_st = 0;
};
static WaveSizes g_wave[9][2];

template <int K, typename T>
static unsigned wave_of(unsigned WaveSizes::*which, int N) {
    const unsigned w = g_wave[K][std::is_same<T, float>::value ? 1 : 0].*which;
    const unsigned nt = rgrid_of<K>(N);
    return w == 0 || w > nt ? nt : w;
}

// incoming face traces of x (the operand of an operator application that no Krylov
// kernel produced: the initial guess, a refinement iterate, a caller's vector)
template <int K, typename T>
__global__ void __launch_bounds__(Rows<K>::THREADS) k_trace_in(MfOp<T> op, const T* __restrict__ x, T* __restrict__ tv,
                                                                T* __restrict__ tg) {
    __shared__ T buf[Rows<K>::WARPS][Rows<K>::EPW][K][K];
    const RowIdx<K> ix(op.g.N, blockIdx.x);
    T row[K];
    int dst[4];
    if (ix.active) {
        load_row<K, T>(x + (size_t)ix.el * K * K + ix.t * K, row);
        load4i(op.g.scat + ((size_t)ix.el * K + ix.t) * 4, dst);
    }
    row_emit_traces<K, T>(op.b, buf[ix.warp][ix.lw], row, dst, tv, tg, ix.t, ix.active);
}

// r = b - A x (x's traces in xtv/xtg), rhat = r; ||r||^2, ||b||^2; element sums of r. Like
// every reducing row kernel it runs as one wave of CTAs, each taking element tiles
// blockIdx.x, blockIdx.x + gridDim.x, ... and reducing once.
template <int K, typename T>
__global__ void __launch_bounds__(Rows<K>::THREADS) k_mf_init(MfOp<T> op, BicgVectors<T> v, ReduceScratch rs) {
    __shared__ RowScratch<K, T> sm[Rows<K>::WARPS];
    const int ntiles = (int)rgrid_of<K>(op.g.N);
    double part[2] = {0.0, 0.0};
    auto tile_body = [&](int tile) {
        const RowIdx<K> ix(op.g.N, tile);
        T y[K];
        row_apply<K, T>(op, v.x, v.xtv, v.xtg, sm[ix.warp], ix, y);
        T rsum = T(0);
        if (ix.active) {
            const size_t p = (size_t)ix.el * K * K + ix.t * K;
            T bb[K], r[K];
            load_row<K, T>(v.b + p, bb);
#pragma unroll
            for (int i = 0; i < K; ++i) {
                r[i] = bb[i] - y[i];
                rsum += r[i];
                part[0] += double(r[i]) * double(r[i]);
                part[1] += double(bb[i]) * double(bb[i]);
            }
            store_row<K, T>(v.r + p, r);
            store_row<K, T>(v.rhat + p, r);
        }
        const T tot = element_total<K, T>(rsum, ix.lw);
        if (ix.active && ix.t == 0) v.er[ix.el] = tot;
    };
    // FP32: one wave of CTAs over the tiles; FP64 keeps one tile per CTA (the loop would
    // push the operator past the register file)
    if constexpr (sizeof(T) == 4) {
#pragma unroll 1
        for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) tile_body(tile);
    } else {
        if ((int)blockIdx.x < ntiles) tile_body(blockIdx.x);
    }
    double out[2];
    if (grid_reduce<2>(part, rs.partials, rs.counter, out) && threadIdx.x == 0) {
        KrylovScalars* sc = rs.sc;
        sc->rnorm2 = out[0];
        sc->bnorm2 = out[1];
        sc->eps2 = sc->tol * sc->tol * out[1];
        sc->rho = out[0];
        sc->rho_old = sc->alpha = sc->omega = 1.0;
        sc->beta = 0.0;
        sc->it = 0;
        sc->breakdown = 0;
        sc->s_exit = 0;
        sc->zero_rhs = out[1] == 0.0;
        sc->done = (out[1] == 0.0) || (out[0] <= sc->eps2);
    }
}

template <typename T>
__global__ void k_zero_if(T* x, size_t n, const KrylovScalars* sc) {
    if (!sc->zero_rhs) return;
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] = T(0);
}


// The smoother's element data (BS): 0 = inverse blocks in T; 1 = inverse blocks as BF16 bit
// patterns (FP32 smoother); 2 = Kronecker-sum factors, with the exact blocks only for the
// elements the fit does not approximate well (FP32 smoother). Each element's data starts on
// a 16-byte boundary (padded_count). A warp's EPW blocks (or factor sets) are one
// contiguous span, copied into shared memory by one bulk copy when the span is at most
// 26 KB (so a CTA's four spans leave room for two CTAs per SM); larger blocks are read
// from global memory directly.
template <int K, typename T, int BS>
struct PostRows {
    using DT = typename std::conditional<BS == 1, unsigned short, T>::type;
    static constexpr int K2 = K * K, K4 = K2 * K2;
    static constexpr int STRIDE = padded_count(K4, (int)sizeof(DT));  // values of DT per element
    static constexpr int KF = 4 * K2 + 2 * K;                      // Kronecker factors per element
    static constexpr int KFS = padded_count(KF, (int)sizeof(T));
    static constexpr int XSTRIDE = padded_count(K4, (int)sizeof(T));  // compact exact blocks (BS 2)
    // bytes of one element's staged data: its inverse block, or (BS 2) its factors
    static constexpr int ELEM = BS == 2 ? KFS * (int)sizeof(T) : STRIDE * (int)sizeof(DT);
    static constexpr int SPAN = Rows<K>::EPW * ELEM;  // bytes per warp
    static constexpr bool kStage = SPAN <= 26 * 1024;
    static constexpr int SMEM = kStage ? Rows<K>::WARPS * SPAN : 0;  // dynamic shared memory
};

__device__ __forceinline__ float block_value(unsigned short b) { return __uint_as_float((unsigned)b << 16); }
template <typename T>
__device__ __forceinline__ T block_value(T v) {
    return v;
}

// K consecutive block values (row t of one r-slice of an element block, [rs][ij] layout),
// widened to T; vector loads as wide as the slice's alignment allows (its offset is a
// multiple of K values from a 16-byte-aligned block start).
template <int K, typename T, typename DT>
__device__ __forceinline__ void load_slice(const DT* p, T (&v)[K]) {
    constexpr int AL = (K * (int)sizeof(DT)) % 16 == 0 ? 16 : ((K * (int)sizeof(DT)) % 8 == 0 ? 8 : ((K * (int)sizeof(DT)) % 4 == 0 ? 4 : (int)sizeof(DT)));
    if constexpr (sizeof(DT) == 2) {
        if constexpr (AL >= 4) {
#pragma unroll
            for (int i = 0; i < K; i += 2) {
                const unsigned w = *reinterpret_cast<const unsigned*>(p + i);
                v[i] = __uint_as_float(w << 16);
                v[i + 1] = __uint_as_float(w & 0xffff0000u);
            }
        } else {
#pragma unroll
            for (int i = 0; i < K; ++i) v[i] = block_value(p[i]);
        }
    } else if constexpr (AL == 16 && sizeof(DT) == 4) {
#pragma unroll
        for (int i = 0; i < K; i += 4) {
            const float4 q = *reinterpret_cast<const float4*>(p + i);
            v[i] = q.x;
            v[i + 1] = q.y;
            v[i + 2] = q.z;
            v[i + 3] = q.w;
        }
    } else if constexpr (AL >= 8 && sizeof(DT) == 4) {
#pragma unroll
        for (int i = 0; i < K; i += 2) {
            const float2 q = *reinterpret_cast<const float2*>(p + i);
            v[i] = q.x;
            v[i + 1] = q.y;
        }
    } else if constexpr (AL == 16 && sizeof(DT) == 8) {
#pragma unroll
        for (int i = 0; i < K; i += 2) {
            const double2 q = *reinterpret_cast<const double2*>(p + i);
            v[i] = q.x;
            v[i + 1] = q.y;
        }
    } else {
#pragma unroll
        for (int i = 0; i < K; ++i) v[i] = T(p[i]);
    }
}

// acc[i] = sum_r blk[r][t K + i] sr[r] over the K^2 values r of the element's residual sr
// (shared memory): row t of D^-1 sr.
template <int K, typename T, typename DT>
__device__ __forceinline__ void block_rows(const DT* blk, const T* sr, int t, T (&acc)[K]) {
    constexpr int K2 = K * K;
#pragma unroll
    for (int i = 0; i < K; ++i) acc[i] = T(0);
#pragma unroll 4
    for (int r = 0; r < K2; ++r) {
        T m[K];
        load_slice<K, T, DT>(blk + r * K2 + t * K, m);
        const T s = sr[r];
#pragma unroll
        for (int i = 0; i < K; ++i) acc[i] += m[i] * s;
    }
}

// The smoother's element inverse M (exact block, BF16 block or Kronecker-sum factors)
// applied to one element vector held in shared memory (srow, K^2 values, [j][i]): row t of
// M srow into acc. For BS 2 the transposes are warp-collective, so every lane runs them;
// zb is a K x K scratch of the element. Warp-collective.
template <int K, typename T, int BS>
__device__ __forceinline__ void smoother_rows(const MfOp<T>& op, const typename PostRows<K, T, BS>::DT* blk,
                                              const T* fk, int kx, const T* srow, T (&zb)[K][K], int t, bool act,
                                              T (&acc)[K]) {
    using PS = PostRows<K, T, BS>;
    constexpr int K2 = K * K;
    if constexpr (BS == 2) {
        // exact block where the fit falls back, Kronecker-sum step (fast diagonalisation,
        // the element body of kron_apply.cuh by rows) for the others
        const bool kr = act && kx < 0;
        if (act && kx >= 0) block_rows<K, T, T>(op.kron_exact + (size_t)kx * PS::XSTRIDE, srow, t, acc);
        const T *vx = fk, *vxi = fk + K2, *vy = fk + 2 * K2, *vyi = fk + 3 * K2, *lx = fk + 4 * K2, *ly = lx + K;
        T c1[K], r1[K], r2[K], c2[K], c3[K], r3[K];
        // column t of Vy^-1 R
#pragma unroll
        for (int j = 0; j < K; ++j) {
            T s = T(0);
            if (kr) {
#pragma unroll
                for (int l = 0; l < K; ++l) s += vyi[j * K + l] * srow[l * K + t];
            }
            c1[j] = s;
        }
        col_to_row<K, T>(zb, c1, r1, t, kr);
        // row t of (Vy^-1 R Vx^-T) ./ (ly_t + lx_i)
#pragma unroll
        for (int i = 0; i < K; ++i) {
            T s = T(0);
            if (kr) {
#pragma unroll
                for (int k = 0; k < K; ++k) s += r1[k] * vxi[i * K + k];
                s = s / (ly[t] + lx[i]);
            }
            r2[i] = s;
        }
        __syncwarp();  // zb is rewritten next
        rows_to_col<K, T>(zb, r2, c2, t, kr);
        // column t of Vy (that), then row t of the product with Vx^T
#pragma unroll
        for (int j = 0; j < K; ++j) {
            T s = T(0);
            if (kr) {
#pragma unroll
                for (int l = 0; l < K; ++l) s += vy[j * K + l] * c2[l];
            }
            c3[j] = s;
        }
        __syncwarp();
        col_to_row<K, T>(zb, c3, r3, t, kr);
        if (kr) {
#pragma unroll
            for (int i = 0; i < K; ++i) {
                T s = T(0);
#pragma unroll
                for (int k = 0; k < K; ++k) s += r3[k] * vx[i * K + k];
                acc[i] = s;
            }
        }
        __syncwarp();  // zb may be reused by the caller
    } else {
        if (act) block_rows<K, T, typename PS::DT>(blk, srow, t, acc);
    }
}

// The warp's smoother element data: one bulk copy of its EPW inverse blocks (or factor
// sets) into its slice of the dynamic shared memory when PostRows::kStage, issued by lane 0
// on barrier bar; blk/fk point at this element's data (staged or global).
template <int K, typename T, int BS>
struct SmootherData {
    const typename PostRows<K, T, BS>::DT* blk = nullptr;
    const T* fk = nullptr;
    int kx = -1;
    int wn = 0;
    __device__ __forceinline__ void start(const MfOp<T>& op, const RowIdx<K>& ix, unsigned char* dyn, uint64_t* bar,
                                          bool issue) {
        using PS = PostRows<K, T, BS>;
        using DT = typename PS::DT;
        constexpr int EPW = Rows<K>::EPW;
        const DT* dsrc;
        if constexpr (BS == 1) dsrc = op.dinv_bf16;
        else dsrc = op.dinv;
        const int wel0 = (blockIdx.x * Rows<K>::WARPS + ix.warp) * EPW;
        wn = min(EPW, op.g.N - wel0);
        blk = dsrc + (size_t)(ix.active ? ix.el : 0) * PS::STRIDE;
        fk = BS == 2 ? op.kron_f + (size_t)(ix.active ? ix.el : 0) * PS::KFS : nullptr;
        if constexpr (BS == 2) {
            if (ix.active) kx = op.kron_x[ix.el];
        }
        if constexpr (PS::kStage) {
            unsigned char* stage = dyn + (size_t)ix.warp * PS::SPAN;
            if (issue && wn > 0 && ix.lane == 0) {
                const unsigned char* src = BS == 2 ? reinterpret_cast<const unsigned char*>(op.kron_f)
                                                   : reinterpret_cast<const unsigned char*>(dsrc);
                mbar_init(bar);
                const unsigned bytes = (unsigned)(wn * PS::ELEM);
                mbar_arrive_expect(bar, bytes);
                bulk_load(stage, src + (size_t)wel0 * PS::ELEM, bytes, bar);
            }
            if constexpr (BS == 2) fk = reinterpret_cast<const T*>(stage + (size_t)ix.lw * PS::ELEM);
            else blk = reinterpret_cast<const DT*>(stage + (size_t)ix.lw * PS::ELEM);
        }
    }
    // wait for the copy; a wait that runs out is recorded for the host, the copy gets a
    // second bounded wait, and the kernel runs on so its reductions stay consistent
    __device__ __forceinline__ void wait(uint64_t* bar, KrylovScalars* sc, int lane) {
        if constexpr (PostRows<K, T, BS>::kStage) {
            if (wn > 0 && !mbar_wait_bounded(bar, 0, kBulkWaitPolls)) {
                if (lane == 0) atomicExch(&sc->dev_error, 1);
                mbar_wait_bounded(bar, 0, kBulkWaitPolls);
            }
        }
    }
};

// Fine part of one preconditioner application, with the BiCGSTAB vector update that
// produces its operand:
//   mode 0:  p = r + beta (p - omega v)  (p = r on the first iteration),  f = p
//   mode 1:  s = r - alpha v, ||s||^2 (s_exit test),                      f = s
// then zf = M f with the smoother's element inverse M (exact FP32/FP64 block, BF16 block or
// Kronecker-sum factors). It needs nothing of the coarse cycle, which runs beside it on a
// second stream; k_post_b combines the two. Mode 0 also stores the element sums of the new
// p for the next iteration. Row-parallel (rows.cuh): thread t of an element owns row t. The
// warp's element data are requested first, by one bulk copy into shared memory
// (PostRows::kStage), so the copy overlaps the vector loads.
template <int K, typename T, int BS = 0>
__global__ void __launch_bounds__(Rows<K>::THREADS) k_post_a(MfOp<T> op, BicgVectors<T> v, int has_coarse,
                                                              ReduceScratch rs, int mode) {
    using R = Rows<K>;
    constexpr int K2 = R::K2, EPW = R::EPW;
    KrylovScalars* sc = rs.sc;
    const int done = sc->done;  // uniform; read early so the round trip overlaps the loads
    extern __shared__ __align__(128) unsigned char post_dyn[];
    __shared__ __align__(8) uint64_t bar[R::WARPS];
    __shared__ __align__(16) T sr[R::WARPS][EPW][K2];
    __shared__ T zb[R::WARPS][EPW][K][K];
    const RowIdx<K> ix(op.g.N, blockIdx.x);
    const int t = ix.t, lw = ix.lw, el = ix.el;
    const bool act = ix.active;
    SmootherData<K, T, BS> sd;
    sd.start(op, ix, post_dyn, &bar[ix.warp], !done);
    const size_t p = (size_t)el * K2 + t * K;
    T rr[K], vv[K], pp[K];
    if (act) {
        load_row<K, T>(v.r + p, rr);
        load_row<K, T>(v.v + p, vv);
        if (mode == 0) load_row<K, T>(v.p + p, pp);
    }
    if (mode == 0 && has_coarse && act && t == 0) {
        const F0<T> f0 = f0_of(v, sc, mode);
        v.ep[(sc->it + 1) & 1][el] = f0[el];
    }
    // the operand: p or s
    T f[K];
    if (mode == 0) {
        if (sc->it == 0) {
#pragma unroll
            for (int i = 0; i < K; ++i) f[i] = rr[i];
        } else {
            const double beta = (sc->rho / sc->rho_old) * (sc->alpha / sc->omega);
            const T om = T(sc->omega);
#pragma unroll
            for (int i = 0; i < K; ++i) f[i] = rr[i] + T(beta) * (pp[i] - om * vv[i]);
        }
    } else {
        const T al = T(sc->alpha);
#pragma unroll
        for (int i = 0; i < K; ++i) f[i] = rr[i] - al * vv[i];
    }
    if (done) return;  // uniform over the grid: no copy was issued
    if (act) {
        store_row<K, T>((mode == 0 ? v.p : v.s) + p, f);
#pragma unroll
        for (int i = 0; i < K; ++i) sr[ix.warp][lw][t * K + i] = f[i];
    }
    __syncwarp();
    sd.wait(&bar[ix.warp], sc, ix.lane);
    T acc[K];
    smoother_rows<K, T, BS>(op, sd.blk, sd.fk, sd.kx, sr[ix.warp][lw], zb[ix.warp][lw], t, act, acc);
    if (act) store_row<K, T>(v.zf + p, acc);
    if (mode == 1) {
        double part[1] = {0.0};
        if (act) {
#pragma unroll
            for (int i = 0; i < K; ++i) part[0] += double(f[i]) * double(f[i]);
        }
        double out[1];
        if (grid_reduce<1>(part, rs.partials, rs.counter, out) && threadIdx.x == 0) {
            sc->snorm2 = out[0];
            sc->s_exit = out[0] <= sc->eps2;
        }
    }
}

// Coarse part of the preconditioner application and the result: the two-level smoothing
// step z = e + w M (f - A e), e = P u0 element-wise constant, as
//   z = u0_self + w (zf - sum_s W_s u0_s),   W_s = M rowsum_s  (k_make_w, at setup),
// where A e = sum over the element's 5 block slots s (itself, its face neighbours) of the
// block row sums times u0 of the slot's element; then z's face traces. Without a coarse
// level (block-Jacobi) z = w zf.
template <int K, typename T>
__global__ void __launch_bounds__(Rows<K>::THREADS) k_post_b(MfOp<T> op, BicgVectors<T> v, CoarseOut<T> co,
                                                              int has_coarse, double w, const KrylovScalars* sc,
                                                              int mode) {
    using R = Rows<K>;
    constexpr int K2 = R::K2;
    if (sc->done) return;  // uniform
    __shared__ T zb[R::WARPS][R::EPW][K][K];
    const RowIdx<K> ix(op.g.N, blockIdx.x);
    const int t = ix.t, el = ix.el;
    const bool act = ix.active;
    const size_t p = (size_t)el * K2 + t * K;
    T zz[K];
    int dst[4];
    if (act) {
        T zf[K];
        load_row<K, T>(v.zf + p, zf);
        load4i(op.g.scat + ((size_t)el * K + t) * 4, dst);
        T ue[5], ws[5][K];
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            ue[q] = has_coarse ? co.ue5[(size_t)el * 5 + q] : T(0);
            if (has_coarse) load_row<K, T>(op.W + ((size_t)el * 5 + q) * K2 + t * K, ws[q]);
        }
#pragma unroll
        for (int i = 0; i < K; ++i) {
            T ae = T(0);
            if (has_coarse) {
#pragma unroll
                for (int q = 0; q < 5; ++q) ae += ws[q][i] * ue[q];
            }
            zz[i] = ue[0] + T(w) * (zf[i] - ae);
        }
        store_row<K, T>((mode == 0 ? v.ph : v.sh) + p, zz);
    }
    row_emit_traces<K, T>(op.b, zb[ix.warp][ix.lw], zz, dst, v.tv, v.tg, t, act);
}

// Setup: W_s = M rowsum_s for the 5 block slots of every element, with the smoother's own
// element inverse M (so the split application k_post_a + k_post_b is exactly the smoothing
// step of the stored smoother).
template <int K, typename T, int BS>
__global__ void __launch_bounds__(Rows<K>::THREADS) k_make_w(MfOp<T> op, T* __restrict__ W, KrylovScalars* sc) {
    using R = Rows<K>;
    constexpr int K2 = R::K2, EPW = R::EPW;
    extern __shared__ __align__(128) unsigned char post_dyn[];
    __shared__ __align__(8) uint64_t bar[R::WARPS];
    __shared__ __align__(16) T sr[R::WARPS][EPW][K2];
    __shared__ T zb[R::WARPS][EPW][K][K];
    const RowIdx<K> ix(op.g.N, blockIdx.x);
    const int t = ix.t, lw = ix.lw, el = ix.el;
    const bool act = ix.active;
    SmootherData<K, T, BS> sd;
    sd.start(op, ix, post_dyn, &bar[ix.warp], true);
    sd.wait(&bar[ix.warp], sc, ix.lane);
    for (int q = 0; q < 5; ++q) {
        const size_t rq = ((size_t)el * 5 + q) * K2 + t * K;
        if (act) {
            T r[K];
            load_row<K, T>(op.rowsum + rq, r);
#pragma unroll
            for (int i = 0; i < K; ++i) sr[ix.warp][lw][t * K + i] = r[i];
        }
        __syncwarp();
        T acc[K];
        smoother_rows<K, T, BS>(op, sd.blk, sd.fk, sd.kx, sr[ix.warp][lw], zb[ix.warp][lw], t, act, acc);
        if (act) store_row<K, T>(W + rq, acc);
        __syncwarp();  // sr is rewritten for the next slot
    }
}

// The FP32 operator's tile loop with its inputs staged in shared memory (apply_stage.cuh):
// the copies of a warp's next tile are issued as soon as the lanes have read the current
// one, so they run under the current tile's arithmetic. body(ix, y, sec_row) finishes
// each tile. A copy whose wait runs out is recorded for the host (dev_error) and gets a
// second bounded wait; after that the warp issues no more copies and runs on, so the
// grid reduction stays consistent.
template <int K, typename Body>
__device__ __forceinline__ void staged_apply_loop(const MfOp<float>& op, const float* x, const float* tvin,
                                                  const float* tgin, const float* sec, RowScratch<K, float>* sm,
                                                  KrylovScalars* sc, Body body) {
    using S = ApplyStage<K>;
    using R = Rows<K>;
    extern __shared__ __align__(128) unsigned char apply_dyn[];
    __shared__ __align__(8) uint64_t bar[R::WARPS];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int N = op.g.N, ntiles = (int)rgrid_of<K>(N);
    float* st = reinterpret_cast<float*>(apply_dyn + (size_t)warp * S::WARP_BYTES);
    auto count = [&](int tile) {
        return tile < ntiles ? max(0, min(R::EPW, N - stage_first<K>(tile, warp))) : 0;
    };
    if (lane == 0) mbar_init(&bar[warp]);
    __syncwarp();
    if (lane == 0 && count(blockIdx.x) > 0)
        stage_issue<K>(st, &bar[warp], op.g, x, tvin, tgin, sec, stage_first<K>(blockIdx.x, warp), count(blockIdx.x));
    unsigned phase = 0;
    bool ok = true;
#pragma unroll 1
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const RowIdx<K> ix(N, tile);
        if (ok && count(tile) > 0) {
            if (!mbar_wait_bounded(&bar[warp], phase & 1u, kBulkWaitPolls)) {
                if (lane == 0) atomicExch(&sc->dev_error, 1);
                ok = mbar_wait_bounded(&bar[warp], phase & 1u, kBulkWaitPolls);
            }
            ++phase;
        }
        ApplyIn<K, float> in;
        float sr[K];
        stage_read<K>(st, op.g, x, sec, stage_first<K>(tile, warp), ix, in, sr);
        __syncwarp();  // every lane has read the slice
        const int next = tile + (int)gridDim.x;
        if (lane == 0 && ok && count(next) > 0) {
            stage_release();
            stage_issue<K>(st, &bar[warp], op.g, x, tvin, tgin, sec, stage_first<K>(next, warp), count(next));
        }
        float y[K];
        row_apply_core<K, float>(op, in, sm[warp], ix, y);
        body(ix, y, sr);
    }
}

// v = A ph; alpha = rho / (rhat, v); element sums of v. ST: the FP32 loop with staged
// inputs (dynamic shared memory ApplyStage<K>::CTA_BYTES).
// (FP32: at most 128 registers, four CTAs per SM)
template <int K, typename T, bool ST = false>
__global__ void __launch_bounds__(Rows<K>::THREADS, sizeof(T) == 4 ? 4 : 1)
    k_mf_v(MfOp<T> op, BicgVectors<T> v, ReduceScratch rs) {
    KrylovScalars* sc = rs.sc;
    // the flag is uniform over the grid (only this kernel's last CTA writes it, after every
    // CTA has read it)
    if (sc->done) return;
    __shared__ RowScratch<K, T> sm[Rows<K>::WARPS];
    const int ntiles = (int)rgrid_of<K>(op.g.N);
    double part[1] = {0.0};
    auto finish = [&](const RowIdx<K>& ix, const T (&y)[K], const T (&rh)[K]) {
        T ysum = T(0);
        if (ix.active) {
            const size_t p = (size_t)ix.el * K * K + ix.t * K;
            store_row<K, T>(v.v + p, y);
#pragma unroll
            for (int i = 0; i < K; ++i) {
                ysum += y[i];
                part[0] += double(rh[i]) * double(y[i]);
            }
        }
        const T tot = element_total<K, T>(ysum, ix.lw);
        if (ix.active && ix.t == 0) v.ev[ix.el] = tot;
    };
    auto tile_body = [&](int tile) {
        const RowIdx<K> ix(op.g.N, tile);
        T y[K];
        row_apply<K, T>(op, v.ph, v.tv, v.tg, sm[ix.warp], ix, y);
        T rh[K];
        if (ix.active) load_row<K, T>(v.rhat + (size_t)ix.el * K * K + ix.t * K, rh);
        finish(ix, y, rh);
    };
    if constexpr (ST && sizeof(T) == 4) {
        staged_apply_loop<K>(op, v.ph, v.tv, v.tg, v.rhat, sm, sc, finish);
    } else if constexpr (sizeof(T) == 4) {
        // FP32: one wave of CTAs over the tiles; FP64 keeps one tile per CTA (the loop
        // would push the operator past the register file)
#pragma unroll 1
        for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
            if (tile + (int)gridDim.x < ntiles)
                prefetch_apply_rows<K, T>(op.g, v.ph, v.tv, v.tg, v.rhat, tile + gridDim.x);
            tile_body(tile);
        }
    } else {
        if ((int)blockIdx.x < ntiles) tile_body(blockIdx.x);
    }
    double out[1];
    if (grid_reduce<1>(part, rs.partials, rs.counter, out) && threadIdx.x == 0) {
        if (out[0] == 0.0 || sc->rho == 0.0) {
            sc->breakdown = 1;
            sc->done = 1;
        } else {
            sc->alpha = sc->rho / out[0];
        }
    }
}

// t = A sh; omega = (t, s) / (t, t). ST as in k_mf_v.
// (FP32: at most 128 registers, four CTAs per SM)
template <int K, typename T, bool ST = false>
__global__ void __launch_bounds__(Rows<K>::THREADS, sizeof(T) == 4 ? 4 : 1)
    k_mf_t(MfOp<T> op, BicgVectors<T> v, ReduceScratch rs) {
    KrylovScalars* sc = rs.sc;
    if (sc->done || sc->s_exit) return;  // uniform
    __shared__ RowScratch<K, T> sm[Rows<K>::WARPS];
    const int ntiles = (int)rgrid_of<K>(op.g.N);
    double part[2] = {0.0, 0.0};
    auto finish = [&](const RowIdx<K>& ix, const T (&y)[K], const T (&sv)[K]) {
        if (ix.active) {
            const size_t p = (size_t)ix.el * K * K + ix.t * K;
            store_row<K, T>(v.t + p, y);
#pragma unroll
            for (int i = 0; i < K; ++i) {
                part[0] += double(y[i]) * double(sv[i]);
                part[1] += double(y[i]) * double(y[i]);
            }
        }
    };
    auto tile_body = [&](int tile) {
        const RowIdx<K> ix(op.g.N, tile);
        T y[K];
        row_apply<K, T>(op, v.sh, v.tv, v.tg, sm[ix.warp], ix, y);
        T sv[K];
        if (ix.active) load_row<K, T>(v.s + (size_t)ix.el * K * K + ix.t * K, sv);
        finish(ix, y, sv);
    };
    if constexpr (ST && sizeof(T) == 4) {
        staged_apply_loop<K>(op, v.sh, v.tv, v.tg, v.s, sm, sc, finish);
    } else if constexpr (sizeof(T) == 4) {
        // FP32: one wave of CTAs over the tiles; FP64 keeps one tile per CTA (the loop
        // would push the operator past the register file)
#pragma unroll 1
        for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
            if (tile + (int)gridDim.x < ntiles)
                prefetch_apply_rows<K, T>(op.g, v.sh, v.tv, v.tg, v.s, tile + gridDim.x);
            tile_body(tile);
        }
    } else {
        if ((int)blockIdx.x < ntiles) tile_body(blockIdx.x);
    }
    double out[2];
    if (grid_reduce<2>(part, rs.partials, rs.counter, out) && threadIdx.x == 0)
        sc->omega = out[1] > 0.0 ? out[0] / out[1] : 0.0;
}

// x += alpha ph + omega sh; r = s - omega t; ||r||^2, (rhat, r); element sums of r;
// convergence test. After an s-exit (||s|| already below tolerance) only x += alpha ph.
// The last CTA to finish ends the iteration: it updates the scalars, sets `done`, and
// inside a captured solve sets the condition of the graph's while node (iterate while
// not done). Every CTA reads `done` and `s_exit` before any CTA arrives at the counter,
// so the last CTA may change them. Every body execution either increments `it` (capped at
// max_iter) or finds `done` set and clears the condition, so the device loop always ends.
// Each thread updates element rows.
template <int K, typename T>
__global__ void __launch_bounds__(Rows<K>::THREADS) k_xr_update(int N, BicgVectors<T> v, ReduceScratch rs,
                                                                 int max_iter, cudaGraphConditionalHandle h,
                                                                 int has_handle) {
    KrylovScalars* sc = rs.sc;
    if (sc->done) {  // the solve ended earlier in this body (breakdown)
        if (has_handle && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(h, 0u);
        return;
    }
    const T alpha = T(sc->alpha);
    const bool s_exit = sc->s_exit;
    const double omega = sc->omega;
    const int ntiles = (int)rgrid_of<K>(N);
    double part[2] = {0.0, 0.0};
#pragma unroll 1
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const RowIdx<K> ix(N, tile);
        const size_t p = (size_t)ix.el * K * K + ix.t * K;
        T rsum = T(0);
        if (ix.active) {
            T x[K], ph[K];
            load_row<K, T>(v.x + p, x);
            load_row<K, T>(v.ph + p, ph);
            if (s_exit) {
#pragma unroll
                for (int i = 0; i < K; ++i) x[i] = x[i] + alpha * ph[i];
                store_row<K, T>(v.x + p, x);
            } else {
                T sh[K], sv[K], tv[K], rh[K], r[K];
                load_row<K, T>(v.sh + p, sh);
                load_row<K, T>(v.s + p, sv);
                load_row<K, T>(v.t + p, tv);
                load_row<K, T>(v.rhat + p, rh);
#pragma unroll
                for (int i = 0; i < K; ++i) {
                    x[i] = x[i] + (alpha * ph[i] + T(omega) * sh[i]);
                    r[i] = sv[i] - T(omega) * tv[i];
                    rsum += r[i];
                    part[0] += double(r[i]) * double(r[i]);
                    part[1] += double(rh[i]) * double(r[i]);
                }
                store_row<K, T>(v.x + p, x);
                store_row<K, T>(v.r + p, r);
            }
        }
        if (!s_exit) {
            const T tot = element_total<K, T>(rsum, ix.lw);
            if (ix.active && ix.t == 0) v.er[ix.el] = tot;
        }
    }
    double out[2];
    if (grid_reduce<2>(part, rs.partials, rs.counter, out) && threadIdx.x == 0) {
        sc->it += 1;
        if (s_exit) {
            sc->rnorm2 = sc->snorm2;
            sc->done = 1;
        } else {
            sc->rnorm2 = out[0];
            sc->rho_old = sc->rho;
            sc->rho = out[1];
            if (out[0] <= sc->eps2 || sc->it >= max_iter || omega == 0.0) sc->done = 1;
        }
        if (has_handle) cudaGraphSetConditional(h, sc->done ? 0u : 1u);
    }
}

__global__ void k_set_loop(const KrylovScalars* sc, cudaGraphConditionalHandle h) {
    cudaGraphSetConditional(h, sc->done ? 0u : 1u);
}

// r = b - A x (FP64 refinement residual); ||r||^2 -> rnorm2, ||b||^2 -> bnorm2
template <int K, typename T>
__global__ void __launch_bounds__(Rows<K>::THREADS) k_mf_residual(MfOp<T> op, const double* __restrict__ b,
                                                                   const T* __restrict__ x, const T* __restrict__ xtv,
                                                                   const T* __restrict__ xtg, double* __restrict__ r,
                                                                   ReduceScratch rs) {
    __shared__ RowScratch<K, T> sm[Rows<K>::WARPS];
    const int ntiles = (int)rgrid_of<K>(op.g.N);
    double part[2] = {0.0, 0.0};
    auto tile_body = [&](int tile) {
        const RowIdx<K> ix(op.g.N, tile);
        T y[K];
        row_apply<K, T>(op, x, xtv, xtg, sm[ix.warp], ix, y);
        if (ix.active) {
            const size_t p = (size_t)ix.el * K * K + ix.t * K;
            double bb[K], rr[K];
            load_row<K, double>(b + p, bb);
#pragma unroll
            for (int i = 0; i < K; ++i) {
                rr[i] = bb[i] - double(y[i]);
                part[0] += rr[i] * rr[i];
                part[1] += bb[i] * bb[i];
            }
            store_row<K, double>(r + p, rr);
        }
    };
    // FP32: one wave of CTAs over the tiles; FP64 keeps one tile per CTA (the loop would
    // push the operator past the register file)
    if constexpr (sizeof(T) == 4) {
#pragma unroll 1
        for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) tile_body(tile);
    } else {
        if ((int)blockIdx.x < ntiles) tile_body(blockIdx.x);
    }
    double out[2];
    if (grid_reduce<2>(part, rs.partials, rs.counter, out) && threadIdx.x == 0) {
        rs.sc->rnorm2 = out[0];
        rs.sc->bnorm2 = out[1];
    }
}

// y = A x (operator only)
template <int K, typename T>
__global__ void __launch_bounds__(Rows<K>::THREADS) k_mf_apply(MfOp<T> op, const T* __restrict__ x,
                                                                const T* __restrict__ xtv, const T* __restrict__ xtg,
                                                                T* __restrict__ y) {
    __shared__ RowScratch<K, T> sm[Rows<K>::WARPS];
    const RowIdx<K> ix(op.g.N, blockIdx.x);
    T yy[K];
    row_apply<K, T>(op, x, xtv, xtg, sm[ix.warp], ix, yy);
    if (ix.active) store_row<K, T>(y + (size_t)ix.el * K * K + ix.t * K, yy);
}

// ---------------------------------------------------------------- FP64 refinement on the device
// The mixed-precision solve as one graph: FP64 residual, then while the refinement
// continues { FP32 right-hand side, inner BiCGSTAB (its own while node), psi += x,
// FP64 residual }. k_refine_ctl decides after every FP64 residual, with the rule the
// host loop uses: stop on a non-finite or zero residual norm, at the target, at the sweep
// cap, or when the last sweep did not halve the residual (stalled: the host finishes the
// solve in FP64); otherwise ask the inner solve for max(inner_tol, 0.3 target / current)
// relative reduction (at most 0.5), so the last sweep does not overshoot.
__global__ void k_refine_begin(KrylovScalars* sc) {
    sc->sweeps = 0;
    sc->iters_total = 0;
    sc->zero_psi = 0;
    sc->finite = 1;
    sc->stalled = 0;
}

__global__ void k_refine_ctl(KrylovScalars* sc, cudaGraphConditionalHandle h) {
    const double bn = sc->bnorm2, rn = sc->rnorm2;
    const bool fin = isfinite(bn) && isfinite(rn);
    double res = bn > 0.0 ? sqrt(rn / bn) : 0.0;
    bool stop = !fin;
    if (fin && bn == 0.0) {
        sc->zero_psi = 1;
        res = 0.0;
        stop = true;
    }
    if (!stop && (rn <= sc->tol_outer * sc->tol_outer * bn || sc->sweeps >= sc->max_sweeps)) stop = true;
    // a sweep that did not halve the residual: iterative refinement with an FP32 inner solve
    // needs cond(A) * eps_32 < 1, which this operator no longer meets
    if (!stop && sc->sweeps > 0 && !(res <= 0.5 * sc->res)) {
        stop = true;
        sc->stalled = 1;
    }
    sc->res = res;
    sc->finite = fin;
    if (!stop) {
        const double need = 0.3 * sc->tol_outer / res;
        sc->tol = fmin(0.5, fmax(sc->inner_tol, need));
        sc->sweeps += 1;
    }
    cudaGraphSetConditional(h, stop ? 0u : 1u);
}

// right-hand side of the inner solve (the FP64 residual rounded to FP32) and its zero
// initial guess
__global__ void k_refine_prep(const double* __restrict__ r, float* __restrict__ b, float* __restrict__ x, size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        b[i] = (float)r[i];
        x[i] = 0.f;
    }
}

// psi += x; the inner iterations are added to the solve's total
__global__ void k_refine_axpy(const float* __restrict__ e, double* __restrict__ x, size_t n, KrylovScalars* sc) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] += (double)e[i];
    if (i == 0) sc->iters_total += sc->it;
}

// a zero right-hand side gives psi = 0
__global__ void k_refine_finish(double* __restrict__ x, size_t n, const KrylovScalars* sc) {
    if (!sc->zero_psi) return;
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] = 0.0;
}

__global__ void k_d2f(const double* a, float* b, size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = (float)a[i];
}
__global__ void k_axpy_f2d(const float* e, double* x, size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] += (double)e[i];
}

// ---------------------------------------------------------------- launchers
#define HO2D_KSWITCH(K, CALL)                              \
    switch (K) {                                           \
        case 1: { constexpr int KK = 1; CALL; } break;      \
        case 2: { constexpr int KK = 2; CALL; } break;      \
        case 3: { constexpr int KK = 3; CALL; } break;      \
        case 4: { constexpr int KK = 4; CALL; } break;      \
        case 5: { constexpr int KK = 5; CALL; } break;      \
        case 6: { constexpr int KK = 6; CALL; } break;      \
        case 7: { constexpr int KK = 7; CALL; } break;      \
        case 8: { constexpr int KK = 8; CALL; } break;      \
        default: return cudaErrorInvalidValue;             \
    }


int krylov_max_blocks(int K, int N) {
    const int k2 = K * K;
    const int epb = (256 / k2) > 32 ? 32 : ((256 / k2) > 0 ? 256 / k2 : 1);
    return (N + epb - 1) / epb;
}

template <typename T>
cudaError_t krylov_init(const MfOp<T>& op, const BicgVectors<T>& v, const ReduceScratch& rs,
                        cudaStream_t s) {
    const int N = op.g.N;
    HO2D_KSWITCH(op.K, (k_trace_in<KK, T><<<rgrid_of<KK>(N), Rows<KK>::THREADS, 0, s>>>(op, v.x, v.xtv, v.xtg)));
    HO2D_KSWITCH(op.K, (k_mf_init<KK, T><<<wave_of<KK, T>(&WaveSizes::init, N), Rows<KK>::THREADS, 0, s>>>(op, v, rs)));
    const size_t n = (size_t)N * op.K * op.K;
    k_zero_if<T><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(v.x, n, rs.sc);
    return cudaGetLastError();
}

// One BiCGSTAB iteration: [coarse cycle on P^T p] -> p update + smoothing (ph) -> v = A ph
// -> [coarse cycle on P^T s] -> s update + smoothing (sh) -> t = A sh -> x, r update and
// loop control.
// A preconditioner application is its coarse cycle (on the side stream when op.side is
// set) beside the fine smoothing part k_post_a, then the combination k_post_b. With ev
// (10 events) everything runs in order on s with the boundaries recorded: ev[0] coarse
// ev[1] fine part ev[2] combination ev[3] operator ev[4] coarse ev[5] fine part ev[6]
// combination ev[7] operator ev[8] update ev[9].
template <int K, typename T>
static void iteration_impl(const MfOp<T>& op, const BicgVectors<T>& v, const ReduceScratch& rs, int max_iter,
                           const Precond<T>& pc, cudaGraphConditionalHandle h, int has_handle, cudaStream_t s,
                           cudaEvent_t* ev = nullptr) {
    auto mark = [&](int i) {
        if (ev) cudaEventRecord(ev[i], s);
    };
    const int N = op.g.N;
    const int mg = pc.nlev > 0;
    const CoarseOut<T> co = mg ? coarse_out(pc) : CoarseOut<T>();
    const unsigned gp = rgrid_of<K>(N);
    constexpr int tp = Rows<K>::THREADS;
    auto post_a = [&](int mode) {
        if constexpr (std::is_same<T, float>::value) {
            if (op.kron_f) {
                k_post_a<K, T, 2><<<gp, tp, PostRows<K, T, 2>::SMEM, s>>>(op, v, mg, rs, mode);
                return;
            }
            if (op.dinv_bf16) {
                k_post_a<K, T, 1><<<gp, tp, PostRows<K, T, 1>::SMEM, s>>>(op, v, mg, rs, mode);
                return;
            }
        }
        k_post_a<K, T, 0><<<gp, tp, PostRows<K, T, 0>::SMEM, s>>>(op, v, mg, rs, mode);
    };
    // one preconditioner application: the coarse cycle beside the fine part (on the side
    // stream, joined before the combination), or after it without a side stream
    auto precond = [&](int mode, int m0) {
        const bool fork = mg && op.side && !ev;  // a profiled iteration runs everything in order
        mark(m0);
        if (fork) {
            cudaEventRecord(op.ev_fork, s);
            cudaStreamWaitEvent(op.side, op.ev_fork, 0);
            coarse_cycle<T>(pc, v, rs.sc, mode, op.side);
            cudaEventRecord(op.ev_join, op.side);
        } else if (mg) {
            coarse_cycle<T>(pc, v, rs.sc, mode, s);
        }
        mark(m0 + 1);
        post_a(mode);
        if (fork) cudaStreamWaitEvent(s, op.ev_join, 0);
        mark(m0 + 2);
        k_post_b<K, T><<<gp, tp, 0, s>>>(op, v, co, mg, pc.omega, rs.sc, mode);
    };
    const unsigned gwv = wave_of<K, T>(&WaveSizes::v, N), gwt = wave_of<K, T>(&WaveSizes::t, N),
                   gwx = wave_of<K, T>(&WaveSizes::xr, N);
    // the FP32 operator with its inputs staged by bulk copies, or read through L2 prefetches
    auto apply_v = [&]() {
        if constexpr (std::is_same<T, float>::value) {
            if (op.staged) {
                k_mf_v<K, T, true><<<wave_of<K, T>(&WaveSizes::v_st, N), Rows<K>::THREADS, ApplyStage<K>::CTA_BYTES,
                                     s>>>(op, v, rs);
                return;
            }
        }
        k_mf_v<K, T><<<gwv, Rows<K>::THREADS, 0, s>>>(op, v, rs);
    };
    auto apply_t = [&]() {
        if constexpr (std::is_same<T, float>::value) {
            if (op.staged) {
                k_mf_t<K, T, true><<<wave_of<K, T>(&WaveSizes::t_st, N), Rows<K>::THREADS, ApplyStage<K>::CTA_BYTES,
                                     s>>>(op, v, rs);
                return;
            }
        }
        k_mf_t<K, T><<<gwt, Rows<K>::THREADS, 0, s>>>(op, v, rs);
    };
    precond(0, 0);
    mark(3);
    apply_v();
    precond(1, 4);
    mark(7);
    apply_t();
    mark(8);
    k_xr_update<K, T><<<gwx, Rows<K>::THREADS, 0, s>>>(N, v, rs, max_iter, h, has_handle);
    mark(9);
}

template <int K, typename T>
static cudaError_t configure_waves() {
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    WaveSizes& ws = g_wave[K][std::is_same<T, float>::value ? 1 : 0];
    auto w = [&](auto kern, unsigned& out, int dyn = 0) {
        int nb = 0;
        if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, Rows<K>::THREADS, dyn);
        out = (unsigned)(nb > 0 ? nb : 1) * (unsigned)sms;
    };
    w(k_xr_update<K, T>, ws.xr);
    if constexpr (sizeof(T) == 4) {  // the FP64 operator kernels take one tile per CTA
        w(k_mf_init<K, T>, ws.init);
        w(k_mf_v<K, T>, ws.v);
        w(k_mf_t<K, T>, ws.t);
        w(k_mf_v<K, T, true>, ws.v_st, ApplyStage<K>::CTA_BYTES);
        w(k_mf_t<K, T, true>, ws.t_st, ApplyStage<K>::CTA_BYTES);
        w(k_mf_residual<K, T>, ws.res);
    }
    return e;
}

// Dynamic shared memory of the smoothing kernels that stage their blocks (above the
// 48 KB a launch gets without asking); once per device before the first launch or capture.
template <int K>
static cudaError_t configure_post() {
    cudaError_t e = cudaSuccess;
    auto one = [&](auto kern, int bytes) {
        if (e == cudaSuccess && bytes > 0)
            e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    };
    one(k_post_a<K, double, 0>, PostRows<K, double, 0>::SMEM);
    one(k_post_a<K, float, 0>, PostRows<K, float, 0>::SMEM);
    one(k_post_a<K, float, 1>, PostRows<K, float, 1>::SMEM);
    one(k_post_a<K, float, 2>, PostRows<K, float, 2>::SMEM);
    one(k_make_w<K, double, 0>, PostRows<K, double, 0>::SMEM);
    one(k_make_w<K, float, 0>, PostRows<K, float, 0>::SMEM);
    one(k_make_w<K, float, 1>, PostRows<K, float, 1>::SMEM);
    one(k_make_w<K, float, 2>, PostRows<K, float, 2>::SMEM);
    return e;
}

cudaError_t krylov_configure(int K) {
    cudaError_t e = cudaSuccess;
    HO2D_KSWITCH(K, (e = configure_post<KK>()));
    if (e == cudaSuccess) HO2D_KSWITCH(K, (e = configure_waves<KK, double>()));
    if (e == cudaSuccess) HO2D_KSWITCH(K, (e = configure_waves<KK, float>()));
    return e;
}

template <typename T>
int krylov_launches_per_iteration(const Precond<T>& pc) {
    return 7 + 2 * coarse_launches(pc);
}

template <int K, typename T>
static cudaError_t make_w_impl(const MfOp<T>& op, T* W, KrylovScalars* sc, cudaStream_t s) {
    const unsigned g = rgrid_of<K>(op.g.N);
    constexpr int tp = Rows<K>::THREADS;
    if constexpr (std::is_same<T, float>::value) {
        if (op.kron_f) {
            k_make_w<K, T, 2><<<g, tp, PostRows<K, T, 2>::SMEM, s>>>(op, W, sc);
            return cudaGetLastError();
        }
        if (op.dinv_bf16) {
            k_make_w<K, T, 1><<<g, tp, PostRows<K, T, 1>::SMEM, s>>>(op, W, sc);
            return cudaGetLastError();
        }
    }
    k_make_w<K, T, 0><<<g, tp, PostRows<K, T, 0>::SMEM, s>>>(op, W, sc);
    return cudaGetLastError();
}

template <typename T>
cudaError_t krylov_make_w(const MfOp<T>& op, T* W, KrylovScalars* sc, cudaStream_t s) {
    cudaError_t e = cudaSuccess;
    HO2D_KSWITCH(op.K, (e = make_w_impl<KK, T>(op, W, sc, s)));
    return e;
}

template <typename T>
cudaError_t krylov_iteration(const MfOp<T>& op, const BicgVectors<T>& v, const ReduceScratch& rs, int max_iter,
                             const Precond<T>& pc, cudaStream_t s) {
    HO2D_KSWITCH(op.K, (iteration_impl<KK, T>(op, v, rs, max_iter, pc, cudaGraphConditionalHandle(), 0, s)));
    return cudaGetLastError();
}

template <typename T>
cudaError_t krylov_iteration_timed(const MfOp<T>& op, const BicgVectors<T>& v, const ReduceScratch& rs, int max_iter,
                                   const Precond<T>& pc, cudaEvent_t* ev, cudaStream_t s) {
    HO2D_KSWITCH(op.K, (iteration_impl<KK, T>(op, v, rs, max_iter, pc, cudaGraphConditionalHandle(), 0, s, ev)));
    return cudaGetLastError();
}

// Captures a whole solve into `*graph_out`: initial residual, then a while node whose body
// is one BiCGSTAB iteration; the loop condition lives on the device, so a solve is one
// graph launch with no host round trip.
template <typename T>
cudaError_t krylov_capture_solve(const MfOp<T>& op, const BicgVectors<T>& v, const ReduceScratch& rs,
                                 int max_iter, const Precond<T>& pc, cudaStream_t s, cudaGraph_t* graph_out) {
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaGraphCreate(&g, 0);
    if (e != cudaSuccess) return e;
    cudaGraphConditionalHandle h;
    if ((e = cudaGraphConditionalHandleCreate(&h, g, 0, 0)) != cudaSuccess) return e;
    if ((e = cudaStreamBeginCaptureToGraph(s, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal)) !=
        cudaSuccess)
        return e;
    krylov_init<T>(op, v, rs, s);
    k_set_loop<<<1, 1, 0, s>>>(rs.sc, h);
    cudaStreamCaptureStatus st;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    cudaGraph_t cg = nullptr;
    if ((e = cudaStreamGetCaptureInfo(s, &st, nullptr, &cg, &deps, &ndeps)) != cudaSuccess) return e;
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t cnode;
    if ((e = cudaGraphAddNode(&cnode, cg, deps, ndeps, &cp)) != cudaSuccess) return e;
    if ((e = cudaStreamUpdateCaptureDependencies(s, &cnode, 1, cudaStreamSetCaptureDependencies)) != cudaSuccess)
        return e;
    if ((e = cudaStreamEndCapture(s, &g)) != cudaSuccess) return e;
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    if ((e = cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal)) !=
        cudaSuccess)
        return e;
    HO2D_KSWITCH(op.K, (iteration_impl<KK, T>(op, v, rs, max_iter, pc, h, 1, s)));
    if ((e = cudaStreamEndCapture(s, &body)) != cudaSuccess) return e;
    *graph_out = g;
    return cudaGetLastError();
}

// Captures a whole mixed-precision solve (FP64 refinement around the FP32 BiCGSTAB) into
// `*graph_out`: the refinement loop and each sweep's BiCGSTAB loop are nested while nodes
// whose conditions are set on the device, so a solve is one graph launch and no host
// round trip. psi64 is updated in place; rhs, the FP64 residual r64 and the FP64 traces
// (xtv64, xtg64) are the refinement's vectors; v32 holds the inner solve's (v32.b is the
// inner right-hand side, v32.x its solution).
cudaError_t krylov_capture_refined_solve(const MfOp<double>& A64, const MfOp<float>& A32,
                                         const BicgVectors<float>& v32, const ReduceScratch& rs, int max_iter,
                                         const Precond<float>& pc, double* psi64, const double* rhs, double* r64,
                                         double* xtv64, double* xtg64, cudaStream_t s, cudaGraph_t* graph_out) {
    const size_t n = (size_t)A64.g.N * A64.K * A64.K;
    const unsigned gn = (unsigned)((n + 255) / 256);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaGraphCreate(&g, 0);
    if (e != cudaSuccess) return e;
    cudaGraphConditionalHandle ho, hi;
    if ((e = cudaGraphConditionalHandleCreate(&ho, g, 0, 0)) != cudaSuccess) return e;
    if ((e = cudaGraphConditionalHandleCreate(&hi, g, 0, 0)) != cudaSuccess) return e;
    // adds a while node on handle h after the capture's current dependencies and returns
    // its body graph; the stream's capture continues after the node
    auto add_while = [&](cudaGraphConditionalHandle h, cudaGraph_t* body) -> cudaError_t {
        cudaStreamCaptureStatus st;
        const cudaGraphNode_t* deps = nullptr;
        size_t ndeps = 0;
        cudaGraph_t cg = nullptr;
        cudaError_t err = cudaStreamGetCaptureInfo(s, &st, nullptr, &cg, &deps, &ndeps);
        if (err != cudaSuccess) return err;
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = h;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t node;
        if ((err = cudaGraphAddNode(&node, cg, deps, ndeps, &cp)) != cudaSuccess) return err;
        if ((err = cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies)) != cudaSuccess)
            return err;
        *body = cp.conditional.phGraph_out[0];
        return cudaSuccess;
    };
    // top level: reset, FP64 residual, decision, the refinement loop, zero-rhs fix-up
    if ((e = cudaStreamBeginCaptureToGraph(s, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal)) !=
        cudaSuccess)
        return e;
    k_refine_begin<<<1, 1, 0, s>>>(rs.sc);
    mf_residual<double>(A64, rhs, psi64, xtv64, xtg64, r64, rs, s);
    k_refine_ctl<<<1, 1, 0, s>>>(rs.sc, ho);
    cudaGraph_t outer = nullptr;
    if ((e = add_while(ho, &outer)) != cudaSuccess) return e;
    k_refine_finish<<<gn, 256, 0, s>>>(psi64, n, rs.sc);
    if ((e = cudaStreamEndCapture(s, &g)) != cudaSuccess) return e;
    // one refinement sweep
    if ((e = cudaStreamBeginCaptureToGraph(s, outer, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal)) !=
        cudaSuccess)
        return e;
    k_refine_prep<<<gn, 256, 0, s>>>(r64, const_cast<float*>(v32.b), v32.x, n);
    krylov_init<float>(A32, v32, rs, s);
    k_set_loop<<<1, 1, 0, s>>>(rs.sc, hi);
    cudaGraph_t inner = nullptr;
    if ((e = add_while(hi, &inner)) != cudaSuccess) return e;
    k_refine_axpy<<<gn, 256, 0, s>>>(v32.x, psi64, n, rs.sc);
    mf_residual<double>(A64, rhs, psi64, xtv64, xtg64, r64, rs, s);
    k_refine_ctl<<<1, 1, 0, s>>>(rs.sc, ho);
    if ((e = cudaStreamEndCapture(s, &outer)) != cudaSuccess) return e;
    // one BiCGSTAB iteration
    if ((e = cudaStreamBeginCaptureToGraph(s, inner, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal)) !=
        cudaSuccess)
        return e;
    HO2D_KSWITCH(A32.K, (iteration_impl<KK, float>(A32, v32, rs, max_iter, pc, hi, 1, s)));
    if ((e = cudaStreamEndCapture(s, &inner)) != cudaSuccess) return e;
    *graph_out = g;
    return cudaGetLastError();
}

// kernel launches of one captured refined solve: begin, residual, decision and fix-up, then
// per sweep right-hand side, initial residual (3), loop set-up, update, residual and
// decision, plus the inner iterations
int krylov_refined_launches(int sweeps, int inner_iters, const Precond<float>& pc) {
    return 5 + sweeps * 9 + inner_iters * krylov_launches_per_iteration(pc);
}

template <typename T>
cudaError_t mf_residual(const MfOp<T>& op, const double* b, const T* x, T* xtv, T* xtg, double* r,
                        const ReduceScratch& rs, cudaStream_t s) {
    HO2D_KSWITCH(op.K, (k_trace_in<KK, T><<<rgrid_of<KK>(op.g.N), Rows<KK>::THREADS, 0, s>>>(op, x, xtv, xtg)));
    HO2D_KSWITCH(op.K, (k_mf_residual<KK, T><<<wave_of<KK, T>(&WaveSizes::res, op.g.N), Rows<KK>::THREADS, 0, s>>>(op, b, x, xtv, xtg, r,
                                                                                                  rs)));
    return cudaGetLastError();
}

template <typename T>
cudaError_t mf_apply_op(const MfOp<T>& op, const T* x, T* xtv, T* xtg, T* y, cudaStream_t s) {
    HO2D_KSWITCH(op.K, (k_trace_in<KK, T><<<rgrid_of<KK>(op.g.N), Rows<KK>::THREADS, 0, s>>>(op, x, xtv, xtg)));
    HO2D_KSWITCH(op.K, (k_mf_apply<KK, T><<<rgrid_of<KK>(op.g.N), Rows<KK>::THREADS, 0, s>>>(op, x, xtv, xtg, y)));
    return cudaGetLastError();
}

template <typename T>
cudaError_t mf_apply_only(const MfOp<T>& op, const T* x, const T* xtv, const T* xtg, T* y, int reps, cudaStream_t s) {
    for (int r = 0; r < reps; ++r)
        HO2D_KSWITCH(op.K, (k_mf_apply<KK, T><<<rgrid_of<KK>(op.g.N), Rows<KK>::THREADS, 0, s>>>(op, x, xtv, xtg, y)));
    return cudaGetLastError();
}

cudaError_t launch_copy_d2f(const double* a, float* b, size_t n, cudaStream_t s) {
    if (n) k_d2f<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(a, b, n);
    return cudaGetLastError();
}
cudaError_t launch_axpy_f2d(const float* e, double* x, size_t n, cudaStream_t s) {
    if (n) k_axpy_f2d<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(e, x, n);
    return cudaGetLastError();
}

#define HO2D_INSTANTIATE_KRYLOV(T)                                                                                \
    template cudaError_t krylov_init<T>(const MfOp<T>&, const BicgVectors<T>&, const ReduceScratch&,             \
                                        cudaStream_t);                                                            \
    template cudaError_t krylov_iteration<T>(const MfOp<T>&, const BicgVectors<T>&, const ReduceScratch&, int,    \
                                             const Precond<T>&, cudaStream_t);                                    \
    template int krylov_launches_per_iteration<T>(const Precond<T>&);                                             \
    template cudaError_t krylov_make_w<T>(const MfOp<T>&, T*, KrylovScalars*, cudaStream_t);                      \
    template cudaError_t krylov_iteration_timed<T>(const MfOp<T>&, const BicgVectors<T>&, const ReduceScratch&,   \
                                                   int, const Precond<T>&, cudaEvent_t*, cudaStream_t);           \
    template cudaError_t krylov_capture_solve<T>(const MfOp<T>&, const BicgVectors<T>&, const ReduceScratch&,     \
                                                 int, const Precond<T>&, cudaStream_t, cudaGraph_t*);             \
    template cudaError_t mf_residual<T>(const MfOp<T>&, const double*, const T*, T*, T*, double*,                 \
                                        const ReduceScratch&, cudaStream_t);                                      \
    template cudaError_t mf_apply_op<T>(const MfOp<T>&, const T*, T*, T*, T*, cudaStream_t);                      \
    template cudaError_t mf_apply_only<T>(const MfOp<T>&, const T*, const T*, const T*, T*, int, cudaStream_t);

HO2D_INSTANTIATE_KRYLOV(double)
HO2D_INSTANTIATE_KRYLOV(float)

}  // namespace ho2d
