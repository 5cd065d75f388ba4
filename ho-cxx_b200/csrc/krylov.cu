// krylov.cu -- matrix-free FR Poisson operator and preconditioned BiCGSTAB (sm_100a).
//
// Operator. The reference assembles the FR Laplacian into a CSR matrix with up to
// 5 K^4 entries per element (src/HO_2D.cpp:1533-1804, 3011-3062) and hands it to AMGCL.
// That matrix is exactly the method-2 FR Laplacian of calc_RHS_diffusion applied with
// homogeneous Poisson boundary values, so here A x is evaluated matrix-free from face
// traces (lap_element in fr_device.cuh): per DOF it reads x, 5 volume metrics and a
// share of the face data instead of 5 K^2 matrix entries. Every kernel that produces
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
#include "bulk_copy.cuh"

namespace ho2d {

namespace {

template <int NV>
__device__ __forceinline__ bool grid_reduce(const double (&v)[NV], double* partials, unsigned* counter,
                                            double (&out)[NV]) {
    __shared__ double red[NV][32];
    __shared__ double fin[NV];
    __shared__ bool s_last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
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
            if (lane == 0) partials[j * gridDim.x + blockIdx.x] = x;
        }
        __threadfence();
    }
    __syncthreads();
    if (threadIdx.x == 0) s_last = (atomicAdd(counter, 1u) == gridDim.x - 1);
    __syncthreads();
    if (!s_last) return false;
    __threadfence();
#pragma unroll
    for (int j = 0; j < NV; ++j) {
        // the partial loads are independent: unrolled, a thread keeps up to 8 in flight
        double x = 0.0;
#pragma unroll 8
        for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) x += __ldcg(&partials[j * gridDim.x + i]);
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
    if (threadIdx.x == 0) *counter = 0u;
    return true;
}

// Scatter destinations of the face points thread ij emits (prefetched at kernel start).
template <int K>
struct TraceDst {
    static constexpr int K2 = K * K, NF = 4 * K, NO = (NF + K2 - 1) / K2;
    int dst[NO];
    __device__ __forceinline__ void load(const int* scat, bool active, int el, int ij) {
#pragma unroll
        for (int q = 0; q < NO; ++q) {
            const int o = ij + q * K2;
            dst[q] = (active && o < NF) ? scat[el * NF + o] : -1;
        }
    }
};

// face traces of an element vector held in shared memory, written to the neighbours'
// incoming slots
template <int K, typename T>
__device__ __forceinline__ void emit_traces(const T* sy, const DevBases<T>& b, const TraceDst<K>& td, T* tv, T* tg,
                                            int ij) {
    constexpr int K2 = K * K;
#pragma unroll
    for (int q = 0; q < TraceDst<K>::NO; ++q) {
        if (td.dst[q] < 0) continue;
        T v, d;
        face_trace<K, T>(sy, b, ij + q * K2, v, d);
        tv[td.dst[q]] = v;
        tg[td.dst[q]] = d;
    }
}

}  // namespace

// ---------------------------------------------------------------- fine-level kernels
// The operator kernels run row-parallel (rows.cuh): K threads per element, Rows<K>::EPC
// elements per CTA.
template <int K>
static __host__ __device__ constexpr unsigned rgrid_of(int N) {
    return (unsigned)((N + Rows<K>::EPC - 1) / Rows<K>::EPC);
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
#pragma unroll
        for (int f = 0; f < 4; ++f) dst[f] = op.g.scat[(size_t)ix.el * 4 * K + f * K + ix.t];
    }
    row_emit_traces<K, T>(op.b, buf[ix.warp][ix.lw], row, dst, tv, tg, ix.t, ix.active);
}

// r = b - A x (x's traces in xtv/xtg), rhat = r; ||r||^2, ||b||^2; element sums of r
template <int K, typename T>
__global__ void __launch_bounds__(Rows<K>::THREADS) k_mf_init(MfOp<T> op, BicgVectors<T> v, ReduceScratch rs) {
    __shared__ RowScratch<K, T> sm[Rows<K>::WARPS];
    const RowIdx<K> ix(op.g.N, blockIdx.x);
    T y[K];
    row_apply<K, T>(op, v.x, v.xtv, v.xtg, sm[ix.warp], ix, y);
    double part[2] = {0.0, 0.0};
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


// Part `part` (0..4) of u0 at element c = S0_c . f0 + Q0_c . u1 (a row of the level-0
// up step): the row entries part, part + 5, ... The first two of each row are loaded
// before any gather, so a part costs two dependent rounds of loads.
template <typename T>
__device__ __forceinline__ T up0_part(const CoarseOut<T>& co, const F0<T>& f0, int c, int part) {
    const size_t rs = (size_t)c * co.S.w, rq = (size_t)c * co.Q.w;
    T sv[2], qv[2];
    int sj[2], qj[2];
#pragma unroll
    for (int m = 0; m < 2; ++m) {
        const int k = part + 5 * m;
        const bool ins = k < co.S.w, inq = k < co.Q.w;
        sv[m] = ins ? co.S.val[rs + k] : T(0);
        sj[m] = ins ? co.S.col[rs + k] : 0;
        qv[m] = inq ? co.Q.val[rq + k] : T(0);
        qj[m] = inq ? co.Q.col[rq + k] : 0;
    }
    T u = sv[0] * f0[sj[0]] + qv[0] * co.u1[qj[0]] + sv[1] * f0[sj[1]] + qv[1] * co.u1[qj[1]];
    for (int k = part + 10; k < co.S.w; k += 5) u += co.S.val[rs + k] * f0[co.S.col[rs + k]];
    for (int k = part + 10; k < co.Q.w; k += 5) u += co.Q.val[rq + k] * co.u1[co.Q.col[rq + k]];
    return u;
}

// The smoother's element data (BS): 0 = inverse blocks in T; 1 = inverse blocks as BF16 bit
// patterns (FP32 smoother); 2 = Kronecker-sum factors, with the exact blocks only for the
// elements the fit does not approximate well (FP32 smoother). Each element's data starts on
// a 16-byte boundary (padded_count). For BS 0 and 1 a warp's EPW blocks are one contiguous
// span, copied into shared memory by one bulk copy when the span is at most 26 KB (so a
// CTA's four spans leave room for two CTAs per SM); larger blocks are read from global
// memory directly.
template <int K, typename T, int BS>
struct PostRows {
    using DT = typename std::conditional<BS == 1, unsigned short, T>::type;
    static constexpr int K2 = K * K, K4 = K2 * K2;
    static constexpr int STRIDE = padded_count(K4, (int)sizeof(DT));  // values of DT per element
    static constexpr int SPAN = Rows<K>::EPW * STRIDE * (int)sizeof(DT);  // bytes per warp
    static constexpr bool kStage = BS != 2 && SPAN <= 26 * 1024;
    static constexpr int SMEM = kStage ? Rows<K>::WARPS * SPAN : 0;  // dynamic shared memory
    static constexpr int KF = 4 * K2 + 2 * K;                      // Kronecker factors per element
    static constexpr int KFS = padded_count(KF, (int)sizeof(T));
    static constexpr int XSTRIDE = padded_count(K4, (int)sizeof(T));  // compact exact blocks (BS 2)
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

// Preconditioner application, with the BiCGSTAB vector update that produces its operand:
//   mode 0:  p = r + beta (p - omega v)  (p = r on the first iteration),  f = p -> ph
//   mode 1:  s = r - alpha v, ||s||^2 (s_exit test),                      f = s -> sh
// then the two-level smoothing step z = e + w D^{-1} (f - A e), e = P u0 element-wise
// constant, with z's face traces. u0 of the element and of its four face neighbours comes
// straight from the coarse cycle (one-level hierarchy), or from the level-0 up step
// u0 = S0 f0 + Q0 u1 evaluated here as 25 partial sums (five per slot) spread over the
// element's threads, or is zero (block-Jacobi, no coarse level). Mode 0 also stores the
// element sums of the new p for the next iteration. Row-parallel (rows.cuh): thread t of
// an element owns row t. The warp's inverse blocks are requested first, by one bulk copy
// into shared memory (PostRows::kStage), so the copy overlaps the up step's dependent
// loads and the vector loads.
template <int K, typename T, int BS = 0>
__global__ void __launch_bounds__(Rows<K>::THREADS) k_mf_post(MfOp<T> op, BicgVectors<T> v, CoarseOut<T> co,
                                                               int has_coarse, double w, ReduceScratch rs, int mode) {
    using R = Rows<K>;
    using PS = PostRows<K, T, BS>;
    using DT = typename PS::DT;
    constexpr int K2 = R::K2, EPW = R::EPW;
    KrylovScalars* sc = rs.sc;
    const int done = sc->done;  // uniform; read early so the round trip overlaps the loads
    extern __shared__ __align__(128) unsigned char post_dyn[];
    __shared__ __align__(8) uint64_t bar[R::WARPS];
    __shared__ T pu[R::WARPS][EPW][25];
    __shared__ __align__(16) T sr[R::WARPS][EPW][K2];
    __shared__ T zb[R::WARPS][EPW][K][K];
    __shared__ __align__(16) T kf[BS == 2 ? R::WARPS : 1][BS == 2 ? EPW : 1][BS == 2 ? PS::KFS : 1];
    const RowIdx<K> ix(op.g.N, blockIdx.x);
    const int t = ix.t, lw = ix.lw, el = ix.el;
    const bool act = ix.active;
    const DT* dsrc;
    if constexpr (BS == 1) dsrc = op.dinv_bf16;
    else dsrc = op.dinv;
    // this warp's blocks: one bulk copy, issued before anything else
    const int wel0 = (blockIdx.x * R::WARPS + ix.warp) * EPW;
    const int wn = min(EPW, op.g.N - wel0);  // elements of this warp (<= 0: none)
    const DT* blk = dsrc + (size_t)el * PS::STRIDE;
    if constexpr (PS::kStage) {
        DT* stage = reinterpret_cast<DT*>(post_dyn + (size_t)ix.warp * PS::SPAN);
        if (!done && wn > 0 && ix.lane == 0) {
            mbar_init(&bar[ix.warp]);
            const unsigned bytes = (unsigned)(wn * PS::STRIDE * (int)sizeof(DT));
            mbar_arrive_expect(&bar[ix.warp], bytes);
            bulk_load(stage, dsrc + (size_t)wel0 * PS::STRIDE, bytes, &bar[ix.warp]);
        }
        blk = stage + (size_t)lw * PS::STRIDE;
    }
    // this thread's rows of the vectors and block row sums, its face points' destinations
    const size_t p = (size_t)el * K2 + t * K;
    T rr[K], vv[K], pp[K], rsum[5][K];
    int dst[4];
    if (act) {
        load_row<K, T>(v.r + p, rr);
        load_row<K, T>(v.v + p, vv);
        if (mode == 0) load_row<K, T>(v.p + p, pp);
#pragma unroll
        for (int s = 0; s < 5; ++s) load_row<K, T>(op.rowsum + ((size_t)el * 5 + s) * K2 + t * K, rsum[s]);
#pragma unroll
        for (int f = 0; f < 4; ++f) dst[f] = op.g.scat[(size_t)el * 4 * K + f * K + t];
    }
    int kx = -1;  // BS 2: this element's exact block, or -1 for its Kronecker factors
    if constexpr (BS == 2) {
        if (act) {
            kx = op.kron_x[el];
            for (int q = t; q < PS::KF; q += K) kf[ix.warp][lw][q] = op.kron_f[(size_t)el * PS::KFS + q];
        }
    }
    const F0<T> f0 = f0_of(v, sc, mode);
    // u0 of block slot s (element bcol[5 el + s]) as five partial sums pu[s][part]
    if (act)
        for (int q = t; q < 25; q += K) {
            const int slot = q / 5, part = q % 5;
            const int c = op.bcol[el * 5 + slot];
            T u = T(0);
            if (c >= 0 && has_coarse) u = co.u0 ? (part == 0 ? co.u0[c] : T(0)) : up0_part(co, f0, c, part);
            pu[ix.warp][lw][q] = u;
        }
    if (mode == 0 && has_coarse && act && t == 0) v.ep[(sc->it + 1) & 1][el] = f0[el];
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
    if (act) store_row<K, T>((mode == 0 ? v.p : v.s) + p, f);
    __syncwarp();
    // the five slot values, each the sum of its five parts (part 0..4 in order), and the
    // smoother's residual row f - A e
    T ue[5];
#pragma unroll
    for (int q = 0; q < 5; ++q) {
        const T* pq = pu[ix.warp][lw] + 5 * q;
        ue[q] = pq[0] + pq[1] + pq[2] + pq[3] + pq[4];
    }
    if (act) {
#pragma unroll
        for (int i = 0; i < K; ++i) {
            T ae = T(0);
#pragma unroll
            for (int s = 0; s < 5; ++s) ae += rsum[s][i] * ue[s];
            sr[ix.warp][lw][t * K + i] = f[i] - ae;
        }
    }
    __syncwarp();
    if constexpr (PS::kStage) {
        if (wn > 0 && !mbar_wait_bounded(&bar[ix.warp], 0, kBulkWaitPolls)) {
            // record the failure for the host and give the copy a second bounded wait; the
            // kernel then runs to its end so the grid-wide reduction stays consistent
            if (ix.lane == 0) atomicExch(&sc->dev_error, 1);
            mbar_wait_bounded(&bar[ix.warp], 0, kBulkWaitPolls);
        }
    }
    T* z = mode == 0 ? v.ph : v.sh;
    const T* srow = sr[ix.warp][lw];
    T acc[K];
    if constexpr (BS == 2) {
        // exact block where the fit falls back, Kronecker-sum step (fast diagonalisation,
        // the element body of kron_apply.cuh by rows) for the others; the transposes are
        // warp-collective, so every lane runs them
        const bool kr = act && kx < 0;
        if (act && kx >= 0) block_rows<K, T, T>(op.kron_exact + (size_t)kx * PS::XSTRIDE, srow, t, acc);
        const T* fk = kf[ix.warp][lw];
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
        col_to_row<K, T>(zb[ix.warp][lw], c1, r1, t, kr);
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
        rows_to_col<K, T>(zb[ix.warp][lw], r2, c2, t, kr);
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
        col_to_row<K, T>(zb[ix.warp][lw], c3, r3, t, kr);
        if (kr) {
#pragma unroll
            for (int i = 0; i < K; ++i) {
                T s = T(0);
#pragma unroll
                for (int k = 0; k < K; ++k) s += r3[k] * vx[i * K + k];
                acc[i] = s;
            }
        }
        __syncwarp();  // zb is the trace buffer below
    } else {
        if (act) block_rows<K, T, DT>(blk, srow, t, acc);
    }
    T zz[K];
    if (act) {
#pragma unroll
        for (int i = 0; i < K; ++i) zz[i] = ue[0] + T(w) * acc[i];
        store_row<K, T>(z + p, zz);
    }
    row_emit_traces<K, T>(op.b, zb[ix.warp][lw], zz, dst, v.tv, v.tg, t, act);
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

// v = A ph; alpha = rho / (rhat, v); element sums of v
template <int K, typename T>
__global__ void __launch_bounds__(Rows<K>::THREADS) k_mf_v(MfOp<T> op, BicgVectors<T> v, ReduceScratch rs) {
    KrylovScalars* sc = rs.sc;
    // read before the operator's loads so the round trips overlap; the flag is uniform
    // over the grid (only this kernel's last CTA writes it, after every CTA has read it)
    const int done = sc->done;
    __shared__ RowScratch<K, T> sm[Rows<K>::WARPS];
    const RowIdx<K> ix(op.g.N, blockIdx.x);
    T y[K];
    row_apply<K, T>(op, v.ph, v.tv, v.tg, sm[ix.warp], ix, y);
    if (done) return;
    double part[1] = {0.0};
    T ysum = T(0);
    if (ix.active) {
        const size_t p = (size_t)ix.el * K * K + ix.t * K;
        T rh[K];
        load_row<K, T>(v.rhat + p, rh);
        store_row<K, T>(v.v + p, y);
#pragma unroll
        for (int i = 0; i < K; ++i) {
            ysum += y[i];
            part[0] += double(rh[i]) * double(y[i]);
        }
    }
    const T tot = element_total<K, T>(ysum, ix.lw);
    if (ix.active && ix.t == 0) v.ev[ix.el] = tot;
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

// t = A sh; omega = (t, s) / (t, t)
template <int K, typename T>
__global__ void __launch_bounds__(Rows<K>::THREADS) k_mf_t(MfOp<T> op, BicgVectors<T> v, ReduceScratch rs) {
    KrylovScalars* sc = rs.sc;
    const bool skip = sc->done || sc->s_exit;  // read early: the round trip overlaps the operator's loads
    __shared__ RowScratch<K, T> sm[Rows<K>::WARPS];
    const RowIdx<K> ix(op.g.N, blockIdx.x);
    T y[K];
    row_apply<K, T>(op, v.sh, v.tv, v.tg, sm[ix.warp], ix, y);
    if (skip) return;
    double part[2] = {0.0, 0.0};
    if (ix.active) {
        const size_t p = (size_t)ix.el * K * K + ix.t * K;
        T sv[K];
        load_row<K, T>(v.s + p, sv);
        store_row<K, T>(v.t + p, y);
#pragma unroll
        for (int i = 0; i < K; ++i) {
            part[0] += double(y[i]) * double(sv[i]);
            part[1] += double(y[i]) * double(y[i]);
        }
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
// Each thread updates one element row; its loads are issued before the flag is read.
template <int K, typename T>
__global__ void __launch_bounds__(Rows<K>::THREADS) k_xr_update(int N, BicgVectors<T> v, ReduceScratch rs,
                                                                 int max_iter, cudaGraphConditionalHandle h,
                                                                 int has_handle) {
    KrylovScalars* sc = rs.sc;
    const RowIdx<K> ix(N, blockIdx.x);
    const size_t p = (size_t)ix.el * K * K + ix.t * K;
    T x[K], ph[K], sh[K], sv[K], tv[K], rh[K];
    if (ix.active) {
        load_row<K, T>(v.x + p, x);
        load_row<K, T>(v.ph + p, ph);
        load_row<K, T>(v.sh + p, sh);
        load_row<K, T>(v.s + p, sv);
        load_row<K, T>(v.t + p, tv);
        load_row<K, T>(v.rhat + p, rh);
    }
    if (sc->done) {  // the solve ended earlier in this body (breakdown)
        if (has_handle && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(h, 0u);
        return;
    }
    const T alpha = T(sc->alpha);
    const bool s_exit = sc->s_exit;
    const double omega = sc->omega;
    double part[2] = {0.0, 0.0};
    T rsum = T(0);
    if (ix.active) {
        if (s_exit) {
#pragma unroll
            for (int i = 0; i < K; ++i) x[i] = x[i] + alpha * ph[i];
            store_row<K, T>(v.x + p, x);
        } else {
            T r[K];
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
    const RowIdx<K> ix(op.g.N, blockIdx.x);
    T y[K];
    row_apply<K, T>(op, x, xtv, xtg, sm[ix.warp], ix, y);
    double part[2] = {0.0, 0.0};
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
// host loop uses: stop on a non-finite or zero residual norm, at the target or at the
// sweep cap; otherwise ask the inner solve for max(inner_tol, 0.3 target / current)
// relative reduction (at most 0.5), so the last sweep does not overshoot.
__global__ void k_refine_begin(KrylovScalars* sc) {
    sc->sweeps = 0;
    sc->iters_total = 0;
    sc->zero_psi = 0;
    sc->finite = 1;
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
    HO2D_KSWITCH(op.K, (k_mf_init<KK, T><<<rgrid_of<KK>(N), Rows<KK>::THREADS, 0, s>>>(op, v, rs)));
    const size_t n = (size_t)N * op.K * op.K;
    k_zero_if<T><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(v.x, n, rs.sc);
    return cudaGetLastError();
}

// One BiCGSTAB iteration: [coarse cycle on P^T p] -> p update + smoothing (ph) -> v = A ph
// -> [coarse cycle on P^T s] -> s update + smoothing (sh) -> t = A sh -> x, r update and
// loop control.
// With ev (8 events) the boundaries between the launches are recorded on the stream:
// ev[0] coarse ev[1] smoothing ev[2] operator ev[3] coarse ev[4] smoothing ev[5] operator
// ev[6] update ev[7].
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
    auto post = [&](int mode) {
        if constexpr (std::is_same<T, float>::value) {
            if (op.kron_f) {
                k_mf_post<K, T, 2><<<gp, tp, PostRows<K, T, 2>::SMEM, s>>>(op, v, co, mg, pc.omega, rs, mode);
                return;
            }
            if (op.dinv_bf16) {
                k_mf_post<K, T, 1><<<gp, tp, PostRows<K, T, 1>::SMEM, s>>>(op, v, co, mg, pc.omega, rs, mode);
                return;
            }
        }
        k_mf_post<K, T, 0><<<gp, tp, PostRows<K, T, 0>::SMEM, s>>>(op, v, co, mg, pc.omega, rs, mode);
    };
    const unsigned gr = rgrid_of<K>(N);
    mark(0);
    if (mg) coarse_cycle<T>(pc, v, rs.sc, 0, s);
    mark(1);
    post(0);
    mark(2);
    k_mf_v<K, T><<<gr, Rows<K>::THREADS, 0, s>>>(op, v, rs);
    mark(3);
    if (mg) coarse_cycle<T>(pc, v, rs.sc, 1, s);
    mark(4);
    post(1);
    mark(5);
    k_mf_t<K, T><<<gr, Rows<K>::THREADS, 0, s>>>(op, v, rs);
    mark(6);
    k_xr_update<K, T><<<gr, Rows<K>::THREADS, 0, s>>>(N, v, rs, max_iter, h, has_handle);
    mark(7);
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
    one(k_mf_post<K, double, 0>, PostRows<K, double, 0>::SMEM);
    one(k_mf_post<K, float, 0>, PostRows<K, float, 0>::SMEM);
    one(k_mf_post<K, float, 1>, PostRows<K, float, 1>::SMEM);
    one(k_mf_post<K, float, 2>, PostRows<K, float, 2>::SMEM);
    return e;
}

cudaError_t krylov_configure(int K) {
    cudaError_t e = cudaSuccess;
    HO2D_KSWITCH(K, (e = configure_post<KK>()));
    return e;
}

template <typename T>
int krylov_launches_per_iteration(const Precond<T>& pc) {
    return 5 + 2 * coarse_launches(pc);
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
    HO2D_KSWITCH(op.K, (k_mf_residual<KK, T><<<rgrid_of<KK>(op.g.N), Rows<KK>::THREADS, 0, s>>>(op, b, x, xtv, xtg, r,
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
