// krylov.cu -- block-sparse Poisson operator and BiCGSTAB on the device (sm_100a).
//
// The assembled FR Laplacian has, per element row, the element's own K^2 x K^2 block and
// up to four neighbour blocks (src/HO_2D.cpp:1533-1804). It is stored as 5 dense blocks
// per element, transposed ([rs][ij]) so that the K^2 threads of an element (one per
// output row) read consecutive addresses: the matrix streams from HBM once per product
// and the x entries of a column block are warp-broadcast loads.
//
// The solver replaces AMGCL's BiCGSTAB (src/HO_2D.hpp:53-54, src/HO_2D.cpp:1960) with a
// right-preconditioned BiCGSTAB (van der Vorst 1992) preconditioned by the inverse
// diagonal (element) blocks. All scalars stay on the device; each kernel fuses its
// vector update with the dot products the next step needs, reduced deterministically
// (per-CTA partials, the last CTA to finish sums them in a fixed order). A `done` flag
// makes the remaining launches of an enqueued batch return immediately, so the host only
// polls for convergence every few iterations.
#include "device.cuh"
#include "fr_launch.hpp"

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
        double x = 0.0;
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

template <int K, typename T, typename TM>
__device__ __forceinline__ T bsr_row(const BsrOp<TM>& A, const T* __restrict__ x, int el, int ij) {
    constexpr int K2 = K * K;
    T acc = T(0);
    const TM* blk = A.blocks + (size_t)el * 5 * K2 * K2 + ij;
#pragma unroll
    for (int s = 0; s < 5; ++s) {
        const int c = A.col[el * 5 + s];
        if (c < 0) continue;
        const T* xc = x + (size_t)c * K2;
        const TM* bs = blk + (size_t)s * K2 * K2;
#pragma unroll
        for (int rs = 0; rs < K2; ++rs) acc += T(__ldg(bs + rs * K2)) * __ldg(xc + rs);
    }
    return acc;
}

// z[el] = Dinv[el] y[el] with y staged in shared memory
template <int K, typename T, typename TM>
__device__ __forceinline__ T block_apply(const TM* __restrict__ dinv, const T* sy, int el, int ij) {
    constexpr int K2 = K * K;
    const TM* d = dinv + (size_t)el * K2 * K2 + ij;
    T acc = T(0);
#pragma unroll
    for (int rs = 0; rs < K2; ++rs) acc += T(__ldg(d + rs * K2)) * sy[rs];
    return acc;
}

}  // namespace

// r = b - A x, rhat = r; ||r||^2, ||b||^2
template <int K, typename T, typename TM>
__global__ void __launch_bounds__(Shape<K>::THREADS) k_init(BsrOp<TM> A, BicgVectors<T> v, ReduceScratch rs,
                                                             double tol) {
    using S = Shape<K>;
    const int le = threadIdx.x / S::K2, ij = threadIdx.x % S::K2;
    const int el = blockIdx.x * S::EPB + le;
    const bool active = le < S::EPB && el < A.N;
    double part[2] = {0.0, 0.0};
    if (active) {
        const int p = el * S::K2 + ij;
        const T bb = v.b[p];
        const T r = bb - bsr_row<K, T, TM>(A, v.x, el, ij);
        v.r[p] = r;
        v.rhat[p] = r;
        part[0] = double(r) * double(r);
        part[1] = double(bb) * double(bb);
    }
    double out[2];
    if (grid_reduce<2>(part, rs.partials, rs.counter, out) && threadIdx.x == 0) {
        KrylovScalars* sc = rs.sc;
        sc->rnorm2 = out[0];
        sc->bnorm2 = out[1];
        sc->eps2 = tol * tol * out[1];
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

// zero right-hand side: x = 0 (the reference's solver returns the zero vector)
template <typename T>
__global__ void k_zero_if(T* x, size_t n, const KrylovScalars* sc) {
    if (!sc->zero_rhs) return;
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] = T(0);
}

// p = r + beta (p - omega v) (p = r on the first iteration); ph = M^{-1} p
template <int K, typename T, typename TM>
__global__ void __launch_bounds__(Shape<K>::THREADS) k_p_update(BsrOp<TM> A, BicgVectors<T> v, ReduceScratch rs) {
    using S = Shape<K>;
    const KrylovScalars* sc = rs.sc;
    if (sc->done) return;
    __shared__ T sp[S::EPB][S::K2];
    const int le = threadIdx.x / S::K2, ij = threadIdx.x % S::K2;
    const int el = blockIdx.x * S::EPB + le;
    const bool active = le < S::EPB && el < A.N;
    const int p = el * S::K2 + ij;
    if (active) {
        T pv;
        if (sc->it == 0) {
            pv = v.r[p];
        } else {
            const double beta = (sc->rho / sc->rho_old) * (sc->alpha / sc->omega);
            pv = v.r[p] + T(beta) * (v.p[p] - T(sc->omega) * v.v[p]);
        }
        v.p[p] = pv;
        sp[le][ij] = pv;
    }
    __syncthreads();
    if (active) v.ph[p] = block_apply<K, T, TM>(A.dinv, sp[le], el, ij);
}

// v = A ph; alpha = rho / (rhat, v)
template <int K, typename T, typename TM>
__global__ void __launch_bounds__(Shape<K>::THREADS) k_spmv_v(BsrOp<TM> A, BicgVectors<T> v, ReduceScratch rs) {
    using S = Shape<K>;
    KrylovScalars* sc = rs.sc;
    if (sc->done) return;
    const int le = threadIdx.x / S::K2, ij = threadIdx.x % S::K2;
    const int el = blockIdx.x * S::EPB + le;
    const bool active = le < S::EPB && el < A.N;
    double part[1] = {0.0};
    if (active) {
        const int p = el * S::K2 + ij;
        const T y = bsr_row<K, T, TM>(A, v.ph, el, ij);
        v.v[p] = y;
        part[0] = double(v.rhat[p]) * double(y);
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

// s = r - alpha v; ||s||^2; sh = M^{-1} s
template <int K, typename T, typename TM>
__global__ void __launch_bounds__(Shape<K>::THREADS) k_s_update(BsrOp<TM> A, BicgVectors<T> v, ReduceScratch rs) {
    using S = Shape<K>;
    KrylovScalars* sc = rs.sc;
    if (sc->done) return;
    __shared__ T sp[S::EPB][S::K2];
    const int le = threadIdx.x / S::K2, ij = threadIdx.x % S::K2;
    const int el = blockIdx.x * S::EPB + le;
    const bool active = le < S::EPB && el < A.N;
    const int p = el * S::K2 + ij;
    double part[1] = {0.0};
    if (active) {
        const T s = v.r[p] - T(sc->alpha) * v.v[p];
        v.s[p] = s;
        sp[le][ij] = s;
        part[0] = double(s) * double(s);
    }
    __syncthreads();
    if (active) v.sh[p] = block_apply<K, T, TM>(A.dinv, sp[le], el, ij);
    double out[1];
    if (grid_reduce<1>(part, rs.partials, rs.counter, out) && threadIdx.x == 0) {
        sc->snorm2 = out[0];
        sc->s_exit = out[0] <= sc->eps2;
    }
}

// t = A sh; omega = (t, s) / (t, t)
template <int K, typename T, typename TM>
__global__ void __launch_bounds__(Shape<K>::THREADS) k_spmv_t(BsrOp<TM> A, BicgVectors<T> v, ReduceScratch rs) {
    using S = Shape<K>;
    KrylovScalars* sc = rs.sc;
    if (sc->done || sc->s_exit) return;
    const int le = threadIdx.x / S::K2, ij = threadIdx.x % S::K2;
    const int el = blockIdx.x * S::EPB + le;
    const bool active = le < S::EPB && el < A.N;
    double part[2] = {0.0, 0.0};
    if (active) {
        const int p = el * S::K2 + ij;
        const T y = bsr_row<K, T, TM>(A, v.sh, el, ij);
        v.t[p] = y;
        part[0] = double(y) * double(v.s[p]);
        part[1] = double(y) * double(y);
    }
    double out[2];
    if (grid_reduce<2>(part, rs.partials, rs.counter, out) && threadIdx.x == 0)
        sc->omega = out[1] > 0.0 ? out[0] / out[1] : 0.0;
}

// x += alpha ph + omega sh; r = s - omega t; ||r||^2, (rhat, r); convergence test
template <int K, typename T, typename TM>
__global__ void __launch_bounds__(Shape<K>::THREADS) k_xr_update(BsrOp<TM> A, BicgVectors<T> v, ReduceScratch rs,
                                                                  int max_iter) {
    using S = Shape<K>;
    KrylovScalars* sc = rs.sc;
    if (sc->done) return;
    const int le = threadIdx.x / S::K2, ij = threadIdx.x % S::K2;
    const int el = blockIdx.x * S::EPB + le;
    const bool active = le < S::EPB && el < A.N;
    const int p = el * S::K2 + ij;
    const double alpha = sc->alpha;
    if (sc->s_exit) {  // ||s|| already below tolerance: x += alpha ph and stop
        if (active) v.x[p] += T(alpha) * v.ph[p];
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            // every CTA read s_exit before any could observe done: done is only read at kernel entry
            sc->rnorm2 = sc->snorm2;
            sc->it += 1;
        }
        return;
    }
    const double omega = sc->omega;
    double part[2] = {0.0, 0.0};
    if (active) {
        v.x[p] += T(alpha) * v.ph[p] + T(omega) * v.sh[p];
        const T r = v.s[p] - T(omega) * v.t[p];
        v.r[p] = r;
        part[0] = double(r) * double(r);
        part[1] = double(v.rhat[p]) * double(r);
    }
    double out[2];
    if (grid_reduce<2>(part, rs.partials, rs.counter, out) && threadIdx.x == 0) {
        sc->rnorm2 = out[0];
        sc->rho_old = sc->rho;
        sc->rho = out[1];
        sc->it += 1;
        if (out[0] <= sc->eps2 || sc->it >= max_iter || omega == 0.0) sc->done = 1;
    }
}

// marks the solve finished after an s-exit iteration (separate launch: all CTAs of
// k_xr_update have read s_exit before this runs)
__global__ void k_finish_s_exit(KrylovScalars* sc) {
    if (!sc->done && sc->s_exit) sc->done = 1;
}

// r = b - A x in FP64; ||r||^2 -> rnorm2, ||b||^2 -> bnorm2
template <int K, typename TM>
__global__ void __launch_bounds__(Shape<K>::THREADS) k_residual64(BsrOp<TM> A, const double* __restrict__ b,
                                                                   const double* __restrict__ x, double* r,
                                                                   ReduceScratch rs) {
    using S = Shape<K>;
    const int le = threadIdx.x / S::K2, ij = threadIdx.x % S::K2;
    const int el = blockIdx.x * S::EPB + le;
    const bool active = le < S::EPB && el < A.N;
    double part[2] = {0.0, 0.0};
    if (active) {
        const int p = el * S::K2 + ij;
        const double y = b[p] - bsr_row<K, double, TM>(A, x, el, ij);
        r[p] = y;
        part[0] = y * y;
        part[1] = b[p] * b[p];
    }
    double out[2];
    if (grid_reduce<2>(part, rs.partials, rs.counter, out) && threadIdx.x == 0) {
        rs.sc->rnorm2 = out[0];
        rs.sc->bnorm2 = out[1];
    }
}

__global__ void k_d2f(const double* a, float* b, size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = (float)a[i];
}
__global__ void k_f2d(const float* a, double* b, size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = (double)a[i];
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

template <int K>
static unsigned kgrid(int N) {
    return (unsigned)((N + Shape<K>::EPB - 1) / Shape<K>::EPB);
}

int krylov_max_blocks(int K, int N) {
    const int k2 = K * K;
    const int epb = (256 / k2) > 64 ? 64 : ((256 / k2) > 0 ? 256 / k2 : 1);
    return (N + epb - 1) / epb;
}

template <typename T, typename TM>
cudaError_t krylov_init(const BsrOp<TM>& A, const BicgVectors<T>& v, const ReduceScratch& rs, double tol,
                        cudaStream_t s) {
    HO2D_KSWITCH(A.K, (k_init<KK, T, TM><<<kgrid<KK>(A.N), Shape<KK>::THREADS, 0, s>>>(A, v, rs, tol)));
    const size_t n = (size_t)A.N * A.K * A.K;
    k_zero_if<T><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(v.x, n, rs.sc);
    return cudaGetLastError();
}

template <int K, typename T, typename TM>
static void iteration_impl(const BsrOp<TM>& A, const BicgVectors<T>& v, const ReduceScratch& rs, int max_iter,
                           cudaStream_t s) {
    const unsigned g = kgrid<K>(A.N);
    constexpr int th = Shape<K>::THREADS;
    k_p_update<K, T, TM><<<g, th, 0, s>>>(A, v, rs);
    k_spmv_v<K, T, TM><<<g, th, 0, s>>>(A, v, rs);
    k_s_update<K, T, TM><<<g, th, 0, s>>>(A, v, rs);
    k_spmv_t<K, T, TM><<<g, th, 0, s>>>(A, v, rs);
    k_xr_update<K, T, TM><<<g, th, 0, s>>>(A, v, rs, max_iter);
}

template <typename T, typename TM>
cudaError_t krylov_iteration(const BsrOp<TM>& A, const BicgVectors<T>& v, const ReduceScratch& rs, int max_iter,
                             cudaStream_t s) {
    HO2D_KSWITCH(A.K, (iteration_impl<KK, T, TM>(A, v, rs, max_iter, s)));
    k_finish_s_exit<<<1, 1, 0, s>>>(rs.sc);
    return cudaGetLastError();
}

template <int K, typename T, typename TM>
__global__ void k_reset_done(KrylovScalars* sc) {
    sc->done = 0;
    sc->s_exit = 0;
    sc->rho = 1.0;
}

template <typename T, typename TM>
cudaError_t krylov_spmv_only(const BsrOp<TM>& A, const BicgVectors<T>& v, const ReduceScratch& rs, int reps,
                             cudaStream_t s) {
    k_reset_done<1, T, TM><<<1, 1, 0, s>>>(rs.sc);
    for (int r = 0; r < reps; ++r) {
        HO2D_KSWITCH(A.K, (k_spmv_v<KK, T, TM><<<kgrid<KK>(A.N), Shape<KK>::THREADS, 0, s>>>(A, v, rs)));
    }
    return cudaGetLastError();
}

template <typename TM>
cudaError_t residual_fp64(const BsrOp<TM>& A, const double* b, const double* x, double* r, const ReduceScratch& rs,
                          cudaStream_t s) {
    HO2D_KSWITCH(A.K, (k_residual64<KK, TM><<<kgrid<KK>(A.N), Shape<KK>::THREADS, 0, s>>>(A, b, x, r, rs)));
    return cudaGetLastError();
}

cudaError_t launch_copy_d2f(const double* a, float* b, size_t n, cudaStream_t s) {
    if (n) k_d2f<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(a, b, n);
    return cudaGetLastError();
}
cudaError_t launch_copy_f2d(const float* a, double* b, size_t n, cudaStream_t s) {
    if (n) k_f2d<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(a, b, n);
    return cudaGetLastError();
}
cudaError_t launch_axpy_f2d(const float* e, double* x, size_t n, cudaStream_t s) {
    if (n) k_axpy_f2d<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(e, x, n);
    return cudaGetLastError();
}

template cudaError_t krylov_init<double, double>(const BsrOp<double>&, const BicgVectors<double>&,
                                                 const ReduceScratch&, double, cudaStream_t);
template cudaError_t krylov_iteration<double, double>(const BsrOp<double>&, const BicgVectors<double>&,
                                                      const ReduceScratch&, int, cudaStream_t);
template cudaError_t krylov_init<float, float>(const BsrOp<float>&, const BicgVectors<float>&, const ReduceScratch&,
                                               double, cudaStream_t);
template cudaError_t krylov_iteration<float, float>(const BsrOp<float>&, const BicgVectors<float>&,
                                                    const ReduceScratch&, int, cudaStream_t);
template cudaError_t krylov_spmv_only<double, double>(const BsrOp<double>&, const BicgVectors<double>&,
                                                      const ReduceScratch&, int, cudaStream_t);
template cudaError_t krylov_spmv_only<float, float>(const BsrOp<float>&, const BicgVectors<float>&,
                                                    const ReduceScratch&, int, cudaStream_t);
template cudaError_t residual_fp64<double>(const BsrOp<double>&, const double*, const double*, double*,
                                           const ReduceScratch&, cudaStream_t);

}  // namespace ho2d
