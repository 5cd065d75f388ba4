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
#include "device.cuh"
#include "fr_device.cuh"
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

// Shared-memory working set of one CTA (EPB elements).
template <int K, typename T>
struct MfShared {
    static constexpr int K2 = K * K, NF = 4 * K, EPB = Shape<K>::EPB;
    T x[EPB][K2], a[EPB][K2], b[EPB][K2];
    T tv[EPB][NF], tg[EPB][NF], com[EPB][NF], cg[EPB][NF], fb[EPB][NF];
};

// y = A x at (el, ij); x's own traces are recomputed, the neighbours' come from tv/tg.
// Collective. Leaves x of the element in sm.x.
template <int K, typename T>
__device__ T mf_apply(const MfOp<T>& op, const T* __restrict__ x, const T* __restrict__ tv, const T* __restrict__ tg,
                      MfShared<K, T>& sm, bool active, int le, int el, int ij) {
    constexpr int K2 = K * K, NF = 4 * K;
    const int lei = active ? le : 0;
    if (active) sm.x[le][ij] = x[el * K2 + ij];
    __syncthreads();
    if (active)
        for (int o = ij; o < NF; o += K2) face_trace<K, T>(sm.x[le], op.b, o, sm.tv[le][o], sm.tg[le][o]);
    __syncthreads();
    return lap_element<K, T>(active, el, ij, op.g, op.b, tv, tg, sm.x[lei], sm.tv[lei], sm.tg[lei], sm.com[lei],
                             sm.cg[lei], sm.a[lei], sm.b[lei], sm.fb[lei], op.g.sw_p, op.zero_bc);
}

// face traces of an element vector held in shared memory
template <int K, typename T>
__device__ __forceinline__ void emit_traces(const T* sy, const DevBases<T>& b, T* tv, T* tg, bool active, int el,
                                            int ij) {
    constexpr int K2 = K * K, NF = 4 * K;
    if (!active) return;
    for (int o = ij; o < NF; o += K2) {
        T v, d;
        face_trace<K, T>(sy, b, o, v, d);
        tv[el * NF + o] = v;
        tg[el * NF + o] = d;
    }
}

// z = Dinv y for one element, y in shared memory (Dinv stored [rs][ij])
template <int K, typename T>
__device__ __forceinline__ T block_apply(const T* __restrict__ dinv, const T* sy, int el, int ij) {
    constexpr int K2 = K * K;
    const T* d = dinv + (size_t)el * K2 * K2 + ij;
    T acc = T(0);
#pragma unroll
    for (int rs = 0; rs < K2; ++rs) acc += __ldg(d + rs * K2) * sy[rs];
    return acc;
}

__device__ __forceinline__ bool pc_skip(const KrylovScalars* sc, int mode) {
    return sc->done || (mode == 1 && sc->s_exit);
}

}  // namespace

// ---------------------------------------------------------------- fine-level kernels
// r = b - A x (x's traces in xtv/xtg), rhat = r; ||r||^2, ||b||^2
template <int K, typename T>
__global__ void __launch_bounds__(Shape<K>::THREADS) k_mf_init(MfOp<T> op, BicgVectors<T> v, ReduceScratch rs,
                                                                double tol) {
    using S = Shape<K>;
    __shared__ MfShared<K, T> sm;
    const int le = threadIdx.x / S::K2, ij = threadIdx.x % S::K2;
    const int el = blockIdx.x * S::EPB + le;
    const bool active = le < S::EPB && el < op.g.N;
    const T y = mf_apply<K, T>(op, v.x, v.xtv, v.xtg, sm, active, le, el, ij);
    double part[2] = {0.0, 0.0};
    if (active) {
        const int p = el * S::K2 + ij;
        const T bb = v.b[p];
        const T r = bb - y;
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

template <typename T>
__global__ void k_zero_if(T* x, size_t n, const KrylovScalars* sc) {
    if (!sc->zero_rhs) return;
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] = T(0);
}

// p = r + beta (p - omega v) (= r on the first iteration); then either ph = D^{-1} p with
// its traces (block-Jacobi) or the element sums of p (two-level: coarse right-hand side)
template <int K, typename T>
__global__ void __launch_bounds__(Shape<K>::THREADS) k_mf_pupdate(MfOp<T> op, BicgVectors<T> v, ReduceScratch rs,
                                                                   T* rc) {
    using S = Shape<K>;
    const KrylovScalars* sc = rs.sc;
    if (sc->done) return;
    __shared__ T sp[S::EPB][S::K2], sz[S::EPB][S::K2];
    const int le = threadIdx.x / S::K2, ij = threadIdx.x % S::K2;
    const int el = blockIdx.x * S::EPB + le;
    const bool active = le < S::EPB && el < op.g.N;
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
    if (rc) {
        if (active && ij == 0) {
            T sum = T(0);
#pragma unroll
            for (int q = 0; q < S::K2; ++q) sum += sp[le][q];
            rc[el] = sum;
        }
        return;
    }
    if (active) {
        const T z = block_apply<K, T>(op.dinv, sp[le], el, ij);
        v.ph[p] = z;
        sz[le][ij] = z;
    }
    __syncthreads();
    emit_traces<K, T>(sz[active ? le : 0], op.b, v.tv, v.tg, active, el, ij);
}

// two-level smoothing step: z = e + w D^{-1} (f - A e), e = P ec element-wise constant;
// writes z and its face traces
template <int K, typename T>
__global__ void __launch_bounds__(Shape<K>::THREADS) k_mf_post(MfOp<T> op, const T* __restrict__ f,
                                                                const T* __restrict__ ec, T* __restrict__ z,
                                                                T* __restrict__ tv, T* __restrict__ tg, double w,
                                                                const KrylovScalars* sc, int mode) {
    using S = Shape<K>;
    constexpr int K2 = S::K2;
    if (pc_skip(sc, mode)) return;
    __shared__ T sr[S::EPB][K2], sz[S::EPB][K2];
    const int le = threadIdx.x / K2, ij = threadIdx.x % K2;
    const int el = blockIdx.x * S::EPB + le;
    const bool active = le < S::EPB && el < op.g.N;
    const int p = el * K2 + ij;
    if (active) {
        T ae = T(0);
#pragma unroll
        for (int s = 0; s < 5; ++s) {
            const int c = op.bcol[el * 5 + s];
            if (c >= 0) ae += op.rowsum[((size_t)el * 5 + s) * K2 + ij] * ec[c];
        }
        sr[le][ij] = f[p] - ae;
    }
    __syncthreads();
    if (active) {
        const T zz = ec[el] + T(w) * block_apply<K, T>(op.dinv, sr[le], el, ij);
        z[p] = zz;
        sz[le][ij] = zz;
    }
    __syncthreads();
    emit_traces<K, T>(sz[active ? le : 0], op.b, tv, tg, active, el, ij);
}

// v = A ph; alpha = rho / (rhat, v)
template <int K, typename T>
__global__ void __launch_bounds__(Shape<K>::THREADS) k_mf_v(MfOp<T> op, BicgVectors<T> v, ReduceScratch rs) {
    using S = Shape<K>;
    KrylovScalars* sc = rs.sc;
    if (sc->done) return;
    __shared__ MfShared<K, T> sm;
    const int le = threadIdx.x / S::K2, ij = threadIdx.x % S::K2;
    const int el = blockIdx.x * S::EPB + le;
    const bool active = le < S::EPB && el < op.g.N;
    const T y = mf_apply<K, T>(op, v.ph, v.tv, v.tg, sm, active, le, el, ij);
    double part[1] = {0.0};
    if (active) {
        const int p = el * S::K2 + ij;
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

// s = r - alpha v; ||s||^2; then sh = D^{-1} s with traces, or the element sums of s
template <int K, typename T>
__global__ void __launch_bounds__(Shape<K>::THREADS) k_mf_supdate(MfOp<T> op, BicgVectors<T> v, ReduceScratch rs,
                                                                   T* rc) {
    using S = Shape<K>;
    KrylovScalars* sc = rs.sc;
    if (sc->done) return;
    __shared__ T sp[S::EPB][S::K2], sz[S::EPB][S::K2];
    const int le = threadIdx.x / S::K2, ij = threadIdx.x % S::K2;
    const int el = blockIdx.x * S::EPB + le;
    const bool active = le < S::EPB && el < op.g.N;
    const int p = el * S::K2 + ij;
    double part[1] = {0.0};
    if (active) {
        const T s = v.r[p] - T(sc->alpha) * v.v[p];
        v.s[p] = s;
        sp[le][ij] = s;
        part[0] = double(s) * double(s);
    }
    __syncthreads();
    if (rc) {
        if (active && ij == 0) {
            T sum = T(0);
#pragma unroll
            for (int q = 0; q < S::K2; ++q) sum += sp[le][q];
            rc[el] = sum;
        }
    } else {
        if (active) {
            const T z = block_apply<K, T>(op.dinv, sp[le], el, ij);
            v.sh[p] = z;
            sz[le][ij] = z;
        }
        __syncthreads();
        emit_traces<K, T>(sz[active ? le : 0], op.b, v.tv, v.tg, active, el, ij);
    }
    double out[1];
    if (grid_reduce<1>(part, rs.partials, rs.counter, out) && threadIdx.x == 0) {
        sc->snorm2 = out[0];
        sc->s_exit = out[0] <= sc->eps2;
    }
}

// t = A sh; omega = (t, s) / (t, t)
template <int K, typename T>
__global__ void __launch_bounds__(Shape<K>::THREADS) k_mf_t(MfOp<T> op, BicgVectors<T> v, ReduceScratch rs) {
    using S = Shape<K>;
    KrylovScalars* sc = rs.sc;
    if (sc->done || sc->s_exit) return;
    __shared__ MfShared<K, T> sm;
    const int le = threadIdx.x / S::K2, ij = threadIdx.x % S::K2;
    const int el = blockIdx.x * S::EPB + le;
    const bool active = le < S::EPB && el < op.g.N;
    const T y = mf_apply<K, T>(op, v.sh, v.tv, v.tg, sm, active, le, el, ij);
    double part[2] = {0.0, 0.0};
    if (active) {
        const int p = el * S::K2 + ij;
        v.t[p] = y;
        part[0] = double(y) * double(v.s[p]);
        part[1] = double(y) * double(y);
    }
    double out[2];
    if (grid_reduce<2>(part, rs.partials, rs.counter, out) && threadIdx.x == 0)
        sc->omega = out[1] > 0.0 ? out[0] / out[1] : 0.0;
}

// x += alpha ph + omega sh; r = s - omega t; ||r||^2, (rhat, r); convergence test
template <int K, typename T>
__global__ void __launch_bounds__(Shape<K>::THREADS) k_xr_update(int N, BicgVectors<T> v, ReduceScratch rs,
                                                                  int max_iter) {
    using S = Shape<K>;
    KrylovScalars* sc = rs.sc;
    if (sc->done) return;
    const int le = threadIdx.x / S::K2, ij = threadIdx.x % S::K2;
    const int el = blockIdx.x * S::EPB + le;
    const bool active = le < S::EPB && el < N;
    const int p = el * S::K2 + ij;
    const double alpha = sc->alpha;
    if (sc->s_exit) {  // ||s|| already below tolerance: x += alpha ph and stop
        if (active) v.x[p] += T(alpha) * v.ph[p];
        if (blockIdx.x == 0 && threadIdx.x == 0) {
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

// ends the solve after an s-exit iteration (a separate launch: every CTA of k_xr_update
// has read s_exit before done changes)
__global__ void k_finish_s_exit(KrylovScalars* sc) {
    if (!sc->done && sc->s_exit) sc->done = 1;
}

// r = b - A x (FP64 refinement residual); ||r||^2 -> rnorm2, ||b||^2 -> bnorm2
template <int K, typename T>
__global__ void __launch_bounds__(Shape<K>::THREADS) k_mf_residual(MfOp<T> op, const double* __restrict__ b,
                                                                    const T* __restrict__ x, const T* __restrict__ xtv,
                                                                    const T* __restrict__ xtg, double* __restrict__ r,
                                                                    ReduceScratch rs) {
    using S = Shape<K>;
    __shared__ MfShared<K, T> sm;
    const int le = threadIdx.x / S::K2, ij = threadIdx.x % S::K2;
    const int el = blockIdx.x * S::EPB + le;
    const bool active = le < S::EPB && el < op.g.N;
    const T y = mf_apply<K, T>(op, x, xtv, xtg, sm, active, le, el, ij);
    double part[2] = {0.0, 0.0};
    if (active) {
        const int p = el * S::K2 + ij;
        const double rr = b[p] - double(y);
        r[p] = rr;
        part[0] = rr * rr;
        part[1] = b[p] * b[p];
    }
    double out[2];
    if (grid_reduce<2>(part, rs.partials, rs.counter, out) && threadIdx.x == 0) {
        rs.sc->rnorm2 = out[0];
        rs.sc->bnorm2 = out[1];
    }
}

// y = A x (operator only)
template <int K, typename T>
__global__ void __launch_bounds__(Shape<K>::THREADS) k_mf_apply(MfOp<T> op, const T* __restrict__ x,
                                                                 const T* __restrict__ xtv, const T* __restrict__ xtg,
                                                                 T* __restrict__ y) {
    using S = Shape<K>;
    __shared__ MfShared<K, T> sm;
    const int le = threadIdx.x / S::K2, ij = threadIdx.x % S::K2;
    const int el = blockIdx.x * S::EPB + le;
    const bool active = le < S::EPB && el < op.g.N;
    const T yy = mf_apply<K, T>(op, x, xtv, xtg, sm, active, le, el, ij);
    if (active) y[el * S::K2 + ij] = yy;
}

// ---------------------------------------------------------------- coarse levels (scalar CSR)
template <typename T>
__device__ __forceinline__ T csr_row(const DevCsr<T>& A, const T* __restrict__ x, int i) {
    T acc = T(0);
    for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k) acc += A.val[k] * x[A.col[k]];
    return acc;
}

template <typename T>
__global__ void k_c_smooth0(int n, const T* __restrict__ m, const T* __restrict__ f, T* __restrict__ u,
                            const KrylovScalars* sc, int mode) {
    if (pc_skip(sc, mode)) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) u[i] = m[i] * f[i];
}

template <typename T>
__global__ void k_c_residual(DevCsr<T> A, const T* __restrict__ f, const T* __restrict__ u, T* __restrict__ t,
                             const KrylovScalars* sc, int mode) {
    if (pc_skip(sc, mode)) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < A.n) t[i] = f[i] - csr_row<T>(A, u, i);
}

template <typename T>
__global__ void k_c_spmv(DevCsr<T> M, const T* __restrict__ x, T* __restrict__ y, const KrylovScalars* sc,
                         int mode) {
    if (pc_skip(sc, mode)) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < M.n) y[i] = csr_row<T>(M, x, i);
}

template <typename T>
__global__ void k_c_prolong_add(DevCsr<T> P, const T* __restrict__ uc, T* __restrict__ u, const KrylovScalars* sc,
                                int mode) {
    if (pc_skip(sc, mode)) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < P.n) u[i] += csr_row<T>(P, uc, i);
}

template <typename T>
__global__ void k_c_smooth(DevCsr<T> A, const T* __restrict__ m, const T* __restrict__ f, const T* __restrict__ u,
                           T* __restrict__ u2, const KrylovScalars* sc, int mode) {
    if (pc_skip(sc, mode)) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < A.n) u2[i] = u[i] + m[i] * (f[i] - csr_row<T>(A, u, i));
}

template <typename T>
__global__ void k_c_dense(int n, const T* __restrict__ inv, const T* __restrict__ f, T* __restrict__ u,
                          const KrylovScalars* sc, int mode) {
    if (pc_skip(sc, mode)) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    T acc = T(0);
    for (int j = 0; j < n; ++j) acc += inv[(size_t)i * n + j] * f[j];
    u[i] = acc;
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

template <int K>
static unsigned kgrid(int N) {
    return (unsigned)((N + Shape<K>::EPB - 1) / Shape<K>::EPB);
}

int krylov_max_blocks(int K, int N) {
    const int k2 = K * K;
    const int epb = (256 / k2) > 64 ? 64 : ((256 / k2) > 0 ? 256 / k2 : 1);
    return (N + epb - 1) / epb;
}

template <typename T>
cudaError_t krylov_init(const MfOp<T>& op, const BicgVectors<T>& v, const ReduceScratch& rs, double tol,
                        cudaStream_t s) {
    const int N = op.g.N;
    cudaError_t e = launch_trace<T>(op.K, N, v.x, v.xtv, v.xtg, op.b, s);
    if (e != cudaSuccess) return e;
    HO2D_KSWITCH(op.K, (k_mf_init<KK, T><<<kgrid<KK>(N), Shape<KK>::THREADS, 0, s>>>(op, v, rs, tol)));
    const size_t n = (size_t)N * op.K * op.K;
    k_zero_if<T><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(v.x, n, rs.sc);
    return cudaGetLastError();
}

template <typename T>
static void coarse_cycle(const Precond<T>& pc, int l, const KrylovScalars* sc, int mode, cudaStream_t s) {
    const CoarseLevel<T>& L = pc.lev[l];
    const unsigned g = (unsigned)((L.n + 127) / 128);
    if (l == pc.nlev - 1) {
        k_c_dense<T><<<g, 128, 0, s>>>(L.n, pc.dense_inv, L.f, L.u, sc, mode);
        return;
    }
    const CoarseLevel<T>& C = pc.lev[l + 1];
    k_c_smooth0<T><<<g, 128, 0, s>>>(L.n, L.m, L.f, L.u, sc, mode);
    k_c_residual<T><<<g, 128, 0, s>>>(L.A, L.f, L.u, L.t, sc, mode);
    k_c_spmv<T><<<(unsigned)((C.n + 127) / 128), 128, 0, s>>>(L.R, L.t, C.f, sc, mode);
    coarse_cycle(pc, l + 1, sc, mode, s);
    k_c_prolong_add<T><<<g, 128, 0, s>>>(L.P, C.out, L.u, sc, mode);
    k_c_smooth<T><<<g, 128, 0, s>>>(L.A, L.m, L.f, L.u, L.u2, sc, mode);
}

template <int K, typename T>
static void iteration_impl(const MfOp<T>& op, const BicgVectors<T>& v, const ReduceScratch& rs, int max_iter,
                           const Precond<T>& pc, cudaStream_t s) {
    const int N = op.g.N;
    const unsigned g = kgrid<K>(N);
    constexpr int th = Shape<K>::THREADS;
    const bool mg = pc.nlev > 0;
    T* rc = mg ? pc.lev[0].f : nullptr;
    k_mf_pupdate<K, T><<<g, th, 0, s>>>(op, v, rs, rc);
    if (mg) {
        coarse_cycle(pc, 0, rs.sc, 0, s);
        k_mf_post<K, T><<<g, th, 0, s>>>(op, v.p, pc.lev[0].out, v.ph, v.tv, v.tg, pc.omega, rs.sc, 0);
    }
    k_mf_v<K, T><<<g, th, 0, s>>>(op, v, rs);
    k_mf_supdate<K, T><<<g, th, 0, s>>>(op, v, rs, rc);
    if (mg) {
        coarse_cycle(pc, 0, rs.sc, 1, s);
        k_mf_post<K, T><<<g, th, 0, s>>>(op, v.s, pc.lev[0].out, v.sh, v.tv, v.tg, pc.omega, rs.sc, 1);
    }
    k_mf_t<K, T><<<g, th, 0, s>>>(op, v, rs);
    k_xr_update<K, T><<<g, th, 0, s>>>(N, v, rs, max_iter);
}

template <typename T>
int krylov_launches_per_iteration(const Precond<T>& pc) {
    if (pc.nlev == 0) return 6;
    const int coarse = 5 * (pc.nlev - 1) + 1;
    return 6 + 2 * (coarse + 1);
}

template <typename T>
cudaError_t krylov_iteration(const MfOp<T>& op, const BicgVectors<T>& v, const ReduceScratch& rs, int max_iter,
                             const Precond<T>& pc, cudaStream_t s) {
    HO2D_KSWITCH(op.K, (iteration_impl<KK, T>(op, v, rs, max_iter, pc, s)));
    k_finish_s_exit<<<1, 1, 0, s>>>(rs.sc);
    return cudaGetLastError();
}

template <typename T>
cudaError_t mf_residual(const MfOp<T>& op, const double* b, const T* x, T* xtv, T* xtg, double* r,
                        const ReduceScratch& rs, cudaStream_t s) {
    cudaError_t e = launch_trace<T>(op.K, op.g.N, x, xtv, xtg, op.b, s);
    if (e != cudaSuccess) return e;
    HO2D_KSWITCH(op.K, (k_mf_residual<KK, T><<<kgrid<KK>(op.g.N), Shape<KK>::THREADS, 0, s>>>(op, b, x, xtv, xtg, r,
                                                                                                  rs)));
    return cudaGetLastError();
}

template <typename T>
cudaError_t mf_apply_op(const MfOp<T>& op, const T* x, T* xtv, T* xtg, T* y, cudaStream_t s) {
    cudaError_t e = launch_trace<T>(op.K, op.g.N, x, xtv, xtg, op.b, s);
    if (e != cudaSuccess) return e;
    HO2D_KSWITCH(op.K, (k_mf_apply<KK, T><<<kgrid<KK>(op.g.N), Shape<KK>::THREADS, 0, s>>>(op, x, xtv, xtg, y)));
    return cudaGetLastError();
}

template <typename T>
cudaError_t mf_apply_only(const MfOp<T>& op, const T* x, const T* xtv, const T* xtg, T* y, int reps, cudaStream_t s) {
    for (int r = 0; r < reps; ++r)
        HO2D_KSWITCH(op.K, (k_mf_apply<KK, T><<<kgrid<KK>(op.g.N), Shape<KK>::THREADS, 0, s>>>(op, x, xtv, xtg, y)));
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
    template cudaError_t krylov_init<T>(const MfOp<T>&, const BicgVectors<T>&, const ReduceScratch&, double,     \
                                        cudaStream_t);                                                            \
    template cudaError_t krylov_iteration<T>(const MfOp<T>&, const BicgVectors<T>&, const ReduceScratch&, int,    \
                                             const Precond<T>&, cudaStream_t);                                    \
    template int krylov_launches_per_iteration<T>(const Precond<T>&);                                             \
    template cudaError_t mf_residual<T>(const MfOp<T>&, const double*, const T*, T*, T*, double*,                 \
                                        const ReduceScratch&, cudaStream_t);                                      \
    template cudaError_t mf_apply_op<T>(const MfOp<T>&, const T*, T*, T*, T*, cudaStream_t);                      \
    template cudaError_t mf_apply_only<T>(const MfOp<T>&, const T*, const T*, const T*, T*, int, cudaStream_t);

HO2D_INSTANTIATE_KRYLOV(double)
HO2D_INSTANTIATE_KRYLOV(float)

}  // namespace ho2d
