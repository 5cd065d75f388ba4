// adjoint.cu -- kernels of the discrete adjoint of the FR stage (sm_100a).
//
//   k_residual_adjoint   reverse of residual_kernel (diffusion + advection type 1)
//   k_velocity_adjoint   reverse of velocity_kernel and update_diffusion_BC
//   k_poisson_transpose  own part of y = A^T x and the neighbours' slots
//   k_gather             own part + transposed traces of the incoming slots
//   k_esum, k_pc_transpose, k_kt_vec   BiCGSTAB on A^T mu = b with its preconditioner
//
// Element kernels: K^2 threads per element, AShape<K>::EPB elements per CTA, every
// element's scratch in shared memory (adjoint_chain.cuh holds the bodies). Reductions
// are per-CTA partial sums added in a fixed order by the last CTA, so results are
// bitwise reproducible.
#include <cmath>

#include "adjoint_launch.hpp"
#include "fr_device.cuh"

namespace ho2d {

namespace {

#define HO2D_ADJ_DISPATCH_K(K, CALL)                      \
    switch (K) {                                          \
        case 1: { constexpr int KK = 1; CALL; } break;     \
        case 2: { constexpr int KK = 2; CALL; } break;     \
        case 3: { constexpr int KK = 3; CALL; } break;     \
        case 4: { constexpr int KK = 4; CALL; } break;     \
        case 5: { constexpr int KK = 5; CALL; } break;     \
        case 6: { constexpr int KK = 6; CALL; } break;     \
        case 7: { constexpr int KK = 7; CALL; } break;     \
        case 8: { constexpr int KK = 8; CALL; } break;     \
        default: return cudaErrorInvalidValue;            \
    }

template <int K>
unsigned agrid(int N) {
    return (unsigned)((N + AShape<K>::EPB - 1) / AShape<K>::EPB);
}

// ---------------------------------------------------------------- stage adjoint
template <int K, typename T>
__global__ void __launch_bounds__(AShape<K>::THREADS) k_residual_adjoint(FrGeom<T> g, DevBases<T> bp,
                                                                          StageAdjArgs<T> a) {
    using S = AShape<K>;
    __shared__ DevBases<T> b;
    __shared__ ResidualAdjScratch<K, T> sm[S::EPB];
    stage_bases(b, bp);
    __syncthreads();
    const int le = threadIdx.x / S::K2, ij = threadIdx.x % S::K2;
    const int el = blockIdx.x * S::EPB + le;
    const bool active = le < S::EPB && el < g.N;
    residual_adjoint_body<K, T>(ElemCtx<S::K2>{ij}, active, el, g, b, a, sm[active ? le : 0]);
}

template <int K, typename T>
__global__ void __launch_bounds__(AShape<K>::THREADS) k_velocity_adjoint(FrGeom<T> g, DevBases<T> bp,
                                                                          StageAdjArgs<T> a) {
    using S = AShape<K>;
    __shared__ DevBases<T> b;
    __shared__ VelocityAdjScratch<K, T> sm[S::EPB];
    stage_bases(b, bp);
    __syncthreads();
    const int le = threadIdx.x / S::K2, ij = threadIdx.x % S::K2;
    const int el = blockIdx.x * S::EPB + le;
    const bool active = le < S::EPB && el < g.N;
    velocity_adjoint_body<K, T>(ElemCtx<S::K2>{ij}, active, el, g, b, a, sm[active ? le : 0]);
}

// ---------------------------------------------------------------- transposed operator
template <int K, typename T>
__global__ void __launch_bounds__(AShape<K>::THREADS) k_poisson_transpose(FrGeom<T> g, DevBases<T> bp,
                                                                           const T* __restrict__ x, T* dir, T* sv,
                                                                           T* sg, const KrylovScalars* sc, int mode) {
    if (sc && pc_skip(sc, mode)) return;
    using S = AShape<K>;
    __shared__ DevBases<T> b;
    __shared__ LapAdjScratch<K, T> sm[S::EPB];
    stage_bases(b, bp);
    __syncthreads();
    const int le = threadIdx.x / S::K2, ij = threadIdx.x % S::K2;
    const int el = blockIdx.x * S::EPB + le;
    const bool active = le < S::EPB && el < g.N;
    poisson_transpose_body<K, T>(ElemCtx<S::K2>{ij}, active, el, g, b, x, dir, sv, sg, sm[active ? le : 0]);
}

template <int K, typename T>
__global__ void __launch_bounds__(AShape<K>::THREADS) k_gather(int N, DevBases<T> bp, const T* __restrict__ dir,
                                                                const T* __restrict__ sv, const T* __restrict__ sg,
                                                                T* __restrict__ out, const KrylovScalars* sc,
                                                                int mode) {
    if (sc && pc_skip(sc, mode)) return;
    using S = AShape<K>;
    __shared__ DevBases<T> b;
    __shared__ GatherScratch<K, T> sm[S::EPB];
    stage_bases(b, bp);
    __syncthreads();
    const int le = threadIdx.x / S::K2, ij = threadIdx.x % S::K2;
    const int el = blockIdx.x * S::EPB + le;
    const bool active = le < S::EPB && el < N;
    gather_body<K, T>(ElemCtx<S::K2>{ij}, active, el, b, dir, sv, sg, out, sm[active ? le : 0]);
}

// ---------------------------------------------------------------- preconditioner
// f0[e] = sum of element e's K^2 values (P^T y), one thread per element, fixed order
template <int K, typename T>
__global__ void __launch_bounds__(256) k_esum(int N, const T* __restrict__ y, T* __restrict__ f0,
                                              const KrylovScalars* sc, int mode) {
    if (pc_skip(sc, mode)) return;
    const int el = blockIdx.x * blockDim.x + threadIdx.x;
    if (el >= N) return;
    constexpr int K2 = K * K;
    T acc = T(0);
#pragma unroll
    for (int q = 0; q < K2; ++q) acc += y[(size_t)el * K2 + q];
    f0[el] = acc;
}

// z = e + omega D^-T (y - A^T e) with e = P u0 (u0 one value per element; e = 0 without a
// coarse level). (A^T P u0) at element el = sum over its 5 block slots of the column sums
// rowsumT times u0 of the slot's element.
template <int K, typename T>
__global__ void __launch_bounds__(AShape<K>::THREADS) k_pc_transpose(int N, const T* __restrict__ dinv,
                                                                      const T* __restrict__ rowsumT,
                                                                      const int* __restrict__ bcol,
                                                                      const T* __restrict__ u0,
                                                                      const T* __restrict__ y, T* __restrict__ z,
                                                                      double omega, const KrylovScalars* sc,
                                                                      int mode) {
    if (pc_skip(sc, mode)) return;
    using S = AShape<K>;
    constexpr int K2 = S::K2;
    __shared__ T q[S::EPB][K2];
    const int le = threadIdx.x / K2, ij = threadIdx.x % K2;
    const int el = blockIdx.x * S::EPB + le;
    const bool active = le < S::EPB && el < N;
    T ue = T(0);
    if (active) {
        const size_t p = (size_t)el * K2 + ij;
        T acc = y[p];
        if (u0) {
            ue = u0[el];
#pragma unroll
            for (int s = 0; s < 5; ++s) {
                const int c = bcol[el * 5 + s];
                if (c >= 0) acc -= rowsumT[((size_t)el * 5 + s) * K2 + ij] * u0[c];
            }
        }
        q[le][ij] = acc;
    }
    __syncthreads();
    if (!active) return;
    // (D^-1)[a][b] is stored at [b][a]; row ij of D^-T is therefore contiguous
    const T* d = dinv + (size_t)el * padded_count(K2 * K2, (int)sizeof(T)) + (size_t)ij * K2;
    T acc = T(0);
#pragma unroll
    for (int rs = 0; rs < K2; ++rs) acc += d[rs] * q[le][rs];
    z[(size_t)el * K2 + ij] = ue + T(omega) * acc;
}

// ---------------------------------------------------------------- BiCGSTAB vector steps
constexpr int kKtThreads = 256;
constexpr int kKtGrid = 2 * 148;

enum KtOp : int { KT_INIT = 0, KT_ALPHA, KT_S, KT_OMEGA, KT_XR, KT_P, KT_RES };

// Scalar step of the last CTA, from the two reduced dot products a, b.
__device__ void kt_finish(int op, double a, double b, KrylovScalars* sc, int max_iter) {
    const double tol2 = sc->tol * sc->tol;
    switch (op) {
        case KT_INIT:
            sc->bnorm2 = a;
            sc->rho = a;
            sc->rnorm2 = a;
            sc->it = 0;
            sc->s_exit = 0;
            sc->breakdown = 0;
            sc->zero_rhs = a == 0.0;
            sc->done = (a == 0.0 || !isfinite(a)) ? 1 : 0;
            break;
        case KT_ALPHA:
            if (a == 0.0 || !isfinite(a)) {
                sc->breakdown = 1;
                sc->done = 1;
            } else {
                sc->alpha = sc->rho / a;
            }
            break;
        case KT_S:
            sc->snorm2 = a;
            sc->s_exit = a <= tol2 * sc->bnorm2 ? 1 : 0;
            break;
        case KT_OMEGA:
            if (b > 0.0 && a != 0.0) {
                sc->omega = a / b;
            } else {
                sc->omega = 0.0;
                sc->breakdown = 1;
            }
            break;
        case KT_XR:
            sc->it += 1;
            if (sc->s_exit) {
                sc->rnorm2 = sc->snorm2;
                sc->done = 1;
            } else {
                sc->rho_old = sc->rho;
                sc->rho = a;
                sc->rnorm2 = b;
                sc->beta = (sc->omega != 0.0 && sc->rho_old != 0.0) ? (a / sc->rho_old) * (sc->alpha / sc->omega) : 0.0;
                sc->done = (b <= tol2 * sc->bnorm2 || sc->it >= max_iter || sc->breakdown || a == 0.0 || !isfinite(b))
                               ? 1
                               : 0;
            }
            break;
        case KT_RES:
            sc->rnorm2 = a;
            sc->bnorm2 = b;
            break;
        default:
            break;
    }
}

// One vector step of the iteration. Every CTA reads `done` and `s_exit` before any CTA
// arrives at the counter, so the last CTA may change them. Inside a captured solve the XR
// step sets the condition of the graph's while node (iterate while not done); a body
// execution either increments `it` (the XR step sets done at max_iter) or finds done set
// and clears the condition, so the device loop always ends.
template <typename T>
__global__ void __launch_bounds__(kKtThreads) k_kt_vec(int op, size_t n, TVectors<T> v, const T* __restrict__ rb,
                                                        const T* __restrict__ ry, T* __restrict__ rr, TReduce red,
                                                        int max_iter, cudaGraphConditionalHandle h, int has_handle) {
    KrylovScalars* sc = red.sc;
    if (op != KT_INIT && op != KT_RES) {
        if (sc->done) {
            if (op == KT_XR && has_handle && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(h, 0u);
            return;
        }
        if (op == KT_OMEGA && sc->s_exit) return;
    }
    const int s_exit = sc->s_exit;
    const T alpha = T(sc->alpha), omega = T(sc->omega), beta = T(sc->beta);
    double d0 = 0.0, d1 = 0.0;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        switch (op) {
            case KT_INIT: {
                const T bi = v.b[i];
                v.x[i] = T(0);
                v.r[i] = bi;
                v.rhat[i] = bi;
                v.p[i] = bi;
                d0 += double(bi) * double(bi);
            } break;
            case KT_ALPHA:
                d0 += double(v.rhat[i]) * double(v.v[i]);
                break;
            case KT_S: {
                const T si = v.r[i] - alpha * v.v[i];
                v.s[i] = si;
                d0 += double(si) * double(si);
            } break;
            case KT_OMEGA: {
                const double ti = double(v.t[i]);
                d0 += ti * double(v.s[i]);
                d1 += ti * ti;
            } break;
            case KT_XR:
                if (s_exit) {
                    v.x[i] += alpha * v.ph[i];
                } else {
                    v.x[i] += alpha * v.ph[i] + omega * v.sh[i];
                    const T ri = v.s[i] - omega * v.t[i];
                    v.r[i] = ri;
                    d0 += double(v.rhat[i]) * double(ri);
                    d1 += double(ri) * double(ri);
                }
                break;
            case KT_P:
                v.p[i] = v.r[i] + beta * (v.p[i] - omega * v.v[i]);
                break;
            case KT_RES: {
                const T bi = rb[i];
                const T ri = bi - ry[i];
                rr[i] = ri;
                d0 += double(ri) * double(ri);
                d1 += double(bi) * double(bi);
            } break;
            default:
                break;
        }
    }
    if (op == KT_P) return;
    __shared__ double s0[kKtThreads], s1[kKtThreads];
    __shared__ bool last;
    s0[threadIdx.x] = d0;
    s1[threadIdx.x] = d1;
    __syncthreads();
    for (int h = kKtThreads / 2; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h) {
            s0[threadIdx.x] += s0[threadIdx.x + h];
            s1[threadIdx.x] += s1[threadIdx.x + h];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        red.partials[blockIdx.x] = s0[0];
        red.partials[gridDim.x + blockIdx.x] = s1[0];
        __threadfence();
        last = atomicAdd(red.counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last || threadIdx.x != 0) return;
    __threadfence();
    double a = 0.0, b = 0.0;
    for (unsigned k = 0; k < gridDim.x; ++k) {
        a += __ldcg(&red.partials[k]);
        b += __ldcg(&red.partials[gridDim.x + k]);
    }
    *red.counter = 0u;
    kt_finish(op, a, b, sc, max_iter);
    if (op == KT_XR && has_handle) cudaGraphSetConditional(h, sc->done ? 0u : 1u);
}

__global__ void k_kt_set_loop(const KrylovScalars* sc, cudaGraphConditionalHandle h) {
    cudaGraphSetConditional(h, sc->done ? 0u : 1u);
}

template <typename T>
cudaError_t kt_vec(int op, size_t n, const TVectors<T>& v, const TReduce& r, int max_iter, cudaStream_t s,
                   const T* rb = nullptr, const T* ry = nullptr, T* rr = nullptr,
                   cudaGraphConditionalHandle h = cudaGraphConditionalHandle(), int has_handle = 0) {
    k_kt_vec<T><<<kKtGrid, kKtThreads, 0, s>>>(op, n, v, rb, ry, rr, r, max_iter, h, has_handle);
    return cudaGetLastError();
}

// z = B^T y (mode 0: y = p; mode 1: y = s, skipped after an early exit)
template <typename T>
cudaError_t pc_transpose_apply(int K, int N, const TPrecond<T>& pc, const T* y, T* z, T* f0, KrylovScalars* sc,
                               int mode, cudaStream_t s) {
    const bool coarse = pc.pc.nlev > 0;
    if (coarse) {
        HO2D_ADJ_DISPATCH_K(K, (k_esum<KK, T><<<(N + 255) / 256, 256, 0, s>>>(N, y, f0, sc, mode)));
        cudaError_t e = coarse_cycle_vec<T>(pc.pc, f0, sc, s);
        if (e != cudaSuccess) return e;
    }
    const T* u0 = coarse ? pc.pc.lev[0].u : nullptr;
    HO2D_ADJ_DISPATCH_K(K, (k_pc_transpose<KK, T><<<agrid<KK>(N), AShape<KK>::THREADS, 0, s>>>(
                               N, pc.dinv, pc.rowsumT, pc.bcol, u0, y, z, pc.pc.omega, sc, mode)));
    return cudaGetLastError();
}

__global__ void k_axpby(size_t n, double* out, double a, const double* x, double c, const double* y) {
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) out[i] = a * x[i] + c * y[i];
}

__global__ void k_sub_scaled(size_t n, double* out, const double* x, const double* J, const double* mu) {
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) out[i] = x[i] - J[i] * mu[i];
}

__global__ void k_copy_f2d(size_t n, const float* x, double* y) {
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) y[i] = double(x[i]);
}

unsigned vec_grid(size_t n) {
    const size_t b = (n + 255) / 256;
    return (unsigned)(b < 1 ? 1 : (b > 4 * 148 ? 4 * 148 : b));
}

}  // namespace

// ---------------------------------------------------------------- launchers
template <typename T>
cudaError_t launch_residual_adjoint(int K, const FrGeom<T>& g, const DevBases<T>& b, const StageAdjArgs<T>& a,
                                    cudaStream_t s) {
    HO2D_ADJ_DISPATCH_K(K, (k_residual_adjoint<KK, T><<<agrid<KK>(g.N), AShape<KK>::THREADS, 0, s>>>(g, b, a)));
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_velocity_adjoint(int K, const FrGeom<T>& g, const DevBases<T>& b, const StageAdjArgs<T>& a,
                                    cudaStream_t s) {
    HO2D_ADJ_DISPATCH_K(K, (k_velocity_adjoint<KK, T><<<agrid<KK>(g.N), AShape<KK>::THREADS, 0, s>>>(g, b, a)));
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_gather(int K, int N, const DevBases<T>& b, const T* dir, const T* sv, const T* sg, T* out,
                          const KrylovScalars* sc, int mode, cudaStream_t s) {
    HO2D_ADJ_DISPATCH_K(K, (k_gather<KK, T><<<agrid<KK>(N), AShape<KK>::THREADS, 0, s>>>(N, b, dir, sv, sg, out, sc,
                                                                                         mode)));
    return cudaGetLastError();
}

template <typename T>
cudaError_t poisson_transpose(int K, const FrGeom<T>& g, const DevBases<T>& b, const T* x, T* y, T* dir, T* sv, T* sg,
                              const KrylovScalars* sc, int mode, cudaStream_t s) {
    HO2D_ADJ_DISPATCH_K(K, (k_poisson_transpose<KK, T><<<agrid<KK>(g.N), AShape<KK>::THREADS, 0, s>>>(
                               g, b, x, dir, sv, sg, sc, mode)));
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return launch_gather<T>(K, g.N, b, dir, sv, sg, y, sc, mode, s);
}

int kt_grid() { return kKtGrid; }

template <typename T>
cudaError_t kt_init(size_t n, const TVectors<T>& v, const TReduce& r, cudaStream_t s) {
    return kt_vec<T>(KT_INIT, n, v, r, 0, s);
}

template <typename T>
cudaError_t kt_iteration_impl(int K, const FrGeom<T>& g, const DevBases<T>& b, const TVectors<T>& v,
                              const TPrecond<T>& pc, const TReduce& r, int max_iter, cudaGraphConditionalHandle h,
                              int has_handle, cudaStream_t s) {
    const int N = g.N;
    const size_t n = (size_t)N * K * K;
    cudaError_t e;
    if ((e = pc_transpose_apply<T>(K, N, pc, v.p, v.ph, v.f0, r.sc, 0, s)) != cudaSuccess) return e;
    if ((e = poisson_transpose<T>(K, g, b, v.ph, v.v, v.dir, v.sv, v.sg, r.sc, 0, s)) != cudaSuccess) return e;
    if ((e = kt_vec<T>(KT_ALPHA, n, v, r, max_iter, s)) != cudaSuccess) return e;
    if ((e = kt_vec<T>(KT_S, n, v, r, max_iter, s)) != cudaSuccess) return e;
    if ((e = pc_transpose_apply<T>(K, N, pc, v.s, v.sh, v.f0, r.sc, 1, s)) != cudaSuccess) return e;
    if ((e = poisson_transpose<T>(K, g, b, v.sh, v.t, v.dir, v.sv, v.sg, r.sc, 1, s)) != cudaSuccess) return e;
    if ((e = kt_vec<T>(KT_OMEGA, n, v, r, max_iter, s)) != cudaSuccess) return e;
    if ((e = kt_vec<T>(KT_XR, n, v, r, max_iter, s, nullptr, nullptr, nullptr, h, has_handle)) != cudaSuccess)
        return e;
    return kt_vec<T>(KT_P, n, v, r, max_iter, s);
}

template <typename T>
cudaError_t kt_iteration(int K, const FrGeom<T>& g, const DevBases<T>& b, const TVectors<T>& v, const TPrecond<T>& pc,
                         const TReduce& r, int max_iter, cudaStream_t s) {
    return kt_iteration_impl<T>(K, g, b, v, pc, r, max_iter, cudaGraphConditionalHandle(), 0, s);
}

// A whole solve as a CUDA graph: init, then a while node whose body is one iteration.
template <typename T>
cudaError_t kt_capture_solve(int K, const FrGeom<T>& g, const DevBases<T>& b, const TVectors<T>& v,
                             const TPrecond<T>& pc, const TReduce& r, int max_iter, cudaStream_t s,
                             cudaGraph_t* graph_out) {
    const size_t n = (size_t)g.N * K * K;
    cudaGraph_t gr = nullptr;
    cudaError_t e = cudaGraphCreate(&gr, 0);
    if (e != cudaSuccess) return e;
    cudaGraphConditionalHandle h;
    if ((e = cudaGraphConditionalHandleCreate(&h, gr, 0, 0)) != cudaSuccess) return e;
    if ((e = cudaStreamBeginCaptureToGraph(s, gr, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal)) !=
        cudaSuccess)
        return e;
    kt_vec<T>(KT_INIT, n, v, r, max_iter, s);
    k_kt_set_loop<<<1, 1, 0, s>>>(r.sc, h);
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
    if ((e = cudaStreamEndCapture(s, &gr)) != cudaSuccess) return e;
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    if ((e = cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal)) !=
        cudaSuccess)
        return e;
    kt_iteration_impl<T>(K, g, b, v, pc, r, max_iter, h, 1, s);
    if ((e = cudaStreamEndCapture(s, &body)) != cudaSuccess) return e;
    *graph_out = gr;
    return cudaGetLastError();
}

template <typename T>
int kt_launches_per_iteration(const TPrecond<T>& pc) {
    const int pcl = (pc.pc.nlev > 0 ? 1 + coarse_vec_launches(pc.pc) : 0) + 1;
    return 2 * pcl + 2 * 2 + 5;
}

template <typename T>
cudaError_t kt_residual(size_t n, const T* b, const T* y, T* r, const TReduce& rr, cudaStream_t s) {
    TVectors<T> v{};
    return kt_vec<T>(KT_RES, n, v, rr, 0, s, b, y, r);
}

cudaError_t launch_axpby(size_t n, double* out, double a, const double* x, double c, const double* y, cudaStream_t s) {
    k_axpby<<<vec_grid(n), 256, 0, s>>>(n, out, a, x, c, y);
    return cudaGetLastError();
}

cudaError_t launch_sub_scaled(size_t n, double* out, const double* x, const double* J, const double* mu,
                              cudaStream_t s) {
    k_sub_scaled<<<vec_grid(n), 256, 0, s>>>(n, out, x, J, mu);
    return cudaGetLastError();
}

cudaError_t launch_copy_f2d(const float* x, double* y, size_t n, cudaStream_t s) {
    k_copy_f2d<<<vec_grid(n), 256, 0, s>>>(n, x, y);
    return cudaGetLastError();
}

template cudaError_t launch_residual_adjoint<double>(int, const FrGeom<double>&, const DevBases<double>&,
                                                     const StageAdjArgs<double>&, cudaStream_t);
template cudaError_t launch_velocity_adjoint<double>(int, const FrGeom<double>&, const DevBases<double>&,
                                                     const StageAdjArgs<double>&, cudaStream_t);

#define HO2D_INSTANTIATE_ADJ(T)                                                                                  \
    template cudaError_t launch_gather<T>(int, int, const DevBases<T>&, const T*, const T*, const T*, T*,         \
                                          const KrylovScalars*, int, cudaStream_t);                              \
    template cudaError_t poisson_transpose<T>(int, const FrGeom<T>&, const DevBases<T>&, const T*, T*, T*, T*, T*, \
                                              const KrylovScalars*, int, cudaStream_t);                          \
    template cudaError_t kt_init<T>(size_t, const TVectors<T>&, const TReduce&, cudaStream_t);                  \
    template cudaError_t kt_iteration<T>(int, const FrGeom<T>&, const DevBases<T>&, const TVectors<T>&,          \
                                         const TPrecond<T>&, const TReduce&, int, cudaStream_t);                 \
    template int kt_launches_per_iteration<T>(const TPrecond<T>&);                                               \
    template cudaError_t kt_capture_solve<T>(int, const FrGeom<T>&, const DevBases<T>&, const TVectors<T>&,      \
                                             const TPrecond<T>&, const TReduce&, int, cudaStream_t, cudaGraph_t*);  \
    template cudaError_t kt_residual<T>(size_t, const T*, const T*, T*, const TReduce&, cudaStream_t);

HO2D_INSTANTIATE_ADJ(double)
HO2D_INSTANTIATE_ADJ(float)

}  // namespace ho2d
