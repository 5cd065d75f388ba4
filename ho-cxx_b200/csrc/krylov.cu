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

// Shared-memory working set of one CTA (EPB elements) for the operator.
template <int K, typename T>
struct MfShared {
    static constexpr int K2 = K * K, NF = 4 * K, EPB = Shape<K>::EPB;
    T x[EPB][K2], a[EPB][K2], b[EPB][K2];
    // own face: traces (recomputed) and metrics; neighbour face: traces and metrics
    T tv[EPB][NF], tg[EPB][NF], fA[EPB][NF], fB[EPB][NF], fJ[EPB][NF];
    T ntv[EPB][NF], ntg[EPB][NF], nfA[EPB][NF], nfB[EPB][NF], nfJ[EPB][NF];
    T com[EPB][NF], cg[EPB][NF], fb[EPB][NF];
    int nb[EPB][4], nijp[EPB][4];  // neighbour element / its face; boundary: -1 - switch
    DevBases<T> bas;               // basis tables staged from the parameter bank
};

// y = A x at (el, ij) for the homogeneous-boundary Poisson operator: the method-2 FR
// Laplacian of fr_device.cuh's lap_element, restaged so that all global data arrive in
// two rounds (own data and connectivity, then the neighbours' face data) and every
// later phase synchronises through shared memory only. Collective.
template <int K, typename T>
__device__ T mf_apply(const MfOp<T>& op, const T* __restrict__ x, const T* __restrict__ tv, const T* __restrict__ tg,
                      MfShared<K, T>& sm, bool active, int le, int el, int ij) {
    constexpr int K2 = K * K, NF = 4 * K, EPB = Shape<K>::EPB;
    const FrGeom<T>& g = op.g;
    stage_bases(sm.bas, op.b);
    const DevBases<T>& b = sm.bas;
    const int j = ij / K, i = ij % K;
    // round 1: x, volume metrics, connectivity
    T xx = T(0), xe = T(0), yx = T(0), ye = T(0), J = T(1);
    if (active) {
        const int p = el * K2 + ij;
        sm.x[le][ij] = x[p];
        xx = g.xxi[p]; xe = g.xeta[p]; yx = g.yxi[p]; ye = g.yeta[p]; J = g.J[p];
    }
    for (int f = threadIdx.x; f < EPB * 4; f += blockDim.x) {
        const int l = f / 4, face = f % 4, e2 = blockIdx.x * EPB + l;
        if (e2 < g.N) {
            const int nb = g.face_nb[e2 * 4 + face];
            sm.nb[l][face] = nb >= 0 ? nb : -1 - g.sw_p[-nb - 1];
            sm.nijp[l][face] = g.face_nijp[e2 * 4 + face];
        }
    }
    __syncthreads();
    // round 2: own face metrics and traces, the neighbours' traces and face metrics
    if (active)
        for (int o = ij; o < NF; o += K2) {
            const int ijp = o / K, k = o % K;
            const int q = (el * 4 + ijp) * K + k;
            sm.fA[le][o] = g.fA[q];
            sm.fB[le][o] = g.fB[q];
            sm.fJ[le][o] = g.fJ[q];
            face_trace<K, T>(sm.x[le], b, o, sm.tv[le][o], sm.tg[le][o]);
            const int nb = sm.nb[le][ijp];
            if (nb >= 0) {
                const int nijp = sm.nijp[le][ijp];
                const int rev = (ijp + nijp - ijp / 2 - nijp / 2 + 1) % 2;
                const int nq = (nb * 4 + nijp) * K + (rev ? K - 1 - k : k);
                sm.ntv[le][o] = tv[nq];
                sm.ntg[le][o] = tg[nq];
                sm.nfA[le][o] = g.fA[nq];
                sm.nfB[le][o] = g.fB[nq];
                sm.nfJ[le][o] = g.fJ[nq];
            }
        }
    __syncthreads();
    // common values: average inside, 0 on Dirichlet faces (homogeneous), Neumann below
    if (active)
        for (int o = ij; o < NF; o += K2) {
            const int nb = sm.nb[le][o / K];
            sm.com[le][o] = nb >= 0 ? T(0.5) * (sm.tv[le][o] + sm.ntv[le][o]) : T(0);
        }
    __syncthreads();
    // homogeneous Neumann faces: K x K system for the common value (src/HO_2D.cpp:2899-2924)
    for (int ijp = ij; active && ijp < 4; ijp += K2) {
        if (sm.nb[le][ijp] != -1 - kNeumann) continue;
        const int lr = ijp & 1;
        T M[K][K], r[K], xs[K];
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const int o = ijp * K + k;
            r[k] = -sm.fA[le][o] * (sm.tg[le][o] - sm.tv[le][o] * b.gp[lr]);
#pragma unroll
            for (int c = 0; c < K; ++c) M[k][c] = -sm.fB[le][o] * b.D[c * K + k];
            M[k][k] += sm.fA[le][o] * b.gp[lr];
        }
#pragma unroll
        for (int c = 0; c < K - 1; ++c)
#pragma unroll
            for (int r2 = c + 1; r2 < K; ++r2) {
                const T fct = M[r2][c] / M[c][c];
                r[r2] -= fct * r[c];
#pragma unroll
                for (int cc = c + 1; cc < K; ++cc) M[r2][cc] -= fct * M[c][cc];
            }
#pragma unroll
        for (int r2 = K - 1; r2 >= 0; --r2) {
            T acc = T(0);
#pragma unroll
            for (int cc = r2 + 1; cc < K; ++cc) acc += M[r2][cc] * xs[cc];
            xs[r2] = (r[r2] - acc) / M[r2][r2];
        }
#pragma unroll
        for (int k = 0; k < K; ++k) sm.com[le][ijp * K + k] = xs[k];
    }
    __syncthreads();
    // corrected normal fluxes, averaged with the neighbour's on interior faces
    if (active)
        for (int o = ij; o < NF; o += K2) {
            const int ijp = o / K, k = o % K, lr = ijp & 1;
            const int nb = sm.nb[le][ijp];
            if (nb == -1 - kNeumann) {
                sm.cg[le][o] = T(0);
                continue;
            }
            const T com = sm.com[le][o];
            T cross = T(0);
#pragma unroll
            for (int m = 0; m < K; ++m) cross += sm.com[le][ijp * K + m] * b.D[m * K + k];
            const T dv = sm.tg[le][o] + (com - sm.tv[le][o]) * b.gp[lr];
            const T fl = (dv * sm.fA[le][o] - cross * sm.fB[le][o]) / sm.fJ[le][o];
            if (nb < 0) {
                sm.cg[le][o] = fl;
            } else {
                const int nijp = sm.nijp[le][ijp];
                const int rev = (ijp + nijp - ijp / 2 - nijp / 2 + 1) % 2;
                const int jn = rev ? K - 1 - k : k;
                T crn = T(0);
#pragma unroll
                for (int m = 0; m < K; ++m) crn += sm.com[le][ijp * K + (rev ? K - 1 - m : m)] * b.D[m * K + jn];
                const T dvn = sm.ntg[le][o] + (com - sm.ntv[le][o]) * b.gp[nijp & 1];
                const T fln = (dvn * sm.nfA[le][o] - crn * sm.nfB[le][o]) / sm.nfJ[le][o];
                sm.cg[le][o] = T(0.5) * (fl + T(2 * ((ijp + nijp) % 2) - 1) * fln);
            }
        }
    __syncthreads();
    // contravariant gradient (src/HO_2D.cpp:2775-2792)
    T ft = T(0), gt = T(0);
    if (active) {
        T dx = T(0), de = T(0);
#pragma unroll
        for (int d = 0; d < K; ++d) {
            dx += sm.x[le][j * K + d] * b.D[d * K + i];
            de += sm.x[le][d * K + i] * b.D[d * K + j];
        }
        dx += (sm.com[le][0 * K + j] - sm.tv[le][0 * K + j]) * b.gR[i * 2 + 0];
        dx += (sm.com[le][1 * K + j] - sm.tv[le][1 * K + j]) * b.gR[i * 2 + 1];
        de += (sm.com[le][2 * K + i] - sm.tv[le][2 * K + i]) * b.gR[j * 2 + 0];
        de += (sm.com[le][3 * K + i] - sm.tv[le][3 * K + i]) * b.gR[j * 2 + 1];
        ft = (dx * (xe * xe + ye * ye) - de * (xx * xe + yx * ye)) / J;
        gt = (de * (xx * xx + yx * yx) - dx * (xx * xe + yx * ye)) / J;
        sm.a[le][ij] = ft;
        sm.b[le][ij] = gt;
    }
    __syncthreads();
    if (active)
        for (int o = ij; o < NF; o += K2) {
            const int ijp = o / K, k = o % K, lr = ijp & 1;
            T v = sm.cg[le][o];
            if (ijp < 2) {
#pragma unroll
                for (int d = 0; d < K; ++d) v -= sm.a[le][k * K + d] * b.sbb[d * 2 + lr];
            } else {
#pragma unroll
                for (int d = 0; d < K; ++d) v -= sm.b[le][d * K + k] * b.sbb[d * 2 + lr];
            }
            sm.fb[le][o] = v;
        }
    __syncthreads();
    if (!active) return T(0);
    T lap = T(0);
#pragma unroll
    for (int d = 0; d < K; ++d) lap += sm.a[le][j * K + d] * b.D[d * K + i];
    lap += sm.fb[le][0 * K + j] * b.gR[i * 2 + 0] + sm.fb[le][1 * K + j] * b.gR[i * 2 + 1];
#pragma unroll
    for (int d = 0; d < K; ++d) lap += sm.b[le][d * K + i] * b.D[d * K + j];
    lap += sm.fb[le][2 * K + i] * b.gR[j * 2 + 0] + sm.fb[le][3 * K + i] * b.gR[j * 2 + 1];
    return lap;
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
    __shared__ DevBases<T> sbas;
    stage_bases(sbas, op.b);
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
    emit_traces<K, T>(sz[active ? le : 0], sbas, v.tv, v.tg, active, el, ij);
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
    __shared__ DevBases<T> sbas;
    stage_bases(sbas, op.b);
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
    emit_traces<K, T>(sz[active ? le : 0], sbas, tv, tg, active, el, ij);
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
    __shared__ DevBases<T> sbas;
    stage_bases(sbas, op.b);
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
        emit_traces<K, T>(sz[active ? le : 0], sbas, v.tv, v.tg, active, el, ij);
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

// same, and sets the condition of the graph's while node: iterate while not done. Every
// body execution either increments `it` (capped at max_iter by k_xr_update) or finds
// `done` set, so the device-side loop always ends.
__global__ void k_finish_loop(KrylovScalars* sc, cudaGraphConditionalHandle h) {
    if (!sc->done && sc->s_exit) sc->done = 1;
    cudaGraphSetConditional(h, sc->done ? 0u : 1u);
}

__global__ void k_set_loop(const KrylovScalars* sc, cudaGraphConditionalHandle h) {
    cudaGraphSetConditional(h, sc->done ? 0u : 1u);
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

// pre-smoothing from zero and residual in one pass: t = f - A (m .* f)
template <typename T>
__global__ void k_c_pre(DevCsr<T> A, const T* __restrict__ m, const T* __restrict__ f, T* __restrict__ t,
                        const KrylovScalars* sc, int mode) {
    if (pc_skip(sc, mode)) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.n) return;
    T acc = T(0);
    for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k) {
        const int j = A.col[k];
        acc += A.val[k] * (m[j] * f[j]);
    }
    t[i] = f[i] - acc;
}

template <typename T>
__global__ void k_c_spmv(DevCsr<T> M, const T* __restrict__ x, T* __restrict__ y, const KrylovScalars* sc,
                         int mode) {
    if (pc_skip(sc, mode)) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < M.n) y[i] = csr_row<T>(M, x, i);
}

// coarse-grid correction and post-smoothing in one pass:
// u' = m .* f + P uc (recomputed per use), u2 = u' + m .* (f - A u')
template <typename T>
__global__ void k_c_post(DevCsr<T> A, DevCsr<T> P, const T* __restrict__ m, const T* __restrict__ f,
                         const T* __restrict__ uc, T* __restrict__ u2, const KrylovScalars* sc, int mode) {
    if (pc_skip(sc, mode)) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.n) return;
    T acc = T(0), ui = T(0);
    for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k) {
        const int j = A.col[k];
        const T uj = m[j] * f[j] + csr_row<T>(P, uc, j);
        acc += A.val[k] * uj;
        if (j == i) ui = uj;
    }
    if (A.ptr[i] == A.ptr[i + 1] || ui == T(0)) ui = m[i] * f[i] + csr_row<T>(P, uc, i);
    u2[i] = ui + m[i] * (f[i] - acc);
}

// coarsest level: u = inv f with the inverse stored column-major (coalesced reads)
template <typename T>
__global__ void k_c_dense(int n, const T* __restrict__ inv_t, const T* __restrict__ f, T* __restrict__ u,
                          const KrylovScalars* sc, int mode) {
    if (pc_skip(sc, mode)) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    T acc = T(0);
    for (int j = 0; j < n; ++j) acc += inv_t[(size_t)j * n + i] * f[j];
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
    const int epb = (256 / k2) > 32 ? 32 : ((256 / k2) > 0 ? 256 / k2 : 1);
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
    k_c_pre<T><<<g, 128, 0, s>>>(L.A, L.m, L.f, L.t, sc, mode);
    k_c_spmv<T><<<(unsigned)((C.n + 127) / 128), 128, 0, s>>>(L.R, L.t, C.f, sc, mode);
    coarse_cycle(pc, l + 1, sc, mode, s);
    k_c_post<T><<<g, 128, 0, s>>>(L.A, L.P, L.m, L.f, C.out, L.u2, sc, mode);
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
    const int coarse = 3 * (pc.nlev - 1) + 1;
    return 6 + 2 * (coarse + 1);
}

template <typename T>
cudaError_t krylov_iteration(const MfOp<T>& op, const BicgVectors<T>& v, const ReduceScratch& rs, int max_iter,
                             const Precond<T>& pc, cudaStream_t s) {
    HO2D_KSWITCH(op.K, (iteration_impl<KK, T>(op, v, rs, max_iter, pc, s)));
    k_finish_s_exit<<<1, 1, 0, s>>>(rs.sc);
    return cudaGetLastError();
}

// Captures a whole solve into `*graph_out`: initial residual, then a while node whose body
// is one BiCGSTAB iteration; the loop condition lives on the device, so a solve is one
// graph launch with no host round trip.
template <typename T>
cudaError_t krylov_capture_solve(const MfOp<T>& op, const BicgVectors<T>& v, const ReduceScratch& rs, double tol,
                                 int max_iter, const Precond<T>& pc, cudaStream_t s, cudaGraph_t* graph_out) {
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaGraphCreate(&g, 0);
    if (e != cudaSuccess) return e;
    cudaGraphConditionalHandle h;
    if ((e = cudaGraphConditionalHandleCreate(&h, g, 0, 0)) != cudaSuccess) return e;
    if ((e = cudaStreamBeginCaptureToGraph(s, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal)) !=
        cudaSuccess)
        return e;
    krylov_init<T>(op, v, rs, tol, s);
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
    HO2D_KSWITCH(op.K, (iteration_impl<KK, T>(op, v, rs, max_iter, pc, s)));
    k_finish_loop<<<1, 1, 0, s>>>(rs.sc, h);
    if ((e = cudaStreamEndCapture(s, &body)) != cudaSuccess) return e;
    *graph_out = g;
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
    template cudaError_t krylov_capture_solve<T>(const MfOp<T>&, const BicgVectors<T>&, const ReduceScratch&,     \
                                                 double, int, const Precond<T>&, cudaStream_t, cudaGraph_t*);     \
    template cudaError_t mf_residual<T>(const MfOp<T>&, const double*, const T*, T*, T*, double*,                 \
                                        const ReduceScratch&, cudaStream_t);                                      \
    template cudaError_t mf_apply_op<T>(const MfOp<T>&, const T*, T*, T*, T*, cudaStream_t);                      \
    template cudaError_t mf_apply_only<T>(const MfOp<T>&, const T*, const T*, const T*, T*, int, cudaStream_t);

HO2D_INSTANTIATE_KRYLOV(double)
HO2D_INSTANTIATE_KRYLOV(float)

}  // namespace ho2d
