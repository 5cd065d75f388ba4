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

// Shared-memory working set of one CTA (EPB elements) for the operator.
template <int K, typename T>
struct MfShared {
    static constexpr int K2 = K * K, NF = 4 * K, EPB = Shape<K>::EPB;
    T x[EPB][K2], a[EPB][K2], b[EPB][K2];
    T tv[EPB][NF], tg[EPB][NF];    // own traces, recomputed from x
    T ntv[EPB][NF], ntg[EPB][NF];  // incoming traces of the neighbours
    T fa[EPB][NF], fb[EPB][NF], nfa[EPB][NF], nfb[EPB][NF];
    T com[EPB][NF], cg[EPB][NF];   // common values; common normal fluxes (then their jumps)
    int code[EPB][4];
    DevBases<T> bas;               // basis tables staged from the parameter bank
};

// y = A x at (el, ij) for the homogeneous-boundary Poisson operator: the method-2 FR
// Laplacian of fr_device.cuh's lap_element. Every global read is one of the element's
// own rows (its x, metric coefficients, face coefficients and incoming traces), so all
// of them are issued in a single round; five barrier phases follow. Collective.
template <int K, typename T>
__device__ T mf_apply_gen(const MfOp<T>& op, const T* __restrict__ x, const T* __restrict__ tv,
                          const T* __restrict__ tg, MfShared<K, T>& sm, bool active, int le, int el, int ij) {
    constexpr int K2 = K * K, NF = 4 * K;
    const PoisGeom<T>& g = op.g;
    const int j = ij / K, i = ij % K;
    // round of loads: everything is indexed by this element only
    T g11 = T(0), g12 = T(0), g22 = T(0);
    if (active) {
        const int p = el * K2 + ij;
        sm.x[le][ij] = x[p];
        g11 = g.G11[p];
        g12 = g.G12[p];
        g22 = g.G22[p];
        for (int o = ij; o < NF; o += K2) {
            const int q = el * NF + o;
            sm.fa[le][o] = g.fa[q];
            sm.fb[le][o] = g.fb[q];
            sm.nfa[le][o] = g.nfa[q];
            sm.nfb[le][o] = g.nfb[q];
            sm.ntv[le][o] = tv[q];
            sm.ntg[le][o] = tg[q];
        }
        for (int c = ij; c < 4; c += K2) sm.code[le][c] = g.code[el * 4 + c];
    }
    stage_bases(sm.bas, op.b);
    __syncthreads();
    const DevBases<T>& b = sm.bas;
    // own traces; common values on interior (average) and Dirichlet (zero) faces
    if (active)
        for (int o = ij; o < NF; o += K2) {
            T v, d;
            face_trace<K, T>(sm.x[le], b, o, v, d);
            sm.tv[le][o] = v;
            sm.tg[le][o] = d;
            sm.com[le][o] = sm.code[le][o / K] >= 0 ? T(0.5) * (v + sm.ntv[le][o]) : T(0);
        }
    __syncthreads();
    // homogeneous Neumann faces: com = Minv r with r_m = -fa_m (tg_m - tv_m g'(+-1)), the
    // K x K common-value system of src/HO_2D.cpp:2899-2924 inverted once at setup
    if (active)
        for (int o = ij; o < NF; o += K2) {
            const int ijp = o / K, k = o % K, c = sm.code[le][ijp];
            if (c > -2) continue;
            const T gp = b.gp[ijp & 1];
            const T* mi = g.minv + ((size_t)(-2 - c) * K + k) * K;
            T acc = T(0);
#pragma unroll
            for (int m = 0; m < K; ++m) {
                const int om = ijp * K + m;
                acc -= mi[m] * sm.fa[le][om] * (sm.tg[le][om] - sm.tv[le][om] * gp);
            }
            sm.com[le][o] = acc;
        }
    __syncthreads();
    // contravariant gradient (src/HO_2D.cpp:2775-2792) and common normal fluxes
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
        sm.a[le][ij] = dx * g11 + de * g12;
        sm.b[le][ij] = de * g22 + dx * g12;
        for (int o = ij; o < NF; o += K2) {
            const int ijp = o / K, k = o % K, c = sm.code[le][ijp];
            if (c <= -2) {
                sm.cg[le][o] = T(0);
                continue;
            }
            const T com = sm.com[le][o];
            T cross = T(0);
#pragma unroll
            for (int m = 0; m < K; ++m) cross += sm.com[le][ijp * K + m] * b.D[m * K + k];
            const T dv = sm.tg[le][o] + (com - sm.tv[le][o]) * b.gp[ijp & 1];
            const T fl = dv * sm.fa[le][o] - cross * sm.fb[le][o];
            if (c < 0) {
                sm.cg[le][o] = fl;
            } else {
                const int nijp = c & 3, rev = c >> 2;
                const int jn = rev ? K - 1 - k : k;
                T crn = T(0);
#pragma unroll
                for (int m = 0; m < K; ++m) crn += sm.com[le][ijp * K + (rev ? K - 1 - m : m)] * b.D[m * K + jn];
                const T dvn = sm.ntg[le][o] + (com - sm.ntv[le][o]) * b.gp[nijp & 1];
                const T fln = dvn * sm.nfa[le][o] - crn * sm.nfb[le][o];
                sm.cg[le][o] = T(0.5) * (fl + T(2 * ((ijp + nijp) % 2) - 1) * fln);
            }
        }
    }
    __syncthreads();
    // flux jumps: common flux minus the interior flux extrapolated to the face
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
            sm.cg[le][o] = v;
        }
    __syncthreads();
    if (!active) return T(0);
    T lap = T(0);
#pragma unroll
    for (int d = 0; d < K; ++d) lap += sm.a[le][j * K + d] * b.D[d * K + i];
    lap += sm.cg[le][0 * K + j] * b.gR[i * 2 + 0] + sm.cg[le][1 * K + j] * b.gR[i * 2 + 1];
#pragma unroll
    for (int d = 0; d < K; ++d) lap += sm.b[le][d * K + i] * b.D[d * K + j];
    lap += sm.cg[le][2 * K + i] * b.gR[j * 2 + 0] + sm.cg[le][3 * K + i] * b.gR[j * 2 + 1];
    return lap;
}

// mf_apply for K >= 4, where every face point has a thread of its own (4K <= K^2): the
// basis values a thread uses (its row and column of D, its Radau derivatives, the
// extrapolation weights of its face point) and its face point's own data stay in
// registers, and shared memory carries only what other threads read. Same arithmetic,
// same order of operations as mf_apply. Collective.
template <int K, typename T>
__device__ T mf_apply_1f(const MfOp<T>& op, const T* __restrict__ x, const T* __restrict__ tv, const T* __restrict__ tg,
                         MfShared<K, T>& sm, bool active, int le, int el, int ij) {
    constexpr int K2 = K * K, NF = 4 * K;
    static_assert(NF <= K2, "one face point per thread");
    const PoisGeom<T>& g = op.g;
    const int j = ij / K, i = ij % K;
    const bool face = active && ij < NF;
    const int ijp = ij / K, k = ij % K, lr = ijp & 1;  // this thread's face point (if face)
    T g11 = T(0), g12 = T(0), g22 = T(0);
    T fa = T(0), fb = T(0), nfa = T(0), nfb = T(0), ntv = T(0), ntg = T(0);
    if (active) {
        const int p = el * K2 + ij;
        sm.x[le][ij] = x[p];
        g11 = g.G11[p];
        g12 = g.G12[p];
        g22 = g.G22[p];
        if (face) {
            const int q = el * NF + ij;
            fa = g.fa[q];
            fb = g.fb[q];
            nfa = g.nfa[q];
            nfb = g.nfb[q];
            ntv = tv[q];
            ntg = tg[q];
            sm.fa[le][ij] = fa;
        }
        if (ij < 4) sm.code[le][ij] = g.code[el * 4 + ij];
    }
    stage_bases(sm.bas, op.b);
    __syncthreads();
    const DevBases<T>& b = sm.bas;
    T Di[K], Dj[K];
#pragma unroll
    for (int d = 0; d < K; ++d) {
        Di[d] = b.D[d * K + i];
        Dj[d] = b.D[d * K + j];
    }
    const T gRi0 = b.gR[i * 2 + 0], gRi1 = b.gR[i * 2 + 1], gRj0 = b.gR[j * 2 + 0], gRj1 = b.gR[j * 2 + 1];
    const int c = face ? sm.code[le][ijp] : -1;
    // own trace and common value (interior: average; Dirichlet: zero)
    T tvv = T(0), tgv = T(0);
    if (face) {
        face_trace<K, T>(sm.x[le], b, ij, tvv, tgv);
        sm.tv[le][ij] = tvv;
        sm.tg[le][ij] = tgv;
        sm.com[le][ij] = c >= 0 ? T(0.5) * (tvv + ntv) : T(0);
    }
    __syncthreads();
    // homogeneous Neumann faces: com = Minv r, r_m = -fa_m (tg_m - tv_m g'(+-1))
    if (face && c <= -2) {
        const T gp = b.gp[lr];
        const T* mi = g.minv + ((size_t)(-2 - c) * K + k) * K;
        T acc = T(0);
#pragma unroll
        for (int m = 0; m < K; ++m) {
            const int om = ijp * K + m;
            acc -= mi[m] * sm.fa[le][om] * (sm.tg[le][om] - sm.tv[le][om] * gp);
        }
        sm.com[le][ij] = acc;
    }
    __syncthreads();
    // contravariant gradient and this face point's common normal flux (kept in a register)
    T cg = T(0);
    if (active) {
        T dx = T(0), de = T(0);
#pragma unroll
        for (int d = 0; d < K; ++d) {
            dx += sm.x[le][j * K + d] * Di[d];
            de += sm.x[le][d * K + i] * Dj[d];
        }
        dx += (sm.com[le][0 * K + j] - sm.tv[le][0 * K + j]) * gRi0;
        dx += (sm.com[le][1 * K + j] - sm.tv[le][1 * K + j]) * gRi1;
        de += (sm.com[le][2 * K + i] - sm.tv[le][2 * K + i]) * gRj0;
        de += (sm.com[le][3 * K + i] - sm.tv[le][3 * K + i]) * gRj1;
        sm.a[le][ij] = dx * g11 + de * g12;
        sm.b[le][ij] = de * g22 + dx * g12;
        if (face && c > -2) {
            const T com = sm.com[le][ij];
            T cross = T(0);
#pragma unroll
            for (int m = 0; m < K; ++m) cross += sm.com[le][ijp * K + m] * b.D[m * K + k];
            const T dv = tgv + (com - tvv) * b.gp[lr];
            const T fl = dv * fa - cross * fb;
            if (c < 0) {
                cg = fl;
            } else {
                const int nijp = c & 3, rev = c >> 2;
                const int jn = rev ? K - 1 - k : k;
                T crn = T(0);
#pragma unroll
                for (int m = 0; m < K; ++m) crn += sm.com[le][ijp * K + (rev ? K - 1 - m : m)] * b.D[m * K + jn];
                const T dvn = ntg + (com - ntv) * b.gp[nijp & 1];
                const T fln = dvn * nfa - crn * nfb;
                cg = T(0.5) * (fl + T(2 * ((ijp + nijp) % 2) - 1) * fln);
            }
        }
    }
    __syncthreads();
    // flux jump at this face point: common flux minus the interior flux extrapolated to it
    if (face) {
        T v = cg;
        if (ijp < 2) {
#pragma unroll
            for (int d = 0; d < K; ++d) v -= sm.a[le][k * K + d] * b.sbb[d * 2 + lr];
        } else {
#pragma unroll
            for (int d = 0; d < K; ++d) v -= sm.b[le][d * K + k] * b.sbb[d * 2 + lr];
        }
        sm.cg[le][ij] = v;
    }
    __syncthreads();
    if (!active) return T(0);
    T lap = T(0);
#pragma unroll
    for (int d = 0; d < K; ++d) lap += sm.a[le][j * K + d] * Di[d];
    lap += sm.cg[le][0 * K + j] * gRi0 + sm.cg[le][1 * K + j] * gRi1;
#pragma unroll
    for (int d = 0; d < K; ++d) lap += sm.b[le][d * K + i] * Dj[d];
    lap += sm.cg[le][2 * K + i] * gRj0 + sm.cg[le][3 * K + i] * gRj1;
    return lap;
}

// y = A x at (el, ij): the register-resident form when every face point has its own
// thread (K >= 4), the general form otherwise. Collective.
template <int K, typename T>
__device__ __forceinline__ T mf_apply(const MfOp<T>& op, const T* __restrict__ x, const T* __restrict__ tv,
                                      const T* __restrict__ tg, MfShared<K, T>& sm, bool active, int le, int el,
                                      int ij) {
    if constexpr (4 * K <= K * K) return mf_apply_1f<K, T>(op, x, tv, tg, sm, active, le, el, ij);
    else return mf_apply_gen<K, T>(op, x, tv, tg, sm, active, le, el, ij);
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

// Element sums of a per-point value: every thread of element le stores its value, then
// thread ij == 0 of each element adds the K^2 values in a fixed order. Collective.
template <int K, typename T>
__device__ __forceinline__ void element_sum(T (&buf)[Shape<K>::EPB][Shape<K>::K2], T val, bool active, int le, int ij,
                                            int el, T* out) {
    __syncthreads();  // buf may still be read by the phase before
    if (active) buf[le][ij] = val;
    __syncthreads();
    if (active && ij == 0) {
        T sum = T(0);
#pragma unroll
        for (int q = 0; q < Shape<K>::K2; ++q) sum += buf[le][q];
        out[el] = sum;
    }
}

}  // namespace

// ---------------------------------------------------------------- fine-level kernels
// incoming face traces of x (the operand of an operator application that no Krylov
// kernel produced: the initial guess, a refinement iterate, a caller's vector)
template <int K, typename T>
__global__ void __launch_bounds__(Shape<K>::THREADS) k_trace_in(MfOp<T> op, const T* __restrict__ x, T* __restrict__ tv,
                                                                 T* __restrict__ tg) {
    using S = Shape<K>;
    __shared__ T sx[S::EPB][S::K2];
    __shared__ DevBases<T> sbas;
    const int le = threadIdx.x / S::K2, ij = threadIdx.x % S::K2;
    const int el = blockIdx.x * S::EPB + le;
    const bool active = le < S::EPB && el < op.g.N;
    TraceDst<K> td;
    td.load(op.g.scat, active, el, ij);
    if (active) sx[le][ij] = x[el * S::K2 + ij];
    stage_bases(sbas, op.b);
    __syncthreads();
    emit_traces<K, T>(sx[active ? le : 0], sbas, td, tv, tg, ij);
}


// r = b - A x (x's traces in xtv/xtg), rhat = r; ||r||^2, ||b||^2
template <int K, typename T>
__global__ void __launch_bounds__(Shape<K>::THREADS) k_mf_init(MfOp<T> op, BicgVectors<T> v, ReduceScratch rs) {
    using S = Shape<K>;
    __shared__ MfShared<K, T> sm;
    const int le = threadIdx.x / S::K2, ij = threadIdx.x % S::K2;
    const int el = blockIdx.x * S::EPB + le;
    const bool active = le < S::EPB && el < op.g.N;
    const T y = mf_apply<K, T>(op, v.x, v.xtv, v.xtg, sm, active, le, el, ij);
    double part[2] = {0.0, 0.0};
    T r = T(0);
    if (active) {
        const int p = el * S::K2 + ij;
        const T bb = v.b[p];
        r = bb - y;
        v.r[p] = r;
        v.rhat[p] = r;
        part[0] = double(r) * double(r);
        part[1] = double(bb) * double(bb);
    }
    element_sum<K, T>(sm.a, r, active, le, ij, el, v.er);
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

// Vector kernels take kVecTiles element tiles per CTA (tile blockIdx.x + t * gridDim.x),
// so the whole vector is covered in one wave of CTAs, and every thread issues its loads
// before it reads the solve's `done` flag: the addresses are valid whatever the flag
// says, so the flag's round trip overlaps the data loads.
constexpr int kVecTiles = 2;

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
// elements the fit does not approximate well (FP32 smoother). For BS 0 and 1, whether
// k_mf_post stages its CTA's inverse blocks (EPB x K^4 values, contiguous in memory) in
// shared memory: when they fit in 32 KB of static shared memory.
template <int K, typename T, int BS = 0>
struct PostStage {
    using DT = typename std::conditional<BS == 1, unsigned short, T>::type;
    static constexpr int K4 = K * K * K * K;
    static constexpr size_t kBytes = (size_t)Shape<K>::EPB * K4 * sizeof(DT) + 32;  // + 16-byte alignment slack
    static constexpr bool kOn = BS != 2 && kBytes <= 32768;
    static constexpr int KF = 4 * K * K + 2 * K;  // Kronecker factors per element (BS 2)
    static constexpr int KE = BS == 2 ? Shape<K>::EPB : 1;
};

__device__ __forceinline__ float block_value(unsigned short b) { return __uint_as_float((unsigned)b << 16); }
template <typename T>
__device__ __forceinline__ T block_value(T v) {
    return v;
}

// Preconditioner application, with the BiCGSTAB vector update that produces its operand:
//   mode 0:  p = r + beta (p - omega v)  (p = r on the first iteration),  f = p -> ph
//   mode 1:  s = r - alpha v, ||s||^2 (s_exit test),                      f = s -> sh
// then the two-level smoothing step z = e + w D^{-1} (f - A e), e = P u0 element-wise
// constant, with z's face traces. u0 of the element and of its four face neighbours comes
// straight from the coarse cycle (one-level hierarchy), or from the level-0 up step
// u0 = S0 f0 + Q0 u1 evaluated here as 25 partial sums (five per slot) spread over the
// element's threads, or is zero (block-Jacobi, no coarse level). Mode 0 also stores the
// element sums of the new p for the next iteration. Everything that does not depend on u0
// starts first: the CTA's inverse blocks are copied into shared memory asynchronously
// (cp.async, 16-byte pieces of the 16-byte-aligned superset of the blocks; the buffer is
// padded past its end), and the block row sums and the vectors are loaded, so all of it
// overlaps the up step's dependent loads.
template <int K, typename T, int BS = 0>
__global__ void __launch_bounds__(Shape<K>::THREADS) k_mf_post(MfOp<T> op, BicgVectors<T> v, CoarseOut<T> co,
                                                                int has_coarse, double w, ReduceScratch rs, int mode) {
    using S = Shape<K>;
    using PS = PostStage<K, T, BS>;
    using DT = typename PS::DT;
    constexpr int K2 = S::K2;
    KrylovScalars* sc = rs.sc;
    const int done = sc->done;  // uniform; read early so the round trip overlaps the loads
    __shared__ T sr[S::EPB][K2], sz[S::EPB][K2], pu[S::EPB][25], ue[S::EPB][5];
    __shared__ DevBases<T> sbas;
    __shared__ __align__(16) unsigned char sd_raw[PS::kOn ? PS::kBytes : 16];
    __shared__ T kf[PS::KE][BS == 2 ? PS::KF : 1], kt[PS::KE][BS == 2 ? K2 : 1], kz[PS::KE][BS == 2 ? K2 : 1];
    const int le = threadIdx.x / K2, ij = threadIdx.x % K2;
    const int el = blockIdx.x * S::EPB + le;
    const bool active = le < S::EPB && el < op.g.N;
    const int p = el * K2 + ij;
    const DT* dsrc;
    if constexpr (BS == 1) dsrc = op.dinv_bf16;
    else dsrc = op.dinv;
    const DT* dblk = dsrc + (size_t)el * PS::K4;  // this element's inverse block ([rs][ij])
    if constexpr (PS::kOn) {
        const int el0 = blockIdx.x * S::EPB;
        const int el1 = min(el0 + S::EPB, op.g.N);
        const size_t b0 = (size_t)el0 * PS::K4 * sizeof(DT), b1 = (size_t)el1 * PS::K4 * sizeof(DT);
        const size_t a0 = b0 & ~size_t(15), a1 = (b1 + 15) & ~size_t(15);
        const char* g = reinterpret_cast<const char*>(dsrc) + a0;
        const unsigned sb = (unsigned)__cvta_generic_to_shared(sd_raw);
        const unsigned nbytes = (unsigned)(a1 - a0);  // < 32 KB
        for (unsigned o = 16u * threadIdx.x; o < nbytes; o += 16u * blockDim.x)
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sb + o), "l"(g + o) : "memory");
        dblk = reinterpret_cast<const DT*>(sd_raw + (b0 - a0)) + (size_t)le * PS::K4;
    }
    TraceDst<K> td;
    td.load(op.g.scat, active, el, ij);
    T rsum[5], rr = T(0), pp = T(0), vv = T(0);
    if (active) {
#pragma unroll
        for (int s = 0; s < 5; ++s) rsum[s] = op.rowsum[((size_t)el * 5 + s) * K2 + ij];
        rr = v.r[p];
        vv = v.v[p];
        if (mode == 0) pp = v.p[p];
    }
    int kx = -1;  // BS 2: this element's exact block, or -1 for its Kronecker factors
    if constexpr (BS == 2) {
        if (active) {
            kx = op.kron_x[el];
            for (int q = ij; q < PS::KF; q += K2) kf[le][q] = op.kron_f[(size_t)el * PS::KF + q];
        }
    }
    stage_bases(sbas, op.b);
    const F0<T> f0 = f0_of(v, sc, mode);
    // u0 of block slot s (element bcol[5 el + s]) as five partial sums pu[s][part]
    if (active)
        for (int t = ij; t < 25; t += K2) {
            const int slot = t / 5, part = t % 5;
            const int c = op.bcol[el * 5 + slot];
            T u = T(0);
            if (c >= 0 && has_coarse) u = co.u0 ? (part == 0 ? co.u0[c] : T(0)) : up0_part(co, f0, c, part);
            pu[le][t] = u;
        }
    if (mode == 0 && has_coarse && active && ij == 0) v.ep[(sc->it + 1) & 1][el] = f0[el];
    // the operand: p or s
    T f;
    if (mode == 0) {
        if (sc->it == 0) {
            f = rr;
        } else {
            const double beta = (sc->rho / sc->rho_old) * (sc->alpha / sc->omega);
            f = rr + T(beta) * (pp - T(sc->omega) * vv);
        }
    } else {
        f = rr - T(sc->alpha) * vv;
    }
    if (active && !done) {
        if (mode == 0) v.p[p] = f;
        else v.s[p] = f;
    }
    if constexpr (PS::kOn) asm volatile("cp.async.wait_all;\n" ::: "memory");
    __syncthreads();
    if (done) return;
    // the five slot values, each the sum of its five parts (part 0..4 in order)
    if (active)
        for (int q = ij; q < 5; q += K2)  // K^2 < 5 threads per element for K <= 2
            ue[le][q] = pu[le][5 * q] + pu[le][5 * q + 1] + pu[le][5 * q + 2] + pu[le][5 * q + 3] + pu[le][5 * q + 4];
    __syncthreads();
    T u_self = T(0);
    if (active) {
        T ae = T(0);
#pragma unroll
        for (int s = 0; s < 5; ++s) ae += rsum[s] * ue[le][s];
        u_self = ue[le][0];
        sr[le][ij] = f - ae;
    }
    __syncthreads();
    T* z = mode == 0 ? v.ph : v.sh;
    T acc = T(0);
    if constexpr (BS == 2) {
        // the exact block where the fit falls back (read before the body reuses sr), then
        // the Kronecker-sum step for the other elements; every thread passes the body's
        // barriers
        if (active && kx >= 0) {
            const T* blk = op.kron_exact + (size_t)kx * PS::K4;
            for (int r = 0; r < K2; ++r) acc += blk[r * K2 + ij] * sr[le][r];
        }
        const int lei = active ? le : 0;
        const ElemCtx<K2> ec{ij};
        kron_apply_body<K, T>(ec, active && kx < 0, kf[lei], kf[lei] + 4 * K2, sr[lei], kt[lei], kz[lei]);
        if (active && kx < 0) acc = kz[le][ij];
    } else if (active) {
#pragma unroll
        for (int r = 0; r < K2; ++r) acc += T(block_value(dblk[r * K2 + ij])) * sr[le][r];
    }
    if (active) {
        const T zz = u_self + T(w) * acc;
        z[p] = zz;
        sz[le][ij] = zz;
    }
    __syncthreads();
    emit_traces<K, T>(sz[active ? le : 0], sbas, td, v.tv, v.tg, ij);
    if (mode == 1) {
        double part[1] = {active ? double(f) * double(f) : 0.0};
        double out[1];
        if (grid_reduce<1>(part, rs.partials, rs.counter, out) && threadIdx.x == 0) {
            sc->snorm2 = out[0];
            sc->s_exit = out[0] <= sc->eps2;
        }
    }
}

// v = A ph; alpha = rho / (rhat, v)
template <int K, typename T>
__global__ void __launch_bounds__(Shape<K>::THREADS) k_mf_v(MfOp<T> op, BicgVectors<T> v, ReduceScratch rs) {
    using S = Shape<K>;
    KrylovScalars* sc = rs.sc;
    // read before the operator's loads so the round trips overlap; the flag is uniform
    // over the grid (only this kernel's last CTA writes it, after every CTA has read it)
    const int done = sc->done;
    __shared__ MfShared<K, T> sm;
    const int le = threadIdx.x / S::K2, ij = threadIdx.x % S::K2;
    const int el = blockIdx.x * S::EPB + le;
    const bool active = le < S::EPB && el < op.g.N;
    const T y = mf_apply<K, T>(op, v.ph, v.tv, v.tg, sm, active, le, el, ij);
    if (done) return;
    double part[1] = {0.0};
    if (active) {
        const int p = el * S::K2 + ij;
        v.v[p] = y;
        part[0] = double(v.rhat[p]) * double(y);
    }
    element_sum<K, T>(sm.a, y, active, le, ij, el, v.ev);
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
__global__ void __launch_bounds__(Shape<K>::THREADS) k_mf_t(MfOp<T> op, BicgVectors<T> v, ReduceScratch rs) {
    using S = Shape<K>;
    KrylovScalars* sc = rs.sc;
    const bool skip = sc->done || sc->s_exit;  // read early: the round trip overlaps the operator's loads
    __shared__ MfShared<K, T> sm;
    const int le = threadIdx.x / S::K2, ij = threadIdx.x % S::K2;
    const int el = blockIdx.x * S::EPB + le;
    const bool active = le < S::EPB && el < op.g.N;
    const T y = mf_apply<K, T>(op, v.sh, v.tv, v.tg, sm, active, le, el, ij);
    if (skip) return;
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

// x += alpha ph + omega sh; r = s - omega t; ||r||^2, (rhat, r); element sums of r;
// convergence test. After an s-exit (||s|| already below tolerance) only x += alpha ph.
// The last CTA to finish ends the iteration: it updates the scalars, sets `done`, and
// inside a captured solve sets the condition of the graph's while node (iterate while
// not done). Every CTA reads `done` and `s_exit` before any CTA arrives at the counter,
// so the last CTA may change them. Every body execution either increments `it` (capped at
// max_iter) or finds `done` set and clears the condition, so the device loop always ends.
template <int K, typename T>
__global__ void __launch_bounds__(Shape<K>::THREADS) k_xr_update(int N, BicgVectors<T> v, ReduceScratch rs,
                                                                  int max_iter, cudaGraphConditionalHandle h,
                                                                  int has_handle) {
    using S = Shape<K>;
    constexpr int NT = kVecTiles;
    KrylovScalars* sc = rs.sc;
    __shared__ T sr[S::EPB][S::K2];
    const int le = threadIdx.x / S::K2, ij = threadIdx.x % S::K2;
    int p[NT], el[NT];
    bool act[NT];
    T x[NT], ph[NT], sh[NT], sv[NT], tv[NT], rh[NT];
#pragma unroll
    for (int t = 0; t < NT; ++t) {
        el[t] = (blockIdx.x + t * gridDim.x) * S::EPB + le;
        act[t] = le < S::EPB && el[t] < N;
        p[t] = el[t] * S::K2 + ij;
        x[t] = act[t] ? v.x[p[t]] : T(0);
        ph[t] = act[t] ? v.ph[p[t]] : T(0);
        sh[t] = act[t] ? v.sh[p[t]] : T(0);
        sv[t] = act[t] ? v.s[p[t]] : T(0);
        tv[t] = act[t] ? v.t[p[t]] : T(0);
        rh[t] = act[t] ? v.rhat[p[t]] : T(0);
    }
    if (sc->done) {  // the solve ended earlier in this body (breakdown)
        if (has_handle && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(h, 0u);
        return;
    }
    const T alpha = T(sc->alpha);
    const bool s_exit = sc->s_exit;
    const double omega = sc->omega;
    double part[2] = {0.0, 0.0};
#pragma unroll
    for (int t = 0; t < NT; ++t) {
        T r = T(0);
        if (s_exit) {
            if (act[t]) v.x[p[t]] = x[t] + alpha * ph[t];
        } else if (act[t]) {
            v.x[p[t]] = x[t] + (alpha * ph[t] + T(omega) * sh[t]);
            r = sv[t] - T(omega) * tv[t];
            v.r[p[t]] = r;
            part[0] += double(r) * double(r);
            part[1] += double(rh[t]) * double(r);
        }
        if (!s_exit) element_sum<K, T>(sr, r, act[t], le, ij, el[t], v.er);
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
cudaError_t krylov_init(const MfOp<T>& op, const BicgVectors<T>& v, const ReduceScratch& rs,
                        cudaStream_t s) {
    const int N = op.g.N;
    HO2D_KSWITCH(op.K, (k_trace_in<KK, T><<<kgrid<KK>(N), Shape<KK>::THREADS, 0, s>>>(op, v.x, v.xtv, v.xtg)));
    HO2D_KSWITCH(op.K, (k_mf_init<KK, T><<<kgrid<KK>(N), Shape<KK>::THREADS, 0, s>>>(op, v, rs)));
    const size_t n = (size_t)N * op.K * op.K;
    k_zero_if<T><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(v.x, n, rs.sc);
    return cudaGetLastError();
}

// One BiCGSTAB iteration: [coarse cycle on P^T p] -> p update + smoothing (ph) -> v = A ph
// -> [coarse cycle on P^T s] -> s update + smoothing (sh) -> t = A sh -> x, r update and
// loop control.
template <int K, typename T>
static void iteration_impl(const MfOp<T>& op, const BicgVectors<T>& v, const ReduceScratch& rs, int max_iter,
                           const Precond<T>& pc, cudaGraphConditionalHandle h, int has_handle, cudaStream_t s) {
    const int N = op.g.N;
    const unsigned g = kgrid<K>(N);
    constexpr int th = Shape<K>::THREADS;
    const int mg = pc.nlev > 0;
    const CoarseOut<T> co = mg ? coarse_out(pc) : CoarseOut<T>();
    const unsigned gv = (g + kVecTiles - 1) / kVecTiles;
    auto post = [&](int mode) {
        if constexpr (std::is_same<T, float>::value) {
            if (op.kron_f) {
                k_mf_post<K, T, 2><<<g, th, 0, s>>>(op, v, co, mg, pc.omega, rs, mode);
                return;
            }
            if (op.dinv_bf16) {
                k_mf_post<K, T, 1><<<g, th, 0, s>>>(op, v, co, mg, pc.omega, rs, mode);
                return;
            }
        }
        k_mf_post<K, T><<<g, th, 0, s>>>(op, v, co, mg, pc.omega, rs, mode);
    };
    if (mg) coarse_cycle<T>(pc, v, rs.sc, 0, s);
    post(0);
    k_mf_v<K, T><<<g, th, 0, s>>>(op, v, rs);
    if (mg) coarse_cycle<T>(pc, v, rs.sc, 1, s);
    post(1);
    k_mf_t<K, T><<<g, th, 0, s>>>(op, v, rs);
    k_xr_update<K, T><<<gv, th, 0, s>>>(N, v, rs, max_iter, h, has_handle);
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

template <typename T>
cudaError_t mf_residual(const MfOp<T>& op, const double* b, const T* x, T* xtv, T* xtg, double* r,
                        const ReduceScratch& rs, cudaStream_t s) {
    HO2D_KSWITCH(op.K, (k_trace_in<KK, T><<<kgrid<KK>(op.g.N), Shape<KK>::THREADS, 0, s>>>(op, x, xtv, xtg)));
    HO2D_KSWITCH(op.K, (k_mf_residual<KK, T><<<kgrid<KK>(op.g.N), Shape<KK>::THREADS, 0, s>>>(op, b, x, xtv, xtg, r,
                                                                                                  rs)));
    return cudaGetLastError();
}

template <typename T>
cudaError_t mf_apply_op(const MfOp<T>& op, const T* x, T* xtv, T* xtg, T* y, cudaStream_t s) {
    HO2D_KSWITCH(op.K, (k_trace_in<KK, T><<<kgrid<KK>(op.g.N), Shape<KK>::THREADS, 0, s>>>(op, x, xtv, xtg)));
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
    template cudaError_t krylov_init<T>(const MfOp<T>&, const BicgVectors<T>&, const ReduceScratch&,             \
                                        cudaStream_t);                                                            \
    template cudaError_t krylov_iteration<T>(const MfOp<T>&, const BicgVectors<T>&, const ReduceScratch&, int,    \
                                             const Precond<T>&, cudaStream_t);                                    \
    template int krylov_launches_per_iteration<T>(const Precond<T>&);                                             \
    template cudaError_t krylov_capture_solve<T>(const MfOp<T>&, const BicgVectors<T>&, const ReduceScratch&,     \
                                                 int, const Precond<T>&, cudaStream_t, cudaGraph_t*);             \
    template cudaError_t mf_residual<T>(const MfOp<T>&, const double*, const T*, T*, T*, double*,                 \
                                        const ReduceScratch&, cudaStream_t);                                      \
    template cudaError_t mf_apply_op<T>(const MfOp<T>&, const T*, T*, T*, T*, cudaStream_t);                      \
    template cudaError_t mf_apply_only<T>(const MfOp<T>&, const T*, const T*, const T*, T*, int, cudaStream_t);

HO2D_INSTANTIATE_KRYLOV(double)
HO2D_INSTANTIATE_KRYLOV(float)

}  // namespace ho2d
