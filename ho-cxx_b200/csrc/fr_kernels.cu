// fr_kernels.cu -- flux-reconstruction kernels of one explicit stage (sm_100a).
//
// Mapping: the velocity and residual kernels run row-parallel (stage_rows.cuh: K threads
// per element, thread t owning row t, column t and face point t of each face); the trace
// and right-hand-side kernels use K^2 threads per element (one per solution point), EPB
// elements per CTA. Neighbour data come from per-element face-trace buffers
// ([el][ijp][k]) written by the previous kernel, so every kernel reads each array once.
//
//   trace_kernel      psi -> psi face values / normal derivatives
//   velocity_kernel   common psi, corrected grad psi, u = dpsi/dy, v = -dpsi/dx
//                     (src/HO_2D.cpp:3174-3366) + velocity_jump / BC_normal_vel side
//                     outputs + no-slip diffusion BC (2647-2664) + the omega and
//                     contravariant-flux face traces the residual kernel needs
//   residual_kernel   Re^-1 Lap(omega) (2666-2927) + BC_vorticity + BC_advection
//                     (2219-2243) + -div(u omega), type 1 (2245-2437) or type 2
//                     (2439-2645) + k = dt (adv + diff) (1833-1836) + the RK update
//                     of solve_advection_diffusion (1465-1531)
//   poisson_rhs_kernel  b = -omega J - sum boundary_source . BC_Poisson (1881-1900)
//   bc_update_kernel  time-dependent BC refresh and h-direction flip (1979-2217)
#include <cmath>

#include <algorithm>

#include "device.cuh"
#include "fr_device.cuh"
#include "fr_launch.hpp"
#include "stage_rows.cuh"

namespace ho2d {

// ----------------------------------------------------------------------------------
template <int K, typename T>
__global__ void __launch_bounds__(Shape<K>::THREADS) trace_kernel(int N, const T* __restrict__ f, T* __restrict__ tv,
                                                                   T* __restrict__ tg, DevBases<T> bp) {
    using S = Shape<K>;
    __shared__ DevBases<T> b;
    stage_bases(b, bp);
    __shared__ T s_f[S::EPB][S::K2];
    const int le = threadIdx.x / S::K2, ij = threadIdx.x % S::K2;
    const int el = blockIdx.x * S::EPB + le;
    const bool active = le < S::EPB && el < N;
    if (active) s_f[le][ij] = f[el * S::K2 + ij];
    __syncthreads();
    if (active) {
        for (int o = ij; o < S::NF; o += S::K2) {
            T v, d;
            face_trace<K, T>(s_f[le], b, o, v, d);
            tv[el * S::NF + o] = v;
            tg[el * S::NF + o] = d;
        }
    }
}

// b = -omega J - sum over the element's boundary edges of boundary_source . BC_Poisson,
// edges taken in increasing index like the reference's loop.
template <int K, typename T>
__global__ void __launch_bounds__(Shape<K>::THREADS) poisson_rhs_kernel(int N, const int* __restrict__ face_nb,
                                                                         const T* __restrict__ w,
                                                                         const T* __restrict__ J,
                                                                         const double* __restrict__ bsrc,
                                                                         const double* __restrict__ bc_p,
                                                                         double* __restrict__ rhs) {
    using S = Shape<K>;
    const int le = threadIdx.x / S::K2, ij = threadIdx.x % S::K2;
    const int el = blockIdx.x * S::EPB + le;
    if (le >= S::EPB || el >= N) return;
    const int p = el * S::K2 + ij;
    double r = -double(w[p]) * double(J[p]);
    int es[4], ne = 0;
#pragma unroll
    for (int f = 0; f < 4; ++f) {
        const int nb = face_nb[el * 4 + f];
        if (nb < 0) es[ne++] = -nb - 1;
    }
    for (int x = 1; x < ne; ++x)
        for (int y = x; y > 0 && es[y - 1] > es[y]; --y) {
            const int t = es[y];
            es[y] = es[y - 1];
            es[y - 1] = t;
        }
    for (int x = 0; x < ne; ++x) {
        const int e = es[x];
        const double* s = bsrc + ((size_t)e * S::K2 + ij) * K;
        double acc = r;
#pragma unroll
        for (int al = 0; al < K; ++al) acc -= s[al] * bc_p[e * K + al];
        r = acc;
    }
    rhs[p] = r;
}

// Time-dependent BC refresh (problem types 2 and 3; hybrid runs, type 11) and the flip of
// normal velocities and Neumann vorticity BCs into the local h direction, one thread per
// edge point. Roles: 1 inlet, 2 top, 3 bottom, 4 object; hybrid 5 open, 6 wall, 7 inlet.
__global__ void bc_update_kernel(int n_eb, int K, int ptype, double tc, double y_min, double y_max,
                                 const int* __restrict__ role, const int* __restrict__ be_ijp,
                                 const int* __restrict__ sw_d, const double* __restrict__ edge_y, BcArrays bc,
                                 HybridBc hb) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n_eb * K) return;
    const int e = idx / K;
    const int r = role[e];
    const double y = edge_y[idx];
    if (ptype == 2) {
        const double h2 = (y_max - y_min) * (y_max - y_min);
        if (r == 1) {
            bc.bc_p[idx] = tc * ((y - y_min) * (y - y_min)) * (3.0 * y_max - y_min - 2.0 * y) / h2;
            bc.bc_d[idx] = tc * 6.0 * (2.0 * y - y_min - y_max) / h2;
            bc.bc_nv[idx] = tc * 6.0 * (y - y_min) * (y - y_max) / h2;
        } else if (r == 2) {
            bc.bc_p[idx] = tc * (y_max - y_min);
        }
    } else if (ptype == 3) {
        if (r == 1) {
            bc.bc_p[idx] = tc * (y - y_min);
            bc.bc_nv[idx] = -tc;
        } else if (r == 2) {
            bc.bc_p[idx] = tc * (y_max - y_min);
            bc.bc_d[idx] = 0.0;
            bc.bc_pv[idx] = -tc;
        } else if (r == 3) {
            bc.bc_pv[idx] = tc;
        } else if (r == 4) {
            bc.bc_p[idx] = tc * 0.5 * (y_max - y_min);
        }
    } else if (ptype == 11) {  // src/HO_2D.cpp:2104-2191
        if (r == 5) {
            const double pv = -(hb.fac1 * hb.vp0[idx] + hb.fac2 * hb.vp1[idx]);
            bc.bc_nv[idx] = -(hb.fac1 * hb.vn0[idx] + hb.fac2 * hb.vn1[idx]);
            bc.bc_pv[idx] = pv;
            bc.bc_p[idx] = pv;
            bc.bc_d[idx] = hb.fac1 * hb.w0[idx] + hb.fac2 * hb.w1[idx];
        } else if (r == 6) {
            bc.bc_nv[idx] = 0.0;
            bc.bc_pv[idx] = 0.0;
        } else if (r == 7) {
            bc.bc_nv[idx] = -hb.inlet_nv[e];
        }
    }
    const double sign = 2.0 * (be_ijp[e] % 2) - 1.0;
    bc.bc_nv[idx] *= sign;
    if (sw_d[e] == kNeumann) bc.bc_d[idx] *= sign;
}

// ----------------------------------------------------------------------------------
// launchers

#define HO2D_DISPATCH_K(K, CALL)                          \
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
static unsigned grid_for(int N) {
    return (unsigned)((N + Shape<K>::EPB - 1) / Shape<K>::EPB);
}

template <typename T>
cudaError_t launch_trace(int K, int N, const T* f, T* tv, T* tg, const DevBases<T>& b, cudaStream_t s) {
    HO2D_DISPATCH_K(K, (trace_kernel<KK, T><<<grid_for<KK>(N), Shape<KK>::THREADS, 0, s>>>(N, f, tv, tg, b)));
    return cudaGetLastError();
}

template <int K>
static unsigned rows_grid(int N) {
    return (unsigned)((N + Rows<K>::EPC - 1) / Rows<K>::EPC);
}

template <typename T, typename TP>
cudaError_t launch_velocity(int K, const FrGeom<TP>& g, const StageCoef<TP>& c, const DevBases<TP>& bp,
                            const DevBases<T>& bw, const BcArrays& bc, const VelocityArgs<T, TP>& a, cudaStream_t s) {
    HO2D_DISPATCH_K(K, (velocity_rows<KK, T, TP><<<rows_grid<KK>(g.N), Rows<KK>::THREADS, 0, s>>>(
                           g, c.G11, c.G12, c.G22, bp, bw, bc, a)));
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_residual(int K, const FrGeom<T>& g, const StageCoef<T>& c, const DevBases<T>& b,
                            const BcArrays& bc, const ResidualArgs<T>& a, cudaStream_t s) {
    HO2D_DISPATCH_K(K, (residual_rows<KK, T><<<rows_grid<KK>(g.N), Rows<KK>::THREADS, 0, s>>>(g, c.G11, c.G12,
                                                                                               c.G22, b, bc, a)));
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_poisson_rhs(int K, int N, const int* face_nb, const T* w, const T* J, const double* bsrc,
                               const double* bc_p, double* rhs, cudaStream_t s) {
    HO2D_DISPATCH_K(K, (poisson_rhs_kernel<KK, T><<<grid_for<KK>(N), Shape<KK>::THREADS, 0, s>>>(
                           N, face_nb, w, J, bsrc, bc_p, rhs)));
    return cudaGetLastError();
}

// A vorticity handed in from the host (staged in `in`) against the device's current one:
// flags[0] = some value is not finite, flags[1] = some value differs bitwise from `cur`.
__global__ void k_vort_check(const double* __restrict__ in, const double* __restrict__ cur, size_t n,
                             int* __restrict__ flags) {
    bool bad = false, diff = false;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const double x = in[i];
        bad |= !isfinite(x);
        diff |= __double_as_longlong(x) != __double_as_longlong(cur[i]);
    }
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(&flags[0], 1);
    if (__any_sync(0xffffffffu, diff) && (threadIdx.x & 31) == 0) atomicOr(&flags[1], 1);
}

cudaError_t launch_vort_check(const double* in, const double* cur, size_t n, int* flags, cudaStream_t s) {
    const unsigned g = (unsigned)std::min<size_t>((n + 255) / 256, 148 * 8);
    k_vort_check<<<g ? g : 1, 256, 0, s>>>(in, cur, n, flags);
    return cudaGetLastError();
}

cudaError_t launch_bc_update(int n_eb, int K, int ptype, double tc, double y_min, double y_max, const int* role,
                             const int* be_ijp, const int* sw_d, const double* edge_y, const BcArrays& bc,
                             const HybridBc& hb, cudaStream_t s) {
    const int n = n_eb * K;
    if (n == 0) return cudaSuccess;
    if (ptype == 11 && !(hb.vn0 && hb.vn1 && hb.vp0 && hb.vp1 && hb.w0 && hb.w1 && hb.inlet_nv))
        return cudaErrorInvalidValue;
    bc_update_kernel<<<(n + 127) / 128, 128, 0, s>>>(n_eb, K, ptype, tc, y_min, y_max, role, be_ijp, sw_d, edge_y,
                                                     bc, hb);
    return cudaGetLastError();
}

template <typename T>
__global__ void hybrid_blend_kernel(size_t n, double* __restrict__ omega, T* __restrict__ w_stage,
                                    const double* __restrict__ wgt, const double* __restrict__ v0,
                                    const double* __restrict__ v1, double fac1, double fac2) {
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const double w = wgt[i];
        const double om = (1.0 - w) * omega[i] + w * (fac1 * v0[i] + fac2 * v1[i]);
        omega[i] = om;
        if (w_stage) w_stage[i] = T(om);
    }
}

template <typename T>
cudaError_t launch_hybrid_blend(size_t n, double* omega, T* w_stage, const double* wgt, const double* v0,
                                const double* v1, double fac1, double fac2, cudaStream_t s) {
    const size_t b = (n + 255) / 256;
    hybrid_blend_kernel<T><<<(unsigned)(b > 1184 ? 1184 : (b < 1 ? 1 : b)), 256, 0, s>>>(n, omega, w_stage, wgt, v0, v1,
                                                                                        fac1, fac2);
    return cudaGetLastError();
}

template cudaError_t launch_hybrid_blend<double>(size_t, double*, double*, const double*, const double*,
                                                 const double*, double, double, cudaStream_t);
template cudaError_t launch_hybrid_blend<float>(size_t, double*, float*, const double*, const double*, const double*,
                                                double, double, cudaStream_t);

#define HO2D_INSTANTIATE_FR(T)                                                                                     \
    template cudaError_t launch_trace<T>(int, int, const T*, T*, T*, const DevBases<T>&, cudaStream_t);            \
    template cudaError_t launch_velocity<T, double>(int, const FrGeom<double>&, const StageCoef<double>&,       \
                                                    const DevBases<double>&, const DevBases<T>&, const BcArrays&, \
                                                    const VelocityArgs<T, double>&, cudaStream_t);                 \
    template cudaError_t launch_residual<T>(int, const FrGeom<T>&, const StageCoef<T>&, const DevBases<T>&,       \
                                            const BcArrays&, const ResidualArgs<T>&, cudaStream_t);                \
    template cudaError_t launch_poisson_rhs<T>(int, int, const int*, const T*, const T*, const double*,           \
                                               const double*, double*, cudaStream_t);

HO2D_INSTANTIATE_FR(double)
HO2D_INSTANTIATE_FR(float)

}  // namespace ho2d
