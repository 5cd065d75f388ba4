// fr_device.cuh -- device routines shared by the FR stage kernels and the matrix-free
// Poisson operator: face traces, Huynh method-2 common values and fluxes (g = g_DG),
// the contravariant gradient with its Radau face corrections, and the FR Laplacian of
// one element (src/HO_2D.cpp:2666-2927; the same discretisation the Poisson matrix of
// src/HO_2D.cpp:1533-1804 assembles, so A x equals lap_element(x) with homogeneous
// boundary values).
#pragma once

#include "device.cuh"

namespace ho2d {

// Copies the 1-D basis tables from the kernel-parameter bank into shared memory: the
// FR loops index them per thread, which would serialise constant-cache reads. The
// caller synchronises before use.
template <typename T>
__device__ __forceinline__ void stage_bases(DevBases<T>& dst, const DevBases<T>& src) {
    constexpr int NW = (int)(sizeof(DevBases<T>) / sizeof(T));
    const T* s = reinterpret_cast<const T*>(&src);
    T* d = reinterpret_cast<T*>(&dst);
    for (int t = threadIdx.x; t < NW; t += blockDim.x) d[t] = s[t];
}

template <int K>
__device__ __forceinline__ int bf_index(int side, int k) {
    return (side / 2) * (K - 2 * k - 1) + k;
}

__device__ __forceinline__ int side_of_ijp(int ijp) {
    // ijp 0 W, 1 E, 2 S, 3 N -> element side (S=0, E=1, N=2, W=3)
    return ijp == 0 ? 3 : (ijp == 1 ? 1 : (ijp == 2 ? 0 : 2));
}

// Face values (basis at -1/+1) and normal derivatives of a K x K block in shared memory.
template <int K, typename T>
__device__ __forceinline__ void face_trace(const T* f, const DevBases<T>& b, int o, T& val, T& der) {
    const int ijp = o / K, k = o % K;
    const int lr = ijp & 1;
    T v = T(0), g = T(0);
    if (ijp < 2) {
#pragma unroll
        for (int m = 0; m < K; ++m) {
            v += f[k * K + m] * b.sbb[m * 2 + lr];
            g += f[k * K + m] * b.sbgb[m * 2 + lr];
        }
    } else {
#pragma unroll
        for (int m = 0; m < K; ++m) {
            v += f[m * K + k] * b.sbb[m * 2 + lr];
            g += f[m * K + k] * b.sbgb[m * 2 + lr];
        }
    }
    val = v;
    der = g;
}

template <int K, typename T>
__device__ __forceinline__ T face_value(const T* f, const DevBases<T>& b, int o) {
    const int ijp = o / K, k = o % K;
    const int lr = ijp & 1;
    T v = T(0);
    if (ijp < 2) {
#pragma unroll
        for (int m = 0; m < K; ++m) v += f[k * K + m] * b.sbb[m * 2 + lr];
    } else {
#pragma unroll
        for (int m = 0; m < K; ++m) v += f[m * K + k] * b.sbb[m * 2 + lr];
    }
    return v;
}

// Common value (s_com) and common normal flux (s_cg) on the 4 faces of one element,
// Huynh's method 2 with g = g_DG: calc_internal_comm_vals_meth2 and
// calc_boundary_comm_vals_meth2 (src/HO_2D.cpp:2833-2927), the face-flux average of
// 2739-2743, for boundary values `bcv` with switches `sw`. `neu_sign` multiplies the
// Neumann values by the h-direction sign (the psi case, src/HO_2D.cpp:3259-3262).
// Must be called by all threads of the CTA (contains __syncthreads).
template <int K, typename T>
__device__ void face_common(bool active, int el, int ij, const FrGeom<T>& g, const DevBases<T>& b,
                            const T* __restrict__ tv_glob, const T* __restrict__ tg_glob, const T* s_tv,
                            const T* s_tg, T* s_com, T* s_cg, const int* __restrict__ sw,
                            const double* __restrict__ bcv, bool neu_sign) {
    constexpr int K2 = K * K, NF = 4 * K;
    // (1) common values of interior and Dirichlet faces
    if (active) {
        for (int o = ij; o < NF; o += K2) {
            const int ijp = o / K, k = o % K;
            const int nb = g.face_nb[el * 4 + ijp];
            T com;
            if (nb >= 0) {
                const int nijp = g.face_nijp[el * 4 + ijp];
                const int rev = (ijp + nijp - ijp / 2 - nijp / 2 + 1) % 2;
                const int jn = rev ? K - 1 - k : k;
                com = T(0.5) * (s_tv[o] + tv_glob[(nb * 4 + nijp) * K + jn]);
            } else {
                const int e = -nb - 1;
                com = sw[e] == kDirichlet ? T(bcv[e * K + bf_index<K>(side_of_ijp(ijp), k)]) : T(0);
            }
            s_com[o] = com;
        }
    }
    __syncthreads();
    // (2) Neumann faces: solve the K x K system for the common value (one thread per face)
    for (int ijp = ij; active && ijp < 4; ijp += K2) {
        const int nb = g.face_nb[el * 4 + ijp];
        if (nb < 0 && sw[-nb - 1] == kNeumann) {
            const int e = -nb - 1, side = side_of_ijp(ijp), lr = ijp & 1;
            const T sgn = neu_sign ? T(2 * (ijp % 2) - 1) : T(1);
            T M[K][K], r[K], x[K];
#pragma unroll
            for (int k = 0; k < K; ++k) {
                const int q = (el * 4 + ijp) * K + k;
                const T cg = sgn * T(bcv[e * K + bf_index<K>(side, k)]) * g.fAn[q];
                s_cg[ijp * K + k] = cg;
                r[k] = g.fJ[q] * cg - g.fA[q] * (s_tg[ijp * K + k] - s_tv[ijp * K + k] * b.gp[lr]);
#pragma unroll
                for (int i = 0; i < K; ++i) M[k][i] = -g.fB[q] * b.D[i * K + k];
                M[k][k] += g.fA[q] * b.gp[lr];
            }
            // Gauss elimination without pivoting (src/MathHelpers.hpp:53-74)
#pragma unroll
            for (int c = 0; c < K - 1; ++c) {
#pragma unroll
                for (int i = c + 1; i < K; ++i) {
                    const T f = M[i][c] / M[c][c];
                    r[i] -= f * r[c];
#pragma unroll
                    for (int j = c + 1; j < K; ++j) M[i][j] -= f * M[c][j];
                }
            }
#pragma unroll
            for (int i = K - 1; i >= 0; --i) {
                T s = T(0);
#pragma unroll
                for (int j = i + 1; j < K; ++j) s += M[i][j] * x[j];
                x[i] = (r[i] - s) / M[i][i];
            }
#pragma unroll
            for (int k = 0; k < K; ++k) s_com[ijp * K + k] = x[k];
        }
    }
    __syncthreads();
    // (3) corrected normal fluxes; interior faces average with the neighbour's flux
    if (active) {
        for (int o = ij; o < NF; o += K2) {
            const int ijp = o / K, k = o % K, lr = ijp & 1;
            const int nb = g.face_nb[el * 4 + ijp];
            if (nb < 0 && sw[-nb - 1] == kNeumann) continue;
            const int q = (el * 4 + ijp) * K + k;
            const T com = s_com[o];
            T cross = T(0);
#pragma unroll
            for (int m = 0; m < K; ++m) cross += s_com[ijp * K + m] * b.D[m * K + k];
            const T dv = s_tg[o] + (com - s_tv[o]) * b.gp[lr];
            const T fl = (dv * g.fA[q] - cross * g.fB[q]) / g.fJ[q];
            if (nb < 0) {
                s_cg[o] = fl;
            } else {
                const int nijp = g.face_nijp[el * 4 + ijp];
                const int rev = (ijp + nijp - ijp / 2 - nijp / 2 + 1) % 2;
                const int jn = rev ? K - 1 - k : k;
                const int nq = (nb * 4 + nijp) * K + jn;
                T crn = T(0);
#pragma unroll
                for (int m = 0; m < K; ++m) crn += s_com[ijp * K + (rev ? K - 1 - m : m)] * b.D[m * K + jn];
                const T dvn = tg_glob[nq] + (com - tv_glob[nq]) * b.gp[nijp & 1];
                const T fln = (dvn * g.fA[nq] - crn * g.fB[nq]) / g.fJ[nq];
                const T sign = T(2 * ((ijp + nijp) % 2) - 1);
                s_cg[o] = T(0.5) * (fl + sign * fln);
            }
        }
    }
    __syncthreads();
}

// f~, g~ at the solution points (src/HO_2D.cpp:2775-2792) and their face corrections
// fB/gB (2795-2803) in s_fb[ijp][k]. Needs s_f, s_tv, s_com, s_cg. Collective.
template <int K, typename T>
__device__ void contravariant_gradient(bool active, int el, int ij, const FrGeom<T>& g, const DevBases<T>& b,
                                       const T* s_f, const T* s_tv, const T* s_com, const T* s_cg, T* s_a,
                                       T* s_b, T* s_fb, T& ft, T& gt) {
    constexpr int K2 = K * K, NF = 4 * K;
    const int j = ij / K, i = ij % K;
    if (active) {
        T dx = T(0), de = T(0);
#pragma unroll
        for (int d = 0; d < K; ++d) {
            dx += s_f[j * K + d] * b.D[d * K + i];
            de += s_f[d * K + i] * b.D[d * K + j];
        }
        dx += (s_com[0 * K + j] - s_tv[0 * K + j]) * b.gR[i * 2 + 0];
        dx += (s_com[1 * K + j] - s_tv[1 * K + j]) * b.gR[i * 2 + 1];
        de += (s_com[2 * K + i] - s_tv[2 * K + i]) * b.gR[j * 2 + 0];
        de += (s_com[3 * K + i] - s_tv[3 * K + i]) * b.gR[j * 2 + 1];
        const int p = el * K2 + ij;
        const T xx = g.xxi[p], xe = g.xeta[p], yx = g.yxi[p], ye = g.yeta[p], J = g.J[p];
        ft = (dx * (xe * xe + ye * ye) - de * (xx * xe + yx * ye)) / J;
        gt = (de * (xx * xx + yx * yx) - dx * (xx * xe + yx * ye)) / J;
        s_a[ij] = ft;
        s_b[ij] = gt;
    }
    __syncthreads();
    if (active) {
        for (int o = ij; o < NF; o += K2) {
            const int ijp = o / K, k = o % K, lr = ijp & 1;
            T v = s_cg[o];
            if (ijp < 2) {
#pragma unroll
                for (int d = 0; d < K; ++d) v -= s_a[k * K + d] * b.sbb[d * 2 + lr];
            } else {
#pragma unroll
                for (int d = 0; d < K; ++d) v -= s_b[d * K + k] * b.sbb[d * 2 + lr];
            }
            s_fb[o] = v;
        }
    }
    __syncthreads();
}


// Raw FR Laplacian J * Lap(x) at (el, ij) from the element's values s_f, its traces
// s_tv/s_tg (computed from s_f by face_trace) and every element's traces in global
// memory; boundary values bcv with switches sw. Collective (all threads of the CTA).
template <int K, typename T>
__device__ T lap_element(bool active, int el, int ij, const FrGeom<T>& g, const DevBases<T>& b,
                         const T* __restrict__ tv_glob, const T* __restrict__ tg_glob, const T* s_f, const T* s_tv,
                         const T* s_tg, T* s_com, T* s_cg, T* s_a, T* s_b, T* s_fb, const int* __restrict__ sw,
                         const double* __restrict__ bcv) {
    face_common<K, T>(active, el, ij, g, b, tv_glob, tg_glob, s_tv, s_tg, s_com, s_cg, sw, bcv, true);
    T ft = T(0), gt = T(0);
    contravariant_gradient<K, T>(active, el, ij, g, b, s_f, s_tv, s_com, s_cg, s_a, s_b, s_fb, ft, gt);
    if (!active) return T(0);
    const int j = ij / K, i = ij % K;
    T lap = T(0);
#pragma unroll
    for (int d = 0; d < K; ++d) lap += s_a[j * K + d] * b.D[d * K + i];
    lap += s_fb[0 * K + j] * b.gR[i * 2 + 0] + s_fb[1 * K + j] * b.gR[i * 2 + 1];
#pragma unroll
    for (int d = 0; d < K; ++d) lap += s_b[d * K + i] * b.D[d * K + j];
    lap += s_fb[2 * K + i] * b.gR[j * 2 + 0] + s_fb[3 * K + i] * b.gR[j * 2 + 1];
    return lap;
}

}  // namespace ho2d
