// kron_apply.cuh -- one element's Kronecker-sum smoother step, z = (I (x) Ax + Ay (x) I)^-1 r,
// by fast diagonalisation (the factors of host_kron.cpp, stored per element as Vx, Vx^-1,
// Vy, Vy^-1 [K][K] row-major and lx, ly [K]). Values are [j][i], j along eta:
//   t = Vy^-1 R Vx^-T,  t ./= (ly_j + lx_i),  Z = Vy t Vx^T,
// four K x K products, one output per thread and a barrier between them; r is overwritten
// (it holds the scaled middle product). Written once for the GPU and the host build
// (elem_ctx.cuh); every thread of the CTA calls it.
#pragma once

#include "elem_ctx.cuh"

namespace ho2d {

template <int K, typename T, class C>
HO2D_HD void kron_apply_body(const C& c, bool active, const T* f, const T* lam, T* r, T* t, T* z) {
    constexpr int K2 = K * K;
    const T *vx = f, *vxi = f + K2, *vy = f + 2 * K2, *vyi = f + 3 * K2;
    const T *lx = lam, *ly = lam + K;
    if (active)
        for (int q = c.tid; q < K2; q += C::nt) {  // t[j][k] = sum_l Vy^-1[j][l] r[l][k]
            const int j = q / K, k = q % K;
            T s = T(0);
            for (int l = 0; l < K; ++l) s += vyi[j * K + l] * r[l * K + k];
            t[q] = s;
        }
    c.sync();
    if (active)
        for (int q = c.tid; q < K2; q += C::nt) {  // r[j][i] = sum_k t[j][k] Vx^-1[i][k] / (ly_j + lx_i)
            const int j = q / K, i = q % K;
            T s = T(0);
            for (int k = 0; k < K; ++k) s += t[j * K + k] * vxi[i * K + k];
            r[q] = s / (ly[j] + lx[i]);
        }
    c.sync();
    if (active)
        for (int q = c.tid; q < K2; q += C::nt) {  // t[j][k] = sum_l Vy[j][l] r[l][k]
            const int j = q / K, k = q % K;
            T s = T(0);
            for (int l = 0; l < K; ++l) s += vy[j * K + l] * r[l * K + k];
            t[q] = s;
        }
    c.sync();
    if (active)
        for (int q = c.tid; q < K2; q += C::nt) {  // z[j][i] = sum_k t[j][k] Vx[i][k]
            const int j = q / K, i = q % K;
            T s = T(0);
            for (int k = 0; k < K; ++k) s += t[j * K + k] * vx[i * K + k];
            z[q] = s;
        }
}

}  // namespace ho2d
