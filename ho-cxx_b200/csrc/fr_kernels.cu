// fr_kernels.cu -- flux-reconstruction kernels of one explicit stage (sm_100a).
//
// Mapping: K^2 threads per element (one per solution point), EPB elements per CTA;
// an element's volume block is staged in shared memory, face work (4K points) is spread
// over the element's threads. Neighbour data come from per-element face-trace buffers
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

#include "device.cuh"
#include "fr_device.cuh"
#include "fr_launch.hpp"

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

template <int K, typename T, typename TP>
__global__ void __launch_bounds__(Shape<K>::THREADS) velocity_kernel(FrGeom<TP> g, DevBases<TP> bp,
                                                                      DevBases<T> bwp, BcArrays bc,
                                                                      VelocityArgs<T, TP> a) {
    using S = Shape<K>;
    __shared__ DevBases<TP> b;
    __shared__ DevBases<T> bw;
    stage_bases(b, bp);
    stage_bases(bw, bwp);
    constexpr int K2 = S::K2, NF = S::NF, EPB = S::EPB;
    __shared__ TP s_f[EPB][K2], s_a[EPB][K2], s_b[EPB][K2];
    __shared__ T s_w[EPB][K2], s_ux[EPB][K2], s_uy[EPB][K2];
    __shared__ TP s_tv[EPB][NF], s_tg[EPB][NF], s_com[EPB][NF], s_cg[EPB][NF], s_fb[EPB][NF];
    const int le = threadIdx.x / K2, ij = threadIdx.x % K2;
    const int el = blockIdx.x * EPB + le;
    const bool active = le < EPB && el < g.N;
    const int lei = active ? le : 0;
    if (active) {
        s_f[le][ij] = a.psi[el * K2 + ij];
        s_w[le][ij] = a.w[el * K2 + ij];
    }
    __syncthreads();
    if (active)
        for (int o = ij; o < NF; o += K2) face_trace<K, TP>(s_f[le], b, o, s_tv[le][o], s_tg[le][o]);
    __syncthreads();
    face_common<K, TP>(active, el, ij, g, b, a.psi_tv, a.psi_tg, s_tv[lei], s_tg[lei], s_com[lei], s_cg[lei], g.sw_p,
                       bc.bc_p, true);
    // boundary side outputs: velocity_jump / BC_normal_vel, then the no-slip diffusion BC
    if (active) {
        for (int o = ij; o < NF; o += K2) {
            const int ijp = o / K, k = o % K;
            const int nb = g.face_nb[el * 4 + ijp];
            if (nb >= 0) continue;
            const int e = -nb - 1;
            const int be = e * K + bf_index<K>(side_of_ijp(ijp), k);
            const int q = (el * 4 + ijp) * K + k;
            double vj = bc.vjump[be];
            if (g.sw_p[e] == kDirichlet) {
                vj = double(s_cg[le][o]) / double(g.fAn[q]);
            } else {
                const TP vsign = TP(1 - 2 * (ijp / 2));
                TP nv = TP(0);
#pragma unroll
                for (int d = 0; d < K; ++d) nv += vsign * s_com[le][ijp * K + d] * b.D[d * K + k];
                bc.bc_nv[be] = double(nv / g.fAn[q]);
            }
            if (g.noslip[g.be_group[e]]) {
                vj += double(2 * (ijp % 2) - 1) * bc.bc_pv[be];
                bc.bc_d[be] = vj / (a.dt * a.re_inv);
            }
            bc.vjump[be] = vj;
        }
    }
    TP ft = TP(0), gt = TP(0);
    contravariant_gradient<K, TP>(active, el, ij, g, b, s_f[lei], s_tv[lei], s_com[lei], s_cg[lei], s_a[lei],
                                  s_b[lei], s_fb[lei], ft, gt);
    if (active) {
        const int j = ij / K, i = ij % K, p = el * K2 + ij;
        const TP tx = ft + s_fb[le][0 * K + j] * b.R[i * 2 + 0] + s_fb[le][1 * K + j] * b.R[i * 2 + 1];
        const TP ty = gt + s_fb[le][2 * K + i] * b.R[j * 2 + 0] + s_fb[le][3 * K + i] * b.R[j * 2 + 1];
        const TP xx = g.xxi[p], xe = g.xeta[p], yx = g.yxi[p], ye = g.yeta[p], J = g.J[p];
        const TP dpdx = (tx * xx + ty * xe) / J;
        const TP dpdy = (tx * yx + ty * ye) / J;
        const TP u = dpdy, v = -dpdx;
        a.u[p] = T(u);
        a.v[p] = T(v);
        s_ux[le][ij] = T(u * ye - v * xe);   // contravariant volumetric fluxes J u.grad(xi), J u.grad(eta)
        s_uy[le][ij] = T(-u * yx + v * xx);
    }
    __syncthreads();
    if (active) {
        for (int o = ij; o < NF; o += K2) {
            const int ijp = o / K;
            T wv, wg;
            face_trace<K, T>(s_w[le], bw, o, wv, wg);
            a.w_tv[el * NF + o] = wv;
            a.w_tg[el * NF + o] = wg;
            a.U_t[el * NF + o] = face_value<K, T>(ijp < 2 ? s_ux[le] : s_uy[le], bw, o);
        }
    }
}

template <int K, typename T>
__global__ void __launch_bounds__(Shape<K>::THREADS) residual_kernel(FrGeom<T> g, DevBases<T> bp, BcArrays bc,
                                                                      ResidualArgs<T> a) {
    using S = Shape<K>;
    __shared__ DevBases<T> b;
    stage_bases(b, bp);
    constexpr int K2 = S::K2, NF = S::NF, EPB = S::EPB;
    __shared__ T s_f[EPB][K2], s_a[EPB][K2], s_b[EPB][K2], s_ux[EPB][K2], s_uy[EPB][K2];
    __shared__ T s_tv[EPB][NF], s_tg[EPB][NF], s_com[EPB][NF], s_cg[EPB][NF], s_fb[EPB][NF], s_ut[EPB][NF],
        s_up[EPB][NF];
    const int le = threadIdx.x / K2, ij = threadIdx.x % K2;
    const int el = blockIdx.x * EPB + le;
    const bool active = le < EPB && el < g.N;
    const int lei = active ? le : 0;
    const int j = ij / K, i = ij % K, p = el * K2 + ij;
    T xx = T(0), xe = T(0), yx = T(0), ye = T(0), J = T(1), w = T(0);
    if (active) {
        w = a.w[p];
        s_f[le][ij] = w;
        xx = g.xxi[p]; xe = g.xeta[p]; yx = g.yxi[p]; ye = g.yeta[p]; J = g.J[p];
        const T u = a.u[p], v = a.v[p];
        s_ux[le][ij] = u * ye - v * xe;
        s_uy[le][ij] = -u * yx + v * xx;
    }
    __syncthreads();
    if (active)
        for (int o = ij; o < NF; o += K2) {
            face_trace<K, T>(s_f[le], b, o, s_tv[le][o], s_tg[le][o]);
            s_ut[le][o] = face_value<K, T>((o / K) < 2 ? s_ux[le] : s_uy[le], b, o);
        }
    __syncthreads();
    // ---- diffusion
    face_common<K, T>(active, el, ij, g, b, a.w_tv, a.w_tg, s_tv[lei], s_tg[lei], s_com[lei], s_cg[lei], g.sw_d,
                      bc.bc_d, false);
    // BC_vorticity (src/HO_2D.cpp:2726-2727) and BC_advection (2219-2243) on boundary faces
    if (active) {
        for (int o = ij; o < NF; o += K2) {
            const int ijp = o / K, k = o % K;
            const int nb = g.face_nb[el * 4 + ijp];
            if (nb >= 0) continue;
            const int e = -nb - 1;
            const int be = e * K + bf_index<K>(side_of_ijp(ijp), k);
            const double wb = double(s_com[le][o]);
            bc.bc_w[be] = wb;
            const double adv = wb * bc.bc_nv[be] * double(g.fAn[(el * 4 + ijp) * K + k]);
            bc.bc_adv[be] = adv;
            s_up[le][o] = T(adv);
        }
    }
    T ft = T(0), gt = T(0);
    contravariant_gradient<K, T>(active, el, ij, g, b, s_f[lei], s_tv[lei], s_com[lei], s_cg[lei], s_a[lei],
                                 s_b[lei], s_fb[lei], ft, gt);
    T diff = T(0);
    if (active) {
        T lap = T(0);
#pragma unroll
        for (int d = 0; d < K; ++d) lap += s_a[le][j * K + d] * b.D[d * K + i];
        lap += s_fb[le][0 * K + j] * b.gR[i * 2 + 0] + s_fb[le][1 * K + j] * b.gR[i * 2 + 1];
#pragma unroll
        for (int d = 0; d < K; ++d) lap += s_b[le][d * K + i] * b.D[d * K + j];
        lap += s_fb[le][2 * K + i] * b.gR[j * 2 + 0] + s_fb[le][3 * K + i] * b.gR[j * 2 + 1];
        diff = lap * (T(a.re_inv) / J);
    }
    __syncthreads();  // s_a / s_b are reused below
    // ---- advection
    if (a.adv_type == 2) {
        // continuous volumetric flux: common flux on faces, Radau-corrected inside
        if (active)
            for (int o = ij; o < NF; o += K2) {
                const int ijp = o / K, k = o % K;
                const int nb = g.face_nb[el * 4 + ijp];
                T cvf;
                if (nb >= 0) {
                    const int nijp = g.face_nijp[el * 4 + ijp];
                    const int rev = (ijp + nijp - ijp / 2 - nijp / 2 + 1) % 2;
                    const int jn = rev ? K - 1 - k : k;
                    const T sign = T(2 * ((ijp + nijp) % 2) - 1);
                    cvf = T(0.5) * (s_ut[le][o] + sign * a.U_t[(nb * 4 + nijp) * K + jn]);
                    const T t = T(ijp % 2);
                    const T wn = a.w_tv[(nb * 4 + nijp) * K + jn];
                    s_up[le][o] = cvf > T(0) ? cvf * (t * s_tv[le][o] + (T(1) - t) * wn)
                                             : cvf * ((T(1) - t) * s_tv[le][o] + t * wn);
                } else {
                    const int e = -nb - 1;
                    cvf = T(bc.bc_nv[e * K + bf_index<K>(side_of_ijp(ijp), k)]) * g.fAn[(el * 4 + ijp) * K + k];
                }
                s_com[le][o] = cvf;  // reuse: common volumetric flux
            }
        __syncthreads();
        if (active) {
            const T cx = s_ux[le][ij] + (s_com[le][0 * K + j] - s_ut[le][0 * K + j]) * b.R[i * 2 + 0] +
                         (s_com[le][1 * K + j] - s_ut[le][1 * K + j]) * b.R[i * 2 + 1];
            const T cy = s_uy[le][ij] + (s_com[le][2 * K + i] - s_ut[le][2 * K + i]) * b.R[j * 2 + 0] +
                         (s_com[le][3 * K + i] - s_ut[le][3 * K + i]) * b.R[j * 2 + 1];
            s_a[le][ij] = cx * w;
            s_b[le][ij] = cy * w;
        }
    } else {
        if (active) {
            s_a[le][ij] = s_ux[le][ij] * w;
            s_b[le][ij] = s_uy[le][ij] * w;
            for (int o = ij; o < NF; o += K2) {
                const int ijp = o / K, k = o % K;
                const int nb = g.face_nb[el * 4 + ijp];
                if (nb < 0) continue;
                const int nijp = g.face_nijp[el * 4 + ijp];
                const int rev = (ijp + nijp - ijp / 2 - nijp / 2 + 1) % 2;
                const int jn = rev ? K - 1 - k : k;
                const int nq = (nb * 4 + nijp) * K + jn;
                const T sign = T(2 * ((ijp + nijp) % 2) - 1);
                const T wl = s_tv[le][o], wr = a.w_tv[nq];
                const T fl = s_ut[le][o] * wl, fr = a.U_t[nq] * wr;
                T up = T(0.5) * (fl + sign * fr);
                const T dw = wl - wr;
                if (fabs(double(dw)) > 1e-4) {  // upwind switch evaluated in double (src/HO_2D.cpp:2370)
                    const T av = (fl - sign * fr) / dw;
                    up += T(0.5) * T((ijp & 1) ? 1 : -1) * fabs(av) * dw;
                }
                s_up[le][o] = up;
            }
        }
    }
    __syncthreads();
    if (active)
        for (int o = ij; o < NF; o += K2) {
            const int ijp = o / K, k = o % K, lr = ijp & 1;
            T v = s_up[le][o];
            if (ijp < 2) {
#pragma unroll
                for (int m = 0; m < K; ++m) v -= s_a[le][k * K + m] * b.sbb[m * 2 + lr];
            } else {
#pragma unroll
                for (int m = 0; m < K; ++m) v -= s_b[le][m * K + k] * b.sbb[m * 2 + lr];
            }
            s_fb[le][o] = v;
        }
    __syncthreads();
    if (!active) return;
    T dv = T(0);
#pragma unroll
    for (int d = 0; d < K; ++d) dv += s_a[le][j * K + d] * b.D[d * K + i];
#pragma unroll
    for (int d = 0; d < K; ++d) dv += s_b[le][d * K + i] * b.D[d * K + j];
    dv += s_fb[le][0 * K + j] * b.gR[i * 2 + 0] + s_fb[le][1 * K + j] * b.gR[i * 2 + 1];
    dv += s_fb[le][2 * K + i] * b.gR[j * 2 + 0] + s_fb[le][3 * K + i] * b.gR[j * 2 + 1];
    const T adv = -dv / J;
    const T kk = T(a.dt) * (adv + diff);
    if (a.rhs_diff) a.rhs_diff[p] = diff;
    if (a.rhs_adv) a.rhs_adv[p] = adv;
    if (a.k_out) a.k_out[p] = kk;
    // ---- RK stage update (src/HO_2D.cpp:1465-1531), FP64 accumulation
    const double k = double(kk);
    if (a.ti_type == 0) return;  // stage only: no update
    double om = a.omega[p];
    if (a.ti_type == 1) {
        om += k;
        a.omega[p] = om;
        if (a.w_next) a.w_next[p] = T(om);
    } else if (a.ti_type == 2) {
        if (a.stage == 0) {
            a.acc[p] = k;
            a.w_next[p] = T(om + 1.0 * k);
        } else {
            om += 0.5 * (a.acc[p] + k);
            a.omega[p] = om;
            if (a.w_next) a.w_next[p] = T(om);
        }
    } else {
        if (a.stage == 0) {
            a.acc[p] = k;
            a.w_next[p] = T(om + 0.5 * k);
        } else if (a.stage == 1) {
            a.acc[p] = a.acc[p] + 2.0 * k;
            a.w_next[p] = T(om + 0.5 * k);
        } else if (a.stage == 2) {
            a.acc[p] = a.acc[p] + 2.0 * k;
            a.w_next[p] = T(om + 1.0 * k);
        } else {
            om += (a.acc[p] + k) / 6.0;
            a.omega[p] = om;
            if (a.w_next) a.w_next[p] = T(om);
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

template <typename T, typename TP>
cudaError_t launch_velocity(int K, const FrGeom<TP>& g, const DevBases<TP>& bp, const DevBases<T>& bw,
                            const BcArrays& bc, const VelocityArgs<T, TP>& a, cudaStream_t s) {
    HO2D_DISPATCH_K(K, (velocity_kernel<KK, T, TP><<<grid_for<KK>(g.N), Shape<KK>::THREADS, 0, s>>>(g, bp, bw, bc,
                                                                                                       a)));
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_residual(int K, const FrGeom<T>& g, const DevBases<T>& b, const BcArrays& bc,
                            const ResidualArgs<T>& a, cudaStream_t s) {
    HO2D_DISPATCH_K(K, (residual_kernel<KK, T><<<grid_for<KK>(g.N), Shape<KK>::THREADS, 0, s>>>(g, b, bc, a)));
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_poisson_rhs(int K, int N, const int* face_nb, const T* w, const T* J, const double* bsrc,
                               const double* bc_p, double* rhs, cudaStream_t s) {
    HO2D_DISPATCH_K(K, (poisson_rhs_kernel<KK, T><<<grid_for<KK>(N), Shape<KK>::THREADS, 0, s>>>(
                           N, face_nb, w, J, bsrc, bc_p, rhs)));
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
    template cudaError_t launch_velocity<T, double>(int, const FrGeom<double>&, const DevBases<double>&,         \
                                                    const DevBases<T>&, const BcArrays&,                          \
                                                    const VelocityArgs<T, double>&, cudaStream_t);                 \
    template cudaError_t launch_residual<T>(int, const FrGeom<T>&, const DevBases<T>&, const BcArrays&,           \
                                            const ResidualArgs<T>&, cudaStream_t);                                 \
    template cudaError_t launch_poisson_rhs<T>(int, int, const int*, const T*, const T*, const double*,           \
                                               const double*, double*, cudaStream_t);

HO2D_INSTANTIATE_FR(double)
HO2D_INSTANTIATE_FR(float)

}  // namespace ho2d
