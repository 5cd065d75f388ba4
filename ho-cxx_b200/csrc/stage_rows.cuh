// stage_rows.cuh -- the FR stage kernels (velocity from psi, vorticity residual with the RK
// update) in the row-parallel mapping of rows.cuh: K threads per element, thread t owns
// row t and column t of the element's K x K blocks and face point t of each of its four
// faces. The arithmetic is the reference's method-2 FR discretisation
// (calc_internal_comm_vals_meth2 / calc_boundary_comm_vals_meth2, calc_RHS_diffusion,
// calc_velocity_vector_from_streamfunction, calc_RHS_advection{,_continuous}:
// src/HO_2D.cpp:2666-2927, 3174-3366, 2245-2645), regrouped by rows and columns: xi passes
// along rows, eta passes down columns, warp-local transposes between.
#pragma once

#include "fr_device.cuh"
#include "rows.cuh"

namespace ho2d {

// Per-warp shared scratch of a stage kernel: the common values of each face (read by all
// K threads of the element for the cross derivatives), the Neumann right-hand sides, and
// three K x K transpose buffers.
template <int K, typename T>
struct StageScratch {
    T com[Rows<K>::EPW][4][K];
    T nr[Rows<K>::EPW][4][K];
    T tr[3][Rows<K>::EPW][K][K];
};

// This face point's neighbour data: the neighbour element (>= 0) or -(edge + 1), the
// neighbour's face, the orientation reversal and the neighbour's index of the point.
struct FacePt {
    int nb, nijp, rev, nq;
};

template <int K, typename T>
__device__ __forceinline__ void face_points(const FrGeom<T>& g, int el, int t, bool act, FacePt (&fp)[4]) {
#pragma unroll
    for (int f = 0; f < 4; ++f) {
        fp[f].nb = act ? g.face_nb[el * 4 + f] : -1;
        fp[f].nijp = 0;
        fp[f].rev = 0;
        fp[f].nq = 0;
        if (fp[f].nb >= 0) {
            const int nijp = g.face_nijp[el * 4 + f];
            const int rev = (f + nijp - f / 2 - nijp / 2 + 1) % 2;
            fp[f].nijp = nijp;
            fp[f].rev = rev;
            fp[f].nq = (fp[f].nb * 4 + nijp) * K + (rev ? K - 1 - t : t);
        }
    }
}

// Method-2 common values com[f] and common normal fluxes cg[f] at face point t of the four
// faces (src/HO_2D.cpp:2833-2927, the face-flux average of 2739-2743): interior faces
// average with the neighbour's own traces
// (tvg/tgg, [N][4][K]); Dirichlet boundary values come from bcv, Neumann ones through the
// precomputed inverse of the face's common-value system (FrGeom::nminv); neu_sign
// multiplies Neumann values by the h-direction sign (the psi case). Leaves every face's
// common values in sm.com. Warp-collective.
template <int K, typename T>
__device__ __forceinline__ void row_face_common(const FrGeom<T>& g, const DevBases<T>& b, int el, int t, int lw,
                                                bool act, const FacePt (&fp)[4], const T* __restrict__ tvg,
                                                const T* __restrict__ tgg, const T (&tv)[4], const T (&tg)[4],
                                                const int* __restrict__ sw, const double* __restrict__ bcv,
                                                bool neu_sign, StageScratch<K, T>& sm, T (&com)[4], T (&cg)[4],
                                                T (&ntv)[4], T (&ntg)[4]) {
    bool neu[4];
    bool any_neu = false;
#pragma unroll
    for (int f = 0; f < 4; ++f) {
        neu[f] = false;
        com[f] = T(0);
        cg[f] = T(0);
        ntv[f] = ntg[f] = T(0);
        if (!act) continue;
        const int nb = fp[f].nb;
        if (nb >= 0) {
            ntv[f] = tvg[fp[f].nq];
            ntg[f] = tgg[fp[f].nq];
            com[f] = T(0.5) * (tv[f] + ntv[f]);
        } else {
            const int e = -nb - 1;
            const int bi = e * K + bf_index<K>(side_of_ijp(f), t);
            if (sw[e] == kDirichlet) {
                com[f] = T(bcv[bi]);
            } else {
                neu[f] = true;
                const int q = (el * 4 + f) * K + t;
                const T sgn = neu_sign ? T(2 * (f % 2) - 1) : T(1);
                cg[f] = sgn * T(bcv[bi]) * g.fAn[q];
                sm.nr[lw][f][t] = cg[f] - g.fA[q] / g.fJ[q] * (tg[f] - tv[f] * b.gp[f & 1]);
            }
        }
        any_neu |= neu[f];
    }
    if (__any_sync(0xffffffffu, any_neu)) {
        __syncwarp();
#pragma unroll
        for (int f = 0; f < 4; ++f) {
            if (!neu[f]) continue;
            const T* mi = g.nminv + ((size_t)(-fp[f].nb - 1) * K + t) * K;
            T acc = T(0);
#pragma unroll
            for (int m = 0; m < K; ++m) acc += mi[m] * sm.nr[lw][f][m];
            com[f] = acc;
        }
    }
    if (act) {
#pragma unroll
        for (int f = 0; f < 4; ++f) sm.com[lw][f][t] = com[f];
    }
    __syncwarp();
    T Dc[K], Dr[K];  // column t and column K-1-t of D (thread-dependent basis entries)
#pragma unroll
    for (int m = 0; m < K; ++m) {
        Dc[m] = b.D[m * K + t];
        Dr[m] = b.D[m * K + (K - 1 - t)];
    }
#pragma unroll
    for (int f = 0; f < 4; ++f) {
        if (!act || neu[f]) continue;
        T cm[K];
#pragma unroll
        for (int m = 0; m < K; ++m) cm[m] = sm.com[lw][f][m];
        T cross = T(0);
#pragma unroll
        for (int m = 0; m < K; ++m) cross += cm[m] * Dc[m];
        const int q = (el * 4 + f) * K + t;
        const T dv = tg[f] + (com[f] - tv[f]) * b.gp[f & 1];
        const T fl = (dv * g.fA[q] - cross * g.fB[q]) / g.fJ[q];
        if (fp[f].nb < 0) {
            cg[f] = fl;
            continue;
        }
        T crn = cross;
        if (fp[f].rev) {
            crn = T(0);
#pragma unroll
            for (int m = 0; m < K; ++m) crn += cm[K - 1 - m] * Dr[m];
        }
        const int nq = fp[f].nq, nijp = fp[f].nijp;
        const T gpn = (nijp & 1) ? b.gp[1] : b.gp[0];
        const T dvn = ntg[f] + (com[f] - ntv[f]) * gpn;
        const T fln = (dvn * g.fA[nq] - crn * g.fB[nq]) / g.fJ[nq];
        cg[f] = T(0.5) * (fl + T(2 * ((f + nijp) % 2) - 1) * fln);
    }
}

// Contravariant gradient (src/HO_2D.cpp:2775-2803): f~ = (f_xi g11 + f_eta g12) along row
// t and g~ = (f_eta g22 + f_xi g12) down column t of the element's field (rows fr, columns
// fc), with the Radau corrections of the own face points, and the flux jumps fb[f] of face
// point t (common flux minus the interior flux extrapolated to it). g11 = (x_eta^2 +
// y_eta^2) / J, g12 = -(x_xi x_eta + y_xi y_eta) / J, g22 = (x_xi^2 + y_xi^2) / J are the
// Poisson operator's metric coefficients (PoisGeom), at row t (g11r, g12r) and column t
// (g22c, g12c). Warp-collective.
template <int K, typename T>
__device__ __forceinline__ void row_contravariant(const DevBases<T>& b, const T (&fr)[K], const T (&fc)[K],
                                                  const T (&tv)[4], const T (&com)[4], const T (&cg)[4],
                                                  const T* __restrict__ G11, const T* __restrict__ G12,
                                                  const T* __restrict__ G22, size_t e2, T (&bufa)[K][K],
                                                  T (&bufb)[K][K], int t, bool act, T (&ft)[K], T (&gt)[K],
                                                  T (&fb)[4]) {
    T dx[K], de[K];
#pragma unroll
    for (int i = 0; i < K; ++i) {
        T s = T(0);
#pragma unroll
        for (int d = 0; d < K; ++d) s += fr[d] * b.D[d * K + i];
        s += (com[0] - tv[0]) * b.gR[i * 2 + 0];
        s += (com[1] - tv[1]) * b.gR[i * 2 + 1];
        dx[i] = s;
    }
#pragma unroll
    for (int j = 0; j < K; ++j) {
        T s = T(0);
#pragma unroll
        for (int d = 0; d < K; ++d) s += fc[d] * b.D[d * K + j];
        s += (com[2] - tv[2]) * b.gR[j * 2 + 0];
        s += (com[3] - tv[3]) * b.gR[j * 2 + 1];
        de[j] = s;
    }
    T der[K], dxc[K];
    col_to_row<K, T>(bufa, de, der, t, act);
    rows_to_col<K, T>(bufb, dx, dxc, t, act);
    T g11[K], g12r[K], g22[K], g12c[K];
    if (act) {
        load_row<K, T>(G11 + e2 + t * K, g11);
        load_row<K, T>(G12 + e2 + t * K, g12r);
        load_col<K, T>(G22 + e2 + t, g22);
        load_col<K, T>(G12 + e2 + t, g12c);
    } else {
#pragma unroll
        for (int i = 0; i < K; ++i) g11[i] = g12r[i] = g22[i] = g12c[i] = T(0);
    }
#pragma unroll
    for (int i = 0; i < K; ++i) {
        ft[i] = dx[i] * g11[i] + der[i] * g12r[i];
        gt[i] = de[i] * g22[i] + dxc[i] * g12c[i];
    }
#pragma unroll
    for (int f = 0; f < 4; ++f) {
        T v = cg[f];
        if (f < 2) {
#pragma unroll
            for (int d = 0; d < K; ++d) v -= ft[d] * b.sbb[d * 2 + (f & 1)];
        } else {
#pragma unroll
            for (int d = 0; d < K; ++d) v -= gt[d] * b.sbb[d * 2 + (f & 1)];
        }
        fb[f] = v;
    }
}

// velocity_kernel by rows (psi and everything derived from it in TP, omega and the outputs
// in T): corrected grad psi, u = dpsi/dy, v = -dpsi/dx, the boundary side outputs
// (velocity_jump, BC_normal_vel, the no-slip diffusion BC) and the omega and
// contravariant-flux face traces the residual kernel gathers.
// (FP32 stage: at most 128 registers, four CTAs per SM)
template <int K, typename T, typename TP>
__global__ void __launch_bounds__(Rows<K>::THREADS, sizeof(T) == 4 ? 4 : 1)
    velocity_rows(FrGeom<TP> g, const TP* __restrict__ G11, const TP* __restrict__ G12, const TP* __restrict__ G22,
                  DevBases<TP> b, DevBases<T> bw, BcArrays bc, VelocityArgs<T, TP> a) {
    __shared__ StageScratch<K, TP> sm[Rows<K>::WARPS];
    __shared__ T wbuf[Rows<K>::WARPS][Rows<K>::EPW][K][K];
    const RowIdx<K> ix(g.N, blockIdx.x);
    const int t = ix.t, lw = ix.lw, el = ix.el;
    const bool act = ix.active;
    StageScratch<K, TP>& S = sm[ix.warp];
    const size_t e2 = (size_t)(act ? el : 0) * K * K;
    TP pr[K], pc[K];
    FacePt fp[4];
    face_points<K, TP>(g, el, t, act, fp);
    if (act) {
        load_row<K, TP>(a.psi + e2 + t * K, pr);
        load_col<K, TP>(a.psi + e2 + t, pc);
    } else {
#pragma unroll
        for (int i = 0; i < K; ++i) pr[i] = pc[i] = TP(0);
    }
    TP tv[4], tg[4], com[4], cg[4], ntv[4], ntg[4];
    row_traces<K, TP>(b, pr, pc, tv, tg);
    row_face_common<K, TP>(g, b, el, t, lw, act, fp, a.psi_tv, a.psi_tg, tv, tg, g.sw_p, bc.bc_p, true, S, com,
                           cg, ntv, ntg);
    // boundary side outputs: velocity_jump / BC_normal_vel, then the no-slip diffusion BC
    if (act) {
#pragma unroll
        for (int f = 0; f < 4; ++f) {
            const int nb = fp[f].nb;
            if (nb >= 0) continue;
            const int e = -nb - 1;
            const int be = e * K + bf_index<K>(side_of_ijp(f), t);
            const int q = (el * 4 + f) * K + t;
            double vj = bc.vjump[be];
            if (g.sw_p[e] == kDirichlet) {
                vj = double(cg[f]) / double(g.fAn[q]);
            } else {
                const TP vsign = TP(1 - 2 * (f / 2));
                TP nv = TP(0);
#pragma unroll
                for (int d = 0; d < K; ++d) nv += vsign * S.com[lw][f][d] * b.D[d * K + t];
                bc.bc_nv[be] = double(nv / g.fAn[q]);
            }
            if (g.noslip[g.be_group[e]]) {
                vj += double(2 * (f % 2) - 1) * bc.bc_pv[be];
                bc.bc_d[be] = vj / (a.dt * a.re_inv);
            }
            bc.vjump[be] = vj;
        }
    }
    TP ft[K], gt[K], fb[4];
    row_contravariant<K, TP>(b, pr, pc, tv, com, cg, G11, G12, G22, e2, S.tr[0][lw], S.tr[1][lw], t, act, ft, gt,
                             fb);
    // d psi / d xi along row t, d psi / d eta down column t (to rows), then u, v at row t
    TP tyc[K], ty[K];
#pragma unroll
    for (int j = 0; j < K; ++j) tyc[j] = gt[j] + fb[2] * b.R[j * 2 + 0] + fb[3] * b.R[j * 2 + 1];
    __syncwarp();  // tr[0] was read by row_contravariant's transposes
    col_to_row<K, TP>(S.tr[0][lw], tyc, ty, t, act);
    TP xx[K], xe[K], yx[K], ye[K], J[K];
    if (act) {
        load_row<K, TP>(g.xxi + e2 + t * K, xx);
        load_row<K, TP>(g.xeta + e2 + t * K, xe);
        load_row<K, TP>(g.yxi + e2 + t * K, yx);
        load_row<K, TP>(g.yeta + e2 + t * K, ye);
        load_row<K, TP>(g.J + e2 + t * K, J);
    } else {
#pragma unroll
        for (int i = 0; i < K; ++i) {
            xx[i] = xe[i] = yx[i] = ye[i] = TP(0);
            J[i] = TP(1);
        }
    }
    T ur[K], vr[K], U[K], V[K];
#pragma unroll
    for (int i = 0; i < K; ++i) {
        const TP tx = ft[i] + fb[0] * b.R[i * 2 + 0] + fb[1] * b.R[i * 2 + 1];
        const TP dpdx = (tx * xx[i] + ty[i] * xe[i]) / J[i];
        const TP dpdy = (tx * yx[i] + ty[i] * ye[i]) / J[i];
        const TP u = dpdy, v = -dpdx;
        ur[i] = T(u);
        vr[i] = T(v);
        U[i] = T(u * ye[i] - v * xe[i]);  // contravariant volumetric fluxes J u.grad(xi), J u.grad(eta)
        V[i] = T(-u * yx[i] + v * xx[i]);
    }
    if (act) {
        store_row<K, T>(a.u + e2 + t * K, ur);
        store_row<K, T>(a.v + e2 + t * K, vr);
    }
    // omega traces and the flux traces: U^xi on W/E from row t, U^eta on S/N from column t
    T Vc[K];
    rows_to_col<K, T>(wbuf[ix.warp][lw], V, Vc, t, act);
    T wr[K], wc[K];
    if (act) {
        load_row<K, T>(a.w + e2 + t * K, wr);
        load_col<K, T>(a.w + e2 + t, wc);
        T wtv[4], wtg[4];
        row_traces<K, T>(bw, wr, wc, wtv, wtg);
        T ut[4];
#pragma unroll
        for (int f = 0; f < 4; ++f) {
            T s = T(0);
            if (f < 2) {
#pragma unroll
                for (int m = 0; m < K; ++m) s += U[m] * bw.sbb[m * 2 + (f & 1)];
            } else {
#pragma unroll
                for (int m = 0; m < K; ++m) s += Vc[m] * bw.sbb[m * 2 + (f & 1)];
            }
            ut[f] = s;
        }
#pragma unroll
        for (int f = 0; f < 4; ++f) {
            const int q = (el * 4 + f) * K + t;
            a.w_tv[q] = wtv[f];
            a.w_tg[q] = wtg[f];
            a.U_t[q] = ut[f];
        }
    }
}

// residual_kernel by rows: Re^-1 Lap(omega) with BC_vorticity and BC_advection, the
// advective divergence (type 1: discontinuous flux with the upwind switch; type 2:
// continuous volumetric flux), k = dt (adv + diff) and the RK update
// (src/HO_2D.cpp:1465-1531, 2219-2645, 2666-2927).
// (FP32: at most 96 registers, five CTAs per SM)
template <int K, typename T>
__global__ void __launch_bounds__(Rows<K>::THREADS, sizeof(T) == 4 ? 5 : 1)
    residual_rows(FrGeom<T> g, const T* __restrict__ G11, const T* __restrict__ G12, const T* __restrict__ G22,
                  DevBases<T> b, BcArrays bc, ResidualArgs<T> a) {
    __shared__ StageScratch<K, T> sm[Rows<K>::WARPS];
    const RowIdx<K> ix(g.N, blockIdx.x);
    const int t = ix.t, lw = ix.lw, el = ix.el;
    const bool act = ix.active;
    StageScratch<K, T>& S = sm[ix.warp];
    const size_t e2 = (size_t)(act ? el : 0) * K * K;
    T wr[K], wc[K], Jr[K];
    FacePt fp[4];
    face_points<K, T>(g, el, t, act, fp);
    if (act) {
        load_row<K, T>(a.w + e2 + t * K, wr);
        load_col<K, T>(a.w + e2 + t, wc);
        load_row<K, T>(g.J + e2 + t * K, Jr);
    } else {
#pragma unroll
        for (int i = 0; i < K; ++i) {
            wr[i] = wc[i] = T(0);
            Jr[i] = T(1);
        }
    }
    T tv[4], tg[4];
    row_traces<K, T>(b, wr, wc, tv, tg);
    // ---- diffusion
    T com[4], cg[4], ntv[4], ntg[4];
    row_face_common<K, T>(g, b, el, t, lw, act, fp, a.w_tv, a.w_tg, tv, tg, g.sw_d, bc.bc_d, false, S, com, cg,
                          ntv, ntg);
    // BC_vorticity (src/HO_2D.cpp:2726-2727) and BC_advection (2219-2243) on boundary faces
    T up[4] = {T(0), T(0), T(0), T(0)};
    if (act) {
#pragma unroll
        for (int f = 0; f < 4; ++f) {
            const int nb = fp[f].nb;
            if (nb >= 0) continue;
            const int e = -nb - 1;
            const int be = e * K + bf_index<K>(side_of_ijp(f), t);
            const double wb = double(com[f]);
            bc.bc_w[be] = wb;
            const double adv = wb * bc.bc_nv[be] * double(g.fAn[(el * 4 + f) * K + t]);
            bc.bc_adv[be] = adv;
            up[f] = T(adv);
        }
    }
    T ft[K], gt[K], fb[4];
    row_contravariant<K, T>(b, wr, wc, tv, com, cg, G11, G12, G22, e2, S.tr[0][lw], S.tr[1][lw], t, act, ft, gt,
                            fb);
    // Laplacian: xi part along row t; eta part down column t, moved to rows
    T lc[K], lcr[K];
#pragma unroll
    for (int j = 0; j < K; ++j) {
        T s = T(0);
#pragma unroll
        for (int d = 0; d < K; ++d) s += gt[d] * b.D[d * K + j];
        s += fb[2] * b.gR[j * 2 + 0] + fb[3] * b.gR[j * 2 + 1];
        lc[j] = s;
    }
    col_to_row<K, T>(S.tr[2][lw], lc, lcr, t, act);
    T diff[K];
#pragma unroll
    for (int i = 0; i < K; ++i) {
        T s = T(0);
#pragma unroll
        for (int d = 0; d < K; ++d) s += ft[d] * b.D[d * K + i];
        s += fb[0] * b.gR[i * 2 + 0] + fb[1] * b.gR[i * 2 + 1];
        diff[i] = (s + lcr[i]) * (T(a.re_inv) / Jr[i]);
    }
    // ---- advection: contravariant volumetric fluxes U^xi = u y_eta - v x_eta along row t and
    // U^eta = -u y_xi + v x_xi down column t, their face values, and the fluxes
    // a = U^xi w along row t, b = U^eta w down column t
    T Ur[K], Vc[K];
    if (act) {
        T ur[K], vr[K], xe[K], ye[K];
        load_row<K, T>(a.u + e2 + t * K, ur);
        load_row<K, T>(a.v + e2 + t * K, vr);
        load_row<K, T>(g.xeta + e2 + t * K, xe);
        load_row<K, T>(g.yeta + e2 + t * K, ye);
#pragma unroll
        for (int i = 0; i < K; ++i) Ur[i] = ur[i] * ye[i] - vr[i] * xe[i];
        T uc[K], vc[K], xx[K], yx[K];
        load_col<K, T>(a.u + e2 + t, uc);
        load_col<K, T>(a.v + e2 + t, vc);
        load_col<K, T>(g.xxi + e2 + t, xx);
        load_col<K, T>(g.yxi + e2 + t, yx);
#pragma unroll
        for (int j = 0; j < K; ++j) Vc[j] = -uc[j] * yx[j] + vc[j] * xx[j];
    } else {
#pragma unroll
        for (int i = 0; i < K; ++i) Ur[i] = Vc[i] = T(0);
    }
    T ut[4];
#pragma unroll
    for (int f = 0; f < 4; ++f) {
        T s = T(0);
        if (f < 2) {
#pragma unroll
            for (int m = 0; m < K; ++m) s += Ur[m] * b.sbb[m * 2 + (f & 1)];
        } else {
#pragma unroll
            for (int m = 0; m < K; ++m) s += Vc[m] * b.sbb[m * 2 + (f & 1)];
        }
        ut[f] = s;
    }
    T fa_[K], fb_[K];
    if (a.adv_type == 2) {
        // continuous volumetric flux: common flux on faces, Radau-corrected inside
        T cvf[4];
#pragma unroll
        for (int f = 0; f < 4; ++f) {
            cvf[f] = T(0);
            if (!act) continue;
            const int nb = fp[f].nb;
            if (nb >= 0) {
                const int nq = fp[f].nq, nijp = fp[f].nijp;
                const T sign = T(2 * ((f + nijp) % 2) - 1);
                cvf[f] = T(0.5) * (ut[f] + sign * a.U_t[nq]);
                const T tt = T(f % 2);
                const T wn = a.w_tv[nq];
                up[f] = cvf[f] > T(0) ? cvf[f] * (tt * tv[f] + (T(1) - tt) * wn)
                                      : cvf[f] * ((T(1) - tt) * tv[f] + tt * wn);
            } else {
                const int e = -nb - 1;
                cvf[f] = T(bc.bc_nv[e * K + bf_index<K>(side_of_ijp(f), t)]) * g.fAn[(el * 4 + f) * K + t];
            }
        }
#pragma unroll
        for (int i = 0; i < K; ++i) {
            fa_[i] = (Ur[i] + (cvf[0] - ut[0]) * b.R[i * 2 + 0] + (cvf[1] - ut[1]) * b.R[i * 2 + 1]) * wr[i];
            fb_[i] = (Vc[i] + (cvf[2] - ut[2]) * b.R[i * 2 + 0] + (cvf[3] - ut[3]) * b.R[i * 2 + 1]) * wc[i];
        }
    } else {
#pragma unroll
        for (int i = 0; i < K; ++i) {
            fa_[i] = Ur[i] * wr[i];
            fb_[i] = Vc[i] * wc[i];
        }
#pragma unroll
        for (int f = 0; f < 4; ++f) {
            if (!act || fp[f].nb < 0) continue;
            const int nq = fp[f].nq, nijp = fp[f].nijp;
            const T sign = T(2 * ((f + nijp) % 2) - 1);
            const T wl = tv[f], wrr = a.w_tv[nq];
            const T fl = ut[f] * wl, fr = a.U_t[nq] * wrr;
            T u = T(0.5) * (fl + sign * fr);
            const T dw = wl - wrr;
            if (fabs(double(dw)) > 1e-4) {  // upwind switch evaluated in double (src/HO_2D.cpp:2370)
                const T av = (fl - sign * fr) / dw;
                u += T(0.5) * T((f & 1) ? 1 : -1) * fabs(av) * dw;
            }
            up[f] = u;
        }
    }
    // flux jumps and the divergence: xi part along row t, eta part down column t
    T jb[4];
#pragma unroll
    for (int f = 0; f < 4; ++f) {
        T v = up[f];
        if (f < 2) {
#pragma unroll
            for (int m = 0; m < K; ++m) v -= fa_[m] * b.sbb[m * 2 + (f & 1)];
        } else {
#pragma unroll
            for (int m = 0; m < K; ++m) v -= fb_[m] * b.sbb[m * 2 + (f & 1)];
        }
        jb[f] = v;
    }
    T dc[K], dcr[K];
#pragma unroll
    for (int j = 0; j < K; ++j) {
        T s = T(0);
#pragma unroll
        for (int d = 0; d < K; ++d) s += fb_[d] * b.D[d * K + j];
        s += jb[2] * b.gR[j * 2 + 0] + jb[3] * b.gR[j * 2 + 1];
        dc[j] = s;
    }
    __syncwarp();  // tr[2] was read above
    col_to_row<K, T>(S.tr[2][lw], dc, dcr, t, act);
    if (!act) return;
    T adv[K], kk[K];
#pragma unroll
    for (int i = 0; i < K; ++i) {
        T s = T(0);
#pragma unroll
        for (int d = 0; d < K; ++d) s += fa_[d] * b.D[d * K + i];
        s += jb[0] * b.gR[i * 2 + 0] + jb[1] * b.gR[i * 2 + 1];
        adv[i] = -(s + dcr[i]) / Jr[i];
        kk[i] = T(a.dt) * (adv[i] + diff[i]);
    }
    const size_t p = e2 + t * K;
    if (a.rhs_diff) store_row<K, T>(a.rhs_diff + p, diff);
    if (a.rhs_adv) store_row<K, T>(a.rhs_adv + p, adv);
    if (a.k_out) store_row<K, T>(a.k_out + p, kk);
    // ---- RK stage update (src/HO_2D.cpp:1465-1531), FP64 accumulation
    if (a.ti_type == 0) return;  // stage only: no update
#pragma unroll
    for (int i = 0; i < K; ++i) {
        const double k = double(kk[i]);
        const size_t q = p + i;
        double om = a.omega[q];
        if (a.ti_type == 1) {
            om += k;
            a.omega[q] = om;
            if (a.w_next) a.w_next[q] = T(om);
        } else if (a.ti_type == 2) {
            if (a.stage == 0) {
                a.acc[q] = k;
                const double wn = om + 1.0 * k;
                a.w_next[q] = T(wn);
                if (a.w_next64) a.w_next64[q] = wn;
            } else {
                om += 0.5 * (a.acc[q] + k);
                a.omega[q] = om;
                if (a.w_next) a.w_next[q] = T(om);
            }
        } else {
            if (a.stage < 3) {
                a.acc[q] = a.stage == 0 ? k : a.acc[q] + 2.0 * k;
                const double wn = om + (a.stage == 2 ? 1.0 : 0.5) * k;
                a.w_next[q] = T(wn);
                if (a.w_next64) a.w_next64[q] = wn;
            } else {
                om += (a.acc[q] + k) / 6.0;
                a.omega[q] = om;
                if (a.w_next) a.w_next[q] = T(om);
            }
        }
    }
}

}  // namespace ho2d
