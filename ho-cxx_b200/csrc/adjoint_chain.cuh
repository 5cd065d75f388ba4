// adjoint_chain.cuh -- element bodies of the discrete adjoint of one FR stage.
//
// Per element, the forward stage (fr_kernels.cu, fr_device.cuh) is a chain of small
// linear maps between the element's point values, its face traces and the traces of its
// neighbours; only the advective upwind flux is nonlinear, and it is linear in the two
// face fluxes once the sign of its wave speed is fixed. These bodies run the chain
// backwards for one element: the transpose of every step, in reverse order, with the
// advective flux linearised at the forward stage's values. A neighbour's traces are
// inputs of an element's forward chain, so their adjoints are outputs here: each body
// writes them into the incoming slot of the neighbour's face point they came from, and
// a later launch adds a slot to that neighbour's own trace adjoints (gather_body).
//
// Every body is written once for two callers: the GPU kernels of adjoint.cu, where the
// K^2 threads of an element share each loop (tid = ij, nt = K^2, sync = __syncthreads),
// and a host build with one thread per element (tid = 0, nt = 1, sync = nothing) that
// checks the bodies against complex-step derivatives of the oracle without a GPU. A body
// is called by every thread of the CTA (it synchronises); `active` masks the threads
// without an element.
//
// Notation: the forward maps are those of calc_RHS_diffusion and the method-2 common
// values (src/HO_2D.cpp:2666-2927), calc_velocity_vector_from_streamfunction
// (3174-3366), update_diffusion_BC (2647-2664), update_advection_BC (2219-2243) and
// calc_RHS_advection (2245-2437); lam_x is the adjoint of x.
#pragma once

#include <cmath>

#include "device.cuh"
#include "elem_ctx.cuh"

namespace ho2d {

// Elements per CTA of the adjoint kernels: at most 128 threads, so that the per-element
// scratch below stays inside the static shared-memory limit for every K <= 8.
template <int K>
struct AShape {
    static constexpr int K2 = K * K, NF = 4 * K;
    static constexpr int EPB = (128 / K2) > 16 ? 16 : ((128 / K2) > 0 ? (128 / K2) : 1);
    static constexpr int THREADS = ((EPB * K2 + 31) / 32) * 32;
};

template <typename T>
HO2D_HD T adj_abs(T x) {
    return x < T(0) ? -x : x;
}

// boundary flux-point index (side/2)(K-2k-1)+k and the ijp -> side map (src/MathHelpers.hpp:23-24)
template <int K>
HO2D_HD int adj_bf(int ijp, int k) {
    const int side = ijp == 0 ? 3 : (ijp == 1 ? 1 : (ijp == 2 ? 0 : 2));
    return (side / 2) * (K - 2 * k - 1) + k;
}

// face point of the neighbour that meets face point (ijp, k) of element el
template <int K, typename T>
HO2D_HD int adj_neighbour_point(const FrGeom<T>& g, int el, int ijp, int k, int nb, int* nijp_out, int* rev_out) {
    const int nijp = g.face_nijp[el * 4 + ijp];
    const int rev = (ijp + nijp - ijp / 2 - nijp / 2 + 1) % 2;
    if (nijp_out) *nijp_out = nijp;
    if (rev_out) *rev_out = rev;
    return (nb * 4 + nijp) * K + (rev ? K - 1 - k : k);
}

// ---------------------------------------------------------------- FR Laplacian chain
// Scratch of one element for lap_adjoint. Entries marked "seed" are set by the caller
// (zero when there is no seed) and synchronised before the call.
template <int K, typename T>
struct LapAdjScratch {
    static constexpr int K2 = K * K, NF = 4 * K;
    T L[K2];             // lam of the raw Laplacian J Lap(f) at the points (lap mode)
    T la[K2], lb[K2];    // lam of f~, g~ (seed)
    T ldx[K2], lde[K2];  // lam of the xi / eta derivatives
    T lf[K2];            // result: lam of f, own traces included
    T lfb[NF];           // lam of the face corrections fB/gB (seed)
    T lcg[NF];           // lam of the common normal fluxes (seed)
    T lcom[NF];          // lam of the common values (seed)
    T ltv[NF], ltg[NF];  // lam of the element's own traces (value, normal derivative)
    T lcr[NF], lcrn[NF]; // lam of the cross derivatives on this side / the neighbour's side
    T ntv[NF], ntg[NF];  // result: lam of the neighbour's traces at each face point
    T lbcv[NF];          // result: lam of the boundary values (Dirichlet value or Neumann flux)
};

// Reverse of the forward method-2 common values and fluxes, the contravariant gradient
// and (when use_lap) the Laplacian of one element (row_face_common, row_contravariant and
// residual_rows in stage_rows.cuh; src/HO_2D.cpp:2666-2927), with boundary switches sw. Result in s.lf, s.ntv, s.ntg,
// s.lbcv. Boundary values do not enter the transposed map (it is linear in f); their
// adjoints come out in s.lbcv.
template <int K, typename T, class C>
HO2D_HD void lap_adjoint(const C& c, bool active, int el, const FrGeom<T>& g, const DevBases<T>& b, const int* sw,
                         bool neu_sign, bool use_lap, LapAdjScratch<K, T>& s) {
    constexpr int K2 = K * K, NF = 4 * K;
    // (1) Laplacian = sum f~ D + sum g~ D + Radau lifts of the face corrections
    if (active && use_lap) {
        for (int o = c.tid; o < NF; o += C::nt) {
            const int ijp = o / K, k = o % K, lr = ijp & 1;
            T acc = T(0);
            if (ijp < 2)
                for (int i = 0; i < K; ++i) acc += s.L[k * K + i] * b.gR[i * 2 + lr];
            else
                for (int j = 0; j < K; ++j) acc += s.L[j * K + k] * b.gR[j * 2 + lr];
            s.lfb[o] += acc;
        }
        for (int ij = c.tid; ij < K2; ij += C::nt) {
            const int hi = ij / K, lo = ij % K;
            T aa = T(0), bb = T(0);
            for (int q = 0; q < K; ++q) {
                aa += s.L[hi * K + q] * b.D[lo * K + q];  // f~ at (j, d) -> Lap at (j, i)
                bb += s.L[q * K + lo] * b.D[hi * K + q];  // g~ at (d, i) -> Lap at (j, i)
            }
            s.la[ij] += aa;
            s.lb[ij] += bb;
        }
    }
    c.sync();
    // (2) fB = cg - f~ extrapolated, gB = cg - g~ extrapolated; f~, g~ from the derivatives
    if (active) {
        for (int o = c.tid; o < NF; o += C::nt) s.lcg[o] += s.lfb[o];
        for (int ij = c.tid; ij < K2; ij += C::nt) {
            const int hi = ij / K, lo = ij % K;
            const T aa = s.la[ij] - s.lfb[0 * K + hi] * b.sbb[lo * 2 + 0] - s.lfb[1 * K + hi] * b.sbb[lo * 2 + 1];
            const T bb = s.lb[ij] - s.lfb[2 * K + lo] * b.sbb[hi * 2 + 0] - s.lfb[3 * K + lo] * b.sbb[hi * 2 + 1];
            const int p = el * K2 + ij;
            const T xx = g.xxi[p], xe = g.xeta[p], yx = g.yxi[p], ye = g.yeta[p], J = g.J[p];
            const T c1 = xe * xe + ye * ye, c2 = xx * xe + yx * ye, c3 = xx * xx + yx * yx;
            s.ldx[ij] = (aa * c1 - bb * c2) / J;
            s.lde[ij] = (bb * c3 - aa * c2) / J;
        }
    }
    c.sync();
    // (3) derivatives -> f, common values and own traces; corrected normal fluxes
    if (active) {
        for (int ij = c.tid; ij < K2; ij += C::nt) {
            const int hi = ij / K, lo = ij % K;
            T acc = T(0);
            for (int q = 0; q < K; ++q) {
                acc += s.ldx[hi * K + q] * b.D[lo * K + q];
                acc += s.lde[q * K + lo] * b.D[hi * K + q];
            }
            s.lf[ij] = acc;
        }
        for (int o = c.tid; o < NF; o += C::nt) {
            const int ijp = o / K, k = o % K, lr = ijp & 1;
            T x = T(0);
            if (ijp < 2)
                for (int i = 0; i < K; ++i) x += s.ldx[k * K + i] * b.gR[i * 2 + lr];
            else
                for (int j = 0; j < K; ++j) x += s.lde[j * K + k] * b.gR[j * 2 + lr];
            T lcom = s.lcom[o] + x;
            T ltv = -x, ltg = T(0), lcr = T(0), lcrn = T(0), ntv = T(0), ntg = T(0);
            const int nb = g.face_nb[el * 4 + ijp];
            const bool neu = nb < 0 && sw[-nb - 1] == kNeumann;
            if (!neu) {
                const int q = (el * 4 + ijp) * K + k;
                const T lcg = s.lcg[o];
                T lfl = lcg, lfln = T(0);
                int nq = 0, nijp = 0;
                if (nb >= 0) {
                    nq = adj_neighbour_point<K, T>(g, el, ijp, k, nb, &nijp, nullptr);
                    const T sign = T(2 * ((ijp + nijp) % 2) - 1);
                    lfl = T(0.5) * lcg;
                    lfln = T(0.5) * sign * lcg;
                }
                // fl = (dv fA - cross fB) / fJ,  dv = tg + (com - tv) g'
                const T ldv = lfl * g.fA[q] / g.fJ[q];
                lcr = -lfl * g.fB[q] / g.fJ[q];
                ltg += ldv;
                lcom += ldv * b.gp[lr];
                ltv -= ldv * b.gp[lr];
                if (nb >= 0) {
                    const T ldvn = lfln * g.fA[nq] / g.fJ[nq];
                    lcrn = -lfln * g.fB[nq] / g.fJ[nq];
                    ntg = ldvn;
                    ntv = -ldvn * b.gp[nijp & 1];
                    lcom += ldvn * b.gp[nijp & 1];
                }
            }
            s.lcom[o] = lcom;
            s.ltv[o] = ltv;
            s.ltg[o] = ltg;
            s.lcr[o] = lcr;
            s.lcrn[o] = lcrn;
            s.ntv[o] = ntv;
            s.ntg[o] = ntg;
        }
    }
    c.sync();
    // (4) cross derivatives sum_m com[m] D[m][k] on both sides of a face -> common values
    if (active) {
        for (int o = c.tid; o < NF; o += C::nt) {
            const int ijp = o / K, m = o % K;
            const int nb = g.face_nb[el * 4 + ijp];
            if (nb < 0 && sw[-nb - 1] == kNeumann) continue;
            T acc = T(0);
            for (int k = 0; k < K; ++k) acc += s.lcr[ijp * K + k] * b.D[m * K + k];
            if (nb >= 0) {
                int rev = 0;
                adj_neighbour_point<K, T>(g, el, ijp, 0, nb, nullptr, &rev);
                const int mm = rev ? K - 1 - m : m;
                for (int k = 0; k < K; ++k) acc += s.lcrn[ijp * K + k] * b.D[mm * K + (rev ? K - 1 - k : k)];
            }
            s.lcom[o] += acc;
        }
    }
    c.sync();
    // (5) common values: interior average, Dirichlet value, Neumann K x K system
    if (active) {
        for (int o = c.tid; o < NF; o += C::nt) {
            const int ijp = o / K;
            const int nb = g.face_nb[el * 4 + ijp];
            if (nb >= 0) {
                s.ltv[o] += T(0.5) * s.lcom[o];
                s.ntv[o] += T(0.5) * s.lcom[o];
                s.lbcv[o] = T(0);
            } else if (sw[-nb - 1] != kNeumann) {
                s.lbcv[o] = s.lcom[o];
            }
        }
        for (int ijp = c.tid; ijp < 4; ijp += C::nt) {
            const int nb = g.face_nb[el * 4 + ijp];
            if (nb >= 0 || sw[-nb - 1] != kNeumann) continue;
            const int lr = ijp & 1;
            const T sgn = neu_sign ? T(2 * (ijp % 2) - 1) : T(1);
            // com = M^-1 r with M[k][i] = -fB_k D[i][k] + delta_ki fA_k g'; lam_r = M^-T lam_com,
            // by Gaussian elimination with partial pivoting on A = M^T
            T A[K][K], y[K];
            for (int k = 0; k < K; ++k) {
                const int q = (el * 4 + ijp) * K + k;
                for (int i = 0; i < K; ++i) A[i][k] = -g.fB[q] * b.D[i * K + k];
                A[k][k] += g.fA[q] * b.gp[lr];
                y[k] = s.lcom[ijp * K + k];
            }
            for (int col = 0; col < K; ++col) {
                int piv = col;
                for (int r = col + 1; r < K; ++r)
                    if (adj_abs(A[r][col]) > adj_abs(A[piv][col])) piv = r;
                if (piv != col) {
                    for (int cc = 0; cc < K; ++cc) {
                        const T t = A[col][cc];
                        A[col][cc] = A[piv][cc];
                        A[piv][cc] = t;
                    }
                    const T t = y[col];
                    y[col] = y[piv];
                    y[piv] = t;
                }
                for (int r = col + 1; r < K; ++r) {
                    const T f = A[r][col] / A[col][col];
                    for (int cc = col; cc < K; ++cc) A[r][cc] -= f * A[col][cc];
                    y[r] -= f * y[col];
                }
            }
            for (int r = K - 1; r >= 0; --r) {
                T acc = y[r];
                for (int cc = r + 1; cc < K; ++cc) acc -= A[r][cc] * y[cc];
                y[r] = acc / A[r][r];
            }
            // r_k = fJ_k cg_k - fA_k (tg_k - tv_k g'),  cg_k = sgn * value_k * fAn_k
            for (int k = 0; k < K; ++k) {
                const int q = (el * 4 + ijp) * K + k, o = ijp * K + k;
                const T lcg = s.lcg[o] + g.fJ[q] * y[k];
                s.lbcv[o] = sgn * g.fAn[q] * lcg;
                s.ltg[o] -= g.fA[q] * y[k];
                s.ltv[o] += g.fA[q] * b.gp[lr] * y[k];
            }
        }
    }
    c.sync();
    // (6) own traces -> f (transposed face_trace)
    if (active) {
        for (int ij = c.tid; ij < K2; ij += C::nt) {
            const int j = ij / K, i = ij % K;
            T acc = s.lf[ij];
            for (int lr = 0; lr < 2; ++lr) {
                acc += s.ltv[lr * K + j] * b.sbb[i * 2 + lr] + s.ltg[lr * K + j] * b.sbgb[i * 2 + lr];
                acc += s.ltv[(2 + lr) * K + i] * b.sbb[j * 2 + lr] + s.ltg[(2 + lr) * K + i] * b.sbgb[j * 2 + lr];
            }
            s.lf[ij] = acc;
        }
    }
    c.sync();
}

// ---------------------------------------------------------------- stage adjoint
// Forward values of the stage (recomputed before the adjoint runs) and the adjoint
// arrays. Volume arrays [N][K][K], slots [N][4K] (indexed by the receiving face point),
// boundary arrays [N_eb][K].
template <typename T>
struct StageAdjArgs {
    const T* w;            // stage input vorticity
    const T* u;            // Cartesian velocity of the stage
    const T* v;
    const T* w_tv;         // omega face values of every element
    const T* U_t;          // contravariant volumetric flux face values of every element
    const double* bc_w;    // common boundary vorticity of the stage (BC_vorticity)
    const double* bc_nv;   // BC_normal_vel of the stage
    const T* lam_k;        // in: lam of k = dt (advective + diffusive RHS)
    T* lw_dir;             // lam of omega from this element's own chain
    T* lux;                // lam of the volumetric fluxes U^xi, U^eta at the points
    T* luy;
    T* slot_wv;            // lam of omega face values / normal derivatives, sent to neighbours
    T* slot_wg;
    T* slot_U;             // lam of U face values, sent to neighbours
    double* lbc_d;         // lam of BC_diffusion
    double* lbc_nv;        // lam of BC_normal_vel (advective boundary flux)
    T* lw_stage;           // out: lam of omega excluding the Poisson solve
    T* lpsi_dir;           // lam of psi from this element's own chain
    T* slot_pv;            // lam of psi traces sent to neighbours
    T* slot_pg;
    double* lpv;           // lam of BC_parl_vel, accumulated over stages
    double dt, re_inv;
    int adv_type = 1;      // 1: discontinuous upwind flux; 2: continuous volumetric flux
};

template <int K, typename T>
struct ResidualAdjScratch {
    static constexpr int K2 = K * K, NF = 4 * K;
    LapAdjScratch<K, T> lap;
    T w[K2], ux[K2], uy[K2], ldv[K2], lA[K2], lB[K2], lw[K2], lux[K2], luy[K2];
    T tvw[NF], ut[NF], lup[NF], lut[NF], ltva[NF], nU[NF], nwv[NF], com[NF];
};

// Step (2) of the residual adjoint for advection type 2. Forward: the common volumetric
// flux com = (U_L + s U_R) / 2 on interior faces and BC_normal_vel |g| on boundary faces;
// the upwind face flux com (c_L omega_L + c_R omega_R), (c_L, c_R) = (t, 1 - t) for com > 0
// and (1 - t, t) otherwise, t = 1 on E/N faces; BC_advection on boundary faces; inside,
// f = cx omega, g = cy omega with cx = U^xi + sum over the W/E faces of (com - U_face) times
// the Radau value at the point (cy likewise with the S/N faces).
template <int K, typename T, class C>
HO2D_HD void residual_adjoint_continuous(const C& c, bool active, int el, const FrGeom<T>& g, const DevBases<T>& b,
                                         const StageAdjArgs<T>& a, ResidualAdjScratch<K, T>& s) {
    constexpr int K2 = K * K, NF = 4 * K;
    LapAdjScratch<K, T>& L = s.lap;
    // (2a) the common volumetric flux of every face
    if (active)
        for (int o = c.tid; o < NF; o += C::nt) {
            const int ijp = o / K, k = o % K;
            const int nb = g.face_nb[el * 4 + ijp];
            if (nb >= 0) {
                int nijp = 0;
                const int nq = adj_neighbour_point<K, T>(g, el, ijp, k, nb, &nijp, nullptr);
                const T sign = T(2 * ((ijp + nijp) % 2) - 1);
                s.com[o] = T(0.5) * (s.ut[o] + sign * a.U_t[nq]);
            } else {
                const int be = (-nb - 1) * K + adj_bf<K>(ijp, k);
                s.com[o] = T(a.bc_nv[be]) * g.fAn[(el * 4 + ijp) * K + k];
            }
        }
    c.sync();
    // (2b) lam of f, g at the points -> lam of omega, and of cx, cy (= lam of U^xi, U^eta)
    if (active)
        for (int ij = c.tid; ij < K2; ij += C::nt) {
            const int hi = ij / K, lo = ij % K;
            const T lA = s.lA[ij] - s.lup[0 * K + hi] * b.sbb[lo * 2 + 0] - s.lup[1 * K + hi] * b.sbb[lo * 2 + 1];
            const T lB = s.lB[ij] - s.lup[2 * K + lo] * b.sbb[hi * 2 + 0] - s.lup[3 * K + lo] * b.sbb[hi * 2 + 1];
            const T cx = s.ux[ij] + (s.com[0 * K + hi] - s.ut[0 * K + hi]) * b.R[lo * 2 + 0] +
                         (s.com[1 * K + hi] - s.ut[1 * K + hi]) * b.R[lo * 2 + 1];
            const T cy = s.uy[ij] + (s.com[2 * K + lo] - s.ut[2 * K + lo]) * b.R[hi * 2 + 0] +
                         (s.com[3 * K + lo] - s.ut[3 * K + lo]) * b.R[hi * 2 + 1];
            s.lw[ij] = lA * cx + lB * cy;
            s.lux[ij] = lA * s.w[ij];
            s.luy[ij] = lB * s.w[ij];
        }
    c.sync();
    // (2c) per face: lam of com from the Radau corrections and from the upwind flux, then
    //      lam of the own and the neighbour's U and omega traces, of BC_vorticity and of
    //      BC_normal_vel
    if (active)
        for (int o = c.tid; o < NF; o += C::nt) {
            const int ijp = o / K, k = o % K, lr = ijp & 1;
            const int nb = g.face_nb[el * 4 + ijp];
            T lcv = T(0);
            if (ijp < 2) {
                for (int i = 0; i < K; ++i) lcv += s.lux[k * K + i] * b.R[i * 2 + lr];
            } else {
                for (int j = 0; j < K; ++j) lcv += s.luy[j * K + k] * b.R[j * 2 + lr];
            }
            const T lup = s.lup[o];
            T lut = -lcv, ltv = T(0), nU = T(0), nwv = T(0);
            if (nb >= 0) {
                int nijp = 0;
                const int nq = adj_neighbour_point<K, T>(g, el, ijp, k, nb, &nijp, nullptr);
                const T sign = T(2 * ((ijp + nijp) % 2) - 1);
                const T wl = s.tvw[o], wr = a.w_tv[nq], cvf = s.com[o], t = T(ijp % 2);
                const T cl = cvf > T(0) ? t : T(1) - t, cr = T(1) - cl;
                const T lcom = lcv + lup * (cl * wl + cr * wr);
                lut += T(0.5) * lcom;
                nU = T(0.5) * sign * lcom;
                ltv = lup * cvf * cl;
                nwv = lup * cvf * cr;
            } else {
                const int be = (-nb - 1) * K + adj_bf<K>(ijp, k);
                const int q = (el * 4 + ijp) * K + k;
                L.lcom[o] = lup * T(a.bc_nv[be]) * g.fAn[q];
                a.lbc_nv[be] = double((lup * T(a.bc_w[be]) + lcv) * g.fAn[q]);
            }
            s.lut[o] = lut;
            s.ltva[o] = ltv;
            s.nU[o] = nU;
            s.nwv[o] = nwv;
        }
    c.sync();
}

// Reverse of residual_kernel without the RK update: lam_k -> lam of omega (own chain), of
// U^xi / U^eta, of the neighbours' omega and U traces, of BC_diffusion and of
// BC_normal_vel. Advection type 1 (discontinuous flux, src/HO_2D.cpp:2245-2437) or type 2
// (continuous volumetric flux, 2439-2645); the upwind choices are those of the forward
// state (fixed where the flux is not differentiable).
template <int K, typename T, class C>
HO2D_HD void residual_adjoint_body(const C& c, bool active, int el, const FrGeom<T>& g, const DevBases<T>& b,
                                   const StageAdjArgs<T>& a, ResidualAdjScratch<K, T>& s) {
    constexpr int K2 = K * K, NF = 4 * K;
    LapAdjScratch<K, T>& L = s.lap;
    const T dt = T(a.dt), re_inv = T(a.re_inv);
    // (0) point values, and the adjoints of the two right-hand sides at the points:
    //     k = dt (adv + diff), diff = Lap re_inv / J, adv = -div / J
    if (active) {
        for (int ij = c.tid; ij < K2; ij += C::nt) {
            const int p = el * K2 + ij;
            const T xx = g.xxi[p], xe = g.xeta[p], yx = g.yxi[p], ye = g.yeta[p], J = g.J[p];
            const T u = a.u[p], v = a.v[p], lk = a.lam_k[p];
            s.w[ij] = a.w[p];
            s.ux[ij] = u * ye - v * xe;
            s.uy[ij] = -u * yx + v * xx;
            L.L[ij] = dt * lk * (re_inv / J);
            s.ldv[ij] = -(dt * lk) / J;
            L.la[ij] = T(0);
            L.lb[ij] = T(0);
        }
        for (int o = c.tid; o < NF; o += C::nt) {
            L.lfb[o] = T(0);
            L.lcg[o] = T(0);
            L.lcom[o] = T(0);
        }
    }
    c.sync();
    // (1) own face values of omega and of the fluxes; the divergence's transposed map
    if (active) {
        for (int o = c.tid; o < NF; o += C::nt) {
            const int ijp = o / K, k = o % K, lr = ijp & 1;
            T tv = T(0), ut = T(0), lfb = T(0);
            if (ijp < 2) {
                for (int m = 0; m < K; ++m) {
                    tv += s.w[k * K + m] * b.sbb[m * 2 + lr];
                    ut += s.ux[k * K + m] * b.sbb[m * 2 + lr];
                    lfb += s.ldv[k * K + m] * b.gR[m * 2 + lr];
                }
            } else {
                for (int m = 0; m < K; ++m) {
                    tv += s.w[m * K + k] * b.sbb[m * 2 + lr];
                    ut += s.uy[m * K + k] * b.sbb[m * 2 + lr];
                    lfb += s.ldv[m * K + k] * b.gR[m * 2 + lr];
                }
            }
            s.tvw[o] = tv;
            s.ut[o] = ut;
            s.lup[o] = lfb;  // lam of the common flux = lam of its jump
        }
        for (int ij = c.tid; ij < K2; ij += C::nt) {
            const int hi = ij / K, lo = ij % K;
            T aa = T(0), bb = T(0);
            for (int q = 0; q < K; ++q) {
                aa += s.ldv[hi * K + q] * b.D[lo * K + q];
                bb += s.ldv[q * K + lo] * b.D[hi * K + q];
            }
            s.lA[ij] = aa;
            s.lB[ij] = bb;
        }
    }
    c.sync();
    if (a.adv_type == 2) {
        residual_adjoint_continuous<K, T>(c, active, el, g, b, a, s);
    } else {
    // (2) volume fluxes U omega; the upwind face flux and the advective boundary flux
    if (active) {
        for (int ij = c.tid; ij < K2; ij += C::nt) {
            const int hi = ij / K, lo = ij % K;
            const T lA = s.lA[ij] - s.lup[0 * K + hi] * b.sbb[lo * 2 + 0] - s.lup[1 * K + hi] * b.sbb[lo * 2 + 1];
            const T lB = s.lB[ij] - s.lup[2 * K + lo] * b.sbb[hi * 2 + 0] - s.lup[3 * K + lo] * b.sbb[hi * 2 + 1];
            s.lw[ij] = lA * s.ux[ij] + lB * s.uy[ij];
            s.lux[ij] = lA * s.w[ij];
            s.luy[ij] = lB * s.w[ij];
        }
        for (int o = c.tid; o < NF; o += C::nt) {
            const int ijp = o / K, k = o % K;
            const int nb = g.face_nb[el * 4 + ijp];
            const T lup = s.lup[o];
            T lut = T(0), ltv = T(0), nU = T(0), nwv = T(0);
            if (nb >= 0) {
                int nijp = 0;
                const int nq = adj_neighbour_point<K, T>(g, el, ijp, k, nb, &nijp, nullptr);
                const T sign = T(2 * ((ijp + nijp) % 2) - 1);
                const T wl = s.tvw[o], wr = a.w_tv[nq], ul = s.ut[o], ur = a.U_t[nq];
                const T fl = ul * wl, fr = ur * wr;
                // up = (fl + sign fr)/2 + [|dw| > 1e-4] (s_lr / 2) |a| dw with a = (fl - sign fr)/dw,
                // i.e. (s_lr / 2) sgn(a) (fl - sign fr): linear in fl, fr for a fixed sgn(a)
                T dfl = T(0.5), dfr = T(0.5) * sign;
                const T dw = wl - wr;
                if (adj_abs(double(dw)) > 1e-4) {
                    const T av = (fl - sign * fr) / dw;
                    const T sg = av > T(0) ? T(1) : (av < T(0) ? T(-1) : T(0));
                    const T h = T(0.5) * T((ijp & 1) ? 1 : -1) * sg;
                    dfl += h;
                    dfr -= h * sign;
                }
                const T lfl = lup * dfl, lfr = lup * dfr;
                lut = lfl * wl;
                ltv = lfl * ul;
                nU = lfr * wr;
                nwv = lfr * ur;
            } else {
                // BC_advection = BC_vorticity BC_normal_vel |g|, BC_vorticity = the diffusion's common value
                const int be = (-nb - 1) * K + adj_bf<K>(ijp, k);
                const int q = (el * 4 + ijp) * K + k;
                L.lcom[o] = lup * T(a.bc_nv[be]) * g.fAn[q];
                a.lbc_nv[be] = double(lup * T(a.bc_w[be]) * g.fAn[q]);
            }
            s.lut[o] = lut;
            s.ltva[o] = ltv;
            s.nU[o] = nU;
            s.nwv[o] = nwv;
        }
    }
    c.sync();
    }
    // (3) transposed face-value maps of the advective part; then the diffusion chain
    if (active) {
        for (int ij = c.tid; ij < K2; ij += C::nt) {
            const int j = ij / K, i = ij % K;
            T lw = s.lw[ij], lux = s.lux[ij], luy = s.luy[ij];
            for (int lr = 0; lr < 2; ++lr) {
                lux += s.lut[lr * K + j] * b.sbb[i * 2 + lr];
                luy += s.lut[(2 + lr) * K + i] * b.sbb[j * 2 + lr];
                lw += s.ltva[lr * K + j] * b.sbb[i * 2 + lr] + s.ltva[(2 + lr) * K + i] * b.sbb[j * 2 + lr];
            }
            s.lw[ij] = lw;
            s.lux[ij] = lux;
            s.luy[ij] = luy;
        }
    }
    lap_adjoint<K, T>(c, active, el, g, b, g.sw_d, false, true, L);
    // (4) outputs
    if (active) {
        for (int ij = c.tid; ij < K2; ij += C::nt) {
            const int p = el * K2 + ij;
            a.lw_dir[p] = s.lw[ij] + L.lf[ij];
            a.lux[p] = s.lux[ij];
            a.luy[p] = s.luy[ij];
        }
        for (int o = c.tid; o < NF; o += C::nt) {
            const int ijp = o / K, k = o % K;
            const int nb = g.face_nb[el * 4 + ijp];
            if (nb >= 0) {
                const int nq = adj_neighbour_point<K, T>(g, el, ijp, k, nb, nullptr, nullptr);
                a.slot_wv[nq] = L.ntv[o] + s.nwv[o];
                a.slot_wg[nq] = L.ntg[o];
                a.slot_U[nq] = s.nU[o];
            } else {
                a.lbc_d[(-nb - 1) * K + adj_bf<K>(ijp, k)] = double(L.lbcv[o]);
            }
        }
    }
}

template <int K, typename T>
struct VelocityAdjScratch {
    static constexpr int NF = 4 * K;
    LapAdjScratch<K, T> lap;
    T gv[NF], gg[NF], gU[NF];
};

// Reverse of velocity_kernel (+ update_diffusion_BC): gathers the neighbours' slots of
// omega and U, finishes lam of omega (lw_stage, the Poisson part still missing), and
// maps lam of u, v, BC_diffusion and BC_normal_vel to lam of psi (own chain + slots) and
// of BC_parl_vel. Velocity_jump on Neumann-psi edges is carried from the previous stage
// in the forward map and is treated as a constant here (no-slip walls are Dirichlet-psi
// in every problem type).
template <int K, typename T, class C>
HO2D_HD void velocity_adjoint_body(const C& c, bool active, int el, const FrGeom<T>& g, const DevBases<T>& b,
                                   const StageAdjArgs<T>& a, VelocityAdjScratch<K, T>& s) {
    constexpr int K2 = K * K, NF = 4 * K;
    LapAdjScratch<K, T>& L = s.lap;
    if (active) {
        for (int o = c.tid; o < NF; o += C::nt) {
            const int q = el * NF + o;
            s.gv[o] = a.slot_wv[q];
            s.gg[o] = a.slot_wg[q];
            s.gU[o] = a.slot_U[q];
            L.lcg[o] = T(0);
            L.lcom[o] = T(0);
            const int ijp = o / K, k = o % K;
            const int nb = g.face_nb[el * 4 + ijp];
            if (nb >= 0) continue;
            const int e = -nb - 1;
            const int be = e * K + adj_bf<K>(ijp, k);
            const int qf = (el * 4 + ijp) * K + k;
            if (g.noslip[g.be_group[e]]) {
                // BC_diffusion = (velocity_jump +- BC_parl_vel) / (dt Re^-1)
                const double lvj = a.lbc_d[be] / (a.dt * a.re_inv);
                a.lpv[be] += double(2 * (ijp % 2) - 1) * lvj;
                if (g.sw_p[e] == kDirichlet) L.lcg[o] = T(lvj / double(g.fAn[qf]));  // velocity_jump = cg / fAn
            }
            if (g.sw_p[e] == kNeumann) {
                // BC_normal_vel[k'] = sum_d vsign com[d] D[d][k'] / fAn[k'] for this face's points k'
                const T vsign = T(1 - 2 * (ijp / 2));
                T acc = T(0);
                for (int kk = 0; kk < K; ++kk) {
                    const int be2 = e * K + adj_bf<K>(ijp, kk);
                    acc += vsign * b.D[k * K + kk] / g.fAn[(el * 4 + ijp) * K + kk] * T(a.lbc_nv[be2]);
                }
                L.lcom[o] = acc;
            }
        }
    }
    c.sync();
    // incoming slots -> lam of omega and of the fluxes; fluxes -> u, v -> grad psi
    if (active) {
        for (int ij = c.tid; ij < K2; ij += C::nt) {
            const int j = ij / K, i = ij % K, p = el * K2 + ij;
            T lw = a.lw_dir[p], lux = a.lux[p], luy = a.luy[p];
            for (int lr = 0; lr < 2; ++lr) {
                lw += s.gv[lr * K + j] * b.sbb[i * 2 + lr] + s.gg[lr * K + j] * b.sbgb[i * 2 + lr];
                lw += s.gv[(2 + lr) * K + i] * b.sbb[j * 2 + lr] + s.gg[(2 + lr) * K + i] * b.sbgb[j * 2 + lr];
                lux += s.gU[lr * K + j] * b.sbb[i * 2 + lr];
                luy += s.gU[(2 + lr) * K + i] * b.sbb[j * 2 + lr];
            }
            a.lw_stage[p] = lw;
            const T xx = g.xxi[p], xe = g.xeta[p], yx = g.yxi[p], ye = g.yeta[p], J = g.J[p];
            // U^xi = u y_eta - v x_eta, U^eta = -u y_xi + v x_xi; u = dpsi/dy, v = -dpsi/dx
            const T lu = lux * ye - luy * yx, lv = -lux * xe + luy * xx;
            const T ldpdx = -lv, ldpdy = lu;
            // dpsi/dx = (tx x_xi + ty x_eta) / J, dpsi/dy = (tx y_xi + ty y_eta) / J
            L.la[ij] = (ldpdx * xx + ldpdy * yx) / J;
            L.lb[ij] = (ldpdx * xe + ldpdy * ye) / J;
        }
    }
    c.sync();
    // tx = f~ + Radau values of fB, ty = g~ + Radau values of gB
    if (active) {
        for (int o = c.tid; o < NF; o += C::nt) {
            const int ijp = o / K, k = o % K, lr = ijp & 1;
            T acc = T(0);
            if (ijp < 2)
                for (int i = 0; i < K; ++i) acc += L.la[k * K + i] * b.R[i * 2 + lr];
            else
                for (int j = 0; j < K; ++j) acc += L.lb[j * K + k] * b.R[j * 2 + lr];
            L.lfb[o] = acc;
        }
    }
    c.sync();
    lap_adjoint<K, T>(c, active, el, g, b, g.sw_p, true, false, L);
    if (active) {
        for (int ij = c.tid; ij < K2; ij += C::nt) a.lpsi_dir[el * K2 + ij] = L.lf[ij];
        for (int o = c.tid; o < NF; o += C::nt) {
            const int ijp = o / K, k = o % K;
            const int nb = g.face_nb[el * 4 + ijp];
            if (nb < 0) continue;
            const int nq = adj_neighbour_point<K, T>(g, el, ijp, k, nb, nullptr, nullptr);
            a.slot_pv[nq] = L.ntv[o];
            a.slot_pg[nq] = L.ntg[o];
        }
    }
}

// ---------------------------------------------------------------- transposed Poisson operator
template <int K, typename T>
struct GatherScratch {
    static constexpr int NF = 4 * K;
    T sv[NF], sg[NF];
};

// out = dir + transposed face_trace of the incoming slots (value, normal derivative) at
// this element's face points. Boundary slots are never written and stay zero.
template <int K, typename T, class C>
HO2D_HD void gather_body(const C& c, bool active, int el, const DevBases<T>& b, const T* dir, const T* sv,
                         const T* sg, T* out, GatherScratch<K, T>& s) {
    constexpr int K2 = K * K, NF = 4 * K;
    if (active)
        for (int o = c.tid; o < NF; o += C::nt) {
            s.sv[o] = sv[el * NF + o];
            s.sg[o] = sg[el * NF + o];
        }
    c.sync();
    if (active)
        for (int ij = c.tid; ij < K2; ij += C::nt) {
            const int j = ij / K, i = ij % K;
            T acc = dir[el * K2 + ij];
            for (int lr = 0; lr < 2; ++lr) {
                acc += s.sv[lr * K + j] * b.sbb[i * 2 + lr] + s.sg[lr * K + j] * b.sbgb[i * 2 + lr];
                acc += s.sv[(2 + lr) * K + i] * b.sbb[j * 2 + lr] + s.sg[(2 + lr) * K + i] * b.sbgb[j * 2 + lr];
            }
            out[el * K2 + ij] = acc;
        }
}

// First half of y = A^T x (A the Poisson operator, psi boundary switches, homogeneous
// values): this element's own part in dir and its neighbours' parts in their slots.
template <int K, typename T, class C>
HO2D_HD void poisson_transpose_body(const C& c, bool active, int el, const FrGeom<T>& g, const DevBases<T>& b,
                                    const T* x, T* dir, T* slot_v, T* slot_g, LapAdjScratch<K, T>& s) {
    constexpr int K2 = K * K, NF = 4 * K;
    if (active) {
        for (int ij = c.tid; ij < K2; ij += C::nt) {
            s.L[ij] = x[el * K2 + ij];
            s.la[ij] = T(0);
            s.lb[ij] = T(0);
        }
        for (int o = c.tid; o < NF; o += C::nt) {
            s.lfb[o] = T(0);
            s.lcg[o] = T(0);
            s.lcom[o] = T(0);
        }
    }
    c.sync();
    lap_adjoint<K, T>(c, active, el, g, b, g.sw_p, true, true, s);
    if (active) {
        for (int ij = c.tid; ij < K2; ij += C::nt) dir[el * K2 + ij] = s.lf[ij];
        for (int o = c.tid; o < NF; o += C::nt) {
            const int ijp = o / K, k = o % K;
            const int nb = g.face_nb[el * 4 + ijp];
            if (nb < 0) continue;
            const int nq = adj_neighbour_point<K, T>(g, el, ijp, k, nb, nullptr, nullptr);
            slot_v[nq] = s.ntv[o];
            slot_g[nq] = s.ntg[o];
        }
    }
}

}  // namespace ho2d
