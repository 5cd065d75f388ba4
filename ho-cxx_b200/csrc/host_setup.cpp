// host_setup.cpp -- bases, metrics, boundary conditions and the block Poisson operator.
//
// bases ............ src/HO_2D.cpp:486-673 (Gauss-Legendre by Newton iteration on the
//                    Legendre three-term recurrence, so any K <= 8 works; the reference's
//                    closed forms stop at K = 5)
// metrics .......... src/HO_2D.cpp:1240-1388
// BCs .............. src/HO_2D.cpp:675-1238 (problem types 1, 2, 3)
// Poisson operator . src/HO_2D.cpp:1533-1804 with the |a| > 1e-14 filter of 3023-3062.
//   The element-interior and face couplings are linear in the metric terms G and GB, so
//   they are evaluated from small precomputed coefficient lists (one entry per
//   (row, column, metric slot)) instead of the reference's nested loops; Neumann faces
//   add the inverse of the K x K face system.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "assemble_element.hpp"
#include "host.hpp"

namespace ho2d {

namespace {

double legendre(int n, double x) {
    if (n == 0) return 1.0;
    double p0 = 1.0, p1 = x;
    for (int i = 2; i <= n; ++i) {
        const double p2 = ((2.0 * i - 1.0) * x * p1 - (i - 1.0) * p0) / i;
        p0 = p1;
        p1 = p2;
    }
    return p1;
}

// Lagrange basis of `nodes` evaluated at x: values V[k], derivatives Dv[k].
void lagrange_at(const std::vector<double>& nodes, double x, double* V, double* Dv) {
    const int n = (int)nodes.size();
    for (int k = 0; k < n; ++k) {
        double den = 1.0, val = 1.0, der = 0.0;
        for (int j = 0; j < n; ++j) {
            if (j == k) continue;
            den *= nodes[k] - nodes[j];
            val *= x - nodes[j];
            double term = 1.0;
            for (int i = 0; i < n; ++i)
                if (i != k && i != j) term *= x - nodes[i];
            der += term;
        }
        V[k] = val / den;
        Dv[k] = der / den;
    }
}

// In-place Gauss-Jordan inverse with partial pivoting of an n x n row-major matrix
// (n <= kMaxK^2). Step k swaps the pivot row into place, scales it, and eliminates column k
// from every other row; column k then holds the inverse's column (its entries start as the
// identity's), so the inverse builds up in a itself and the row swaps are undone as column
// swaps at the end: n^3 multiply-adds and no scratch beyond two rows. The row update is
// compiled twice, for AVX2 and for the baseline, and picked at load time; neither contracts
// to FMA, so both give the same bits as the textbook two-matrix form.
__attribute__((target_clones("avx2", "default"))) bool invert(int n, double* m) {
    constexpr int kMax = kMaxK * kMaxK;
    if (n < 1 || n > kMax) return false;
    int piv[kMax];
    double rk[kMax];  // the scaled pivot row, kept apart so the row updates vectorise
    for (int k = 0; k < n; ++k) {
        int p = k;
        for (int i = k + 1; i < n; ++i)
            if (std::fabs(m[(size_t)i * n + k]) > std::fabs(m[(size_t)p * n + k])) p = i;
        if (m[(size_t)p * n + k] == 0.0) return false;
        piv[k] = p;
        if (p != k)
            for (int j = 0; j < n; ++j) std::swap(m[(size_t)k * n + j], m[(size_t)p * n + j]);
        double* row = m + (size_t)k * n;
        const double d = 1.0 / row[k];
        row[k] = 1.0;
        for (int j = 0; j < n; ++j) rk[j] = row[j] * d;
        for (int j = 0; j < n; ++j) row[j] = rk[j];
        for (int i = 0; i < n; ++i) {
            if (i == k) continue;
            double* __restrict__ ri = m + (size_t)i * n;
            const double l = ri[k];
            if (l == 0.0) continue;
            ri[k] = 0.0;
            for (int j = 0; j < n; ++j) ri[j] -= l * rk[j];
        }
    }
    for (int k = n - 1; k >= 0; --k)
        if (piv[k] != k)
            for (int i = 0; i < n; ++i) std::swap(m[(size_t)i * n + k], m[(size_t)i * n + piv[k]]);
    return true;
}

}  // namespace

Error make_bases(int K, int L, Bases& B) {
    if (K < 1 || K > kMaxK) return {4, "Knod out of range"};
    if (L < 2 || L > 4) return {4, "Lnod must be 2, 3 or 4"};
    B.K = K;
    B.L = L;
    B.xs.assign(K, 0.0);
    B.w.assign(K, 0.0);
    // Gauss-Legendre nodes: Newton on P_K from the Chebyshev-like initial guess
    for (int i = 0; i < K; ++i) {
        double x = std::cos(M_PI * (i + 0.75) / (K + 0.5));
        double dp = 1.0;
        for (int it = 0; it < 100; ++it) {
            const double p = legendre(K, x), pm = legendre(K - 1, x);
            dp = K * (x * p - pm) / (x * x - 1.0);
            const double dx = p / dp;
            x -= dx;
            if (std::fabs(dx) < 1e-16) break;
        }
        const double p = legendre(K, x), pm = legendre(K - 1, x);
        dp = K * (x * p - pm) / (x * x - 1.0);
        B.xs[K - 1 - i] = x;
        B.w[K - 1 - i] = 2.0 / ((1.0 - x * x) * dp * dp);
    }
    if (K == 1) { B.xs[0] = 0.0; B.w[0] = 2.0; }
    if (K % 2 == 1) B.xs[K / 2] = 0.0;
    for (int i = 0; i < K / 2; ++i) {  // exact symmetry
        const double a = 0.5 * (B.xs[K - 1 - i] - B.xs[i]);
        B.xs[i] = -a;
        B.xs[K - 1 - i] = a;
        const double w = 0.5 * (B.w[i] + B.w[K - 1 - i]);
        B.w[i] = B.w[K - 1 - i] = w;
    }
    std::vector<double> gx(L);
    for (int i = 0; i < L; ++i) gx[i] = -1.0 + 2.0 * i / (L - 1);
    std::vector<double> V(std::max(K, L)), Dv(std::max(K, L));
    B.sbb.assign(K * 2, 0.0);
    B.sbgb.assign(K * 2, 0.0);
    for (int lr = 0; lr < 2; ++lr) {
        lagrange_at(B.xs, lr ? 1.0 : -1.0, V.data(), Dv.data());
        for (int k = 0; k < K; ++k) { B.sbb[k * 2 + lr] = V[k]; B.sbgb[k * 2 + lr] = Dv[k]; }
    }
    B.D.assign(K * K, 0.0);
    for (int m = 0; m < K; ++m) {
        lagrange_at(B.xs, B.xs[m], V.data(), Dv.data());
        for (int k = 0; k < K; ++k) B.D[k * K + m] = Dv[k];
    }
    B.gsb.assign(L * K, 0.0);
    B.gsgb.assign(L * K, 0.0);
    for (int m = 0; m < K; ++m) {
        lagrange_at(gx, B.xs[m], V.data(), Dv.data());
        for (int k = 0; k < L; ++k) { B.gsb[k * K + m] = V[k]; B.gsgb[k * K + m] = Dv[k]; }
    }
    B.gbb.assign(L * 2, 0.0);
    B.gbgb.assign(L * 2, 0.0);
    for (int lr = 0; lr < 2; ++lr) {
        lagrange_at(gx, lr ? 1.0 : -1.0, V.data(), Dv.data());
        for (int k = 0; k < L; ++k) { B.gbb[k * 2 + lr] = V[k]; B.gbgb[k * 2 + lr] = Dv[k]; }
    }
    B.R.assign(K * 2, 0.0);
    B.gR.assign(K * 2, 0.0);
    if (K == 1) {
        B.R[0] = B.R[1] = 0.5;
        B.gR[0] = -0.5;
        B.gR[1] = 0.5;
    } else {
        // right Radau R_K(x) = (-1)^K/2 (P_K - P_{K-1}); the left one is its mirror
        const double sg = (K % 2 == 0) ? 1.0 : -1.0;
        const double c = 0.5 * sg, cd = 0.5 * K * sg;
        for (int i = 0; i < K; ++i) {
            const double x = B.xs[i];
            B.R[i * 2 + 0] = c * (legendre(K, x) - legendre(K - 1, x));
            B.R[i * 2 + 1] = c * (legendre(K, -x) - legendre(K - 1, -x));
            B.gR[i * 2 + 0] = cd * (legendre(K, x) + legendre(K - 1, x)) / (1.0 + x);
            B.gR[i * 2 + 1] = -cd * (legendre(K, -x) + legendre(K - 1, -x)) / (1.0 - x);
        }
    }
    B.gp[0] = -0.5 * K * (K + 1.0);
    B.gp[1] = 0.5 * K * (K + 1.0);
    return {0, ""};
}

void make_metrics(const Mesh& mesh, const Bases& B, Metrics& M) {
    const int N = mesh.n_el, K = B.K, L = B.L, lin = L - 1;
    const size_t nv = (size_t)N * K * K;
    M.xxi.assign(nv, 0.0); M.xeta.assign(nv, 0.0); M.yxi.assign(nv, 0.0); M.yeta.assign(nv, 0.0);
    M.J.assign(nv, 0.0);
    M.G.assign(nv * 4, 0.0);
    M.GB.assign((size_t)N * 4 * K * 2, 0.0);
    M.fA.assign((size_t)N * 4 * K, 0.0); M.fB = M.fA; M.fJ = M.fA; M.fAn = M.fA;
#pragma omp parallel for schedule(static)
    for (int el = 0; el < N; ++el) {
        double X[4][4], Y[4][4];
        for (int j = 0; j < L; ++j)
            for (int i = 0; i < L; ++i) {
                const int nd = mesh.elem_nodes[el][tensor2fem(i, j, lin)];
                X[j][i] = mesh.node_xy[2 * nd];
                Y[j][i] = mesh.node_xy[2 * nd + 1];
            }
        for (int j = 0; j < K; ++j)
            for (int i = 0; i < K; ++i) {
                double xx = 0, yx = 0, xe = 0, ye = 0;
                for (int n = 0; n < L; ++n)
                    for (int m = 0; m < L; ++m) {
                        const double a = B.gsgb[m * K + i] * B.gsb[n * K + j];
                        const double b = B.gsgb[n * K + j] * B.gsb[m * K + i];
                        xx += a * X[n][m]; yx += a * Y[n][m];
                        xe += b * X[n][m]; ye += b * Y[n][m];
                    }
                const size_t p = ((size_t)el * K + j) * K + i;
                M.xxi[p] = xx; M.yxi[p] = yx; M.xeta[p] = xe; M.yeta[p] = ye;
                const double J = xx * ye - xe * yx;
                M.J[p] = J;
                const double g[2][2] = {{-xe, ye}, {xx, -yx}};
                for (int r = 0; r < 2; ++r)
                    for (int s = 0; s < 2; ++s)
                        M.G[p * 4 + r * 2 + s] = (g[r][0] * g[s][0] + g[r][1] * g[s][1]) / J;
            }
        for (int ijp = 0; ijp < 4; ++ijp) {
            const int d = ijp / 2, t = ijp % 2;
            for (int k = 0; k < K; ++k) {
                double xx = 0, yx = 0, xe = 0, ye = 0;
                for (int j = 0; j < L; ++j)
                    for (int i = 0; i < L; ++i) {
                        double a, b;  // weights of d/dxi and d/deta
                        if (d == 0) {
                            a = B.gbgb[i * 2 + t] * B.gsb[j * K + k];
                            b = B.gbb[i * 2 + t] * B.gsgb[j * K + k];
                        } else {
                            a = B.gbb[j * 2 + t] * B.gsgb[i * K + k];
                            b = B.gbgb[j * 2 + t] * B.gsb[i * K + k];
                        }
                        xx += a * X[j][i]; yx += a * Y[j][i];
                        xe += b * X[j][i]; ye += b * Y[j][i];
                    }
                const size_t q = ((size_t)el * 4 + ijp) * K + k;
                const double fJ = xx * ye - xe * yx;
                M.fJ[q] = fJ;
                M.fA[q] = d == 0 ? xe * xe + ye * ye : xx * xx + yx * yx;
                M.fB[q] = xx * xe + yx * ye;
                M.fAn[q] = std::sqrt(M.fA[q]);
                const double g[2][2] = {{-xe, ye}, {xx, -yx}};
                for (int r = 0; r < 2; ++r)
                    M.GB[((((size_t)el * 2 + d) * 2 + t) * K + k) * 2 + r] =
                        (g[d][0] * g[r][0] + g[d][1] * g[r][1]) / fJ;
            }
        }
    }
}

namespace {

std::vector<double> edge_y(const Mesh& m, const Bases& B, int e) {
    std::vector<double> y(B.K, 0.0);
    const int lin = m.lnod - 1;
    for (int k = 0; k < B.K; ++k)
        for (int j = 0; j < m.lnod; ++j) y[k] += B.gsb[j * B.K + k] * m.node_xy[2 * m.edge_nodes[e][tensor2fem_1d(j, lin)] + 1];
    return y;
}

}  // namespace

namespace {

#define HO2D_SETUP_TRY(expr)    \
    do {                        \
        Error _e = (expr);      \
        if (_e.code) return _e; \
    } while (0)

// Problem type 11 (src/HO_2D.cpp:893-1134). Boundaries by name: "open" (Neumann psi,
// Dirichlet vorticity, values set every stage from the driver's data), "wall" (no slip),
// "inlet" (Dirichlet psi and vorticity), "outlet" (Neumann psi and vorticity, zero). With
// inlets, psi is marched along the chain of non-open boundary edges (each edge's second
// node is the next edge's first): an inlet edge of length L with normal velocity v lowers
// psi by L v and gets psi linear along it, the mean velocity's difference quotients with
// its neighbours as vorticity and -v as BC_normal_vel; an outlet lowers psi the same way;
// a wall takes the psi reached. The chain starts at the first edge that is neither inlet
// nor outlet and assumes 2-node edges.
Error setup_hybrid_bcs(const Mesh& m, const Bases& B, BoundaryConditions& bc) {
    const int K = B.K, neb = m.n_eb, ng = (int)m.group_names.size();
    enum { T_OTHER, T_OPEN, T_WALL, T_INLET, T_OUTLET };
    std::vector<int> type(neb, T_OTHER);
    bool have_inlets = false;
    for (int g = 0; g < ng; ++g) {
        const std::string& nm = m.group_names[g];
        int t;
        if (nm == "open") t = T_OPEN;
        else if (nm == "wall") t = T_WALL;
        else if (nm == "inlet") t = T_INLET;
        else if (nm == "outlet") t = T_OUTLET;
        else return {4, "hybrid run: boundary \"" + nm + "\" is not wall, open, inlet or outlet"};
        bc.noslip[g] = t == T_WALL ? 1 : 0;
        have_inlets = have_inlets || (t == T_INLET && !m.group_edges[g].empty());
        for (int e : m.group_edges[g]) {
            type[e] = t;
            const size_t q0 = (size_t)e * K;
            if (t == T_OPEN) {
                bc.sw_p[e] = NEUMANN;
                bc.sw_d[e] = DIRICHLET;
                bc.role[e] = ROLE_OPEN;
            } else if (t == T_WALL) {
                bc.sw_p[e] = DIRICHLET;
                bc.sw_d[e] = NEUMANN;
                bc.role[e] = ROLE_WALL_H;
            } else if (t == T_INLET) {
                bc.sw_p[e] = DIRICHLET;
                bc.sw_d[e] = DIRICHLET;
                bc.role[e] = ROLE_INLET_H;
            } else {
                bc.sw_p[e] = NEUMANN;
                bc.sw_d[e] = NEUMANN;
            }
            if (t == T_INLET || t == T_OUTLET) {
                const double v = e < (int)m.edge_normvel.size() ? m.edge_normvel[e] : std::nan("");
                if (!std::isfinite(v)) return {1, "hybrid run: an inlet or outlet edge has no normal velocity"};
                if (t == T_INLET) bc.inlet_nv[e] = v;
            }
            std::fill_n(bc.bc_p.begin() + q0, K, 0.0);
            std::fill_n(bc.bc_nv.begin() + q0, K, 0.0);
            std::fill_n(bc.bc_pv.begin() + q0, K, 0.0);
            std::fill_n(bc.bc_d.begin() + q0, K, 0.0);
        }
    }
    if (!have_inlets) return {0, ""};
    if (m.lnod != 2) return {4, "hybrid run: inlets need 2-node edges (Lnod = 2)"};
    const int nnodes = (int)m.node_xy.size() / 2;
    std::vector<int> firstnode(nnodes, 0);
    for (int e = 0; e < neb; ++e)
        if (type[e] != T_OPEN) firstnode[m.edge_nodes[e][0]] = e;
    int istart = 0;
    while (istart < neb && (type[istart] == T_INLET || type[istart] == T_OUTLET)) ++istart;
    if (istart == neb) return {3, "hybrid run: every boundary edge is an inlet or outlet"};
    std::vector<int> chain = {istart};
    for (;;) {
        const int next = firstnode[m.edge_nodes[chain.back()][1]];
        if (next == chain.front()) break;
        chain.push_back(next);
        if ((int)chain.size() > neb) return {3, "hybrid run: the boundary edges do not close into a loop"};
    }
    const int nc = (int)chain.size();
    std::vector<double> len(nc);
    for (int i = 0; i < nc; ++i) {
        const auto& en = m.edge_nodes[chain[i]];
        const double dx = m.node_xy[2 * en[1]] - m.node_xy[2 * en[0]], dy = m.node_xy[2 * en[1] + 1] - m.node_xy[2 * en[0] + 1];
        len[i] = std::sqrt(dx * dx + dy * dy);
    }
    auto inlet_v = [&](int i) { return type[chain[i]] == T_INLET ? m.edge_normvel[chain[i]] : 0.0; };
    double psi_end = 0.0;
    for (int i = 0; i < nc; ++i) {
        const int e = chain[i];
        const double psi_start = psi_end;
        const size_t q0 = (size_t)e * K;
        if (type[e] == T_INLET) {
            const double v = m.edge_normvel[e];
            psi_end -= len[i] * v;
            const int ip = i == 0 ? nc - 1 : i - 1, in = i == nc - 1 ? 0 : i + 1;
            const double w = (inlet_v(in) - v) / (len[in] + len[i]) + (v - inlet_v(ip)) / (len[i] + len[ip]);
            for (int k = 0; k < K; ++k) {
                bc.bc_p[q0 + k] = B.gsb[0 * K + k] * psi_start + B.gsb[1 * K + k] * psi_end;
                bc.bc_d[q0 + k] = w;
                bc.bc_nv[q0 + k] = -v;
            }
        } else if (type[e] == T_OUTLET) {
            psi_end -= len[i] * m.edge_normvel[e];
        } else if (type[e] == T_WALL) {
            std::fill_n(bc.bc_p.begin() + q0, K, psi_end);
        }
    }
    return {0, ""};
}

}  // namespace

Error setup_bcs(const Input& in, const Mesh& m, const Bases& B, BoundaryConditions& bc) {
    const int K = B.K, neb = m.n_eb, ng = (int)m.group_names.size();
    bc.sw_p.assign(neb, DIRICHLET);
    bc.sw_d.assign(neb, DIRICHLET);
    bc.noslip.assign(ng, 0);
    bc.bc_p.assign((size_t)neb * K, 0.0);
    bc.bc_nv = bc.bc_p; bc.bc_pv = bc.bc_p; bc.bc_d = bc.bc_p;
    bc.edge_y.assign((size_t)neb * K, 0.0);
    bc.role.assign(neb, ROLE_NONE);
    for (int e = 0; e < neb; ++e) {
        const auto y = edge_y(m, B, e);
        std::copy(y.begin(), y.end(), bc.edge_y.begin() + (size_t)e * K);
    }
    auto fill = [&](std::vector<double>& a, int e, double v) { std::fill_n(a.begin() + (size_t)e * K, K, v); };
    bc.inlet_nv.assign(neb, 0.0);
    const int pt = in.problem_type;
    if (pt == 11) {  // hybrid run (src/HO_2D.cpp:893-1134)
        HO2D_SETUP_TRY(setup_hybrid_bcs(m, B, bc));
    } else if (pt == 1) {  // lid-driven cavity (src/HO_2D.cpp:700-727)
        std::fill(bc.noslip.begin(), bc.noslip.end(), 1);
        std::fill(bc.sw_p.begin(), bc.sw_p.end(), DIRICHLET);
        std::fill(bc.sw_d.begin(), bc.sw_d.end(), NEUMANN);
        for (int g = 0; g < ng; ++g)
            if (m.group_names[g] == "top")
                for (int e : m.group_edges[g]) fill(bc.bc_pv, e, -1.0);
    } else {  // backward-facing step (729-817) and flow over an object (819-906)
        bool have_inlet = false;
        for (int g = 0; g < ng; ++g) {
            if (m.group_names[g] != "inlet" || m.group_edges[g].empty()) continue;
            have_inlet = true;
            const int n0 = m.edge_nodes[m.group_edges[g][0]][0];
            bc.y_min = bc.y_max = m.node_xy[2 * n0 + 1];
            for (int e : m.group_edges[g])
                for (int c = 0; c < 2; ++c) {
                    const double y = m.node_xy[2 * m.edge_nodes[e][c] + 1];
                    bc.y_min = std::min(bc.y_min, y);
                    bc.y_max = std::max(bc.y_max, y);
                }
        }
        (void)have_inlet;
        const double ymin = bc.y_min, ymax = bc.y_max, h2 = (ymax - ymin) * (ymax - ymin);
        for (int g = 0; g < ng; ++g) {
            const std::string& nm = m.group_names[g];
            for (int e : m.group_edges[g]) {
                const double* y = &bc.edge_y[(size_t)e * K];
                if (nm == "inlet") {
                    bc.sw_d[e] = DIRICHLET;
                    bc.sw_p[e] = DIRICHLET;
                    bc.role[e] = ROLE_INLET;
                    for (int k = 0; k < K; ++k) {
                        const size_t q = (size_t)e * K + k;
                        if (pt == 2) {
                            bc.bc_p[q] = (y[k] - ymin) * (y[k] - ymin) * (3.0 * ymax - ymin - 2.0 * y[k]) / h2;
                            bc.bc_d[q] = 6.0 * (2.0 * y[k] - ymin - ymax) / h2;
                            bc.bc_nv[q] = 6.0 * (y[k] - ymin) * (y[k] - ymax) / h2;
                        } else {
                            bc.bc_p[q] = y[k] - ymin;
                            bc.bc_d[q] = 0.0;
                            bc.bc_nv[q] = -1.0;
                        }
                    }
                } else if (nm == "outlet") {
                    bc.sw_d[e] = NEUMANN;
                    bc.sw_p[e] = NEUMANN;
                    fill(bc.bc_d, e, 0.0);
                    fill(bc.bc_p, e, 0.0);
                } else if (nm == "top" || nm == "bottom") {
                    bc.sw_p[e] = DIRICHLET;
                    bc.sw_d[e] = NEUMANN;
                    bc.role[e] = nm == "top" ? ROLE_TOP : ROLE_BOTTOM;
                    fill(bc.bc_p, e, nm == "top" ? ymax - ymin : 0.0);
                    fill(bc.bc_nv, e, 0.0);
                    fill(bc.bc_pv, e, pt == 2 ? 0.0 : (nm == "top" ? -1.0 : 1.0));
                } else if (nm == "object" && pt == 3) {
                    bc.sw_p[e] = DIRICHLET;
                    bc.sw_d[e] = NEUMANN;
                    bc.role[e] = ROLE_OBJECT;
                    fill(bc.bc_p, e, 0.5 * (ymax - ymin));
                    fill(bc.bc_nv, e, 0.0);
                    fill(bc.bc_pv, e, 0.0);
                }
            }
            if (nm == "inlet" || nm == "outlet") bc.noslip[g] = 0;
            else if (nm == "top" || nm == "bottom") bc.noslip[g] = pt == 2 ? 1 : 0;
            else if (nm == "object" && pt == 3) bc.noslip[g] = 1;
        }
    }
    // outward normal values into the local h direction (src/HO_2D.cpp:1228-1237)
    for (int e = 0; e < neb; ++e) {
        const int ijp = kF2I[m.be_side[e]];
        const double sign = 2.0 * (ijp % 2) - 1.0;
        for (int k = 0; k < K; ++k) {
            bc.bc_nv[(size_t)e * K + k] *= sign;
            if (bc.sw_d[e] == NEUMANN) bc.bc_d[(size_t)e * K + k] *= sign;
        }
    }
    return {0, ""};
}

namespace {

// Element-interior coupling: Lc[ij][rs] += c * G[el][b][a][r][d] (src/HO_2D.cpp:1567-1596).
std::vector<AsmEntry> volume_entries(const Bases& B) {
    const int K = B.K, K2 = K * K;
    std::vector<AsmEntry> out;
    for (int j = 0; j < K; ++j)
        for (int i = 0; i < K; ++i)
            for (int m = 0; m < K; ++m)
                for (int r = 0; r < 2; ++r) {
                    const int a = m * (1 - r) + i * r, b = m * r + j * (1 - r);
                    const int cr = j * r + i * (1 - r);
                    const double tmp3 = B.sbb[m * 2] * B.gR[cr * 2] + B.sbb[m * 2 + 1] * B.gR[cr * 2 + 1];
                    const double sn = B.D[m * K + i * (1 - r) + j * r];
                    for (int d = 0; d < 2; ++d) {
                        const int t1 = a * (1 - d) + b * d;
                        for (int p = 0; p < K; ++p) {
                            const int rs = (p * d + b * (1 - d)) * K + (p * (1 - d) + a * d);
                            const double tmp2 = 0.5 * (B.sbb[p * 2] * B.gR[t1 * 2] + B.sbb[p * 2 + 1] * B.gR[t1 * 2 + 1]);
                            const double c = sn * (B.D[p * K + t1] - tmp2) + tmp3 * (-B.D[p * K + t1] + tmp2);
                            out.push_back({(j * K + i) * K2 + rs, ((b * K + a) * 2 + r) * 2 + d, c});
                        }
                    }
                }
    return out;
}

// Face weights W[ij][q] = sum c * G[el][b][a][r][d] for face (d, t) (src/HO_2D.cpp:1614-1637).
std::vector<AsmEntry> face_entries(const Bases& B, int d, int t) {
    const int K = B.K;
    std::vector<AsmEntry> out;
    for (int j = 0; j < K; ++j)
        for (int i = 0; i < K; ++i)
            for (int m = 0; m < K; ++m)
                for (int r = 0; r < 2; ++r) {
                    const int a = m * (1 - r) + i * r, b = m * r + j * (1 - r);
                    const int q = a * d + b * (1 - d);
                    const int cr = j * r + i * (1 - r);
                    const double sn = B.D[m * K + i * (1 - r) + j * r];
                    const double ngr = B.gR[(a * (1 - d) + b * d) * 2 + t];
                    const double tmp2 = B.sbb[m * 2] * B.gR[cr * 2] + B.sbb[m * 2 + 1] * B.gR[cr * 2 + 1];
                    out.push_back({(j * K + i) * K + q, ((b * K + a) * 2 + r) * 2 + d, (sn - tmp2) * ngr});
                }
    return out;
}


}  // namespace

void assemble_poisson(const Mesh& mesh, const Bases& B, const Metrics& M, const BoundaryConditions& bc,
                      PoissonOperator& op, bool keep_blocks, KronSmoother* kron) {
    const int N = mesh.n_el, K = B.K, K2 = K * K, K4 = K2 * K2;
    op.K2 = K2;
    op.blocks.assign(keep_blocks ? (size_t)N * 5 * K4 : 0, 0.0);
    op.block_col.assign((size_t)N * 5, -1);
    op.bsrc.assign((size_t)mesh.n_eb * K2 * K, 0.0);
    op.dinv.assign((size_t)N * K4, 0.0);
    op.rowsum.assign((size_t)N * 5 * K2, 0.0);
    op.colsum.assign((size_t)N * 5 * K2, 0.0);
    op.bsum.assign((size_t)N * 5, 0.0);
    if (kron) {
        kron->K = K;
        kron->v.assign((size_t)N * 4 * K * K, 0.0);
        kron->lam.assign((size_t)N * 2 * K, 0.0);
        kron->exact.assign(N, 1);
        kron->defect.assign(N, 0.0);
    }
    const AsmCoefficients co = assembly_coefficients(B);
    const AsmBases ab = asm_bases(B);
    const AsmTables tb = co.tables();
    const AsmMesh am{M.G.data(), M.GB.data(), M.fJ.data(), mesh.bidx.data(), mesh.nbr.data(), mesh.nbr_side.data(),
                     bc.sw_p.data()};
    const AsmOut ao{op.bsrc.data(), op.rowsum.data(), op.colsum.data(), op.bsum.data(),
                    keep_blocks ? op.blocks.data() : nullptr, op.block_col.data()};
    int64_t nnz = 0;
#pragma omp parallel reduction(+ : nnz)
    {
        std::vector<double> Lc(K4), L(K4), W((size_t)K2 * K), WN((size_t)K2 * K), Nm((size_t)K * K);
        const AsmScratch sc{{Lc.data(), 1}, {L.data(), 1}, {W.data(), 1}, {WN.data(), 1}, {Nm.data(), 1}};
#pragma omp for schedule(dynamic, 16)
        for (int el = 0; el < N; ++el) {
            nnz += assemble_element(el, ab, tb, am, ao, sc, [](int n, Str<double> a) { return invert(n, a.p); });
            if (kron) {  // the Kronecker-sum fit of the filtered diagonal block ([ij][rs])
                KronFit f;
                const bool ok = kron_fit(K, Lc.data(), f);
                kron_store(ok ? &f : nullptr, ok ? kron_defect(f, Lc.data()) : 0.0, el, *kron);
            }
            // inverse of the filtered diagonal block, stored transposed like the blocks
            invert(K2, Lc.data());
            double* di = &op.dinv[(size_t)el * K4];
            for (int ij = 0; ij < K2; ++ij)
                for (int rs = 0; rs < K2; ++rs) di[rs * K2 + ij] = Lc[ij * K2 + rs];
        }
    }
    op.nnz = nnz;
}

AsmBases asm_bases(const Bases& B) {
    return AsmBases{B.K, B.sbb.data(), B.sbgb.data(), B.gR.data(), B.D.data(), {B.gp[0], B.gp[1]}};
}

AsmCoefficients assembly_coefficients(const Bases& B) {
    AsmCoefficients c;
    c.vol = volume_entries(B);
    for (int d = 0; d < 2; ++d)
        for (int t = 0; t < 2; ++t) c.fw[d * 2 + t] = face_entries(B, d, t);
    return c;
}

}  // namespace ho2d
