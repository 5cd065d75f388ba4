// shim_linalg.hpp -- project-written CPU sparse linear algebra behind the oracle's
// Eigen/AMGCL API shim.
//
// TEST INFRASTRUCTURE ONLY. This header lets the reference's own, unmodified
// src/HO_2D.cpp and src/Mesh.cpp compile in an image that has neither Eigen nor
// AMGCL. Only the names and signatures the reference calls are mirrored
// (src/HO_2D.hpp:34-54, src/HO_2D.cpp:1548,1669,2954-3086,1917,1960); every
// algorithm below is written from the published methods, not from those libraries:
//   * smoothed-aggregation AMG: Vanek, Mandel & Brezina, Computing 56 (1996) --
//     strength threshold eps_strong=0.08, plain greedy aggregation, piecewise
//     constant tentative prolongator, one damped-Jacobi prolongator smoothing step
//     on the filtered matrix with omega = (4/3)/rho(D^-1 A_f) (Gershgorin bound),
//     Galerkin coarse operators R A P with R = P^T;
//   * SPAI-0 smoother: Broeker & Grote (2002), m_i = a_ii / sum_j a_ij^2;
//   * BiCGSTAB: van der Vorst (1992), right preconditioned, stopping on the true
//     residual ||r|| <= tol * ||b|| (or maxiter);
//   * coarsest level: dense LU with partial pivoting once n <= 500 rows.
// Parity at this boundary is mathematical (same A, same b, converged psi), not
// iterate-for-iterate: these are not AMGCL 1.4.0 or Eigen 3.3.9.
#pragma once

#include <algorithm>
#include <cassert>
#include <cmath>
#include <cstdint>
#include <iomanip>
#include <iostream>
#include <limits>
#include <sstream>
#include <tuple>
#include <vector>

namespace shimla {

struct Csr {
    int n = 0, m = 0;  // rows, cols
    std::vector<int> ptr, col;
    std::vector<double> val;
    size_t nnz() const { return val.size(); }
};

inline void spmv(const Csr& A, const double* x, double* y) {
    for (int i = 0; i < A.n; ++i) {
        double s = 0.0;
        for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k) s += A.val[k] * x[A.col[k]];
        y[i] = s;
    }
}

inline Csr transpose(const Csr& A) {
    Csr T;
    T.n = A.m;
    T.m = A.n;
    T.ptr.assign(T.n + 1, 0);
    for (size_t k = 0; k < A.col.size(); ++k) T.ptr[A.col[k] + 1]++;
    for (int i = 0; i < T.n; ++i) T.ptr[i + 1] += T.ptr[i];
    T.col.resize(A.nnz());
    T.val.resize(A.nnz());
    std::vector<int> pos(T.ptr.begin(), T.ptr.end() - 1);
    for (int i = 0; i < A.n; ++i)
        for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k) {
            const int p = pos[A.col[k]]++;
            T.col[p] = i;
            T.val[p] = A.val[k];
        }
    return T;
}

// Gustavson row-by-row product with a dense accumulator.
inline Csr spgemm(const Csr& A, const Csr& B) {
    Csr C;
    C.n = A.n;
    C.m = B.m;
    C.ptr.assign(C.n + 1, 0);
    std::vector<int> marker(B.m, -1);
    std::vector<double> acc(B.m, 0.0);
    std::vector<int> cols;
    for (int i = 0; i < A.n; ++i) {
        cols.clear();
        for (int ka = A.ptr[i]; ka < A.ptr[i + 1]; ++ka) {
            const int j = A.col[ka];
            const double a = A.val[ka];
            for (int kb = B.ptr[j]; kb < B.ptr[j + 1]; ++kb) {
                const int c = B.col[kb];
                if (marker[c] != i) {
                    marker[c] = i;
                    acc[c] = 0.0;
                    cols.push_back(c);
                }
                acc[c] += a * B.val[kb];
            }
        }
        std::sort(cols.begin(), cols.end());
        for (int c : cols) {
            C.col.push_back(c);
            C.val.push_back(acc[c]);
        }
        C.ptr[i + 1] = (int)C.col.size();
    }
    return C;
}

struct DenseLU {
    int n = 0;
    std::vector<double> a;  // row-major LU factors
    std::vector<int> piv;
    void factor(const Csr& A) {
        n = A.n;
        a.assign((size_t)n * n, 0.0);
        piv.resize(n);
        for (int i = 0; i < n; ++i)
            for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k) a[(size_t)i * n + A.col[k]] += A.val[k];
        for (int k = 0; k < n; ++k) {
            int p = k;
            double best = std::fabs(a[(size_t)k * n + k]);
            for (int i = k + 1; i < n; ++i)
                if (std::fabs(a[(size_t)i * n + k]) > best) { best = std::fabs(a[(size_t)i * n + k]); p = i; }
            piv[k] = p;
            if (p != k)
                for (int j = 0; j < n; ++j) std::swap(a[(size_t)k * n + j], a[(size_t)p * n + j]);
            const double d = a[(size_t)k * n + k];
            if (d == 0.0) continue;  // singular pivot: leave the row alone
            for (int i = k + 1; i < n; ++i) {
                const double l = a[(size_t)i * n + k] / d;
                a[(size_t)i * n + k] = l;
                if (l != 0.0)
                    for (int j = k + 1; j < n; ++j) a[(size_t)i * n + j] -= l * a[(size_t)k * n + j];
            }
        }
    }
    void solve(const double* b, double* x) const {
        std::vector<double> y(b, b + n);
        for (int k = 0; k < n; ++k) std::swap(y[k], y[piv[k]]);
        for (int i = 0; i < n; ++i) {
            double s = y[i];
            for (int j = 0; j < i; ++j) s -= a[(size_t)i * n + j] * y[j];
            y[i] = s;
        }
        for (int i = n - 1; i >= 0; --i) {
            double s = y[i];
            for (int j = i + 1; j < n; ++j) s -= a[(size_t)i * n + j] * y[j];
            const double d = a[(size_t)i * n + i];
            y[i] = d != 0.0 ? s / d : 0.0;
        }
        std::copy(y.begin(), y.end(), x);
    }
};

class SaAmg {
  public:
    double eps_strong = 0.08;
    int coarse_enough = 500;
    int max_levels = 30;

    void build(const Csr& A0) {
        levels_.clear();
        levels_.emplace_back();
        levels_[0].A = A0;
        while ((int)levels_.size() < max_levels && levels_.back().A.n > coarse_enough) {
            Level& L = levels_.back();
            Csr P;
            if (!coarsen(L.A, P)) break;
            L.P = P;
            L.R = transpose(P);
            Csr AP = spgemm(L.A, P);
            Level next;
            next.A = spgemm(L.R, AP);
            if (next.A.n == 0 || next.A.n >= L.A.n) { L.P = Csr(); L.R = Csr(); break; }
            levels_.push_back(std::move(next));
        }
        for (auto& L : levels_) {
            L.m.assign(L.A.n, 0.0);
            for (int i = 0; i < L.A.n; ++i) {
                double d = 0.0, s = 0.0;
                for (int k = L.A.ptr[i]; k < L.A.ptr[i + 1]; ++k) {
                    s += L.A.val[k] * L.A.val[k];
                    if (L.A.col[k] == i) d = L.A.val[k];
                }
                L.m[i] = s > 0.0 ? d / s : 0.0;
            }
            L.f.assign(L.A.n, 0.0);
            L.u.assign(L.A.n, 0.0);
            L.t.assign(L.A.n, 0.0);
        }
        lu_.factor(levels_.back().A);
    }

    // z = M^{-1} r via one V(1,1) cycle from a zero initial guess.
    void apply(const double* r, double* z) {
        std::copy(r, r + levels_[0].A.n, levels_[0].f.begin());
        cycle(0);
        std::copy(levels_[0].u.begin(), levels_[0].u.end(), z);
    }

  private:
    struct Level {
        Csr A, P, R;
        std::vector<double> m, f, u, t;
    };
    std::vector<Level> levels_;
    DenseLU lu_;

    void smooth(Level& L) {  // u += M (f - A u)
        spmv(L.A, L.u.data(), L.t.data());
        for (int i = 0; i < L.A.n; ++i) L.u[i] += L.m[i] * (L.f[i] - L.t[i]);
    }

    void cycle(size_t l) {
        Level& L = levels_[l];
        if (l + 1 == levels_.size()) {
            lu_.solve(L.f.data(), L.u.data());
            return;
        }
        std::fill(L.u.begin(), L.u.end(), 0.0);
        smooth(L);
        spmv(L.A, L.u.data(), L.t.data());
        for (int i = 0; i < L.A.n; ++i) L.t[i] = L.f[i] - L.t[i];
        Level& C = levels_[l + 1];
        spmv(L.R, L.t.data(), C.f.data());
        cycle(l + 1);
        spmv(L.P, C.u.data(), L.t.data());
        for (int i = 0; i < L.A.n; ++i) L.u[i] += L.t[i];
        smooth(L);
    }

    // Strength graph, plain aggregation, tentative and smoothed prolongator.
    bool coarsen(const Csr& A, Csr& P) {
        const int n = A.n;
        std::vector<double> diag(n, 0.0);
        for (int i = 0; i < n; ++i)
            for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k)
                if (A.col[k] == i) diag[i] = A.val[k];
        std::vector<char> strong(A.nnz(), 0);
        for (int i = 0; i < n; ++i)
            for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k) {
                const int j = A.col[k];
                if (j == i) continue;
                const double a = A.val[k];
                strong[k] = (a * a > eps_strong * eps_strong * std::fabs(diag[i] * diag[j]));
            }
        const int UNDONE = -1, REMOVED = -2;
        std::vector<int> agg(n, UNDONE);
        for (int i = 0; i < n; ++i) {
            bool any = false;
            for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k) any = any || strong[k];
            if (!any) agg[i] = REMOVED;  // isolated: left to the smoother
        }
        int nagg = 0;
        // pass 1: roots whose whole strong neighbourhood is still free
        for (int i = 0; i < n; ++i) {
            if (agg[i] != UNDONE) continue;
            bool free = true;
            for (int k = A.ptr[i]; k < A.ptr[i + 1] && free; ++k)
                if (strong[k] && agg[A.col[k]] >= 0) free = false;
            if (!free) continue;
            agg[i] = nagg;
            for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k)
                if (strong[k] && agg[A.col[k]] == UNDONE) agg[A.col[k]] = nagg;
            ++nagg;
        }
        // pass 2: attach leftovers to a strongly connected aggregate
        std::vector<int> agg1 = agg;
        for (int i = 0; i < n; ++i) {
            if (agg[i] != UNDONE) continue;
            for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k)
                if (strong[k] && agg[A.col[k]] >= 0) { agg1[i] = agg[A.col[k]]; break; }
        }
        agg.swap(agg1);
        // pass 3: whatever is left starts new aggregates
        for (int i = 0; i < n; ++i) {
            if (agg[i] != UNDONE) continue;
            agg[i] = nagg;
            for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k)
                if (strong[k] && agg[A.col[k]] == UNDONE) agg[A.col[k]] = nagg;
            ++nagg;
        }
        if (nagg == 0 || nagg >= n) return false;
        // filtered matrix diagonal: weak connections lumped into the diagonal
        std::vector<double> dfil(diag);
        for (int i = 0; i < n; ++i)
            for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k)
                if (A.col[k] != i && !strong[k]) dfil[i] += A.val[k];
        // Gershgorin bound of rho(D_f^{-1} A_f)
        double rho = 0.0;
        for (int i = 0; i < n; ++i) {
            if (dfil[i] == 0.0) continue;
            double s = std::fabs(dfil[i]);
            for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k)
                if (A.col[k] != i && strong[k]) s += std::fabs(A.val[k]);
            rho = std::max(rho, s / std::fabs(dfil[i]));
        }
        const double omega = rho > 0.0 ? (4.0 / 3.0) / rho : 0.0;
        // P = (I - omega D_f^{-1} A_f) P_tent
        P = Csr();
        P.n = n;
        P.m = nagg;
        P.ptr.assign(n + 1, 0);
        std::vector<int> marker(nagg, -1);
        std::vector<double> acc(nagg, 0.0);
        std::vector<int> cols;
        for (int i = 0; i < n; ++i) {
            cols.clear();
            auto add = [&](int c, double v) {
                if (marker[c] != i) { marker[c] = i; acc[c] = 0.0; cols.push_back(c); }
                acc[c] += v;
            };
            const double s = dfil[i] != 0.0 ? omega / dfil[i] : 0.0;
            if (agg[i] >= 0) add(agg[i], 1.0);
            for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k) {
                const int j = A.col[k];
                if (agg[j] < 0) continue;
                double aij;
                if (j == i) aij = dfil[i];
                else if (strong[k]) aij = A.val[k];
                else continue;
                add(agg[j], -s * aij);
            }
            std::sort(cols.begin(), cols.end());
            for (int c : cols)
                if (acc[c] != 0.0) { P.col.push_back(c); P.val.push_back(acc[c]); }
            P.ptr[i + 1] = (int)P.col.size();
        }
        return true;
    }
};

// Direct solver for golden-vector generation: reverse Cuthill-McKee ordering
// (Cuthill & McKee 1969; George 1971) followed by a banded LU with partial pivoting
// in LAPACK's band layout (the dgbtf2 elimination order).
class BandedLU {
  public:
    void factor(const Csr& A) {
        n_ = A.n;
        // symmetric adjacency for the ordering
        std::vector<std::vector<int>> adj(n_);
        for (int i = 0; i < n_; ++i)
            for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k) {
                const int j = A.col[k];
                if (j == i) continue;
                adj[i].push_back(j);
                adj[j].push_back(i);
            }
        for (auto& a : adj) {
            std::sort(a.begin(), a.end());
            a.erase(std::unique(a.begin(), a.end()), a.end());
        }
        std::vector<int> order;
        order.reserve(n_);
        std::vector<char> seen(n_, 0);
        while ((int)order.size() < n_) {
            int start = -1;
            for (int i = 0; i < n_; ++i)
                if (!seen[i] && (start < 0 || adj[i].size() < adj[start].size())) start = i;
            size_t head = order.size();
            order.push_back(start);
            seen[start] = 1;
            while (head < order.size()) {
                const int v = order[head++];
                std::vector<int> nb;
                for (int w : adj[v])
                    if (!seen[w]) { seen[w] = 1; nb.push_back(w); }
                std::sort(nb.begin(), nb.end(), [&](int a, int b) { return adj[a].size() < adj[b].size(); });
                order.insert(order.end(), nb.begin(), nb.end());
            }
        }
        std::reverse(order.begin(), order.end());
        perm_.assign(n_, 0);  // perm_[old] = new
        for (int i = 0; i < n_; ++i) perm_[order[i]] = i;
        kl_ = ku_ = 0;
        for (int i = 0; i < n_; ++i)
            for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k) {
                const int d = perm_[i] - perm_[A.col[k]];
                kl_ = std::max(kl_, d);
                ku_ = std::max(ku_, -d);
            }
        kv_ = kl_ + ku_;
        ld_ = 2 * kl_ + ku_ + 1;
        ab_.assign((size_t)ld_ * n_, 0.0);
        for (int i = 0; i < n_; ++i)
            for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k) at(perm_[i], perm_[A.col[k]]) += A.val[k];
        piv_.assign(n_, 0);
        int ju = 0;
        for (int j = 0; j < n_; ++j) {
            const int km = std::min(kl_, n_ - 1 - j);
            int jp = 0;
            double best = std::fabs(at(j, j));
            for (int t = 1; t <= km; ++t)
                if (std::fabs(at(j + t, j)) > best) { best = std::fabs(at(j + t, j)); jp = t; }
            piv_[j] = j + jp;
            if (best == 0.0) continue;
            ju = std::max(ju, std::min(j + ku_ + jp, n_ - 1));
            if (jp != 0)
                for (int c = j; c <= ju; ++c) std::swap(at(j, c), at(j + jp, c));
            const double d = at(j, j);
            for (int t = 1; t <= km; ++t) at(j + t, j) /= d;
            for (int c = j + 1; c <= ju; ++c) {
                const double f = at(j, c);
                if (f == 0.0) continue;
                for (int t = 1; t <= km; ++t) at(j + t, c) -= at(j + t, j) * f;
            }
        }
    }
    void solve(const double* b, double* x) {
        std::vector<double> y(n_);
        for (int i = 0; i < n_; ++i) y[perm_[i]] = b[i];
        for (int j = 0; j < n_; ++j) {
            std::swap(y[j], y[piv_[j]]);
            const int km = std::min(kl_, n_ - 1 - j);
            for (int t = 1; t <= km; ++t) y[j + t] -= at(j + t, j) * y[j];
        }
        for (int j = n_ - 1; j >= 0; --j) {
            y[j] = at(j, j) != 0.0 ? y[j] / at(j, j) : 0.0;
            for (int i = std::max(0, j - kv_); i < j; ++i) y[i] -= at(i, j) * y[j];
        }
        for (int i = 0; i < n_; ++i) x[i] = y[perm_[i]];
    }

  private:
    int n_ = 0, kl_ = 0, ku_ = 0, kv_ = 0, ld_ = 0;
    std::vector<double> ab_;
    std::vector<int> piv_, perm_;
    double& at(int i, int j) { return ab_[(size_t)(kv_ + i - j) + (size_t)j * ld_]; }
};

// Right-preconditioned BiCGSTAB; returns (iterations, ||b - A x|| / ||b||).
inline std::tuple<int, double> bicgstab(const Csr& A, SaAmg& M, const double* b, double* x, double tol,
                                        int maxiter) {
    const int n = A.n;
    auto dot = [n](const std::vector<double>& u, const std::vector<double>& v) {
        double s = 0.0;
        for (int i = 0; i < n; ++i) s += u[i] * v[i];
        return s;
    };
    std::vector<double> r(n), rhat(n), p(n, 0.0), v(n, 0.0), s(n), t(n), ph(n), sh(n);
    double nb = 0.0;
    for (int i = 0; i < n; ++i) nb += b[i] * b[i];
    nb = std::sqrt(nb);
    if (nb == 0.0) {
        std::fill(x, x + n, 0.0);
        return std::make_tuple(0, 0.0);
    }
    spmv(A, x, r.data());
    for (int i = 0; i < n; ++i) r[i] = b[i] - r[i];
    rhat = r;
    double res = std::sqrt(dot(r, r));
    const double eps = tol * nb;
    double rho_old = 1.0, alpha = 1.0, omega = 1.0;
    int it = 0;
    for (; it < maxiter && res > eps; ++it) {
        const double rho = dot(rhat, r);
        if (rho == 0.0) break;
        if (it == 0) p = r;
        else {
            const double beta = (rho / rho_old) * (alpha / omega);
            for (int i = 0; i < n; ++i) p[i] = r[i] + beta * (p[i] - omega * v[i]);
        }
        M.apply(p.data(), ph.data());
        spmv(A, ph.data(), v.data());
        const double rv = dot(rhat, v);
        if (rv == 0.0) break;
        alpha = rho / rv;
        for (int i = 0; i < n; ++i) s[i] = r[i] - alpha * v[i];
        const double ress = std::sqrt(dot(s, s));
        if (ress <= eps) {
            for (int i = 0; i < n; ++i) x[i] += alpha * ph[i];
            res = ress;
            ++it;
            break;
        }
        M.apply(s.data(), sh.data());
        spmv(A, sh.data(), t.data());
        const double tt = dot(t, t);
        omega = tt > 0.0 ? dot(t, s) / tt : 0.0;
        for (int i = 0; i < n; ++i) {
            x[i] += alpha * ph[i] + omega * sh[i];
            r[i] = s[i] - omega * t[i];
        }
        rho_old = rho;
        res = std::sqrt(dot(r, r));
        if (omega == 0.0) { ++it; break; }
    }
    return std::make_tuple(it, res / nb);
}

}  // namespace shimla
