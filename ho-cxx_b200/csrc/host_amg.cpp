// host_amg.cpp -- coarse space of the Poisson preconditioner, built once on the host.
//
// The device preconditioner is two-level: damped element block-Jacobi on the FR operator
// (exact solves of each element's K^2 x K^2 diagonal block) plus a correction in the
// space of element-wise constants (P0). The P0 Galerkin operator A1 = P^T A P has one
// row per element and the element adjacency as its pattern (5 entries per row); it is
// solved approximately by one V-cycle of smoothed-aggregation AMG -- the coarsening
// family of the reference's AMGCL setup (src/HO_2D.hpp:54, src/HO_2D.cpp:3066-3072),
// written here from the published method (Vanek, Mandel & Brezina 1996):
//   strength |a_ij| > 0.08 sqrt(|a_ii a_jj|), greedy plain aggregation, piecewise-constant
//   tentative prolongator, one damped-Jacobi smoothing step of it on the filtered matrix
//   with omega = (4/3) / rho(D^-1 A_f) (Gershgorin bound), R = P^T, A_c = R A P;
//   SPAI-0 smoothers (Broeker & Grote 2002); dense inverse of the last level.
#include <algorithm>
#include <cmath>

#include "host_amg.hpp"

namespace ho2d {

namespace {

Csr transpose(const Csr& A) {
    Csr T;
    T.n = A.m;
    T.m = A.n;
    T.ptr.assign(T.n + 1, 0);
    for (int c : A.col) T.ptr[c + 1]++;
    for (int i = 0; i < T.n; ++i) T.ptr[i + 1] += T.ptr[i];
    T.col.resize(A.col.size());
    T.val.resize(A.val.size());
    std::vector<int> pos(T.ptr.begin(), T.ptr.end() - 1);
    for (int i = 0; i < A.n; ++i)
        for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k) {
            const int p = pos[A.col[k]]++;
            T.col[p] = i;
            T.val[p] = A.val[k];
        }
    return T;
}

Csr multiply(const Csr& A, const Csr& B) {
    Csr C;
    C.n = A.n;
    C.m = B.m;
    C.ptr.assign(C.n + 1, 0);
    std::vector<int> mark(B.m, -1), cols;
    std::vector<double> acc(B.m, 0.0);
    for (int i = 0; i < A.n; ++i) {
        cols.clear();
        for (int ka = A.ptr[i]; ka < A.ptr[i + 1]; ++ka) {
            const int j = A.col[ka];
            for (int kb = B.ptr[j]; kb < B.ptr[j + 1]; ++kb) {
                const int c = B.col[kb];
                if (mark[c] != i) {
                    mark[c] = i;
                    acc[c] = 0.0;
                    cols.push_back(c);
                }
                acc[c] += A.val[ka] * B.val[kb];
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

// I - diag(l) A diag(r); an empty l or r means no scaling on that side. Every row gets an
// explicit diagonal entry.
Csr identity_minus_scaled(const Csr& A, const std::vector<double>& l, const std::vector<double>& r) {
    Csr C;
    C.n = A.n;
    C.m = A.m;
    C.ptr.assign(A.n + 1, 0);
    for (int i = 0; i < A.n; ++i) {
        bool diag = false;
        for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k) {
            const int j = A.col[k];
            if (!diag && j > i) {
                C.col.push_back(i);
                C.val.push_back(1.0);
                diag = true;
            }
            double v = -A.val[k] * (l.empty() ? 1.0 : l[i]) * (r.empty() ? 1.0 : r[j]);
            if (j == i) {
                v += 1.0;
                diag = true;
            }
            C.col.push_back(j);
            C.val.push_back(v);
        }
        if (!diag) {
            C.col.push_back(i);
            C.val.push_back(1.0);
        }
        C.ptr[i + 1] = (int)C.col.size();
    }
    return C;
}

// 2 diag(m) - diag(m) A diag(m)
Csr smoothing_part(const Csr& A, const std::vector<double>& m) {
    Csr C = identity_minus_scaled(A, m, m);  // I - mAm, with an explicit diagonal
    for (int i = 0; i < C.n; ++i)
        for (int k = C.ptr[i]; k < C.ptr[i + 1]; ++k)
            if (C.col[k] == i) C.val[k] += 2.0 * m[i] - 1.0;
    return C;
}

std::vector<double> spai0(const Csr& A) {
    std::vector<double> m(A.n, 0.0);
    for (int i = 0; i < A.n; ++i) {
        double d = 0.0, s = 0.0;
        for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k) {
            s += A.val[k] * A.val[k];
            if (A.col[k] == i) d = A.val[k];
        }
        m[i] = s > 0.0 ? d / s : 0.0;
    }
    return m;
}

// Smoothed-aggregation prolongator of A; returns false when A does not coarsen.
bool sa_prolongator(const Csr& A, Csr& P) {
    const int n = A.n;
    const double eps = 0.08;
    std::vector<double> diag(n, 0.0);
    for (int i = 0; i < n; ++i)
        for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k)
            if (A.col[k] == i) diag[i] = A.val[k];
    std::vector<char> strong(A.val.size(), 0);
    for (int i = 0; i < n; ++i)
        for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k) {
            const int j = A.col[k];
            if (j != i) strong[k] = A.val[k] * A.val[k] > eps * eps * std::fabs(diag[i] * diag[j]);
        }
    const int FREE = -1, ISOLATED = -2;
    std::vector<int> agg(n, FREE);
    for (int i = 0; i < n; ++i) {
        bool any = false;
        for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k) any = any || strong[k];
        if (!any) agg[i] = ISOLATED;
    }
    int na = 0;
    for (int i = 0; i < n; ++i) {  // roots with an entirely free neighbourhood
        if (agg[i] != FREE) continue;
        bool ok = true;
        for (int k = A.ptr[i]; k < A.ptr[i + 1] && ok; ++k)
            if (strong[k] && agg[A.col[k]] >= 0) ok = false;
        if (!ok) continue;
        agg[i] = na;
        for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k)
            if (strong[k] && agg[A.col[k]] == FREE) agg[A.col[k]] = na;
        ++na;
    }
    std::vector<int> joined = agg;
    for (int i = 0; i < n; ++i) {  // leftovers join a strongly connected aggregate
        if (agg[i] != FREE) continue;
        for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k)
            if (strong[k] && agg[A.col[k]] >= 0) {
                joined[i] = agg[A.col[k]];
                break;
            }
    }
    agg.swap(joined);
    for (int i = 0; i < n; ++i) {  // the rest start new aggregates
        if (agg[i] != FREE) continue;
        agg[i] = na;
        for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k)
            if (strong[k] && agg[A.col[k]] == FREE) agg[A.col[k]] = na;
        ++na;
    }
    if (na == 0 || na >= n) return false;
    std::vector<double> df(diag);  // filtered diagonal
    for (int i = 0; i < n; ++i)
        for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k)
            if (A.col[k] != i && !strong[k]) df[i] += A.val[k];
    double rho = 0.0;
    for (int i = 0; i < n; ++i) {
        if (df[i] == 0.0) continue;
        double s = std::fabs(df[i]);
        for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k)
            if (A.col[k] != i && strong[k]) s += std::fabs(A.val[k]);
        rho = std::max(rho, s / std::fabs(df[i]));
    }
    const double omega = rho > 0.0 ? (4.0 / 3.0) / rho : 0.0;
    P = Csr();
    P.n = n;
    P.m = na;
    P.ptr.assign(n + 1, 0);
    std::vector<int> mark(na, -1), cols;
    std::vector<double> acc(na, 0.0);
    for (int i = 0; i < n; ++i) {
        cols.clear();
        auto add = [&](int c, double v) {
            if (mark[c] != i) {
                mark[c] = i;
                acc[c] = 0.0;
                cols.push_back(c);
            }
            acc[c] += v;
        };
        const double s = df[i] != 0.0 ? omega / df[i] : 0.0;
        if (agg[i] >= 0) add(agg[i], 1.0);
        for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k) {
            const int j = A.col[k];
            if (agg[j] < 0) continue;
            if (j == i) add(agg[j], -s * df[i]);
            else if (strong[k]) add(agg[j], -s * A.val[k]);
        }
        std::sort(cols.begin(), cols.end());
        for (int c : cols)
            if (acc[c] != 0.0) {
                P.col.push_back(c);
                P.val.push_back(acc[c]);
            }
        P.ptr[i + 1] = (int)P.col.size();
    }
    return true;
}

// Inverse by LU with partial pivoting (rows updated in parallel), then one forward and
// back substitution per column of the identity (columns in parallel).
bool dense_inverse(int n, const Csr& A, std::vector<double>& inv) {
    std::vector<double> a((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i)
        for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k) a[(size_t)i * n + A.col[k]] += A.val[k];
    std::vector<int> piv(n);
    for (int k = 0; k < n; ++k) {
        int p = k;
        for (int i = k + 1; i < n; ++i)
            if (std::fabs(a[(size_t)i * n + k]) > std::fabs(a[(size_t)p * n + k])) p = i;
        if (a[(size_t)p * n + k] == 0.0) return false;
        piv[k] = p;
        if (p != k)
            for (int j = 0; j < n; ++j) std::swap(a[(size_t)k * n + j], a[(size_t)p * n + j]);
        const double d = 1.0 / a[(size_t)k * n + k];
        const double* rk = &a[(size_t)k * n];
#pragma omp parallel for schedule(static) if (n - k > 256)
        for (int i = k + 1; i < n; ++i) {
            double* ri = &a[(size_t)i * n];
            const double l = ri[k] * d;
            ri[k] = l;
            if (l != 0.0)
                for (int j = k + 1; j < n; ++j) ri[j] -= l * rk[j];
        }
    }
    inv.assign((size_t)n * n, 0.0);
#pragma omp parallel
    {
        std::vector<double> x(n);
#pragma omp for schedule(dynamic, 16)
        for (int c = 0; c < n; ++c) {
            std::fill(x.begin(), x.end(), 0.0);
            x[c] = 1.0;
            for (int k = 0; k < n; ++k) std::swap(x[k], x[piv[k]]);
            for (int i = 1; i < n; ++i) {
                const double* ri = &a[(size_t)i * n];
                double s = x[i];
                for (int j = 0; j < i; ++j) s -= ri[j] * x[j];
                x[i] = s;
            }
            for (int i = n - 1; i >= 0; --i) {
                const double* ri = &a[(size_t)i * n];
                double s = x[i];
                for (int j = i + 1; j < n; ++j) s -= ri[j] * x[j];
                x[i] = s / ri[i];
            }
            for (int i = 0; i < n; ++i) inv[(size_t)i * n + c] = x[i];
        }
    }
    return true;
}

}  // namespace

Ell to_ell(const Csr& A) {
    Ell E;
    E.n = A.n;
    E.m = A.m;
    for (int i = 0; i < A.n; ++i) E.w = std::max(E.w, A.ptr[i + 1] - A.ptr[i]);
    E.w = (E.w + 3) / 4 * 4;  // rows start on 16-byte boundaries
    E.col.assign((size_t)E.n * E.w, 0);
    E.val.assign((size_t)E.n * E.w, 0.0);
    for (int i = 0; i < A.n; ++i)
        for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k) {
            E.col[(size_t)i * E.w + (k - A.ptr[i])] = A.col[k];
            E.val[(size_t)i * E.w + (k - A.ptr[i])] = A.val[k];
        }
    return E;
}

Csr p0_coarse_operator(const PoissonOperator& op, int N) {
    Csr A;
    A.n = A.m = N;
    A.ptr.assign(N + 1, 0);
    for (int el = 0; el < N; ++el) {
        std::vector<std::pair<int, double>> row;
        for (int s = 0; s < 5; ++s) {
            const int c = op.block_col[(size_t)el * 5 + s];
            if (c < 0) continue;
            row.push_back({c, op.bsum[(size_t)el * 5 + s]});
        }
        std::sort(row.begin(), row.end());
        for (size_t k = 0; k < row.size(); ++k) {
            if (!A.col.empty() && (int)A.col.size() > A.ptr[el] && A.col.back() == row[k].first)
                A.val.back() += row[k].second;
            else {
                A.col.push_back(row[k].first);
                A.val.push_back(row[k].second);
            }
        }
        A.ptr[el + 1] = (int)A.col.size();
    }
    return A;
}

Error build_coarse_hierarchy(const Csr& A1, CoarseHierarchy& H, int dense_max, int dense_max_first, bool invert_dense) {
    H = CoarseHierarchy();
    H.levels.emplace_back();
    H.levels[0].A = A1;
    auto coarsen = [&]() {
        const int n = H.levels.back().A.n;
        return n > (H.levels.size() == 1 ? dense_max_first : dense_max);
    };
    while (coarsen() && H.levels.size() < 16) {
        AmgLevel& L = H.levels.back();
        Csr P;
        if (!sa_prolongator(L.A, P)) break;
        Csr R = transpose(P);
        Csr Ac = multiply(R, multiply(L.A, P));
        if (Ac.n >= L.A.n) break;
        L.P = P;
        L.R = R;
        AmgLevel next;
        next.A = Ac;
        H.levels.push_back(next);
    }
    for (auto& L : H.levels) L.m = spai0(L.A);
    for (size_t l = 0; l + 1 < H.levels.size(); ++l) {
        AmgLevel& L = H.levels[l];
        L.M = multiply(L.R, identity_minus_scaled(L.A, {}, L.m));
        L.S = smoothing_part(L.A, L.m);
        L.Q = multiply(identity_minus_scaled(L.A, L.m, {}), L.P);
    }
    const Csr& Ab = H.levels.back().A;
    if (Ab.n > 2 * std::max(dense_max, kDenseMax))
        return {4, "coarse Poisson problem did not coarsen below the dense-solve size"};
    H.n_dense = Ab.n;
    if (invert_dense && !dense_inverse(Ab.n, Ab, H.dense_inv)) return {3, "singular coarsest Poisson operator"};
    return {0, ""};
}

}  // namespace ho2d
