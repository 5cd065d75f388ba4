// host_kron.cpp -- the Kronecker-sum approximation of an element's diagonal Poisson block,
// for a smoother that stores O(K^2) values per element instead of the K^4 of the inverse.
//
// The diagonal block D (K^2 x K^2, row ij = (j, i), j along eta) is fitted in the least-
// squares sense by I (x) Ax + Ay (x) I, i.e. D[(j,i),(l,k)] ~ delta_jl Ax[i][k] + Ay[j][l]
// delta_ik: the off-diagonal entries of Ax (Ay) are the averages of the matching entries of
// D over j (over i), and the K x K array of D's diagonal entries d[j][i] ~ Ax[i][i] +
// Ay[j][j] is split by row and column means. With Ax = Vx diag(lx) Vx^-1 and Ay = Vy
// diag(ly) Vy^-1 (fast diagonalisation; Lynch, Rice & Thomas 1964) the fitted block's
// inverse applies to R[j][i] as  X = Vy [ (Vy^-1 R Vx^-T) ./ (ly_j + lx_i) ] Vx^T.
//
// Eigenvalues: Householder reduction to Hessenberg form, then the QR algorithm with a
// Wilkinson shift, one Givens sweep per step, deflating from the bottom (Golub & Van Loan,
// Matrix Computations, ch. 7). A complex pair (a 2 x 2 block with negative discriminant)
// or a missed convergence rejects the fit. Eigenvectors: two steps of inverse iteration
// with the computed eigenvalue on the original matrix.
#include <algorithm>
#include <cmath>
#include <vector>

#include "host.hpp"

namespace ho2d {

namespace {

// LU with partial pivoting of the n x n row-major a (in place); false if singular
bool lu(int n, std::vector<double>& a, std::vector<int>& piv) {
    piv.resize(n);
    for (int k = 0; k < n; ++k) {
        int p = k;
        for (int i = k + 1; i < n; ++i)
            if (std::fabs(a[i * n + k]) > std::fabs(a[p * n + k])) p = i;
        piv[k] = p;
        if (a[p * n + k] == 0.0) return false;
        if (p != k)
            for (int j = 0; j < n; ++j) std::swap(a[k * n + j], a[p * n + j]);
        for (int i = k + 1; i < n; ++i) {
            const double l = a[i * n + k] / a[k * n + k];
            a[i * n + k] = l;
            for (int j = k + 1; j < n; ++j) a[i * n + j] -= l * a[k * n + j];
        }
    }
    return true;
}

void lu_solve(int n, const std::vector<double>& a, const std::vector<int>& piv, double* x) {
    for (int k = 0; k < n; ++k) std::swap(x[k], x[piv[k]]);
    for (int i = 1; i < n; ++i)
        for (int j = 0; j < i; ++j) x[i] -= a[i * n + j] * x[j];
    for (int i = n - 1; i >= 0; --i) {
        for (int j = i + 1; j < n; ++j) x[i] -= a[i * n + j] * x[j];
        x[i] /= a[i * n + i];
    }
}

}  // namespace

bool real_eigenvalues(int n, const double* A, double* lambda) {
    std::vector<double> h(A, A + (size_t)n * n);
    // Householder reduction to upper Hessenberg form: zero column k below row k + 1
    for (int k = 0; k + 2 < n; ++k) {
        double alpha = 0.0;
        for (int i = k + 1; i < n; ++i) alpha += h[i * n + k] * h[i * n + k];
        alpha = std::sqrt(alpha);
        if (alpha == 0.0) continue;
        if (h[(k + 1) * n + k] > 0.0) alpha = -alpha;
        std::vector<double> v(n, 0.0);
        v[k + 1] = h[(k + 1) * n + k] - alpha;
        for (int i = k + 2; i < n; ++i) v[i] = h[i * n + k];
        double vv = 0.0;
        for (int i = k + 1; i < n; ++i) vv += v[i] * v[i];
        if (vv == 0.0) continue;
        // h = (I - 2 v v^T / vv) h (I - 2 v v^T / vv)
        for (int j = 0; j < n; ++j) {
            double s = 0.0;
            for (int i = k + 1; i < n; ++i) s += v[i] * h[i * n + j];
            s *= 2.0 / vv;
            for (int i = k + 1; i < n; ++i) h[i * n + j] -= s * v[i];
        }
        for (int i = 0; i < n; ++i) {
            double s = 0.0;
            for (int j = k + 1; j < n; ++j) s += h[i * n + j] * v[j];
            s *= 2.0 / vv;
            for (int j = k + 1; j < n; ++j) h[i * n + j] -= s * v[j];
        }
    }
    // shifted QR on the active window [lo, hi]
    const double eps = 1e-15;
    int hi = n - 1, iter = 0;
    while (hi >= 0) {
        if (hi == 0) {
            lambda[0] = h[0];
            break;
        }
        int lo = hi;  // bottom of the unreduced block
        while (lo > 0 &&
               std::fabs(h[lo * n + lo - 1]) > eps * (std::fabs(h[lo * n + lo]) + std::fabs(h[(lo - 1) * n + lo - 1])))
            --lo;
        if (lo == hi) {  // a 1 x 1 block has split off
            lambda[hi] = h[hi * n + hi];
            --hi;
            iter = 0;
            continue;
        }
        const double a = h[(hi - 1) * n + hi - 1], b = h[(hi - 1) * n + hi], c = h[hi * n + hi - 1],
                     d = h[hi * n + hi];
        const double disc = 0.25 * (a - d) * (a - d) + b * c;
        if (lo == hi - 1) {  // a 2 x 2 block: real pair or reject
            if (disc < 0.0) return false;
            const double m = 0.5 * (a + d), r = std::sqrt(disc);
            lambda[hi] = m + r;
            lambda[hi - 1] = m - r;
            hi -= 2;
            iter = 0;
            continue;
        }
        if (++iter > 60) return false;
        // Wilkinson shift: the eigenvalue of the trailing 2 x 2 block nearer to d (its real
        // part when the pair is complex, which keeps the iteration real)
        double mu = d;
        if (disc >= 0.0) {
            const double m = 0.5 * (a + d), r = std::sqrt(disc);
            mu = std::fabs(m + r - d) < std::fabs(m - r - d) ? m + r : m - r;
        } else {
            mu = 0.5 * (a + d);
        }
        if (iter % 11 == 10) mu += std::fabs(h[hi * n + hi - 1]);  // exceptional shift
        // one QR step on rows/columns lo..hi: H - mu I = Q R, H <- R Q + mu I (Givens)
        std::vector<double> cs(n), sn(n);
        for (int k = lo; k <= hi; ++k) h[k * n + k] -= mu;
        for (int k = lo; k < hi; ++k) {
            const double x = h[k * n + k], y = h[(k + 1) * n + k];
            const double r = std::hypot(x, y);
            const double cc = r == 0.0 ? 1.0 : x / r, ss = r == 0.0 ? 0.0 : y / r;
            cs[k] = cc;
            sn[k] = ss;
            for (int j = k; j < n; ++j) {
                const double t1 = h[k * n + j], t2 = h[(k + 1) * n + j];
                h[k * n + j] = cc * t1 + ss * t2;
                h[(k + 1) * n + j] = -ss * t1 + cc * t2;
            }
        }
        for (int k = lo; k < hi; ++k) {
            const double cc = cs[k], ss = sn[k];
            for (int i = 0; i <= std::min(k + 2, hi); ++i) {
                const double t1 = h[i * n + k], t2 = h[i * n + k + 1];
                h[i * n + k] = cc * t1 + ss * t2;
                h[i * n + k + 1] = -ss * t1 + cc * t2;
            }
        }
        for (int k = lo; k <= hi; ++k) h[k * n + k] += mu;
    }
    return true;
}

bool eigenvectors(int n, const double* A, const double* lambda, double* V) {
    std::vector<double> b((size_t)n * n), x(n);
    std::vector<int> piv;
    for (int c = 0; c < n; ++c) {
        // inverse iteration with the eigenvalue moved off by a relative 1e-10, so that the
        // shifted matrix factors
        const double shift = lambda[c] + 1e-10 * (1.0 + std::fabs(lambda[c]));
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) b[i * n + j] = A[i * n + j] - (i == j ? shift : 0.0);
        if (!lu(n, b, piv)) return false;
        for (int i = 0; i < n; ++i) x[i] = 1.0 + 0.1 * i;
        for (int it = 0; it < 2; ++it) {
            lu_solve(n, b, piv, x.data());
            double nrm = 0.0;
            for (double v : x) nrm += v * v;
            nrm = std::sqrt(nrm);
            if (!(nrm > 0.0) || !std::isfinite(nrm)) return false;
            for (double& v : x) v /= nrm;
        }
        for (int i = 0; i < n; ++i) V[i * n + c] = x[i];
    }
    return true;
}

bool kron_fit(int K, const double* D, KronFit& f) {
    const int K2 = K * K;
    auto at = [&](int j, int i, int l, int k) { return D[(size_t)(j * K + i) * K2 + l * K + k]; };
    std::vector<double> ax((size_t)K * K, 0.0), ay((size_t)K * K, 0.0);
    for (int i = 0; i < K; ++i)
        for (int k = 0; k < K; ++k) {
            if (i == k) continue;
            double sx = 0.0, sy = 0.0;
            for (int j = 0; j < K; ++j) {
                sx += at(j, i, j, k);  // Ax[i][k]: mean over j of D[(j,i),(j,k)]
                sy += at(i, j, k, j);  // Ay[i][k]: mean over j of D[(i,j),(k,j)]
            }
            ax[i * K + k] = sx / K;
            ay[i * K + k] = sy / K;
        }
    // diagonal d[j][i] ~ Ax[i][i] + Ay[j][j]: column means to Ax, row means minus the grand
    // mean to Ay
    double grand = 0.0;
    std::vector<double> rowm(K, 0.0), colm(K, 0.0);
    for (int j = 0; j < K; ++j)
        for (int i = 0; i < K; ++i) {
            const double d = at(j, i, j, i);
            rowm[j] += d / K;
            colm[i] += d / K;
            grand += d / (K * K);
        }
    for (int i = 0; i < K; ++i) ax[i * K + i] = colm[i];
    for (int j = 0; j < K; ++j) ay[j * K + j] = rowm[j] - grand;
    f.K = K;
    f.lx.assign(K, 0.0);
    f.ly.assign(K, 0.0);
    f.vx.assign((size_t)K * K, 0.0);
    f.vy.assign((size_t)K * K, 0.0);
    if (!real_eigenvalues(K, ax.data(), f.lx.data()) || !real_eigenvalues(K, ay.data(), f.ly.data())) return false;
    if (!eigenvectors(K, ax.data(), f.lx.data(), f.vx.data()) || !eigenvectors(K, ay.data(), f.ly.data(), f.vy.data()))
        return false;
    for (int j = 0; j < K; ++j)
        for (int i = 0; i < K; ++i)
            if (!(std::fabs(f.ly[j] + f.lx[i]) > 0.0)) return false;
    f.vxi = f.vx;
    f.vyi = f.vy;
    std::vector<int> piv;
    for (std::vector<double>* m : {&f.vxi, &f.vyi}) {  // inverses by LU, column by column
        std::vector<double> a(*m), e(K);
        if (!lu(K, a, piv)) return false;
        for (int c = 0; c < K; ++c) {
            std::fill(e.begin(), e.end(), 0.0);
            e[c] = 1.0;
            lu_solve(K, a, piv, e.data());
            for (int r = 0; r < K; ++r) (*m)[r * K + c] = e[r];
        }
    }
    return true;
}

void kron_apply(const KronFit& f, const double* r, double* z) {
    const int K = f.K;
    std::vector<double> t((size_t)K * K, 0.0), u((size_t)K * K, 0.0);
    // t = Vy^-1 R Vx^-T, scaled by 1 / (ly_j + lx_i)
    for (int j = 0; j < K; ++j)
        for (int i = 0; i < K; ++i) {
            double s = 0.0;
            for (int l = 0; l < K; ++l)
                for (int k = 0; k < K; ++k) s += f.vyi[j * K + l] * r[l * K + k] * f.vxi[i * K + k];
            t[j * K + i] = s / (f.ly[j] + f.lx[i]);
        }
    // z = Vy t Vx^T
    for (int j = 0; j < K; ++j)
        for (int i = 0; i < K; ++i) {
            double s = 0.0;
            for (int l = 0; l < K; ++l)
                for (int k = 0; k < K; ++k) s += f.vy[j * K + l] * t[l * K + k] * f.vx[i * K + k];
            z[j * K + i] = s;
        }
}

double kron_defect(const KronFit& f, const double* D) {
    const int K = f.K, K2 = K * K;
    // E = I - M D, column c = e_c - M (D e_c)
    std::vector<double> E((size_t)K2 * K2), col(K2), z(K2);
    for (int c = 0; c < K2; ++c) {
        for (int r = 0; r < K2; ++r) col[r] = D[(size_t)r * K2 + c];
        kron_apply(f, col.data(), z.data());
        for (int r = 0; r < K2; ++r) E[(size_t)r * K2 + c] = (r == c ? 1.0 : 0.0) - z[r];
    }
    // ||E||_2 by power iteration on E^T E (an estimate from below; it serves as a threshold)
    std::vector<double> x(K2, 1.0), y(K2);
    double sigma2 = 0.0;
    for (int it = 0; it < 100; ++it) {
        for (int r = 0; r < K2; ++r) {
            double s = 0.0;
            for (int c = 0; c < K2; ++c) s += E[(size_t)r * K2 + c] * x[c];
            y[r] = s;
        }
        for (int c = 0; c < K2; ++c) {
            double s = 0.0;
            for (int r = 0; r < K2; ++r) s += E[(size_t)r * K2 + c] * y[r];
            x[c] = s;
        }
        double nrm = 0.0;
        for (double v : x) nrm += v * v;
        nrm = std::sqrt(nrm);
        if (!(nrm > 0.0) || !std::isfinite(nrm)) return nrm == 0.0 ? 0.0 : INFINITY;
        sigma2 = nrm;  // ||E^T E x|| with ||x|| = 1 from the second step on
        for (double& v : x) v /= nrm;
    }
    return std::sqrt(sigma2);
}

void kron_store(const KronFit* f, double defect, int el, KronSmoother& ks) {
    const int K = ks.K;
    ks.defect[el] = f ? defect : INFINITY;
    ks.exact[el] = !f || !(defect <= kKronDefectMax);
    if (!f) return;
    const std::vector<double>* m[4] = {&f->vx, &f->vxi, &f->vy, &f->vyi};
    for (int a = 0; a < 4; ++a) std::copy(m[a]->begin(), m[a]->end(), ks.v.begin() + ((size_t)el * 4 + a) * K * K);
    std::copy(f->lx.begin(), f->lx.end(), ks.lam.begin() + (size_t)el * 2 * K);
    std::copy(f->ly.begin(), f->ly.end(), ks.lam.begin() + ((size_t)el * 2 + 1) * K);
}

void kron_fit_blocks(int K, int N, const double* diag, KronSmoother& ks) {
    const size_t K4 = (size_t)K * K * K * K;
    ks.K = K;
    ks.v.assign((size_t)N * 4 * K * K, 0.0);
    ks.lam.assign((size_t)N * 2 * K, 0.0);
    ks.exact.assign(N, 1);
    ks.defect.assign(N, 0.0);
#pragma omp parallel for schedule(dynamic, 64)
    for (int el = 0; el < N; ++el) {
        const double* D = diag + (size_t)el * K4;
        KronFit f;
        const bool ok = kron_fit(K, D, f);
        kron_store(ok ? &f : nullptr, ok ? kron_defect(f, D) : 0.0, el, ks);
    }
}

void kron_factor_arrays(const KronSmoother& ks, std::vector<double>& factors, std::vector<int>& exact_index) {
    const int K = ks.K, K2 = K * K, per = 4 * K2 + 2 * K;
    const int N = (int)ks.exact.size();
    factors.assign((size_t)N * per, 0.0);
    exact_index.assign(N, -1);
    int n_exact = 0;
    for (int el = 0; el < N; ++el) {
        if (ks.exact[el]) {
            exact_index[el] = n_exact++;
            continue;
        }
        std::copy(ks.v.begin() + (size_t)el * 4 * K2, ks.v.begin() + (size_t)(el + 1) * 4 * K2,
                  factors.begin() + (size_t)el * per);
        std::copy(ks.lam.begin() + (size_t)el * 2 * K, ks.lam.begin() + (size_t)(el + 1) * 2 * K,
                  factors.begin() + (size_t)el * per + 4 * K2);
    }
}

void kron_device_arrays(const KronSmoother& ks, const std::vector<double>& dinv, std::vector<double>& factors,
                        std::vector<int>& exact_index, std::vector<double>& exact_blocks) {
    const size_t K4 = (size_t)ks.K * ks.K * ks.K * ks.K;
    kron_factor_arrays(ks, factors, exact_index);
    exact_blocks.clear();
    for (size_t el = 0; el < exact_index.size(); ++el)
        if (exact_index[el] >= 0)
            exact_blocks.insert(exact_blocks.end(), dinv.begin() + el * K4, dinv.begin() + (el + 1) * K4);
}

}  // namespace ho2d
