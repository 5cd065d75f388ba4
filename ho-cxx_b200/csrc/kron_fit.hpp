// kron_fit.hpp -- the Kronecker-sum fit of an element's diagonal Poisson block, as one
// source for the host (host_kron.cpp) and the device (setup_device.cu, one element per
// thread).
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
// with the computed eigenvalue on the original matrix. The fit's quality is ||I - M D||_2
// by power iteration on E^T E.
//
// Only IEEE operations, fabs and sqrt are used (the Givens radius is a scaled square root
// written out here), and the device file is compiled with -fmad=false, so the host and
// the device fits agree bit for bit.
#pragma once

#include <cmath>

#include "assemble_element.hpp"  // Str, HO2D_ASM_HD

namespace ho2d {

constexpr int kKronMaxK = 8;

struct KronFitHD {
    int K;
    double vx[kKronMaxK * kKronMaxK], vxi[kKronMaxK * kKronMaxK];
    double vy[kKronMaxK * kKronMaxK], vyi[kKronMaxK * kKronMaxK];
    double lx[kKronMaxK], ly[kKronMaxK];
};

// x is neither infinite nor NaN
HO2D_ASM_HD inline bool kf_finite(double x) { return x - x == 0.0; }

// sqrt(x^2 + y^2) without overflow: the larger magnitude times sqrt(1 + r^2)
HO2D_ASM_HD inline double kf_radius(double x, double y) {
    const double ax = fabs(x), ay = fabs(y);
    const double m = ax > ay ? ax : ay, s = ax > ay ? ay : ax;
    if (m == 0.0) return 0.0;
    const double r = s / m;
    return m * sqrt(1.0 + r * r);
}

// LU with partial pivoting of the n x n row-major a (in place); false if singular
HO2D_ASM_HD inline bool kf_lu(int n, double* a, int* piv) {
    for (int k = 0; k < n; ++k) {
        int p = k;
        for (int i = k + 1; i < n; ++i)
            if (fabs(a[i * n + k]) > fabs(a[p * n + k])) p = i;
        piv[k] = p;
        if (a[p * n + k] == 0.0) return false;
        if (p != k)
            for (int j = 0; j < n; ++j) {
                const double t = a[k * n + j];
                a[k * n + j] = a[p * n + j];
                a[p * n + j] = t;
            }
        for (int i = k + 1; i < n; ++i) {
            const double l = a[i * n + k] / a[k * n + k];
            a[i * n + k] = l;
            for (int j = k + 1; j < n; ++j) a[i * n + j] -= l * a[k * n + j];
        }
    }
    return true;
}

HO2D_ASM_HD inline void kf_lu_solve(int n, const double* a, const int* piv, double* x) {
    for (int k = 0; k < n; ++k) {
        const double t = x[k];
        x[k] = x[piv[k]];
        x[piv[k]] = t;
    }
    for (int i = 1; i < n; ++i)
        for (int j = 0; j < i; ++j) x[i] -= a[i * n + j] * x[j];
    for (int i = n - 1; i >= 0; --i) {
        for (int j = i + 1; j < n; ++j) x[i] -= a[i * n + j] * x[j];
        x[i] /= a[i * n + i];
    }
}

// Real eigenvalues of the n x n row-major A (false if a complex pair or no convergence).
HO2D_ASM_HD inline bool kf_real_eigenvalues(int n, const double* A, double* lambda) {
    double h[kKronMaxK * kKronMaxK], v[kKronMaxK], cs[kKronMaxK], sn[kKronMaxK];
    for (int i = 0; i < n * n; ++i) h[i] = A[i];
    // Householder reduction to upper Hessenberg form: zero column k below row k + 1
    for (int k = 0; k + 2 < n; ++k) {
        double alpha = 0.0;
        for (int i = k + 1; i < n; ++i) alpha += h[i * n + k] * h[i * n + k];
        alpha = sqrt(alpha);
        if (alpha == 0.0) continue;
        if (h[(k + 1) * n + k] > 0.0) alpha = -alpha;
        for (int i = 0; i < n; ++i) v[i] = 0.0;
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
               fabs(h[lo * n + lo - 1]) > eps * (fabs(h[lo * n + lo]) + fabs(h[(lo - 1) * n + lo - 1])))
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
            const double m = 0.5 * (a + d), r = sqrt(disc);
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
            const double m = 0.5 * (a + d), r = sqrt(disc);
            mu = fabs(m + r - d) < fabs(m - r - d) ? m + r : m - r;
        } else {
            mu = 0.5 * (a + d);
        }
        if (iter % 11 == 10) mu += fabs(h[hi * n + hi - 1]);  // exceptional shift
        // one QR step on rows/columns lo..hi: H - mu I = Q R, H <- R Q + mu I (Givens)
        for (int k = lo; k <= hi; ++k) h[k * n + k] -= mu;
        for (int k = lo; k < hi; ++k) {
            const double x = h[k * n + k], y = h[(k + 1) * n + k];
            const double r = kf_radius(x, y);
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
            const int top = k + 2 < hi ? k + 2 : hi;
            for (int i = 0; i <= top; ++i) {
                const double t1 = h[i * n + k], t2 = h[i * n + k + 1];
                h[i * n + k] = cc * t1 + ss * t2;
                h[i * n + k + 1] = -ss * t1 + cc * t2;
            }
        }
        for (int k = lo; k <= hi; ++k) h[k * n + k] += mu;
    }
    return true;
}

// Eigenvectors for those eigenvalues as the columns of V (false if that fails).
HO2D_ASM_HD inline bool kf_eigenvectors(int n, const double* A, const double* lambda, double* V) {
    double b[kKronMaxK * kKronMaxK], x[kKronMaxK];
    int piv[kKronMaxK];
    for (int c = 0; c < n; ++c) {
        // inverse iteration with the eigenvalue moved off by a relative 1e-10, so that the
        // shifted matrix factors
        const double shift = lambda[c] + 1e-10 * (1.0 + fabs(lambda[c]));
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) b[i * n + j] = A[i * n + j] - (i == j ? shift : 0.0);
        if (!kf_lu(n, b, piv)) return false;
        for (int i = 0; i < n; ++i) x[i] = 1.0 + 0.1 * i;
        for (int it = 0; it < 2; ++it) {
            kf_lu_solve(n, b, piv, x);
            double nrm = 0.0;
            for (int i = 0; i < n; ++i) nrm += x[i] * x[i];
            nrm = sqrt(nrm);
            if (!(nrm > 0.0) || !kf_finite(nrm)) return false;
            for (int i = 0; i < n; ++i) x[i] /= nrm;
        }
        for (int i = 0; i < n; ++i) V[i * n + c] = x[i];
    }
    return true;
}

// Fit and factor D ([ij][rs], K2 x K2 row-major view); false when an eigenvalue is complex,
// a factor is singular or some ly_j + lx_i vanishes.
HO2D_ASM_HD inline bool kf_fit(int K, Str<double> D, KronFitHD& f) {
    const int K2 = K * K;
    auto at = [&](int j, int i, int l, int k) { return D[(long long)(j * K + i) * K2 + l * K + k]; };
    double ax[kKronMaxK * kKronMaxK], ay[kKronMaxK * kKronMaxK];
    for (int i = 0; i < K * K; ++i) ax[i] = ay[i] = 0.0;
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
    double grand = 0.0, rowm[kKronMaxK], colm[kKronMaxK];
    for (int i = 0; i < K; ++i) rowm[i] = colm[i] = 0.0;
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
    for (int i = 0; i < K; ++i) f.lx[i] = f.ly[i] = 0.0;
    for (int i = 0; i < K * K; ++i) f.vx[i] = f.vy[i] = 0.0;
    if (!kf_real_eigenvalues(K, ax, f.lx) || !kf_real_eigenvalues(K, ay, f.ly)) return false;
    if (!kf_eigenvectors(K, ax, f.lx, f.vx) || !kf_eigenvectors(K, ay, f.ly, f.vy)) return false;
    for (int j = 0; j < K; ++j)
        for (int i = 0; i < K; ++i)
            if (!(fabs(f.ly[j] + f.lx[i]) > 0.0)) return false;
    // inverses by LU, column by column
    double a[kKronMaxK * kKronMaxK], e[kKronMaxK];
    int piv[kKronMaxK];
    for (int w = 0; w < 2; ++w) {
        const double* m = w ? f.vy : f.vx;
        double* mi = w ? f.vyi : f.vxi;
        for (int i = 0; i < K * K; ++i) a[i] = m[i];
        if (!kf_lu(K, a, piv)) return false;
        for (int c = 0; c < K; ++c) {
            for (int r = 0; r < K; ++r) e[r] = 0.0;
            e[c] = 1.0;
            kf_lu_solve(K, a, piv, e);
            for (int r = 0; r < K; ++r) mi[r * K + c] = e[r];
        }
    }
    return true;
}

// z = (I (x) Ax + Ay (x) I)^-1 r for r, z [j][i]
HO2D_ASM_HD inline void kf_apply(const KronFitHD& f, const double* r, double* z) {
    const int K = f.K;
    double t[kKronMaxK * kKronMaxK];
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

// ||I - M D||_2 of the fitted inverse M against D ([ij][rs] view), by 100 steps of power
// iteration on E^T E (an estimate from below; it serves as a threshold); E is K^4 scratch.
HO2D_ASM_HD inline double kf_defect(const KronFitHD& f, Str<double> D, Str<double> E) {
    const int K = f.K, K2 = K * K;
    double col[kKronMaxK * kKronMaxK], z[kKronMaxK * kKronMaxK];
    // E = I - M D, column c = e_c - M (D e_c)
    for (int c = 0; c < K2; ++c) {
        for (int r = 0; r < K2; ++r) col[r] = D[(long long)r * K2 + c];
        kf_apply(f, col, z);
        for (int r = 0; r < K2; ++r) E[(long long)r * K2 + c] = (r == c ? 1.0 : 0.0) - z[r];
    }
    double x[kKronMaxK * kKronMaxK], y[kKronMaxK * kKronMaxK];
    for (int i = 0; i < K2; ++i) x[i] = 1.0;
    double sigma2 = 0.0;
    for (int it = 0; it < 100; ++it) {
        for (int r = 0; r < K2; ++r) {
            double s = 0.0;
            for (int c = 0; c < K2; ++c) s += E[(long long)r * K2 + c] * x[c];
            y[r] = s;
        }
        for (int c = 0; c < K2; ++c) {
            double s = 0.0;
            for (int r = 0; r < K2; ++r) s += E[(long long)r * K2 + c] * y[r];
            x[c] = s;
        }
        double nrm = 0.0;
        for (int i = 0; i < K2; ++i) nrm += x[i] * x[i];
        nrm = sqrt(nrm);
        if (!(nrm > 0.0) || !kf_finite(nrm)) return nrm == 0.0 ? 0.0 : INFINITY;
        sigma2 = nrm;  // ||E^T E x|| with ||x|| = 1 from the second step on
        for (int i = 0; i < K2; ++i) x[i] /= nrm;
    }
    return sqrt(sigma2);
}

}  // namespace ho2d
