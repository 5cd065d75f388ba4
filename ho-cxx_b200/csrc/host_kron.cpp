// host_kron.cpp -- the Kronecker-sum approximation of an element's diagonal Poisson block,
// for a smoother that stores O(K^2) values per element instead of the K^4 of the inverse.
// The fit itself (kron_fit.hpp) is shared with the device setup; this file holds the host
// entry points and the per-element storage.
#include <algorithm>
#include <cmath>
#include <vector>

#include "host.hpp"
#include "kron_fit.hpp"

namespace ho2d {

namespace {

KronFit to_host(const KronFitHD& h) {
    const int K = h.K;
    KronFit f;
    f.K = K;
    f.vx.assign(h.vx, h.vx + K * K);
    f.vxi.assign(h.vxi, h.vxi + K * K);
    f.vy.assign(h.vy, h.vy + K * K);
    f.vyi.assign(h.vyi, h.vyi + K * K);
    f.lx.assign(h.lx, h.lx + K);
    f.ly.assign(h.ly, h.ly + K);
    return f;
}

KronFitHD to_hd(const KronFit& f) {
    KronFitHD h{};
    const int K = f.K;
    h.K = K;
    std::copy(f.vx.begin(), f.vx.begin() + K * K, h.vx);
    std::copy(f.vxi.begin(), f.vxi.begin() + K * K, h.vxi);
    std::copy(f.vy.begin(), f.vy.begin() + K * K, h.vy);
    std::copy(f.vyi.begin(), f.vyi.begin() + K * K, h.vyi);
    std::copy(f.lx.begin(), f.lx.begin() + K, h.lx);
    std::copy(f.ly.begin(), f.ly.begin() + K, h.ly);
    return h;
}

}  // namespace

bool real_eigenvalues(int n, const double* A, double* lambda) {
    if (n < 1 || n > kKronMaxK) return false;
    return kf_real_eigenvalues(n, A, lambda);
}

bool eigenvectors(int n, const double* A, const double* lambda, double* V) {
    if (n < 1 || n > kKronMaxK) return false;
    return kf_eigenvectors(n, A, lambda, V);
}

bool kron_fit(int K, const double* D, KronFit& f) {
    if (K < 1 || K > kKronMaxK) return false;
    KronFitHD h{};
    const bool ok = kf_fit(K, Str<double>{const_cast<double*>(D), 1}, h);
    f = to_host(h);
    return ok;
}

void kron_apply(const KronFit& f, const double* r, double* z) {
    const KronFitHD h = to_hd(f);
    kf_apply(h, r, z);
}

double kron_defect(const KronFit& f, const double* D) {
    const int K2 = f.K * f.K;
    std::vector<double> E((size_t)K2 * K2);
    const KronFitHD h = to_hd(f);
    return kf_defect(h, Str<double>{const_cast<double*>(D), 1}, Str<double>{E.data(), 1});
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
    const bool have = ks.v.size() == (size_t)N * 4 * K2;  // (a device fit keeps only the flags)
    factors.assign(have ? (size_t)N * per : 0, 0.0);
    exact_index.assign(N, -1);
    int n_exact = 0;
    for (int el = 0; el < N; ++el) {
        if (ks.exact[el]) {
            exact_index[el] = n_exact++;
            continue;
        }
        if (!have) continue;
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
