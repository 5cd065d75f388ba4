// shim_eigen.hpp -- the subset of the Eigen API that src/HO_2D.cpp calls
// (src/HO_2D.hpp:34-41,51,133-141; src/HO_2D.cpp:1548,1669,1917,2954-3009).
// TEST INFRASTRUCTURE ONLY: names and signatures follow Eigen 3.3 so the reference
// compiles unmodified; the arithmetic is shimla's (shim_linalg.hpp).
#pragma once

#include "shim_linalg.hpp"

namespace Eigen {

template <typename T>
class Triplet {
  public:
    Triplet(int r = 0, int c = 0, const T& v = T(0)) : r_(r), c_(c), v_(v) {}
    int row() const { return r_; }
    int col() const { return c_; }
    const T& value() const { return v_; }

  private:
    int r_, c_;
    T v_;
};

class VectorXd {
  public:
    VectorXd() {}
    explicit VectorXd(int n) : v_(n, 0.0) {}
    void resize(int n) { v_.assign(n, 0.0); }
    int size() const { return (int)v_.size(); }
    double& operator()(int i) { return v_[i]; }
    double operator()(int i) const { return v_[i]; }
    double* data() { return v_.data(); }
    const double* data() const { return v_.data(); }

  private:
    std::vector<double> v_;
};

class MatrixXd {
  public:
    MatrixXd() : r_(0), c_(0) {}
    MatrixXd(int r, int c) : r_(r), c_(c), a_((size_t)r * c, 0.0) {}
    double& operator()(int i, int j) { return a_[(size_t)i * c_ + j]; }
    double operator()(int i, int j) const { return a_[(size_t)i * c_ + j]; }
    int rows() const { return r_; }
    int cols() const { return c_; }
    // Gauss-Jordan inverse with partial pivoting.
    MatrixXd inverse() const {
        const int n = r_;
        MatrixXd a(*this), inv(n, n);
        for (int i = 0; i < n; ++i) inv(i, i) = 1.0;
        for (int k = 0; k < n; ++k) {
            int p = k;
            for (int i = k + 1; i < n; ++i)
                if (std::fabs(a(i, k)) > std::fabs(a(p, k))) p = i;
            if (p != k)
                for (int j = 0; j < n; ++j) { std::swap(a(k, j), a(p, j)); std::swap(inv(k, j), inv(p, j)); }
            const double d = a(k, k);
            for (int j = 0; j < n; ++j) { a(k, j) /= d; inv(k, j) /= d; }
            for (int i = 0; i < n; ++i) {
                if (i == k) continue;
                const double l = a(i, k);
                if (l == 0.0) continue;
                for (int j = 0; j < n; ++j) { a(i, j) -= l * a(k, j); inv(i, j) -= l * inv(k, j); }
            }
        }
        return inv;
    }

  private:
    int r_, c_;
    std::vector<double> a_;
};

template <typename T, int Options = 0>
class SparseMatrix {
  public:
    struct Storage {
        void squeeze() {}
    };
    void resize(int r, int c) { csr_ = shimla::Csr(); csr_.n = r; csr_.m = c; csr_.ptr.assign(r + 1, 0); }
    Storage& data() { return storage_; }
    template <typename It>
    void setFromTriplets(It begin, It end) {  // duplicates are summed
        std::vector<std::vector<std::pair<int, double>>> rows(csr_.n);
        for (It it = begin; it != end; ++it) rows[it->row()].push_back({it->col(), it->value()});
        csr_.col.clear();
        csr_.val.clear();
        for (int i = 0; i < csr_.n; ++i) {
            auto& r = rows[i];
            std::sort(r.begin(), r.end(), [](const std::pair<int, double>& a, const std::pair<int, double>& b) {
                return a.first < b.first;
            });
            for (size_t k = 0; k < r.size(); ++k) {
                if (!csr_.col.empty() && (int)csr_.col.size() > csr_.ptr[i] && csr_.col.back() == r[k].first)
                    csr_.val.back() += r[k].second;
                else { csr_.col.push_back(r[k].first); csr_.val.push_back(r[k].second); }
            }
            csr_.ptr[i + 1] = (int)csr_.col.size();
        }
    }
    void makeCompressed() {}
    const shimla::Csr& csr() const { return csr_; }

  private:
    shimla::Csr csr_;
    Storage storage_;
};

enum { RowMajor = 1, Lower = 1, Upper = 2 };

template <typename T>
class IncompleteLUT {};  // the preconditioner type is only named; shimla's AMG is used

template <typename MatrixType, typename Preconditioner = IncompleteLUT<double>>
class BiCGSTAB {
  public:
    void compute(const MatrixType& A) {
        A_ = &A.csr();
        amg_.build(*A_);
    }
    VectorXd solve(const VectorXd& b) {
        VectorXd x(b.size());
        auto r = shimla::bicgstab(*A_, amg_, b.data(), x.data(), std::numeric_limits<double>::epsilon(),
                                  2 * b.size());
        iters_ = std::get<0>(r);
        err_ = std::get<1>(r);
        return x;
    }
    int iterations() const { return iters_; }
    double error() const { return err_; }

  private:
    const shimla::Csr* A_ = nullptr;
    shimla::SaAmg amg_;
    int iters_ = 0;
    double err_ = 0.0;
};

}  // namespace Eigen
