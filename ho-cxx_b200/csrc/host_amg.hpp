// host_amg.hpp -- P0 coarse operator and its smoothed-aggregation hierarchy (host setup).
#pragma once

#include <vector>

#include "host.hpp"

namespace ho2d {

// The coarsest level is inverted densely once it has at most this many rows; the device
// applies the inverse as one grid-wide matrix-vector product (4096^2 FP32 values = 64 MB).
// Level 0 is inverted densely only below kDenseMaxFirst rows: beyond that one coarsening
// step is cheaper than a large dense P0 level.
constexpr int kDenseMax = 4096;
constexpr int kDenseMaxFirst = 1024;

struct Csr {
    int n = 0, m = 0;
    std::vector<int> ptr, col;
    std::vector<double> val;
};

struct AmgLevel {
    Csr A, P, R;            // P, R empty on the coarsest level
    std::vector<double> m;  // SPAI-0 smoother weights
    // The V(1,1) cycle of this level with pre-smoothing from zero, u' = m .* f, and
    // post-smoothing u = u'' + m .* (f - A u''), u'' = u' + P u_c, as three fixed operators:
    //   f_c = M f,  u = S f + Q u_c   with
    //   M = R (I - A diag(m)),  S = 2 diag(m) - diag(m) A diag(m),  Q = (I - diag(m) A) P.
    Csr M, S, Q;  // empty on the coarsest level
};

// Row-padded (ELL) copy of a sparse matrix: every row holds exactly w entries (w a
// multiple of 4), padding entries have column 0 and value 0, so a row is read without a
// row pointer and every row starts on a 16-byte boundary.
struct Ell {
    int n = 0, m = 0, w = 0;
    std::vector<int> col;     // [n][w]
    std::vector<double> val;  // [n][w]
};
Ell to_ell(const Csr& A);

struct CoarseHierarchy {
    std::vector<AmgLevel> levels;  // levels[0] is the P0 (one value per element) operator
    int n_dense = 0;
    std::vector<double> dense_inv;  // row-major inverse of the coarsest operator
};

// A1 = P^T A P for P = element indicator: the sum of each K^2 x K^2 block.
Csr p0_coarse_operator(const PoissonOperator& op, int N);
// Coarsens A1 until a level has at most dense_max rows (level 0 itself: at most
// dense_max_first rows) and inverts that level densely.
// invert_dense = false leaves H.dense_inv empty (the caller inverts the last level).
Error build_coarse_hierarchy(const Csr& A1, CoarseHierarchy& H, int dense_max = kDenseMax,
                             int dense_max_first = kDenseMaxFirst, bool invert_dense = true);

}  // namespace ho2d
