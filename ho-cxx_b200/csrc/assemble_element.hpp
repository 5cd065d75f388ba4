// assemble_element.hpp -- one element's rows of the block Poisson operator, as one source
// for the host (host_setup.cpp, one element per OpenMP iteration) and the device
// (setup_device.cu, one element per thread).
//
// Follows src/HO_2D.cpp:1533-1804 (form_Laplace_operator_matrix) with the |a| > 1e-14
// filter of 3023-3062: the element-interior and face couplings are linear in the metric
// terms G and GB, so they are evaluated from precomputed coefficient lists (AsmEntry, one
// per (row, metric slot)); Dirichlet faces add to the boundary source, Neumann faces add
// the inverse of the K x K face system, interior faces fill the neighbour's block.
//
// Both compilations run the same IEEE operations in the same order: the host code is built
// for baseline x86-64 (no fused multiply-add) and the device file with -fmad=false, and
// the only math functions used are fabs and sqrt (exact on both). So the device assembly
// reproduces the host's bits.
//
// Scratch arrays are strided views: stride 1 on the host; on the device the elements of a
// chunk are interleaved (stride = chunk size), so a warp's accesses coalesce.
#pragma once

#include <cmath>
#include <cstdint>

#ifdef __CUDACC__
#define HO2D_ASM_HD __host__ __device__
#else
#define HO2D_ASM_HD
#endif

namespace ho2d {

struct AsmEntry {
    int row, g;  // output row, metric slot
    double c;
};

template <typename T>
struct Str {
    T* p;
    long long s;
    HO2D_ASM_HD T& operator[](long long i) const { return p[i * s]; }
};

struct AsmBases {
    int K;
    const double *sbb, *sbgb, *gR, *D;  // [K][2], [K][2], [K][2], [K][K]
    double gp[2];
};

// coefficient lists: volume (rows ij * K2 + rs over G) and the four faces (d, t) -> d * 2 + t
// (rows ij * K + q over G)
struct AsmTables {
    const AsmEntry* vol;
    int nvol;
    const AsmEntry* fw[4];
    int nfw[4];
};

struct AsmMesh {
    const double *G, *GB, *fJ;           // [N][K2][2][2], [N][2][2][K][2], [N][4][K]
    const int *bidx, *nbr, *nbr_side;    // [N][4] by element side
    const int* sw_p;                     // [N_eb]
};

// outputs: slot-indexed arrays as in PoissonOperator (host.hpp); blocks (optional) in the
// transposed [rs][ij] storage
struct AsmOut {
    double *bsrc, *rowsum, *colsum, *bsum, *blocks;
    int* block_col;
};

struct AsmScratch {
    Str<double> Lc, L, W, WN, Nm;  // K4, K4, K3, K3, K2
};

HO2D_ASM_HD inline int asm_rs_of(int p, int q, int d, int K) {
    return (p * d + q * (1 - d)) * K + (p * (1 - d) + q * d);
}
HO2D_ASM_HD inline int asm_bf_of(int side, int k, int K) { return (side / 2) * (K - 2 * k - 1) + k; }

// In-place Gauss-Jordan inverse with partial pivoting of the n x n row-major a (the
// reference algorithm of host_setup.cpp's invert, on a strided view): pivot row scaled
// into rk, eliminated from every other row, row swaps undone as column swaps.
HO2D_ASM_HD inline bool asm_invert(int n, Str<double> m, double* rk, int* piv) {
    for (int k = 0; k < n; ++k) {
        int p = k;
        for (int i = k + 1; i < n; ++i)
            if (fabs(m[(long long)i * n + k]) > fabs(m[(long long)p * n + k])) p = i;
        if (m[(long long)p * n + k] == 0.0) return false;
        piv[k] = p;
        if (p != k)
            for (int j = 0; j < n; ++j) {
                const double t = m[(long long)k * n + j];
                m[(long long)k * n + j] = m[(long long)p * n + j];
                m[(long long)p * n + j] = t;
            }
        const double d = 1.0 / m[(long long)k * n + k];
        m[(long long)k * n + k] = 1.0;
        for (int j = 0; j < n; ++j) rk[j] = m[(long long)k * n + j] * d;
        for (int j = 0; j < n; ++j) m[(long long)k * n + j] = rk[j];
        for (int i = 0; i < n; ++i) {
            if (i == k) continue;
            const double l = m[(long long)i * n + k];
            if (l == 0.0) continue;
            m[(long long)i * n + k] = 0.0;
            for (int j = 0; j < n; ++j) m[(long long)i * n + j] -= l * rk[j];
        }
    }
    for (int k = n - 1; k >= 0; --k)
        if (piv[k] != k)
            for (int i = 0; i < n; ++i) {
                const double t = m[(long long)i * n + k];
                m[(long long)i * n + k] = m[(long long)i * n + piv[k]];
                m[(long long)i * n + piv[k]] = t;
            }
    return true;
}

// Filter one block (|a| > 1e-14 survives), in place in src ([ij][rs]), and reduce it: row
// sums over rs (ascending), column sums over ij (ascending), the block sum in the stored
// order (rs outer, ij inner); the transposed block into blocks when kept. Returns the
// surviving entries.
HO2D_ASM_HD inline int64_t asm_store(int K2, Str<double> src, size_t slot_index, const AsmOut& o) {
    int64_t cnt = 0;
    for (int ij = 0; ij < K2; ++ij)
        for (int rs = 0; rs < K2; ++rs) {
            double v = src[(long long)ij * K2 + rs];
            if (!(fabs(v) > 1e-14)) v = 0.0;
            else ++cnt;
            src[(long long)ij * K2 + rs] = v;
        }
    double* rsum = o.rowsum + slot_index * K2;
    double* csum = o.colsum + slot_index * K2;
    for (int ij = 0; ij < K2; ++ij) {
        double acc = 0.0;
        for (int rs = 0; rs < K2; ++rs) acc += src[(long long)ij * K2 + rs];
        rsum[ij] = acc;
    }
    double tot = 0.0;
    for (int rs = 0; rs < K2; ++rs) {
        double acc = 0.0;
        for (int ij = 0; ij < K2; ++ij) {
            const double v = src[(long long)ij * K2 + rs];
            tot += v;
            acc += v;
        }
        csum[rs] = acc;
    }
    o.bsum[slot_index] = tot;
    if (o.blocks) {
        double* T = o.blocks + slot_index * (size_t)K2 * K2;
        for (int rs = 0; rs < K2; ++rs)
            for (int ij = 0; ij < K2; ++ij) T[(size_t)rs * K2 + ij] = src[(long long)ij * K2 + rs];
    }
    return cnt;
}

// Element el: the four face blocks stored (slots 1..4, empty slots zeroed), the boundary
// source of its boundary faces, and its own block filtered in s.Lc ([ij][rs]), reduced into
// slot 0 but not yet inverted. inv(n, view) inverts the K x K Neumann face systems.
// Returns the surviving entries of all five blocks.
template <class Inv>
HO2D_ASM_HD int64_t assemble_element(int el, const AsmBases& B, const AsmTables& tb, const AsmMesh& m,
                                     const AsmOut& o, const AsmScratch& s, Inv inv) {
    constexpr int i2f[4] = {3, 1, 0, 2};  // ijp -> element side (W, E, S, N)
    constexpr int f2i[4] = {2, 1, 3, 0};  // element side -> ijp
    const int K = B.K, K2 = K * K, K4 = K2 * K2;
    const double* gp = B.gp;
    const Str<double> Lc = s.Lc, L = s.L, W = s.W, WN = s.WN, Nm = s.Nm;
    for (int i = 0; i < K4; ++i) Lc[i] = 0.0;
    const double* G = m.G + (size_t)el * K2 * 4;
    for (int n = 0; n < tb.nvol; ++n) {
        const AsmEntry e = tb.vol[n];
        Lc[e.row] += e.c * G[e.g];
    }
    int64_t nnz = 0;
    o.block_col[(size_t)el * 5] = el;
    for (int ijp = 0; ijp < 4; ++ijp) {
        const int d = ijp / 2, t = ijp % 2, side = i2f[ijp];
        const size_t slot = (size_t)el * 5 + 1 + ijp;
        for (int i = 0; i < K2 * K; ++i) W[i] = 0.0;
        const AsmEntry* fw = tb.fw[d * 2 + t];
        for (int n = 0; n < tb.nfw[d * 2 + t]; ++n) {
            const AsmEntry e = fw[n];
            W[e.row] += e.c * G[e.g];
        }
        const double* GBe = m.GB + (((size_t)el * 2 + d) * 2 + t) * K * 2;
        const int eb = m.bidx[(size_t)el * 4 + side];
        if (eb >= 0) {
            o.block_col[slot] = -1;
            for (int i = 0; i < K2; ++i) o.rowsum[slot * K2 + i] = o.colsum[slot * K2 + i] = 0.0;
            o.bsum[slot] = 0.0;
            if (o.blocks)
                for (int i = 0; i < K4; ++i) o.blocks[slot * K4 + i] = 0.0;
            double* bs = o.bsrc + (size_t)eb * K2 * K;
            for (int i = 0; i < K2 * K; ++i) bs[i] = 0.0;
            for (int ij = 0; ij < K2; ++ij)
                for (int q = 0; q < K; ++q)
                    for (int p = 0; p < K; ++p)
                        Lc[(long long)ij * K2 + asm_rs_of(p, q, d, K)] -= 0.5 * W[ij * K + q] * B.sbb[p * 2 + t];
            if (m.sw_p[eb] == 0) {  // Dirichlet face (src/HO_2D.cpp:1640-1658)
                for (int ij = 0; ij < K2; ++ij) {
                    const int j = ij / K, i = ij % K;
                    for (int q = 0; q < K; ++q) bs[ij * K + asm_bf_of(side, q, K)] += W[ij * K + q];
                    const int alpha = i * d + j * (1 - d);
                    const double ngr = B.gR[(j * d + i * (1 - d)) * 2 + t];
                    const double A = GBe[alpha * 2 + d], Bc = GBe[alpha * 2 + 1 - d];
                    for (int mm = 0; mm < K; ++mm)
                        Lc[(long long)ij * K2 + asm_rs_of(mm, alpha, d, K)] +=
                            A * (B.sbgb[mm * 2 + t] - gp[t] * B.sbb[mm * 2 + t]) * ngr;
                    bs[ij * K + asm_bf_of(side, alpha, K)] += A * gp[t] * ngr;
                    for (int mm = 0; mm < K; ++mm) bs[ij * K + asm_bf_of(side, mm, K)] += Bc * B.D[mm * K + alpha] * ngr;
                }
            } else {  // Neumann face (src/HO_2D.cpp:1660-1714)
                for (int r = 0; r < K; ++r) {
                    for (int c = 0; c < K; ++c) Nm[r * K + c] = -GBe[r * 2 + 1 - d] * B.D[c * K + r];
                    Nm[r * K + r] += -GBe[r * 2 + d] * gp[t];
                }
                inv(K, Nm);
                const double sign = t ? 1.0 : -1.0;
                double sq[8];
                for (int p = 0; p < K; ++p) sq[p] = sqrt(GBe[p * 2 + d] * m.fJ[((size_t)el * 4 + ijp) * K + p]);
                for (int ij = 0; ij < K2; ++ij)
                    for (int c = 0; c < K; ++c) {
                        double acc = 0.0;
                        for (int q = 0; q < K; ++q) acc += W[ij * K + q] * Nm[q * K + c];
                        WN[ij * K + c] = acc;
                    }
                for (int ij = 0; ij < K2; ++ij) {
                    const int j = ij / K, i = ij % K;
                    const int alpha = i * d + j * (1 - d);
                    const double ngr = B.gR[(j * d + i * (1 - d)) * 2 + t];
                    bs[ij * K + asm_bf_of(side, alpha, K)] += sign * ngr * sq[alpha];
                    for (int p = 0; p < K; ++p) {
                        bs[ij * K + asm_bf_of(side, p, K)] -= sign * WN[ij * K + p] * sq[p];
                        const double tmp4 = B.sbgb[p * 2 + t] - gp[t] * B.sbb[p * 2 + t];
                        for (int c = 0; c < K; ++c)
                            Lc[(long long)ij * K2 + asm_rs_of(p, c, d, K)] += WN[ij * K + c] * tmp4 * GBe[c * 2 + d];
                    }
                }
            }
            continue;
        }
        // interior face (src/HO_2D.cpp:1716-1792): this face's neighbour block
        const int eln = m.nbr[(size_t)el * 4 + side];
        const int ijpm = f2i[m.nbr_side[(size_t)el * 4 + side]];
        const int dn = ijpm / 2, tn = ijpm % 2;
        const int rev = (d + t + dn + tn + 1) % 2;
        for (int i = 0; i < K4; ++i) L[i] = 0.0;
        for (int ij = 0; ij < K2; ++ij)
            for (int q = 0; q < K; ++q) {
                const int Mq = rev * (K - 2 * q - 1) + q;
                for (int p = 0; p < K; ++p)
                    L[(long long)ij * K2 + asm_rs_of(p, Mq, dn, K)] += 0.5 * W[ij * K + q] * B.sbb[p * 2 + tn];
            }
        const double* GBn = m.GB + (((size_t)eln * 2 + dn) * 2 + tn) * K * 2;
        const double sign = (t == tn) ? -1.0 : 1.0;
        for (int ij = 0; ij < K2; ++ij) {
            const int j = ij / K, i = ij % K;
            const int alpha = i * d + j * (1 - d);
            const int Ma = rev * (K - 2 * alpha - 1) + alpha;
            const double A = GBe[alpha * 2 + d], Bc = GBe[alpha * 2 + 1 - d];
            const double An = GBn[Ma * 2 + dn], Bn = GBn[Ma * 2 + 1 - dn];
            const double ngr = B.gR[(j * d + i * (1 - d)) * 2 + t];
            for (int mm = 0; mm < K; ++mm) {
                const int Mm = rev * (K - 2 * mm - 1) + mm;
                Lc[(long long)ij * K2 + asm_rs_of(mm, alpha, d, K)] +=
                    (0.5 * A * B.sbgb[mm * 2 + t] - 0.25 * gp[t] * A * B.sbb[mm * 2 + t] +
                     0.25 * sign * gp[tn] * An * B.sbb[mm * 2 + t]) * ngr;
                L[(long long)ij * K2 + asm_rs_of(mm, Ma, dn, K)] +=
                    (0.5 * sign * An * B.sbgb[mm * 2 + tn] - 0.25 * sign * gp[tn] * An * B.sbb[mm * 2 + tn] +
                     0.25 * gp[t] * A * B.sbb[mm * 2 + tn]) * ngr;
                const double coeff = 0.25 * (Bc * B.D[mm * K + alpha] + sign * Bn * B.D[Mm * K + Ma]) * ngr;
                for (int p = 0; p < K; ++p) {
                    Lc[(long long)ij * K2 + asm_rs_of(p, mm, d, K)] += coeff * B.sbb[p * 2 + t];
                    L[(long long)ij * K2 + asm_rs_of(p, Mm, dn, K)] += coeff * B.sbb[p * 2 + tn];
                }
            }
        }
        o.block_col[slot] = eln;
        nnz += asm_store(K2, L, slot, o);
    }
    nnz += asm_store(K2, Lc, (size_t)el * 5, o);
    return nnz;
}

}  // namespace ho2d
