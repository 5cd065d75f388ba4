// setup_device.cu -- Poisson setup on the device: the block assembly with the inverse of
// every diagonal block, the dense inverse of the coarsest level, and the conversions of
// the setup arrays to the FP32 / BF16 copies the preconditioner reads.
//
// Assembly (src/HO_2D.cpp:1533-1804 with the filter of 3023-3062): one thread per element
// runs assemble_element (assemble_element.hpp, the same source the host assembly runs)
// over interleaved scratch, then inverts its filtered diagonal block by the same
// Gauss-Jordan steps as the host. This file is compiled with -fmad=false, so every value
// matches the host assembly bit for bit.
//
// Coarsest level (the dense solve of src/HO_2D.cpp:3066-3072's AMG hierarchy, here the
// last level of the P0 / smoothed-aggregation hierarchy): Gauss-Jordan with partial
// pivoting, one pivot per step (a one-CTA pivot kernel, then a row-parallel elimination),
// in place in the row-padded FP64 storage the coarse cycle reads.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "assemble_element.hpp"
#include "kron_fit.hpp"
#include "device.cuh"
#include "fr_launch.hpp"
#include "host_amg.hpp"
#include "solver.hpp"
#include "solver_state.hpp"

namespace ho2d {

namespace {

// ---------------------------------------------------------------- block assembly
// Per element scratch (doubles): Lc K4, L K4, W K3, WN K3, Nm K2 -- element t of a chunk
// of n at t + i n.
inline size_t asm_scratch_values(int K) { return (size_t)2 * K * K * K * K + 2 * K * K * K + K * K; }

__global__ void __launch_bounds__(128) k_assemble(int el0, int n, AsmBases B, AsmTables tb, AsmMesh m, AsmOut o,
                                                  double* __restrict__ dinv, long long dstride,
                                                  double* __restrict__ diag, double* __restrict__ scratch,
                                                  unsigned long long* __restrict__ nnz) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int el = el0 + t;
    const int K = B.K, K2 = K * K, K3 = K2 * K, K4 = K2 * K2;
    const long long S = n;
    double* base = scratch + t;
    const AsmScratch sc{{base, S},
                        {base + (size_t)K4 * S, S},
                        {base + (size_t)2 * K4 * S, S},
                        {base + ((size_t)2 * K4 + K3) * S, S},
                        {base + ((size_t)2 * K4 + 2 * K3) * S, S}};
    double rk[kMaxK * kMaxK];
    int piv[kMaxK * kMaxK];
    auto inv = [&](int nn, Str<double> a) { return asm_invert(nn, a, rk, piv); };
    const int64_t cnt = assemble_element(el, B, tb, m, o, sc, inv);
    if (diag)  // the filtered diagonal block ([ij][rs]) for a host-side fit
        for (int i = 0; i < K4; ++i) diag[(size_t)el * K4 + i] = sc.Lc[i];
    asm_invert(K2, sc.Lc, rk, piv);
    double* di = dinv + (size_t)el * dstride;
    for (int ij = 0; ij < K2; ++ij)
        for (int rs = 0; rs < K2; ++rs) di[rs * K2 + ij] = sc.Lc[(long long)ij * K2 + rs];
    atomicAdd(nnz, (unsigned long long)cnt);
}

// ---------------------------------------------------------------- Kronecker-sum fit
// One thread per element: the fit of its filtered diagonal block (diag [N][K4]) and its
// defect ||I - M D||_2 (E: K4 interleaved scratch); the FP32 factors [vx vxi vy vyi lx ly]
// of a kept fit at el * fstride, zeros and exact[el] = 1 where the exact block stays.
__global__ void __launch_bounds__(128) k_kron_fit(int el0, int n, int K, const double* __restrict__ diag,
                                                  double* __restrict__ scratch, float* __restrict__ factors,
                                                  long long fstride, unsigned char* __restrict__ exact) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int el = el0 + t, K2 = K * K, K4 = K2 * K2, per = 4 * K2 + 2 * K;
    const Str<double> D{const_cast<double*>(diag) + (size_t)el * K4, 1};
    KronFitHD f;
    const bool ok = kf_fit(K, D, f);
    const double defect = ok ? kf_defect(f, D, Str<double>{scratch + t, n}) : 0.0;
    const bool ex = !ok || !(defect <= kKronDefectMax);
    exact[el] = ex ? 1 : 0;
    float* fo = factors + (size_t)el * fstride;
    if (ex) {
        for (int i = 0; i < per; ++i) fo[i] = 0.f;
        return;
    }
    const double* src[4] = {f.vx, f.vxi, f.vy, f.vyi};
    for (int a = 0; a < 4; ++a)
        for (int i = 0; i < K2; ++i) fo[a * K2 + i] = (float)src[a][i];
    for (int i = 0; i < K; ++i) {
        fo[4 * K2 + i] = (float)f.lx[i];
        fo[4 * K2 + K + i] = (float)f.ly[i];
    }
}

// ---------------------------------------------------------------- dense Gauss-Jordan
constexpr int kPivotThreads = 1024;

// Step k: the pivot (largest |a[i][k]|, i >= k, first index on ties), the row swap, the
// scaled pivot row into rk and the row itself, the multipliers of column k into lcol
// (zero for the pivot row). A zero pivot sets *err and every later step does nothing.
__global__ void __launch_bounds__(kPivotThreads) k_gj_pivot(double* __restrict__ a, int n, int w, int k,
                                                            double* __restrict__ rk, double* __restrict__ lcol,
                                                            int* __restrict__ piv, int* __restrict__ err) {
    if (*err) return;
    __shared__ double sv[kPivotThreads / 32];
    __shared__ int si[kPivotThreads / 32];
    __shared__ int sp;
    __shared__ double sd;
    double best = -1.0;
    int bi = n;
    for (int i = k + threadIdx.x; i < n; i += blockDim.x) {
        const double v = fabs(a[(size_t)i * w + k]);
        if (v > best) {
            best = v;
            bi = i;
        }
    }
    auto better = [](double v, int i, double bv, int bj) { return v > bv || (v == bv && i < bj); };
    for (int off = 16; off > 0; off >>= 1) {
        const double ov = __shfl_down_sync(0xffffffffu, best, off);
        const int oi = __shfl_down_sync(0xffffffffu, bi, off);
        if (better(ov, oi, best, bi)) {
            best = ov;
            bi = oi;
        }
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) {
        sv[wid] = best;
        si[wid] = bi;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = sv[0];
        int p = si[0];
        for (int q = 1; q < (int)(blockDim.x >> 5); ++q)
            if (better(sv[q], si[q], b, p)) {
                b = sv[q];
                p = si[q];
            }
        if (!(b > 0.0) || p >= n) {
            *err = 1;
            p = -1;
        }
        sp = p;
        if (p >= 0) piv[k] = p;
    }
    __syncthreads();
    const int p = sp;
    if (p < 0) return;
    if (p != k)
        for (int j = threadIdx.x; j < n; j += blockDim.x) {
            const double x = a[(size_t)k * w + j];
            a[(size_t)k * w + j] = a[(size_t)p * w + j];
            a[(size_t)p * w + j] = x;
        }
    __syncthreads();
    if (threadIdx.x == 0) sd = 1.0 / a[(size_t)k * w + k];
    __syncthreads();
    const double d = sd;
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        const double v = j == k ? 1.0 : a[(size_t)k * w + j];
        const double r = v * d;
        rk[j] = r;
        a[(size_t)k * w + j] = r;
    }
    for (int i = threadIdx.x; i < n; i += blockDim.x) lcol[i] = i == k ? 0.0 : a[(size_t)i * w + k];
}

// a[i][j] -= l_i rk[j] for every row but the pivot row (a[i][k] starts from zero)
__global__ void k_gj_elim(double* __restrict__ a, int n, int w, int k, const double* __restrict__ rk,
                          const double* __restrict__ lcol, const int* __restrict__ err) {
    if (*err) return;
    const int i = blockIdx.y, j = blockIdx.x * blockDim.x + threadIdx.x;
    const double l = lcol[i];
    if (l == 0.0 || j >= n) return;
    const double v = j == k ? 0.0 : a[(size_t)i * w + j];
    a[(size_t)i * w + j] = v - l * rk[j];
}

// the row swaps undone as column swaps, last pivot first (each thread one row)
__global__ void k_gj_unswap(double* __restrict__ a, int n, int w, const int* __restrict__ piv,
                            const int* __restrict__ err) {
    if (*err) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double* r = a + (size_t)i * w;
    for (int k = n - 1; k >= 0; --k) {
        const int p = piv[k];
        if (p != k) {
            const double x = r[k];
            r[k] = r[p];
            r[p] = x;
        }
    }
}

// ---------------------------------------------------------------- conversions
// rows x cols values, row strides ss (source) and ds (destination); idx (optional) picks the
// source row of each destination row
__global__ void k_rows_f32(const double* __restrict__ src, long long ss, const int* __restrict__ idx,
                           float* __restrict__ dst, long long ds, int rows, int cols) {
    const size_t total = (size_t)rows * cols;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += (size_t)gridDim.x * blockDim.x) {
        const size_t r = q / cols, c = q % cols;
        const size_t sr = idx ? (size_t)idx[r] : r;
        dst[r * ds + c] = (float)src[sr * ss + c];
    }
}

// BF16 of the FP32 rounding, to nearest with ties to even (finite values)
template <typename S>
__global__ void k_rows_bf16(const S* __restrict__ src, long long ss, unsigned short* __restrict__ dst, long long ds,
                            int rows, int cols) {
    const size_t total = (size_t)rows * cols;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += (size_t)gridDim.x * blockDim.x) {
        const size_t r = q / cols, c = q % cols;
        unsigned u = __float_as_uint((float)src[r * ss + c]);
        u += 0x7FFFu + ((u >> 16) & 1u);
        dst[r * ds + c] = (unsigned short)(u >> 16);
    }
}

unsigned conv_grid(size_t total) { return (unsigned)std::min<size_t>((total + 255) / 256, 148 * 16); }

}  // namespace

cudaError_t rows_to_f32(const double* src, long long ss, const int* idx, float* dst, long long ds, int rows, int cols,
                        cudaStream_t s) {
    if (rows <= 0 || cols <= 0) return cudaSuccess;
    k_rows_f32<<<conv_grid((size_t)rows * cols), 256, 0, s>>>(src, ss, idx, dst, ds, rows, cols);
    return cudaGetLastError();
}

cudaError_t rows_to_bf16(const double* src, long long ss, unsigned short* dst, long long ds, int rows, int cols,
                         cudaStream_t s) {
    if (rows <= 0 || cols <= 0) return cudaSuccess;
    k_rows_bf16<double><<<conv_grid((size_t)rows * cols), 256, 0, s>>>(src, ss, dst, ds, rows, cols);
    return cudaGetLastError();
}

// In-place inverse of the n x n matrix a (row stride w) on the device; *singular on a zero
// pivot. 2n + 1 launches on stream s, then one synchronisation for the flag.
cudaError_t dense_invert_device(double* a, int n, int w, cudaStream_t s, bool* singular) {
    *singular = false;
    if (n <= 0) return cudaSuccess;
    DeviceBuffer rk, lcol, piv, err;
    cudaError_t e;
    if ((e = rk.alloc((size_t)n * sizeof(double))) != cudaSuccess) return e;
    if ((e = lcol.alloc((size_t)n * sizeof(double))) != cudaSuccess) return e;
    if ((e = piv.alloc((size_t)n * sizeof(int))) != cudaSuccess) return e;
    if ((e = err.alloc(sizeof(int))) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(err.get(), 0, sizeof(int), s)) != cudaSuccess) return e;
    const dim3 eg((n + 255) / 256, n);
    for (int k = 0; k < n; ++k) {
        k_gj_pivot<<<1, kPivotThreads, 0, s>>>(a, n, w, k, rk.as<double>(), lcol.as<double>(), piv.as<int>(),
                                               err.as<int>());
        k_gj_elim<<<eg, 256, 0, s>>>(a, n, w, k, rk.as<double>(), lcol.as<double>(), err.as<int>());
    }
    k_gj_unswap<<<(n + 255) / 256, 256, 0, s>>>(a, n, w, piv.as<int>(), err.as<int>());
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    int h = 0;
    if ((e = cudaMemcpyAsync(&h, err.get(), sizeof(int), cudaMemcpyDeviceToHost, s)) != cudaSuccess) return e;
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;
    *singular = h != 0;
    return cudaSuccess;
}

// Poisson assembly on the device into the solver's buffers: inverse diagonal blocks
// (dinv64, padded rows), block row sums (rowsum64), column sums (colsum64), the boundary
// source (bsrc) and the block columns (bcol); the block sums, block columns and entry count
// come back to op_ for the coarse hierarchy. With kron_fit, the Kronecker-sum fit of every
// filtered diagonal block runs on the device too: its FP32 factors go to kron_f and the
// per-element exact-block flags to kron_ on the host.
Error Solver::assemble_device(bool kron_fit) {
    DeviceState& d = *d_;
    const int N = mesh_.n_el, K = in_.knod, K2 = K * K, K4 = K2 * K2, neb = mesh_.n_eb;
    op_ = PoissonOperator();
    op_.K2 = K2;
    // coefficient lists and bases
    const AsmCoefficients co = assembly_coefficients(B_);
    std::vector<AsmEntry> ent(co.vol);
    size_t off[5] = {0, 0, 0, 0, 0};
    for (int f = 0; f < 4; ++f) {
        off[f + 1] = ent.size();
        ent.insert(ent.end(), co.fw[f].begin(), co.fw[f].end());
    }
    std::vector<double> bas;
    for (const std::vector<double>* v : {&B_.sbb, &B_.sbgb, &B_.gR, &B_.D}) bas.insert(bas.end(), v->begin(), v->end());
    DeviceBuffer dent, dbas, dG, dGB, dfJ, dbidx, dnbr, dnside, dbsum, dnnz, scratch, ddiag;
    HO2D_CUDA(upload(dent, ent), "upload assembly coefficients");
    HO2D_CUDA(upload(dbas, bas), "upload bases");
    HO2D_CUDA(upload(dG, M_.G), "upload metrics");
    HO2D_CUDA(upload(dGB, M_.GB), "upload metrics");
    HO2D_CUDA(upload(dfJ, M_.fJ), "upload metrics");
    HO2D_CUDA(upload(dbidx, mesh_.bidx), "upload mesh tables");
    HO2D_CUDA(upload(dnbr, mesh_.nbr), "upload mesh tables");
    HO2D_CUDA(upload(dnside, mesh_.nbr_side), "upload mesh tables");
    const double* db = dbas.as<double>();
    const AsmBases ab{K, db, db + 2 * K, db + 4 * K, db + 6 * K, {B_.gp[0], B_.gp[1]}};
    const AsmEntry* de = dent.as<AsmEntry>();
    AsmTables tb{de, (int)co.vol.size(), {}, {}};
    for (int f = 0; f < 4; ++f) {
        tb.fw[f] = de + off[f + 1];
        tb.nfw[f] = (int)co.fw[f].size();
    }
    const AsmMesh am{dG.as<double>(),   dGB.as<double>(),   dfJ.as<double>(), dbidx.as<int>(),
                     dnbr.as<int>(),    dnside.as<int>(),   d.sw_p.as<int>()};
    // outputs
    const long long dstride = padded_count(K4, 8);
    HO2D_CUDA(d.dinv64.alloc(((size_t)N * dstride + 1) * sizeof(double)), "alloc block-Jacobi");
    HO2D_CUDA(cudaMemsetAsync(d.dinv64.get(), 0, d.dinv64.bytes(), d.stream), "memset");
    HO2D_CUDA(d.rowsum64.alloc((size_t)N * 5 * K2 * sizeof(double)), "alloc block row sums");
    HO2D_CUDA(d.colsum64.alloc((size_t)N * 5 * K2 * sizeof(double)), "alloc block column sums");
    HO2D_CUDA(d.bsrc.alloc((size_t)std::max(1, neb) * K2 * K * sizeof(double)), "alloc boundary source");
    HO2D_CUDA(d.bcol.alloc((size_t)N * 5 * sizeof(int)), "alloc block columns");
    HO2D_CUDA(dbsum.alloc((size_t)N * 5 * sizeof(double)), "alloc block sums");
    HO2D_CUDA(dnnz.alloc(sizeof(unsigned long long)), "alloc");
    HO2D_CUDA(cudaMemsetAsync(dnnz.get(), 0, sizeof(unsigned long long), d.stream), "memset");
    if (kron_fit) HO2D_CUDA(ddiag.alloc((size_t)N * K4 * sizeof(double)), "alloc diagonal blocks");
    const AsmOut ao{d.bsrc.as<double>(), d.rowsum64.as<double>(), d.colsum64.as<double>(), dbsum.as<double>(), nullptr,
                    d.bcol.as<int>()};
    // chunks of at most ~2 GB of scratch, a multiple of the CTA size
    const size_t per = asm_scratch_values(K) * sizeof(double);
    int chunk = (int)std::min<size_t>((size_t)N, std::max<size_t>(128, ((size_t)2 << 30) / per));
    chunk = (chunk + 127) / 128 * 128;
    HO2D_CUDA(scratch.alloc((size_t)chunk * per), "alloc assembly scratch");
    for (int el0 = 0; el0 < N; el0 += chunk) {
        const int n = std::min(chunk, N - el0);
        k_assemble<<<(n + 127) / 128, 128, 0, d.stream>>>(el0, n, ab, tb, am, ao, d.dinv64.as<double>(), dstride,
                                                          kron_fit ? ddiag.as<double>() : nullptr,
                                                          scratch.as<double>(), dnnz.as<unsigned long long>());
        HO2D_CUDA(cudaGetLastError(), "block assembly");
    }
    HO2D_CUDA(cudaStreamSynchronize(d.stream), "block assembly");
    op_.bsum.resize((size_t)N * 5);
    op_.block_col.resize((size_t)N * 5);
    unsigned long long nnz = 0;
    HO2D_CUDA(cudaMemcpy(op_.bsum.data(), dbsum.get(), op_.bsum.size() * sizeof(double), cudaMemcpyDeviceToHost),
              "download block sums");
    HO2D_CUDA(cudaMemcpy(op_.block_col.data(), d.bcol.get(), op_.block_col.size() * sizeof(int),
                         cudaMemcpyDeviceToHost),
              "download block columns");
    HO2D_CUDA(cudaMemcpy(&nnz, dnnz.get(), sizeof(nnz), cudaMemcpyDeviceToHost), "download entry count");
    op_.nnz = (int64_t)nnz;
    if (kron_fit) {
        const int per = 4 * K2 + 2 * K;
        const long long fstride = padded_count(per, 4);
        HO2D_CUDA(d.kron_f.alloc(((size_t)N * fstride + 1) * sizeof(float)), "alloc Kronecker factors");
        HO2D_CUDA(cudaMemsetAsync(d.kron_f.get(), 0, d.kron_f.bytes(), d.stream), "memset");
        DeviceBuffer dex, kscr;
        HO2D_CUDA(dex.alloc((size_t)N), "alloc exact flags");
        int kchunk = (int)std::min<size_t>((size_t)N, std::max<size_t>(128, ((size_t)2 << 30) / ((size_t)K4 * 8)));
        kchunk = (kchunk + 127) / 128 * 128;
        HO2D_CUDA(kscr.alloc((size_t)kchunk * K4 * sizeof(double)), "alloc fit scratch");
        for (int el0 = 0; el0 < N; el0 += kchunk) {
            const int n = std::min(kchunk, N - el0);
            k_kron_fit<<<(n + 127) / 128, 128, 0, d.stream>>>(el0, n, K, ddiag.as<double>(), kscr.as<double>(),
                                                              d.kron_f.as<float>(), fstride, dex.as<unsigned char>());
            HO2D_CUDA(cudaGetLastError(), "Kronecker-sum fit");
        }
        kron_ = KronSmoother();
        kron_.K = K;
        kron_.exact.resize(N);
        // (the handle's stream does not synchronise with the legacy stream's copies)
        HO2D_CUDA(cudaStreamSynchronize(d.stream), "Kronecker-sum fit");
        HO2D_CUDA(cudaMemcpy(kron_.exact.data(), dex.get(), (size_t)N, cudaMemcpyDeviceToHost), "download exact flags");
        kron_on_device_ = true;
    }
    return {0, ""};
}

Error Solver::get_poisson_setup(int which, int64_t len, double* out) {
    DeviceState& d = *d_;
    const int N = mesh_.n_el, K = in_.knod, K2 = K * K, K4 = K2 * K2;
    const int64_t need[6] = {(int64_t)N * K4, (int64_t)N * 5 * K2, (int64_t)N * 5 * K2, (int64_t)N * 5,
                             (int64_t)mesh_.n_eb * K2 * K, (int64_t)N * 5};
    if (which < 0 || which > 5) return {1, "unknown setup array"};
    if (len != need[which]) return {1, "buffer length does not match the setup array"};
    if (len == 0) return {0, ""};
    switch (which) {
        case 0:
            HO2D_CUDA(cudaMemcpy2D(out, (size_t)K4 * sizeof(double), d.dinv64.get(),
                                   (size_t)padded_count(K4, 8) * sizeof(double), (size_t)K4 * sizeof(double), N,
                                   cudaMemcpyDeviceToHost),
                      "download inverse blocks");
            break;
        case 1:
            HO2D_CUDA(cudaMemcpy(out, d.rowsum64.get(), len * sizeof(double), cudaMemcpyDeviceToHost), "download");
            break;
        case 2:
            HO2D_TRY(ensure_host_colsum());
            std::copy(op_.colsum.begin(), op_.colsum.end(), out);
            break;
        case 3:
            std::copy(op_.bsum.begin(), op_.bsum.end(), out);
            break;
        case 4:
            HO2D_CUDA(cudaMemcpy(out, d.bsrc.get(), len * sizeof(double), cudaMemcpyDeviceToHost), "download");
            break;
        default:
            for (int64_t i = 0; i < len; ++i) out[i] = (double)op_.block_col[i];
    }
    return {0, ""};
}

}  // namespace ho2d
