// fr_launch.hpp -- argument blocks and launchers of the FR and Krylov kernels.
#pragma once

#include <cuda_runtime.h>

#include "device.cuh"

namespace ho2d {

template <typename T>
struct VelocityArgs {
    const T* psi;     // [N][K][K]
    const T* psi_tv;  // psi face traces (values, normal derivatives)
    const T* psi_tg;
    const T* w;       // stage input vorticity
    T* u;             // Cartesian velocity
    T* v;
    T* w_tv;          // omega face traces for the residual kernel
    T* w_tg;
    T* U_t;           // contravariant volumetric flux traces (U^xi on W/E, U^eta on S/N)
    double dt, re_inv;
};

template <typename T>
struct ResidualArgs {
    const T* w;       // stage input vorticity
    const T* u;
    const T* v;
    const T* w_tv;    // face traces written by the velocity kernel (all elements)
    const T* w_tg;
    const T* U_t;
    double dt, re_inv;
    int adv_type;     // 1 or 2
    int ti_type;      // 0 = stage only (no RK update), 1, 2, 4
    int stage;        // RK stage index
    double* omega;    // vorticity at time level n (FP64)
    double* acc;      // RK accumulator (FP64)
    T* w_next;        // next stage input (may alias nothing in the stage-only mode)
    T* rhs_diff;      // optional outputs (nullptr to skip)
    T* rhs_adv;
    T* k_out;
};

template <typename T>
cudaError_t launch_trace(int K, int N, const T* f, T* tv, T* tg, const DevBases<T>& b, cudaStream_t s);
template <typename T>
cudaError_t launch_velocity(int K, const FrGeom<T>& g, const DevBases<T>& b, const BcArrays& bc,
                            const VelocityArgs<T>& a, cudaStream_t s);
template <typename T>
cudaError_t launch_residual(int K, const FrGeom<T>& g, const DevBases<T>& b, const BcArrays& bc,
                            const ResidualArgs<T>& a, cudaStream_t s);
template <typename T>
cudaError_t launch_poisson_rhs(int K, int N, const int* face_nb, const T* w, const T* J, const double* bsrc,
                               const double* bc_p, double* rhs, cudaStream_t s);
cudaError_t launch_bc_update(int n_eb, int K, int ptype, double tc, double y_min, double y_max, const int* role,
                             const int* be_ijp, const int* sw_d, const double* edge_y, const BcArrays& bc,
                             cudaStream_t s);

// ---- Krylov (krylov.cu)
// Block-sparse operator: 5 K^2 x K^2 blocks per element row, transposed ([rs][ij]).
template <typename TM>
struct BsrOp {
    int N, K;
    const TM* blocks;  // [N][5][K2][K2]
    const int* col;    // [N][5]
    const TM* dinv;    // [N][K2][K2] inverse diagonal block (transposed), block-Jacobi
};

template <typename T>
struct BicgVectors {
    T *x, *r, *rhat, *p, *v, *s, *t, *ph, *sh;
    const T* b;
};

struct ReduceScratch {
    double* partials;    // [4 * max_blocks]
    unsigned* counter;   // 1 word, zero between launches
    KrylovScalars* sc;   // device scalars
};

template <typename T, typename TM>
cudaError_t krylov_init(const BsrOp<TM>& A, const BicgVectors<T>& v, const ReduceScratch& rs, double tol,
                        cudaStream_t s);
template <typename T, typename TM>
cudaError_t krylov_iteration(const BsrOp<TM>& A, const BicgVectors<T>& v, const ReduceScratch& rs, int max_iter,
                             cudaStream_t s);
// `reps` back-to-back launches of the solver's SpMV kernel (v = A ph, fused (rhat, v))
template <typename T, typename TM>
cudaError_t krylov_spmv_only(const BsrOp<TM>& A, const BicgVectors<T>& v, const ReduceScratch& rs, int reps,
                             cudaStream_t s);
// y = b - A x in FP64 (x in T64 = double); fused ||y||^2, ||b||^2 -> sc->rnorm2, sc->bnorm2
template <typename TM>
cudaError_t residual_fp64(const BsrOp<TM>& A, const double* b, const double* x, double* r, const ReduceScratch& rs,
                          cudaStream_t s);
int krylov_max_blocks(int K, int N);

// elementwise helpers
cudaError_t launch_copy_d2f(const double* a, float* b, size_t n, cudaStream_t s);
cudaError_t launch_copy_f2d(const float* a, double* b, size_t n, cudaStream_t s);
cudaError_t launch_axpy_f2d(const float* e, double* x, size_t n, cudaStream_t s);  // x += e

}  // namespace ho2d
