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
// Matrix-free FR Laplacian (the Poisson operator) plus the preconditioner's element data.
template <typename T>
struct MfOp {
    int K;
    FrGeom<T> g;            // metrics, connectivity, Poisson BC switches (g.sw_p)
    DevBases<T> b;
    const double* zero_bc;  // [N_eb * K] zeros: homogeneous boundary values
    const T* dinv;          // [N][K2][K2] inverse diagonal blocks, transposed ([rs][ij])
    const T* rowsum;        // [N][5][K2] row sums of the 5 blocks of each element row
    const int* bcol;        // [N][5] element of each block (slot 0 = self, 1 + ijp = neighbours)
};

template <typename T>
struct BicgVectors {
    T *x, *r, *rhat, *p, *v, *s, *t, *ph, *sh;
    const T* b;
    T *tv, *tg;    // face traces of the operand of the next operator application (ph or sh)
    T *xtv, *xtg;  // face traces of x (initial residual)
};

struct ReduceScratch {
    double* partials;    // [4 * max_blocks]
    unsigned* counter;   // 1 word, zero between launches
    KrylovScalars* sc;   // device scalars
};

// scalar CSR matrix on the device
template <typename T>
struct DevCsr {
    int n;
    const int* ptr;
    const int* col;
    const T* val;
};

// one coarse level of the two-level preconditioner (level 0 = one value per element)
template <typename T>
struct CoarseLevel {
    int n;
    DevCsr<T> A, P, R;  // P, R unused on the coarsest level
    const T* m;         // SPAI-0 weights
    T *f, *u, *t, *u2;  // right-hand side, iterate, residual, smoothed iterate
    T* out;             // where this level's cycle leaves its result (u2, or u when coarsest)
};

constexpr int kMaxLevels = 24;

// preconditioner: nlev == 0 -> block-Jacobi; otherwise the two-level V(0,1) cycle
template <typename T>
struct Precond {
    int nlev = 0;
    double omega = 1.0;  // weight of the block-Jacobi smoothing step
    CoarseLevel<T> lev[kMaxLevels];
    const T* dense_inv = nullptr;  // inverse of the coarsest operator
};

template <typename T>
cudaError_t krylov_init(const MfOp<T>& op, const BicgVectors<T>& v, const ReduceScratch& rs, double tol,
                        cudaStream_t s);
template <typename T>
cudaError_t krylov_iteration(const MfOp<T>& op, const BicgVectors<T>& v, const ReduceScratch& rs, int max_iter,
                             const Precond<T>& pc, cudaStream_t s);
template <typename T>
int krylov_launches_per_iteration(const Precond<T>& pc);
// a whole solve (initial residual + device-side while loop of iterations) as a CUDA graph
template <typename T>
cudaError_t krylov_capture_solve(const MfOp<T>& op, const BicgVectors<T>& v, const ReduceScratch& rs, double tol,
                                 int max_iter, const Precond<T>& pc, cudaStream_t s, cudaGraph_t* graph_out);
// r = b - A x with ||r||^2 -> sc->rnorm2, ||b||^2 -> sc->bnorm2 (traces of x into xtv/xtg)
template <typename T>
cudaError_t mf_residual(const MfOp<T>& op, const double* b, const T* x, T* xtv, T* xtg, double* r,
                        const ReduceScratch& rs, cudaStream_t s);
// y = A x (traces of x into xtv/xtg first)
template <typename T>
cudaError_t mf_apply_op(const MfOp<T>& op, const T* x, T* xtv, T* xtg, T* y, cudaStream_t s);
// `reps` launches of the operator kernel alone on x whose traces are already in xtv/xtg
template <typename T>
cudaError_t mf_apply_only(const MfOp<T>& op, const T* x, const T* xtv, const T* xtg, T* y, int reps, cudaStream_t s);
int krylov_max_blocks(int K, int N);

// elementwise helpers
cudaError_t launch_copy_d2f(const double* a, float* b, size_t n, cudaStream_t s);
cudaError_t launch_axpy_f2d(const float* e, double* x, size_t n, cudaStream_t s);  // x += e

}  // namespace ho2d
