// adjoint_launch.hpp -- launchers of the discrete-adjoint kernels (adjoint.cu).
#pragma once

#include <cuda_runtime.h>

#include "adjoint_chain.cuh"
#include "fr_launch.hpp"

namespace ho2d {

// ---- stage adjoint (one launch per body; the launches run in this order)
template <typename T>
cudaError_t launch_residual_adjoint(int K, const FrGeom<T>& g, const DevBases<T>& b, const StageAdjArgs<T>& a,
                                    cudaStream_t s);
template <typename T>
cudaError_t launch_velocity_adjoint(int K, const FrGeom<T>& g, const DevBases<T>& b, const StageAdjArgs<T>& a,
                                    cudaStream_t s);
// out = dir + transposed traces of the incoming slots sv (values) and sg (normal
// derivatives); skipped when sc says so (sc may be null: never skipped)
template <typename T>
cudaError_t launch_gather(int K, int N, const DevBases<T>& b, const T* dir, const T* sv, const T* sg, T* out,
                          const KrylovScalars* sc, int mode, cudaStream_t s);

// ---- transposed Poisson operator: y = A^T x in two launches (own part + neighbour
// slots, then the gather); dir, sv, sg are scratch ([N][K][K], [N][4K], [N][4K]; the
// boundary entries of sv, sg must be zero and stay so)
template <typename T>
cudaError_t poisson_transpose(int K, const FrGeom<T>& g, const DevBases<T>& b, const T* x, T* y, T* dir, T* sv, T* sg,
                              const KrylovScalars* sc, int mode, cudaStream_t s);

// ---- BiCGSTAB on A^T mu = b, right-preconditioned with the transpose-problem's
// two-level preconditioner: z = e + omega D^-T (f - A^T e), e = P cycle(P^T f), the cycle
// built from (P^T A P)^T on the host.
template <typename T>
struct TVectors {
    T *x, *r, *rhat, *p, *v, *s, *t, *ph, *sh;
    const T* b;
    T *dir, *sv, *sg;  // scratch of the operator
    T* f0;             // element sums (N entries, zero-padded to a multiple of 4)
};

template <typename T>
struct TPrecond {
    Precond<T> pc;        // coarse hierarchy of the transposed P0 problem (nlev 0: block-Jacobi only)
    const T* dinv;        // inverse diagonal blocks of A, [N][K2][K2] stored [rs][ij]: read transposed
    const T* rowsumT;     // [N][5][K2]: column sums of the 5 blocks of A^T's element row
    const int* bcol;      // [N][5]
};

struct TReduce {
    double* partials;   // [2 * kt_grid()]
    unsigned* counter;  // one word, zero between launches
    KrylovScalars* sc;
};
int kt_grid();

// x = 0, r = rhat = p = b; ||b||^2; done if b == 0
template <typename T>
cudaError_t kt_init(size_t n, const TVectors<T>& v, const TReduce& r, cudaStream_t s);
// one iteration; every kernel returns at once when the solve is done
template <typename T>
cudaError_t kt_iteration(int K, const FrGeom<T>& g, const DevBases<T>& b, const TVectors<T>& v, const TPrecond<T>& pc,
                         const TReduce& r, int max_iter, cudaStream_t s);
template <typename T>
int kt_launches_per_iteration(const TPrecond<T>& pc);
// a whole solve (init + device-side while loop of iterations) as a CUDA graph
template <typename T>
cudaError_t kt_capture_solve(int K, const FrGeom<T>& g, const DevBases<T>& b, const TVectors<T>& v,
                             const TPrecond<T>& pc, const TReduce& r, int max_iter, cudaStream_t s,
                             cudaGraph_t* graph_out);
// r = b - y with ||r||^2 -> sc->rnorm2 and ||b||^2 -> sc->bnorm2
template <typename T>
cudaError_t kt_residual(size_t n, const T* b, const T* y, T* r, const TReduce& rr, cudaStream_t s);

// ---- vector helpers (FP64)
// out = a x + c y (out may alias x or y)
cudaError_t launch_axpby(size_t n, double* out, double a, const double* x, double c, const double* y, cudaStream_t s);
// y = x (FP32 -> FP64)
cudaError_t launch_copy_f2d(const float* x, double* y, size_t n, cudaStream_t s);
// out = x - J .* mu
cudaError_t launch_sub_scaled(size_t n, double* out, const double* x, const double* J, const double* mu,
                              cudaStream_t s);

}  // namespace ho2d
