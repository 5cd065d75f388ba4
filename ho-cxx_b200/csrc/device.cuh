// device.cuh -- device-side data structures shared by the FR and Krylov kernels.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace ho2d {

constexpr int kDirichlet = 0, kNeumann = 1;

// Per-element stride, in values of elem_bytes bytes, of the preconditioner's element data
// (the K^4 inverse blocks, the Kronecker-sum factors): n rounded up to a whole number of
// 16-byte pieces, so that every element's data starts on a 16-byte boundary.
__host__ __device__ constexpr int padded_count(int n, int elem_bytes) {
    return (n * elem_bytes + 15) / 16 * 16 / elem_bytes;
}

// Threads: K^2 per element (one per solution point), EPB elements per CTA.
template <int K>
struct Shape {
    static constexpr int K2 = K * K;
    static constexpr int EPB = (256 / K2) > 32 ? 32 : ((256 / K2) > 0 ? (256 / K2) : 1);
    static constexpr int THREADS = ((EPB * K2 + 31) / 32) * 32;  // whole warps; tail threads idle
    static constexpr int NF = 4 * K;  // face points per element
};

// 1-D bases, passed by value (kernel parameter space); T is the arithmetic type.
template <typename T>
struct DevBases {
    T D[64];     // D[k*K+m] = l_k'(x_m)
    T sbb[16];   // [k*2+lr] l_k(-1), l_k(+1)
    T sbgb[16];  // [k*2+lr] l_k'(-1), l_k'(+1)
    T R[16];     // [k*2+lr] Radau values (left, right)
    T gR[16];    // [k*2+lr] Radau derivatives
    T gp[2];     // g'(-1), g'(+1)
};

// Everything an FR kernel reads. Pointers are device pointers; volume arrays are
// [N][K][K], face arrays [N][4][K] (ijp order), boundary arrays [N_eb][K].
template <typename T>
struct FrGeom {
    int N, n_eb;
    const int* face_nb;     // [N*4] neighbour element (>= 0) or -(edge + 1) on the boundary
    const int* face_nijp;   // [N*4] neighbour's face ijp across this face
    const T* xxi;           // volume metrics
    const T* xeta;
    const T* yxi;
    const T* yeta;
    const T* J;
    const T* fA;            // face metrics g.g (normal), g1.g2, face Jacobian, |g|
    const T* fB;
    const T* fJ;
    const T* fAn;
    const int* be_group;    // [N_eb]
    const int* sw_p;        // [N_eb]
    const int* sw_d;        // [N_eb]
    const int* noslip;      // [n_groups]
    // [N_eb][K][K] inverse of the Neumann common-value system of every boundary edge with a
    // Neumann psi or vorticity condition, rows scaled by 1/J_f (zero elsewhere)
    const T* nminv;
};

// Boundary-edge arrays, always double (they carry the 1/(dt Re^-1) wall flux).
struct BcArrays {
    double* bc_p;
    double* bc_nv;
    double* bc_pv;
    double* bc_d;
    double* bc_w;
    double* vjump;
    double* bc_adv;
};

// Scalars of one Krylov solve, resident on the device.
struct KrylovScalars {
    double rho, rho_old, alpha, omega, beta;
    double bnorm2, rnorm2, snorm2, eps2;
    int it, done, breakdown, s_exit, zero_rhs, pad;
    double tol;  // relative tolerance of the next solve, written by the host before it starts
    // FP64 iterative refinement around the FP32 solve when it runs on the device (one graph
    // per solve): the target on the FP64 residual, the smallest inner reduction asked of a
    // sweep and the sweep cap (written by the host), then the sweeps done, the inner
    // iterations summed over them, the last relative FP64 residual, whether it was finite
    // and whether the right-hand side was zero (written by the device)
    double tol_outer, inner_tol;
    int max_sweeps, sweeps, iters_total, finite, zero_psi;
    int dev_error;  // nonzero: a kernel's bounded wait ran out (the host reports it)
    double res;
    // the refinement stopped because a sweep cut the FP64 residual by less than half (the
    // FP32 solve is no longer accurate enough for this operator; the host finishes in FP64)
    int stalled, pad2;
};

// A preconditioner application is skipped once the solve is done, and the second one of
// an iteration (mode 1) also when the iteration exits early after its s update.
__device__ __forceinline__ bool pc_skip(const KrylovScalars* sc, int mode) {
    return sc->done || (mode == 1 && sc->s_exit);
}

}  // namespace ho2d
