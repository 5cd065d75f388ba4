// forces.cu -- FP64 force on a no-slip body (drag and lift), no counterpart in the reference.
//
// In the vorticity formulation the wall traction follows from the wall vorticity and its
// normal flux (Koumoutsakos & Leonard, JFM 1995): along a stationary no-slip wall the
// momentum equation gives dp/ds = nu d(omega)/dn, with n the normal pointing from the body
// into the fluid and s running along t = z x n, and the viscous traction is nu omega t.
// Integrating the pressure force by parts around the closed body removes the pressure
// itself:
//   F = nu * closed-integral of ( y d(omega)/dn + omega t_x,  -x d(omega)/dn + omega t_y ) ds.
// Every factor but the two boundary arrays is static, so setup folds position, tangent,
// Gauss weight, face length and the orientation of the stored normal derivative into four
// coefficients per boundary point (Solver::setup_forces); this kernel only forms the
// weighted sum, in one CTA and a fixed order (bitwise reproducible).
#include "device.cuh"
#include "fr_launch.hpp"

namespace ho2d {

namespace {

constexpr int kForceThreads = 256;

// out[0..1] = sum_p (cdx_p, cdy_p) dwdn[idx_p] + (cwx_p, cwy_p) wall[idx_p]
__global__ void __launch_bounds__(kForceThreads) k_body_force(int npts, const double* __restrict__ coef,
                                                              const int* __restrict__ idx,
                                                              const double* __restrict__ dwdn,
                                                              const double* __restrict__ wall, double* out) {
    __shared__ double red[2][kForceThreads];
    double fx = 0.0, fy = 0.0;
    for (int p = threadIdx.x; p < npts; p += kForceThreads) {
        const double dn = dwdn[idx[p]], w = wall[idx[p]];
        fx += coef[4 * p + 0] * dn + coef[4 * p + 2] * w;
        fy += coef[4 * p + 1] * dn + coef[4 * p + 3] * w;
    }
    red[0][threadIdx.x] = fx;
    red[1][threadIdx.x] = fy;
    __syncthreads();
    for (int h = kForceThreads / 2; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h) {
            red[0][threadIdx.x] += red[0][threadIdx.x + h];
            red[1][threadIdx.x] += red[1][threadIdx.x + h];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[0] = red[0][0];
        out[1] = red[1][0];
    }
}

}  // namespace

cudaError_t launch_body_force(int npts, const double* coef, const int* idx, const double* dwdn, const double* wall,
                              double* out, cudaStream_t s) {
    k_body_force<<<1, kForceThreads, 0, s>>>(npts, coef, idx, dwdn, wall, out);
    return cudaGetLastError();
}

}  // namespace ho2d
