// fr_device.cuh -- small device routines shared by the FR kernels: staging of the 1-D
// basis tables, the boundary flux-point index and side tables, and face traces of an
// element block held in shared memory by the K^2-thread kernels (trace_kernel, the
// adjoint's element bodies).
#pragma once

#include "device.cuh"

namespace ho2d {

// Copies the 1-D basis tables from the kernel-parameter bank into shared memory: the
// FR loops index them per thread, which would serialise constant-cache reads. The
// caller synchronises before use.
template <typename T>
__device__ __forceinline__ void stage_bases(DevBases<T>& dst, const DevBases<T>& src) {
    constexpr int NW = (int)(sizeof(DevBases<T>) / sizeof(T));
    const T* s = reinterpret_cast<const T*>(&src);
    T* d = reinterpret_cast<T*>(&dst);
    for (int t = threadIdx.x; t < NW; t += blockDim.x) d[t] = s[t];
}

template <int K>
__device__ __forceinline__ int bf_index(int side, int k) {
    return (side / 2) * (K - 2 * k - 1) + k;
}

__device__ __forceinline__ int side_of_ijp(int ijp) {
    // ijp 0 W, 1 E, 2 S, 3 N -> element side (S=0, E=1, N=2, W=3)
    return ijp == 0 ? 3 : (ijp == 1 ? 1 : (ijp == 2 ? 0 : 2));
}

// Face values (basis at -1/+1) and normal derivatives of a K x K block in shared memory.
template <int K, typename T>
__device__ __forceinline__ void face_trace(const T* f, const DevBases<T>& b, int o, T& val, T& der) {
    const int ijp = o / K, k = o % K;
    const int lr = ijp & 1;
    T v = T(0), g = T(0);
    if (ijp < 2) {
#pragma unroll
        for (int m = 0; m < K; ++m) {
            v += f[k * K + m] * b.sbb[m * 2 + lr];
            g += f[k * K + m] * b.sbgb[m * 2 + lr];
        }
    } else {
#pragma unroll
        for (int m = 0; m < K; ++m) {
            v += f[m * K + k] * b.sbb[m * 2 + lr];
            g += f[m * K + k] * b.sbgb[m * 2 + lr];
        }
    }
    val = v;
    der = g;
}

template <int K, typename T>
__device__ __forceinline__ T face_value(const T* f, const DevBases<T>& b, int o) {
    const int ijp = o / K, k = o % K;
    const int lr = ijp & 1;
    T v = T(0);
    if (ijp < 2) {
#pragma unroll
        for (int m = 0; m < K; ++m) v += f[k * K + m] * b.sbb[m * 2 + lr];
    } else {
#pragma unroll
        for (int m = 0; m < K; ++m) v += f[m * K + k] * b.sbb[m * 2 + lr];
    }
    return v;
}

}  // namespace ho2d
