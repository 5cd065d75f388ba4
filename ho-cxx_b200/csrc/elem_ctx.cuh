// elem_ctx.cuh -- the two pieces that let an element body be written once for the GPU
// (the K^2 threads of an element share each loop, tid = ij, nt = K^2, sync = __syncthreads)
// and for a host build (one thread per element, tid = 0, nt = 1, sync = nothing) that checks
// it without a GPU.
#pragma once

#if defined(__CUDACC__)
#define HO2D_HD __host__ __device__ __forceinline__
#else
#define HO2D_HD inline
#endif

namespace ho2d {

// Threads of one element and their barrier.
template <int NT>
struct ElemCtx {
    int tid;
    static constexpr int nt = NT;
    HO2D_HD void sync() const {
#if defined(__CUDA_ARCH__)
        __syncthreads();
#endif
    }
};

}  // namespace ho2d
