// noalloc.cu -- fixed scratch for the allocation-free Poisson operator entry point.
//
// ho2d_apply_poisson_noalloc applies the device Poisson operator to caller-owned device
// buffers without allocating anything. The one piece of working memory it needs -- the
// face traces (value and normal derivative at every face point) of the operand -- lives
// in the file-scope array below instead of a cudaMalloc'd buffer. Every GPU that loads
// the library holds this array until the process exits.
//
// The array's host-side name is only a stand-in for the symbol, not a device address, so
// its device address is looked up with cudaGetSymbolAddress once per device, with that
// device current; Solver::setup does this for the handle's device.
#include <mutex>

#include "noalloc.hpp"

namespace ho2d {

namespace {

// 2 trace arrays of N_el * 4 * Knod doubles each
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles];

constexpr int kMaxDevices = 64;
double* g_scratch_ptr[kMaxDevices] = {nullptr};
std::mutex g_scratch_mutex;

}  // namespace

Error noalloc_scratch(int device, double** ptr) {
    if (device < 0 || device >= kMaxDevices) return {1, "device index out of range for the fixed scratch table"};
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_ptr[device]) {
        int current = -1;
        cudaError_t e = cudaGetDevice(&current);
        if (e != cudaSuccess) return {5, std::string("cudaGetDevice: ") + cudaGetErrorString(e)};
        if (current != device) return {1, "noalloc scratch set-up must run with its device current"};
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return {5, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e)};
        g_scratch_ptr[device] = static_cast<double*>(p);
    }
    *ptr = g_scratch_ptr[device];
    return {0, ""};
}

}  // namespace ho2d
