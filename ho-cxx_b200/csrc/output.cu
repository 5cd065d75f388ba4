// output.cu -- the reference's VTK output (src/HO_2D.cpp:3369-3692) of the device fields:
// the smooth file's node averages and sample values are made on the device
// (output_device.cu), the solution-point fields and those are copied to the host and
// written by write_vtk_files (output_host.cpp), on the caller's thread for trigger_write
// and on VtkQueue's thread for the time loop's dumps.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "host.hpp"
#include "solver_state.hpp"

namespace ho2d {

namespace {

template <typename T>
cudaError_t fetch(std::vector<double>& out, const DeviceBuffer& b, size_t n) {
    std::vector<T> tmp(n);
    cudaError_t e = cudaMemcpy(tmp.data(), b.get(), n * sizeof(T), cudaMemcpyDeviceToHost);
    out.assign(tmp.begin(), tmp.end());
    return e;
}

}  // namespace

// Host copies of the fields the VTK files are written from.
Error Solver::vtk_job(int indx, int subidx, const std::string& dir, VtkQueue::Job& j) {
    DeviceState& d = *d_;
    HO2D_CUDA(cudaStreamSynchronize(d.stream), "sync");
    const int K = in_.knod;
    const size_t nv = (size_t)mesh_.n_el * K * K;
    // the smooth file's node values are made on the device unless HO2D_HOST_OUTPUT=1; then
    // only the vorticity file's fields come back
    const char* ho = std::getenv("HO2D_HOST_OUTPUT");
    const bool on_device = !(ho && std::string(ho) == "1");
    if (on_device) HO2D_TRY(vtk_nodes_device(j));
    HO2D_CUDA(fetch<double>(j.w, d.omega, nv), "copy");
    if (!on_device) HO2D_CUDA(fetch<double>(j.psi, d.psi64, nv), "copy");
    if (stage32_) {
        HO2D_CUDA(fetch<float>(j.u, d.u, nv), "copy");
        HO2D_CUDA(fetch<float>(j.v, d.v, nv), "copy");
        HO2D_CUDA(fetch<float>(j.rhs_diff, d.rhs_diff, nv), "copy");
        HO2D_CUDA(fetch<float>(j.rhs_adv, d.rhs_adv, nv), "copy");
    } else {
        HO2D_CUDA(fetch<double>(j.u, d.u, nv), "copy");
        HO2D_CUDA(fetch<double>(j.v, d.v, nv), "copy");
        HO2D_CUDA(fetch<double>(j.rhs_diff, d.rhs_diff, nv), "copy");
        HO2D_CUDA(fetch<double>(j.rhs_adv, d.rhs_adv, nv), "copy");
    }
    const size_t nb = (size_t)mesh_.n_eb * K;
    if (!on_device) {
        HO2D_CUDA(fetch<double>(j.bc_w, d.bc_w, nb), "copy");
        HO2D_CUDA(fetch<double>(j.bc_nv, d.bc_nv, nb), "copy");
        HO2D_CUDA(fetch<double>(j.bc_pv, d.bc_pv, nb), "copy");
    }
    j.problem_type = in_.problem_type;
    j.indx = indx;
    j.subidx = subidx;
    j.dir = dir;
    return {0, ""};
}

// trigger_write: the files are complete on return (after any dump still being written)
Error Solver::write_vtk(int indx, int subidx, const std::string& dir) {
    const NvtxRange nvtx_range("ho2d.write_vtk");
    if (!setup_done_) return {1, "not set up"};
    HO2D_TRY(vtk_queue_.wait());
    VtkQueue::Job j;
    HO2D_TRY(vtk_job(indx, subidx, dir, j));
    return write_vtk_files(mesh_, B_, in_.problem_type, j.fields(), indx, subidx, dir, &samples_);
}

// a dump of the time loop: written on the queue's thread while the loop goes on
Error Solver::queue_vtk(int indx, const std::string& dir) {
    const NvtxRange nvtx_range("ho2d.queue_vtk");
    VtkQueue::Job j;
    HO2D_TRY(vtk_job(indx, -1, dir, j));
    return vtk_queue_.submit(mesh_, B_, &samples_, std::move(j));
}

}  // namespace ho2d
