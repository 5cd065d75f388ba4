// output.cu -- the reference's VTK output (src/HO_2D.cpp:3369-3692) of the device fields:
// the fields are copied to the host and written by write_vtk_files (output_host.cpp), on
// the caller's thread for trigger_write and on VtkQueue's thread for the time loop's dumps.
#include <cmath>
#include <cstdio>
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
    HO2D_CUDA(fetch<double>(j.w, d.omega, nv), "copy");
    HO2D_CUDA(fetch<double>(j.psi, d.psi64, nv), "copy");
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
    HO2D_CUDA(fetch<double>(j.bc_w, d.bc_w, nb), "copy");
    HO2D_CUDA(fetch<double>(j.bc_nv, d.bc_nv, nb), "copy");
    HO2D_CUDA(fetch<double>(j.bc_pv, d.bc_pv, nb), "copy");
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
    VtkFields fl{j.w.data(),       j.psi.data(),  j.u.data(),     j.v.data(),    j.rhs_diff.data(),
                 j.rhs_adv.data(), j.bc_w.data(), j.bc_nv.data(), j.bc_pv.data()};
    return write_vtk_files(mesh_, B_, in_.problem_type, fl, indx, subidx, dir, &samples_);
}

// a dump of the time loop: written on the queue's thread while the loop goes on
Error Solver::queue_vtk(int indx, const std::string& dir) {
    const NvtxRange nvtx_range("ho2d.queue_vtk");
    VtkQueue::Job j;
    HO2D_TRY(vtk_job(indx, -1, dir, j));
    return vtk_queue_.submit(mesh_, B_, &samples_, std::move(j));
}

}  // namespace ho2d
