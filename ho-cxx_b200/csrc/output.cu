// output.cu -- the reference's VTK output (src/HO_2D.cpp:3369-3692) of the device fields:
// the fields are copied to the host and written by write_vtk_files (output_host.cpp).
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

Error Solver::write_vtk(int indx, int subidx, const std::string& dir) {
    if (!setup_done_) return {1, "not set up"};
    DeviceState& d = *d_;
    HO2D_CUDA(cudaStreamSynchronize(d.stream), "sync");
    const int K = in_.knod;
    const size_t nv = (size_t)mesh_.n_el * K * K;
    std::vector<double> w, psi, u, v, rd, ra, bw, bnv, bpv;
    HO2D_CUDA(fetch<double>(w, d.omega, nv), "copy");
    HO2D_CUDA(fetch<double>(psi, d.psi64, nv), "copy");
    if (stage32_) {
        HO2D_CUDA(fetch<float>(u, d.u, nv), "copy");
        HO2D_CUDA(fetch<float>(v, d.v, nv), "copy");
        HO2D_CUDA(fetch<float>(rd, d.rhs_diff, nv), "copy");
        HO2D_CUDA(fetch<float>(ra, d.rhs_adv, nv), "copy");
    } else {
        HO2D_CUDA(fetch<double>(u, d.u, nv), "copy");
        HO2D_CUDA(fetch<double>(v, d.v, nv), "copy");
        HO2D_CUDA(fetch<double>(rd, d.rhs_diff, nv), "copy");
        HO2D_CUDA(fetch<double>(ra, d.rhs_adv, nv), "copy");
    }
    const size_t nb = (size_t)mesh_.n_eb * K;
    HO2D_CUDA(fetch<double>(bw, d.bc_w, nb), "copy");
    HO2D_CUDA(fetch<double>(bnv, d.bc_nv, nb), "copy");
    HO2D_CUDA(fetch<double>(bpv, d.bc_pv, nb), "copy");
    VtkFields fl{w.data(), psi.data(), u.data(), v.data(), rd.data(), ra.data(), bw.data(), bnv.data(), bpv.data()};
    return write_vtk_files(mesh_, B_, in_.problem_type, fl, indx, subidx, dir, &samples_);
}

}  // namespace ho2d
