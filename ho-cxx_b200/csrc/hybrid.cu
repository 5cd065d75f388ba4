// hybrid.cu -- the hybrid-operation entry points of the reference's HO_2D
// (src/HO_2D.hpp:251-290, src/HO_2D.cpp:3698-4278): an external Lagrangian (vortex)
// solver loads the mesh from arrays, sets the open-boundary velocity and vorticity and the
// vorticity it wants blended in at the start and end of each outer step, and advances
// with solveto_d. On the device the open-boundary values are interpolated in time and the
// blend is applied at every BC update (update_bcs in solver.cu, kernels in fr_kernels.cu).
#include <cmath>
#include <cstdio>

#include "solver_state.hpp"

namespace ho2d {

// set_defaults (src/HO_2D.cpp:3698-3713)
void Solver::set_defaults() {
    Input in;
    in.knod = 3;
    in.reyn_inv = 1.0;
    in.huynh = 2;
    in.ti_type = 2;
    in.adv_type = 2;
    in.problem_type = 11;
    in.num_steps = 0;
    in.dt = 1.0;
    in.dump_freq = 100;
    in.fast = 0;
    in.lhs_type = 3;
    in_ = in;
    hybrid_ = false;
    input_done_ = true;
    setup_done_ = false;
    t_start_ = t_end_ = 0.0;
}

Error Solver::set_elemorder(int k) {
    if (k < 1 || k > 8) return {4, "element order (Knod) must be 1..8"};
    in_.knod = k;
    return {0, ""};
}

Error Solver::load_mesh_arrays(int iorder, int nxy, const double* xy, int nidx, const int* idx, int nwall,
                               const int* wall, int nopen, const int* open) {
    setup_done_ = false;
    vtk_queue_.wait();  // a dump still being written reads the mesh
    return mesh_from_arrays(iorder, nxy, xy, nidx, idx, nwall, wall, nopen, open, mesh_);
}

// load_inout_arrays_d (src/HO_2D.cpp:3884-3898): inlets, then outlets, each edge with its
// normal velocity
Error Solver::load_inout_arrays(int ninval, const double* velin, int nin, const int* idxin, int noutval,
                                const double* velout, int nout, const int* idxout) {
    if (mesh_.elem_nodes.empty()) return {1, "load the mesh arrays first"};
    vtk_queue_.wait();
    HO2D_TRY(add_boundary_arrays(mesh_, "inlet", nin, idxin, ninval, velin));
    return add_boundary_arrays(mesh_, "outlet", nout, idxout, noutval, velout);
}

// process_mesh_input (src/HO_2D.cpp:3901-3937)
Error Solver::process_mesh_input() {
    if (!input_done_) return {1, "call ho2d_set_defaults (or ho2d_read_input) first"};
    if (mesh_.elem_nodes.empty()) return {1, "load the mesh arrays first"};
    vtk_queue_.wait();  // a dump still being written reads the mesh
    HO2D_TRY(process_mesh(mesh_));
    samples_ = SamplePoints();  // the reference reads no sample points here
    return setup_from_mesh();
}

// Device arrays of a hybrid run (zero until the driver sets them) and the unit outward
// normals of the open edges (open_normals, host_hybrid.cpp).
Error Solver::hybrid_upload() {
    DeviceState& d = *d_;
    const int K = in_.knod, neb = std::max(1, mesh_.n_eb);
    const size_t nv = (size_t)mesh_.n_el * K * K, nb = (size_t)neb * K;
    const std::vector<double> zb(nb, 0.0), zv(nv, 0.0);
    for (auto& b : d.hyb) HO2D_CUDA(upload(b, zb), "alloc hybrid boundary data");
    for (auto& b : d.hvort) HO2D_CUDA(upload(b, zv), "alloc hybrid vorticity");
    std::vector<double> inl(bc_.inlet_nv);
    inl.resize(neb, 0.0);
    HO2D_CUDA(upload(d.hyb_inlet_nv, inl), "upload inlet velocities");
    for (auto& h : h_open_) h.assign(nb, 0.0);
    open_normals(mesh_, B_, M_, bc_, open_normal_);
    open_normal_.resize(nb * 2, 0.0);
    return {0, ""};
}

int Solver::open_point_count() const { return ho2d::open_point_count(mesh_, in_.knod); }

// getopenpts_d (src/HO_2D.cpp:4004-4042)
Error Solver::get_open_points(double* out) {
    if (!setup_done_) return {1, "not set up"};
    open_points(mesh_, B_, out);
    return {0, ""};
}

// setopenvels_d (src/HO_2D.cpp:4047-4122): the end values become the start values; the new
// Cartesian velocities, split into normal (outward) and parallel parts
// (split_open_velocities), become the end values.
Error Solver::set_open_velocities(const double* xyvel) {
    if (!setup_done_ || in_.problem_type != 11) return {1, "not a set-up hybrid run (problem type 11)"};
    DeviceState& d = *d_;
    h_open_[0] = h_open_[1];
    h_open_[2] = h_open_[3];
    split_open_velocities(mesh_, in_.knod, open_normal_, xyvel, h_open_[1].data(), h_open_[3].data());
    for (int a = 0; a < 4; ++a)
        HO2D_CUDA(cudaMemcpy(d.hyb[a].get(), h_open_[a].data(), h_open_[a].size() * 8, cudaMemcpyHostToDevice),
                  "upload open velocities");
    return {0, ""};
}

// setopenvort_d (src/HO_2D.cpp:4125-4145)
Error Solver::set_open_vorticity(const double* w) {
    if (!setup_done_ || in_.problem_type != 11) return {1, "not a set-up hybrid run (problem type 11)"};
    DeviceState& d = *d_;
    const std::vector<int>* oe = open_boundary_edges(mesh_);
    const int K = in_.knod;
    h_open_[4] = h_open_[5];
    if (oe)
        for (size_t i = 0; i < oe->size(); ++i)
            for (int j = 0; j < K; ++j) h_open_[5][(size_t)(*oe)[i] * K + j] = w[i * K + j];
    for (int a = 4; a < 6; ++a)
        HO2D_CUDA(cudaMemcpy(d.hyb[a].get(), h_open_[a].data(), h_open_[a].size() * 8, cudaMemcpyHostToDevice),
                  "upload open vorticity");
    return {0, ""};
}

// setptogweights_d (src/HO_2D.cpp:4174-4187)
Error Solver::set_ptog_weights(const double* w) {
    if (!setup_done_ || !d_->hvort[2].get()) return {1, "not a set-up hybrid run (problem type 11)"};
    const size_t nv = (size_t)mesh_.n_el * in_.knod * in_.knod;
    HO2D_CUDA(cudaStreamSynchronize(d_->stream), "sync");
    HO2D_CUDA(cudaMemcpy(d_->hvort[2].get(), w, nv * 8, cudaMemcpyHostToDevice), "upload weights");
    return {0, ""};
}

// getsolnareas_d (src/HO_2D.cpp:3982-3992)
Error Solver::get_solution_areas(double* out) {
    if (!setup_done_) return {1, "not set up"};
    solution_areas(B_, M_, mesh_.n_el, out);
    return {0, ""};
}

// get_hoquad_weights_d (src/HO_2D.cpp:4252-4259)
Error Solver::get_hoquad_weights(double* out) {
    if (!setup_done_) return {1, "not set up"};
    const int K = in_.knod;
    for (int j = 0; j < K; ++j)
        for (int k = 0; k < K; ++k) out[j * K + k] = 0.25 * B_.w[j] * B_.w[k];
    return {0, ""};
}

// clean_up (src/HO_2D.cpp:4275-4278): releases the device state; the handle can be set up again
void Solver::release() {
    vtk_queue_.wait();
    adj_.reset();
    d_.reset(new DeviceState);
    setup_done_ = false;
}

}  // namespace ho2d
