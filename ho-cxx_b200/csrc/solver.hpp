// solver.hpp -- one solver instance: host setup tables plus everything resident on the GPU.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "host.hpp"

namespace ho2d {

// Owning device allocation.
class DeviceBuffer {
  public:
    DeviceBuffer() = default;
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    ~DeviceBuffer() { reset(); }
    cudaError_t alloc(size_t bytes);
    void reset();
    void* get() const { return p_; }
    size_t bytes() const { return n_; }
    template <typename T>
    T* as() const { return static_cast<T*>(p_); }

  private:
    void* p_ = nullptr;
    size_t n_ = 0;
};

struct DeviceState;   // solver_state.hpp
struct AdjointState;  // solver_state.hpp
struct LevelBufs;     // solver_state.hpp
struct CoarseHierarchy;
template <typename T>
struct Precond;

class Solver {
  public:
    Solver();
    ~Solver();

    Error read_input(const std::string& path);
    Error setup();
    Error step(int nsteps);
    Error stage(double coeff);
    Error solve();
    Error solveto(double outerdt, int numstep, int integtype, double reyn);
    Error set_precision(int mode);
    Error time_steps(int nsteps, double* total_ms, double* poisson_ms);
    Error profile_spmv(int reps, double* avg_ms, double* bytes);
    Error profile_krylov(int reps, double* ms, double* bytes);  // [5] each
    Error apply_poisson(const double* x, double* y);
    Error apply_poisson_noalloc(const double* dx, double* dy);

    Error get_volume(int which, double* out);  // [N][K][K]
    Error get_velocity(double* out);           // [N][K][K][2]
    Error set_vorticity(const double* in);
    Error get_boundary(int which, double* out);
    Error set_boundary(int which, const double* in);
    Error get_solution_points(double* out);
    Error get_boundary_points(double* out);  // [N_eb][K][2] in boundary-array order
    // save_vorticity_vtk + save_smooth_vtk of the current fields into dir (output.cu)
    Error write_vtk(int indx, int subidx, const std::string& dir);
    // directory for the VTK files ho2d_solve writes at dump steps ("" = none written)
    void set_output_dir(const std::string& dir) { output_dir_ = dir; }
    // FP64 force (ρ = 1) on the boundary group named "object", from the wall vorticity and
    // its normal flux of the latest stage
    Error get_forces(double* fx, double* fy);

    // ---- hybrid operation (hybrid.cu), the _d entry points of src/HO_2D.hpp:251-290
    void set_defaults();
    void enable_hybrid() { hybrid_ = true; }
    Error set_elemorder(int k);
    Error load_mesh_arrays(int iorder, int nxy, const double* xy, int nidx, const int* idx, int nwall,
                           const int* wall, int nopen, const int* open);
    Error load_inout_arrays(int ninval, const double* velin, int nin, const int* idxin, int noutval,
                            const double* velout, int nout, const int* idxout);
    Error process_mesh_input();
    Error get_solution_areas(double* out);     // [N][K][K] w_j w_k J
    int open_point_count() const;              // 2 * (open edges) * K
    Error get_open_points(double* out);        // [open edges][K][x, y]
    Error set_open_velocities(const double* xyvel);  // [open edges][K][u, v]
    Error set_open_vorticity(const double* w);       // [open edges][K]
    Error set_ptog_weights(const double* w);         // [N][K][K]
    Error get_hoquad_weights(double* out);           // [K][K] 0.25 w_j w_k
    bool hybrid() const { return hybrid_; }
    void release();                                  // clean_up: device memory freed, setup undone

    // ---- discrete adjoint (adjoint_driver.cu)
    // nsteps time steps from the current state, keeping the vorticity every ckpt_every
    // steps for the backward sweep
    Error adjoint_forward(int nsteps, int ckpt_every);
    // gradient of J(omega(T)) with respect to omega at the start of the last
    // adjoint_forward and to BC_parl_vel, from dJ/d(omega(T)); the state at T is kept
    Error adjoint_backward(const double* dJ_dw, double* grad_w0, double* grad_pv);
    // adjoint of one stage (stage(coeff)) at the current state: lam_k -> lam of the stage
    // input vorticity and of BC_parl_vel
    Error stage_adjoint(double coeff, const double* lam_k, double* lam_w, double* lam_pv);
    // y = A^T x with the transposed matrix-free Poisson operator (FP64)
    Error apply_poisson_transpose(const double* x, double* y);
    int adjoint_steps() const;
    // FP32 (true) or FP64 storage of checkpoints and recomputed stage states
    void set_adjoint_storage(bool fp32) { adj_state32_ = fp32; }
    int last_adjoint_iterations() const { return last_adj_iters_; }
    double last_adjoint_residual() const { return last_adj_res_; }

    bool is_setup() const { return setup_done_; }
    const Input& input() const { return in_; }
    int n_el() const { return mesh_.n_el; }
    int knod() const { return in_.knod; }
    int n_eb() const { return mesh_.n_eb; }
    int lnod() const { return mesh_.lnod; }
    double time() const { return time_; }
    void set_time(double t) {
        time_ = t;
        hist_count_ = 0;
    }
    double dt() const { return in_.dt; }
    int precision() const { return krylov32_ ? (stage32_ ? 1 : 2) : 0; }
    // smoother of the FP32 preconditioner: 0 exact inverse blocks in FP32, 1 the same blocks
    // in BF16, 2 Kronecker-sum factors with exact blocks where the fit is poor; -1 = from the
    // environment (HO2D_SMOOTHER_KRON=1, HO2D_SMOOTHER_BF16=1). Takes effect at setup.
    Error set_smoother(int kind);
    // where the Poisson operator is assembled and its diagonal blocks inverted: on the
    // device (true, the default) or on the host (false, or HO2D_HOST_SETUP=1); both give the
    // same bits. Takes effect at setup.
    void set_device_setup(bool on) { device_setup_req_ = on ? 1 : 0; }
    bool device_setup() const { return device_setup_; }
    // one assembled array (ho2d_get_poisson_setup's which), len values into out
    Error get_poisson_setup(int which, int64_t len, double* out);
    int smoother() const { return smoother_kind_; }
    int smoother_exact_blocks() const { return smoother_exact_; }
    int last_poisson_iterations() const { return last_iters_; }
    double last_poisson_residual() const { return last_res_; }
    int64_t launches() const { return launches_; }
    // cumulative since setup: Poisson solves, inner Krylov iterations, refinement sweeps
    void counters(int64_t* solves, int64_t* iters, int64_t* sweeps) const {
        if (solves) *solves = n_solves_;
        if (iters) *iters = iters_total_;
        if (sweeps) *sweeps = sweeps_total_;
    }
    int64_t fp64_finishes() const { return fp64_finishes_; }
    void set_poisson_tolerance(double tol, int max_iter) {
        tol_ = tol;
        max_iter_ = max_iter;
    }

  private:
    Error stage_impl(double coeff, int rk_stage, bool update);
    Error poisson_solve();
    Error vtk_job(int indx, int subidx, const std::string& dir, VtkQueue::Job& j);  // output.cu
    Error queue_vtk(int indx, const std::string& dir);
    Error vtk_device_tables();                  // output_device.cu
    Error vtk_nodes_device(VtkQueue::Job& j);   // node averages and sample values on the device
    template <typename T>
    Error stage_t(double coeff, int rk_stage, bool update, bool solve = true);
    template <typename T>
    Error velocity_only_t();
    template <typename T>
    Error update_bcs(double t, bool into_stage);
    Error setup_from_mesh();
    Error assemble_device(bool kron_fit);  // setup_device.cu
    Error ensure_host_colsum();  // block column sums on the host (the adjoint's coarse problem)
    Error hybrid_upload();
    Error upload_precision_arrays();
    Error setup_preconditioner();
    Error build_poisson_geometry(const std::vector<int>& fnb, const std::vector<int>& fnijp);
    Error setup_forces();
    Error upload_hierarchy(const CoarseHierarchy& H, double omega, std::vector<std::unique_ptr<LevelBufs>>& lev,
                           DeviceBuffer& dense64, DeviceBuffer& dense32, Precond<double>& pc64, Precond<float>& pc32,
                           std::vector<int>* sizes);
    Error adjoint_prepare();
    Error stage_adjoint_dev(double coeff, double* out);
    Error transposed_solve(const double* rhs, double* mu);
    Error store_state(void* dst, const double* src);
    Error load_state(double* dst, const void* src);
    bool adj_state32_ = false;
    template <typename T>
    Error kt_run(T* x, const T* b, bool f32, double tol, int& iters);
    int force_points_ = 0;  // boundary points of the "object" group (0: none)
    Error cuda(cudaError_t e, const char* what);

    Input in_;
    Mesh mesh_;
    Bases B_;
    Metrics M_;
    BoundaryConditions bc_;
    PoissonOperator op_;
    bool input_done_ = false, setup_done_ = false;
    bool stage32_ = false;   // FR stage kernels in FP32 (HO2D_MIXED)
    bool krylov32_ = false;  // FP32 BiCGSTAB inside FP64 refinement (HO2D_MIXED, HO2D_MIXED_KRYLOV)
    double time_ = 0.0;
    // outer time step of solveto_d (src/HO_2D.cpp:4208-4210): hybrid BCs interpolate in it
    double t_start_ = 0.0, t_end_ = 0.0;
    bool hybrid_ = false;                     // enable_hybrid: set_vort feeds the blend target
    std::string output_dir_;                  // where solve() writes its VTK files (empty: none)
    SamplePoints samples_;                    // the input's sample points (VTK output)
    VtkQueue vtk_queue_;                      // dumps being written (declared after what it reads)
    KronSmoother kron_;                       // Kronecker-sum smoother data (smoother kind 2)
    int smoother_req_ = -1;                   // requested smoother kind (-1: environment)
    int smoother_kind_ = 0;                   // kind in use since the last setup
    int smoother_exact_ = 0;                  // kind 2: elements that keep their exact block
    int device_setup_req_ = -1;               // requested setup place (-1: environment)
    bool device_setup_ = true;                // Poisson assembly on the device since the last setup
    bool kron_on_device_ = false;             // the Kronecker-sum factors were fitted on the device
    // initial guess of each stage's Poisson solve: 0/1 = the last psi; 2, 3 = the same RK
    // stage of the last 2 or 3 steps extrapolated in time (HO2D_PSI_EXTRAP)
    int psi_extrap_ = 3;
    int hist_count_ = 0, hist_step_ = 0, hist_ns_ = 0;
    double hist_dt_ = 0.0;
    std::vector<double> open_normal_;         // [N_eb][K][2] unit outward normal on open edges
    std::vector<double> h_open_[6];           // host copies of the open-boundary data (start/end)
    double tol_ = 1e-12;
    int max_iter_ = 500;
    int last_iters_ = 0, prev_iters_ = 8;
    double last_res_ = 0.0;
    int64_t launches_ = 0;
    long n_solves_ = 0;
    int64_t iters_total_ = 0, sweeps_total_ = 0;
    int64_t fp64_finishes_ = 0;  // mixed solves whose refinement stalled and the FP64 solve finished
    int coarse_levels_ = 0;
    std::vector<int> coarse_sizes_;
    double inner_tol_ = 1e-4;        // FP32 inner solve: relative reduction per refinement sweep
    int max_sweeps_ = 30;            // refinement sweep cap (HO2D_MAX_SWEEPS)
    bool verbose_ = false;           // HO2D_VERBOSE=1: coarse levels and one line per Poisson solve on stderr
    bool use_graphs_ = true;         // HO2D_GRAPHS=0: host-driven Krylov loop instead of a CUDA graph
    bool timing_ = false;
    double poisson_ms_acc_ = 0.0;
    std::unique_ptr<DeviceState> d_;
    std::unique_ptr<AdjointState> adj_;
    int last_adj_iters_ = 0, adj_prev_iters_ = 8;
    double last_adj_res_ = 0.0;
};

}  // namespace ho2d
