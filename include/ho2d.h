/*
 * ho2d.h -- C ABI of the B200-native HO-CXX vorticity-streamfunction FR solver.
 *
 * One opaque handle drives one mesh, like one instance of the reference's HO_2D class
 * (src/HO_2D.hpp:69-291). Every entry point returns an int status (0 = success, as the
 * reference's char/int returns at src/main.cpp:49-59); no C++ exception crosses this
 * boundary. Buffers are caller-owned (int32 length, double* data) pairs in the
 * reference's ordering: volume fields [el][j][i] with el in .msh file order, boundary
 * arrays [edge][k] in boundary-edge order (src/HO_2D.cpp:4148-4250 use the same pairs).
 * Calls are synchronous at return and not thread-safe on one handle. Every handle owns
 * one CUDA stream on the device that is current when ho2d_setup runs.
 */
#ifndef HO2D_H
#define HO2D_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ho2d_solver ho2d_solver;

enum ho2d_status {
    HO2D_OK = 0,
    HO2D_ERR_ARG = 1,            /* null handle/buffer, wrong length, call out of order */
    HO2D_ERR_IO = 2,             /* input.dat or .msh cannot be opened (reference: exit(1)) */
    HO2D_ERR_MESH = 3,           /* malformed mesh, unsupported element type (reference: returns 2/3) */
    HO2D_ERR_UNSUPPORTED = 4,    /* Knod, Lnod, scheme or problem type outside what is implemented */
    HO2D_ERR_CUDA = 5,           /* a CUDA runtime error; ho2d_last_error has the text */
    HO2D_ERR_NOT_CONVERGED = 6,  /* Poisson solve hit its iteration cap above tolerance */
    HO2D_ERR_NONFINITE = 7       /* NaN/Inf detected in the vorticity */
};

enum ho2d_precision {
    HO2D_FP64 = 0,          /* every device array and operation in double precision */
    HO2D_MIXED = 1,         /* FP32 FR residual and Krylov, FP64 refinement residual and RK accumulation */
    HO2D_MIXED_KRYLOV = 2   /* FP64 FR residual; FP32 Krylov inside FP64 refinement of the Poisson solve */
};

/* Smoother of the FP32 Poisson preconditioner (HO2D_MIXED, HO2D_MIXED_KRYLOV). No
 * counterpart in the reference, whose AMGCL relaxation is fixed at compile time
 * (src/HO_2D.hpp:54). The FP64 solve always uses exact FP64 inverse blocks. */
enum ho2d_smoother {
    HO2D_SMOOTHER_BLOCKS = 0,  /* exact inverse of each element's diagonal block, FP32 */
    HO2D_SMOOTHER_BF16 = 1,    /* the same blocks stored in BF16 (half the bytes) */
    HO2D_SMOOTHER_KRON = 2     /* Kronecker-sum fit of each block, inverted by fast
                                  diagonalisation (4K^2+2K values per element); the exact
                                  block where the fit is poor */
};

/* which boundary-edge array [N_eb][Knod] ho2d_get_boundary / ho2d_set_boundary address */
enum ho2d_boundary_array {
    HO2D_BC_POISSON = 0,        /* BC_Poisson: psi or d(psi)/dn */
    HO2D_BC_NORMAL_VEL = 1,     /* BC_normal_vel (local h direction) */
    HO2D_BC_PARL_VEL = 2,       /* BC_parl_vel (counter-clockwise tangential velocity) */
    HO2D_BC_DIFFUSION = 3,      /* BC_diffusion: vorticity or its normal derivative */
    HO2D_BC_VORTICITY = 4,      /* BC_vorticity: common vorticity on the boundary */
    HO2D_BC_VELOCITY_JUMP = 5,  /* velocity_jump: d(psi)/dn on Dirichlet-psi edges */
    HO2D_BC_ADVECTION = 6       /* BC_advection */
};

/* which volume array [N_el][Knod][Knod] ho2d_get_field addresses */
enum ho2d_field {
    HO2D_FIELD_VORTICITY = 0,
    HO2D_FIELD_STREAMFUNCTION = 1,
    HO2D_FIELD_RHS_DIFFUSIVE = 2,  /* Re^-1 Laplacian(omega) of the last stage */
    HO2D_FIELD_RHS_ADVECTIVE = 3,  /* -div(u omega) of the last stage */
    HO2D_FIELD_STAGE_K = 4,        /* k = dt (advective + diffusive) of the last stage */
    HO2D_FIELD_JACOBIAN = 5        /* vol_jac at the solution points */
};

/* Replaces HO_2D::HO_2D() (src/HO_2D.hpp:184-198). */
int ho2d_create(ho2d_solver** handle);
/* Replaces HO_2D::~HO_2D / release_memory (src/HO_2D.cpp:125-211); frees device memory. */
int ho2d_destroy(ho2d_solver* handle);
/* Replaces HO_2D::read_input_file (src/HO_2D.cpp:213-317); the mesh path in the file is
 * resolved relative to the directory of `path`. */
int ho2d_read_input(ho2d_solver* handle, const char* path);
/* Replaces the setup sequence of src/main.cpp:49-75: setup_mesh, allocate_arrays,
 * setup_sps_gps, form_bases, form_metrics, setup_IC_BC_SRC, form_Laplace_operator_matrix
 * (src/HO_2D.cpp:476-1804, 3011-3086). Uploads everything to the current CUDA device. */
int ho2d_setup(ho2d_solver* handle);
/* Replaces HO_2D::solve_vorticity_streamfunction (src/HO_2D.cpp:1390-1463) for
 * num_time_steps steps from the initial vorticity, including the extra Poisson solve and
 * velocity recovery at every dump step; there it writes the reference's two VTK files
 * (ho2d_write_vtk) into the directory set by ho2d_set_output_dir, if one is set. */
int ho2d_solve(ho2d_solver* handle);
/* Directory for the VTK files of ho2d_solve (NULL or "" = write none, the default). */
int ho2d_set_output_dir(ho2d_solver* handle, const char* dir);
/* Replaces save_vorticity_vtk and save_smooth_vtk (src/HO_2D.cpp:3369-3692), and
 * trigger_write (4262-4271): writes vorticity<p>_K<K>[_<subidx>]_<indx>.vtk (solution
 * points) and problem<p>_K<K>[_<subidx>]_<indx>.vtk (node averages) of the current fields
 * into dir (NULL: the working directory); subidx < 0 leaves it out of the names. When the
 * input names a sample-points file (read_process_sample_points, src/HO_2D.cpp:319-474,
 * read at ho2d_setup relative to the input's directory), also
 * sampling_points<p>_K<K>_L<Lnod>_<indx>.dat: x, y, vorticity, u, v per point
 * (src/HO_2D.cpp:3592-3614). */
int ho2d_write_vtk(ho2d_solver* handle, int32_t indx, int32_t subidx, const char* dir);
/* Replaces nsteps calls of HO_2D::solve_advection_diffusion (src/HO_2D.cpp:1465-1531),
 * advancing the solver time by dt after each. */
int ho2d_step(ho2d_solver* handle, int32_t nsteps);
/* Replaces one HO_2D::Euler_time_integrate(vorticity, k, coeff) (src/HO_2D.cpp:1806-1839)
 * on the current vorticity, without advancing time; results via ho2d_get_field. */
int ho2d_stage(ho2d_solver* handle, double coeff);
/* Replaces HO_2D::solveto_d (src/HO_2D.cpp:4194-4233) for the non-hybrid problem types:
 * dt = outerdt / numstep, integrator `integtype`, Re = reyn, numstep steps. `region` only
 * names the reference's optional substep VTK files (src/HO_2D.cpp:4217-4230); no files are
 * written here, so it is accepted and has no effect. */
int ho2d_solveto(ho2d_solver* handle, double outerdt, int32_t numstep, int32_t integtype, double reyn,
                 int32_t region);

/* Sizes after ho2d_setup: elements, Knod, boundary edges, geometry nodes per edge. */
int ho2d_get_sizes(ho2d_solver* handle, int32_t* n_el, int32_t* knod, int32_t* n_edges_boundary,
                   int32_t* lnod);
/* Vorticity in/out (like setsolnvort_d / getallvorts_d, src/HO_2D.cpp:4148-4250);
 * len = N_el*Knod*Knod. ho2d_set_vort also sets the initial vorticity used by ho2d_solve. */
int ho2d_get_vort(ho2d_solver* handle, int32_t len, double* buf);
int ho2d_set_vort(ho2d_solver* handle, int32_t len, const double* buf);
/* Stream function, len = N_el*Knod*Knod. */
int ho2d_get_psi(ho2d_solver* handle, int32_t len, double* buf);
/* Cartesian velocity [el][j][i][u,v] (velocity_cart), len = 2*N_el*Knod*Knod. */
int ho2d_get_vel(ho2d_solver* handle, int32_t len, double* buf);
/* Any volume array of enum ho2d_field, len = N_el*Knod*Knod. */
int ho2d_get_field(ho2d_solver* handle, int32_t which, int32_t len, double* buf);
/* Boundary-edge arrays of enum ho2d_boundary_array, len = N_eb*Knod. Setting
 * HO2D_BC_PARL_VEL replaces a lid/wall velocity profile (the reference's BC_parl_vel). */
int ho2d_get_boundary(ho2d_solver* handle, int32_t which, int32_t len, double* buf);
int ho2d_set_boundary(ho2d_solver* handle, int32_t which, int32_t len, const double* buf);
/* Solution-point coordinates [el][j][i][x,y] (like getsolnpts_d, src/HO_2D.cpp:3946-3980),
 * len = 2*N_el*Knod*Knod. */
int ho2d_get_solution_points(ho2d_solver* handle, int32_t len, double* buf);
/* No counterpart in the reference. Coordinates of the boundary flux points [N_eb][Knod][x,y]
 * in the order of the boundary-edge arrays (ho2d_get_boundary), len = 2*N_eb*Knod: the
 * points where BC_parl_vel and the other boundary arrays live. */
int ho2d_get_boundary_points(ho2d_solver* handle, int32_t len, double* buf);

/* HO2D_FP64 (default), HO2D_MIXED or HO2D_MIXED_KRYLOV; may be called before or after
 * ho2d_setup. */
int ho2d_set_precision(ho2d_solver* handle, int32_t mode);
/* Selects the FP32 preconditioner's smoother (enum ho2d_smoother) for the next
 * ho2d_setup; -1 restores the default (HO2D_SMOOTHER_KRON=1 or HO2D_SMOOTHER_BF16=1 in the
 * environment, else HO2D_SMOOTHER_BLOCKS). No counterpart in the reference. */
int ho2d_set_smoother(ho2d_solver* handle, int32_t kind);
/* The smoother in use since the last ho2d_setup and, for HO2D_SMOOTHER_KRON, how many
 * elements keep their exact inverse block (0 otherwise). */
int ho2d_get_smoother(ho2d_solver* handle, int32_t* kind, int32_t* exact_blocks);
/* Where the next ho2d_setup assembles the Poisson operator (src/HO_2D.cpp:1533-1804),
 * inverts its diagonal blocks and the coarsest level's dense matrix: 1 = on the device
 * (the default), 0 = on the host (also HO2D_HOST_SETUP=1 in the environment). Both give
 * the same bits for the assembled arrays. No counterpart in the reference. */
int ho2d_set_device_setup(ho2d_solver* handle, int32_t on);
/* One array of the assembled Poisson operator after ho2d_setup, as doubles:
 * HO2D_SETUP_DINV   inverse diagonal blocks [N_el][K^2 (rs)][K^2 (ij)] (the inverse's
 *                   transpose, the layout the smoother reads);
 * HO2D_SETUP_ROWSUM sums over rs of each block row [N_el][5][K^2] (slot 0 = the element,
 *                   1..4 = its neighbour across face ijp 0..3, zero for boundary faces);
 * HO2D_SETUP_COLSUM sums over ij of each block column [N_el][5][K^2];
 * HO2D_SETUP_BSUM   each block's entry sum [N_el][5];
 * HO2D_SETUP_BSRC   the boundary source [N_eb][K^2][K] (src/HO_2D.cpp:1640-1714);
 * HO2D_SETUP_BCOL   each slot's column element (-1 = none) [N_el][5].
 * len must equal the array's length. */
enum ho2d_setup_array {
    HO2D_SETUP_DINV = 0,
    HO2D_SETUP_ROWSUM = 1,
    HO2D_SETUP_COLSUM = 2,
    HO2D_SETUP_BSUM = 3,
    HO2D_SETUP_BSRC = 4,
    HO2D_SETUP_BCOL = 5
};
int ho2d_get_poisson_setup(ho2d_solver* handle, int32_t which, int64_t len, double* buf);
/* Poisson solve controls: relative tolerance on ||b - A psi|| / ||b|| (default 1e-12)
 * and iteration cap (default 500). */
int ho2d_set_poisson_tolerance(ho2d_solver* handle, double rel_tol, int32_t max_iter);
/* Statistics of the last Poisson solve: Krylov iterations (inner iterations summed over
 * refinement sweeps) and final relative residual. */
int ho2d_poisson_stats(ho2d_solver* handle, int32_t* iterations, double* rel_residual);
/* No counterpart in the reference. Totals since ho2d_setup: Poisson solves, Krylov
 * iterations (inner iterations of all refinement sweeps in the mixed modes) and FP64
 * refinement sweeps (0 in HO2D_FP64). Any pointer may be NULL. */
int ho2d_solve_counters(ho2d_solver* handle, int64_t* solves, int64_t* iterations, int64_t* sweeps);
/* Mixed-precision Poisson solves since setup whose FP64 refinement stalled (a sweep that did
 * not halve the residual: the FP32 inner solve is not accurate enough for the operator) or
 * hit its sweep cap, and which the FP64 solve then finished from the refined iterate. No
 * counterpart in the reference. */
int ho2d_fp64_finishes(ho2d_solver* handle, int64_t* count);
/* Current solver time and time-step size. */
int ho2d_get_time(ho2d_solver* handle, double* time, double* dt);
/* Sets the current solver time (the reference's time_start / current_time,
 * src/HO_2D.hpp:164), e.g. to restart a run or to start inside the pulsatile inflow
 * cycle of problem types 2 and 3. */
int ho2d_set_time(ho2d_solver* handle, double time);
/* Runs nsteps time steps and reports device time between CUDA events recorded on the
 * handle's stream around each step: total milliseconds and the part spent in Poisson
 * solves. Before each step (outside its events) a 256 MiB device buffer is written, so
 * no step starts with the previous step's data in the 126 MB L2. */
int ho2d_time_steps(ho2d_solver* handle, int32_t nsteps, double* total_ms, double* poisson_ms);
/* Runs the Poisson operator kernel (matrix-free y = A psi, the kernel every operator
 * application of the Krylov solve uses) `reps` times back to back on the current psi, in
 * the active precision, between CUDA events on the handle's stream; returns the average
 * launch duration and the algorithmic bytes one launch must move. */
int ho2d_profile_spmv(ho2d_solver* handle, int32_t reps, double* avg_ms, double* bytes_per_launch);
/* No counterpart in the reference. Device time of the Krylov kernels inside `iterations`
 * BiCGSTAB iterations of the active precision's Poisson solve on the current state (run
 * without a CUDA graph and in order, CUDA events between the launches on the handle's
 * stream; psi is not changed), and their algorithmic bytes per launch. ms[5] and
 * bytes[5]: [0] fine part of the smoothing step, [1] operator kernel, [2] x/r update,
 * [3] one coarse cycle, [4] combination of the smoothing step; per launch averages. */
int ho2d_profile_krylov(ho2d_solver* handle, int32_t iterations, double* ms, double* bytes);
/* y = A x in FP64 with the device's Poisson operator: the matrix the reference assembles
 * in form_Laplace_operator_matrix (src/HO_2D.cpp:1533-1804), applied matrix-free;
 * len = N_el*Knod*Knod. */
int ho2d_apply_poisson(ho2d_solver* handle, int32_t len, const double* x, double* y);
/* No counterpart in the reference. Allocation-free variant of ho2d_apply_poisson for
 * callers that cannot let a library call cudaMalloc: codes that own all device memory
 * through their own pool or a fixed budget, or that must not trigger the implicit device
 * synchronisation an allocation can cause in the middle of their own work. x_device and
 * y_device are caller-owned DEVICE buffers of len = N_el*Knod*Knod doubles on the
 * handle's device, each 16-byte aligned as cudaMalloc returns them (HO2D_ERR_ARG
 * otherwise) (y = A x, FP64, synchronous at return: y_device is complete when the
 * call returns). The call runs on the handle's own non-blocking stream, which is not
 * ordered after the caller's streams or the legacy default stream: whatever wrote
 * x_device must have completed before the call (synchronise the stream or event that
 * wrote it). The
 * only working memory is a fixed 8 MiB array compiled into the library (face traces of
 * x), so meshes with N_el*Knod > 131072 are rejected with HO2D_ERR_ARG. Its device
 * address is looked up once per device inside ho2d_setup; this call itself allocates
 * nothing. Every call on a device shares that array and nothing in it needs clearing
 * (it is fully rewritten from x before it is read), so calls that overlap on the GPU --
 * from different handles or streams on the same device -- race on it. */
int ho2d_apply_poisson_noalloc(ho2d_solver* handle, int32_t len, const double* x_device, double* y_device);
/* No counterpart in the reference. FP64 force per unit depth (density 1) on the boundary
 * group named "object" (problem type 3): fx (drag) and fy (lift) from the wall vorticity and
 * its normal flux of the latest stage, dp/ds = nu d(omega)/dn plus the skin friction
 * nu omega t (Koumoutsakos & Leonard, JFM 1995). Drag and lift coefficients are 2 F / (U^2 D).
 * HO2D_ERR_ARG when the mesh has no "object" group. */
int ho2d_get_forces(ho2d_solver* handle, double* fx, double* fy);
/* ---- Hybrid operation: the entry points an external Lagrangian driver calls
 * (src/HO_2D.hpp:251-290). Sequence: ho2d_set_defaults, ho2d_enable_hybrid,
 * ho2d_set_elemorder, ho2d_load_mesh_arrays, ho2d_load_inout_arrays (optional),
 * ho2d_process_mesh_input; then per outer step ho2d_set_open_velocities,
 * ho2d_set_open_vorticity, ho2d_set_vort (the vorticity to blend in; hybrid mode only),
 * ho2d_set_ptog_weights, ho2d_solveto and ho2d_get_vort. Problem type 11. */
/* Replaces set_defaults (src/HO_2D.cpp:3698-3713): Knod 3, Re^-1 1, RK2, advection type 2,
 * problem type 11, dt 1; takes the place of ho2d_read_input. */
int ho2d_set_defaults(ho2d_solver* handle);
/* Replaces enable_hybrid (3714-3716): ho2d_set_vort then sets the blend target. */
int ho2d_enable_hybrid(ho2d_solver* handle);
/* Replaces set_elemorder (3718-3720): Knod. */
int ho2d_set_elemorder(ho2d_solver* handle, int32_t knod);
/* Replaces load_mesh_arrays_d (3832-3886): geometry order iorder (Lnod - 1); nxy doubles of
 * node coordinates (x, y pairs); nidx element node indices (Lnod^2 per element, Gmsh
 * order, 0-based); nwall / nopen node indices of the "wall" / "open" boundary edges (Lnod
 * per edge, in the element's counter-clockwise orientation). */
int ho2d_load_mesh_arrays(ho2d_solver* handle, int32_t iorder, int32_t nxy, const double* xy, int32_t nidx,
                          const int32_t* idx, int32_t nwall, const int32_t* idxwall, int32_t nopen,
                          const int32_t* idxopen);
/* Replaces load_inout_arrays_d (3889-3904): "inlet" and "outlet" edges, each with one
 * normal velocity per edge (or two values: parallel, normal). */
int ho2d_load_inout_arrays(ho2d_solver* handle, int32_t ninval, const double* velin, int32_t nin,
                           const int32_t* idxin, int32_t noutval, const double* velout, int32_t nout,
                           const int32_t* idxout);
/* Replaces process_mesh_input (3907-3940): mesh processing and the device setup. */
int ho2d_process_mesh_input(ho2d_solver* handle);
/* Replaces getsolnareas_d (3983-3994): w_j w_k J per solution point, len = N_el*Knod*Knod. */
int ho2d_get_solution_areas(ho2d_solver* handle, int32_t len, double* buf);
/* Replaces getopenptlen (3996-4004): 2 * (open edges) * Knod. */
int ho2d_get_open_point_count(ho2d_solver* handle, int32_t* len);
/* Replaces getopenpts_d (4006-4031): [open edge][Knod][x, y] along each edge. */
int ho2d_get_open_points(ho2d_solver* handle, int32_t len, double* buf);
/* Replaces setopenvels_d (4035-4106): Cartesian velocity [open edge][Knod][u, v] at the end
 * of the outer step; the previous values become the start values. */
int ho2d_set_open_velocities(ho2d_solver* handle, int32_t len, const double* buf);
/* Replaces setopenvort_d (4109-4129): vorticity [open edge][Knod] at the end of the outer step. */
int ho2d_set_open_vorticity(ho2d_solver* handle, int32_t len, const double* buf);
/* Replaces setptogweights_d (4156-4170): blend weights per solution point, len = N_el*Knod*Knod. */
int ho2d_set_ptog_weights(ho2d_solver* handle, int32_t len, const double* buf);
/* Replaces get_hoquad_weights_d (4252-4260): 0.25 w_j w_k, len = Knod*Knod. */
int ho2d_get_hoquad_weights(ho2d_solver* handle, int32_t len, double* buf);
/* Replaces clean_up (4274-4277): frees the device state; the handle stays valid. The
 * reference's trigger_write (VTK files) is not provided. */
int ho2d_clean_up(ho2d_solver* handle);

/* ---- Discrete adjoint. No counterpart in the reference: gradients of a scalar
 * J(omega(T)) of the vorticity after nsteps time steps with respect to the initial
 * vorticity and to BC_parl_vel (the wall velocity of no-slip walls, constant in time),
 * by the transpose of the discrete time loop of solve_advection_diffusion
 * (src/HO_2D.cpp:1465-1531): stage kernels run backwards, a transposed Poisson solve per
 * stage. Advection types 1 and 2, every precision: with HO2D_MIXED_KRYLOV the forward and
 * transposed Poisson solves are FP32 Krylov inside FP64 refinement; with HO2D_MIXED the
 * forward sweep and its recomputation follow the FP32-stage trajectory and each stage is
 * linearised in FP64 at its states. Hybrid runs (problem type 11) are rejected with
 * HO2D_ERR_UNSUPPORTED. */
/* Storage of the adjoint's checkpoints and recomputed stage states: 0 = FP64 (default),
 * 1 = FP32 (half the memory; the backward sweep then linearises about a trajectory
 * recomputed from FP32-rounded states). Takes effect at the next ho2d_adjoint_forward. */
int ho2d_set_adjoint_storage(ho2d_solver* handle, int32_t fp32);
/* Runs nsteps time steps from the current state (as ho2d_step) and keeps the vorticity
 * every ckpt_every steps for the backward sweep. */
int ho2d_adjoint_forward(ho2d_solver* handle, int32_t nsteps, int32_t ckpt_every);
/* From dJ/d(omega(T)) (len = N_el*Knod*Knod) returns dJ/d(omega) at the start of the last
 * ho2d_adjoint_forward (same length) and dJ/d(BC_parl_vel) (len_pv = N_eb*Knod; 0 with a
 * null buffer skips it). Each segment of ckpt_every steps is recomputed from its
 * checkpoint; afterwards the solver is back at the state and time reached by the forward
 * sweep. */
int ho2d_adjoint_backward(ho2d_solver* handle, int32_t len, const double* dJ_domegaT, double* grad_omega0,
                          int32_t len_pv, double* grad_parl_vel);
/* Adjoint of one ho2d_stage(coeff) at the current state: lam_k, the adjoint of the
 * stage's k (len = N_el*Knod*Knod), to lam_w, the adjoint of the stage input, and lam_pv,
 * the adjoint of BC_parl_vel (len_pv = N_eb*Knod, or 0 with a null buffer). */
int ho2d_stage_adjoint(ho2d_solver* handle, double coeff, int32_t len, const double* lam_k, double* lam_w,
                       int32_t len_pv, double* lam_pv);
/* y = A^T x in FP64 with the transposed matrix-free Poisson operator; len = N_el*Knod*Knod. */
int ho2d_apply_poisson_transpose(ho2d_solver* handle, int32_t len, const double* x, double* y);
/* Krylov iterations (summed over refinement sweeps) and final relative residual of the
 * last transposed Poisson solve. */
int ho2d_adjoint_stats(ho2d_solver* handle, int32_t* iterations, double* rel_residual);

/* Total number of kernel launches this handle has issued since it was created. */
int ho2d_last_launch_count(ho2d_solver* handle, int64_t* launches);
/* Text of the last error on this handle ("" if none). The pointer stays valid until the
 * next call on the handle. */
const char* ho2d_last_error(ho2d_solver* handle);

#ifdef __cplusplus
}
#endif

#endif /* HO2D_H */
