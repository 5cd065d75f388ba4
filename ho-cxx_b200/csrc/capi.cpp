// capi.cpp -- the extern "C" boundary declared in include/ho2d.h. Every entry point
// catches exceptions and turns them into status codes plus a per-handle message.
#include <cmath>
#include <cstring>
#include <exception>
#include <new>
#include <string>

#include "../../include/ho2d.h"
#include "solver.hpp"

struct ho2d_solver {
    ho2d::Solver s;
    std::string err;
};

namespace {

int finish(ho2d_solver* h, const ho2d::Error& e) {
    h->err = e.code ? e.msg : std::string();
    return e.code;
}

template <typename F>
int guarded(ho2d_solver* h, F&& f) {
    if (!h) return HO2D_ERR_ARG;
    try {
        return finish(h, f());
    } catch (const std::bad_alloc&) {
        h->err = "host out of memory";
        return HO2D_ERR_ARG;
    } catch (const std::exception& ex) {
        h->err = ex.what();
        return HO2D_ERR_ARG;
    } catch (...) {
        h->err = "unknown exception";
        return HO2D_ERR_ARG;
    }
}

ho2d::Error check_len(const ho2d_solver* h, int32_t len, size_t expect, const void* buf) {
    if (!h->s.is_setup()) return {HO2D_ERR_ARG, "call ho2d_setup first"};
    if (!buf) return {HO2D_ERR_ARG, "null buffer"};
    if (len < 0 || (size_t)len != expect)
        return {HO2D_ERR_ARG, "buffer length " + std::to_string(len) + " != expected " + std::to_string(expect)};
    return {0, ""};
}

size_t nvol(const ho2d_solver* h) { return (size_t)h->s.n_el() * h->s.knod() * h->s.knod(); }
size_t nbnd(const ho2d_solver* h) { return (size_t)h->s.n_eb() * h->s.knod(); }

}  // namespace

extern "C" {

int ho2d_create(ho2d_solver** handle) {
    if (!handle) return HO2D_ERR_ARG;
    try {
        *handle = new ho2d_solver();
    } catch (...) {
        *handle = nullptr;
        return HO2D_ERR_ARG;
    }
    return HO2D_OK;
}

int ho2d_destroy(ho2d_solver* handle) {
    if (!handle) return HO2D_ERR_ARG;
    delete handle;
    return HO2D_OK;
}

int ho2d_read_input(ho2d_solver* h, const char* path) {
    return guarded(h, [&]() -> ho2d::Error {
        if (!path) return {HO2D_ERR_ARG, "null path"};
        return h->s.read_input(path);
    });
}

int ho2d_setup(ho2d_solver* h) {
    return guarded(h, [&]() { return h->s.setup(); });
}

int ho2d_solve(ho2d_solver* h) {
    return guarded(h, [&]() { return h->s.solve(); });
}

int ho2d_step(ho2d_solver* h, int32_t nsteps) {
    return guarded(h, [&]() { return h->s.step(nsteps); });
}

int ho2d_stage(ho2d_solver* h, double coeff) {
    return guarded(h, [&]() { return h->s.stage(coeff); });
}

int ho2d_solveto(ho2d_solver* h, double outerdt, int32_t numstep, int32_t integtype, double reyn, int32_t region) {
    (void)region;  // names output files in the reference; nothing is written here
    return guarded(h, [&]() { return h->s.solveto(outerdt, numstep, integtype, reyn); });
}

int ho2d_get_sizes(ho2d_solver* h, int32_t* n_el, int32_t* knod, int32_t* n_edges_boundary, int32_t* lnod) {
    return guarded(h, [&]() -> ho2d::Error {
        if (!h->s.is_setup()) return {HO2D_ERR_ARG, "call ho2d_setup first"};
        if (n_el) *n_el = h->s.n_el();
        if (knod) *knod = h->s.knod();
        if (n_edges_boundary) *n_edges_boundary = h->s.n_eb();
        if (lnod) *lnod = h->s.lnod();
        return {0, ""};
    });
}

int ho2d_get_vort(ho2d_solver* h, int32_t len, double* buf) {
    return guarded(h, [&]() -> ho2d::Error {
        ho2d::Error e = check_len(h, len, nvol(h), buf);
        return e.code ? e : h->s.get_volume(HO2D_FIELD_VORTICITY, buf);
    });
}

int ho2d_set_vort(ho2d_solver* h, int32_t len, const double* buf) {
    return guarded(h, [&]() -> ho2d::Error {
        ho2d::Error e = check_len(h, len, nvol(h), buf);
        return e.code ? e : h->s.set_vorticity(buf);
    });
}

int ho2d_get_psi(ho2d_solver* h, int32_t len, double* buf) {
    return guarded(h, [&]() -> ho2d::Error {
        ho2d::Error e = check_len(h, len, nvol(h), buf);
        return e.code ? e : h->s.get_volume(HO2D_FIELD_STREAMFUNCTION, buf);
    });
}

int ho2d_get_vel(ho2d_solver* h, int32_t len, double* buf) {
    return guarded(h, [&]() -> ho2d::Error {
        ho2d::Error e = check_len(h, len, 2 * nvol(h), buf);
        return e.code ? e : h->s.get_velocity(buf);
    });
}

int ho2d_get_field(ho2d_solver* h, int32_t which, int32_t len, double* buf) {
    return guarded(h, [&]() -> ho2d::Error {
        ho2d::Error e = check_len(h, len, nvol(h), buf);
        return e.code ? e : h->s.get_volume(which, buf);
    });
}

int ho2d_get_boundary(ho2d_solver* h, int32_t which, int32_t len, double* buf) {
    return guarded(h, [&]() -> ho2d::Error {
        ho2d::Error e = check_len(h, len, nbnd(h), buf);
        return e.code ? e : h->s.get_boundary(which, buf);
    });
}

int ho2d_set_boundary(ho2d_solver* h, int32_t which, int32_t len, const double* buf) {
    return guarded(h, [&]() -> ho2d::Error {
        ho2d::Error e = check_len(h, len, nbnd(h), buf);
        return e.code ? e : h->s.set_boundary(which, buf);
    });
}

int ho2d_get_boundary_points(ho2d_solver* h, int32_t len, double* buf) {
    return guarded(h, [&]() -> ho2d::Error {
        ho2d::Error e = check_len(h, len, 2 * nbnd(h), buf);
        return e.code ? e : h->s.get_boundary_points(buf);
    });
}

int ho2d_get_solution_points(ho2d_solver* h, int32_t len, double* buf) {
    return guarded(h, [&]() -> ho2d::Error {
        ho2d::Error e = check_len(h, len, 2 * nvol(h), buf);
        return e.code ? e : h->s.get_solution_points(buf);
    });
}

int ho2d_set_precision(ho2d_solver* h, int32_t mode) {
    return guarded(h, [&]() { return h->s.set_precision(mode); });
}

int ho2d_profile_krylov(ho2d_solver* h, int32_t iterations, double* ms, double* bytes) {
    return guarded(h, [&]() { return h->s.profile_krylov(iterations, ms, bytes); });
}

int ho2d_set_smoother(ho2d_solver* h, int32_t kind) {
    return guarded(h, [&]() { return h->s.set_smoother(kind); });
}

int ho2d_get_smoother(ho2d_solver* h, int32_t* kind, int32_t* exact_blocks) {
    return guarded(h, [&]() -> ho2d::Error {
        if (!h->s.is_setup()) return {HO2D_ERR_ARG, "call ho2d_setup first"};
        if (kind) *kind = h->s.smoother();
        if (exact_blocks) *exact_blocks = h->s.smoother_exact_blocks();
        return {0, ""};
    });
}

int ho2d_set_device_setup(ho2d_solver* h, int32_t on) {
    return guarded(h, [&]() -> ho2d::Error {
        if (on != 0 && on != 1) return {HO2D_ERR_ARG, "on must be 0 or 1"};
        h->s.set_device_setup(on == 1);
        return {0, ""};
    });
}

int ho2d_get_poisson_setup(ho2d_solver* h, int32_t which, int64_t len, double* buf) {
    return guarded(h, [&]() -> ho2d::Error {
        if (!h->s.is_setup()) return {HO2D_ERR_ARG, "call ho2d_setup first"};
        if (!buf) return {HO2D_ERR_ARG, "null buffer"};
        return h->s.get_poisson_setup(which, len, buf);
    });
}

int ho2d_set_poisson_tolerance(ho2d_solver* h, double rel_tol, int32_t max_iter) {
    return guarded(h, [&]() -> ho2d::Error {
        if (!(rel_tol > 0.0) || max_iter <= 0) return {HO2D_ERR_ARG, "tolerance and iteration cap must be positive"};
        h->s.set_poisson_tolerance(rel_tol, max_iter);
        return {0, ""};
    });
}

int ho2d_poisson_stats(ho2d_solver* h, int32_t* iterations, double* rel_residual) {
    return guarded(h, [&]() -> ho2d::Error {
        if (iterations) *iterations = h->s.last_poisson_iterations();
        if (rel_residual) *rel_residual = h->s.last_poisson_residual();
        return {0, ""};
    });
}

int ho2d_solve_counters(ho2d_solver* h, int64_t* solves, int64_t* iterations, int64_t* sweeps) {
    return guarded(h, [&]() -> ho2d::Error {
        h->s.counters(solves, iterations, sweeps);
        return {0, ""};
    });
}

int ho2d_fp64_finishes(ho2d_solver* h, int64_t* count) {
    return guarded(h, [&]() -> ho2d::Error {
        if (!count) return {HO2D_ERR_ARG, "null pointer"};
        *count = h->s.fp64_finishes();
        return {0, ""};
    });
}

int ho2d_get_time(ho2d_solver* h, double* time, double* dt) {
    return guarded(h, [&]() -> ho2d::Error {
        if (time) *time = h->s.time();
        if (dt) *dt = h->s.dt();
        return {0, ""};
    });
}

int ho2d_set_time(ho2d_solver* h, double time) {
    return guarded(h, [&]() -> ho2d::Error {
        if (!std::isfinite(time)) return {HO2D_ERR_ARG, "time must be finite"};
        h->s.set_time(time);
        return {0, ""};
    });
}

int ho2d_time_steps(ho2d_solver* h, int32_t nsteps, double* total_ms, double* poisson_ms) {
    return guarded(h, [&]() { return h->s.time_steps(nsteps, total_ms, poisson_ms); });
}

int ho2d_profile_spmv(ho2d_solver* h, int32_t reps, double* avg_ms, double* bytes_per_launch) {
    return guarded(h, [&]() { return h->s.profile_spmv(reps, avg_ms, bytes_per_launch); });
}

int ho2d_apply_poisson(ho2d_solver* h, int32_t len, const double* x, double* y) {
    return guarded(h, [&]() -> ho2d::Error {
        ho2d::Error e = check_len(h, len, nvol(h), x);
        if (e.code) return e;
        if (!y) return {HO2D_ERR_ARG, "null output buffer"};
        return h->s.apply_poisson(x, y);
    });
}

int ho2d_apply_poisson_noalloc(ho2d_solver* h, int32_t len, const double* x_device, double* y_device) {
    return guarded(h, [&]() -> ho2d::Error {
        ho2d::Error e = check_len(h, len, nvol(h), x_device);
        if (e.code) return e;
        return h->s.apply_poisson_noalloc(x_device, y_device);
    });
}

int ho2d_get_forces(ho2d_solver* h, double* fx, double* fy) {
    return guarded(h, [&]() { return h->s.get_forces(fx, fy); });
}

int ho2d_set_output_dir(ho2d_solver* h, const char* dir) {
    return guarded(h, [&]() -> ho2d::Error {
        h->s.set_output_dir(dir ? dir : "");
        return {0, ""};
    });
}

int ho2d_write_vtk(ho2d_solver* h, int32_t indx, int32_t subidx, const char* dir) {
    return guarded(h, [&]() { return h->s.write_vtk(indx, subidx, dir ? dir : ""); });
}

int ho2d_set_defaults(ho2d_solver* h) {
    return guarded(h, [&]() -> ho2d::Error {
        h->s.set_defaults();
        return {0, ""};
    });
}

int ho2d_enable_hybrid(ho2d_solver* h) {
    return guarded(h, [&]() -> ho2d::Error {
        h->s.enable_hybrid();
        return {0, ""};
    });
}

int ho2d_set_elemorder(ho2d_solver* h, int32_t knod) {
    return guarded(h, [&]() { return h->s.set_elemorder(knod); });
}

int ho2d_load_mesh_arrays(ho2d_solver* h, int32_t iorder, int32_t nxy, const double* xy, int32_t nidx,
                          const int32_t* idx, int32_t nwall, const int32_t* idxwall, int32_t nopen,
                          const int32_t* idxopen) {
    return guarded(h, [&]() -> ho2d::Error {
        if (!xy || !idx || (nwall > 0 && !idxwall) || (nopen > 0 && !idxopen)) return {HO2D_ERR_ARG, "null buffer"};
        return h->s.load_mesh_arrays(iorder, nxy, xy, nidx, idx, nwall, idxwall, nopen, idxopen);
    });
}

int ho2d_load_inout_arrays(ho2d_solver* h, int32_t ninval, const double* velin, int32_t nin, const int32_t* idxin,
                           int32_t noutval, const double* velout, int32_t nout, const int32_t* idxout) {
    return guarded(h, [&]() {
        return h->s.load_inout_arrays(ninval, velin, nin, idxin, noutval, velout, nout, idxout);
    });
}

int ho2d_process_mesh_input(ho2d_solver* h) {
    return guarded(h, [&]() { return h->s.process_mesh_input(); });
}

int ho2d_get_solution_areas(ho2d_solver* h, int32_t len, double* buf) {
    return guarded(h, [&]() -> ho2d::Error {
        ho2d::Error e = check_len(h, len, nvol(h), buf);
        return e.code ? e : h->s.get_solution_areas(buf);
    });
}

int ho2d_get_open_point_count(ho2d_solver* h, int32_t* len) {
    return guarded(h, [&]() -> ho2d::Error {
        if (!len) return {HO2D_ERR_ARG, "null output"};
        *len = h->s.open_point_count();
        return {0, ""};
    });
}

int ho2d_get_open_points(ho2d_solver* h, int32_t len, double* buf) {
    return guarded(h, [&]() -> ho2d::Error {
        ho2d::Error e = check_len(h, len, (size_t)h->s.open_point_count(), buf);
        return e.code ? e : h->s.get_open_points(buf);
    });
}

int ho2d_set_open_velocities(ho2d_solver* h, int32_t len, const double* buf) {
    return guarded(h, [&]() -> ho2d::Error {
        ho2d::Error e = check_len(h, len, (size_t)h->s.open_point_count(), buf);
        return e.code ? e : h->s.set_open_velocities(buf);
    });
}

int ho2d_set_open_vorticity(ho2d_solver* h, int32_t len, const double* buf) {
    return guarded(h, [&]() -> ho2d::Error {
        ho2d::Error e = check_len(h, len, (size_t)h->s.open_point_count() / 2, buf);
        return e.code ? e : h->s.set_open_vorticity(buf);
    });
}

int ho2d_set_ptog_weights(ho2d_solver* h, int32_t len, const double* buf) {
    return guarded(h, [&]() -> ho2d::Error {
        ho2d::Error e = check_len(h, len, nvol(h), buf);
        return e.code ? e : h->s.set_ptog_weights(buf);
    });
}

int ho2d_get_hoquad_weights(ho2d_solver* h, int32_t len, double* buf) {
    return guarded(h, [&]() -> ho2d::Error {
        ho2d::Error e = check_len(h, len, (size_t)h->s.knod() * h->s.knod(), buf);
        return e.code ? e : h->s.get_hoquad_weights(buf);
    });
}

int ho2d_clean_up(ho2d_solver* h) {
    return guarded(h, [&]() -> ho2d::Error {
        h->s.release();
        return {0, ""};
    });
}

int ho2d_set_adjoint_storage(ho2d_solver* h, int32_t fp32) {
    return guarded(h, [&]() -> ho2d::Error {
        if (fp32 != 0 && fp32 != 1) return {HO2D_ERR_ARG, "storage must be 0 (FP64) or 1 (FP32)"};
        h->s.set_adjoint_storage(fp32 == 1);
        return {0, ""};
    });
}

int ho2d_adjoint_forward(ho2d_solver* h, int32_t nsteps, int32_t ckpt_every) {
    return guarded(h, [&]() -> ho2d::Error {
        if (!h->s.is_setup()) return {HO2D_ERR_ARG, "call ho2d_setup first"};
        return h->s.adjoint_forward(nsteps, ckpt_every);
    });
}

int ho2d_adjoint_backward(ho2d_solver* h, int32_t len, const double* dJ_domegaT, double* grad_omega0, int32_t len_pv,
                          double* grad_parl_vel) {
    return guarded(h, [&]() -> ho2d::Error {
        ho2d::Error e = check_len(h, len, nvol(h), dJ_domegaT);
        if (e.code) return e;
        if (!grad_omega0) return {HO2D_ERR_ARG, "null output buffer"};
        if (grad_parl_vel || len_pv) {
            e = check_len(h, len_pv, nbnd(h), grad_parl_vel);
            if (e.code) return e;
        }
        return h->s.adjoint_backward(dJ_domegaT, grad_omega0, grad_parl_vel);
    });
}

int ho2d_stage_adjoint(ho2d_solver* h, double coeff, int32_t len, const double* lam_k, double* lam_w, int32_t len_pv,
                       double* lam_pv) {
    return guarded(h, [&]() -> ho2d::Error {
        ho2d::Error e = check_len(h, len, nvol(h), lam_k);
        if (e.code) return e;
        if (!lam_w) return {HO2D_ERR_ARG, "null output buffer"};
        if (lam_pv || len_pv) {
            e = check_len(h, len_pv, nbnd(h), lam_pv);
            if (e.code) return e;
        }
        return h->s.stage_adjoint(coeff, lam_k, lam_w, lam_pv);
    });
}

int ho2d_apply_poisson_transpose(ho2d_solver* h, int32_t len, const double* x, double* y) {
    return guarded(h, [&]() -> ho2d::Error {
        ho2d::Error e = check_len(h, len, nvol(h), x);
        if (e.code) return e;
        if (!y) return {HO2D_ERR_ARG, "null output buffer"};
        return h->s.apply_poisson_transpose(x, y);
    });
}

int ho2d_adjoint_stats(ho2d_solver* h, int32_t* iterations, double* rel_residual) {
    return guarded(h, [&]() -> ho2d::Error {
        if (iterations) *iterations = h->s.last_adjoint_iterations();
        if (rel_residual) *rel_residual = h->s.last_adjoint_residual();
        return {0, ""};
    });
}

int ho2d_last_launch_count(ho2d_solver* h, int64_t* launches) {
    return guarded(h, [&]() -> ho2d::Error {
        if (launches) *launches = h->s.launches();
        return {0, ""};
    });
}

const char* ho2d_last_error(ho2d_solver* h) {
    if (!h) return "null handle";
    return h->err.c_str();
}

}  // extern "C"
