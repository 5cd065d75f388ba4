/*
 * HO_2D.hpp -- header-only C++ wrapper that keeps the member spelling of the reference's
 * HO_2D class (src/HO_2D.hpp:219-290) on top of the C ABI in ho2d.h, so a caller written
 * against the reference (src/main.cpp:44-77, or a hybrid driver calling solveto_d /
 * getallvorts_d) switches by changing the include and the link line (-lho2d).
 * Methods return the reference's success codes (0) or throw HO2DException.
 */
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "ho2d.h"

class HO2DException : public std::runtime_error {
  public:
    HO2DException(int code, const std::string& msg) : std::runtime_error(msg), code_(code) {}
    int code() const { return code_; }

  private:
    int code_;
};

class HO_2D {
  public:
    HO_2D() {
        if (ho2d_create(&h_) != HO2D_OK) throw HO2DException(HO2D_ERR_ARG, "ho2d_create failed");
    }
    ~HO_2D() { ho2d_destroy(h_); }
    HO_2D(const HO_2D&) = delete;
    HO_2D& operator=(const HO_2D&) = delete;

    int read_input_file(const std::string& filename) { return check(ho2d_read_input(h_, filename.c_str())); }
    // setup_mesh ... form_Laplace_operator_matrix: one device setup, run by the first call
    char setup_mesh() { return ensure_setup(); }
    char allocate_arrays() { return ensure_setup(); }
    void setup_sps_gps() { ensure_setup(); }
    void read_process_sample_points() {}  // the setup reads the input's sample points
    void form_bases() { ensure_setup(); }
    void form_metrics() { ensure_setup(); }
    void setup_IC_BC_SRC() { ensure_setup(); }
    void form_Laplace_operator_matrix() { ensure_setup(); }
    // the time loop; like the reference, writes the dump-step VTK (and sample-point) files
    // into the working directory unless set_output_dir chose another one ("" = none)
    char solve_vorticity_streamfunction() {
        if (!output_dir_set_) set_output_dir(".");
        return (char)check(ho2d_solve(h_));
    }
    void set_output_dir(const std::string& dir) {
        check(ho2d_set_output_dir(h_, dir.c_str()));
        output_dir_set_ = true;
    }
    char solve_advection_diffusion() { return (char)check(ho2d_step(h_, 1)); }
    void solveto_d(double outerdt, int32_t numstep, int32_t integtype, double reyn, int32_t region = 0) {
        check(ho2d_solveto(h_, outerdt, numstep, integtype, reyn, region));
    }
    void setsolnvort_d(int32_t len, const double* v) { check(ho2d_set_vort(h_, len, v)); }
    void getallvorts_d(int32_t len, double* v) { check(ho2d_get_vort(h_, len, v)); }
    void getsolnpts_d(int32_t len, double* xy) { check(ho2d_get_solution_points(h_, len, xy)); }
    // length of the getsolnpts_d array: x, y per solution point (src/HO_2D.cpp:3942-3944)
    int32_t getsolnptlen() { return 2 * getsolnlen(); }
    // length of the getallvorts_d / setsolnvort_d arrays: N_el * Knod^2 (no counterpart in
    // the reference, which takes the length from getsolnptlen / 2)
    int32_t getsolnlen() {
        int32_t n = 0, k = 0;
        check(ho2d_get_sizes(h_, &n, &k, nullptr, nullptr));
        return n * k * k;
    }

    // hybrid operation (src/HO_2D.hpp:251-290)
    void set_defaults() { check(ho2d_set_defaults(h_)); }
    void enable_hybrid() { check(ho2d_enable_hybrid(h_)); }
    void set_elemorder(int32_t eorder) { check(ho2d_set_elemorder(h_, eorder)); }
    void load_mesh_arrays_d(int32_t iorder, int32_t nnodes, const double* xynodes, int32_t nelems,
                            const int32_t* idxelems, int32_t nwall, const int32_t* idxwall, int32_t nopen,
                            const int32_t* idxopen) {
        check(ho2d_load_mesh_arrays(h_, iorder, nnodes, xynodes, nelems, idxelems, nwall, idxwall, nopen, idxopen));
    }
    void load_inout_arrays_d(int32_t ninval, const double* velin, int32_t nin, const int32_t* idxin,
                             int32_t noutval, const double* velout, int32_t nout, const int32_t* idxout) {
        check(ho2d_load_inout_arrays(h_, ninval, velin, nin, idxin, noutval, velout, nout, idxout));
    }
    void process_mesh_input() {
        check(ho2d_process_mesh_input(h_));
        setup_ = true;
    }
    void getsolnareas_d(int32_t len, double* areas) { check(ho2d_get_solution_areas(h_, len, areas)); }
    int32_t getopenptlen() {
        int32_t n = 0;
        check(ho2d_get_open_point_count(h_, &n));
        return n;
    }
    void getopenpts_d(int32_t len, double* xy) { check(ho2d_get_open_points(h_, len, xy)); }
    void setopenvels_d(int32_t len, const double* xyvel) { check(ho2d_set_open_velocities(h_, len, xyvel)); }
    void setopenvort_d(int32_t len, const double* vort) { check(ho2d_set_open_vorticity(h_, len, vort)); }
    void setptogweights_d(int32_t len, const double* wgt) { check(ho2d_set_ptog_weights(h_, len, wgt)); }
    void get_hoquad_weights_d(int32_t len, double* w) { check(ho2d_get_hoquad_weights(h_, len, w)); }
    // the two VTK files of the current fields into the working directory
    void trigger_write(int32_t indx, int32_t subidx) { check(ho2d_write_vtk(h_, indx, subidx, nullptr)); }
    void clean_up() {
        check(ho2d_clean_up(h_));
        setup_ = false;
    }
    void set_precision(int mode) { check(ho2d_set_precision(h_, mode)); }
    // smoother of the FP32 preconditioner (enum ho2d_smoother) for the next setup
    void set_smoother(int kind) { check(ho2d_set_smoother(h_, kind)); }
    ho2d_solver* handle() { return h_; }

  private:
    int check(int code) {
        if (code != HO2D_OK) throw HO2DException(code, ho2d_last_error(h_));
        return 0;
    }
    char ensure_setup() {
        if (!setup_) {
            check(ho2d_setup(h_));
            setup_ = true;
        }
        return 0;
    }
    ho2d_solver* h_ = nullptr;
    bool setup_ = false;
    bool output_dir_set_ = false;
};
