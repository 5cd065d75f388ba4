// adjoint_driver.cu -- the discrete adjoint of the time loop: checkpointed forward sweep,
// recomputation of one segment at a time, the reverse sweep over the RK stages, and the
// transposed Poisson solve.
//
// No counterpart in the reference. The forward map of a step is the stage sequence of
// solve_advection_diffusion (src/HO_2D.cpp:1465-1531) with the stages of
// Euler_time_integrate (1806-1839). Its adjoint here is the transpose of the discrete
// map (adjoint_chain.cuh for the stage kernels, BiCGSTAB on A^T for the Poisson solve),
// exact up to the Poisson tolerance of the forward recomputation and of the transposed
// solve.
//
// Memory: one FP64 vorticity per checkpoint (every ckpt_every steps) and, during the
// backward sweep, the stage inputs and streamfunctions of one segment
// (ckpt_every x stages x 2 FP64 fields); the trajectory is never stored whole.
#include <cmath>
#include <cstdio>
#include <cstdlib>

#include "adjoint_launch.hpp"
#include "solver_state.hpp"

namespace ho2d {

namespace {

// Explicit schemes of solve_advection_diffusion as Butcher tableaux: stage inputs
// w_s = omega + sum_r a[s][r] k_r at time t + c[s] dt, and omega' = omega + sum_s b[s] k_s.
struct Tableau {
    int ns = 1;
    double c[4] = {0, 0, 0, 0};
    double b[4] = {1, 0, 0, 0};
    double a[4][4] = {};
};

Tableau tableau(int ti_type) {
    Tableau t;
    if (ti_type == 4) {
        t.ns = 4;
        const double c[4] = {0.0, 0.5, 0.5, 1.0}, b[4] = {1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0};
        for (int s = 0; s < 4; ++s) {
            t.c[s] = c[s];
            t.b[s] = b[s];
        }
        t.a[1][0] = 0.5;
        t.a[2][1] = 0.5;
        t.a[3][2] = 1.0;
    } else if (ti_type == 2) {
        t.ns = 2;
        t.c[1] = 1.0;
        t.b[0] = t.b[1] = 0.5;
        t.a[1][0] = 1.0;
    }
    return t;
}

Csr transpose_csr(const Csr& A) {
    Csr T;
    T.n = A.m;
    T.m = A.n;
    T.ptr.assign((size_t)T.n + 1, 0);
    for (int c : A.col) ++T.ptr[(size_t)c + 1];
    for (int i = 0; i < T.n; ++i) T.ptr[(size_t)i + 1] += T.ptr[i];
    T.col.resize(A.col.size());
    T.val.resize(A.val.size());
    std::vector<int> pos(T.ptr.begin(), T.ptr.end() - 1);
    for (int r = 0; r < A.n; ++r)
        for (int q = A.ptr[r]; q < A.ptr[(size_t)r + 1]; ++q) {
            const int dst = pos[A.col[q]]++;
            T.col[dst] = r;
            T.val[dst] = A.val[q];
        }
    return T;
}

template <typename T>
const DevBases<T>& bases_of(const DeviceState& d, bool f32) {
    return *reinterpret_cast<const DevBases<T>*>(f32 ? (const void*)&d.b32 : (const void*)&d.b64);
}

}  // namespace

int Solver::adjoint_steps() const { return adj_ ? adj_->nsteps : -1; }

// Buffers and the preconditioner of the transposed Poisson problem, built once per setup.
Error Solver::adjoint_prepare() {
    if (!setup_done_) return {1, "call ho2d_setup first"};
    if (!adj_) adj_.reset(new AdjointState);
    AdjointState& a = *adj_;
    if (a.ready) return {0, ""};
    DeviceState& d = *d_;
    HO2D_CUDA(cudaSetDevice(d.device), "cudaSetDevice");
    if (krylov32_) HO2D_TRY(upload_precision_arrays());
    const int N = mesh_.n_el, K = in_.knod, K2 = K * K, neb = std::max(1, mesh_.n_eb);
    const size_t nv = (size_t)N * K2, nf = (size_t)N * 4 * K;
    const std::vector<double> zv(nv, 0.0), zf(nf, 0.0), zb((size_t)neb * K, 0.0);
    for (auto& b : a.kv) HO2D_CUDA(upload(b, zv), "alloc adjoint Krylov");
    for (DeviceBuffer* b : {&a.res64, &a.x32, &a.b32, &a.lam_k, &a.lw_out, &a.lw_dir, &a.lux, &a.luy, &a.lw_stage,
                            &a.lpsi_dir, &a.lpsi, &a.mu, &a.lam, &a.wT, &a.psiT})
        HO2D_CUDA(upload(*b, zv), "alloc adjoint fields");
    for (auto& b : a.mus) HO2D_CUDA(upload(b, zv), "alloc adjoint fields");
    for (DeviceBuffer* b : {&a.sv, &a.sg, &a.swv, &a.swg, &a.sU, &a.spv, &a.spg})
        HO2D_CUDA(upload(*b, zf), "alloc adjoint slots");
    for (DeviceBuffer* b : {&a.lbc_d, &a.lbc_nv, &a.lpv}) HO2D_CUDA(upload(*b, zb), "alloc adjoint boundary");
    HO2D_CUDA(upload(a.f0, std::vector<double>((size_t)N + 4, 0.0)), "alloc element sums");
    HO2D_CUDA(upload(a.partials, std::vector<double>((size_t)2 * kt_grid(), 0.0)), "alloc partials");
    HO2D_CUDA(upload(a.counter, std::vector<unsigned>(1, 0u)), "alloc counter");
    HO2D_CUDA(a.scalars.alloc(sizeof(KrylovScalars)), "alloc scalars");
    HO2D_CUDA(cudaMemset(a.scalars.get(), 0, sizeof(KrylovScalars)), "memset");
    // column sums of A's blocks: (A^T P u)(el, ij) = sum over the 5 block slots of el of
    // u[c] * sum_r A[(c, r), (el, ij)], c = the slot's element: the column sums (over rows
    // r, ascending) of block (c, s2), the slot of c whose column element is el
    HO2D_TRY(ensure_host_colsum());
    std::vector<double> rsT((size_t)N * 5 * K2, 0.0);
    for (int el = 0; el < N; ++el)
        for (int s = 0; s < 5; ++s) {
            const int c = op_.block_col[(size_t)el * 5 + s];
            if (c < 0) continue;
            int s2 = -1;
            for (int q = 0; q < 5; ++q)
                if (op_.block_col[(size_t)c * 5 + q] == el) s2 = q;
            if (s2 < 0) return {3, "Poisson block structure is not symmetric"};
            const double* cs = &op_.colsum[((size_t)c * 5 + s2) * K2];
            std::copy(cs, cs + K2, rsT.begin() + ((size_t)el * 5 + s) * K2);
        }
    HO2D_CUDA(upload(a.rowsumT64, rsT), "upload transposed row sums");
    HO2D_CUDA(upload_as<float>(a.rowsumT32, rsT), "upload transposed row sums");
    // coarse hierarchy of the transposed P0 problem (same settings as the forward one)
    a.pc64 = Precond<double>();
    a.pc32 = Precond<float>();
    a.lev.clear();
    const char* mode = std::getenv("HO2D_PRECOND");
    const char* om = std::getenv("HO2D_MG_OMEGA");
    const double omega = om ? std::atof(om) : kSmoothingWeight;
    a.pc64.omega = a.pc32.omega = omega;
    if (!(mode && std::string(mode) == "bj")) {
        const char* dm = std::getenv("HO2D_DENSE_MAX");
        const int dmax = dm ? std::max(1, std::atoi(dm)) : kDenseMax;
        CoarseHierarchy H;
        HO2D_TRY(build_coarse_hierarchy(transpose_csr(p0_coarse_operator(op_, N)), H, dmax, dm ? dmax : kDenseMaxFirst,
                                        !device_setup_));
        HO2D_TRY(upload_hierarchy(H, omega, a.lev, a.dense64, a.dense32, a.pc64, a.pc32, nullptr));
    }
    HO2D_CUDA(cudaDeviceSynchronize(), "adjoint setup");
    a.ready = true;
    return {0, ""};
}

// BiCGSTAB on A^T x = b in precision T to relative tolerance tol; x starts at zero.
template <typename T>
Error Solver::kt_run(T* x, const T* b, bool f32, double tol, int& iters) {
    DeviceState& d = *d_;
    AdjointState& a = *adj_;
    const int K = in_.knod;
    const size_t n = (size_t)mesh_.n_el * K * K;
    TVectors<T> v;
    v.x = x;
    v.r = a.kv[0].as<T>();
    v.rhat = a.kv[1].as<T>();
    v.p = a.kv[2].as<T>();
    v.v = a.kv[3].as<T>();
    v.s = a.kv[4].as<T>();
    v.t = a.kv[5].as<T>();
    v.ph = a.kv[6].as<T>();
    v.sh = a.kv[7].as<T>();
    v.dir = a.kv[8].as<T>();
    v.b = b;
    v.sv = a.sv.as<T>();
    v.sg = a.sg.as<T>();
    v.f0 = a.f0.as<T>();
    TPrecond<T> pc;
    pc.pc = *reinterpret_cast<const Precond<T>*>(f32 ? (const void*)&a.pc32 : (const void*)&a.pc64);
    pc.dinv = f32 ? (const T*)d.dinv32.get() : (const T*)d.dinv64.get();
    pc.rowsumT = f32 ? (const T*)a.rowsumT32.get() : (const T*)a.rowsumT64.get();
    pc.bcol = d.bcol.as<int>();
    const TReduce red{a.partials.as<double>(), a.counter.as<unsigned>(), a.scalars.as<KrylovScalars>()};
    const FrGeom<T> g = geom_of<T>(d, mesh_, f32);
    const DevBases<T>& bb = bases_of<T>(d, f32);
    // the element sums' padding and the boundary entries of the slots must read as zero in
    // precision T; these buffers are shared by the FP64 and FP32 solves
    HO2D_CUDA(cudaMemsetAsync(a.f0.get(), 0, a.f0.bytes(), d.stream), "memset");
    HO2D_CUDA(cudaMemsetAsync(a.sv.get(), 0, a.sv.bytes(), d.stream), "memset");
    HO2D_CUDA(cudaMemsetAsync(a.sg.get(), 0, a.sg.bytes(), d.stream), "memset");
    d.h_sc->tol = tol;  // the stream is idle: the last read of h_sc was synchronised
    HO2D_CUDA(cudaMemcpyAsync(&red.sc->tol, &d.h_sc->tol, sizeof(double), cudaMemcpyHostToDevice, d.stream), "tol");
    if (use_graphs_) {
        // one launch of the captured solve (init and a device-side while loop); the graph
        // bakes in the operands, so it is recaptured when they change
        const int gi = f32 ? 1 : 0;
        SolveGraph& sg = a.graph[gi];
        if (!sg.exec || sg.max_iter != max_iter_ || a.graph_x[gi] != (const void*)x || a.graph_b[gi] != (const void*)b) {
            sg.reset();
            HO2D_CUDA(kt_capture_solve<T>(K, g, bb, v, pc, red, max_iter_, d.stream, &sg.graph), "graph capture");
            HO2D_CUDA(cudaGraphInstantiate(&sg.exec, sg.graph, 0), "graph instantiate");
            sg.max_iter = max_iter_;
            a.graph_x[gi] = x;
            a.graph_b[gi] = b;
        }
        HO2D_CUDA(cudaGraphLaunch(sg.exec, d.stream), "graph launch");
        HO2D_CUDA(cudaMemcpyAsync(d.h_sc, red.sc, sizeof(KrylovScalars), cudaMemcpyDeviceToHost, d.stream), "poll");
        HO2D_CUDA(cudaStreamSynchronize(d.stream), "poll");
        iters = d.h_sc->it;
        launches_ += 2 + (int64_t)iters * kt_launches_per_iteration<T>(pc);
        return {0, ""};
    }
    HO2D_CUDA(kt_init<T>(n, v, red, d.stream), "transposed init");
    launches_ += 1;
    // batches of iterations between polls of the done flag; an iteration enqueued after
    // the solve finished returns at once in every kernel
    int chunk = std::max(1, adj_prev_iters_ - 1);
    for (;;) {
        for (int c = 0; c < chunk; ++c) {
            HO2D_CUDA(kt_iteration<T>(K, g, bb, v, pc, red, max_iter_, d.stream), "transposed iteration");
            launches_ += kt_launches_per_iteration<T>(pc);
        }
        HO2D_CUDA(cudaMemcpyAsync(d.h_sc, red.sc, sizeof(KrylovScalars), cudaMemcpyDeviceToHost, d.stream), "poll");
        HO2D_CUDA(cudaStreamSynchronize(d.stream), "poll");
        if (d.h_sc->done) break;
        chunk = 2;
    }
    iters = d.h_sc->it;
    return {0, ""};
}

// mu = A^-T rhs (FP64 vectors): FP64 BiCGSTAB, or with a mixed-precision Krylov mode FP32
// BiCGSTAB inside FP64 iterative refinement on the FP64 transposed residual.
Error Solver::transposed_solve(const double* rhs, double* mu) {
    const NvtxRange nvtx_range("ho2d.poisson_transpose");
    DeviceState& d = *d_;
    AdjointState& a = *adj_;
    const int N = mesh_.n_el, K = in_.knod;
    const size_t nv = (size_t)N * K * K;
    const TReduce red{a.partials.as<double>(), a.counter.as<unsigned>(), a.scalars.as<KrylovScalars>()};
    bool finite = true;
    last_adj_iters_ = 0;
    int sweeps = 0;
    if (!krylov32_) {
        int it = 0;
        HO2D_TRY(kt_run<double>(mu, rhs, false, tol_, it));
        last_adj_iters_ = it;
        const double bn = d.h_sc->bnorm2, rn = d.h_sc->rnorm2;
        finite = std::isfinite(bn) && std::isfinite(rn);
        last_adj_res_ = bn > 0 ? std::sqrt(rn / bn) : 0.0;
    } else {
        const FrGeom<double> g = geom_of<double>(d, mesh_, false);
        HO2D_CUDA(cudaMemsetAsync(mu, 0, nv * 8, d.stream), "memset");
        for (;; ++sweeps) {
            HO2D_CUDA(cudaMemsetAsync(a.sv.get(), 0, a.sv.bytes(), d.stream), "memset");  // shared with FP32
            HO2D_CUDA(cudaMemsetAsync(a.sg.get(), 0, a.sg.bytes(), d.stream), "memset");
            HO2D_CUDA(poisson_transpose<double>(K, g, d.b64, mu, a.kv[9].as<double>(), a.kv[8].as<double>(),
                                                a.sv.as<double>(), a.sg.as<double>(), nullptr, 0, d.stream),
                      "transposed operator");
            HO2D_CUDA(kt_residual<double>(nv, rhs, a.kv[9].as<double>(), a.res64.as<double>(), red, d.stream),
                      "transposed residual");
            launches_ += 3;
            HO2D_CUDA(cudaMemcpyAsync(d.h_sc, red.sc, sizeof(KrylovScalars), cudaMemcpyDeviceToHost, d.stream), "poll");
            HO2D_CUDA(cudaStreamSynchronize(d.stream), "poll");
            const double bn = d.h_sc->bnorm2, rn = d.h_sc->rnorm2;
            finite = std::isfinite(bn) && std::isfinite(rn);
            last_adj_res_ = bn > 0 ? std::sqrt(rn / bn) : 0.0;
            if (!finite || bn == 0.0) break;
            if (rn <= tol_ * tol_ * bn || sweeps >= 30) break;
            HO2D_CUDA(launch_copy_d2f(a.res64.as<double>(), a.b32.as<float>(), nv, d.stream), "d2f");
            const double need = 0.3 * tol_ / last_adj_res_;
            const double itol = std::min(0.5, std::max(inner_tol_, need));
            int it = 0;
            HO2D_TRY(kt_run<float>(a.x32.as<float>(), a.b32.as<float>(), true, itol, it));
            last_adj_iters_ += it;
            HO2D_CUDA(launch_axpy_f2d(a.x32.as<float>(), mu, nv, d.stream), "axpy");
            launches_ += 2;
        }
    }
    adj_prev_iters_ = std::max(1, krylov32_ ? last_adj_iters_ / std::max(1, sweeps) : last_adj_iters_);
    if (!finite) return {7, "non-finite values in the transposed Poisson solve"};
    return {0, ""};
}

// Adjoint of one stage at the stage input in d.w_stage with its streamfunction in
// d.psi64 (both set by the caller, time_ at the step's start): lam of k in a.lam_k ->
// lam of the stage input in out; lam of BC_parl_vel accumulates in a.lpv.
Error Solver::stage_adjoint_dev(double coeff, double* out) {
    DeviceState& d = *d_;
    AdjointState& a = *adj_;
    const int N = mesh_.n_el, K = in_.knod;
    const size_t nv = (size_t)N * K * K;
    HO2D_TRY(stage_t<double>(coeff, 0, false, false));  // the stage's fields from its psi
    const FrGeom<double> g = geom_of<double>(d, mesh_, false);
    StageAdjArgs<double> sa;
    sa.w = d.w_stage.as<double>();
    sa.u = d.u.as<double>();
    sa.v = d.v.as<double>();
    sa.w_tv = d.w_tv.as<double>();
    sa.U_t = d.U_t.as<double>();
    sa.bc_w = d.bc_w.as<double>();
    sa.bc_nv = d.bc_nv.as<double>();
    sa.lam_k = a.lam_k.as<double>();
    sa.lw_dir = a.lw_dir.as<double>();
    sa.lux = a.lux.as<double>();
    sa.luy = a.luy.as<double>();
    sa.slot_wv = a.swv.as<double>();
    sa.slot_wg = a.swg.as<double>();
    sa.slot_U = a.sU.as<double>();
    sa.lbc_d = a.lbc_d.as<double>();
    sa.lbc_nv = a.lbc_nv.as<double>();
    sa.lw_stage = a.lw_stage.as<double>();
    sa.lpsi_dir = a.lpsi_dir.as<double>();
    sa.slot_pv = a.spv.as<double>();
    sa.slot_pg = a.spg.as<double>();
    sa.lpv = a.lpv.as<double>();
    sa.dt = in_.dt;
    sa.re_inv = in_.reyn_inv;
    sa.adv_type = in_.adv_type;
    HO2D_CUDA(launch_residual_adjoint<double>(K, g, d.b64, sa, d.stream), "residual adjoint");
    HO2D_CUDA(launch_velocity_adjoint<double>(K, g, d.b64, sa, d.stream), "velocity adjoint");
    HO2D_CUDA(launch_gather<double>(K, N, d.b64, a.lpsi_dir.as<double>(), a.spv.as<double>(), a.spg.as<double>(),
                                    a.lpsi.as<double>(), nullptr, 0, d.stream),
              "psi gather");
    launches_ += 3;
    // psi = A^-1 (-J omega - boundary terms): lam of omega -= J A^-T lam of psi
    HO2D_TRY(transposed_solve(a.lpsi.as<double>(), a.mu.as<double>()));
    HO2D_CUDA(launch_sub_scaled(nv, out, a.lw_stage.as<double>(), d.m64[4].as<double>(), a.mu.as<double>(), d.stream),
              "combine");
    launches_ += 1;
    return {0, ""};
}

// Advection types 1 and 2 (residual_adjoint_continuous for type 2); both are checked on the
// host and on the GPU against complex-step derivatives of the oracle. Every precision: with
// the FP32 stage (HO2D_MIXED) the forward sweep and the segment recomputation follow the
// mixed trajectory, and each stage is linearised in FP64 at its states.
static Error adjoint_supported(const Input& in) {
    if (in.adv_type != 1 && in.adv_type != 2) return {4, "the adjoint covers advection types 1 and 2"};
    if (in.problem_type == 11) return {4, "the adjoint does not cover hybrid runs (problem type 11)"};
    return {0, ""};
}

Error Solver::stage_adjoint(double coeff, const double* lam_k, double* lam_w, double* lam_pv) {
    HO2D_TRY(adjoint_supported(in_));
    HO2D_TRY(adjoint_prepare());
    DeviceState& d = *d_;
    AdjointState& a = *adj_;
    const size_t nv = (size_t)mesh_.n_el * in_.knod * in_.knod, nb = (size_t)mesh_.n_eb * in_.knod;
    if (stage32_) {  // the FP32 stage input kept, and widened in place for the FP64 stage
        if (a.w32_save.bytes() < nv * 4) HO2D_CUDA(a.w32_save.alloc(nv * 4), "alloc");
        HO2D_CUDA(cudaMemcpyAsync(a.w32_save.get(), d.w_stage.get(), nv * 4, cudaMemcpyDeviceToDevice, d.stream),
                  "copy");
        HO2D_CUDA(launch_copy_f2d(a.w32_save.as<float>(), d.w_stage.as<double>(), nv, d.stream), "f2d");
    }
    HO2D_TRY(stage_t<double>(coeff, 0, false, true));  // the stage at the current state: psi of this input
    HO2D_CUDA(cudaMemcpyAsync(a.lam_k.get(), lam_k, nv * 8, cudaMemcpyHostToDevice, d.stream), "copy");
    HO2D_CUDA(cudaMemsetAsync(a.lpv.get(), 0, a.lpv.bytes(), d.stream), "memset");
    HO2D_TRY(stage_adjoint_dev(coeff, a.lw_out.as<double>()));
    HO2D_CUDA(cudaMemcpyAsync(lam_w, a.lw_out.get(), nv * 8, cudaMemcpyDeviceToHost, d.stream), "copy");
    if (lam_pv && nb) HO2D_CUDA(cudaMemcpyAsync(lam_pv, a.lpv.get(), nb * 8, cudaMemcpyDeviceToHost, d.stream), "copy");
    if (stage32_)  // the FP32 stage input back
        HO2D_CUDA(cudaMemcpyAsync(d.w_stage.get(), a.w32_save.get(), nv * 4, cudaMemcpyDeviceToDevice, d.stream),
                  "copy");
    HO2D_CUDA(cudaStreamSynchronize(d.stream), "stage adjoint");
    return {0, ""};
}

Error Solver::apply_poisson_transpose(const double* x, double* y) {
    HO2D_TRY(adjoint_prepare());
    DeviceState& d = *d_;
    AdjointState& a = *adj_;
    const size_t nv = (size_t)mesh_.n_el * in_.knod * in_.knod;
    HO2D_CUDA(cudaMemcpyAsync(a.lpsi.get(), x, nv * 8, cudaMemcpyHostToDevice, d.stream), "copy");
    HO2D_CUDA(cudaMemsetAsync(a.sv.get(), 0, a.sv.bytes(), d.stream), "memset");  // shared with FP32
    HO2D_CUDA(cudaMemsetAsync(a.sg.get(), 0, a.sg.bytes(), d.stream), "memset");
    const FrGeom<double> g = geom_of<double>(d, mesh_, false);
    HO2D_CUDA(poisson_transpose<double>(in_.knod, g, d.b64, a.lpsi.as<double>(), a.mu.as<double>(),
                                        a.kv[8].as<double>(), a.sv.as<double>(), a.sg.as<double>(), nullptr, 0,
                                        d.stream),
              "transposed operator");
    launches_ += 2;
    HO2D_CUDA(cudaMemcpyAsync(y, a.mu.get(), nv * 8, cudaMemcpyDeviceToHost, d.stream), "copy");
    HO2D_CUDA(cudaStreamSynchronize(d.stream), "apply transpose");
    return {0, ""};
}

// One stored FP64 field of the time loop (checkpoint, segment stage input or psi), kept in
// FP64 or, with FP32 state storage, rounded to FP32.
Error Solver::store_state(void* dst, const double* src) {
    DeviceState& d = *d_;
    const size_t nv = (size_t)mesh_.n_el * in_.knod * in_.knod;
    if (adj_->state_bytes == 4) HO2D_CUDA(launch_copy_d2f(src, static_cast<float*>(dst), nv, d.stream), "store state");
    else HO2D_CUDA(cudaMemcpyAsync(dst, src, nv * 8, cudaMemcpyDeviceToDevice, d.stream), "store state");
    return {0, ""};
}

Error Solver::load_state(double* dst, const void* src) {
    DeviceState& d = *d_;
    const size_t nv = (size_t)mesh_.n_el * in_.knod * in_.knod;
    if (adj_->state_bytes == 4) HO2D_CUDA(launch_copy_f2d(static_cast<const float*>(src), dst, nv, d.stream), "load state");
    else HO2D_CUDA(cudaMemcpyAsync(dst, src, nv * 8, cudaMemcpyDeviceToDevice, d.stream), "load state");
    return {0, ""};
}

// The stage input d.w_stage from omega, in the stage precision (FP32 under HO2D_MIXED).
static cudaError_t stage_input_from(const DeviceState& d, bool stage32, const double* w, size_t nv) {
    if (stage32) return launch_copy_d2f(w, d.w_stage.as<float>(), nv, d.stream);
    return cudaMemcpyAsync(d.w_stage.get(), w, nv * 8, cudaMemcpyDeviceToDevice, d.stream);
}

Error Solver::adjoint_forward(int nsteps, int ckpt_every) {
    const NvtxRange nvtx_range("ho2d.adjoint_forward");
    HO2D_TRY(adjoint_supported(in_));
    if (nsteps < 0 || ckpt_every < 1) return {1, "adjoint_forward needs nsteps >= 0 and ckpt_every >= 1"};
    HO2D_TRY(adjoint_prepare());
    DeviceState& d = *d_;
    AdjointState& a = *adj_;
    const size_t nv = (size_t)mesh_.n_el * in_.knod * in_.knod;
    const int nck = (nsteps + ckpt_every - 1) / ckpt_every;
    const size_t wb = adj_state32_ ? 4 : 8;  // bytes per stored value
    if (a.state_bytes != wb) {
        a.ckpt.clear();
        a.seg_w.reset();
        a.seg_psi.reset();
        a.state_bytes = wb;
    }
    while ((int)a.ckpt.size() < nck) {
        std::unique_ptr<DeviceBuffer> b(new DeviceBuffer);
        HO2D_CUDA(b->alloc(nv * wb), "alloc checkpoint");
        a.ckpt.push_back(std::move(b));
    }
    a.nsteps = -1;  // valid again once the sweep completes
    a.t0 = time_;
    a.every = ckpt_every;
    // the stage input of a step is omega itself
    HO2D_CUDA(stage_input_from(d, stage32_, d.omega.as<double>(), nv), "copy");
    for (int n = 0; n < nsteps; ++n) {
        if (n % ckpt_every == 0) HO2D_TRY(store_state(a.ckpt[n / ckpt_every]->get(), d.omega.as<double>()));
        HO2D_TRY(step(1));
    }
    HO2D_CUDA(cudaMemcpyAsync(a.wT.get(), d.omega.get(), nv * 8, cudaMemcpyDeviceToDevice, d.stream), "copy");
    HO2D_CUDA(cudaMemcpyAsync(a.psiT.get(), d.psi64.get(), nv * 8, cudaMemcpyDeviceToDevice, d.stream), "copy");
    HO2D_CUDA(cudaStreamSynchronize(d.stream), "adjoint forward");
    a.nsteps = nsteps;
    return {0, ""};
}

Error Solver::adjoint_backward(const double* dJ_dw, double* grad_w0, double* grad_pv) {
    const NvtxRange nvtx_range("ho2d.adjoint_backward");
    HO2D_TRY(adjoint_supported(in_));
    if (!adj_ || adj_->nsteps < 0) return {1, "ho2d_adjoint_backward needs a completed ho2d_adjoint_forward"};
    HO2D_TRY(adjoint_prepare());
    DeviceState& d = *d_;
    AdjointState& a = *adj_;
    HO2D_CUDA(cudaSetDevice(d.device), "cudaSetDevice");
    const size_t nv = (size_t)mesh_.n_el * in_.knod * in_.knod, nb = (size_t)mesh_.n_eb * in_.knod;
    const Tableau tb = tableau(in_.ti_type);
    const int ns = tb.ns, every = a.every, nsteps = a.nsteps;
    const size_t wb = a.state_bytes;
    const size_t seg_bytes = (size_t)every * ns * nv * wb;
    if (a.seg_w.bytes() < seg_bytes) {
        HO2D_CUDA(a.seg_w.alloc(seg_bytes), "alloc segment");
        HO2D_CUDA(a.seg_psi.alloc(seg_bytes), "alloc segment");
    }
    char* seg_w = static_cast<char*>(a.seg_w.get());
    char* seg_psi = static_cast<char*>(a.seg_psi.get());
    double* lam = a.lam.as<double>();
    double* lk = a.lam_k.as<double>();
    auto copy = [&](void* dst, const void* src) -> Error {
        HO2D_CUDA(cudaMemcpyAsync(dst, src, nv * 8, cudaMemcpyDeviceToDevice, d.stream), "copy");
        return {0, ""};
    };
    HO2D_CUDA(cudaMemcpyAsync(lam, dJ_dw, nv * 8, cudaMemcpyHostToDevice, d.stream), "copy");
    HO2D_CUDA(cudaMemsetAsync(a.lpv.get(), 0, a.lpv.bytes(), d.stream), "memset");
    const int nseg = (nsteps + every - 1) / every;
    for (int seg = nseg - 1; seg >= 0; --seg) {
        const int n0 = seg * every, n1 = std::min(nsteps, n0 + every);
        // recompute the segment from its checkpoint, keeping every stage input and psi; the
        // stages are the FP64 ones the adjoint linearises (under HO2D_MIXED the checkpoints
        // come from the FP32-stage trajectory and each segment is recomputed in FP64 from them)
        HO2D_TRY(load_state(d.omega.as<double>(), a.ckpt[seg]->get()));
        HO2D_TRY(copy(d.w_stage.get(), d.omega.get()));
        for (int n = n0; n < n1; ++n) {
            time_ = a.t0 + n * in_.dt;
            for (int s = 0; s < ns; ++s) {
                const size_t off = ((size_t)(n - n0) * ns + s) * nv * wb;
                HO2D_TRY(store_state(seg_w + off, d.w_stage.as<double>()));
                HO2D_TRY(stage_t<double>(tb.c[s], s, true));
                HO2D_TRY(store_state(seg_psi + off, d.psi64.as<double>()));
            }
        }
        // reverse sweep: lam_k_s = b_s lam + sum_{r > s} a_rs mu_r, lam += sum_s mu_s
        for (int n = n1 - 1; n >= n0; --n) {
            for (int s = ns - 1; s >= 0; --s) {
                const size_t off = ((size_t)(n - n0) * ns + s) * nv * wb;
                HO2D_CUDA(launch_axpby(nv, lk, tb.b[s], lam, 0.0, lam, d.stream), "lam_k");
                for (int r = s + 1; r < ns; ++r)
                    if (tb.a[r][s] != 0.0) HO2D_CUDA(launch_axpby(nv, lk, 1.0, lk, tb.a[r][s], a.mus[r].as<double>(), d.stream), "lam_k");
                HO2D_TRY(load_state(d.w_stage.as<double>(), seg_w + off));
                HO2D_TRY(load_state(d.psi64.as<double>(), seg_psi + off));
                time_ = a.t0 + n * in_.dt;
                HO2D_TRY(stage_adjoint_dev(tb.c[s], a.mus[s].as<double>()));
            }
            for (int s = 0; s < ns; ++s) HO2D_CUDA(launch_axpby(nv, lam, 1.0, lam, 1.0, a.mus[s].as<double>(), d.stream), "lam");
            launches_ += 2 * ns + 1;
        }
    }
    HO2D_CUDA(cudaMemcpyAsync(grad_w0, lam, nv * 8, cudaMemcpyDeviceToHost, d.stream), "copy");
    if (grad_pv && nb) HO2D_CUDA(cudaMemcpyAsync(grad_pv, a.lpv.get(), nb * 8, cudaMemcpyDeviceToHost, d.stream), "copy");
    // back to the state at T
    HO2D_TRY(copy(d.omega.get(), a.wT.get()));
    HO2D_CUDA(stage_input_from(d, stage32_, a.wT.as<double>(), nv), "copy");
    HO2D_TRY(copy(d.psi64.get(), a.psiT.get()));
    time_ = a.t0 + nsteps * in_.dt;
    HO2D_CUDA(cudaStreamSynchronize(d.stream), "adjoint backward");
    return {0, ""};
}

template Error Solver::kt_run<double>(double*, const double*, bool, double, int&);
template Error Solver::kt_run<float>(float*, const float*, bool, double, int&);

}  // namespace ho2d
