// solver.cu -- device state and the stage / step / Poisson drivers.
//
// One stage (src/HO_2D.cpp:1806-1839) on the device:
//   bc_update      update_BCs(t + c dt)                     (1979-2217)
//   poisson_rhs    RHS of solve_Poisson                    (1881-1900)
//   Krylov solve   replaces (*AMGCL_solver)(RHS, x)         (1960), warm start = last psi
//   trace + velocity   calc_velocity_vector_from_streamfunction + update_diffusion_BC
//   residual       calc_RHS_diffusion + update_advection_BC + calc_RHS_advection[_continuous]
//                  + k = dt (adv + diff) + the RK combination of solve_advection_diffusion
// Nothing crosses PCIe inside a step except the Krylov convergence flag polled by the host.
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <type_traits>

#include "device.cuh"
#include "fr_launch.hpp"
#include "host_amg.hpp"
#include "noalloc.hpp"
#include "solver.hpp"
#include "solver_state.hpp"
#include "adjoint_launch.hpp"

namespace ho2d {

// Every buffer gets 16 bytes past its end: a bulk copy that rounds a span's end up to the
// next 16-byte boundary (apply_stage.cuh) stays inside the allocation.
cudaError_t DeviceBuffer::alloc(size_t bytes) {
    reset();
    if (bytes == 0) return cudaSuccess;
    cudaError_t e = cudaMalloc(&p_, bytes + 16);
    if (e == cudaSuccess) n_ = bytes;
    else p_ = nullptr;
    return e;
}

void DeviceBuffer::reset() {
    if (p_) cudaFree(p_);
    p_ = nullptr;
    n_ = 0;
}


Solver::Solver() : d_(new DeviceState) {
    const char* pe = std::getenv("HO2D_PSI_EXTRAP");
    if (pe) psi_extrap_ = std::atoi(pe);
    const char* os = std::getenv("HO2D_OP_STAGE");
    if (os && os[0]) d_->op_staged = std::atoi(os) != 0;
    const char* v = std::getenv("HO2D_VERBOSE");
    verbose_ = v && v[0] && v[0] != '0';
    const char* g = std::getenv("HO2D_GRAPHS");
    use_graphs_ = !(g && g[0] == '0');
    const char* it = std::getenv("HO2D_INNER_TOL");
    if (it && std::atof(it) > 0.0 && std::atof(it) < 1.0) inner_tol_ = std::atof(it);
    const char* ms = std::getenv("HO2D_MAX_SWEEPS");
    if (ms && std::atoi(ms) >= 1) max_sweeps_ = std::atoi(ms);
}
Solver::~Solver() = default;

Error Solver::cuda(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return {0, ""};
    return {5, std::string(what) + ": " + cudaGetErrorString(e)};
}


Error Solver::read_input(const std::string& path) {
    Input in;
    Error e = ho2d::read_input(path, in);
    if (e.code) return e;
    in_ = in;
    input_done_ = true;
    setup_done_ = false;
    return {0, ""};
}

Error Solver::setup() {
    const NvtxRange nvtx_range("ho2d.setup");
    if (!input_done_) return {1, "ho2d_setup called before ho2d_read_input"};
    vtk_queue_.wait();  // a dump still being written reads the mesh replaced here
    std::string mesh_path = in_.mesh_file;
    if (!mesh_path.empty() && mesh_path[0] != '/') mesh_path = in_.base_dir + "/" + mesh_path;
    mesh_ = Mesh();
    HO2D_TRY(read_msh(mesh_path, in_.occ, mesh_));
    // read_process_sample_points (src/main.cpp:65): the file name is taken relative to the
    // input's directory, like the mesh file
    std::string sample_path = in_.sample_file;
    if (!sample_path.empty() && sample_path[0] != '/') sample_path = in_.base_dir + "/" + sample_path;
    HO2D_TRY(read_sample_points(sample_path, mesh_, samples_));
    return setup_from_mesh();
}

// Everything after the mesh (src/main.cpp:55-75, or process_mesh_input for a mesh loaded
// from arrays): bases, metrics, BCs, the Poisson operator and its preconditioner, and the
// device state.
Error Solver::setup_from_mesh() {
    setup_done_ = false;
    adj_.reset();
    HO2D_TRY(make_bases(in_.knod, mesh_.lnod, B_));
    make_metrics(mesh_, B_, M_);
    for (double j : M_.J)
        if (!(j > 0.0)) return {3, "non-positive element Jacobian: check the element orientation"};
    HO2D_TRY(setup_bcs(in_, mesh_, B_, bc_));
    // smoother of the FP32 preconditioner: the requested kind, else the environment
    // (HO2D_SMOOTHER_KRON=1, HO2D_SMOOTHER_BF16=1), else exact FP32 blocks
    smoother_kind_ = smoother_req_;
    if (smoother_kind_ < 0) {
        auto on = [](const char* nm) {
            const char* e = std::getenv(nm);
            return e && std::string(e) == "1";
        };
        smoother_kind_ = on("HO2D_SMOOTHER_KRON") ? 2 : (on("HO2D_SMOOTHER_BF16") ? 1 : 0);
    }
    // the Poisson operator: assembled on the device unless the host is asked for
    // (set_device_setup(false) or HO2D_HOST_SETUP=1); smoother kind 2 adds the Kronecker-sum
    // fit of every diagonal block
    device_setup_ = device_setup_req_ >= 0 ? device_setup_req_ == 1 : [] {
        const char* e = std::getenv("HO2D_HOST_SETUP");
        return !(e && std::string(e) == "1");
    }();
    kron_ = KronSmoother();
    if (!device_setup_) assemble_poisson(mesh_, B_, M_, bc_, op_, false, smoother_kind_ == 2 ? &kron_ : nullptr);

    DeviceState& d = *d_;
    HO2D_CUDA(cudaGetDevice(&d.device), "cudaGetDevice");
    if (!d.stream) HO2D_CUDA(cudaStreamCreateWithFlags(&d.stream, cudaStreamNonBlocking), "cudaStreamCreate");
    if (!d.side) {
        // the coarse cycle's stream at the highest priority: its short dependent kernels get
        // SM slots ahead of the wide fine-smoothing kernel they run beside, which has slack
        int lo = 0, hi = 0;
        HO2D_CUDA(cudaDeviceGetStreamPriorityRange(&lo, &hi), "cudaDeviceGetStreamPriorityRange");
        HO2D_CUDA(cudaStreamCreateWithPriority(&d.side, cudaStreamNonBlocking, hi), "cudaStreamCreate");
    }
    for (cudaEvent_t* e : {&d.ev_fork, &d.ev_join})
        if (!*e) HO2D_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming), "cudaEventCreate");
    for (cudaEvent_t* e : {&d.ev0, &d.ev1, &d.evp0, &d.evp1})
        if (!*e) HO2D_CUDA(cudaEventCreate(e), "cudaEventCreate");
    if (!d.h_sc) HO2D_CUDA(cudaMallocHost(&d.h_sc, sizeof(KrylovScalars)), "cudaMallocHost");
    HO2D_TRY(noalloc_scratch(d.device, &d.noalloc_scratch));  // once per device, this device current
    HO2D_CUDA(krylov_configure(in_.knod), "kernel set-up");

    const int N = mesh_.n_el, K = in_.knod, K2 = K * K, neb = mesh_.n_eb;
    const size_t nv = (size_t)N * K2, nf = (size_t)N * 4 * K;
    // connectivity in ijp order
    std::vector<int> fnb((size_t)N * 4), fnijp((size_t)N * 4), beijp(neb);
    for (int el = 0; el < N; ++el)
        for (int ijp = 0; ijp < 4; ++ijp) {
            const int side = kI2F[ijp];
            const int nb = mesh_.nbr[(size_t)el * 4 + side];
            if (nb >= 0) {
                fnb[(size_t)el * 4 + ijp] = nb;
                fnijp[(size_t)el * 4 + ijp] = kF2I[mesh_.nbr_side[(size_t)el * 4 + side]];
            } else {
                fnb[(size_t)el * 4 + ijp] = -(mesh_.bidx[(size_t)el * 4 + side] + 1);
                fnijp[(size_t)el * 4 + ijp] = -1;
            }
        }
    for (int e = 0; e < neb; ++e) beijp[e] = kF2I[mesh_.be_side[e]];
    HO2D_CUDA(upload(d.face_nb, fnb), "upload");
    HO2D_CUDA(upload(d.face_nijp, fnijp), "upload");
    HO2D_CUDA(upload(d.be_group, mesh_.be_group), "upload");
    HO2D_CUDA(upload(d.sw_p, bc_.sw_p), "upload");
    HO2D_CUDA(upload(d.sw_d, bc_.sw_d), "upload");
    HO2D_CUDA(upload(d.noslip, bc_.noslip.empty() ? std::vector<int>{0} : bc_.noslip), "upload");
    HO2D_CUDA(upload(d.role, bc_.role), "upload");
    HO2D_CUDA(upload(d.be_ijp, beijp), "upload");
    d.b64 = make_dev_bases<double>(B_);
    d.b32 = make_dev_bases<float>(B_);
    const std::vector<double>* mets[9] = {&M_.xxi, &M_.xeta, &M_.yxi, &M_.yeta, &M_.J, &M_.fA, &M_.fB, &M_.fJ, &M_.fAn};
    for (int i = 0; i < 9; ++i) HO2D_CUDA(upload(d.m64[i], *mets[i]), "upload metrics");
    d.have32 = false;
    HO2D_CUDA(upload(d.bc_p, bc_.bc_p), "upload");
    HO2D_CUDA(upload(d.bc_nv, bc_.bc_nv), "upload");
    HO2D_CUDA(upload(d.bc_pv, bc_.bc_pv), "upload");
    HO2D_CUDA(upload(d.bc_d, bc_.bc_d), "upload");
    HO2D_CUDA(upload(d.edge_y, bc_.edge_y), "upload");
    const std::vector<double> zb((size_t)neb * K, 0.0);
    HO2D_CUDA(upload(d.bc_w, zb), "upload");
    HO2D_CUDA(upload(d.vjump, zb), "upload");
    HO2D_CUDA(upload(d.bc_adv, zb), "upload");
    // fields (typed fields sized for double so either precision fits)
    const std::vector<double> zv(nv, 0.0);
    for (DeviceBuffer* b : {&d.omega, &d.acc, &d.psi64, &d.rhs, &d.rres, &d.w_stage, &d.psiT, &d.u, &d.v, &d.rhs_diff,
                            &d.rhs_adv, &d.kout, &d.w_stage64})
        HO2D_CUDA(upload(*b, zv), "alloc fields");
    const std::vector<double> zf(nf, 0.0);
    for (DeviceBuffer* b : {&d.psi_tv, &d.psi_tg, &d.w_tv, &d.w_tg, &d.U_t}) HO2D_CUDA(upload(*b, zf), "alloc traces");
    // Poisson operator: the inverse diagonal blocks and the row sums of every block (the
    // two-level smoother's A e for element-wise constant e), from assemble_poisson
    // every element's block starts on a 16-byte boundary (padded_count): the smoothing
    // kernel stages blocks with bulk copies
    const int K4 = K2 * K2;
    d.vtk.ready = false;  // the VTK node tables follow the mesh
    d.colsum64.reset();
    kron_on_device_ = false;
    if (device_setup_) {
        // kind 2: the Kronecker-sum fit on the device from the assembled diagonal blocks
        HO2D_TRY(assemble_device(smoother_kind_ == 2));
    } else {
        HO2D_CUDA(upload(d.bsrc, op_.bsrc.empty() ? std::vector<double>{0.0} : op_.bsrc), "upload");
        HO2D_CUDA(upload(d.dinv64, padded_rows<double>(op_.dinv, N, K4, padded_count(K4, 8))), "upload block-Jacobi");
        HO2D_CUDA(upload(d.rowsum64, op_.rowsum), "upload block row sums");
        HO2D_CUDA(upload(d.bcol, op_.block_col), "upload block columns");
    }
    smoother_exact_ = 0;
    for (unsigned char x : kron_.exact) smoother_exact_ += x ? 1 : 0;
    HO2D_CUDA(d.W64.alloc((size_t)N * 5 * K2 * sizeof(double)), "alloc smoothed row sums");
    HO2D_CUDA(d.W32.alloc((size_t)N * 5 * K2 * sizeof(float)), "alloc smoothed row sums");
    HO2D_CUDA(d.zf.alloc((size_t)N * K2 * sizeof(double)), "alloc smoother vector");
    {
        // where the coarse cycle delivers each element's level-0 value: every block slot
        // (el, s) with block_col[5 el + s] = c reads u0 of element c
        std::vector<int> dst((size_t)N * 5, -1), cnt(N, 0);
        for (int el = 0; el < N; ++el)
            for (int sl = 0; sl < 5; ++sl) {
                const int c = op_.block_col[(size_t)el * 5 + sl];
                if (c < 0) continue;
                if (cnt[c] >= 5) return {3, "an element is a block neighbour of more than four elements"};
                dst[(size_t)c * 5 + cnt[c]++] = el * 5 + sl;
            }
        HO2D_CUDA(upload(d.u0dst, dst), "upload coarse slot table");
        HO2D_CUDA(upload(d.ue5, std::vector<double>((size_t)N * 5, 0.0)), "alloc coarse slot values");
        HO2D_CUDA(upload(d.ue5_32, std::vector<float>((size_t)N * 5, 0.f)), "alloc coarse slot values");
    }
    HO2D_TRY(build_poisson_geometry(fnb, fnijp));
    HO2D_TRY(setup_forces());
    for (DeviceBuffer* b : {&d.ktv, &d.ktg, &d.kxtv, &d.kxtg}) HO2D_CUDA(upload(*b, zf), "alloc Krylov traces");
    d.dinv32.reset();
    d.dinv_bf16.reset();
    for (DeviceBuffer* b : {&d.kron_x, &d.kron_exact}) b->reset();
    if (!kron_on_device_) d.kron_f.reset();
    d.rowsum32.reset();
    for (auto& b : d.pg32) b.reset();
    HO2D_TRY(setup_preconditioner());
    for (auto& b : d.kv) HO2D_CUDA(upload(b, zv), "alloc Krylov");
    for (auto& b : d.esum) HO2D_CUDA(upload(b, std::vector<double>((size_t)N + 4, 0.0)), "alloc element sums");
    const int mb = krylov_max_blocks(K, N);
    HO2D_CUDA(upload(d.partials, std::vector<double>((size_t)4 * mb, 0.0)), "alloc partials");
    // the grid reductions' counters: one for the groups of 64 CTAs, one per group
    HO2D_CUDA(upload(d.counter, std::vector<unsigned>(2 + mb / 64, 0u)), "alloc counter");
    HO2D_CUDA(d.scalars.alloc(sizeof(KrylovScalars)), "alloc scalars");
    HO2D_CUDA(cudaMemset(d.scalars.get(), 0, sizeof(KrylovScalars)), "memset");
    // the FP64 smoother applied to the block row sums (the split smoothing step)
    HO2D_CUDA(krylov_make_w<double>(make_op<double>(d, mesh_, K, false), d.W64.as<double>(),
                                    d.scalars.as<KrylovScalars>(), d.stream),
              "smoothed row sums");
    time_ = 0.0;
    t_start_ = t_end_ = 0.0;
    hist_count_ = 0;
    if (in_.problem_type == 11) HO2D_TRY(hybrid_upload());
    setup_done_ = true;
    if (stage32_ || krylov32_) HO2D_TRY(upload_precision_arrays());
    HO2D_CUDA(cudaDeviceSynchronize(), "setup");
    return {0, ""};
}

// Static data of the matrix-free Poisson operator (PoisGeom in fr_launch.hpp): metric and
// face coefficients with the divisions by J and J_f done here, the neighbour's face
// coefficients gathered into this element's rows, face codes, the inverted K x K
// common-value system of every Neumann edge, and the trace scatter table.
Error Solver::build_poisson_geometry(const std::vector<int>& fnb, const std::vector<int>& fnijp) {
    DeviceState& d = *d_;
    const int N = mesh_.n_el, K = in_.knod, K2 = K * K, NF = 4 * K, neb = mesh_.n_eb;
    const size_t nv = (size_t)N * K2, nf = (size_t)N * NF;
    std::vector<double>* h = d.pg_host;
    for (int a = 0; a < 3; ++a) h[a].assign(nv, 0.0);
    for (int a = 3; a < 7; ++a) h[a].assign(nf, 0.0);
    h[7].assign((size_t)std::max(1, neb) * K * K, 0.0);
    for (size_t p = 0; p < nv; ++p) {
        const double xx = M_.xxi[p], xe = M_.xeta[p], yx = M_.yxi[p], ye = M_.yeta[p], J = M_.J[p];
        h[0][p] = (xe * xe + ye * ye) / J;
        h[1][p] = -(xx * xe + yx * ye) / J;
        h[2][p] = (xx * xx + yx * yx) / J;
    }
    for (size_t q = 0; q < nf; ++q) {
        h[3][q] = M_.fA[q] / M_.fJ[q];
        h[4][q] = M_.fB[q] / M_.fJ[q];
    }
    std::vector<int> code((size_t)N * 4), scat(nf, -1);
    for (int el = 0; el < N; ++el)
        for (int ijp = 0; ijp < 4; ++ijp) {
            const int nb = fnb[(size_t)el * 4 + ijp];
            if (nb >= 0) {
                const int nijp = fnijp[(size_t)el * 4 + ijp];
                const int rev = (ijp + nijp - ijp / 2 - nijp / 2 + 1) % 2;
                code[(size_t)el * 4 + ijp] = nijp + 4 * rev;
                for (int k = 0; k < K; ++k) {
                    const size_t q = ((size_t)el * 4 + ijp) * K + k;
                    const size_t nq = ((size_t)nb * 4 + nijp) * K + (rev ? K - 1 - k : k);
                    h[5][q] = h[3][nq];
                    h[6][q] = h[4][nq];
                    scat[nq] = (int)q;  // the neighbour's point feeds this element's slot
                }
                continue;
            }
            const int e = -nb - 1;
            code[(size_t)el * 4 + ijp] = bc_.sw_p[e] == kNeumann ? -2 - e : -1;
            // the inverse serves the operator (Neumann psi) and the stage kernels (Neumann
            // psi or vorticity): the system depends on the face geometry only
            if (bc_.sw_p[e] != kNeumann && bc_.sw_d[e] != kNeumann) continue;
            // M[k][c] = -fb_k l_c'(x_k) + fa_k g'(+-1) delta_kc (rows scaled by 1/J_f)
            const int lr = ijp & 1;
            std::vector<double> A((size_t)K * K), I((size_t)K * K, 0.0);
            for (int k = 0; k < K; ++k) {
                const size_t q = ((size_t)el * 4 + ijp) * K + k;
                for (int c = 0; c < K; ++c) A[(size_t)k * K + c] = -h[4][q] * B_.D[(size_t)c * K + k];
                A[(size_t)k * K + k] += h[3][q] * B_.gp[lr];
                I[(size_t)k * K + k] = 1.0;
            }
            for (int c = 0; c < K; ++c) {  // Gauss-Jordan with partial pivoting
                int piv = c;
                for (int r = c + 1; r < K; ++r)
                    if (std::fabs(A[(size_t)r * K + c]) > std::fabs(A[(size_t)piv * K + c])) piv = r;
                if (A[(size_t)piv * K + c] == 0.0) return {3, "singular Neumann common-value system"};
                for (int m = 0; m < K; ++m) {
                    std::swap(A[(size_t)c * K + m], A[(size_t)piv * K + m]);
                    std::swap(I[(size_t)c * K + m], I[(size_t)piv * K + m]);
                }
                const double inv = 1.0 / A[(size_t)c * K + c];
                for (int m = 0; m < K; ++m) {
                    A[(size_t)c * K + m] *= inv;
                    I[(size_t)c * K + m] *= inv;
                }
                for (int r = 0; r < K; ++r) {
                    if (r == c) continue;
                    const double f = A[(size_t)r * K + c];
                    for (int m = 0; m < K; ++m) {
                        A[(size_t)r * K + m] -= f * A[(size_t)c * K + m];
                        I[(size_t)r * K + m] -= f * I[(size_t)c * K + m];
                    }
                }
            }
            std::copy(I.begin(), I.end(), h[7].begin() + (size_t)e * K * K);
        }
    // device layout of the face data and of the trace slots: [N][K][4], the four faces of
    // one face-point index together, so the thread that owns face point k of every face
    // (row-parallel operator) reads them as one vector
    auto perm = [K, NF](size_t q) {
        const size_t el = q / NF, r = q % NF;
        return (el * K + r % K) * 4 + r / K;
    };
    for (int a = 3; a < 7; ++a) {
        std::vector<double> t(nf);
        for (size_t q = 0; q < nf; ++q) t[perm(q)] = h[a][q];
        h[a].swap(t);
    }
    std::vector<int> scat_p(nf, -1);
    for (size_t q = 0; q < nf; ++q)
        if (scat[q] >= 0) scat_p[perm(q)] = (int)perm((size_t)scat[q]);
    for (int a = 0; a < 8; ++a) HO2D_CUDA(upload(d.pg64[a], h[a]), "upload Poisson operator data");
    HO2D_CUDA(upload(d.pcode, code), "upload Poisson face codes");
    HO2D_CUDA(upload(d.pscat, scat_p), "upload trace scatter table");
    return {0, ""};
}

// Per boundary point of the group "object": the coefficients of the body force
// (forces.cu) F = sum (cdx, cdy) dw/dn_stored + (cwx, cwy) w_wall, where
//   cdx = nu w_k |g| sigma y,  cdy = -nu w_k |g| sigma x,  cwx = nu w_k |g| t_x,  cwy = nu w_k |g| t_y,
// (x, y) the point, |g| the face length per unit of the face coordinate, w_k the Gauss
// weight, t = z x n with n the inward normal of the element (from the body into the
// fluid), and sigma = +1 on W/S faces, -1 on E/N faces: the stored normal derivative is
// taken towards the +xi / +eta side of the face (the element interior on W/S faces).
Error Solver::setup_forces() {
    DeviceState& d = *d_;
    force_points_ = 0;
    int grp = -1;
    for (size_t g = 0; g < mesh_.group_names.size(); ++g)
        if (mesh_.group_names[g] == "object") grp = (int)g;
    if (grp < 0) return {0, ""};
    const int K = in_.knod, L = mesh_.lnod, lin = L - 1;
    const double nu = in_.reyn_inv;
    std::vector<double> coef;
    std::vector<int> idx;
    for (int e = 0; e < mesh_.n_eb; ++e) {
        if (mesh_.be_group[e] != grp) continue;
        const int el = mesh_.be_el[e], side = mesh_.be_side[e], ijp = kF2I[side];
        const int dd = ijp / 2, t = ijp % 2;
        const double sigma = (ijp % 2 == 0) ? 1.0 : -1.0;
        const double tsign = (ijp == 1 || ijp == 2) ? 1.0 : -1.0;  // counter-clockwise traversal
        for (int k = 0; k < K; ++k) {
            double x = 0, y = 0, dx = 0, dy = 0;  // position and derivative along the face
            for (int j = 0; j < L; ++j)
                for (int i = 0; i < L; ++i) {
                    const int nd = mesh_.elem_nodes[el][tensor2fem(i, j, lin)];
                    const double X = mesh_.node_xy[2 * nd], Y = mesh_.node_xy[2 * nd + 1];
                    double w0, w1;
                    if (dd == 0) {  // W/E face: xi = -+1, eta = x_k
                        w0 = B_.gbb[i * 2 + t] * B_.gsb[j * K + k];
                        w1 = B_.gbb[i * 2 + t] * B_.gsgb[j * K + k];
                    } else {  // S/N face: eta = -+1, xi = x_k
                        w0 = B_.gsb[i * K + k] * B_.gbb[j * 2 + t];
                        w1 = B_.gsgb[i * K + k] * B_.gbb[j * 2 + t];
                    }
                    x += w0 * X;
                    y += w0 * Y;
                    dx += w1 * X;
                    dy += w1 * Y;
                }
            const double len = std::sqrt(dx * dx + dy * dy);
            const double tcx = tsign * dx / len, tcy = tsign * dy / len;  // element's ccw tangent
            const double tx = -tcx, ty = -tcy;                            // t = z x n = -t_ccw
            const double ds = nu * B_.w[k] * len;
            coef.insert(coef.end(), {ds * sigma * y, -ds * sigma * x, ds * tx, ds * ty});
            idx.push_back(e * K + (side / 2) * (K - 2 * k - 1) + k);
        }
    }
    force_points_ = (int)idx.size();
    HO2D_CUDA(upload(d.fcoef, coef), "upload force coefficients");
    HO2D_CUDA(upload(d.fidx, idx), "upload force indices");
    HO2D_CUDA(d.fout.alloc(2 * sizeof(double)), "alloc force result");
    return {0, ""};
}

Error Solver::get_forces(double* fx, double* fy) {
    if (!setup_done_) return {1, "not set up"};
    if (force_points_ == 0) return {1, "the mesh has no boundary group named \"object\""};
    DeviceState& d = *d_;
    HO2D_CUDA(cudaSetDevice(d.device), "cudaSetDevice");
    HO2D_CUDA(launch_body_force(force_points_, d.fcoef.as<double>(), d.fidx.as<int>(), d.bc_d.as<double>(),
                                d.bc_w.as<double>(), d.fout.as<double>(), d.stream),
              "body force");
    launches_ += 1;
    double out[2];
    HO2D_CUDA(cudaMemcpyAsync(out, d.fout.get(), sizeof(out), cudaMemcpyDeviceToHost, d.stream), "copy");
    HO2D_CUDA(cudaStreamSynchronize(d.stream), "sync");
    if (fx) *fx = out[0];
    if (fy) *fy = out[1];
    return {0, ""};
}

// Uploads a coarse hierarchy (cycle operators of every level, level vectors, padded dense
// inverse of the coarsest level) and fills the device views of both precisions.
Error Solver::upload_hierarchy(const CoarseHierarchy& H, double omega, std::vector<std::unique_ptr<LevelBufs>>& lev,
                               DeviceBuffer& dense64, DeviceBuffer& dense32, Precond<double>& pc64,
                               Precond<float>& pc32, std::vector<int>* sizes) {
    if ((int)H.levels.size() > kMaxLevels) return {4, "coarse hierarchy too deep"};
    const int nl = (int)H.levels.size();
    lev.clear();
    std::vector<Ell> eM(nl), eS(nl), eQ(nl);
    for (int l = 0; l < nl; ++l) {
        const AmgLevel& L = H.levels[l];
        auto b = std::unique_ptr<LevelBufs>(new LevelBufs);
        if (l + 1 < nl) {
            eM[l] = to_ell(L.M);
            eS[l] = to_ell(L.S);
            eQ[l] = to_ell(L.Q);
            HO2D_CUDA(upload_ell(b->M, eM[l]), "upload coarse M");
            HO2D_CUDA(upload_ell(b->S, eS[l]), "upload coarse S");
            HO2D_CUDA(upload_ell(b->Q, eQ[l]), "upload coarse Q");
        }
        const std::vector<double> z((size_t)L.A.n + 8, 0.0);  // zero padding for 16-byte reads
        for (DeviceBuffer* v : {&b->f, &b->u}) HO2D_CUDA(upload(*v, z), "alloc coarse vectors");
        lev.push_back(std::move(b));
    }
    // coarsest inverse, rows padded to a multiple of 4 entries (16-byte row starts): the
    // host's, or inverted on the device in place when the hierarchy comes without it
    const int nd = H.n_dense, wd = (nd + 3) / 4 * 4;
    std::vector<double> dpad((size_t)nd * wd, 0.0);
    const bool on_device = H.dense_inv.empty();
    if (on_device) {
        const Csr& Ab = H.levels.back().A;
        for (int i = 0; i < nd; ++i)
            for (int k = Ab.ptr[i]; k < Ab.ptr[i + 1]; ++k) dpad[(size_t)i * wd + Ab.col[k]] += Ab.val[k];
    } else {
        for (int i = 0; i < nd; ++i)
            std::copy(H.dense_inv.begin() + (size_t)i * nd, H.dense_inv.begin() + (size_t)(i + 1) * nd,
                      dpad.begin() + (size_t)i * wd);
    }
    HO2D_CUDA(upload(dense64, dpad), "upload dense");
    if (on_device) {
        bool singular = false;
        HO2D_CUDA(dense_invert_device(dense64.as<double>(), nd, wd, d_->stream, &singular), "dense inverse");
        if (singular) return {3, "singular coarsest Poisson operator"};
    }
    // the FP32 preconditioner's coarsest inverse in BF16 (half the bytes of the largest
    // coarse read; the preconditioner's precision changes only the iteration count) when
    // it is a level below the element level
    const bool dense16 = nl > 1;
    const int w16 = (nd + 7) / 8 * 8;
    if (dense16) {
        HO2D_CUDA(dense32.alloc(((size_t)nd * w16 + 8) * sizeof(uint16_t)), "alloc dense");
        HO2D_CUDA(cudaMemsetAsync(dense32.get(), 0, dense32.bytes(), d_->stream), "memset");
        HO2D_CUDA(rows_to_bf16(dense64.as<double>(), wd, dense32.as<uint16_t>(), w16, nd, nd, d_->stream), "dense");
    } else {
        HO2D_CUDA(dense32.alloc(((size_t)nd * wd + 1) * sizeof(float)), "alloc dense");
        HO2D_CUDA(cudaMemsetAsync(dense32.get(), 0, dense32.bytes(), d_->stream), "memset");
        HO2D_CUDA(rows_to_f32(dense64.as<double>(), wd, nullptr, dense32.as<float>(), wd, nd, nd, d_->stream), "dense");
    }
    HO2D_CUDA(cudaStreamSynchronize(d_->stream), "dense");
    auto fill = [&](auto& pc, bool f32) {
        using T = typename std::remove_const<typename std::remove_pointer<decltype(pc.dense.val)>::type>::type;
        pc.nlev = nl;
        pc.omega = omega;
        pc.dense.n = nd;
        pc.dense.w = wd;
        pc.dense.g = 32;
        pc.dense.col = nullptr;
        pc.dense.val = f32 ? (const T*)dense32.get() : (const T*)dense64.get();
        if (f32 && dense16) {
            pc.dense.val = nullptr;
            pc.dense.val16 = dense32.as<unsigned short>();
            pc.dense.w = w16;
        }
        for (int l = 0; l < nl; ++l) {
            auto& b = *lev[l];
            auto& c = pc.lev[l];
            c.n = H.levels[l].A.n;
            if (l + 1 < nl) {
                c.M = view<T>(b.M, eM[l], lanes_for(eM[l].w), f32);
                const int g = lanes_for(std::max(eS[l].w, eQ[l].w));
                c.S = view<T>(b.S, eS[l], g, f32);
                c.Q = view<T>(b.Q, eQ[l], g, f32);
            }
            c.f = b.f.as<T>();
            c.u = b.u.as<T>();
        }
        pc.ue5 = f32 ? d_->ue5_32.as<T>() : d_->ue5.as<T>();
        pc.u0dst = d_->u0dst.as<int>();
    };
    fill(pc64, false);
    fill(pc32, true);
    if (sizes) {
        sizes->clear();
        for (const auto& L : H.levels) sizes->push_back(L.A.n);
    }
    return {0, ""};
}

// The block column sums on the host: kept by the host assembly, downloaded once after the
// device assembly.
Error Solver::ensure_host_colsum() {
    if (!op_.colsum.empty()) return {0, ""};
    DeviceState& d = *d_;
    if (!d.colsum64.get()) return {3, "block column sums unavailable"};
    op_.colsum.resize(d.colsum64.bytes() / sizeof(double));
    HO2D_CUDA(cudaMemcpy(op_.colsum.data(), d.colsum64.get(), d.colsum64.bytes(), cudaMemcpyDeviceToHost),
              "download block column sums");
    return {0, ""};
}

// Builds the P0 coarse hierarchy on the host and the device views of both precisions.
// HO2D_PRECOND=bj selects plain block-Jacobi; HO2D_MG_OMEGA sets the smoother weight;
// HO2D_DENSE_MAX bounds the dense coarsest level (a test hook for other hierarchy shapes).
Error Solver::setup_preconditioner() {
    DeviceState& d = *d_;
    const int N = mesh_.n_el;
    d.pc64 = Precond<double>();
    d.pc32 = Precond<float>();
    d.graph64.reset();
    d.graph32.reset();
    d.graph_mixed.reset();
    d.lev.clear();
    const char* mode = std::getenv("HO2D_PRECOND");
    if (mode && std::string(mode) == "bj") return {0, ""};
    const char* om = std::getenv("HO2D_MG_OMEGA");
    const double omega = om ? std::atof(om) : kSmoothingWeight;
    const char* dm = std::getenv("HO2D_DENSE_MAX");
    const int dmax = dm ? std::max(1, std::atoi(dm)) : kDenseMax;
    CoarseHierarchy H;
    HO2D_TRY(build_coarse_hierarchy(p0_coarse_operator(op_, N), H, dmax, dm ? dmax : kDenseMaxFirst,
                                    !device_setup_));
    HO2D_TRY(upload_hierarchy(H, omega, d.lev, d.dense64, d.dense32, d.pc64, d.pc32, &coarse_sizes_));
    coarse_levels_ = (int)coarse_sizes_.size();
    if (verbose_) {
        std::fprintf(stderr, "  coarse levels:");
        for (int n : coarse_sizes_) std::fprintf(stderr, " %d", n);
        std::fprintf(stderr, " (the last inverted densely)\n");
    }
    return {0, ""};
}

Error Solver::upload_precision_arrays() {
    DeviceState& d = *d_;
    if (d.have32) return {0, ""};
    const std::vector<double>* mets[9] = {&M_.xxi, &M_.xeta, &M_.yxi, &M_.yeta, &M_.J, &M_.fA, &M_.fB, &M_.fJ, &M_.fAn};
    for (int i = 0; i < 9; ++i) HO2D_CUDA(upload_as<float>(d.m32[i], *mets[i]), "upload fp32 metrics");
    const int N = mesh_.n_el, K = in_.knod, K2 = K * K, K4 = K2 * K2;
    // the FP32 (and BF16) copies are made on the device from the FP64 arrays
    const long long s8 = padded_count(K4, 8), s4 = padded_count(K4, 4);
    HO2D_CUDA(d.dinv32.alloc(((size_t)N * s4 + 1) * sizeof(float)), "alloc fp32 block-Jacobi");
    HO2D_CUDA(cudaMemsetAsync(d.dinv32.get(), 0, d.dinv32.bytes(), d.stream), "memset");
    HO2D_CUDA(rows_to_f32(d.dinv64.as<double>(), s8, nullptr, d.dinv32.as<float>(), s4, N, K4, d.stream),
              "fp32 block-Jacobi");
    // smoother kind 1: the FP32 smoother reads a BF16 copy of the inverse blocks (half the
    // bytes; the preconditioner's precision changes only the inner iteration count)
    if (smoother_kind_ == 1) {
        const long long st = padded_count(K4, 2);
        HO2D_CUDA(d.dinv_bf16.alloc(((size_t)N * st + 1) * sizeof(uint16_t)), "alloc bf16 block-Jacobi");
        HO2D_CUDA(cudaMemsetAsync(d.dinv_bf16.get(), 0, d.dinv_bf16.bytes(), d.stream), "memset");
        HO2D_CUDA(rows_to_bf16(d.dinv64.as<double>(), s8, d.dinv_bf16.as<uint16_t>(), st, N, K4, d.stream),
                  "bf16 block-Jacobi");
    }
    if (kron_.K > 0) {  // the Kronecker-sum smoother's arrays (FP32), smoother kind 2
        std::vector<double> f;
        std::vector<int> xi, rows;
        kron_factor_arrays(kron_, f, xi);
        for (int el = 0; el < N; ++el)
            if (xi[el] >= 0) rows.push_back(el);
        const int per = 4 * K2 + 2 * K;
        if (!kron_on_device_)  // (the device fit wrote its factors in place)
            HO2D_CUDA(upload(d.kron_f, padded_rows<float>(f, N, per, padded_count(per, 4))),
                      "upload Kronecker factors");
        HO2D_CUDA(upload(d.kron_x, xi), "upload Kronecker exact-block index");
        DeviceBuffer drows;
        HO2D_CUDA(upload(drows, rows.empty() ? std::vector<int>{0} : rows), "upload exact rows");
        HO2D_CUDA(d.kron_exact.alloc(((size_t)rows.size() * s4 + 1) * sizeof(float)), "alloc Kronecker exact blocks");
        HO2D_CUDA(cudaMemsetAsync(d.kron_exact.get(), 0, d.kron_exact.bytes(), d.stream), "memset");
        HO2D_CUDA(rows_to_f32(d.dinv64.as<double>(), s8, drows.as<int>(), d.kron_exact.as<float>(), s4,
                              (int)rows.size(), K4, d.stream),
                  "Kronecker exact blocks");
        HO2D_CUDA(cudaStreamSynchronize(d.stream), "Kronecker exact blocks");
    }
    HO2D_CUDA(d.rowsum32.alloc((size_t)N * 5 * K2 * sizeof(float)), "alloc fp32 block row sums");
    HO2D_CUDA(rows_to_f32(d.rowsum64.as<double>(), K2, nullptr, d.rowsum32.as<float>(), K2, N * 5, K2, d.stream),
              "fp32 block row sums");
    for (int a = 0; a < 8; ++a) HO2D_CUDA(upload_as<float>(d.pg32[a], d.pg_host[a]), "upload fp32 operator data");
    // the FP32 smoother (exact, BF16 or Kronecker-sum) applied to the block row sums
    HO2D_CUDA(krylov_make_w<float>(make_op<float>(d, mesh_, K, true), d.W32.as<float>(), d.scalars.as<KrylovScalars>(),
                                   d.stream),
              "smoothed row sums");
    HO2D_CUDA(cudaStreamSynchronize(d.stream), "smoothed row sums");
    d.have32 = true;
    return {0, ""};
}

Error Solver::set_smoother(int kind) {
    if (kind < -1 || kind > 2)
        return {1, "smoother must be HO2D_SMOOTHER_BLOCKS (0), HO2D_SMOOTHER_BF16 (1) or HO2D_SMOOTHER_KRON (2)"};
    smoother_req_ = kind;
    return {0, ""};
}

Error Solver::set_precision(int mode) {
    if (mode < 0 || mode > 2)
        return {1, "precision must be HO2D_FP64 (0), HO2D_MIXED (1) or HO2D_MIXED_KRYLOV (2)"};
    const bool was = stage32_;
    stage32_ = mode == 1;
    krylov32_ = mode != 0;
    if (setup_done_) {
        if (stage32_ || krylov32_) HO2D_TRY(upload_precision_arrays());
        if (stage32_ != was) {
            // re-derive the stage input in the new precision from the FP64 vorticity
            DeviceState& d = *d_;
            const size_t nv = (size_t)mesh_.n_el * in_.knod * in_.knod;
            if (stage32_) HO2D_CUDA(launch_copy_d2f(d.omega.as<double>(), d.w_stage.as<float>(), nv, d.stream), "d2f");
            else
                HO2D_CUDA(cudaMemcpyAsync(d.w_stage.get(), d.omega.get(), nv * 8, cudaMemcpyDeviceToDevice, d.stream),
                          "copy");
            HO2D_CUDA(cudaStreamSynchronize(d.stream), "sync");
        }
    }
    return {0, ""};
}

// ------------------------------------------------------------------ Poisson
Error Solver::poisson_solve() {
    const NvtxRange nvtx_range("ho2d.poisson");
    DeviceState& d = *d_;
    const int N = mesh_.n_el, K = in_.knod;
    const size_t nv = (size_t)N * K * K;
    ReduceScratch rs{d.partials.as<double>(), d.counter.as<unsigned>(), d.scalars.as<KrylovScalars>()};
    if (timing_) HO2D_CUDA(cudaEventRecord(d.evp0, d.stream), "event");
    auto poll = [&]() -> Error {
        HO2D_CUDA(cudaMemcpyAsync(d.h_sc, d.scalars.get(), sizeof(KrylovScalars), cudaMemcpyDeviceToHost, d.stream),
                  "poll");
        HO2D_CUDA(cudaStreamSynchronize(d.stream), "poll");
        if (d.h_sc->dev_error) return {5, "a device-side wait for a bulk copy ran out (the GPU did not complete it)"};
        return {0, ""};
    };
    // runs BiCGSTAB to completion on (A, v); returns iterations
    // one solve: by default a single launch of the captured graph (initial residual and a
    // device-side while loop); with HO2D_GRAPHS=0 the host enqueues batches of iterations
    // and polls the done flag between batches
    auto run = [&](auto A, auto v, const auto& pc, double tol, int& iters, SolveGraph& sg) -> Error {
        // the tolerance travels in the device scalars, so one captured graph serves any
        // tolerance (the stream is idle here: every earlier read of h_sc was synchronised)
        d.h_sc->tol = tol;
        HO2D_CUDA(cudaMemcpyAsync(&d.scalars.as<KrylovScalars>()->tol, &d.h_sc->tol, sizeof(double),
                                  cudaMemcpyHostToDevice, d.stream),
                  "tolerance");
        if (use_graphs_) {
            if (!sg.exec || sg.max_iter != max_iter_) {
                sg.reset();
                HO2D_CUDA(krylov_capture_solve(A, v, rs, max_iter_, pc, d.stream, &sg.graph), "graph capture");
                // per-node priorities: the coarse cycle's nodes keep their stream's high priority
                HO2D_CUDA(cudaGraphInstantiate(&sg.exec, sg.graph, cudaGraphInstantiateFlagUseNodePriority),
                          "graph instantiate");
                sg.max_iter = max_iter_;
            }
            HO2D_CUDA(cudaGraphLaunch(sg.exec, d.stream), "graph launch");
            HO2D_TRY(poll());
            iters = d.h_sc->it;
            launches_ += 4 + (int64_t)iters * krylov_launches_per_iteration(pc);
            return {0, ""};
        }
        HO2D_CUDA(krylov_init(A, v, rs, d.stream), "krylov init");
        launches_ += 3;
        HO2D_TRY(poll());
        int chunk = std::max(1, prev_iters_ - 1);
        while (!d.h_sc->done) {
            for (int c = 0; c < chunk; ++c) {
                HO2D_CUDA(krylov_iteration(A, v, rs, max_iter_, pc, d.stream), "krylov iteration");
                launches_ += krylov_launches_per_iteration(pc);
            }
            HO2D_TRY(poll());
            chunk = 2;
        }
        iters = d.h_sc->it;
        return {0, ""};
    };
    last_iters_ = 0;
    int sweeps = 0;
    bool finite = true;
    double refined_res = -1.0;  // the refinement's residual when the FP64 solve finished it
    // the FP64 solve from the current psi (the FP64 mode, and the finish of a mixed solve
    // whose refinement stalled)
    auto fp64_solve = [&]() -> Error {
        const MfOp<double> A = make_op<double>(d, mesh_, K, false);
        const BicgVectors<double> v = krylov_vectors<double>(d, d.psi64.as<double>(), d.rhs.as<double>());
        int it = 0;
        HO2D_TRY(run(A, v, d.pc64, tol_, it, d.graph64));
        last_iters_ += it;
        const double bn = d.h_sc->bnorm2, rn = d.h_sc->rnorm2;
        finite = std::isfinite(bn) && std::isfinite(rn);
        last_res_ = bn > 0 ? std::sqrt(rn / bn) : 0.0;
        return {0, ""};
    };
    if (!krylov32_) {
        HO2D_TRY(fp64_solve());
    } else if (use_graphs_) {
        // FP64 iterative refinement around an FP32 BiCGSTAB, both loops on the device: one
        // graph launch and one read of the scalars per solve
        const MfOp<double> A64 = make_op<double>(d, mesh_, K, false);
        const MfOp<float> A32 = make_op<float>(d, mesh_, K, true);
        const BicgVectors<float> v = krylov_vectors<float>(d, d.kv[8].as<float>(), d.kv[9].as<float>());
        SolveGraph& sg = d.graph_mixed;
        if (!sg.exec || sg.max_iter != max_iter_) {
            sg.reset();
            HO2D_CUDA(krylov_capture_refined_solve(A64, A32, v, rs, max_iter_, d.pc32, d.psi64.as<double>(),
                                                   d.rhs.as<double>(), d.rres.as<double>(), d.kxtv.as<double>(),
                                                   d.kxtg.as<double>(), d.stream, &sg.graph),
                      "graph capture");
            // per-node priorities: the coarse cycle's nodes keep their stream's high priority
            HO2D_CUDA(cudaGraphInstantiate(&sg.exec, sg.graph, cudaGraphInstantiateFlagUseNodePriority),
                      "graph instantiate");
            sg.max_iter = max_iter_;
        }
        // the refinement's controls travel in the device scalars (the stream is idle: every
        // earlier read of h_sc was synchronised)
        d.h_sc->tol_outer = tol_;
        d.h_sc->inner_tol = inner_tol_;
        d.h_sc->max_sweeps = max_sweeps_;
        static_assert(offsetof(KrylovScalars, inner_tol) == offsetof(KrylovScalars, tol_outer) + sizeof(double) &&
                          offsetof(KrylovScalars, max_sweeps) == offsetof(KrylovScalars, inner_tol) + sizeof(double),
                      "refinement controls are contiguous");
        HO2D_CUDA(cudaMemcpyAsync(&d.scalars.as<KrylovScalars>()->tol_outer, &d.h_sc->tol_outer,
                                  2 * sizeof(double) + sizeof(int), cudaMemcpyHostToDevice, d.stream),
                  "refinement controls");
        HO2D_CUDA(cudaGraphLaunch(sg.exec, d.stream), "graph launch");
        HO2D_TRY(poll());
        sweeps = d.h_sc->sweeps;
        last_iters_ = d.h_sc->iters_total;
        finite = d.h_sc->finite != 0;
        last_res_ = d.h_sc->res;
        launches_ += krylov_refined_launches(sweeps, last_iters_, d.pc32);
        if (finite && !(last_res_ <= tol_)) {  // stalled or capped: the FP64 solve finishes
            ++fp64_finishes_;
            refined_res = last_res_;
            HO2D_TRY(fp64_solve());
        }
    } else {
        // FP64 iterative refinement around an FP32 BiCGSTAB on the same operator, driven
        // from the host (HO2D_GRAPHS=0): every exit passes through an FP64 residual of the
        // current psi
        const MfOp<double> A64 = make_op<double>(d, mesh_, K, false);
        const MfOp<float> A32 = make_op<float>(d, mesh_, K, true);
        const BicgVectors<float> v = krylov_vectors<float>(d, d.kv[8].as<float>(), d.kv[9].as<float>());
        bool stalled = false;
        for (;; ++sweeps) {
            HO2D_CUDA(mf_residual<double>(A64, d.rhs.as<double>(), d.psi64.as<double>(), d.kxtv.as<double>(),
                                          d.kxtg.as<double>(), d.rres.as<double>(), rs, d.stream),
                      "fp64 residual");
            launches_ += 2;
            HO2D_TRY(poll());
            const double bn = d.h_sc->bnorm2, rn = d.h_sc->rnorm2;
            const double prev = last_res_;
            finite = std::isfinite(bn) && std::isfinite(rn);
            last_res_ = bn > 0 ? std::sqrt(rn / bn) : 0.0;
            if (!finite) break;
            if (bn == 0.0) {
                HO2D_CUDA(cudaMemsetAsync(d.psi64.get(), 0, nv * 8, d.stream), "memset");
                last_res_ = 0.0;
                break;
            }
            if (rn <= tol_ * tol_ * bn || sweeps >= max_sweeps_) break;
            if (sweeps > 0 && !(last_res_ <= 0.5 * prev)) {  // the same stall rule as the graph
                stalled = true;
                break;
            }
            HO2D_CUDA(launch_copy_d2f(d.rres.as<double>(), d.kv[9].as<float>(), nv, d.stream), "d2f");
            HO2D_CUDA(cudaMemsetAsync(d.kv[8].get(), 0, nv * sizeof(float), d.stream), "memset");
            launches_ += 1;
            // ask the inner solve for no more reduction than this sweep needs: the last
            // sweep typically needs one order of magnitude, not inner_tol_'s four
            const double need = 0.3 * tol_ / last_res_;
            const double itol = std::min(0.5, std::max(inner_tol_, need));
            int it = 0;
            HO2D_TRY(run(A32, v, d.pc32, itol, it, d.graph32));
            last_iters_ += it;
            HO2D_CUDA(launch_axpy_f2d(d.kv[8].as<float>(), d.psi64.as<double>(), nv, d.stream), "axpy");
            launches_ += 1;
        }
        if (finite && (stalled || !(last_res_ <= tol_))) {
            ++fp64_finishes_;
            refined_res = last_res_;
            HO2D_TRY(fp64_solve());
        }
    }
    ++n_solves_;
    iters_total_ += last_iters_;
    sweeps_total_ += krylov32_ ? sweeps : 0;
    if (verbose_) {
        std::fprintf(stderr, "  poisson solve %ld: iters %d sweeps %d rel. residual %.3e (FP64 finishes so far %ld)",
                     n_solves_, last_iters_, sweeps, last_res_, (long)fp64_finishes_);
        if (refined_res >= 0.0) std::fprintf(stderr, "; finished in FP64 from %.3e", refined_res);
        std::fprintf(stderr, "\n");
    }
    prev_iters_ = std::max(1, krylov32_ ? last_iters_ / std::max(1, sweeps) : last_iters_);
    if (timing_) {
        HO2D_CUDA(cudaEventRecord(d.evp1, d.stream), "event");
        HO2D_CUDA(cudaEventSynchronize(d.evp1), "event");
        float ms = 0.f;
        HO2D_CUDA(cudaEventElapsedTime(&ms, d.evp0, d.evp1), "event");
        poisson_ms_acc_ += ms;
    }
    if (!finite || !std::isfinite(last_res_))
        return {7, "non-finite values in the Poisson solve (vorticity blew up)"};
    return {0, ""};
}

// ------------------------------------------------------------------ stages
// update_BCs(t) (src/HO_2D.cpp:1979-2217) on the device: the time-dependent BC values of
// problem types 2, 3 and 11 and the h-direction flip. For a hybrid run (type 11) it also
// blends omega towards the driver's vorticity with the particle-to-grid weights, as the
// reference does at every call; into_stage also blends the stage input, which is omega
// itself in the first stage.
template <typename T>
Error Solver::update_bcs(double t, bool into_stage) {
    DeviceState& d = *d_;
    BcArrays bc{d.bc_p.as<double>(), d.bc_nv.as<double>(), d.bc_pv.as<double>(), d.bc_d.as<double>(),
                d.bc_w.as<double>(), d.vjump.as<double>(), d.bc_adv.as<double>()};
    const double tc = 2.0 * std::fabs(std::sin(M_PI / 40.0 * t));
    HybridBc hb;
    const bool hyb = in_.problem_type == 11;
    if (hyb) {
        // weight of the start values: (t - t_start) / (t_end - t_start), as in the reference
        // (so the end values apply at the outer step's start); end values before any outer step
        hb.fac1 = t_end_ > t_start_ ? (t - t_start_) / (t_end_ - t_start_) : 0.0;
        hb.fac2 = 1.0 - hb.fac1;
        hb.vn0 = d.hyb[0].as<double>();
        hb.vn1 = d.hyb[1].as<double>();
        hb.vp0 = d.hyb[2].as<double>();
        hb.vp1 = d.hyb[3].as<double>();
        hb.w0 = d.hyb[4].as<double>();
        hb.w1 = d.hyb[5].as<double>();
        hb.inlet_nv = d.hyb_inlet_nv.as<double>();
    }
    HO2D_CUDA(launch_bc_update(mesh_.n_eb, in_.knod, in_.problem_type, tc, bc_.y_min, bc_.y_max, d.role.as<int>(),
                               d.be_ijp.as<int>(), d.sw_d.as<int>(), d.edge_y.as<double>(), bc, hb, d.stream),
              "bc_update");
    launches_ += 1;
    if (hyb) {
        const size_t nv = (size_t)mesh_.n_el * in_.knod * in_.knod;
        HO2D_CUDA(launch_hybrid_blend<T>(nv, d.omega.as<double>(), into_stage ? d.w_stage.as<T>() : nullptr,
                                         d.hvort[2].as<double>(), d.hvort[0].as<double>(), d.hvort[1].as<double>(),
                                         hb.fac1, hb.fac2, d.stream),
                  "hybrid blend");
        launches_ += 1;
    }
    return {0, ""};
}

// One stage at the current stage input. With solve == false the Poisson solve is skipped
// and the stage works from the psi already in place (the adjoint recomputes a stored
// stage's fields this way).
template <typename T>
Error Solver::stage_t(double coeff, int rk_stage, bool update, bool solve) {
    const NvtxRange nvtx_range("ho2d.stage");
    DeviceState& d = *d_;
    const int N = mesh_.n_el, K = in_.knod;
    const size_t nv = (size_t)N * K * K;
    const bool f32 = sizeof(T) == 4;
    const DevBases<T>& b = *reinterpret_cast<const DevBases<T>*>(f32 ? (const void*)&d.b32 : (const void*)&d.b64);
    const FrGeom<T> g = geom_of<T>(d, mesh_, f32);
    BcArrays bc{d.bc_p.as<double>(), d.bc_nv.as<double>(), d.bc_pv.as<double>(), d.bc_d.as<double>(),
                d.bc_w.as<double>(), d.vjump.as<double>(), d.bc_adv.as<double>()};
    HO2D_TRY(update_bcs<T>(time_ + coeff * in_.dt, rk_stage == 0));
    const FrGeom<double> g64 = geom_of<double>(d, mesh_, false);
    // Inside a time step the FP32 stage takes its Poisson right-hand side from the FP64
    // stage input: omega for the first stage, the residual kernel's FP64 copy of the next
    // stage input for the others. The FP32 rounding of the stage vorticity is noise that the
    // extrapolated initial guess cannot predict, so a right-hand side built from it starts
    // every solve at about 1e-7 relative residual.
    const bool rhs64 = f32 && update;
    if (solve) {
        if (rhs64)
            HO2D_CUDA(launch_poisson_rhs<double>(K, N, d.face_nb.as<int>(),
                                                 rk_stage == 0 ? d.omega.as<double>() : d.w_stage64.as<double>(),
                                                 g64.J, d.bsrc.as<double>(), d.bc_p.as<double>(),
                                                 d.rhs.as<double>(), d.stream),
                      "poisson_rhs");
        else
            HO2D_CUDA(launch_poisson_rhs<T>(K, N, d.face_nb.as<int>(), d.w_stage.as<T>(), g.J, d.bsrc.as<double>(),
                                            d.bc_p.as<double>(), d.rhs.as<double>(), d.stream),
                      "poisson_rhs");
        launches_ += 1;
        HO2D_TRY(poisson_solve());
    }
    // the velocity is derived from psi in FP64 in both precisions (VelocityArgs)
    const double* psi = d.psi64.as<double>();
    HO2D_CUDA(launch_trace<double>(K, N, psi, d.psi_tv.as<double>(), d.psi_tg.as<double>(), d.b64, d.stream), "trace");
    VelocityArgs<T, double> va{psi, d.psi_tv.as<double>(), d.psi_tg.as<double>(), d.w_stage.as<T>(), d.u.as<T>(),
                               d.v.as<T>(), d.w_tv.as<T>(), d.w_tg.as<T>(), d.U_t.as<T>(), in_.dt, in_.reyn_inv};
    HO2D_CUDA((launch_velocity<T, double>(K, g64, stage_coef<double>(d, false), d.b64, b, bc, va, d.stream)), "velocity");
    ResidualArgs<T> ra;
    ra.w = d.w_stage.as<T>();
    ra.u = d.u.as<T>();
    ra.v = d.v.as<T>();
    ra.w_tv = d.w_tv.as<T>();
    ra.w_tg = d.w_tg.as<T>();
    ra.U_t = d.U_t.as<T>();
    ra.dt = in_.dt;
    ra.re_inv = in_.reyn_inv;
    ra.adv_type = in_.adv_type;
    ra.ti_type = update ? in_.ti_type : 0;
    ra.stage = rk_stage;
    ra.omega = d.omega.as<double>();
    ra.acc = d.acc.as<double>();
    ra.w_next = update ? d.w_stage.as<T>() : nullptr;
    ra.w_next64 = rhs64 ? d.w_stage64.as<double>() : nullptr;
    // the RHS terms are kept from a lone stage and from the last stage of a step (the
    // reference's RHS arrays hold the last stage computed; its VTK output writes them)
    const int ns = in_.ti_type == 4 ? 4 : (in_.ti_type == 2 ? 2 : 1);
    const bool keep_rhs = !update || rk_stage == ns - 1;
    ra.rhs_diff = keep_rhs ? d.rhs_diff.as<T>() : nullptr;
    ra.rhs_adv = keep_rhs ? d.rhs_adv.as<T>() : nullptr;
    ra.k_out = update ? nullptr : d.kout.as<T>();
    HO2D_CUDA(launch_residual<T>(K, g, stage_coef<T>(d, f32), b, bc, ra, d.stream), "residual");
    launches_ += 3;
    return {0, ""};
}

template <typename T>
Error Solver::velocity_only_t() {
    // update_BCs(t) + solve_Poisson(vorticity) + velocity, as at dump steps (src/HO_2D.cpp:1411-1416)
    DeviceState& d = *d_;
    const int N = mesh_.n_el, K = in_.knod;
    const size_t nv = (size_t)N * K * K;
    const bool f32 = sizeof(T) == 4;
    const DevBases<T>& b = *reinterpret_cast<const DevBases<T>*>(f32 ? (const void*)&d.b32 : (const void*)&d.b64);
    const FrGeom<T> g = geom_of<T>(d, mesh_, f32);
    BcArrays bc{d.bc_p.as<double>(), d.bc_nv.as<double>(), d.bc_pv.as<double>(), d.bc_d.as<double>(),
                d.bc_w.as<double>(), d.vjump.as<double>(), d.bc_adv.as<double>()};
    HO2D_TRY(update_bcs<T>(time_, true));
    HO2D_CUDA(launch_poisson_rhs<T>(K, N, d.face_nb.as<int>(), d.w_stage.as<T>(), g.J, d.bsrc.as<double>(),
                                    d.bc_p.as<double>(), d.rhs.as<double>(), d.stream),
              "poisson_rhs");
    HO2D_TRY(poisson_solve());
    const double* psi = d.psi64.as<double>();
    const FrGeom<double> g64 = geom_of<double>(d, mesh_, false);
    HO2D_CUDA(launch_trace<double>(K, N, psi, d.psi_tv.as<double>(), d.psi_tg.as<double>(), d.b64, d.stream), "trace");
    VelocityArgs<T, double> va{psi, d.psi_tv.as<double>(), d.psi_tg.as<double>(), d.w_stage.as<T>(), d.u.as<T>(),
                               d.v.as<T>(), d.w_tv.as<T>(), d.w_tg.as<T>(), d.U_t.as<T>(), in_.dt, in_.reyn_inv};
    HO2D_CUDA((launch_velocity<T, double>(K, g64, stage_coef<double>(d, false), d.b64, b, bc, va, d.stream)), "velocity");
    launches_ += 4;
    return {0, ""};
}

Error Solver::stage_impl(double coeff, int rk_stage, bool update) {
    return stage32_ ? stage_t<float>(coeff, rk_stage, update) : stage_t<double>(coeff, rk_stage, update);
}

Error Solver::step(int nsteps) {
    const NvtxRange nvtx_range("ho2d.step");
    if (!setup_done_) return {1, "ho2d_step called before ho2d_setup"};
    if (nsteps < 0) return {1, "nsteps must be non-negative"};
    HO2D_CUDA(cudaSetDevice(d_->device), "cudaSetDevice");
    static const double c4[4] = {0.0, 0.5, 0.5, 1.0};
    static const double c2[2] = {0.0, 1.0};
    const int ns = in_.ti_type == 4 ? 4 : (in_.ti_type == 2 ? 2 : 1);
    const double* c = in_.ti_type == 4 ? c4 : c2;
    DeviceState& d = *d_;
    const size_t nv = (size_t)mesh_.n_el * in_.knod * in_.knod;
    const int order = psi_extrap_;
    if (order >= 2 && !d.psi_hist[0][0].get())
        for (auto& row : d.psi_hist)
            for (auto& b : row) HO2D_CUDA(b.alloc(nv * 8), "alloc psi history");
    if (hist_dt_ != in_.dt || hist_ns_ != ns) {
        hist_count_ = 0;
        hist_dt_ = in_.dt;
        hist_ns_ = ns;
    }
    for (int i = 0; i < nsteps; ++i) {
        const int k = hist_step_;
        for (int s = 0; s < ns; ++s) {
            if (order >= 2 && hist_count_ >= order) {
                // initial guess of this stage's Poisson solve: the same stage of the last
                // steps, extrapolated in time (they are dt apart); the solve's tolerance is
                // unchanged, only its starting point moves closer
                double* psi = d.psi64.as<double>();
                const double* h1 = d.psi_hist[(k + 2) % 3][s].as<double>();
                const double* h2 = d.psi_hist[(k + 1) % 3][s].as<double>();
                if (order == 2) {
                    HO2D_CUDA(launch_axpby(nv, psi, 2.0, h1, -1.0, h2, d.stream), "psi guess");
                } else {
                    const double* h3 = d.psi_hist[k % 3][s].as<double>();
                    HO2D_CUDA(launch_axpby(nv, psi, 3.0, h1, -3.0, h2, d.stream), "psi guess");
                    HO2D_CUDA(launch_axpby(nv, psi, 1.0, psi, 1.0, h3, d.stream), "psi guess");
                }
                launches_ += order - 1;
            }
            HO2D_TRY(stage_impl(c[s], s, true));
            if (order >= 2)
                HO2D_CUDA(cudaMemcpyAsync(d.psi_hist[k % 3][s].get(), d.psi64.get(), nv * 8, cudaMemcpyDeviceToDevice,
                                          d.stream),
                          "psi history");
        }
        time_ += in_.dt;
        hist_step_ = (k + 1) % 3;
        hist_count_ = std::min(hist_count_ + 1, 3);
    }
    HO2D_CUDA(cudaStreamSynchronize(d_->stream), "step");
    HO2D_CUDA(cudaGetLastError(), "step");
    return {0, ""};
}

Error Solver::stage(double coeff) {
    if (!setup_done_) return {1, "ho2d_stage called before ho2d_setup"};
    HO2D_CUDA(cudaSetDevice(d_->device), "cudaSetDevice");
    HO2D_TRY(stage_impl(coeff, 0, false));
    HO2D_CUDA(cudaStreamSynchronize(d_->stream), "stage");
    return {0, ""};
}

Error Solver::solve() {
    const NvtxRange nvtx_range("ho2d.solve");
    if (!setup_done_) return {1, "ho2d_solve called before ho2d_setup"};
    HO2D_CUDA(cudaSetDevice(d_->device), "cudaSetDevice");
    const int nt = in_.num_steps, df = std::max(1, in_.dump_freq);
    // dumps are written on the VTK queue's thread while the loop goes on; all are on disk
    // when solve returns
    for (int ti = 0; ti < nt; ++ti) {
        if (ti % df == 0) {
            HO2D_TRY(stage32_ ? velocity_only_t<float>() : velocity_only_t<double>());
            if (!output_dir_.empty()) HO2D_TRY(queue_vtk(ti, output_dir_));
        }
        HO2D_TRY(step(1));
    }
    if (nt % df == 0) {
        HO2D_TRY(stage32_ ? velocity_only_t<float>() : velocity_only_t<double>());
        if (!output_dir_.empty()) HO2D_TRY(queue_vtk(nt, output_dir_));
    }
    HO2D_CUDA(cudaStreamSynchronize(d_->stream), "solve");
    return vtk_queue_.wait();
}

Error Solver::solveto(double outerdt, int numstep, int integtype, double reyn) {
    // src/HO_2D.cpp:4194-4233 for the non-hybrid problem types
    if (!setup_done_) return {1, "ho2d_solveto called before ho2d_setup"};
    if (numstep <= 0 || !(outerdt > 0.0)) return {1, "solveto needs numstep > 0 and outerdt > 0"};
    if (integtype != 1 && integtype != 2 && integtype != 4) return {4, "integtype must be 1, 2 or 4"};
    in_.dt = outerdt / numstep;
    in_.ti_type = integtype;
    in_.reyn_inv = reyn > 1e-3 ? 1.0 / reyn : -1.0;
    // the outer step runs from the previous outer step's end (src/HO_2D.cpp:4208-4210)
    t_start_ = t_end_;
    time_ = t_start_;
    t_end_ += outerdt;
    return step(numstep);
}

Error Solver::time_steps(int nsteps, double* total_ms, double* poisson_ms) {
    if (!setup_done_) return {1, "ho2d_time_steps called before ho2d_setup"};
    DeviceState& d = *d_;
    HO2D_CUDA(cudaSetDevice(d.device), "cudaSetDevice");
    // twice the 126 MB L2: writing it before a step evicts what the previous step left there
    constexpr size_t kFlushBytes = size_t(256) << 20;
    if (!d.l2flush.get()) HO2D_CUDA(d.l2flush.alloc(kFlushBytes), "cudaMalloc");
    HO2D_CUDA(cudaStreamSynchronize(d.stream), "sync");
    timing_ = true;
    poisson_ms_acc_ = 0.0;
    double total = 0.0;
    for (int s = 0; s < nsteps; ++s) {
        HO2D_CUDA(cudaMemsetAsync(d.l2flush.get(), s & 0xff, kFlushBytes, d.stream), "L2 flush");
        HO2D_CUDA(cudaEventRecord(d.ev0, d.stream), "event");
        Error e = step(1);
        if (e.code) {
            timing_ = false;
            return e;
        }
        HO2D_CUDA(cudaEventRecord(d.ev1, d.stream), "event");
        HO2D_CUDA(cudaEventSynchronize(d.ev1), "event");
        float ms = 0.f;
        HO2D_CUDA(cudaEventElapsedTime(&ms, d.ev0, d.ev1), "event");
        total += ms;
    }
    timing_ = false;
    if (total_ms) *total_ms = total;
    if (poisson_ms) *poisson_ms = poisson_ms_acc_;
    return {0, ""};
}

// Average duration of the Poisson operator kernel (k_mf_apply: y = A x, matrix-free, the
// same device code as every operator application inside the Krylov solve) over `reps`
// launches between CUDA events on the handle's stream, and its algorithmic bytes per
// launch: per point x, the 3 metric coefficients and y; per face point the 4 face
// coefficients and the 2 incoming traces; 4 face codes per element.
Error Solver::profile_spmv(int reps, double* avg_ms, double* bytes) {
    if (!setup_done_) return {1, "not set up"};
    if (reps <= 0) return {1, "reps must be positive"};
    DeviceState& d = *d_;
    HO2D_CUDA(cudaSetDevice(d.device), "cudaSetDevice");
    const int N = mesh_.n_el, K = in_.knod;
    const size_t w = krylov32_ ? 4 : 8;
    if (bytes) *bytes = double((size_t)N * ((5 * (size_t)K * K + 24 * (size_t)K) * w + 16));
    if (!krylov32_) {
        const MfOp<double> op = make_op<double>(d, mesh_, K, false);
        HO2D_CUDA(mf_apply_op<double>(op, d.psi64.as<double>(), d.kxtv.as<double>(), d.kxtg.as<double>(),
                                      d.kv[5].as<double>(), d.stream), "apply");
        HO2D_CUDA(cudaEventRecord(d.ev0, d.stream), "event");
        HO2D_CUDA(mf_apply_only<double>(op, d.psi64.as<double>(), d.kxtv.as<double>(), d.kxtg.as<double>(),
                                        d.kv[5].as<double>(), reps, d.stream), "apply");
    } else {
        const MfOp<float> op = make_op<float>(d, mesh_, K, true);
        HO2D_CUDA(launch_copy_d2f(d.psi64.as<double>(), d.psiT.as<float>(), (size_t)N * K * K, d.stream), "d2f");
        HO2D_CUDA(mf_apply_op<float>(op, d.psiT.as<float>(), d.kxtv.as<float>(), d.kxtg.as<float>(),
                                     d.kv[5].as<float>(), d.stream), "apply");
        HO2D_CUDA(cudaEventRecord(d.ev0, d.stream), "event");
        HO2D_CUDA(mf_apply_only<float>(op, d.psiT.as<float>(), d.kxtv.as<float>(), d.kxtg.as<float>(),
                                       d.kv[5].as<float>(), reps, d.stream), "apply");
    }
    HO2D_CUDA(cudaEventRecord(d.ev1, d.stream), "event");
    HO2D_CUDA(cudaEventSynchronize(d.ev1), "event");
    float ms = 0.f;
    HO2D_CUDA(cudaEventElapsedTime(&ms, d.ev0, d.ev1), "event");
    if (avg_ms) *avg_ms = ms / reps;
    return {0, ""};
}

// Per-launch device time of the Krylov kernels inside BiCGSTAB iterations of the active
// precision's solve, and their algorithmic bytes per launch: [0] the fine part of the
// smoothing step (vector update + the smoother's element inverse), [1] the operator kernels
// (v = A ph, t = A sh), [2] the x/r update, [3] one coarse cycle, [4] the combination of
// the smoothing step (coarse correction + face traces). The iterations run on the current
// state without a CUDA graph and in order on the handle's stream (the coarse cycle does not
// run beside the fine part here), with events between the launches: the FP32 solve of a
// refinement sweep on the FP64 residual of the current psi (mixed modes), or the FP64 solve
// of the last right-hand side from a zero guess (FP64). Their tolerance is zero, so none of
// them ends early; psi is not changed.
Error Solver::profile_krylov(int reps, double* ms, double* bytes) {
    if (!setup_done_) return {1, "not set up"};
    if (reps <= 0 || reps > 1000) return {1, "reps must be in 1..1000"};
    DeviceState& d = *d_;
    HO2D_CUDA(cudaSetDevice(d.device), "cudaSetDevice");
    const int N = mesh_.n_el, K = in_.knod, K2 = K * K;
    const size_t nv = (size_t)N * K2;
    for (cudaEvent_t& e : d.prof_ev)
        if (!e) HO2D_CUDA(cudaEventCreate(&e), "cudaEventCreate");
    ReduceScratch rs{d.partials.as<double>(), d.counter.as<unsigned>(), d.scalars.as<KrylovScalars>()};
    HO2D_CUDA(cudaStreamSynchronize(d.stream), "sync");
    d.h_sc->tol = 0.0;
    HO2D_CUDA(cudaMemcpyAsync(&d.scalars.as<KrylovScalars>()->tol, &d.h_sc->tol, sizeof(double),
                              cudaMemcpyHostToDevice, d.stream),
              "tolerance");
    double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    auto run = [&](auto A, auto v, const auto& pc) -> Error {
        HO2D_CUDA(krylov_init(A, v, rs, d.stream), "krylov init");
        for (int r = 0; r < reps; ++r) {
            HO2D_CUDA(krylov_iteration_timed(A, v, rs, 1 << 30, pc, d.prof_ev, d.stream), "krylov iteration");
            HO2D_CUDA(cudaEventSynchronize(d.prof_ev[9]), "event");
            float t[9];
            for (int i = 0; i < 9; ++i) HO2D_CUDA(cudaEventElapsedTime(&t[i], d.prof_ev[i], d.prof_ev[i + 1]), "event");
            acc[3] += t[0] + t[4];
            acc[0] += t[1] + t[5];
            acc[4] += t[2] + t[6];
            acc[1] += t[3] + t[7];
            acc[2] += t[8];
        }
        return {0, ""};
    };
    const int bw = krylov32_ ? 4 : 8;
    int coarse_bytes = 0;
    if (krylov32_) {
        const MfOp<double> A64 = make_op<double>(d, mesh_, K, false);
        const MfOp<float> A32 = make_op<float>(d, mesh_, K, true);
        const BicgVectors<float> v = krylov_vectors<float>(d, d.kv[8].as<float>(), d.kv[9].as<float>());
        HO2D_CUDA(mf_residual<double>(A64, d.rhs.as<double>(), d.psi64.as<double>(), d.kxtv.as<double>(),
                                      d.kxtg.as<double>(), d.rres.as<double>(), rs, d.stream),
                  "fp64 residual");
        HO2D_CUDA(launch_copy_d2f(d.rres.as<double>(), d.kv[9].as<float>(), nv, d.stream), "d2f");
        HO2D_CUDA(cudaMemsetAsync(d.kv[8].get(), 0, nv * sizeof(float), d.stream), "memset");
        HO2D_TRY(run(A32, v, d.pc32));
        coarse_bytes = coarse_cycle_bytes(d.pc32);
    } else {
        const MfOp<double> A = make_op<double>(d, mesh_, K, false);
        const BicgVectors<double> v = krylov_vectors<double>(d, d.kv[8].as<double>(), d.rhs.as<double>());
        HO2D_CUDA(cudaMemsetAsync(d.kv[8].get(), 0, nv * sizeof(double), d.stream), "memset");
        HO2D_TRY(run(A, v, d.pc64));
        coarse_bytes = coarse_cycle_bytes(d.pc64);
    }
    HO2D_CUDA(cudaMemcpyAsync(d.h_sc, d.scalars.get(), sizeof(KrylovScalars), cudaMemcpyDeviceToHost, d.stream),
              "poll");
    HO2D_CUDA(cudaStreamSynchronize(d.stream), "sync");
    if (d.h_sc->done && d.h_sc->it < reps)
        return {1, "the profiled iterations ended early (breakdown): no per-kernel times"};
    if (ms) {
        ms[0] = acc[0] / (2.0 * reps);
        ms[1] = acc[1] / (2.0 * reps);
        ms[2] = acc[2] / reps;
        ms[3] = acc[3] / (2.0 * reps);
        ms[4] = acc[4] / (2.0 * reps);
    }
    if (bytes) {
        // fine part, per element: the smoother's element data (inverse block in its storage,
        // or the Kronecker factors plus the exact blocks of the elements that keep them), r
        // and v (and p in mode 0: half the launches) read, p or s and M f written
        const double K4 = (double)K2 * K2;
        double blk = K4 * bw;
        if (krylov32_ && smoother_kind_ == 1) blk = K4 * 2;
        if (krylov32_ && smoother_kind_ == 2) blk = (4.0 * K2 + 2 * K) * 4 + (double)smoother_exact_ / N * K4 * 4;
        bytes[0] = (double)N * (blk + 4.5 * K2 * bw);
        // per element: operand, 3 metric coefficients, rhat or s, result; 4 face coefficients
        // and 2 incoming traces per face point; 4 face codes; the element sum
        bytes[1] = (double)N * ((6.0 * K2 + 24.0 * K) * bw + 16.0 + bw);
        // x, ph, sh, s, t, rhat read; x and r written; the element sum of r
        bytes[2] = (double)N * (8.0 * K2 * bw + bw);
        bytes[3] = coarse_bytes;
        // combination, per element: M f, the 5 smoothed row sums and the 5 coarse values
        // read, z and its 4K face traces (value, derivative) written, 4K destinations read
        bytes[4] = (double)N * ((7.0 * K2 + 8.0 * K) * bw + 5.0 * bw + 16.0 * K);
    }
    return {0, ""};
}

// y = A x on caller-owned device buffers without allocating: the operand's face traces
// go to the fixed scratch of noalloc.cu (shared by every call on this device).
Error Solver::apply_poisson_noalloc(const double* dx, double* dy) {
    if (!setup_done_) return {1, "not set up"};
    if (!dx || !dy) return {1, "null device buffer"};
    // the operator kernels move element rows in 16-byte pieces
    if ((reinterpret_cast<uintptr_t>(dx) | reinterpret_cast<uintptr_t>(dy)) % 16 != 0)
        return {1, "device buffers must be 16-byte aligned (cudaMalloc's alignment)"};
    DeviceState& d = *d_;
    const int N = mesh_.n_el, K = in_.knod;
    const size_t need = 2 * (size_t)N * 4 * K;
    if (need > kNoAllocScratchDoubles)
        return {1, "mesh too large for the fixed scratch of the allocation-free entry point: N_el*Knod = " +
                       std::to_string((size_t)N * K) + " exceeds " + std::to_string(kNoAllocScratchDoubles / 8)};
    HO2D_CUDA(cudaSetDevice(d.device), "cudaSetDevice");
    double* tv = d.noalloc_scratch;
    double* tg = tv + (size_t)N * 4 * K;
    const MfOp<double> op = make_op<double>(d, mesh_, K, false);
    HO2D_CUDA(mf_apply_op<double>(op, dx, tv, tg, dy, d.stream), "apply");
    HO2D_CUDA(cudaStreamSynchronize(d.stream), "sync");
    return {0, ""};
}

// y = A psi on the device in FP64 (the matrix-free Poisson operator), for checks
Error Solver::apply_poisson(const double* x, double* y) {
    if (!setup_done_) return {1, "not set up"};
    DeviceState& d = *d_;
    HO2D_CUDA(cudaSetDevice(d.device), "cudaSetDevice");
    const size_t nv = (size_t)mesh_.n_el * in_.knod * in_.knod;
    HO2D_CUDA(cudaStreamSynchronize(d.stream), "sync");
    HO2D_CUDA(cudaMemcpy(d.kv[4].get(), x, nv * 8, cudaMemcpyHostToDevice), "copy");
    const MfOp<double> op = make_op<double>(d, mesh_, in_.knod, false);
    HO2D_CUDA(mf_apply_op<double>(op, d.kv[4].as<double>(), d.kxtv.as<double>(), d.kxtg.as<double>(),
                                  d.kv[5].as<double>(), d.stream), "apply");
    HO2D_CUDA(cudaStreamSynchronize(d.stream), "sync");
    HO2D_CUDA(cudaMemcpy(y, d.kv[5].get(), nv * 8, cudaMemcpyDeviceToHost), "copy");
    return {0, ""};
}

// ------------------------------------------------------------------ data access
Error Solver::get_volume(int which, double* out) {
    if (!setup_done_) return {1, "not set up"};
    DeviceState& d = *d_;
    const size_t nv = (size_t)mesh_.n_el * in_.knod * in_.knod;
    HO2D_CUDA(cudaStreamSynchronize(d.stream), "sync");
    const void* src = nullptr;
    bool typed = false;
    switch (which) {
        case 0: src = d.omega.get(); break;
        case 1: src = d.psi64.get(); break;
        case 2: src = d.rhs_diff.get(); typed = true; break;
        case 3: src = d.rhs_adv.get(); typed = true; break;
        case 4: src = d.kout.get(); typed = true; break;
        case 5:
            std::copy(M_.J.begin(), M_.J.end(), out);
            return {0, ""};
        default: return {1, "unknown field"};
    }
    if (typed && stage32_) {
        std::vector<float> tmp(nv);
        HO2D_CUDA(cudaMemcpy(tmp.data(), src, nv * 4, cudaMemcpyDeviceToHost), "copy");
        std::copy(tmp.begin(), tmp.end(), out);
    } else {
        HO2D_CUDA(cudaMemcpy(out, src, nv * 8, cudaMemcpyDeviceToHost), "copy");
    }
    return {0, ""};
}

Error Solver::get_velocity(double* out) {
    if (!setup_done_) return {1, "not set up"};
    DeviceState& d = *d_;
    const size_t nv = (size_t)mesh_.n_el * in_.knod * in_.knod;
    HO2D_CUDA(cudaStreamSynchronize(d.stream), "sync");
    std::vector<double> u(nv), v(nv);
    if (stage32_) {
        std::vector<float> uf(nv), vf(nv);
        HO2D_CUDA(cudaMemcpy(uf.data(), d.u.get(), nv * 4, cudaMemcpyDeviceToHost), "copy");
        HO2D_CUDA(cudaMemcpy(vf.data(), d.v.get(), nv * 4, cudaMemcpyDeviceToHost), "copy");
        std::copy(uf.begin(), uf.end(), u.begin());
        std::copy(vf.begin(), vf.end(), v.begin());
    } else {
        HO2D_CUDA(cudaMemcpy(u.data(), d.u.get(), nv * 8, cudaMemcpyDeviceToHost), "copy");
        HO2D_CUDA(cudaMemcpy(v.data(), d.v.get(), nv * 8, cudaMemcpyDeviceToHost), "copy");
    }
    for (size_t i = 0; i < nv; ++i) {
        out[2 * i] = u[i];
        out[2 * i + 1] = v[i];
    }
    return {0, ""};
}

Error Solver::set_vorticity(const double* in) {
    if (!setup_done_) return {1, "not set up"};
    DeviceState& d = *d_;
    const size_t nv = (size_t)mesh_.n_el * in_.knod * in_.knod;
    HO2D_CUDA(cudaStreamSynchronize(d.stream), "sync");
    // staged on the device and checked there: finite everywhere, and whether it differs from
    // the current vorticity at all (a caller handing back the state it read continues the
    // trajectory, so the streamfunction history stays valid)
    if (d.vort_in.bytes() < nv * 8) HO2D_CUDA(d.vort_in.alloc(nv * 8), "alloc");
    if (!d.vort_flags.get()) HO2D_CUDA(d.vort_flags.alloc(2 * sizeof(int)), "alloc");
    HO2D_CUDA(cudaMemsetAsync(d.vort_flags.get(), 0, 2 * sizeof(int), d.stream), "memset");
    HO2D_CUDA(cudaMemcpyAsync(d.vort_in.get(), in, nv * 8, cudaMemcpyHostToDevice, d.stream), "copy");
    HO2D_CUDA(launch_vort_check(d.vort_in.as<double>(), d.omega.as<double>(), nv, d.vort_flags.as<int>(), d.stream),
              "check");
    int flags[2] = {0, 0};
    HO2D_CUDA(cudaMemcpyAsync(flags, d.vort_flags.get(), sizeof(flags), cudaMemcpyDeviceToHost, d.stream), "copy");
    HO2D_CUDA(cudaStreamSynchronize(d.stream), "sync");
    if (flags[0]) return {7, "non-finite value in the vorticity passed in"};
    if (hybrid_ && d.hvort[1].get()) {
        // hybrid operation (setsolnvort_d, src/HO_2D.cpp:4148-4170): the vorticity to blend
        // in at the end of the outer step; the previous one becomes the start value
        HO2D_CUDA(cudaMemcpy(d.hvort[0].get(), d.hvort[1].get(), nv * 8, cudaMemcpyDeviceToDevice), "copy");
        HO2D_CUDA(cudaMemcpy(d.hvort[1].get(), in, nv * 8, cudaMemcpyHostToDevice), "copy");
        return {0, ""};
    }
    if (flags[1]) {  // a new state: the trajectory restarts, no psi history to extrapolate from
        hist_count_ = 0;
        HO2D_CUDA(cudaMemcpyAsync(d.omega.get(), d.vort_in.get(), nv * 8, cudaMemcpyDeviceToDevice, d.stream), "copy");
    }
    // the stage input is the vorticity either way (a single ho2d_stage starts from it)
    if (stage32_) HO2D_CUDA(launch_copy_d2f(d.omega.as<double>(), d.w_stage.as<float>(), nv, d.stream), "d2f");
    else HO2D_CUDA(cudaMemcpyAsync(d.w_stage.get(), d.omega.get(), nv * 8, cudaMemcpyDeviceToDevice, d.stream), "copy");
    HO2D_CUDA(cudaStreamSynchronize(d.stream), "sync");
    return {0, ""};
}

static DeviceBuffer* boundary_buffer(DeviceState& d, int which) {
    switch (which) {
        case 0: return &d.bc_p;
        case 1: return &d.bc_nv;
        case 2: return &d.bc_pv;
        case 3: return &d.bc_d;
        case 4: return &d.bc_w;
        case 5: return &d.vjump;
        case 6: return &d.bc_adv;
        default: return nullptr;
    }
}

Error Solver::get_boundary(int which, double* out) {
    if (!setup_done_) return {1, "not set up"};
    DeviceBuffer* b = boundary_buffer(*d_, which);
    if (!b) return {1, "unknown boundary array"};
    HO2D_CUDA(cudaStreamSynchronize(d_->stream), "sync");
    HO2D_CUDA(cudaMemcpy(out, b->get(), (size_t)mesh_.n_eb * in_.knod * 8, cudaMemcpyDeviceToHost), "copy");
    return {0, ""};
}

Error Solver::set_boundary(int which, const double* in) {
    if (!setup_done_) return {1, "not set up"};
    DeviceBuffer* b = boundary_buffer(*d_, which);
    if (!b) return {1, "unknown boundary array"};
    HO2D_CUDA(cudaStreamSynchronize(d_->stream), "sync");
    HO2D_CUDA(cudaMemcpy(b->get(), in, (size_t)mesh_.n_eb * in_.knod * 8, cudaMemcpyHostToDevice), "copy");
    return {0, ""};
}

// Coordinates of the boundary flux points in the order of the boundary arrays
// ([N_eb][K][x, y], index e*K + (side/2)(K-2k-1) + k for face point k of edge e's face).
Error Solver::get_boundary_points(double* out) {
    if (!setup_done_) return {1, "not set up"};
    const int K = in_.knod, L = mesh_.lnod, lin = L - 1;
    for (int e = 0; e < mesh_.n_eb; ++e) {
        const int el = mesh_.be_el[e], side = mesh_.be_side[e], ijp = kF2I[side];
        const int dd = ijp / 2, t = ijp % 2;
        for (int k = 0; k < K; ++k) {
            double x = 0.0, y = 0.0;
            for (int j = 0; j < L; ++j)
                for (int i = 0; i < L; ++i) {
                    const int nd = mesh_.elem_nodes[el][tensor2fem(i, j, lin)];
                    const double w = dd == 0 ? B_.gbb[i * 2 + t] * B_.gsb[j * K + k] : B_.gsb[i * K + k] * B_.gbb[j * 2 + t];
                    x += w * mesh_.node_xy[2 * nd];
                    y += w * mesh_.node_xy[2 * nd + 1];
                }
            const size_t q = (size_t)e * K + (side / 2) * (K - 2 * k - 1) + k;
            out[2 * q] = x;
            out[2 * q + 1] = y;
        }
    }
    return {0, ""};
}

Error Solver::get_solution_points(double* out) {
    if (!setup_done_) return {1, "not set up"};
    const int N = mesh_.n_el, K = in_.knod, L = mesh_.lnod;
    for (int el = 0; el < N; ++el)
        for (int j = 0; j < K; ++j)
            for (int i = 0; i < K; ++i) {
                double x = 0.0, y = 0.0;
                for (int ly = 0; ly < L; ++ly)
                    for (int lx = 0; lx < L; ++lx) {
                        const int nd = mesh_.elem_nodes[el][tensor2fem(lx, ly, L - 1)];
                        const double wgt = B_.gsb[ly * K + j] * B_.gsb[lx * K + i];
                        x += wgt * mesh_.node_xy[2 * nd];
                        y += wgt * mesh_.node_xy[2 * nd + 1];
                    }
                const size_t p = ((size_t)el * K + j) * K + i;
                out[2 * p] = x;
                out[2 * p + 1] = y;
            }
    return {0, ""};
}

// the adjoint driver (adjoint_driver.cu) recomputes stages in FP64
template Error Solver::stage_t<double>(double, int, bool, bool);

}  // namespace ho2d
