// solver_state.hpp -- device state of one solver instance and the helpers that build its
// kernel arguments; shared by solver.cu (stage, step, Poisson) and adjoint_driver.cu.
#pragma once

#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <type_traits>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "device.cuh"
#include "fr_launch.hpp"
#include "host_amg.hpp"
#include "solver.hpp"

namespace ho2d {

// A named NVTX range for the lifetime of a scope: setup, steps, stages, Poisson solves,
// adjoint sweeps and VTK dumps show up by name in a profiler's timeline (ncu --nvtx
// --nvtx-include); without an attached tool each push and pop is a cheap no-op.
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

// Device copy of one row-padded matrix (FP64 and FP32 values) and of one coarse level.
struct EllBufs {
    DeviceBuffer col, v64, v32;
};
struct LevelBufs {
    EllBufs M, S, Q;
    DeviceBuffer f, u;
};

// A captured Krylov solve and the parameters baked into it.
struct SolveGraph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int max_iter = -1;
    void reset() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
        max_iter = -1;
    }
    ~SolveGraph() { reset(); }
};

// Device tables and scratch of the VTK node values (output_device.cu), built at the first
// dump after a setup.
struct VtkDevice {
    bool ready = false;
    int nbel = 0, nn = 0;
    DeviceBuffer sgb, t2f, nodes, node_xy, be_el, be_side, bases, bptr, bedges, nptr, nslot, sel, shape;
    DeviceBuffer om, ps, vx, vy, cvx, cvy, avg, samp, u64, v64;
};

struct DeviceState {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, evp0 = nullptr, evp1 = nullptr;
    cudaEvent_t prof_ev[10] = {};  // launch boundaries of a profiled Krylov iteration
    // the coarse cycle's stream beside the fine smoothing part, and its fork/join events
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    // connectivity and boundary tables
    DeviceBuffer face_nb, face_nijp, be_group, sw_p, sw_d, noslip, role, be_ijp;
    DevBases<double> b64;
    DevBases<float> b32;
    // metrics: xxi, xeta, yxi, yeta, J, fA, fB, fJ, fAn
    DeviceBuffer m64[9], m32[9];
    bool have32 = false;
    // boundary arrays (double)
    DeviceBuffer bc_p, bc_nv, bc_pv, bc_d, bc_w, vjump, bc_adv, edge_y, bsrc;
    // fields
    DeviceBuffer omega, acc, psi64, rhs, rres;
    DeviceBuffer vort_in, vort_flags;  // set_vorticity: the staged field and its check flags
    DeviceBuffer w_stage, psiT, u, v, psi_tv, psi_tg, w_tv, w_tg, U_t, rhs_diff, rhs_adv, kout;
    // FP64 value of the next stage input, written beside the FP32 one by the stage kernels
    // of HO2D_MIXED; the Poisson right-hand side of the stages after the first reads it
    DeviceBuffer w_stage64;
    // Poisson operator and Krylov workspace
    // Poisson operator: matrix-free; block-Jacobi inverses and block row sums from setup
    DeviceBuffer dinv64, dinv32, rowsum64, rowsum32, bcol;
    DeviceBuffer colsum64;  // block column sums (device assembly only)
    VtkDevice vtk;
    DeviceBuffer W64, W32, zf;  // smoother applied to the block row sums; fine part of z
    // level-0 coarse values per element slot (one buffer per precision: the cycle writes only
    // the slots that have a block neighbour, so a shared buffer would leave the other
    // precision's bytes in the rest), and where each value goes
    DeviceBuffer ue5, ue5_32, u0dst;
    DeviceBuffer dinv_bf16;  // BF16 copy of dinv for the FP32 smoother (HO2D_SMOOTHER_BF16=1)
    // Kronecker-sum smoother for the FP32 solve (HO2D_SMOOTHER_KRON=1): factors, exact-block
    // index per element, compact exact blocks
    DeviceBuffer kron_f, kron_x, kron_exact;
    // matrix-free operator data: G11, G12, G22, fa, fb, nfa, nfb, minv (PoisGeom)
    DeviceBuffer pg64[8], pg32[8], pcode, pscat;
    std::vector<double> pg_host[8];  // kept for the FP32 copies made on demand
    DeviceBuffer kv[10];  // r, rhat, p, v, s, t, ph, sh, x (inner), b (inner)
    // FP32 operator inputs staged by bulk copies (HO2D_OP_STAGE=1) instead of read through
    // L2 prefetches (the default: 51 against 60 us per launch on the 256 x 512 O-grid, K = 6)
    bool op_staged = false;
    DeviceBuffer esum[4];  // element sums of r, v, p (two alternating buffers), N + 4 entries
    DeviceBuffer ktv, ktg, kxtv, kxtg;  // face traces of the Krylov operand and of x
    DeviceBuffer partials, counter, scalars;
    KrylovScalars* h_sc = nullptr;
    // two-level preconditioner: per coarse level the row-padded cycle operators M, S, Q
    // (FP64 and FP32 values) and the level's f and u (sized for FP64, reused for FP32)
    using EllBufs = ho2d::EllBufs;
    using LevelBufs = ho2d::LevelBufs;
    std::vector<std::unique_ptr<LevelBufs>> lev;
    DeviceBuffer dense64, dense32;
    Precond<double> pc64;
    Precond<float> pc32;
    SolveGraph graph64, graph32;  // captured Krylov solves (FP64 solve, FP32 inner solve)
    SolveGraph graph_mixed;       // captured mixed-precision solve (refinement loop included)
    double* noalloc_scratch = nullptr;  // device address of noalloc.cu's fixed scratch
    DeviceBuffer l2flush;               // written between timed steps to evict L2
    DeviceBuffer fcoef, fidx, fout;     // body-force coefficients, boundary indices, result
    // hybrid runs: open-boundary normal / parallel velocity and vorticity at the outer step's
    // start and end [N_eb][K]; inlet normal velocity [N_eb]; the driver's vorticity at
    // start and end and the particle-to-grid weights [N][K][K]
    DeviceBuffer hyb[6], hyb_inlet_nv, hvort[3];
    // psi of each RK stage of the last three steps (the next solve's initial guess)
    DeviceBuffer psi_hist[3][4];

    ~DeviceState() {
        if (h_sc) cudaFreeHost(h_sc);
        for (cudaEvent_t e : {ev0, ev1, evp0, evp1})
            if (e) cudaEventDestroy(e);
        for (cudaEvent_t e : prof_ev)
            if (e) cudaEventDestroy(e);
        for (cudaEvent_t e : {ev_fork, ev_join})
            if (e) cudaEventDestroy(e);
        if (side) cudaStreamDestroy(side);
        if (stream) cudaStreamDestroy(stream);
    }
};

// Device state of the discrete adjoint, allocated on first use.
struct AdjointState {
    bool ready = false;
    // preconditioner of the transposed Poisson problem: column sums of A's blocks, and the
    // coarse hierarchy of (P^T A P)^T
    std::vector<std::unique_ptr<LevelBufs>> lev;
    DeviceBuffer dense64, dense32, rowsumT64, rowsumT32;
    Precond<double> pc64;
    Precond<float> pc32;
    // BiCGSTAB on A^T: x r rhat p v s t ph sh dir (sized for FP64), element sums, slots
    DeviceBuffer kv[10];
    DeviceBuffer f0, sv, sg, partials, counter, scalars;
    DeviceBuffer res64, x32, b32;  // refinement: FP64 residual, FP32 correction and right-hand side
    SolveGraph graph[2];           // captured transposed solves (FP64, FP32) and their operands
    const void* graph_x[2] = {nullptr, nullptr};
    const void* graph_b[2] = {nullptr, nullptr};
    // stage adjoint: lam of k (in), of omega (out) and the intermediate arrays
    DeviceBuffer lam_k, lw_out, lw_dir, lux, luy, lw_stage, lpsi_dir, lpsi, mu;
    DeviceBuffer swv, swg, sU, spv, spg;  // incoming slots [N][4K] (boundary entries stay zero)
    DeviceBuffer lbc_d, lbc_nv, lpv;      // boundary adjoints [N_eb][K]
    // time loop: lam of omega, per-stage results, checkpoints and one segment of stages
    DeviceBuffer lam, mus[4];
    std::vector<std::unique_ptr<DeviceBuffer>> ckpt;
    DeviceBuffer seg_w, seg_psi, wT, psiT;
    DeviceBuffer w32_save;  // the FP32 stage input kept across a single-stage adjoint (HO2D_MIXED)
    int nsteps = -1, every = 1;
    double t0 = 0.0;
    size_t state_bytes = 8;  // 8: FP64 state storage, 4: FP32
};

namespace {

template <typename T>
DevBases<T> make_dev_bases(const Bases& B) {
    DevBases<T> d;
    std::memset(&d, 0, sizeof(d));
    for (int i = 0; i < B.K * B.K; ++i) d.D[i] = T(B.D[i]);
    for (int i = 0; i < B.K * 2; ++i) {
        d.sbb[i] = T(B.sbb[i]);
        d.sbgb[i] = T(B.sbgb[i]);
        d.R[i] = T(B.R[i]);
        d.gR[i] = T(B.gR[i]);
    }
    d.gp[0] = T(B.gp[0]);
    d.gp[1] = T(B.gp[1]);
    return d;
}

template <typename T>
cudaError_t upload(DeviceBuffer& buf, const std::vector<T>& h) {
    cudaError_t e = buf.alloc(h.size() * sizeof(T));
    if (e != cudaSuccess || h.empty()) return e;
    return cudaMemcpy(buf.get(), h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice);
}

template <typename T>
cudaError_t upload_as(DeviceBuffer& buf, const std::vector<double>& h) {
    std::vector<T> c(h.begin(), h.end());
    return upload(buf, c);
}

// n rows of `len` values from h, each padded with zeros to `stride` values (the device
// layout of the per-element preconditioner data, padded_count in device.cuh), converted
// to T.
template <typename T>
std::vector<T> padded_rows(const std::vector<double>& h, size_t n, int len, int stride) {
    std::vector<T> out(n * (size_t)stride + 1, T(0));  // one spare value: never an empty allocation
    for (size_t r = 0; r < n; ++r)
        for (int i = 0; i < len; ++i) out[r * stride + i] = T(h[r * len + i]);
    return out;
}

inline cudaError_t upload_ell(DeviceState::EllBufs& b, const Ell& A) {
    cudaError_t e;
    if ((e = upload(b.col, A.col.empty() ? std::vector<int>{0} : A.col)) != cudaSuccess) return e;
    if ((e = upload(b.v64, A.val.empty() ? std::vector<double>{0.0} : A.val)) != cudaSuccess) return e;
    return upload_as<float>(b.v32, A.val.empty() ? std::vector<double>{0.0} : A.val);
}

// lanes per row for a row-padded matrix of width w: about w/2, a power of two in [4, 32]
inline int lanes_for(int w) {
    int g = 4;
    while (g < 32 && 2 * g <= std::max(1, w / 2)) g *= 2;
    return g;
}

template <typename TM>
DevEll<TM> view(const DeviceState::EllBufs& b, const Ell& A, int g, bool f32) {
    DevEll<TM> v;
    v.n = A.n;
    v.w = A.w;
    v.g = g;
    v.col = b.col.as<int>();
    v.val = f32 ? (const TM*)b.v32.get() : (const TM*)b.v64.get();
    return v;
}


template <typename T>
FrGeom<T> geom_of(DeviceState& d, const Mesh& m, bool f32) {
    DeviceBuffer* mm = f32 ? d.m32 : d.m64;
    FrGeom<T> g;
    g.N = m.n_el;
    g.n_eb = m.n_eb;
    g.face_nb = d.face_nb.as<int>();
    g.face_nijp = d.face_nijp.as<int>();
    g.xxi = mm[0].as<T>();
    g.xeta = mm[1].as<T>();
    g.yxi = mm[2].as<T>();
    g.yeta = mm[3].as<T>();
    g.J = mm[4].as<T>();
    g.fA = mm[5].as<T>();
    g.fB = mm[6].as<T>();
    g.fJ = mm[7].as<T>();
    g.fAn = mm[8].as<T>();
    g.be_group = d.be_group.as<int>();
    g.sw_p = d.sw_p.as<int>();
    g.sw_d = d.sw_d.as<int>();
    g.noslip = d.noslip.as<int>();
    g.nminv = (f32 ? d.pg32[7] : d.pg64[7]).as<T>();
    return g;
}

template <typename T>
StageCoef<T> stage_coef(DeviceState& d, bool f32) {
    const DeviceBuffer* pg = f32 ? d.pg32 : d.pg64;
    return {pg[0].as<T>(), pg[1].as<T>(), pg[2].as<T>()};
}

template <typename T>
MfOp<T> make_op(DeviceState& d, const Mesh& m, int K, bool f32) {
    MfOp<T> op;
    op.K = K;
    op.g.N = m.n_el;
    const DeviceBuffer* pg = f32 ? d.pg32 : d.pg64;
    op.g.G11 = pg[0].as<T>();
    op.g.G12 = pg[1].as<T>();
    op.g.G22 = pg[2].as<T>();
    op.g.fa = pg[3].as<T>();
    op.g.fb = pg[4].as<T>();
    op.g.nfa = pg[5].as<T>();
    op.g.nfb = pg[6].as<T>();
    op.g.minv = pg[7].as<T>();
    op.g.code = d.pcode.as<int>();
    op.g.scat = d.pscat.as<int>();
    op.b = *reinterpret_cast<const DevBases<T>*>(f32 ? (const void*)&d.b32 : (const void*)&d.b64);
    op.dinv = f32 ? (const T*)d.dinv32.get() : (const T*)d.dinv64.get();
    op.dinv_bf16 = f32 ? (const unsigned short*)d.dinv_bf16.get() : nullptr;
    const bool kron = f32 && d.kron_f.get();
    op.kron_f = kron ? (const T*)d.kron_f.get() : nullptr;
    op.kron_x = kron ? d.kron_x.as<int>() : nullptr;
    op.kron_exact = kron ? (const T*)d.kron_exact.get() : nullptr;
    op.rowsum = f32 ? (const T*)d.rowsum32.get() : (const T*)d.rowsum64.get();
    op.bcol = d.bcol.as<int>();
    op.W = f32 ? (const T*)d.W32.get() : (const T*)d.W64.get();
    op.staged = f32 && d.op_staged ? 1 : 0;
    op.side = d.side;
    op.ev_fork = d.ev_fork;
    op.ev_join = d.ev_join;
    return op;
}

template <typename T>
BicgVectors<T> krylov_vectors(DeviceState& d, T* x, const T* b) {
    BicgVectors<T> v;
    v.x = x;
    v.r = d.kv[0].as<T>();
    v.rhat = d.kv[1].as<T>();
    v.p = d.kv[2].as<T>();
    v.v = d.kv[3].as<T>();
    v.s = d.kv[4].as<T>();
    v.t = d.kv[5].as<T>();
    v.ph = d.kv[6].as<T>();
    v.sh = d.kv[7].as<T>();
    v.b = b;
    v.tv = d.ktv.as<T>();
    v.tg = d.ktg.as<T>();
    v.xtv = d.kxtv.as<T>();
    v.xtg = d.kxtg.as<T>();
    v.er = d.esum[0].as<T>();
    v.ev = d.esum[1].as<T>();
    v.ep[0] = d.esum[2].as<T>();
    v.ep[1] = d.esum[3].as<T>();
    v.zf = d.zf.as<T>();
    return v;
}


}  // namespace

// Inside Solver members: return the first failing status.
#define HO2D_TRY(expr)                 \
    do {                               \
        Error _e = (expr);             \
        if (_e.code) return _e;        \
    } while (0)
#define HO2D_CUDA(call, what) HO2D_TRY(cuda((call), what))

}  // namespace ho2d
