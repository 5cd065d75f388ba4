// fr_launch.hpp -- argument blocks and launchers of the FR and Krylov kernels.
#pragma once

#include <cuda_runtime.h>

#include "device.cuh"

namespace ho2d {

// TP is the precision of psi and of everything derived from it (face values, common
// values, the gradient, the wall velocity jump); T that of omega and of the outputs. The
// FP32 stage keeps TP = double: the velocity is a derivative of psi, and the wall's
// velocity jump is divided by dt Re^-1 into the diffusion BC, which would carry FP32
// round-off of psi amplified by both.
template <typename T, typename TP = T>
struct VelocityArgs {
    const TP* psi;     // [N][K][K]
    const TP* psi_tv;  // psi face traces (values, normal derivatives)
    const TP* psi_tg;
    const T* w;       // stage input vorticity
    T* u;             // Cartesian velocity
    T* v;
    T* w_tv;          // omega face traces for the residual kernel
    T* w_tg;
    T* U_t;           // contravariant volumetric flux traces (U^xi on W/E, U^eta on S/N)
    double dt, re_inv;
};

template <typename T>
struct ResidualArgs {
    const T* w;       // stage input vorticity
    const T* u;
    const T* v;
    const T* w_tv;    // face traces written by the velocity kernel (all elements)
    const T* w_tg;
    const T* U_t;
    double dt, re_inv;
    int adv_type;     // 1 or 2
    int ti_type;      // 0 = stage only (no RK update), 1, 2, 4
    int stage;        // RK stage index
    double* omega;    // vorticity at time level n (FP64)
    double* acc;      // RK accumulator (FP64)
    T* w_next;        // next stage input (may alias nothing in the stage-only mode)
    double* w_next64 = nullptr;  // optional FP64 copy of the next stage input (FP32 stage)
    T* rhs_diff;      // optional outputs (nullptr to skip)
    T* rhs_adv;
    T* k_out;
};

template <typename T>
cudaError_t launch_trace(int K, int N, const T* f, T* tv, T* tg, const DevBases<T>& b, cudaStream_t s);
// The metric coefficients g11, g12, g22 of the contravariant gradient ([N][K][K], the
// Poisson operator's PoisGeom G11/G12/G22) in the stage kernels' precision.
template <typename T>
struct StageCoef {
    const T *G11, *G12, *G22;
};
// g, c and bp in the precision of psi (TP), bw in that of omega (T)
template <typename T, typename TP>
cudaError_t launch_velocity(int K, const FrGeom<TP>& g, const StageCoef<TP>& c, const DevBases<TP>& bp,
                            const DevBases<T>& bw, const BcArrays& bc, const VelocityArgs<T, TP>& a, cudaStream_t s);
template <typename T>
cudaError_t launch_residual(int K, const FrGeom<T>& g, const StageCoef<T>& c, const DevBases<T>& b,
                            const BcArrays& bc, const ResidualArgs<T>& a, cudaStream_t s);
template <typename T>
cudaError_t launch_poisson_rhs(int K, int N, const int* face_nb, const T* w, const T* J, const double* bsrc,
                               const double* bc_p, double* rhs, cudaStream_t s);
// Hybrid runs (problem type 11): the driver's open-boundary data at the start and end of
// the outer time step ([N_eb][K], zero off the open boundary), the inlets' normal velocity
// [N_eb], and the weights of the two ends at the stage's time.
struct HybridBc {
    const double *vn0 = nullptr, *vn1 = nullptr;  // normal velocity (outward)
    const double *vp0 = nullptr, *vp1 = nullptr;  // parallel velocity
    const double *w0 = nullptr, *w1 = nullptr;    // vorticity
    const double* inlet_nv = nullptr;
    double fac1 = 0.0, fac2 = 1.0;
};
cudaError_t launch_bc_update(int n_eb, int K, int ptype, double tc, double y_min, double y_max, const int* role,
                             const int* be_ijp, const int* sw_d, const double* edge_y, const BcArrays& bc,
                             const HybridBc& hb, cudaStream_t s);
// omega = (1 - wgt) omega + wgt (fac1 v0 + fac2 v1) (src/HO_2D.cpp:2183-2189); also into the
// stage input when w_stage is given (the first stage, whose input is omega itself)
template <typename T>
cudaError_t launch_hybrid_blend(size_t n, double* omega, T* w_stage, const double* wgt, const double* v0,
                                const double* v1, double fac1, double fac2, cudaStream_t s);

// ---- Krylov (krylov.cu)
// Static data of the matrix-free Poisson operator (the method-2 FR Laplacian with
// homogeneous boundary values), laid out so that an element reads only its own rows:
//   G11, G12, G22  [N][K2]  contravariant metric coefficients: (g_eta.g_eta)/J,
//                           -(g_xi.g_eta)/J, (g_xi.g_xi)/J
//   fa, fb         [N][4K]  face coefficients g.g/J_f and g1.g2/J_f of this element
//   nfa, nfb       [N][4K]  the same coefficients of the neighbour across each face point
//   code           [N][4]   interior face: nijp + 4 * rev; Dirichlet: -1;
//                           Neumann: -2 - boundary edge index
//   minv           [N_eb][K][K]  inverse of the common-value system of a Neumann edge
//   scat           [N][4K]  where a face point's traces go in the neighbour's incoming
//                           slots (-1 on the boundary): producers of an operand write
//                           its traces there, so the operator reads them as its own rows
template <typename T>
struct PoisGeom {
    int N = 0;
    const T *G11 = nullptr, *G12 = nullptr, *G22 = nullptr;
    const T *fa = nullptr, *fb = nullptr, *nfa = nullptr, *nfb = nullptr;
    const T* minv = nullptr;
    const int* code = nullptr;
    const int* scat = nullptr;
};

// Matrix-free FR Laplacian (the Poisson operator) plus the preconditioner's element data.
// Weight of the preconditioner's block smoothing step, z = e + w M (f - A e). Under-relaxing
// the exact (or fitted) block inverse pays: on the 256 x 512 cylinder O-grid at K = 6 the
// inner iterations per step fell by 18% (mixed) and 14% (FP64) from w = 1 to 0.7, and on
// the backward-facing step by 5%.
constexpr double kSmoothingWeight = 0.7;

template <typename T>
struct MfOp {
    int K;
    PoisGeom<T> g;
    DevBases<T> b;
    const T* dinv;          // [N][K2][K2] inverse diagonal blocks, transposed ([rs][ij])
    const T* rowsum;        // [N][5][K2] row sums of the 5 blocks of each element row
    const int* bcol;        // [N][5] element of each block (slot 0 = self, 1 + ijp = neighbours)
    // optional BF16 copy of dinv (bit patterns), read by the FP32 smoother when present
    const unsigned short* dinv_bf16 = nullptr;
    // optional Kronecker-sum smoother (FP32): factors [N][4K^2 + 2K], the compact index of
    // each element's exact block or -1 [N], and those exact blocks [n][K2][K2] ([rs][ij])
    const T* kron_f = nullptr;
    const int* kron_x = nullptr;
    const T* kron_exact = nullptr;
    // [N][5][K2] the smoother's element inverse applied to each block row sum (k_make_w)
    const T* W = nullptr;
    // FP32 operator kernels stage their inputs in shared memory by bulk copies
    // (apply_stage.cuh) instead of reading them through L2 prefetches
    int staged = 0;
    // host side: a second stream and two events; when set, each coarse cycle runs on the
    // second stream beside the fine part of the smoothing step (k_post_a)
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
};

template <typename T>
struct BicgVectors {
    T *x, *r, *rhat, *p, *v, *s, *t, *ph, *sh;
    const T* b;
    T *tv, *tg;    // incoming face traces of the operand of the next operator application
    T *xtv, *xtg;  // incoming face traces of x (initial residual)
    // element sums (N entries, zero-padded) of r, of v, and of p in two buffers that
    // alternate with the iteration count: the coarse right-hand sides P^T p and P^T s are
    // linear combinations of them, formed wherever they are read
    T *er, *ev, *ep[2];
    T* zf;  // the fine part M f of the current preconditioner application (k_post_a)
};

// The level-0 coarse right-hand side of one preconditioner application, formed where it
// is read: f0[e] = a[e] + cb b[e] + cc c[e].
//   mode 0 (p = r + beta (p - omega v)):  f0 = er + beta ep_prev - beta omega ev
//                                          (= er on the first iteration)
//   mode 1 (s = r - alpha v):             f0 = er - alpha ev
template <typename T>
struct F0 {
    const T *a, *b, *c;
    T cb, cc;
    __device__ __forceinline__ T operator[](int e) const { return a[e] + cb * b[e] + cc * c[e]; }
};

template <typename T>
__device__ __forceinline__ F0<T> f0_of(const BicgVectors<T>& v, const KrylovScalars* sc, int mode) {
    F0<T> f;
    f.a = v.er;
    f.b = f.c = v.er;  // zero weight unless set below
    f.cb = f.cc = T(0);
    if (mode == 1) {
        f.b = v.ev;
        f.cb = T(-sc->alpha);
    } else if (sc->it > 0) {
        const double beta = (sc->rho / sc->rho_old) * (sc->alpha / sc->omega);
        f.b = v.ep[sc->it & 1];
        f.c = v.ev;
        f.cb = T(beta);
        f.cc = T(-beta * sc->omega);
    }
    return f;
}

struct ReduceScratch {
    double* partials;    // [4 * max_blocks]
    unsigned* counter;   // 1 word, zero between launches
    KrylovScalars* sc;   // device scalars
};

// Row-padded sparse matrix on the device: row i holds w entries at [i * w, (i + 1) * w);
// padding entries have column 0 and value 0. col == nullptr means dense (column = k).
template <typename T>
struct DevEll {
    int n = 0, w = 0;
    int g = 1;  // lanes that cooperate on one row (a power of two <= 32)
    const int* col = nullptr;
    const T* val = nullptr;
    // the dense coarsest inverse of the FP32 preconditioner is stored as BF16 bit patterns
    // (rows padded to a multiple of 8 values); val is then null
    const unsigned short* val16 = nullptr;
};

// One level of the coarse hierarchy (level 0 = one value per element). Its V(1,1) cycle
// is f_next = M f and u = S f + Q u_next (host_amg.hpp has the formulas).
template <typename T>
struct CoarseLevel {
    int n = 0;
    DevEll<T> M, S, Q;  // empty on the coarsest level
    T* f = nullptr;     // right-hand side (zero-padded past n)
    T* u = nullptr;     // result
};

constexpr int kMaxLevels = 16;

// Preconditioner: nlev == 0 -> block-Jacobi; otherwise the two-level cycle (coarse.cu)
template <typename T>
struct Precond {
    int nlev = 0;
    double omega = 1.0;  // weight of the block-Jacobi smoothing step
    CoarseLevel<T> lev[kMaxLevels];
    DevEll<T> dense;  // row-major inverse of the coarsest operator (col == nullptr)
    // level-0 result delivered per element: ue5[5 el + s] = u0 of the element in block slot s
    // of element el (s = 0 itself, 1 + ijp its face neighbours; 0 where there is none);
    // u0dst[5 c + k] lists the slots element c's value goes to (-1: unused)
    T* ue5 = nullptr;
    const int* u0dst = nullptr;
};

// What the fine smoothing step needs of the coarse result: u0 at each element's five block
// slots (the whole cycle, level 0's up step included, ran before it).
template <typename T>
struct CoarseOut {
    const T* ue5 = nullptr;  // [N][5]: u0 of each element's five block slots (Precond::ue5)
};

// enqueues the coarse part of one preconditioner application (mode 0: on P^T p, mode 1:
// on P^T s, both formed from the element sums in v)
template <typename T>
cudaError_t coarse_cycle(const Precond<T>& pc, const BicgVectors<T>& v, const KrylovScalars* sc, int mode,
                         cudaStream_t s);
template <typename T>
int coarse_launches(const Precond<T>& pc);
// the whole cycle on a plain level-0 right-hand side: u0 -> pc.lev[0].u (coarse.cu)
template <typename T>
cudaError_t coarse_cycle_vec(const Precond<T>& pc, const T* f0, const KrylovScalars* sc, cudaStream_t s);
template <typename T>
int coarse_vec_launches(const Precond<T>& pc);
template <typename T>
CoarseOut<T> coarse_out(const Precond<T>& pc);
template <typename T>
int coarse_cycle_bytes(const Precond<T>& pc);

template <typename T>
cudaError_t krylov_init(const MfOp<T>& op, const BicgVectors<T>& v, const ReduceScratch& rs, cudaStream_t s);
template <typename T>
cudaError_t krylov_iteration(const MfOp<T>& op, const BicgVectors<T>& v, const ReduceScratch& rs, int max_iter,
                             const Precond<T>& pc, cudaStream_t s);
template <typename T>
int krylov_launches_per_iteration(const Precond<T>& pc);
// one iteration as krylov_iteration, in order on s, with the boundaries between its
// launches recorded on 10 events (coarse, fine smoothing part, combination, operator,
// coarse, fine smoothing part, combination, operator, update)
template <typename T>
cudaError_t krylov_iteration_timed(const MfOp<T>& op, const BicgVectors<T>& v, const ReduceScratch& rs, int max_iter,
                                   const Precond<T>& pc, cudaEvent_t* ev, cudaStream_t s);
// a whole solve (initial residual + device-side while loop of iterations) as a CUDA graph
template <typename T>
cudaError_t krylov_capture_solve(const MfOp<T>& op, const BicgVectors<T>& v, const ReduceScratch& rs, int max_iter,
                                 const Precond<T>& pc, cudaStream_t s, cudaGraph_t* graph_out);
// a whole mixed-precision solve (FP64 refinement around the FP32 BiCGSTAB, both loops on
// the device) as a CUDA graph; the refinement controls are read from the scalars
// (tol_outer, inner_tol, max_sweeps) and its results written there (krylov.cu)
cudaError_t krylov_capture_refined_solve(const MfOp<double>& A64, const MfOp<float>& A32,
                                         const BicgVectors<float>& v32, const ReduceScratch& rs, int max_iter,
                                         const Precond<float>& pc, double* psi64, const double* rhs, double* r64,
                                         double* xtv64, double* xtg64, cudaStream_t s, cudaGraph_t* graph_out);
int krylov_refined_launches(int sweeps, int inner_iters, const Precond<float>& pc);
// r = b - A x with ||r||^2 -> sc->rnorm2, ||b||^2 -> sc->bnorm2 (traces of x into xtv/xtg)
template <typename T>
cudaError_t mf_residual(const MfOp<T>& op, const double* b, const T* x, T* xtv, T* xtg, double* r,
                        const ReduceScratch& rs, cudaStream_t s);
// y = A x (traces of x into xtv/xtg first)
template <typename T>
cudaError_t mf_apply_op(const MfOp<T>& op, const T* x, T* xtv, T* xtg, T* y, cudaStream_t s);
// `reps` launches of the operator kernel alone on x whose traces are already in xtv/xtg
template <typename T>
cudaError_t mf_apply_only(const MfOp<T>& op, const T* x, const T* xtv, const T* xtg, T* y, int reps, cudaStream_t s);
int krylov_max_blocks(int K, int N);
// per-device set-up of the Krylov kernels for order K (krylov.cu): before the first launch
// or graph capture on the device
cudaError_t krylov_configure(int K);

// setup_device.cu: rows x cols values between row-strided arrays (idx, optional, gives the
// source row of each destination row), to FP32 or to BF16 (round to nearest even); the
// in-place dense inverse (row stride w) of the coarsest level
cudaError_t rows_to_f32(const double* src, long long ss, const int* idx, float* dst, long long ds, int rows, int cols,
                        cudaStream_t s);
cudaError_t rows_to_bf16(const double* src, long long ss, unsigned short* dst, long long ds, int rows, int cols,
                         cudaStream_t s);
cudaError_t dense_invert_device(double* a, int n, int w, cudaStream_t s, bool* singular);
// W = M rowsum for the 5 block slots of every element ([N][5][K2], T), with the smoother
// op selects (its element inverse M: exact blocks, BF16 blocks or Kronecker-sum factors)
template <typename T>
cudaError_t krylov_make_w(const MfOp<T>& op, T* W, KrylovScalars* sc, cudaStream_t s);

// out[0..1] = FP64 force on a body from its boundary points' precomputed coefficients
// (forces.cu): coef [npts][4], idx = index of each point in the boundary arrays
cudaError_t launch_body_force(int npts, const double* coef, const int* idx, const double* dwdn, const double* wall,
                              double* out, cudaStream_t s);

// elementwise helpers
cudaError_t launch_copy_d2f(const double* a, float* b, size_t n, cudaStream_t s);
// flags[0] |= some in[i] is not finite; flags[1] |= some in[i] differs bitwise from cur[i]
cudaError_t launch_vort_check(const double* in, const double* cur, size_t n, int* flags, cudaStream_t s);
cudaError_t launch_axpy_f2d(const float* e, double* x, size_t n, cudaStream_t s);  // x += e

}  // namespace ho2d
