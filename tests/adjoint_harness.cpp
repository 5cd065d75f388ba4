// adjoint_harness.cpp -- host build of the adjoint's element bodies, for CPU tests.
//
// Compiles ho-cxx_b200/csrc/adjoint_chain.cuh with g++ and runs each body over all
// elements with one thread per element, in the order the GPU launches run them
// (residual adjoint, then velocity adjoint, then the psi gather; Poisson transpose =
// body + gather). The test (test_adjoint_cpu.py) feeds it the oracle's geometry and
// forward state and compares the results with complex-step derivatives of the oracle.
// Never part of the library.
#include <cstring>
#include <vector>

#include "adjoint_chain.cuh"

using namespace ho2d;

namespace {

struct HostGeom {
    FrGeom<double> g;
    DevBases<double> b;
};

// met: [5][N*K2] xxi, xeta, yxi, yeta, J; fmet: [4][N*4K] fA, fB, fJ, fAn;
// bases: D[64], sbb[16], sbgb[16], R[16], gR[16], gp[2]
HostGeom make_geom(int K, int N, int n_eb, const int* face_nb, const int* face_nijp, const double* met,
                   const double* fmet, const int* be_group, const int* sw_p, const int* sw_d, const int* noslip,
                   const double* bases) {
    HostGeom h;
    const size_t nv = (size_t)N * K * K, nf = (size_t)N * 4 * K;
    h.g.N = N;
    h.g.n_eb = n_eb;
    h.g.face_nb = face_nb;
    h.g.face_nijp = face_nijp;
    h.g.xxi = met;
    h.g.xeta = met + nv;
    h.g.yxi = met + 2 * nv;
    h.g.yeta = met + 3 * nv;
    h.g.J = met + 4 * nv;
    h.g.fA = fmet;
    h.g.fB = fmet + nf;
    h.g.fJ = fmet + 2 * nf;
    h.g.fAn = fmet + 3 * nf;
    h.g.be_group = be_group;
    h.g.sw_p = sw_p;
    h.g.sw_d = sw_d;
    h.g.noslip = noslip;
    std::memcpy(&h.b, bases, sizeof(DevBases<double>));
    return h;
}

// omega face values and the volumetric-flux face values of every element, as the
// forward velocity kernel writes them
template <int K>
void forward_traces(const HostGeom& h, const double* w, const double* u, const double* v, std::vector<double>& w_tv,
                    std::vector<double>& U_t) {
    constexpr int K2 = K * K, NF = 4 * K;
    const int N = h.g.N;
    w_tv.assign((size_t)N * NF, 0.0);
    U_t.assign((size_t)N * NF, 0.0);
    for (int el = 0; el < N; ++el) {
        double ux[K2], uy[K2];
        for (int ij = 0; ij < K2; ++ij) {
            const int p = el * K2 + ij;
            ux[ij] = u[p] * h.g.yeta[p] - v[p] * h.g.xeta[p];
            uy[ij] = -u[p] * h.g.yxi[p] + v[p] * h.g.xxi[p];
        }
        for (int o = 0; o < NF; ++o) {
            const int ijp = o / K, k = o % K, lr = ijp & 1;
            double tv = 0, ut = 0;
            for (int m = 0; m < K; ++m) {
                const int idx = ijp < 2 ? k * K + m : m * K + k;
                tv += w[el * K2 + idx] * h.b.sbb[m * 2 + lr];
                ut += (ijp < 2 ? ux[idx] : uy[idx]) * h.b.sbb[m * 2 + lr];
            }
            w_tv[(size_t)el * NF + o] = tv;
            U_t[(size_t)el * NF + o] = ut;
        }
    }
}

template <int K>
int stage_adjoint_k(const HostGeom& h, const double* w, const double* u, const double* v, const double* bc_w,
                    const double* bc_nv, const double* lam_k, double dt, double re_inv, double* lw_stage, double* lpsi,
                    double* lpv, int adv_type) {
    constexpr int K2 = K * K, NF = 4 * K;
    const int N = h.g.N, neb = h.g.n_eb;
    std::vector<double> w_tv, U_t;
    forward_traces<K>(h, w, u, v, w_tv, U_t);
    const size_t nv = (size_t)N * K2, nf = (size_t)N * NF;
    std::vector<double> lw_dir(nv), lux(nv), luy(nv), lpsi_dir(nv);
    std::vector<double> swv(nf, 0.0), swg(nf, 0.0), sU(nf, 0.0), spv(nf, 0.0), spg(nf, 0.0);
    std::vector<double> lbc_d((size_t)neb * K, 0.0), lbc_nv((size_t)neb * K, 0.0);
    StageAdjArgs<double> a;
    a.w = w;
    a.u = u;
    a.v = v;
    a.w_tv = w_tv.data();
    a.U_t = U_t.data();
    a.bc_w = bc_w;
    a.bc_nv = bc_nv;
    a.lam_k = lam_k;
    a.lw_dir = lw_dir.data();
    a.lux = lux.data();
    a.luy = luy.data();
    a.slot_wv = swv.data();
    a.slot_wg = swg.data();
    a.slot_U = sU.data();
    a.lbc_d = lbc_d.data();
    a.lbc_nv = lbc_nv.data();
    a.lw_stage = lw_stage;
    a.lpsi_dir = lpsi_dir.data();
    a.slot_pv = spv.data();
    a.slot_pg = spg.data();
    a.lpv = lpv;
    a.dt = dt;
    a.re_inv = re_inv;
    a.adv_type = adv_type;
    const ElemCtx<1> c{0};
    {
        auto* s = new ResidualAdjScratch<K, double>;
        for (int el = 0; el < N; ++el) residual_adjoint_body<K, double>(c, true, el, h.g, h.b, a, *s);
        delete s;
    }
    {
        auto* s = new VelocityAdjScratch<K, double>;
        for (int el = 0; el < N; ++el) velocity_adjoint_body<K, double>(c, true, el, h.g, h.b, a, *s);
        delete s;
    }
    GatherScratch<K, double> gs;
    for (int el = 0; el < N; ++el) gather_body<K, double>(c, true, el, h.b, lpsi_dir.data(), spv.data(), spg.data(), lpsi, gs);
    return 0;
}

template <int K>
int poisson_transpose_k(const HostGeom& h, const double* x, double* y) {
    constexpr int K2 = K * K, NF = 4 * K;
    const int N = h.g.N;
    std::vector<double> dir((size_t)N * K2), sv((size_t)N * NF, 0.0), sg((size_t)N * NF, 0.0);
    const ElemCtx<1> c{0};
    auto* s = new LapAdjScratch<K, double>;
    for (int el = 0; el < N; ++el) poisson_transpose_body<K, double>(c, true, el, h.g, h.b, x, dir.data(), sv.data(), sg.data(), *s);
    delete s;
    GatherScratch<K, double> gs;
    for (int el = 0; el < N; ++el) gather_body<K, double>(c, true, el, h.b, dir.data(), sv.data(), sg.data(), y, gs);
    return 0;
}

#define HARNESS_DISPATCH(K, CALL)                     \
    switch (K) {                                      \
        case 2: { constexpr int KK = 2; return CALL; } \
        case 3: { constexpr int KK = 3; return CALL; } \
        case 4: { constexpr int KK = 4; return CALL; } \
        case 5: { constexpr int KK = 5; return CALL; } \
        case 6: { constexpr int KK = 6; return CALL; } \
        default: return 1;                            \
    }

}  // namespace

extern "C" int stage_adjoint_host(int K, int N, int n_eb, const int* face_nb, const int* face_nijp, const double* met,
                                  const double* fmet, const int* be_group, const int* sw_p, const int* sw_d,
                                  const int* noslip, const double* bases, const double* w, const double* u,
                                  const double* v, const double* bc_w, const double* bc_nv, const double* lam_k,
                                  double dt, double re_inv, double* lw_stage, double* lpsi, double* lpv,
                                  int adv_type) {
    const HostGeom h = make_geom(K, N, n_eb, face_nb, face_nijp, met, fmet, be_group, sw_p, sw_d, noslip, bases);
    HARNESS_DISPATCH(K, stage_adjoint_k<KK>(h, w, u, v, bc_w, bc_nv, lam_k, dt, re_inv, lw_stage, lpsi, lpv, adv_type))
}

extern "C" int poisson_transpose_host(int K, int N, int n_eb, const int* face_nb, const int* face_nijp,
                                      const double* met, const double* fmet, const int* be_group, const int* sw_p,
                                      const int* sw_d, const int* noslip, const double* bases, const double* x,
                                      double* y) {
    const HostGeom h = make_geom(K, N, n_eb, face_nb, face_nijp, met, fmet, be_group, sw_p, sw_d, noslip, bases);
    HARNESS_DISPATCH(K, poisson_transpose_k<KK>(h, x, y))
}
