// host_harness.cpp -- host build of the library's setup code (ho-cxx_b200/csrc/host_io.cpp,
// host_setup.cpp, host_hybrid.cpp, host_amg.cpp) for CPU tests against the reference's own
// setup arrays and the coarse hierarchy's defining identities:
// a case is set up from an input.dat + Gmsh mesh, or from the arrays a hybrid driver
// passes, and its tables are read out by name. Never part of the library.
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "host.hpp"
#include "host_amg.hpp"
#include "kron_apply.cuh"

namespace {

struct Case {
    ho2d::Input in;
    ho2d::Mesh m;
    ho2d::Bases B;
    ho2d::Metrics M;
    ho2d::BoundaryConditions bc;
    ho2d::PoissonOperator op;
    std::vector<double> nrm;  // open-edge normals (problem type 11)
    std::vector<double> tmp;
    ho2d::CoarseHierarchy H;
};

const ho2d::Csr* level_matrix(const Case* c, int level, const std::string& which) {
    if (level < 0 || level >= (int)c->H.levels.size()) return nullptr;
    const ho2d::AmgLevel& L = c->H.levels[level];
    if (which == "A") return &L.A;
    if (which == "P") return &L.P;
    if (which == "R") return &L.R;
    if (which == "M") return &L.M;
    if (which == "S") return &L.S;
    if (which == "Q") return &L.Q;
    return nullptr;
}

// the steps after the mesh, in the order of Solver::setup_from_mesh
int finish(Case* c) {
    ho2d::Error e = ho2d::make_bases(c->in.knod, c->m.lnod, c->B);
    if (e.code) return e.code;
    ho2d::make_metrics(c->m, c->B, c->M);
    e = ho2d::setup_bcs(c->in, c->m, c->B, c->bc);
    if (e.code) return e.code;
    ho2d::assemble_poisson(c->m, c->B, c->M, c->bc, c->op, /*keep_blocks=*/true);
    if (c->in.problem_type == 11) ho2d::open_normals(c->m, c->B, c->M, c->bc, c->nrm);
    return 0;
}

void* done(Case* c, int code, int* out) {
    *out = code;
    if (code) {
        delete c;
        return nullptr;
    }
    return c;
}

template <typename T>
long copy_out(const std::vector<T>& v, double* out) {
    if (out)
        for (size_t i = 0; i < v.size(); ++i) out[i] = (double)v[i];
    return (long)v.size();
}

}  // namespace

extern "C" void* case_from_input(const char* path, int* code) {
    auto* c = new Case;
    ho2d::Error e = ho2d::read_input(path, c->in);
    if (!e.code) {
        std::string mp = c->in.mesh_file;
        if (!mp.empty() && mp[0] != '/') mp = c->in.base_dir + "/" + mp;
        e = ho2d::read_msh(mp, c->in.occ, c->m);
    }
    return done(c, e.code ? e.code : finish(c), code);
}

// A hybrid case (problem type 11, Knod knod) from the arrays of load_mesh_arrays_d and
// load_inout_arrays_d, then process_mesh_input.
extern "C" void* case_from_arrays(int knod, int iorder, int nxy, const double* xy, int nidx, const int* idx,
                                  int nwall, const int* wall, int nopen, const int* open, int ninval,
                                  const double* velin, int nin, const int* idxin, int noutval, const double* velout,
                                  int nout, const int* idxout, int* code) {
    auto* c = new Case;
    c->in.knod = knod;
    c->in.problem_type = 11;
    c->in.adv_type = 2;
    c->in.ti_type = 2;
    ho2d::Error e = ho2d::mesh_from_arrays(iorder, nxy, xy, nidx, idx, nwall, wall, nopen, open, c->m);
    if (!e.code) e = ho2d::add_boundary_arrays(c->m, "inlet", nin, idxin, ninval, velin);
    if (!e.code) e = ho2d::add_boundary_arrays(c->m, "outlet", nout, idxout, noutval, velout);
    if (!e.code) e = ho2d::process_mesh(c->m);
    return done(c, e.code ? e.code : finish(c), code);
}

extern "C" void case_free(void* h) { delete static_cast<Case*>(h); }

// N_el, Knod, Lnod, N_eb, boundary groups, Poisson entries above the 1e-14 filter
extern "C" void case_dims(void* h, long* d) {
    const Case* c = static_cast<Case*>(h);
    d[0] = c->m.n_el;
    d[1] = c->in.knod;
    d[2] = c->m.lnod;
    d[3] = c->m.n_eb;
    d[4] = (long)c->m.group_names.size();
    d[5] = (long)c->op.nnz;
}

extern "C" int case_group_name(void* h, int g, char* buf, int cap) {
    const Case* c = static_cast<Case*>(h);
    if (g < 0 || g >= (int)c->m.group_names.size() || cap < 1) return -1;
    std::strncpy(buf, c->m.group_names[g].c_str(), cap - 1);
    buf[cap - 1] = 0;
    return 0;
}

// Length of the named array (and its values as doubles when out is not null); -1 if unknown.
extern "C" long case_get(void* h, const char* name, double* out) {
    Case* c = static_cast<Case*>(h);
    const std::string n = name;
    const ho2d::Mesh& m = c->m;
    const ho2d::Bases& B = c->B;
    const ho2d::Metrics& M = c->M;
    const ho2d::BoundaryConditions& bc = c->bc;
    const ho2d::PoissonOperator& op = c->op;
    if (n == "node_xy") return copy_out(m.node_xy, out);
    if (n == "elem_nodes" || n == "bedge_nodes") {  // [N][Lnod^2] node slots, [N_eb][Lnod] edge nodes
        std::vector<int> flat;
        if (n == "elem_nodes")
            for (const auto& e : m.elem_nodes) flat.insert(flat.end(), e.begin(), e.end());
        else
            for (int e = 0; e < m.n_eb; ++e) flat.insert(flat.end(), m.edge_nodes[e].begin(), m.edge_nodes[e].end());
        return copy_out(flat, out);
    }
    if (n == "nbr") return copy_out(m.nbr, out);
    if (n == "nbr_side") return copy_out(m.nbr_side, out);
    if (n == "bidx") return copy_out(m.bidx, out);
    if (n == "be_el") return copy_out(m.be_el, out);
    if (n == "be_side") return copy_out(m.be_side, out);
    if (n == "be_group") return copy_out(m.be_group, out);
    if (n == "xs") return copy_out(B.xs, out);
    if (n == "w") return copy_out(B.w, out);
    if (n == "sbb") return copy_out(B.sbb, out);
    if (n == "sbgb") return copy_out(B.sbgb, out);
    if (n == "D") return copy_out(B.D, out);
    if (n == "R") return copy_out(B.R, out);
    if (n == "gR") return copy_out(B.gR, out);
    if (n == "J") return copy_out(M.J, out);
    if (n == "xxi") return copy_out(M.xxi, out);
    if (n == "xeta") return copy_out(M.xeta, out);
    if (n == "yxi") return copy_out(M.yxi, out);
    if (n == "yeta") return copy_out(M.yeta, out);
    if (n == "G") return copy_out(M.G, out);
    if (n == "GB") return copy_out(M.GB, out);
    if (n == "fA") return copy_out(M.fA, out);
    if (n == "fB") return copy_out(M.fB, out);
    if (n == "fJ") return copy_out(M.fJ, out);
    if (n == "fAn") return copy_out(M.fAn, out);
    if (n == "sw_p") return copy_out(bc.sw_p, out);
    if (n == "sw_d") return copy_out(bc.sw_d, out);
    if (n == "noslip") return copy_out(bc.noslip, out);
    if (n == "role") return copy_out(bc.role, out);
    if (n == "bc_p") return copy_out(bc.bc_p, out);
    if (n == "bc_nv") return copy_out(bc.bc_nv, out);
    if (n == "bc_pv") return copy_out(bc.bc_pv, out);
    if (n == "bc_d") return copy_out(bc.bc_d, out);
    if (n == "blocks") return copy_out(op.blocks, out);
    if (n == "block_col") return copy_out(op.block_col, out);
    if (n == "bsrc") return copy_out(op.bsrc, out);
    if (n == "dinv") return copy_out(op.dinv, out);
    if (n == "open_normals") return copy_out(c->nrm, out);
    if (n == "areas") {
        c->tmp.assign((size_t)m.n_el * B.K * B.K, 0.0);
        ho2d::solution_areas(B, M, m.n_el, c->tmp.data());
        return copy_out(c->tmp, out);
    }
    if (n == "openpts") {
        c->tmp.assign((size_t)ho2d::open_point_count(m, B.K), 0.0);
        ho2d::open_points(m, B, c->tmp.data());
        return copy_out(c->tmp, out);
    }
    return -1;
}

// The block reductions assemble_poisson streams (row sums, column sums, block sums) against
// the same sums taken from the kept blocks in the order their consumers summed them when
// the blocks were stored (rs, then ij ascending; rows ascending; stored order), and a second
// assembly without the blocks against the first. Returns the number of values that differ
// in any bit, or -1 if the assembly without blocks kept some.
extern "C" long case_check_block_reductions(void* h) {
    const Case* c = static_cast<Case*>(h);
    const ho2d::PoissonOperator& op = c->op;
    const int K2 = op.K2;
    const size_t nb = (size_t)c->m.n_el * 5;
    long bad = 0;
    for (size_t eb = 0; eb < nb; ++eb) {
        const double* blk = &op.blocks[eb * K2 * K2];
        std::vector<double> rs(K2, 0.0);
        double tot = 0.0;
        for (int r = 0; r < K2; ++r)
            for (int ij = 0; ij < K2; ++ij) rs[ij] += blk[r * K2 + ij];
        for (int q = 0; q < K2 * K2; ++q) tot += blk[q];
        for (int x = 0; x < K2; ++x) {
            double acc = 0.0;
            for (int r = 0; r < K2; ++r) acc += blk[(size_t)x * K2 + r];
            bad += std::memcmp(&acc, &op.colsum[eb * K2 + x], 8) != 0;
            bad += std::memcmp(&rs[x], &op.rowsum[eb * K2 + x], 8) != 0;
        }
        bad += std::memcmp(&tot, &op.bsum[eb], 8) != 0;
    }
    ho2d::PoissonOperator s;
    ho2d::assemble_poisson(c->m, c->B, c->M, c->bc, s);
    if (!s.blocks.empty()) return -1;
    auto diff = [](const std::vector<double>& a, const std::vector<double>& b) {
        if (a.size() != b.size()) return (long)std::max(a.size(), b.size());
        return (long)(std::memcmp(a.data(), b.data(), a.size() * 8) != 0);
    };
    bad += diff(s.dinv, op.dinv) + diff(s.rowsum, op.rowsum) + diff(s.colsum, op.colsum) + diff(s.bsum, op.bsum) +
           diff(s.bsrc, op.bsrc) + (s.nnz != op.nnz) + (s.block_col != op.block_col);
    return bad;
}

// The coarse hierarchy of the case's P0 operator (p0_coarse_operator, build_coarse_hierarchy)
// with the given dense-solve thresholds; returns the number of levels, or -code.
extern "C" int case_build_hierarchy(void* h, int dense_max, int dense_max_first) {
    Case* c = static_cast<Case*>(h);
    const ho2d::Csr A1 = ho2d::p0_coarse_operator(c->op, c->m.n_el);
    const ho2d::Error e = ho2d::build_coarse_hierarchy(A1, c->H, dense_max, dense_max_first);
    return e.code ? -e.code : (int)c->H.levels.size();
}

// Matrix `which` (A, P, R, M, S, Q) of a level as CSR: dims = rows, columns, entries; the
// arrays are filled when not null. Returns 0, or -1 for an unknown level or matrix.
extern "C" int case_level_csr(void* h, int level, const char* which, long* dims, int* ptr, int* col, double* val) {
    const ho2d::Csr* A = level_matrix(static_cast<Case*>(h), level, which);
    if (!A) return -1;
    dims[0] = A->n;
    dims[1] = A->m;
    dims[2] = (long)A->val.size();
    if (ptr) std::copy(A->ptr.begin(), A->ptr.end(), ptr);
    if (col) std::copy(A->col.begin(), A->col.end(), col);
    if (val) std::copy(A->val.begin(), A->val.end(), val);
    return 0;
}

// The same matrix as ELL (to_ell): dims = rows, columns, row width.
extern "C" int case_level_ell(void* h, int level, const char* which, long* dims, int* col, double* val) {
    const ho2d::Csr* A = level_matrix(static_cast<Case*>(h), level, which);
    if (!A) return -1;
    const ho2d::Ell E = ho2d::to_ell(*A);
    dims[0] = E.n;
    dims[1] = E.m;
    dims[2] = E.w;
    if (col) std::copy(E.col.begin(), E.col.end(), col);
    if (val) std::copy(E.val.begin(), E.val.end(), val);
    return 0;
}

// SPAI-0 weights of a level (length = its rows), or the dense inverse of the last level
// (level = -1; length n_dense^2). Returns the length, or -1.
extern "C" long case_level_vec(void* h, int level, double* out) {
    const Case* c = static_cast<Case*>(h);
    const std::vector<double>* v = level == -1 ? &c->H.dense_inv
                                  : (level >= 0 && level < (int)c->H.levels.size() ? &c->H.levels[level].m : nullptr);
    if (!v) return -1;
    if (out) std::copy(v->begin(), v->end(), out);
    return (long)v->size();
}

// split_open_velocities of the driver's open-boundary velocities into vn, vp [N_eb][K]
extern "C" void case_split_open(void* h, const double* xyvel, double* vn, double* vp) {
    const Case* c = static_cast<Case*>(h);
    ho2d::split_open_velocities(c->m, c->in.knod, c->nrm, xyvel, vn, vp);
}

// ---- Kronecker-sum smoother pieces (host_kron.cpp)

extern "C" int kron_eigs(int n, const double* A, double* lam) { return ho2d::real_eigenvalues(n, A, lam) ? 1 : 0; }

extern "C" int kron_vecs(int n, const double* A, const double* lam, double* V) {
    return ho2d::eigenvectors(n, A, lam, V) ? 1 : 0;
}

// The fit of element el's diagonal block (from the kept blocks): applies the fitted inverse
// to r ([j][i]) into z and returns ||I - M D||_2 in *defect; returns 1, or 0 if rejected.
extern "C" int case_kron(void* h, int el, const double* r, double* z, double* defect) {
    const Case* c = static_cast<Case*>(h);
    const int K2 = c->op.K2, K = c->in.knod;
    const double* blk = &c->op.blocks[(size_t)el * 5 * K2 * K2];  // slot 0, [rs][ij]
    std::vector<double> D((size_t)K2 * K2);
    for (int ij = 0; ij < K2; ++ij)
        for (int rs = 0; rs < K2; ++rs) D[(size_t)ij * K2 + rs] = blk[(size_t)rs * K2 + ij];
    ho2d::KronFit f;
    if (!ho2d::kron_fit(K, D.data(), f)) return 0;
    ho2d::kron_apply(f, r, z);
    *defect = ho2d::kron_defect(f, D.data());
    return 1;
}

// assemble_poisson again with the Kronecker-sum smoother data; returns the number of
// elements that keep the exact inverse block, and their defects in defect[N] if not null
extern "C" long case_kron_smoother(void* h, double* defect) {
    Case* c = static_cast<Case*>(h);
    ho2d::PoissonOperator op;
    ho2d::KronSmoother ks;
    ho2d::assemble_poisson(c->m, c->B, c->M, c->bc, op, false, &ks);
    long n = 0;
    for (int el = 0; el < c->m.n_el; ++el) {
        n += ks.exact[el];
        if (defect) defect[el] = ks.defect[el];
    }
    return n;
}

// make_bases(K, L) alone: the named table (xs, w, sbb, sbgb, D, R, gR, gsb, gsgb, gbb, gbgb,
// gp) into out when not null; returns its length, or -code / -100 for an unknown name.
extern "C" long bases_get(int K, int L, const char* name, double* out) {
    ho2d::Bases B;
    const ho2d::Error e = ho2d::make_bases(K, L, B);
    if (e.code) return -e.code;
    const std::string n = name;
    const std::vector<double>* v = n == "xs" ? &B.xs : n == "w" ? &B.w : n == "sbb" ? &B.sbb : n == "sbgb" ? &B.sbgb
                                 : n == "D" ? &B.D : n == "R" ? &B.R : n == "gR" ? &B.gR : n == "gsb" ? &B.gsb
                                 : n == "gsgb" ? &B.gsgb : n == "gbb" ? &B.gbb : n == "gbgb" ? &B.gbgb : nullptr;
    if (n == "gp") {
        if (out) out[0] = B.gp[0], out[1] = B.gp[1];
        return 2;
    }
    if (!v) return -100;
    if (out) std::copy(v->begin(), v->end(), out);
    return (long)v->size();
}

// bf16_bits over an array (the rounding of the optional BF16 smoother blocks)
extern "C" void bf16_array(const float* x, uint16_t* out, int n) {
    for (int i = 0; i < n; ++i) out[i] = ho2d::bf16_bits(x[i]);
}

namespace {
template <int K>
void kron_body_k(const ho2d::KronFit& f, const double* r_in, double* z) {
    constexpr int K2 = K * K;
    double fac[4 * K2], lam[2 * K], r[K2], t[K2];
    const std::vector<double>* m[4] = {&f.vx, &f.vxi, &f.vy, &f.vyi};
    for (int a = 0; a < 4; ++a) std::copy(m[a]->begin(), m[a]->end(), fac + a * K2);
    std::copy(f.lx.begin(), f.lx.end(), lam);
    std::copy(f.ly.begin(), f.ly.end(), lam + K);
    std::copy(r_in, r_in + K2, r);
    const ho2d::ElemCtx<1> c{0};
    ho2d::kron_apply_body<K, double>(c, true, fac, lam, r, t, z);
}
}  // namespace

// The element body of the Kronecker-sum smoother (kron_apply.cuh, one thread) on element
// el's fitted factors, applied to r into z; 0 if the fit is rejected.
extern "C" int case_kron_body(void* h, int el, const double* r, double* z) {
    const Case* c = static_cast<Case*>(h);
    const int K2 = c->op.K2, K = c->in.knod;
    const double* blk = &c->op.blocks[(size_t)el * 5 * K2 * K2];
    std::vector<double> D((size_t)K2 * K2);
    for (int ij = 0; ij < K2; ++ij)
        for (int rs = 0; rs < K2; ++rs) D[(size_t)ij * K2 + rs] = blk[(size_t)rs * K2 + ij];
    ho2d::KronFit f;
    if (!ho2d::kron_fit(K, D.data(), f)) return 0;
    switch (K) {
        case 1: kron_body_k<1>(f, r, z); break;
        case 2: kron_body_k<2>(f, r, z); break;
        case 3: kron_body_k<3>(f, r, z); break;
        case 4: kron_body_k<4>(f, r, z); break;
        case 5: kron_body_k<5>(f, r, z); break;
        case 6: kron_body_k<6>(f, r, z); break;
        case 7: kron_body_k<7>(f, r, z); break;
        case 8: kron_body_k<8>(f, r, z); break;
        default: return 0;
    }
    return 1;
}

// kron_device_arrays of the case: the elements' packed factors applied by the element body
// (or their exact block) to r, as the device smoother will; returns the number of exact
// elements. z [N][K^2], r [N][K^2].
extern "C" long case_kron_device(void* h, const double* r, double* z) {
    Case* c = static_cast<Case*>(h);
    const int K = c->in.knod, K2 = K * K, K4 = K2 * K2, per = 4 * K2 + 2 * K;
    ho2d::PoissonOperator op;
    ho2d::KronSmoother ks;
    ho2d::assemble_poisson(c->m, c->B, c->M, c->bc, op, false, &ks);
    std::vector<double> f, ex;
    std::vector<int> xi;
    ho2d::kron_device_arrays(ks, op.dinv, f, xi, ex);
    long n_exact = 0;
    for (int el = 0; el < c->m.n_el; ++el) {
        const double* re = r + (size_t)el * K2;
        double* ze = z + (size_t)el * K2;
        if (xi[el] >= 0) {
            ++n_exact;
            const double* blk = &ex[(size_t)xi[el] * K4];
            for (int ij = 0; ij < K2; ++ij) {
                double acc = 0.0;
                for (int rs = 0; rs < K2; ++rs) acc += blk[rs * K2 + ij] * re[rs];
                ze[ij] = acc;
            }
            continue;
        }
        std::vector<double> rr(re, re + K2), t(K2);
        const double* fe = &f[(size_t)el * per];
        const ho2d::ElemCtx<1> cx{0};
        switch (K) {
            case 3: ho2d::kron_apply_body<3, double>(cx, true, fe, fe + 4 * K2, rr.data(), t.data(), ze); break;
            case 4: ho2d::kron_apply_body<4, double>(cx, true, fe, fe + 4 * K2, rr.data(), t.data(), ze); break;
            case 5: ho2d::kron_apply_body<5, double>(cx, true, fe, fe + 4 * K2, rr.data(), t.data(), ze); break;
            case 7: ho2d::kron_apply_body<7, double>(cx, true, fe, fe + 4 * K2, rr.data(), t.data(), ze); break;
            default: return -1;
        }
    }
    return n_exact;
}
