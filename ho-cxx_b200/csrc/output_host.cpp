// output_host.cpp -- the reference's two VTK writers (src/HO_2D.cpp:3369-3692) on host
// arrays: save_vorticity_vtk (values at the solution points) and save_smooth_vtk (values at
// the geometry nodes, averaged over the elements sharing a node). Same file names, layout
// and number format (%g, the default of the reference's iostreams), the reference's node
// numbering (the mesh reader's first-use order, src/Mesh.cpp:296-333), and the same
// boundary treatment in the smooth file: boundary nodes take BC_vorticity and the Cartesian
// velocity rebuilt from BC_normal_vel (local h direction) and BC_parl_vel. With sample
// points, also the sample-point file of save_smooth_vtk (src/HO_2D.cpp:3592-3614): x, y and
// the node-averaged vorticity and velocity interpolated with the geometry shape functions.
#include <cmath>
#include <cstdio>
#include <exception>
#include <memory>
#include <new>
#include <string>
#include <system_error>
#include <vector>

#include "host.hpp"
#include "vtk_nodes.hpp"

namespace ho2d {

namespace {

struct File {
    FILE* f = nullptr;
    explicit File(const std::string& path) : f(std::fopen(path.c_str(), "w")) {}
    ~File() {
        if (f) std::fclose(f);
    }
};

}  // namespace

VtkGeoHost::VtkGeoHost(const Mesh& m, const Bases& B) : mesh(m), bases(B) {
    const int K = B.K, L = m.lnod, L2 = L * L;
    sgb.resize((size_t)K * L);
    for (int k = 0; k < K; ++k)
        for (int l = 0; l < L; ++l) {
            const double x = L > 1 ? -1.0 + 2.0 * l / (L - 1) : 0.0;
            double p = 1.0;
            for (int q = 0; q < K; ++q)
                if (q != k) p *= (x - B.xs[q]) / (B.xs[k] - B.xs[q]);
            sgb[(size_t)k * L + l] = p;
        }
    t2f.resize(L2);
    for (int ly = 0; ly < L; ++ly)
        for (int lx = 0; lx < L; ++lx) t2f[ly * L + lx] = tensor2fem(lx, ly, L - 1);
    nodes.resize((size_t)m.n_el * L2);
    for (int el = 0; el < m.n_el; ++el)
        for (int l = 0; l < L2; ++l) nodes[(size_t)el * L2 + l] = m.elem_nodes[el][l];
}

VtkGeo VtkGeoHost::geo() const {
    return VtkGeo{mesh.n_el,       bases.K,          mesh.lnod,         mesh.n_eb,          sgb.data(),
                  t2f.data(),      nodes.data(),     mesh.node_xy.data(), mesh.be_el.data(), mesh.be_side.data(),
                  bases.gbgb.data(), bases.gbb.data(), bases.gsb.data(),   bases.gsgb.data()};
}

Error write_vtk_files(const Mesh& mesh_, const Bases& B_, int problem_type, const VtkFields& fl, int indx, int subidx,
                      const std::string& dir, const SamplePoints* samples) {
    const int N = mesh_.n_el, K = B_.K, K2 = K * K, L = mesh_.lnod, lin = L - 1, L2 = L * L;
    const size_t nv = (size_t)N * K2, nb = (size_t)mesh_.n_eb * K;
    const double *w = fl.w, *psi = fl.psi, *u = fl.u, *v = fl.v, *rd = fl.rhs_diff, *ra = fl.rhs_adv;
    const double *bw = fl.bc_w, *bnv = fl.bc_nv, *bpv = fl.bc_pv;
    char tag[64];
    if (subidx > -1) std::snprintf(tag, sizeof(tag), "%d_K%d_%02d_%05d.vtk", problem_type, K, subidx, indx);
    else std::snprintf(tag, sizeof(tag), "%d_K%d_%05d.vtk", problem_type, K, indx);
    const std::string pre = dir.empty() ? std::string() : dir + "/";

    // ---- save_vorticity_vtk: values at the solution points
    {
        std::vector<double> xy(2 * nv);  // solution points (getsolnpts_d)
        for (int el = 0; el < N; ++el)
            for (int j = 0; j < K; ++j)
                for (int i = 0; i < K; ++i) {
                    double x = 0.0, y = 0.0;
                    for (int ly = 0; ly < L; ++ly)
                        for (int lx = 0; lx < L; ++lx) {
                            const int nd = mesh_.elem_nodes[el][tensor2fem(lx, ly, lin)];
                            const double wgt = B_.gsb[ly * K + j] * B_.gsb[lx * K + i];
                            x += wgt * mesh_.node_xy[2 * nd];
                            y += wgt * mesh_.node_xy[2 * nd + 1];
                        }
                    const size_t p = ((size_t)el * K + j) * K + i;
                    xy[2 * p] = x;
                    xy[2 * p + 1] = y;
                }
        File fh(pre + "vorticity" + tag);
        if (!fh.f) return {2, "cannot write " + pre + "vorticity" + tag};
        FILE* f = fh.f;
        std::fprintf(f, "# vtk DataFile Version 3.0\n2D Unstructured Grid of Quads\nASCII\n\nDATASET POLYDATA\n");
        std::fprintf(f, "POINTS %zu double\n", nv);
        for (size_t p = 0; p < nv; ++p) std::fprintf(f, "%g %g  0.\n", xy[2 * p], xy[2 * p + 1]);
        std::fprintf(f, "POINT_DATA %zu\n", nv);
        const char* names[3] = {"vorticity", "rhs_diffusive", "rhs_advective"};
        const double* vals[3] = {w, rd, ra};
        for (int a = 0; a < 3; ++a) {
            std::fprintf(f, "SCALARS %s double 1 \nLOOKUP_TABLE default \n", names[a]);
            for (int el = 0; el < N; ++el) {
                for (int q = 0; q < K2; ++q) std::fprintf(f, "%g ", vals[a][(size_t)el * K2 + q]);
                std::fprintf(f, "\n");
            }
        }
        std::fprintf(f, "VECTORS velocity double \n");
        for (size_t p = 0; p < nv; ++p) std::fprintf(f, "%g %g 0.\n", u[p], v[p]);
    }

    // ---- save_smooth_vtk: values at the geometry nodes, averaged over the elements
    // sharing a node (vtk_nodes.hpp), unless the caller brings them (the device's)
    const size_t nn = mesh_.node_xy.size() / 2;
    std::vector<double> hw, hp, hux, huy, hs;
    const double *nw = fl.nw, *np = fl.np, *nux = fl.nux, *nuy = fl.nuy, *samp = fl.samp;
    if (!nw) {
        const VtkGeoHost gh(mesh_, B_);
        const VtkGeo g = gh.geo();
        std::vector<double> om((size_t)N * L2, 0.0), ps((size_t)N * L2, 0.0), vx((size_t)N * L2, 0.0),
            vy((size_t)N * L2, 0.0);
        for (int el = 0; el < N; ++el)
            vtk_element_nodes(g, el, w, psi, u, v, om.data(), ps.data(), vx.data(), vy.data());
        std::vector<double> cvx(nb, 0.0), cvy(nb, 0.0);
        for (int e = 0; e < mesh_.n_eb; ++e) vtk_edge_velocity(g, e, bnv, bpv, cvx.data(), cvy.data());
        for (int e = 0; e < mesh_.n_eb; ++e) vtk_edge_nodes(g, e, bw, cvx.data(), cvy.data(), om.data(), vx.data(), vy.data());
        // nodes in the compact numbering of the mesh reader (first use: edges, then
        // elements), which is the reference's numbering (src/Mesh.cpp:296-333)
        hw.assign(nn, 0.0);
        hp.assign(nn, 0.0);
        hux.assign(nn, 0.0);
        huy.assign(nn, 0.0);
        std::vector<int> rep(nn, 0);
        for (int el = 0; el < N; ++el)
            for (int l = 0; l < L2; ++l) {
                const size_t q = (size_t)el * L2 + l;
                const int nd = mesh_.elem_nodes[el][l];
                hux[nd] += vx[q];
                huy[nd] += vy[q];
                hw[nd] += om[q];
                hp[nd] += ps[q];
                ++rep[nd];
            }
        for (size_t n = 0; n < nn; ++n) vtk_node_average(rep[n], hw[n], hp[n], hux[n], huy[n]);
        nw = hw.data();
        np = hp.data();
        nux = hux.data();
        nuy = huy.data();
        if (samples && samples->size() > 0) {
            hs.assign(3 * samples->size(), 0.0);
            for (size_t si = 0; si < samples->size(); ++si) {
                const int el = samples->elem[si];
                vtk_sample(L2, mesh_.elem_nodes[el].data(), &samples->shape[si * L2], nw, nux, nuy, &hs[3 * si]);
            }
            samp = hs.data();
        }
    }
    File fh(pre + "problem" + tag);
    if (!fh.f) return {2, "cannot write " + pre + "problem" + tag};
    FILE* f = fh.f;
    std::fprintf(f, "# vtk DataFile Version 3.0\n2D Unstructured Grid of Quads\nASCII\n\nDATASET UNSTRUCTURED_GRID\n");
    std::fprintf(f, "POINTS %zu double\n", nn);
    for (size_t n = 0; n < nn; ++n) std::fprintf(f, "%g %g 0.0\n", mesh_.node_xy[2 * n], mesh_.node_xy[2 * n + 1]);
    std::fprintf(f, "CELLS %d %d\n", N, N * (L2 + 1));
    for (int el = 0; el < N; ++el) {
        std::fprintf(f, "%d", L2);
        for (int l = 0; l < L2; ++l) std::fprintf(f, " %d", mesh_.elem_nodes[el][l]);
        std::fprintf(f, "\n");
    }
    std::fprintf(f, "CELL_TYPES %d\n", N);
    for (int el = 0; el < N; ++el) std::fprintf(f, "70\n");
    std::fprintf(f, "POINT_DATA %zu\n", nn);
    std::fprintf(f, "SCALARS vorticity double 1 \nLOOKUP_TABLE default \n");
    for (size_t n = 0; n < nn; ++n) std::fprintf(f, "%g\n", nw[n]);
    std::fprintf(f, "SCALARS psi double 1 \nLOOKUP_TABLE default \n");
    for (size_t n = 0; n < nn; ++n) std::fprintf(f, "%g\n", np[n]);
    std::fprintf(f, "VECTORS velocity double \n");
    for (size_t n = 0; n < nn; ++n) std::fprintf(f, "%g %g 0.0\n", nux[n], nuy[n]);
    if (!samples || samples->size() == 0) return {0, ""};
    char sname[96];
    std::snprintf(sname, sizeof(sname), "sampling_points%d_K%d_L%d_%05d.dat", problem_type, K, L, indx);
    File sh(pre + sname);
    if (!sh.f) return {2, "cannot write " + pre + sname};
    for (size_t si = 0; si < samples->size(); ++si)
        std::fprintf(sh.f, "%g %g %g %g %g\n", samples->xy[2 * si], samples->xy[2 * si + 1], samp[3 * si],
                     samp[3 * si + 1], samp[3 * si + 2]);
    return {0, ""};
}

Error VtkQueue::submit(const Mesh& mesh, const Bases& B, const SamplePoints* samples, Job job) {
    Error e = wait();
    if (e.code) return e;
    auto owned = std::make_shared<Job>(std::move(job));
    auto work = [this, &mesh, &B, samples, owned]() {
        const Job& j = *owned;
        const VtkFields f = j.fields();
        // nothing may leave the writer thread: every exception becomes an error status, and
        // building the message (which allocates) may itself throw, so it has a fixed fallback
        try {
            try {
                err_ = write_vtk_files(mesh, B, j.problem_type, f, j.indx, j.subidx, j.dir, samples);
            } catch (const std::bad_alloc&) {
                err_ = {5, "out of host memory writing the VTK files"};
            } catch (const std::exception& ex) {
                err_ = {5, std::string("writing the VTK files: ") + ex.what()};
            }
        } catch (...) {
            err_.code = 5;
            err_.msg = "VTK write fail";  // 14 characters: fits the string's inline buffer
        }
    };
    try {
        thread_ = std::thread(work);
    } catch (const std::system_error&) {  // no thread to be had: write here
        work();
    }
    return {0, ""};
}

Error VtkQueue::wait() {
    if (thread_.joinable()) thread_.join();
    Error e = err_;
    err_ = {0, ""};
    return e;
}

}  // namespace ho2d
