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
    // sharing a node. sgb[k][l]: solution basis k at geometry node l (equispaced in [-1, 1]).
    std::vector<double> sgb((size_t)K * L);
    for (int k = 0; k < K; ++k)
        for (int l = 0; l < L; ++l) {
            const double x = L > 1 ? -1.0 + 2.0 * l / (L - 1) : 0.0;
            double p = 1.0;
            for (int m = 0; m < K; ++m)
                if (m != k) p *= (x - B_.xs[m]) / (B_.xs[k] - B_.xs[m]);
            sgb[(size_t)k * L + l] = p;
        }
    std::vector<double> om((size_t)N * L2, 0.0), ps((size_t)N * L2, 0.0), vx((size_t)N * L2, 0.0),
        vy((size_t)N * L2, 0.0);
    for (int el = 0; el < N; ++el)
        for (int ly = 0; ly < L; ++ly)
            for (int lx = 0; lx < L; ++lx) {
                const size_t g = (size_t)el * L2 + tensor2fem(lx, ly, lin);
                double a = 0, b = 0, c = 0, e = 0;
                for (int ky = 0; ky < K; ++ky)
                    for (int kx = 0; kx < K; ++kx) {
                        const double coeff = sgb[(size_t)ky * L + ly] * sgb[(size_t)kx * L + lx];
                        const size_t p = (size_t)el * K2 + ky * K + kx;
                        a += coeff * w[p];
                        b += coeff * psi[p];
                        c += coeff * u[p];
                        e += coeff * v[p];
                    }
                om[g] = a;
                ps[g] = b;
                vx[g] = c;
                vy[g] = e;
            }
    // boundary nodes: BC_vorticity, and the Cartesian velocity from the normal (local h
    // direction) and counter-clockwise tangential components (src/HO_2D.cpp:3440-3513)
    std::vector<double> cvx(nb, 0.0), cvy(nb, 0.0);
    for (int e = 0; e < mesh_.n_eb; ++e) {
        const int el = mesh_.be_el[e], side = mesh_.be_side[e], ijp = kF2I[side], dd = ijp / 2, t = ijp % 2;
        const double parl_sign = -1.0 + 2.0 * (side / 2);
        for (int k = 0; k < K; ++k) {
            double xx = 0, xe = 0, yx = 0, ye = 0;  // d(x, y)/d(xi, eta) at face point k
            for (int j = 0; j < L; ++j)
                for (int i = 0; i < L; ++i) {
                    const int nd = mesh_.elem_nodes[el][tensor2fem(i, j, lin)];
                    const double X = mesh_.node_xy[2 * nd], Y = mesh_.node_xy[2 * nd + 1];
                    double wx, we;
                    if (dd == 0) {  // W/E face: xi = -+1, eta = x_k
                        wx = B_.gbgb[i * 2 + t] * B_.gsb[j * K + k];
                        we = B_.gbb[i * 2 + t] * B_.gsgb[j * K + k];
                    } else {  // S/N face: eta = -+1, xi = x_k
                        wx = B_.gsgb[i * K + k] * B_.gbb[j * 2 + t];
                        we = B_.gsb[i * K + k] * B_.gbgb[j * 2 + t];
                    }
                    xx += wx * X;
                    yx += wx * Y;
                    xe += we * X;
                    ye += we * Y;
                }
            const size_t q = (size_t)e * K + (side / 2) * (K - 2 * k - 1) + k;
            if (dd == 0) {
                const double g2 = std::sqrt(xe * xe + ye * ye), un = bnv[q], ut = parl_sign * bpv[q];
                cvx[q] = (1.0 / g2) * (un * ye + ut * xe);
                cvy[q] = (1.0 / g2) * (-un * xe + ut * ye);
            } else {
                const double g1 = std::sqrt(xx * xx + yx * yx), un = bnv[q], ut = parl_sign * bpv[q];
                cvx[q] = (1.0 / g1) * (-un * yx + ut * xx);
                cvy[q] = (1.0 / g1) * (un * xx + ut * yx);
            }
        }
    }
    for (int e = 0; e < mesh_.n_eb; ++e) {
        const int el = mesh_.be_el[e], side = mesh_.be_side[e], ijp = kF2I[side], dd = ijp / 2, t = ijp % 2;
        for (int l = 0; l < L; ++l) {
            const int su2pv = l * ((1 - dd) * L + dd) + t * (L - 1) * (dd * (L - 1) + 1);
            const size_t g = (size_t)el * L2 + tensor2fem(su2pv % L, su2pv / L, lin);
            double a = 0, c = 0, f2 = 0;
            for (int m = 0; m < K; ++m) {
                const double coeff = sgb[(size_t)m * L + l];
                const size_t q = (size_t)e * K + (side / 2) * (K - 2 * m - 1) + m;
                a += coeff * bw[q];
                c += coeff * cvx[q];
                f2 += coeff * cvy[q];
            }
            om[g] = a;
            vx[g] = c;
            vy[g] = f2;
        }
    }
    // nodes in the compact numbering of the mesh reader (first use: edges, then elements),
    // which is the reference's numbering (src/Mesh.cpp:296-333)
    const size_t nn = mesh_.node_xy.size() / 2;
    std::vector<double> nw(nn, 0.0), np(nn, 0.0), nux(nn, 0.0), nuy(nn, 0.0);
    std::vector<int> rep(nn, 0);
    for (int el = 0; el < N; ++el)
        for (int l = 0; l < L2; ++l) {
            const size_t g = (size_t)el * L2 + l;
            const int nd = mesh_.elem_nodes[el][l];
            nux[nd] += vx[g];
            nuy[nd] += vy[g];
            nw[nd] += om[g];
            np[nd] += ps[g];
            ++rep[nd];
        }
    for (size_t n = 0; n < nn; ++n) {
        nw[n] /= rep[n];
        np[n] /= rep[n];
        nux[n] *= 1.0 / rep[n];
        nuy[n] *= 1.0 / rep[n];
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
    for (size_t s = 0; s < samples->size(); ++s) {
        const int el = samples->elem[s];
        const double* sf = &samples->shape[s * L2];
        double om_s = 0.0, ux = 0.0, uy = 0.0;
        for (int l = 0; l < L2; ++l) {
            const int nd = mesh_.elem_nodes[el][l];
            om_s += sf[l] * nw[nd];
            ux += sf[l] * nux[nd];
            uy += sf[l] * nuy[nd];
        }
        std::fprintf(sh.f, "%g %g %g %g %g\n", samples->xy[2 * s], samples->xy[2 * s + 1], om_s, ux, uy);
    }
    return {0, ""};
}

Error VtkQueue::submit(const Mesh& mesh, const Bases& B, const SamplePoints* samples, Job job) {
    Error e = wait();
    if (e.code) return e;
    auto owned = std::make_shared<Job>(std::move(job));
    auto work = [this, &mesh, &B, samples, owned]() {
        const Job& j = *owned;
        const VtkFields f{j.w.data(),       j.psi.data(),  j.u.data(),     j.v.data(),    j.rhs_diff.data(),
                          j.rhs_adv.data(), j.bc_w.data(), j.bc_nv.data(), j.bc_pv.data()};
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
