// vtk_nodes.hpp -- the node values of save_smooth_vtk (src/HO_2D.cpp:3392-3614), as one
// source for the host writer (output_host.cpp) and the device (output_device.cu):
//   * every element's fields interpolated to its geometry nodes (solution basis at the
//     equispaced node positions, sgb[k][l]);
//   * on boundary edges, BC_vorticity and the Cartesian velocity rebuilt from BC_normal_vel
//     (local h direction) and the counter-clockwise BC_parl_vel, interpolated to the edge's
//     nodes, the later edge of an element winning at a shared corner node;
//   * per mesh node, the average over the element node slots that share it, summed in
//     ascending (element, slot) order;
//   * the sample points' values: the nodes' averages weighted by the geometry shape
//     functions of the point's element.
// The device file is compiled with -fmad=false, so both give the same bits.
#pragma once

#include <cmath>

#ifdef __CUDACC__
#define HO2D_VTK_HD __host__ __device__
#else
#define HO2D_VTK_HD
#endif

namespace ho2d {

struct VtkGeo {
    int N, K, L, neb;
    const double* sgb;         // [K][L] solution basis k at geometry node position l
    const int* t2f;            // [L][L] (ly, lx) -> Gmsh node slot
    const int* elem_nodes;     // [N][L^2] mesh node of each slot
    const double* node_xy;     // [nodes][2]
    const int *be_el, *be_side;  // [neb]
    const double *gbgb, *gbb;  // [L][2] geometry basis (derivative) at -1, +1
    const double *gsb, *gsgb;  // [L][K] geometry basis (derivative) at the solution points
};

// element el: om, ps, vx, vy [N][L^2] from w, psi, u, v [N][K][K]
HO2D_VTK_HD inline void vtk_element_nodes(const VtkGeo& g, int el, const double* w, const double* psi,
                                          const double* u, const double* v, double* om, double* ps, double* vx,
                                          double* vy) {
    const int K = g.K, L = g.L, K2 = K * K, L2 = L * L;
    for (int ly = 0; ly < L; ++ly)
        for (int lx = 0; lx < L; ++lx) {
            const size_t q = (size_t)el * L2 + g.t2f[ly * L + lx];
            double a = 0, b = 0, c = 0, e = 0;
            for (int ky = 0; ky < K; ++ky)
                for (int kx = 0; kx < K; ++kx) {
                    const double coeff = g.sgb[ky * L + ly] * g.sgb[kx * L + lx];
                    const size_t p = (size_t)el * K2 + ky * K + kx;
                    a += coeff * w[p];
                    b += coeff * psi[p];
                    c += coeff * u[p];
                    e += coeff * v[p];
                }
            om[q] = a;
            ps[q] = b;
            vx[q] = c;
            vy[q] = e;
        }
}

// boundary edge e: the Cartesian velocity at its K points (boundary-array order) into
// cvx, cvy [neb][K] (src/HO_2D.cpp:3440-3513)
HO2D_VTK_HD inline void vtk_edge_velocity(const VtkGeo& g, int e, const double* bnv, const double* bpv,
                                          double* cvx, double* cvy) {
    constexpr int f2i[4] = {2, 1, 3, 0};
    const int K = g.K, L = g.L, L2 = L * L;
    const int el = g.be_el[e], side = g.be_side[e], ijp = f2i[side], dd = ijp / 2, t = ijp % 2;
    const double parl_sign = -1.0 + 2.0 * (side / 2);
    for (int k = 0; k < K; ++k) {
        double xx = 0, xe = 0, yx = 0, ye = 0;  // d(x, y)/d(xi, eta) at face point k
        for (int j = 0; j < L; ++j)
            for (int i = 0; i < L; ++i) {
                const int nd = g.elem_nodes[(size_t)el * L2 + g.t2f[j * L + i]];
                const double X = g.node_xy[2 * (size_t)nd], Y = g.node_xy[2 * (size_t)nd + 1];
                double wx, we;
                if (dd == 0) {  // W/E face: xi = -+1, eta = x_k
                    wx = g.gbgb[i * 2 + t] * g.gsb[j * K + k];
                    we = g.gbb[i * 2 + t] * g.gsgb[j * K + k];
                } else {  // S/N face: eta = -+1, xi = x_k
                    wx = g.gsgb[i * K + k] * g.gbb[j * 2 + t];
                    we = g.gsb[i * K + k] * g.gbgb[j * 2 + t];
                }
                xx += wx * X;
                yx += wx * Y;
                xe += we * X;
                ye += we * Y;
            }
        const size_t q = (size_t)e * K + (side / 2) * (K - 2 * k - 1) + k;
        if (dd == 0) {
            const double g2 = sqrt(xe * xe + ye * ye), un = bnv[q], ut = parl_sign * bpv[q];
            cvx[q] = (1.0 / g2) * (un * ye + ut * xe);
            cvy[q] = (1.0 / g2) * (-un * xe + ut * ye);
        } else {
            const double g1 = sqrt(xx * xx + yx * yx), un = bnv[q], ut = parl_sign * bpv[q];
            cvx[q] = (1.0 / g1) * (-un * yx + ut * xx);
            cvy[q] = (1.0 / g1) * (un * xx + ut * yx);
        }
    }
}

// boundary edge e: BC_vorticity and the rebuilt velocity at the edge's L node slots
HO2D_VTK_HD inline void vtk_edge_nodes(const VtkGeo& g, int e, const double* bw, const double* cvx, const double* cvy,
                                       double* om, double* vx, double* vy) {
    constexpr int f2i[4] = {2, 1, 3, 0};
    const int K = g.K, L = g.L, L2 = L * L;
    const int el = g.be_el[e], side = g.be_side[e], ijp = f2i[side], dd = ijp / 2, t = ijp % 2;
    for (int l = 0; l < L; ++l) {
        const int su2pv = l * ((1 - dd) * L + dd) + t * (L - 1) * (dd * (L - 1) + 1);
        const size_t q = (size_t)el * L2 + g.t2f[(su2pv / L) * L + su2pv % L];
        double a = 0, c = 0, f2 = 0;
        for (int m = 0; m < K; ++m) {
            const double coeff = g.sgb[m * L + l];
            const size_t p = (size_t)e * K + (side / 2) * (K - 2 * m - 1) + m;
            a += coeff * bw[p];
            c += coeff * cvx[p];
            f2 += coeff * cvy[p];
        }
        om[q] = a;
        vx[q] = c;
        vy[q] = f2;
    }
}

// the averages of one node from its sums and slot count
HO2D_VTK_HD inline void vtk_node_average(int rep, double& w, double& p, double& ux, double& uy) {
    w /= rep;
    p /= rep;
    ux *= 1.0 / rep;
    uy *= 1.0 / rep;
}

// one sample point: vorticity and velocity from the node averages
HO2D_VTK_HD inline void vtk_sample(int L2, const int* nodes, const double* sf, const double* nw, const double* nux,
                                   const double* nuy, double* out) {
    double om_s = 0.0, ux = 0.0, uy = 0.0;
    for (int l = 0; l < L2; ++l) {
        const int nd = nodes[l];
        om_s += sf[l] * nw[nd];
        ux += sf[l] * nux[nd];
        uy += sf[l] * nuy[nd];
    }
    out[0] = om_s;
    out[1] = ux;
    out[2] = uy;
}

}  // namespace ho2d
