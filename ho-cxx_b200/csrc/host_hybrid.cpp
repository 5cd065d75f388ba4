// host_hybrid.cpp -- host arithmetic of the hybrid entry points (src/HO_2D.cpp:3982-4122):
// solution-point areas, the points of the open boundary, the outward unit normals of the
// open edges and the split of a driver's Cartesian velocities into normal and parallel
// parts. The device side (hybrid.cu) uploads what these compute.
#include <cmath>

#include "host.hpp"

namespace ho2d {

const std::vector<int>* open_boundary_edges(const Mesh& m) {
    for (size_t g = 0; g < m.group_names.size(); ++g)
        if (m.group_names[g] == "open") return &m.group_edges[g];
    return nullptr;
}

// getopenptlen (src/HO_2D.cpp:3994-4002): x, y of K points per open edge
int open_point_count(const Mesh& m, int K) {
    const std::vector<int>* oe = open_boundary_edges(m);
    return oe ? 2 * (int)oe->size() * K : 0;
}

// getsolnareas_d (src/HO_2D.cpp:3982-3992): w_j w_k |J| at each solution point
void solution_areas(const Bases& B, const Metrics& M, int n_el, double* out) {
    const int K = B.K;
    for (int el = 0; el < n_el; ++el)
        for (int j = 0; j < K; ++j)
            for (int k = 0; k < K; ++k) {
                const size_t p = ((size_t)el * K + j) * K + k;
                out[p] = B.w[j] * B.w[k] * M.J[p];
            }
}

// getopenpts_d (src/HO_2D.cpp:4004-4042): the geometry map of each open edge (its Lnod
// nodes from the first to the last) at the K solution points, in open-boundary order
void open_points(const Mesh& m, const Bases& B, double* out) {
    const std::vector<int>* oe = open_boundary_edges(m);
    if (!oe) return;
    const int K = B.K, L = m.lnod, lin = L - 1;
    for (size_t i = 0; i < oe->size(); ++i) {
        const auto& en = m.edge_nodes[(*oe)[i]];
        for (int j = 0; j < K; ++j) {
            double x = 0.0, y = 0.0;
            for (int l = 0; l < L; ++l) {
                const int nd = en[tensor2fem_1d(l, lin)];
                x += B.gsb[l * K + j] * m.node_xy[2 * nd];
                y += B.gsb[l * K + j] * m.node_xy[2 * nd + 1];
            }
            out[2 * (i * K + j)] = x;
            out[2 * (i * K + j) + 1] = y;
        }
    }
}

// The unit outward normal at face point k of the element that owns each open edge
// (src/HO_2D.cpp:4087-4100): the derivative of the geometry map along the face, rotated a
// quarter turn towards the outside and divided by its length |g| (face_Anorm). Layout
// [n_eb][K][2]; zero on the other edges.
void open_normals(const Mesh& m, const Bases& B, const Metrics& M, const BoundaryConditions& bc,
                  std::vector<double>& nrm) {
    const int K = B.K, L = m.lnod, lin = L - 1;
    nrm.assign((size_t)m.n_eb * K * 2, 0.0);
    for (int e = 0; e < m.n_eb; ++e) {
        if (bc.role[e] != ROLE_OPEN) continue;
        const int el = m.be_el[e], ijp = kF2I[m.be_side[e]];
        const int dd = ijp / 2, t = ijp % 2;
        const double coeff = 2.0 * t - 1.0;
        for (int k = 0; k < K; ++k) {
            double dx = 0.0, dy = 0.0;  // derivative along the face (xi on S/N faces, eta on W/E)
            for (int j = 0; j < L; ++j)
                for (int i = 0; i < L; ++i) {
                    const int nd = m.elem_nodes[el][tensor2fem(i, j, lin)];
                    const double w = dd == 0 ? B.gbb[i * 2 + t] * B.gsgb[j * K + k] : B.gsgb[i * K + k] * B.gbb[j * 2 + t];
                    dx += w * m.node_xy[2 * nd];
                    dy += w * m.node_xy[2 * nd + 1];
                }
            const double an = M.fAn[((size_t)el * 4 + ijp) * K + k];
            const double nx = dd == 1 ? -dy : dy, ny = dd == 1 ? dx : -dx;
            nrm[((size_t)e * K + k) * 2] = nx * coeff / an;
            nrm[((size_t)e * K + k) * 2 + 1] = ny * coeff / an;
        }
    }
}

// setopenvels_d (src/HO_2D.cpp:4047-4122): the driver's velocity (u, v) at point j of open
// edge i becomes n.(u, v) in vn and n x (u, v) in vp, at [edge][j] of the open edge's
// boundary-edge index. Point j is paired with the normal at face point j of the owning
// element, as in the reference.
void split_open_velocities(const Mesh& m, int K, const std::vector<double>& nrm, const double* xyvel, double* vn,
                           double* vp) {
    const std::vector<int>* oe = open_boundary_edges(m);
    if (!oe) return;
    for (size_t i = 0; i < oe->size(); ++i) {
        const int e = (*oe)[i];
        for (int j = 0; j < K; ++j) {
            const size_t q = (size_t)e * K + j;
            const double u = xyvel[2 * (i * K + j)], v = xyvel[2 * (i * K + j) + 1];
            const double nx = nrm[2 * q], ny = nrm[2 * q + 1];
            vn[q] = nx * u + ny * v;
            vp[q] = nx * v - ny * u;
        }
    }
}

}  // namespace ho2d
