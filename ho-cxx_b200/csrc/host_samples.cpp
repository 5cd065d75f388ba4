// host_samples.cpp -- the sample points of the input's sample-points file
// (read_process_sample_points, src/HO_2D.cpp:319-474): for each point, the element that
// holds it and the Lnod^2 geometry shape functions at its local coordinates. The VTK
// output interpolates the node-averaged vorticity and velocity with them
// (src/HO_2D.cpp:3592-3614, write_vtk_files).
//
// Element search: the first element, in element order, whose boundary polygon (the straight
// segments between consecutive geometry nodes along its four edges) contains the point, by
// a crossing count along the +x ray. The reference casts the ray at a slope drawn from the
// clock-seeded rand(); the answer is the same except for points on an element's boundary,
// which either element may hold. A point in no polygon goes to the element with the node
// nearest to it (first in element, then node-slot order; src/HO_2D.cpp:380-394).
//
// Local coordinates: Newton's method on x(xi, eta) = p from (0.08, 0.08), stopped when both
// steps are at most 1e-3, as in the reference; the shape functions are those of the
// iterate the last step was computed at, as the reference keeps them. The reference's
// iteration has no limit; here it stops after 100 steps.
#include <cmath>
#include <cstdlib>
#include <fstream>
#include <iterator>
#include <string>
#include <vector>

#include "host.hpp"

namespace ho2d {

namespace {

// Lagrange basis on the L equispaced nodes of [-1, 1] and its derivative at x
void equispaced_basis(int L, double x, double* val, double* der) {
    double nodes[4];
    for (int k = 0; k < L; ++k) nodes[k] = L > 1 ? -1.0 + 2.0 * k / (L - 1) : 0.0;
    for (int k = 0; k < L; ++k) {
        double den = 1.0, v = 1.0, d = 0.0;
        for (int m = 0; m < L; ++m) {
            if (m == k) continue;
            den *= nodes[k] - nodes[m];
            v *= x - nodes[m];
            double prod = 1.0;  // d/dx of prod_{m' != k} (x - x_m'): drop factor m
            for (int q = 0; q < L; ++q)
                if (q != k && q != m) prod *= x - nodes[q];
            d += prod;
        }
        val[k] = v / den;
        der[k] = d / den;
    }
}

// crossing count of the +x ray from (px, py) with the element's boundary polygon
bool polygon_contains(const Mesh& m, int el, double px, double py) {
    const int L = m.lnod, lin = L - 1;
    std::vector<int> ring;  // perimeter of the L x L node grid, counter-clockwise
    for (int i = 0; i < L; ++i) ring.push_back(tensor2fem(i, 0, lin));
    for (int j = 1; j < L; ++j) ring.push_back(tensor2fem(L - 1, j, lin));
    for (int i = L - 2; i >= 0; --i) ring.push_back(tensor2fem(i, L - 1, lin));
    for (int j = L - 2; j >= 1; --j) ring.push_back(tensor2fem(0, j, lin));
    bool in = false;
    const size_t n = ring.size();
    for (size_t a = 0; a < n; ++a) {
        const int na = m.elem_nodes[el][ring[a]], nb = m.elem_nodes[el][ring[(a + 1) % n]];
        const double xa = m.node_xy[2 * na], ya = m.node_xy[2 * na + 1];
        const double xb = m.node_xy[2 * nb], yb = m.node_xy[2 * nb + 1];
        if ((ya <= py) != (yb <= py)) {
            const double xc = xa + (py - ya) / (yb - ya) * (xb - xa);
            if (xc > px) in = !in;
        }
    }
    return in;
}

int locate(const Mesh& m, double px, double py) {
    const int L = m.lnod, lin = L - 1;
    for (int el = 0; el < m.n_el; ++el) {
        double x0 = INFINITY, x1 = -INFINITY, y0 = INFINITY, y1 = -INFINITY;
        for (int j = 0; j < L; ++j)
            for (int i = 0; i < L; ++i) {
                if (i != 0 && i != lin && j != 0 && j != lin) continue;  // edge nodes only
                const int nd = m.elem_nodes[el][tensor2fem(i, j, lin)];
                x0 = std::fmin(x0, m.node_xy[2 * nd]);
                x1 = std::fmax(x1, m.node_xy[2 * nd]);
                y0 = std::fmin(y0, m.node_xy[2 * nd + 1]);
                y1 = std::fmax(y1, m.node_xy[2 * nd + 1]);
            }
        if (px < x0 || px > x1 || py < y0 || py > y1) continue;
        if (polygon_contains(m, el, px, py)) return el;
    }
    // nearest geometry node; the search starts one unit above the distance to element 0's
    // first node, so that element 0 always takes part
    const int n0 = m.elem_nodes[0][0];
    double best = std::hypot(px - m.node_xy[2 * n0], py - m.node_xy[2 * n0 + 1]) + 1.0;
    int hold = -1;
    for (int el = 0; el < m.n_el; ++el)
        for (int nd : m.elem_nodes[el]) {
            const double d = std::hypot(px - m.node_xy[2 * nd], py - m.node_xy[2 * nd + 1]);
            if (d < best) {
                best = d;
                hold = el;
            }
        }
    return hold;
}

void local_shape(const Mesh& m, int el, double px, double py, double* shape) {
    const int L = m.lnod, lin = L - 1;
    double bx[4], dbx[4], by[4], dby[4];
    double xi = 0.08, eta = 0.08;
    for (int it = 0; it < 100; ++it) {
        equispaced_basis(L, xi, bx, dbx);
        equispaced_basis(L, eta, by, dby);
        double X = 0, Y = 0, Xxi = 0, Xeta = 0, Yxi = 0, Yeta = 0;
        for (int j = 0; j < L; ++j)
            for (int i = 0; i < L; ++i) {
                const int nd = m.elem_nodes[el][tensor2fem(i, j, lin)];
                const double x = m.node_xy[2 * nd], y = m.node_xy[2 * nd + 1];
                X += bx[i] * by[j] * x;
                Y += bx[i] * by[j] * y;
                Xxi += dbx[i] * by[j] * x;
                Yxi += dbx[i] * by[j] * y;
                Xeta += bx[i] * dby[j] * x;
                Yeta += bx[i] * dby[j] * y;
            }
        const double det = Xxi * Yeta - Xeta * Yxi, rx = px - X, ry = py - Y;
        const double dxi = (rx * Yeta - ry * Xeta) / det, deta = (ry * Xxi - rx * Yxi) / det;
        if (!std::isfinite(dxi) || !std::isfinite(deta)) break;
        xi += dxi;
        eta += deta;
        if (std::fabs(dxi) <= 1e-3 && std::fabs(deta) <= 1e-3) break;
    }
    for (int j = 0; j < L; ++j)
        for (int i = 0; i < L; ++i) shape[tensor2fem(i, j, lin)] = bx[i] * by[j];
}

}  // namespace

Error read_sample_points(const std::string& path, const Mesh& m, SamplePoints& sp) {
    sp = SamplePoints();
    std::ifstream f(path, std::ios::binary);
    if (!f) return {0, ""};  // no file: no sample points, as in the reference
    const std::string text((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
    // x y pairs separated by white space, up to the first token that is not a number
    std::vector<double> v;
    const char* p = text.c_str();
    for (;;) {
        char* end = nullptr;
        const double x = std::strtod(p, &end);
        if (end == p) break;
        v.push_back(x);
        p = end;
    }
    size_t n = v.size() / 2;
    // The reference reads pairs until end of file and drops the last point when it repeats
    // the one before it (within 1e-6). After trailing white space its final read fails and
    // leaves a copy of the last point, which that check removes; a file that ends on its last
    // number instead loses a genuinely repeated last point.
    const bool ends_on_number = n > 0 && v.size() % 2 == 0 && *p == '\0';
    if (ends_on_number && n >= 2 &&
        std::hypot(v[2 * n - 2] - v[2 * n - 4], v[2 * n - 1] - v[2 * n - 3]) < 1e-6)
        --n;
    if (n > 0 && m.n_el == 0) return {3, "sample points given for a mesh without elements"};
    const int L2 = m.lnod * m.lnod;
    sp.xy.assign(v.begin(), v.begin() + 2 * n);
    sp.elem.resize(n);
    sp.shape.assign(n * L2, 0.0);
    for (size_t s = 0; s < n; ++s) {
        sp.elem[s] = locate(m, sp.xy[2 * s], sp.xy[2 * s + 1]);
        local_shape(m, sp.elem[s], sp.xy[2 * s], sp.xy[2 * s + 1], &sp.shape[s * L2]);
    }
    return {0, ""};
}

}  // namespace ho2d
