// host_io.cpp -- input.dat and Gmsh 4.1 readers.
//
// read_input follows the positional format of HO_2D::read_input_file
// (src/HO_2D.cpp:213-317): every value is preceded by one comment line, two extra lines
// follow the OCC flag, and anything after the sample-points file name is ignored.
//
// read_msh follows Mesh::read_msh_file and Mesh::process_mesh (src/Mesh.cpp:93-487):
// dimension-1 physical names become the named boundaries; line elements of curves that
// carry a physical tag become boundary edges in file order; quads are read in slot
// order and reoriented when the OCC flag is set. Neighbours are found through a hash of
// each edge's corner pair (O(N)), which yields the same tables as the reference's
// O(N^2) scan because every interior edge has exactly two owners; boundary edges take
// the orientation of their element (src/Mesh.cpp:373-375).
#include <algorithm>
#include <cmath>
#include <fstream>
#include <limits>
#include <sstream>
#include <unordered_map>

#include "host.hpp"

namespace ho2d {

#define HO2D_HOST_TRY(expr)     \
    do {                        \
        Error _e = (expr);      \
        if (_e.code) return _e; \
    } while (0)

namespace {

std::string dirname_of(const std::string& path) {
    const size_t s = path.find_last_of('/');
    return s == std::string::npos ? std::string(".") : path.substr(0, s);
}

std::string rstrip(std::string s) {
    while (!s.empty() && (s.back() == '\r' || s.back() == ' ' || s.back() == '\t')) s.pop_back();
    return s;
}

}  // namespace

int tensor2fem_1d(int i, int lnod_in) { return i == 0 ? 0 : (i == lnod_in ? 1 : i + 1); }

int tensor2fem(int i, int j, int lnod_in) {
    static const int q2[3][3] = {{0, 4, 1}, {7, 8, 5}, {3, 6, 2}};
    static const int q3[4][4] = {{0, 4, 5, 1}, {11, 12, 13, 6}, {10, 15, 14, 7}, {3, 9, 8, 2}};
    if (lnod_in == 1) return i + 3 * j - 2 * i * j;
    if (lnod_in == 2) return q2[j][i];
    if (lnod_in == 3) return q3[j][i];
    return -1;
}

Error read_input(const std::string& path, Input& in) {
    std::ifstream f(path);
    if (!f) return {2, "cannot open input file " + path};
    std::string line;
    auto skip = [&]() { std::getline(f, line); };
    auto rest = [&]() { f.ignore(std::numeric_limits<std::streamsize>::max(), '\n'); };
    char comma = 0;
    double reyn = 0.0;
    skip(); f >> in.nel_i >> comma >> in.nel_j; rest();
    skip(); f >> in.knod; rest();
    skip(); f >> in.lnod_in; rest();
    skip(); f >> in.mesh_file; rest();
    skip(); f >> in.occ; rest();
    skip(); skip();
    skip(); f >> reyn; rest();
    skip(); f >> in.dx_ratio; rest();
    skip(); f >> in.fac; rest();
    skip(); f >> in.huynh; rest();
    skip(); f >> in.ti_type; rest();
    skip(); f >> in.adv_type; rest();
    skip(); f >> in.problem_type; rest();
    skip(); f >> in.num_steps; rest();
    skip(); f >> in.dt; rest();
    skip(); f >> in.dump_freq; rest();
    skip(); f >> in.fast; rest();
    skip(); f >> in.lhs_type; rest();
    skip(); f >> in.sample_file; rest();
    if (f.fail() && !f.eof()) return {2, "malformed input file " + path};
    if (in.mesh_file.empty()) return {2, "input file " + path + " names no mesh file"};
    in.reyn_inv = reyn > 1e-3 ? 1.0 / reyn : -1.0;  // src/HO_2D.cpp:255
    in.base_dir = dirname_of(path);
    if (in.knod < 1 || in.knod > kMaxK) return {4, "Knod must be in 1.." + std::to_string(kMaxK)};
    if (in.huynh != 2) return {4, "only HuynhSolver_type 2 (g_DG) is implemented"};
    if (in.ti_type != 1 && in.ti_type != 2 && in.ti_type != 4) return {4, "time integration must be 1, 2 or 4"};
    if (in.adv_type != 1 && in.adv_type != 2) return {4, "advection type must be 1 or 2"};
    if (in.problem_type < 1 || in.problem_type > 3) return {4, "problem types 1, 2 and 3 are implemented"};
    if (!(in.dt > 0.0)) return {1, "dt must be positive"};
    if (in.dump_freq <= 0) in.dump_freq = 1;
    return {0, ""};
}

namespace {

bool locate(std::ifstream& f, const std::string& key) {
    std::string line;
    while (std::getline(f, line))
        if (rstrip(line) == key) return true;
    return false;
}

int edge_nodes_of_type(int t) {
    switch (t) {
        case 1: return 2;
        case 8: return 3;
        case 26: return 4;
        case 27: return 5;
        case 28: return 6;
        default: return -1;
    }
}

int face_nodes_of_type(int t) {
    switch (t) {
        case 3: return 4;
        case 10: return 9;
        case 16: return 8;
        case 36: return 16;
        case 37: return 25;
        default: return -1;
    }
}

int face_edge_nodes(int n_face_nodes) {
    switch (n_face_nodes) {
        case 4: return 2;
        case 9: return 3;
        case 8: return 3;
        case 16: return 4;
        case 25: return 5;
        default: return -1;
    }
}

}  // namespace

Error read_msh(const std::string& path, int occ, Mesh& m) {
    std::ifstream f(path);
    if (!f) return {2, "cannot open mesh file " + path};
    std::string line;
    if (!locate(f, "$PhysicalNames")) return {3, "no $PhysicalNames section in " + path};
    int nphys = 0;
    f >> nphys;
    std::getline(f, line);
    std::vector<int> btags;
    for (int i = 0; i < nphys; ++i) {
        if (!std::getline(f, line)) return {3, "truncated $PhysicalNames"};
        std::istringstream ls(line);
        int dim = 0, tag = 0;
        std::string name;
        ls >> dim >> tag >> name;
        if (dim != 1) continue;
        if (name.size() >= 2 && name.front() == '"') name = name.substr(1, name.size() - 2);
        btags.push_back(tag);
        m.group_names.push_back(name);
    }
    m.group_edges.assign(btags.size(), {});
    if (!locate(f, "$Entities")) return {3, "no $Entities section in " + path};
    int npt = 0, ncv = 0, nsf = 0, nvol = 0;
    f >> npt >> ncv >> nsf >> nvol;
    std::getline(f, line);
    if (nvol != 0) return {3, "the mesh has volumes; a 2-D mesh is expected"};
    for (int i = 0; i < npt; ++i) std::getline(f, line);
    std::unordered_map<int, int> curve_phys;
    for (int i = 0; i < ncv; ++i) {
        if (!std::getline(f, line)) return {3, "truncated $Entities"};
        std::istringstream ls(line);
        int tag = 0, nt = 0, ph = 0;
        double bb[6];
        ls >> tag >> bb[0] >> bb[1] >> bb[2] >> bb[3] >> bb[4] >> bb[5] >> nt;
        if (nt > 0) ls >> ph;
        curve_phys[tag] = nt > 0 ? ph : 0;
    }
    if (!locate(f, "$Nodes")) return {3, "no $Nodes section in " + path};
    long nblk = 0, nnodes = 0, nmin = 0, nmax = 0;
    f >> nblk >> nnodes >> nmin >> nmax;
    std::getline(f, line);
    if (nmax < nmin || nnodes <= 0) return {3, "bad $Nodes header"};
    std::vector<double> raw_xy(2 * (size_t)(nmax - nmin + 1), std::nan(""));
    for (long b = 0; b < nblk; ++b) {
        int edim = 0, etag = 0, param = 0;
        long cnt = 0;
        f >> edim >> etag >> param >> cnt;
        std::getline(f, line);
        std::vector<long> tags(cnt);
        for (long k = 0; k < cnt; ++k) {
            f >> tags[k];
            std::getline(f, line);
        }
        for (long k = 0; k < cnt; ++k) {
            double x = 0, y = 0, z = 0;
            f >> x >> y >> z;
            std::getline(f, line);
            const long t = tags[k] - nmin;
            if (t < 0 || t >= (long)raw_xy.size() / 2) return {3, "node tag out of range"};
            raw_xy[2 * t] = x;
            raw_xy[2 * t + 1] = y;
        }
    }
    if (!f) return {3, "truncated $Nodes section"};
    if (!locate(f, "$Elements")) return {3, "no $Elements section in " + path};
    long eblk = 0, nelem = 0, emin = 0, emax = 0;
    f >> eblk >> nelem >> emin >> emax;
    std::getline(f, line);
    std::vector<std::vector<long>> edges_raw, quads_raw;
    int last_edge_nodes = -1;
    for (long b = 0; b < eblk; ++b) {
        int edim = 0, etag = 0, etype = 0;
        long cnt = 0;
        f >> edim >> etag >> etype >> cnt;
        std::getline(f, line);
        if (edim == 0) {
            for (long k = 0; k < cnt; ++k) std::getline(f, line);
        } else if (edim == 1) {
            const int nn = edge_nodes_of_type(etype);
            if (nn < 0) return {3, "unsupported line element type " + std::to_string(etype)};
            last_edge_nodes = nn;
            auto it = curve_phys.find(etag);
            const int ph = it == curve_phys.end() ? 0 : it->second;
            if (ph == 0) {  // interface curve without a physical name: skipped
                for (long k = 0; k < cnt; ++k) std::getline(f, line);
                continue;
            }
            const auto gi = std::find(btags.begin(), btags.end(), ph);
            if (gi == btags.end()) return {3, "curve references an unknown physical tag"};
            const int g = (int)(gi - btags.begin());
            for (long k = 0; k < cnt; ++k) {
                long tag = 0;
                f >> tag;
                std::vector<long> nodes(nn);
                for (int j = 0; j < nn; ++j) f >> nodes[j];
                std::getline(f, line);
                m.group_edges[g].push_back((int)edges_raw.size());
                edges_raw.push_back(nodes);
            }
        } else if (edim == 2) {
            const int nn = face_nodes_of_type(etype);
            if (nn < 0) return {3, "unsupported surface element type " + std::to_string(etype)};
            for (long k = 0; k < cnt; ++k) {
                long tag = 0;
                f >> tag;
                std::vector<long> nodes(nn);
                for (int j = 0; j < nn; ++j) f >> nodes[j];
                std::getline(f, line);
                quads_raw.push_back(nodes);
            }
        } else {
            return {3, "elements of dimension 3 in a 2-D mesh"};
        }
        if (!f) return {3, "truncated $Elements section"};
    }
    if (quads_raw.empty()) return {3, "the mesh has no quadrilateral elements"};
    if (last_edge_nodes < 2) return {3, "the mesh has no boundary line elements"};
    m.lnod = last_edge_nodes;
    const int lin = m.lnod - 1;
    if (m.lnod > 4) return {4, "geometry order above cubic (Lnod > 4) is not supported"};
    for (auto& q : quads_raw)
        if (face_edge_nodes((int)q.size()) != m.lnod || (int)q.size() != m.lnod * m.lnod) {
            if (face_edge_nodes((int)q.size()) != m.lnod) return {3, "quad and line element orders differ"};
            return {4, "serendipity quads are not supported"};
        }
    if (occ) {  // src/Mesh.cpp:276-287
        for (auto& q : quads_raw) {
            std::vector<long> old = q;
            for (int jo = 0; jo < m.lnod; ++jo)
                for (int io = 0; io < m.lnod; ++io)
                    q[tensor2fem(lin - jo, lin - io, lin)] = old[tensor2fem(io, jo, lin)];
        }
    }
    // compact node numbering over the nodes actually referenced
    std::vector<int> remap(raw_xy.size() / 2, -1);
    auto use = [&](long tag) -> int {
        const long t = tag - nmin;
        if (t < 0 || t >= (long)remap.size() || std::isnan(raw_xy[2 * t])) return -1;
        if (remap[t] < 0) {
            remap[t] = (int)(m.node_xy.size() / 2);
            m.node_xy.push_back(raw_xy[2 * t]);
            m.node_xy.push_back(raw_xy[2 * t + 1]);
        }
        return remap[t];
    };
    m.edge_nodes.resize(edges_raw.size());
    for (size_t e = 0; e < edges_raw.size(); ++e)
        for (long t : edges_raw[e]) {
            const int v = use(t);
            if (v < 0) return {3, "a line element references a missing node"};
            m.edge_nodes[e].push_back(v);
        }
    m.elem_nodes.resize(quads_raw.size());
    for (size_t q = 0; q < quads_raw.size(); ++q)
        for (long t : quads_raw[q]) {
            const int v = use(t);
            if (v < 0) return {3, "a quad references a missing node"};
            m.elem_nodes[q].push_back(v);
        }
    return process_mesh(m);
}

// Neighbour search and boundary-edge ownership (src/Mesh.cpp:342-487, hash-based): fills
// n_el, n_eb, nbr, nbr_side, bidx, be_el, be_side, be_group from node_xy, elem_nodes,
// edge_nodes (boundary edges, group by group) and group_edges. Boundary edges take the
// orientation of the element side they cover.
Error process_mesh(Mesh& m) {
    m.n_el = (int)m.elem_nodes.size();
    m.n_eb = (int)m.edge_nodes.size();
    if (m.n_el == 0) return {3, "the mesh has no elements"};
    // process_mesh: identify edges by their corner pair
    auto key = [](int a, int b) { return ((uint64_t)(uint32_t)std::min(a, b) << 32) | (uint32_t)std::max(a, b); };
    std::unordered_map<uint64_t, int> edge_of;
    edge_of.reserve(2 * (size_t)m.n_el + m.n_eb);
    for (int e = 0; e < m.n_eb; ++e) edge_of.emplace(key(m.edge_nodes[e][0], m.edge_nodes[e][1]), e);
    const int ene = m.lnod;
    std::vector<int> elem_edge((size_t)m.n_el * 4);
    int next_edge = m.n_eb;
    for (int el = 0; el < m.n_el; ++el) {
        const auto& q = m.elem_nodes[el];
        for (int s = 0; s < 4; ++s) {
            const int a = q[s], b = q[(s + 1) % 4];
            auto it = edge_of.find(key(a, b));
            int e;
            if (it == edge_of.end()) {
                e = next_edge++;
                edge_of.emplace(key(a, b), e);
            } else {
                e = it->second;
                if (e < m.n_eb) {  // boundary edge: adopt the element's orientation
                    std::vector<int> en = {a, b};
                    for (int k = 0; k < ene - 2; ++k) en.push_back(q[4 + s * (ene - 2) + k]);
                    m.edge_nodes[e] = en;
                }
            }
            elem_edge[(size_t)el * 4 + s] = e;
        }
    }
    // owners of each edge, lowest (element, side) first as in the reference's scan order
    std::vector<int> own_a((size_t)next_edge, -1), own_b((size_t)next_edge, -1);
    for (int el = 0; el < m.n_el; ++el)
        for (int s = 0; s < 4; ++s) {
            const int e = elem_edge[(size_t)el * 4 + s];
            const int code = el * 4 + s;
            if (own_a[e] < 0) own_a[e] = code;
            else if (own_b[e] < 0) own_b[e] = code;
            else return {3, "an edge is shared by more than two elements"};
        }
    m.nbr.assign((size_t)m.n_el * 4, -1);
    m.nbr_side.assign((size_t)m.n_el * 4, -1);
    m.bidx.assign((size_t)m.n_el * 4, -1);
    m.be_el.assign(m.n_eb, -1);
    m.be_side.assign(m.n_eb, -1);
    for (int el = 0; el < m.n_el; ++el)
        for (int s = 0; s < 4; ++s) {
            const int e = elem_edge[(size_t)el * 4 + s];
            const int me = el * 4 + s;
            const int other = own_a[e] == me ? own_b[e] : own_a[e];
            if (other >= 0) {
                m.nbr[(size_t)el * 4 + s] = other / 4;
                m.nbr_side[(size_t)el * 4 + s] = other % 4;
            } else {
                if (e >= m.n_eb) return {3, "an element side lies on the boundary but no boundary line covers it"};
                m.bidx[(size_t)el * 4 + s] = e;
                m.be_el[e] = el;
                m.be_side[e] = s;
            }
        }
    for (int e = 0; e < m.n_eb; ++e)
        if (m.be_el[e] < 0) return {3, "a boundary line element matches no element side"};
    m.be_group.assign(m.n_eb, -1);
    for (size_t g = 0; g < m.group_edges.size(); ++g)
        for (int e : m.group_edges[g]) m.be_group[e] = (int)g;
    return {0, ""};
}

// load_mesh_arrays_d (src/HO_2D.cpp:3823-3881): nodes [nxy/2][2], elements of Lnod^2 node
// indices each (Gmsh order), then the boundaries named "wall" and "open" as Lnod-node
// edges. Boundaries "inlet" and "outlet" follow through add_boundary_arrays.
Error mesh_from_arrays(int iorder, int nxy, const double* xy, int nidx, const int* idx, int nwall, const int* wall,
                       int nopen, const int* open, Mesh& m) {
    m = Mesh();
    m.lnod = iorder + 1;
    if (m.lnod < 2 || m.lnod > 4) return {4, "geometry order must be 1, 2 or 3 (Lnod 2..4)"};
    if (nxy < 2 || nxy % 2 || !xy) return {1, "node array must hold x, y pairs"};
    m.node_xy.assign(xy, xy + nxy);
    const int nper = m.lnod * m.lnod, nn = nxy / 2;
    if (nidx <= 0 || nidx % nper || !idx) return {1, "element index array is not a multiple of Lnod^2"};
    m.elem_nodes.resize(nidx / nper);
    for (size_t e = 0; e < m.elem_nodes.size(); ++e) {
        m.elem_nodes[e].assign(idx + e * nper, idx + (e + 1) * nper);
        for (int v : m.elem_nodes[e])
            if (v < 0 || v >= nn) return {3, "an element references a node outside the node array"};
    }
    if (nwall > 0) HO2D_HOST_TRY(add_boundary_arrays(m, "wall", nwall, wall, 0, nullptr));
    if (nopen > 0) HO2D_HOST_TRY(add_boundary_arrays(m, "open", nopen, open, 0, nullptr));
    return {0, ""};
}

// arrays_to_boundary (src/HO_2D.cpp:3724-3820): one boundary group of n/Lnod edges, with
// nval optional values: one per edge (normal velocity) or two (parallel, then normal).
Error add_boundary_arrays(Mesh& m, const std::string& name, int n, const int* idx, int nval, const double* vals) {
    if (n <= 0) return {0, ""};
    if (!idx || n % m.lnod) return {1, "boundary " + name + ": index array is not a multiple of Lnod"};
    const int ne = n / m.lnod, nn = (int)m.node_xy.size() / 2;
    int per = 0;
    if (nval > 0) {
        if (!vals || nval % ne || nval / ne > 2) return {1, "boundary " + name + ": expected 1 or 2 values per edge"};
        per = nval / ne;
    }
    m.group_names.push_back(name);
    m.group_edges.emplace_back();
    for (int i = 0; i < ne; ++i) {
        std::vector<int> en(idx + (size_t)i * m.lnod, idx + (size_t)(i + 1) * m.lnod);
        for (int v : en)
            if (v < 0 || v >= nn) return {3, "boundary " + name + " references a node outside the node array"};
        m.group_edges.back().push_back((int)m.edge_nodes.size());
        m.edge_nodes.push_back(en);
        m.edge_normvel.push_back(per == 1 ? vals[i] : (per == 2 ? vals[2 * i + 1] : std::nan("")));
        m.edge_parlvel.push_back(per == 2 ? vals[2 * i] : std::nan(""));
    }
    return {0, ""};
}

}  // namespace ho2d
