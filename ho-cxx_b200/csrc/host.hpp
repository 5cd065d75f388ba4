// host.hpp -- host-side setup of the B200 HO-CXX solver: input.dat, Gmsh mesh, bases,
// metrics, boundary conditions and the Poisson operator in block form.
//
// Layouts (all flat, row-major):
//   volume fields      [el][j][i]            (j = eta index, i = xi index)
//   face traces        [el][ijp][k]          ijp 0 = W (xi=-1), 1 = E, 2 = S (eta=-1), 3 = N
//   boundary arrays    [edge][k]             edge in boundary-edge (file) order
//   Poisson blocks     [el][slot][rs][ij]    slot 0 = element itself, 1..4 = face ijp 0..3;
//                      stored transposed (column rs outer) so that consecutive threads
//                      (one per output row ij) read consecutive addresses.
#pragma once

#include <cstdint>
#include <string>
#include <thread>
#include <vector>

#include "assemble_element.hpp"
#include "vtk_nodes.hpp"

namespace ho2d {

constexpr int kMaxK = 8;
constexpr int DIRICHLET = 0, NEUMANN = 1;
// element sides (counter-clockwise from the bottom, src/Mesh.hpp:114-119)
constexpr int SOUTH = 0, EAST = 1, NORTH = 2, WEST = 3;
// ijp -> element side and back (src/MathHelpers.hpp:23-24)
constexpr int kI2F[4] = {WEST, EAST, SOUTH, NORTH};
constexpr int kF2I[4] = {2, 1, 3, 0};

struct Error {
    int code;
    std::string msg;
};

// Positional input.dat fields (src/HO_2D.cpp:213-317).
struct Input {
    int nel_i = 0, nel_j = 0;
    int knod = 2;
    int lnod_in = 1;
    std::string mesh_file;
    std::string base_dir;
    int occ = 0;
    double reyn_inv = 0.001;
    double dx_ratio = 1.0, fac = 0.0;
    int huynh = 2;
    int ti_type = 4;
    int adv_type = 1;
    int problem_type = 1;
    int num_steps = 0;
    double dt = 0.001;
    int dump_freq = 1000;
    int fast = 0;
    int lhs_type = 3;
    std::string sample_file;
};

// Mesh after reading and processing; element sides in SENW order.
struct Mesh {
    int n_el = 0, lnod = 2, n_eb = 0;
    std::vector<double> node_xy;               // [n_nodes][2]
    std::vector<std::vector<int>> elem_nodes;  // Gmsh node slots per element
    std::vector<std::vector<int>> edge_nodes;  // boundary edges first (file order), element CCW orientation
    std::vector<std::string> group_names;
    std::vector<std::vector<int>> group_edges;
    std::vector<int> nbr, nbr_side, bidx;      // [n_el][4] by side; -1 where absent
    std::vector<int> be_el, be_side, be_group; // [n_eb]
    // boundaries loaded from arrays (hybrid drivers): per-edge normal / parallel velocity
    // given with the edge (NaN where none was given)
    std::vector<double> edge_normvel, edge_parlvel;
};

// 1-D bases on the K Gauss-Legendre solution points and the L equispaced geometry nodes.
struct Bases {
    int K = 0, L = 0;
    std::vector<double> xs, w;          // [K]
    std::vector<double> sbb, sbgb;      // [K][2]  l_k(-1), l_k(+1) and derivatives
    std::vector<double> D;              // [K][K]  D[k][m] = l_k'(x_m)
    std::vector<double> R, gR;          // [K][2]  Radau g_L/g_R values and derivatives
    std::vector<double> gsb, gsgb;      // [L][K]  geometry basis (and derivative) at the sps
    std::vector<double> gbb, gbgb;      // [L][2]  geometry basis (and derivative) at -1, +1
    double gp[2] = {0.0, 0.0};          // g'(-1), g'(+1) of g_DG
};

struct Metrics {
    std::vector<double> xxi, xeta, yxi, yeta, J;  // [N][K][K]
    std::vector<double> G;                        // [N][K][K][2][2]  (g_r . g_s) / J
    std::vector<double> GB;                       // [N][2][2][K][2]
    std::vector<double> fA, fB, fJ, fAn;          // [N][4][K]
};

struct BoundaryConditions {
    std::vector<int> sw_p, sw_d;                   // [N_eb] DIRICHLET / NEUMANN
    std::vector<int> noslip;                       // [n_groups]
    std::vector<double> bc_p, bc_nv, bc_pv, bc_d;  // [N_eb][K]
    std::vector<double> edge_y;                    // [N_eb][K] y at the edge's solution points
    std::vector<int> role;                         // [N_eb] time-dependent role (see BcRole)
    std::vector<double> inlet_nv;                  // [N_eb] hybrid inlets: the edge's normal velocity
    double y_min = 0.0, y_max = 0.0;
};

// Per-edge role in the time-dependent BC refresh of src/HO_2D.cpp:1979-2217.
// ROLE_OPEN / ROLE_WALL_H / ROLE_INLET_H: the "open", "wall" and "inlet" boundaries of a
// hybrid run (problem type 11, 2104-2191).
enum BcRole {
    ROLE_NONE = 0,
    ROLE_INLET = 1,
    ROLE_TOP = 2,
    ROLE_BOTTOM = 3,
    ROLE_OBJECT = 4,
    ROLE_OPEN = 5,
    ROLE_WALL_H = 6,
    ROLE_INLET_H = 7
};

// Poisson operator: 5 K^2 x K^2 blocks per element (transposed) and the boundary source.
// The device applies the operator matrix-free; of the blocks it needs only the inverse
// diagonal blocks and sums, so the blocks themselves (5 K^4 values per element, 25 GB at
// 262,144 elements and K = 7) are kept only on request.
struct PoissonOperator {
    int K2 = 0;
    std::vector<double> blocks;   // [N][5][K2][K2] (rs outer, ij inner); empty unless kept
    std::vector<int> block_col;   // [N][5] column element (-1 = empty slot)
    std::vector<double> bsrc;     // [N_eb][K2][K]
    std::vector<double> dinv;     // [N][K2][K2] inverse of the diagonal block (rs outer)
    std::vector<double> rowsum;   // [N][5][K2] sum over rs of each block row (rs ascending)
    std::vector<double> colsum;   // [N][5][K2] sum over ij of each block column (ij ascending)
    std::vector<double> bsum;     // [N][5] sum of each block's entries (stored order)
    int64_t nnz = 0;              // entries surviving the |a| > 1e-14 filter
};

Error read_input(const std::string& path, Input& in);
Error read_msh(const std::string& path, int occ, Mesh& mesh);
Error process_mesh(Mesh& mesh);
Error mesh_from_arrays(int iorder, int nxy, const double* xy, int nidx, const int* idx, int nwall, const int* wall,
                       int nopen, const int* open, Mesh& m);
Error add_boundary_arrays(Mesh& m, const std::string& name, int n, const int* idx, int nval, const double* vals);
Error make_bases(int K, int L, Bases& B);
void make_metrics(const Mesh& mesh, const Bases& B, Metrics& M);
Error setup_bcs(const Input& in, const Mesh& mesh, const Bases& B, BoundaryConditions& bc);
// Per-element data of the Kronecker-sum smoother (host_kron.cpp): the factors of each
// element's fitted diagonal block, and the elements that keep the exact inverse block
// (fit rejected, or ||I - M D||_2 > kKronDefectMax).
constexpr double kKronDefectMax = 0.5;
struct KronSmoother {
    int K = 0;
    std::vector<double> v;              // [N][4][K][K]: Vx, Vx^-1, Vy, Vy^-1
    std::vector<double> lam;            // [N][2][K]: lx, ly
    std::vector<unsigned char> exact;   // [N]: 1 = the exact inverse block is used
    std::vector<double> defect;         // [N]: ||I - M D||_2 (infinity where rejected)
};
struct KronFit;
void kron_store(const KronFit* f, double defect, int el, KronSmoother& ks);
// The device arrays of the Kronecker-sum smoother: per element its 4K^2 factors and 2K
// eigenvalues [N][4K^2 + 2K] (zero where the exact block is used), the index of its exact
// inverse block in the compact array, or -1 [N], and those blocks [n_exact][K^2][K^2]
// taken from dinv (same [rs][ij] layout).
// The fit of every element's filtered diagonal block diag [N][K2][K2] (row ij, column rs),
// as assemble_poisson makes it while the blocks stream by.
void kron_fit_blocks(int K, int N, const double* diag, KronSmoother& ks);
// The packed factors [N][4 K2 + 2 K] (zero for exact elements) and the exact-block index
// (-1 for fitted elements, else the element's rank among the exact ones).
void kron_factor_arrays(const KronSmoother& ks, std::vector<double>& factors, std::vector<int>& exact_index);
void kron_device_arrays(const KronSmoother& ks, const std::vector<double>& dinv, std::vector<double>& factors,
                        std::vector<int>& exact_index, std::vector<double>& exact_blocks);

void assemble_poisson(const Mesh& mesh, const Bases& B, const Metrics& M, const BoundaryConditions& bc,
                      PoissonOperator& op, bool keep_blocks = false, KronSmoother* kron = nullptr);
// The coefficient lists of the block assembly (one entry per (row, metric slot)): volume
// rows ij * K2 + rs, face (d, t) rows ij * K + q at index d * 2 + t.
struct AsmCoefficients {
    std::vector<AsmEntry> vol, fw[4];
    AsmTables tables() const {
        AsmTables t{vol.data(), (int)vol.size(), {}, {}};
        for (int f = 0; f < 4; ++f) {
            t.fw[f] = fw[f].data();
            t.nfw[f] = (int)fw[f].size();
        }
        return t;
    }
};
AsmCoefficients assembly_coefficients(const Bases& B);
AsmBases asm_bases(const Bases& B);
int tensor2fem(int i, int j, int lnod_in);

// Fields written by the VTK output: volume arrays [N][K][K] (vorticity, streamfunction,
// Cartesian velocity components, the two RHS terms), boundary arrays [N_eb][K]
// (BC_vorticity, BC_normal_vel in the local h direction, BC_parl_vel).
struct VtkFields {
    const double *w, *psi, *u, *v, *rhs_diff, *rhs_adv;
    const double *bc_w, *bc_nv, *bc_pv;
    // the smooth file's node averages [nodes] and sample values [n][3] when already made
    // (on the device); null: made on the host from the fields above
    const double *nw = nullptr, *np = nullptr, *nux = nullptr, *nuy = nullptr, *samp = nullptr;
};
// Tables of the node interpolation (vtk_nodes.hpp) for a mesh: sgb [K][L], the Gmsh slot of
// each (ly, lx) and the element node slots flattened [N][L^2].
struct VtkGeoHost {
    VtkGeoHost(const Mesh& m, const Bases& B);
    VtkGeo geo() const;
    const Mesh& mesh;
    const Bases& bases;
    std::vector<double> sgb;
    std::vector<int> t2f, nodes;
};
// Points of the input's sample-points file (read_process_sample_points, host_samples.cpp):
// coordinates [n][2], the element that holds each point, and the Lnod^2 geometry shape
// functions (Gmsh node slots) at its local coordinates [n][Lnod^2].
struct SamplePoints {
    std::vector<double> xy;
    std::vector<int> elem;
    std::vector<double> shape;
    size_t size() const { return elem.size(); }
};
// A missing file gives no points (no error), as in the reference.
Error read_sample_points(const std::string& path, const Mesh& m, SamplePoints& sp);

// save_vorticity_vtk + save_smooth_vtk (src/HO_2D.cpp:3369-3692) into dir ("" = working
// directory); subidx < 0 leaves it out of the file names. With sample points (may be null)
// also sampling_points<p>_K<K>_L<Lnod>_<indx>.dat.
Error write_vtk_files(const Mesh& mesh, const Bases& B, int problem_type, const VtkFields& f, int indx, int subidx,
                      const std::string& dir, const SamplePoints* samples = nullptr);
int tensor2fem_1d(int i, int lnod_in);

// The VTK files of one dump written on a background thread, so that the time loop goes on
// while the ASCII files are formatted. The job owns host copies of the fields; the mesh,
// bases and sample points are read in place and must not change until wait() returns.
// One write is in flight at a time: submit() first waits for the previous one. wait()
// returns the first error since the last wait(); the destructor waits.
class VtkQueue {
  public:
    struct Job {
        std::vector<double> w, psi, u, v, rhs_diff, rhs_adv, bc_w, bc_nv, bc_pv;
        std::vector<double> nw, np, nux, nuy, samp;  // node averages and sample values (device-made)
        VtkFields fields() const {
            auto p = [](const std::vector<double>& v) { return v.empty() ? nullptr : v.data(); };
            return VtkFields{p(w),     p(psi),   p(u),     p(v),   p(rhs_diff), p(rhs_adv), p(bc_w),
                             p(bc_nv), p(bc_pv), p(nw),    p(np),  p(nux),      p(nuy),     p(samp)};
        }
        int problem_type = 0, indx = 0, subidx = -1;
        std::string dir;
    };
    VtkQueue() = default;
    VtkQueue(const VtkQueue&) = delete;
    VtkQueue& operator=(const VtkQueue&) = delete;
    ~VtkQueue() { wait(); }
    Error submit(const Mesh& mesh, const Bases& B, const SamplePoints* samples, Job job);
    Error wait();

  private:
    std::thread thread_;
    Error err_{0, ""};
};

// Kronecker-sum approximation of an element's diagonal Poisson block (host_kron.cpp):
// D ([ij][rs], K^2 x K^2) ~ I (x) Ax + Ay (x) I with Ax = Vx diag(lx) Vx^-1 and
// Ay = Vy diag(ly) Vy^-1, all [K][K] row-major, eigenvectors as columns.
struct KronFit {
    int K = 0;
    std::vector<double> vx, vxi, vy, vyi, lx, ly;
};
// Real eigenvalues of the n x n row-major A (false if a complex pair or no convergence).
bool real_eigenvalues(int n, const double* A, double* lambda);
// Eigenvectors for those eigenvalues as the columns of V (false if that fails).
bool eigenvectors(int n, const double* A, const double* lambda, double* V);
// Fit and factor; false when an eigenvalue is complex, a factor is singular or some
// ly_j + lx_i vanishes (the exact inverse block is then the smoother's).
bool kron_fit(int K, const double* D, KronFit& f);
// z = (I (x) Ax + Ay (x) I)^-1 r for r, z [j][i]
void kron_apply(const KronFit& f, const double* r, double* z);
// ||I - M D||_2 of the fitted inverse M against the block it approximates (power
// iteration: an estimate from below, to about 1e-3 relative)
double kron_defect(const KronFit& f, const double* D);

// The BF16 bit pattern of a finite float, rounded to nearest with ties to even (the upper
// 16 bits after adding 0x7FFF plus the lowest kept bit).
inline uint16_t bf16_bits(float f) {
    uint32_t u;
    static_assert(sizeof(u) == sizeof(f), "float is 32 bits");
    __builtin_memcpy(&u, &f, 4);
    u += 0x7FFFu + ((u >> 16) & 1u);
    return (uint16_t)(u >> 16);
}

// Hybrid operation (host_hybrid.cpp): the edges of the "open" boundary (null if none), the
// getopenpts_d array length, solution-point areas [N][K][K], open-boundary points
// [open edge][K][x, y], outward unit normals of the open edges [N_eb][K][2], and the
// normal / parallel split of the driver's open-boundary velocities into [N_eb][K] arrays.
const std::vector<int>* open_boundary_edges(const Mesh& m);
int open_point_count(const Mesh& m, int K);
void solution_areas(const Bases& B, const Metrics& M, int n_el, double* out);
void open_points(const Mesh& m, const Bases& B, double* out);
void open_normals(const Mesh& m, const Bases& B, const Metrics& M, const BoundaryConditions& bc,
                  std::vector<double>& nrm);
void split_open_velocities(const Mesh& m, int K, const std::vector<double>& nrm, const double* xyvel, double* vn,
                           double* vp);

}  // namespace ho2d
