// sanitizer_driver.cpp -- the library's host code (mesh reader, setup, streamed and
// Kronecker-sum assembly, coarse hierarchy and its ELL copies, sample points, the VTK queue,
// hybrid geometry) run end to end on the given inputs, for a build with AddressSanitizer
// and UndefinedBehaviorSanitizer (tests/test_host_setup_cpu.py). Arguments: pairs of
// input.dat and sample-points file ("-" for none), and the directory the VTK files go to.
// Never part of the library.
#include <algorithm>
#include <cstdio>
#include <string>
#include "host.hpp"
#include "host_amg.hpp"
using namespace ho2d;
static int run(const char* input, const char* samples, bool kron, const char* outdir) {
    Input in; Error e = read_input(input, in); if (e.code) { printf("input %s\n", e.msg.c_str()); return 1; }
    Mesh m; e = read_msh(in.base_dir + "/" + in.mesh_file, in.occ, m); if (e.code) { printf("msh %s\n", e.msg.c_str()); return 1; }
    Bases B; make_bases(in.knod, m.lnod, B); Metrics M; make_metrics(m, B, M);
    BoundaryConditions bc; e = setup_bcs(in, m, B, bc); if (e.code) { printf("bc %s\n", e.msg.c_str()); return 1; }
    PoissonOperator op; KronSmoother ks; assemble_poisson(m, B, M, bc, op, true, kron ? &ks : nullptr);
    Csr A1 = p0_coarse_operator(op, m.n_el); CoarseHierarchy H; e = build_coarse_hierarchy(A1, H, 8, 8);
    for (auto& L : H.levels) { to_ell(L.A); if (!L.M.val.empty()) { to_ell(L.M); to_ell(L.S); to_ell(L.Q); } }
    SamplePoints sp; if (samples) read_sample_points(samples, m, sp);
    const size_t nv = (size_t)m.n_el * B.K * B.K, nb = (size_t)m.n_eb * B.K;
    std::vector<double> f(nv, 0.5), g(nb, 0.25);
    VtkQueue q;
    VtkQueue::Job j; j.w = f; j.psi = f; j.u = f; j.v = f; j.rhs_diff = f; j.rhs_adv = f; j.bc_w = g; j.bc_nv = g; j.bc_pv = g;
    j.problem_type = in.problem_type; j.indx = 1; j.dir = outdir;
    q.submit(m, B, &sp, std::move(j)); e = q.wait();
    std::vector<double> areas(nv), opts(open_point_count(m, B.K) + 1); solution_areas(B, M, m.n_el, areas.data()); open_points(m, B, opts.data());
    printf("%s: N %d K %d L %d levels %zu samples %zu kron-exact %zu vtk %d\n", input, m.n_el, B.K, m.lnod, H.levels.size(), sp.size(),
           kron ? (size_t)std::count(ks.exact.begin(), ks.exact.end(), 1) : 0, e.code);
    return 0;
}
int main(int argc, char** argv) {
    int rc = 0;
    for (int i = 1; i + 2 < argc; i += 2)
        rc |= run(argv[i], std::string(argv[i + 1]) == "-" ? nullptr : argv[i + 1], true, argv[argc - 1]);
    return rc;
}
