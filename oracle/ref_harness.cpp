// ref_harness.cpp -- drives the reference's own HO_2D class (src/HO_2D.cpp, src/Mesh.cpp,
// compiled unmodified against the oracle API shim) and dumps its internal arrays.
//
// TEST INFRASTRUCTURE ONLY. It generates golden vectors for the parity tests and, in
// --time mode, times the reference's CPU time loop for the bench's reference arm.
// Nothing in the product links or calls it.
//
// Sequence mirrored from src/main.cpp:44-77 (read_input_file, setup_mesh,
// allocate_arrays, setup_sps_gps, form_bases, form_metrics, setup_IC_BC_SRC,
// form_Laplace_operator_matrix); the time loop mirrors
// src/HO_2D.cpp:1407-1447 without the VTK writers (dump_frequency output only).
// read_process_sample_points (src/HO_2D.cpp:319) runs only with --samples: it is
// output-only and seeds its ray casting from time(0).
//
// usage: ho2d_ref INPUT.dat OUTDIR [options]
//   --setup                dump mesh tables, bases, metrics, BCs, Poisson matrix
//   --init-vort FILE.npy   replace the initial vorticity [N_el][K][K]
//   --lid FILE.npy         replace BC_parl_vel [N_eb][K] after setup (before the h-flip
//                          convention is irrelevant: parl_vel is never flipped)
//   --dt X                 override dt
//   --stage COEFF          run one Euler_time_integrate(vorticity, k1, COEFF) and dump
//                          the stage arrays (psi, velocity, RHS terms, BC arrays)
//   --steps N              run N time steps, dumping vorticity/psi every --every steps
//   --every M              dump period for --steps (default N)
//   --time N               time N steps (no dumps) and print a JSON line
//   --time-stages N        time N RK stages (Euler_time_integrate on the current vorticity,
//                          coefficients cycling 0, .5, .5, 1) and print a JSON line
//   --t0 T                 start the time loop at time T instead of 0
//   --solve                run solve_vorticity_streamfunction (writes the reference's VTK
//                          files into the input's directory), dump the fields the last
//                          files were written from (solve_*.npy) and stop
//   --samples              run read_process_sample_points after setup_sps_gps, as
//                          src/main.cpp:65 does (the sample file named in the input,
//                          opened from the input's directory); --solve then also writes
//                          the reference's sampling_points*.dat files
//   --verbose              keep the reference's stdout
// or:   ho2d_ref --hybrid SPECDIR OUTDIR [--verbose]   (see run_hybrid)
#include "HO_2D.hpp"

#include <sys/stat.h>
#include <unistd.h>

#include <chrono>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>

namespace {

void write_npy(const std::string& path, const char* descr, const std::vector<size_t>& shape, const void* data,
               size_t itemsize) {
    std::string hdr = std::string("{'descr': '") + descr + "', 'fortran_order': False, 'shape': (";
    size_t count = 1;
    for (size_t i = 0; i < shape.size(); ++i) {
        hdr += std::to_string(shape[i]);
        hdr += (shape.size() == 1 || i + 1 < shape.size()) ? ", " : "";
        count *= shape[i];
    }
    hdr += "), }";
    const size_t pre = 10;
    size_t total = pre + hdr.size() + 1;
    const size_t pad = (64 - total % 64) % 64;
    hdr += std::string(pad, ' ');
    hdr += '\n';
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) { std::perror(path.c_str()); std::exit(3); }
    const unsigned char magic[8] = {0x93, 'N', 'U', 'M', 'P', 'Y', 1, 0};
    std::fwrite(magic, 1, 8, f);
    const uint16_t hl = (uint16_t)hdr.size();
    std::fwrite(&hl, 2, 1, f);
    std::fwrite(hdr.data(), 1, hdr.size(), f);
    std::fwrite(data, itemsize, count, f);
    std::fclose(f);
}

void dump_f64(const std::string& dir, const std::string& name, const std::vector<size_t>& shape, const double* p) {
    write_npy(dir + "/" + name + ".npy", "<f8", shape, p, 8);
}
void dump_i32(const std::string& dir, const std::string& name, const std::vector<size_t>& shape,
              const std::vector<int32_t>& v) {
    write_npy(dir + "/" + name + ".npy", "<i4", shape, v.data(), 4);
}

std::vector<double> read_npy_f64(const std::string& path, size_t expect) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) { std::perror(path.c_str()); std::exit(3); }
    unsigned char pre[10];
    if (std::fread(pre, 1, 10, f) != 10) std::exit(3);
    const uint16_t hl = (uint16_t)(pre[8] | (pre[9] << 8));
    std::string hdr(hl, ' ');
    if (std::fread(&hdr[0], 1, hl, f) != hl) std::exit(3);
    if (hdr.find("<f8") == std::string::npos || hdr.find("'fortran_order': False") == std::string::npos) {
        std::fprintf(stderr, "%s: expected a C-ordered float64 array\n", path.c_str());
        std::exit(3);
    }
    std::vector<double> v(expect);
    if (std::fread(v.data(), 8, expect, f) != expect) {
        std::fprintf(stderr, "%s: short read (expected %zu values)\n", path.c_str(), expect);
        std::exit(3);
    }
    std::fclose(f);
    return v;
}

struct NullBuf : std::streambuf {
    int overflow(int c) override { return c; }
};

// A whole .npy file of the given dtype ("<f8" or "<i4"); missing file: empty.
template <typename T>
std::vector<T> read_npy_any(const std::string& path, const char* descr) {
    std::vector<T> v;
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) return v;
    unsigned char pre[10];
    if (std::fread(pre, 1, 10, f) != 10) std::exit(3);
    const uint16_t hl = (uint16_t)(pre[8] | (pre[9] << 8));
    std::string hdr(hl, ' ');
    if (std::fread(&hdr[0], 1, hl, f) != hl) std::exit(3);
    if (hdr.find(descr) == std::string::npos) {
        std::fprintf(stderr, "%s: expected dtype %s\n", path.c_str(), descr);
        std::exit(3);
    }
    const size_t a = hdr.find("'shape': (") + 10, b = hdr.find(')', a);
    size_t count = 1;
    std::string sh = hdr.substr(a, b - a);
    size_t pos = 0;
    while (pos < sh.size()) {
        const size_t c = sh.find(',', pos);
        const std::string tok = sh.substr(pos, c == std::string::npos ? std::string::npos : c - pos);
        if (tok.find_first_of("0123456789") != std::string::npos) count *= std::stoul(tok);
        if (c == std::string::npos) break;
        pos = c + 1;
    }
    v.resize(count);
    if (count && std::fread(v.data(), sizeof(T), count, f) != count) std::exit(3);
    std::fclose(f);
    return v;
}

// --hybrid SPECDIR OUTDIR: the reference's hybrid sequence (src/HO_2D.hpp:251-290) on
// arrays from SPECDIR: spec.txt ("key value" lines: knod iorder nouter numstep outerdt
// integ reyn), nodes.npy, elems.npy, wall.npy, open.npy, inlet.npy / inletvel.npy,
// outlet.npy / outletvel.npy, ptog.npy, and per outer step s = -1 .. nouter-1 the driver
// data vort_<s>.npy, openvel_<s>.npy, openvort_<s>.npy (s = -1 fills the "start" values
// before the first step). Dumps vort_out_<s>.npy after each outer step, the setup it starts
// from (setup_*.npy) and the split of each new open-boundary velocity (open_vel*_end_<s>.npy).
int run_hybrid(const std::string& spec, const std::string& outdir_in, bool verbose) {
    std::map<std::string, double> kv;
    {
        std::ifstream f(spec + "/spec.txt");
        std::string k;
        double v;
        while (f >> k >> v) kv[k] = v;
    }
    mkdir(outdir_in.c_str(), 0755);
    char absout[4096];
    if (!realpath(outdir_in.c_str(), absout)) { std::perror("realpath"); return 3; }
    const std::string outdir = absout;
    auto f8 = [&](const std::string& n) { return read_npy_any<double>(spec + "/" + n + ".npy", "<f8"); };
    auto i4 = [&](const std::string& n) { return read_npy_any<int32_t>(spec + "/" + n + ".npy", "<i4"); };
    std::vector<double> xy = f8("nodes"), inv = f8("inletvel"), outv = f8("outletvel"), ptog = f8("ptog");
    std::vector<int32_t> el = i4("elems"), wall = i4("wall"), open = i4("open"), inl = i4("inlet"), outl = i4("outlet");
    NullBuf nullbuf;
    std::streambuf* saved = std::cout.rdbuf();
    if (!verbose) std::cout.rdbuf(&nullbuf);
    HO_2D s;
    s.set_defaults();
    s.enable_hybrid();
    s.set_elemorder((int32_t)kv["knod"]);
    s.load_mesh_arrays_d((int32_t)kv["iorder"], (int32_t)xy.size(), xy.data(), (int32_t)el.size(), el.data(),
                         (int32_t)wall.size(), wall.data(), (int32_t)open.size(), open.data());
    s.load_inout_arrays_d((int32_t)inv.size(), inv.data(), (int32_t)inl.size(), inl.data(), (int32_t)outv.size(),
                          outv.data(), (int32_t)outl.size(), outl.data());
    s.process_mesh_input();
    const int32_t nv = s.mesh.N_el * s.Knod * s.Knod;
    const int32_t nopen = s.getopenptlen();
    // the setup the hybrid sequence starts from (setup_*.npy): mesh tables, Jacobians and
    // the boundary conditions of problem type 11
    const size_t N = s.mesh.N_el, K = s.Knod, Neb = s.mesh.N_edges_boundary;
    {
        std::vector<int32_t> nbr(N * 4), nside(N * 4), be_el(Neb), be_side(Neb), be_group(Neb, -1), swp(Neb), swd(Neb),
            nsl(s.mesh.N_Gboundary);
        for (size_t e = 0; e < N; ++e)
            for (int q = 0; q < 4; ++q) {
                const auto& en = s.mesh.elem_neighbor[e];
                nbr[e * 4 + q] = en.is_on_boundary[q] ? -1 : (int32_t)en.neighbor[q];
                nside[e * 4 + q] = en.is_on_boundary[q] ? -1 : en.neighbor_common_side[q];
            }
        for (size_t b = 0; b < Neb; ++b) {
            be_el[b] = s.mesh.boundary_edges[b].element_index;
            be_side[b] = s.mesh.boundary_edges[b].side;
            swp[b] = s.BC_switch_Poisson[b];
            swd[b] = s.BC_switch_diffusion[b];
        }
        for (int g = 0; g < s.mesh.N_Gboundary; ++g) {
            for (unsigned e : s.mesh.boundaries[g].edges) be_group[e] = g;
            nsl[g] = s.BC_no_slip[g] ? 1 : 0;
        }
        dump_i32(outdir, "setup_elem_neighbor", {N, 4}, nbr);
        dump_i32(outdir, "setup_elem_neighbor_side", {N, 4}, nside);
        dump_i32(outdir, "setup_bedge_element", {Neb}, be_el);
        dump_i32(outdir, "setup_bedge_side", {Neb}, be_side);
        dump_i32(outdir, "setup_bedge_group", {Neb}, be_group);
        dump_i32(outdir, "setup_BC_switch_Poisson", {Neb}, swp);
        dump_i32(outdir, "setup_BC_switch_diffusion", {Neb}, swd);
        dump_i32(outdir, "setup_BC_no_slip", {(size_t)s.mesh.N_Gboundary}, nsl);
        dump_f64(outdir, "setup_vol_jac", {N, K, K}, &s.vol_jac[0][0][0]);
        dump_f64(outdir, "setup_face_Anorm", {N, 4, K}, &s.face_Anorm[0][0][0]);
        dump_f64(outdir, "setup_BC_Poisson", {Neb, K}, &s.BC_Poisson[0][0]);
        dump_f64(outdir, "setup_BC_normal_vel", {Neb, K}, &s.BC_normal_vel[0][0]);
        dump_f64(outdir, "setup_BC_parl_vel", {Neb, K}, &s.BC_parl_vel[0][0]);
        dump_f64(outdir, "setup_BC_diffusion", {Neb, K}, &s.BC_diffusion[0][0]);
        dump_f64(outdir, "setup_boundary_source", {Neb, K * K, K}, &s.boundary_source[0][0][0]);
    }
    if (!ptog.empty()) s.setptogweights_d(nv, ptog.data());
    const int nouter = (int)kv["nouter"];
    for (int st = -1; st < nouter; ++st) {
        const std::string t = std::to_string(st);
        std::vector<double> v = f8("vort_" + t), ov = f8("openvel_" + t), ow = f8("openvort_" + t);
        if (!v.empty()) s.setsolnvort_d(nv, v.data());
        if (!ov.empty()) {
            s.setopenvels_d(nopen, ov.data());
            // the normal / parallel split of the new open-boundary velocities (rows: open
            // edges in open-boundary order)
            dump_f64(outdir, "open_velnorm_end_" + t, {(size_t)nopen / (2 * K), K}, &s.BC_VelNorm_end[0][0]);
            dump_f64(outdir, "open_velparl_end_" + t, {(size_t)nopen / (2 * K), K}, &s.BC_VelParl_end[0][0]);
        }
        if (!ow.empty()) s.setopenvort_d(nopen / 2, ow.data());
        if (st < 0) continue;
        s.solveto_d(kv["outerdt"], (int32_t)kv["numstep"], (int32_t)kv["integ"], kv["reyn"]);
        std::vector<double> out(nv);
        s.getallvorts_d(nv, out.data());
        dump_f64(outdir, "vort_out_" + t, {(size_t)nv}, out.data());
    }
    std::vector<double> areas(nv), opts(std::max(1, nopen));
    s.getsolnareas_d(nv, areas.data());
    dump_f64(outdir, "areas", {(size_t)nv}, areas.data());
    if (nopen > 0) {
        s.getopenpts_d(nopen, opts.data());
        dump_f64(outdir, "openpts", {(size_t)nopen}, opts.data());
    }
    std::cout.rdbuf(saved);
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc >= 4 && std::string(argv[1]) == "--hybrid")
        return run_hybrid(argv[2], argv[3], argc > 4 && std::string(argv[4]) == "--verbose");
    if (argc < 3) {
        std::fprintf(stderr, "usage: %s INPUT.dat OUTDIR [options]\n", argv[0]);
        return 2;
    }
    std::string input = argv[1], outdir = argv[2];
    bool do_setup = false, verbose = false, do_stage = false, do_solve = false, do_samples = false;
    double stage_coeff = 0.0, dt_override = -1.0, t0 = 0.0;
    long nsteps = 0, every = 0, ntime = 0, nstages = 0;
    std::string init_vort, lid;
    for (int i = 3; i < argc; ++i) {
        std::string a = argv[i];
        if (a == "--setup") do_setup = true;
        else if (a == "--verbose") verbose = true;
        else if (a == "--init-vort" && i + 1 < argc) init_vort = argv[++i];
        else if (a == "--lid" && i + 1 < argc) lid = argv[++i];
        else if (a == "--dt" && i + 1 < argc) dt_override = std::atof(argv[++i]);
        else if (a == "--stage" && i + 1 < argc) { do_stage = true; stage_coeff = std::atof(argv[++i]); }
        else if (a == "--steps" && i + 1 < argc) nsteps = std::atol(argv[++i]);
        else if (a == "--every" && i + 1 < argc) every = std::atol(argv[++i]);
        else if (a == "--time" && i + 1 < argc) ntime = std::atol(argv[++i]);
        else if (a == "--time-stages" && i + 1 < argc) nstages = std::atol(argv[++i]);
        else if (a == "--t0" && i + 1 < argc) t0 = std::atof(argv[++i]);
        else if (a == "--solve") do_solve = true;
        else if (a == "--samples") do_samples = true;
        else { std::fprintf(stderr, "unknown option %s\n", a.c_str()); return 2; }
    }
    mkdir(outdir.c_str(), 0755);
    char absout[4096];
    if (!realpath(outdir.c_str(), absout)) { std::perror("realpath"); return 3; }
    outdir = absout;
    // the reference opens the mesh file relative to the working directory
    std::string dir = ".", base = input;
    const size_t slash = input.find_last_of('/');
    if (slash != std::string::npos) { dir = input.substr(0, slash); base = input.substr(slash + 1); }
    if (chdir(dir.c_str()) != 0) { std::perror("chdir"); return 3; }

    NullBuf nullbuf;
    std::streambuf* saved = std::cout.rdbuf();
    if (!verbose) std::cout.rdbuf(&nullbuf);

    const auto t_setup0 = std::chrono::steady_clock::now();
    HO_2D ho;
    if (ho.read_input_file(base) != 0) { std::cout.rdbuf(saved); std::fprintf(stderr, "read_input_file failed\n"); return 4; }
    if (dt_override > 0) ho.dt = dt_override;
    if (ho.setup_mesh() != 0) { std::cout.rdbuf(saved); std::fprintf(stderr, "setup_mesh failed\n"); return 4; }
    if (ho.allocate_arrays() != 0) { std::cout.rdbuf(saved); std::fprintf(stderr, "allocate_arrays failed\n"); return 4; }
    ho.setup_sps_gps();
    if (do_samples) ho.read_process_sample_points();
    ho.form_bases();
    ho.form_metrics();
    ho.setup_IC_BC_SRC();
    ho.form_Laplace_operator_matrix();
    const double setup_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_setup0).count();

    const size_t N = ho.mesh.N_el, K = ho.Knod, Neb = ho.mesh.N_edges_boundary, L = ho.mesh.Lnod;
    if (!init_vort.empty()) {
        std::vector<double> w = read_npy_f64(init_vort, N * K * K);
        std::copy(w.begin(), w.end(), &ho.initial_vorticity[0][0][0]);
    }
    if (!lid.empty()) {
        std::vector<double> w = read_npy_f64(lid, Neb * K);
        std::copy(w.begin(), w.end(), &ho.BC_parl_vel[0][0]);
    }
    for (size_t i = 0; i < N * K * K; ++i) ho.vorticity[0][0][i] = ho.initial_vorticity[0][0][i];
    ho.current_time = ho.time_start + t0;

    if (do_setup) {
        std::vector<int32_t> nbr(N * 4), nside(N * 4), onb(N * 4), bidx(N * 4);
        for (size_t e = 0; e < N; ++e)
            for (int s = 0; s < 4; ++s) {
                const auto& en = ho.mesh.elem_neighbor[e];
                onb[e * 4 + s] = en.is_on_boundary[s] ? 1 : 0;
                nbr[e * 4 + s] = en.is_on_boundary[s] ? -1 : (int32_t)en.neighbor[s];
                nside[e * 4 + s] = en.is_on_boundary[s] ? -1 : en.neighbor_common_side[s];
                bidx[e * 4 + s] = en.is_on_boundary[s] ? (int32_t)en.boundary_index[s] : -1;
            }
        dump_i32(outdir, "elem_neighbor", {N, 4}, nbr);
        dump_i32(outdir, "elem_neighbor_side", {N, 4}, nside);
        dump_i32(outdir, "elem_on_boundary", {N, 4}, onb);
        dump_i32(outdir, "elem_boundary_index", {N, 4}, bidx);
        std::vector<int32_t> be_el(Neb), be_side(Neb), be_group(Neb, -1);
        for (size_t b = 0; b < Neb; ++b) {
            be_el[b] = ho.mesh.boundary_edges[b].element_index;
            be_side[b] = ho.mesh.boundary_edges[b].side;
        }
        for (int g = 0; g < ho.mesh.N_Gboundary; ++g)
            for (unsigned e : ho.mesh.boundaries[g].edges) be_group[e] = g;
        dump_i32(outdir, "bedge_element", {Neb}, be_el);
        dump_i32(outdir, "bedge_side", {Neb}, be_side);
        dump_i32(outdir, "bedge_group", {Neb}, be_group);
        std::vector<double> xy(N * L * L * 2);
        for (size_t e = 0; e < N; ++e)
            for (size_t j = 0; j < L; ++j)
                for (size_t i = 0; i < L; ++i) {
                    const auto& c = ho.mesh.nodes[ho.mesh.elements[e].nodes[ho.mesh.tensor2FEM((int)i, (int)j)]].coor;
                    xy[((e * L + j) * L + i) * 2 + 0] = c.x;
                    xy[((e * L + j) * L + i) * 2 + 1] = c.y;
                }
        dump_f64(outdir, "elem_nodes_xy", {N, L, L, 2}, xy.data());
        dump_f64(outdir, "sps_local_coor", {K}, ho.sps_local_coor);
        dump_f64(outdir, "sps_weight", {K}, ho.sps_weight);
        dump_f64(outdir, "sps_boundary_basis", {K, 2}, &ho.sps_boundary_basis[0][0]);
        dump_f64(outdir, "sps_boundary_grad_basis", {K, 2}, &ho.sps_boundary_grad_basis[0][0]);
        dump_f64(outdir, "sps_sps_grad_basis", {K, K}, &ho.sps_sps_grad_basis[0][0]);
        dump_f64(outdir, "sps_radau", {K, 2}, &ho.sps_radau[0][0]);
        dump_f64(outdir, "sps_grad_radau", {K, 2}, &ho.sps_grad_radau[0][0]);
        dump_f64(outdir, "gps_sps_basis", {L, K}, &ho.gps_sps_basis[0][0]);
        dump_f64(outdir, "gps_sps_grad_basis", {L, K}, &ho.gps_sps_grad_basis[0][0]);
        dump_f64(outdir, "vol_Dx_Dxsi", {N, K, K, 2}, &ho.vol_Dx_Dxsi[0][0][0].x);
        dump_f64(outdir, "vol_Dy_Dxsi", {N, K, K, 2}, &ho.vol_Dy_Dxsi[0][0][0].x);
        dump_f64(outdir, "vol_jac", {N, K, K}, &ho.vol_jac[0][0][0]);
        dump_f64(outdir, "vol_Dxsi_Dx", {N, K, K, 2, 2}, &ho.vol_Dxsi_Dx[0][0][0][0][0]);
        dump_f64(outdir, "G", {N, K, K, 2, 2}, &ho.G[0][0][0][0][0]);
        dump_f64(outdir, "GB", {N, 2, 2, K, 2}, &ho.GB[0][0][0][0][0]);
        dump_f64(outdir, "face_Acoef", {N, 4, K}, &ho.face_Acoef[0][0][0]);
        dump_f64(outdir, "face_Bcoef", {N, 4, K}, &ho.face_Bcoef[0][0][0]);
        dump_f64(outdir, "face_jac", {N, 4, K}, &ho.face_jac[0][0][0]);
        dump_f64(outdir, "face_Anorm", {N, 4, K}, &ho.face_Anorm[0][0][0]);
        std::vector<int32_t> swp(Neb), swd(Neb), nsl(ho.mesh.N_Gboundary);
        for (size_t b = 0; b < Neb; ++b) { swp[b] = ho.BC_switch_Poisson[b]; swd[b] = ho.BC_switch_diffusion[b]; }
        for (int g = 0; g < ho.mesh.N_Gboundary; ++g) nsl[g] = ho.BC_no_slip[g] ? 1 : 0;
        dump_i32(outdir, "BC_switch_Poisson", {Neb}, swp);
        dump_i32(outdir, "BC_switch_diffusion", {Neb}, swd);
        dump_i32(outdir, "BC_no_slip", {(size_t)ho.mesh.N_Gboundary}, nsl);
        dump_f64(outdir, "BC_Poisson", {Neb, K}, &ho.BC_Poisson[0][0]);
        dump_f64(outdir, "BC_normal_vel", {Neb, K}, &ho.BC_normal_vel[0][0]);
        dump_f64(outdir, "BC_parl_vel", {Neb, K}, &ho.BC_parl_vel[0][0]);
        dump_f64(outdir, "BC_diffusion", {Neb, K}, &ho.BC_diffusion[0][0]);
        dump_f64(outdir, "boundary_source", {Neb, K * K, K}, &ho.boundary_source[0][0][0]);
        if (ho.LHS_type == 3) {
            const shimla::Csr& A = ho.AMGCL_solver->matrix();
            std::vector<int32_t> ptr(A.ptr.begin(), A.ptr.end()), col(A.col.begin(), A.col.end());
            dump_i32(outdir, "A_ptr", {ptr.size()}, ptr);
            dump_i32(outdir, "A_col", {col.size()}, col);
            dump_f64(outdir, "A_val", {A.val.size()}, A.val.data());
        }
        FILE* f = std::fopen((outdir + "/meta.json").c_str(), "w");
        std::fprintf(f, "{\"N_el\": %zu, \"Knod\": %zu, \"Lnod\": %zu, \"N_edges_boundary\": %zu, ", N, K, L, Neb);
        std::fprintf(f, "\"Reyn_inv\": %.17g, \"dt\": %.17g, \"problem_type\": %d, \"advection_type\": %d, ",
                     ho.Reyn_inv, ho.dt, ho.problem_type, ho.advection_type);
        std::fprintf(f, "\"time_integration_type\": %d, \"boundaries\": [", ho.time_integration_type);
        for (int g = 0; g < ho.mesh.N_Gboundary; ++g)
            std::fprintf(f, "%s\"%s\"", g ? ", " : "", ho.mesh.boundaries[g].name.c_str());
        std::fprintf(f, "], \"setup_seconds\": %.6f}\n", setup_s);
        std::fclose(f);
    }

    if (do_solve) {
        // the reference's whole time loop with its own VTK output (written into the input's
        // directory, the working directory here)
        ho.solve_vorticity_streamfunction();
        // the fields the last VTK files were written from
        dump_f64(outdir, "solve_vorticity", {N, K, K}, &ho.vorticity[0][0][0]);
        dump_f64(outdir, "solve_psi", {N, K, K}, &ho.stream_function[0][0][0]);
        std::vector<double> vel(N * K * K * 2);
        for (size_t i = 0; i < N * K * K; ++i) {
            vel[2 * i] = (&ho.velocity_cart[0][0][0])[i].x;
            vel[2 * i + 1] = (&ho.velocity_cart[0][0][0])[i].y;
        }
        dump_f64(outdir, "solve_vel", {N, K, K, 2}, vel.data());
        dump_f64(outdir, "solve_rhs_diff", {N, K, K}, &ho.RHS_diffusive[0][0][0]);
        dump_f64(outdir, "solve_rhs_adv", {N, K, K}, &ho.RHS_advective[0][0][0]);
        dump_f64(outdir, "solve_bc_w", {Neb, K}, &ho.BC_vorticity[0][0]);
        dump_f64(outdir, "solve_bc_nv", {Neb, K}, &ho.BC_normal_vel[0][0]);
        dump_f64(outdir, "solve_bc_pv", {Neb, K}, &ho.BC_parl_vel[0][0]);
        std::cout.rdbuf(saved);
        return 0;
    }
    if (do_stage) {
        ho.Euler_time_integrate(ho.vorticity, ho.k1, stage_coeff);
        dump_f64(outdir, "stage_psi", {N, K, K}, &ho.stream_function[0][0][0]);
        dump_f64(outdir, "stage_vel", {N, K, K, 2}, &ho.velocity_cart[0][0][0].x);
        dump_f64(outdir, "stage_rhs_diff", {N, K, K}, &ho.RHS_diffusive[0][0][0]);
        dump_f64(outdir, "stage_rhs_adv", {N, K, K}, &ho.RHS_advective[0][0][0]);
        dump_f64(outdir, "stage_k", {N, K, K}, &ho.k1[0][0][0]);
        dump_f64(outdir, "stage_BC_vorticity", {Neb, K}, &ho.BC_vorticity[0][0]);
        dump_f64(outdir, "stage_velocity_jump", {Neb, K}, &ho.velocity_jump[0][0]);
        dump_f64(outdir, "stage_BC_diffusion", {Neb, K}, &ho.BC_diffusion[0][0]);
        dump_f64(outdir, "stage_BC_advection", {Neb, K}, &ho.BC_advection[0][0]);
        dump_f64(outdir, "stage_BC_normal_vel", {Neb, K}, &ho.BC_normal_vel[0][0]);
        dump_f64(outdir, "stage_BC_Poisson", {Neb, K}, &ho.BC_Poisson[0][0]);
        dump_f64(outdir, "stage_BC_parl_vel", {Neb, K}, &ho.BC_parl_vel[0][0]);
    }

    if (nsteps > 0) {
        if (every <= 0) every = nsteps;
        for (long ti = 0; ti < nsteps; ++ti) {
            ho.ti = (int)ti;
            ho.solve_advection_diffusion();
            ho.current_time += ho.dt;
            if ((ti + 1) % every == 0) {
                const std::string tag = std::to_string(ti + 1);
                dump_f64(outdir, "traj_vort_" + tag, {N, K, K}, &ho.vorticity[0][0][0]);
                dump_f64(outdir, "traj_psi_" + tag, {N, K, K}, &ho.stream_function[0][0][0]);
            }
        }
    }

    if (ntime > 0) {
        amgcl::shim_solve_seconds() = 0.0;
        amgcl::shim_solve_iterations() = 0;
        const auto t0 = std::chrono::steady_clock::now();
        for (long ti = 0; ti < ntime; ++ti) {
            ho.ti = (int)ti;
            ho.solve_advection_diffusion();
            ho.current_time += ho.dt;
        }
        const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        std::cout.rdbuf(saved);
        std::printf("{\"steps\": %ld, \"seconds\": %.6f, \"poisson_seconds\": %.6f, \"poisson_iterations\": %ld, "
                    "\"setup_seconds\": %.6f, \"N_el\": %zu, \"Knod\": %zu, \"dof\": %zu}\n",
                    ntime, sec, amgcl::shim_solve_seconds(), amgcl::shim_solve_iterations(), setup_s, N, K, N * K * K);
    }
    if (nstages > 0) {
        static const double c4[4] = {0.0, 0.5, 0.5, 1.0};
        amgcl::shim_solve_seconds() = 0.0;
        amgcl::shim_solve_iterations() = 0;
        const auto t0 = std::chrono::steady_clock::now();
        for (long s = 0; s < nstages; ++s) ho.Euler_time_integrate(ho.vorticity, ho.k1, c4[s % 4]);
        const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        std::cout.rdbuf(saved);
        std::printf("{\"stages\": %ld, \"seconds\": %.6f, \"poisson_seconds\": %.6f, \"poisson_iterations\": %ld, "
                    "\"setup_seconds\": %.6f, \"N_el\": %zu, \"Knod\": %zu, \"dof\": %zu}\n",
                    nstages, sec, amgcl::shim_solve_seconds(), amgcl::shim_solve_iterations(), setup_s, N, K, N * K * K);
    }
    std::cout.rdbuf(saved);
    return 0;
}
