// vtk_harness.cpp -- host build of the library's VTK writer (ho-cxx_b200/csrc/output_host.cpp)
// with its mesh reader and bases, for a CPU test: the test passes fields the reference
// wrote its own VTK files from and compares the files. Never part of the library.
#include "host.hpp"

extern "C" int write_vtk_host(const char* msh, int occ, int knod, int problem_type, const double* w, const double* psi,
                              const double* u, const double* v, const double* rd, const double* ra, const double* bw,
                              const double* bnv, const double* bpv, int indx, int subidx, const char* dir) {
    ho2d::Mesh m;
    ho2d::Error e = ho2d::read_msh(msh, occ, m);
    if (e.code) return e.code;
    ho2d::Bases B;
    e = ho2d::make_bases(knod, m.lnod, B);
    if (e.code) return e.code;
    const ho2d::VtkFields f{w, psi, u, v, rd, ra, bw, bnv, bpv};
    return ho2d::write_vtk_files(m, B, problem_type, f, indx, subidx, dir).code;
}
