// vtk_harness.cpp -- host build of the library's VTK writer (ho-cxx_b200/csrc/output_host.cpp)
// with its mesh reader, bases and sample-point search (host_samples.cpp), for a CPU test: the
// test passes fields the reference wrote its own VTK and sample-point files from and compares
// the files. Never part of the library.
#include "host.hpp"

extern "C" int write_vtk_host(const char* msh, int occ, int knod, int problem_type, const double* w, const double* psi,
                              const double* u, const double* v, const double* rd, const double* ra, const double* bw,
                              const double* bnv, const double* bpv, int indx, int subidx, const char* dir,
                              const char* samples) {
    ho2d::Mesh m;
    ho2d::Error e = ho2d::read_msh(msh, occ, m);
    if (e.code) return e.code;
    ho2d::Bases B;
    e = ho2d::make_bases(knod, m.lnod, B);
    if (e.code) return e.code;
    ho2d::SamplePoints sp;
    if (samples && *samples) {
        e = ho2d::read_sample_points(samples, m, sp);
        if (e.code) return e.code;
    }
    const ho2d::VtkFields f{w, psi, u, v, rd, ra, bw, bnv, bpv};
    return ho2d::write_vtk_files(m, B, problem_type, f, indx, subidx, dir, &sp).code;
}

// read_sample_points alone: the element and the Lnod^2 shape functions of each point
// (elem [n], shape [n][Lnod^2]); returns the number of points, or -code on error.
extern "C" long sample_points_host(const char* msh, int occ, const char* samples, int* elem, double* shape,
                                   long cap) {
    ho2d::Mesh m;
    ho2d::Error e = ho2d::read_msh(msh, occ, m);
    if (e.code) return -e.code;
    ho2d::SamplePoints sp;
    e = ho2d::read_sample_points(samples, m, sp);
    if (e.code) return -e.code;
    const size_t L2 = (size_t)m.lnod * m.lnod;
    for (size_t s = 0; s < sp.size() && (long)s < cap; ++s) {
        elem[s] = sp.elem[s];
        for (size_t l = 0; l < L2; ++l) shape[s * L2 + l] = sp.shape[s * L2 + l];
    }
    return (long)sp.size();
}

// The same fields written twice through VtkQueue (dump indices indx and indx + 1, the
// second submitted while the first may still be on the queue's thread), then waited for.
extern "C" int write_vtk_queued_host(const char* msh, int occ, int knod, int problem_type, const double* w,
                                     const double* psi, const double* u, const double* v, const double* rd,
                                     const double* ra, const double* bw, const double* bnv, const double* bpv,
                                     int indx, const char* dir, const char* samples) {
    ho2d::Mesh m;
    ho2d::Error e = ho2d::read_msh(msh, occ, m);
    if (e.code) return e.code;
    ho2d::Bases B;
    e = ho2d::make_bases(knod, m.lnod, B);
    if (e.code) return e.code;
    ho2d::SamplePoints sp;
    if (samples && *samples) {
        e = ho2d::read_sample_points(samples, m, sp);
        if (e.code) return e.code;
    }
    const size_t nv = (size_t)m.n_el * knod * knod, nb = (size_t)m.n_eb * knod;
    ho2d::VtkQueue q;
    for (int r = 0; r < 2; ++r) {
        ho2d::VtkQueue::Job j;
        j.w.assign(w, w + nv);
        j.psi.assign(psi, psi + nv);
        j.u.assign(u, u + nv);
        j.v.assign(v, v + nv);
        j.rhs_diff.assign(rd, rd + nv);
        j.rhs_adv.assign(ra, ra + nv);
        j.bc_w.assign(bw, bw + nb);
        j.bc_nv.assign(bnv, bnv + nb);
        j.bc_pv.assign(bpv, bpv + nb);
        j.problem_type = problem_type;
        j.indx = indx + r;
        j.dir = dir;
        e = q.submit(m, B, &sp, std::move(j));
        if (e.code) return e.code;
    }
    return q.wait().code;
}
