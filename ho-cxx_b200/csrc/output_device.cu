// output_device.cu -- the node values of save_smooth_vtk (src/HO_2D.cpp:3392-3614) made on
// the device with the writer's own routines (vtk_nodes.hpp): element fields to geometry
// nodes, the boundary edges' BC values, the per-node averages and the sample points. Only
// the node averages and sample values come back to the host for the smooth file (instead
// of the streamfunction and the boundary arrays). Compiled with -fmad=false: the values
// equal the host writer's bit for bit, so the files do too.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "solver.hpp"
#include "solver_state.hpp"
#include "vtk_nodes.hpp"

namespace ho2d {

namespace {

__global__ void k_vtk_elem(VtkGeo g, const double* __restrict__ w, const double* __restrict__ psi,
                           const double* __restrict__ u, const double* __restrict__ v, double* om, double* ps,
                           double* vx, double* vy) {
    const int el = blockIdx.x * blockDim.x + threadIdx.x;
    if (el < g.N) vtk_element_nodes(g, el, w, psi, u, v, om, ps, vx, vy);
}

__global__ void k_vtk_edge_vel(VtkGeo g, const double* __restrict__ bnv, const double* __restrict__ bpv, double* cvx,
                               double* cvy) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < g.neb) vtk_edge_velocity(g, e, bnv, bpv, cvx, cvy);
}

// one thread per element with boundary edges, its edges in ascending order (the later edge
// wins at a corner node, as in the host loop over edges)
__global__ void k_vtk_edge_nodes(VtkGeo g, int nbel, const int* __restrict__ ptr, const int* __restrict__ edges,
                                 const double* __restrict__ bw, const double* __restrict__ cvx,
                                 const double* __restrict__ cvy, double* om, double* vx, double* vy) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nbel) return;
    for (int k = ptr[i]; k < ptr[i + 1]; ++k) vtk_edge_nodes(g, edges[k], bw, cvx, cvy, om, vx, vy);
}

// one thread per mesh node: the sums over its slots in ascending (element, slot) order,
// then the averages; out = [nw | np | nux | nuy]
__global__ void k_vtk_average(int nn, const int* __restrict__ ptr, const int* __restrict__ slot,
                              const double* __restrict__ om, const double* __restrict__ ps,
                              const double* __restrict__ vx, const double* __restrict__ vy, double* __restrict__ out) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= nn) return;
    double a = 0.0, b = 0.0, c = 0.0, d = 0.0;
    for (int k = ptr[n]; k < ptr[n + 1]; ++k) {
        const int q = slot[k];
        c += vx[q];
        d += vy[q];
        a += om[q];
        b += ps[q];
    }
    vtk_node_average(ptr[n + 1] - ptr[n], a, b, c, d);
    out[n] = a;
    out[(size_t)nn + n] = b;
    out[2 * (size_t)nn + n] = c;
    out[3 * (size_t)nn + n] = d;
}

__global__ void k_vtk_samples(int ns, int L2, const int* __restrict__ sel, const double* __restrict__ shape,
                              const int* __restrict__ nodes, int nn, const double* __restrict__ avg,
                              double* __restrict__ out) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= ns) return;
    vtk_sample(L2, nodes + (size_t)sel[s] * L2, shape + (size_t)s * L2, avg, avg + 2 * (size_t)nn,
               avg + 3 * (size_t)nn, out + 3 * (size_t)s);
}

__global__ void k_f2d(const float* __restrict__ a, double* __restrict__ b, size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = (double)a[i];
}

unsigned blocks_for(size_t n) { return (unsigned)std::max<size_t>(1, (n + 127) / 128); }

}  // namespace

// Static tables of the device node interpolation, once per setup.
Error Solver::vtk_device_tables() {
    DeviceState& d = *d_;
    VtkDevice& t = d.vtk;
    if (t.ready) return {0, ""};
    const int N = mesh_.n_el, K = in_.knod, L = mesh_.lnod, L2 = L * L, neb = mesh_.n_eb;
    const VtkGeoHost gh(mesh_, B_);
    const int nn = (int)(mesh_.node_xy.size() / 2);
    HO2D_CUDA(upload(t.sgb, gh.sgb), "upload");
    HO2D_CUDA(upload(t.t2f, gh.t2f), "upload");
    HO2D_CUDA(upload(t.nodes, gh.nodes), "upload");
    HO2D_CUDA(upload(t.node_xy, mesh_.node_xy), "upload");
    HO2D_CUDA(upload(t.be_el, mesh_.be_el.empty() ? std::vector<int>{0} : mesh_.be_el), "upload");
    HO2D_CUDA(upload(t.be_side, mesh_.be_side.empty() ? std::vector<int>{0} : mesh_.be_side), "upload");
    std::vector<double> bas;
    for (const std::vector<double>* v : {&B_.gbgb, &B_.gbb, &B_.gsb, &B_.gsgb}) bas.insert(bas.end(), v->begin(), v->end());
    HO2D_CUDA(upload(t.bases, bas), "upload");
    // boundary edges by element (elements in ascending order, edges ascending)
    std::vector<std::vector<int>> by_el(N);
    for (int e = 0; e < neb; ++e) by_el[mesh_.be_el[e]].push_back(e);
    std::vector<int> bptr{0}, bedges;
    for (int el = 0; el < N; ++el) {
        if (by_el[el].empty()) continue;
        bedges.insert(bedges.end(), by_el[el].begin(), by_el[el].end());
        bptr.push_back((int)bedges.size());
    }
    t.nbel = (int)bptr.size() - 1;
    HO2D_CUDA(upload(t.bptr, bptr), "upload");
    HO2D_CUDA(upload(t.bedges, bedges.empty() ? std::vector<int>{0} : bedges), "upload");
    // element node slots by mesh node, ascending (element, slot)
    std::vector<int> nptr(nn + 1, 0), nslot((size_t)N * L2);
    for (int v : gh.nodes) ++nptr[v + 1];
    for (int n = 0; n < nn; ++n) nptr[n + 1] += nptr[n];
    std::vector<int> fill(nptr.begin(), nptr.end() - 1);
    for (size_t q = 0; q < gh.nodes.size(); ++q) nslot[fill[gh.nodes[q]]++] = (int)q;
    HO2D_CUDA(upload(t.nptr, nptr), "upload");
    HO2D_CUDA(upload(t.nslot, nslot), "upload");
    const size_t ns = samples_.size();
    if (ns > 0) {
        HO2D_CUDA(upload(t.sel, samples_.elem), "upload");
        HO2D_CUDA(upload(t.shape, samples_.shape), "upload");
        HO2D_CUDA(t.samp.alloc(3 * ns * sizeof(double)), "alloc");
    }
    for (DeviceBuffer* b : {&t.om, &t.ps, &t.vx, &t.vy}) HO2D_CUDA(b->alloc((size_t)N * L2 * sizeof(double)), "alloc");
    for (DeviceBuffer* b : {&t.cvx, &t.cvy})
        HO2D_CUDA(b->alloc((size_t)std::max(1, neb) * K * sizeof(double)), "alloc");
    HO2D_CUDA(t.avg.alloc((size_t)4 * std::max(1, nn) * sizeof(double)), "alloc");
    t.nn = nn;
    t.ready = true;
    return {0, ""};
}

// The smooth file's node averages and sample values of the current fields into j.
Error Solver::vtk_nodes_device(VtkQueue::Job& j) {
    HO2D_TRY(vtk_device_tables());
    DeviceState& d = *d_;
    VtkDevice& t = d.vtk;
    const int N = mesh_.n_el, K = in_.knod, L = mesh_.lnod, neb = mesh_.n_eb;
    const size_t nv = (size_t)N * K * K;
    const double* gb = t.bases.as<double>();
    const VtkGeo g{N,
                   K,
                   L,
                   neb,
                   t.sgb.as<double>(),
                   t.t2f.as<int>(),
                   t.nodes.as<int>(),
                   t.node_xy.as<double>(),
                   t.be_el.as<int>(),
                   t.be_side.as<int>(),
                   gb,
                   gb + 2 * L,
                   gb + 4 * L,
                   gb + 4 * L + (size_t)L * K};
    const double *u = d.u.as<double>(), *v = d.v.as<double>();
    if (stage32_) {  // the FP32 stage's velocity, widened exactly as the host copy would be
        HO2D_CUDA(t.u64.alloc(nv * sizeof(double)), "alloc");
        HO2D_CUDA(t.v64.alloc(nv * sizeof(double)), "alloc");
        k_f2d<<<blocks_for(nv), 128, 0, d.stream>>>(d.u.as<float>(), t.u64.as<double>(), nv);
        k_f2d<<<blocks_for(nv), 128, 0, d.stream>>>(d.v.as<float>(), t.v64.as<double>(), nv);
        u = t.u64.as<double>();
        v = t.v64.as<double>();
    }
    k_vtk_elem<<<blocks_for(N), 128, 0, d.stream>>>(g, d.omega.as<double>(), d.psi64.as<double>(), u, v,
                                                     t.om.as<double>(), t.ps.as<double>(), t.vx.as<double>(),
                                                     t.vy.as<double>());
    if (neb > 0) {
        k_vtk_edge_vel<<<blocks_for(neb), 128, 0, d.stream>>>(g, d.bc_nv.as<double>(), d.bc_pv.as<double>(),
                                                               t.cvx.as<double>(), t.cvy.as<double>());
        k_vtk_edge_nodes<<<blocks_for(t.nbel), 128, 0, d.stream>>>(g, t.nbel, t.bptr.as<int>(), t.bedges.as<int>(),
                                                                    d.bc_w.as<double>(), t.cvx.as<double>(),
                                                                    t.cvy.as<double>(), t.om.as<double>(),
                                                                    t.vx.as<double>(), t.vy.as<double>());
    }
    k_vtk_average<<<blocks_for(t.nn), 128, 0, d.stream>>>(t.nn, t.nptr.as<int>(), t.nslot.as<int>(), t.om.as<double>(),
                                                          t.ps.as<double>(), t.vx.as<double>(), t.vy.as<double>(),
                                                          t.avg.as<double>());
    const size_t ns = samples_.size();
    if (ns > 0)
        k_vtk_samples<<<blocks_for(ns), 128, 0, d.stream>>>((int)ns, L * L, t.sel.as<int>(), t.shape.as<double>(),
                                                            t.nodes.as<int>(), t.nn, t.avg.as<double>(),
                                                            t.samp.as<double>());
    HO2D_CUDA(cudaGetLastError(), "node values");
    std::vector<double> avg((size_t)4 * t.nn);
    HO2D_CUDA(cudaMemcpyAsync(avg.data(), t.avg.get(), avg.size() * sizeof(double), cudaMemcpyDeviceToHost, d.stream),
              "copy");
    j.samp.assign(3 * ns, 0.0);
    if (ns > 0)
        HO2D_CUDA(cudaMemcpyAsync(j.samp.data(), t.samp.get(), 3 * ns * sizeof(double), cudaMemcpyDeviceToHost,
                                  d.stream),
                  "copy");
    HO2D_CUDA(cudaStreamSynchronize(d.stream), "node values");
    const size_t nn = (size_t)t.nn;
    j.nw.assign(avg.begin(), avg.begin() + nn);
    j.np.assign(avg.begin() + nn, avg.begin() + 2 * nn);
    j.nux.assign(avg.begin() + 2 * nn, avg.begin() + 3 * nn);
    j.nuy.assign(avg.begin() + 3 * nn, avg.begin() + 4 * nn);
    return {0, ""};
}

}  // namespace ho2d
