// ho2d_main.cpp -- command-line drop-in for the reference's src/main.cpp: reads
// input.dat (or argv[1]), runs the setup sequence and the time loop on the GPU.
// Options after the input file: --mixed (FP32 residual/Krylov in FP64 refinement).
// VTK output is not written; the final vorticity statistics and timing are printed.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "HO_2D.hpp"

int main(int argc, char const* argv[]) {
    std::string input = "input.dat";
    bool mixed = false;
    for (int i = 1; i < argc; ++i) {
        if (std::strcmp(argv[i], "--mixed") == 0) mixed = true;
        else if (argv[i][0] == '-') {
            std::printf("\nUsage:\n  %s [input.dat] [--mixed]\n\n", argv[0]);
            return -1;
        } else input = argv[i];
    }
    try {
        HO_2D ho;
        ho.read_input_file(input);
        if (mixed) ho.set_precision(HO2D_MIXED);
        const auto t0 = std::chrono::steady_clock::now();
        ho.setup_mesh();
        ho.form_Laplace_operator_matrix();
        const auto t1 = std::chrono::steady_clock::now();
        ho.solve_vorticity_streamfunction();
        const auto t2 = std::chrono::steady_clock::now();
        const int32_t n = ho.getsolnptlen();
        std::vector<double> w(n);
        ho.getallvorts_d(n, w.data());
        double l2 = 0.0, mx = 0.0;
        for (double v : w) {
            l2 += v * v;
            mx = std::fmax(mx, std::fabs(v));
        }
        std::printf("setup %.3f s, time loop %.3f s, DOF %d, |omega|_2 %.12e, max|omega| %.12e\n",
                    std::chrono::duration<double>(t1 - t0).count(), std::chrono::duration<double>(t2 - t1).count(),
                    n, std::sqrt(l2), mx);
    } catch (const HO2DException& e) {
        std::printf("error %d: %s\n", e.code(), e.what());
        return e.code();
    }
    return 0;
}
