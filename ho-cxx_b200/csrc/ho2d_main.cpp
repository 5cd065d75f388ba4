// ho2d_main.cpp -- command-line drop-in for the reference's src/main.cpp: reads
// input.dat (or argv[1]), runs the setup sequence and the time loop on the GPU, and writes
// the VTK files of the dump steps (and the sample-point files, when the input names a
// sample-points file) into the working directory, as the reference does. Then prints the
// final vorticity norms and the timing.
// Options after the input file: --mixed (FP32 BiCGSTAB inside FP64 iterative refinement,
// FP64 stage: HO2D_MIXED_KRYLOV), --mixed-stage (the FR stage in FP32 too: HO2D_MIXED),
// --no-output (write no files).
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "HO_2D.hpp"

int main(int argc, char const* argv[]) {
    std::string input = "input.dat";
    int precision = HO2D_FP64;
    bool output = true;
    for (int i = 1; i < argc; ++i) {
        if (std::strcmp(argv[i], "--mixed") == 0) precision = HO2D_MIXED_KRYLOV;
        else if (std::strcmp(argv[i], "--mixed-stage") == 0) precision = HO2D_MIXED;
        else if (std::strcmp(argv[i], "--no-output") == 0) output = false;
        else if (argv[i][0] == '-') {
            std::printf("\nUsage:\n  %s [input.dat] [--mixed | --mixed-stage] [--no-output]\n\n", argv[0]);
            return -1;
        } else input = argv[i];
    }
    try {
        HO_2D ho;
        ho.read_input_file(input);
        ho.set_precision(precision);
        if (!output) ho.set_output_dir("");
        const auto t0 = std::chrono::steady_clock::now();
        ho.setup_mesh();
        ho.form_Laplace_operator_matrix();
        const auto t1 = std::chrono::steady_clock::now();
        ho.solve_vorticity_streamfunction();
        const auto t2 = std::chrono::steady_clock::now();
        const int32_t n = ho.getsolnlen();
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
