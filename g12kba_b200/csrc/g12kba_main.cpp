// g12kba: drop-in replacement for the reference executable
// (G12KBA-GW/src/main/Main.cpp:44-62).  Reads ./input, prepares G0, runs
// adiabatic switching and RK4 on the GPU, and writes real_G1.txt,
// imag_G1.txt, dipole.txt and progress.txt in the working directory with the
// reference's formats and stdout lines.
//
// Extension input keys (ignored by the reference): precision (fp64 | bf16oz |
// tf32x3 | tf32x6 | fp32 | fp64sym), device, G0_file (n*n complex128 binary replacing make_G0), plus
// V_law, quench_gate and AS_dt handled by g12_read_input.
#include "g12kba.h"

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

static std::string ext_value(const char *key)
{
    std::ifstream f("input");
    std::string line, prev;
    bool hit = false;
    while (std::getline(f, line)) {
        if (hit) return line;
        if (line == key) hit = true;
    }
    return "";
}

int main(int argc, char **argv)
{
    (void)argc;
    (void)argv;
    g12_params P;
    std::vector<char> log(1 << 16);
    int rc = g12_read_input("input", &P, log.data(), int(log.size()));
    std::cout << log.data();
    if (rc) {
        std::cerr << "g12kba: an input value could not be converted (the reference's stod/stoi throws)\n";
        return 1;
    }
    int prec = G12_PREC_FP64;
    std::string pv = ext_value("precision");
    if (pv == "tf32x3") prec = G12_PREC_TF32X3;
    else if (pv == "tf32x6") prec = G12_PREC_TF32X6;
    else if (pv == "bf16oz") prec = G12_PREC_BF16OZ;
    else if (pv == "fp32") prec = G12_PREC_FP32;
    else if (pv == "fp64sym") prec = G12_PREC_FP64SYM;
    int device = 0;
    std::string dv = ext_value("device");
    if (!dv.empty()) device = std::atoi(dv.c_str());

    const int n = P.Ns * P.Nb;
    std::vector<double> G1(size_t(2) * n * n);
    g12_make_G0(&P, P.Ns / 2, G1.data());  // Main.cpp:52: p_number = int(Ns/2)
    std::string g0 = ext_value("G0_file");
    if (!g0.empty()) {
        FILE *f = std::fopen(g0.c_str(), "rb");
        if (!f || std::fread(G1.data(), sizeof(double), G1.size(), f) != G1.size()) {
            std::cerr << "g12kba: cannot read G0_file " << g0 << "\n";
            return 1;
        }
        std::fclose(f);
    }

    g12_ctx *ctx = nullptr;
    rc = g12_create(&P, prec, device, &ctx);
    if (rc) {
        std::cerr << "g12kba: " << g12_last_error(nullptr) << "\n";
        return 1;
    }
    rc = g12_set_state(ctx, G1.data(), nullptr, nullptr);
    if (rc) {
        std::cerr << "g12kba: " << g12_last_error(ctx) << "\n";
        return 1;
    }

    // AS.h:65-212
    std::cout << "Beginning Adiabatic Switching Procedure\n";
    auto t0 = std::chrono::steady_clock::now();
    int64_t done = 0;
    rc = g12_adiabatic_switch(ctx, &done);
    if (rc < 0) {
        std::cerr << "g12kba: " << g12_last_error(ctx) << "\n";
        return 1;
    }
    std::cout << "U = " << P.U << "\r";
    auto t1 = std::chrono::steady_clock::now();
    std::cout << "Adiabatic Switching complete, elapsed time:" << std::chrono::duration<double>(t1 - t0).count()
              << " sec \n";

    // RK_solver.h:66-224
    const int64_t T = g12_rk_iterations(&P);
    std::cout << "Beginning Time Stepping Procedure\n";
    auto t2 = std::chrono::steady_clock::now();
    std::vector<double> traj(size_t(2) * n * n * size_t(std::max<int64_t>(T, 1)));
    rc = g12_propagate(ctx, T, traj.data(), &done);
    auto t3 = std::chrono::steady_clock::now();
    const double tmax = double(P.time_steps) * P.dt;
    double t = 0;
    for (int64_t s = 0; s < done; ++s) t += P.dt;
    if (rc == G12_GUARD_TRIPPED) {
        const double nd = 2 * traj[size_t(2) * n * n * size_t(done - 1) + 1];
        std::cout << "ERROR: Unphysical Number Density on site 1:" << nd
                  << " elapsed time:" << std::chrono::duration<double>(t3 - t2).count() << " sec \n";
    } else if (rc < 0) {
        std::cerr << "g12kba: " << g12_last_error(ctx) << "\n";
        return 1;
    } else {
        std::cout << double(t) / (tmax) * 100 << "%\r";
        std::cout << "\n Execution Succesful, elapsed time:" << std::chrono::duration<double>(t3 - t2).count()
                  << " sec \n";
    }
    // progress.txt holds the last step's percentage (RK_solver.h:219-220)
    if (done > 0 && rc != G12_GUARD_TRIPPED) {
        double pr = double(t) / (tmax) * 100;
        g12_write_rfile("progress.txt", &pr, 1);
    }

    // Main.cpp:55-58
    std::vector<double> p(size_t(std::max<int64_t>(done, 1)));
    g12_dipole(traj.data(), done, n, p.data());
    g12_write_cfile2D("G1.txt", traj.data(), done, n * n);
    g12_write_rfile("dipole.txt", p.data(), done);
    g12_destroy(ctx);
    return 0;
}
