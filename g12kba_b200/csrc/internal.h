// Internal declarations shared by the host (host.cpp) and device (engine.cu)
// halves of libg12kba.so.  Not part of the C ABI.
#pragma once

#include <string>

namespace g12 {

// fermi_func.h:21-24, evaluated on the host in FP64 (glibc exp) so that the
// schedule scalars and the AS termination test match the reference bit for bit.
double fermi(double t, double t0, double tau);

void log_append(std::string *log, const std::string &s);

// Per-stage scalars of one RK4 step (AS.h:114-141, RK_solver.h:122-151).
struct StageP {
    double U;       // U_eff: U (RK4) or U_AS = fermi(t_RK)*U (AS)
    double wq;      // quench amplitude added to h on sites i < nq
    double c_next;  // dt of the next stage: tmp_{k+1} = Y + c_next*K_k
    double w;       // RK weight 1, 2, 2, 1
    double dt;      // full step (the final Y += RK*dt/6)
    int nq;         // quench extent
    int pad;
};

struct StepP {
    StageP st[4];
    int record;  // RK4 phase: snapshot + density guard at the step head
    int pad[3];
};

}  // namespace g12
