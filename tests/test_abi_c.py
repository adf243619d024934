"""The C ABI from plain C: a C99 program that includes include/g12kba.h, links
libg12kba.so and calls the host-side entry points (input defaults, schedule
counts, G0, dipole, particle number), and checks that device creation fails
loudly without a GPU.  Compiles and runs on CPU."""
import os
import shutil
import subprocess

import pytest

C_SRC = r"""
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include "g12kba.h"

int main(void)
{
    g12_params p;
    g12_params_default(&p);
    p.Ns = 4; p.Nb = 1; p.Nq = 2; p.U = 1.0; p.dt = 0.02; p.time_steps = 2000;
    p.AS_rate = 0.5; p.AS_midpoint = 10.0;
    const int n = p.Ns * p.Nb;
    if (g12_as_steps(&p) != 304) { printf("as_steps %lld\n", (long long)g12_as_steps(&p)); return 1; }
    if (g12_rk_iterations(&p) != 2000) return 2;
    double *G1 = calloc(2 * n * n, sizeof(double));
    if (g12_make_G0(&p, p.Ns / 2, G1) != G12_OK) return 3;
    double N = 0, dip = 0;
    if (g12_particle_number(G1, 1, n, &N) != G12_OK || fabs(N - 2.0 * (p.Ns / 2)) > 1e-6) { printf("N %g\n", N); return 4; }
    if (g12_dipole(G1, 1, n, &dip) != G12_OK) return 5;
    g12_ctx *ctx = NULL;
    int rc = g12_create(&p, G12_PREC_FP64, 0, &ctx);
    if (rc == G12_OK) { g12_destroy(ctx); printf("device\n"); return 0; }
    if (rc != G12_ERR_NO_DEVICE || ctx != NULL) return 6;
    printf("no device: %s\n", g12_last_error(NULL));
    free(G1);
    return 0;
}
"""


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_c_program_binds_the_abi(g12, tmp_path):
    src = tmp_path / "abi.c"
    src.write_text(C_SRC)
    exe = tmp_path / "abi"
    pkg = os.path.dirname(g12.LIB_PATH)
    inc = os.path.dirname(g12.HEADER)
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", inc, str(src), "-o", str(exe), "-L", pkg,
                        "-lg12kba", f"-Wl,-rpath,{pkg}", "-lm"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    assert "no device" in r.stdout or "device" in r.stdout
