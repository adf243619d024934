/*
 * Oracle test infrastructure (never linked into the product).
 *
 * Compiles the reference's own headers (G12KBA-GW/src/headers/*.h, taken from
 * a temporary copy with the patch set applied by oracle/build_ref.sh) into
 *   oracle/_ref/g12_ref        - a driver equivalent to G12KBA-GW/src/main/Main.cpp:44-62
 *                                plus full-precision binary dumps, and
 *   oracle/_ref/libg12ref.so   - extern "C" wrappers around each reference routine,
 *                                for per-function parity tests.
 *
 * Behaviour fixes that need no source change are made here, on globals:
 *   - epsilon is resized to Nb zeros (read_input.h:43 sizes it for Nb=1, so
 *     HF.h:65 reads past its end for Nb>=2);
 *   - the global V is sized Ns-1 when EHM=true.  AS.h:68-73 and
 *     RK_solver.h:70-76 fill a block-local V that shadows the global one, and
 *     AS.h:138 then writes into the empty global vector (segfault).  Once the
 *     global has the right size, AS.h:136-140 refreshes it every stage with
 *     U_AS*law(r), and RK4 then runs with the final U*law(r).
 */
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <complex>
#include <chrono>
#include <fstream>
#include <iostream>

/* long-range interaction law used by the patched AS.h / RK_solver.h
 * (build_ref.sh replaces exp(-decay_rate*(i+1)) with G12_VLAW(i+1)) */
double G12_VLAW(int r);

#include "write_to_file.h"
#include "RK_solver.h"
#include "AS.h"
#include "init_G.h"
#include "dipole.h"
#include "read_input.h"

using namespace std;

complex<double> im = {0, 1};

/* 0: U*exp(-decay_rate*r) as in AS.h:138 / RK_solver.h:74;  1: U/(1+r). */
static int g_vlaw = 0;

double G12_VLAW(int r)
{
    if (g_vlaw == 1) return 1.0 / (1.0 + double(r));
    return exp(-decay_rate * r);
}

typedef complex<double> cd;

static vector<cd> from_raw(const double *p, size_t n)
{
    vector<cd> v(n);
    if (p) for (size_t i = 0; i < n; ++i) v[i] = cd(p[2 * i], p[2 * i + 1]);
    return v;
}

static void to_raw(const vector<cd> &v, double *p)
{
    for (size_t i = 0; i < v.size(); ++i) { p[2 * i] = v[i].real(); p[2 * i + 1] = v[i].imag(); }
}

static vector<double> vvec(const double *V, int nV)
{
    vector<double> v;
    for (int i = 0; i < nV; ++i) v.push_back(V[i]);
    return v;
}

static void set_dims(int ns, int nb)
{
    Ns = ns; Nb = nb; Ns2 = ns * ns; Nb2 = nb * nb;
    epsilon.assign(nb, 0.0);
}

extern "C" {

double ref_fermi(double t, double t0, double tau) { return fermi(t, t0, tau); }

/* HF.h:57-104 */
void ref_h_HFx_quench(double *h_out, const double *G1, int ns, int nb, double u,
                      double tt1, double tt2, double w, const double *V, int nV, int nq)
{
    set_dims(ns, nb);
    size_t n2 = size_t(ns * nb) * size_t(ns * nb);
    vector<cd> h(n2), g = from_raw(G1, n2);
    vector<double> vv = vvec(V, nV);
    h_HFx_quench(h, g, g, ns, nb, u, tt1, tt2, w, epsilon, vv, nq);
    to_raw(h, h_out);
}

/* commutators.h:28-51 */
void ref_hG_commutator(const double *G, const double *h, double *comm, int n)
{
    size_t n2 = size_t(n) * n;
    vector<cd> g = from_raw(G, n2), hh = from_raw(h, n2), c(n2);
    hG_commutator(g, hh, c);
    to_raw(c, comm);
}

/* commutators.h:53-99 */
void ref_h2_commutator(const double *G2, const double *h, double *comm, int ns, int nb)
{
    set_dims(ns, nb);
    size_t n = size_t(ns * nb), n4 = n * n * n * n;
    vector<cd> g = from_raw(G2, n4), hh = from_raw(h, n * n), c(n4);
    h2xyG2xyxy_commutator(g, hh, hh, c, ns, nb);
    to_raw(c, comm);
}

/* psi.h:157-276 */
void ref_psi_xxxx(double *psi, const double *G1, int ns, int nb, double u, const double *V, int nV)
{
    set_dims(ns, nb);
    size_t n = size_t(ns * nb), n4 = n * n * n * n;
    vector<cd> p(n4), g = from_raw(G1, n * n);
    vector<double> vv = vvec(V, nV);
    Psi_xxxx(p, g, ns, nb, u, vv);
    to_raw(p, psi);
}

/* psi.h:26-154 */
void ref_psi_xyxy(double *psi, const double *G1, int ns, int nb, double u, const double *V, int nV)
{
    set_dims(ns, nb);
    size_t n = size_t(ns * nb), n4 = n * n * n * n;
    vector<cd> p(n4), g = from_raw(G1, n * n);
    vector<double> vv = vvec(V, nV);
    Psi_xyxy(p, g, ns, nb, u, vv);
    to_raw(p, psi);
}

/* pi.h:25-95; called as Pi(pi_xx,G1,G2xy,G2xx) and Pi(pi_xy,G1,G2xx,G2xy) */
void ref_pi(double *pi, const double *G1, const double *G2a, const double *G2b, double u,
            int ns, int nb, const double *V, int nV)
{
    set_dims(ns, nb);
    size_t n = size_t(ns * nb), n4 = n * n * n * n;
    vector<cd> p(n4), g = from_raw(G1, n * n), a = from_raw(G2a, n4), b = from_raw(G2b, n4);
    vector<double> vv = vvec(V, nV);
    Pi_xyxy(p, g, a, b, u, ns, nb, vv);
    to_raw(p, pi);
}

/* collision_integral.h:27-69 */
void ref_collision(double *I, const double *G2xy, const double *G2xx, int ns, int nb, double u,
                   const double *V, int nV)
{
    set_dims(ns, nb);
    size_t n = size_t(ns * nb), n4 = n * n * n * n;
    vector<cd> ii(n * n), a = from_raw(G2xy, n4), b = from_raw(G2xx, n4);
    vector<double> vv = vvec(V, nV);
    collision_int(ii, a, b, ns, nb, u, vv);
    to_raw(ii, I);
}

/* G1_G2_t_step.h:24-47 (K overwritten, RK accumulated in place) */
void ref_G1_step(const double *comm, const double *I, double *K, double *RK, double w, int ns, int nb)
{
    size_t n = size_t(ns * nb);
    vector<cd> c = from_raw(comm, n * n), ii = from_raw(I, n * n), k(n * n), rk = from_raw(RK, n * n);
    G1_step(c, ii, k, rk, w, ns, nb);
    to_raw(k, K);
    to_raw(rk, RK);
}

/* G1_G2_t_step.h:55-86 */
void ref_G2_step(const double *comm, const double *psi, const double *pi, double *K, double *RK,
                 double w, int ns, int nb)
{
    set_dims(ns, nb);
    size_t n = size_t(ns * nb), n4 = n * n * n * n;
    vector<cd> c = from_raw(comm, n4), ps = from_raw(psi, n4), pp = from_raw(pi, n4), k(n4),
               rk = from_raw(RK, n4);
    G2_step(c, ps, pp, k, rk, w, ns, nb);
    to_raw(k, K);
    to_raw(rk, RK);
}

/* init_G.h:57-75 with the MKL shim's cheev */
void ref_make_G0(double *G1, int ns, int nb, int p_number, double tt1, double tt2)
{
    set_dims(ns, nb);
    size_t n = size_t(ns * nb);
    vector<cd> g(n * n);
    make_G0(g, ns, nb, p_number, 0, tt1, tt2, 0, epsilon);
    to_raw(g, G1);
}

/* dipole.h:25-32 over T snapshots of n2 entries */
void ref_dipole(double *p, const double *traj, int T, int n2)
{
    vector<vector<cd>> tr(T);
    for (int t = 0; t < T; ++t) tr[t] = from_raw(traj + size_t(2) * n2 * t, n2);
    vector<double> pp(T);
    dipole(pp, tr);
    for (int t = 0; t < T; ++t) p[t] = pp[t];
}

} /* extern "C" */

#ifdef G12_REF_MAIN

static void dump(const string &dir, const string &name, const vector<cd> &v)
{
    FILE *f = fopen((dir + "/" + name).c_str(), "wb");
    if (!f) { perror(name.c_str()); exit(2); }
    fwrite(v.data(), sizeof(cd), v.size(), f);
    fclose(f);
}

/*
 * Usage: g12_ref [--vlaw exp|inv] [--dump DIR] [--g0 FILE] [--no-text]
 *                [--skip-as] [--time-rk W K] [--print-params]
 * Reads ./input exactly as G12KBA-GW/src/main/Main.cpp does.
 */
int main(int argc, char **argv)
{
    string dumpdir, g0file;
    bool no_text = false, skip_as = false, print_params = false;
    long time_w = -1, time_k = -1;
    for (int a = 1; a < argc; ++a) {
        string s = argv[a];
        if (s == "--vlaw" && a + 1 < argc) { string v = argv[++a]; g_vlaw = (v == "inv") ? 1 : 0; }
        else if (s == "--dump" && a + 1 < argc) dumpdir = argv[++a];
        else if (s == "--g0" && a + 1 < argc) g0file = argv[++a];
        else if (s == "--no-text") no_text = true;
        else if (s == "--skip-as") skip_as = true;
        else if (s == "--print-params") print_params = true;
        else if (s == "--time-rk" && a + 2 < argc) { time_w = atol(argv[++a]); time_k = atol(argv[++a]); }
        else { fprintf(stderr, "g12_ref: unknown argument %s\n", s.c_str()); return 2; }
    }

    assign_vals();
    if (print_params) {
        /* the globals read_input.h:85-146 produced, for reader parity tests */
        printf("{\"Ns\": %d, \"Nb\": %d, \"Nq\": %d, \"time_steps\": %d, \"HF\": %d, \"EHM\": %d, "
               "\"q_type\": \"%s\", \"t1\": %.17g, \"t2\": %.17g, \"t3\": %.17g, \"U\": %.17g, "
               "\"dt\": %.17g, \"quench_strength\": %.17g, \"AS_rate\": %.17g, \"AS_midpoint\": %.17g, "
               "\"quench_rate\": %.17g, \"quench_on_midpoint\": %.17g, \"quench_off_midpoint\": %.17g}\n",
               Ns, Nb, Nq, time_steps, int(HF), int(EHM), q_type.c_str(), t1, t2, t3, U, dt_fixed,
               quench_strength, AS_rate, AS_midpoint, quench_rate, quench_on_midpoint, quench_off_midpoint);
        return 0;
    }
    epsilon.assign(Nb, 0.0);
    if (EHM) V.assign(Ns > 1 ? Ns - 1 : 0, 0.0);

    vector<cd> G1x(Ns * Ns * Nb * Nb);
    vector<cd> G2xxxx(Ns2 * Ns2 * Nb2 * Nb2);
    vector<cd> G2xydy(Ns2 * Ns2 * Nb2 * Nb2);
    vector<vector<cd>> G1x_diag;
    make_G0(G1x, Ns, Nb, int(Ns / 2), 0, t1, t2, t3, epsilon);
    if (!g0file.empty()) {
        FILE *f = fopen(g0file.c_str(), "rb");
        if (!f || fread(G1x.data(), sizeof(cd), G1x.size(), f) != G1x.size()) {
            fprintf(stderr, "g12_ref: cannot read %s\n", g0file.c_str());
            return 2;
        }
        fclose(f);
    }
    if (!dumpdir.empty()) dump(dumpdir, "g0.bin", G1x);

    if (time_k >= 0) {
        /* CPU-baseline timing: RK4 steps only, from G0 with G2 = 0 (the cost
         * of a step does not depend on the state values). */
        if (EHM) for (int i = 0; i < Ns - 1; ++i) V[i] = U * G12_VLAW(i + 1);
        int saved = time_steps;
        time_steps = int(time_w);
        vector<vector<cd>> warm;
        if (time_w > 0) RK4(G1x, G2xxxx, G2xydy, warm);
        time_steps = int(time_k);
        auto t0 = chrono::steady_clock::now();
        RK4(G1x, G2xxxx, G2xydy, G1x_diag);
        auto t1c = chrono::steady_clock::now();
        time_steps = saved;
        double sec = chrono::duration<double>(t1c - t0).count();
        printf("\n{\"rk_iterations\": %zu, \"seconds\": %.9f}\n", G1x_diag.size(), sec);
        return 0;
    }

    if (!skip_as) Adiabatic_switching(G1x, G2xxxx, G2xydy, G1x_diag);
    else if (EHM) for (int i = 0; i < Ns - 1; ++i) V[i] = U * G12_VLAW(i + 1);
    if (!dumpdir.empty()) {
        dump(dumpdir, "g1_as.bin", G1x);
        dump(dumpdir, "g2xx_as.bin", G2xxxx);
        dump(dumpdir, "g2xy_as.bin", G2xydy);
    }
    int rc = RK4(G1x, G2xxxx, G2xydy, G1x_diag);
    vector<double> p(G1x_diag.size());
    if (!G1x_diag.empty()) dipole(p, G1x_diag);
    if (!no_text) {
        write_to_cfile2D("G1.txt", G1x_diag);
        write_to_rfile("dipole.txt", p);
    }
    if (!dumpdir.empty()) {
        vector<cd> flat;
        for (auto &g : G1x_diag) flat.insert(flat.end(), g.begin(), g.end());
        dump(dumpdir, "traj.bin", flat);
        dump(dumpdir, "g2xx.bin", G2xxxx);
        dump(dumpdir, "g2xy.bin", G2xydy);
        FILE *f = fopen((dumpdir + "/dipole.bin").c_str(), "wb");
        fwrite(p.data(), sizeof(double), p.size(), f);
        fclose(f);
        f = fopen((dumpdir + "/meta.txt").c_str(), "w");
        fprintf(f, "T %zu\nNs %d\nNb %d\nrk_status %d\n", G1x_diag.size(), Ns, Nb, rc);
        fclose(f);
    }
    return 0;
}
#endif
