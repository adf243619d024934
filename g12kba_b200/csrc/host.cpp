// Host-side half of the C ABI: input reader, schedule counts, initial state,
// dipole and text writers.  No CUDA here; the propagation lives in engine.cu.
#include "g12kba.h"
#include "internal.h"

#include <cerrno>
#include <climits>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <thread>
#include <vector>

namespace g12 {

void log_append(std::string *log, const std::string &s)
{
    if (log) *log += s;
}

}  // namespace g12

using namespace g12;

extern "C" void g12_params_default(g12_params *p)
{
    // read_input.h:27-49
    std::memset(p, 0, sizeof(*p));
    p->HF = 0;
    p->EHM = 0;
    p->t1 = 1;
    p->t2 = 0;
    p->t3 = 0;
    p->U = .5;
    p->time_steps = 1000;
    p->dt = .02;
    p->quench_strength = 1;
    p->Ns = 2;
    p->Nq = 0;
    p->Nb = 1;
    p->q_type = G12_QUENCH_FULL;
    p->AS_rate = 3;
    p->AS_midpoint = 25;
    p->quench_rate = .2;
    p->quench_on_midpoint = 50;
    p->quench_off_midpoint = 55;
    p->v_law = G12_VLAW_EXP;
    p->quench_gate = 50;   // RK_solver.h:141
    p->as_dt = .1;         // AS.h:114-121
    p->decay_rate = .7;    // read_input.h:29
}

namespace {

// The input file as std::getline sees it (read_input.h:53-83).
struct InputLines {
    std::vector<std::string> lines;
    bool exists = false;
    bool last_newline = false;
};

InputLines load_lines(const char *path)
{
    InputLines L;
    std::ifstream f(path, std::ios::binary);
    if (!f.is_open()) return L;
    L.exists = true;
    std::string all((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
    size_t start = 0;
    while (start < all.size()) {
        size_t nl = all.find('\n', start);
        if (nl == std::string::npos) {
            L.lines.push_back(all.substr(start));
            L.last_newline = false;
            return L;
        }
        L.lines.push_back(all.substr(start, nl - start));
        start = nl + 1;
    }
    L.last_newline = !all.empty();
    return L;
}

// read_input.h:53-83.  The value is the line after the first line that
// contains `var`; reading past the end leaves std::getline's last string in
// place, which is "" unless the file lacks a final newline.
std::string read_var_val(const InputLines &L, const std::string &var, std::string *log)
{
    size_t counter = 0;
    for (size_t i = 0; i < L.lines.size(); ++i) {
        counter++;
        if (L.lines[i].find(var) != std::string::npos) break;
    }
    std::string s;
    if (counter + 1 <= L.lines.size()) s = L.lines[counter];
    else if (L.exists && !L.lines.empty() && !L.last_newline) s = L.lines.back();
    if (s.empty()) {
        log_append(log, "Missing value for " + var + " initialising to 0\n");
        return "0";
    }
    return s;
}

// std::stod / std::stoi semantics: leading whitespace skipped, trailing text
// ignored, no conversion or ERANGE rejected.
bool parse_double(const std::string &s, double *out)
{
    const char *b = s.c_str();
    char *e = nullptr;
    errno = 0;
    double v = std::strtod(b, &e);
    if (e == b || errno == ERANGE) return false;
    *out = v;
    return true;
}

bool parse_int(const std::string &s, int32_t *out)
{
    const char *b = s.c_str();
    char *e = nullptr;
    errno = 0;
    long v = std::strtol(b, &e, 10);
    if (e == b || errno == ERANGE || v < INT_MIN || v > INT_MAX) return false;
    *out = int32_t(v);
    return true;
}

bool has_key(const InputLines &L, const std::string &key)
{
    for (auto &l : L.lines)
        if (l == key) return true;
    return false;
}

}  // namespace

extern "C" int g12_read_input(const char *path, g12_params *p, char *logbuf, int32_t logcap)
{
    if (!path || !p) return G12_ERR_INVALID;
    std::string log;
    InputLines L = load_lines(path);
    g12_params_default(p);
    // read_input.h:88-106, in the reference's order (messages depend on it)
    bool ok = true;
    auto rd = [&](const char *k, double *v) {
        if (ok && !parse_double(read_var_val(L, k, &log), v)) ok = false;
    };
    auto ri = [&](const char *k, int32_t *v) {
        if (ok && !parse_int(read_var_val(L, k, &log), v)) ok = false;
    };
    rd("t1", &p->t1);
    rd("t2", &p->t2);
    rd("t3", &p->t3);
    rd("U", &p->U);
    ri("time_steps", &p->time_steps);
    rd("dt", &p->dt);
    rd("quench_strength", &p->quench_strength);
    ri("Ns", &p->Ns);
    ri("Nb", &p->Nb);
    ri("Nq", &p->Nq);
    rd("AS_rate", &p->AS_rate);
    rd("AS_midpoint", &p->AS_midpoint);
    rd("quench_on_midpoint", &p->quench_on_midpoint);
    rd("quench_off_midpoint", &p->quench_off_midpoint);
    rd("quench_rate", &p->quench_rate);
    if (!ok) {
        if (logbuf && logcap > 0) std::snprintf(logbuf, size_t(logcap), "%s", log.c_str());
        return G12_ERR_PARSE;
    }
    // read_input.h:109-144
    if (read_var_val(L, "HF", &log) == "true") p->HF = 1;
    else if (read_var_val(L, "HF", &log) == "false") p->HF = 0;
    else {
        log += "Invalid specification of HF calculation parameter, performing full HF-GKBA calculation.\n";
        p->HF = 0;
    }
    if (read_var_val(L, "EHM", &log) == "true") p->EHM = 1;
    else if (read_var_val(L, "EHM", &log) == "false") p->EHM = 0;
    else {
        log += "Invalid specification for EHM parameter. performing full calculation for onsite model.\n";
        p->EHM = 0;
    }
    if (read_var_val(L, "q_type", &log) == "full") p->q_type = G12_QUENCH_FULL;
    else if (read_var_val(L, "q_type", &log) == "pulse") p->q_type = G12_QUENCH_PULSE;
    else if (read_var_val(L, "q_type", &log) == "none") {
        p->quench_strength = 0;
        p->Nq = 0;
    } else {
        log += "Invalid specification of quench type, no quench initiated\n";
    }
    // Extension keys (the reference ignores unknown keys).  Only read when the
    // key line is present verbatim, so reference inputs never change meaning.
    if (has_key(L, "V_law")) {
        std::string v = read_var_val(L, "V_law", nullptr);
        if (v == "inv") p->v_law = G12_VLAW_INV;
        else if (v == "exp") p->v_law = G12_VLAW_EXP;
        else log += "Invalid V_law, using exp\n";
    }
    if (has_key(L, "quench_gate")) {
        double g;
        if (parse_double(read_var_val(L, "quench_gate", nullptr), &g)) p->quench_gate = g;
    }
    if (has_key(L, "AS_dt")) {
        double g;
        if (parse_double(read_var_val(L, "AS_dt", nullptr), &g)) p->as_dt = g;
    }
    if (logbuf && logcap > 0) std::snprintf(logbuf, size_t(logcap), "%s", log.c_str());
    return G12_OK;
}

// fermi_func.h:21-24
double g12::fermi(double t, double t0, double tau) { return 1.0 / (1 + std::exp((t0 - t) / tau)); }

extern "C" int64_t g12_as_steps(const g12_params *p)
{
    // AS.h:96-100,114-121: the loop head counts |U_AS - U| <= 0, where U_AS
    // is the previous step's last-stage value (unset before the first step).
    if (!p) return -1;
    double t = 0, u_as = NAN;
    int count = 0;
    int64_t steps = 0;
    while (count < 20) {
        if (std::fabs(u_as - p->U) <= 0) count += 1;
        u_as = fermi(t + p->as_dt, p->AS_midpoint, p->AS_rate) * p->U;
        t += p->as_dt;
        if (++steps > (int64_t(1) << 40)) return -1;
    }
    return steps;
}

extern "C" int64_t g12_rk_iterations(const g12_params *p)
{
    // RK_solver.h:66,96,216: while(t < tmax) with t += dt in floating point
    if (!p) return -1;
    double tmax = double(p->time_steps) * p->dt, t = 0;
    int64_t it = 0;
    while (t < tmax) {
        ++it;
        t += p->dt;
        if (it > (int64_t(1) << 40)) return -1;
    }
    return it;
}

namespace {

typedef std::complex<double> cd;

// HF.h:57-104 on the host, for the initial Hamiltonian (U = 0, no quench, no V).
void host_h_hf0(std::vector<cd> &h, int Ns, int Nb, double t1, double t2)
{
    const cd im(0, 1);
    const int n = Ns * Nb;
    std::vector<cd> G1(size_t(n) * n);  // zero: make_G0 passes the empty G1
    const double U = 0;
    for (int i = 0; i < Ns; ++i) {
        for (int a = 0; a < Nb; ++a) {
            h[(i + a * Ns) * n + (i + a * Ns)] += 0.0;
            if (i < Ns - 1) {
                h[((i + 1) + a * Ns) * n + (i + a * Ns)] += -t1;
                h[(i + a * Ns) * n + ((i + 1) + a * Ns)] += -t1;
            }
            if (a < Nb - 1) {
                h[(i + a * Ns) * n + (i + (a + 1) * Ns)] += -t2;
                h[(i + (a + 1) * Ns) * n + (i + a * Ns)] += -t2;
            }
            h[(i + a * Ns) * n + (i + a * Ns)] += -im * U * G1[(i + a * Ns) * n + (i + a * Ns)];
            for (int g = 0; g < Nb; ++g) {
                h[(i + a * Ns) * n + (i + g * Ns)] +=
                    im * U * cd(double(a != g)) * G1[(i + g * Ns) * n + (i + a * Ns)];
                if (g != a) h[(i + a * Ns) * n + (i + a * Ns)] += -2.0 * im * U * G1[(i + g * Ns) * n + (i + g * Ns)];
            }
        }
    }
}

// Cyclic complex Jacobi (Jacobi 1846; Rutishauser's real update formulas with
// the phase of a_pq rotated onto the real axis), FP64, interleaved re/im.
void jacobi_hermitian(int n, double *A, double *V)
{
#define RE(M, r, c) (M)[2 * ((r) * n + (c))]
#define IM(M, r, c) (M)[2 * ((r) * n + (c)) + 1]
    for (int r = 0; r < n; ++r)
        for (int c = 0; c < n; ++c) {
            RE(V, r, c) = (r == c) ? 1.0 : 0.0;
            IM(V, r, c) = 0.0;
        }
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0, tot = 0.0;
        for (int p = 0; p < n; ++p) {
            tot += RE(A, p, p) * RE(A, p, p);
            for (int q = p + 1; q < n; ++q) off += RE(A, p, q) * RE(A, p, q) + IM(A, p, q) * IM(A, p, q);
        }
        tot += 2.0 * off;
        if (off == 0.0 || off <= 1e-36 * tot) break;
        for (int p = 0; p < n - 1; ++p) {
            for (int q = p + 1; q < n; ++q) {
                double apr = RE(A, p, q), api = IM(A, p, q);
                double mag = std::hypot(apr, api);
                if (mag == 0.0) continue;
                double er = apr / mag, ei = api / mag;
                double theta = (RE(A, q, q) - RE(A, p, p)) / (2.0 * mag);
                double t;
                if (std::fabs(theta) > 1e150) t = 0.5 / theta;
                else t = (theta >= 0.0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                double cs = 1.0 / std::sqrt(t * t + 1.0);
                double sn = t * cs;
                double sr = sn * er, si = -sn * ei;
                double cr = cs * er, ci = -cs * ei;
                for (int r = 0; r < n; ++r) {
                    if (r == p || r == q) continue;
                    double xr = RE(A, r, p), xi = IM(A, r, p);
                    double yr = RE(A, r, q), yi = IM(A, r, q);
                    double nrp_r = cs * xr - (sr * yr - si * yi);
                    double nrp_i = cs * xi - (sr * yi + si * yr);
                    double nrq_r = sn * xr + (cr * yr - ci * yi);
                    double nrq_i = sn * xi + (cr * yi + ci * yr);
                    RE(A, r, p) = nrp_r;
                    IM(A, r, p) = nrp_i;
                    RE(A, r, q) = nrq_r;
                    IM(A, r, q) = nrq_i;
                    RE(A, p, r) = nrp_r;
                    IM(A, p, r) = -nrp_i;
                    RE(A, q, r) = nrq_r;
                    IM(A, q, r) = -nrq_i;
                }
                RE(A, p, p) = RE(A, p, p) - t * mag;
                IM(A, p, p) = 0.0;
                RE(A, q, q) = RE(A, q, q) + t * mag;
                IM(A, q, q) = 0.0;
                RE(A, p, q) = 0.0;
                IM(A, p, q) = 0.0;
                RE(A, q, p) = 0.0;
                IM(A, q, p) = 0.0;
                for (int r = 0; r < n; ++r) {
                    double xr = RE(V, r, p), xi = IM(V, r, p);
                    double yr = RE(V, r, q), yi = IM(V, r, q);
                    RE(V, r, p) = cs * xr - (sr * yr - si * yi);
                    IM(V, r, p) = cs * xi - (sr * yi + si * yr);
                    RE(V, r, q) = sn * xr + (cr * yr - ci * yi);
                    IM(V, r, q) = sn * xi + (cr * yi + ci * yr);
                }
            }
        }
    }
#undef RE
#undef IM
}

// LAPACK cheev contract (jobz='V', uplo='L'): ascending eigenvalues, columns
// of `a` the eigenvectors; phase fixed so the first largest-modulus component
// is real positive; FP64 Jacobi on the float-rounded input, rounded to float.
void eig_c64(int n, std::vector<float> &a /* 2*n*n, row-major interleaved */, std::vector<float> &w)
{
    std::vector<double> A(size_t(2) * n * n), V(size_t(2) * n * n);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j <= i; ++j) {
            double re = double(a[2 * (i * n + j)]), im = double(a[2 * (i * n + j) + 1]);
            if (i == j) im = 0.0;
            A[2 * (i * n + j)] = re;
            A[2 * (i * n + j) + 1] = im;
            A[2 * (j * n + i)] = re;
            A[2 * (j * n + i) + 1] = -im;
        }
    jacobi_hermitian(n, A.data(), V.data());
    std::vector<int> ord(n);
    for (int i = 0; i < n; ++i) ord[i] = i;
    for (int i = 1; i < n; ++i) {
        int key = ord[i];
        double kv = A[2 * (key * n + key)];
        int j = i - 1;
        while (j >= 0 && A[2 * (ord[j] * n + ord[j])] > kv) {
            ord[j + 1] = ord[j];
            --j;
        }
        ord[j + 1] = key;
    }
    w.assign(n, 0.f);
    for (int k = 0; k < n; ++k) {
        int src = ord[k];
        w[k] = float(A[2 * (src * n + src)]);
        int m = 0;
        double best = -1.0;
        for (int i = 0; i < n; ++i) {
            double mr = V[2 * (i * n + src)], mi = V[2 * (i * n + src) + 1];
            double mm = mr * mr + mi * mi;
            if (mm > best) {
                best = mm;
                m = i;
            }
        }
        double pr = V[2 * (m * n + src)], pi = V[2 * (m * n + src) + 1];
        double pm = std::hypot(pr, pi);
        double ur = pr / pm, ui = -pi / pm;
        for (int i = 0; i < n; ++i) {
            double vr = V[2 * (i * n + src)], vi = V[2 * (i * n + src) + 1];
            double nr = vr * ur - vi * ui, ni = vr * ui + vi * ur;
            a[2 * (i * n + k)] = float(nr);
            a[2 * (i * n + k) + 1] = float(ni);
        }
    }
}

}  // namespace

extern "C" int g12_make_G0(const g12_params *p, int32_t p_number, double *G1_out)
{
    if (!p || !G1_out || p->Ns < 1 || p->Nb < 1 || p->Ns * p->Nb > 4096) return G12_ERR_INVALID;
    const int Ns = p->Ns, Nb = p->Nb, n = Ns * Nb;
    std::vector<cd> h(size_t(n) * n);
    host_h_hf0(h, Ns, Nb, p->t1, p->t2);
    // init_G.h:28-43: lower triangle to complex64, cheev, back to complex128
    std::vector<float> a(size_t(2) * n * n, 0.f), w;
    for (int j = 0; j < n; ++j)
        for (int i = j; i < n; ++i) {
            a[2 * (i * n + j)] = float(h[i * n + j].real());
            a[2 * (i * n + j) + 1] = float(h[i * n + j].imag());
        }
    eig_c64(n, a, w);
    std::vector<cd> ev(size_t(n) * n);
    for (int x = 0; x < n * n; ++x) ev[x] = cd(a[2 * x], a[2 * x + 1]);
    // init_G.h:67-74
    const cd im(0, 1);
    std::vector<cd> G(size_t(n) * n);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            G[i * n + j] = 0;
            for (int k = 0; k < p_number; ++k) G[i * n + j] += ev[i * n + k] * std::conj(ev[j * n + k]) * im;
        }
    for (int x = 0; x < n * n; ++x) {
        G1_out[2 * x] = G[x].real();
        G1_out[2 * x + 1] = G[x].imag();
    }
    return G12_OK;
}

extern "C" int g12_dipole(const double *traj, int64_t T, int32_t n, double *p_out)
{
    // dipole.h:25-32 (the flattened orbital index is mirrored, bands included)
    if (!traj || !p_out || n < 1) return G12_ERR_INVALID;
    const int64_t N = int64_t(n) * n;
    const double sq = std::sqrt(double(N));
    for (int64_t t = 0; t < T; ++t) p_out[t] = 0.0;
    for (int i = 0; i < int(sq / 2); ++i)
        for (int64_t t = 0; t < T; ++t)
            p_out[t] += 2 * (sq / 2 - i - .5) *
                        (traj[2 * (t * N + i * (int(sq) + 1)) + 1] - traj[2 * (t * N + N - i * (int(sq) + 1) - 1) + 1]) / sq;
    return G12_OK;
}

extern "C" int g12_particle_number(const double *traj, int64_t T, int32_t n, double *N_out)
{
    // N = 2 Tr Im G1 (two spin projections of rho = -i G1); the G1-G2
    // equations conserve it exactly (RK_solver.h:101 guards its site-0 part)
    if (!traj || !N_out || n < 1) return G12_ERR_INVALID;
    const int64_t NN = int64_t(n) * n;
    for (int64_t t = 0; t < T; ++t) {
        double s = 0.0;
        for (int i = 0; i < n; ++i) s += traj[2 * (t * NN + int64_t(i) * (n + 1)) + 1];
        N_out[t] = 2.0 * s;
    }
    return G12_OK;
}

namespace {

// std::ostream << double with default flags and precision 6 == "%.6g".
inline int fmt_g6(char *buf, double v) { return std::snprintf(buf, 32, "%g", v); }

bool write_rows(const std::string &path, const double *traj, int64_t T, int32_t n2, int part)
{
    FILE *f = std::fopen(path.c_str(), "wb");
    if (!f) return false;
    // rows are independent: format blocks of rows on several threads
    const int nthreads = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    const int64_t block = 64;
    std::vector<std::string> out(static_cast<size_t>(nthreads));
    for (int64_t r0 = 0; r0 < n2; r0 += block * nthreads) {
        std::vector<std::thread> th;
        for (int w = 0; w < nthreads; ++w) {
            th.emplace_back([&, w]() {
                std::string &s = out[size_t(w)];
                s.clear();
                char buf[40];
                const int64_t a = r0 + int64_t(w) * block, b = std::min<int64_t>(a + block, n2);
                for (int64_t j = a; j < b; ++j) {
                    for (int64_t i = 0; i < T; ++i) {
                        int len = fmt_g6(buf, traj[2 * (i * int64_t(n2) + j) + part]);
                        s.append(buf, size_t(len));
                        s.push_back(' ');
                    }
                    s.push_back('\n');
                }
            });
        }
        for (auto &t : th) t.join();
        for (auto &s : out) std::fwrite(s.data(), 1, s.size(), f);
    }
    std::fclose(f);
    return true;
}

}  // namespace

extern "C" int g12_write_cfile2D(const char *name, const double *traj, int64_t T, int32_t n2)
{
    // write_to_file.h:52-69: one row per G1 element, one column per snapshot
    if (!name || (!traj && T > 0)) return G12_ERR_INVALID;
    std::string nm(name);
    if (!write_rows("imag_" + nm, traj, T, n2, 1)) return G12_ERR_INVALID;
    if (!write_rows("real_" + nm, traj, T, n2, 0)) return G12_ERR_INVALID;
    return G12_OK;
}

extern "C" int g12_write_rfile(const char *name, const double *data, int64_t count)
{
    // write_to_file.h:26-34
    FILE *f = std::fopen(name, "wb");
    if (!f) return G12_ERR_INVALID;
    char buf[40];
    for (int64_t i = 0; i < count; ++i) {
        int len = fmt_g6(buf, data[i]);
        buf[len] = '\n';
        std::fwrite(buf, 1, size_t(len) + 1, f);
    }
    std::fclose(f);
    return G12_OK;
}
