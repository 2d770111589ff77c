// cfd_driver.cpp -- cfd_b200_solver: the reference program's driver on the B200 library.
//
// The reference's main() constructs a Solver from INP.DAT (PSolver.cpp:502-1043) and runs
// timeLoop() (PSolver.cpp:1051-2065): it prints "loop dmax" every step (PSolver.cpp:1890)
// and, every 100 steps, rewrites spt100.dat and SURF_DIST.dat and appends to COEFF_HIS.dat
// and COEFF_HIS_pr_vor.dat (PSolver.cpp:1989-2040). This program does the same through the
// C ABI of include/cfd_b200.h; the physics constants the reference hard-codes are options.
//
//   cfd_b200_solver [INP.DAT] [--steps N] [--Re x] [--Ri x] [--Pr x] [--F x] [--time-accurate] [--alpha deg]
//                   [--dt x] [--profile ogrid|cavity] [--precision fp64|mixed]
//                   [--tol-mom x] [--tol-p x] [--atol-mom x] [--atol-p x] [--maxit-mom N]
//                   [--maxit-p N] [--out-every N] [--solve-to tol] [--quiet] [--dir DIR]
//
// --solve-to runs until the steady residual (relative to the first step) is below tol or
// --steps steps have run, writing the outputs once at the end. Exit status: 0 on success,
// 1 on bad input, 2 on a solver error (message on stderr).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/cfd_b200.h"

namespace {

struct Grid {
    int n0 = 0, n1 = 0;
    double dxi0 = 0, dxi1 = 0, p_grid = 0, a_grid = 0, ar = 0;
    std::vector<double> x, y, xix, xiy, etx, ety, alph, beta, gam, jac;  // n1*n0, [j][i]
    std::vector<double> xnix, xniy, xnox, xnoy;                           // n0
};

// INP.DAT in the reference's token order (PSolver.cpp:517-547)
bool read_inp(const std::string& path, Grid& g, std::string& err) {
    std::ifstream in(path);
    if (!in) {
        err = "cannot open " + path;
        return false;
    }
    std::vector<double> t;
    t.reserve(1 << 20);
    std::string tok;
    while (in >> tok) {
        char* end = nullptr;
        const double v = std::strtod(tok.c_str(), &end);
        if (end == tok.c_str() || *end) {
            err = path + ": non-numeric token '" + tok + "'";
            return false;
        }
        t.push_back(v);
    }
    if (t.size() < 11) {
        err = path + ": bad header";
        return false;
    }
    g.n0 = (int)t[0];
    g.n1 = (int)t[1];
    if (g.n0 < 6 || g.n1 < 5) {
        err = path + ": grid too small";
        return false;
    }
    const size_t np = (size_t)g.n0 * g.n1;
    const size_t need = 11 + np * 12 + 4 * (size_t)g.n0;
    if (t.size() < need) {
        err = path + ": truncated (" + std::to_string(t.size()) + " tokens, need " + std::to_string(need) + ")";
        return false;
    }
    g.dxi0 = t[2];
    g.dxi1 = t[3];
    g.p_grid = t[4];
    g.a_grid = t[5];
    g.ar = t[6];
    size_t p = 11;
    std::vector<double>* b1[4] = {nullptr, nullptr, &g.x, &g.y};  // xi eta x y
    std::vector<double>* b2[4] = {&g.xix, &g.xiy, &g.etx, &g.ety};
    std::vector<double>* b3[3] = {&g.alph, &g.beta, &g.gam};
    for (auto* v : {&g.x, &g.y, &g.xix, &g.xiy, &g.etx, &g.ety, &g.alph, &g.beta, &g.gam, &g.jac}) v->resize(np);
    for (size_t k = 0; k < np; k++, p += 4)
        for (int m = 0; m < 4; m++)
            if (b1[m]) (*b1[m])[k] = t[p + m];
    for (size_t k = 0; k < np; k++, p += 4)
        for (int m = 0; m < 4; m++) (*b2[m])[k] = t[p + m];
    for (size_t k = 0; k < np; k++, p += 3)
        for (int m = 0; m < 3; m++) (*b3[m])[k] = t[p + m];
    for (size_t k = 0; k < np; k++, p++) g.jac[k] = t[p];
    for (auto* v : {&g.xnix, &g.xniy, &g.xnox, &g.xnoy}) v->resize(g.n0);
    for (int i = 0; i < g.n0; i++, p += 4) {
        g.xnix[i] = t[p];
        g.xniy[i] = t[p + 1];
        g.xnox[i] = t[p + 2];
        g.xnoy[i] = t[p + 3];
    }
    return true;
}

cfd_grid as_abi(const Grid& g) {
    cfd_grid c{};
    c.n0 = g.n0;
    c.n1 = g.n1;
    c.dxi0 = g.dxi0;
    c.dxi1 = g.dxi1;
    c.p_grid = g.p_grid;
    c.a_grid = g.a_grid;
    c.ar = g.ar;
    c.x = g.x.data();
    c.y = g.y.data();
    c.xix = g.xix.data();
    c.xiy = g.xiy.data();
    c.etx = g.etx.data();
    c.ety = g.ety.data();
    c.alph = g.alph.data();
    c.beta = g.beta.data();
    c.gam = g.gam.data();
    c.jac = g.jac.data();
    c.xnix = g.xnix.data();
    c.xniy = g.xniy.data();
    c.xnox = g.xnox.data();
    c.xnoy = g.xnoy.data();
    return c;
}

// spt100.dat: Tecplot zone, x y fixed 9 decimals, u v T p si vort scientific 13 digits,
// j outer / i inner, a blank line after every j row (PSolver.cpp:1991-2004)
bool write_spt(const std::string& path, const Grid& g, const std::vector<double>* f) {
    FILE* o = std::fopen(path.c_str(), "w");
    if (!o) return false;
    std::fprintf(o, "zone\nI=%d\nJ=%d\n", g.n0, g.n1);
    for (int j = 0; j < g.n1; j++) {
        for (int i = 0; i < g.n0; i++) {
            const size_t k = (size_t)j * g.n0 + i;
            std::fprintf(o, "%.9f %.9f %.13e %.13e %.13e %.13e %.13e %.13e\n", g.x[k], g.y[k], f[0][k], f[1][k],
                         f[2][k], f[3][k], f[4][k], f[5][k]);
        }
        std::fprintf(o, "\n");
    }
    return std::fclose(o) == 0;
}

// COEFF_HIS.dat / COEFF_HIS_pr_vor.dat: appended, the int time and four fixed 8-decimal
// values (PSolver.cpp:2018-2026); in time-accurate mode the time as a fixed 8-decimal value
bool append_his(const std::string& path, double time, bool as_int, double a, double b, double c, double d) {
    FILE* o = std::fopen(path.c_str(), "a");
    if (!o) return false;
    if (as_int) std::fprintf(o, "%d %.8f %.8f %.8f %.8f\n", (int)time, a, b, c, d);
    else std::fprintf(o, "%.8f %.8f %.8f %.8f %.8f\n", time, a, b, c, d);
    return std::fclose(o) == 0;
}

// SURF_DIST.dat: xi, p, vorticity and dT/dn on the wall row j = 0, default stream
// formatting (6 significant digits) (PSolver.cpp:2032-2039)
bool write_surf(const std::string& path, const Grid& g, const std::vector<double>* f) {
    FILE* o = std::fopen(path.c_str(), "w");
    if (!o) return false;
    const std::vector<double>&T = f[2], &P = f[3], &VO = f[5];
    const int n0 = g.n0;
    for (int i = 0; i < n0; i++) {
        double dthdn = -(4 * T[n0 + i] - 3 * T[i] - T[2 * n0 + i]) / (2 * g.dxi1);
        dthdn = dthdn * std::sqrt(g.etx[i] * g.etx[i] + g.ety[i] * g.ety[i]);
        std::fprintf(o, "%g %g %g %g\n", i * g.dxi0, P[i], VO[i], dthdn);
    }
    return std::fclose(o) == 0;
}

int usage() {
    std::fprintf(stderr,
                 "usage: cfd_b200_solver [INP.DAT] [--steps N] [--Re x] [--Ri x] [--Pr x] [--F x] [--time-accurate] [--alpha deg]\n"
                 "       [--dt x] [--profile ogrid|cavity] [--precision fp64|mixed] [--tol-mom x] [--tol-p x]\n"
                 "       [--atol-mom x] [--atol-p x] [--maxit-mom N] [--maxit-p N]\n"
                 "       [--out-every N] [--solve-to tol] [--quiet] [--dir DIR]\n");
    return 1;
}

}  // namespace

int main(int argc, char** argv) {
    std::string inp = "INP.DAT", dir = ".";
    long long steps = 1000;
    int out_every = 100;
    bool quiet = false;
    double solve_to = -1.0;
    cfd_params prm;
    cfd_params_default(&prm);
    for (int a = 1; a < argc; a++) {
        const std::string k = argv[a];
        auto val = [&]() -> const char* { return a + 1 < argc ? argv[++a] : nullptr; };
        auto num = [&](double& out) {
            const char* v = val();
            if (!v) return false;
            char* e = nullptr;
            out = std::strtod(v, &e);
            return e != v && !*e;
        };
        double d = 0;
        // a count: a whole number in [0, 2^31 - 1]
        auto count = [&]() { return num(d) && d >= 0 && d <= 2147483647.0 && d == std::floor(d); };
        if (k == "--steps") { if (!count()) return usage(); steps = (long long)d; }
        else if (k == "--Re") { if (!num(prm.Re)) return usage(); }
        else if (k == "--Ri") { if (!num(prm.Ri)) return usage(); }
        else if (k == "--Pr") { if (!num(prm.Pr)) return usage(); }
        else if (k == "--F") { if (!num(prm.F)) return usage(); }
        else if (k == "--alpha") { if (!num(prm.alpha_deg)) return usage(); }
        else if (k == "--dt") { if (!num(prm.dt)) return usage(); }
        else if (k == "--tol-mom") { if (!num(prm.tol_mom)) return usage(); }
        else if (k == "--tol-p") { if (!num(prm.tol_p)) return usage(); }
        else if (k == "--atol-mom") { if (!num(prm.atol_mom)) return usage(); }
        else if (k == "--atol-p") { if (!num(prm.atol_p)) return usage(); }
        else if (k == "--maxit-mom") { if (!count() || d < 2) return usage(); prm.maxit_mom = (int)d; }
        else if (k == "--maxit-p") { if (!count() || d < 1) return usage(); prm.maxit_p = (int)d; }
        else if (k == "--out-every") { if (!count()) return usage(); out_every = (int)d; }
        else if (k == "--solve-to") { if (!num(solve_to)) return usage(); }
        else if (k == "--quiet") quiet = true;
        else if (k == "--time-accurate") prm.time_accurate = 1;
        else if (k == "--dir") { const char* v = val(); if (!v) return usage(); dir = v; }
        else if (k == "--profile") {
            const char* v = val();
            if (!v) return usage();
            if (!std::strcmp(v, "ogrid")) prm.profile = CFD_PROFILE_OGRID;
            else if (!std::strcmp(v, "cavity")) prm.profile = CFD_PROFILE_CAVITY;
            else return usage();
        } else if (k == "--precision") {
            const char* v = val();
            if (!v) return usage();
            if (!std::strcmp(v, "fp64")) prm.precision = CFD_PRECISION_FP64;
            else if (!std::strcmp(v, "mixed")) prm.precision = CFD_PRECISION_MIXED;
            else return usage();
        } else if (!k.empty() && k[0] != '-') inp = k;
        else return usage();
    }
    // the cavity uses the Fortran-intent T coefficient (the C++ slot bug destabilises T on
    // skewed grids); the O-grid keeps the reference's C++ behaviour
    if (prm.profile == CFD_PROFILE_CAVITY) prm.fix_T_annw = 1;
    Grid g;
    std::string err;
    if (!read_inp(inp, g, err)) {
        std::fprintf(stderr, "cfd_b200_solver: %s\n", err.c_str());
        return 1;
    }
    const cfd_grid cg = as_abi(g);
    cfd_case* c = nullptr;
    if (cfd_case_create(&cg, &prm, &c) != CFD_OK) {
        std::fprintf(stderr, "cfd_b200_solver: %s\n", cfd_last_error());
        return 2;
    }
    const size_t np = (size_t)g.n0 * g.n1;
    std::vector<double> f[6];
    for (auto& v : f) v.resize(np);
    double time = 0;  // the reference's time is an int (PSolver.cpp:186), unless time-accurate
    const bool int_time = !prm.time_accurate;
    auto outputs = [&](const cfd_step_stats& st) -> bool {
        if (cfd_case_get_fields(c, f[0].data(), f[1].data(), f[2].data(), f[3].data(), f[4].data(), f[5].data()))
            return false;
        return write_spt(dir + "/spt100.dat", g, f) &&
               append_his(dir + "/COEFF_HIS.dat", time, int_time, st.cl, st.cd, st.cm, st.nu) &&
               append_his(dir + "/COEFF_HIS_pr_vor.dat", time, int_time, st.cl_pr, st.cd_pr, st.cl_vor, st.cd_vor) &&
               write_surf(dir + "/SURF_DIST.dat", g, f);
    };
    int rc = 0;
    cfd_step_stats st{};
    if (solve_to > 0) {
        rc = cfd_case_solve_to(c, solve_to, (int)steps, &st);
        if (rc == CFD_OK || rc == CFD_E_NOTCONV) {
            std::printf("steps %d steady_res_rel %.6e nu %.12f status %d\n", st.steps, st.steady_res_rel, st.nu,
                        rc == CFD_OK ? 0 : 1);
            if (!outputs(st)) rc = CFD_E_ARG;
            else rc = CFD_OK;
        }
    } else {
        for (long long loop = 0; loop < steps && rc == CFD_OK; loop++) {
            rc = cfd_case_step(c, 1, &st);
            if (rc) break;
            time = st.time;  // (int)(time + dt) in the reference's int mode
            if (!quiet) std::printf("%lld %g\n", loop, st.dmax);  // "loop dmax", PSolver.cpp:1890
            if (out_every > 0 && loop % out_every == 0 && !outputs(st)) rc = CFD_E_ARG;
        }
    }
    if (rc != CFD_OK) std::fprintf(stderr, "cfd_b200_solver: %s\n", cfd_last_error());
    cfd_case_destroy(c);
    return rc == CFD_OK ? 0 : 2;
}
