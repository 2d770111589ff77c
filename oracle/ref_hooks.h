/*
 * ref_hooks.h -- TEST INFRASTRUCTURE ONLY (part of the oracle, never shipped).
 *
 * Force-included (g++ -include) into the reference build that oracle/build_ref.sh
 * makes from the reference's own s.cpp. The build script rewrites a handful of
 * literal initialisers of the reference so they read the values below from the
 * environment; nothing of the reference's arithmetic is changed:
 *
 *   CFD_MAXSTEP   time steps of the constructor's time loop (s.cpp:178)
 *   CFD_RE/RI/PR/F/ALPHA/DT   physics members (s.cpp:159-173)
 *   CFD_TOL_SIP, CFD_MAXIT_SIP  sip9p's local tol / maxiter (s.cpp:2085-2086)
 *   CFD_TOL_GS,  CFD_MAXIT_GS   gauss's local tol / maxiter (s.cpp:2289-2290)
 *   CFD_DIAG      file receiving 12 float64 per step (loop, time, dmax, cl, cd,
 *                 cm, Nu, circ, CL_pr, CD_pr, CL_vor, CD_vor), written where the
 *                 reference computes Nuss (s.cpp:1982)
 *   CFD_DUMP      file receiving the final fields (replaces main's second
 *                 timeLoop call, s.cpp:2450)
 *   CFD_DUMP_COEF file receiving the assembled coefficient planes
 *
 * Dump format: int32 n0, int32 n1, int32 nplanes, then nplanes planes of
 * n1*n0 float64 in [j][i] order (i fastest), in the order of the name lists
 * below (mirrored by oracle/refrun.py).
 */
#ifndef CFD_REF_HOOKS_H
#define CFD_REF_HOOKS_H
#include <cstdio>
#include <cstdlib>

/* s.cpp keeps the grid size in the global `int n[2]` (s.cpp:8). */
extern int n[2];

static double ref_cfg_d(const char* key, double dflt) {
    const char* s = std::getenv(key);
    return s ? std::strtod(s, nullptr) : dflt;
}
static int ref_cfg_i(const char* key, int dflt) {
    const char* s = std::getenv(key);
    return s ? std::atoi(s) : dflt;
}

static FILE* ref_diag_file() {
    static FILE* fp = nullptr;
    static bool opened = false;
    if (!opened) {
        opened = true;
        const char* path = std::getenv("CFD_DIAG");
        if (path) fp = std::fopen(path, "wb");
    }
    return fp;
}

static void ref_diag(int loop, int time, double dmax, double cl, double cd, double cm,
                     double nu, double circ, double clp, double cdp, double clv,
                     double cdv) {
    FILE* fp = ref_diag_file();
    if (!fp) return;
    double rec[12] = {(double)loop, (double)time, dmax, cl, cd, cm, nu, circ,
                      clp, cdp, clv, cdv};
    std::fwrite(rec, sizeof(double), 12, fp);
    std::fflush(fp);
}

template <class S>
static void ref_write_plane(FILE* fp, S& s, double** a) {
    for (int j = 0; j < n[1]; j++)
        for (int i = 0; i < n[0]; i++) std::fwrite(&a[i][j], sizeof(double), 1, fp);
}

template <class S>
static void ref_dump(S& s) {
    const char* path = std::getenv("CFD_DUMP");
    if (path) {
        FILE* fp = std::fopen(path, "wb");
        double** planes[] = {s.u[0],  s.u[1],  s.u[2],  s.p,    s.up[0], s.up[1],
                             s.us[0], s.us[1], s.pcor,  s.q,    s.qu,    s.qv,
                             s.qt,    s.qup,   s.qvp,   s.si,   s.dil,   s.vort,
                             s.uxi,   s.uet};
        int hdr[3] = {n[0], n[1], (int)(sizeof(planes) / sizeof(planes[0]))};
        std::fwrite(hdr, sizeof(int), 3, fp);
        for (double** a : planes) ref_write_plane(fp, s, a);
        std::fclose(fp);
    }
    const char* cpath = std::getenv("CFD_DUMP_COEF");
    if (cpath) {
        FILE* fp = std::fopen(cpath, "wb");
        double** planes[] = {
            s.aup,    s.aue,    s.auw,    s.aun,    s.aus,    s.aune,   s.aunw,
            s.ause,   s.ausw,   s.auee,   s.auww,   s.aunn,   s.auss,   s.aunnee,
            s.aunnww, s.aussee, s.aussww, s.aunne,  s.aunnw,  s.ausse,  s.aussw,
            s.aunee,  s.aunww,  s.ausee,  s.ausww,  s.atp,    s.ate,    s.atw,
            s.atn,    s.ats,    s.atne,   s.atnw,   s.atse,   s.atsw,   s.atee,
            s.atww,   s.atnn,   s.atss,   s.atnnee, s.atnnww, s.atssee, s.atssww,
            s.atnne,  s.atnnw,  s.atsse,  s.atssw,  s.atnee,  s.atnww,  s.atsee,
            s.atsww,  s.ap,     s.ae,     s.aw,     s.an,     s.as,     s.ane,
            s.anw,    s.ase,    s.asw};
        int hdr[3] = {n[0], n[1], (int)(sizeof(planes) / sizeof(planes[0]))};
        std::fwrite(hdr, sizeof(int), 3, fp);
        for (double** a : planes) ref_write_plane(fp, s, a);
        std::fclose(fp);
    }
}
#endif
