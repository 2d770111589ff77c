/*
 * cfd_oracle.c -- TEST INFRASTRUCTURE ONLY. FP64 CPU restatement of the
 * reference solver's time step (mhsuhail00/CFD_Solver, PSolver.cpp), used as
 * the parity checker for the CUDA path. Only tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg may load it; the product never does.
 *
 * Layout: every plane is n1*n0 float64 in [j][i] order (i fastest), the order
 * of INP.DAT. The reference's arrays are [i][j]; only the storage differs.
 *
 * Profile OGRID restates the reference exactly, loop order and expression
 * association included, so that it can be pinned to the compiled reference
 * (oracle/_ref) bit for bit:
 *   coefficient assembly            PSolver.cpp:752-940, 944-1040
 *   contravariant velocities        PSolver.cpp:1063-1069
 *   convection + right-hand sides   PSolver.cpp:1075-1237
 *   five gauss() solves             PSolver.cpp:1241-1350, body 2280-2446
 *   up/vp far-field condition       PSolver.cpp:1356-1382
 *   face velocities -> q            PSolver.cpp:1390-1449
 *   sip9p() pressure correction     PSolver.cpp:1453-1466, body 2067-2278
 *   pcor boundary conditions        PSolver.cpp:1471-1499
 *   velocity / pressure correction  PSolver.cpp:1505-1542
 *   far-field vr/vth, circulation   PSolver.cpp:1549-1609
 *   u/v/T boundary update           PSolver.cpp:1617-1656
 *   boundary pressure               PSolver.cpp:1668-1783
 *   stream function                 PSolver.cpp:1789-1801
 *   dilatation / vorticity / dmax   PSolver.cpp:1807-1888
 *   forces, moment, Nusselt         PSolver.cpp:1901-1983
 * The reference's C++ quirks are kept by default: the T solve passes atnw in
 * the annw slot (PSolver.cpp:1290), `time` is an int (PSolver.cpp:186), the
 * circulation spacing is 1/(n0-2) (PSolver.cpp:1571). fix_T_annw / fix_circ_de
 * switch to the Fortran intent (solver.for:907, :1197).
 *
 * Profile CAVITY (no reference implementation) reuses the same interior
 * discretisation with xi non-periodic: lid-driven unit square, lid u = lid_u on
 * j = n1-1, no-slip elsewhere, T = 1 on j = 0, T = 0 on j = n1-1, adiabatic
 * i-walls. Its boundary treatment is this project's definition:
 *   - 9-point operator on the ring of cells next to any wall, 25-point inside;
 *   - boundary couplings are not folded: solves read the fixed wall values;
 *   - xi-derivatives next to an i-wall are 2nd-order central;
 *   - pcor frozen at 0 on walls during the solve, then copied from the
 *     adjacent interior (zero normal gradient), p likewise, corners averaged;
 *   - adiabatic walls T = (4 T1 - T2) / 3.
 * The inner solvers stay lexicographic Gauss-Seidel and SIP(0.92).
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define ORC_OGRID 0
#define ORC_CAVITY 1

typedef struct {
    double Re, Ri, Pr, F, alpha_deg, dt;
    double tol_gs, tol_sip;
    int maxit_gs, maxit_sip;
    int profile;
    int fix_T_annw;
    int fix_circ_de;
    double omega_p; /* p += omega_p * pcor (the reference: 1) */
    double lid_u;   /* cavity lid velocity */
    int time_accurate; /* 1: the wall motion sees t = n dt (a double); 0: the reference's int time */
    /* absolute L1 residual floors of the gauss() / sip9p() stop rules (not in the reference;
     * 0 keeps its relative-only rule). A converged run needs them: the first residual of a
     * solve started from the previous step's solution shrinks with the step-to-step change,
     * so a relative rule alone asks for residuals below rounding near the steady state. */
    double atol_gs, atol_sip;
} orc_params;

/* per-step diagnostics record */
enum {
    D_LOOP, D_TIME, D_DMAX, D_CL, D_CD, D_CM, D_NU, D_CIRC, D_CLP, D_CDP, D_CLV, D_CDV,
    D_QL1, D_QL2, D_QMAX, D_DTL1, D_DTMAX, D_DUL1,
    D_IT_U, D_IT_V, D_IT_T, D_IT_UP, D_IT_VP, D_IT_SIP,
    D_COUNT
};

enum {
    /* 25 velocity and 25 temperature coefficient planes */
    C_P, C_E, C_W, C_N, C_S, C_NE, C_NW, C_SE, C_SW, C_EE, C_WW, C_NN, C_SS,
    C_NNEE, C_NNWW, C_SSEE, C_SSWW, C_NNE, C_NNW, C_SSE, C_SSW, C_NEE, C_NWW,
    C_SEE, C_SWW, C_NCOEF
};

typedef struct {
    int n0, n1;
    double d0, d1, ar;
    orc_params prm;
    double Pi, uinf, vinf, speed_amp, accn_amp, thetamax;
    int loop, time;
    double timed; /* time as a double (time-accurate mode) */
    /* grid */
    double *x, *y, *xix, *xiy, *etx, *ety, *alph, *beta, *gam, *jac;
    double *xnix, *xniy, *xnox, *xnoy;
    /* state */
    double *u, *v, *T, *p, *up, *vp, *us, *vs, *uold, *vold, *Told;
    double *pcor, *q, *qu, *qv, *qt, *qup, *qvp, *sol, *uxi, *uet, *si, *dil, *vort;
    double *vr0, *vr1, *vth0, *vth1;
    /* coefficients */
    double *au[C_NCOEF], *at[C_NCOEF];
    double *bus, *buse, *busw, *bts, *btse, *btsw, *bun, *bune, *bunw, *btn, *btne, *btnw;
    double *ap, *ae, *aw, *an, *as, *ane, *anw, *ase, *asw;
    /* SIP factors (pure function of the pressure coefficients) and scratch */
    double *fbe, *fbw, *fbs, *fbn, *fbne, *fbsw, *fbp, *res, *qp, *del;
    /* previous fields for residual diagnostics */
    double *Tprev, *uprev, *vprev;
    double diag[D_COUNT];
    int sip_factored;
} orc_case;

#define IX(i, j) ((size_t)(j) * (size_t)n0 + (size_t)(i))

static double* plane(const orc_case* c) {
    return (double*)calloc((size_t)c->n0 * (size_t)c->n1, sizeof(double));
}

/* ------------------------------------------------------------------ */
/* periodic neighbour indices of the reference (xi periodic, seam n0-1) */
static inline int og_inn(int i, int n0) { return i == 0 ? n0 - 2 : i - 1; }
static inline int og_inn2(int i, int n0) { return i == 0 ? n0 - 3 : (i == 1 ? n0 - 2 : i - 2); }
static inline int og_ipp2(int i, int n0) { return i == n0 - 2 ? 1 : i + 2; }

static inline int is_cav(const orc_case* c) { return c->prm.profile == ORC_CAVITY; }
static inline int ilo(const orc_case* c) { return is_cav(c) ? 1 : 0; }
static inline int ihi(const orc_case* c) { return c->n0 - 2; } /* inclusive */

static inline void nbr(const orc_case* c, int i, int* inn, int* ipp, int* inn2, int* ipp2) {
    int n0 = c->n0;
    if (is_cav(c)) {
        *inn = i - 1; *ipp = i + 1; *inn2 = i - 2; *ipp2 = i + 2;
    } else {
        *inn = og_inn(i, n0); *ipp = i + 1; *inn2 = og_inn2(i, n0); *ipp2 = og_ipp2(i, n0);
    }
}

/* the 9-point ring: rows next to the j-walls, and for the cavity the i-walls */
static inline int near_wall(const orc_case* c, int i, int j) {
    if (j == 1 || j == c->n1 - 2) return 1;
    if (is_cav(c) && (i == 1 || i == c->n0 - 2)) return 1;
    return 0;
}

/* ------------------------------------------------------------------ */
/* u/v/T coefficient assembly, PSolver.cpp:752-940 */
static void assemble_uvT(orc_case* c) {
    const int n0 = c->n0, n1 = c->n1;
    const double d0 = c->d0, d1 = c->d1, dt = c->prm.dt, Re = c->prm.Re, Pr = c->prm.Pr;
    double** A = c->au;
    double** B = c->at;
    for (int j = 1; j < n1 - 1; j++) {
        for (int i = ilo(c); i <= ihi(c); i++) {
            const size_t k = IX(i, j);
            const double al = c->alph[k], be = c->beta[k], ga = c->gam[k];
            if (near_wall(c, i, j)) {
                A[C_E][k] = -dt * (al / (d0 * d0)) / Re;
                A[C_W][k] = -dt * (al / (d0 * d0)) / Re;
                A[C_N][k] = -dt * (ga / (d1 * d1)) / Re;
                A[C_S][k] = -dt * (ga / (d1 * d1)) / Re;
                A[C_NE][k] = dt * be / (2.0 * d0 * d1 * Re);
                A[C_SW][k] = A[C_NE][k];
                A[C_NW][k] = -dt * be / (2.0 * d0 * d1 * Re);
                A[C_SE][k] = A[C_NW][k];
                A[C_P][k] = 1 + dt * 2.0 * (al / (d0 * d0) + ga / (d1 * d1)) / Re;
                B[C_E][k] = -dt * (al / (d0 * d0)) / (Re * Pr);
                B[C_W][k] = -dt * (al / (d0 * d0)) / (Re * Pr);
                B[C_N][k] = -dt * (ga / (d1 * d1)) / (Re * Pr);
                B[C_S][k] = -dt * (ga / (d1 * d1)) / (Re * Pr);
                B[C_NE][k] = dt * (be / (2.0 * d0 * d1)) / (Re * Pr);
                B[C_SW][k] = B[C_NE][k];
                B[C_NW][k] = -dt * (be / (2.0 * d0 * d1)) / (Re * Pr);
                B[C_SE][k] = B[C_NW][k];
                B[C_P][k] = 1 + dt * 2.0 * (al / (d0 * d0) + ga / (d1 * d1)) / (Re * Pr);
            } else {
                A[C_E][k] = (-dt) * ((4.0 * al) / (3.0 * d0 * d0)) / Re;
                A[C_W][k] = (-dt) * ((4.0 * al) / (3.0 * d0 * d0)) / Re;
                A[C_N][k] = (-dt) * ((4.0 * ga) / (3.0 * d1 * d1)) / Re;
                A[C_S][k] = (-dt) * ((4.0 * ga) / (3.0 * d1 * d1)) / Re;
                A[C_NE][k] = (-dt) * (-8.0 * be / (9.0 * d0 * d1)) / Re;
                A[C_NW][k] = (-dt) * (8.0 * be / (9.0 * d0 * d1)) / Re;
                A[C_SE][k] = A[C_NW][k];
                A[C_SW][k] = A[C_NE][k];
                A[C_NN][k] = (-dt) * (-ga / (12.0 * d1 * d1)) / Re;
                A[C_SS][k] = (-dt) * (-ga / (12.0 * d1 * d1)) / Re;
                A[C_EE][k] = (-dt) * (-al / (12.0 * d0 * d0)) / Re;
                A[C_WW][k] = (-dt) * (-al / (12.0 * d0 * d0)) / Re;
                A[C_NNEE][k] = (-dt) * (-be / (72.0 * d0 * d1)) / Re;
                A[C_NNWW][k] = (-dt) * (be / (72.0 * d0 * d1)) / Re;
                A[C_SSEE][k] = A[C_NNWW][k];
                A[C_SSWW][k] = A[C_NNEE][k];
                A[C_NNE][k] = (-dt) * (be / (9.0 * d0 * d1)) / Re;
                A[C_NNW][k] = (-dt) * (-be / (9.0 * d0 * d1)) / Re;
                A[C_SSE][k] = A[C_NNW][k];
                A[C_SSW][k] = A[C_NNE][k];
                A[C_NEE][k] = A[C_NNE][k];
                A[C_NWW][k] = A[C_NNW][k];
                A[C_SEE][k] = A[C_NNW][k];
                A[C_SWW][k] = A[C_NNE][k];
                A[C_P][k] = 1 + dt * (5.0 * al / (2.0 * d0 * d0) + 5.0 * ga / (2.0 * d1 * d1)) / Re;
                for (int m = 1; m < C_NCOEF; m++) B[m][k] = A[m][k] / Pr;
                B[C_P][k] = 1 + dt * (5.0 * al / (2.0 * d0 * d0) + 5.0 * ga / (2.0 * d1 * d1)) / (Re * Pr);
            }
            if (!is_cav(c)) {
                /* fold the wall-row couplings into b-vectors (PSolver.cpp:851-882) */
                if (j == 1) {
                    c->bus[i] = A[C_S][k]; c->buse[i] = A[C_SE][k]; c->busw[i] = A[C_SW][k];
                    c->bts[i] = B[C_S][k]; c->btse[i] = B[C_SE][k]; c->btsw[i] = B[C_SW][k];
                    A[C_S][k] = 0; A[C_SE][k] = 0; A[C_SW][k] = 0;
                    B[C_S][k] = 0; B[C_SE][k] = 0; B[C_SW][k] = 0;
                }
                if (j == n1 - 2) {
                    c->bun[i] = A[C_N][k]; c->bune[i] = A[C_NE][k]; c->bunw[i] = A[C_NW][k];
                    c->btn[i] = B[C_N][k]; c->btne[i] = B[C_NE][k]; c->btnw[i] = B[C_NW][k];
                    A[C_N][k] = 0; A[C_NE][k] = 0; A[C_NW][k] = 0;
                    B[C_N][k] = 0; B[C_NE][k] = 0; B[C_NW][k] = 0;
                }
                if (i == 0) {
                    for (int m = 0; m < C_NCOEF; m++) {
                        A[m][IX(n0 - 1, j)] = A[m][k];
                        B[m][IX(n0 - 1, j)] = B[m][k];
                    }
                }
            }
        }
    }
}

/* pressure 9-point assembly, PSolver.cpp:944-1040 */
static void assemble_p(orc_case* c) {
    const int n0 = c->n0, n1 = c->n1;
    const double d0 = c->d0, d1 = c->d1;
    const double *X = c->xix, *Y = c->xiy, *E = c->etx, *G = c->ety;
    for (int j = 1; j < n1 - 1; j++) {
        for (int i = ilo(c); i <= ihi(c); i++) {
            int inn, ipp, inn2, ipp2;
            nbr(c, i, &inn, &ipp, &inn2, &ipp2);
            const int jpp = j + 1, jnn = j - 1;
            const size_t k = IX(i, j);
            const size_t kE = IX(ipp, j), kW = IX(inn, j), kN = IX(i, jpp), kS = IX(i, jnn);
            double aae = (X[k] / (2.0 * d0 * d0)) * (X[k] + X[kE]);
            double bbe = (E[k] / (8.0 * d0 * d1)) * (X[kN] - X[kS]);
            double cce = (Y[k] / (2.0 * d0 * d0)) * (Y[k] + Y[kE]);
            double dde = (G[k] / (8.0 * d0 * d1)) * (Y[kN] - Y[kS]);
            c->ae[k] = aae + bbe + cce + dde;
            double aaw = (X[k] / (2.0 * d0 * d0)) * (X[k] + X[kW]);
            double bbw = (E[k] / (8.0 * d0 * d1)) * (X[kS] - X[kN]);
            double ccw = (Y[k] / (2.0 * d0 * d0)) * (Y[k] + Y[kW]);
            double ddw = (G[k] / (8.0 * d0 * d1)) * (Y[kS] - Y[kN]);
            c->aw[k] = aaw + bbw + ccw + ddw;
            double aan = (X[k] / (8.0 * d0 * d1)) * (E[kE] - E[kW]);
            double bbn = (E[k] / (2.0 * d1 * d1)) * (E[k] + E[kN]);
            double ccn = (Y[k] / (8.0 * d0 * d1)) * (G[kE] - G[kW]);
            double ddn = (G[k] / (2.0 * d1 * d1)) * (G[k] + G[kN]);
            c->an[k] = aan + bbn + ccn + ddn;
            double aas = (X[k] / (8.0 * d0 * d1)) * (E[kW] - E[kE]);
            double bbs = (E[k] / (2.0 * d1 * d1)) * (E[k] + E[kS]);
            double ccs = (Y[k] / (8.0 * d0 * d1)) * (G[kW] - G[kE]);
            double dds = (G[k] / (2.0 * d1 * d1)) * (G[k] + G[kS]);
            c->as[k] = aas + bbs + ccs + dds;
            double aane = (X[k] / (8.0 * d0 * d1)) * (E[k] + E[kE]);
            double bbne = (E[k] / (8.0 * d0 * d1)) * (X[k] + X[kN]);
            double ccne = (Y[k] / (8.0 * d0 * d1)) * (G[k] + G[kE]);
            double ddne = (G[k] / (8.0 * d0 * d1)) * (Y[k] + Y[kN]);
            c->ane[k] = aane + bbne + ccne + ddne;
            double aasw = (X[k] / (8.0 * d0 * d1)) * (E[k] + E[kW]);
            double bbsw = (E[k] / (8.0 * d0 * d1)) * (X[k] + X[kS]);
            double ccsw = (Y[k] / (8.0 * d0 * d1)) * (G[k] + G[kW]);
            double ddsw = (G[k] / (8.0 * d0 * d1)) * (Y[k] + Y[kS]);
            c->asw[k] = aasw + bbsw + ccsw + ddsw;
            double aanw = -(X[k] / (8.0 * d0 * d1)) * (E[k] + E[kW]);
            double bbnw = -(E[k] / (8.0 * d0 * d1)) * (X[k] + X[kN]);
            double ccnw = -(Y[k] / (8.0 * d0 * d1)) * (G[k] + G[kW]);
            double ddnw = -(G[k] / (8.0 * d0 * d1)) * (Y[k] + Y[kN]);
            c->anw[k] = aanw + bbnw + ccnw + ddnw;
            double aase = -(X[k] / (8.0 * d0 * d1)) * (E[k] + E[kE]);
            double bbse = -(E[k] / (8.0 * d0 * d1)) * (X[k] + X[kS]);
            double ccse = -(Y[k] / (8.0 * d0 * d1)) * (G[k] + G[kE]);
            double ddse = -(G[k] / (8.0 * d0 * d1)) * (Y[k] + Y[kS]);
            c->ase[k] = aase + bbse + ccse + ddse;
            double pxi = 1.0 / (2. * d0 * d0);
            double pet = 1.0 / (2. * d1 * d1);
            double aap = -X[k] * (2. * X[k] + X[kW] + X[kE]);
            double bbp = -E[k] * (2. * E[k] + E[kS] + E[kN]);
            double ccp = -Y[k] * (2. * Y[k] + Y[kW] + Y[kE]);
            double ddp = -G[k] * (2. * G[k] + G[kS] + G[kN]);
            c->ap[k] = aap * pxi + bbp * pet + ccp * pxi + ddp * pet;
            if (!is_cav(c) && i == 0) {
                const size_t s = IX(n0 - 1, j);
                c->ae[s] = c->ae[k]; c->aw[s] = c->aw[k]; c->an[s] = c->an[k];
                c->as[s] = c->as[k]; c->ane[s] = c->ane[k]; c->ase[s] = c->ase[k];
                c->asw[s] = c->asw[k]; c->anw[s] = c->anw[k]; c->ap[s] = c->ap[k];
            }
        }
    }
}

/* ------------------------------------------------------------------ */
/* gauss(), PSolver.cpp:2280-2446: relative-L1 stopped lexicographic GS on
 * the 9-point (near-wall) / 25-point operator. Returns the iteration count. */
static int gauss(orc_case* c, double* const* a, double* annw_plane, double* phi, const double* q) {
    const int n0 = c->n0, n1 = c->n1;
    const double tol = c->prm.tol_gs, atol = c->prm.atol_gs;
    const int maxit = c->prm.maxit_gs;
    const double *ap = a[C_P], *ae = a[C_E], *as = a[C_S], *an = a[C_N], *aw = a[C_W];
    const double *ase = a[C_SE], *asw = a[C_SW], *ane = a[C_NE], *anw = a[C_NW];
    const double *ass = a[C_SS], *assee = a[C_SSEE], *assww = a[C_SSWW], *asse = a[C_SSE];
    const double *assw = a[C_SSW], *asee = a[C_SEE], *asww = a[C_SWW], *ann = a[C_NN];
    const double *annee = a[C_NNEE], *annww = a[C_NNWW], *anne = a[C_NNE];
    const double *annw = annw_plane, *anee = a[C_NEE], *anww = a[C_NWW];
    const double *aee = a[C_EE], *aww = a[C_WW];
    double sumnor = 1.0;
    int iter;
    for (iter = 0; iter < maxit; iter++) {
        double ssum = 0.0;
        for (int pass = 0; pass < 2; pass++) {
            /* pass 0: residual + L1 sum; pass 1: in-place update */
            for (int j = 1; j < n1 - 1; j++) {
                for (int i = ilo(c); i <= ihi(c); i++) {
                    int inn, ipp, inn2, ipp2;
                    nbr(c, i, &inn, &ipp, &inn2, &ipp2);
                    const int jpp = j + 1, jpp2 = j + 2, jnn = j - 1, jnn2 = j - 2;
                    const size_t k = IX(i, j);
                    double acc;
                    if (pass == 0) acc = q[k] - ap[k] * phi[k];
                    else acc = q[k];
                    acc = acc - ae[k] * phi[IX(ipp, j)] - an[k] * phi[IX(i, jpp)] -
                          as[k] * phi[IX(i, jnn)] - aw[k] * phi[IX(inn, j)] -
                          anw[k] * phi[IX(inn, jpp)] - ane[k] * phi[IX(ipp, jpp)] -
                          asw[k] * phi[IX(inn, jnn)] - ase[k] * phi[IX(ipp, jnn)];
                    if (!near_wall(c, i, j)) {
                        acc = acc - aee[k] * phi[IX(ipp2, j)] - aww[k] * phi[IX(inn2, j)] -
                              annee[k] * phi[IX(ipp2, jpp2)] - anee[k] * phi[IX(ipp2, jpp)] -
                              asee[k] * phi[IX(ipp2, jnn)] - assee[k] * phi[IX(ipp2, jnn2)] -
                              anne[k] * phi[IX(ipp, jpp2)] - asse[k] * phi[IX(ipp, jnn2)] -
                              annw[k] * phi[IX(inn, jpp2)] - assw[k] * phi[IX(inn, jnn2)] -
                              annww[k] * phi[IX(inn2, jpp2)] - anww[k] * phi[IX(inn2, jpp)] -
                              asww[k] * phi[IX(inn2, jnn)] - assww[k] * phi[IX(inn2, jnn2)] -
                              ann[k] * phi[IX(i, jpp2)] - ass[k] * phi[IX(i, jnn2)];
                    }
                    if (pass == 0) {
                        ssum += fabs(acc);
                    } else {
                        phi[k] = acc / ap[k];
                        if (!is_cav(c) && i == 0) phi[IX(n0 - 1, j)] = phi[k];
                    }
                }
            }
            if (pass == 0) {
                if (iter == 0) sumnor = (ssum != 0.0) ? ssum : 1.0;
            }
        }
        if (ssum / sumnor < tol || ssum <= atol) { iter++; break; }
    }
    return iter;
}

/* SIP factorisation (PSolver.cpp:2091-2154); a pure function of the pressure
 * coefficients, so it is computed once and reused by every solve. */
static void sip_factor(orc_case* c) {
    const int n0 = c->n0, n1 = c->n1;
    const double alp = 0.92;
    const size_t N = (size_t)n0 * n1;
    memset(c->fbsw, 0, N * sizeof(double)); memset(c->fbn, 0, N * sizeof(double));
    memset(c->fbs, 0, N * sizeof(double)); memset(c->fbne, 0, N * sizeof(double));
    memset(c->fbe, 0, N * sizeof(double)); memset(c->fbw, 0, N * sizeof(double));
    memset(c->fbp, 0, N * sizeof(double));
    double *bsw = c->fbsw, *bw = c->fbw, *bs = c->fbs, *bp = c->fbp, *bn = c->fbn;
    double *be = c->fbe, *bne = c->fbne;
    for (int j = 1; j < n1 - 1; j++) {
        for (int i = ilo(c); i <= ihi(c); i++) {
            int inn, ipp, inn2, ipp2;
            nbr(c, i, &inn, &ipp, &inn2, &ipp2);
            const int jnn = j - 1;
            const size_t k = IX(i, j);
            bsw[k] = c->asw[k];
            bw[k] = (c->aw[k] + alp * c->anw[k] - bsw[k] * bn[IX(inn, jnn)]) /
                    (1.0 + alp * bn[IX(inn, j)]);
            bs[k] = (c->as[k] + alp * c->ase[k] - bsw[k] * be[IX(inn, jnn)]) /
                    (1.0 + alp * be[IX(i, jnn)]);
            double ad = c->anw[k] + c->ase[k] - bs[k] * be[IX(i, jnn)] - bw[k] * bn[IX(inn, j)];
            bp[k] = c->ap[k] - alp * ad - bs[k] * bn[IX(i, jnn)] - bw[k] * be[IX(inn, j)] -
                    bsw[k] * bne[IX(inn, jnn)];
            bn[k] = (c->an[k] + alp * c->anw[k] - alp * bw[k] * bn[IX(inn, j)] -
                     bw[k] * bne[IX(inn, j)]) / bp[k];
            be[k] = (c->ae[k] + alp * c->ase[k] - alp * bs[k] * be[IX(i, jnn)] -
                     bs[k] * bne[IX(i, jnn)]) / bp[k];
            bne[k] = c->ane[k] / bp[k];
            if (!is_cav(c) && i == 0) {
                const size_t s = IX(n0 - 1, j);
                bsw[s] = bsw[k]; bn[s] = bn[k]; bs[s] = bs[k]; bne[s] = bne[k];
                be[s] = be[k]; bw[s] = bw[k]; bp[s] = bp[k];
            }
        }
    }
    c->sip_factored = 1;
}

/* sip9p() iterations, PSolver.cpp:2156-2262. Returns the iteration count. */
static int sip9p(orc_case* c, double* phi, const double* q) {
    const int n0 = c->n0, n1 = c->n1;
    const size_t N = (size_t)n0 * n1;
    if (!c->sip_factored) sip_factor(c);
    const double *bsw = c->fbsw, *bw = c->fbw, *bs = c->fbs, *bp = c->fbp, *bn = c->fbn;
    const double *be = c->fbe, *bne = c->fbne;
    double *res = c->res, *qp = c->qp, *del = c->del;
    memset(qp, 0, N * sizeof(double));
    memset(del, 0, N * sizeof(double));
    const double tol = c->prm.tol_sip, atol = c->prm.atol_sip;
    double sumnor = 1.0;
    int iter;
    for (iter = 0; iter < c->prm.maxit_sip; iter++) {
        double ssum = 0.0;
        for (int j = 1; j < n1 - 1; j++) {
            for (int i = ilo(c); i <= ihi(c); i++) {
                int inn, ipp, inn2, ipp2;
                nbr(c, i, &inn, &ipp, &inn2, &ipp2);
                const int jpp = j + 1, jnn = j - 1;
                const size_t k = IX(i, j);
                res[k] = q[k] - c->ap[k] * phi[k] - c->ae[k] * phi[IX(ipp, j)] -
                         c->an[k] * phi[IX(i, jpp)] - c->as[k] * phi[IX(i, jnn)] -
                         c->aw[k] * phi[IX(inn, j)] - c->anw[k] * phi[IX(inn, jpp)] -
                         c->ane[k] * phi[IX(ipp, jpp)] - c->asw[k] * phi[IX(inn, jnn)] -
                         c->ase[k] * phi[IX(ipp, jnn)];
                ssum += fabs(res[k]);
                qp[k] = (res[k] - bs[k] * qp[IX(i, jnn)] - bw[k] * qp[IX(inn, j)] -
                         bsw[k] * qp[IX(inn, jnn)]) / bp[k];
                if (!is_cav(c) && i == 0) {
                    res[IX(n0 - 1, j)] = res[k];
                    qp[IX(n0 - 1, j)] = qp[k];
                }
            }
        }
        if (iter == 0) sumnor = (ssum != 0.0) ? ssum : 1.0;
        double sumav = ssum / sumnor;
        for (int j = n1 - 2; j >= 1; j--) {
            for (int i = ihi(c); i >= ilo(c); i--) {
                int inn, ipp, inn2, ipp2;
                nbr(c, i, &inn, &ipp, &inn2, &ipp2);
                const int jpp = j + 1;
                const size_t k = IX(i, j);
                del[k] = qp[k] - bn[k] * del[IX(i, jpp)] - be[k] * del[IX(ipp, j)] -
                         bne[k] * del[IX(ipp, jpp)];
                phi[k] = phi[k] + del[k];
                if (!is_cav(c) && i == 0) phi[IX(n0 - 1, j)] = phi[k];
            }
        }
        if (sumav < tol || ssum <= atol) { iter++; break; }
    }
    return iter;
}

/* ------------------------------------------------------------------ */
/* initial conditions and boundary conditions, PSolver.cpp:614-748 */
static void initial_state(orc_case* c) {
    const int n0 = c->n0, n1 = c->n1;
    const size_t N = (size_t)n0 * n1;
    c->loop = 1;
    c->time = 0;
    c->timed = 0.0;
    for (size_t k = 0; k < N; k++) {
        if (is_cav(c)) {
            c->u[k] = 0.0; c->v[k] = 0.0; c->T[k] = 0.0;
            c->up[k] = 0.0; c->vp[k] = 0.0;
        } else {
            c->u[k] = c->uinf; c->v[k] = c->vinf; c->T[k] = 0.0;
            c->up[k] = c->uinf; c->vp[k] = c->vinf;
        }
        c->uxi[k] = 0; c->uet[k] = 0; c->p[k] = 0; c->pcor[k] = 0; c->si[k] = 0;
    }
    if (is_cav(c)) {
        /* lid-driven unit square: u = lid_u on the lid, T = 1 bottom / 0 top,
         * adiabatic sides start at the interior value (0) */
        for (int i = 0; i < n0; i++) {
            c->u[IX(i, n1 - 1)] = c->prm.lid_u;
            c->up[IX(i, n1 - 1)] = c->prm.lid_u;
            c->T[IX(i, 0)] = 1.0;
        }
        /* the lid's end points belong to the side walls */
        c->u[IX(0, n1 - 1)] = 0.0; c->up[IX(0, n1 - 1)] = 0.0;
        c->u[IX(n0 - 1, n1 - 1)] = 0.0; c->up[IX(n0 - 1, n1 - 1)] = 0.0;
        return;
    }
    /* wall j = 0 (PSolver.cpp:698-714) */
    for (int i = 0; i < n0; i++) {
        const size_t k = IX(i, 0);
        c->u[k] = -c->speed_amp * c->y[k];
        c->v[k] = c->speed_amp * c->x[k];
        c->up[k] = c->u[k];
        c->vp[k] = c->v[k];
        c->T[k] = 1.0;
    }
    /* far field j = n1-1 (PSolver.cpp:720-748) */
    const int j = n1 - 1;
    for (int i = 0; i < n0 - 1; i++) {
        const size_t k = IX(i, j);
        double vnn = c->u[k] * c->xnox[i] + c->v[k] * c->xnoy[i];
        if (vnn >= 0) {
            c->u[k] = c->uinf; c->v[k] = c->vinf; c->T[k] = 0.0;
            c->up[k] = c->u[k]; c->vp[k] = c->v[k];
        } else {
            const size_t kb = IX(i, j - 1);
            c->u[k] = c->u[kb]; c->v[k] = c->v[kb]; c->T[k] = c->T[kb];
            if (i == 0) {
                const size_t s = IX(n0 - 1, j);
                c->u[s] = c->u[k]; c->v[s] = c->v[k]; c->T[s] = c->T[k];
            }
        }
    }
}

/* ------------------------------------------------------------------ */
/* one time step of PSolver.cpp:1058-1983 */
static void time_step(orc_case* c) {
    const int n0 = c->n0, n1 = c->n1;
    const size_t N = (size_t)n0 * n1;
    const double d0 = c->d0, d1 = c->d1, dt = c->prm.dt, Re = c->prm.Re, Pr = c->prm.Pr;
    const double Ri = c->prm.Ri, Pi = c->Pi;
    const double uinf = c->uinf, vinf = c->vinf;
    const int cav = is_cav(c);
    double* fld[3] = {c->u, c->v, c->T};

    memcpy(c->Tprev, c->T, N * sizeof(double));
    memcpy(c->uprev, c->u, N * sizeof(double));
    memcpy(c->vprev, c->v, N * sizeof(double));

    c->time = (int)((double)c->time + dt);
    c->timed = c->timed + dt;
    /* the time the wall motion sees: the reference's int (PSolver.cpp:186), or t = n dt */
    const double tw = c->prm.time_accurate ? c->timed : (double)c->time;

    /* contravariant velocities, PSolver.cpp:1063-1069 */
    for (size_t k = 0; k < N; k++) {
        c->uxi[k] = c->xix[k] * c->u[k] + c->xiy[k] * c->v[k];
        c->uet[k] = c->etx[k] * c->u[k] + c->ety[k] * c->v[k];
        c->Told[k] = c->T[k];
    }

    /* convection + predictor right-hand sides, PSolver.cpp:1075-1237 */
    for (int j = 1; j < n1 - 1; j++) {
        for (int i = ilo(c); i <= ihi(c); i++) {
            int inn, ipp, inn2, ipp2;
            nbr(c, i, &inn, &ipp, &inn2, &ipp2);
            const int jpp = j + 1, jnn = j - 1, jpp2 = j + 2, jnn2 = j - 2;
            const size_t k = IX(i, j);
            const double ux = c->uxi[k], ue = c->uet[k];
            const int near_i = cav && (i == 1 || i == n0 - 2);
            const int near_j = (j == 1 || j == n1 - 2);
            double conv[3];
            for (int m = 0; m < 3; m++) {
                const double* f = fld[m];
                double pec1, pec2;
                if (m <= 1) {
                    pec1 = ux * Re * d0 / c->alph[k];
                    pec2 = ue * Re * d1 / c->gam[k];
                } else {
                    pec1 = ux * Re * Pr * d0 / c->alph[k];
                    pec2 = ue * Re * Pr * d1 / c->gam[k];
                }
                double du_xi, du_et;
                if (near_i) {
                    du_xi = 0.5 * (f[IX(ipp, j)] - f[IX(inn, j)]) / d0;
                } else if (!near_j && pec1 <= 2 && pec1 > -2) {
                    double xpp = 8.0 * (f[IX(ipp, j)] - f[IX(inn, j)]);
                    double xnn = f[IX(ipp2, j)] - f[IX(inn2, j)];
                    du_xi = (1.0 / 12.0) * (xpp - xnn) / d0;
                } else if (!near_j) {
                    double ak1 = ux * (-f[IX(ipp2, j)] + 8 * f[IX(ipp, j)] - 8 * f[IX(inn, j)] +
                                       f[IX(inn2, j)]) / (12.0 * d0);
                    double ak2 = fabs(ux) * (f[IX(ipp2, j)] - 4 * f[IX(ipp, j)] + 6 * f[k] -
                                             4 * f[IX(inn, j)] + f[IX(inn2, j)]) / (4.0 * d0);
                    ak1 = ak1 + ak2;
                    du_xi = ak1 / ux;
                } else {
                    double xpp = 8.0 * (f[IX(ipp, j)] - f[IX(inn, j)]);
                    double xnn = f[IX(ipp2, j)] - f[IX(inn2, j)];
                    du_xi = (1.0 / 12.0) * (xpp - xnn) / d0;
                }
                if (near_j) {
                    du_et = 0.5 * (f[IX(i, jpp)] - f[IX(i, jnn)]) / d1;
                } else if (near_i || (pec2 <= 2 && pec2 > -2)) {
                    double ypp = 8.0 * (f[IX(i, jpp)] - f[IX(i, jnn)]);
                    double ynn = f[IX(i, jpp2)] - f[IX(i, jnn2)];
                    du_et = (1.0 / 12.0) * (ypp - ynn) / d1;
                } else {
                    double ak3 = ue * (-f[IX(i, jpp2)] + 8 * f[IX(i, jpp)] - 8 * f[IX(i, jnn)] +
                                       f[IX(i, jnn2)]) / (12.0 * d1);
                    double ak4 = fabs(ue) * (f[IX(i, jpp2)] - 4 * f[IX(i, jpp)] + 6 * f[k] -
                                             4 * f[IX(i, jnn)] + f[IX(i, jnn2)]) / (4.0 * d1);
                    ak3 = ak3 + ak4;
                    du_et = ak3 / ue;
                }
                conv[m] = ux * du_xi + ue * du_et;
            }
            double dp_dxi = (c->p[IX(ipp, j)] - c->p[IX(inn, j)]) / (2.0 * d0);
            double dp_de = (c->p[IX(i, jpp)] - c->p[IX(i, jnn)]) / (2.0 * d1);
            double dp_dx = c->xix[k] * dp_dxi + c->etx[k] * dp_de;
            double dp_dy = c->xiy[k] * dp_dxi + c->ety[k] * dp_de;
            c->qu[k] = dt * (-conv[0] - dp_dx) + c->u[k];
            c->qv[k] = dt * (-conv[1] - dp_dy + Ri * c->T[k]) + c->v[k];
            c->qt[k] = -dt * conv[2] + c->T[k];
            c->qup[k] = c->qu[k] + dt * dp_dx;
            c->qvp[k] = c->qv[k] + dt * dp_dy;
            if (!cav && j == 1) {
                const size_t s0 = IX(i, jnn), s1 = IX(ipp, jnn), s2 = IX(inn, jnn);
                double sumu = c->bus[i] * c->u[s0] + c->buse[i] * c->u[s1] + c->busw[i] * c->u[s2];
                c->qu[k] = c->qu[k] - sumu;
                double sumv = c->bus[i] * c->v[s0] + c->buse[i] * c->v[s1] + c->busw[i] * c->v[s2];
                c->qv[k] = c->qv[k] - sumv;
                double sumt = c->bts[i] * c->T[s0] + c->btse[i] * c->T[s1] + c->btsw[i] * c->T[s2];
                c->qt[k] = c->qt[k] - sumt;
                sumu = c->bus[i] * c->up[s0] + c->buse[i] * c->up[s1] + c->busw[i] * c->up[s2];
                c->qup[k] = c->qup[k] - sumu;
                sumv = c->bus[i] * c->vp[s0] + c->buse[i] * c->vp[s1] + c->busw[i] * c->vp[s2];
                c->qvp[k] = c->qvp[k] - sumv;
            }
            if (!cav && j == n1 - 2) {
                const size_t s0 = IX(i, jpp), s1 = IX(ipp, jpp), s2 = IX(inn, jpp);
                double sumu = c->bun[i] * c->u[s0] + c->bune[i] * c->u[s1] + c->bunw[i] * c->u[s2];
                c->qu[k] = c->qu[k] - sumu;
                double sumv = c->bun[i] * c->v[s0] + c->bune[i] * c->v[s1] + c->bunw[i] * c->v[s2];
                c->qv[k] = c->qv[k] - sumv;
                double sumt = c->btn[i] * c->T[s0] + c->btne[i] * c->T[s1] + c->btnw[i] * c->T[s2];
                c->qt[k] = c->qt[k] - sumt;
                sumu = c->bun[i] * c->up[s0] + c->bune[i] * c->up[s1] + c->bunw[i] * c->up[s2];
                c->qup[k] = c->qup[k] - sumu;
                sumv = c->bun[i] * c->vp[s0] + c->bune[i] * c->vp[s1] + c->bunw[i] * c->vp[s2];
                c->qvp[k] = c->qvp[k] - sumv;
            }
            if (!cav && i == 0) {
                const size_t s = IX(n0 - 1, j);
                c->qu[s] = c->qu[k]; c->qv[s] = c->qv[k]; c->qt[s] = c->qt[k];
                c->qup[s] = c->qup[k]; c->qvp[s] = c->qvp[k];
            }
        }
    }

    /* the five momentum / energy solves, PSolver.cpp:1241-1350 */
    double* annw_T = c->prm.fix_T_annw ? c->at[C_NNW] : c->at[C_NW];
    struct { double* rhs; double* init; double* out; int ufield; int zero_start; int it; } sv[5] = {
        {c->qu, c->u, c->us, 1, 0, D_IT_U},
        {c->qv, c->v, c->vs, 1, 0, D_IT_V},
        {c->qt, c->T, c->T, 0, 0, D_IT_T},
        {c->qup, c->up, c->up, 1, 1, D_IT_UP},
        {c->qvp, c->vp, c->vp, 1, 1, D_IT_VP},
    };
    for (int s = 0; s < 5; s++) {
        if (!sv[s].zero_start) {
            memcpy(c->sol, sv[s].init, N * sizeof(double));
        } else if (!cav) {
            /* up/vp start from zero with the wall row kept (PSolver.cpp:1304-1312) */
            for (size_t k = 0; k < N; k++) c->sol[k] = 0.0;
            for (int i = 0; i < n0; i++) c->sol[IX(i, 0)] = sv[s].init[IX(i, 0)];
        } else {
            /* cavity: zero interior start, all wall values kept */
            memcpy(c->sol, sv[s].init, N * sizeof(double));
            for (int j = 1; j < n1 - 1; j++)
                for (int i = 1; i < n0 - 1; i++) c->sol[IX(i, j)] = 0.0;
        }
        int it = gauss(c, sv[s].ufield ? c->au : c->at, sv[s].ufield ? c->au[C_NNW] : annw_T,
                       c->sol, sv[s].rhs);
        c->diag[sv[s].it] = it;
        for (int j = 1; j < n1 - 1; j++) {
            for (int i = ilo(c); i <= ihi(c); i++) {
                sv[s].out[IX(i, j)] = c->sol[IX(i, j)];
                if (!cav && i == 0) sv[s].out[IX(n0 - 1, j)] = c->sol[IX(i, j)];
            }
        }
    }

    if (!cav) {
        /* up/vp far-field condition, PSolver.cpp:1356-1382 */
        const int j = n1 - 1;
        for (int i = 0; i < n0 - 1; i++) {
            const size_t k = IX(i, j);
            double vnn = uinf * c->xnox[i] + vinf * c->xnoy[i];
            if (vnn >= 0) {
                c->up[k] = c->u[k];
                c->vp[k] = c->v[k];
            } else {
                const int jnn = j - 1;
                c->up[k] = (5.0 * c->up[IX(i, jnn)] - 4.0 * c->up[IX(i, jnn - 1)] + c->up[IX(i, jnn - 2)]) / 2.0;
                c->vp[k] = (5.0 * c->vp[IX(i, jnn)] - 4.0 * c->vp[IX(i, jnn - 1)] + c->vp[IX(i, jnn - 2)]) / 2.0;
            }
            if (i == 0) {
                c->up[IX(n0 - 1, j)] = c->up[k];
                c->vp[IX(n0 - 1, j)] = c->vp[k];
            }
        }
    }

    /* face velocities -> continuity source q, PSolver.cpp:1390-1449 */
    {
        const double *P = c->p, *U = c->up, *V = c->vp;
        const double *X = c->xix, *Y = c->xiy, *E = c->etx, *G = c->ety;
        for (int j = 1; j < n1 - 1; j++) {
            for (int i = ilo(c); i <= ihi(c); i++) {
                int inn, ipp, inn2, ipp2;
                nbr(c, i, &inn, &ipp, &inn2, &ipp2);
                const int jpp = j + 1, jnn = j - 1;
                const size_t k = IX(i, j), kE = IX(ipp, j), kW = IX(inn, j);
                const size_t kN = IX(i, jpp), kS = IX(i, jnn);
                double dpdxi_ip = (P[kE] - P[k]) / d0;
                double dpde_ip = (P[IX(ipp, jpp)] + P[kN] - P[kS] - P[IX(ipp, jnn)]) / (4.0 * d1);
                double dpdxi_in = (P[k] - P[kW]) / d0;
                double dpde_in = (P[kN] + P[IX(inn, jpp)] - P[kS] - P[IX(inn, jnn)]) / (4.0 * d1);
                double dpdxi_jp = (P[IX(ipp, jpp)] - P[IX(inn, jpp)] + P[kE] - P[kW]) / (4.0 * d0);
                double dpde_jp = (P[kN] - P[k]) / d1;
                double dpdxi_jn = (P[kE] - P[kW] + P[IX(ipp, jnn)] - P[IX(inn, jnn)]) / (4.0 * d0);
                double dpde_jn = (P[k] - P[kS]) / d1;
                double us_ip = 0.5 * (U[k] + U[kE]) - 0.5 * dt * ((X[k] + X[kE]) * dpdxi_ip + (E[k] + E[kE]) * dpde_ip);
                double us_in = 0.5 * (U[k] + U[kW]) - 0.5 * dt * ((X[k] + X[kW]) * dpdxi_in + (E[k] + E[kW]) * dpde_in);
                double us_jp = 0.5 * (U[k] + U[kN]) - 0.5 * dt * ((X[k] + X[kN]) * dpdxi_jp + (E[k] + E[kN]) * dpde_jp);
                double us_jn = 0.5 * (U[k] + U[kS]) - 0.5 * dt * ((X[k] + X[kS]) * dpdxi_jn + (E[k] + E[kS]) * dpde_jn);
                double vs_ip = 0.5 * (V[k] + V[kE]) - 0.5 * dt * ((Y[k] + Y[kE]) * dpdxi_ip + (G[k] + G[kE]) * dpde_ip);
                double vs_in = 0.5 * (V[k] + V[kW]) - 0.5 * dt * ((Y[k] + Y[kW]) * dpdxi_in + (G[k] + G[kW]) * dpde_in);
                double vs_jp = 0.5 * (V[k] + V[kN]) - 0.5 * dt * ((Y[k] + Y[kN]) * dpdxi_jp + (G[k] + G[kN]) * dpde_jp);
                double vs_jn = 0.5 * (V[k] + V[kS]) - 0.5 * dt * ((Y[k] + Y[kS]) * dpdxi_jn + (G[k] + G[kS]) * dpde_jn);
                double dusdxi = (us_ip - us_in) / d0;
                double dusde = (us_jp - us_jn) / d1;
                double dvsdxi = (vs_ip - vs_in) / d0;
                double dvsde = (vs_jp - vs_jn) / d1;
                double qq = (X[k] * dusdxi) + (E[k] * dusde) + (Y[k] * dvsdxi) + (G[k] * dvsde);
                c->q[k] = qq / dt;
            }
        }
    }
    {
        double l1 = 0.0, l2 = 0.0, mx = 0.0;
        for (int j = 1; j < n1 - 1; j++)
            for (int i = ilo(c); i <= ihi(c); i++) {
                double a = fabs(c->q[IX(i, j)]);
                l1 += a; l2 += a * a; if (a > mx) mx = a;
            }
        c->diag[D_QL1] = l1; c->diag[D_QL2] = sqrt(l2); c->diag[D_QMAX] = mx;
    }

    /* pressure correction, PSolver.cpp:1453-1466 */
    for (size_t k = 0; k < N; k++) {
        c->pcor[k] = 0;
        c->uold[k] = c->u[k];
        c->vold[k] = c->v[k];
    }
    c->diag[D_IT_SIP] = sip9p(c, c->pcor, c->q);

    /* pcor boundary conditions, PSolver.cpp:1471-1499 */
    if (!cav) {
        for (int i = 0; i < n0 - 1; i++) {
            c->pcor[IX(i, 0)] = c->pcor[IX(i, 1)];
            if (i == 0) c->pcor[IX(n0 - 1, 0)] = c->pcor[IX(i, 0)];
        }
        const int j = n1 - 1;
        for (int i = 0; i < n0 - 1; i++) {
            double vnn = uinf * c->xnox[i] + vinf * c->xnoy[i];
            c->pcor[IX(i, j)] = 0;
            if (vnn >= 0) c->pcor[IX(i, j)] = c->pcor[IX(i, j - 1)];
            if (i == 0) c->pcor[IX(n0 - 1, j)] = c->pcor[IX(i, j)];
        }
    } else {
        for (int i = 1; i < n0 - 1; i++) {
            c->pcor[IX(i, 0)] = c->pcor[IX(i, 1)];
            c->pcor[IX(i, n1 - 1)] = c->pcor[IX(i, n1 - 2)];
        }
        for (int j = 1; j < n1 - 1; j++) {
            c->pcor[IX(0, j)] = c->pcor[IX(1, j)];
            c->pcor[IX(n0 - 1, j)] = c->pcor[IX(n0 - 2, j)];
        }
        c->pcor[IX(0, 0)] = 0.5 * (c->pcor[IX(1, 0)] + c->pcor[IX(0, 1)]);
        c->pcor[IX(n0 - 1, 0)] = 0.5 * (c->pcor[IX(n0 - 2, 0)] + c->pcor[IX(n0 - 1, 1)]);
        c->pcor[IX(0, n1 - 1)] = 0.5 * (c->pcor[IX(1, n1 - 1)] + c->pcor[IX(0, n1 - 2)]);
        c->pcor[IX(n0 - 1, n1 - 1)] = 0.5 * (c->pcor[IX(n0 - 2, n1 - 1)] + c->pcor[IX(n0 - 1, n1 - 2)]);
    }

    /* velocity correction, PSolver.cpp:1505-1532 (i outer, j inner) */
    for (int i = ilo(c); i <= ihi(c); i++) {
        for (int j = 1; j < n1 - 1; j++) {
            int inn, ipp, inn2, ipp2;
            nbr(c, i, &inn, &ipp, &inn2, &ipp2);
            const int jpp = j + 1, jnn = j - 1;
            const size_t k = IX(i, j);
            double dpcor_dxi = 0.5 * (c->pcor[IX(ipp, j)] - c->pcor[IX(inn, j)]) / d0;
            double dpcor_de = 0.5 * (c->pcor[IX(i, jpp)] - c->pcor[IX(i, jnn)]) / d1;
            c->u[k] = c->us[k] - dt * (c->xix[k] * dpcor_dxi + c->etx[k] * dpcor_de);
            c->v[k] = c->vs[k] - dt * (c->xiy[k] * dpcor_dxi + c->ety[k] * dpcor_de);
            if (!cav && i == 0) {
                c->u[IX(n0 - 1, j)] = c->u[k];
                c->v[IX(n0 - 1, j)] = c->v[k];
            }
        }
    }
    /* p += pcor, PSolver.cpp:1534-1542 */
    for (int i = ilo(c); i <= ihi(c); i++) {
        for (int j = 1; j < n1 - 1; j++) {
            const size_t k = IX(i, j);
            if (c->prm.omega_p == 1.0) c->p[k] = c->p[k] + c->pcor[k];
            else c->p[k] = c->p[k] + c->prm.omega_p * c->pcor[k];
            if (!cav && i == 0) c->p[IX(n0 - 1, j)] = c->p[k];
        }
    }

    if (!cav) {
        /* vr / vth just inside the far field, PSolver.cpp:1549-1562 */
        int j = n1 - 2;
        for (int i = 0; i < n0 - 1; i++) {
            const size_t k = IX(i, j);
            double costh = c->x[k] / sqrt(c->x[k] * c->x[k] + c->y[k] * c->y[k]);
            double sinth = c->y[k] / sqrt(c->x[k] * c->x[k] + c->y[k] * c->y[k]);
            c->vr0[i] = c->u[k] * costh + c->v[k] * sinth;
            c->vth0[i] = -c->u[k] * sinth + c->v[k] * costh;
            if (i == 0) { c->vr0[n0 - 1] = c->vr0[i]; c->vth0[n0 - 1] = c->vth0[i]; }
        }
        /* circulation, PSolver.cpp:1568-1576 */
        double circ = 0.0;
        for (int i = 0; i < n0 - 1; i++) {
            double de = c->prm.fix_circ_de ? 1.0 / (n0 - 1) : 1.0 / (n0 - 2);
            const size_t k = IX(i, j), kp = IX(i + 1, j);
            double f1 = (c->u[k] * c->ety[k] - c->v[k] * c->etx[k]) * fabs(c->jac[k]);
            double f2 = (c->u[kp] * c->ety[kp] - c->v[kp] * c->etx[kp]) * fabs(c->jac[kp]);
            circ = circ + de * 0.5 * (f1 + f2);
        }
        c->diag[D_CIRC] = circ;
        /* far-field prediction, PSolver.cpp:1582-1609 */
        j = n1 - 1;
        for (int i = 0; i < n0 - 1; i++) {
            const double eps = 1e-2;
            const size_t k = IX(i, j), kb = IX(i, j - 1);
            double cr = sqrt(c->x[kb] * c->x[kb] + c->y[kb] * c->y[kb]) /
                        sqrt(c->x[k] * c->x[k] + c->y[k] * c->y[k]);
            double costh = c->x[k] / sqrt(c->x[k] * c->x[k] + c->y[k] * c->y[k]);
            double sinth = c->y[k] / sqrt(c->x[k] * c->x[k] + c->y[k] * c->y[k]);
            double vrinf = uinf * costh + vinf * sinth;
            double vtinf = -uinf * sinth + vinf * costh;
            int kk = fabs(circ) > eps ? 1 : 2;
            double cr2 = pow(cr, 2), crk = pow(cr, kk);
            c->vr1[i] = c->vr0[i] * cr2 + vrinf * (1 - cr2);
            c->vth1[i] = c->vth0[i] * crk + vtinf * (1 - crk);
            if (i == 0) { c->vr1[n0 - 1] = c->vr1[i]; c->vth1[n0 - 1] = c->vth1[i]; }
        }
        /* wall velocity, PSolver.cpp:1617-1630 */
        for (int i = 0; i < n0; i++) {
            const size_t k = IX(i, 0);
            c->u[k] = -c->speed_amp * cos(2.0 * Pi * c->prm.F * tw) * c->y[k];
            c->up[k] = c->u[k];
            c->v[k] = c->speed_amp * cos(2.0 * Pi * c->prm.F * tw) * c->x[k];
            c->vp[k] = c->v[k];
        }
        /* far-field u/v/T, PSolver.cpp:1632-1656 */
        for (int i = 0; i < n0 - 1; i++) {
            const size_t k = IX(i, j);
            double vnn = uinf * c->xnox[i] + vinf * c->xnoy[i];
            if (vnn >= 0) {
                c->u[k] = uinf; c->v[k] = vinf; c->T[k] = 0.0;
            } else {
                double costh = c->x[k] / sqrt(c->x[k] * c->x[k] + c->y[k] * c->y[k]);
                double sinth = c->y[k] / sqrt(c->x[k] * c->x[k] + c->y[k] * c->y[k]);
                c->u[k] = costh * c->vr1[i] - sinth * c->vth1[i];
                c->v[k] = sinth * c->vr1[i] + costh * c->vth1[i];
                c->T[k] = c->Told[k] - (c->uet[k] * dt / d1) * (c->Told[k] - c->Told[IX(i, j - 1)]);
            }
            if (i == 0) {
                const size_t s = IX(n0 - 1, j), z = IX(0, j);
                c->u[s] = c->u[z]; c->v[s] = c->v[z]; c->T[s] = c->T[z];
            }
        }
    } else {
        /* cavity: walls are static, only the adiabatic T walls move */
        for (int j = 1; j < n1 - 1; j++) {
            c->T[IX(0, j)] = (4.0 * c->T[IX(1, j)] - c->T[IX(2, j)]) / 3.0;
            c->T[IX(n0 - 1, j)] = (4.0 * c->T[IX(n0 - 2, j)] - c->T[IX(n0 - 3, j)]) / 3.0;
        }
    }

    /* contravariant velocities from the updated field, PSolver.cpp:1668-1673 */
    for (size_t k = 0; k < N; k++) {
        c->uxi[k] = c->xix[k] * c->u[k] + c->xiy[k] * c->v[k];
        c->uet[k] = c->etx[k] * c->u[k] + c->ety[k] * c->v[k];
    }

    if (!cav) {
        /* wall pressure from the normal momentum equation, PSolver.cpp:1677-1729 */
        double dp_dx = 0.0, dp_dy = 0.0;
        int j = 0;
        for (int i = 0; i < n0 - 1; i++) {
            for (int m = 0; m < 2; m++) {
                const double* f = fld[m];
                int ipp = i + 1, inn = (i == 0) ? n0 - 2 : i - 1;
                const int jpp = j + 1, jpp2 = j + 2;
                const size_t k = IX(i, j);
                double aa = c->alph[k] * (f[IX(ipp, j)] + f[IX(inn, j)] - 2 * f[k]) / (d0 * d0);
                double gg = c->gam[k] * (f[IX(i, jpp + 1)] + f[k] - 2 * f[IX(i, jpp)]) / (d1 * d1);
                double bb = c->beta[k] * (f[IX(ipp, jpp)] + f[IX(inn, j)] - f[IX(inn, jpp)] - f[IX(ipp, j)]) /
                            (2 * d0 * d1);
                (void)jpp2;
                double d2u = aa + gg - 2 * bb + 0.0;
                double cv = c->uxi[k] * 0.5 * (f[IX(ipp, j)] - f[IX(inn, j)]) / d0;
                cv = cv + c->uet[k] * (f[IX(i, jpp)] - f[k]) / d1;
                double alc;
                if (m == 0) alc = c->accn_amp * sin(2.0 * Pi * c->prm.F * tw) * c->y[k];
                else alc = -c->accn_amp * sin(2.0 * Pi * c->prm.F * tw) * c->x[k];
                if (m == 0) dp_dx = 1.0 * d2u / Re - cv - alc;
                if (m == 1) dp_dy = 1.0 * d2u / Re - cv - alc + Ri * c->T[k];
            }
            const size_t k = IX(i, j);
            c->p[k] = c->p[IX(i, j + 1)] - (dp_dx * (-c->xiy[k] * c->jac[k]) + dp_dy * (c->xix[k] * c->jac[k])) * d1;
            if (i == 0) c->p[IX(n0 - 1, j)] = c->p[k];
        }
        /* far-field pressure: momentum equation at inflow, Gresho at outflow,
         * PSolver.cpp:1733-1783 */
        j = n1 - 1;
        for (int i = 0; i < n0 - 1; i++) {
            double vnn = uinf * c->xnox[i] + vinf * c->xnoy[i];
            const size_t k = IX(i, j);
            if (vnn >= 0) {
                for (int m = 0; m < 2; m++) {
                    const double* f = fld[m];
                    const double* fo = (m == 0) ? c->uold : c->vold;
                    int ipp = i + 1, inn = i - 1;
                    if (i == 0) inn = n0 - 2;
                    const int jnn = j - 1, jnn2 = j - 2;
                    double aa = c->alph[k] * (f[IX(ipp, j)] + f[IX(inn, j)] - 2 * f[k]) / (d0 * d0);
                    double gg = c->gam[k] * (f[k] + f[IX(i, jnn - 1)] - 2 * f[IX(i, jnn)]) / (d1 * d1);
                    double bb = c->beta[k] * (f[IX(ipp, j)] + f[IX(inn, jnn)] - f[IX(ipp, jnn)] - f[IX(inn, j)]) /
                                (2 * d0 * d1);
                    double d2u = aa + gg - 2 * bb + 0.0;
                    double cv = c->uxi[k] * 0.5 * (f[IX(ipp, j)] - f[IX(inn, j)]) / d0;
                    cv = cv + c->uet[k] * (3.0 * f[k] - 4 * f[IX(i, jnn)] + f[IX(i, jnn2)]) / (2 * d1);
                    double alc = (f[k] - fo[k]) / dt;
                    if (m == 0) dp_dx = 1.0 * d2u / Re - cv - alc;
                    if (m == 1) dp_dy = 1.0 * d2u / Re - cv - alc + Ri * c->T[k];
                }
                c->p[k] = c->p[IX(i, j - 1)] + (dp_dx * (-c->xiy[k] * c->jac[k]) + dp_dy * (c->xix[k] * c->jac[k])) * d1;
            } else {
                c->p[k] = 0.5 * (1.0 / Re) * ((3 * c->uet[k] - 4 * c->uet[IX(i, j - 1)] + c->uet[IX(i, j - 2)]) / d1);
            }
            if (i == 0) c->p[IX(n0 - 1, j)] = c->p[k];
        }
    } else {
        /* cavity: zero normal pressure gradient on every wall, corners averaged */
        for (int i = 1; i < n0 - 1; i++) {
            c->p[IX(i, 0)] = c->p[IX(i, 1)];
            c->p[IX(i, n1 - 1)] = c->p[IX(i, n1 - 2)];
        }
        for (int j = 1; j < n1 - 1; j++) {
            c->p[IX(0, j)] = c->p[IX(1, j)];
            c->p[IX(n0 - 1, j)] = c->p[IX(n0 - 2, j)];
        }
        c->p[IX(0, 0)] = 0.5 * (c->p[IX(1, 0)] + c->p[IX(0, 1)]);
        c->p[IX(n0 - 1, 0)] = 0.5 * (c->p[IX(n0 - 2, 0)] + c->p[IX(n0 - 1, 1)]);
        c->p[IX(0, n1 - 1)] = 0.5 * (c->p[IX(1, n1 - 1)] + c->p[IX(0, n1 - 2)]);
        c->p[IX(n0 - 1, n1 - 1)] = 0.5 * (c->p[IX(n0 - 2, n1 - 1)] + c->p[IX(n0 - 1, n1 - 2)]);
    }

    /* stream function, PSolver.cpp:1789-1801 */
    for (int i = 0; i < n0; i++) c->si[IX(i, 0)] = 0;
    for (int i = 0; i < n0; i++) {
        for (int j = 1; j < n1; j++) {
            const size_t k = IX(i, j), kb = IX(i, j - 1);
            double ca = (c->xix[k] * c->u[k] * fabs(c->jac[k]) + c->xix[kb] * c->u[kb] * fabs(c->jac[kb]));
            double cb = (c->xiy[k] * c->v[k] * fabs(c->jac[k]) + c->xiy[kb] * c->v[kb] * fabs(c->jac[kb]));
            c->si[k] = c->si[kb] + (ca + cb) * 0.5 * d1;
        }
    }

    /* dilatation, vorticity and dmax, PSolver.cpp:1807-1853 */
    double dmax = 0.0;
    for (int i = ilo(c); i <= ihi(c); i++) {
        for (int j = 1; j < n1 - 1; j++) {
            int inn, ipp, inn2, ipp2;
            nbr(c, i, &inn, &ipp, &inn2, &ipp2);
            const int jpp = j + 1, jnn = j - 1;
            const size_t k = IX(i, j);
            const double *U = c->u, *V = c->v;
            c->dil[k] = c->xix[k] * (U[IX(ipp, j)] - U[IX(inn, j)]) / (2 * d0) +
                        c->etx[k] * (U[IX(i, jpp)] - U[IX(i, jnn)]) / (2 * d1) +
                        c->ety[k] * (V[IX(i, jpp)] - V[IX(i, jnn)]) / (2 * d1) +
                        c->xiy[k] * (V[IX(ipp, j)] - V[IX(inn, j)]) / (2 * d0);
            double dv_dxi = 0.5 / d0 * (V[IX(ipp, j)] - V[IX(inn, j)]);
            double dv_det = 0.5 / d1 * (V[IX(i, jpp)] - V[IX(i, jnn)]);
            double dv_dx = c->xix[k] * dv_dxi + c->etx[k] * dv_det;
            double du_dxi = 0.5 / d0 * (U[IX(ipp, j)] - U[IX(inn, j)]);
            double du_det = 0.5 / d1 * (U[IX(i, jpp)] - U[IX(i, jnn)]);
            double du_dy = c->xiy[k] * du_dxi + c->ety[k] * du_det;
            c->vort[k] = dv_dx - du_dy;
            if (!cav && i == 0) {
                c->dil[IX(n0 - 1, j)] = c->dil[k];
                c->vort[IX(n0 - 1, j)] = c->vort[k];
            }
            if (c->dil[k] > dmax) dmax = c->dil[k];
        }
    }
    /* wall / far-field vorticity, PSolver.cpp:1855-1888 */
    for (int j = 0; j < n1; j += n1 - 1) {
        for (int i = ilo(c); i <= ihi(c); i++) {
            int inn, ipp, inn2, ipp2;
            nbr(c, i, &inn, &ipp, &inn2, &ipp2);
            const int jpp = j + 1, jnn = j - 1;
            const size_t k = IX(i, j);
            const double *U = c->u, *V = c->v;
            double dv_dxi = 0.5 / d0 * (V[IX(ipp, j)] - V[IX(inn, j)]);
            double dv_det = (j == 0) ? 1.0 / d1 * (V[IX(i, jpp)] - V[k]) : 1.0 / d1 * (V[k] - V[IX(i, jnn)]);
            double dv_dx = c->xix[k] * dv_dxi + c->etx[k] * dv_det;
            double du_dxi = 0.5 / d0 * (U[IX(ipp, j)] - U[IX(inn, j)]);
            double du_det = (j == 0) ? 1.0 / d1 * (U[IX(i, jpp)] - U[k]) : 1.0 / d1 * (U[k] - U[IX(i, jnn)]);
            double du_dy = c->xiy[k] * du_dxi + c->ety[k] * du_det;
            c->vort[k] = dv_dx - du_dy;
            if (!cav && i == 0) c->vort[IX(n0 - 1, j)] = c->vort[k];
        }
    }
    c->diag[D_DMAX] = dmax;

    /* forces, moment and Nusselt number on j = 0, PSolver.cpp:1901-1983 */
    {
        const int j = 0;
        const double sa = sin(c->prm.alpha_deg * Pi / 180.0), ca_ = cos(c->prm.alpha_deg * Pi / 180.0);
        double pr_x = 0.0, pr_y = 0.0, vor_x = 0.0, vor_y = 0.0;
        double press_i = 0.0, vor_i = 0.0, temp_i = 0.0;
        const int i0 = 0, i1 = n0 - 2;
        for (int i = i0; i <= i1; i++) {
            const size_t k = IX(i, j), kp = IX(i + 1, j);
            double PJ1 = c->p[k] * c->jac[k], pj2 = c->p[kp] * c->jac[kp];
            double VJ1 = c->vort[k] * c->jac[k], VJ2 = c->vort[kp] * c->jac[kp];
            double fp1_x = PJ1 * c->etx[k], fp2_x = pj2 * c->etx[kp];
            double fp1_y = PJ1 * c->ety[k], fp2_y = pj2 * c->ety[kp];
            double fv1_x = VJ1 * c->ety[k], fv2_x = VJ2 * c->ety[kp];
            double fv1_y = VJ1 * c->etx[k], fv2_y = VJ2 * c->etx[kp];
            pr_x = pr_x + 0.5 * d0 * (fp1_x + fp2_x);
            pr_y = pr_y + 0.5 * d0 * (fp1_y + fp2_y);
            vor_x = vor_x + 0.5 * d0 * (fv1_x + fv2_x);
            vor_y = vor_y + 0.5 * d0 * (fv1_y + fv2_y);
        }
        double cx = 2 * pr_x + (2.0 / Re) * vor_x;
        double cy = 2 * pr_y - (2.0 / Re) * vor_y;
        c->diag[D_CLP] = 2 * pr_y * sa - 2 * pr_x * ca_;
        c->diag[D_CDP] = 2 * pr_y * ca_ + 2 * pr_x * sa;
        c->diag[D_CLV] = -(2.0 / Re) * vor_y * sa - (2.0 / Re) * vor_x * ca_;
        c->diag[D_CDV] = -(2.0 / Re) * vor_y * ca_ + (2.0 / Re) * vor_x * sa;
        c->diag[D_CL] = cy * sa - cx * ca_;
        c->diag[D_CD] = cy * ca_ + cx * sa;
        for (int i = i0; i <= i1; i++) {
            const size_t k = IX(i, j), kp = IX(i + 1, j);
            double PJ1 = c->p[k] * c->jac[k], pj2 = c->p[kp] * c->jac[kp];
            double VJ1 = c->vort[k] * c->jac[k], VJ2 = c->vort[kp] * c->jac[kp];
            double TJ1 = c->jac[k] * (c->etx[k] * c->etx[k] + c->ety[k] * c->ety[k]);
            double TJ2 = c->jac[kp] * (c->etx[kp] * c->etx[kp] + c->ety[kp] * c->ety[kp]);
            double fp1 = PJ1 * (c->x[k] * c->ety[k] - c->y[k] * c->etx[k]);
            double fp2 = pj2 * (c->x[kp] * c->ety[kp] - c->y[kp] * c->etx[kp]);
            double fv1 = VJ1 * (c->x[k] * c->etx[k] + c->y[k] * c->ety[k]);
            double fv2 = VJ2 * (c->x[kp] * c->etx[kp] + c->y[kp] * c->ety[kp]);
            double fh1 = TJ1 * (4 * c->T[IX(i, j + 1)] - 3 * c->T[k] - c->T[IX(i, j + 2)]) / (2 * d1);
            double fh2 = TJ2 * (4 * c->T[IX(i + 1, j + 1)] - 3 * c->T[kp] - c->T[IX(i + 1, j + 2)]) / (2 * d1);
            press_i = press_i + 0.5 * d0 * (fp1 + fp2);
            vor_i = vor_i + 0.5 * d0 * (fv1 + fv2);
            temp_i = temp_i + 0.5 * (fh1 + fh2) * d0;
        }
        c->diag[D_CM] = 2 * press_i - (2.0 / Re) * vor_i;
        const double ar = c->ar;
        if (!cav)
            c->diag[D_NU] = (2 * temp_i) / (Pi * (3 * (1 + (1.0 / ar)) - sqrt((3 + (1.0 / ar)) * ((3.0 / ar) + 1))));
        else
            c->diag[D_NU] = -temp_i; /* wall length 1, right-handed grid (J > 0) */
    }

    /* residual diagnostics (not in the reference) */
    {
        double dtl1 = 0.0, dtmx = 0.0, dul1 = 0.0;
        for (int j = 1; j < n1 - 1; j++)
            for (int i = ilo(c); i <= ihi(c); i++) {
                const size_t k = IX(i, j);
                double a = fabs(c->T[k] - c->Tprev[k]);
                dtl1 += a; if (a > dtmx) dtmx = a;
                dul1 += fabs(c->u[k] - c->uprev[k]) + fabs(c->v[k] - c->vprev[k]);
            }
        c->diag[D_DTL1] = dtl1; c->diag[D_DTMAX] = dtmx; c->diag[D_DUL1] = dul1;
    }
}

/* ------------------------------------------------------------------ */
/* C ABI of the oracle (ctypes) */

orc_case* orc_create(int n0, int n1, double dxi0, double dxi1, double ar,
                     const double* planes, const double* normals, const orc_params* prm) {
    if (n0 < 7 || n1 < 6 || !planes || !normals || !prm) return NULL;
    orc_case* c = (orc_case*)calloc(1, sizeof(orc_case));
    c->n0 = n0; c->n1 = n1; c->d0 = dxi0; c->d1 = dxi1; c->ar = ar;
    c->prm = *prm;
    c->Pi = acos(-1.0);
    c->thetamax = c->Pi / 12.0;
    c->speed_amp = c->thetamax * 2.0 * c->Pi * prm->F;
    c->accn_amp = 2.0 * c->Pi * prm->F * c->speed_amp;
    c->uinf = sin(prm->alpha_deg * c->Pi / 180.0);
    c->vinf = cos(prm->alpha_deg * c->Pi / 180.0);
    const size_t N = (size_t)n0 * n1;
    double** g[] = {&c->x, &c->y, &c->xix, &c->xiy, &c->etx, &c->ety, &c->alph, &c->beta, &c->gam, &c->jac};
    for (int m = 0; m < 10; m++) {
        *g[m] = plane(c);
        memcpy(*g[m], planes + (size_t)m * N, N * sizeof(double));
    }
    double** nv[] = {&c->xnix, &c->xniy, &c->xnox, &c->xnoy,
                     &c->bus, &c->buse, &c->busw, &c->bts, &c->btse, &c->btsw,
                     &c->bun, &c->bune, &c->bunw, &c->btn, &c->btne, &c->btnw,
                     &c->vr0, &c->vr1, &c->vth0, &c->vth1};
    for (int m = 0; m < 20; m++) *nv[m] = (double*)calloc((size_t)n0, sizeof(double));
    for (int m = 0; m < 4; m++) memcpy(*nv[m], normals + (size_t)m * n0, n0 * sizeof(double));
    double** st[] = {&c->u, &c->v, &c->T, &c->p, &c->up, &c->vp, &c->us, &c->vs, &c->uold,
                     &c->vold, &c->Told, &c->pcor, &c->q, &c->qu, &c->qv, &c->qt, &c->qup,
                     &c->qvp, &c->sol, &c->uxi, &c->uet, &c->si, &c->dil, &c->vort,
                     &c->ap, &c->ae, &c->aw, &c->an, &c->as, &c->ane, &c->anw, &c->ase, &c->asw,
                     &c->fbe, &c->fbw, &c->fbs, &c->fbn, &c->fbne, &c->fbsw, &c->fbp, &c->res,
                     &c->qp, &c->del, &c->Tprev, &c->uprev, &c->vprev};
    for (size_t m = 0; m < sizeof(st) / sizeof(st[0]); m++) *st[m] = plane(c);
    for (int m = 0; m < C_NCOEF; m++) { c->au[m] = plane(c); c->at[m] = plane(c); }
    initial_state(c);
    c->loop = 0; /* timeLoop counts from 0 (PSolver.cpp:1058) */
    assemble_uvT(c);
    assemble_p(c);
    return c;
}

void orc_destroy(orc_case* c) {
    if (!c) return;
    double* all[] = {c->x, c->y, c->xix, c->xiy, c->etx, c->ety, c->alph, c->beta, c->gam, c->jac,
                     c->xnix, c->xniy, c->xnox, c->xnoy, c->bus, c->buse, c->busw, c->bts,
                     c->btse, c->btsw, c->bun, c->bune, c->bunw, c->btn, c->btne, c->btnw,
                     c->vr0, c->vr1, c->vth0, c->vth1, c->u, c->v, c->T, c->p, c->up, c->vp,
                     c->us, c->vs, c->uold, c->vold, c->Told, c->pcor, c->q, c->qu, c->qv,
                     c->qt, c->qup, c->qvp, c->sol, c->uxi, c->uet, c->si, c->dil, c->vort,
                     c->ap, c->ae, c->aw, c->an, c->as, c->ane, c->anw, c->ase, c->asw, c->fbe,
                     c->fbw, c->fbs, c->fbn, c->fbne, c->fbsw, c->fbp, c->res, c->qp, c->del,
                     c->Tprev, c->uprev, c->vprev};
    for (size_t m = 0; m < sizeof(all) / sizeof(all[0]); m++) free(all[m]);
    for (int m = 0; m < C_NCOEF; m++) { free(c->au[m]); free(c->at[m]); }
    free(c);
}

/* advance nsteps; if hist != NULL it receives nsteps*D_COUNT records */
int orc_step(orc_case* c, int nsteps, double* hist) {
    for (int s = 0; s < nsteps; s++) {
        time_step(c);
        c->diag[D_LOOP] = c->loop;
        c->diag[D_TIME] = c->prm.time_accurate ? c->timed : (double)c->time;
        c->loop++;
        if (hist) memcpy(hist + (size_t)s * D_COUNT, c->diag, D_COUNT * sizeof(double));
    }
    return 0;
}

int orc_diag_count(void) { return D_COUNT; }

/* pointer to an internal plane (n1*n0) or vector (n0) by name, NULL if unknown */
double* orc_field(orc_case* c, const char* name) {
    struct { const char* n; double* p; } t[] = {
        {"u", c->u}, {"v", c->v}, {"T", c->T}, {"p", c->p}, {"up", c->up}, {"vp", c->vp},
        {"us", c->us}, {"vs", c->vs}, {"pcor", c->pcor}, {"q", c->q}, {"qu", c->qu},
        {"qv", c->qv}, {"qt", c->qt}, {"qup", c->qup}, {"qvp", c->qvp}, {"si", c->si},
        {"dil", c->dil}, {"vort", c->vort}, {"uxi", c->uxi}, {"uet", c->uet},
        {"ap", c->ap}, {"ae", c->ae}, {"aw", c->aw}, {"an", c->an}, {"as", c->as},
        {"ane", c->ane}, {"anw", c->anw}, {"ase", c->ase}, {"asw", c->asw},
        {"bus", c->bus}, {"buse", c->buse}, {"busw", c->busw}, {"bun", c->bun},
        {"bune", c->bune}, {"bunw", c->bunw}, {"bts", c->bts}, {"btse", c->btse},
        {"btsw", c->btsw}, {"btn", c->btn}, {"btne", c->btne}, {"btnw", c->btnw},
    };
    for (size_t m = 0; m < sizeof(t) / sizeof(t[0]); m++)
        if (strcmp(t[m].n, name) == 0) return t[m].p;
    static const char* cn[C_NCOEF] = {"p", "e", "w", "n", "s", "ne", "nw", "se", "sw", "ee", "ww",
                                      "nn", "ss", "nnee", "nnww", "ssee", "ssww", "nne", "nnw",
                                      "sse", "ssw", "nee", "nww", "see", "sww"};
    if (name[0] == 'a' && (name[1] == 'u' || name[1] == 't')) {
        for (int m = 0; m < C_NCOEF; m++)
            if (strcmp(name + 2, cn[m]) == 0) return name[1] == 'u' ? c->au[m] : c->at[m];
    }
    return NULL;
}
