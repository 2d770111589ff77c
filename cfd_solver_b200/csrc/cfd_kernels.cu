// cfd_kernels.cu -- sm_100a kernels of one projection time step, batched over a case table.
//
// Reference mapping (mhsuhail00/CFD_Solver, PSolver.cpp):
//   k_assemble_p     pressure 9-point stencil            PSolver.cpp:944-1040
//   k_rhs            contravariant velocities,           PSolver.cpp:1063-1069
//                    convection + predictor RHS          PSolver.cpp:1075-1237
//   k_sweep_*        the five gauss() systems            PSolver.cpp:1241-1350, 2280-2446
//   (cfd_sweep.cu)   (u/v/T coefficients assembled in     PSolver.cpp:752-940
//                     shared memory from alpha, beta, gamma; k_sweep_fin, k_mom_fix,
//                     k_mom_update finish each sweep / solve)
//   k_upbc           up/vp far-field condition           PSolver.cpp:1356-1382
//   k_face_q         face velocities -> continuity q     PSolver.cpp:1390-1449
//   k_bicg_* / k_mg_*  pressure correction (replaces      PSolver.cpp:1453-1466, 2067-2278
//                    sip9p): BiCGStab on the stored 9-point stencil, preconditioned by a
//                    Galerkin multigrid V-cycle with multicolour Gauss-Seidel smoothing
//   k_correct        pcor BCs + velocity / p correction  PSolver.cpp:1471-1542
//   k_bc             far-field / wall BCs, circulation,  PSolver.cpp:1549-1783
//                    boundary pressure, wall integrals   PSolver.cpp:1901-1983
//   k_diag           dilatation, vorticity, dmax         PSolver.cpp:1807-1853
//   k_si             stream function (output only)       PSolver.cpp:1789-1801
#include <type_traits>

#include "cfd_common.cuh"
#include "cfd_reduce.cuh"
#include "cfd_kernels.cuh"
#include "cfd_bulk.cuh"

namespace cfd {

#define AT(ptr, ii, jj) (ptr)[(long long)(jj) * ld + (ii)]

constexpr int JTW = TX + 4;   // 32 x 16 tile columns incl. a 2-cell halo
constexpr int JTH = TYJ + 4;  // 32 x 16 tile rows incl. a 2-cell halo

// plane that holds the final multigrid V-cycle result of level l of case c (x on the
// case's coarsest level; otherwise fixed by the numbers of pre- and post-sweeps)
__device__ __forceinline__ int mg_result_plane(const BatchDev& b, const CaseDev& c, int l) {
    return l == c.nlev - 1 ? M_X : b.mg_res;
}

__device__ __forceinline__ bool near_wall(const CaseDev& c, int i, int j) {
    if (j == 1 || j == c.n1 - 2) return true;
    return c.profile == CAVITY && (i == 1 || i == c.n0 - 2);
}

// ---------------------------------------------------------------------------
// The 9-point pressure stencil at one cell (PSolver.cpp:944-1040) from the four metric
// planes X = xi_x, Y = xi_y, E = eta_x, G = eta_y at the cell and its four neighbours,
// in the order ap, ae, aw, an, as, ane, anw, ase, asw. c1 = 1 / (2 dxi0^2), c2 = 1 / (8 dxi0
// dxi1), c3 = 1 / (2 dxi1^2) (the reference divides by these; multiplying by reciprocals
// moves each coefficient by at most a unit in the last place). The stencil is stored
// once (k_assemble_p): rebuilding it inside the SpMV was measured slower (about 100 FP64
// operations per cell against 40 bytes saved).
template <typename T>
struct P9In {
    T x, xe, xw, xn, xs, y, ye, yw, yn, ys, e, ee, ew, en, es, g, ge, gw, gn, gs;
};

template <typename T>
__device__ __forceinline__ void p9_coefs(const P9In<T>& m, T c1, T c2, T c3, T (&a)[9]) {
    const T X = m.x, Y = m.y, E = m.e, G = m.g;
    a[1] = (X * c1) * (X + m.xe) + (E * c2) * (m.xn - m.xs) + (Y * c1) * (Y + m.ye) + (G * c2) * (m.yn - m.ys);
    a[2] = (X * c1) * (X + m.xw) + (E * c2) * (m.xs - m.xn) + (Y * c1) * (Y + m.yw) + (G * c2) * (m.ys - m.yn);
    a[3] = (X * c2) * (m.ee - m.ew) + (E * c3) * (E + m.en) + (Y * c2) * (m.ge - m.gw) + (G * c3) * (G + m.gn);
    a[4] = (X * c2) * (m.ew - m.ee) + (E * c3) * (E + m.es) + (Y * c2) * (m.gw - m.ge) + (G * c3) * (G + m.gs);
    a[5] = (X * c2) * (E + m.ee) + (E * c2) * (X + m.xn) + (Y * c2) * (G + m.ge) + (G * c2) * (Y + m.yn);
    a[8] = (X * c2) * (E + m.ew) + (E * c2) * (X + m.xs) + (Y * c2) * (G + m.gw) + (G * c2) * (Y + m.ys);
    a[6] = -((X * c2) * (E + m.ew)) - (E * c2) * (X + m.xn) - (Y * c2) * (G + m.gw) - (G * c2) * (Y + m.yn);
    a[7] = -((X * c2) * (E + m.ee)) - (E * c2) * (X + m.xs) - (Y * c2) * (G + m.ge) - (G * c2) * (Y + m.ys);
    a[0] = (-X * (T(2) * X + m.xw + m.xe)) * c1 + (-E * (T(2) * E + m.es + m.en)) * c3 +
           (-Y * (T(2) * Y + m.yw + m.ye)) * c1 + (-G * (T(2) * G + m.gs + m.gn)) * c3;
}

// the metrics around flat index k of planes X, Y, E, G with row pitch ld
template <typename T, typename S>
__device__ __forceinline__ P9In<T> p9_load(const S* X, const S* Y, const S* E, const S* G, long long k, int ld) {
    P9In<T> m;
    m.x = X[k]; m.xe = X[k + 1]; m.xw = X[k - 1]; m.xn = X[k + ld]; m.xs = X[k - ld];
    m.y = Y[k]; m.ye = Y[k + 1]; m.yw = Y[k - 1]; m.yn = Y[k + ld]; m.ys = Y[k - ld];
    m.e = E[k]; m.ee = E[k + 1]; m.ew = E[k - 1]; m.en = E[k + ld]; m.es = E[k - ld];
    m.g = G[k]; m.ge = G[k + 1]; m.gw = G[k - 1]; m.gn = G[k + ld]; m.gs = G[k - ld];
    return m;
}

// pressure stencil assembly, also the set-up of multigrid level 0 (stencil and the FP32
// metric copies its matrix-free sweeps read)
__global__ void __launch_bounds__(NT) k_assemble_p(BatchDev b, int toff) {
    const Tile t = b.ftiles[toff + blockIdx.x];
    const CaseDev& c = b.cases[t.c];
    const int i = t.i0 + (int)(threadIdx.x % TX), j = t.j0 + (int)(threadIdx.x / TX);
    if (i < c.ilo || i > c.ihi || j > c.n1 - 2) return;
    const int ld = c.ld, W = c.W, per = c.periodic;
    const long long k = (long long)j * ld + i;
    const P9In<double> m = p9_load<double>(plane(b, c, P_XIX), plane(b, c, P_XIY), plane(b, c, P_ETX),
                                           plane(b, c, P_ETY), k, ld);
    double vals[9];
    p9_coefs<double>(m, c.pc1, c.pc2, c.pc3, vals);
    const LevelDev& L0 = c.lev[0];
    const int ld0 = L0.ld;
#pragma unroll
    for (int q = 0; q < 9; q++) {
        store_mirrored(plane(b, c, P_AP + q), ld, i, j, W, per, vals[q]);
        store_mirrored(mplane(b, L0, M_AP + q), ld0, i, j, W, per, (float)vals[q]);
    }
}

// ---------------------------------------------------------------------------
// u/v/T operator coefficients, PSolver.cpp:765-849, computed in registers
struct Coef25 {
    double p, e, w, n, s, ne, nw, se, sw;
    double ee, ww, nn, ss, nnee, nnww, ssee, ssww, nne, nnw, sse, ssw, nee, nww, see, sww;
};

__device__ __forceinline__ void build_coefs(const CaseDev& c, double al, double be, double ga,
                                            bool nearw, int j, Coef25& A, Coef25& T) {
    const double d0 = c.d0, d1 = c.d1, dt = c.dt, Re = c.Re, Pr = c.Pr;
    if (nearw) {
        A.e = A.w = -dt * (al / (d0 * d0)) / Re;
        A.n = A.s = -dt * (ga / (d1 * d1)) / Re;
        A.ne = A.sw = dt * be / (2.0 * d0 * d1 * Re);
        A.nw = A.se = -dt * be / (2.0 * d0 * d1 * Re);
        A.p = 1 + dt * 2.0 * (al / (d0 * d0) + ga / (d1 * d1)) / Re;
        T.e = T.w = -dt * (al / (d0 * d0)) / (Re * Pr);
        T.n = T.s = -dt * (ga / (d1 * d1)) / (Re * Pr);
        T.ne = T.sw = dt * (be / (2.0 * d0 * d1)) / (Re * Pr);
        T.nw = T.se = -dt * (be / (2.0 * d0 * d1)) / (Re * Pr);
        T.p = 1 + dt * 2.0 * (al / (d0 * d0) + ga / (d1 * d1)) / (Re * Pr);
        if (c.profile == OGRID) {
            // wall-row couplings are folded into the right-hand side (PSolver.cpp:851-882)
            if (j == 1) { A.s = A.se = A.sw = 0.0; T.s = T.se = T.sw = 0.0; }
            if (j == c.n1 - 2) { A.n = A.ne = A.nw = 0.0; T.n = T.ne = T.nw = 0.0; }
        }
        A.ee = A.ww = A.nn = A.ss = A.nnee = A.nnww = A.ssee = A.ssww = 0.0;
        A.nne = A.nnw = A.sse = A.ssw = A.nee = A.nww = A.see = A.sww = 0.0;
        T.ee = T.ww = T.nn = T.ss = T.nnee = T.nnww = T.ssee = T.ssww = 0.0;
        T.nne = T.nnw = T.sse = T.ssw = T.nee = T.nww = T.see = T.sww = 0.0;
    } else {
        A.e = A.w = (-dt) * ((4.0 * al) / (3.0 * d0 * d0)) / Re;
        A.n = A.s = (-dt) * ((4.0 * ga) / (3.0 * d1 * d1)) / Re;
        A.ne = A.sw = (-dt) * (-8.0 * be / (9.0 * d0 * d1)) / Re;
        A.nw = A.se = (-dt) * (8.0 * be / (9.0 * d0 * d1)) / Re;
        A.nn = A.ss = (-dt) * (-ga / (12.0 * d1 * d1)) / Re;
        A.ee = A.ww = (-dt) * (-al / (12.0 * d0 * d0)) / Re;
        A.nnee = A.ssww = (-dt) * (-be / (72.0 * d0 * d1)) / Re;
        A.nnww = A.ssee = (-dt) * (be / (72.0 * d0 * d1)) / Re;
        A.nne = A.ssw = A.nee = A.sww = (-dt) * (be / (9.0 * d0 * d1)) / Re;
        A.nnw = A.sse = A.nww = A.see = (-dt) * (-be / (9.0 * d0 * d1)) / Re;
        A.p = 1 + dt * (5.0 * al / (2.0 * d0 * d0) + 5.0 * ga / (2.0 * d1 * d1)) / Re;
        T.e = A.e / Pr; T.w = A.w / Pr; T.n = A.n / Pr; T.s = A.s / Pr;
        T.ne = A.ne / Pr; T.nw = A.nw / Pr; T.se = A.se / Pr; T.sw = A.sw / Pr;
        T.nn = A.nn / Pr; T.ss = A.ss / Pr; T.ee = A.ee / Pr; T.ww = A.ww / Pr;
        T.nnee = A.nnee / Pr; T.nnww = A.nnww / Pr; T.ssee = A.ssee / Pr; T.ssww = A.ssww / Pr;
        T.nne = A.nne / Pr; T.nnw = A.nnw / Pr; T.sse = A.sse / Pr; T.ssw = A.ssw / Pr;
        T.nee = A.nee / Pr; T.nww = A.nww / Pr; T.see = A.see / Pr; T.sww = A.sww / Pr;
        T.p = 1 + dt * (5.0 * al / (2.0 * d0 * d0) + 5.0 * ga / (2.0 * d1 * d1)) / (Re * Pr);
        // the reference's T solve passes atnw in the annw slot (PSolver.cpp:1290)
        if (!c.fix_T_annw) T.nnw = T.nw;
    }
}

// sum of the off-centre couplings, in the order of gauss() (PSolver.cpp:2408-2425)
__device__ __forceinline__ double offsum(const double* F, long long k, int ld, const Coef25& a, bool nearw) {
    double s = a.e * F[k + 1] + a.n * F[k + ld] + a.s * F[k - ld] + a.w * F[k - 1] +
               a.nw * F[k + ld - 1] + a.ne * F[k + ld + 1] + a.sw * F[k - ld - 1] + a.se * F[k - ld + 1];
    if (!nearw) {
        const long long l2 = 2LL * ld;
        s += a.ee * F[k + 2] + a.ww * F[k - 2] + a.nnee * F[k + l2 + 2] + a.nee * F[k + ld + 2] +
             a.see * F[k - ld + 2] + a.ssee * F[k - l2 + 2] + a.nne * F[k + l2 + 1] +
             a.sse * F[k - l2 + 1] + a.nnw * F[k + l2 - 1] + a.ssw * F[k - l2 - 1] +
             a.nnww * F[k + l2 - 2] + a.nww * F[k + ld - 2] + a.sww * F[k - ld - 2] +
             a.ssww * F[k - l2 - 2] + a.nn * F[k + l2] + a.ss * F[k - l2];
    }
    return s;
}

// ---------------------------------------------------------------------------
// contravariant velocities + convection + the five right-hand sides
// (PSolver.cpp:1063-1237); also seeds the five solves' iterates. A CTA owns a 32 x 16 tile
// (two cells per thread); u, v, T, p, up, vp with a 2-cell halo and the seven metric
// planes of the tile arrive by tensor TMA into shared memory.
constexpr int RHS_HALO = 6, RHS_INT = 7;
constexpr size_t RHS_SMEM = (size_t)(RHS_HALO * JTW * JTH + RHS_INT * TX * TYJ) * sizeof(double) + 128;
const size_t kRhsSmem = RHS_SMEM;

// One convective term ux df/dxi + ue df/deta of field F at tile offset o
// (PSolver.cpp:1110-1180): 4th-order central differences when the cell Peclet number is in
// (-2, 2] (and always in the rows / columns next to a wall, where the reference uses
// 2nd-order central), otherwise 3rd-order upwind. The reference forms du = (ux D1 +
// |ux| D4) / ux and multiplies by ux again; here the product is formed directly, and every
// division by a grid spacing is a multiplication by its reciprocal.
__device__ __forceinline__ double conv_one(const double* F, int o, bool near_i, bool near_j, double ux,
                                           double ue, bool cen_i, bool cen_j, double rd0, double rd1) {
    constexpr int R = JTW;
    const double fc = F[o], fe = F[o + 1], fw = F[o - 1];
    const double fn = F[o + R], fs = F[o - R];
    double cx, cy;
    if (near_i) {
        cx = ux * (0.5 * (fe - fw) * rd0);
    } else {
        const double fee = F[o + 2], fww = F[o - 2];
        if (near_j || cen_i) {
            cx = ux * ((1.0 / 12.0) * (8.0 * (fe - fw) - (fee - fww)) * rd0);
        } else {
            cx = (ux * ((1.0 / 12.0) * (-fee + 8.0 * fe - 8.0 * fw + fww)) +
                  fabs(ux) * (0.25 * (fee - 4.0 * fe + 6.0 * fc - 4.0 * fw + fww))) * rd0;
        }
    }
    if (near_j) {
        cy = ue * (0.5 * (fn - fs) * rd1);
    } else {
        const double fnn = F[o + 2 * R], fss = F[o - 2 * R];
        if (near_i || cen_j) {
            cy = ue * ((1.0 / 12.0) * (8.0 * (fn - fs) - (fnn - fss)) * rd1);
        } else {
            cy = (ue * ((1.0 / 12.0) * (-fnn + 8.0 * fn - 8.0 * fs + fss)) +
                  fabs(ue) * (0.25 * (fnn - 4.0 * fn + 6.0 * fc - 4.0 * fs + fss))) * rd1;
        }
    }
    return cx + cy;
}

// Three CTAs per SM (80 registers, 36 bytes of spills; the 63 KB staged per CTA fits three
// times): while one CTA computes, two others' copies are in flight. Two CTAs per SM at 122
// registers left the SM idle between a CTA's copies and its arithmetic (431 vs 373 us per
// step on the 256-case twin sweep).
__global__ void __launch_bounds__(NT, 3) k_rhs(BatchDev b) {
    extern __shared__ __align__(128) unsigned char rraw[];
    __shared__ __align__(8) uint64_t bar;
    double* sm = reinterpret_cast<double*>((reinterpret_cast<uintptr_t>(rraw) + 127) & ~uintptr_t(127));
    const Tile t = b.jtiles[blockIdx.x];
    const CaseDev& c = b.cases[t.c];
    const int tid = threadIdx.x;
    const int cur = b.cur, nxt = cur ^ 1;
    // halo tiles: u, v, T, p, up, vp; interior tiles: xix, xiy, etx, ety, alpha, gamma, beta
    double* SI = sm + RHS_HALO * JTW * JTH;
    const bool active = b.iscal[(long long)t.c * NISCAL + I_ACTIVE] != 0;
    if (tid == 0 && t.k == 0) {
        int* is = b.iscal + (long long)t.c * NISCAL;
        int word = active ? (1 << NFIELD) - 1 : 0;
        for (int f = 0; f < NFIELD; f++) {
            is[I_MDONE0 + f] = active ? 0 : 1;
            is[I_MIT0 + f] = 0;
            is[I_MODD0 + f] = 0;
            is[I_MFLIP0 + f] = b.mixed ? 0 : is[I_MNEXT0 + f];
            word |= (is[I_MFLIP0 + f] != 0) << (NFIELD + f);
        }
        is[I_MWORD] = word;
        if (active) atomicAdd(b.mactive, NFIELD);
        else is[I_PDONE] = 1;  // an empty slot takes no part in the step
    }
    if (tid == 0) {  // the sweep kernel's word for this tile (I_MWORD of the case)
        int word = active ? (1 << NFIELD) - 1 : 0;
        if (active && !b.mixed)
            for (int f = 0; f < NFIELD; f++)
                word |= (b.iscal[(long long)t.c * NISCAL + I_MNEXT0 + f] != 0) << (NFIELD + f);
        b.tword[blockIdx.x] = word;
    }
    if (!active) return;
    if (tid == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
        const char* maps = b.tmaps + (size_t)t.c * TMAP_STRIDE;
        mbar_arrive_expect_tx(&bar, (RHS_HALO * JTW * JTH + RHS_INT * TX * TYJ) * sizeof(double));
        const int hp[RHS_HALO] = {P_U, P_V, P_T0 + cur, P_P, P_UP0 + cur, P_VP0 + cur};
        const int ip[RHS_INT] = {P_XIX, P_XIY, P_ETX, P_ETY, P_ALPH, P_GAM, P_BETA};
        for (int m = 0; m < RHS_HALO; m++) tma_load_3d(sm + m * JTW * JTH, maps, t.i0, t.j0 - 2, hp[m], &bar);
        for (int m = 0; m < RHS_INT; m++) tma_load_3d(SI + m * TX * TYJ, maps + 128, t.i0 + 2, t.j0, ip[m], &bar);
    }
    // the case's constants and planes, loaded while the copies are in flight
    const int ld = c.ld, W = c.W, per = c.periodic, n1 = c.n1, n0 = c.n0, ilo = c.ilo, ihi = c.ihi;
    const bool cav = c.profile == CAVITY;
    const double d0 = c.d0, d1 = c.d1, dt = c.dt, Re = c.Re, Pr = c.Pr, Ri = c.Ri;
    const double rd0 = 1.0 / d0, rd1 = 1.0 / d1;
    double* const fb = b.f64 + c.base + H;  // plane 0 of the case; plane k at fb + k * ps
    const long long ps = c.ps;
    const bool warm = c.warm_up != 0;
    int nextm = 0;  // fields whose first iterate goes into the scratch plane (FP64 form)
    if (!b.mixed)
        for (int f = 0; f < NFIELD; f++) nextm |= (b.iscal[(long long)t.c * NISCAL + I_MNEXT0 + f] != 0) << f;
    __syncthreads();
    const bool ok = __syncthreads_and(mbar_wait_bounded(&bar, 0, b.wait_polls));
    if (!ok) {
        if (tid == 0) {
            atomicExch(b.error, 1);
            mbar_wait_bounded(&bar, 0);  // the copies land before the CTA leaves
        }
        return;
    }
    const double *Us = sm, *Vs = sm + JTW * JTH, *Ts = sm + 2 * JTW * JTH, *Ps = sm + 3 * JTW * JTH,
                 *UPs = sm + 4 * JTW * JTH, *VPs = sm + 5 * JTW * JTH;
    const double* U = fb + P_U * ps;
    const double* V = fb + P_V * ps;
    const double* T = fb + (P_T0 + cur) * ps;
    const double* UP = fb + (P_UP0 + cur) * ps;
    const double* VP = fb + (P_VP0 + cur) * ps;
    // iterate buffers of field f: A (the solution) and B (the Jacobi scratch)
    auto Ap = [&](int f) { return fb + (f < 2 ? P_US + f : P_T0 + 2 * (f - 2) + nxt) * ps; };
    auto Bp = [&](int f) { return fb + (P_BU + f) * ps; };
    const int li = tid % TX, lj = tid / TX;
    const int i = t.i0 + li;
#pragma unroll 1
    for (int h = 0; h < 2; h++) {
        const int j = t.j0 + lj + h * TY;
        if (i < ilo || i > ihi || j > n1 - 2) continue;
        const int o = (lj + h * TY + 2) * JTW + (li + 2);
        const int oi = (lj + h * TY) * TX + li;
        const long long k = (long long)j * ld + i;
        const double xix = SI[oi], xiy = SI[TX * TYJ + oi], etx = SI[2 * TX * TYJ + oi], ety = SI[3 * TX * TYJ + oi];
        const double al = SI[4 * TX * TYJ + oi], ga = SI[5 * TX * TYJ + oi];
        const double uc = Us[o], vc = Vs[o], tc = Ts[o];
        const double ux = xix * uc + xiy * vc;
        const double ue = etx * uc + ety * vc;
        const bool near_j = (j == 1 || j == n1 - 2);
        const bool near_i = cav && (i == 1 || i == n0 - 2);
        // cell Peclet numbers ux Re dxi / alpha, ue Re deta / gamma (x Pr for T)
        const double pu1 = ux * (Re * d0) / al, pu2 = ue * (Re * d1) / ga;
        const double pt1 = pu1 * Pr, pt2 = pu2 * Pr;
        const bool cu1 = pu1 <= 2 && pu1 > -2, cu2 = pu2 <= 2 && pu2 > -2;
        const bool ct1 = pt1 <= 2 && pt1 > -2, ct2 = pt2 <= 2 && pt2 > -2;
        const double cv0 = conv_one(Us, o, near_i, near_j, ux, ue, cu1, cu2, rd0, rd1);
        const double cv1 = conv_one(Vs, o, near_i, near_j, ux, ue, cu1, cu2, rd0, rd1);
        const double cv2 = conv_one(Ts, o, near_i, near_j, ux, ue, ct1, ct2, rd0, rd1);
        const double dp_dxi = (Ps[o + 1] - Ps[o - 1]) * (0.5 * rd0);
        const double dp_de = (Ps[o + JTW] - Ps[o - JTW]) * (0.5 * rd1);
        const double dp_dx = xix * dp_dxi + etx * dp_de;
        const double dp_dy = xiy * dp_dxi + ety * dp_de;
        double qu = dt * (-cv0 - dp_dx) + uc;
        double qv = dt * (-cv1 - dp_dy + Ri * tc) + vc;
        double qt = -dt * cv2 + tc;
        double qup = qu + dt * dp_dx;
        double qvp = qv + dt * dp_dy;
        if (!cav && near_j) {
            // folded wall-row couplings (PSolver.cpp:1195-1227)
            const double be = SI[6 * TX * TYJ + oi];
            const double bs = -dt * (ga / (d1 * d1)) / Re;
            const double bpos = dt * be / (2.0 * d0 * d1 * Re);
            const double bneg = -dt * be / (2.0 * d0 * d1 * Re);
            const double ts = -dt * (ga / (d1 * d1)) / (Re * Pr);
            const double tpos = dt * (be / (2.0 * d0 * d1)) / (Re * Pr);
            const double tneg = -dt * (be / (2.0 * d0 * d1)) / (Re * Pr);
            int s0, s1, s2;
            double c1, c2, t1, t2;
            if (j == 1) {  // bus, buse (= ause), busw (= ausw)
                s0 = o - JTW; s1 = o - JTW + 1; s2 = o - JTW - 1;
                c1 = bneg; c2 = bpos; t1 = tneg; t2 = tpos;
            } else {       // bun, bune (= aune), bunw (= aunw)
                s0 = o + JTW; s1 = o + JTW + 1; s2 = o + JTW - 1;
                c1 = bpos; c2 = bneg; t1 = tpos; t2 = tneg;
            }
            double sumu = bs * Us[s0] + c1 * Us[s1] + c2 * Us[s2];
            qu = qu - sumu;
            double sumv = bs * Vs[s0] + c1 * Vs[s1] + c2 * Vs[s2];
            qv = qv - sumv;
            double sumt = ts * Ts[s0] + t1 * Ts[s1] + t2 * Ts[s2];
            qt = qt - sumt;
            sumu = bs * UPs[s0] + c1 * UPs[s1] + c2 * UPs[s2];
            qup = qup - sumu;
            sumv = bs * VPs[s0] + c1 * VPs[s1] + c2 * VPs[s2];
            qvp = qvp - sumv;
        }
        fb[P_RU * ps + k] = qu;
        fb[P_RV * ps + k] = qv;
        fb[P_RT * ps + k] = qt;
        fb[P_RUP * ps + k] = qup;
        fb[P_RVP * ps + k] = qvp;
        // seed the iterates (PSolver.cpp:1241-1337): u*, v*, T from the current fields;
        // up/vp from the previous solution (warm start) or zero. A solve predicted to stop
        // after an odd number of sweeps starts in the scratch plane, so that its result
        // ends in the iterate plane (the prediction is the previous step's parity; FP64 form)
        auto X0 = [&](int f) { return ((nextm >> f) & 1) ? Bp(f) : Ap(f); };
        store_mirrored(X0(F_U), ld, i, j, W, per, uc);
        store_mirrored(X0(F_V), ld, i, j, W, per, vc);
        store_mirrored(X0(F_T), ld, i, j, W, per, tc);
        store_mirrored(X0(F_UP), ld, i, j, W, per, warm ? UPs[o] : 0.0);
        store_mirrored(X0(F_VP), ld, i, j, W, per, warm ? VPs[o] : 0.0);
        // boundary values the stencils read (both iterate buffers)
        auto put_bnd = [&](int bi, int bj) {
            const long long kb = (long long)bj * ld + bi;
            const bool zero_far = !cav && bj == n1 - 1;  // up/vp solves see zero on the far row
#pragma unroll 1
            for (int f = 0; f < NFIELD; f++) {
                const double* src = f == F_U ? U : f == F_V ? V : f == F_T ? T : f == F_UP ? UP : VP;
                const double val = (zero_far && f >= F_UP) ? 0.0 : src[kb];
                store_mirrored(Ap(f), ld, bi, bj, W, per, val);
                store_mirrored(Bp(f), ld, bi, bj, W, per, val);
            }
        };
        if (j == 1) put_bnd(i, 0);
        if (j == n1 - 2) put_bnd(i, n1 - 1);
        if (cav) {
            if (i == 1) {
                put_bnd(0, j);
                if (j == 1) put_bnd(0, 0);
                if (j == n1 - 2) put_bnd(0, n1 - 1);
            }
            if (i == n0 - 2) {
                put_bnd(n0 - 1, j);
                if (j == 1) put_bnd(n0 - 1, 0);
                if (j == n1 - 2) put_bnd(n0 - 1, n1 - 1);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// up/vp far-field condition (PSolver.cpp:1356-1382), one CTA per O-grid case
__global__ void __launch_bounds__(BC_THREADS) k_upbc(BatchDev b) {
    const CaseDev& c = b.cases[blockIdx.x];
    if (c.profile != OGRID || !b.iscal[(long long)blockIdx.x * NISCAL + I_ACTIVE]) return;
    const int ld = c.ld, j = c.n1 - 1, nxt = b.cur ^ 1;
    double* UP = plane(b, c, P_UP0 + nxt);
    double* VP = plane(b, c, P_VP0 + nxt);
    const double* U = plane(b, c, P_U);
    const double* V = plane(b, c, P_V);
    const double* VEC = plane(b, c, P_VEC);
    for (int i = threadIdx.x; i < c.W; i += blockDim.x) {
        const double vnn = c.uinf * VEC[2LL * ld + i] + c.vinf * VEC[3LL * ld + i];
        const long long k = (long long)j * ld + i;
        double a, bb;
        if (vnn >= 0) {
            a = U[k];
            bb = V[k];
        } else {
            a = (5.0 * UP[k - ld] - 4.0 * UP[k - 2LL * ld] + UP[k - 3LL * ld]) / 2.0;
            bb = (5.0 * VP[k - ld] - 4.0 * VP[k - 2LL * ld] + VP[k - 3LL * ld]) / 2.0;
        }
        store_mirrored(UP, ld, i, j, c.W, 1, a);
        store_mirrored(VP, ld, i, j, c.W, 1, bb);
    }
}

// ---------------------------------------------------------------------------
// face velocities -> continuity source q (PSolver.cpp:1390-1449) with the
// mass-residual reductions; seeds the BiCGStab residual. 32 x 16 tiles, two cells per
// thread; p, up, vp and the four metric planes with their halo arrive by tensor TMA.
constexpr int FQ_HALO = 7;
constexpr size_t FQ_SMEM = (size_t)FQ_HALO * JTW * JTH * sizeof(double) + 128;
const size_t kFaceQSmem = FQ_SMEM;

__global__ void __launch_bounds__(NT, 4) k_face_q(BatchDev b) {
    extern __shared__ __align__(128) unsigned char fraw[];
    __shared__ __align__(8) uint64_t bar;
    double* sm = reinterpret_cast<double*>((reinterpret_cast<uintptr_t>(fraw) + 127) & ~uintptr_t(127));
    const Tile t = b.jtiles[blockIdx.x];
    const CaseDev& c = b.cases[t.c];
    const int tid = threadIdx.x;
    const int nxt = b.cur ^ 1;
    if (!b.iscal[(long long)t.c * NISCAL + I_ACTIVE]) return;  // uniform over the case
    if (tid == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
        const char* maps = b.tmaps + (size_t)t.c * TMAP_STRIDE;
        mbar_arrive_expect_tx(&bar, FQ_HALO * JTW * JTH * sizeof(double));
        const int hp[FQ_HALO] = {P_P, P_UP0 + nxt, P_VP0 + nxt, P_XIX, P_XIY, P_ETX, P_ETY};
        for (int m = 0; m < FQ_HALO; m++) tma_load_3d(sm + m * JTW * JTH, maps, t.i0, t.j0 - 2, hp[m], &bar);
    }
    // the case's constants and output planes, loaded while the copies are in flight
    const int ld = c.ld, ilo = c.ilo, ihi = c.ihi, n1 = c.n1, ld0 = c.lev[0].ld;
    double* QP = plane(b, c, P_Q);
    double* KRP = plane(b, c, P_KR);
    float* B0 = mplane(b, c.lev[0], M_B);
    // reciprocals once per thread: the per-cell quotients become products (each within an
    // ulp of the quotient; 1 / (4 d) is 0.25 / d exactly)
    const double dt = c.dt, rd0 = 1.0 / c.d0, rd1 = 1.0 / c.d1, q0 = 0.25 * rd0, q1 = 0.25 * rd1;
    const double hdt = 0.5 * dt, rdt = 1.0 / dt;
    __syncthreads();
    const bool ok = __syncthreads_and(mbar_wait_bounded(&bar, 0, b.wait_polls));
    if (!ok) {
        if (tid == 0) {
            atomicExch(b.error, 1);
            mbar_wait_bounded(&bar, 0);  // the copies land before the CTA leaves
        }
        return;
    }
    const double *P = sm, *U = sm + JTW * JTH, *V = sm + 2 * JTW * JTH, *X = sm + 3 * JTW * JTH,
                 *Y = sm + 4 * JTW * JTH, *E = sm + 5 * JTW * JTH, *G = sm + 6 * JTW * JTH;
    const int li = tid % TX, lj = tid / TX;
    const int i = t.i0 + li;
    double red[3] = {0.0, 0.0, 0.0};
    for (int h = 0; h < 2; h++) {
        const int j = t.j0 + lj + h * TY;
        if (!ok || i < ilo || i > ihi || j > n1 - 2) continue;
        const int k = (lj + h * TY + 2) * JTW + (li + 2);
        const int kE = k + 1, kW = k - 1, kN = k + JTW, kS = k - JTW;
        double dpdxi_ip = (P[kE] - P[k]) * rd0;
        double dpde_ip = (P[kN + 1] + P[kN] - P[kS] - P[kS + 1]) * q1;
        double dpdxi_in = (P[k] - P[kW]) * rd0;
        double dpde_in = (P[kN] + P[kN - 1] - P[kS] - P[kS - 1]) * q1;
        double dpdxi_jp = (P[kN + 1] - P[kN - 1] + P[kE] - P[kW]) * q0;
        double dpde_jp = (P[kN] - P[k]) * rd1;
        double dpdxi_jn = (P[kE] - P[kW] + P[kS + 1] - P[kS - 1]) * q0;
        double dpde_jn = (P[k] - P[kS]) * rd1;
        double us_ip = 0.5 * (U[k] + U[kE]) - hdt * ((X[k] + X[kE]) * dpdxi_ip + (E[k] + E[kE]) * dpde_ip);
        double us_in = 0.5 * (U[k] + U[kW]) - hdt * ((X[k] + X[kW]) * dpdxi_in + (E[k] + E[kW]) * dpde_in);
        double us_jp = 0.5 * (U[k] + U[kN]) - hdt * ((X[k] + X[kN]) * dpdxi_jp + (E[k] + E[kN]) * dpde_jp);
        double us_jn = 0.5 * (U[k] + U[kS]) - hdt * ((X[k] + X[kS]) * dpdxi_jn + (E[k] + E[kS]) * dpde_jn);
        double vs_ip = 0.5 * (V[k] + V[kE]) - hdt * ((Y[k] + Y[kE]) * dpdxi_ip + (G[k] + G[kE]) * dpde_ip);
        double vs_in = 0.5 * (V[k] + V[kW]) - hdt * ((Y[k] + Y[kW]) * dpdxi_in + (G[k] + G[kW]) * dpde_in);
        double vs_jp = 0.5 * (V[k] + V[kN]) - hdt * ((Y[k] + Y[kN]) * dpdxi_jp + (G[k] + G[kN]) * dpde_jp);
        double vs_jn = 0.5 * (V[k] + V[kS]) - hdt * ((Y[k] + Y[kS]) * dpdxi_jn + (G[k] + G[kS]) * dpde_jn);
        double dusdxi = (us_ip - us_in) * rd0;
        double dusde = (us_jp - us_jn) * rd1;
        double dvsdxi = (vs_ip - vs_in) * rd0;
        double dvsde = (vs_jp - vs_jn) * rd1;
        double qq = (X[k] * dusdxi) + (E[k] * dusde) + (Y[k] * dvsdxi) + (G[k] * dvsde);
        const double q = qq * rdt;
        // q doubles as BiCGStab's shadow residual r_hat; p, v and the iterate pcor are
        // initialised by the first iteration's kernels (beta = 0, x = 0)
        const long long kg = (long long)j * ld + i;
        QP[kg] = q;
        KRP[kg] = q;
        // the first iteration's p = r_0 = q, as the preconditioner's right-hand side (k_bicg_p
        // has nothing to do in the first iteration; the second reads p_1 from the q plane)
        B0[(long long)j * ld0 + i] = (float)q;
        red[0] += fabs(q);
        red[1] += q * q;
        red[2] = fmax(red[2], fabs(q));
    }
    if (case_reduce<3, 0x4u>(b, t.c, blockIdx.x, c.jt_begin, c.jt_count, red) && tid == 0) {
        double* sc = b.scal + (long long)t.c * NSCAL;
        int* is = b.iscal + (long long)t.c * NISCAL;
        sc[S_QL1] = red[0];
        sc[S_QL2] = sqrt(red[1]);
        if (is[I_NSTEP] == 0) sc[S_QL2_0] = sqrt(red[1]);
        sc[S_QMAX] = red[2];
        sc[S_RHO] = red[1];
        sc[S_ALPHA] = 1.0;
        sc[S_OMEGA] = 1.0;
        sc[S_BETA] = 0.0;
        sc[S_NB1] = red[0];
        sc[S_RL1] = red[0];
        is[I_PIT] = 0;
        // this step's solver status starts with the momentum / energy solves: a field still
        // iterating when their loop ended stopped at the sweep cap
        is[I_PSTATUS] = (is[I_MWORD] & ((1 << NFIELD) - 1)) ? ST_MAXITER : 0;
        if (red[0] == 0.0 || !isfinite(red[0])) {
            is[I_PDONE] = 1;
            if (!isfinite(red[0])) is[I_STATUS] |= ST_NAN;
        } else {
            is[I_PDONE] = 0;
            atomicAdd(b.active, 1);
        }
    }
}

// ---------------------------------------------------------------------------
// BiCGStab, right-preconditioned, FP64 vectors; per-case scalars live on the device
// The BiCGStab kernels run on the 32 x 16 tiles, two cells per thread (rows lj and
// lj + 8), every load of both cells issued before the arithmetic.
__global__ void __launch_bounds__(NT, 3) k_bicg_p(BatchDev b) {
    const Tile t = b.jtiles[blockIdx.x];
    if (b.iscal[(long long)t.c * NISCAL + I_PDONE]) return;
    // p_{k+1} = r_k + beta (p_k - omega v_k), launched at the end of iteration k (after
    // k_bicg_x has counted it and formed beta). p_1 = r_0 = q is k_face_q's, written as the
    // preconditioner's right-hand side, so after the first iteration p_1 is read from the q
    // plane. Before any iteration (it == 0) there is nothing to do.
    const int it = b.iscal[(long long)t.c * NISCAL + I_PIT];
    if (it == 0) return;
    const CaseDev& c = b.cases[t.c];
    const int i = t.i0 + (int)(threadIdx.x % TX), j0 = t.j0 + (int)(threadIdx.x / TX);
    const double* sc = b.scal + (long long)t.c * NSCAL;
    const double beta = sc[S_BETA], omega = sc[S_OMEGA];
    double* Pv = plane(b, c, P_KP);
    const double* Pold = it == 1 ? plane(b, c, P_Q) : Pv;
    const double* R = plane(b, c, P_KR);
    const double* Vv = plane(b, c, P_KV);
    const LevelDev& L = c.lev[0];
    bool in[2];
    long long k[2];
    double r[2], po[2], v[2];
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const int j = j0 + h * TY;
        in[h] = i >= c.ilo && i <= c.ihi && j <= c.n1 - 2;
        k[h] = in[h] ? (long long)j * c.ld + i : (long long)c.ld + c.ilo;
        r[h] = R[k[h]];
        po[h] = Pold[k[h]];
        v[h] = Vv[k[h]];
    }
#pragma unroll
    for (int h = 0; h < 2; h++) {
        if (!in[h]) continue;
        const int j = j0 + h * TY;
        const double p = r[h] + beta * (po[h] - omega * v[h]);
        Pv[k[h]] = p;
        mplane(b, L, M_B)[(long long)j * L.ld + i] = (float)p;
        store_mirrored(mplane(b, L, M_X), L.ld, i, j, L.W, c.periodic, 0.0f);
    }
}

// y = A * x with x = (double) MG level-0 result; mode 0: p_hat, v, (r_hat, v) -> alpha
//                                               mode 1: s_hat, t, (t, s), (t, t) -> omega
__global__ void __launch_bounds__(NT, 5) k_spmv(BatchDev b, int mode) {
    const Tile t = b.jtiles[blockIdx.x];
    if (b.iscal[(long long)t.c * NISCAL + I_PDONE]) return;
    const CaseDev& c = b.cases[t.c];
    const int i = t.i0 + (int)(threadIdx.x % TX), j0 = t.j0 + (int)(threadIdx.x / TX);
    const int ld = c.ld;
    const LevelDev& L = c.lev[0];
    const int l0 = L.ld;
    const float* X = mplane(b, L, mg_result_plane(b, c, 0));
    const double* DOT = plane(b, c, mode == 0 ? P_Q : P_KS);
    bool in[2];
    long long k[2];
    double y[2], xc[2], dv[2];
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const int j = j0 + h * TY;
        in[h] = i >= c.ilo && i <= c.ihi && j <= c.n1 - 2;
        const int jj = in[h] ? j : 1, ii = in[h] ? i : c.ilo;
        const long long kk = (long long)jj * ld + ii, q = (long long)jj * l0 + ii;
        k[h] = kk;
        xc[h] = (double)X[q];
        y[h] = plane(b, c, P_AP)[kk] * xc[h] + plane(b, c, P_AE)[kk] * (double)X[q + 1] +
               plane(b, c, P_AW)[kk] * (double)X[q - 1] + plane(b, c, P_AN)[kk] * (double)X[q + l0] +
               plane(b, c, P_AS)[kk] * (double)X[q - l0] + plane(b, c, P_ANE)[kk] * (double)X[q + l0 + 1] +
               plane(b, c, P_ANW)[kk] * (double)X[q + l0 - 1] + plane(b, c, P_ASE)[kk] * (double)X[q - l0 + 1] +
               plane(b, c, P_ASW)[kk] * (double)X[q - l0 - 1];
        dv[h] = DOT[kk];
    }
    double red[2] = {0.0, 0.0};
#pragma unroll
    for (int h = 0; h < 2; h++) {
        if (!in[h]) continue;
        if (mode == 0) {
            plane(b, c, P_KPH)[k[h]] = xc[h];
            plane(b, c, P_KV)[k[h]] = y[h];
            red[0] += dv[h] * y[h];
        } else {
            plane(b, c, P_KSH)[k[h]] = xc[h];
            plane(b, c, P_KT)[k[h]] = y[h];
            red[0] += y[h] * dv[h];
            red[1] += y[h] * y[h];
        }
    }
    if (case_reduce<2, 0u>(b, t.c, blockIdx.x, c.jt_begin, c.jt_count, red) && threadIdx.x == 0) {
        double* sc = b.scal + (long long)t.c * NSCAL;
        int* is = b.iscal + (long long)t.c * NISCAL;
        if (mode == 0) {
            if (red[0] == 0.0 || !isfinite(red[0])) {
                is[I_PSTATUS] |= ST_BREAKDOWN;
                is[I_PDONE] = 1;
                atomicSub(b.active, 1);
            } else {
                sc[S_ALPHA] = sc[S_RHO] / red[0];
            }
        } else {
            sc[S_OMEGA] = red[1] > 0.0 ? red[0] / red[1] : 0.0;
        }
    }
}

// s = r - alpha v, and the half step x += alpha p_hat; when |s| already meets the stop rule
// the solve ends here (the standard early exit: x + alpha p_hat is the iterate whose
// residual is s) and the second preconditioner application of the iteration is skipped
__global__ void __launch_bounds__(NT, 5) k_bicg_s(BatchDev b) {
    const Tile t = b.jtiles[blockIdx.x];
    if (b.iscal[(long long)t.c * NISCAL + I_PDONE]) return;
    const bool first = b.iscal[(long long)t.c * NISCAL + I_PIT] == 0;
    const CaseDev& c = b.cases[t.c];
    const int i = t.i0 + (int)(threadIdx.x % TX), j0 = t.j0 + (int)(threadIdx.x / TX);
    const double alpha = b.scal[(long long)t.c * NSCAL + S_ALPHA];
    double* X = plane(b, c, P_PCOR);
    const double *R = plane(b, c, P_KR), *Vv = plane(b, c, P_KV), *PH = plane(b, c, P_KPH);
    const LevelDev& L = c.lev[0];
    bool in[2];
    long long k[2];
    double x0[2], r[2], v[2], ph[2];
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const int j = j0 + h * TY;
        in[h] = i >= c.ilo && i <= c.ihi && j <= c.n1 - 2;
        k[h] = in[h] ? (long long)j * c.ld + i : (long long)c.ld + c.ilo;
        x0[h] = first ? 0.0 : X[k[h]];
        r[h] = R[k[h]];
        v[h] = Vv[k[h]];
        ph[h] = PH[k[h]];
    }
    double red[1] = {0.0};
#pragma unroll
    for (int h = 0; h < 2; h++) {
        if (!in[h]) continue;
        const int j = j0 + h * TY;
        const double s = r[h] - alpha * v[h];
        const double x = x0[h] + alpha * ph[h];
        plane(b, c, P_KS)[k[h]] = s;
        store_mirrored(X, c.ld, i, j, c.W, c.periodic, x);
        mplane(b, L, M_B)[(long long)j * L.ld + i] = (float)s;
        store_mirrored(mplane(b, L, M_X), L.ld, i, j, L.W, c.periodic, 0.0f);
        red[0] += fabs(s);
    }
    if (case_reduce<1, 0u>(b, t.c, blockIdx.x, c.jt_begin, c.jt_count, red) && threadIdx.x == 0) {
        double* sc = b.scal + (long long)t.c * NSCAL;
        int* is = b.iscal + (long long)t.c * NISCAL;
        const bool conv = red[0] <= c.tol_p * sc[S_NB1] || red[0] <= c.atol_p;
        if (conv || !isfinite(red[0])) {
            is[I_PIT] += 1;
            sc[S_RL1] = red[0];
            if (!isfinite(red[0])) is[I_STATUS] |= ST_NAN;
            is[I_PDONE] = 1;
            atomicSub(b.active, 1);
        }
    }
}

__global__ void __launch_bounds__(NT, 5) k_bicg_x(BatchDev b, int maxit) {
    const Tile t = b.jtiles[blockIdx.x];
    if (b.iscal[(long long)t.c * NISCAL + I_PDONE]) return;
    const CaseDev& c = b.cases[t.c];
    const int i = t.i0 + (int)(threadIdx.x % TX), j0 = t.j0 + (int)(threadIdx.x / TX);
    const double* sc0 = b.scal + (long long)t.c * NSCAL;
    const double alpha = sc0[S_ALPHA], omega = sc0[S_OMEGA];
    const int ld = c.ld;
    double* X = plane(b, c, P_PCOR);
    const double *SH = plane(b, c, P_KSH), *S = plane(b, c, P_KS), *T = plane(b, c, P_KT), *Q = plane(b, c, P_Q);
    bool in[2];
    long long k[2];
    double x0[2], sh[2], s[2], tt[2], q[2];
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const int j = j0 + h * TY;
        in[h] = i >= c.ilo && i <= c.ihi && j <= c.n1 - 2;
        k[h] = in[h] ? (long long)j * ld + i : (long long)ld + c.ilo;
        x0[h] = X[k[h]];
        sh[h] = SH[k[h]];
        s[h] = S[k[h]];
        tt[h] = T[k[h]];
        q[h] = Q[k[h]];
    }
    double red[2] = {0.0, 0.0};
#pragma unroll
    for (int h = 0; h < 2; h++) {
        if (!in[h]) continue;
        const int j = j0 + h * TY;
        // x already carries the half step alpha p_hat (k_bicg_s)
        store_mirrored(X, ld, i, j, c.W, c.periodic, x0[h] + omega * sh[h]);
        const double r = s[h] - omega * tt[h];
        plane(b, c, P_KR)[k[h]] = r;
        red[0] += q[h] * r;
        red[1] += fabs(r);
    }
    if (case_reduce<2, 0u>(b, t.c, blockIdx.x, c.jt_begin, c.jt_count, red) && threadIdx.x == 0) {
        double* sc = b.scal + (long long)t.c * NSCAL;
        int* is = b.iscal + (long long)t.c * NISCAL;
        const int it = ++is[I_PIT];
        const double rho_new = red[0];
        sc[S_RL1] = red[1];
        const bool conv = red[1] <= c.tol_p * sc[S_NB1] || red[1] <= c.atol_p;
        bool stop = conv;
        if (!isfinite(red[1])) { is[I_STATUS] |= ST_NAN; stop = true; }
        else if (!conv && (omega == 0.0 || rho_new == 0.0)) { is[I_PSTATUS] |= ST_BREAKDOWN; stop = true; }
        else if (!conv && it >= maxit) { is[I_PSTATUS] |= ST_MAXITER; stop = true; }
        if (!stop) {
            sc[S_BETA] = (rho_new / sc[S_RHO]) * (alpha / omega);
            sc[S_RHO] = rho_new;
        } else {
            is[I_PDONE] = 1;
            atomicSub(b.active, 1);
        }
    }
}

// ---------------------------------------------------------------------------
// multigrid preconditioner, FP32, level tiles.
//
// One V-cycle: on the way down, level l is pre-smoothed from zero and its residual formed
// and restricted into b_{l+1} -- either by k_mg_gs (mode 0: writes x_l) followed by
// k_mg_rr, or (schedule form 2) by k_mg_prr in one pass over overlapping regions; then one
// k_mg_coarse launch smooths every case's coarsest level (one CTA per case, in place in x);
// on the way up, k_mg_gs (mode 2) adds the prolonged coarse result and post-smooths,
// writing the level's result into its r plane. No kernel reads a plane that another CTA of
// the same launch writes, so the V-cycle is a fixed linear map (the same bits whatever the
// CTA schedule), as the Krylov method needs. The level's final result lives in r (x for a
// case whose coarsest level it is).

// stored column of level column gi, gi in [-W, inf): the periodic wrap without a division
// in the common case (gi within one width of the level)
__device__ __forceinline__ int mg_wrap(int gi, int W) {
    int col = gi < 0 ? gi + W : gi;
    if (col >= W) col = col >= 2 * W ? col % W : col - W;
    return col;
}

__device__ __forceinline__ int mg_colour(int i, int j, int W, int periodic) {
    // 4 colours by parity; an odd periodic width gets 2 extra colours for its last column
    if (periodic && (W & 1) && i == W - 1) return 4 + (j & 1);
    return (i & 1) | ((j & 1) << 1);
}


// Residual r = b - A x of level l on the fine points a coarse tile of level l + 1 needs,
// in shared memory, then full-weighting restriction into b_{l+1} (tiles of level l + 1;
// x_{l+1} is zeroed for the coarse solve). Fine points that are not unknowns contribute 0.
__global__ void __launch_bounds__(NT) k_mg_rr(BatchDev b, int l, int src) {
    constexpr int RW = 2 * TX + 1, RH = 2 * TY + 1;  // fine residual region
    constexpr int XW = RW + 2, XH = RH + 2;          // fine x region (one-cell halo)
    __shared__ float xs[XH * XW];
    __shared__ float rs[RH * RW];
    const Tile t = b.atiles[l + 1][blockIdx.x];
    if (b.iscal[(long long)t.c * NISCAL + I_PDONE]) return;
    const CaseDev& c = b.cases[t.c];
    const LevelDev& F = c.lev[l];
    const LevelDev& C = c.lev[l + 1];
    const int tid = threadIdx.x;
    const int fl = F.ld, per = c.periodic;
    const int fi0 = 2 * t.i0 - 1, fj0 = 2 * t.j0 - 1;
    const float* X = mplane(b, F, src);
    for (int e = tid; e < XH * XW; e += NT) {
        const int gj = fj0 - 1 + e / XW, gi = fi0 - 1 + e % XW;
        float v = 0.0f;
        if (gj >= 0 && gj < F.n1 && gi >= -H && gi < F.W + H) v = X[(long long)gj * fl + gi];
        xs[e] = v;
    }
    __syncthreads();
    // fine unknown columns in stored form: periodic -1 .. W (halo mirrors), else ilo .. ihi
    const int clo = per ? -1 : F.ilo, chi = per ? F.W : F.ihi;
    for (int e = tid; e < RH * RW; e += NT) {
        const int rj = e / RW, ri = e % RW;
        const int gj = fj0 + rj, gi = fi0 + ri;
        float r = 0.0f;
        if (gj >= 1 && gj <= F.n1 - 2 && gi >= clo && gi <= chi) {
            const long long k = (long long)gj * fl + gi;
            const int o = (rj + 1) * XW + (ri + 1);
            const float ax = mplane(b, F, M_AP)[k] * xs[o] + mplane(b, F, M_AE)[k] * xs[o + 1] +
                             mplane(b, F, M_AW)[k] * xs[o - 1] + mplane(b, F, M_AN)[k] * xs[o + XW] +
                             mplane(b, F, M_AS)[k] * xs[o - XW] + mplane(b, F, M_ANE)[k] * xs[o + XW + 1] +
                             mplane(b, F, M_ANW)[k] * xs[o + XW - 1] + mplane(b, F, M_ASE)[k] * xs[o - XW + 1] +
                             mplane(b, F, M_ASW)[k] * xs[o - XW - 1];
            r = mplane(b, F, M_B)[k] - ax;
        }
        rs[e] = r;
    }
    __syncthreads();
    const int li = tid % TX, lj = tid / TX;
    const int I = t.i0 + li, J = t.j0 + lj;
    if (I < C.ilo || I > C.ihi || J > C.n1 - 2) return;
    const int f = (2 * lj + 1) * RW + (2 * li + 1);  // fine (2I, 2J) in the residual region
    const float v = 0.0625f * (rs[f - RW - 1] + rs[f - RW + 1] + rs[f + RW - 1] + rs[f + RW + 1]) +
                    0.125f * (rs[f - RW] + rs[f + RW] + rs[f - 1] + rs[f + 1]) + 0.25f * rs[f];
    const long long kc = (long long)J * C.ld + I;
    mplane(b, C, M_B)[kc] = v;
    store_mirrored(mplane(b, C, M_X), C.ld, I, J, C.W, per, 0.0f);
}

// Pre-smoothing folded into the residual + restriction pass (schedule form `fused` = 2).
// One CTA per 32 x 8 tile of level l + 1. Its fine region E (the 65 x 17 fine points the
// restriction reads plus a one-cell ring: 67 x 19) is smoothed from zero in shared memory,
// zero outside E, by `inner` multicolour Gauss-Seidel sweeps; the residual is formed from
// that x and restricted into b_{l+1}; x is stored for the fine points the tile owns
// (columns 2 i0 .. 2 i0 + 63, rows 2 j0 - 1 .. 2 j0 + 14, and in the last tile row also the
// rows up to n1 - 2), where the post-smoother starts. Neighbouring regions overlap by up to
// three cells, and on a region's ring the residual uses the region's own smoothed x, not
// the owner's stored one. The V-cycle stays a fixed linear map (each CTA reads only level
// planes no CTA of the launch writes); it is a different map from form 1's, with the
// level's pre-smoothing pass and its read of the stencil saved.
constexpr int MPR_EW = 2 * TX + 3, MPR_EH = 2 * TY + 3;  // smoothed region E
constexpr int MPR_RW = 2 * TX + 1, MPR_RH = 2 * TY + 1;  // fine residual region
constexpr int MPR_BX = (MPR_EW + 1) / 2, MPR_BY = (MPR_EH + 1) / 2;  // 2 x 2 blocks of E: 34 x 10
// x of E with a zero ring (69 x 21 points), split by column parity; a parity half has rows
// of 40 words, and the second half starts 16 banks after the first
constexpr int MPR_XW = MPR_EW + 2, MPR_XH = MPR_EH + 2;
constexpr int MPR_XS = 40, MPR_XP = MPR_XH * MPR_XS + 8;
static_assert(MPR_XS >= (MPR_XW + 1) / 2 && MPR_XP % 32 == 16, "split layout of the region's x");
static_assert(MG_PRR_THREADS >= MPR_BX * MPR_BY && MG_PRR_THREADS >= TX * TY && MG_PRR_THREADS % 32 == 0,
              "one thread per 2 x 2 block of E, one per coarse point");

__device__ __forceinline__ int mpr_at(int xx, int ry) {  // point (xx, ry) of the ringed region
    return (xx & 1) * MPR_XP + ry * MPR_XS + (xx >> 1);
}
// the fine residual region (65 x 17 points), split by column parity like x: the blocks write
// it and the restriction reads it at column stride 2, which a plain row-major tile serves
// with two-way bank conflicts; split, consecutive threads touch consecutive words
constexpr int MPR_RS = 33, MPR_RP = MPR_RH * MPR_RS + 16;
__device__ __forceinline__ int mpr_rat(int x, int y) { return (x & 1) * MPR_RP + y * MPR_RS + (x >> 1); }

// Each thread owns one 2 x 2 block of E, which holds one point of each colour (E starts at
// an even column and row, and a level with a coarser one has an even width when periodic,
// so the colours are the four parity classes); its four stencils stay in registers.
__global__ void __launch_bounds__(MG_PRR_THREADS, 3) k_mg_prr(BatchDev b, int l, int dst, int inner) {
    __shared__ float xs[2 * MPR_XP];
    __shared__ float rs[2 * MPR_RP];
    const Tile t = b.atiles[l + 1][blockIdx.x];
    if (b.iscal[(long long)t.c * NISCAL + I_PDONE]) return;
    const CaseDev& c = b.cases[t.c];
    const LevelDev& F = c.lev[l];
    const LevelDev& C = c.lev[l + 1];
    const int tid = threadIdx.x;
    const int fl = F.ld, W = F.W, per = c.periodic, n1 = F.n1;
    if (per && (W & 1)) {
        if (tid == 0) atomicExch(b.error, 1);
        return;
    }
    const int ei0 = 2 * t.i0 - 2, ej0 = 2 * t.j0 - 2;  // level-l (column, row) of E's first point
    const bool own = tid < MPR_BX * MPR_BY;
    const int bx = own ? tid % MPR_BX : 0, by = own ? tid / MPR_BX : 0;
    const int gi0 = ei0 + 2 * bx;
    int c0, c1;  // stored columns of the block's two columns (c1 = c0 + 1 when both exist)
    if (per) {
        c0 = mg_wrap(gi0, W);
        c1 = c0 + 1;
    } else {
        c0 = (gi0 >= 0 && gi0 < W) ? gi0 : -1;
        c1 = (gi0 + 1 >= 0 && gi0 + 1 < W) ? gi0 + 1 : -1;
    }
    float a[2][2][10];  // [dy][dx][ap, ae, aw, an, as, ane, anw, ase, asw, b]
    bool ok[2][2];
#pragma unroll
    for (int dy = 0; dy < 2; dy++) {
        const int gj = ej0 + 2 * by + dy;
        const bool rowok = own && gj >= 1 && gj <= n1 - 2 && 2 * by + dy < MPR_EH;
        ok[dy][0] = rowok && c0 >= F.ilo && c0 <= F.ihi;
        ok[dy][1] = rowok && c1 >= F.ilo && c1 <= F.ihi && 2 * bx + 1 < MPR_EW;
        // the even column and its right neighbour, 8-byte aligned (safe row / column outside)
        const long long k = (long long)((gj >= 0 && gj < n1) ? gj : 1) * fl + (c0 >= 0 ? c0 : 0);
#pragma unroll
        for (int q = 0; q < 10; q++) {
            const float2 v = *reinterpret_cast<const float2*>(mplane(b, F, q < 9 ? M_AP + q : M_B) + k);
            a[dy][0][q] = v.x;
            a[dy][1][q] = v.y;
        }
    }
    for (int e = tid; e < 2 * MPR_XP; e += MG_PRR_THREADS) xs[e] = 0.0f;
    __syncthreads();
    // point of colour cc in the block: (dx, dy) = (cc & 1, cc >> 1); its ringed position is
    // (2 bx + dx + 1, 2 by + dy + 1)
    float xr[2][2] = {{0.0f, 0.0f}, {0.0f, 0.0f}};
    // the first sweep from zero: a colour's neighbours of the colours not yet relaxed are
    // still zero, so colour 0 reads none, colour 1 its E/W neighbours (colour 0), colour 2
    // its N/S (colour 0) and diagonal (colour 1) neighbours, colour 3 all eight
    auto relax0 = [&](auto cc_) {
        constexpr int cc = decltype(cc_)::value;
        constexpr int dx = cc & 1, dy = cc >> 1;
        if (ok[dy][dx]) {
            const float(&f)[10] = a[dy][dx];
            const int xx = 2 * bx + dx + 1, ry = 2 * by + dy + 1;
            float sm = 0.0f;
            if (cc == 1) sm = f[1] * xs[mpr_at(xx + 1, ry)] + f[2] * xs[mpr_at(xx - 1, ry)];
            if (cc == 2)
                sm = f[3] * xs[mpr_at(xx, ry + 1)] + f[4] * xs[mpr_at(xx, ry - 1)] +
                     f[5] * xs[mpr_at(xx + 1, ry + 1)] + f[6] * xs[mpr_at(xx - 1, ry + 1)] +
                     f[7] * xs[mpr_at(xx + 1, ry - 1)] + f[8] * xs[mpr_at(xx - 1, ry - 1)];
            if (cc == 3)
                sm = f[1] * xs[mpr_at(xx + 1, ry)] + f[2] * xs[mpr_at(xx - 1, ry)] +
                     f[3] * xs[mpr_at(xx, ry + 1)] + f[4] * xs[mpr_at(xx, ry - 1)] +
                     f[5] * xs[mpr_at(xx + 1, ry + 1)] + f[6] * xs[mpr_at(xx - 1, ry + 1)] +
                     f[7] * xs[mpr_at(xx + 1, ry - 1)] + f[8] * xs[mpr_at(xx - 1, ry - 1)];
            const float v = (f[9] - sm) / f[0];
            xs[mpr_at(xx, ry)] = v;
            xr[dy][dx] = v;
        }
        __syncthreads();
    };
    auto relax = [&](auto cc_) {
        constexpr int cc = decltype(cc_)::value;
        constexpr int dx = cc & 1, dy = cc >> 1;
        if (ok[dy][dx]) {
            const float(&f)[10] = a[dy][dx];
            const int xx = 2 * bx + dx + 1, ry = 2 * by + dy + 1;
            const float sm = f[1] * xs[mpr_at(xx + 1, ry)] + f[2] * xs[mpr_at(xx - 1, ry)] +
                             f[3] * xs[mpr_at(xx, ry + 1)] + f[4] * xs[mpr_at(xx, ry - 1)] +
                             f[5] * xs[mpr_at(xx + 1, ry + 1)] + f[6] * xs[mpr_at(xx - 1, ry + 1)] +
                             f[7] * xs[mpr_at(xx + 1, ry - 1)] + f[8] * xs[mpr_at(xx - 1, ry - 1)];
            const float v = (f[9] - sm) / f[0];
            xs[mpr_at(xx, ry)] = v;
            xr[dy][dx] = v;
        }
        __syncthreads();
    };
    using C0 = std::integral_constant<int, 0>;
    using C1 = std::integral_constant<int, 1>;
    using C2 = std::integral_constant<int, 2>;
    using C3 = std::integral_constant<int, 3>;
    if (inner > 0) {
        relax0(C0{}); relax0(C1{}); relax0(C2{}); relax0(C3{});
    }
    for (int n = 1; n < inner; n++) {
        relax(C0{}); relax(C1{}); relax(C2{}); relax(C3{});
    }
    // residual on the restriction's fine points (E without its ring), x of the owned points
    float* OUT = mplane(b, F, dst);
    const int jhi = (t.j0 + TY > C.n1 - 2) ? n1 - 2 : min(2 * t.j0 + 14, n1 - 2);
#pragma unroll
    for (int dy = 0; dy < 2; dy++)
#pragma unroll
        for (int dx = 0; dx < 2; dx++) {
            const int x = 2 * bx + dx, y = 2 * by + dy;
            if (!own || x < 1 || x > MPR_RW || y < 1 || y > MPR_RH) continue;
            float r = 0.0f;
            if (ok[dy][dx]) {
                const float(&f)[10] = a[dy][dx];
                const int xx = x + 1, ry = y + 1;
                const float ax = f[0] * xr[dy][dx] + f[1] * xs[mpr_at(xx + 1, ry)] + f[2] * xs[mpr_at(xx - 1, ry)] +
                                 f[3] * xs[mpr_at(xx, ry + 1)] + f[4] * xs[mpr_at(xx, ry - 1)] +
                                 f[5] * xs[mpr_at(xx + 1, ry + 1)] + f[6] * xs[mpr_at(xx - 1, ry + 1)] +
                                 f[7] * xs[mpr_at(xx + 1, ry - 1)] + f[8] * xs[mpr_at(xx - 1, ry - 1)];
                r = f[9] - ax;
            }
            rs[mpr_rat(x - 1, y - 1)] = r;
            // owned: columns 2 i0 .. 2 i0 + 63 (E columns 2 .. 65), rows 2 j0 - 1 .. jhi
            const int gi = ei0 + x, gj = ej0 + y;
            if (x >= 2 && gi >= F.ilo && gi <= F.ihi && gj <= jhi)
                store_mirrored(OUT, fl, gi, gj, W, per, ok[dy][dx] ? xr[dy][dx] : 0.0f);
        }
    __syncthreads();
    if (tid >= TX * TY) return;
    const int li = tid % TX, lj = tid / TX;
    const int I = t.i0 + li, J = t.j0 + lj;
    if (I < C.ilo || I > C.ihi || J > C.n1 - 2) return;
    const int fx = 2 * li + 1, fy = 2 * lj + 1;  // fine (2I, 2J) in the residual region
    const float r4 = 0.0625f * (rs[mpr_rat(fx - 1, fy - 1)] + rs[mpr_rat(fx + 1, fy - 1)] + rs[mpr_rat(fx - 1, fy + 1)] +
                                rs[mpr_rat(fx + 1, fy + 1)]) +
                     0.125f * (rs[mpr_rat(fx, fy - 1)] + rs[mpr_rat(fx, fy + 1)] + rs[mpr_rat(fx - 1, fy)] +
                               rs[mpr_rat(fx + 1, fy)]) +
                     0.25f * rs[mpr_rat(fx, fy)];
    mplane(b, C, M_B)[(long long)J * C.ld + I] = r4;
    store_mirrored(mplane(b, C, M_X), C.ld, I, J, C.W, per, 0.0f);
}

// bilinear prolongation of the coarse result at fine point (i, j), i in [0, W)
__device__ __forceinline__ float mg_prolong_at(const float* XC, int cl, int i, int j) {
    const int I = i >> 1, J = j >> 1;
    const long long q = (long long)J * cl + I;
    if (!(i & 1) && !(j & 1)) return XC[q];
    if (!(j & 1)) return 0.5f * (XC[q] + XC[q + 1]);
    if (!(i & 1)) return 0.5f * (XC[q] + XC[q + cl]);
    return 0.25f * (XC[q] + XC[q + 1] + XC[q + cl] + XC[q + cl + 1]);
}

// Multicolour Gauss-Seidel sweeps of level l on a 32 x 16 tile (block Gauss-Seidel at tile
// edges: the halo ring holds the neighbouring tiles' values from before the first sweep).
// The sweeps read plane `src` and write plane `dst` != src, so nothing is read that another
// CTA writes.
//   mode 0: from x = 0, colours in order (first pre-sweep; src unused)
//   mode 1: from src, colours in order (further pre-sweeps)
//   mode 2: from src plus the prolonged result of level l + 1, colours reversed (first
//           post-sweep)
//   mode 3: from src, colours reversed (further post-sweeps)
// `inner` sweeps run back to back in shared memory (one launch and one read of the stencil
// for several sweeps, at the price of weaker coupling between tiles).
//
// A level with a coarser one has an even width when periodic, so its colours are the four
// parity classes. Tiles start at an even column and an odd row, so every 2 x 2 block of the
// tile holds one point of each colour: a thread owns one block (16 x 8 blocks, 128
// threads), keeps its four stencils in registers (loaded as column pairs) and relaxes one
// point per colour. x with its halo is held in shared memory split by column parity, rows
// padded so that a warp's two block rows fall in different banks: every read of a
// colour pass is free of bank conflicts.
constexpr int MG_GS_XW = TX + 2, MG_GS_XH = TYJ + 2;  // x halo region
constexpr int MG_GS_XS = 24;                           // row stride of a parity half
constexpr int MG_GS_XP = MG_GS_XH * MG_GS_XS;          // 432 = 16 mod 32 words
static_assert(MG_GS_XS >= (MG_GS_XW + 1) / 2 && (2 * MG_GS_XS) % 32 == 16 && MG_GS_XP % 32 == 16,
              "parity halves must keep a colour pass free of bank conflicts");
static_assert(MG_GS_THREADS == (TX / 2) * (TYJ / 2), "one thread per 2 x 2 block");

__device__ __forceinline__ int mg_gs_at(int xx, int ry) {  // halo point (xx, ry) in the split layout
    return (xx & 1) * MG_GS_XP + ry * MG_GS_XS + (xx >> 1);
}

__global__ void __launch_bounds__(MG_GS_THREADS, 8) k_mg_gs(BatchDev b, int l, int mode, int src, int dst, int inner) {
    __shared__ float xs[2 * MG_GS_XP];
    const Tile t = b.mtiles[l][blockIdx.x];
    if (b.iscal[(long long)t.c * NISCAL + I_PDONE]) return;
    const CaseDev& c = b.cases[t.c];
    const LevelDev& L = c.lev[l];
    const int tid = threadIdx.x;
    const int ld = L.ld, W = L.W, per = c.periodic, n1 = L.n1;
    if (per && (W & 1)) {
        if (tid == 0) atomicExch(b.error, 1);
        return;
    }
    const bool zero = mode == 0, prolong = mode == 2, reverse = mode >= 2;
    const float* X = mplane(b, L, src);
    const float* XC = prolong ? mplane(b, c.lev[l + 1], mg_result_plane(b, c, l + 1)) : nullptr;
    const int cl = prolong ? c.lev[l + 1].ld : 0;
    // stored column of level column gi (periodic wrap), or -1 outside the level
    auto column = [&](int gi) -> int {
        if (per) return mg_wrap(gi, W);
        return (gi >= 0 && gi < W) ? gi : -1;
    };
    // this thread's 2 x 2 block: tile columns 2 bx, 2 bx + 1, rows 2 by, 2 by + 1
    const int bx = tid % (TX / 2), by = tid / (TX / 2);
    const int gi0 = t.i0 + 2 * bx;
    const int c0 = column(gi0), c1 = column(gi0 + 1);  // c1 = c0 + 1 whenever both are in the level
    float a[2][2][10];  // [dy][dx][ap^-1, ae, aw, an, as, ane, anw, ase, asw, b]
    bool ok[2][2];
#pragma unroll
    for (int dy = 0; dy < 2; dy++) {
        const int gj = t.j0 + 2 * by + dy;
        ok[dy][0] = gj >= 1 && gj <= n1 - 2 && c0 >= L.ilo && c0 <= L.ihi;
        ok[dy][1] = gj >= 1 && gj <= n1 - 2 && c1 >= L.ilo && c1 <= L.ihi;
        // an even column and its right neighbour, 8-byte aligned (safe row / column when outside)
        const long long k = (long long)((gj >= 0 && gj < n1) ? gj : 1) * ld + (c0 >= 0 ? c0 : 0);
#pragma unroll
        for (int q = 0; q < 10; q++) {
            const float2 v = *reinterpret_cast<const float2*>(mplane(b, L, q < 9 ? M_AP + q : M_B) + k);
            a[dy][0][q] = v.x;
            a[dy][1][q] = v.y;
        }
    }
    // x and its halo (with the prolonged coarse correction in mode 2)
    constexpr int NXL = (MG_GS_XW * MG_GS_XH + MG_GS_THREADS - 1) / MG_GS_THREADS;
    float xv[NXL];
#pragma unroll
    for (int m = 0; m < NXL; m++) {
        const int e = tid + m * MG_GS_THREADS;
        const int gj = t.j0 - 1 + e / MG_GS_XW, col = column(t.i0 - 1 + e % MG_GS_XW);
        float v = 0.0f;
        if (!zero && e < MG_GS_XW * MG_GS_XH && gj >= 0 && gj < n1 && col >= 0) {
            v = X[(long long)gj * ld + col];
            if (prolong && gj >= 1 && gj <= n1 - 2 && col >= L.ilo && col <= L.ihi)
                v += mg_prolong_at(XC, cl, col, gj);
        }
        xv[m] = v;
    }
#pragma unroll
    for (int m = 0; m < NXL; m++) {
        const int e = tid + m * MG_GS_THREADS;
        if (e < MG_GS_XW * MG_GS_XH) xs[mg_gs_at(e % MG_GS_XW, e / MG_GS_XW)] = xv[m];
    }
#pragma unroll
    for (int dy = 0; dy < 2; dy++)
#pragma unroll
        for (int dx = 0; dx < 2; dx++) a[dy][dx][0] = ok[dy][dx] ? 1.0f / a[dy][dx][0] : 0.0f;
    __syncthreads();
    // point of colour cc in this thread's block: (dx, dy) = (cc & 1, 1 - (cc >> 1)) (the tile's
    // first row is odd); its halo position is (2 bx + dx + 1, 2 by + dy + 1)
    auto relax = [&](auto cc_) {
        constexpr int cc = decltype(cc_)::value;
        constexpr int dx = cc & 1, dy = 1 - (cc >> 1);
        if (ok[dy][dx]) {
            const float(&f)[10] = a[dy][dx];
            const int xx = 2 * bx + dx + 1, ry = 2 * by + dy + 1;
            const float sm = f[1] * xs[mg_gs_at(xx + 1, ry)] + f[2] * xs[mg_gs_at(xx - 1, ry)] +
                             f[3] * xs[mg_gs_at(xx, ry + 1)] + f[4] * xs[mg_gs_at(xx, ry - 1)] +
                             f[5] * xs[mg_gs_at(xx + 1, ry + 1)] + f[6] * xs[mg_gs_at(xx - 1, ry + 1)] +
                             f[7] * xs[mg_gs_at(xx + 1, ry - 1)] + f[8] * xs[mg_gs_at(xx - 1, ry - 1)];
            xs[mg_gs_at(xx, ry)] = (f[9] - sm) * f[0];
        }
        __syncthreads();
    };
    using C0 = std::integral_constant<int, 0>;
    using C1 = std::integral_constant<int, 1>;
    using C2 = std::integral_constant<int, 2>;
    using C3 = std::integral_constant<int, 3>;
    for (int n = 0; n < inner; n++) {
        if (reverse) { relax(C3{}); relax(C2{}); relax(C1{}); relax(C0{}); }
        else { relax(C0{}); relax(C1{}); relax(C2{}); relax(C3{}); }
    }
    float* OUT = mplane(b, L, dst);
#pragma unroll
    for (int dy = 0; dy < 2; dy++)
#pragma unroll
        for (int dx = 0; dx < 2; dx++) {
            const int i = gi0 + dx, j = t.j0 + 2 * by + dy;
            if (i < L.ilo || i > L.ihi || j > n1 - 2) continue;
            store_mirrored(OUT, ld, i, j, W, per, xs[mg_gs_at(2 * bx + dx + 1, 2 * by + dy + 1)]);
        }
}

// coarsest level: `sweeps` multicolour GS sweeps by one CTA per case, x in shared memory
// and each thread's stencil in registers when the level fits (one unknown per thread);
// larger levels (a case whose grid does not coarsen) sweep through global memory
constexpr int MGC_THREADS = 1024, MGC_SMEM = 4096;
__global__ void __launch_bounds__(MGC_THREADS) k_mg_coarse(BatchDev b, int l, int sweeps) {
    __shared__ float xs[MGC_SMEM];
    // l < 0: one launch for every case, each on its own coarsest level (the case lists of
    // all levels are stored back to back from ccases[0])
    const int cid = l >= 0 ? b.ccases[l][blockIdx.x] : b.ccases[0][blockIdx.x];
    if (b.iscal[(long long)cid * NISCAL + I_PDONE]) return;
    const CaseDev& c = b.cases[cid];
    const LevelDev& L = c.lev[l >= 0 ? l : c.nlev - 1];
    const int ld = L.ld, per = c.periodic;
    const int nx = L.ihi - L.ilo + 1, ny = L.n1 - 2;
    float* X = mplane(b, L, M_X);
    const float* Bv = mplane(b, L, M_B);
    const int ncol = (per && (L.W & 1)) ? 6 : 4;
    const int sw = L.W + 2 * H;  // shared copy: all rows, columns -H .. W+H-1
    if (nx * ny <= MGC_THREADS && L.n1 * sw <= MGC_SMEM) {
        for (int e = threadIdx.x; e < L.n1 * sw; e += MGC_THREADS) xs[e] = 0.0f;  // x = 0 (and boundaries)
        const int e = threadIdx.x;
        const bool in = e < nx * ny;
        const int i = L.ilo + (in ? e % nx : 0), j = 1 + (in ? e / nx : 0);
        const long long k = (long long)j * ld + i;
        float ap = 1.f, ae = 0.f, aw = 0.f, an = 0.f, as = 0.f, ane = 0.f, anw = 0.f, ase = 0.f, asw = 0.f, bv = 0.f;
        int col = -1;
        if (in) {
            ap = mplane(b, L, M_AP)[k]; ae = mplane(b, L, M_AE)[k]; aw = mplane(b, L, M_AW)[k];
            an = mplane(b, L, M_AN)[k]; as = mplane(b, L, M_AS)[k]; ane = mplane(b, L, M_ANE)[k];
            anw = mplane(b, L, M_ANW)[k]; ase = mplane(b, L, M_ASE)[k]; asw = mplane(b, L, M_ASW)[k];
            bv = Bv[k];
            col = mg_colour(i, j, L.W, per);
        }
        const int o = j * sw + i + H;
        const int m = mirror_col(i, L.W, per);
        __syncthreads();
        for (int s = 0; s < sweeps; s++) {
            for (int cc = 0; cc < ncol; cc++) {
                if (col == cc) {
                    const float sm = ae * xs[o + 1] + aw * xs[o - 1] + an * xs[o + sw] + as * xs[o - sw] +
                                     ane * xs[o + sw + 1] + anw * xs[o + sw - 1] + ase * xs[o - sw + 1] +
                                     asw * xs[o - sw - 1];
                    const float v = (bv - sm) / ap;
                    xs[o] = v;
                    if (m > -1000000) xs[j * sw + m + H] = v;
                }
                __syncthreads();
            }
        }
        if (in) store_mirrored(X, ld, i, j, L.W, per, xs[o]);
        return;
    }
    for (int e = threadIdx.x; e < nx * ny; e += blockDim.x) {  // x = 0
        const int i = L.ilo + e % nx, j = 1 + e / nx;
        store_mirrored(X, ld, i, j, L.W, per, 0.0f);
    }
    __syncthreads();
    for (int s = 0; s < sweeps; s++) {
        for (int col = 0; col < ncol; col++) {
            for (int e = threadIdx.x; e < nx * ny; e += blockDim.x) {
                const int i = L.ilo + e % nx, j = 1 + e / nx;
                if (mg_colour(i, j, L.W, per) != col) continue;
                const long long k = (long long)j * ld + i;
                const float sm = mplane(b, L, M_AE)[k] * X[k + 1] + mplane(b, L, M_AW)[k] * X[k - 1] +
                                 mplane(b, L, M_AN)[k] * X[k + ld] + mplane(b, L, M_AS)[k] * X[k - ld] +
                                 mplane(b, L, M_ANE)[k] * X[k + ld + 1] + mplane(b, L, M_ANW)[k] * X[k + ld - 1] +
                                 mplane(b, L, M_ASE)[k] * X[k - ld + 1] + mplane(b, L, M_ASW)[k] * X[k - ld - 1];
                store_mirrored(X, ld, i, j, L.W, per, (Bv[k] - sm) / mplane(b, L, M_AP)[k]);
            }
            __syncthreads();
        }
    }
}

// Galerkin coarse operator A_{l+1} = R A_l P (R full weighting, P bilinear, R = P^T / 4)
__device__ __forceinline__ bool lev_unknown(const LevelDev& L, int periodic, int i, int j) {
    if (j < 1 || j > L.n1 - 2) return false;
    if (periodic) return true;
    return i >= L.ilo && i <= L.ihi;
}

__global__ void __launch_bounds__(NT) k_mg_galerkin(BatchDev b, int l, int toff) {
    const Tile t = b.atiles[l + 1][toff + blockIdx.x];
    const CaseDev& c = b.cases[t.c];
    const LevelDev& F = c.lev[l];
    const LevelDev& C = c.lev[l + 1];
    const int I = t.i0 + (int)(threadIdx.x % TX), J = t.j0 + (int)(threadIdx.x / TX);
    if (I < C.ilo || I > C.ihi || J > C.n1 - 2) return;
    const int per = c.periodic;
    const int fl = F.ld;
    const float* fa[9];
#pragma unroll
    for (int m = 0; m < 9; m++) fa[m] = mplane(b, F, M_AP + m);
    // stencil offsets in M_AP.. order: p, e, w, n, s, ne, nw, se, sw
    const int ox[9] = {0, 1, -1, 0, 0, 1, -1, 1, -1};
    const int oy[9] = {0, 0, 0, 1, -1, 1, 1, -1, -1};
    double acc[9];  // indexed (dy + 1) * 3 + (dx + 1)
#pragma unroll
    for (int m = 0; m < 9; m++) acc[m] = 0.0;
    for (int bj = -1; bj <= 1; bj++) {
        for (int bi = -1; bi <= 1; bi++) {
            const int fi = 2 * I + bi, fj = 2 * J + bj;
            if (!lev_unknown(F, per, fi, fj)) continue;
            const double wr = 0.25 * (bi == 0 ? 1.0 : 0.5) * (bj == 0 ? 1.0 : 0.5);
            const long long kf = (long long)fj * fl + fi;
            for (int m = 0; m < 9; m++) {
                const int gi = fi + ox[m], gj = fj + oy[m];
                if (!lev_unknown(F, per, gi, gj)) continue;
                const double a = wr * (double)fa[m][kf];
                // coarse parents of fine point (gi, gj)
                int pi[2], pj[2];
                double wi[2], wj[2];
                int ni, nj;
                if (!(gi & 1)) { pi[0] = gi >> 1; wi[0] = 1.0; ni = 1; }
                else { pi[0] = (gi - 1) >> 1; pi[1] = (gi + 1) >> 1; wi[0] = wi[1] = 0.5; ni = 2; }
                if (!(gj & 1)) { pj[0] = gj >> 1; wj[0] = 1.0; nj = 1; }
                else { pj[0] = (gj - 1) >> 1; pj[1] = (gj + 1) >> 1; wj[0] = wj[1] = 0.5; nj = 2; }
                for (int x = 0; x < ni; x++) {
                    for (int y = 0; y < nj; y++) {
                        if (!lev_unknown(C, per, pi[x], pj[y])) continue;
                        const int dx = pi[x] - I, dy = pj[y] - J;
                        acc[(dy + 1) * 3 + (dx + 1)] += a * wi[x] * wj[y];
                    }
                }
            }
        }
    }
    const long long kc = (long long)J * C.ld + I;
    const int idx[9] = {4, 5, 3, 7, 1, 8, 6, 2, 0};  // p, e, w, n, s, ne, nw, se, sw
#pragma unroll
    for (int m = 0; m < 9; m++)
        store_mirrored(mplane(b, C, M_AP + m), C.ld, I, J, C.W, per, (float)acc[idx[m]]);
    (void)kc;
}

// ---------------------------------------------------------------------------
// pcor boundary conditions + velocity / pressure correction (PSolver.cpp:1471-1542);
// also the momentum part of the steady residual, sum |u^{n+1} - u^n| + |v^{n+1} - v^n|
__global__ void __launch_bounds__(NT, 4) k_correct(BatchDev b) {
    // a 32 x 16 tile, two cells per thread (rows lj and lj + 8): every load of both cells
    // is issued before any arithmetic
    const Tile t = b.jtiles[blockIdx.x];
    const CaseDev& c = b.cases[t.c];
    const int* isc = b.iscal + (long long)t.c * NISCAL;
    if (!isc[I_ACTIVE]) return;  // uniform over the case
    // no pressure iteration ran (q vanished or broke down at once): pcor = 0
    const bool none = isc[I_PIT] == 0;
    const int ld = c.ld, W = c.W, per = c.periodic, n1 = c.n1, n0 = c.n0;
    const bool cav = c.profile == CAVITY;
    double* PC = plane(b, c, P_PCOR);
    double* U = plane(b, c, P_U);
    double* V = plane(b, c, P_V);
    double* P = plane(b, c, P_P);
    const double* US = plane(b, c, P_US);
    const double* VS = plane(b, c, P_VS);
    const double* XIX = plane(b, c, P_XIX);
    const double* XIY = plane(b, c, P_XIY);
    const double* ETX = plane(b, c, P_ETX);
    const double* ETY = plane(b, c, P_ETY);
    const double* VEC = plane(b, c, P_VEC);
    const int i = t.i0 + (int)(threadIdx.x % TX);
    bool in[2];
    long long kk[2];
    double pc0[2], pn0[2], ps0[2], pe0[2], pw0[2], us[2], vs[2], xix[2], etx[2], xiy[2], ety[2], u0[2], v0[2],
        p0[2];
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const int j = t.j0 + (int)(threadIdx.x / TX) + h * TY;
        in[h] = i >= c.ilo && i <= c.ihi && j <= n1 - 2;
        const long long k = in[h] ? (long long)j * ld + i : (long long)ld + c.ilo;  // a safe cell when out
        kk[h] = k;
        pc0[h] = PC[k]; pn0[h] = PC[k + ld]; ps0[h] = PC[k - ld]; pe0[h] = PC[k + 1]; pw0[h] = PC[k - 1];
        us[h] = US[k]; vs[h] = VS[k];
        xix[h] = XIX[k]; etx[h] = ETX[k]; xiy[h] = XIY[k]; ety[h] = ETY[k];
        u0[h] = U[k]; v0[h] = V[k]; p0[h] = P[k];
    }
    const double vnn = c.uinf * VEC[2LL * ld + i] + c.vinf * VEC[3LL * ld + i];
    const double h0 = 0.5 / c.d0, h1 = 0.5 / c.d1, dt = c.dt;  // the gradients' quotients as products
    double red[1] = {0.0};
#pragma unroll
    for (int h = 0; h < 2; h++) {
        if (!in[h]) continue;
        const int j = t.j0 + (int)(threadIdx.x / TX) + h * TY;
        const long long k = kk[h];
        const double pc = none ? 0.0 : pc0[h];
        // pcor on the boundary after its conditions: wall copy, far field 0 / copy at inflow
        const double far = (!cav && vnn >= 0) ? pc : 0.0;
        const double pN = none ? 0.0 : (j == n1 - 2) ? (cav ? pc : far) : pn0[h];
        const double pS = none ? 0.0 : (j == 1) ? pc : ps0[h];
        const double pE = none ? 0.0 : (cav && i == n0 - 2) ? pc : pe0[h];
        const double pW = none ? 0.0 : (cav && i == 1) ? pc : pw0[h];
        const double dpcor_dxi = (pE - pW) * h0;
        const double dpcor_de = (pN - pS) * h1;
        const double un = us[h] - dt * (xix[h] * dpcor_dxi + etx[h] * dpcor_de);
        const double vn = vs[h] - dt * (xiy[h] * dpcor_dxi + ety[h] * dpcor_de);
        red[0] += fabs(un - u0[h]) + fabs(vn - v0[h]);
        store_mirrored(U, ld, i, j, W, per, un);
        store_mirrored(V, ld, i, j, W, per, vn);
        const double pn = (c.omega_p == 1.0) ? p0[h] + pc : p0[h] + c.omega_p * pc;
        store_mirrored(P, ld, i, j, W, per, pn);
        if (none) store_mirrored(PC, ld, i, j, W, per, 0.0);
        // record the boundary pcor (output only)
        if (j == 1) store_mirrored(PC, ld, i, 0, W, per, pc);
        if (j == n1 - 2) store_mirrored(PC, ld, i, n1 - 1, W, per, cav ? pc : far);
        if (cav) {
            if (i == 1) PC[k - 1] = pc;
            if (i == n0 - 2) PC[k + 1] = pc;
            if (i == 1 && j == 1) PC[0] = pc;
            if (i == n0 - 2 && j == 1) PC[n0 - 1] = pc;
            if (i == 1 && j == n1 - 2) PC[(long long)(n1 - 1) * ld] = pc;
            if (i == n0 - 2 && j == n1 - 2) PC[(long long)(n1 - 1) * ld + n0 - 1] = pc;
        }
    }
    if (case_reduce<1, 0u>(b, t.c, blockIdx.x, c.jt_begin, c.jt_count, red) && threadIdx.x == 0)
        b.scal[(long long)t.c * NSCAL + S_DUL1] = red[0];
}

// ---------------------------------------------------------------------------
// boundary update, boundary pressure and wall integrals: one CTA per case
// (O-grid: PSolver.cpp:1549-1783 and 1855-1983; cavity: this project's walls)
__global__ void __launch_bounds__(BC_THREADS, 2) k_bc(BatchDev b) {
    const int cid = blockIdx.x;
    const CaseDev& c = b.cases[cid];
    if (!b.iscal[(long long)cid * NISCAL + I_ACTIVE]) return;
    const int ld = c.ld, W = c.W, per = c.periodic, n1 = c.n1, n0 = c.n0;
    const int cur = b.cur, nxt = cur ^ 1;
    const bool cav = c.profile == CAVITY;
    const double d0 = c.d0, d1 = c.d1, dt = c.dt, Re = c.Re, Ri = c.Ri, Pi = c.Pi;
    double* U = plane(b, c, P_U);
    double* V = plane(b, c, P_V);
    double* Tn = plane(b, c, P_T0 + nxt);
    const double* To = plane(b, c, P_T0 + cur);
    double* UPn = plane(b, c, P_UP0 + nxt);
    double* VPn = plane(b, c, P_VP0 + nxt);
    double* P = plane(b, c, P_P);
    double* VORT = plane(b, c, P_VORT);
    const double* X = plane(b, c, P_X);
    const double* Yc = plane(b, c, P_Y);
    const double* XIX = plane(b, c, P_XIX);
    const double* XIY = plane(b, c, P_XIY);
    const double* ETX = plane(b, c, P_ETX);
    const double* ETY = plane(b, c, P_ETY);
    const double* ALPH = plane(b, c, P_ALPH);
    const double* BETA = plane(b, c, P_BETA);
    const double* GAM = plane(b, c, P_GAM);
    const double* JAC = plane(b, c, P_JAC);
    const double* VEC = plane(b, c, P_VEC);
    __shared__ double red[16 * 32];
    __shared__ double s_circ;
    int* is = b.iscal + (long long)cid * NISCAL;
    double* sc = b.scal + (long long)cid * NSCAL;
    const int time_new = (int)((double)is[I_TIME] + dt);
    // the time the wall motion sees: the reference's int (PSolver.cpp:186), or t = n dt
    const double t_new = c.time_accurate ? sc[S_TIME] + dt : (double)time_new;
    const int jf = n1 - 1;
    // far-field u/v before this update (uold of PSolver.cpp:1456); W <= 4096
    extern __shared__ double s_old[];  // 2 * (W + 1)

    if (!cav) {
        // circulation at j = n1-2 (PSolver.cpp:1568-1576)
        {
            const int j = n1 - 2;
            const double de = c.fix_circ_de ? 1.0 / (n0 - 1) : 1.0 / (n0 - 2);
            double acc[1] = {0.0};
            for (int i = threadIdx.x; i < W; i += blockDim.x) {
                const long long k = (long long)j * ld + i, kp = k + 1;
                double f1 = (U[k] * ETY[k] - V[k] * ETX[k]) * fabs(JAC[k]);
                double f2 = (U[kp] * ETY[kp] - V[kp] * ETX[kp]) * fabs(JAC[kp]);
                acc[0] += de * 0.5 * (f1 + f2);
                const long long kf = (long long)jf * ld + i;
                s_old[i] = U[kf];
                s_old[W + 1 + i] = V[kf];
            }
            block_sum<1>(acc, red);
            if (threadIdx.x == 0) s_circ = acc[0];
            __syncthreads();
        }
        const double circ = s_circ;
        const double cwall = cos(2.0 * Pi * c.F * t_new);
        for (int i = threadIdx.x; i < W; i += blockDim.x) {
            // vr/vth just inside (PSolver.cpp:1549-1562) and their far-field prediction (:1582-1609)
            const long long kb = (long long)(jf - 1) * ld + i, k = (long long)jf * ld + i;
            const double costb = X[kb] / sqrt(X[kb] * X[kb] + Yc[kb] * Yc[kb]);
            const double sintb = Yc[kb] / sqrt(X[kb] * X[kb] + Yc[kb] * Yc[kb]);
            const double vr0 = U[kb] * costb + V[kb] * sintb;
            const double vth0 = -U[kb] * sintb + V[kb] * costb;
            const double cr = sqrt(X[kb] * X[kb] + Yc[kb] * Yc[kb]) / sqrt(X[k] * X[k] + Yc[k] * Yc[k]);
            const double costh = X[k] / sqrt(X[k] * X[k] + Yc[k] * Yc[k]);
            const double sinth = Yc[k] / sqrt(X[k] * X[k] + Yc[k] * Yc[k]);
            const double vrinf = c.uinf * costh + c.vinf * sinth;
            const double vtinf = -c.uinf * sinth + c.vinf * costh;
            const double cr2 = cr * cr;
            const double crk = fabs(circ) > 1e-2 ? cr : cr2;
            const double vr1 = vr0 * cr2 + vrinf * (1 - cr2);
            const double vth1 = vth0 * crk + vtinf * (1 - crk);
            // far-field u/v/T (PSolver.cpp:1632-1656)
            const double vnn = c.uinf * VEC[2LL * ld + i] + c.vinf * VEC[3LL * ld + i];
            double un, vn, tn;
            if (vnn >= 0) {
                un = c.uinf; vn = c.vinf; tn = 0.0;
            } else {
                un = costh * vr1 - sinth * vth1;
                vn = sinth * vr1 + costh * vth1;
                const double uet_old = ETX[k] * s_old[i] + ETY[k] * s_old[W + 1 + i];
                tn = To[k] - (uet_old * dt / d1) * (To[k] - To[k - ld]);
            }
            store_mirrored(U, ld, i, jf, W, per, un);
            store_mirrored(V, ld, i, jf, W, per, vn);
            store_mirrored(Tn, ld, i, jf, W, per, tn);
            // wall velocity (PSolver.cpp:1617-1630)
            const double uw = -c.speed_amp * cwall * Yc[i];
            const double vw = c.speed_amp * cwall * X[i];
            store_mirrored(U, ld, i, 0, W, per, uw);
            store_mirrored(V, ld, i, 0, W, per, vw);
            store_mirrored(UPn, ld, i, 0, W, per, uw);
            store_mirrored(VPn, ld, i, 0, W, per, vw);
        }
        __syncthreads();
        // boundary pressure (PSolver.cpp:1668-1783)
        const double swall = sin(2.0 * Pi * c.F * t_new);
        const double* Fl[2] = {U, V};
        for (int i = threadIdx.x; i < W; i += blockDim.x) {
            {   // wall, j = 0
                const long long k = i;
                double dpd[2];
                const double uxi = XIX[k] * U[k] + XIY[k] * V[k];
                const double uet = ETX[k] * U[k] + ETY[k] * V[k];
                for (int m = 0; m < 2; m++) {
                    const double* f = Fl[m];
                    const double aa = ALPH[k] * (f[k + 1] + f[k - 1] - 2 * f[k]) / (d0 * d0);
                    const double gg = GAM[k] * (f[k + 2LL * ld] + f[k] - 2 * f[k + ld]) / (d1 * d1);
                    const double bb = BETA[k] * (f[k + ld + 1] + f[k - 1] - f[k + ld - 1] - f[k + 1]) / (2 * d0 * d1);
                    const double d2u = aa + gg - 2 * bb;
                    double cv = uxi * 0.5 * (f[k + 1] - f[k - 1]) / d0;
                    cv = cv + uet * (f[k + ld] - f[k]) / d1;
                    const double alc = (m == 0) ? c.accn_amp * swall * Yc[k] : -c.accn_amp * swall * X[k];
                    dpd[m] = 1.0 * d2u / Re - cv - alc + (m == 1 ? Ri * Tn[k] : 0.0);
                }
                const double pw = P[k + ld] - (dpd[0] * (-XIY[k] * JAC[k]) + dpd[1] * (XIX[k] * JAC[k])) * d1;
                store_mirrored(P, ld, i, 0, W, per, pw);
            }
            {   // far field, j = n1-1
                const long long k = (long long)jf * ld + i;
                const double vnn = c.uinf * VEC[2LL * ld + i] + c.vinf * VEC[3LL * ld + i];
                double pf;
                if (vnn >= 0) {
                    const double uxi = XIX[k] * U[k] + XIY[k] * V[k];
                    const double uet = ETX[k] * U[k] + ETY[k] * V[k];
                    double dpd[2];
                    for (int m = 0; m < 2; m++) {
                        const double* f = Fl[m];
                        const double fo = s_old[m * (W + 1) + i];
                        const double aa = ALPH[k] * (f[k + 1] + f[k - 1] - 2 * f[k]) / (d0 * d0);
                        const double gg = GAM[k] * (f[k] + f[k - 2LL * ld] - 2 * f[k - ld]) / (d1 * d1);
                        const double bb = BETA[k] * (f[k + 1] + f[k - ld - 1] - f[k - ld + 1] - f[k - 1]) / (2 * d0 * d1);
                        const double d2u = aa + gg - 2 * bb;
                        double cv = uxi * 0.5 * (f[k + 1] - f[k - 1]) / d0;
                        cv = cv + uet * (3.0 * f[k] - 4 * f[k - ld] + f[k - 2LL * ld]) / (2 * d1);
                        const double alc = (f[k] - fo) / dt;
                        dpd[m] = 1.0 * d2u / Re - cv - alc + (m == 1 ? Ri * Tn[k] : 0.0);
                    }
                    pf = P[k - ld] + (dpd[0] * (-XIY[k] * JAC[k]) + dpd[1] * (XIX[k] * JAC[k])) * d1;
                } else {
                    const double e0 = ETX[k] * U[k] + ETY[k] * V[k];
                    const long long k1 = k - ld, k2 = k - 2LL * ld;
                    const double e1 = ETX[k1] * U[k1] + ETY[k1] * V[k1];
                    const double e2 = ETX[k2] * U[k2] + ETY[k2] * V[k2];
                    pf = 0.5 * (1.0 / Re) * ((3 * e0 - 4 * e1 + e2) / d1);
                }
                store_mirrored(P, ld, i, jf, W, per, pf);
            }
        }
    } else {
        // cavity: adiabatic side walls, zero normal pressure gradient, static walls
        for (int j = 1 + threadIdx.x; j <= n1 - 2; j += blockDim.x) {
            const long long r = (long long)j * ld;
            Tn[r] = (4.0 * Tn[r + 1] - Tn[r + 2]) / 3.0;
            Tn[r + n0 - 1] = (4.0 * Tn[r + n0 - 2] - Tn[r + n0 - 3]) / 3.0;
            P[r] = P[r + 1];
            P[r + n0 - 1] = P[r + n0 - 2];
        }
        for (int i = 1 + threadIdx.x; i <= n0 - 2; i += blockDim.x) {
            P[i] = P[i + ld];
            P[(long long)jf * ld + i] = P[(long long)(jf - 1) * ld + i];
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            P[0] = 0.5 * (P[1] + P[ld]);
            P[n0 - 1] = 0.5 * (P[n0 - 2] + P[ld + n0 - 1]);
            const long long r = (long long)jf * ld;
            P[r] = 0.5 * (P[r + 1] + P[r - ld]);
            P[r + n0 - 1] = 0.5 * (P[r + n0 - 2] + P[r - ld + n0 - 1]);
        }
    }
    __syncthreads();
    // vorticity on the j-boundaries (PSolver.cpp:1855-1888)
    for (int e = threadIdx.x; e < 2 * (c.ihi - c.ilo + 1); e += blockDim.x) {
        const int nb = c.ihi - c.ilo + 1;
        const int i = c.ilo + e % nb;
        const int j = (e < nb) ? 0 : jf;
        const long long k = (long long)j * ld + i;
        const double dv_dxi = 0.5 / d0 * (V[k + 1] - V[k - 1]);
        const double dv_det = (j == 0) ? 1.0 / d1 * (V[k + ld] - V[k]) : 1.0 / d1 * (V[k] - V[k - ld]);
        const double dv_dx = XIX[k] * dv_dxi + ETX[k] * dv_det;
        const double du_dxi = 0.5 / d0 * (U[k + 1] - U[k - 1]);
        const double du_det = (j == 0) ? 1.0 / d1 * (U[k + ld] - U[k]) : 1.0 / d1 * (U[k] - U[k - ld]);
        const double du_dy = XIY[k] * du_dxi + ETY[k] * du_det;
        store_mirrored(VORT, ld, i, j, W, per, dv_dx - du_dy);
    }
    __syncthreads();
    // forces, moment, Nusselt number on j = 0 (PSolver.cpp:1901-1983)
    double acc[7] = {0, 0, 0, 0, 0, 0, 0};
    for (int i = threadIdx.x; i <= n0 - 2; i += blockDim.x) {
        const long long k = i, kp = i + 1;
        const double PJ1 = P[k] * JAC[k], pj2 = P[kp] * JAC[kp];
        const double VJ1 = VORT[k] * JAC[k], VJ2 = VORT[kp] * JAC[kp];
        acc[0] += 0.5 * d0 * (PJ1 * ETX[k] + pj2 * ETX[kp]);
        acc[1] += 0.5 * d0 * (PJ1 * ETY[k] + pj2 * ETY[kp]);
        acc[2] += 0.5 * d0 * (VJ1 * ETY[k] + VJ2 * ETY[kp]);
        acc[3] += 0.5 * d0 * (VJ1 * ETX[k] + VJ2 * ETX[kp]);
        const double TJ1 = JAC[k] * (ETX[k] * ETX[k] + ETY[k] * ETY[k]);
        const double TJ2 = JAC[kp] * (ETX[kp] * ETX[kp] + ETY[kp] * ETY[kp]);
        const double fp1 = PJ1 * (X[k] * ETY[k] - Yc[k] * ETX[k]);
        const double fp2 = pj2 * (X[kp] * ETY[kp] - Yc[kp] * ETX[kp]);
        const double fv1 = VJ1 * (X[k] * ETX[k] + Yc[k] * ETY[k]);
        const double fv2 = VJ2 * (X[kp] * ETX[kp] + Yc[kp] * ETY[kp]);
        const double fh1 = TJ1 * (4 * Tn[k + ld] - 3 * Tn[k] - Tn[k + 2LL * ld]) / (2 * d1);
        const double fh2 = TJ2 * (4 * Tn[kp + ld] - 3 * Tn[kp] - Tn[kp + 2LL * ld]) / (2 * d1);
        acc[4] += 0.5 * d0 * (fp1 + fp2);
        acc[5] += 0.5 * d0 * (fv1 + fv2);
        acc[6] += 0.5 * (fh1 + fh2) * d0;
    }
    block_sum<7>(acc, red);
    if (threadIdx.x == 0) {
        const double pr_x = acc[0], pr_y = acc[1], vor_x = acc[2], vor_y = acc[3];
        const double cx = 2 * pr_x + (2.0 / Re) * vor_x;
        const double cy = 2 * pr_y - (2.0 / Re) * vor_y;
        const double sa = c.sa, ca = c.ca;
        sc[S_CLP] = 2 * pr_y * sa - 2 * pr_x * ca;
        sc[S_CDP] = 2 * pr_y * ca + 2 * pr_x * sa;
        sc[S_CLV] = -(2.0 / Re) * vor_y * sa - (2.0 / Re) * vor_x * ca;
        sc[S_CDV] = -(2.0 / Re) * vor_y * ca + (2.0 / Re) * vor_x * sa;
        sc[S_CL] = cy * sa - cx * ca;
        sc[S_CD] = cy * ca + cx * sa;
        sc[S_CM] = 2 * acc[4] - (2.0 / Re) * acc[5];
        const double ar = c.ar;
        if (!cav)
            sc[S_NU] = (2 * acc[6]) / (Pi * (3 * (1 + (1.0 / ar)) - sqrt((3 + (1.0 / ar)) * ((3.0 / ar) + 1))));
        else
            sc[S_NU] = -acc[6];
        sc[S_CIRC] = cav ? 0.0 : s_circ;
        is[I_TIME] = time_new;
        sc[S_TIME] = t_new;
    }
}

// ---------------------------------------------------------------------------
// dilatation, interior vorticity, dmax and the energy residual (PSolver.cpp:1807-1853)
__global__ void __launch_bounds__(NT, 3) k_diag(BatchDev b) {
    // a 32 x 16 tile, two cells per thread; all loads of both cells first
    const Tile t = b.jtiles[blockIdx.x];
    const CaseDev& c = b.cases[t.c];
    if (!b.iscal[(long long)t.c * NISCAL + I_ACTIVE]) return;  // uniform over the case
    const int ld = c.ld, W = c.W, per = c.periodic;
    const int i = t.i0 + (int)(threadIdx.x % TX);
    const double* U = plane(b, c, P_U);
    const double* V = plane(b, c, P_V);
    const double* XIX = plane(b, c, P_XIX);
    const double* XIY = plane(b, c, P_XIY);
    const double* ETX = plane(b, c, P_ETX);
    const double* ETY = plane(b, c, P_ETY);
    const double* TN = plane(b, c, P_T0 + (b.cur ^ 1));
    const double* TO = plane(b, c, P_T0 + b.cur);
    bool in[2];
    double ue[2], uw[2], un[2], us[2], ve[2], vw[2], vn[2], vs[2], xix[2], xiy[2], etx[2], ety[2], tn[2], to[2];
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const int j = t.j0 + (int)(threadIdx.x / TX) + h * TY;
        in[h] = i >= c.ilo && i <= c.ihi && j <= c.n1 - 2;
        const long long k = in[h] ? (long long)j * ld + i : (long long)ld + c.ilo;  // a safe cell when out
        ue[h] = U[k + 1]; uw[h] = U[k - 1]; un[h] = U[k + ld]; us[h] = U[k - ld];
        ve[h] = V[k + 1]; vw[h] = V[k - 1]; vn[h] = V[k + ld]; vs[h] = V[k - ld];
        xix[h] = XIX[k]; xiy[h] = XIY[k]; etx[h] = ETX[k]; ety[h] = ETY[k];
        tn[h] = TN[k]; to[h] = TO[k];
    }
    // 0.5 / d is 1 / (2 d) exactly: the dilatation's quotients become products
    const double h0 = 0.5 / c.d0, h1 = 0.5 / c.d1;
    double red[3] = {-1.0e300, 0.0, 0.0};
#pragma unroll
    for (int h = 0; h < 2; h++) {
        if (!in[h]) continue;
        const int j = t.j0 + (int)(threadIdx.x / TX) + h * TY;
        const double dil = xix[h] * (ue[h] - uw[h]) * h0 + etx[h] * (un[h] - us[h]) * h1 +
                           ety[h] * (vn[h] - vs[h]) * h1 + xiy[h] * (ve[h] - vw[h]) * h0;
        const double dv_dxi = h0 * (ve[h] - vw[h]);
        const double dv_det = h1 * (vn[h] - vs[h]);
        const double du_dxi = h0 * (ue[h] - uw[h]);
        const double du_det = h1 * (un[h] - us[h]);
        const double vort = (xix[h] * dv_dxi + etx[h] * dv_det) - (xiy[h] * du_dxi + ety[h] * du_det);
        store_mirrored(plane(b, c, P_VORT), ld, i, j, W, per, vort);
        store_mirrored(plane(b, c, P_DIL), ld, i, j, W, per, dil);
        const double dT = fabs(tn[h] - to[h]);
        red[0] = fmax(red[0], dil);
        red[1] += dT;
        red[2] = fmax(red[2], dT);
    }
    if (case_reduce<3, 0x5u>(b, t.c, blockIdx.x, c.jt_begin, c.jt_count, red) && threadIdx.x == 0) {
        double* sc = b.scal + (long long)t.c * NSCAL;
        int* is = b.iscal + (long long)t.c * NISCAL;
        sc[S_DMAX] = fmax(red[0], 0.0);
        sc[S_DTL1] = red[1];
        sc[S_DTMAX] = red[2];
        // steady residual: mean (|du| + |dv| + |dT|) / dt over the unknown cells
        const double ncell = (double)(c.ihi - c.ilo + 1) * (c.n1 - 2);
        sc[S_SR] = (sc[S_DUL1] + red[1]) / (c.dt * ncell);
        if (is[I_NSTEP] == 0) sc[S_SR0] = sc[S_SR];
        is[I_NSTEP] += 1;
    }
}

// stream function, a scan along j per column (PSolver.cpp:1789-1801)
__global__ void __launch_bounds__(BC_THREADS) k_si(BatchDev b) {
    const CaseDev& c = b.cases[blockIdx.x];
    const int ld = c.ld;
    double* SI = plane(b, c, P_SI);
    const double* U = plane(b, c, P_U);
    const double* V = plane(b, c, P_V);
    const double* XIX = plane(b, c, P_XIX);
    const double* XIY = plane(b, c, P_XIY);
    const double* JAC = plane(b, c, P_JAC);
    const int ncol = c.periodic ? c.W : c.n0;
    for (int i = threadIdx.x; i < ncol; i += blockDim.x) {
        double s = 0.0;
        store_mirrored(SI, ld, i, 0, c.W, c.periodic, 0.0);
        for (int j = 1; j < c.n1; j++) {
            const long long k = (long long)j * ld + i, kb = k - ld;
            const double ca = (XIX[k] * U[k] * fabs(JAC[k]) + XIX[kb] * U[kb] * fabs(JAC[kb]));
            const double cb = (XIY[k] * V[k] * fabs(JAC[k]) + XIY[kb] * V[kb] * fabs(JAC[kb]));
            s = s + (ca + cb) * 0.5 * c.d1;
            store_mirrored(SI, ld, i, j, c.W, c.periodic, s);
        }
    }
}

// condition of a graph while-loop: keep looping while `*flag > 0` and fewer than `maxc`
// iterations ran this step; `total` accumulates iterations over all steps
__global__ void k_loop_cond(cudaGraphConditionalHandle h, const int* flag, int* counter, int maxc,
                            int* total) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        const int n = ++(*counter);
        atomicAdd(total, 1);
        cudaGraphSetConditional(h, (*flag > 0 && n < maxc) ? 1u : 0u);
    }
}

// condition of a graph if-node: run the body when `*flag > 0`; `total` counts the runs
__global__ void k_if_cond(cudaGraphConditionalHandle h, const int* flag, int* total) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        const bool go = *flag > 0;
        if (go) atomicAdd(total, 1);
        cudaGraphSetConditional(h, go ? 1u : 0u);
    }
}

#undef AT
// ---------------------------------------------------------------------------
// Resident state <-> one contiguous staging buffer (so a state snapshot crosses PCIe as one
// copy per direction). Per case: the six state planes u, v, p, T, up, vp, each n1 rows of the
// stored columns (n0 for the cavity, W = n0 - 1 for the periodic O-grid), then 16 doubles:
// int time and int steps taken, then the first-step steady residual and continuity norm (the
// references of the relative residuals), then the time as a double. Unpacking writes the periodic halo mirrors too.
// blockIdx.x = case * 7 + m (m = 6: the counter slot); one warp per row.
__global__ void __launch_bounds__(256) k_state_pack(BatchDev b, double* stage, const long long* off, int to_stage) {
    const int c = blockIdx.x / 7, m = blockIdx.x % 7;
    const CaseDev& d = b.cases[c];
    const int nc = d.periodic ? d.W : d.n0;
    double* dst = stage + off[c] + (long long)m * d.n1 * nc;
    if (m == 6) {
        // the case's counters: the reference's int time, the steps taken, and the
        // first-step references of the relative residuals
        int* is = b.iscal + (long long)c * NISCAL;
        double* sc = b.scal + (long long)c * NSCAL;
        int* di = reinterpret_cast<int*>(dst);
        if (threadIdx.x == 0) {
            if (to_stage) {
                di[0] = is[I_TIME];
                di[1] = is[I_NSTEP];
                dst[1] = sc[S_SR0];
                dst[2] = sc[S_QL2_0];
                dst[3] = sc[S_TIME];
                for (int k = 4; k < 16; k++) dst[k] = 0.0;
            } else {
                is[I_TIME] = di[0];
                is[I_NSTEP] = di[1];
                sc[S_SR0] = dst[1];
                sc[S_QL2_0] = dst[2];
                sc[S_TIME] = dst[3];
            }
        }
        return;
    }
    const int ids[6] = {P_U, P_V, P_P, P_T0 + b.cur, P_UP0 + b.cur, P_VP0 + b.cur};
    double* P = plane(b, d, ids[m]);
    const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int j = threadIdx.x >> 5; j < d.n1; j += nw) {
        double* row = P + (long long)j * d.ld;
        double* srow = dst + (long long)j * nc;
        if (to_stage) {
            for (int i = lane; i < nc; i += 32) srow[i] = row[i];
        } else {
            for (int i = lane; i < nc; i += 32) store_mirrored(row, 0, i, 0, d.W, d.periodic, srow[i]);
        }
    }
}

}  // namespace cfd

// ---------------------------------------------------------------------------
// The sip9p() seam (cfd_sip_solve, PSolver.cpp:2067-2278): a one-case batch whose pressure
// stencil is the caller's nine stored planes instead of the grid's. The solve is the step's
// own BiCGStab + multigrid, run on the correction e of A (phi0 + e) = q with e = 0 on the
// boundary rows (and, without periodic xi, the boundary columns), as sip9p holds them.
namespace cfd {

// caller's [j][i] arrays -> case 0's padded planes: the stencil on the unknown cells (zero
// elsewhere, as k_assemble_p leaves it) in FP64 and as multigrid level 0, phi0 into P_SI and
// q into P_VORT at every stored point; a periodic case's halo columns take the wrap
__global__ void k_sip_pack(BatchDev b, SipIn in) {
    const CaseDev& c = b.cases[0];
    const int W = c.W, per = c.periodic;
    const int ncols = W + 2 * H;  // padded columns -H .. W + H - 1
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long long)c.n1 * ncols) return;
    const int j = (int)(e / ncols), col = (int)(e % ncols) - H;
    int i = col;  // the caller's column
    if (per) i = col < 0 ? col + W : (col >= W ? col - W : col);
    else if (col < 0 || col >= c.n0) return;
    const long long src = (long long)j * in.n0 + i;
    const long long k = (long long)j * c.ld + col;
    const bool unknown = j >= 1 && j <= c.n1 - 2 && i >= c.ilo && i <= c.ihi;
    const LevelDev& L0 = c.lev[0];
    const long long k0 = (long long)j * L0.ld + col;
#pragma unroll
    for (int q = 0; q < 9; q++) {
        const double v = unknown ? in.a[q][src] : 0.0;
        plane(b, c, P_AP + q)[k] = v;
        mplane(b, L0, M_AP + q)[k0] = (float)v;
    }
    plane(b, c, P_SI)[k] = in.phi[src];
    plane(b, c, P_VORT)[k] = in.q[src];
}

// r0 = q - A phi0 on the unknown cells (phi0's boundary values enter through the stencil),
// then the pressure solve's start as k_face_q leaves it for a step: r0 is the right-hand
// side, the shadow residual and the first preconditioner input; the iterate starts at zero
__global__ void __launch_bounds__(NT) k_sip_init(BatchDev b) {
    const Tile t = b.jtiles[blockIdx.x];
    const CaseDev& c = b.cases[t.c];
    const int tid = threadIdx.x, li = tid % TX, lj = tid / TX, i = t.i0 + li;
    const int ld = c.ld;
    const double* X = plane(b, c, P_SI);
    const double* Q = plane(b, c, P_VORT);
    const LevelDev& L0 = c.lev[0];
    double red[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const int j = t.j0 + lj + h * TY;
        if (i < c.ilo || i > c.ihi || j > c.n1 - 2) continue;
        const long long k = (long long)j * ld + i;
        const double ax = plane(b, c, P_AP)[k] * X[k] + plane(b, c, P_AE)[k] * X[k + 1] +
                          plane(b, c, P_AW)[k] * X[k - 1] + plane(b, c, P_AN)[k] * X[k + ld] +
                          plane(b, c, P_AS)[k] * X[k - ld] + plane(b, c, P_ANE)[k] * X[k + ld + 1] +
                          plane(b, c, P_ANW)[k] * X[k + ld - 1] + plane(b, c, P_ASE)[k] * X[k - ld + 1] +
                          plane(b, c, P_ASW)[k] * X[k - ld - 1];
        const double r = Q[k] - ax;
        plane(b, c, P_Q)[k] = r;
        plane(b, c, P_KR)[k] = r;
        mplane(b, L0, M_B)[(long long)j * L0.ld + i] = (float)r;
        red[0] += fabs(r);
        red[1] += r * r;
        red[2] = fmax(red[2], fabs(r));
    }
    if (case_reduce<3, 0x4u>(b, t.c, blockIdx.x, c.jt_begin, c.jt_count, red) && tid == 0) {
        double* sc = b.scal + (long long)t.c * NSCAL;
        int* is = b.iscal + (long long)t.c * NISCAL;
        sc[S_QL1] = red[0];
        sc[S_QL2] = sqrt(red[1]);
        sc[S_QMAX] = red[2];
        sc[S_RHO] = red[1];
        sc[S_ALPHA] = 1.0;
        sc[S_OMEGA] = 1.0;
        sc[S_BETA] = 0.0;
        sc[S_NB1] = red[0];
        sc[S_RL1] = red[0];
        is[I_PIT] = 0;
        is[I_PSTATUS] = 0;
        if (red[0] == 0.0 || !isfinite(red[0])) {
            is[I_PDONE] = 1;
            if (!isfinite(red[0])) is[I_STATUS] |= ST_NAN;
        } else {
            is[I_PDONE] = 0;
            atomicAdd(b.active, 1);
        }
    }
}

// phi = phi0 + e on the unknown cells of the caller's [j][i] array (a periodic case's seam
// column n0 - 1 repeats column 0); boundary values are left as the caller gave them
__global__ void k_sip_out(BatchDev b, double* phi, int n0) {
    const CaseDev& c = b.cases[0];
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long long)c.n1 * n0) return;
    const int j = (int)(e / n0), i = (int)(e % n0);
    const int col = (c.periodic && i == n0 - 1) ? 0 : i;
    if (j < 1 || j > c.n1 - 2 || col < c.ilo || col > c.ihi) return;
    const long long k = (long long)j * c.ld + col;
    phi[e] = plane(b, c, P_SI)[k] + plane(b, c, P_PCOR)[k];
}

}  // namespace cfd
