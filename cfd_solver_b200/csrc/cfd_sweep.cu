// cfd_sweep.cu -- the Chebyshev-Jacobi sweeps of the five u/v/T/up/vp systems
// (replacing gauss(), PSolver.cpp:2280-2446) as one persistent, pipelined kernel.
//
// One CTA sweeps one 32 x 16 tile of one case for all of its still-iterating fields.
// The fields stream through two shared-memory buffers: each field's x tile with its
// 2-cell halo, its right-hand side and (after the first sweep) the previous iterate
// arrive by tensor copies completed on the buffer's mbarrier, and the copies of field
// k+2 are issued as soon as field k has been read into registers, so they overlap the
// arithmetic of field k and the wait for field k+1. The first field also brings alpha,
// beta, gamma; every thread turns its own cells' values into the operator (E, G, B and
// the two inverse diagonals) in place, in a thread-private part of shared memory that
// needs no barrier and costs no registers.
//
// A warp owns four consecutive rows of the tile, a lane one column: the thread reads its
// eight-row x five-column window once into registers, so its four cells cost ten
// shared-memory loads each instead of twenty-five. Each cell's off-centre sum (25-point, or
// 9-point on the near-wall cells) is formed just before its update, and the per-CTA
// constants and each field's warp residual sums sit in shared memory, so the kernel holds
// its 128 registers with little spilling. The per-tile L1 residuals go to one partial row
// per tile that k_sweep_fin sums per case in a fixed order after the launch.
//
// Three modes share the code:
//   SW_F64    FP64 iterates x_k (the plain path);
//   SW_MX0    first sweep of the precision form: the residual r = rhs - A x0 in FP64
//             from the FP64 iterate, stored as FP32 together with the first FP32
//             correction d_1 = g D^-1 r;
//   SW_MX     later sweeps of the precision form on the FP32 correction d_k for
//             A d = r (x = x0 + d is formed by k_mom_update after the last sweep).
// The stop rule is the reference's (relative L1 residual of the system before the
// sweep, PSolver.cpp:2318-2330), evaluated with deterministic per-case reductions.
//
// Chebyshev acceleration: with the Jacobi value xJ = (rhs - sum_nb a_nb x_k) / ap the
// three-term recurrence is
//     x_{k+1} = w_{k+1} (x_k + g (xJ - x_k) - x_{k-1}) + x_{k-1},  g = 2 / (a + b),
// w_1 = 1, w_2 = 1 / (1 - 1 / (2 s^2)), w_{k+1} = 1 / (1 - w_k / (4 s^2)), s = (b + a) / (b - a),
// for eigenvalues of D^-1 A in [a, b] (bounds computed per case on the host).
// x_{k+1} overwrites x_{k-1} in place, so the iterates ping-pong between the solution
// buffer and the scratch; sweeps come in pairs and end in the solution buffer.
//
// Per cell the operator is fixed by E = dt alpha/(Re dxi0^2), G = dt gamma/(Re dxi1^2) and
// B = dt beta/(Re dxi0 dxi1): 4th-order rows (PSolver.cpp:791-821) have
//   ae = aw = -4/3 E, aee = aww = E/12, an = as = -4/3 G, ann = ass = G/12,
//   ane = asw = 8/9 B, anw = ase = -8/9 B, annee = assww = B/72, annww = assee = -B/72,
//   anne = assw = anee = asww = -B/9, annw = asse = anww = asee = B/9, ap = 1 + 5/2 (E + G);
// 9-point rows (PSolver.cpp:766-775): ae = aw = -E, an = as = -G, ane = asw = B/2,
// anw = ase = -B/2, ap = 1 + 2 (E + G), with the wall-row couplings folded out on the
// O-grid (PSolver.cpp:851-882). The T system divides E, G, B by Pr.
#include "cfd_bulk.cuh"
#include "cfd_common.cuh"
#include "cfd_reduce.cuh"
#include "cfd_sweep.cuh"

namespace cfd {

namespace {

template <int MODE>
struct SwCfg;
template <>
struct SwCfg<SW_F64> {
    using XT = double;  // x tile (with halo)
    using RT = double;  // right-hand side / residual tile
    using ST = double;  // arithmetic of the sweep
    static constexpr int XW = TX + 4, XO = 2;  // halo tile row length, column of cell 0 in it
    static constexpr bool PREV = true;
};
template <>
struct SwCfg<SW_MX0> {
    using XT = double;
    using RT = double;
    using ST = double;
    static constexpr int XW = TX + 4, XO = 2;
    static constexpr bool PREV = false;
};
template <>
struct SwCfg<SW_MX> {
    using XT = float;
    using RT = float;
    using ST = float;
    static constexpr int XW = TX + 8, XO = 4;  // FP32 boxes start 4 columns left (16-byte x)
    static constexpr bool PREV = true;
};

constexpr int SW_HALO_ROWS = TYJ + 4;
constexpr int SW_CELLS = TX * TYJ;
constexpr int align128(int x) { return (x + 127) / 128 * 128; }

// shared-memory layout: two field buffers, then alpha/beta/gamma (FP64, 3 planes) which
// every thread overwrites with its cells' operator (3 planes of ST: E, G, B -- in place for
// FP64, behind them for FP32, whose 4-byte slots would overlap other threads' unread 8-byte
// inputs), then the two inverse diagonals 1/ap_u, 1/ap_T in FP32. The diagonal only scales
// each Jacobi correction (the residual is exact in ST), so its precision moves no fixed
// point; holding it in FP32 lets five CTAs share an SM.
template <int MODE>
struct SwLayout {
    using C = SwCfg<MODE>;
    static constexpr unsigned XBYTES = C::XW * SW_HALO_ROWS * sizeof(typename C::XT);
    static constexpr unsigned RBYTES = SW_CELLS * sizeof(typename C::RT);
    static constexpr unsigned PBYTES = SW_CELLS * sizeof(typename C::XT);
    static constexpr unsigned MBYTES = 3 * SW_CELLS * sizeof(double);
    static constexpr int X = 0;
    static constexpr int RHS = align128(XBYTES);
    static constexpr int PREV = RHS + align128(RBYTES);
    static constexpr int BUF = PREV + (C::PREV ? align128(PBYTES) : 0);
    static constexpr int MET = 2 * BUF;
    static constexpr int OPS = sizeof(typename C::ST) == 8 ? MET : MET + (int)MBYTES;
    static constexpr int RAP = OPS + 3 * SW_CELLS * (int)sizeof(typename C::ST);  // 1/ap_u, 1/ap_T (FP32)
    static constexpr int TOTAL = RAP + 2 * SW_CELLS * (int)sizeof(float);
};

// FP64 plane of field f's iterate for state parity nxt (u*, v*, T, up, vp)
__device__ __forceinline__ int sw_iter_plane(int f, int nxt) { return f < 2 ? P_US + f : P_T0 + 2 * (f - 2) + nxt; }

// issue the tensor copies of field f of tile t into buffer `sm` (with alpha, beta, gamma)
template <int MODE>
__device__ __forceinline__ void sw_issue(const Tile& t, int f, int sweep, int nxt, const char* maps,
                                         unsigned char* sm, unsigned char* met, uint64_t* bar, bool flip) {
    using L = SwLayout<MODE>;
    const int pa = sw_iter_plane(f, nxt);
    unsigned bytes = L::XBYTES + L::RBYTES + (met ? L::MBYTES : 0u);
    bool prev = false;
    int xs = 0, ps = 0;
    if (MODE == SW_F64) {
        // x_s is in the iterate plane when s is even, unless the solve started in the scratch plane
        const bool to_scratch = ((sweep & 1) == 0) != flip;
        xs = to_scratch ? pa : P_BU + f;
        ps = to_scratch ? P_BU + f : pa;
        prev = sweep > 0;
    } else if (MODE == SW_MX0) {
        xs = pa;
    } else {
        const int to_scratch = (sweep & 1) == 0;
        xs = to_scratch ? X_DA + f : X_DB + f;
        ps = to_scratch ? X_DB + f : X_DA + f;
        prev = sweep > 1;
    }
    if (prev) bytes += L::PBYTES;
    fence_proxy_async_smem();
    mbar_arrive_expect_tx(bar, bytes);
    if (MODE == SW_MX) {
        tma_load_3d(sm + L::X, maps + TMAP_X32_HALO, t.i0, t.j0 - 2, xs, bar);
        tma_load_3d(sm + L::RHS, maps + TMAP_X32_TILE, t.i0 + 4, t.j0, X_R + f, bar);
        if (prev) tma_load_3d(sm + L::PREV, maps + TMAP_X32_TILE, t.i0 + 4, t.j0, ps, bar);
    } else {
        tma_load_3d(sm + L::X, maps + TMAP_F64_HALO, t.i0, t.j0 - 2, xs, bar);
        tma_load_3d(sm + L::RHS, maps + TMAP_F64_TILE, t.i0 + 2, t.j0, P_RU + f, bar);
        if (prev) tma_load_3d(sm + L::PREV, maps + TMAP_F64_TILE, t.i0 + 2, t.j0, ps, bar);
    }
    // alpha, beta, gamma: three consecutive planes in one box
    if (met) tma_load_3d(met, maps + TMAP_F64_TILE3, t.i0 + 2, t.j0, P_ALPH, bar);
}

// off-centre sums of the u-type operator for the cell whose window centre row is `r0 + 2`:
// the 25-point (4th-order) rows and the 9-point near-wall rows
#define WX(dy, dx) w[r0 + 2 + (dy)][2 + (dx)]
template <typename ST>
__device__ __forceinline__ ST sw_sum25(const ST (&w)[8][5], int r0, ST E, ST G, ST B) {
    const ST ex = ST(-4.0 / 3.0) * (WX(0, 1) + WX(0, -1)) + ST(1.0 / 12.0) * (WX(0, 2) + WX(0, -2));
    const ST gy = ST(-4.0 / 3.0) * (WX(1, 0) + WX(-1, 0)) + ST(1.0 / 12.0) * (WX(2, 0) + WX(-2, 0));
    const ST bx = ST(8.0 / 9.0) * (WX(1, 1) + WX(-1, -1) - WX(1, -1) - WX(-1, 1)) +
                  ST(1.0 / 72.0) * (WX(2, 2) + WX(-2, -2) - WX(2, -2) - WX(-2, 2)) +
                  ST(1.0 / 9.0) * (WX(2, -1) + WX(-2, 1) + WX(1, -2) + WX(-1, 2) - WX(2, 1) - WX(-2, -1) -
                                   WX(1, 2) - WX(-1, -2));
    return E * ex + G * gy + B * bx;
}
template <typename ST>
__device__ __forceinline__ ST sw_sum9(const ST (&w)[8][5], int r0, ST E, ST G, ST B, bool drop_s, bool drop_n) {
    ST s = -E * (WX(0, 1) + WX(0, -1));
    const ST n = -G * WX(1, 0) + ST(0.5) * B * (WX(1, 1) - WX(1, -1));
    const ST so = -G * WX(-1, 0) + ST(0.5) * B * (WX(-1, -1) - WX(-1, 1));
    if (!drop_n) s += n;
    if (!drop_s) s += so;
    return s;
}
#undef WX

template <int MODE>
__device__ __forceinline__ void sweep_tile(const BatchDev& b, unsigned char* sm, uint64_t* bar) {
    using C = SwCfg<MODE>;
    using L = SwLayout<MODE>;
    using XT = typename C::XT;
    using RT = typename C::RT;
    using ST = typename C::ST;
    const Tile t = b.jtiles[blockIdx.x];
    const CaseDev& c = b.cases[t.c];
    // one word (the case's I_MWORD, kept per tile so that it is read in the same round trip as
    // the tile): the fields still iterating, those whose first iterate is in the scratch plane
    // (FP64 form), and the sweeps done (the same for every still-active field of the case)
    const int word = b.tword[blockIdx.x];
    const int mask = word & ((1 << NFIELD) - 1);
    if (mask == 0) return;  // uniform over the case's CTAs
    const int sweep = word >> (2 * NFIELD);
    const int flipm = MODE == SW_F64 ? (word >> NFIELD) & ((1 << NFIELD) - 1) : 0;
    const int tid = threadIdx.x, lane = tid & 31, wrp = tid >> 5;
    const int nxt = b.cur ^ 1;
    const int nf = __popc(mask);
    const char* maps = b.tmaps + (size_t)t.c * TMAP_STRIDE;
    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        fence_mbar_init();
        const int m1 = mask & (mask - 1);
        const int f0 = __ffs(mask) - 1;
        sw_issue<MODE>(t, f0, sweep, nxt, maps, sm, sm + L::MET, &bar[0], (flipm >> f0) & 1);
        if (m1) {
            const int f1 = __ffs(m1) - 1;
            sw_issue<MODE>(t, f1, sweep, nxt, maps, sm + L::BUF, nullptr, &bar[1], (flipm >> f1) & 1);
        }
    }
    // per-case constants (uniform)
    const double* sc = b.scal + (long long)t.c * NSCAL;
    const bool weighted = MODE == SW_MX ? true : sweep > 0;
    const bool has_prev = MODE == SW_MX ? sweep > 1 : (MODE == SW_F64 && sweep > 0);
    // per-CTA constants of the sweeps (Chebyshev step g and weight w of the u-type and T
    // systems, 1/Pr) and the tile's per-warp residual sums, in shared memory
    __shared__ ST sconst[5];
    __shared__ double sred[SW_WARPS * NFIELD];
    const double rPr64 = c.rPr;
    if (tid < SW_WARPS * NFIELD) sred[tid] = 0.0;
    if (tid == 0) {
        sconst[0] = (ST)(2.0 / (c.cheb_a[0] + c.cheb_b[0]));
        sconst[1] = (ST)(2.0 / (c.cheb_a[1] + c.cheb_b[1]));
        sconst[2] = weighted ? (ST)sc[S_CW0] : ST(1);
        sconst[3] = weighted ? (ST)sc[S_CW1] : ST(1);
        sconst[4] = (ST)rPr64;
    }
    const int ld = c.ld, xld = c.xld, W = c.W, per = c.periodic;
    const int i = t.i0 + lane;
    bool inq[SW_ROWS], nearw[SW_ROWS], drop_s[SW_ROWS], drop_n[SW_ROWS];
#pragma unroll
    for (int q = 0; q < SW_ROWS; q++) {
        const int j = t.j0 + wrp * SW_ROWS + q;
        inq[q] = i >= c.ilo && i <= c.ihi && j <= c.n1 - 2;
        nearw[q] = j == 1 || j == c.n1 - 2 || (c.profile == CAVITY && (i == 1 || i == c.n0 - 2));
        drop_s[q] = c.profile == OGRID && j == 1;
        drop_n[q] = c.profile == OGRID && j == c.n1 - 2;
    }
    __syncthreads();

    ST* OPS = reinterpret_cast<ST*>(sm + L::OPS);
    float* RAP = reinterpret_cast<float*>(sm + L::RAP);
    // the thread's periodic mirror column (written alongside column i), or none
    const int mcol = mirror_col(i, W, per);
    bool ok = true;
    int k = 0;
    for (int fm = mask; fm; fm &= fm - 1, k++) {
        const int f = __ffs(fm) - 1;
        const int bi = k & 1;
        // one thread polls the buffer's mbarrier; the barrier after it orders the other
        // threads' reads of the landed copies after its observation (the others wait in the
        // barrier instead of spending issue slots on polls)
        bool got = true;
        if (tid == 0) got = mbar_wait_bounded(&bar[bi], (k >> 1) & 1, b.wait_polls);
        ok = __syncthreads_and(got) && ok;
        if (!ok) break;
        const unsigned char* buf = sm + bi * L::BUF;
        if (k == 0) {
            // alpha, beta, gamma of the thread's own cells -> E, G, B, 1/ap_u, 1/ap_T
            const double* MET = reinterpret_cast<const double*>(sm + L::MET);
            const double kE = c.swk[0], kG = c.swk[1], kB = c.swk[2];
#pragma unroll
            for (int q = 0; q < SW_ROWS; q++) {
                const int o = (wrp * SW_ROWS + q) * TX + lane;
                const double E = kE * MET[o], B = kB * MET[SW_CELLS + o], G = kG * MET[2 * SW_CELLS + o];
                const double D = (nearw[q] ? 2.0 : 2.5) * (E + G);
                OPS[o] = (ST)E;
                OPS[SW_CELLS + o] = (ST)G;
                OPS[2 * SW_CELLS + o] = (ST)B;
                // the correctly rounded reciprocal (the value 1.0 / x gives, in fewer instructions)
                RAP[o] = (float)__drcp_rn(1.0 + D);
                RAP[SW_CELLS + o] = (float)__drcp_rn(1.0 + D * rPr64);
            }
        }
        const bool isT = f == F_T;
        const XT* X = reinterpret_cast<const XT*>(buf + L::X);
        const RT* R = reinterpret_cast<const RT*>(buf + L::RHS);
        const XT* P = reinterpret_cast<const XT*>(buf + L::PREV);
        // the thread's window: rows wrp*4 - 2 .. wrp*4 + 5, columns lane - 2 .. lane + 2
        ST w[8][5];
        ST rhs[SW_ROWS], xm[SW_ROWS];
#pragma unroll
        for (int q = 0; q < SW_ROWS; q++) {
            const int o = (wrp * SW_ROWS + q) * TX + lane;
            rhs[q] = (ST)R[o];
            xm[q] = has_prev ? (ST)P[o] : ST(0);
        }
#pragma unroll
        for (int rr = 0; rr < 8; rr++)
#pragma unroll
            for (int cl = 0; cl < 5; cl++) w[rr][cl] = (ST)X[(wrp * SW_ROWS + rr) * C::XW + lane + cl + C::XO - 2];
        __syncthreads();  // the buffer has been read: refill it with the field after next
        if (tid == 0) {
            int nx = fm & (fm - 1);
            nx &= nx - 1;
            if (nx) {
                const int f2 = __ffs(nx) - 1;
                sw_issue<MODE>(t, f2, sweep, nxt, maps, sm + bi * L::BUF, nullptr, &bar[bi], (flipm >> f2) & 1);
            }
        }

        const ST g = sconst[isT ? 1 : 0], wgt = sconst[isT ? 3 : 2];
        const ST scale = isT ? sconst[4] : ST(1);
        // the reference's T solve passes atnw in the annw slot (PSolver.cpp:1290): the
        // (i-1, j+2) coefficient of the 25-point T rows becomes anw = -8/9 B instead of B/9
        const bool tbug = isT && !c.fix_T_annw;
        const int rapoff = isT ? SW_CELLS : 0;
        double* dst64 = nullptr;
        float* dst32 = nullptr;
        float* res32 = nullptr;
        int dld = ld;
        if (MODE == SW_F64) {
            dst64 = plane(b, c, (((sweep & 1) == 0) != (((flipm >> f) & 1) != 0)) ? P_BU + f : sw_iter_plane(f, nxt));
        } else if (MODE == SW_MX0) {
            dst32 = xplane(b, c, X_DB + f);
            res32 = xplane(b, c, X_R + f);
            dld = xld;
        } else {
            dst32 = xplane(b, c, (sweep & 1) == 0 ? X_DB + f : X_DA + f);
            dld = xld;
        }
        double racc = 0.0;
#pragma unroll
        for (int q = 0; q < SW_ROWS; q++) {
            const int o = (wrp * SW_ROWS + q) * TX + lane;
            const ST E = OPS[o], G = OPS[SW_CELLS + o], B = OPS[2 * SW_CELLS + o];
            // off-centre sum: the 25-point form, or the 9-point form on the near-wall cells
            ST sm_ = nearw[q] ? sw_sum9<ST>(w, q, E, G, B, drop_s[q], drop_n[q]) : sw_sum25<ST>(w, q, E, G, B);
            if (tbug && !nearw[q]) sm_ -= B * w[q + 4][1];
            sm_ *= scale;
            const ST D = (nearw[q] ? ST(2) : ST(2.5)) * (E + G);
            const ST ap = ST(1) + D * scale;
            const ST rap = (ST)RAP[rapoff + o];
            const ST xk = w[q + 2][2];
            const ST res = rhs[q] - ap * xk - sm_;
            racc += inq[q] ? fabs((double)res) : 0.0;
            const long long kk = (long long)(t.j0 + wrp * SW_ROWS + q) * dld;
            if (MODE == SW_MX0) {
                const float d1 = (float)(g * res * rap), rr = (float)res;
                if (inq[q]) {
                    dst32[kk + i] = d1;
                    res32[kk + i] = rr;
                    if (mcol > -1000000) {
                        dst32[kk + mcol] = d1;
                        res32[kk + mcol] = rr;
                    }
                }
            } else {
                ST xn = xk + g * res * rap;
                if (weighted) xn = wgt * (xn - xm[q]) + xm[q];
                if (inq[q]) {
                    if (MODE == SW_F64) {
                        dst64[kk + i] = (double)xn;
                        if (mcol > -1000000) dst64[kk + mcol] = (double)xn;
                    } else {
                        dst32[kk + i] = (float)xn;
                        if (mcol > -1000000) dst32[kk + mcol] = (float)xn;
                    }
                }
            }
        }
        // the field's warp residual (lane 0), summed as the tile's partial after the last field
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) racc += __shfl_down_sync(0xffffffffu, racc, o);
        if (lane == 0) sred[wrp * NFIELD + f] = racc;
    }
    if (!ok) {
        if (tid == 0) {
            atomicExch(b.error, 1);
            // let the copies still in flight land before the CTA leaves (the long default limit)
            for (int m = k; m < nf && m < k + 2; m++) mbar_wait_bounded(&bar[m & 1], (m >> 1) & 1);
        }
        return;
    }
    // the tile's partial L1 residuals, one row per tile (summed per case by k_sweep_fin):
    // the tile's four warp sums in a fixed order
    __syncthreads();
    if (tid < NFIELD) {
        double x = 0.0;
#pragma unroll
        for (int w = 0; w < SW_WARPS; w++) x += sred[w * NFIELD + tid];
        b.partial[(long long)blockIdx.x * PSTRIDE + tid] = x;
    }
}

}  // namespace

__global__ void __launch_bounds__(SW_THREADS, 4) k_sweep_f64(BatchDev b) {
    extern __shared__ __align__(128) unsigned char swraw[];
    __shared__ __align__(8) uint64_t bar[2];
    unsigned char* sm = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(swraw) + 127) & ~uintptr_t(127));
    sweep_tile<SW_F64>(b, sm, bar);
}

// precision form, the step's first sweep (every still-iterating field of every case starts
// at sweep 0 together): the FP64 residual r = rhs - A x0 and the first FP32 correction
__global__ void __launch_bounds__(SW_THREADS, 4) k_sweep_mx0(BatchDev b) {
    extern __shared__ __align__(128) unsigned char swraw[];
    __shared__ __align__(8) uint64_t bar[2];
    unsigned char* sm = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(swraw) + 127) & ~uintptr_t(127));
    sweep_tile<SW_MX0>(b, sm, bar);
}

// precision form, the later sweeps: FP32 throughout. Compiled apart from the FP64 first
// sweep it needs 80 registers and no spills, so six CTAs (37 KB of shared memory each)
// share an SM instead of four
__global__ void __launch_bounds__(SW_THREADS, 6) k_sweep_mx1(BatchDev b) {
    extern __shared__ __align__(128) unsigned char swraw[];
    __shared__ __align__(8) uint64_t bar[2];
    unsigned char* sm = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(swraw) + 127) & ~uintptr_t(127));
    sweep_tile<SW_MX>(b, sm, bar);
}

// What the case's bookkeeping after a sweep reads, loaded by thread 0 of k_sweep_fin at its
// start so that the loads overlap the partial sums (the sweep count, the fields still
// iterating and their start planes come from the case's packed word).
struct FinIn {
    double mr0[NFIELD];   // first-sweep residuals (the rule's reference)
    double cw[2];         // Chebyshev weights of the sweep just done
    double ca[2], cb[2];  // eigenvalue bounds (u-type, T)
    double tol, atol;
    unsigned long long ncell;
};

__device__ __forceinline__ void fin_load(const BatchDev& b, const CaseDev& c, int cid, FinIn& in) {
    const double* scw = b.scal + (long long)cid * NSCAL;
#pragma unroll
    for (int f = 0; f < NFIELD; f++) in.mr0[f] = scw[S_MR0 + f];
#pragma unroll
    for (int ty = 0; ty < 2; ty++) {
        in.cw[ty] = scw[S_CW0 + ty];
        in.ca[ty] = c.cheb_a[ty];
        in.cb[ty] = c.cheb_b[ty];
    }
    in.tol = c.tol_mom;
    in.atol = c.atol_mom;
    in.ncell = (unsigned long long)(c.ihi - c.ilo + 1) * (c.n1 - 2);
}

// the case's bookkeeping after a sweep (thread 0 of k_sweep_fin): stop decisions, the next
// Chebyshev weights, the sweep kernel's new word (returned) and the traffic counters
__device__ __forceinline__ int fin_case(const BatchDev& b, int cid, int* is, int word, const double (&v)[NFIELD],
                                        const FinIn& in) {
    double* scw = b.scal + (long long)cid * NSCAL;
    const int mask = word & ((1 << NFIELD) - 1), flipm = (word >> NFIELD) & ((1 << NFIELD) - 1);
    const int sweep = word >> (2 * NFIELD);
    int nmask = mask;
    // the rule is tested after every sweep (on the residual of the sweep's input iterate; the
    // sweep's output, one sweep further, is the result)
#pragma unroll
    for (int f = 0; f < NFIELD; f++) {
        if (!(mask & (1 << f))) continue;
        const double mr0 = sweep == 0 ? ((v[f] != 0.0) ? v[f] : 1.0) : in.mr0[f];
        if (sweep == 0) {
            scw[S_MR0 + f] = mr0;
            is[I_MNEXT0 + f] = 0;  // next step: start in the iterate plane, unless this solve stops odd
        }
        scw[S_MR + f] = v[f];
        is[I_MIT0 + f] = sweep + 1;
        bool done = (v[f] / mr0 < in.tol) || (v[f] <= in.atol);
        if (!isfinite(v[f])) {
            is[I_STATUS] |= ST_NAN;
            done = true;
        }
        if (done) {
            // the result x_{sweep+1} is in the scratch plane when the sweep's parity equals
            // the solve's start plane flag; predict the next step's start from this parity
            is[I_MDONE0 + f] = 1;
            is[I_MODD0 + f] = (sweep & 1) == ((flipm >> f) & 1);
            is[I_MNEXT0 + f] = (sweep & 1) == 0;
            atomicSub(b.mactive, 1);
            nmask &= ~(1 << f);
        }
    }
    const int nword = nmask | (flipm << NFIELD) | ((sweep + 1) << (2 * NFIELD));
    is[I_MWORD] = nword;
#pragma unroll
    for (int ty = 0; ty < 2; ty++) {  // Chebyshev weight of the next sweep
        const double ca = in.ca[ty], cb = in.cb[ty];
        const double s2 = ((cb + ca) / (cb - ca)) * ((cb + ca) / (cb - ca));
        scw[S_CW0 + ty] = (sweep == 0) ? 1.0 / (1.0 - 1.0 / (2.0 * s2)) : 1.0 / (1.0 - in.cw[ty] / (4.0 * s2));
    }
    // algorithmic-traffic counters (cells and field-cells swept)
    const unsigned long long nf = (unsigned long long)__popc(mask) * in.ncell;
    atomicAdd(&b.work[0], nf);
    atomicAdd(&b.work[1], in.ncell);
    if (sweep == 0) atomicAdd(&b.work[2], nf);
    if (sweep == 1) atomicAdd(&b.work[3], nf);
    return nword;
}

// per case after every sweep launch: sum the tile rows in a fixed order, count the
// sweep, decide the stop (after every sweep), advance the Chebyshev weights, and hand every
// tile of the case the sweep kernel's new word (the stores spread over the CTA's threads:
// a 1025 x 1025 case has 2,048 tiles)
__global__ void __launch_bounds__(SWF_THREADS) k_sweep_fin(BatchDev b) {
    __shared__ double red[NFIELD * 32];
    __shared__ int s_word;
    const int cid = blockIdx.x;
    const CaseDev& c = b.cases[cid];
    int* is = b.iscal + (long long)cid * NISCAL;
    const int word = is[I_MWORD];
    if (!(word & ((1 << NFIELD) - 1))) return;
    const int tid = threadIdx.x;
    FinIn in;
    if (tid == 0) fin_load(b, c, cid, in);
    double v[NFIELD] = {0.0, 0.0, 0.0, 0.0, 0.0};
    const int np = c.jt_count;  // one row per tile
    for (int e = tid; e < np; e += blockDim.x) {
        const double* src = b.partial + ((long long)c.jt_begin + e) * PSTRIDE;
#pragma unroll
        for (int f = 0; f < NFIELD; f++) v[f] += src[f];
    }
    block_sum<NFIELD>(v, red);
    if (tid == 0) s_word = fin_case(b, cid, is, word, v, in);
    __syncthreads();
    // the new word into every tile of the case, by all threads
    const int nword = s_word;
    for (int k = tid; k < c.jt_count; k += blockDim.x) b.tword[c.jt_begin + k] = nword;
}


size_t sweep_smem_f64() { return (size_t)SwLayout<SW_F64>::TOTAL + 128; }
size_t sweep_smem_mx0() { return (size_t)SwLayout<SW_MX0>::TOTAL + 128; }
size_t sweep_smem_mx1() { return (size_t)SwLayout<SW_MX>::TOTAL + 128; }

// x0 += d for every field of the precision form (after the last sweep, d_final in X_DA)
// A solve whose result is in the scratch plane (FP64 form; it stopped after a sweep count of
// the other parity than predicted): copy it into the iterate plane. 32 x 16 tiles, two
// cells per thread; the CTAs of a case with no such solve leave at once.
__global__ void __launch_bounds__(NT) k_mom_fix(BatchDev b) {
    const Tile t = b.jtiles[blockIdx.x];
    const int* is = b.iscal + (long long)t.c * NISCAL;
    int odd = 0;  // solves whose result is in the scratch plane: stopped there, or ran to the
                  // sweep cap (an even count) after starting there
#pragma unroll
    for (int f = 0; f < NFIELD; f++) odd |= (is[I_MDONE0 + f] ? is[I_MODD0 + f] != 0 : is[I_MFLIP0 + f] != 0) << f;
    if (!odd || !is[I_ACTIVE]) return;
    const CaseDev& c = b.cases[t.c];
    const int nxt = b.cur ^ 1;
    const int i = t.i0 + (int)(threadIdx.x % TX);
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const int j = t.j0 + (int)(threadIdx.x / TX) + h * TY;
        if (i < c.ilo || i > c.ihi || j > c.n1 - 2) continue;
        const long long k = (long long)j * c.ld + i;
#pragma unroll
        for (int f = 0; f < NFIELD; f++)
            if (odd & (1 << f))
                store_mirrored(plane(b, c, sw_iter_plane(f, nxt)), c.ld, i, j, c.W, c.periodic, plane(b, c, P_BU + f)[k]);
    }
}

__global__ void __launch_bounds__(NT) k_mom_update(BatchDev b) {
    const Tile t = b.ftiles[blockIdx.x];
    const CaseDev& c = b.cases[t.c];
    if (!b.iscal[(long long)t.c * NISCAL + I_ACTIVE]) return;  // uniform over the case
    const int i = t.i0 + (int)(threadIdx.x % TX), j = t.j0 + (int)(threadIdx.x / TX);
    if (i < c.ilo || i > c.ihi || j > c.n1 - 2) return;
    const int nxt = b.cur ^ 1;
    const long long k = (long long)j * c.ld + i, kx = (long long)j * c.xld + i;
    double x[NFIELD];
    float d[NFIELD];
#pragma unroll
    for (int f = 0; f < NFIELD; f++) {
        x[f] = plane(b, c, sw_iter_plane(f, nxt))[k];
        // the correction after an even number of sweeps is in X_DA, after an odd one in X_DB
        d[f] = xplane(b, c, (b.iscal[(long long)t.c * NISCAL + I_MODD0 + f] ? X_DB : X_DA) + f)[kx];
    }
#pragma unroll
    for (int f = 0; f < NFIELD; f++)
        store_mirrored(plane(b, c, sw_iter_plane(f, nxt)), c.ld, i, j, c.W, c.periodic, x[f] + (double)d[f]);
}

}  // namespace cfd
