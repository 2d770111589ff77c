// cfd_common.cuh -- device data layout shared by the CUDA kernels and the host runtime.
//
// A batch packs many cases (grids of uneven size and parameters) into one FP64
// arena and one FP32 arena. Each case owns NPLANES FP64 planes; plane `k` of
// case `c` stores point (i, j) at
//     f64[c.base + k * c.ps + j * c.ld + H + i]
// with j in [0, n1) (all rows of the reference, boundary rows included) and
// i in [-H, W + H): W = n0 - 1 unique columns for the periodic O-grid (the
// reference's seam column n0-1 is the halo column i = W, the copy of i = 0),
// W = n0 for the cavity. The two halo columns on each side hold the periodic
// wrap; every kernel that writes column 0, 1, W-2 or W-1 of a periodic case
// also writes its halo mirror, so stencils never use modular indexing.
//
// Work is split into 32 x 8 tiles of the unknown cells (j in [1, n1-2],
// i in [ilo, ihi]); a tile table lists (case, i0, j0, tile-in-case) for every
// tile of every case, so one launch covers the whole batch.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace cfd {

constexpr int H = 2;          // halo columns on each side
constexpr int TX = 32;        // tile width (cells), one warp per tile row
constexpr int TY = 8;         // tile height
constexpr int TYJ = 16;       // tile height of the u/v/T sweep kernel (two cells per thread)
constexpr int NT = TX * TY;   // threads per tile kernel
constexpr int MAXLEV = 12;    // multigrid levels per case
constexpr int BC_THREADS = 256;

enum Profile { OGRID = 0, CAVITY = 1 };

// FP64 plane slots of a case
enum Plane {
    P_X, P_Y, P_XIX, P_XIY, P_ETX, P_ETY, P_ALPH, P_BETA, P_GAM, P_JAC,  // grid
    P_AP, P_AE, P_AW, P_AN, P_AS, P_ANE, P_ANW, P_ASE, P_ASW,            // pressure stencil
    P_U, P_V, P_P, P_T0, P_T1, P_UP0, P_UP1, P_VP0, P_VP1,               // state (T, up, vp double-buffered)
    P_US, P_VS,                                                          // u*, v*
    P_RU, P_RV, P_RT, P_RUP, P_RVP,                                      // right-hand sides
    P_BU, P_BV, P_BT, P_BUP, P_BVP,                                      // Jacobi scratch
    P_Q, P_PCOR, P_VORT, P_SI, P_DIL,                                    // q, pcor, diagnostics
    P_VEC,    // rows 0..3: normals xnix, xniy, xnox, xnoy (one value per column)
    P_KR, P_KRH, P_KP, P_KV, P_KS, P_KT, P_KPH, P_KSH,                   // BiCGStab vectors
    NPLANES
};

// FP32 multigrid planes of one level
enum MgPlane { M_AP, M_AE, M_AW, M_AN, M_AS, M_ANE, M_ANW, M_ASE, M_ASW, M_X, M_B, M_R, NMG };

// momentum / energy systems solved each step
enum Field { F_U, F_V, F_T, F_UP, F_VP, NFIELD };

// FP32 planes of the precision form (per case, after its multigrid levels): the two
// correction buffers and the FP32 residual of each of the five systems. Column i of
// row j of plane k sits at f32[c.xbase + k * c.xps + j * c.xld + H32 + i]; the 4
// columns left of column 0 keep every tensor box of these planes 16-byte aligned.
enum MxPlane { X_DA = 0, X_DB = NFIELD, X_R = 2 * NFIELD, NXPLANES = 3 * NFIELD };
constexpr int H32 = 4;

// per-case CUtensorMaps (128 bytes each) in BatchDev::tmaps, TMAP_STRIDE bytes per case:
// FP64 planes with x = column + 2: box 36 x 20 (tile + 2-cell halo), box 32 x 16 (tile),
// box 32 x 16 x 3 planes; FP32 correction planes with x = column + 4: box 40 x 20, 32 x 16
constexpr int TMAP_F64_HALO = 0, TMAP_F64_TILE = 128, TMAP_F64_TILE3 = 256, TMAP_X32_HALO = 384,
              TMAP_X32_TILE = 512, TMAP_STRIDE = 640;

// per-case scalar slots (FP64) of the pressure solve and step statistics
enum Scalar {
    S_RHO, S_ALPHA, S_OMEGA, S_BETA, S_NB1, S_RL1, S_RL1_0,
    S_QL1, S_QL2, S_QMAX, S_DMAX, S_CL, S_CD, S_CM, S_NU, S_CIRC, S_CLP, S_CDP, S_CLV, S_CDV,
    S_DTL1, S_DTMAX, S_DUL1, S_CW0, S_CW1,  // Chebyshev weights of the u-type / T systems
    S_QL2_0, S_SR, S_SR0,                   // first-step q_l2; steady residual (now, first step)
    S_MR0 = 29,           // 5 initial momentum residuals (L1)
    S_MR = S_MR0 + NFIELD,  // 5 latest momentum residuals
    S_TIME = S_MR + NFIELD,  // time as a double (time-accurate mode)
    NSCAL = S_TIME + 2
};

// per-case integer slots
enum IScalar {
    I_PDONE, I_PIT, I_PSTATUS, I_TIME,
    I_MDONE0,                 // 5 momentum done flags
    I_MIT0 = I_MDONE0 + NFIELD,  // 5 momentum sweep counts
    I_MODD0 = I_MIT0 + NFIELD,   // 5 flags: the solve's result is in the scratch plane
    I_MFLIP0 = I_MODD0 + NFIELD,  // 5 flags: this step's first iterate is in the scratch plane
    I_MNEXT0 = I_MFLIP0 + NFIELD, // 5 flags: the same, predicted for the next step
    I_MWORD = I_MNEXT0 + NFIELD,  // the sweep kernel's one read: bits 0-4 fields still iterating,
                                  // 5-9 I_MFLIP0 bits, 10+ sweeps done (same for every active field)
    I_STATUS,
    I_ACTIVE,                 // 0: an empty slot, skipped by every kernel
    I_NSTEP,                  // steps taken since the case was admitted
    NISCAL
};

enum Status { ST_OK = 0, ST_MAXITER = 1, ST_BREAKDOWN = 2, ST_NAN = 4 };

struct LevelDev {
    int W, n1, ld, nlo;   // stored width, rows, pitch; nlo = ilo for this level
    int ilo, ihi;         // unknown columns (inclusive)
    long long base;       // FP32 arena offset of this level's plane 0 origin
    long long ps;         // FP32 plane stride
    int tile_begin, tile_count;  // tiles of this case in the level's tile table
};

struct CaseDev {
    int W, n0, n1, ld;
    int periodic, ilo, ihi, profile;
    long long base, ps;
    int tile_begin, tile_count;     // fine-grid tiles of this case
    int jt_begin, jt_count;         // 32 x 16 tiles of this case (u/v/T sweeps)
    int nlev;
    int xld;                        // FP32 precision-form planes: pitch, base, stride
    long long xbase, xps;
    int fix_T_annw, fix_circ_de, warm_up;
    int time_accurate;              // 1: time is a double (t = n dt), 0: the reference's int
    double d0, d1, dt, Re, Pr, Ri, F;
    double uinf, vinf, speed_amp, accn_amp, Pi, ar, omega_p, lid_u, sa, ca;
    double tol_mom, atol_mom, tol_p, atol_p;
    double cheb_a[2], cheb_b[2];  // eigenvalue bounds of D^-1 A (u-type, T) for the Chebyshev sweeps
    double swk[3];                // dt / (Re dxi0^2), dt / (Re dxi1^2), dt / (Re dxi0 dxi1): E, G, B per metric
    double rPr;                   // 1 / Pr
    double pc1, pc2, pc3;         // 1 / (2 dxi0^2), 1 / (8 dxi0 dxi1), 1 / (2 dxi1^2): pressure stencil
    LevelDev lev[MAXLEV];
};

struct Tile {
    int c, i0, j0, k;  // case, first column, first row, tile index within the case
};

// everything a kernel needs, passed by value
struct BatchDev {
    const CaseDev* cases;
    int ncases;
    double* f64;
    float* f32;
    double* scal;          // ncases * NSCAL
    int* iscal;            // ncases * NISCAL
    double* partial;       // reduction partials: ntiles_max * 8
    unsigned int* counter; // per case, last-block detection
    int* active;           // global count of cases still iterating (pressure)
    int* mactive;          // global count of (case, field) pairs still iterating (momentum)
    int* error;            // set when a bounded wait in a kernel gives up
    unsigned wait_polls;   // polls of a kernel's bounded mbarrier waits before they give up
    int mixed;             // 1: the precision form (momentum iterates are FP32 corrections)
    int* tword;            // per 32 x 16 tile: its case's I_MWORD, so the sweep kernel reads it
                           // in the same round trip as the tile itself
    const Tile* ftiles;    // fine-grid tiles of every case (FP64 kernels, multigrid level 0)
    int nftiles;
    const Tile* jtiles;    // 32 x 16 tiles of every case (u/v/T sweeps)
    int njtiles;
    const Tile* mtiles[MAXLEV];   // level-l 32 x 16 tiles of the cases for which l is not the coarsest level
    int nmtiles[MAXLEV];
    const Tile* atiles[MAXLEV];   // level-l tiles of every case that has level l (set-up)
    int natiles[MAXLEV];
    const int* ccases[MAXLEV];    // cases whose coarsest level is l
    int nccases[MAXLEV];
    unsigned long long* work;  // [0] field-cells and [1] cells swept by k_jac, [2] field-cells of sweep 0
    const char* tmaps;     // per case TMAP_STRIDE bytes of CUtensorMaps (TMAP_* offsets)
    int cur;               // which of T0/T1 (up0/up1, vp0/vp1) holds the current state
    int mg_res;            // multigrid plane (M_X or M_R) holding a non-coarsest level's V-cycle result
};

// ------------------------------------------------------------------------
__device__ __forceinline__ double* plane(const BatchDev& b, const CaseDev& c, int k) {
    return b.f64 + c.base + (long long)k * c.ps + H;
}
__device__ __forceinline__ float* mplane(const BatchDev& b, const LevelDev& L, int k) {
    return b.f32 + L.base + (long long)k * L.ps + H;
}
__device__ __forceinline__ float* xplane(const BatchDev& b, const CaseDev& c, int k) {
    return b.f32 + c.xbase + (long long)k * c.xps + H32;
}

// periodic halo mirror of column i (or -1 if none)
__device__ __forceinline__ int mirror_col(int i, int W, int periodic) {
    if (!periodic) return -1000000;
    if (i < 2) return i + W;
    if (i >= W - 2) return i - W;
    return -1000000;
}

template <typename T>
__device__ __forceinline__ void store_mirrored(T* p, int ld, int i, int j, int W, int periodic, T v) {
    p[(long long)j * ld + i] = v;
    int m = mirror_col(i, W, periodic);
    if (m > -1000000) p[(long long)j * ld + m] = v;
}

// block-wide sum of NV values (blockDim.x == nthreads, multiple of 32); result valid in thread 0
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double* smem /* NV * 32 */) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; k++) {
        double x = v[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) smem[k * 32 + warp] = x;
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < NV; k++) {
            double x = lane < nw ? smem[k * 32 + lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
            v[k] = x;
        }
    }
    __syncthreads();
}

template <int NV>
__device__ __forceinline__ void block_max(double (&v)[NV], double* smem) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; k++) {
        double x = v[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x = fmax(x, __shfl_down_sync(0xffffffffu, x, o));
        if (lane == 0) smem[k * 32 + warp] = x;
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < NV; k++) {
            double x = lane < nw ? smem[k * 32 + lane] : -1.0e300;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) x = fmax(x, __shfl_down_sync(0xffffffffu, x, o));
            v[k] = x;
        }
    }
    __syncthreads();
}

}  // namespace cfd
