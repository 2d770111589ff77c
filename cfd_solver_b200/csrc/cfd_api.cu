// cfd_api.cu -- host runtime and C ABI (include/cfd_b200.h).
//
// A batch owns one FP64 arena (NPLANES planes per case), one FP32 arena (the
// multigrid hierarchy), a device case table, the tile tables of every level
// and one CUDA stream. One time step of every case in the batch is a fixed
// sequence of launches (the step of PSolver.cpp:1058-1983); the inner solves
// iterate on the device and the host only reads a 4-byte "cases still
// iterating" counter to decide when to stop launching.
#include <cuda.h>  // CUtensorMap types (the encoder is fetched through the runtime)
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/cfd_b200.h"
#include "cfd_bulk.cuh"
#include "cfd_common.cuh"
#include "cfd_kernels.cuh"
#include "cfd_reduce.cuh"
#include "cfd_sweep.cuh"

using namespace cfd;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}
}  // namespace

// lets the other translation units of the library report through cfd_last_error()
void cfd_internal_set_error(const char* msg) { g_err = msg ? msg : ""; }

namespace {

#define CK(call)                                                                          \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return fail(e_ == cudaErrorMemoryAllocation ? CFD_E_OOM : CFD_E_CUDA,         \
                        std::string(#call) + ": " + cudaGetErrorString(e_));              \
    } while (0)

long long rup(long long x, long long a) { return (x + a - 1) / a * a; }

constexpr int NFLAGS = 10;  // device flag words of a batch

enum KernelId {
    K_ASSEMBLE_P, K_RHS, K_SWEEP, K_UPBC, K_FACE_Q, K_BICG_P, K_SPMV, K_BICG_S, K_BICG_X,
    K_MG_SMOOTH, K_MG_RR, K_MG_POST, K_MG_COARSE, K_MG_GALERKIN,
    K_CORRECT, K_BC, K_DIAG, K_SI, K_MOM_UPDATE, K_SWEEP_FIN, K_MG_PRR, K_MOM_FIX, NKERNEL
};
const char* kKernelNames[NKERNEL] = {
    "k_assemble_p", "k_rhs", "k_sweep", "k_upbc", "k_face_q", "k_bicg_p", "k_spmv", "k_bicg_s",
    "k_bicg_x", "k_mg_presmooth", "k_mg_rr", "k_mg_postsmooth", "k_mg_coarse",
    "k_mg_galerkin", "k_correct", "k_bc", "k_diag", "k_si", "k_mom_update", "k_sweep_fin", "k_mg_prr", "k_mom_fix"};

struct LevelGeom {
    int W, n1, ld, ilo, ihi;
    long long ps;
};

// multigrid hierarchy of a case: coarsen by 2 while the level stays even-sized
std::vector<LevelGeom> build_levels(int W, int n1, int periodic) {
    std::vector<LevelGeom> L;
    int w = W, n = n1;
    for (int l = 0; l < MAXLEV; l++) {
        LevelGeom g;
        g.W = w;
        g.n1 = n;
        g.ld = (int)rup(w + 2 * H, 32);
        g.ps = rup(32 + (long long)n * g.ld, 32);
        g.ilo = periodic ? 0 : 1;
        g.ihi = periodic ? w - 1 : w - 2;
        L.push_back(g);
        if ((long long)(g.ihi - g.ilo + 1) * (n - 2) <= 64) break;
        bool can;
        int wc, nc;
        if (periodic) {
            can = (w % 2 == 0) && (w / 2 >= 4);
            wc = w / 2;
        } else {
            can = ((w - 1) % 2 == 0) && ((w - 1) / 2 + 1 >= 5);
            wc = (w - 1) / 2 + 1;
        }
        can = can && ((n - 1) % 2 == 0) && ((n - 1) / 2 + 1 >= 4);
        nc = (n - 1) / 2 + 1;
        if (!can) break;
        w = wc;
        n = nc;
    }
    return L;
}

struct CaseGeom {
    int W, ld, ilo, ihi, periodic;
    long long ps;
    int xld;         // FP32 precision-form planes: pitch (columns -4 .. W+1 and slack), stride
    long long xps;
    std::vector<LevelGeom> lev;
    long long bytes64() const { return (long long)NPLANES * ps + 16; }
    long long words32() const {
        long long s = 0;
        for (auto& g : lev) s += (long long)NMG * g.ps + 32;
        return s + (long long)NXPLANES * xps + 32;
    }
};

CaseGeom case_geom(int n0, int n1, int profile) {
    CaseGeom g;
    g.periodic = profile == CFD_PROFILE_OGRID;
    g.W = g.periodic ? n0 - 1 : n0;
    g.ld = (int)rup(g.W + 2 * H + 2, 16);  // 2 columns of slack for 16-byte row copies
    g.ps = rup(16 + (long long)n1 * g.ld, 16);
    g.ilo = g.periodic ? 0 : 1;
    g.ihi = g.periodic ? g.W - 1 : n0 - 2;
    g.lev = build_levels(g.W, n1, g.periodic);
    g.xld = (int)rup(g.W + H32 + H + 2, 32);
    g.xps = rup((long long)n1 * g.xld + 32, 32);
    return g;
}

struct Launch {
    int id;
    cudaEvent_t e0, e1;
};

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn tensor_map_encoder() {
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    }
    return fn;
}

}  // namespace

struct cfd_batch {
    int n = 0;
    std::vector<CaseDev> hc;
    std::vector<cfd_params> prm;
    std::vector<CaseGeom> geom;
    std::vector<double> q_l2_first, sr_first;  // unused (first-step references live on the device)
    CaseDev* dc = nullptr;
    double* f64 = nullptr;
    float* f32 = nullptr;
    long long n64 = 0, n32 = 0;
    double* scal = nullptr;
    int* iscal = nullptr;
    double* partial = nullptr;
    unsigned int* counter = nullptr;
    // device flags: [0] cases still in the pressure solve, [1] (case, field) pairs still in
    // the momentum solves, [2] / [3] this step's momentum-pair / pressure-iteration counts,
    // [4] kernel wait timeout, [5] / [6] cumulative pair / iteration counts (graph steps),
    // [7] this step's momentum sweep launches, [8] cumulative count of pressure iterations
    // whose second half ran (graph steps)
    int* flags = nullptr;
    bool use_graph = true;
    cudaGraphExec_t gexec[2] = {nullptr, nullptr};
    int launches_per_pair = 2, launches_per_iter = 0, launches_per_half = 0, launches_fixed = 0;
    int flags_total0[3] = {0, 0, 0};
    int* tword = nullptr;                // per tile: the case's momentum-loop word
    unsigned long long* work = nullptr;  // k_jac traffic counters
    long long launches = 0;              // kernels launched since creation
    int* h_flags = nullptr;
    double* stage = nullptr;        // state snapshot staging (allocated on first use)
    long long* stage_off = nullptr; // per-case offsets into it (doubles)
    Tile* dtiles = nullptr;
    int* dcc = nullptr;
    size_t cap_tiles = 0, cap_cc = 0, cap_partial = 0, cap_tword = 0;  // table allocations (entries)
    int ntable_cases = 0;    // cases in the tile tables (one coarsest level each)
    char* dtmaps = nullptr;  // two CUtensorMaps per case
    // slot pool (cfd_pool_create): cases are placed in one byte arena at admission
    bool is_pool = false;
    size_t pool_bytes = 0;
    std::vector<std::pair<size_t, size_t>> pool_free;  // free regions (offset, bytes), sorted
    std::vector<std::pair<size_t, size_t>> pool_region; // per case: its region, or (0, 0)
    size_t stage_bytes = 0;
    BatchDev bd{};
    int nlev_max = 0;
    int ncol[MAXLEV] = {};
    int maxit_mom = 100, maxit_p = 200;
    int precision = CFD_PRECISION_FP64;
    int sw_grid = 0;      // CTAs of the sweep kernel (one per 32 x 16 tile)
    size_t sw_smem = 0;   // its dynamic shared memory (the precision form: the first sweep's)
    size_t sw_smem1 = 0;  // the precision form's later sweeps (k_sweep_mx1)
    int coarse_sweeps = 12;
    int mg_pre = 1, mg_post = 3;  // multigrid sweeps before / after the coarse correction
    int mg_fused = 2;             // 1: a smoothing phase's sweeps in one launch; 2: and the
                                  // pre-smoothing inside the residual + restriction launch
    int swf_threads = 128;  // k_sweep_fin CTA size: 512 when a case has >= 1024 tiles
    int max_W = 0;
    int cur = 0;
    long long steps_done = 0;
    cudaStream_t st = nullptr;
    int dev = 0;
    // profiling
    bool prof = false;
    std::vector<Launch> pending;
    std::vector<cudaEvent_t> pool;
    double kt_ms[NKERNEL] = {};
    long long kt_n[NKERNEL] = {};
    // host staging
    std::vector<double> hscal;
    std::vector<int> hiscal;
};

namespace {

cudaEvent_t get_event(cfd_batch* b) {
    if (!b->pool.empty()) {
        cudaEvent_t e = b->pool.back();
        b->pool.pop_back();
        return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
}

struct Prof {
    cfd_batch* b;
    int id;
    cudaEvent_t e0{}, e1{};
    Prof(cfd_batch* b_, int id_) : b(b_), id(id_) {
        b->launches++;
        if (b->prof) {
            e0 = get_event(b);
            e1 = get_event(b);
            cudaEventRecord(e0, b->st);
        }
    }
    ~Prof() {
        if (b->prof) {
            cudaEventRecord(e1, b->st);
            b->pending.push_back({id, e0, e1});
        }
    }
};

int flush_profile(cfd_batch* b) {
    if (b->pending.empty()) return CFD_OK;
    CK(cudaStreamSynchronize(b->st));
    for (auto& l : b->pending) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, l.e0, l.e1);
        b->kt_ms[l.id] += ms;
        b->kt_n[l.id] += 1;
        b->pool.push_back(l.e0);
        b->pool.push_back(l.e1);
    }
    b->pending.clear();
    return CFD_OK;
}

// reads the device flags (one copy); fails if a kernel's bounded wait gave up
int read_flag(cfd_batch* b, int idx, int* out) {
    CK(cudaMemcpyAsync(b->h_flags, b->flags, NFLAGS * sizeof(int), cudaMemcpyDeviceToHost, b->st));
    CK(cudaStreamSynchronize(b->st));
    *out = b->h_flags[idx];
    if (b->h_flags[4]) return fail(CFD_E_CUDA, "a bounded wait inside a kernel timed out");
    return CFD_OK;
}

// host copy of one padded plane: [j][i] with n0 columns (the seam column of the
// O-grid is the halo copy of column 0)
void pad_plane(const CaseDev& c, const double* src, std::vector<double>& dst) {
    dst.assign((size_t)c.ps, 0.0);
    double* o = dst.data() + 16;  // column 0 of row 0
    for (int j = 0; j < c.n1; j++) {
        double* row = o + (long long)j * c.ld;
        const double* s = src + (size_t)j * c.n0;
        if (c.periodic) {
            for (int i = 0; i < c.W; i++) row[i] = s[i];
            row[-2] = s[c.W - 2];
            row[-1] = s[c.W - 1];
            row[c.W] = s[0];
            row[c.W + 1] = s[1];
        } else {
            for (int i = 0; i < c.n0; i++) row[i] = s[i];
        }
    }
}

void unpad_plane(const CaseDev& c, const double* padded, double* out) {
    const double* o = padded + 16;
    for (int j = 0; j < c.n1; j++) {
        const double* row = o + (long long)j * c.ld;
        double* d = out + (size_t)j * c.n0;
        if (c.periodic) {
            for (int i = 0; i < c.W; i++) d[i] = row[i];
            d[c.n0 - 1] = row[c.W];
        } else {
            for (int i = 0; i < c.n0; i++) d[i] = row[i];
        }
    }
}

// the checks of a case's parameters that do not read its grid
int check_case_params(const cfd_params* p) {
    if (!p) return fail(CFD_E_ARG, "null params");
    if (p->profile != CFD_PROFILE_OGRID && p->profile != CFD_PROFILE_CAVITY)
        return fail(CFD_E_ARG, "unknown profile");
    if (!(p->dt > 0) || !(p->Re > 0) || !(p->Pr > 0)) return fail(CFD_E_ARG, "dt, Re, Pr must be > 0");
    if (p->maxit_mom < 2 || p->maxit_p < 1) return fail(CFD_E_ARG, "iteration caps too small");
    if (p->precision != CFD_PRECISION_FP64 && p->precision != CFD_PRECISION_MIXED)
        return fail(CFD_E_ARG, "unknown precision");
    return CFD_OK;
}

int check_params(const cfd_grid* g, const cfd_params* p) {
    if (!g || !p) return fail(CFD_E_ARG, "null grid or params");
    if (int rc = check_case_params(p)) return rc;
    if (g->n0 < 8 || g->n1 < 6) return fail(CFD_E_ARG, "grid too small (need n0 >= 8, n1 >= 6)");
    if (g->n0 > 8192 || g->n1 > 8192) return fail(CFD_E_ARG, "grid too large (n0, n1 <= 8192)");
    if (!(g->dxi0 > 0) || !(g->dxi1 > 0)) return fail(CFD_E_ARG, "non-positive grid spacing");
    if (!g->x || !g->y || !g->xix || !g->xiy || !g->etx || !g->ety || !g->alph || !g->beta ||
        !g->gam || !g->jac || !g->xnix || !g->xniy || !g->xnox || !g->xnoy)
        return fail(CFD_E_ARG, "missing grid plane");
    const size_t N = (size_t)g->n0 * g->n1;
    for (size_t k = 0; k < N; k++) {
        if (!(g->alph[k] > 0) || !(g->gam[k] > 0) || !std::isfinite(g->beta[k]) || !std::isfinite(g->jac[k]))
            return fail(CFD_E_ARG, "grid metrics invalid (alpha, gamma must be > 0)");
    }
    return CFD_OK;
}

// initial state of PSolver.cpp:614-748 (O-grid) or the cavity's
void initial_state(const cfd_grid* g, const cfd_params* p, const CaseDev& c, std::vector<double>* st) {
    // st: u, v, T, up, vp, p (n1*n0, [j][i])
    const int n0 = g->n0, n1 = g->n1;
    const size_t N = (size_t)n0 * n1;
    for (int m = 0; m < 6; m++) st[m].assign(N, 0.0);
    if (p->profile == CFD_PROFILE_CAVITY) {
        for (int i = 1; i < n0 - 1; i++) {
            st[0][(size_t)(n1 - 1) * n0 + i] = p->lid_u;
            st[3][(size_t)(n1 - 1) * n0 + i] = p->lid_u;
        }
        for (int i = 0; i < n0; i++) st[2][i] = 1.0;
        return;
    }
    for (size_t k = 0; k < N; k++) {
        st[0][k] = c.uinf; st[1][k] = c.vinf; st[3][k] = c.uinf; st[4][k] = c.vinf;
    }
    for (int i = 0; i < n0; i++) {
        st[0][i] = -c.speed_amp * g->y[i];
        st[1][i] = c.speed_amp * g->x[i];
        st[3][i] = st[0][i];
        st[4][i] = st[1][i];
        st[2][i] = 1.0;
    }
    const int j = n1 - 1;
    for (int i = 0; i < n0 - 1; i++) {
        const size_t k = (size_t)j * n0 + i;
        const double vnn = st[0][k] * g->xnox[i] + st[1][k] * g->xnoy[i];
        if (vnn >= 0) {
            st[0][k] = c.uinf; st[1][k] = c.vinf; st[2][k] = 0.0;
            st[3][k] = st[0][k]; st[4][k] = st[1][k];
        } else {
            const size_t kb = k - n0;
            st[0][k] = st[0][kb]; st[1][k] = st[1][kb]; st[2][k] = st[2][kb];
            if (i == 0) {
                const size_t s = (size_t)j * n0 + n0 - 1;
                st[0][s] = st[0][k]; st[1][s] = st[1][k]; st[2][s] = st[2][k];
            }
        }
    }
}

// Eigenvalue bounds of D^-1 A for the Chebyshev sweeps. With E = dt/Re (alpha/dxi0^2 +
// gamma/dxi1^2) the smooth modes of the 25-point operator sit at 1/(1 + 2.5 E) and Gershgorin
// bounds the top: 1 + ((17/6) E + 4.5 |beta| dt/(Re dxi0 dxi1)) / (1 + 2.5 E); the 9-point
// rows lie inside both (margins: cheb_finish). T uses Re*Pr; the reference's T slot bug
// (atnw for annw) adds 7/9 |beta| c to the off-diagonal sum.
// Per-system constants of the bound scan: dt/scale, the cross-term factor, dt/(scale dxi0
// dxi1), dxi0^2, dxi1^2 (index 0: u, v, up, vp with scale Re; 1: T with scale Re Pr).
struct ChebScan {
    double dts[2], cross[2], cc[2], d00, d11;
};

ChebScan cheb_consts(const cfd_params& p, double dxi0, double dxi1) {
    ChebScan cs;
    for (int ty = 0; ty < 2; ty++) {
        const double scale = ty == 0 ? p.Re : p.Re * p.Pr;
        cs.dts[ty] = p.dt / scale;
        cs.cross[ty] = (ty == 1 && !p.fix_T_annw) ? 4.5 + 7.0 / 9.0 : 4.5;
        cs.cc[ty] = p.dt / (scale * dxi0 * dxi1);
    }
    cs.d00 = dxi0 * dxi0;
    cs.d11 = dxi1 * dxi1;
    return cs;
}

// The interval [a0, b0] = [1/(1 + 2.5 E), 1 + rmax] widened on each side by 2 % of its
// width, but by at most 10 % of a0 below and 5 % of b0 above. The mass-dominated systems of
// small time steps have narrow intervals (w << a0): width margins keep them narrow, and their
// solves meet the stop rule after two sweeps instead of three. Large time steps give wide
// intervals whose smallest eigenvalue lies within a few per cent of a0 (a0 = 0.053, w = 2.45
// for a 257 x 257 cavity at E = 7): there the lower margin must stay a fraction of a0, since
// a0 - 0.02 w would put the lower end near zero and triple the sweep count.
void cheb_finish(const double* emax, const double* rmax, CaseDev& d) {
    for (int ty = 0; ty < 2; ty++) {
        const double a0 = 1.0 / (1.0 + 2.5 * emax[ty]), b0 = 1.0 + rmax[ty], w = b0 - a0;
        d.cheb_a[ty] = a0 - std::min(0.1 * a0, 0.02 * w);
        d.cheb_b[ty] = b0 + std::min(0.05 * b0, 0.02 * w);
    }
}

void cheb_bounds(const cfd_grid& g, const cfd_params& p, CaseDev& d) {
    const int n0 = g.n0, n1 = g.n1;
    const ChebScan cs = cheb_consts(p, g.dxi0, g.dxi1);
    double emax[2], rmax[2];
    for (int ty = 0; ty < 2; ty++) {
        emax[ty] = 0.0;
        rmax[ty] = 0.0;
        for (int j = 1; j < n1 - 1; j++)
            for (int i = 0; i < n0; i++) {
                const size_t k = (size_t)j * n0 + i;
                const double E = cs.dts[ty] * (g.alph[k] / cs.d00 + g.gam[k] / cs.d11);
                emax[ty] = std::max(emax[ty], E);
                rmax[ty] = std::max(rmax[ty], ((17.0 / 6.0) * E + cs.cross[ty] * std::fabs(g.beta[k]) * cs.cc[ty]) /
                                                  (1.0 + 2.5 * E));
            }
    }
    cheb_finish(emax, rmax, d);
}

// The bound scan of cheb_bounds() over a grid that is in device memory (the 10 planes
// of a generated grid), with each product, quotient and sum rounded on its own as the
// host evaluates them, so both give the same bits. Also counts the points whose metrics
// are invalid (the test of check_params()). The maxima are of non-negative doubles, so
// they are taken on the bit patterns as unsigned integers. out: emax[2], rmax[2] (bit
// patterns), invalid points; zeroed by the caller.
constexpr int SCAN_THREADS = 256;
__global__ void __launch_bounds__(SCAN_THREADS) k_grid_scan(const double* planes, int n0, int n1, ChebScan cs,
                                                            unsigned long long* out) {
    const long long np = (long long)n0 * n1;
    const double* alph = planes + (long long)P_ALPH * np;
    const double* beta = planes + (long long)P_BETA * np;
    const double* gam = planes + (long long)P_GAM * np;
    const double* jac = planes + (long long)P_JAC * np;
    double em[2] = {0.0, 0.0}, rm[2] = {0.0, 0.0};
    unsigned long long bad = 0;
    for (long long k = (long long)blockIdx.x * SCAN_THREADS + threadIdx.x; k < np;
         k += (long long)gridDim.x * SCAN_THREADS) {
        const double a = alph[k], g = gam[k], be = beta[k];
        if (!(a > 0) || !(g > 0) || !isfinite(be) || !isfinite(jac[k])) bad++;
        const int j = (int)(k / n0);
        if (j < 1 || j > n1 - 2) continue;
        const double sm = __dadd_rn(__ddiv_rn(a, cs.d00), __ddiv_rn(g, cs.d11));
#pragma unroll
        for (int ty = 0; ty < 2; ty++) {
            const double E = __dmul_rn(cs.dts[ty], sm);
            const double num = __dadd_rn(__dmul_rn(17.0 / 6.0, E), __dmul_rn(__dmul_rn(cs.cross[ty], fabs(be)), cs.cc[ty]));
            const double r = __ddiv_rn(num, __dadd_rn(1.0, __dmul_rn(2.5, E)));
            em[ty] = fmax(em[ty], E);
            rm[ty] = fmax(rm[ty], r);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        for (int ty = 0; ty < 2; ty++) {
            em[ty] = fmax(em[ty], __shfl_xor_sync(0xffffffffu, em[ty], o));
            rm[ty] = fmax(rm[ty], __shfl_xor_sync(0xffffffffu, rm[ty], o));
        }
        bad += __shfl_xor_sync(0xffffffffu, bad, o);
    }
    if ((threadIdx.x & 31) == 0) {
        for (int ty = 0; ty < 2; ty++) {
            atomicMax(out + ty, (unsigned long long)__double_as_longlong(em[ty]));
            atomicMax(out + 2 + ty, (unsigned long long)__double_as_longlong(rm[ty]));
        }
        if (bad) atomicAdd(out + 4, bad);
    }
}

// Writes a generated grid (10 planes of [n1][n0], then 4 rows of n0 normals) into a case's
// padded planes the way pad_plane() does on the host: `region` is the start of the case's
// plane 0 (plane q at region + q * ps, point (j, i) at 16 + j * ld + i); for a periodic case
// padded columns -H..W+H-1 take source column i mod W; normals go to rows 0..3 of P_VEC,
// zero in the other rows. The planes' other entries are zeroed by the caller.
__global__ void k_grid_to_slot(const double* gen, int n0, int n1, int W, int periodic, double* region,
                               long long ps, int ld) {
    const int ncols = periodic ? W + 2 * H : n0;
    const long long per = (long long)n1 * ncols;
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= 11 * per) return;
    const int q = (int)(e / per);
    const long long r = e - q * per;
    const int j = (int)(r / ncols), cpad = (int)(r % ncols);
    const int col = periodic ? cpad - H : cpad;
    const int i = col < 0 ? col + W : (col >= W ? col - W : col);
    const long long np = (long long)n0 * n1;
    double v;
    if (q < 10)
        v = gen[q * np + (long long)j * n0 + i];
    else
        v = j < 4 ? gen[10 * np + (long long)j * n0 + i] : 0.0;
    const int pid = q < 10 ? q : P_VEC;
    region[(long long)pid * ps + 16 + (long long)j * ld + col] = v;
}

// The initial state (initial_state() on the host, PSolver.cpp:614-748) of a case whose grid
// was generated on the device, written straight into its six state planes in the padded
// layout pad_plane() gives (the planes are zeroed by the caller; a periodic case's halo
// columns take the wrap). `x0`, `y0` are row 0 of x and y. Cavity: zero fields,
// lid u = up = lid_u on row n1-1 (columns 1 .. n0-2), T = 1 on row 0. O-grid: the uniform
// stream (uinf, vinf) with T = p = 0, and on the wall row the rotating-wall velocity
// (-w y, w x) with T = 1; the far-field row keeps the stream (either branch of the inflow
// test there copies the stream from the row below).
__global__ void k_init_state(double* region, long long ps, int ld, int n0, int n1, int W, int periodic,
                             int cavity, const double* x0, const double* y0, double uinf, double vinf,
                             double speed_amp,
                             double lid_u, int pu, int pv, int pT, int pup, int pvp) {
    const int ncols = periodic ? W + 2 * H : n0;
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long long)n1 * ncols) return;
    const int j = (int)(e / ncols), cpad = (int)(e % ncols);
    const int col = periodic ? cpad - H : cpad;
    const int i = col < 0 ? col + W : (col >= W && periodic ? col - W : col);
    double u, v, T, up, vp;
    if (cavity) {
        u = (j == n1 - 1 && i >= 1 && i <= n0 - 2) ? lid_u : 0.0;
        up = u;
        v = vp = 0.0;
        T = j == 0 ? 1.0 : 0.0;
    } else if (j == 0) {
        u = -speed_amp * y0[i];
        v = speed_amp * x0[i];
        up = u;
        vp = v;
        T = 1.0;
    } else {
        u = up = uinf;
        v = vp = vinf;
        T = 0.0;
    }
    const long long k = 16 + (long long)j * ld + col;
    region[(long long)pu * ps + k] = u;
    region[(long long)pv * ps + k] = v;
    region[(long long)pT * ps + k] = T;
    region[(long long)pup * ps + k] = up;
    region[(long long)pvp * ps + k] = vp;
}

static_assert(P_X == 0 && P_Y == 1 && P_XIX == 2 && P_XIY == 3 && P_ETX == 4 && P_ETY == 5 && P_ALPH == 6 &&
                  P_BETA == 7 && P_GAM == 8 && P_JAC == 9,
              "grid planes 0..9 in the order of cfd_grid_generate's planes");

// physics and numerics of one case into its descriptor (all but the Chebyshev bounds)
void case_scalars_to_dev(CaseDev& d, double dxi0, double dxi1, double ar, const cfd_params& p) {
    const cfd_grid g{0, 0, dxi0, dxi1, 0.0, 0.0, ar};
    d.fix_T_annw = p.fix_T_annw; d.fix_circ_de = p.fix_circ_de; d.warm_up = p.warm_start;
    d.time_accurate = p.time_accurate != 0;
    d.d0 = g.dxi0; d.d1 = g.dxi1; d.dt = p.dt; d.Re = p.Re; d.Pr = p.Pr; d.Ri = p.Ri; d.F = p.F;
    d.Pi = acos(-1.0);
    const double thetamax = d.Pi / 12.0;
    d.speed_amp = thetamax * 2.0 * d.Pi * p.F;
    d.accn_amp = 2.0 * d.Pi * p.F * d.speed_amp;
    d.uinf = sin(p.alpha_deg * d.Pi / 180.0);
    d.vinf = cos(p.alpha_deg * d.Pi / 180.0);
    d.sa = sin(p.alpha_deg * d.Pi / 180.0);
    d.ca = cos(p.alpha_deg * d.Pi / 180.0);
    d.ar = g.ar; d.omega_p = p.omega_p; d.lid_u = p.lid_u;
    d.tol_mom = p.tol_mom; d.atol_mom = p.atol_mom; d.tol_p = p.tol_p; d.atol_p = p.atol_p;
    // the sweeps' per-case factors, formed once here rather than by every thread of every CTA
    d.swk[0] = d.dt / (d.Re * d.d0 * d.d0);
    d.swk[1] = d.dt / (d.Re * d.d1 * d.d1);
    d.swk[2] = d.dt / (d.Re * d.d0 * d.d1);
    d.rPr = 1.0 / d.Pr;
    d.pc1 = 1.0 / (2.0 * g.dxi0 * g.dxi0);
    d.pc2 = 1.0 / (8.0 * g.dxi0 * g.dxi1);
    d.pc3 = 1.0 / (2.0 * g.dxi1 * g.dxi1);
}

// physics, numerics and Chebyshev bounds of one case into its descriptor
void case_params_to_dev(CaseDev& d, const cfd_grid& g, const cfd_params& p) {
    case_scalars_to_dev(d, g.dxi0, g.dxi1, g.ar, p);
    cheb_bounds(g, p, d);
}

void make_tiles(int ilo, int ihi, int n1, int cid, std::vector<Tile>& out, int ty = TY) {
    int k = 0;
    for (int j0 = 1; j0 <= n1 - 2; j0 += ty)
        for (int i0 = (ilo / TX) * TX; i0 <= ihi; i0 += TX) out.push_back({cid, i0, j0, k++});
}

// --------------------------------------------------------------------------
// one time step of every case in the batch
// planes of the pre-smoothed x and of the V-cycle result of a non-coarsest level: sweeps
// alternate between x and r, starting in x
int mg_pre_plane(int nu_pre, int fused) { return (fused || (nu_pre & 1)) ? M_X : M_R; }
int mg_res_plane(int nu_pre, int nu_post, int fused) {
    const int p = mg_pre_plane(nu_pre, fused);
    const int q = p == M_X ? M_R : M_X;
    return (fused || (nu_post & 1)) ? q : p;
}

// One V-cycle. Smoothing phases of several sweeps run either as one launch per sweep
// (each sweep sees the neighbouring tiles' latest values) or, `mg_fused`, as one launch
// doing all of the phase's sweeps in shared memory; `mg_fused` = 2 also folds each level's
// pre-smoothing into its residual + restriction launch (k_mg_prr).
int run_vcycle(cfd_batch* b) {
    BatchDev& bd = b->bd;
    const int fused = b->mg_fused;
    const int pre = mg_pre_plane(b->mg_pre, fused);
    const int npre = fused ? 1 : b->mg_pre, inpre = fused ? b->mg_pre : 1;
    const int npost = fused ? 1 : b->mg_post, inpost = fused ? b->mg_post : 1;
    // down: pre-smoothing, residual and restriction level by level; then one launch solves
    // every case on its own coarsest level (a case's coarse solve needs only its own
    // restriction, done by then, and is read first by the post-smoothing of the level above)
    for (int l = 0; l < b->nlev_max; l++) {
        if (bd.nmtiles[l] > 0 && fused == 2) {
            Prof pr(b, K_MG_PRR);
            k_mg_prr<<<bd.natiles[l + 1], MG_PRR_THREADS, 0, b->st>>>(bd, l, pre, b->mg_pre);
        } else if (bd.nmtiles[l] > 0) {
            for (int s = 0; s < npre; s++) {  // pre-smoothing from zero
                Prof pr(b, K_MG_SMOOTH);
                const int dst = (s & 1) ? M_R : M_X;
                k_mg_gs<<<bd.nmtiles[l], MG_GS_THREADS, 0, b->st>>>(bd, l, s == 0 ? 0 : 1, dst == M_X ? M_R : M_X, dst,
                                                                  inpre);
            }
            Prof pr(b, K_MG_RR);
            k_mg_rr<<<bd.natiles[l + 1], NT, 0, b->st>>>(bd, l, pre);
        }
    }
    {
        Prof pr(b, K_MG_COARSE);
        k_mg_coarse<<<b->ntable_cases, 1024, 0, b->st>>>(bd, -1, b->coarse_sweeps);
    }
    for (int l = b->nlev_max - 2; l >= 0; l--) {
        if (bd.nmtiles[l] == 0) continue;
        int src = pre;
        for (int s = 0; s < npost; s++) {
            Prof pr(b, K_MG_POST);
            const int dst = src == M_X ? M_R : M_X;
            k_mg_gs<<<bd.nmtiles[l], MG_GS_THREADS, 0, b->st>>>(bd, l, s == 0 ? 2 : 3, src, dst, inpost);
            src = dst;
        }
    }
    return CFD_OK;
}

// ---- the pieces of one step (also captured into the step graph)
void enq_begin(cfd_batch* b, BatchDev& bd) {
    cudaMemsetAsync(b->flags, 0, 4 * sizeof(int), b->st);
    Prof pr(b, K_RHS);
    k_rhs<<<bd.njtiles, NT, kRhsSmem, b->st>>>(bd);
}
// FP64 form: sweeps in pairs (the iterates ping-pong between two planes)
void enq_mom_pair(cfd_batch* b, BatchDev& bd) {
    for (int s = 0; s < 2; s++) {
        {
            Prof pr(b, K_SWEEP);
            k_sweep_f64<<<b->sw_grid, SW_THREADS, b->sw_smem, b->st>>>(bd);
        }
        Prof pr(b, K_SWEEP_FIN);
        k_sweep_fin<<<b->n, b->swf_threads, 0, b->st>>>(bd);
    }
}
// precision form: the step's first sweep (FP64 residual, k_sweep_mx0), then one FP32
// sweep (k_sweep_mx1) per loop iteration
void enq_mom_mx_first(cfd_batch* b, BatchDev& bd) {
    {
        Prof pr(b, K_SWEEP);
        k_sweep_mx0<<<b->sw_grid, SW_THREADS, b->sw_smem, b->st>>>(bd);
    }
    Prof pr(b, K_SWEEP_FIN);
    k_sweep_fin<<<b->n, b->swf_threads, 0, b->st>>>(bd);
}
void enq_mom_mx_next(cfd_batch* b, BatchDev& bd) {
    {
        Prof pr(b, K_SWEEP);
        k_sweep_mx1<<<b->sw_grid, SW_THREADS, b->sw_smem1, b->st>>>(bd);
    }
    Prof pr(b, K_SWEEP_FIN);
    k_sweep_fin<<<b->n, b->swf_threads, 0, b->st>>>(bd);
}
// loop iterations that bound the momentum / energy solves at maxit_mom sweeps
int mom_loop_cap(const cfd_batch* b) {
    return b->precision == CFD_PRECISION_MIXED ? std::max(1, b->maxit_mom - 1) : std::max(1, b->maxit_mom / 2);
}
void enq_mid(cfd_batch* b, BatchDev& bd) {
    if (b->precision == CFD_PRECISION_MIXED) {
        Prof pr(b, K_MOM_UPDATE);
        k_mom_update<<<bd.nftiles, NT, 0, b->st>>>(bd);
    } else {
        Prof pr(b, K_MOM_FIX);
        k_mom_fix<<<bd.njtiles, NT, 0, b->st>>>(bd);
    }
    {
        Prof pr(b, K_UPBC);
        k_upbc<<<b->n, BC_THREADS, 0, b->st>>>(bd);
    }
    Prof pr(b, K_FACE_Q);
    k_face_q<<<bd.njtiles, NT, kFaceQSmem, b->st>>>(bd);
}
// one BiCGStab iteration in two halves: up to the half-step exit (k_bicg_s), and the rest,
// which the step graph skips when every case stopped at the half step. The next iteration's
// direction p_{k+1} is formed at the end of the second half (k_bicg_p, from the beta and
// omega k_bicg_x has just computed), so the first iteration, whose p_1 = r_0 k_face_q writes,
// and every step whose cases all stop at the first half step launch no k_bicg_p.
void enq_p_first(cfd_batch* b, BatchDev& bd) {
    const int nf = bd.njtiles;  // the BiCGStab kernels run on the 32 x 16 tiles
    run_vcycle(b);
    { Prof pr(b, K_SPMV); k_spmv<<<nf, NT, 0, b->st>>>(bd, 0); }
    { Prof pr(b, K_BICG_S); k_bicg_s<<<nf, NT, 0, b->st>>>(bd); }
}
void enq_p_second(cfd_batch* b, BatchDev& bd) {
    const int nf = bd.njtiles;
    run_vcycle(b);
    { Prof pr(b, K_SPMV); k_spmv<<<nf, NT, 0, b->st>>>(bd, 1); }
    { Prof pr(b, K_BICG_X); k_bicg_x<<<nf, NT, 0, b->st>>>(bd, b->maxit_p); }
    { Prof pr(b, K_BICG_P); k_bicg_p<<<nf, NT, 0, b->st>>>(bd); }
}
void enq_p_iter(cfd_batch* b, BatchDev& bd) {
    enq_p_first(b, bd);
    enq_p_second(b, bd);
}
void enq_end(cfd_batch* b, BatchDev& bd) {
    { Prof pr(b, K_CORRECT); k_correct<<<bd.njtiles, NT, 0, b->st>>>(bd); }
    { Prof pr(b, K_BC); k_bc<<<b->n, BC_THREADS, 2 * (b->max_W + 1) * sizeof(double), b->st>>>(bd); }
    { Prof pr(b, K_DIAG); k_diag<<<bd.njtiles, NT, 0, b->st>>>(bd); }
}

// one step with host-side loop control (per-kernel profiling works on this path)
int one_step_direct(cfd_batch* b) {
    BatchDev& bd = b->bd;
    bd.cur = b->cur;
    enq_begin(b, bd);
    // momentum / energy solves: sweeps (in pairs in the FP64 form) until every (case, field)
    // stopped; the counter is read every second loop iteration (a finished case's CTAs
    // leave at once)
    const bool mixed = b->precision == CFD_PRECISION_MIXED;
    if (mixed) enq_mom_mx_first(b, bd);
    const int npairs = mom_loop_cap(b);
    for (int pair = 0; pair < npairs; pair++) {
        if (mixed) enq_mom_mx_next(b, bd);
        else enq_mom_pair(b, bd);
        if (pair % 2 == 1 || pair == npairs - 1) {
            int m = 0;
            int rc = read_flag(b, 1, &m);
            if (rc) return rc;
            if (m <= 0) break;
        }
    }
    enq_mid(b, bd);
    // pressure correction: the first iteration is launched without a check (a case whose
    // q vanished is flagged done by k_face_q and its CTAs leave at once)
    for (int it = 0; it < b->maxit_p; it++) {
        if (it > 0) {
            int a = 0;
            int rc = read_flag(b, 0, &a);
            if (rc) return rc;
            if (a <= 0) break;
        }
        enq_p_iter(b, bd);
    }
    enq_end(b, bd);
    CK(cudaGetLastError());
    return CFD_OK;
}

// Build the step graph for state parity `cur`: child graphs for the straight segments and
// two while-loops whose condition kernels read the device counters of still-iterating work.
int build_step_graph(cfd_batch* b, int cur) {
    const bool prof = b->prof;
    b->prof = false;
    const long long l0 = b->launches;
    BatchDev bd = b->bd;
    bd.cur = cur;
    cudaGraph_t g = nullptr;
    CK(cudaGraphCreate(&g, 0));
    cudaGraphNode_t prev = nullptr;
    auto child = [&](auto&& enqueue) -> int {
        cudaGraph_t seg = nullptr;
        CK(cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal));
        enqueue();
        CK(cudaStreamEndCapture(b->st, &seg));
        cudaGraphNode_t n = nullptr;
        CK(cudaGraphAddChildGraphNode(&n, g, prev ? &prev : nullptr, prev ? 1 : 0, seg));
        cudaGraphDestroy(seg);
        prev = n;
        return CFD_OK;
    };
    auto loop = [&](auto&& enqueue, int* flag, int* counter, int maxc, int* total) -> int {
        cudaGraphConditionalHandle h;
        CK(cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault));
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = h;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t n = nullptr;
        CK(cudaGraphAddNode(&n, g, prev ? &prev : nullptr, prev ? 1 : 0, &cp));
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        CK(cudaStreamBeginCaptureToGraph(b->st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        enqueue();
        k_loop_cond<<<1, 32, 0, b->st>>>(h, flag, counter, maxc, total);
        cudaGraph_t out = nullptr;
        CK(cudaStreamEndCapture(b->st, &out));
        prev = n;
        return CFD_OK;
    };
    // the pressure loop: the iteration's first half, a condition kernel, an if-node holding
    // the second half (run while some case is still iterating), the loop condition
    long long lh0 = 0, lh1 = 0, lh2 = 0;
    auto p_loop = [&]() -> int {
        cudaGraphConditionalHandle h;
        CK(cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault));
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = h;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t n = nullptr;
        CK(cudaGraphAddNode(&n, g, prev ? &prev : nullptr, prev ? 1 : 0, &cp));
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        cudaGraphConditionalHandle hif;
        CK(cudaGraphConditionalHandleCreate(&hif, body, 0, cudaGraphCondAssignDefault));
        CK(cudaStreamBeginCaptureToGraph(b->st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        lh0 = b->launches;
        enq_p_first(b, bd);
        lh1 = b->launches;
        k_if_cond<<<1, 32, 0, b->st>>>(hif, b->flags + 0, b->flags + 8);
        cudaStreamCaptureStatus cst;
        const cudaGraphNode_t* deps = nullptr;
        size_t ndeps = 0;
        CK(cudaStreamGetCaptureInfo(b->st, &cst, nullptr, nullptr, &deps, &ndeps));
        std::vector<cudaGraphNode_t> tail(deps, deps + ndeps);
        cudaGraph_t out = nullptr;
        CK(cudaStreamEndCapture(b->st, &out));
        cudaGraphNodeParams ip = {};
        ip.type = cudaGraphNodeTypeConditional;
        ip.conditional.handle = hif;
        ip.conditional.type = cudaGraphCondTypeIf;
        ip.conditional.size = 1;
        cudaGraphNode_t ifn = nullptr;
        CK(cudaGraphAddNode(&ifn, body, tail.data(), tail.size(), &ip));
        CK(cudaStreamBeginCaptureToGraph(b->st, ip.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                         cudaStreamCaptureModeThreadLocal));
        enq_p_second(b, bd);
        lh2 = b->launches;
        CK(cudaStreamEndCapture(b->st, &out));
        CK(cudaStreamBeginCaptureToGraph(b->st, body, &ifn, nullptr, 1, cudaStreamCaptureModeThreadLocal));
        k_loop_cond<<<1, 32, 0, b->st>>>(h, b->flags + 0, b->flags + 3, b->maxit_p, b->flags + 6);
        CK(cudaStreamEndCapture(b->st, &out));
        prev = n;
        return CFD_OK;
    };
    const bool mixed = b->precision == CFD_PRECISION_MIXED;
    int rc = child([&] {
        enq_begin(b, bd);
        if (mixed) enq_mom_mx_first(b, bd);
    });
    const long long la = b->launches;
    if (!rc) rc = loop([&] {
        if (mixed) enq_mom_mx_next(b, bd);
        else enq_mom_pair(b, bd);
    }, b->flags + 1, b->flags + 2, mom_loop_cap(b), b->flags + 5);
    const long long lm = b->launches;
    if (!rc) rc = child([&] { enq_mid(b, bd); });
    const long long lp0 = b->launches;
    if (!rc) rc = p_loop();
    const long long lp1 = b->launches;
    if (!rc) rc = child([&] { enq_end(b, bd); });
    if (!rc) {
        // kernels per straight segment, per loop iteration (+2: the two condition kernels),
        // per executed second half
        b->launches_per_pair = (int)(lm - la) + 1;
        b->launches_per_iter = (int)(lh1 - lh0) + 2;
        b->launches_per_half = (int)(lh2 - lh1);
        b->launches_fixed = (int)((la - l0) + (lp0 - lm) + (b->launches - lp1));
        if (cudaGraphInstantiate(&b->gexec[cur], g, 0) != cudaSuccess) rc = fail(CFD_E_CUDA, "graph instantiation failed");
    }
    cudaGraphDestroy(g);
    b->launches = l0;
    b->prof = prof;
    return rc;
}

int one_step(cfd_batch* b) {
    int rc;
    if (b->ntable_cases == 0) return CFD_OK;  // an empty slot pool: nothing to step
    if (b->use_graph && !b->prof) {
        if (!b->gexec[b->cur]) {
            rc = build_step_graph(b, b->cur);
            if (rc) return rc;
        }
        CK(cudaGraphLaunch(b->gexec[b->cur], b->st));
        b->launches += b->launches_fixed;  // the loops' share is added from the device counters
    } else {
        rc = one_step_direct(b);
        if (rc) return rc;
    }
    b->cur ^= 1;
    b->steps_done++;
    if (b->prof) return flush_profile(b);
    return CFD_OK;
}

// adds the loop launches of graph steps (from the cumulative device counters) to the count
void drop_graphs(cfd_batch* b) {
    for (int k = 0; k < 2; k++)
        if (b->gexec[k]) {
            cudaGraphExecDestroy(b->gexec[k]);
            b->gexec[k] = nullptr;
        }
}

int account_graph_launches(cfd_batch* b) {
    if (!b->use_graph) return CFD_OK;
    int dummy = 0;
    int rc = read_flag(b, 0, &dummy);
    if (rc) return rc;
    const int tp = b->h_flags[5], ti = b->h_flags[6], th = b->h_flags[8];
    b->launches += (long long)(tp - b->flags_total0[0]) * b->launches_per_pair +
                   (long long)(ti - b->flags_total0[1]) * b->launches_per_iter +
                   (long long)(th - b->flags_total0[2]) * b->launches_per_half;
    b->flags_total0[0] = tp;
    b->flags_total0[1] = ti;
    b->flags_total0[2] = th;
    return CFD_OK;
}

int fetch_scalars(cfd_batch* b) {
    b->hscal.resize((size_t)b->n * NSCAL);
    b->hiscal.resize((size_t)b->n * NISCAL);
    CK(cudaMemcpyAsync(b->hscal.data(), b->scal, b->hscal.size() * sizeof(double), cudaMemcpyDeviceToHost, b->st));
    CK(cudaMemcpyAsync(b->hiscal.data(), b->iscal, b->hiscal.size() * sizeof(int), cudaMemcpyDeviceToHost, b->st));
    CK(cudaStreamSynchronize(b->st));

    return CFD_OK;
}

void fill_stats(cfd_batch* b, int c, cfd_step_stats* s) {
    const double* sc = b->hscal.data() + (size_t)c * NSCAL;
    const int* is = b->hiscal.data() + (size_t)c * NISCAL;
    memset(s, 0, sizeof(*s));
    s->status = is[I_STATUS] | is[I_PSTATUS];
    for (int f = 0; f < NFIELD; f++) s->it_mom[f] = is[I_MIT0 + f];
    s->it_p = is[I_PIT];
    s->dmax = sc[S_DMAX];
    s->cl = sc[S_CL]; s->cd = sc[S_CD]; s->cm = sc[S_CM]; s->nu = sc[S_NU]; s->circ = sc[S_CIRC];
    s->cl_pr = sc[S_CLP]; s->cd_pr = sc[S_CDP]; s->cl_vor = sc[S_CLV]; s->cd_vor = sc[S_CDV];
    s->q_l1 = sc[S_QL1]; s->q_l2 = sc[S_QL2]; s->q_max = sc[S_QMAX];
    s->dT_l1 = sc[S_DTL1]; s->dT_max = sc[S_DTMAX];
    s->p_res_rel = sc[S_NB1] > 0 ? sc[S_RL1] / sc[S_NB1] : 0.0;
    const double q0 = sc[S_QL2_0];
    s->mass_res_rel = q0 > 0 ? sc[S_QL2] / q0 : (sc[S_QL2] == 0 ? 0.0 : 1.0);
    s->steady_res = sc[S_SR];
    const double r0 = sc[S_SR0];
    s->steady_res_rel = r0 > 0 ? s->steady_res / r0 : (s->steady_res == 0 ? 0.0 : 1.0);
    s->steps = is[I_NSTEP];
    s->time = b->prm[c].time_accurate ? sc[S_TIME] : (double)is[I_TIME];
}

int plane_id(const char* name, int cur) {
    struct { const char* n; int id; } t[] = {
        {"x", P_X}, {"y", P_Y}, {"xix", P_XIX}, {"xiy", P_XIY}, {"etx", P_ETX}, {"ety", P_ETY},
        {"alph", P_ALPH}, {"beta", P_BETA}, {"gam", P_GAM}, {"jac", P_JAC},
        {"ap", P_AP}, {"ae", P_AE}, {"aw", P_AW}, {"an", P_AN}, {"as", P_AS}, {"ane", P_ANE},
        {"anw", P_ANW}, {"ase", P_ASE}, {"asw", P_ASW},
        {"u", P_U}, {"v", P_V}, {"p", P_P}, {"T", P_T0 + cur}, {"up", P_UP0 + cur}, {"vp", P_VP0 + cur},
        {"us", P_US}, {"vs", P_VS}, {"qu", P_RU}, {"qv", P_RV}, {"qt", P_RT}, {"qup", P_RUP},
        {"qvp", P_RVP}, {"q", P_Q}, {"pcor", P_PCOR}, {"vort", P_VORT}, {"si", P_SI}, {"dil", P_DIL}};
    for (auto& e : t)
        if (strcmp(e.n, name) == 0) return e.id;
    return -1;
}

}  // namespace

// Grid, normals, initial state, descriptor and per-case scalars of case `c` (a slot of the
// batch); with `setup` also its pressure stencil and multigrid hierarchy. Every copy goes on
// the batch's stream: that stream is non-blocking, so a copy on the legacy default stream
// would not be ordered before the kernels that read it (a synchronous copy from pageable
// memory may return before its DMA lands). From pageable memory the call returns once the
// source is staged, so the host vectors may be reused or freed right after it.
namespace {
// plane `plane_id` of case `d` from a host [n1][n0] array, padded
int put_plane(cfd_batch* b, const CaseDev& d, int plane_id, const double* src, std::vector<double>& pad) {
    pad_plane(d, src, pad);
    CK(cudaMemcpyAsync(b->f64 + d.base + H - 16 + (long long)plane_id * d.ps, pad.data(), sizeof(double) * d.ps,
                       cudaMemcpyHostToDevice, b->st));
    return CFD_OK;
}

// Initial state, descriptor and per-case scalars of case `c` once its grid planes are in
// place, and with `setup` its pressure stencil and multigrid hierarchy. The initial state
// reads only n0, n1, row 0 of x and y and the outer normals xnox, xnoy of `g`; with
// `state_on_device` the caller has written the state planes already (k_init_state).
int upload_state(cfd_batch* b, int c, const cfd_grid& g, const cfd_params& p, bool setup,
                 bool state_on_device = false) {
    CaseDev& d = b->hc[c];
    if (!state_on_device) {
        std::vector<double> pad;
        std::vector<double> st[6];
        initial_state(&g, &p, d, st);
        const int sid[6] = {P_U, P_V, P_T0 + b->cur, P_UP0 + b->cur, P_VP0 + b->cur, P_P};
        for (int m = 0; m < 6; m++)
            if (int rc = put_plane(b, d, sid[m], st[m].data(), pad)) return rc;
    }
    CK(cudaMemcpyAsync(b->dc + c, &d, sizeof(CaseDev), cudaMemcpyHostToDevice, b->st));
    std::vector<double> sc(NSCAL, 0.0);
    std::vector<int> is(NISCAL, 0);
    is[I_ACTIVE] = 1;
    CK(cudaMemcpyAsync(b->scal + (size_t)c * NSCAL, sc.data(), sizeof(double) * NSCAL, cudaMemcpyHostToDevice, b->st));
    CK(cudaMemcpyAsync(b->iscal + (size_t)c * NISCAL, is.data(), sizeof(int) * NISCAL, cudaMemcpyHostToDevice, b->st));
    if (setup) {
        BatchDev bd = b->bd;
        k_assemble_p<<<d.tile_count, NT, 0, b->st>>>(bd, d.tile_begin);
        for (int l = 0; l + 1 < d.nlev; l++)
            k_mg_galerkin<<<d.lev[l + 1].tile_count, NT, 0, b->st>>>(bd, l, d.lev[l + 1].tile_begin);
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(b->st));
    }
    return CFD_OK;
}
}  // namespace

int upload_case(cfd_batch* b, int c, const cfd_grid& g, const cfd_params& p, bool setup) {
    CaseDev& d = b->hc[c];
    case_params_to_dev(d, g, p);
    b->prm[c] = p;
    std::vector<double> pad;
    auto put = [&](int plane_id, const double* src) -> int { return put_plane(b, d, plane_id, src, pad); };
    const double* gp[10] = {g.x, g.y, g.xix, g.xiy, g.etx, g.ety, g.alph, g.beta, g.gam, g.jac};
    const int gid[10] = {P_X, P_Y, P_XIX, P_XIY, P_ETX, P_ETY, P_ALPH, P_BETA, P_GAM, P_JAC};
    for (int m = 0; m < 10; m++)
        if (int rc = put(gid[m], gp[m])) return rc;
    std::vector<double> vec((size_t)g.n0 * g.n1, 0.0);  // normals as rows 0..3 of P_VEC
    const double* nv[4] = {g.xnix, g.xniy, g.xnox, g.xnoy};
    for (int r = 0; r < 4 && r < g.n1; r++)
        for (int i = 0; i < g.n0; i++) vec[(size_t)r * g.n0 + i] = nv[r][i];
    if (int rc = put(P_VEC, vec.data())) return rc;
    return upload_state(b, c, g, p, setup);
}

namespace {
// ---- a case's place in the arenas, and the tile tables over a set of cases

// the multigrid levels and the precision-form planes of case d in the FP32 arena from
// offset off32 (words, 32-aligned): G.words32() words
void place_levels(CaseDev& d, const CaseGeom& G, long long off32) {
    d.nlev = (int)G.lev.size();
    for (int l = 0; l < d.nlev; l++) {
        const LevelGeom& lg = G.lev[l];
        LevelDev& L = d.lev[l];
        L.W = lg.W; L.n1 = lg.n1; L.ld = lg.ld; L.ilo = lg.ilo; L.ihi = lg.ihi; L.nlo = lg.ilo;
        L.base = off32 + 32 - H;
        L.ps = lg.ps;
        off32 += (long long)NMG * lg.ps + 32;
        off32 = rup(off32, 32);
    }
    d.xld = G.xld;
    d.xps = G.xps;
    d.xbase = off32 + 32 - H32;
}

int set_kernel_attributes(cfd_batch* b) {
    b->sw_smem = b->precision == CFD_PRECISION_MIXED ? sweep_smem_mx0() : sweep_smem_f64();
    const void* swk = b->precision == CFD_PRECISION_MIXED ? (const void*)k_sweep_mx0 : (const void*)k_sweep_f64;
    CK(cudaFuncSetAttribute(swk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b->sw_smem));
    if (b->precision == CFD_PRECISION_MIXED) {
        // six CTAs of the FP32 sweep per SM need the largest shared-memory carve-out
        b->sw_smem1 = sweep_smem_mx1();
        CK(cudaFuncSetAttribute(k_sweep_mx1, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b->sw_smem1));
        CK(cudaFuncSetAttribute(k_sweep_mx1, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
    }
    CK(cudaFuncSetAttribute(swk, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
    CK(cudaFuncSetAttribute(k_rhs, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kRhsSmem));
    CK(cudaFuncSetAttribute(k_face_q, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFaceQSmem));
    return CFD_OK;
}

// grows a device table to at least `need` entries of `sz` bytes (contents not kept)
template <typename T>
int grow(T*& ptr, size_t& cap, size_t need) {
    need = std::max<size_t>(need, 1);
    if (need <= cap) return CFD_OK;
    cudaFree(ptr);
    ptr = nullptr;
    cap = 0;
    const cudaError_t e = cudaMalloc((void**)&ptr, sizeof(T) * need);
    if (e != cudaSuccess) return fail(CFD_E_OOM, std::string("tile tables: ") + cudaGetErrorString(e));
    cap = need;
    return CFD_OK;
}

// The tile tables of the cases `ids` (in that order; a case's tiles in row-major tile order,
// so every per-case reduction sums in the same order whatever else is in the tables), each
// case's offsets into them, the batch-wide maxima the launches use, and the device copies.
// The step graphs hold the old tables and are dropped.
int build_tables(cfd_batch* b, const std::vector<int>& ids) {
    CK(cudaStreamSynchronize(b->st));
    std::vector<Tile> ftiles, jtiles;
    std::vector<std::vector<Tile>> at(MAXLEV), mt(MAXLEV);
    std::vector<std::vector<int>> cc(MAXLEV);
    b->nlev_max = 0;
    b->max_W = 0;
    b->maxit_mom = 0;
    b->maxit_p = 0;
    for (int l = 0; l < MAXLEV; l++) b->ncol[l] = 0;
    int jt_max = 0;
    for (int c : ids) {
        CaseDev& d = b->hc[c];
        d.tile_begin = (int)ftiles.size();
        make_tiles(d.ilo, d.ihi, d.n1, c, ftiles);
        d.tile_count = (int)ftiles.size() - d.tile_begin;
        d.jt_begin = (int)jtiles.size();
        make_tiles(d.ilo, d.ihi, d.n1, c, jtiles, TYJ);
        d.jt_count = (int)jtiles.size() - d.jt_begin;
        for (int l = 0; l < d.nlev; l++) {
            LevelDev& L = d.lev[l];
            L.tile_begin = (int)at[l].size();
            make_tiles(L.ilo, L.ihi, L.n1, c, at[l]);
            L.tile_count = (int)at[l].size() - L.tile_begin;
            if (l < d.nlev - 1) make_tiles(L.ilo, L.ihi, L.n1, c, mt[l], TYJ);
            else cc[l].push_back(c);
            b->ncol[l] = std::max(b->ncol[l], (d.periodic && (L.W & 1)) ? 6 : 4);
        }
        b->nlev_max = std::max(b->nlev_max, d.nlev);
        b->max_W = std::max(b->max_W, d.W);
        b->maxit_mom = std::max(b->maxit_mom, b->prm[c].maxit_mom);
        b->maxit_p = std::max(b->maxit_p, b->prm[c].maxit_p);
        jt_max = std::max(jt_max, d.jt_count);
    }
    std::vector<Tile> all(ftiles);
    const size_t pos_jt = all.size();
    all.insert(all.end(), jtiles.begin(), jtiles.end());
    std::vector<int> allcc;
    size_t pos_at[MAXLEV], pos_mt[MAXLEV], pos_cc[MAXLEV];
    for (int l = 0; l < MAXLEV; l++) {
        pos_at[l] = all.size();
        all.insert(all.end(), at[l].begin(), at[l].end());
        pos_mt[l] = all.size();
        all.insert(all.end(), mt[l].begin(), mt[l].end());
        pos_cc[l] = allcc.size();
        allcc.insert(allcc.end(), cc[l].begin(), cc[l].end());
    }
    if (int rc = grow(b->dtiles, b->cap_tiles, all.size())) return rc;
    if (int rc = grow(b->dcc, b->cap_cc, allcc.size())) return rc;
    if (int rc = grow(b->partial, b->cap_partial, PSTRIDE * std::max(ftiles.size(), jtiles.size() * SW_WARPS)))
        return rc;
    if (int rc = grow(b->tword, b->cap_tword, jtiles.size())) return rc;
    if (!all.empty())
        CK(cudaMemcpyAsync(b->dtiles, all.data(), sizeof(Tile) * all.size(), cudaMemcpyHostToDevice, b->st));
    if (!allcc.empty())
        CK(cudaMemcpyAsync(b->dcc, allcc.data(), sizeof(int) * allcc.size(), cudaMemcpyHostToDevice, b->st));
    CK(cudaMemcpyAsync(b->dc, b->hc.data(), sizeof(CaseDev) * b->n, cudaMemcpyHostToDevice, b->st));
    BatchDev& bd = b->bd;
    bd.partial = b->partial;
    bd.tword = b->tword;
    bd.ftiles = b->dtiles;
    bd.nftiles = (int)ftiles.size();
    bd.jtiles = b->dtiles + pos_jt;
    bd.njtiles = (int)jtiles.size();
    for (int l = 0; l < MAXLEV; l++) {
        bd.atiles[l] = b->dtiles + pos_at[l]; bd.natiles[l] = (int)at[l].size();
        bd.mtiles[l] = b->dtiles + pos_mt[l]; bd.nmtiles[l] = (int)mt[l].size();
        bd.ccases[l] = b->dcc + pos_cc[l]; bd.nccases[l] = (int)cc[l].size();
    }
    b->ntable_cases = (int)ids.size();
    b->sw_grid = (int)jtiles.size();  // one CTA per 32 x 16 tile
    b->swf_threads = jt_max >= 1024 ? SWF_THREADS : 128;
    const size_t bc_smem = 2 * (size_t)(b->max_W + 1) * sizeof(double);
    if (bc_smem > 48 * 1024)
        CK(cudaFuncSetAttribute(k_bc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bc_smem));
    drop_graphs(b);
    CK(cudaStreamSynchronize(b->st));
    return CFD_OK;
}

// the case's five 3-D tensor maps (x, y = row, z = plane): over the FP64 planes from the halo
// column -2 (x = column + 2), boxes 36 x 20 (tile + halo), 32 x 16 (tile) and 32 x 16 x 3
// (three consecutive planes); over the FP32 correction planes from column -4 (x = column + 4,
// so both boxes start on 16-byte boundaries), 40 x 20 and 32 x 16
int encode_tmaps(cfd_batch* b, const CaseDev& d, unsigned char* mc) {
    EncodeTiledFn enc = tensor_map_encoder();
    if (!enc) return fail(CFD_E_CUDA, "cuTensorMapEncodeTiled unavailable");
    const cuuint32_t es[3] = {1, 1, 1};
    auto make = [&](int off, CUtensorMapDataType ty, void* gaddr, const cuuint64_t* dims, const cuuint64_t* strides,
                    const cuuint32_t* box) {
        return enc(reinterpret_cast<CUtensorMap*>(mc + off), ty, 3, gaddr, dims, strides, box, es,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    };
    const cuuint64_t d64[3] = {(cuuint64_t)d.ld, (cuuint64_t)d.n1, (cuuint64_t)NPLANES};
    const cuuint64_t s64[2] = {(cuuint64_t)d.ld * 8, (cuuint64_t)d.ps * 8};
    const cuuint32_t bh[3] = {TX + 4, TYJ + 4, 1}, bt[3] = {TX, TYJ, 1}, bt3[3] = {TX, TYJ, 3};
    const cuuint64_t d32[3] = {(cuuint64_t)d.xld, (cuuint64_t)d.n1, (cuuint64_t)NXPLANES};
    const cuuint64_t s32[2] = {(cuuint64_t)d.xld * 4, (cuuint64_t)d.xps * 4};
    const cuuint32_t xh[3] = {TX + 8, TYJ + 4, 1};
    void* g64 = b->f64 + d.base + H - 2;
    void* g32 = b->f32 + d.xbase;
    CUresult r = make(TMAP_F64_HALO, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, g64, d64, s64, bh);
    if (r == CUDA_SUCCESS) r = make(TMAP_F64_TILE, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, g64, d64, s64, bt);
    if (r == CUDA_SUCCESS) r = make(TMAP_F64_TILE3, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, g64, d64, s64, bt3);
    if (r == CUDA_SUCCESS) r = make(TMAP_X32_HALO, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, g32, d32, s32, xh);
    if (r == CUDA_SUCCESS) r = make(TMAP_X32_TILE, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, g32, d32, s32, bt);
    if (r != CUDA_SUCCESS) return fail(CFD_E_CUDA, "cuTensorMapEncodeTiled failed");
    return CFD_OK;
}
}  // namespace

int cfd_internal_grid_gen(const cfd_grid_spec* spec, double* d_planes, double* d_normals, cudaStream_t stream);

// Case `c` from a grid generated on the device into `gen` (10 planes, 4 normal rows, 5
// scan words): the bound scan and metric check run on the device and only their results,
// row 0 of x and y and the normals come back; the slot's grid planes are written from
// `gen` on the device, and only after the check has passed.
int upload_case_generated(cfd_batch* b, int c, const cfd_grid_spec& spec, const cfd_params& p, double* gen) {
    CaseDev& d = b->hc[c];
    const int n0 = spec.n0, n1 = spec.n1;
    const long long np = (long long)n0 * n1;
    double* nrm = gen + 10 * np;
    unsigned long long* scan = reinterpret_cast<unsigned long long*>(nrm + 4LL * n0);
    if (int rc = cfd_internal_grid_gen(&spec, gen, nrm, b->st)) return rc;
    const double dxi0 = 1.0 / (n0 - 1), dxi1 = 1.0 / (n1 - 1);
    const ChebScan cs = cheb_consts(p, dxi0, dxi1);
    CK(cudaMemsetAsync(scan, 0, 5 * sizeof(unsigned long long), b->st));
    const int sblocks = (int)std::min<long long>((np + SCAN_THREADS - 1) / SCAN_THREADS, 148LL * 8);
    k_grid_scan<<<sblocks, SCAN_THREADS, 0, b->st>>>(gen, n0, n1, cs, scan);
    CK(cudaGetLastError());
    unsigned long long hs[5];
    CK(cudaMemcpyAsync(hs, scan, sizeof(hs), cudaMemcpyDeviceToHost, b->st));
    CK(cudaStreamSynchronize(b->st));
    if (hs[4] != 0) return fail(CFD_E_ARG, "grid metrics invalid (alpha, gamma must be > 0)");
    double emax[2], rmax[2];
    for (int ty = 0; ty < 2; ty++) {
        memcpy(&emax[ty], &hs[ty], sizeof(double));
        memcpy(&rmax[ty], &hs[2 + ty], sizeof(double));
    }
    // the slot's grid planes: zero (as pad_plane leaves every entry it does not set), then fill
    double* region = b->f64 + d.base + H - 16;
    CK(cudaMemsetAsync(region, 0, sizeof(double) * 10 * d.ps, b->st));
    CK(cudaMemsetAsync(region + (long long)P_VEC * d.ps, 0, sizeof(double) * d.ps, b->st));
    const long long nput = 11LL * n1 * (d.periodic ? d.W + 2 * H : n0);
    k_grid_to_slot<<<(unsigned)((nput + 255) / 256), 256, 0, b->st>>>(gen, n0, n1, d.W, d.periodic, region, d.ps,
                                                                      d.ld);
    CK(cudaGetLastError());
    const double ar = spec.profile == CFD_PROFILE_OGRID ? spec.ar : 1.0;
    case_scalars_to_dev(d, dxi0, dxi1, ar, p);
    cheb_finish(emax, rmax, d);
    b->prm[c] = p;
    // the initial state on the device as well: nothing of the case crosses PCIe
    const int sid[6] = {P_U, P_V, P_T0 + b->cur, P_UP0 + b->cur, P_VP0 + b->cur, P_P};
    for (int m = 0; m < 6; m++) CK(cudaMemsetAsync(region + (long long)sid[m] * d.ps, 0, sizeof(double) * d.ps, b->st));
    const long long nst = (long long)n1 * (d.periodic ? d.W + 2 * H : n0);
    k_init_state<<<(unsigned)((nst + 255) / 256), 256, 0, b->st>>>(
        region, d.ps, d.ld, n0, n1, d.W, d.periodic, spec.profile == CFD_PROFILE_CAVITY, gen + (long long)P_X * np,
        gen + (long long)P_Y * np, d.uinf, d.vinf, d.speed_amp, d.lid_u, sid[0], sid[1], sid[2], sid[3], sid[4]);
    CK(cudaGetLastError());
    cfd_grid g{};
    g.n0 = n0;
    g.n1 = n1;
    g.dxi0 = dxi0;
    g.dxi1 = dxi1;
    g.ar = ar;
    return upload_state(b, c, g, p, true, true);
}

// ==========================================================================
extern "C" {

void cfd_params_default(cfd_params* p) {
    if (!p) return;
    memset(p, 0, sizeof(*p));
    p->Re = 1000.0; p->Ri = 0.0; p->Pr = 0.71; p->F = 0.0; p->alpha_deg = 82.0; p->dt = 0.01e-2;
    p->tol_mom = 0.75e-2; p->atol_mom = 0.0; p->tol_p = 0.75e-2; p->atol_p = 0.0;
    p->maxit_mom = 100; p->maxit_p = 200;
    p->profile = CFD_PROFILE_OGRID;
    p->fix_T_annw = 0; p->fix_circ_de = 0; p->warm_start = 1;
    p->omega_p = 1.0; p->lid_u = 1.0;
    p->precision = CFD_PRECISION_FP64;
    p->time_accurate = 0;
}

const char* cfd_last_error(void) { return g_err.c_str(); }

int cfd_set_device(int device) {
    CK(cudaSetDevice(device));
    return CFD_OK;
}

int cfd_device_count(int* count) {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (count) *count = (e == cudaSuccess) ? n : 0;
    if (e != cudaSuccess) return fail(CFD_E_CUDA, std::string("cudaGetDeviceCount: ") + cudaGetErrorString(e));
    return CFD_OK;
}

size_t cfd_case_bytes(int n0, int n1, int profile) {
    if (n0 < 8 || n1 < 6) return 0;
    CaseGeom g = case_geom(n0, n1, profile);
    long long ntiles = (long long)((n1 - 2 + TY - 1) / TY) * ((g.W + TX - 1) / TX + 1);
    return (size_t)(g.bytes64() * 8 + g.words32() * 4 + ntiles * (PSTRIDE * 8 + sizeof(Tile) * 3) +
                    sizeof(CaseDev) + (NSCAL * 8 + NISCAL * 4));
}

int cfd_batch_create(int ncases, const cfd_grid* grids, const cfd_params* params, cfd_batch** out) {
    if (!out || ncases <= 0 || !grids || !params) return fail(CFD_E_ARG, "bad batch arguments");
    *out = nullptr;
    for (int c = 0; c < ncases; c++) {
        int rc = check_params(&grids[c], &params[c]);
        if (rc) return fail(rc, "case " + std::to_string(c) + ": " + g_err);
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(CFD_E_CUDA, "no CUDA device available (this library has no CPU path)");
    cfd_batch* b = new cfd_batch();
    b->n = ncases;
    cudaGetDevice(&b->dev);
    auto cleanup = [&](int rc) { cfd_batch_destroy(b); return rc; };
    if (cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking) != cudaSuccess)
        return cleanup(fail(CFD_E_CUDA, "stream creation failed"));

    // ---- geometry, offsets
    long long off64 = 0, off32 = 0;
    b->hc.resize(ncases);
    b->prm.assign(params, params + ncases);
    b->q_l2_first.assign(ncases, -1.0);
    b->sr_first.assign(ncases, -1.0);
    for (int c = 0; c < ncases; c++) {
        const cfd_grid& g = grids[c];
        const cfd_params& p = params[c];
        CaseGeom G = case_geom(g.n0, g.n1, p.profile);
        b->geom.push_back(G);
        CaseDev& d = b->hc[c];
        memset(&d, 0, sizeof(d));
        d.W = G.W; d.n0 = g.n0; d.n1 = g.n1; d.ld = G.ld;
        d.periodic = G.periodic; d.ilo = G.ilo; d.ihi = G.ihi; d.profile = p.profile;
        d.base = off64 + 16 - H;
        d.ps = G.ps;
        off64 += G.bytes64() - 16 + 16;
        off64 = rup(off64, 16);
        case_params_to_dev(d, g, p);
        place_levels(d, G, off32);
        off32 += G.words32();
        off32 = rup(off32, 32);
        b->max_W = std::max(b->max_W, d.W);
        if (c == 0) b->precision = p.precision;
        if (p.precision != b->precision)
            return cleanup(fail(CFD_E_ARG, "all cases of a batch must use the same precision"));
    }
    if (b->max_W > 4096) return cleanup(fail(CFD_E_ARG, "grid width above 4096 columns"));
    b->n64 = off64 + 16;
    b->n32 = off32 + 32;

    // ---- device allocations (the tile tables: build_tables)
#define ALLOC(ptr, bytes)                                                         \
    do {                                                                          \
        cudaError_t e_ = cudaMalloc((void**)&(ptr), (bytes));                     \
        if (e_ != cudaSuccess)                                                    \
            return cleanup(fail(CFD_E_OOM, std::string("cudaMalloc ") + #ptr + ": " + cudaGetErrorString(e_))); \
    } while (0)
    ALLOC(b->f64, (size_t)b->n64 * sizeof(double));
    ALLOC(b->f32, (size_t)b->n32 * sizeof(float));
    ALLOC(b->dc, sizeof(CaseDev) * ncases);
    ALLOC(b->scal, sizeof(double) * NSCAL * ncases);
    ALLOC(b->iscal, sizeof(int) * NISCAL * ncases);
    ALLOC(b->counter, sizeof(unsigned) * ncases);
    ALLOC(b->flags, sizeof(int) * NFLAGS);
    ALLOC(b->work, sizeof(unsigned long long) * 4);
    ALLOC(b->dtmaps, (size_t)TMAP_STRIDE * ncases);
#undef ALLOC
    if (cudaHostAlloc((void**)&b->h_flags, sizeof(int) * NFLAGS, cudaHostAllocDefault) != cudaSuccess)
        return cleanup(fail(CFD_E_CUDA, "pinned allocation failed"));
    cudaMemsetAsync(b->f64, 0, (size_t)b->n64 * sizeof(double), b->st);
    cudaMemsetAsync(b->f32, 0, (size_t)b->n32 * sizeof(float), b->st);
    cudaMemsetAsync(b->scal, 0, sizeof(double) * NSCAL * ncases, b->st);
    cudaMemsetAsync(b->iscal, 0, sizeof(int) * NISCAL * ncases, b->st);
    cudaMemsetAsync(b->counter, 0, sizeof(unsigned) * ncases, b->st);
    cudaMemsetAsync(b->work, 0, sizeof(unsigned long long) * 4, b->st);
    cudaMemsetAsync(b->flags, 0, sizeof(int) * NFLAGS, b->st);
    CK(cudaStreamSynchronize(b->st));
    {
        const size_t smem = 2 * (size_t)(b->max_W + 1) * sizeof(double);
        if (smem > 48 * 1024)
            CK(cudaFuncSetAttribute(k_bc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        if (int rc = set_kernel_attributes(b)) return cleanup(rc);
    }

    BatchDev& bd = b->bd;
    bd.cases = b->dc; bd.ncases = ncases; bd.f64 = b->f64; bd.f32 = b->f32;
    bd.scal = b->scal; bd.iscal = b->iscal; bd.counter = b->counter;
    bd.active = b->flags; bd.mactive = b->flags + 1;
    bd.work = b->work;
    bd.tmaps = b->dtmaps;
    // ---- tile tables over every case
    {
        std::vector<int> ids(ncases);
        for (int c = 0; c < ncases; c++) ids[c] = c;
        if (int rc = build_tables(b, ids)) return cleanup(rc);
    }
    {
        std::vector<unsigned char> maps((size_t)TMAP_STRIDE * ncases);
        for (int c = 0; c < ncases; c++)
            if (int rc = encode_tmaps(b, b->hc[c], maps.data() + (size_t)TMAP_STRIDE * c))
                return cleanup(rc);
        CK(cudaMemcpyAsync(b->dtmaps, maps.data(), maps.size(), cudaMemcpyHostToDevice, b->st));
    }
    bd.error = b->flags + 4;
    bd.wait_polls = kWaitPolls;
    bd.mg_res = mg_res_plane(b->mg_pre, b->mg_post, b->mg_fused);
    bd.mixed = b->precision == CFD_PRECISION_MIXED;

    // ---- upload grid + initial state (padded planes with halos)
    b->cur = 0;
    bd.cur = 0;
    for (int c = 0; c < ncases; c++) {
        int rc = upload_case(b, c, grids[c], params[c], false);
        if (rc) return cleanup(rc);
    }
    // ---- set-up kernels: pressure stencil, multigrid hierarchy
    {
        Prof pr(b, K_ASSEMBLE_P);
        k_assemble_p<<<bd.nftiles, NT, 0, b->st>>>(bd, 0);
    }
    for (int l = 0; l + 1 < b->nlev_max; l++) {
        if (bd.natiles[l + 1] == 0) continue;
        Prof pr(b, K_MG_GALERKIN);
        k_mg_galerkin<<<bd.natiles[l + 1], NT, 0, b->st>>>(bd, l, 0);
    }
    if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(b->st) != cudaSuccess)
        return cleanup(fail(CFD_E_CUDA, "set-up kernels failed"));
    flush_profile(b);
    *out = b;
    return CFD_OK;
}

// ---- slot pool: cases placed in one byte arena at admission (no counterpart in the reference)
namespace {
constexpr size_t kPoolAlign = 256;

// the bytes a case takes in a pool: its FP64 planes, then its FP32 levels and planes
size_t pool_case_bytes(const CaseGeom& G) {
    return rup((long long)G.bytes64() * 8, kPoolAlign) + rup((long long)G.words32() * 4, kPoolAlign);
}

// first fit in the sorted free list; returns false when no region is large enough
bool pool_take(cfd_batch* b, size_t bytes, size_t* off) {
    for (size_t k = 0; k < b->pool_free.size(); k++) {
        auto& f = b->pool_free[k];
        if (f.second < bytes) continue;
        *off = f.first;
        f.first += bytes;
        f.second -= bytes;
        if (f.second == 0) b->pool_free.erase(b->pool_free.begin() + (long)k);
        return true;
    }
    return false;
}

// returns a region to the free list, merging it with its neighbours
void pool_give(cfd_batch* b, size_t off, size_t bytes) {
    auto& v = b->pool_free;
    auto it = std::lower_bound(v.begin(), v.end(), std::make_pair(off, (size_t)0));
    it = v.insert(it, {off, bytes});
    if (it + 1 != v.end() && it->first + it->second == (it + 1)->first) {
        it->second += (it + 1)->second;
        v.erase(it + 1);
    }
    if (it != v.begin() && (it - 1)->first + (it - 1)->second == it->first) {
        (it - 1)->second += it->second;
        v.erase(it);
    }
}

std::vector<int> pool_ids(const cfd_batch* b) {
    std::vector<int> ids;
    for (int c = 0; c < b->n; c++)
        if (b->pool_region[c].second) ids.push_back(c);
    return ids;
}
}  // namespace

int cfd_pool_create(size_t hbm_budget, int max_cases, int precision, cfd_batch** out) {
    if (!out || max_cases <= 0 || max_cases > (1 << 16) || hbm_budget < (1u << 20) ||
        (precision != CFD_PRECISION_FP64 && precision != CFD_PRECISION_MIXED))
        return fail(CFD_E_ARG, "cfd_pool_create: bad arguments");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(CFD_E_CUDA, "no CUDA device available (this library has no CPU path)");
    cfd_batch* b = new cfd_batch();
    b->n = max_cases;
    b->is_pool = true;
    b->precision = precision;
    cudaGetDevice(&b->dev);
    auto cleanup = [&](int rc) { cfd_batch_destroy(b); return rc; };
    if (cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking) != cudaSuccess)
        return cleanup(fail(CFD_E_CUDA, "stream creation failed"));
    b->hc.assign(max_cases, CaseDev{});
    cfd_params dp;
    cfd_params_default(&dp);
    dp.precision = precision;
    b->prm.assign(max_cases, dp);
    b->geom.assign(max_cases, CaseGeom{});
    b->pool_region.assign(max_cases, {0, 0});
    b->pool_bytes = hbm_budget / kPoolAlign * kPoolAlign;
    b->pool_free.push_back({0, b->pool_bytes});
#define ALLOC(ptr, bytes)                                                         \
    do {                                                                          \
        cudaError_t e_ = cudaMalloc((void**)&(ptr), (bytes));                     \
        if (e_ != cudaSuccess)                                                    \
            return cleanup(fail(CFD_E_OOM, std::string("cudaMalloc ") + #ptr + ": " + cudaGetErrorString(e_))); \
    } while (0)
    ALLOC(b->f64, b->pool_bytes);
    b->f32 = reinterpret_cast<float*>(b->f64);  // one arena: a case's FP32 part follows its FP64 part
    b->n64 = (long long)(b->pool_bytes / 8);
    b->n32 = (long long)(b->pool_bytes / 4);
    ALLOC(b->dc, sizeof(CaseDev) * max_cases);
    ALLOC(b->scal, sizeof(double) * NSCAL * max_cases);
    ALLOC(b->iscal, sizeof(int) * NISCAL * max_cases);
    ALLOC(b->counter, sizeof(unsigned) * max_cases);
    ALLOC(b->flags, sizeof(int) * NFLAGS);
    ALLOC(b->work, sizeof(unsigned long long) * 4);
    ALLOC(b->dtmaps, (size_t)TMAP_STRIDE * max_cases);
#undef ALLOC
    if (cudaHostAlloc((void**)&b->h_flags, sizeof(int) * NFLAGS, cudaHostAllocDefault) != cudaSuccess)
        return cleanup(fail(CFD_E_CUDA, "pinned allocation failed"));
    // every slot starts empty: inactive, its pressure solve done, no momentum word
    std::vector<int> is((size_t)NISCAL * max_cases, 0);
    for (int c = 0; c < max_cases; c++) is[(size_t)c * NISCAL + I_PDONE] = 1;
    if (cudaMemsetAsync(b->scal, 0, sizeof(double) * NSCAL * max_cases, b->st) != cudaSuccess ||
        cudaMemcpyAsync(b->iscal, is.data(), sizeof(int) * is.size(), cudaMemcpyHostToDevice, b->st) != cudaSuccess ||
        cudaMemsetAsync(b->counter, 0, sizeof(unsigned) * max_cases, b->st) != cudaSuccess ||
        cudaMemsetAsync(b->work, 0, sizeof(unsigned long long) * 4, b->st) != cudaSuccess ||
        cudaMemsetAsync(b->flags, 0, sizeof(int) * NFLAGS, b->st) != cudaSuccess ||
        cudaStreamSynchronize(b->st) != cudaSuccess)
        return cleanup(fail(CFD_E_CUDA, "pool initialisation failed"));
    if (int rc = set_kernel_attributes(b)) return cleanup(rc);
    BatchDev& bd = b->bd;
    bd.cases = b->dc; bd.ncases = max_cases; bd.f64 = b->f64; bd.f32 = b->f32;
    bd.scal = b->scal; bd.iscal = b->iscal; bd.counter = b->counter;
    bd.active = b->flags; bd.mactive = b->flags + 1;
    bd.work = b->work;
    bd.tmaps = b->dtmaps;
    bd.error = b->flags + 4;
    bd.wait_polls = kWaitPolls;
    bd.mg_res = mg_res_plane(b->mg_pre, b->mg_post, b->mg_fused);
    bd.mixed = precision == CFD_PRECISION_MIXED;
    if (int rc = build_tables(b, {})) return cleanup(rc);
    *out = b;
    return CFD_OK;
}

int cfd_pool_admit(cfd_batch* b, const cfd_grid* g, const cfd_params* p, int* slot) {
    if (!b || !b->is_pool || !slot) return fail(CFD_E_ARG, "cfd_pool_admit: not a slot pool");
    *slot = -1;
    int rc = check_params(g, p);
    if (rc) return rc;
    if (p->precision != b->precision) return fail(CFD_E_ARG, "case precision differs from the pool's");
    int c = 0;
    while (c < b->n && b->pool_region[c].second) c++;
    if (c == b->n) return fail(CFD_E_OOM, "every case slot of the pool is taken");
    const CaseGeom G = case_geom(g->n0, g->n1, p->profile);
    if (G.W > 4096) return fail(CFD_E_ARG, "grid width above 4096 columns");
    const size_t bytes = pool_case_bytes(G);
    size_t off = 0;
    if (!pool_take(b, bytes, &off)) return fail(CFD_E_OOM, "no free region of the pool's budget fits this case");
    CK(cudaStreamSynchronize(b->st));
    CaseDev& d = b->hc[c];
    memset(&d, 0, sizeof(d));
    d.W = G.W; d.n0 = g->n0; d.n1 = g->n1; d.ld = G.ld;
    d.periodic = G.periodic; d.ilo = G.ilo; d.ihi = G.ihi; d.profile = p->profile;
    d.base = (long long)(off / 8) + 16 - H;
    d.ps = G.ps;
    case_params_to_dev(d, *g, *p);
    place_levels(d, G, (long long)((off + rup((long long)G.bytes64() * 8, kPoolAlign)) / 4));
    b->geom[c] = G;
    b->prm[c] = *p;
    b->pool_region[c] = {off, bytes};
    std::vector<unsigned char> maps(TMAP_STRIDE);
    auto undo = [&](int code) {
        pool_give(b, off, bytes);
        b->pool_region[c] = {0, 0};
        memset(&b->hc[c], 0, sizeof(CaseDev));
        build_tables(b, pool_ids(b));
        return code;
    };
    rc = encode_tmaps(b, d, maps.data());
    if (rc) return undo(rc);
    // the region may hold a retired case's planes: every plane starts from zero
    if (cudaMemsetAsync(reinterpret_cast<char*>(b->f64) + off, 0, bytes, b->st) != cudaSuccess ||
        cudaMemcpyAsync(b->dtmaps + (size_t)TMAP_STRIDE * c, maps.data(), TMAP_STRIDE, cudaMemcpyHostToDevice,
                        b->st) != cudaSuccess ||
        cudaMemsetAsync(b->scal + (size_t)c * NSCAL, 0, sizeof(double) * NSCAL, b->st) != cudaSuccess)
        return undo(fail(CFD_E_CUDA, "cfd_pool_admit: slot initialisation failed"));
    rc = build_tables(b, pool_ids(b));
    if (rc) return undo(rc);
    rc = upload_case(b, c, *g, *p, true);
    if (rc) return undo(rc);
    *slot = c;
    return CFD_OK;
}

int cfd_pool_release(cfd_batch* b, int slot) {
    if (!b || !b->is_pool || slot < 0 || slot >= b->n || !b->pool_region[slot].second)
        return fail(CFD_E_ARG, "cfd_pool_release: not an occupied slot of a pool");
    CK(cudaStreamSynchronize(b->st));
    // the entry leaves every launch: inactive, its pressure solve done, no momentum word
    int w[NISCAL];
    CK(cudaMemcpy(w, b->iscal + (size_t)slot * NISCAL, sizeof(w), cudaMemcpyDeviceToHost));
    w[I_ACTIVE] = 0;
    w[I_PDONE] = 1;
    w[I_MWORD] = 0;
    CK(cudaMemcpy(b->iscal + (size_t)slot * NISCAL, w, sizeof(w), cudaMemcpyHostToDevice));
    pool_give(b, b->pool_region[slot].first, b->pool_region[slot].second);
    b->pool_region[slot] = {0, 0};
    memset(&b->hc[slot], 0, sizeof(CaseDev));
    b->geom[slot] = CaseGeom{};
    return build_tables(b, pool_ids(b));
}

int cfd_pool_free(cfd_batch* b, size_t* free_bytes, size_t* largest) {
    if (!b || !b->is_pool) return fail(CFD_E_ARG, "cfd_pool_free: not a slot pool");
    size_t tot = 0, big = 0;
    for (auto& f : b->pool_free) {
        tot += f.second;
        big = std::max(big, f.second);
    }
    if (free_bytes) *free_bytes = tot;
    if (largest) *largest = big;
    return CFD_OK;
}

size_t cfd_pool_case_bytes(int n0, int n1, int profile) {
    if (n0 < 8 || n1 < 6) return 0;
    return pool_case_bytes(case_geom(n0, n1, profile));
}

int cfd_batch_step(cfd_batch* b, int nsteps) {
    if (!b || nsteps < 0) return fail(CFD_E_ARG, "bad arguments");
    for (int s = 0; s < nsteps; s++) {
        int rc = one_step(b);
        if (rc) return rc;
    }
    CK(cudaStreamSynchronize(b->st));
    return account_graph_launches(b);
}

int cfd_batch_stats(cfd_batch* b, int case_index, cfd_step_stats* out) {
    if (!b || !out || case_index < 0 || case_index >= b->n) return fail(CFD_E_ARG, "bad arguments");
    int rc = fetch_scalars(b);
    if (rc) return rc;
    fill_stats(b, case_index, out);
    return CFD_OK;
}

int cfd_batch_get_plane(cfd_batch* b, int case_index, const char* name, double* out) {
    if (!b || !name || !out || case_index < 0 || case_index >= b->n) return fail(CFD_E_ARG, "bad arguments");
    const CaseDev& d = b->hc[case_index];
    const int id = plane_id(name, b->cur);
    if (id < 0) return fail(CFD_E_ARG, std::string("unknown plane ") + name);
    if (id == P_SI) {
        b->bd.cur = b->cur;
        Prof pr(b, K_SI);
        k_si<<<b->n, BC_THREADS, 0, b->st>>>(b->bd);
    }
    std::vector<double> pad((size_t)d.ps);
    CK(cudaMemcpyAsync(pad.data(), b->f64 + d.base + H - 16 + (long long)id * d.ps, sizeof(double) * d.ps,
                       cudaMemcpyDeviceToHost, b->st));
    CK(cudaStreamSynchronize(b->st));
    unpad_plane(d, pad.data(), out);
    return CFD_OK;
}

int cfd_batch_destroy(cfd_batch* b) {
    if (!b) return CFD_OK;
    if (b->st) cudaStreamSynchronize(b->st);
    drop_graphs(b);
    for (auto& l : b->pending) { cudaEventDestroy(l.e0); cudaEventDestroy(l.e1); }
    for (auto e : b->pool) cudaEventDestroy(e);
    if ((void*)b->f32 != (void*)b->f64) cudaFree(b->f32);
    cudaFree(b->f64); cudaFree(b->dc); cudaFree(b->scal); cudaFree(b->iscal);
    cudaFree(b->stage); cudaFree(b->stage_off);
    cudaFree(b->partial); cudaFree(b->counter); cudaFree(b->flags); cudaFree(b->work); cudaFree(b->tword); cudaFree(b->dtiles); cudaFree(b->dcc); cudaFree(b->dtmaps);
    if (b->h_flags) cudaFreeHost(b->h_flags);
    if (b->st) cudaStreamDestroy(b->st);
    delete b;
    return CFD_OK;
}

int cfd_batch_set_mg(cfd_batch* b, int nu_pre, int nu_post, int coarse_sweeps, int fused) {
    if (!b) return fail(CFD_E_ARG, "null batch");
    if (nu_pre < 1 || nu_pre > 8 || nu_post < 1 || nu_post > 8 || coarse_sweeps < 1 || coarse_sweeps > 256 ||
        fused < 0 || fused > 2)
        return fail(CFD_E_ARG, "multigrid schedule out of range (sweeps 1..8, coarse sweeps 1..256, fused 0..2)");
    CK(cudaStreamSynchronize(b->st));
    b->mg_pre = nu_pre;
    b->mg_post = nu_post;
    b->coarse_sweeps = coarse_sweeps;
    b->mg_fused = fused;
    b->bd.mg_res = mg_res_plane(nu_pre, nu_post, fused);
    drop_graphs(b);  // the step graphs hold the old schedule
    return CFD_OK;
}

int cfd_batch_set_wait_limit(cfd_batch* b, long long polls) {
    if (!b) return fail(CFD_E_ARG, "null batch");
    CK(cudaStreamSynchronize(b->st));
    b->bd.wait_polls = polls < 0 ? kWaitPolls : (unsigned)std::min<long long>(polls, 0xffffffffll);
    drop_graphs(b);  // the step graphs hold the old limit in their kernel parameters
    return CFD_OK;
}

int cfd_batch_get_mg(cfd_batch* b, int* nu_pre, int* nu_post, int* coarse_sweeps, int* fused) {
    if (!b) return fail(CFD_E_ARG, "null batch");
    if (nu_pre) *nu_pre = b->mg_pre;
    if (nu_post) *nu_post = b->mg_post;
    if (coarse_sweeps) *coarse_sweeps = b->coarse_sweeps;
    if (fused) *fused = b->mg_fused;
    return CFD_OK;
}

// Times each candidate multigrid schedule over `steps` steps from the batch's current state
// (saved on the device and restored before every candidate and at the end), keeps the
// fastest and reports its time per step. The batch's state is unchanged on return.
int cfd_batch_autotune(cfd_batch* b, int steps, int* out_schedule, double* out_ms_per_step) {
    if (!b || steps < 1) return fail(CFD_E_ARG, "bad arguments");
    static const int cand[][4] = {{1, 1, 12, 0}, {1, 2, 12, 0}, {2, 1, 12, 0}, {2, 2, 12, 0},
                                  {1, 2, 12, 1}, {1, 3, 12, 1}, {2, 2, 12, 1}, {2, 3, 12, 1},
                                  {1, 2, 12, 2}, {1, 3, 12, 2}, {1, 4, 12, 2}, {1, 3, 8, 2},
                                  {2, 2, 12, 2}, {2, 3, 12, 2}};
    const int ncand = (int)(sizeof(cand) / sizeof(cand[0]));
    const size_t n64 = (size_t)b->n64 * sizeof(double), nsc = sizeof(double) * NSCAL * b->n,
                 nis = sizeof(int) * NISCAL * b->n;
    char* snap = nullptr;
    CK(cudaStreamSynchronize(b->st));
    if (cudaMalloc((void**)&snap, n64 + nsc + nis) != cudaSuccess)
        return fail(CFD_E_OOM, "autotune: no device memory for the state snapshot");
    const int cur0 = b->cur;
    const long long steps0 = b->steps_done, launches0 = b->launches;
    auto copy = [&](bool save) -> int {
        char* p = snap;
        const void* src[3] = {b->f64, b->scal, b->iscal};
        void* dst[3] = {b->f64, b->scal, b->iscal};
        const size_t nb[3] = {n64, nsc, nis};
        for (int k = 0; k < 3; k++) {
            cudaError_t e = save ? cudaMemcpyAsync(p, src[k], nb[k], cudaMemcpyDeviceToDevice, b->st)
                                 : cudaMemcpyAsync(dst[k], p, nb[k], cudaMemcpyDeviceToDevice, b->st);
            if (e != cudaSuccess) return fail(CFD_E_CUDA, "autotune: snapshot copy failed");
            p += nb[k];
        }
        b->cur = cur0;
        b->steps_done = steps0;
        return CFD_OK;
    };
    const int mp = b->mg_pre, mq = b->mg_post, mc = b->coarse_sweeps, mf = b->mg_fused;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    int rc = copy(true), best = -1;
    float best_ms = 0.f;
    for (int k = 0; k < ncand && !rc; k++) {
        rc = cfd_batch_set_mg(b, cand[k][0], cand[k][1], cand[k][2], cand[k][3]);
        if (!rc) rc = copy(false);
        if (!rc) rc = cfd_batch_step(b, 1);  // builds the step graphs of this schedule
        if (!rc) rc = copy(false);
        if (rc) break;
        cudaEventRecord(e0, b->st);
        rc = cfd_batch_step(b, steps);
        cudaEventRecord(e1, b->st);
        if (rc) break;
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (best < 0 || ms < best_ms) {
            best = k;
            best_ms = ms;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    int rc2 = rc ? cfd_batch_set_mg(b, mp, mq, mc, mf)
                 : cfd_batch_set_mg(b, cand[best][0], cand[best][1], cand[best][2], cand[best][3]);
    int rc3 = copy(false);
    if (!rc3) rc3 = cudaStreamSynchronize(b->st) == cudaSuccess ? CFD_OK : fail(CFD_E_CUDA, "autotune sync");
    cudaFree(snap);
    b->launches = launches0;
    if (rc) return rc;
    if (rc2) return rc2;
    if (rc3) return rc3;
    if (out_schedule)
        for (int q = 0; q < 4; q++) out_schedule[q] = cand[best][q];
    if (out_ms_per_step) *out_ms_per_step = best_ms / steps;
    return CFD_OK;
}

int cfd_batch_profile(cfd_batch* b, int enable) {
    if (!b) return fail(CFD_E_ARG, "null batch");
    int rc = flush_profile(b);
    b->prof = enable != 0;
    for (int k = 0; k < NKERNEL; k++) { b->kt_ms[k] = 0; b->kt_n[k] = 0; }
    return rc;
}

int cfd_batch_kernel_times(cfd_batch* b, const char** names, double* total_ms, long long* launches, int cap) {
    if (!b) return fail(CFD_E_ARG, "null batch");
    flush_profile(b);
    for (int k = 0; k < NKERNEL && k < cap; k++) {
        if (names) names[k] = kKernelNames[k];
        if (total_ms) total_ms[k] = b->kt_ms[k];
        if (launches) launches[k] = b->kt_n[k];
    }
    return NKERNEL;
}

int cfd_batch_sync(cfd_batch* b) {
    if (!b) return fail(CFD_E_ARG, "null batch");
    CK(cudaStreamSynchronize(b->st));
    return CFD_OK;
}

int cfd_batch_admit(cfd_batch* b, int slot, const cfd_grid* g, const cfd_params* p) {
    if (!b || slot < 0 || slot >= b->n) return fail(CFD_E_ARG, "bad slot");
    int rc = check_params(g, p);
    if (rc) return rc;
    const CaseDev& d = b->hc[slot];
    if (g->n0 != d.n0 || g->n1 != d.n1 || p->profile != d.profile)
        return fail(CFD_E_ARG, "case does not match the slot's geometry (n0, n1, profile)");
    if (p->precision != b->precision) return fail(CFD_E_ARG, "case precision differs from the batch's");
    CK(cudaStreamSynchronize(b->st));
    return upload_case(b, slot, *g, *p, true);
}

int cfd_batch_admit_spec(cfd_batch* b, int slot, const cfd_grid_spec* spec, const cfd_params* p) {
    if (!b || slot < 0 || slot >= b->n) return fail(CFD_E_ARG, "bad slot");
    if (!spec) return fail(CFD_E_ARG, "null grid spec");
    int rc = check_case_params(p);
    if (rc) return rc;
    const CaseDev& d = b->hc[slot];
    if (spec->n0 != d.n0 || spec->n1 != d.n1 || spec->profile != d.profile || p->profile != d.profile)
        return fail(CFD_E_ARG, "case does not match the slot's geometry (n0, n1, profile)");
    if (p->precision != b->precision) return fail(CFD_E_ARG, "case precision differs from the batch's");
    CK(cudaStreamSynchronize(b->st));
    const long long np = (long long)spec->n0 * spec->n1;
    double* gen = nullptr;
    CK(cudaMallocAsync((void**)&gen, sizeof(double) * (size_t)(10 * np + 4LL * spec->n0 + 5), b->st));
    rc = upload_case_generated(b, slot, *spec, *p, gen);
    cudaFreeAsync(gen, b->st);
    const cudaError_t e = cudaStreamSynchronize(b->st);
    if (rc) return rc;
    CK(e);
    return CFD_OK;
}

int cfd_batch_set_active(cfd_batch* b, int slot, int active) {
    if (!b || slot < 0 || slot >= b->n) return fail(CFD_E_ARG, "bad slot");
    const int v = active ? 1 : 0;
    CK(cudaMemcpyAsync(b->iscal + (size_t)slot * NISCAL + I_ACTIVE, &v, sizeof(int), cudaMemcpyHostToDevice, b->st));
    CK(cudaStreamSynchronize(b->st));
    return CFD_OK;
}

int cfd_batch_fetch_stats(cfd_batch* b, cfd_step_stats* out, int cap) {
    if (!b || !out) return fail(CFD_E_ARG, "bad arguments");
    int rc = fetch_scalars(b);
    if (rc) return rc;
    for (int c = 0; c < b->n && c < cap; c++) fill_stats(b, c, out + c);
    return CFD_OK;
}

void* cfd_batch_stream(cfd_batch* b) { return b ? (void*)b->st : nullptr; }

long long cfd_batch_launches(cfd_batch* b) { return b ? b->launches : -1; }

int cfd_batch_work(cfd_batch* b, unsigned long long* out4) {
    if (!b || !out4) return fail(CFD_E_ARG, "bad arguments");
    CK(cudaMemcpyAsync(out4, b->work, 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, b->st));
    CK(cudaStreamSynchronize(b->st));
    return CFD_OK;
}

// the resident state of every case: u, v, p, T, up, vp (n1 rows of the stored columns each,
// in case order) and 16 doubles of counters
static const int kStatePlanes = 6;

static long long state_doubles(const CaseDev& d) {
    return (long long)kStatePlanes * d.n1 * (d.periodic ? d.W : d.n0) + 16;
}

size_t cfd_batch_state_bytes(cfd_batch* b) {
    if (!b) return 0;
    size_t s = 0;
    for (auto& d : b->hc) s += (size_t)state_doubles(d) * sizeof(double);
    return s;
}

// The state crosses PCIe as one copy per direction: a kernel packs (or unpacks) every
// case's state planes into a device staging buffer laid out as the host buffer.
static int state_copy(cfd_batch* b, void* host, size_t bytes, bool to_host) {
    if (!b || !host) return fail(CFD_E_ARG, "bad arguments");
    const size_t need = cfd_batch_state_bytes(b);
    if (bytes < need) return fail(CFD_E_ARG, "state buffer too small");
    // per-case offsets into the image (a slot pool's cases change with admissions)
    std::vector<long long> off(b->n);
    long long o = 0;
    for (int c = 0; c < b->n; c++) {
        off[c] = o;
        o += state_doubles(b->hc[c]);
    }
    if (need > b->stage_bytes) {
        CK(cudaStreamSynchronize(b->st));
        cudaFree(b->stage);
        b->stage = nullptr;
        b->stage_bytes = 0;
        CK(cudaMalloc((void**)&b->stage, need));
        b->stage_bytes = need;
    }
    if (!b->stage_off) CK(cudaMalloc((void**)&b->stage_off, sizeof(long long) * b->n));
    CK(cudaMemcpyAsync(b->stage_off, off.data(), sizeof(long long) * b->n, cudaMemcpyHostToDevice, b->st));
    b->bd.cur = b->cur;
    if (to_host) {
        k_state_pack<<<b->n * 7, 256, 0, b->st>>>(b->bd, b->stage, b->stage_off, 1);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(host, b->stage, need, cudaMemcpyDeviceToHost, b->st));
    } else {
        CK(cudaMemcpyAsync(b->stage, host, need, cudaMemcpyHostToDevice, b->st));
        k_state_pack<<<b->n * 7, 256, 0, b->st>>>(b->bd, b->stage, b->stage_off, 0);
        CK(cudaGetLastError());
    }
    CK(cudaStreamSynchronize(b->st));
    return CFD_OK;
}

// Checkpoint file (replaces the reference's spa100.dat restart writer, PSolver.cpp:2006-2016):
//   "CFDB200C" | u32 version 3 | u32 cases | per case i32 n0, n1, profile, precision and a
//   u64 grid fingerprint | the state image of cfd_batch_get_state | u64 FNV-1a hash of all
//   preceding bytes
namespace {
const char kCkptMagic[8] = {'C', 'F', 'D', 'B', '2', '0', '0', 'C'};
// 1: padded device planes in the state image; 2: stored columns only; 3: a grid fingerprint per case
const uint32_t kCkptVersion = 3;
constexpr size_t kCkptCaseHdr = 24;  // i32 n0, n1, profile, precision; u64 grid fingerprint
uint64_t fnv1a(const unsigned char* p, size_t n, uint64_t h = 1469598103934665603ull) {
    for (size_t k = 0; k < n; k++) {
        h ^= p[k];
        h *= 1099511628211ull;
    }
    return h;
}

// the splitmix64 output function (Steele, Lea and Flood 2014): a bijective 64-bit mixer
__device__ __forceinline__ unsigned long long mix64(unsigned long long x) {
    x ^= x >> 30;
    x *= 0xbf58476d1ce4e5b9ull;
    x ^= x >> 27;
    x *= 0x94d049bb133111ebull;
    x ^= x >> 31;
    return x;
}

// A fingerprint of every case's grid (the ten grid planes over the stored columns, one CTA
// per case): the wrapping sum of a mixed word per value and position, so the result is the
// same whatever order the threads add in.
__global__ void k_grid_hash(BatchDev b, unsigned long long* out) {
    const CaseDev& c = b.cases[blockIdx.x];
    const int ncols = c.periodic ? c.W : c.n0;
    const long long per = (long long)c.n1 * ncols;
    unsigned long long h = 0;
    for (long long e = threadIdx.x; e < 10 * per; e += blockDim.x) {
        const int q = (int)(e / per);
        const long long r = e - q * per;
        const int j = (int)(r / ncols), i = (int)(r % ncols);
        const double v = plane(b, c, q)[(long long)j * c.ld + i];
        h += mix64((unsigned long long)__double_as_longlong(v) ^ mix64((unsigned long long)e));
    }
    atomicAdd(out + blockIdx.x, h);
}

int grid_fingerprints(cfd_batch* b, std::vector<uint64_t>& out) {
    unsigned long long* d = nullptr;
    CK(cudaMalloc((void**)&d, sizeof(unsigned long long) * b->n));
    out.assign(b->n, 0);
    cudaError_t e = cudaMemsetAsync(d, 0, sizeof(unsigned long long) * b->n, b->st);
    if (e == cudaSuccess) {
        k_grid_hash<<<b->n, 256, 0, b->st>>>(b->bd, d);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(out.data(), d, sizeof(uint64_t) * b->n, cudaMemcpyDeviceToHost, b->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->st);
    cudaFree(d);
    if (e != cudaSuccess) return fail(CFD_E_CUDA, std::string("grid fingerprint: ") + cudaGetErrorString(e));
    return CFD_OK;
}
}  // namespace

int cfd_batch_save(cfd_batch* b, const char* path) {
    if (!b || !path) return fail(CFD_E_ARG, "bad arguments");
    const size_t sb = cfd_batch_state_bytes(b);
    std::vector<uint64_t> fp;
    if (int rc = grid_fingerprints(b, fp)) return rc;
    std::vector<unsigned char> buf(8 + 8 + kCkptCaseHdr * b->n + sb + 8);
    unsigned char* p = buf.data();
    memcpy(p, kCkptMagic, 8);
    const uint32_t hdr[2] = {kCkptVersion, (uint32_t)b->n};
    memcpy(p + 8, hdr, 8);
    for (int c = 0; c < b->n; c++) {
        const int32_t g[4] = {b->hc[c].n0, b->hc[c].n1, b->hc[c].profile, b->prm[c].precision};
        memcpy(p + 16 + kCkptCaseHdr * c, g, 16);
        memcpy(p + 16 + kCkptCaseHdr * c + 16, &fp[c], 8);
    }
    unsigned char* st = p + 16 + kCkptCaseHdr * b->n;
    if (int rc = cfd_batch_get_state(b, st, sb)) return rc;
    const uint64_t h = fnv1a(p, buf.size() - 8);
    memcpy(p + buf.size() - 8, &h, 8);
    FILE* f = fopen(path, "wb");
    if (!f) return fail(CFD_E_ARG, std::string("cannot write ") + path);
    const bool ok = fwrite(p, 1, buf.size(), f) == buf.size();
    if (fclose(f) != 0 || !ok) return fail(CFD_E_ARG, std::string("write failed: ") + path);
    return CFD_OK;
}

int cfd_batch_load(cfd_batch* b, const char* path) {
    if (!b || !path) return fail(CFD_E_ARG, "bad arguments");
    FILE* f = fopen(path, "rb");
    if (!f) return fail(CFD_E_ARG, std::string("cannot open ") + path);
    std::vector<unsigned char> buf;
    unsigned char tmp[1 << 16];
    size_t n;
    while ((n = fread(tmp, 1, sizeof(tmp), f)) > 0) buf.insert(buf.end(), tmp, tmp + n);
    fclose(f);
    const size_t sb = cfd_batch_state_bytes(b);
    const size_t need = 8 + 8 + kCkptCaseHdr * b->n + sb + 8;
    if (buf.size() < 16 || memcmp(buf.data(), kCkptMagic, 8) != 0) return fail(CFD_E_ARG, "not a checkpoint file");
    uint32_t hdr[2];
    memcpy(hdr, buf.data() + 8, 8);
    if (hdr[0] != kCkptVersion) return fail(CFD_E_ARG, "unsupported checkpoint version");
    if ((int)hdr[1] != b->n || buf.size() != need)
        return fail(CFD_E_ARG, "checkpoint does not match the batch (number of cases or sizes)");
    uint64_t h;
    memcpy(&h, buf.data() + need - 8, 8);
    if (h != fnv1a(buf.data(), need - 8)) return fail(CFD_E_ARG, "checkpoint is corrupt (hash mismatch)");
    std::vector<uint64_t> fp;
    if (int rc = grid_fingerprints(b, fp)) return rc;
    for (int c = 0; c < b->n; c++) {
        int32_t g[4];
        uint64_t gh;
        memcpy(g, buf.data() + 16 + kCkptCaseHdr * c, 16);
        memcpy(&gh, buf.data() + 16 + kCkptCaseHdr * c + 16, 8);
        if (g[0] != b->hc[c].n0 || g[1] != b->hc[c].n1 || g[2] != b->hc[c].profile || g[3] != b->prm[c].precision)
            return fail(CFD_E_ARG, "checkpoint case " + std::to_string(c) + " has another geometry or precision");
        if (gh != fp[c])
            return fail(CFD_E_ARG, "checkpoint case " + std::to_string(c) + " was saved on another grid");
    }
    return cfd_batch_set_state(b, buf.data() + 16 + kCkptCaseHdr * b->n, sb);
}

int cfd_batch_get_state(cfd_batch* b, void* host, size_t bytes) { return state_copy(b, host, bytes, true); }
int cfd_batch_set_state(cfd_batch* b, const void* host, size_t bytes) {
    return state_copy(b, const_cast<void*>(host), bytes, false);
}

// ---- the sip9p() seam (replaces PSolver.cpp:2067-2278, called at :1466)
// A one-case batch of the caller's size carries the solve: its pressure stencil and
// multigrid hierarchy come from the caller's nine planes (the grid the batch is created
// with only sizes it), and the step's own BiCGStab + V-cycle kernels run host-driven on the
// correction of phi0, with the reference's relative L1 stop rule.
int cfd_sip_solve(int n0, int n1, int periodic, const double* const* coef9, double* phi, const double* q,
                  double tol, int maxit, int* iters, void* stream) {
    if (iters) *iters = 0;
    if (n0 < 8 || n1 < (periodic ? 6 : 7) || !coef9 || !phi || !q || maxit < 1 || !(tol >= 0.0))
        return fail(CFD_E_ARG, "cfd_sip_solve: bad arguments");
    for (int m = 0; m < 9; m++)
        if (!coef9[m]) return fail(CFD_E_ARG, "cfd_sip_solve: null coefficient plane");
    // the caller's arrays are complete once its stream has drained
    CK(cudaStreamSynchronize((cudaStream_t)stream));
    cfd_grid_spec spec{};
    spec.profile = periodic ? CFD_PROFILE_OGRID : CFD_PROFILE_CAVITY;
    spec.n0 = n0;
    spec.n1 = n1;
    spec.ar = 2.0;
    spec.r_outer = 20.0;
    const size_t np = (size_t)n0 * n1;
    std::vector<double> planes(10 * np), normals(4 * (size_t)n0);
    int rc = cfd_grid_generate(&spec, planes.data(), normals.data());
    if (rc) return rc;
    cfd_grid g{};
    g.n0 = n0;
    g.n1 = n1;
    g.dxi0 = 1.0 / (n0 - 1);
    g.dxi1 = 1.0 / (n1 - 1);
    g.ar = spec.ar;
    const double** gp[10] = {&g.x, &g.y, &g.xix, &g.xiy, &g.etx, &g.ety, &g.alph, &g.beta, &g.gam, &g.jac};
    for (int m = 0; m < 10; m++) *gp[m] = planes.data() + m * np;
    g.xnix = normals.data();
    g.xniy = normals.data() + n0;
    g.xnox = normals.data() + 2 * n0;
    g.xnoy = normals.data() + 3 * n0;
    cfd_params p;
    cfd_params_default(&p);
    p.profile = spec.profile;
    p.tol_p = tol;
    p.atol_p = 0.0;
    p.maxit_p = maxit;
    cfd_batch* b = nullptr;
    rc = cfd_batch_create(1, &g, &p, &b);
    if (rc) return rc;
    auto finish = [&](int code) {
        cudaStreamSynchronize(b->st);
        cfd_batch_destroy(b);
        return code;
    };
    BatchDev& bd = b->bd;
    const CaseDev& d = b->hc[0];
    // sip9p's argument order (ap, ae, as, an, aw, ase, asw, ane, anw) -> P_AP .. P_ASW
    SipIn in;
    const int order[9] = {0, 1, 4, 3, 2, 7, 8, 5, 6};
    for (int m = 0; m < 9; m++) in.a[m] = coef9[order[m]];
    in.phi = phi;
    in.q = q;
    in.n0 = n0;
    const long long npad = (long long)n1 * (d.W + 2 * H);
    k_sip_pack<<<(unsigned)((npad + 255) / 256), 256, 0, b->st>>>(bd, in);
    for (int l = 0; l + 1 < b->nlev_max; l++)
        if (bd.natiles[l + 1] > 0) k_mg_galerkin<<<bd.natiles[l + 1], NT, 0, b->st>>>(bd, l, 0);
    if (cudaMemsetAsync(b->flags, 0, 4 * sizeof(int), b->st) != cudaSuccess)
        return finish(fail(CFD_E_CUDA, "cfd_sip_solve: flag reset failed"));
    k_sip_init<<<bd.njtiles, NT, 0, b->st>>>(bd);
    for (int it = 0; it < maxit; it++) {
        if (it > 0) {
            int a = 0;
            rc = read_flag(b, 0, &a);
            if (rc) return finish(rc);
            if (a <= 0) break;
        }
        enq_p_iter(b, bd);
    }
    k_sip_out<<<(unsigned)(((long long)np + 255) / 256), 256, 0, b->st>>>(bd, phi, n0);
    if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(b->st) != cudaSuccess)
        return finish(fail(CFD_E_CUDA, "cfd_sip_solve: kernel failure"));
    int is[NISCAL];
    if (cudaMemcpy(is, b->iscal, sizeof(is), cudaMemcpyDeviceToHost) != cudaSuccess)
        return finish(fail(CFD_E_CUDA, "cfd_sip_solve: status read failed"));
    if (iters) *iters = is[I_PIT];
    const int st = is[I_STATUS] | is[I_PSTATUS];
    if (st & ST_NAN) return finish(fail(CFD_E_DIVERGED, "cfd_sip_solve: residual not finite"));
    if (st & ST_BREAKDOWN) return finish(fail(CFD_E_BREAKDOWN, "cfd_sip_solve: Krylov breakdown"));
    if (st & ST_MAXITER) return finish(fail(CFD_E_MAXITER, "cfd_sip_solve: maxit reached"));
    return finish(CFD_OK);
}

// ---- single case
int cfd_case_create(const cfd_grid* g, const cfd_params* prm, cfd_case** out) {
    return cfd_batch_create(1, g, prm, out);
}

int cfd_case_step(cfd_case* c, int nsteps, cfd_step_stats* last) {
    int rc = cfd_batch_step(c, nsteps);
    if (rc) return rc;
    if (last) {
        rc = cfd_batch_stats(c, 0, last);
        if (rc) return rc;
        last->steps = nsteps;
        if (last->status & ST_NAN) return fail(CFD_E_DIVERGED, "NaN in the solution");
        if (last->status & ST_BREAKDOWN) return fail(CFD_E_BREAKDOWN, "pressure solve: Krylov breakdown");
        if (last->status & ST_MAXITER) return fail(CFD_E_MAXITER, "an inner solve stopped at its iteration cap");
    }
    return CFD_OK;
}

int cfd_case_solve_to(cfd_case* c, double tol, int max_steps, cfd_step_stats* last) {
    if (!c || max_steps < 0) return fail(CFD_E_ARG, "bad arguments");
    cfd_step_stats s{};
    int done = 0;
    const int chunk = 10;
    while (done < max_steps) {
        const int n = std::min(chunk, max_steps - done);
        int rc = cfd_batch_step(c, n);
        if (rc) return rc;
        done += n;
        rc = cfd_batch_stats(c, 0, &s);
        if (rc) return rc;
        if (s.status & ST_NAN) {
            s.steps = done;
            if (last) *last = s;
            return fail(CFD_E_DIVERGED, "NaN in the solution");
        }
        if (s.steady_res_rel <= tol) break;
    }
    s.steps = done;
    if (last) *last = s;
    if (s.steady_res_rel > tol) return fail(CFD_E_NOTCONV, "max_steps reached before the steady residual reached tol");
    return CFD_OK;
}

int cfd_case_get_fields(cfd_case* c, double* u, double* v, double* T, double* p, double* si, double* vort) {
    if (!c) return fail(CFD_E_ARG, "null case");
    struct { const char* n; double* o; } f[] = {{"u", u}, {"v", v}, {"T", T}, {"p", p}, {"si", si}, {"vort", vort}};
    for (auto& e : f) {
        if (!e.o) continue;
        int rc = cfd_batch_get_plane(c, 0, e.n, e.o);
        if (rc) return rc;
    }
    return CFD_OK;
}

int cfd_case_destroy(cfd_case* c) { return cfd_batch_destroy(c); }

}  // extern "C"
