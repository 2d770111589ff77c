/*
 * cfd_b200.h -- C ABI of the B200 (sm_100a) projection-step solver.
 *
 * Drop-in boundary for the hot path of mhsuhail00/CFD_Solver. The reference is
 * one C++ class (`class Solver`, PSolver.cpp:11-2447) with no plugin or FFI
 * interface; its per-step body `Solver::timeLoop()` (PSolver.cpp:1051-2065)
 * and the two solver members it calls,
 *     void gauss(double** ap, ..., double** phi, double** q)   PSolver.cpp:2280-2286
 *     void sip9p(double** ap, ..., double** phi, double** q)   PSolver.cpp:2067-2069
 * are what this library replaces. The grid comes from the reference's INP.DAT
 * (PSolver.cpp:517-547); the physics constants that the reference hard-codes
 * as members (PSolver.cpp:160-183) and the solver tolerances it keeps as
 * locals (PSolver.cpp:2086-2088, 2290-2291) are per-case parameters here.
 *
 * Conventions
 *  - Every call returns CFD_OK (0) or a negative CFD_E_* code; cfd_last_error()
 *    gives the message of the last failure on the calling thread.
 *  - Host arrays are float64, n1*n0 in [j][i] order (i fastest) -- the order of
 *    INP.DAT -- with the O-grid's seam column i = n0-1 included.
 *  - The library owns all device memory; the caller owns every host buffer.
 *  - A handle is driven by one host thread at a time; each batch has its own
 *    CUDA stream. There is no CPU fallback: without a usable CUDA device every
 *    entry point that needs one fails with CFD_E_CUDA.
 */
#ifndef CFD_B200_H
#define CFD_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CFD_OK 0
#define CFD_E_ARG (-1)      /* bad argument / grid */
#define CFD_E_CUDA (-2)     /* CUDA error or no device */
#define CFD_E_OOM (-3)      /* device memory exhausted / over budget */
#define CFD_E_DIVERGED (-4) /* NaN in a case */
#define CFD_E_MAXITER (-5)  /* an inner solve hit its iteration cap */
#define CFD_E_BREAKDOWN (-6)/* Krylov breakdown */
#define CFD_E_NOTCONV (-7)  /* solve_to: max_steps reached */

#define CFD_PROFILE_OGRID 0  /* the reference's O-grid (periodic xi, body + far field) */
#define CFD_PROFILE_CAVITY 1 /* lid-driven unit square on a curvilinear grid */

#define CFD_PRECISION_FP64 0  /* every sweep and Krylov vector in FP64 (the plain path) */
#define CFD_PRECISION_MIXED 1 /* FP32 inner sweeps / Krylov work inside FP64 defect correction */

/* One INP.DAT grid (PSolver.cpp:517-547); planes are n1*n0 host float64, [j][i]. */
typedef struct cfd_grid {
    int n0, n1;
    double dxi0, dxi1;
    double p_grid, a_grid, ar;
    const double *x, *y;
    const double *xix, *xiy, *etx, *ety; /* xi_x, xi_y, eta_x, eta_y */
    const double *alph, *beta, *gam;     /* alpha, beta, gamma */
    const double *jac;                   /* J = x_xi y_eta - x_eta y_xi */
    const double *xnix, *xniy, *xnox, *xnoy; /* n0 each */
} cfd_grid;

/* Analytic grid of a case, generated on the GPU by cfd_grid_generate (the reference reads
 * its grid from INP.DAT, written by an external generator). */
typedef struct cfd_grid_spec {
    int profile;           /* CFD_PROFILE_OGRID: elliptic-cylinder O-grid; CFD_PROFILE_CAVITY */
    int n0, n1;            /* grid points (O-grid: n0 >= 8, n1 >= 6; cavity: both >= 7) */
    double ar;             /* O-grid semi-axis ratio (>= 1; 1 = circle): semi-axes 1 and 1/ar */
    double r_outer;        /* O-grid far-field radius */
    double skew;           /* skew amplitude s: O-grid mu = mu0 + L[eta + s eta(1-eta) sin 2 pi xi];
                              cavity x = xi + s xi(1-xi) sin 2 pi eta, y = eta + s eta(1-eta) sin 2 pi xi */
} cfd_grid_spec;

/* Per-case parameters. cfd_params_default() gives the reference's values. */
typedef struct cfd_params {
    double Re, Ri, Pr, F, alpha_deg, dt;  /* PSolver.cpp:160-174 */
    double tol_mom, atol_mom;  /* u/v/T solves: relative / absolute L1 residual (ref 0.75e-2, 0) */
    double tol_p, atol_p;      /* pressure correction: relative / absolute L1 residual */
    int maxit_mom, maxit_p;    /* iteration caps per solve */
    int profile;               /* CFD_PROFILE_* */
    int fix_T_annw;            /* 1: T solve uses atnnw (Fortran intent); 0: reference C++ */
    int fix_circ_de;           /* 1: circulation spacing 1/(n0-1) (Fortran); 0: 1/(n0-2) */
    int warm_start;            /* 1: up/vp solves start from the previous step; 0: from zero */
    double omega_p;            /* p += omega_p * pcor (reference: 1) */
    double lid_u;              /* cavity lid velocity */
    int precision;             /* CFD_PRECISION_FP64 (plain) or CFD_PRECISION_MIXED; one per batch */
    int time_accurate;         /* 0: time is the reference's int (PSolver.cpp:186; the oscillating
                                  wall of PSolver.cpp:1617-1630 then sees t = 0 while dt < 1);
                                  1: time is a double, t = n dt, for unsteady oscillating-cylinder
                                  runs (F != 0) */
} cfd_params;

/* Statistics of the last completed step of a case. */
typedef struct cfd_step_stats {
    int steps;        /* steps taken by the call */
    int status;       /* bit set of the CFD solver status flags (0 = clean) */
    int it_mom[5];    /* sweeps of the u*, v*, T, up, vp solves */
    int it_p;         /* pressure-correction iterations */
    double dmax;      /* max dilatation, the reference's per-step print (PSolver.cpp:1890) */
    double cl, cd, cm, nu, circ;
    double cl_pr, cd_pr, cl_vor, cd_vor;
    double q_l1, q_l2, q_max; /* continuity source q (mass residual) norms */
    double dT_l1, dT_max;     /* energy residual: |T^{n+1} - T^n| */
    double p_res_rel;         /* final relative L1 residual of the pressure solve */
    double mass_res_rel;      /* q_l2 / q_l2 of the case's first step */
    double steady_res;        /* mean (|du| + |dv| + |dT|) / dt over the unknown cells */
    double steady_res_rel;    /* steady_res / steady_res of the case's first step */
    double time;              /* the case's time after the step (an integer unless time_accurate) */
} cfd_step_stats;

typedef struct cfd_batch cfd_batch;
typedef cfd_batch cfd_case; /* a single case is a batch of one */

void cfd_params_default(cfd_params* p);
const char* cfd_last_error(void);
int cfd_device_count(int* count);
/* make `device` current for this thread's later calls (one process per GPU) */
int cfd_set_device(int device);

/* status bits of cfd_step_stats.status (the reference reports none: its solves loop to
 * maxiter = 100000 silently, PSolver.cpp:2087, 2291, and it never checks for NaN) */
#define CFD_STATUS_MAXITER 1   /* this step: a u/v/T/up/vp or pressure solve stopped at its cap */
#define CFD_STATUS_BREAKDOWN 2 /* this step: the pressure BiCGStab broke down (rho or omega = 0) */
#define CFD_STATUS_NAN 4       /* sticky: a non-finite residual; the case's fields are invalid */

/* ---- single case (replaces Solver::Solver() + Solver::timeLoop()) ---- */
int cfd_case_create(const cfd_grid* g, const cfd_params* prm, cfd_case** out);
/* advance nsteps time steps (the body of timeLoop, PSolver.cpp:1058-1983). With `last`,
 * the last step's status is also returned: CFD_E_DIVERGED (NaN), CFD_E_BREAKDOWN or
 * CFD_E_MAXITER; the steps have been taken either way. */
int cfd_case_step(cfd_case* c, int nsteps, cfd_step_stats* last);
/* step until steady_res_rel <= tol (or max_steps: CFD_E_NOTCONV). The continuity source q
 * of this projection scheme keeps a compatibility defect in a closed cavity (the pressure
 * level drifts uniformly), so convergence is judged on the steady residual. */
int cfd_case_solve_to(cfd_case* c, double tol, int max_steps, cfd_step_stats* last);
/* host copies of the fields, n1*n0 each, [j][i]; any pointer may be NULL */
int cfd_case_get_fields(cfd_case* c, double* u, double* v, double* T, double* p, double* si,
                        double* vort);
int cfd_case_destroy(cfd_case* c);

/* ---- batch: many cases of uneven size and parameters in one set of launches ---- */
int cfd_batch_create(int ncases, const cfd_grid* grids, const cfd_params* params,
                     cfd_batch** out);
int cfd_batch_step(cfd_batch* b, int nsteps);
int cfd_batch_stats(cfd_batch* b, int case_index, cfd_step_stats* out);
/* named plane of one case ("u", "v", "T", "p", "up", "vp", "us", "vs", "pcor", "q",
 * "qu", "qv", "qt", "qup", "qvp", "si", "vort", "dil", "ap", "ae", ...) as n1*n0 [j][i] */
int cfd_batch_get_plane(cfd_batch* b, int case_index, const char* name, double* out);
int cfd_batch_destroy(cfd_batch* b);
/* device bytes a case of this size needs (admission by HBM budget) */
size_t cfd_case_bytes(int n0, int n1, int profile);
/* the stats of every case (cap entries at most), one device -> host copy */
int cfd_batch_fetch_stats(cfd_batch* b, cfd_step_stats* out, int cap);

/* ---- multigrid schedule of the pressure preconditioner (no counterpart in the reference,
 * whose SIP solver has none): pre- and post-sweeps per level (1..8), sweeps on the
 * coarsest level (1..256) and `fused` (1: a smoothing phase's sweeps run in one launch,
 * tile halos held; 0: one launch per sweep; 2: as 1, with each level's pre-smoothing done
 * inside its residual + restriction launch on overlapping regions); defaults 1, 3, 12, 2.
 * cfd_batch_autotune() times a fixed list of candidate schedules over `steps` steps each from the batch's
 * current state (restored before each candidate and on return, so the batch continues
 * exactly where it was), keeps the fastest and reports it as {pre, post, coarse, fused}
 * with its time per step. */
int cfd_batch_set_mg(cfd_batch* b, int nu_pre, int nu_post, int coarse_sweeps, int fused);
/* Polls a kernel's wait for its bulk copies makes before it gives up (no counterpart in the
 * reference; default 2^24, about 0.1-1 s; negative restores the default; 0 gives up at
 * once, which only tests the error path). A wait that gives up sets the batch's error
 * flag and the kernel returns (after its copies have landed); the step then fails with
 * CFD_E_CUDA ("a bounded wait inside a kernel timed out") and the batch's fields are
 * invalid: destroy it. The device stays usable. */
int cfd_batch_set_wait_limit(cfd_batch* b, long long polls);
int cfd_batch_get_mg(cfd_batch* b, int* nu_pre, int* nu_post, int* coarse_sweeps, int* fused);
int cfd_batch_autotune(cfd_batch* b, int steps, int* out_schedule4, double* out_ms_per_step);

/* ---- slots: continuous batching over a batch of fixed-geometry slots ----
 * Every case of a batch is a slot. cfd_batch_admit() writes a new case into slot `slot`
 * (same n0, n1 and profile as the slot): grid, initial state, parameters and its pressure
 * stencil / multigrid set-up, while the other slots keep their resident state; the case
 * then takes part in every cfd_batch_step(). cfd_batch_set_active(b, slot, 0) empties a
 * slot (its kernels skip it), 1 re-activates it. */
int cfd_batch_admit(cfd_batch* b, int slot, const cfd_grid* g, const cfd_params* p);
/* cfd_batch_admit() of the grid cfd_grid_generate() makes for `spec`, generated straight
 * into the slot's device planes together with the case's initial state: nothing of the
 * case crosses PCIe (five words of the metric scan come back). The slot's Chebyshev bounds
 * and metric check are computed on the device with the same per-point arithmetic as the
 * host path, so the case steps bit for bit like cfd_batch_admit() of that grid. spec->n0, n1, profile must
 * match the slot; CFD_E_ARG (the slot untouched) for a mismatch or an invalid spec. */
int cfd_batch_admit_spec(cfd_batch* b, int slot, const cfd_grid_spec* spec, const cfd_params* p);
int cfd_batch_set_active(cfd_batch* b, int slot, int active);

/* ---- slot pool: admission by free device memory (no counterpart in the reference, which
 * runs one case per process) ----
 * A pool is a batch whose cases are placed in one device arena of hbm_budget bytes as they
 * are admitted, whatever their size, and give their memory back when released; every
 * cfd_batch_* call works on it. Its case indices are slots 0 .. max_cases-1; an empty slot
 * takes part in no launch. cfd_pool_admit() places a new case in the first free region
 * that fits it and writes its slot; CFD_E_OOM (nothing changed) when no free region of the
 * budget fits or every slot is taken -- retry after a release. The other cases keep their
 * resident state and step on bit for bit as they would alone (each case's tiles keep their
 * order in the launches). cfd_pool_release() frees a slot and its memory at once.
 * cfd_pool_case_bytes() is the arena bytes a case takes; cfd_pool_free() reports the free
 * bytes and the largest free region. */
int cfd_pool_create(size_t hbm_budget, int max_cases, int precision, cfd_batch** out);
int cfd_pool_admit(cfd_batch* b, const cfd_grid* g, const cfd_params* p, int* slot);
int cfd_pool_release(cfd_batch* b, int slot);
int cfd_pool_free(cfd_batch* b, size_t* free_bytes, size_t* largest);
size_t cfd_pool_case_bytes(int n0, int n1, int profile);

/* ---- serving session: requests with arrival times over slot classes ---- */
typedef struct cfd_request {
    double arrival_s;     /* seconds after the session starts */
    const cfd_grid* grid; /* must match a slot class (n0, n1, params.profile) */
    cfd_params params;
    double tol;           /* converged when steady_res_rel <= tol */
    int max_steps;        /* step cap (result CFD_E_NOTCONV) */
} cfd_request;

typedef struct cfd_result {
    int status; /* CFD_OK (converged), CFD_E_NOTCONV, CFD_E_DIVERGED */
    int slot, steps;
    double arrival_s, admit_s, done_s, latency_s;
    double nu, steady_res_rel, mass_res_rel;
} cfd_result;

typedef struct cfd_serve_config {
    int nclasses;                /* fixed slots only: the slot classes */
    const cfd_grid* class_grids; /* one template grid per slot class (sets n0, n1) */
    const int* class_profile;    /* CFD_PROFILE_* of each class */
    const int* class_slots;      /* slots per class; NULL: admission by free device memory --
                                    a slot pool (cfd_pool_create) of hbm_budget bytes takes
                                    requests of any size, the classes are not used */
    size_t hbm_budget;           /* device bytes of the pool when class_slots is NULL */
    int steps_per_tick;          /* steps between convergence checks / admissions */
    int precision;               /* CFD_PRECISION_* of every slot (requests must match) */
} cfd_serve_config;

typedef struct cfd_serve_stats {
    double makespan_s, cases_per_s, p50_latency_s, p99_latency_s, mean_latency_s;
    long long steps, cell_updates;
    int converged, failed, slots;
} cfd_serve_stats;

/* Runs a serving session in real time: requests are admitted as they arrive -- by free
 * device memory (class_slots NULL: oldest first into the first free region of the budget
 * that fits; a smaller request may pass a larger one that does not fit yet, until the
 * oldest has waited 20 ticks) or into free slots of their class -- all admitted cases
 * advance together, converged cases are retired and their memory or slots reused.
 * results[i] belongs to reqs[i]. */
int cfd_serve(const cfd_serve_config* cfg, const cfd_request* reqs, int nreq, cfd_result* results,
              cfd_serve_stats* stats);

/* ---- timing: per-kernel CUDA-event durations accumulated on the batch's stream ---- */
int cfd_batch_profile(cfd_batch* b, int enable);
/* fills up to cap entries; returns the number of kernel names known */
int cfd_batch_kernel_times(cfd_batch* b, const char** names, double* total_ms, long long* launches,
                           int cap);
int cfd_batch_sync(cfd_batch* b);
/* the batch's CUDA stream (cudaStream_t), for callers that time or order work on it */
void* cfd_batch_stream(cfd_batch* b);
/* kernels launched by the batch since creation */
long long cfd_batch_launches(cfd_batch* b);
/* algorithmic-traffic counters of the u/v/T sweeps: [0] field-cells swept, [1] cells swept,
 * [2] field-cells of first sweeps, [3] field-cells of second sweeps (the sweeps that read
 * one array less in the FP64 path and in the precision form respectively) */
int cfd_batch_work(cfd_batch* b, unsigned long long* out4);

/* ---- the gauss() seam on device arrays (replaces PSolver.cpp:2280-2446) ----
 * Solves one momentum / energy system given its 25 stored coefficient planes in
 * gauss()'s argument order (ap, ae, as, an, aw, ase, asw, ane, anw, ass, assee, assww,
 * asse, assw, asee, asww, ann, annee, annww, anne, annw, anee, anww, aee, aww), each a
 * device array of n1*n0 float64 in [j][i] order. phi (device, in/out) carries the
 * initial guess and the boundary values; q is the right-hand side. periodic = 1: xi is
 * periodic with the seam column n0-1 duplicating column 0 (the reference's O-grid);
 * 0: columns 0 and n0-1 are fixed. Chebyshev-accelerated Jacobi sweeps until the
 * relative L1 residual before a sweep is below tol (gauss()'s rule, PSolver.cpp:2438).
 * Sweeps run in pairs, the stop tested after each pair on the host (the call waits for
 * its work), so at most maxit rounded down to even sweeps are taken.
 * Scratch (a second iterate and reduction partials) is allocated and freed per call.
 * Returns CFD_OK, CFD_E_MAXITER or CFD_E_DIVERGED; *sweeps receives the sweep count. */
int cfd_gauss_solve(int n0, int n1, int periodic, const double* const* coef, double* phi,
                    const double* q, double tol, int maxit, int* sweeps, void* stream);

/* ---- the sip9p() seam on device arrays (replaces PSolver.cpp:2067-2278, called at :1466)
 * Solves the pressure-correction system given its 9 stored coefficient planes in sip9p()'s
 * argument order (ap, ae, as, an, aw, ase, asw, ane, anw), each a device array of n1*n0
 * float64 in [j][i] order; phi (device, in/out) carries the initial guess and the boundary
 * values, which stay fixed as sip9p holds them (rows j = 0 and n1-1, and with periodic = 0
 * columns 0 and n0-1); q is the right-hand side. periodic = 1: xi is periodic with the seam
 * column n0-1 duplicating column 0. BiCGStab preconditioned by a Galerkin multigrid V-cycle
 * built from the given planes (replacing the SIP iteration, which has no parallel form)
 * until the L1 residual is below tol times the initial one (sip9p's rule,
 * PSolver.cpp:2259). The call allocates a one-case batch for the solve (device memory of
 * about cfd_case_bytes(n0, n1, profile)), waits for `stream` before it starts, and returns
 * once phi is written. Returns CFD_OK, CFD_E_MAXITER, CFD_E_BREAKDOWN or CFD_E_DIVERGED;
 * *iters receives the BiCGStab iterations. */
int cfd_sip_solve(int n0, int n1, int periodic, const double* const* coef9, double* phi,
                  const double* q, double tol, int maxit, int* iters, void* stream);

/* Same solve as cfd_gauss_solve() for callers that cannot allocate device memory: hosts
 * whose device memory belongs to another allocator or budget, loops that must not take
 * the allocator's locks or meet an out-of-memory failure mid-step. No counterpart in the
 * reference (its gauss() allocates two full arrays per call, PSolver.cpp:2288-2289).
 * The scratch lives in one static device array sized for n0*n1 <= CFD_NOALLOC_MAX_POINTS
 * (about 8.4 MB, held by every GPU that loads the library until the process exits);
 * larger grids are rejected with CFD_E_ARG. The first call on a device looks up the
 * array's device address (make that first call before any stream capture). All calls
 * on a device share the array: calls that overlap on the GPU race, so serialise them
 * (one stream, or one call at a time). The call allocates nothing; it clears the part
 * of the scratch that must start at zero itself. */
#define CFD_NOALLOC_MAX_POINTS (1 << 20)
int cfd_gauss_solve_noalloc(int n0, int n1, int periodic, const double* const* coef, double* phi,
                            const double* q, double tol, int maxit, int* sweeps, void* stream);

/* ---- grid generation on the GPU
 * Generates the grid of `spec` on the current device (coordinates and metrics from the
 * analytic map and its derivatives; the O-grid's seam column n0 - 1 repeats column 0) and
 * copies it to host memory: `planes` gets 10 * n1 * n0 doubles, the planes x, y, xi_x, xi_y,
 * eta_x, eta_y, alpha, beta, gamma, J in that order, each [j][i]; `normals` gets 4 * n0
 * doubles: the inner and outer boundary normals xnix, xniy, xnox, xnoy (the INP.DAT blocks,
 * PSolver.cpp:517-547). CFD_E_ARG for an invalid spec. */
int cfd_grid_generate(const cfd_grid_spec* spec, double* planes, double* normals);

/* ---- resident state snapshot (checkpoint / restart, host-owned stepping) ----
 * An image of every case's u, v, p, T, up, vp, int time, steps taken and the first-step
 * references of the relative residuals. Per case, in case order: the six fields as
 * row-major doubles, n1 rows of the stored columns (n0 for the cavity; n0 - 1 for the
 * periodic O-grid, whose column n0 - 1 repeats column 0), then 16 doubles (int time and
 * int steps in the first, the two references in the next two, the time as a double in the
 * fourth). cfd_batch_state_bytes()
 * gives its size. Use pinned host memory for speed. Restoring an image and stepping gives
 * the same bits as the steps taken from it. */
size_t cfd_batch_state_bytes(cfd_batch* b);
int cfd_batch_get_state(cfd_batch* b, void* host, size_t bytes);
int cfd_batch_set_state(cfd_batch* b, const void* host, size_t bytes);
/* Checkpoint files, in place of the reference's restart file spa100.dat (PSolver.cpp:2006-2016,
 * whose C++ writer dumps pointers): "CFDB200C", u32 version (3), u32 number of cases, per
 * case i32 n0, n1, profile, precision and a u64 fingerprint of its grid (x, y, the metrics
 * and J), the state image above, u64 FNV-1a hash of all preceding bytes (little-endian).
 * cfd_batch_load() checks magic, version, every case's geometry, precision and grid
 * fingerprint against the batch, and the hash, and fails with CFD_E_ARG (the batch
 * untouched) on any mismatch. */
int cfd_batch_save(cfd_batch* b, const char* path);
int cfd_batch_load(cfd_batch* b, const char* path);

#ifdef __cplusplus
}
#endif
#endif
