// cfd_seam.cu -- the fine-grained gauss() seam: one stored-coefficient system solve.
//
// The reference's gauss() (PSolver.cpp:2280-2446) takes the 25 coefficient planes
// of one momentum / energy system, the iterate phi (initial guess, boundary values)
// and the right-hand side q, and runs relative-L1-stopped lexicographic Gauss-Seidel.
// cfd_gauss_solve() takes the same planes as device arrays in the reference's
// argument order and solves with Chebyshev-accelerated Jacobi sweeps instead (the
// spectrum bounds of D^-1 A come from the coefficients: smooth modes at 1/max(ap),
// Gershgorin on top). Layout: n1*n0 float64, [j][i]; with `periodic` the seam
// column n0-1 duplicates column 0 as in the reference, unknowns i = 0..n0-2;
// otherwise columns 0 and n0-1 are fixed. 9-point rows: j = 1, n1-2 (and, when not
// periodic, i = 1, n0-2).
#include <cuda_runtime.h>

#include <cmath>

#include "../../include/cfd_b200.h"

namespace cfd_seam {

constexpr int BS = 256;

// scratch layout (doubles): [0..7] scalars, [8..8+nblk) partials, then the second iterate
enum { SC_MAXAP, SC_MAXOFF, SC_R0, SC_R, SC_W, SC_DONE, SC_CNT, SC_A };

struct Sys {
    int n0, n1, periodic;
    const double* c[25];  // gauss() argument order
    double* x0;           // caller's phi
    double* x1;           // scratch iterate
    const double* q;
    double* sc;           // scalars
    double* part;         // per-block partials
    unsigned int* cnt;
};

// gauss() argument order: ap, ae, as, an, aw, ase, asw, ane, anw, ass, assee, assww, asse,
// assw, asee, asww, ann, annee, annww, anne, annw, anee, anww, aee, aww
__constant__ int kDx[25] = {0, 1, 0, 0, -1, 1, -1, 1, -1, 0, 2, -2, 1, -1, 2, -2, 0, 2, -2, 1, -1, 2, -2, 2, -2};
__constant__ int kDy[25] = {0, 0, -1, 1, 0, -1, -1, 1, 1, -2, -2, -2, -2, -2, -1, -1, 2, 2, 2, 2, 2, 1, 1, 0, 0};

__device__ __forceinline__ bool cell_of(const Sys& s, int e, int& i, int& j) {
    const int ilo = s.periodic ? 0 : 1, ihi = s.n0 - 2;
    const int nx = ihi - ilo + 1, ny = s.n1 - 2;
    if (e >= nx * ny) return false;
    i = ilo + e % nx;
    j = 1 + e / nx;
    return true;
}

__device__ __forceinline__ int wrap(const Sys& s, int i) {
    if (!s.periodic) return i;
    const int P = s.n0 - 1;
    return i < 0 ? i + P : (i >= P ? i - P : i);
}

__device__ __forceinline__ bool near9(const Sys& s, int i, int j) {
    if (j == 1 || j == s.n1 - 2) return true;
    return !s.periodic && (i == 1 || i == s.n0 - 2);
}

__device__ double block_sum(double v, double* sm) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = v;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x < 32) {
        r = threadIdx.x < (blockDim.x >> 5) ? sm[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
    }
    __syncthreads();
    return r;
}

__device__ double block_max(double v, double* sm) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = v;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x < 32) {
        r = threadIdx.x < (blockDim.x >> 5) ? sm[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) r = fmax(r, __shfl_down_sync(0xffffffffu, r, o));
    }
    __syncthreads();
    return r;
}

// spectrum bounds: max ap and max sum|a_nb|/ap over the unknowns (all values >= 0)
__global__ void __launch_bounds__(BS) k_seam_bounds(Sys s) {
    __shared__ double sm[32];
    int i, j;
    double ap = 0.0, off = 0.0;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (cell_of(s, e, i, j)) {
        const long long k = (long long)j * s.n0 + i;
        ap = fabs(s.c[0][k]);
        const int nc = near9(s, i, j) ? 9 : 25;
        for (int m = 1; m < nc; m++) off += fabs(s.c[m][k]);
        off /= ap;
    }
    const double a = block_max(ap, sm), o = block_max(off, sm);
    if (threadIdx.x == 0) {
        atomicMax((unsigned long long*)&s.sc[SC_MAXAP], __double_as_longlong(a));
        atomicMax((unsigned long long*)&s.sc[SC_MAXOFF], __double_as_longlong(o));
    }
}

// one Chebyshev-Jacobi sweep src -> dst (x_{k+1} overwrites x_{k-1} in dst)
__global__ void __launch_bounds__(BS) k_seam_sweep(Sys s, int to_scratch, int sweep, double tol) {
    __shared__ double sm[32];
    __shared__ int last;
    if (s.sc[SC_DONE] != 0.0) return;
    const double* src = to_scratch ? s.x0 : s.x1;
    double* dst = to_scratch ? s.x1 : s.x0;
    const double a = 0.9 / s.sc[SC_MAXAP], b = 1.05 * (1.0 + s.sc[SC_MAXOFF]);
    const double g = 2.0 / (a + b);
    const double w = sweep == 0 ? 1.0 : s.sc[SC_W];
    int i, j;
    double r = 0.0;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (cell_of(s, e, i, j)) {
        const int n0 = s.n0;
        const long long k = (long long)j * n0 + i;
        const int nc = near9(s, i, j) ? 9 : 25;
        double sum = 0.0;
        for (int m = 1; m < nc; m++) {
            const int ii = wrap(s, i + kDx[m]), jj = j + kDy[m];
            sum += s.c[m][k] * src[(long long)jj * n0 + ii];
        }
        const double ap = s.c[0][k], rhs = s.q[k], xk = src[k];
        const double xj = (rhs - sum) / ap;
        double xn = xk + g * (xj - xk);
        if (sweep > 0) {
            const double xm = dst[k];
            xn = w * (xk + g * (xj - xk) - xm) + xm;
        }
        dst[k] = xn;
        if (s.periodic && i == 0) dst[(long long)j * n0 + n0 - 1] = xn;  // seam column
        r = fabs(rhs - ap * xk - sum);
    }
    r = block_sum(r, sm);
    if (threadIdx.x == 0) {
        s.part[blockIdx.x] = r;
        __threadfence();
        last = atomicAdd(s.cnt, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double t = 0.0;
    for (int m = threadIdx.x; m < (int)gridDim.x; m += blockDim.x) t += __ldcg(s.part + m);
    t = block_sum(t, sm);
    if (threadIdx.x == 0) {
        *s.cnt = 0u;
        if (sweep == 0) s.sc[SC_R0] = t != 0.0 ? t : 1.0;
        s.sc[SC_R] = t;
        const double s2 = ((b + a) / (b - a)) * ((b + a) / (b - a));
        s.sc[SC_W] = sweep == 0 ? 1.0 / (1.0 - 1.0 / (2.0 * s2)) : 1.0 / (1.0 - s.sc[SC_W] / (4.0 * s2));
        // pairs end in the caller's array; the stop is decided on the second sweep of a pair
        if (!to_scratch && (t / s.sc[SC_R0] < tol || !isfinite(t))) s.sc[SC_DONE] = isfinite(t) ? 1.0 : 2.0;
    }
}

}  // namespace cfd_seam

void cfd_internal_set_error(const char* msg);

// shared driver: `scratch` holds (8 + nblk) doubles, a second n1*n0 iterate, and a counter
int cfd_seam_solve(int n0, int n1, int periodic, const double* const* coef, double* phi, const double* q,
                   double tol, int maxit, int* sweeps, void* stream, double* scratch) {
    using namespace cfd_seam;
    cudaStream_t st = (cudaStream_t)stream;
    Sys s;
    s.n0 = n0; s.n1 = n1; s.periodic = periodic;
    for (int m = 0; m < 25; m++) s.c[m] = coef[m];
    const int nx = periodic ? n0 - 1 : n0 - 2, ny = n1 - 2;
    const int ncell = nx * ny;
    const int nblk = (ncell + BS - 1) / BS;
    s.sc = scratch;
    s.part = scratch + 8;
    s.x0 = phi;
    s.x1 = scratch + 8 + ((nblk + 31) / 32) * 32;
    s.cnt = (unsigned int*)(s.x1 + (size_t)n0 * n1);
    s.q = q;
    if (cudaMemsetAsync(scratch, 0, 8 * sizeof(double), st) != cudaSuccess ||
        cudaMemsetAsync(s.cnt, 0, sizeof(unsigned int), st) != cudaSuccess ||
        cudaMemcpyAsync(s.x1, phi, sizeof(double) * (size_t)n0 * n1, cudaMemcpyDeviceToDevice, st) != cudaSuccess) {
        cfd_internal_set_error("gauss seam: scratch initialisation failed");
        return CFD_E_CUDA;
    }
    k_seam_bounds<<<nblk, BS, 0, st>>>(s);
    int done = 0;
    double flag = 0.0;
    // sweeps run in pairs (the pair ends in the caller's array), so at most maxit rounded
    // down to even sweeps are taken
    for (int k = 0; k + 2 <= maxit && !done; k += 2) {
        k_seam_sweep<<<nblk, BS, 0, st>>>(s, 1, k, tol);
        k_seam_sweep<<<nblk, BS, 0, st>>>(s, 0, k + 1, tol);
        if (cudaMemcpyAsync(&flag, s.sc + SC_DONE, sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess) {
            cfd_internal_set_error("gauss seam: stream error");
            return CFD_E_CUDA;
        }
        if (sweeps) *sweeps = k + 2;
        done = flag != 0.0;
    }
    if (cudaGetLastError() != cudaSuccess) {
        cfd_internal_set_error("gauss seam: kernel launch failed");
        return CFD_E_CUDA;
    }
    if (flag == 2.0) {
        cfd_internal_set_error("gauss seam: residual not finite");
        return CFD_E_DIVERGED;
    }
    if (!done) cfd_internal_set_error("gauss seam: maxit reached");
    return done ? CFD_OK : CFD_E_MAXITER;
}

size_t cfd_seam_scratch_doubles(int n0, int n1, int periodic) {
    const int nx = periodic ? n0 - 1 : n0 - 2, ny = n1 - 2;
    const int nblk = (nx * ny + cfd_seam::BS - 1) / cfd_seam::BS;
    return 8 + ((size_t)(nblk + 31) / 32) * 32 + (size_t)n0 * n1 + 1;
}

extern "C" int cfd_gauss_solve(int n0, int n1, int periodic, const double* const* coef, double* phi,
                               const double* q, double tol, int maxit, int* sweeps, void* stream) {
    if (n0 < 8 || n1 < 6 || !coef || !phi || !q || maxit < 2) {
        cfd_internal_set_error("cfd_gauss_solve: bad arguments");
        return CFD_E_ARG;
    }
    for (int m = 0; m < 25; m++)
        if (!coef[m]) {
            cfd_internal_set_error("cfd_gauss_solve: null coefficient plane");
            return CFD_E_ARG;
        }
    double* scratch = nullptr;
    const size_t nd = cfd_seam_scratch_doubles(n0, n1, periodic);
    if (cudaMalloc((void**)&scratch, nd * sizeof(double)) != cudaSuccess) {
        cfd_internal_set_error("cfd_gauss_solve: cudaMalloc of the scratch failed");
        return CFD_E_OOM;
    }
    int rc = cfd_seam_solve(n0, n1, periodic, coef, phi, q, tol, maxit, sweeps, stream, scratch);
    cudaStreamSynchronize((cudaStream_t)stream);
    cudaFree(scratch);
    return rc;
}
