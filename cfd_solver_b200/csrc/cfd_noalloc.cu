// cfd_noalloc.cu -- cfd_gauss_solve_noalloc(): the gauss() seam without any allocation.
//
// Some callers cannot call cudaMalloc: a host application whose device memory is owned
// by another allocator or pool that must not be bypassed (a framework's caching allocator,
// a memory budget enforced by the embedding program), and real-time loops that must not
// take the allocator's locks or risk an out-of-memory failure in the middle of a step.
// For them this entry point runs the same solve as cfd_gauss_solve() with its scratch
// (the second iterate, the reduction partials and a few scalars) in one file-scope
// device array of fixed size, so the call itself allocates nothing. The solve reads its
// stop flag on the host after every pair of sweeps, so each call waits for its own work.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/cfd_b200.h"

int cfd_seam_solve(int n0, int n1, int periodic, const double* const* coef, double* phi, const double* q,
                   double tol, int maxit, int* sweeps, void* stream, double* scratch);
size_t cfd_seam_scratch_doubles(int n0, int n1, int periodic);
void cfd_internal_set_error(const char* msg);

namespace {

// largest grid (n0 * n1 points) the static scratch serves: 2^20 points (1025 x 1023)
constexpr long long kMaxPoints = CFD_NOALLOC_MAX_POINTS;
// second iterate + one partial per 256 cells (rounded) + scalars + counter
constexpr long long kScratchDoubles = kMaxPoints + (kMaxPoints / 256 + 64) + 16;

// Every GPU that loads this library holds this array (about 8.4 MB) until the process
// exits. All calls on a device share it, and each call leaves its contents behind.
__device__ __align__(256) double g_gauss_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
double* g_scratch_ptr[kMaxDevices] = {};
std::mutex g_scratch_mu;

}  // namespace

extern "C" int cfd_gauss_solve_noalloc(int n0, int n1, int periodic, const double* const* coef,
                                       double* phi, const double* q, double tol, int maxit,
                                       int* sweeps, void* stream) {
    if (n0 < 8 || n1 < 6 || !coef || !phi || !q || maxit < 2) {
        cfd_internal_set_error("cfd_gauss_solve_noalloc: bad arguments");
        return CFD_E_ARG;
    }
    for (int m = 0; m < 25; m++)
        if (!coef[m]) {
            cfd_internal_set_error("cfd_gauss_solve_noalloc: null coefficient plane");
            return CFD_E_ARG;
        }
    if ((long long)n0 * n1 > kMaxPoints ||
        (long long)cfd_seam_scratch_doubles(n0, n1, periodic) > kScratchDoubles) {
        cfd_internal_set_error(("cfd_gauss_solve_noalloc: grid of " + std::to_string((long long)n0 * n1) +
                                " points exceeds the static scratch limit of " + std::to_string(kMaxPoints) +
                                " points (CFD_NOALLOC_MAX_POINTS)").c_str());
        return CFD_E_ARG;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        cfd_internal_set_error("cfd_gauss_solve_noalloc: no usable current device");
        return CFD_E_CUDA;
    }
    double* scratch = nullptr;
    {
        // set-up, once per device and with that device current: the device address of the
        // array (in host code its name is only a host-side stand-in)
        std::lock_guard<std::mutex> lock(g_scratch_mu);
        if (!g_scratch_ptr[dev]) {
            double* p = nullptr;
            cudaError_t e = cudaGetSymbolAddress((void**)&p, g_gauss_scratch);
            if (e != cudaSuccess || !p) {
                cfd_internal_set_error((std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e)).c_str());
                return CFD_E_CUDA;
            }
            g_scratch_ptr[dev] = p;
        }
        scratch = g_scratch_ptr[dev];
    }
    // cfd_seam_solve clears the scalars and the counter it relies on before its first sweep
    const int rc = cfd_seam_solve(n0, n1, periodic, coef, phi, q, tol, maxit, sweeps, stream, scratch);
    // an error return can leave sweeps of this call queued on the stream; they must finish
    // before the caller's next call reuses the shared array
    if (rc == CFD_E_CUDA) cudaStreamSynchronize((cudaStream_t)stream);
    return rc;
}
