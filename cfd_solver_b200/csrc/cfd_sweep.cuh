// cfd_sweep.cuh -- the persistent momentum / energy sweep kernels (cfd_sweep.cu).
#pragma once
#include "cfd_common.cuh"

namespace cfd {
enum SweepMode { SW_F64 = 0, SW_MX0 = 1, SW_MX = 2 };
constexpr int SW_WARPS = 4;                       // warps per CTA (one 32 x 16 tile)
constexpr int SW_THREADS = 32 * SW_WARPS;
constexpr int SW_ROWS = TYJ / SW_WARPS;           // rows of the tile per thread
constexpr int SWF_THREADS = 512;                  // per-case finalisation, most threads (a batch with a
                                                   // case of >= 1024 tiles; 128 otherwise)

__global__ void k_sweep_f64(BatchDev b);
__global__ void k_sweep_mx0(BatchDev b);
__global__ void k_sweep_mx1(BatchDev b);
__global__ void k_sweep_fin(BatchDev b);
__global__ void k_mom_update(BatchDev b);
__global__ void k_mom_fix(BatchDev b);
size_t sweep_smem_f64();
size_t sweep_smem_mx0();
size_t sweep_smem_mx1();
}  // namespace cfd
