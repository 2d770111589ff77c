// cfd_kernels.cuh -- kernel entry points launched by the host runtime (cfd_api.cu).
#pragma once
#include "cfd_common.cuh"

namespace cfd {
__global__ void k_assemble_p(BatchDev b, int toff);
__global__ void k_rhs(BatchDev b);
extern const size_t kRhsSmem;
extern const size_t kFaceQSmem;
__global__ void k_upbc(BatchDev b);
__global__ void k_face_q(BatchDev b);
__global__ void k_bicg_p(BatchDev b);
__global__ void k_spmv(BatchDev b, int mode);
__global__ void k_bicg_s(BatchDev b);
__global__ void k_bicg_x(BatchDev b, int maxit);
__global__ void k_mg_smooth(BatchDev b, int l, int colour);
__global__ void k_mg_smooth_blk(BatchDev b, int l, int reverse, int zero_init);
__global__ void k_mg_resid(BatchDev b, int l);
__global__ void k_mg_restrict(BatchDev b, int l);
__global__ void k_mg_prolong(BatchDev b, int l);
__global__ void k_mg_coarse(BatchDev b, int l, int sweeps);
__global__ void k_mg_galerkin(BatchDev b, int l, int toff);
__global__ void k_correct(BatchDev b);
__global__ void k_bc(BatchDev b);
__global__ void k_diag(BatchDev b);
__global__ void k_si(BatchDev b);
__global__ void k_loop_cond(cudaGraphConditionalHandle h, const int* flag, int* counter, int maxc, int* total);
}  // namespace cfd
