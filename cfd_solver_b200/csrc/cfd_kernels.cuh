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
__global__ void k_mg_gs(BatchDev b, int l, int mode, int src, int dst, int inner);
constexpr int MG_GS_THREADS = 128;  // k_mg_gs: one thread per 2 x 2 block of a 32 x 16 tile
__global__ void k_mg_rr(BatchDev b, int l, int src);
__global__ void k_mg_prr(BatchDev b, int l, int dst, int inner);
constexpr int MG_PRR_THREADS = 352;  // k_mg_prr: one thread per 2 x 2 block of its 67 x 19 region
__global__ void k_mg_coarse(BatchDev b, int l, int sweeps);
__global__ void k_mg_galerkin(BatchDev b, int l, int toff);
__global__ void k_correct(BatchDev b);
__global__ void k_bc(BatchDev b);
__global__ void k_diag(BatchDev b);
__global__ void k_si(BatchDev b);
__global__ void k_state_pack(BatchDev b, double* stage, const long long* off, int to_stage);
__global__ void k_loop_cond(cudaGraphConditionalHandle h, const int* flag, int* counter, int maxc, int* total);
__global__ void k_if_cond(cudaGraphConditionalHandle h, const int* flag, int* total);
// the sip9p() seam: the caller's stencil (in the plane order P_AP .. P_ASW), phi0 and q
struct SipIn {
    const double* a[9];
    const double* phi;
    const double* q;
    int n0;
};
__global__ void k_sip_pack(BatchDev b, SipIn in);
__global__ void k_sip_init(BatchDev b);
__global__ void k_sip_out(BatchDev b, double* phi, int n0);
}  // namespace cfd
