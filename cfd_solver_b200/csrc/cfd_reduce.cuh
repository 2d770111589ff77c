// cfd_reduce.cuh -- deterministic per-case reductions over a tile table.
//
// Every CTA of a tile kernel reduces its values, writes one partial per tile,
// and the last CTA of each case (detected with a per-case arrival counter)
// sums that case's partials in a fixed order and runs the finaliser. The
// result does not depend on CTA scheduling or on which other cases share the
// launch, so a case gives the same bits alone and inside any batch.
#pragma once
#include "cfd_common.cuh"

namespace cfd {

constexpr int PSTRIDE = 8;  // doubles per tile partial

// op bit k set => value k is a max, else a sum
template <int NV, unsigned MAXMASK>
__device__ __forceinline__ void block_reduce_mixed(double (&v)[NV], double* smem) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; k++) {
        const bool mx = (MAXMASK >> k) & 1u;
        double x = v[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            double y = __shfl_down_sync(0xffffffffu, x, o);
            x = mx ? fmax(x, y) : x + y;
        }
        if (lane == 0) smem[k * 32 + warp] = x;
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < NV; k++) {
            const bool mx = (MAXMASK >> k) & 1u;
            double x = lane < nw ? smem[k * 32 + lane] : (mx ? -1.0e300 : 0.0);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                double y = __shfl_down_sync(0xffffffffu, x, o);
                x = mx ? fmax(x, y) : x + y;
            }
            v[k] = x;
        }
    }
    __syncthreads();
}

// Returns true (in every thread of the CTA) when this CTA is the last of case
// `cid`; then `v` holds the case totals in thread 0.
template <int NV, unsigned MAXMASK>
__device__ __forceinline__ bool case_reduce(const BatchDev& b, int cid, int tile_global,
                                            int tile_begin, int tile_count, double (&v)[NV]) {
    static_assert(NV <= PSTRIDE, "too many reduction values");
    __shared__ double smem[NV * 32];
    __shared__ int is_last;
    block_reduce_mixed<NV, MAXMASK>(v, smem);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; k++) b.partial[(long long)tile_global * PSTRIDE + k] = v[k];
        __threadfence();
        unsigned prev = atomicAdd(&b.counter[cid], 1u);
        is_last = (prev == (unsigned)(tile_count - 1));
    }
    __syncthreads();
    if (!is_last) return false;
    __threadfence();
    double acc[NV];
#pragma unroll
    for (int k = 0; k < NV; k++) acc[k] = ((MAXMASK >> k) & 1u) ? -1.0e300 : 0.0;
    for (int t = threadIdx.x; t < tile_count; t += blockDim.x) {
        const double* src = b.partial + (long long)(tile_begin + t) * PSTRIDE;
#pragma unroll
        for (int k = 0; k < NV; k++) {
            double x = __ldcg(src + k);
            acc[k] = ((MAXMASK >> k) & 1u) ? fmax(acc[k], x) : acc[k] + x;
        }
    }
    block_reduce_mixed<NV, MAXMASK>(acc, smem);
#pragma unroll
    for (int k = 0; k < NV; k++) v[k] = acc[k];
    if (threadIdx.x == 0) b.counter[cid] = 0u;
    return true;
}

}  // namespace cfd
