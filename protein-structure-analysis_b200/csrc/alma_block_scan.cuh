// Block-wide exclusive scan of int64 values (used by the list builders).
#pragma once
#include "alma_common.cuh"

namespace alma {

// Exclusive block scan of one int64 per thread; returns the block total.
__device__ __forceinline__ int64_t block_exclusive_scan(int64_t v, int64_t &excl, int64_t *smem /*32*/) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int64_t inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int64_t t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
    }
    if (lane == 31) smem[wid] = inc;
    __syncthreads();
    if (wid == 0) {
        const int nw = blockDim.x >> 5;
        int64_t w = lane < nw ? smem[lane] : 0;
        int64_t wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int64_t t = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += t;
        }
        if (lane < nw) smem[lane] = wi - w;  // exclusive warp offsets
        if (lane == nw - 1) smem[32] = wi;   // block total
    }
    __syncthreads();
    excl = smem[wid] + inc - v;
    const int64_t total = smem[32];
    __syncthreads();
    return total;
}

}  // namespace alma
