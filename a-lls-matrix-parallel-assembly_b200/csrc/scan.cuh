// Block-wide exclusive scan shared by the consolidation and the colouring
// kernels.
#pragma once

namespace fem {

constexpr int kScanThreads = 256;

// Block-wide exclusive scan of one long long per thread (kScanThreads threads).
__device__ __forceinline__ long long block_exclusive_scan(long long v, long long* s_warp, long long& total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    long long inc = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const long long o = __shfl_up_sync(0xFFFFFFFFu, inc, d);
        if (lane >= d) inc += o;
    }
    if (lane == 31) s_warp[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        long long w = lane < kScanThreads / 32 ? s_warp[lane] : 0;
        long long wi = w;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const long long o = __shfl_up_sync(0xFFFFFFFFu, wi, d);
            if (lane >= d) wi += o;
        }
        if (lane < kScanThreads / 32) s_warp[lane] = wi - w;
        if (lane == kScanThreads / 32 - 1) s_warp[kScanThreads / 32] = wi;
    }
    __syncthreads();
    total = s_warp[kScanThreads / 32];
    const long long out = s_warp[warp] + inc - v;
    __syncthreads();  // s_warp may be reused by the caller's next scan
    return out;
}

}  // namespace fem
