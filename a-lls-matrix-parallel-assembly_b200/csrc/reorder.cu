// Element processing order for the 2-D scatter.
//
// The scatter's cost is dominated by the L2 / HBM traffic of the row lists it
// touches. Elements given in a shuffled order (the T3 and mixed benchmark
// meshes) touch lists all over the pool at once; processing them grouped by
// their lowest node id keeps the lists of a band of nodes hot in L2 while all
// of their elements are scattered. The order is a stable-per-bucket counting
// sort computed on the device every call:
//   k_bucket_count    key = type * NB + (min node id >> kBucketShift); histogram
//   k_bucket_scan     one CTA: exclusive scan of the histogram; the element
//                     range of each element type (Q4 first, then T3)
//   k_bucket_scatter  perm[offset[key]++] = e
// The input arrays are not modified; only the order in which the scatter
// visits elements changes (and with it the order of the FP64 atomic adds).
#include <algorithm>

#include "launch.h"

namespace fem {
namespace {

constexpr int kBucketShift = 8;  // 256 nodes per bucket
constexpr int kThreads = 256;

__device__ __forceinline__ int element_key(const MeshView& m, int e, int NB) {
    const int* c = m.conn + (size_t)e * m.stride;
    const bool t3 = m.types ? __ldg(m.types + e) != FEM_Q4 : m.stride == 3;
    const int npe = t3 ? 3 : 4;
    int lo = 0x7FFFFFFF;
    for (int a = 0; a < npe; a++) {
        const int n = __ldg(c + a);
        lo = min(lo, (n >= 0 && n < m.N) ? n : 0);  // bad ids are reported by the scatter
    }
    return (m.types && t3 ? NB : 0) + (lo >> kBucketShift);
}

__global__ void k_bucket_count(MeshView m, int NB, int* __restrict__ hist) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < m.E_count; e += gridDim.x * blockDim.x)
        atomicAdd(hist + element_key(m, e, NB), 1);
}

// Exclusive scan of hist[0..nkeys) in place; ranges = {q4 begin, q4 end, t3 begin, t3 end}.
__global__ void __launch_bounds__(1024) k_bucket_scan(int* __restrict__ hist, int nkeys, int NB, int mixed,
                                                      int* __restrict__ ranges) {
    __shared__ int s_warp[33];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int carry = 0;
    for (int base = 0; base < nkeys; base += 1024) {
        const int k = base + threadIdx.x;
        const int v = k < nkeys ? hist[k] : 0;
        int inc = v;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int o = __shfl_up_sync(0xFFFFFFFFu, inc, d);
            if (lane >= d) inc += o;
        }
        if (lane == 31) s_warp[warp] = inc;
        __syncthreads();
        if (warp == 0) {
            const int w = s_warp[lane];
            int wi = w;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const int o = __shfl_up_sync(0xFFFFFFFFu, wi, d);
                if (lane >= d) wi += o;
            }
            s_warp[lane] = wi - w;
            if (lane == 31) s_warp[32] = wi;
        }
        __syncthreads();
        const int ex = carry + s_warp[warp] + inc - v;
        if (k < nkeys) hist[k] = ex;
        if (mixed && k == NB) ranges[1] = ex;  // first T3 key: number of Q4 elements
        carry += s_warp[32];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        if (mixed) {
            ranges[0] = 0;
            ranges[2] = ranges[1];
            ranges[3] = carry;
        } else {
            ranges[0] = 0;
            ranges[1] = carry;
            ranges[2] = 0;
            ranges[3] = carry;
        }
    }
}

__global__ void k_bucket_scatter(MeshView m, int NB, int* __restrict__ offsets, int* __restrict__ perm) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < m.E_count; e += gridDim.x * blockDim.x)
        perm[atomicAdd(offsets + element_key(m, e, NB), 1)] = e;
}

}  // namespace

int reorder_buckets(int num_nodes) { return (num_nodes >> kBucketShift) + 1; }

cudaError_t launch_reorder(const MeshView& m, int* hist, int* ranges, int* perm, int sms, cudaStream_t s) {
    const int NB = reorder_buckets(m.N);
    const int nkeys = (m.types ? 2 : 1) * NB;
    cudaError_t err = cudaMemsetAsync(hist, 0, (size_t)nkeys * sizeof(int), s);
    if (err) return err;
    const long long want = ((long long)m.E_count + kThreads - 1) / kThreads;
    const int grid = (int)std::min<long long>(want > 0 ? want : 1, (long long)sms * 8);
    k_bucket_count<<<grid, kThreads, 0, s>>>(m, NB, hist);
    k_bucket_scan<<<1, 1024, 0, s>>>(hist, nkeys, NB, m.types ? 1 : 0, ranges);
    k_bucket_scatter<<<grid, kThreads, 0, s>>>(m, NB, hist, perm);
    return cudaGetLastError();
}

}  // namespace fem
