// Element processing order for the scatter kernels.
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
// When the key table fits in shared memory (up to 40 K keys), one CTA per SM
// counts and places its elements with shared-memory atomics instead
// (k_key_count_sm, k_key_scatter_sm), one global atomic per non-zero key.
// The input arrays are not modified; only the order in which the scatter
// visits elements changes (and with it the order of the FP64 atomic adds).
//
// Hex20 meshes use a spatial order instead: a row node's elements (up to 8)
// should be scattered close together in time, or its list lines are evicted
// from L2 between their visits (in natural x-y-z order they are a whole z-layer
// of elements apart). The key is the 3-D Morton code of the midpoint of each
// element's corner diagonal (nodes 0 and 6), quantized on a 2^b grid over the
// node bounding box (k_bbox), counting-sorted the same way.
#include <algorithm>

#include "launch.h"

namespace fem {
namespace {

constexpr int kBucketShift = 8;  // 256 nodes per bucket
constexpr int kThreads = 256;
constexpr int kMaxMortonBits = 5;  // at most 32^3 spatial buckets

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

// Order-preserving map of a double to an unsigned 64-bit integer.
__device__ __forceinline__ unsigned long long ordered_bits(double v) {
    const unsigned long long u = (unsigned long long)__double_as_longlong(v);
    return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}
__device__ __forceinline__ double from_ordered_bits(unsigned long long u) {
    return __longlong_as_double((long long)((u >> 63) ? (u & 0x7FFFFFFFFFFFFFFFull) : ~u));
}

// bbox = {min x, min y, min z, max x, max y, max z} as ordered bits.
__global__ void k_bbox_init(unsigned long long* bbox) {
    if (threadIdx.x < 3) bbox[threadIdx.x] = ~0ull;
    else if (threadIdx.x < 6) bbox[threadIdx.x] = 0ull;
}

__global__ void k_bbox(MeshView m, unsigned long long* bbox) {
    unsigned long long lo[3] = {~0ull, ~0ull, ~0ull}, hi[3] = {0ull, 0ull, 0ull};
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < m.N; n += gridDim.x * blockDim.x) {
        const unsigned long long v[3] = {ordered_bits(__ldg(m.x + n)), ordered_bits(__ldg(m.y + n)),
                                         ordered_bits(__ldg(m.z + n))};
#pragma unroll
        for (int d = 0; d < 3; d++) {
            lo[d] = v[d] < lo[d] ? v[d] : lo[d];
            hi[d] = v[d] > hi[d] ? v[d] : hi[d];
        }
    }
#pragma unroll
    for (int d = 0; d < 3; d++) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long l2 = __shfl_xor_sync(0xFFFFFFFFu, lo[d], o);
            const unsigned long long h2 = __shfl_xor_sync(0xFFFFFFFFu, hi[d], o);
            lo[d] = l2 < lo[d] ? l2 : lo[d];
            hi[d] = h2 > hi[d] ? h2 : hi[d];
        }
    }
    if ((threadIdx.x & 31) == 0) {
#pragma unroll
        for (int d = 0; d < 3; d++) {
            atomicMin(bbox + d, lo[d]);
            atomicMax(bbox + 3 + d, hi[d]);
        }
    }
}

// Spreads the low 10 bits of v to every third bit.
__device__ __forceinline__ unsigned spread3(unsigned v) {
    v &= 0x3FFu;
    v = (v | (v << 16)) & 0x030000FFu;
    v = (v | (v << 8)) & 0x0300F00Fu;
    v = (v | (v << 4)) & 0x030C30C3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

__device__ __forceinline__ int morton_key(const MeshView& m, int e, const unsigned long long* bbox, int bits) {
    const int* c = m.conn + (size_t)e * m.stride;
    int n0 = __ldg(c + 0), n6 = __ldg(c + 6);
    n0 = (n0 >= 0 && n0 < m.N) ? n0 : 0;  // bad ids are reported by the scatter
    n6 = (n6 >= 0 && n6 < m.N) ? n6 : 0;
    const double p[3] = {0.5 * (__ldg(m.x + n0) + __ldg(m.x + n6)), 0.5 * (__ldg(m.y + n0) + __ldg(m.y + n6)),
                         0.5 * (__ldg(m.z + n0) + __ldg(m.z + n6))};
    const int cells = 1 << bits;
    unsigned q[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const double lo = from_ordered_bits(bbox[d]), hi = from_ordered_bits(bbox[3 + d]);
        const double t = hi > lo ? (p[d] - lo) / (hi - lo) : 0.0;
        int qi = (int)(t * cells);
        q[d] = (unsigned)min(max(qi, 0), cells - 1);
    }
    return (int)(spread3(q[0]) | (spread3(q[1]) << 1) | (spread3(q[2]) << 2));
}

__global__ void k_morton_count(MeshView m, const unsigned long long* bbox, int bits, int* __restrict__ hist) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < m.E_count; e += gridDim.x * blockDim.x)
        atomicAdd(hist + morton_key(m, e, bbox, bits), 1);
}

__global__ void k_morton_scatter(MeshView m, const unsigned long long* bbox, int bits, int* __restrict__ offsets,
                                 int* __restrict__ perm) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < m.E_count; e += gridDim.x * blockDim.x)
        perm[atomicAdd(offsets + morton_key(m, e, bbox, bits), 1)] = e;
}

// Keys of the two orders as functors for the shared-memory histogram kernels.
struct BucketKey {
    MeshView m;
    int NB;
    __device__ __forceinline__ int operator()(int e) const { return element_key(m, e, NB); }
};
struct MortonKey {
    MeshView m;
    const unsigned long long* bbox;
    int bits;
    __device__ __forceinline__ int operator()(int e) const { return morton_key(m, e, bbox, bits); }
};

// Shared-memory histograms (when the key table fits): a CTA counts its
// elements' keys with shared-memory atomics and flushes each non-zero counter
// with one global atomic, instead of one global atomic per element.
constexpr int kSmThreads = 1024;
constexpr int kMaxSmemKeys = 160 * 1024 / 4;

template <typename Key>
__global__ void __launch_bounds__(kSmThreads) k_key_count_sm(Key key, int E, int nkeys, int* __restrict__ hist) {
    extern __shared__ int s_cnt[];
    for (int k = threadIdx.x; k < nkeys; k += blockDim.x) s_cnt[k] = 0;
    __syncthreads();
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < E; e += gridDim.x * blockDim.x)
        atomicAdd(&s_cnt[key(e)], 1);
    __syncthreads();
    for (int k = threadIdx.x; k < nkeys; k += blockDim.x)
        if (s_cnt[k]) atomicAdd(hist + k, s_cnt[k]);
}

// offsets: the exclusive scan of the histogram. A CTA counts its elements'
// keys again, reserves one range per key (one global atomic per non-zero key)
// and places its elements inside the ranges with shared-memory atomics.
template <typename Key>
__global__ void __launch_bounds__(kSmThreads) k_key_scatter_sm(Key key, int E, int nkeys, int* __restrict__ offsets,
                                                               int* __restrict__ perm) {
    extern __shared__ int s_pos[];
    for (int k = threadIdx.x; k < nkeys; k += blockDim.x) s_pos[k] = 0;
    __syncthreads();
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < E; e += gridDim.x * blockDim.x)
        atomicAdd(&s_pos[key(e)], 1);
    __syncthreads();
    for (int k = threadIdx.x; k < nkeys; k += blockDim.x) {
        const int c = s_pos[k];
        if (c) s_pos[k] = atomicAdd(offsets + k, c);
    }
    __syncthreads();
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < E; e += gridDim.x * blockDim.x)
        perm[atomicAdd(&s_pos[key(e)], 1)] = e;
}

// The shared-memory kernels' attribute (dynamic shared memory above 48 KB) is
// set once per device.
template <typename Key>
cudaError_t smem_kernels_ready() {
    static DeviceCache cache;
    int ok = 0;
    return per_device(cache, [](int& v) {
        cudaError_t e = cudaFuncSetAttribute(k_key_count_sm<Key>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             kMaxSmemKeys * (int)sizeof(int));
        if (!e)
            e = cudaFuncSetAttribute(k_key_scatter_sm<Key>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     kMaxSmemKeys * (int)sizeof(int));
        v = 1;
        return e;
    }, ok);
}

// Counting sort of the elements by key: histogram, scan (ranges), scatter.
template <typename Key, typename CountK, typename ScatterK>
cudaError_t counting_sort(const Key& key, int E, int nkeys, int NB, int mixed, int* hist, int* ranges, int* perm,
                          int sms, CountK count_global, ScatterK scatter_global, cudaStream_t s) {
    if (nkeys <= kMaxSmemKeys) {
        cudaError_t err = smem_kernels_ready<Key>();
        if (err) return err;
        const long long want = ((long long)E + kSmThreads - 1) / kSmThreads;
        const int grid = (int)std::min<long long>(want > 0 ? want : 1, (long long)sms);
        const size_t smem = (size_t)nkeys * sizeof(int);
        k_key_count_sm<Key><<<grid, kSmThreads, smem, s>>>(key, E, nkeys, hist);
        k_bucket_scan<<<1, 1024, 0, s>>>(hist, nkeys, NB, mixed, ranges);
        k_key_scatter_sm<Key><<<grid, kSmThreads, smem, s>>>(key, E, nkeys, hist, perm);
    } else {
        const long long want = ((long long)E + kThreads - 1) / kThreads;
        const int grid = (int)std::min<long long>(want > 0 ? want : 1, (long long)sms * 8);
        count_global(grid);
        k_bucket_scan<<<1, 1024, 0, s>>>(hist, nkeys, NB, mixed, ranges);
        scatter_global(grid);
    }
    return cudaGetLastError();
}

}  // namespace

int reorder_buckets(int num_nodes) { return (num_nodes >> kBucketShift) + 1; }

int morton_bits(int num_elems) {
    int b = 1;
    while (b < kMaxMortonBits && (1ll << (3 * b)) * 4 < (long long)num_elems) b++;
    return b;
}

cudaError_t launch_reorder_3d(const MeshView& m, int* hist, int* ranges, int* perm, unsigned long long* bbox, int sms,
                              cudaStream_t s) {
    const int bits = morton_bits(m.E_count);
    const int nkeys = 1 << (3 * bits);
    cudaError_t err = cudaMemsetAsync(hist, 0, (size_t)nkeys * sizeof(int), s);
    if (err) return err;
    k_bbox_init<<<1, 32, 0, s>>>(bbox);
    const long long wn = ((long long)m.N + kThreads - 1) / kThreads;
    k_bbox<<<(int)std::min<long long>(wn > 0 ? wn : 1, (long long)sms * 4), kThreads, 0, s>>>(m, bbox);
    return counting_sort(
        MortonKey{m, bbox, bits}, m.E_count, nkeys, nkeys, 0, hist, ranges, perm, sms,
        [&](int grid) { k_morton_count<<<grid, kThreads, 0, s>>>(m, bbox, bits, hist); },
        [&](int grid) { k_morton_scatter<<<grid, kThreads, 0, s>>>(m, bbox, bits, hist, perm); }, s);
}

cudaError_t launch_reorder(const MeshView& m, int* hist, int* ranges, int* perm, int sms, cudaStream_t s) {
    const int NB = reorder_buckets(m.N);
    const int nkeys = (m.types ? 2 : 1) * NB;
    cudaError_t err = cudaMemsetAsync(hist, 0, (size_t)nkeys * sizeof(int), s);
    if (err) return err;
    return counting_sort(
        BucketKey{m, NB}, m.E_count, nkeys, NB, m.types ? 1 : 0, hist, ranges, perm, sms,
        [&](int grid) { k_bucket_count<<<grid, kThreads, 0, s>>>(m, NB, hist); },
        [&](int grid) { k_bucket_scatter<<<grid, kThreads, 0, s>>>(m, NB, hist, perm); }, s);
}

}  // namespace fem
