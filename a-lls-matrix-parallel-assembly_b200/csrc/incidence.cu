// Node -> element incidence lists (CSR over the nodes) of a mesh: the
// colouring baseline's neighbour structure (colour.cu) and, for Hex20, the
// ownership test of the list scatter's element groups (claim_hex20.cuh).
//
//   k_inc_count                  cnt[n] = elements with node n (a node twice
//                                in one element counts twice)
//   k_tile_sums / k_tile_scan /  off = exclusive prefix of cnt in tiles of
//   k_tile_apply                 kScanTile nodes; cnt cleared for the fill
//   k_inc_fill                   inc[off[n] ..] = the elements, in no order;
//                                cnt[n] is the count again afterwards
#include <algorithm>

#include "launch.h"
#include "scan.cuh"

namespace fem {
namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ int elem_npe(const MeshView& m, int e) {
    if (m.types) return __ldg(m.types + e) == FEM_Q4 ? 4 : 3;
    return m.stride;
}

__global__ void k_inc_count(MeshView m, int* __restrict__ cnt, int* status) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < m.E_count; e += gridDim.x * blockDim.x) {
        const int npe = elem_npe(m, e);
        for (int k = 0; k < npe; k++) {
            const int n = __ldg(m.conn + (size_t)e * m.stride + k);
            if (n < 0 || n >= m.N) {
                atomicOr(status, 1 << FEM_ERR_BAD_MESH);
                continue;
            }
            atomicAdd(cnt + n, 1);
        }
    }
}

// Tile sums of cnt (kScanTile entries per CTA).
__global__ void __launch_bounds__(kScanThreads) k_tile_sums(const int* __restrict__ cnt, int N,
                                                            long long* __restrict__ tiles) {
    __shared__ long long s_warp[kScanThreads / 32 + 1];
    long long sum = 0;
    for (int i = 0; i < kScanTile / kScanThreads; i++) {
        const long long n = (long long)blockIdx.x * kScanTile + (long long)i * kScanThreads + threadIdx.x;
        if (n < N) sum += cnt[n];
    }
    long long total;
    block_exclusive_scan(sum, s_warp, total);
    if (threadIdx.x == 0) tiles[blockIdx.x] = total;
}

// Exclusive scan of the tile sums in place (one CTA); off[N] = total.
__global__ void __launch_bounds__(kScanThreads) k_tile_scan(long long* __restrict__ tiles, int num_tiles,
                                                            int* __restrict__ off_end, int* status) {
    __shared__ long long s_warp[kScanThreads / 32 + 1];
    long long carry = 0;
    for (int base = 0; base < num_tiles; base += kScanThreads) {
        const int t = base + threadIdx.x;
        const long long v = t < num_tiles ? tiles[t] : 0;
        long long total;
        const long long ex = block_exclusive_scan(v, s_warp, total);
        if (t < num_tiles) tiles[t] = carry + ex;
        carry += total;
    }
    if (threadIdx.x == 0) {
        *off_end = (int)carry;
        if (carry > 0x7FFFFFFFll) atomicOr(status, 1 << FEM_ERR_RANGE);
    }
}

// off[n] = exclusive prefix of cnt; cnt is cleared for the fill pass.
__global__ void __launch_bounds__(kScanThreads) k_tile_apply(int* __restrict__ cnt, int N,
                                                             const long long* __restrict__ tiles,
                                                             int* __restrict__ off) {
    constexpr int kItems = kScanTile / kScanThreads;
    __shared__ long long s_warp[kScanThreads / 32 + 1];
    const long long base = (long long)blockIdx.x * kScanTile + (long long)threadIdx.x * kItems;
    int c[kItems];
    long long sum = 0;
#pragma unroll
    for (int i = 0; i < kItems; i++) {
        c[i] = base + i < N ? cnt[base + i] : 0;
        sum += c[i];
    }
    long long total;
    long long o = tiles[blockIdx.x] + block_exclusive_scan(sum, s_warp, total);
#pragma unroll
    for (int i = 0; i < kItems; i++) {
        if (base + i < N) {
            off[base + i] = (int)o;
            cnt[base + i] = 0;
        }
        o += c[i];
    }
}

__global__ void k_inc_fill(MeshView m, const int* __restrict__ off, int* __restrict__ cursor, int* __restrict__ inc) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < m.E_count; e += gridDim.x * blockDim.x) {
        const int npe = elem_npe(m, e);
        for (int k = 0; k < npe; k++) {
            const int n = __ldg(m.conn + (size_t)e * m.stride + k);
            if (n < 0 || n >= m.N) continue;
            inc[off[n] + atomicAdd(cursor + n, 1)] = e;
        }
    }
}

}  // namespace

cudaError_t launch_incidence(const MeshView& m, int* cnt, int* off, int* inc, long long* tiles, int* status, int sms,
                             cudaStream_t s) {
    cudaError_t err = cudaMemsetAsync(cnt, 0, (size_t)m.N * sizeof(int), s);
    if (err) return err;
    const int num_tiles = (m.N + kScanTile - 1) / kScanTile;
    const int ge = (int)std::max<long long>(1, std::min<long long>(((long long)m.E_count + kThreads - 1) / kThreads,
                                                                   (long long)sms * 8));
    if (m.E_count > 0) k_inc_count<<<ge, kThreads, 0, s>>>(m, cnt, status);
    k_tile_sums<<<num_tiles, kScanThreads, 0, s>>>(cnt, m.N, tiles);
    k_tile_scan<<<1, kScanThreads, 0, s>>>(tiles, num_tiles, off + m.N, status);
    k_tile_apply<<<num_tiles, kScanThreads, 0, s>>>(cnt, m.N, tiles, off);
    if (m.E_count > 0) k_inc_fill<<<ge, kThreads, 0, s>>>(m, off, cnt, inc);
    return cudaGetLastError();
}

}  // namespace fem
