// Hex20 A-LLS scatter, pass 1 of 2: list entries (the pattern) and the slot
// map.
//
// Replaces the insert half of assembleGlobalStiffnessKernelALLSFixedArray
// (ALLS_Hex20_3D_Assembly_Performance.cu:226-256: a linear scan of the row's
// columns, a slot claimed with atomicAdd on the row count, no fence), whose
// racing inserts duplicate or drop columns.
//
// One warp per element, persistent over the elements perm[i0, i1) (a wave of
// the spatial element order). For each of the element's 20 row nodes the warp
// copies the node's first list chunk (next link + S1 hashed slots, at most
// 384 bytes) into shared memory with cp.async, all 20 rows at once, so the
// element costs one round trip for its list reads instead of one per row.
// Each lane then resolves its share of the 400 (row node, column node) pairs
// in the shared copy: a column found on its probe sequence is an existing
// entry; otherwise the first empty slot of the sequence is claimed with
// atomicCAS(0 -> column + 1), all of the lane's claims in flight together. A
// CAS that meets another column moves on along the sequence (slots are never
// freed, so a column is found or placed at the first empty slot of its
// sequence, never twice); a full chunk continues in the row's overflow chunks
// (taken from the pool and linked with atomicCAS), read from global memory.
//
// The claimer of a slot zeroes the slot's value block and counts the entry
// for its row; every pair's global slot id goes to the slot map (i - i0) * 400
// + 20 * I + J, which the value pass (values_hex20.cu, or the tensor-core form
// in ke_tcgen05.cu) reads to add the element's Ke blocks with FP64 atomics.
// The two passes are separate launches, so every value block is zeroed before
// any addition reaches it and no entry is ever in a half-written state: no
// pending flags, no fences, no waits.
#include <algorithm>

#include "claim_hex20.cuh"

namespace fem {
namespace {

constexpr int kWarps = 4;
constexpr int kThreads = kWarps * 32;

__global__ void __launch_bounds__(kThreads) k_claim_hex20(MeshView m, ListLayout L, const int* __restrict__ perm,
                                                          int i0, int i1, int* __restrict__ map) {
    __shared__ ClaimWarpSmem sm[kWarps];
    const int w = threadIdx.x >> 5;
    claim_warp(m, L, perm, (long long)i0 + blockIdx.x * kWarps + w, (long long)gridDim.x * kWarps, i1, i0, map, sm[w]);
}

}  // namespace

cudaError_t launch_claim_hex20(const MeshView& m, const ListLayout& L, const int* perm, int i0, int i1, int* map,
                               cudaStream_t s) {
    if (i1 <= i0) return cudaSuccess;
    static DeviceCache cache;
    int per_sm = 0;
    const cudaError_t err = per_device(cache, [](int& v) {
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, k_claim_hex20, kThreads, 0);
    }, per_sm);
    if (err) return err;
    const long long need = (i1 - i0 + kWarps - 1) / kWarps;
    const long long grid = std::max<long long>(1, std::min<long long>(need, (long long)per_sm * sm_count()));
    k_claim_hex20<<<(int)grid, kThreads, 0, s>>>(m, L, perm, i0, i1, map);
    return cudaGetLastError();
}

}  // namespace fem
