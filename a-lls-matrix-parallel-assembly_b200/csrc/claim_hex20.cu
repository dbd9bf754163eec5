// Hex20 A-LLS scatter, pass 1 of 2: list entries (the pattern) and the
// records of the element groups.
//
// Replaces the insert half of assembleGlobalStiffnessKernelALLSFixedArray
// (ALLS_Hex20_3D_Assembly_Performance.cu:226-256: a linear scan of the row's
// columns, a slot claimed with atomicAdd on the row count, no fence), whose
// racing inserts duplicate or drop columns.
//
// One CTA per element group (group_hex20.cuh: kGroup consecutive positions of
// the spatial order), persistent over the groups of a wave. The CTA numbers
// the group's nodes and node pairs and writes the group's record: node ids,
// the block table of its elements (pair index, orientation, sole block), and
// the slot word of every ordered pair (row node, column node), found or
// claimed once however many of the group's elements share it.
//
// Claims (claim_group, the batched kernel): the group's rows' first chunks
// are copied into shared memory with cp.async; every ordered pair is probed
// in the copy; each absent column is claimed with atomicCAS(0 -> column + 1)
// at the first slot empty in the copy, all of a thread's claims in flight
// together, each outcome written back to the copy (which so only ever holds
// what the slot truly holds); a CAS that met another claimer's column walks
// on along its probe sequence (slots are never freed, so a column is found or
// placed at the first empty slot of its sequence, never twice); a full first
// chunk continues in the row's overflow chunks (taken from the pool and
// linked with atomicCAS). Ownership: a pair belongs to the group alone when
// no element outside the group has both nodes (64-bit masks of the outside
// elements, from the mesh's node -> element incidence; without it every pair
// counts as shared). The claimer of a shared pair's slot zeroes its value
// block; each claimed entry is counted for its row.
//
// Lookup (k_claim_hex20, the single-mesh path): the wave's row pass
// (rows_hex20.cu) has inserted every column already, with the pairs' shared
// flags in the slot words; the group finds its slots in the copies and
// writes the record.
//
// The value pass (values_hex20.cu) is a separate launch, so every value block
// is zeroed before any addition reaches it and no entry is ever in a
// half-written state: no pending flags, no fences, no waits.
#include <algorithm>

#include "claim_hex20.cuh"

namespace fem {
namespace {

__global__ void __launch_bounds__(kClaimThreads, 3) k_claim_hex20(MeshView m, ListLayout L, const int* __restrict__ perm,
                                                                   int i0, int i1, int* __restrict__ map) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ClaimSmem& sm = *reinterpret_cast<ClaimSmem*>(smem_raw);
    const int ngroups = (i1 - i0 + kGroup - 1) / kGroup;
    for (int g = blockIdx.x; g < ngroups; g += gridDim.x) {
        const long long g0 = (long long)i0 + (long long)g * kGroup;
        claim_group<true>(m, L, perm, nullptr, nullptr, g0, min(kGroup, i1 - (int)g0), map + (size_t)g * kGroupRecWords,
                          sm);
    }
}

}  // namespace

cudaError_t launch_claim_hex20(const MeshView& m, const ListLayout& L, const int* perm, int i0, int i1, int* map,
                               cudaStream_t s) {
    if (i1 <= i0) return cudaSuccess;
    static DeviceCache cache;
    const size_t smem = sizeof(ClaimSmem);
    int per_sm = 0;
    const cudaError_t err = per_device(cache, [&](int& v) {
        cudaError_t e = cudaFuncSetAttribute(k_claim_hex20, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (!e) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, k_claim_hex20, kClaimThreads, smem);
        return e;
    }, per_sm);
    if (err) return err;
    const long long need = (i1 - i0 + kGroup - 1) / kGroup;
    const long long grid = std::max<long long>(1, std::min<long long>(need, (long long)per_sm * sm_count()));
    k_claim_hex20<<<(int)grid, kClaimThreads, smem, s>>>(m, L, perm, i0, i1, map);
    return cudaGetLastError();
}

}  // namespace fem
