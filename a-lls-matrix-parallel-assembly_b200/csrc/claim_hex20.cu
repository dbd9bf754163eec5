// Hex20 A-LLS scatter, pass 1 of 2: list entries (the pattern) and the map
// records of the element groups.
//
// Replaces the insert half of assembleGlobalStiffnessKernelALLSFixedArray
// (ALLS_Hex20_3D_Assembly_Performance.cu:226-256: a linear scan of the row's
// columns, a slot claimed with atomicAdd on the row count, no fence), whose
// racing inserts duplicate or drop columns.
//
// One CTA per element group (group_hex20.cuh: kGroup consecutive positions of
// the spatial order), persistent over the groups of a wave. The CTA numbers
// the group's nodes and node pairs, so an ordered pair (row node, column node)
// that several of the group's elements share is resolved once. Row nodes go
// in batches of kClaimRows: the batch's first list chunks (next link + S1
// hashed slots, at most 384 bytes each) are copied into shared memory with
// cp.async, then the batch's ordered pairs are resolved in placement rounds
// (claim_hex20.cuh): each pending column takes the first slot of its probe
// sequence that is empty in the copy (a shared-memory CAS, so the group's own
// columns never meet in global memory), all of a round's claims go to the list
// as atomicCAS(0 -> column + 1), and a CAS that met another group's column
// moves on in the next round. Slots are never freed, so a column is found or
// placed at the first empty slot of its sequence; the rare second copy that a
// race between groups leaves is retired with a tombstone key before the
// value pass. A full first chunk continues in the row's overflow chunks
// (taken from the pool and linked with atomicCAS), read from global memory.
// The groups are claimed by class g mod 8 (the parities of a brick's
// coordinates in a brick-structured Morton order), so the groups claiming at
// the same time rarely share a row.
//
// Ownership: a pair {u, v} belongs to the group alone when no element outside
// the group has both nodes: the elements of u and of v outside the group
// (from the mesh's node -> element incidence lists, built once per mesh)
// have none in common. The value pass stores such a pair's blocks once; the
// claimer of any other slot zeroes its value block for the atomic adds of
// several groups. Each claimed entry is counted for its row, and the slot id
// (with the shared flag) goes to the group's map record. The two passes are
// separate launches, so every value block is zeroed before any addition
// reaches it and no entry is ever in a half-written state: no pending flags,
// no fences, no waits.
#include <algorithm>

#include "claim_hex20.cuh"

namespace fem {
namespace {

__global__ void __launch_bounds__(kClaimThreads, 3) k_claim_hex20(MeshView m, ListLayout L, const int* __restrict__ perm,
                                                          const int* __restrict__ inc_off, const int* __restrict__ inc,
                                                          int i0, int i1, int* __restrict__ map) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ClaimSmem& sm = *reinterpret_cast<ClaimSmem*>(smem_raw);
    const int ngroups = (i1 - i0 + kGroup - 1) / kGroup;
    // groups by class g mod 8 (for a brick-structured Morton order, the
    // parities of the brick's coordinates), classes ordered so that
    // consecutive ones differ in two or three parities: the groups claiming
    // at the same time rarely share a row node
    const int per = (ngroups + 7) / 8;
    for (int j = blockIdx.x; j < 8 * per; j += gridDim.x) {
        const int g = (j % per) * 8 + ((0x43526170 >> (4 * (j / per))) & 7);
        if (g >= ngroups) continue;
        const long long g0 = (long long)i0 + (long long)g * kGroup;
        claim_group(m, L, perm, inc_off, inc, g0, min(kGroup, i1 - (int)g0), map + (size_t)g * kGroupRecWords, sm);
    }
}

}  // namespace

cudaError_t launch_claim_hex20(const MeshView& m, const ListLayout& L, const int* perm, const int* inc_off,
                               const int* inc, int i0, int i1, int* map, cudaStream_t s) {
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
    k_claim_hex20<<<(int)grid, kClaimThreads, smem, s>>>(m, L, perm, inc_off, inc, i0, i1, map);
    return cudaGetLastError();
}

}  // namespace fem
