// K1 for 2-D meshes: fused Q4 / T3 element stiffness + A-LLS row-list scatter.
//
// Replaces assembleGlobalStiffnessKernelALLS
// (ALLS_Quad2D_Assembly_Accuracy_Analysis.cu:394-468,
//  ALLS_T3_Unstructed_Elements_Assemble_Performance.cu:227-290,
//  ALLS_Q4_T3_Mixed_Elements_Assembly_Performance.cu:248-312).
//
// One thread per element, as in the reference, but:
//  * Ke is computed in registers in node-block form (upper blocks only);
//  * each row node's list is read one 64-byte chunk row at a time (next pointer
//    and 14 hashed slots in four 16-byte L2 loads) and all of the element's
//    column nodes are resolved against that view: a column is looked up along
//    its probe sequence and, if absent, its slot is claimed with atomicCAS
//    (empty -> col|pending) — one slot per column and row, never a duplicate;
//  * the claimer stores its block values with plain 16-byte stores, fences, and
//    publishes the column; found columns are accumulated with atomicAdd
//    (red.global.add.f64), after a bounded wait if the slot is still pending.
//    A thread publishes its own claims before it waits on anyone else's, so
//    no wait can be circular.
// The reference instead walks a pointer list per (row, col) pair and can lose a
// contribution or insert a column twice (its head-insert race, Q4A:452-463).
#include "element2d.cuh"
#include "launch.h"

namespace fem {
namespace {

enum SlotState : int { kUnresolved = 0, kFound = 1, kFoundPending = 2, kClaimed = 3 };
constexpr int kMask14 = (1 << k2DSlots) - 1;

__device__ __forceinline__ unsigned rot14(unsigned m, int h) {
    return ((m >> h) | (m << (k2DSlots - h))) & kMask14;
}

template <int NPE>
__device__ __forceinline__ void scatter_element_2d(const MeshView& m, const ListLayout& L, int e, int& spare) {
    using Blk = Blocks2D<NPE>;
    int nodes[NPE];
    bool bad = false;
#pragma unroll
    for (int a = 0; a < NPE; a++) {
        nodes[a] = __ldg(m.conn + (size_t)e * m.stride + a);
        bad |= (nodes[a] < 0) | (nodes[a] >= m.N);
    }
    if (bad) {
        raise_status(L.info, FEM_ERR_BAD_MESH);
        return;
    }
    double xe[NPE], ye[NPE];
#pragma unroll
    for (int a = 0; a < NPE; a++) {
        xe[a] = __ldg(m.x + nodes[a]);
        ye[a] = __ldg(m.y + nodes[a]);
    }
    const double E = m.E ? __ldg(m.E + e) : m.E0;
    const double nu = m.nu ? __ldg(m.nu + e) : m.nu0;
    double kb[Blk::kCount][4];
    double det;
    if constexpr (NPE == 4) {
        det = ke_q4_blocks(xe, ye, E, nu, m.t, kb);
    } else {
        det = ke_t3_blocks(xe, ye, E, nu, m.t, kb);
    }
    if (!(det > 0.0)) raise_status(L.info, FEM_ERR_DETJ);

#pragma unroll
    for (int a = 0; a < NPE; a++) {
        int state[NPE];
        unsigned gid[NPE];
        int* word[NPE];
#pragma unroll
        for (int b = 0; b < NPE; b++) {
            state[b] = kUnresolved;
            gid[b] = 0;
            word[b] = nullptr;
        }
        // Resolve the slot of every column node of the element in row node a.
        // A failed CAS means the register view of the chunk is stale; the chunk
        // is then re-read before the remaining columns are resolved (a column
        // another thread has just claimed must be found, not claimed again).
        int c = nodes[a];
        for (int step = 0; step < kMaxChainSteps; step++) {
            int* meta = chunk_meta(L, c);
            const int4 w0 = ld_cg4(meta), w1 = ld_cg4(meta + 4), w2 = ld_cg4(meta + 8), w3 = ld_cg4(meta + 12);
            const int cols[k2DSlots] = {w0.z, w0.w, w1.x, w1.y, w1.z, w1.w, w2.x,
                                        w2.y, w2.z, w2.w, w3.x, w3.y, w3.z, w3.w};
            unsigned empty = 0, pend = 0;
#pragma unroll
            for (int s = 0; s < k2DSlots; s++) {
                empty |= (cols[s] == 0 ? 1u : 0u) << s;
                pend |= (cols[s] < 0 ? 1u : 0u) << s;
            }
            bool all = true, full = false, stale = false;
#pragma unroll
            for (int b = 0; b < NPE; b++) {
                if (state[b] == kUnresolved && !stale) {
                    const int key = nodes[b] + 1;
                    unsigned match = 0;
#pragma unroll
                    for (int s = 0; s < k2DSlots; s++) match |= (((cols[s] & kColMask) == key) ? 1u : 0u) << s;
                    const int h = probe_start(key, k2DSlots);
                    const unsigned cand = rot14(match | empty, h);
                    if (!cand) {
                        full = true;  // no free slot on this chunk's probe sequence
                    } else {
                        int pos = h + __ffs(cand) - 1;
                        pos -= pos >= k2DSlots ? k2DSlots : 0;
                        if (match & (1u << pos)) {
                            state[b] = (pend >> pos) & 1u ? kFoundPending : kFound;
                        } else {
                            const int old = atomicCAS(meta + 2 + pos, 0, key | kPending);
                            if (old == 0) {
                                state[b] = kClaimed;
                                empty &= ~(1u << pos);
                            } else if ((old & kColMask) == key) {
                                state[b] = old < 0 ? kFoundPending : kFound;
                            } else {
                                stale = true;  // slot taken by another column: re-read the chunk
                            }
                        }
                        if (state[b] != kUnresolved) {
                            gid[b] = slot_gid(L, c, pos);
                            word[b] = meta + 2 + pos;
                        }
                    }
                }
                all &= state[b] != kUnresolved;
            }
            if (all) break;
            if (stale || !full) continue;  // same chunk, fresh view
            c = next_chunk(L, c, spare);
            if (c < 0) break;  // pool overflow: status raised, the rest of the row is dropped
        }
        // Claimed slots: store values, fence, publish. Found slots: atomicAdd.
        bool claimed = false;
#pragma unroll
        for (int b = 0; b < NPE; b++) {
            if (state[b] == kUnresolved || state[b] == kFoundPending) continue;
            double* p = L.vals + (size_t)gid[b] * 4;
            const double v0 = block_entry<NPE>(kb, a, b, 0), v1 = block_entry<NPE>(kb, a, b, 1);
            const double v2 = block_entry<NPE>(kb, a, b, 2), v3 = block_entry<NPE>(kb, a, b, 3);
            if (state[b] == kClaimed) {
                reinterpret_cast<double2*>(p)[0] = make_double2(v0, v1);
                reinterpret_cast<double2*>(p)[1] = make_double2(v2, v3);
                claimed = true;
            } else {
                atomicAdd(p + 0, v0);
                atomicAdd(p + 1, v1);
                atomicAdd(p + 2, v2);
                atomicAdd(p + 3, v3);
            }
        }
        if (claimed) {
            __threadfence();
#pragma unroll
            for (int b = 0; b < NPE; b++)
                if (state[b] == kClaimed) atomicExch(word[b], nodes[b] + 1);
        }
        // Columns another thread is still writing: wait for them, then add.
#pragma unroll
        for (int b = 0; b < NPE; b++) {
            if (state[b] != kFoundPending) continue;
            if (!wait_published(L, word[b])) continue;
            double* p = L.vals + (size_t)gid[b] * 4;
#pragma unroll
            for (int v = 0; v < 4; v++) atomicAdd(p + v, block_entry<NPE>(kb, a, b, v));
        }
    }
}

template <int NPE>
__global__ void __launch_bounds__(128) k_scatter_2d(MeshView m, ListLayout L, const int* __restrict__ elist,
                                                   const int* __restrict__ ecount) {
    const int count = ecount ? *ecount : m.E_count;
    int spare = -1;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const int e = elist ? __ldg(elist + i) : i;
        scatter_element_2d<NPE>(m, L, e, spare);
    }
}

// Splits a mixed mesh into Q4 and T3 element lists (warp-aggregated appends).
__global__ void k_partition_2d(MeshView m, int* __restrict__ list_q4, int* __restrict__ list_t3,
                               int* __restrict__ counts) {
    const int lane = threadIdx.x & 31;
    for (int base = (blockIdx.x * blockDim.x + threadIdx.x) & ~31; base < m.E_count;
         base += gridDim.x * blockDim.x) {
        const int e = base + lane;
        const bool valid = e < m.E_count;
        const bool q4 = valid && __ldg(m.types + e) == FEM_Q4;
        const bool t3 = valid && !q4;
        const unsigned mq = __ballot_sync(0xFFFFFFFFu, q4), mt = __ballot_sync(0xFFFFFFFFu, t3);
        int bq = 0, bt = 0;
        if (lane == 0) {
            if (mq) bq = atomicAdd(counts + 0, __popc(mq));
            if (mt) bt = atomicAdd(counts + 1, __popc(mt));
        }
        bq = __shfl_sync(0xFFFFFFFFu, bq, 0);
        bt = __shfl_sync(0xFFFFFFFFu, bt, 0);
        const unsigned below = (1u << lane) - 1u;
        if (q4) list_q4[bq + __popc(mq & below)] = e;
        if (t3) list_t3[bt + __popc(mt & below)] = e;
    }
}

int sm_count() {
    static int n = 0;
    if (!n) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (n <= 0) n = 148;
    }
    return n;
}

}  // namespace

cudaError_t launch_scatter_2d(const MeshView& m, const ListLayout& L, int npe, const int* elist,
                              const int* ecount, cudaStream_t s) {
    const int threads = 128;
    long long want = ((long long)m.E_count + threads - 1) / threads;
    int grid = (int)(want < (long long)sm_count() * 64 ? (want > 0 ? want : 1) : (long long)sm_count() * 64);
    if (npe == 4)
        k_scatter_2d<4><<<grid, threads, 0, s>>>(m, L, elist, ecount);
    else
        k_scatter_2d<3><<<grid, threads, 0, s>>>(m, L, elist, ecount);
    return cudaGetLastError();
}

cudaError_t launch_partition_2d(const MeshView& m, int* list_q4, int* list_t3, int* counts, cudaStream_t s) {
    cudaError_t err = cudaMemsetAsync(counts, 0, 2 * sizeof(int), s);
    if (err) return err;
    const int threads = 256;
    long long want = ((long long)m.E_count + threads - 1) / threads;
    int grid = (int)(want < (long long)sm_count() * 16 ? (want > 0 ? want : 1) : (long long)sm_count() * 16);
    k_partition_2d<<<grid, threads, 0, s>>>(m, list_q4, list_t3, counts);
    return cudaGetLastError();
}

}  // namespace fem
