// K1 for 2-D meshes: fused Q4 / T3 element stiffness + A-LLS row-list scatter.
//
// Replaces assembleGlobalStiffnessKernelALLS
// (ALLS_Quad2D_Assembly_Accuracy_Analysis.cu:394-468,
//  ALLS_T3_Unstructed_Elements_Assemble_Performance.cu:227-290,
//  ALLS_Q4_T3_Mixed_Elements_Assembly_Performance.cu:248-312).
//
// One thread per (element, row node) instead of one per element:
//  * elements are visited in a node-local order (reorder.cu) so the lists they
//    touch stay in L2;
//  * the thread computes its row of Ke in registers (node-block form) and reads
//    its row node's list one 64-byte chunk row at a time (next pointer and 14
//    hashed slots in four 16-byte L2 loads); every column node of the element
//    is looked up along its probe sequence and, if absent, its slot is claimed
//    with atomicCAS (empty -> col|pending) — one slot per column and row, never
//    a duplicate; a failed CAS re-reads the chunk before the next column;
//  * the claimer stores its block values with plain 16-byte stores, fences, and
//    publishes the column; found columns are accumulated with atomicAdd
//    (red.global.add.f64), after a bounded wait if the slot is still pending.
//    A thread publishes its own claims before it waits on anyone else's, so
//    no wait can be circular. Claims are counted per row node for the scan.
// The reference instead walks a pointer list per (row, col) pair and can lose a
// contribution or insert a column twice (its head-insert race, Q4A:452-463).
#include <algorithm>

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
__device__ __forceinline__ void scatter_row_2d(const MeshView& m, const ListLayout& L, int e, int a, int& spare) {
    int nodes[NPE];
    bool bad = false;
#pragma unroll
    for (int a = 0; a < NPE; a++) {
        nodes[a] = __ldg(m.conn + (size_t)e * m.stride + a);
        bad |= (nodes[a] < 0) | (nodes[a] >= m.N);
    }
    if (bad) {
        if (a == 0) raise_status(L.info, FEM_ERR_BAD_MESH);
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
    double kr[NPE][4];  // blocks K_ab of this thread's row a
    double det;
    if constexpr (NPE == 4) {
        det = ke_q4_row(xe, ye, E, nu, m.t, a, kr);
    } else {
        det = ke_t3_row(xe, ye, E, nu, m.t, a, kr);
    }
    if (a == 0 && !(det > 0.0)) raise_status(L.info, FEM_ERR_DETJ);
    int row_node = nodes[0];
#pragma unroll
    for (int i = 1; i < NPE; i++) row_node = a == i ? nodes[i] : row_node;
    {
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
        int c = row_node;
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
        // Claimed slots: store values, fence, publish — before any atomic, so the
        // fence waits only for these stores and the slots stay pending briefly.
        int nclaimed = 0;
#pragma unroll
        for (int b = 0; b < NPE; b++) nclaimed += state[b] == kClaimed;
        if (nclaimed) {
            atomicAdd(L.counts + row_node, nclaimed);
#pragma unroll
            for (int b = 0; b < NPE; b++) {
                if (state[b] != kClaimed) continue;
                double* p = L.vals + (size_t)gid[b] * 4;
                reinterpret_cast<double2*>(p)[0] = make_double2(kr[b][0], kr[b][1]);
                reinterpret_cast<double2*>(p)[1] = make_double2(kr[b][2], kr[b][3]);
            }
            __threadfence();
#pragma unroll
            for (int b = 0; b < NPE; b++)
                if (state[b] == kClaimed) atomicExch(word[b], nodes[b] + 1);
        }
        // Found (published) slots: atomicAdd.
#pragma unroll
        for (int b = 0; b < NPE; b++) {
            if (state[b] != kFound) continue;
            double* p = L.vals + (size_t)gid[b] * 4;
#pragma unroll
            for (int v = 0; v < 4; v++) atomicAdd(p + v, kr[b][v]);
        }
        // Columns another thread is still writing: wait for them, then add.
#pragma unroll
        for (int b = 0; b < NPE; b++) {
            if (state[b] != kFoundPending) continue;
            if (!wait_published(L, word[b])) continue;
            double* p = L.vals + (size_t)gid[b] * 4;
#pragma unroll
            for (int v = 0; v < 4; v++) atomicAdd(p + v, kr[b][v]);
        }
    }
}

template <int NPE>
__global__ void __launch_bounds__(256, NPE == 3 ? 3 : 2) k_scatter_2d(MeshView m, ListLayout L, const int* __restrict__ perm,
                                                   const int* __restrict__ range) {
    const int begin = range[0], count = range[1] - range[0];
    const long long work = (long long)count * NPE;
    int spare = -1;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < work;
         t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t / NPE), a = (int)(t - (long long)i * NPE);
        scatter_row_2d<NPE>(m, L, __ldg(perm + begin + i), a, spare);
    }
}

}  // namespace

cudaError_t launch_scatter_2d(const MeshView& m, const ListLayout& L, int npe, const int* perm, const int* range,
                              cudaStream_t s) {
    const int threads = 256;
    const long long want = ((long long)m.E_count * npe + threads - 1) / threads;
    const int grid = (int)std::min<long long>(want > 0 ? want : 1, (long long)sm_count() * 8);
    if (npe == 4)
        k_scatter_2d<4><<<grid, threads, 0, s>>>(m, L, perm, range);
    else
        k_scatter_2d<3><<<grid, threads, 0, s>>>(m, L, perm, range);
    return cudaGetLastError();
}

}  // namespace fem
