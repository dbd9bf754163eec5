// Device code of the 2-D A-LLS scatter (scatter2d.cu), shared with the
// batched persistent kernel (batched.cu). See scatter2d.cu for the method.
#pragma once

#include "element2d.cuh"
#include "launch.h"

namespace fem {
namespace {

enum SlotState : int { kUnresolved = 0, kFound = 1, kClaimed = 3, kSkip = 4 };
constexpr int kMask14 = (1 << k2DSlots) - 1;
constexpr int kThreads2D = 256;
constexpr int kWarps2D = kThreads2D / 32;

__device__ __forceinline__ unsigned rot14(unsigned m, int h) {
    return ((m >> h) | (m << (k2DSlots - h))) & kMask14;
}

// Finds or claims the slot of column key `key` in the row list of node `row`.
// Returns the slot state (kFound, kClaimed, or kSkip on pool overflow); gid is
// the slot's global id.
// view: the row's first chunk, loaded by the caller (possibly some time ago:
// a stale view only costs failed CASes, never a wrong slot).
__device__ __forceinline__ int resolve_2d(const ListLayout& L, int row, int key, const int4 (&view)[4], int& spare,
                                          unsigned& gid) {
    int c = row;
    for (int step = 0; step < kMaxChainSteps; step++) {
        int* meta = chunk_meta(L, c);
        int4 w0 = view[0], w1 = view[1], w2 = view[2], w3 = view[3];
        if (step > 0) {
            w0 = ld_cg4(meta);
            w1 = ld_cg4(meta + 4);
            w2 = ld_cg4(meta + 8);
            w3 = ld_cg4(meta + 12);
        }
        const int cols[k2DSlots] = {w0.z, w0.w, w1.x, w1.y, w1.z, w1.w, w2.x,
                                    w2.y, w2.z, w2.w, w3.x, w3.y, w3.z, w3.w};
        unsigned empty = 0, match = 0;
#pragma unroll
        for (int s = 0; s < k2DSlots; s++) {
            empty |= (cols[s] == 0 ? 1u : 0u) << s;
            match |= (cols[s] == key ? 1u : 0u) << s;
        }
        int state = kUnresolved, pos = 0;
        if (match) {
            pos = __ffs(match) - 1;
            state = kFound;
        } else {
            const int h = probe_start(key, k2DSlots);
            for (int tries = 0; tries < k2DSlots; tries++) {
                const unsigned cand = rot14(empty, h);
                if (!cand) break;  // probe sequence full in this chunk: go on in the next one
                pos = h + __ffs(cand) - 1;
                pos -= pos >= k2DSlots ? k2DSlots : 0;
                const int old = atomicCAS(meta + 2 + pos, 0, key);
                if (old == 0) {
                    state = kClaimed;
                    break;
                }
                if (old == key) {
                    state = kFound;
                    break;
                }
                empty &= ~(1u << pos);  // taken by another column meanwhile
            }
        }
        if (state != kUnresolved) {
            gid = slot_gid(L, c, pos);
            return state;
        }
        c = next_chunk<true>(L, c, spare);
        if (c < 0) return kSkip;  // pool overflow: status raised, the block is dropped
    }
    raise_status(L.info, FEM_ERR_TIMEOUT);
    return kSkip;
}

// Element id of work item `i` of this lane (valid: inside the range).
// want_type >= 0: only the elements of that type (mixed meshes without a
// type-grouped order) are taken; the others leave their lanes idle.
__device__ __forceinline__ int element_of(const MeshView& m, const int* perm, int begin, int count, long long i,
                                          bool ok, int want_type, bool& valid) {
    valid = ok && i < count;
    const int e = valid ? (perm ? FEM_LDG(perm + begin + i) : begin + (int)i) : 0;
    if (valid && want_type >= 0) valid = FEM_LDG(m.types + e) == want_type;
    return e;
}

// Resident CTAs per SM the register budget is set for (build-time tuning knobs).
#ifndef FEM_T3_MIN_CTAS
#define FEM_T3_MIN_CTAS 4
#endif
#ifndef FEM_Q4_MIN_CTAS
#define FEM_Q4_MIN_CTAS 2
#endif

// Warp-level shared memory of the 2-D scatter: the warp's blocks and slot ids,
// transposed so that each red instruction covers whole 32-byte blocks.
struct Scatter2DWarpSmem {
    double val[32][4];
    unsigned gid[32];
};

// The scatter of the elements perm[begin + i], i in [0, count) (perm NULL:
// element begin + i), by one warp among num_warps: the warp takes items
// warp_id * EPW, (warp_id + num_warps) * EPW, ... Every lane of the warp calls it.
template <int NPE, typename T>
__device__ __forceinline__ void scatter2d_warp(const MeshView& m, const ListLayout& L, const int* __restrict__ perm,
                                               int begin, int count, long long warp_id, long long num_warps,
                                               Scatter2DWarpSmem& ws, int want_type = -1) {
    constexpr int G = NPE * NPE;   // lanes per element
    constexpr int EPW = 32 / G;    // elements per warp
    constexpr unsigned kFull = 0xFFFFFFFFu;
    const int lane = threadIdx.x & 31;
    const int eslot = lane / G, sub = lane - eslot * G;
    const int a = sub / NPE, b = sub - (sub / NPE) * NPE;
    const bool lane_used = eslot < EPW;
    const unsigned row_group = ((1u << NPE) - 1u) << (eslot * G + a * NPE);
    const long long stride = num_warps * EPW;
    int spare = -1;

    // Software pipeline over this warp's work items k = 0, 1, 2, ...:
    // iteration k works on element k (nodes, coordinates and material loaded
    // during iteration k-1) while element k+1's node ids and element k+2's id
    // are in flight.
    long long base = warp_id * EPW;
    bool valid, valid1, valid2;
    int e = element_of(m, perm, begin, count, base + eslot, lane_used, want_type, valid);
    int e1 = element_of(m, perm, begin, count, base + stride + eslot, lane_used, want_type, valid1);
    int nodes[NPE], nodes1[NPE];
#pragma unroll
    for (int k = 0; k < NPE; k++) {
        nodes[k] = valid ? FEM_LDG(m.conn + (size_t)e * m.stride + k) : 0;
        nodes1[k] = valid1 ? FEM_LDG(m.conn + (size_t)e1 * m.stride + k) : 0;
    }
    int e2 = element_of(m, perm, begin, count, base + 2 * stride + eslot, lane_used, want_type, valid2);
    double xe[NPE], ye[NPE], Ee = 0.0, nue = 0.0;
    auto load_element = [&]() {
        bool bad = false;
#pragma unroll
        for (int k = 0; k < NPE; k++) bad |= (nodes[k] < 0) | (nodes[k] >= m.N);
        if (valid && bad) {
            if (sub == 0) raise_status(L.info, FEM_ERR_BAD_MESH);
            valid = false;
        }
#pragma unroll
        for (int k = 0; k < NPE; k++) {
            xe[k] = valid ? FEM_LDG(m.x + nodes[k]) : 0.0;
            ye[k] = valid ? FEM_LDG(m.y + nodes[k]) : 0.0;
        }
        Ee = !valid ? 0.0 : (m.E ? FEM_LDG(m.E + e) : m.E0);
        nue = !valid ? 0.0 : (m.nu ? FEM_LDG(m.nu + e) : m.nu0);
    };
    load_element();

    for (; base < count; base += stride) {
        int row = nodes[0], col = nodes[0];
#pragma unroll
        for (int k = 1; k < NPE; k++) {
            row = a == k ? nodes[k] : row;
            col = b == k ? nodes[k] : col;
        }
        int4 view[4] = {make_int4(0, 0, 0, 0), make_int4(0, 0, 0, 0), make_int4(0, 0, 0, 0), make_int4(0, 0, 0, 0)};
        if (valid) {
            const int* meta = chunk_meta(L, row);
#pragma unroll
            for (int q = 0; q < 4; q++) view[q] = ld_cg4(meta + 4 * q);
        }
        double kv[4] = {0.0, 0.0, 0.0, 0.0};
        int state = kSkip;
        unsigned gid = 0;
        if (valid) {
            const double det = ke_block_2d<NPE, T>(xe, ye, Ee, nue, m.t, a, b, kv);
            if (sub == 0 && !(det > 0.0)) raise_status(L.info, FEM_ERR_DETJ);
            state = resolve_2d(L, row, col + 1, view, spare, gid);
        }
        // claims of each (element, row) group: one counter atomic per group
        const unsigned claimed = __ballot_sync(kFull, state == kClaimed);
        if (valid && b == 0 && (claimed & row_group)) atomicAdd(L.counts + row, __popc(claimed & row_group));
        // every block (claimed or found) is added to its zero-initialised slot
        // with red.add, four consecutive lanes per block
        ws.gid[lane] = state != kSkip ? gid : 0xFFFFFFFFu;
        ws.val[lane][0] = kv[0];
        ws.val[lane][1] = kv[1];
        ws.val[lane][2] = kv[2];
        ws.val[lane][3] = kv[3];
        __syncwarp();
#pragma unroll
        for (int r = 0; r < 4; r++) {
            const int src = 8 * r + (lane >> 2), v = lane & 3;
            const unsigned g = ws.gid[src];
            if (g != 0xFFFFFFFFu) atomicAdd(L.vals + (size_t)g * 4 + v, ws.val[src][v]);
        }
        __syncwarp();
        // advance the pipeline
        e = e1;
        valid = valid1;
#pragma unroll
        for (int k = 0; k < NPE; k++) nodes[k] = nodes1[k];
        e1 = e2;
        valid1 = valid2;
#pragma unroll
        for (int k = 0; k < NPE; k++) nodes1[k] = valid1 ? FEM_LDG(m.conn + (size_t)e1 * m.stride + k) : 0;
        e2 = element_of(m, perm, begin, count, base + 3 * stride + eslot, lane_used, want_type, valid2);
        load_element();
    }
}

}  // namespace
}  // namespace fem
