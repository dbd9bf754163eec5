// Device code of the Hex20 claim pass (claim_hex20.cu), shared with the
// batched persistent kernel (batched.cu). See claim_hex20.cu for the method.
#pragma once

#include "launch.h"

namespace fem {
namespace {

constexpr int kClaimMaxWords = 96;   // first-chunk meta rows of at most 96 words (S1 <= 94, checked on the host)
constexpr int kPairs = 400;
constexpr int kPerLane = (kPairs + 31) / 32;  // 13

enum : unsigned char { kCFound = 0, kCTry = 1, kCClaimed = 2, kCChain = 3 };

// Shared memory of one claiming warp.
struct ClaimWarpSmem {
    alignas(16) int view[20][kClaimMaxWords];  // first chunks of the element's 20 row nodes
    int node[20];
    int claims[20];                            // entries claimed per row node
};

__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Zeroes the 72-byte value block of a slot (16-byte stores where aligned).
__device__ __forceinline__ void zero_block(double* v) {
    if ((reinterpret_cast<uintptr_t>(v) & 15) == 0) {
        double2* q = reinterpret_cast<double2*>(v);
        q[0] = q[1] = q[2] = q[3] = make_double2(0.0, 0.0);
        v[8] = 0.0;
    } else {
        v[0] = 0.0;
        double2* q = reinterpret_cast<double2*>(v + 1);
        q[0] = q[1] = q[2] = q[3] = make_double2(0.0, 0.0);
    }
}

// Resolves `key` in the overflow chunks of row node n (global memory, after
// the first chunk was found full). Returns the slot id, sets `claimed`; -1 on
// pool overflow or when the chain bound is hit (status raised).
__device__ int resolve_chain(const ListLayout& L, int n, int key, int& spare, bool& claimed) {
    claimed = false;
    int c = n;
    for (int step = 0; step < kMaxChainSteps; step++) {
        c = next_chunk(L, c, spare);
        if (c < 0) return -1;  // pool overflow, raised by alloc_chunk
        int* meta = chunk_meta(L, c);
        const int S = chunk_cap(L, c);
        const int p0 = probe_start(key, S);
        for (int t = 0; t < S; t++) {
            int s = p0 + t;
            if (s >= S) s -= S;
            int v = ld_cg(meta + 2 + s);
            if (v == 0) {
                v = atomicCAS(meta + 2 + s, 0, key);
                if (v == 0) {
                    claimed = true;
                    return (int)slot_gid(L, c, s);
                }
            }
            if (v == key) return (int)slot_gid(L, c, s);
        }
    }
    raise_status(L.info, FEM_ERR_TIMEOUT);
    return -1;
}

// Claims of the elements at positions i = i_first, i_first + i_stride, ...
// below i1 of the visit order perm (perm NULL: element i), by one warp; the
// slot ids of position i go to map row i - map_origin. Every lane of the
// warp calls it.
__device__ __forceinline__ void claim_warp(const MeshView& m, const ListLayout& L, const int* __restrict__ perm,
                                           long long i_first, long long i_stride, int i1, int map_origin,
                                           int* __restrict__ map, ClaimWarpSmem& ws) {
    const int lane = threadIdx.x & 31;
    const int S1 = L.S1, H1 = L.H1;
    int spare = -1;
    int (*view)[kClaimMaxWords] = ws.view;
    for (long long ii = i_first; ii < i1; ii += i_stride) {
        const int i = (int)ii;
        const int e = perm ? FEM_LDG(perm + i) : i;
        int n = 0;
        if (lane < 20) n = FEM_LDG(m.conn + (size_t)e * 20 + lane);
        const bool bad = __any_sync(0xFFFFFFFFu, lane < 20 && (n < 0 || n >= m.N));
        int* out = map + (size_t)(i - map_origin) * kPairs;
        if (bad) {
            if (lane == 0) raise_status(L.info, FEM_ERR_BAD_MESH);
            for (int p = lane; p < kPairs; p += 32) out[p] = -1;
            continue;
        }
        if (lane < 20) {
            ws.node[lane] = n;
            ws.claims[lane] = 0;
        }
        __syncwarp();
        // the 20 first chunks, H1 / 4 16-byte pieces each
        const int pieces = H1 >> 2;
        for (int q = lane; q < 20 * pieces; q += 32) {
            const int I = q / pieces, k = q - I * pieces;
            cp_async16(&view[I][4 * k], L.meta1 + (size_t)ws.node[I] * H1 + 4 * k);
        }
        cp_async_wait_all();
        __syncwarp();
        // resolve this lane's pairs p = lane + 32 k: row I = p / 20, column J = p % 20
        int slot[kPerLane];
        unsigned char st[kPerLane];
#pragma unroll
        for (int k = 0; k < kPerLane; k++) {
            const int p = lane + 32 * k;
            st[k] = kCFound;
            slot[k] = -1;
            if (p < kPairs) {
                const int I = p / 20, J = p - 20 * I;
                const int key = ws.node[J] + 1;
                const int* v = view[I] + 2;
                const int p0 = probe_start(key, S1);
                st[k] = kCChain;
                for (int t = 0; t < S1; t++) {
                    int s = p0 + t;
                    if (s >= S1) s -= S1;
                    const int x = v[s];
                    if (x == key) {
                        st[k] = kCFound;
                        slot[k] = s;
                        break;
                    }
                    if (x == 0) {
                        st[k] = kCTry;
                        slot[k] = s;
                        break;
                    }
                }
            }
        }
        // all claims of the lane in flight at once
        int old[kPerLane];
#pragma unroll
        for (int k = 0; k < kPerLane; k++) {
            old[k] = 0;
            if (st[k] == kCTry) {
                const int p = lane + 32 * k, I = p / 20, J = p - 20 * I;
                old[k] = atomicCAS(L.meta1 + (size_t)ws.node[I] * H1 + 2 + slot[k], 0, ws.node[J] + 1);
            }
        }
#pragma unroll
        for (int k = 0; k < kPerLane; k++) {
            if (st[k] != kCTry) continue;
            const int p = lane + 32 * k, I = p / 20, J = p - 20 * I;
            const int key = ws.node[J] + 1;
            const int p0 = probe_start(key, S1);
            int* meta = L.meta1 + (size_t)ws.node[I] * H1 + 2;
            int s = slot[k], x = old[k];
            st[k] = kCChain;
            // walk on from the contested slot: slots non-empty in the copy stay
            // non-empty, so only its empty ones are candidates
            for (int t = 0; t < S1; t++) {
                if (x == 0) {
                    st[k] = kCClaimed;
                    break;
                }
                if (x == key) {
                    st[k] = kCFound;
                    break;
                }
                int u = -1;
                for (int r = 1; r < S1; r++) {
                    int s2 = s + r;
                    if (s2 >= S1) s2 -= S1;
                    if (s2 == p0) break;  // wrapped around the sequence
                    const int y = view[I][2 + s2];
                    if (y == key) {
                        u = s2;
                        x = key;
                        break;
                    }
                    if (y == 0) {
                        u = s2;
                        x = atomicCAS(meta + s2, 0, key);
                        break;
                    }
                }
                if (u < 0) break;  // no empty slot left on the sequence: overflow chunks
                s = u;
            }
            slot[k] = s;
        }
        // global slot ids; overflow chunks for rows whose first chunk is full
#pragma unroll
        for (int k = 0; k < kPerLane; k++) {
            const int p = lane + 32 * k;
            if (p >= kPairs) continue;
            const int I = p / 20, J = p - 20 * I;
            const int rn = ws.node[I];
            int gid;
            if (st[k] == kCChain) {
                bool claimed = false;
                gid = resolve_chain(L, rn, ws.node[J] + 1, spare, claimed);
                if (claimed) st[k] = kCClaimed;
            } else {
                gid = (int)slot_gid(L, rn, slot[k]);
            }
            if (st[k] == kCClaimed && gid >= 0) {
                // values are kept for upper blocks only (row node <= column node)
                if (rn <= ws.node[J]) zero_block(L.vals + (size_t)(unsigned)gid * 9);
                atomicAdd(&ws.claims[I], 1);
            }
            out[p] = gid;
        }
        __syncwarp();
        if (lane < 20 && ws.claims[lane]) atomicAdd(L.counts + ws.node[lane], ws.claims[lane]);
        __syncwarp();
    }
}

}  // namespace
}  // namespace fem
