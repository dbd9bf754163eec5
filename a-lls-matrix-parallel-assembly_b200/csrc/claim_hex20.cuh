// Device code of the Hex20 claim pass (claim_hex20.cu), shared with the
// batched persistent kernel (batched.cu). See claim_hex20.cu for the method.
#pragma once

#include "group_hex20.cuh"

namespace fem {
namespace {

constexpr int kClaimMaxWords = 96;  // first-chunk meta rows of at most 96 words (S1 <= 94, checked on the host)
constexpr int kClaimRows = 32;      // row nodes whose first chunks are copied at once
constexpr int kExtMax = 8;          // elements outside the group kept per node (more: its pairs count as shared)

enum : unsigned char { kCFound = 0, kCTry = 1, kCClaimed = 2, kCChain = 3 };

// Shared memory of one claiming CTA.
struct ClaimSmem {
    GroupTopo T;
    alignas(16) int view[kClaimRows][kClaimMaxWords];  // first chunks of a batch of row nodes
    int claims[kClaimRows];                            // entries claimed per row node of the batch
    int obase[kClaimRows + 1];                         // ordered pairs before each row of the batch
    int ext[kGroupOcc][kExtMax];                       // node u's elements outside the group, ascending
    unsigned char next[kGroupOcc];                     // their number (kExtMax + 1: more than kExtMax)
    int gelem[kGroup];                                 // the group's elements
};

// Whether every element with both group-local nodes u and v is in the group:
// no element outside the group has both.
__device__ __forceinline__ bool pair_owned(const ClaimSmem& sm, int u, int v) {
    const int cu = sm.next[u], cv = sm.next[v];
    if (cu == 0 || cv == 0) return true;
    if (cu > kExtMax || cv > kExtMax) return false;
    int i = 0, j = 0;
    while (i < cu && j < cv) {
        const int a = sm.ext[u][i], b = sm.ext[v][j];
        if (a == b) return false;
        if (a < b) i++;
        else j++;
    }
    return true;
}

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

// Finds or claims column key `key` in the first chunk of row node rn, whose
// copy (taken at the start of the batch) is `view`: the key's probe sequence
// in the copy; the first slot empty in the copy is claimed with atomicCAS.
// A CAS that meets another column moves on along the sequence: slots are
// never freed, so a column sits at the first slot of its sequence that was
// empty when it was inserted and is never inserted twice. Returns the slot
// (state kCFound / kCClaimed) or kCChain when the first chunk's sequence is
// full.
__device__ __forceinline__ unsigned char claim_first_chunk(const ListLayout& L, int rn, const int* view, int key,
                                                           int& slot) {
    const int S1 = L.S1;
    const int p0 = probe_start(key, S1);
    int* meta = L.meta1 + (size_t)rn * L.H1 + 2;
    const int* v = view + 2;
    for (int t = 0; t < S1; t++) {
        int s = p0 + t;
        if (s >= S1) s -= S1;
        const int x = v[s];
        if (x == key) {
            slot = s;
            return kCFound;
        }
        if (x != 0) continue;
        const int old = atomicCAS(meta + s, 0, key);
        if (old == 0) {
            slot = s;
            return kCClaimed;
        }
        if (old == key) {
            slot = s;
            return kCFound;
        }
    }
    return kCChain;
}

// Claim pass of the group of positions [g0, g0 + ne) of the visit order
// (perm NULL: element i). inc_off / inc: the mesh's node -> element incidence
// lists; NULL makes every pair shared (every claimed block is zeroed). rec:
// the group's map record. Every thread of the CTA calls it.
__device__ void claim_group(const MeshView& m, const ListLayout& L, const int* __restrict__ perm,
                            const int* __restrict__ inc_off, const int* __restrict__ inc, long long g0, int ne,
                            unsigned* __restrict__ rec, ClaimSmem& sm) {
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31;
    GroupTopo& T = sm.T;
    if (tid < ne) sm.gelem[tid] = perm ? FEM_LDG(perm + g0 + tid) : (int)(g0 + tid);
    group_topology(m, perm, g0, ne, T);
    if (T.bad) {
        if (tid == 0) raise_status(L.info, FEM_ERR_BAD_MESH);
        __syncthreads();
        return;
    }
    const int nu = T.nu;
    // each node's elements outside the group (sorted, at most kExtMax kept)
    for (int u = tid; u < nu; u += nt) {
        int c = kExtMax + 1;
        if (inc_off) {
            const int n = T.node[u];
            const int o1 = FEM_LDG(inc_off + n + 1);
            c = 0;
            for (int k = FEM_LDG(inc_off + n); k < o1; k++) {
                const int e = FEM_LDG(inc + k);
                bool in = false;
                for (int w = 0; w < ne; w++) in |= sm.gelem[w] == e;
                if (in) continue;
                if (c < kExtMax) {
                    int p = c;
                    while (p > 0 && sm.ext[u][p - 1] > e) {
                        sm.ext[u][p] = sm.ext[u][p - 1];
                        p--;
                    }
                    sm.ext[u][p] = e;
                }
                c++;
            }
            c = min(c, kExtMax + 1);
        }
        sm.next[u] = (unsigned char)c;
    }
    int spare = -1;
    for (int rb = 0; rb < nu; rb += kClaimRows) {
        const int nrows = min(kClaimRows, nu - rb);
        // the batch's first chunks, H1 / 4 16-byte pieces each
        const int pieces = L.H1 >> 2;
        for (int q = tid; q < nrows * pieces; q += nt) {
            const int r = q / pieces, k = q - r * pieces;
            cp_async16(&sm.view[r][4 * k], L.meta1 + (size_t)T.node[rb + r] * L.H1 + 4 * k);
        }
        if (tid < 32) {
            int c = 0;
            if (lane < nrows) {
#pragma unroll
                for (int w = 0; w < kNbWords; w++) c += __popc(T.nb[rb + lane][w]);
            }
            int incl = c;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const int y = __shfl_up_sync(0xFFFFFFFFu, incl, d);
                if (lane >= d) incl += y;
            }
            if (lane < nrows) {
                sm.obase[lane] = incl - c;
                sm.claims[lane] = 0;
            }
            if (lane == nrows - 1) sm.obase[nrows] = incl;
        }
        cp_async_wait_all();
        __syncthreads();
        const int total = sm.obase[nrows];
        for (int f = tid; f < total; f += nt) {
            int lo = 0, hi = nrows - 1;  // the last row whose first pair is <= f
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (sm.obase[mid] <= f) lo = mid;
                else hi = mid - 1;
            }
            const int r = lo, u = rb + r;
            const int v = nb_member(T, u, f - sm.obase[r]);
            const int rn = T.node[u], key = T.node[v] + 1;
            int slot = -1;
            unsigned char st = claim_first_chunk(L, rn, sm.view[r], key, slot);
            int gid;
            if (st == kCChain) {
                bool claimed = false;
                gid = resolve_chain(L, rn, key, spare, claimed);
                st = claimed ? kCClaimed : kCFound;
            } else {
                gid = (int)slot_gid(L, rn, slot);
            }
            const bool owned = pair_owned(sm, u, v);
            if (gid >= 0 && st == kCClaimed) {
                if (!owned) zero_block(L.vals + (size_t)(unsigned)gid * 9);
                atomicAdd(&sm.claims[r], 1);
            }
            const unsigned word = gid < 0 ? kMapNone : ((unsigned)gid | (owned ? 0u : kPairShared));
            if (u <= v) {
                const int p = pair_index(T, u, v);
                rec[2 * p] = word;
                if (u == v) rec[2 * p + 1] = kMapNone;
            } else {
                rec[2 * pair_index(T, v, u) + 1] = word;
            }
        }
        __syncthreads();
        if (tid < nrows && sm.claims[tid]) atomicAdd(L.counts + T.node[rb + tid], sm.claims[tid]);
        __syncthreads();  // the batch's copies and counters are free
    }
}

}  // namespace
}  // namespace fem
