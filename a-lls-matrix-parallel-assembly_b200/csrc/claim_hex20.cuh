// Device code of the Hex20 claim pass (claim_hex20.cu), shared with the
// batched persistent kernel (batched.cu). See claim_hex20.cu for the method.
#pragma once

#include "group_hex20.cuh"

namespace fem {
namespace {

constexpr int kClaimMaxWords = 96;  // first-chunk meta rows of at most 96 words (S1 <= 94, checked on the host)
constexpr int kViewStride = 100;    // words between the copied rows (16-byte rows, banks spread)
constexpr int kClaimRows = 96;      // row nodes whose first chunks are copied at once (a 2x2x2 brick has 81)
constexpr int kExtMax = 8;          // elements outside the group kept per node (more: its pairs count as shared)

enum : unsigned char { kCFound = 0, kCTry = 1, kCClaimed = 2, kCChain = 3, kCNone = 4 };

// Shared memory of one claiming CTA.
struct ClaimSmem {
    GroupTopo T;
    alignas(16) int view[kClaimRows][kViewStride];     // first chunks of a batch of row nodes
    int claims[kClaimRows];                            // entries claimed per row node of the batch
    int obase[kClaimRows + 1];                         // ordered pairs before each row of the batch
    unsigned char cols[kGroup * 400];                  // the batch's ordered pairs: column node of each
    int mult[kGroupPairs];                             // blocks of the group's elements on each node pair
    unsigned short tab[kGroup * 210];                  // the block table before it is written
    int ext[kGroupOcc][kExtMax];                       // node u's elements outside the group, ascending
    int inc_lo[kGroupOcc], inc_n[kGroupOcc];           // node u's incidence list (offset, length)
    int inc_base[kGroupOcc + 1];                       // flattened incidence entries before node u
    int next[kGroupOcc];                               // elements outside the group kept for u (capped)
    int gelem[kGroup];                                 // the group's elements
};

// Whether every element with both group-local nodes u and v is in the group:
// no element outside the group has both.
__device__ __forceinline__ bool pair_owned(const ClaimSmem& sm, int u, int v) {
    const int cu = min(sm.next[u], kExtMax + 1), cv = min(sm.next[v], kExtMax + 1);
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

// Walks the probe sequence of column key `key` in the first chunk of row node
// rn from step t0 on, against `view`, the chunk's copy in shared memory: a
// slot holding the key is found; the first slot empty in the copy is claimed
// with atomicCAS. The copy only ever holds what the slot truly holds: each
// CAS's outcome is written back to it (the key, or the column another claimer
// put there), so the other threads of the CTA see it. A CAS that meets another
// column moves on along the sequence: slots are never freed, so a column sits
// at the first slot of its sequence that was empty when it was inserted and is
// never inserted twice. Returns kCFound / kCClaimed with the slot, or kCChain
// when the first chunk's sequence is full.
__device__ unsigned char claim_walk(const ListLayout& L, int rn, volatile int* view, int key, int t0, int& slot) {
    const int S1 = L.S1;
    const int p0 = probe_start(key, S1);
    int* meta = L.meta1 + (size_t)rn * L.H1 + 2;
    for (int t = t0; t < S1; t++) {
        int s = p0 + t;
        if (s >= S1) s -= S1;
        const int x = view[s];
        if (x == key) {
            slot = s;
            return kCFound;
        }
        if (x != 0) continue;
        const int old = atomicCAS(meta + s, 0, key);
        view[s] = old == 0 ? key : old;
        if (old == 0 || old == key) {
            slot = s;
            return old == 0 ? kCClaimed : kCFound;
        }
    }
    return kCChain;
}

constexpr int kClaimThreads = 256;
constexpr int kClaimInFlight = 10;  // ordered pairs a thread resolves at once (a brick's 2,485: one round)

// Claim pass of the group of positions [g0, g0 + ne) of the visit order
// (perm NULL: element i). inc_off / inc: the mesh's node -> element incidence
// lists; NULL makes every pair shared (every claimed block is zeroed). rec:
// the group's record (group_hex20.cuh). Every thread of the CTA calls it.
__device__ void claim_group(const MeshView& m, const ListLayout& L, const int* __restrict__ perm,
                            const int* __restrict__ inc_off, const int* __restrict__ inc, long long g0, int ne,
                            int* __restrict__ rec, ClaimSmem& sm) {
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nwarps = nt >> 5;
    GroupTopo& T = sm.T;
    if (tid < ne) sm.gelem[tid] = perm ? FEM_LDG(perm + g0 + tid) : (int)(g0 + tid);
    group_topology(m, perm, g0, ne, T);
    if (T.bad) {
        if (tid == 0) {
            raise_status(L.info, FEM_ERR_BAD_MESH);
            rec[0] = 0;
            rec[1] = 0;
        }
        __syncthreads();
        return;
    }
    const int nu = T.nu;
    // the record: header, node ids, block table
    if (tid == 0) {
        rec[0] = T.npairs;
        rec[1] = ne;
    }
    if (tid < ne) rec[2 + tid] = sm.gelem[tid];
    for (int k = tid; k < ne * 20; k += nt) rec[kRecOcc + k] = T.occ[k];
    for (int k = tid; k < T.npairs; k += nt) sm.mult[k] = 0;
    __syncthreads();
    for (int k = tid; k < ne * 210; k += nt) {
        const int w = k / 210, p = k - 210 * w;
        int I = 0;
        while (I < 19 && packed_block(I + 1, I + 1) <= p) I++;
        const int J = I + p - packed_block(I, I);
        const int u = T.lidx[20 * w + I], v = T.lidx[20 * w + J];
        unsigned e = u <= v ? (unsigned)pair_index(T, u, v) : ((unsigned)pair_index(T, v, u) | kTabTransposed);
        if (u == v && I != J) e |= kTabBoth;
        sm.tab[k] = (unsigned short)e;
        atomicAdd(&sm.mult[e & kTabPair], (e & kTabBoth) ? 2 : 1);
    }
    __syncthreads();
    unsigned short* tab = reinterpret_cast<unsigned short*>(rec + kRecTab);
    for (int k = tid; k < ne * 210; k += nt) {
        const unsigned e = sm.tab[k];
        tab[k] = (unsigned short)(sm.mult[e & kTabPair] == 1 ? e | kTabSole : e);
    }
    // each node's elements outside the group (at most kExtMax kept, sorted):
    // the incidence entries of all the group's nodes are read in parallel
    for (int u = tid; u < nu; u += nt) {
        sm.next[u] = inc_off ? 0 : kExtMax + 1;
        if (inc_off) {
            const int n = T.node[u];
            const int lo = FEM_LDG(inc_off + n);
            sm.inc_lo[u] = lo;
            sm.inc_n[u] = FEM_LDG(inc_off + n + 1) - lo;
        } else {
            sm.inc_n[u] = 0;
        }
    }
    __syncthreads();
    if (tid < 32) {
        int carry = 0;
        for (int u0 = 0; u0 < nu; u0 += 32) {
            const int c = u0 + lane < nu ? sm.inc_n[u0 + lane] : 0;
            int incl = c;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const int y = __shfl_up_sync(0xFFFFFFFFu, incl, d);
                if (lane >= d) incl += y;
            }
            if (u0 + lane < nu) sm.inc_base[u0 + lane] = carry + incl - c;
            carry += __shfl_sync(0xFFFFFFFFu, incl, 31);
        }
        if (lane == 0) sm.inc_base[nu] = carry;
    }
    __syncthreads();
    for (int q = tid; q < sm.inc_base[nu]; q += nt) {
        int lo = 0, hi = nu - 1;  // the last node whose first entry is <= q
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (sm.inc_base[mid] <= q) lo = mid;
            else hi = mid - 1;
        }
        const int e = FEM_LDG(inc + sm.inc_lo[lo] + q - sm.inc_base[lo]);
        bool in = false;
        for (int w = 0; w < ne; w++) in |= sm.gelem[w] == e;
        if (!in) {
            const int k = atomicAdd(&sm.next[lo], 1);
            if (k < kExtMax) sm.ext[lo][k] = e;
        }
    }
    __syncthreads();
    for (int u = tid; u < nu; u += nt) {
        const int c = min(sm.next[u], kExtMax);
        for (int i = 1; i < c; i++) {
            const int e = sm.ext[u][i];
            int p = i;
            while (p > 0 && sm.ext[u][p - 1] > e) {
                sm.ext[u][p] = sm.ext[u][p - 1];
                p--;
            }
            sm.ext[u][p] = e;
        }
    }
    unsigned* map = reinterpret_cast<unsigned*>(rec + kRecMap);
    int spare = -1;
    const int S1 = L.S1;
    for (int rb = 0; rb < nu; rb += kClaimRows) {
        const int nrows = min(kClaimRows, nu - rb);
        // the batch's first chunks, H1 / 4 16-byte pieces each
        const int pieces = L.H1 >> 2;
        for (int q = tid; q < nrows * pieces; q += nt) {
            const int r = q / pieces, k = q - r * pieces;
            cp_async16(&sm.view[r][4 * k], L.meta1 + (size_t)T.node[rb + r] * L.H1 + 4 * k);
        }
        if (tid < 32) {
            int carry = 0;
            for (int r0 = 0; r0 < nrows; r0 += 32) {
                const int r = r0 + lane;
                int c = 0;
                if (r < nrows) {
#pragma unroll
                    for (int w = 0; w < kNbWords; w++) c += __popc(T.nb[rb + r][w]);
                }
                int incl = c;
#pragma unroll
                for (int d = 1; d < 32; d <<= 1) {
                    const int y = __shfl_up_sync(0xFFFFFFFFu, incl, d);
                    if (lane >= d) incl += y;
                }
                if (r < nrows) {
                    sm.obase[r] = carry + incl - c;
                    sm.claims[r] = 0;
                }
                carry += __shfl_sync(0xFFFFFFFFu, incl, 31);
            }
            if (lane == 0) sm.obase[nrows] = carry;
        }
        __syncthreads();
        // the batch's ordered pairs as a flat list of column nodes, row by row
        for (int r = warp; r < nrows; r += nwarps) {
            int base = sm.obase[r];
#pragma unroll
            for (int w = 0; w < kNbWords; w++) {
                const unsigned bits = T.nb[rb + r][w];
                if ((bits >> lane) & 1u) sm.cols[base + __popc(bits & ((1u << lane) - 1u))] = (unsigned char)(32 * w + lane);
                base += __popc(bits);
            }
        }
        cp_async_wait_all();
        __syncthreads();
        const int total = sm.obase[nrows];
        for (int f0 = tid; f0 < total; f0 += nt * kClaimInFlight) {
            int row[kClaimInFlight], col[kClaimInFlight], slot[kClaimInFlight], old[kClaimInFlight], gids[kClaimInFlight];
            unsigned char st[kClaimInFlight];
            // probe the copies
#pragma unroll
            for (int j = 0; j < kClaimInFlight; j++) {
                const int f = f0 + j * nt;
                st[j] = kCNone;
                row[j] = 0;
                col[j] = 0;
                slot[j] = 0;
                if (f < total) {
                    int lo = 0, hi = nrows - 1;  // the last row whose first pair is <= f
                    while (lo < hi) {
                        const int mid = (lo + hi + 1) >> 1;
                        if (sm.obase[mid] <= f) lo = mid;
                        else hi = mid - 1;
                    }
                    row[j] = lo;
                    col[j] = sm.cols[f];
                    const int key = T.node[col[j]] + 1;
                    const volatile int* v = sm.view[lo] + 2;
                    const int p0 = probe_start(key, S1);
                    st[j] = kCChain;
                    for (int t = 0; t < S1; t++) {
                        int s = p0 + t;
                        if (s >= S1) s -= S1;
                        const int x = v[s];
                        if (x == key || x == 0) {
                            st[j] = x == key ? kCFound : kCTry;
                            slot[j] = x == key ? s : t;  // kCTry: the step of the sequence
                            break;
                        }
                    }
                }
            }
            // the claims in flight at once
#pragma unroll
            for (int j = 0; j < kClaimInFlight; j++) {
                old[j] = 0;
                if (st[j] == kCTry) {
                    const int key = T.node[col[j]] + 1;
                    int s = probe_start(key, S1) + slot[j];
                    if (s >= S1) s -= S1;
                    old[j] = atomicCAS(L.meta1 + (size_t)T.node[rb + row[j]] * L.H1 + 2 + s, 0, key);
                    sm.view[row[j]][2 + s] = old[j] == 0 ? key : old[j];
                }
            }
#pragma unroll
            for (int j = 0; j < kClaimInFlight; j++) {
                if (st[j] == kCNone) continue;
                const int r = row[j], u = rb + r, v = col[j];
                const int rn = T.node[u], key = T.node[v] + 1;
                int gid = -1;
                if (st[j] == kCTry) {
                    const int t = slot[j];
                    int s = probe_start(key, S1) + t;
                    if (s >= S1) s -= S1;
                    if (old[j] == 0 || old[j] == key) {
                        st[j] = old[j] == 0 ? kCClaimed : kCFound;
                        slot[j] = s;
                    } else {
                        st[j] = claim_walk(L, rn, sm.view[r] + 2, key, t + 1, slot[j]);
                    }
                }
                if (st[j] == kCChain) {
                    bool claimed = false;
                    gid = resolve_chain(L, rn, key, spare, claimed);
                    st[j] = claimed ? kCClaimed : kCFound;
                } else {
                    gid = (int)slot_gid(L, rn, slot[j]);
                }
                gids[j] = gid;
            }
            // the stores after every atomic of the round
#pragma unroll
            for (int j = 0; j < kClaimInFlight; j++) {
                if (st[j] == kCNone) continue;
                const int r = row[j], u = rb + r, v = col[j], gid = gids[j];
                const bool owned = pair_owned(sm, u, v);
                if (gid >= 0 && st[j] == kCClaimed) {
                    if (!owned) zero_block(L.vals + (size_t)(unsigned)gid * 9);
                    atomicAdd(&sm.claims[r], 1);
                }
                const unsigned word = gid < 0 ? kMapNone : ((unsigned)gid | (owned ? 0u : kPairShared));
                if (u <= v) {
                    const int p = pair_index(T, u, v);
                    map[2 * p] = word;
                    if (u == v) map[2 * p + 1] = kMapNone;
                } else {
                    map[2 * pair_index(T, v, u) + 1] = word;
                }
            }
        }
        __syncthreads();
        for (int r = tid; r < nrows; r += nt)
            if (sm.claims[r]) atomicAdd(L.counts + T.node[rb + r], sm.claims[r]);
        __syncthreads();  // the batch's copies and counters are free
    }
}

}  // namespace
}  // namespace fem
