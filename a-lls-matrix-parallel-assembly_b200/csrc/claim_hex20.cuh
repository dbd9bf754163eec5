// Device code of the Hex20 claim pass (claim_hex20.cu), shared with the
// batched persistent kernel (batched.cu). See claim_hex20.cu for the method.
#pragma once

#include <cooperative_groups.h>

#include "group_hex20.cuh"

namespace fem {
namespace {

namespace cg = cooperative_groups;

constexpr int kClaimMaxWords = 96;  // first-chunk meta rows of at most 96 words (S1 <= 94, checked on the host)
constexpr int kViewStride = 100;    // words between the copied rows (16-byte rows, banks spread)
constexpr int kClaimRows = 96;      // row nodes whose first chunks are copied at once (a 2x2x2 brick has 81)
constexpr int kOutBits = 64;        // elements outside the group that get a bit of the ownership masks
constexpr int kOutTable = 256;      // hash table of the outside elements

enum : unsigned char { kCFound = 0, kCTry = 1, kCClaimed = 2, kCChain = 3, kCNone = 4, kCFail = 5, kCTent = 6 };

// State of a batch pair: the probe step (0xFF: none, a full first chunk) in
// the high byte, the state in the low byte, so that of two slots found to
// hold one column the smaller word names the earlier one.
constexpr int kNoStep = 0xFF;
__device__ __forceinline__ unsigned short pair_res(int step, int state) { return (unsigned short)((step << 8) | state); }

// Key word of a slot that held a second copy of a column and was retired:
// occupied for every probe, no column for the consolidation (kColMask clears it).
constexpr int kTombKey = (int)0x80000000u;

constexpr int kPlaceIters = 8;  // placement rounds before the remaining claims walk one by one

// Shared memory of one claiming CTA. The block-table scratch and the
// incidence bounds are used before the row batches, the chunk copies and the
// pair list during them.
struct ClaimSmem {
    GroupTopo T;
    union {
        struct {
            int mult[kGroupPairs];                 // blocks of the group's elements on each node pair, then fill counters
            int cofs[kGroupPairs + 1];             // first entry of each pair's blocks
            unsigned short tab[kGroup * 210];      // each element block's pair index and orientation bits
            int inc_lo[kGroupOcc], inc_n[kGroupOcc];  // incidence list of each node
        } pre;
        struct {
            alignas(16) int view[kClaimRows][kViewStride];  // first chunks of a batch of row nodes
            unsigned pairs[kGroup * 400];          // the batch's ordered pairs: row | column << 8 | record word << 16
            unsigned short res[kGroup * 400];      // each pair's probe step << 8 | state (pair_res)
            unsigned char home[kGroup * 400];      // earliest probe step a met claim showed holding the pair's column (0xFF: none)
        } batch;
    };
    unsigned long long extm[kGroupOcc];   // node u's elements outside the group (mask bits)
    unsigned unk[kNbWords];               // nodes with an outside element that has no mask bit
    int okey[kOutTable];                  // outside elements (hash table, -1 empty)
    unsigned char obit[kOutTable];        // their mask bits (kOutBits: none)
    unsigned ouse[kOutTable / 32];        // occupancy of the table
    int claims[kClaimRows];               // entries claimed per row node of the batch
    int obase[kClaimRows + 1];            // ordered pairs before each row of the batch
    unsigned short pdec[210];             // packed block p -> I | J << 8
    int gelem[kGroup];                    // the group's elements
};

// Whether every element with both group-local nodes u and v is in the group:
// no element outside the group has both (the masks of their outside
// elements do not meet; a node with an unnumbered outside element only
// decides when the other node has no outside element at all).
__device__ __forceinline__ bool pair_owned(const ClaimSmem& sm, int u, int v) {
    const bool ku = (sm.unk[u >> 5] >> (u & 31)) & 1u, kv = (sm.unk[v >> 5] >> (v & 31)) & 1u;
    const unsigned long long mu = sm.extm[u], mv = sm.extm[v];
    if ((!ku && mu == 0) || (!kv && mv == 0)) return true;
    return !ku && !kv && (mu & mv) == 0;
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
__device__ __forceinline__ unsigned char claim_walk(const ListLayout& L, int rn, volatile int* view, int key, int t0,
                                                    int& slot) {
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

// Slot of probe step t of a sequence starting at p0 in a chunk of S slots.
__device__ __forceinline__ int probe_slot(int p0, int t, int S) {
    const int s = p0 + t;
    return s >= S ? s - S : s;
}

// Group-local node of node id n (-1 when the group has no such node).
__device__ __forceinline__ int local_node(const GroupTopo& T, int n) {
    int h = (int)(((unsigned)n * 2654435761u) >> 23) % (2 * kGroupOcc);
    for (int i = 0; i < 2 * kGroupOcc; i++) {
        const int k = T.hkey[h];
        if (k == n) return T.lidx[T.hfirst[h]];
        if (k == -1) return -1;
        h = h + 1 == 2 * kGroupOcc ? 0 : h + 1;
    }
    return -1;
}

// Exclusive prefix sum of f(i) for i < n into out[0..n] by the first warp.
template <typename F>
__device__ __forceinline__ void warp_scan_into(int n, int* out, F f) {
    const int lane = threadIdx.x & 31;
    int carry = 0;
    for (int i0 = 0; i0 < n; i0 += 32) {
        const int i = i0 + lane;
        const int c = i < n ? f(i) : 0;
        int incl = c;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int y = __shfl_up_sync(0xFFFFFFFFu, incl, d);
            if (lane >= d) incl += y;
        }
        if (i < n) out[i] = carry + incl - c;
        carry += __shfl_sync(0xFFFFFFFFu, incl, 31);
    }
    if (lane == 0) out[n] = carry;
}

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
    if (tid < 20) {
        const int p0 = packed_block(tid, tid);
        for (int J = tid; J < 20; J++) sm.pdec[p0 + J - tid] = (unsigned short)(tid | (J << 8));
    }
    for (int k = tid; k < kOutTable; k += nt) sm.okey[k] = -1;
    for (int k = tid; k < kGroupOcc; k += nt) sm.extm[k] = 0ull;
    if (tid < kNbWords) sm.unk[tid] = 0u;
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
    // the record: header, node ids, then each element block's pair and orientation
    if (tid == 0) {
        rec[0] = T.npairs;
        rec[1] = ne;
    }
    if (tid < ne) rec[2 + tid] = sm.gelem[tid];
    for (int k = tid; k < ne * 20; k += nt) rec[kRecOcc + k] = T.occ[k];
    for (int k = tid; k < T.npairs; k += nt) sm.pre.mult[k] = 0;
    for (int u = tid; u < nu; u += nt) {
        if (inc_off) {
            const int n = T.node[u];
            const int lo = FEM_LDG(inc_off + n);
            sm.pre.inc_lo[u] = lo;
            sm.pre.inc_n[u] = FEM_LDG(inc_off + n + 1) - lo;
        } else {
            sm.pre.inc_n[u] = 0;
            atomicOr(&sm.unk[u >> 5], 1u << (u & 31));  // no incidence: every pair counts as shared
        }
    }
    __syncthreads();
    // the pair-major block order is read by the group value pass only; the
    // batched kernel (no incidence lists) adds element by element
    if (inc_off) {
        for (int k = tid; k < ne * 210; k += nt) {
            const int w = k / 210, d = sm.pdec[k - 210 * w], I = d & 0xFF, J = d >> 8;
            const int u = T.lidx[20 * w + I], v = T.lidx[20 * w + J];
            unsigned e = u <= v ? (unsigned)pair_index(T, u, v) : ((unsigned)pair_index(T, v, u) | kTabTransposed);
            if (u == v && I != J) e |= kTabBoth;
            sm.pre.tab[k] = (unsigned short)e;
            atomicAdd(&sm.pre.mult[e & kTabPair], 1);
        }
        __syncthreads();
        // the pair-major order of the element blocks: each pair's first position
        // (a scan of the counts), then each block's position, its pair's next free one
        if (tid < 32) warp_scan_into(T.npairs, sm.pre.cofs, [&](int r) { return sm.pre.mult[r]; });
        __syncthreads();
        unsigned short* cofs = reinterpret_cast<unsigned short*>(rec + kRecCofs);
        for (int r = tid; r <= T.npairs; r += nt) {
            cofs[r] = (unsigned short)sm.pre.cofs[r];
            if (r < T.npairs) sm.pre.mult[r] = sm.pre.cofs[r];
        }
        __syncthreads();
        unsigned short* cpos = reinterpret_cast<unsigned short*>(rec + kRecCpos);
        for (int k = tid; k < ne * 210; k += nt) {
            const unsigned e = sm.pre.tab[k];
            cpos[k] = (unsigned short)(atomicAdd(&sm.pre.mult[e & kTabPair], 1) | (e & (kTabTransposed | kTabBoth)));
        }
    }
    // ownership masks: the elements outside the group that have a node of
    // the group, numbered through a hash table (the first kOutBits get a bit)
    // (thread per node and entry rank modulo 8: no search for the entry's node)
    auto outside = [&](int u, int k) {
        const int e = FEM_LDG(inc + sm.pre.inc_lo[u] + k);
        for (int w = 0; w < ne; w++)
            if (sm.gelem[w] == e) return -1;
        return e;
    };
    auto out_slot = [&](int e) { return (int)(((unsigned)e * 2654435761u) >> 24); };
    for (int t = tid; t < nu * 8; t += nt) {
        const int u = t >> 3;
        for (int k = t & 7; k < sm.pre.inc_n[u]; k += 8) {
            const int e = outside(u, k);
            if (e < 0) continue;
            int h = out_slot(e);
            for (int i = 0; i < kOutTable; i++) {
                const int old = atomicCAS(&sm.okey[h], -1, e);
                if (old == -1 || old == e) break;
                h = (h + 1) & (kOutTable - 1);
            }
        }
    }
    __syncthreads();
    for (int s0 = warp * 32; s0 < kOutTable; s0 += nwarps * 32) {
        const unsigned b = __ballot_sync(0xFFFFFFFFu, sm.okey[s0 + lane] != -1);
        if (lane == 0) sm.ouse[s0 >> 5] = b;
    }
    __syncthreads();
    for (int s = tid; s < kOutTable; s += nt) {
        int r = __popc(sm.ouse[s >> 5] & ((1u << (s & 31)) - 1u));
        for (int w = 0; w < (s >> 5); w++) r += __popc(sm.ouse[w]);
        sm.obit[s] = (unsigned char)min(r, kOutBits);
    }
    __syncthreads();
    for (int t = tid; t < nu * 8; t += nt) {
        const int u = t >> 3;
        for (int k = t & 7; k < sm.pre.inc_n[u]; k += 8) {
            const int e = outside(u, k);
            if (e < 0) continue;
            int h = out_slot(e), b = kOutBits;
            for (int i = 0; i < kOutTable; i++) {
                if (sm.okey[h] == e) {
                    b = sm.obit[h];
                    break;
                }
                h = (h + 1) & (kOutTable - 1);
            }
            if (b < kOutBits) atomicOr(&sm.extm[u], 1ull << b);
            else atomicOr(&sm.unk[u >> 5], 1u << (u & 31));
        }
    }
    unsigned* map = reinterpret_cast<unsigned*>(rec + kRecMap);
    int spare = -1;
    const int S1 = L.S1;
    for (int rb = 0; rb < nu; rb += kClaimRows) {
        const int nrows = min(kClaimRows, nu - rb);
        __syncthreads();  // the block-table scratch (first batch) or the previous batch is free
        // the batch's first chunks, H1 / 4 16-byte pieces each
        const int pieces = L.H1 >> 2;
        for (int q = tid; q < nrows * pieces; q += nt) {
            const int r = q / pieces, k = q - r * pieces;
            cp_async16(&sm.batch.view[r][4 * k], L.meta1 + (size_t)T.node[rb + r] * L.H1 + 4 * k);
        }
        for (int r = tid; r < nrows; r += nt) sm.claims[r] = 0;
        if (tid < 32)
            warp_scan_into(nrows, sm.obase, [&](int r) {
                int c = 0;
#pragma unroll
                for (int w = 0; w < kNbWords; w++) c += __popc(T.nb[rb + r][w]);
                return c;
            });
        __syncthreads();
        // the batch's ordered pairs, row by row: column, and the record word of
        // the pair's slot (2 pair_index(u, v) for u <= v, 2 pair_index(v, u) + 1 else)
        for (int r = warp; r < nrows; r += nwarps) {
            const int u = rb + r, base = sm.obase[r], below = T.nbbelow[u];
            int cum = 0;
#pragma unroll
            for (int w = 0; w < kNbWords; w++) {
                const unsigned bits = T.nb[u][w];
                if ((bits >> lane) & 1u) {
                    const int k = cum + __popc(bits & ((1u << lane) - 1u)), v = 32 * w + lane;
                    const int word = u <= v ? 2 * (T.ubase[u] + k - below) : 2 * pair_index(T, v, u) + 1;
                    sm.batch.pairs[base + k] = (unsigned)r | ((unsigned)v << 8) | ((unsigned)word << 16);
                    sm.batch.res[base + k] = pair_res(0, kCTry);  // the first round probes from step 0
                    sm.batch.home[base + k] = 0xFF;
                }
                cum += __popc(bits);
            }
        }
        cp_async_wait_all();
        __syncthreads();
        const int total = sm.obase[nrows];
        // 1.-3. placement rounds. Each round first places every pending
        // column in the copy (shared-memory CAS: the first slot of its
        // sequence empty in the copy becomes its tentative slot, so the
        // CTA's own columns never meet in global memory), then issues all
        // tentative claims to the list at once (atomicCAS(0 -> key)), and
        // writes each outcome back to the copy, which so holds only what the
        // slots truly hold again. A claim that met another group's column
        // goes on from the next step in the next round.
        //
        // A column's tentative slot can lie beyond a slot that another of the
        // CTA's columns held tentatively. If another group put the column
        // itself there meanwhile, the claim met there reports it: the column's
        // entry is the earliest slot of its sequence known to hold it
        // (collected per pair as a byte minimum, applied after a barrier), and
        // a later slot this CTA claimed for it is retired with kTombKey. Other groups never map the
        // column to that later slot: their probes reach the earlier one first.
        for (int it = 0; it < kPlaceIters; it++) {
            int pend = 0;
            for (int f = tid; f < total; f += nt) {
                const unsigned short res = sm.batch.res[f];
                const int st = res & 0xFF;
                if (st != kCTry && st != kCFail) continue;
                const unsigned pr = sm.batch.pairs[f];
                const int r = pr & 0xFF, key = T.node[(pr >> 8) & 0xFF] + 1;
                int* v = sm.batch.view[r] + 2;
                const int p0 = probe_start(key, S1);
                unsigned short out = pair_res(kNoStep, kCChain);
                for (int t = (res >> 8) + (st == kCFail ? 1 : 0); t < S1; t++) {
                    const int s = probe_slot(p0, t, S1);
                    int x = reinterpret_cast<volatile int*>(v)[s];
                    if (x == 0) {
                        x = atomicCAS(v + s, 0, key);
                        if (x == 0) {
                            out = pair_res(t, kCTent);
                            break;
                        }
                    }
                    if (x == key) {
                        out = pair_res(t, kCFound);
                        break;
                    }
                }
                sm.batch.res[f] = out;
                pend = 1;
            }
            if (!__syncthreads_or(pend)) break;
#pragma unroll 8
            for (int f = tid; f < total; f += nt) {
                const unsigned short res = sm.batch.res[f];
                if ((res & 0xFF) != kCTent) continue;
                const unsigned pr = sm.batch.pairs[f];
                const int r = pr & 0xFF, key = T.node[(pr >> 8) & 0xFF] + 1;
                const int t = res >> 8, s = probe_slot(probe_start(key, S1), t, S1);
                const int old = atomicCAS(L.meta1 + (size_t)T.node[rb + r] * L.H1 + 2 + s, 0, key);
                if (old != 0 && old != key) sm.batch.view[r][2 + s] = old;
                sm.batch.res[f] = pair_res(t, old == 0 ? kCClaimed : (old == key ? kCFound : kCFail));
            }
            __syncthreads();
            // claims that met a column of this group's row: the earliest step
            // at which a slot is known to hold it (a byte minimum), ...
            int met = 0;
            for (int f = tid; f < total; f += nt) {
                const unsigned short res = sm.batch.res[f];
                if ((res & 0xFF) != kCFail) continue;
                const unsigned pr = sm.batch.pairs[f];
                const int r = pr & 0xFF, u = rb + r, key = T.node[(pr >> 8) & 0xFF] + 1;
                const int w = sm.batch.view[r][2 + probe_slot(probe_start(key, S1), res >> 8, S1)];
                if (w <= 0) continue;  // a retired slot
                const int vw = local_node(T, w - 1);
                if (vw < 0 || !((T.nb[u][vw >> 5] >> (vw & 31)) & 1u)) continue;
                const int fw = sm.obase[r] + T.nbpre[u][vw >> 5] + __popc(T.nb[u][vw >> 5] & ((1u << (vw & 31)) - 1u));
                int tw = probe_slot(probe_start(key, S1), res >> 8, S1) - probe_start(w, S1);
                if (tw < 0) tw += S1;
                unsigned* word = reinterpret_cast<unsigned*>(&sm.batch.home[fw & ~3]);
                const int sh = (fw & 3) * 8;
                unsigned cur = *reinterpret_cast<volatile unsigned*>(word);
                while (((cur >> sh) & 0xFFu) > (unsigned)tw) {
                    const unsigned seen = atomicCAS(word, cur, (cur & ~(0xFFu << sh)) | ((unsigned)tw << sh));
                    if (seen == cur) break;
                    cur = seen;
                }
                met = 1;
            }
            if (!__syncthreads_or(met)) continue;
            // ... which becomes the pair's entry unless it already has an
            // earlier one or its next probe step comes first; a slot this CTA
            // claimed later in the sequence is retired
            for (int f = tid; f < total; f += nt) {
                const int h = sm.batch.home[f];
                if (h == 0xFF) continue;
                sm.batch.home[f] = 0xFF;
                const unsigned short res = sm.batch.res[f];
                const int st = res & 0xFF, t = res >> 8;
                if (st == kCFail ? t < h : (st != kCChain && t <= h)) continue;
                sm.batch.res[f] = pair_res(h, kCFound);
                if (st == kCClaimed) {
                    const unsigned pr = sm.batch.pairs[f];
                    const int r = pr & 0xFF, key = T.node[(pr >> 8) & 0xFF] + 1;
                    const int so = probe_slot(probe_start(key, S1), t, S1);
                    atomicExch(L.meta1 + (size_t)T.node[rb + r] * L.H1 + 2 + so, kTombKey);
                    sm.batch.view[r][2 + so] = kTombKey;
                }
            }
            __syncthreads();
        }
        // 4. what the rounds left (claim by claim), overflow chains, then the stores
        for (int f = tid; f < total; f += nt) {
            const unsigned pr = sm.batch.pairs[f];
            const int r = pr & 0xFF, v = (pr >> 8) & 0xFF, word_idx = pr >> 16, u = rb + r;
            const int rn = T.node[u], key = T.node[v] + 1;
            const unsigned res = sm.batch.res[f];
            unsigned char st = (unsigned char)(res & 0xFF);
            int slot = st == kCChain ? 0 : probe_slot(probe_start(key, S1), res >> 8, S1);
            if (st == kCFail) st = claim_walk(L, rn, sm.batch.view[r] + 2, key, (res >> 8) + 1, slot);
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
                // one count per row among the lanes claiming together
                const cg::coalesced_group claimers = cg::coalesced_threads();
                const cg::coalesced_group row = cg::labeled_partition(claimers, r);
                if (row.thread_rank() == 0) atomicAdd(&sm.claims[r], (int)row.size());
            }
            map[word_idx] = gid < 0 ? kMapNone : ((unsigned)gid | (owned ? 0u : kPairShared));
            if (u == v) map[word_idx + 1] = kMapNone;
        }
        __syncthreads();
        for (int r = tid; r < nrows; r += nt)
            if (sm.claims[r]) atomicAdd(L.counts + T.node[rb + r], sm.claims[r]);
    }
    __syncthreads();  // the shared memory is free for the next group
}

}  // namespace
}  // namespace fem
