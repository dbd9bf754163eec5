// Internal definitions shared by the kernels and the C ABI of the assembler.
//
// Row lists ("A-LLS" lists, after the reference's ALLSNode pool,
// ALLS_Quad2D_Assembly_Accuracy_Analysis.cu:63-67,384-391) live in a device
// pool of fixed-size chunks. Every node n owns chunk n (its "first chunk");
// further chunks come from an overflow pool through an atomic bump counter and
// are linked with atomicCAS on the previous chunk's `next` word. A list entry
// (slot) holds one column NODE and the dof_per_node^2 block of values of that
// (row node, column node) pair, so the dpn rows of a node share one list.
//
// Chunk metadata is a row of H = S + 2 int32 words:
//     word 0 = reserved (0)
//     word 1 = next  (chunk id + 1 of the next chunk, 0 = none)
//     word 2+s = slot s: 0 = empty, col+1 = column node col
// Within a chunk a column's slot is found by open addressing (linear probing
// from a hash of the column); a chunk with no free slot on the probe sequence
// continues in the next chunk. A slot is claimed by atomicCAS(0 -> col+1), so
// every column appears at most once per row. Block values are never written by
// a claim: they are zero before the first addition (2-D: the value array is
// cleared with the lists; Hex20: the claimer zeroes the block in the claim
// pass, and values are added in a later launch), so no contributor ever waits
// for another.
// Slot values are stored slot-major: vals[gid * B + v], B = dpn^2, where gid is
// the global slot id (first-chunk slots first, then overflow-chunk slots), so a
// slot's block is contiguous (one 32-byte sector in 2-D, 72 bytes for Hex20).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "fem_alls.h"

namespace fem {

constexpr int kBlockThreads = 256;
constexpr int kScanTile = 4096;  // nodes per scan tile (256 threads x 16)

// Device-resident info word; its first bytes are laid out exactly as fem_info.
struct DevInfo {
    long long nnz;
    long long list_entries;
    int status_bits;
    int overflow_chunks;   // overflow-pool bump counter (may overshoot the capacity)
    int pool_chunks;
    int max_row_entries;
    int tile_ticket;       // consolidation tile dispenser
    int pad0;
    long long pad1[3];
};
static_assert(sizeof(DevInfo) == 64, "DevInfo size");
static_assert(offsetof(DevInfo, max_row_entries) == offsetof(fem_info, max_row_entries), "fem_info layout");

struct ListLayout {
    int N;          // nodes (= first chunks)
    int S1, S2;     // slots per first / overflow chunk
    int H1, H2;     // int32 words per first / overflow chunk meta row (S + 2)
    int B;          // values per slot (dpn^2)
    int cap2;       // overflow chunk capacity
    int* meta1;     // [N * H1]
    int* meta2;     // [cap2 * H2]
    double* vals;   // [(N*S1 + cap2*S2) * B]
    int* counts;    // [N] list entries of each row node (incremented by the claimers)
    DevInfo* info;
};

// Bits of DevInfo::status_bits are 1 << FEM_ERR_*.
__device__ __forceinline__ void raise_status(DevInfo* info, int code) {
    atomicOr(&info->status_bits, 1 << code);
}

__device__ __forceinline__ int* chunk_meta(const ListLayout& L, int c) {
    return c < L.N ? L.meta1 + (size_t)c * L.H1 : L.meta2 + (size_t)(c - L.N) * L.H2;
}
__device__ __forceinline__ int chunk_cap(const ListLayout& L, int c) { return c < L.N ? L.S1 : L.S2; }
__device__ __forceinline__ unsigned slot_gid(const ListLayout& L, int c, int s) {
    return c < L.N ? (unsigned)c * (unsigned)L.S1 + (unsigned)s
                   : (unsigned)L.N * (unsigned)L.S1 + (unsigned)(c - L.N) * (unsigned)L.S2 + (unsigned)s;
}
// Chunk id and slot of a global slot id.
__device__ __forceinline__ void gid_chunk(const ListLayout& L, unsigned gid, int& c, int& s) {
    unsigned first = (unsigned)L.N * (unsigned)L.S1;
    if (gid < first) {
        c = (int)(gid / (unsigned)L.S1);
        s = (int)(gid % (unsigned)L.S1);
    } else {
        unsigned g2 = gid - first;
        c = L.N + (int)(g2 / (unsigned)L.S2);
        s = (int)(g2 % (unsigned)L.S2);
    }
}

// Loads of data that no kernel of the launch writes go through the read-only
// path. The batched persistent kernel (batched.cu), whose work items read what
// earlier items of the same launch wrote, defines FEM_LDG as an L2 load before
// it includes the kernels' device code.
#ifndef FEM_LDG
#define FEM_LDG(p) __ldg(p)
#endif

// L2-coherent loads (bypass L1: list words change under other SMs' writes).
__device__ __forceinline__ int ld_cg(const int* p) { return __ldcg(p); }
__device__ __forceinline__ int4 ld_cg4(const int* p) { return __ldcg(reinterpret_cast<const int4*>(p)); }

// Takes one chunk from the overflow pool and zeroes its meta row (and, with
// kZeroVals, its slots' values, for lists whose contributions are all
// atomic adds). Returns the chunk id, or -1 (and raises FEM_ERR_POOL_OVERFLOW)
// when the pool is empty. The caller must __threadfence() before publishing
// the chunk.
template <bool kZeroVals = false>
__device__ __forceinline__ int alloc_chunk(const ListLayout& L) {
    int k = atomicAdd(&L.info->overflow_chunks, 1);
    if (k >= L.cap2) {
        raise_status(L.info, FEM_ERR_POOL_OVERFLOW);
        return -1;
    }
    int* m = L.meta2 + (size_t)k * L.H2;
    for (int i = 0; i < L.H2; i += 4) *reinterpret_cast<int4*>(m + i) = make_int4(0, 0, 0, 0);
    if (kZeroVals) {
        double2* v = reinterpret_cast<double2*>(L.vals + (size_t)slot_gid(L, L.N + k, 0) * L.B);
        for (int i = 0; i < L.S2 * L.B / 2; i++) v[i] = make_double2(0.0, 0.0);
    }
    return L.N + k;
}

// Bound on retry loops (chunk chains, claims); hitting it raises FEM_ERR_TIMEOUT.
constexpr int kMaxChainSteps = 1 << 20;

constexpr int kColMask = 0x7FFFFFFF;

// Start of the probe sequence of column key `key` (col + 1) in a chunk of S slots.
__device__ __forceinline__ int probe_start(int key, int S) {
    return (int)__umulhi((unsigned)key * 2654435761u, (unsigned)S);
}

// Next chunk of chunk c, allocating and atomicCAS-linking a new one if there is
// none. Returns -1 on pool overflow (status raised). `spare` keeps a chunk that
// lost a link race for this thread's next allocation (-1 = none).
template <bool kZeroVals = false>
__device__ __forceinline__ int next_chunk(const ListLayout& L, int c, int& spare) {
    int* m = chunk_meta(L, c);
    int nx = ld_cg(m + 1);
    if (nx == 0) {
        int nc = spare >= 0 ? spare : alloc_chunk<kZeroVals>(L);
        spare = -1;
        if (nc < 0) return -1;
        __threadfence();  // the zeroed meta row is visible before the link
        int old = atomicCAS(m + 1, 0, nc + 1);
        if (old == 0) {
            nx = nc + 1;
        } else {
            spare = nc;
            nx = old;
        }
    }
    return nx - 1;
}

// Host-side layout description (sizes in bytes, offsets from the workspace base).
struct HostLayout {
    int kind, dpn, B, N, E;
    int S1, S2, H1, H2, cap2;
    int num_tiles;  // scan tiles of kScanTile nodes
    size_t off_info, off_meta1, off_meta2, off_vals, off_counts, off_ucounts, off_tiles, off_elist, off_inc, off_map,
        off_stage, total;
    size_t meta1_bytes;
};

}  // namespace fem
