// Element groups of the Hex20 list scatter (claim_hex20.cuh, values_group.cuh,
// and the batched kernel).
//
// A group is kGroup consecutive positions of the spatial element order (a
// 2x2x2 brick of a structured mesh in Morton order). Its kGroup * 20 node
// occurrences name nu <= 160 distinct nodes, numbered u = 0..nu-1 in order of
// first occurrence ("group-local nodes"). Two group-local nodes are
// neighbours when some element of the group has both; node u's neighbour set
// nb[u] (u included) is a 160-bit set, and the group's node pairs {u <= v}
// (v in nb[u]) are numbered by
//     pair_index(u, v) = ubase[u] + #{v' in nb[u] : u <= v' < v},
// so pair {u, u} is ubase[u] and the pairs of u are contiguous.
//
// The claim pass resolves every ordered pair (row node u, column node v) of
// the group once, however many of the group's elements have both nodes, and
// writes the group's record (int32 words):
//   [0] number of node pairs, [1] elements (0: the group has a bad node id),
//   [2 + w] element id of the group's element w;
//   kRecOcc + 20 w + a: node id of node a of element w;
//   kRecCpos + (210 w + p) / 2: for element w's packed upper block p (I <= J,
//     p = 20 I - I (I - 1) / 2 + J - I), a 16-bit entry: the block's position
//     in the pair-major order of the group's blocks (bits 0-10), bit 15 set
//     when it lies transposed in its pair (u > v), bit 14 set when both
//     orientations fall on one diagonal block (an element with a repeated
//     node);
//   kRecCofs: 16-bit offsets, pair r's blocks take positions [cofs[r], cofs[r + 1]);
//   (these two sections are written for the group value pass only: a claim
//   without incidence lists, the batched kernel's, leaves them unset);
//   kRecMap + 2 r: slot id of (row u, column v) of pair r = {u <= v}, and
//   kRecMap + 2 r + 1: slot id of (row v, column u) (kMapNone for a diagonal
//     pair or an unresolved slot). Bit 31 (kPairShared) marks a pair that
//     elements outside the group also have: its slots are zeroed by their
//     claimer and receive atomic adds; the other pairs belong to this group
//     alone and their blocks are stored once.
#pragma once

#include "launch.h"

namespace fem {
namespace {

constexpr int kGroup = 8;                        // elements per group
constexpr int kGroupOcc = kGroup * 20;           // node occurrences of a group
constexpr int kNbWords = kGroupOcc / 32;         // words of a set of group-local nodes
constexpr int kGroupPairs = kGroup * 210;        // bound on a group's node pairs {u <= v}
constexpr int kGroupMapWords = 2 * kGroupPairs;  // map record words per group
constexpr unsigned kPairShared = 0x80000000u;    // map word flag: other groups add to the pair
constexpr unsigned kMapNone = 0xFFFFFFFFu;       // map word of no slot
constexpr int kRecOcc = 16;                                  // record words: header, then occurrences,
constexpr int kRecCpos = kRecOcc + kGroupOcc;                // block positions (two 16-bit entries a word),
constexpr int kRecCofs = kRecCpos + kGroup * 210 / 2;        // each pair's first position,
constexpr int kRecMap = kRecCofs + (kGroupPairs + 1 + 7) / 8 * 4;  // slot words
constexpr int kGroupRecWords = kRecMap + kGroupMapWords;
constexpr unsigned kTabTransposed = 0x8000u, kTabBoth = 0x4000u, kTabPair = 0x07FFu, kPosMask = 0x07FFu;
static_assert(kNbWords * 32 == kGroupOcc, "whole words of group-local nodes");
static_assert(kGroupPairs <= kTabPair + 1, "pair index in 11 bits");
static_assert(kRecCpos % 4 == 0 && kRecCofs % 4 == 0 && kRecMap % 4 == 0 && kGroupRecWords % 4 == 0, "16-byte sections");
static_assert(kGroup * 210 <= kPosMask + 1, "block position in 11 bits");
static_assert(kGroup == kHex20GroupSize && kGroupRecWords == kHex20GroupRecWords, "host-side sizes");
static_assert(kHex20Wave % kGroup == 0 && kBatchHex20Wave % kGroup == 0, "waves of whole groups");

// Whether a map word names a slot (slot ids are below 2^31 - 1: the layout
// keeps the slot count below 2^31).
__device__ __forceinline__ bool map_has_slot(unsigned w) { return (w & ~kPairShared) != (kMapNone & ~kPairShared); }

// Packed index of the upper block (I, J), I <= J, of a Hex20 element.
__device__ __forceinline__ int packed_block(int I, int J) { return I * 20 - I * (I - 1) / 2 + J - I; }

struct GroupTopo {
    int node[kGroupOcc];                   // group-local node u -> node id (u < nu)
    int occ[kGroupOcc];                    // occurrence 20 e + a -> node id of node a of element e
    unsigned nb[kGroupOcc][kNbWords];      // neighbour sets
    unsigned first[kNbWords];              // occurrences that are their node's first
    unsigned short ubase[kGroupOcc + 1];   // pair index of {u, u}; ubase[nu] = number of pairs
    unsigned char nbpre[kGroupOcc][kNbWords];  // neighbours of u in the words before w
    unsigned char nbbelow[kGroupOcc];      // neighbours of u before u
    unsigned char lidx[kGroupOcc];         // occurrence -> group-local node
    unsigned short hslot[kGroupOcc];       // occurrence -> its node's entry in the hash table
    int hkey[2 * kGroupOcc];               // node id hash table (first occurrences), -1 = empty
    int hfirst[2 * kGroupOcc];
    int ne, nu, npairs, bad;
};

// Pair index of {u, v}, u <= v, v in nb[u]: v's rank among u's neighbours
// from u on.
__device__ __forceinline__ int pair_index(const GroupTopo& T, int u, int v) {
    return T.ubase[u] + T.nbpre[u][v >> 5] + __popc(T.nb[u][v >> 5] & ((1u << (v & 31)) - 1u)) - T.nbbelow[u];
}

// Topology of the group of positions [g0, g0 + ne) of the visit order perm
// (NULL: element i is position i). Every thread of the CTA calls it; it ends
// with a barrier. A node id outside [0, N) sets T.bad (and leaves the rest
// undefined).
__device__ void group_topology(const MeshView& m, const int* __restrict__ perm, long long g0, int ne, GroupTopo& T) {
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31;
    const int nocc = ne * 20;
    if (tid == 0) {
        T.bad = 0;
        T.ne = ne;
    }
    if (tid < kNbWords) T.first[tid] = 0;
    for (int k = tid; k < kGroupOcc * kNbWords; k += nt) (&T.nb[0][0])[k] = 0u;
    for (int k = tid; k < 2 * kGroupOcc; k += nt) {
        T.hkey[k] = -1;
        T.hfirst[k] = kGroupOcc;
    }
    __syncthreads();
    for (int k = tid; k < nocc; k += nt) {
        const long long i = g0 + k / 20;
        const int e = perm ? FEM_LDG(perm + i) : (int)i;
        const int n = FEM_LDG(m.conn + (size_t)e * 20 + k % 20);
        T.occ[k] = n;
        if (n < 0 || n >= m.N) T.bad = 1;
    }
    __syncthreads();
    if (T.bad) return;  // uniform
    // first occurrence of each occurrence's node, through a hash table of the node ids
    for (int k = tid; k < nocc; k += nt) {
        const int n = T.occ[k];
        int h = (int)(((unsigned)n * 2654435761u) >> 23) % (2 * kGroupOcc);
        for (;;) {
            const int old = atomicCAS(&T.hkey[h], -1, n);
            if (old == -1 || old == n) break;
            h = h + 1 == 2 * kGroupOcc ? 0 : h + 1;
        }
        T.hslot[k] = (unsigned short)h;
        atomicMin(&T.hfirst[h], k);
    }
    __syncthreads();
    for (int k = tid; k < nocc; k += nt) {
        const int j = T.hfirst[T.hslot[k]];
        T.lidx[k] = (unsigned char)j;
        if (j == k) atomicOr(&T.first[k >> 5], 1u << (k & 31));
    }
    __syncthreads();
    // group-local node = rank of the first occurrence among the first occurrences
    for (int k = tid; k < nocc; k += nt) {
        const int j = T.lidx[k];
        int u = __popc(T.first[j >> 5] & ((1u << (j & 31)) - 1u));
        for (int w = 0; w < (j >> 5); w++) u += __popc(T.first[w]);
        T.lidx[k] = (unsigned char)u;
        if (j == k) T.node[u] = T.occ[k];
    }
    __syncthreads();
    // neighbour sets (every node pair of every element, the node itself included)
    for (int k = tid; k < ne * 400; k += nt) {
        const int e = k / 400, p = k - 400 * e, a = p / 20, b = p - 20 * a;
        const int u = T.lidx[20 * e + a], v = T.lidx[20 * e + b];
        atomicOr(&T.nb[u][v >> 5], 1u << (v & 31));
    }
    __syncthreads();
    // neighbour-rank tables of pair_index
    for (int u = tid; u < kGroupOcc; u += nt) {
        int c = 0, below = 0;
#pragma unroll
        for (int w = 0; w < kNbWords; w++) {
            const unsigned bits = T.nb[u][w];
            T.nbpre[u][w] = (unsigned char)c;
            if (w < (u >> 5)) below += __popc(bits);
            else if (w == (u >> 5)) below += __popc(bits & ((1u << (u & 31)) - 1u));
            c += __popc(bits);
        }
        T.nbbelow[u] = (unsigned char)below;
    }
    // pair numbering: ubase = exclusive prefix of the counts of {u <= v}
    if (tid < 32) {
        int nu = 0;
#pragma unroll
        for (int w = 0; w < kNbWords; w++) nu += __popc(T.first[w]);
        int carry = 0;
        for (int u0 = 0; u0 < nu; u0 += 32) {
            const int u = u0 + lane;
            int c = 0;
            if (u < nu) {
#pragma unroll
                for (int w = 0; w < kNbWords; w++) {
                    unsigned bits = T.nb[u][w];
                    if (w < (u >> 5)) bits = 0u;
                    else if (w == (u >> 5)) bits &= ~0u << (u & 31);
                    c += __popc(bits);
                }
            }
            int incl = c;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const int y = __shfl_up_sync(0xFFFFFFFFu, incl, d);
                if (lane >= d) incl += y;
            }
            if (u < nu) T.ubase[u] = (unsigned short)(carry + incl - c);
            carry += __shfl_sync(0xFFFFFFFFu, incl, 31);
        }
        if (lane == 0) {
            T.ubase[nu] = (unsigned short)carry;
            T.nu = nu;
            T.npairs = carry;
        }
    }
    __syncthreads();
}

}  // namespace
}  // namespace fem
