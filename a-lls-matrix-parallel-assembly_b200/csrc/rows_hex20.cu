// Hex20 list scatter, pass 1a (single-mesh path): the list entries of a
// wave, inserted row by row.
//
// Replaces the insert half of assembleGlobalStiffnessKernelALLSFixedArray
// (ALLS_Hex20_3D_Assembly_Performance.cu:226-256: a linear scan of the row's
// columns, a slot claimed with atomicAdd on the row count, no fence), whose
// racing inserts duplicate or drop columns.
//
// One warp per row node that an element of the wave has (the wave's node
// list, built once per mesh): the warp reads the node's incident elements
// (node -> element incidence) and their node ids, and collects in a
// shared-memory hash table every column node with
//   - whether an element of this wave has it (only those are inserted now;
//     the others belong to another wave's pass), and
//   - the lowest and highest element group (visit position / 8) among all
//     elements with both nodes: the node pair belongs to one group alone when
//     they are equal.
// The warp then inserts the wave's new columns into the row's first chunk:
// the chunk is copied into shared memory, each lane claims the first empty
// slot of its column's probe sequence there with a shared-memory atomicCAS
// (lanes of one warp are the only writers of the row in this launch, so the
// copy is the row), and the claimed slot words go back to the list with the
// pair's shared flag in bit 31. A full first chunk continues in the row's
// overflow chunks (taken from the pool and linked with atomicCAS). The value
// block of every new shared pair is zeroed for the atomic adds of several
// groups; an owned pair's block is left for the one store of its group. The
// row's entry count grows by its new entries.
//
// Warp-aggregated insertion: the list still takes one entry per (row node,
// column node) pair with atomic slot claims and atomic value additions, but a
// row's claims are gathered in one warp instead of racing from every element.
#include <algorithm>

#include "claim_hex20.cuh"

namespace fem {
namespace {

constexpr int kRowWarps = 8;
constexpr int kRowThreads = kRowWarps * 32;
constexpr int kRowHash = 512;   // column hash table per warp (a row has at most a few hundred columns)
constexpr int kRowElems = 8;    // incident elements read at once

struct RowWarpSmem {
    int key[kRowHash];       // column node + 1 (0 = empty)
    int gmin[kRowHash], gmax[kRowHash];
    int inw[kRowHash];       // an element of this wave has the column
    alignas(16) int chunk[kClaimMaxWords];
    int elem[kRowElems], grp[kRowElems], wave[kRowElems];
};

__device__ __forceinline__ int row_hash(int key) { return (int)(((unsigned)key * 2654435761u) >> 23); }

// Inserts key (column + 1, flag in bit 31 of the stored word) into the row's
// overflow chunks after its first chunk was found full, as resolve_chain
// (the stored words carry the flag, so columns are compared under kColMask).
// Returns the slot id (-1: pool overflow or chain bound, status raised) and
// whether it was new.
__device__ int row_chain_insert(const ListLayout& L, int n, int key, unsigned flag, int& spare, bool& fresh) {
    fresh = false;
    int c = n;
    for (int step = 0; step < kMaxChainSteps; step++) {
        c = next_chunk(L, c, spare);
        if (c < 0) return -1;
        int* meta = chunk_meta(L, c);
        const int S = chunk_cap(L, c);
        const int p0 = probe_start(key, S);
        for (int t = 0; t < S; t++) {
            int s = p0 + t;
            if (s >= S) s -= S;
            int v = ld_cg(meta + 2 + s);
            if (v == 0) {
                v = atomicCAS(meta + 2 + s, 0, (int)((unsigned)key | flag));
                if (v == 0) {
                    fresh = true;
                    return (int)slot_gid(L, c, s);
                }
            }
            if ((v & kColMask) == key) return (int)slot_gid(L, c, s);
        }
    }
    raise_status(L.info, FEM_ERR_TIMEOUT);
    return -1;
}

__global__ void __launch_bounds__(kRowThreads) k_rows_hex20(MeshView m, ListLayout L, const int* __restrict__ inc_off,
                                                           const int* __restrict__ inc,
                                                           const int* __restrict__ pos_of, int i0, int i1,
                                                           const int* __restrict__ wnodes,
                                                           const int* __restrict__ woff, int w) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    RowWarpSmem& sm = reinterpret_cast<RowWarpSmem*>(smem_raw)[warp];
    const int S1 = L.S1, H1 = L.H1;
    const int first = woff[w], count = woff[w + 1] - first;
    int spare = -1;
    for (long long q = (long long)blockIdx.x * kRowWarps + warp; q < count; q += (long long)gridDim.x * kRowWarps) {
        const int n = __ldg(wnodes + first + q);
        for (int h = lane; h < kRowHash; h += 32) {
            sm.key[h] = 0;
            sm.gmin[h] = 0x7FFFFFFF;
            sm.gmax[h] = -1;
            sm.inw[h] = 0;
        }
        // the row's first chunk (its slot words from earlier waves)
        for (int k = lane; k < (H1 >> 2); k += 32)
            *reinterpret_cast<int4*>(&sm.chunk[4 * k]) = ld_cg4(L.meta1 + (size_t)n * H1 + 4 * k);
        __syncwarp();
        // the columns of the node's elements
        const int lo = __ldg(inc_off + n), deg = __ldg(inc_off + n + 1) - lo;
        for (int j0 = 0; j0 < deg; j0 += kRowElems) {
            const int cnt = min(kRowElems, deg - j0);
            if (lane < cnt) {
                const int e = __ldg(inc + lo + j0 + lane);
                const int pos = __ldg(pos_of + e);
                sm.elem[lane] = e;
                sm.grp[lane] = pos >> 3;
                sm.wave[lane] = pos >= i0 && pos < i1;
            }
            __syncwarp();
            for (int idx = lane; idx < cnt * 20; idx += 32) {
                const int j = idx / 20;
                const int c = __ldg(m.conn + (size_t)sm.elem[j] * 20 + idx - 20 * j);
                if (c < 0 || c >= m.N) continue;  // reported by the lookup pass
                const int key = c + 1;
                int h = row_hash(key) & (kRowHash - 1);
                bool placed = false;
                for (int t = 0; t < kRowHash && !placed; t++) {
                    const int old = atomicCAS(&sm.key[h], 0, key);
                    placed = old == 0 || old == key;
                    if (!placed) h = (h + 1) & (kRowHash - 1);
                }
                if (!placed) {  // more distinct columns than the table holds
                    raise_status(L.info, FEM_ERR_RANGE);
                    continue;
                }
                atomicMin(&sm.gmin[h], sm.grp[j]);
                atomicMax(&sm.gmax[h], sm.grp[j]);
                if (sm.wave[j]) sm.inw[h] = 1;
            }
            __syncwarp();
        }
        // the wave's columns into the row: found, or claimed in the copy
        int fresh = 0;
        for (int h = lane; h < kRowHash; h += 32) {
            const int key = sm.key[h];
            if (key == 0 || !sm.inw[h]) continue;
            const unsigned flag = sm.gmin[h] == sm.gmax[h] ? 0u : kPairShared;
            const int p0 = probe_start(key, S1);
            int gid = -1;
            bool is_new = false, full = true;
            for (int t = 0; t < S1; t++) {
                int s = p0 + t;
                if (s >= S1) s -= S1;
                int x = sm.chunk[2 + s];
                if (x == 0) {
                    x = atomicCAS(&sm.chunk[2 + s], 0, (int)((unsigned)key | flag));
                    if (x == 0) {
                        L.meta1[(size_t)n * H1 + 2 + s] = (int)((unsigned)key | flag);
                        gid = (int)slot_gid(L, n, s);
                        is_new = true;
                        full = false;
                        break;
                    }
                }
                if ((x & kColMask) == key) {
                    full = false;
                    break;  // an entry of an earlier wave
                }
            }
            if (full) gid = row_chain_insert(L, n, key, flag, spare, is_new);
            if (is_new) {
                fresh++;
                if (flag && gid >= 0) zero_block(L.vals + (size_t)(unsigned)gid * 9);
            }
        }
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) fresh += __shfl_xor_sync(0xFFFFFFFFu, fresh, d);
        if (lane == 0 && fresh) L.counts[n] += fresh;  // this warp is the row's only writer in the launch
        __syncwarp();
    }
}

// pos_of[perm[i]] = i.
__global__ void k_positions(const int* __restrict__ perm, int E, int* __restrict__ pos_of) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < E; i += gridDim.x * blockDim.x) pos_of[__ldg(perm + i)] = i;
}

// Waves a node's elements fall in (bit w of a 64-bit mask); mode 0 counts the
// nodes of each wave, mode 1 lists them.
__global__ void k_node_waves(int N, const int* __restrict__ inc_off, const int* __restrict__ inc,
                             const int* __restrict__ pos_of, int wave, int mode, int* __restrict__ wcount,
                             const int* __restrict__ woff, int* __restrict__ wnodes) {
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < N; n += gridDim.x * blockDim.x) {
        unsigned long long mask = 0ull;
        for (int k = __ldg(inc_off + n); k < __ldg(inc_off + n + 1); k++) mask |= 1ull << (__ldg(pos_of + __ldg(inc + k)) / wave);
        while (mask) {
            const int w = __ffsll((long long)mask) - 1;
            mask &= mask - 1ull;
            const int slot = atomicAdd(wcount + w, 1);
            if (mode) wnodes[woff[w] + slot] = n;
        }
    }
}

__global__ void k_wave_offsets(int* __restrict__ wcount, int nw, int* __restrict__ woff) {
    if (threadIdx.x == 0) {
        int o = 0;
        for (int w = 0; w < nw; w++) {
            woff[w] = o;
            o += wcount[w];
            wcount[w] = 0;  // the list pass counts again
        }
        woff[nw] = o;
    }
}

}  // namespace

cudaError_t launch_wave_nodes(const MeshView& m, const int* perm, const int* inc_off, const int* inc, int wave,
                              int nwaves, int* pos_of, int* wcount, int* woff, int* wnodes, cudaStream_t s) {
    if (nwaves > 64) return cudaErrorInvalidValue;
    const int g = std::max(1, std::min((m.E_count + 255) / 256, 8 * sm_count()));
    const int gn = std::max(1, std::min((m.N + 255) / 256, 8 * sm_count()));
    cudaError_t err = cudaMemsetAsync(wcount, 0, (size_t)nwaves * sizeof(int), s);
    if (err) return err;
    k_positions<<<g, 256, 0, s>>>(perm, m.E_count, pos_of);
    k_node_waves<<<gn, 256, 0, s>>>(m.N, inc_off, inc, pos_of, wave, 0, wcount, nullptr, nullptr);
    k_wave_offsets<<<1, 32, 0, s>>>(wcount, nwaves, woff);
    k_node_waves<<<gn, 256, 0, s>>>(m.N, inc_off, inc, pos_of, wave, 1, wcount, woff, wnodes);
    return cudaGetLastError();
}

cudaError_t launch_rows_hex20(const MeshView& m, const ListLayout& L, const int* inc_off, const int* inc,
                              const int* pos_of, int i0, int i1, const int* wnodes, const int* woff, int w,
                              cudaStream_t s) {
    static DeviceCache cache;
    const size_t smem = kRowWarps * sizeof(RowWarpSmem);
    int per_sm = 0;
    const cudaError_t err = per_device(cache, [&](int& v) {
        cudaError_t e = cudaFuncSetAttribute(k_rows_hex20, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (!e) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, k_rows_hex20, kRowThreads, smem);
        return e;
    }, per_sm);
    if (err) return err;
    // the wave's node count is on the device: a persistent grid of every resident CTA
    k_rows_hex20<<<per_sm * sm_count(), kRowThreads, smem, s>>>(m, L, inc_off, inc, pos_of, i0, i1, wnodes, woff, w);
    return cudaGetLastError();
}

}  // namespace fem
