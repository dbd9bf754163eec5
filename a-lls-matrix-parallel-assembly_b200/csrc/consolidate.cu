// K2-K4 fused: list -> CSR consolidation.
//
// Replaces both the reference's host pattern build (buildCSRStructure,
// ALLS_Quad2D_Assembly_Accuracy_Analysis.cu:605-645; buildCSRStructureHex20,
// ALLS_Hex20_3D_Assembly_Performance.cu:364-392) and its convert kernels
// (convertALLStoCSRKernel, Q4A:471-501; ...FixedArray, H20:259-278), which walk
// each row's list and binary-search the host-built col_ind.
//
// One CTA handles a tile of NPT consecutive nodes; a group of G lanes serves
// one node (all dpn dof rows of it):
//   1. gather the node's list entries (column node, slot) — the non-empty
//      hashed slots of its chunk chain — into shared memory as 64-bit keys
//      (col << 32 | slot);
//   2. bitonic sort of the G*KPL keys across the group (shuffles + registers);
//   3. mark the first key of every column run and count unique columns u (the
//      scatter inserts each column once per row; runs longer than one would be
//      summed all the same);
//   4. tile-wide scan of u, then a single-pass decoupled look-back over tiles
//      (tiles are handed out in launch order through an atomic ticket, so every
//      predecessor is already running; waits are bounded);
//   5. write row_ptr and, row by row, col_idx = col*dpn + b and the value
//      (sum of the run's slot values) with consecutive lanes on consecutive
//      entries.
// The result is the reference's pattern exactly: every dof row of node n holds
// {c*dpn + b : c in adj(n)} in increasing order.
#include "launch.h"

namespace fem {
namespace {

constexpr unsigned long long kEmptyKey = ~0ull;
constexpr unsigned long long kFlagAggregate = 1ull << 62;
constexpr unsigned long long kFlagPrefix = 2ull << 62;
constexpr unsigned long long kValueMask = (1ull << 62) - 1;
constexpr long long kMaxSpin = 1ll << 22;

__device__ __forceinline__ unsigned long long shfl_xor_u64(unsigned long long v, int m) {
    unsigned lo = (unsigned)v, hi = (unsigned)(v >> 32);
    lo = __shfl_xor_sync(0xFFFFFFFFu, lo, m);
    hi = __shfl_xor_sync(0xFFFFFFFFu, hi, m);
    return ((unsigned long long)hi << 32) | lo;
}

// Ascending bitonic sort of G*KPL keys held as keys[i] at position lane*KPL + i
// of a G-lane group. Every lane of the warp must call it.
template <int G, int KPL>
__device__ __forceinline__ void group_sort(unsigned long long (&keys)[KPL], int glane) {
    constexpr int N = G * KPL;
#pragma unroll
    for (int size = 2; size <= N; size <<= 1) {
#pragma unroll
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            if (stride >= KPL) {
                const int lstride = stride / KPL;
#pragma unroll
                for (int i = 0; i < KPL; i++) {
                    const int pos = glane * KPL + i;
                    const unsigned long long other = shfl_xor_u64(keys[i], lstride);
                    const bool up = (pos & size) == 0;
                    const bool lower = (pos & stride) == 0;
                    const unsigned long long mn = keys[i] < other ? keys[i] : other;
                    const unsigned long long mx = keys[i] < other ? other : keys[i];
                    keys[i] = (lower == up) ? mn : mx;
                }
            } else {
#pragma unroll
                for (int i = 0; i < KPL; i++) {
                    const int j = i ^ stride;
                    if (j > i) {
                        const int pos = glane * KPL + i;
                        const bool up = (pos & size) == 0;
                        const unsigned long long a = keys[i], b = keys[j];
                        const bool swap = up ? (a > b) : (a < b);
                        keys[i] = swap ? b : a;
                        keys[j] = swap ? a : b;
                    }
                }
            }
        }
    }
}

// Slow path for rows with more list entries than a group can sort at once (a
// node of unusually high degree). Iterated minimum extraction: each unique
// column is found as the smallest column above the previous one, with a
// group-wide min over the row's entries; duplicate slots are summed by the same
// walk. O(unique * entries / G) work, exact for any row length.
template <int G>
__device__ __forceinline__ unsigned group_mask(int grp_in_warp) {
    return G == 32 ? 0xFFFFFFFFu : (((1u << G) - 1u) << (grp_in_warp * G));
}

template <int G>
__device__ int long_row_next_col(const ListLayout& L, int n, int after, int glane, unsigned mask) {
    int best = 0x7FFFFFFF;
    int c = n;
    for (int step = 0; step < kMaxChainSteps; step++) {
        const int* meta = chunk_meta(L, c);
        const int cap = chunk_cap(L, c);
        const int next = __ldg(meta + 1);
        for (int s = glane; s < cap; s += G) {
            const int col = (__ldg(meta + 2 + s) & kColMask) - 1;
            if (col > after && col < best) best = col;
        }
        if (next == 0) break;
        c = next - 1;
    }
#pragma unroll
    for (int d = G / 2; d > 0; d >>= 1) best = min(best, __shfl_xor_sync(mask, best, d));
    return best;
}

template <int DPN, int G>
__device__ int long_row_count(const ListLayout& L, int n, int T, int glane, unsigned mask) {
    int u = 0, last = -1;
    for (int it = 0; it < T; it++) {
        const int c = long_row_next_col<G>(L, n, last, glane, mask);
        if (c == 0x7FFFFFFF) break;
        u++;
        last = c;
    }
    return u;
}

template <int DPN, int G>
__device__ void long_row_write(const ListLayout& L, int n, int u, long long base, int glane, unsigned mask,
                               int* __restrict__ col_idx, double* __restrict__ values) {
    constexpr int B = DPN * DPN;
    int last = -1;
    for (int k = 0; k < u; k++) {
        const int col = long_row_next_col<G>(L, n, last, glane, mask);
        last = col;
        double sum[B];
#pragma unroll
        for (int v = 0; v < B; v++) sum[v] = 0.0;
        int c = n;
        for (int step = 0; step < kMaxChainSteps; step++) {
            const int* meta = chunk_meta(L, c);
            const int cap = chunk_cap(L, c);
            const int next = __ldg(meta + 1);
            for (int s = glane; s < cap; s += G) {
                if ((__ldg(meta + 2 + s) & kColMask) - 1 == col) {
                    const double* p = L.vals + (size_t)slot_gid(L, c, s) * B;
#pragma unroll
                    for (int v = 0; v < B; v++) sum[v] += __ldg(p + v);
                }
            }
            if (next == 0) break;
            c = next - 1;
        }
#pragma unroll
        for (int v = 0; v < B; v++) {
#pragma unroll
            for (int d = G / 2; d > 0; d >>= 1) sum[v] += __shfl_xor_sync(mask, sum[v], d);
        }
        if (glane == 0) {
#pragma unroll
            for (int a = 0; a < DPN; a++)
#pragma unroll
                for (int b = 0; b < DPN; b++) {
                    const long long pos = base + (long long)a * DPN * u + (long long)k * DPN + b;
                    col_idx[pos] = col * DPN + b;
                    values[pos] = sum[a * DPN + b];
                }
        }
    }
}

template <int DPN, int G, int KPL>
__global__ void __launch_bounds__(kBlockThreads) k_consolidate(ListLayout L, int* __restrict__ row_ptr,
                                                               int* __restrict__ col_idx, double* __restrict__ values,
                                                               long long capacity, unsigned long long* tile_state,
                                                               int num_tiles) {
    constexpr int NPT = kBlockThreads / G;  // nodes per tile
    constexpr int NK = G * KPL;             // key capacity per node
    constexpr int B = DPN * DPN;
    __shared__ unsigned long long s_keys[NPT][NK];
    __shared__ short s_head[NPT][NK + 1];
    __shared__ int s_u[NPT], s_ex[NPT], s_T[NPT];
    __shared__ int s_tile;
    __shared__ long long s_prefix, s_total;

    const int tid = threadIdx.x;
    if (tid == 0) s_tile = atomicAdd(&L.info->tile_ticket, 1);
    __syncthreads();
    const int tile = s_tile;
    if (tile >= num_tiles) return;  // uniform
    const int grp = tid / G, glane = tid % G;
    const int n = tile * NPT + grp;
    const bool valid = n < L.N;

    const unsigned gmask = group_mask<G>((tid & 31) / G);
    const int gshift = G == 32 ? 0 : ((tid & 31) / G) * G;
    // 1. gather (non-empty hashed slots of every chunk of the row)
    int T = 0;
    bool long_row = false;
    if (valid) {
        int c = n;
        for (int step = 0; step < kMaxChainSteps; step++) {
            const int* meta = chunk_meta(L, c);
            const int cap = chunk_cap(L, c);
            const int next = __ldg(meta + 1);
            for (int s0 = 0; s0 < cap; s0 += G) {
                const int s = s0 + glane;
                const int col = s < cap ? (__ldg(meta + 2 + s) & kColMask) : 0;
                const unsigned used = __ballot_sync(gmask, col != 0) >> gshift;
                const int e = T + __popc(used & ((1u << glane) - 1u));
                if (col != 0 && e < NK)
                    s_keys[grp][e] = ((unsigned long long)(unsigned)(col - 1) << 32) | slot_gid(L, c, s);
                T += __popc(used);
            }
            if (next == 0) break;
            c = next - 1;
        }
        long_row = T > NK;
    }
    const int Ts = long_row ? 0 : T;  // entries sorted in registers
    __syncwarp();
    // 2. sort
    unsigned long long keys[KPL];
#pragma unroll
    for (int i = 0; i < KPL; i++) {
        const int p = glane * KPL + i;
        keys[i] = p < Ts ? s_keys[grp][p] : kEmptyKey;
    }
    group_sort<G, KPL>(keys, glane);
#pragma unroll
    for (int i = 0; i < KPL; i++) s_keys[grp][glane * KPL + i] = keys[i];
    __syncwarp();
    // 3. run heads
    int heads = 0;
    bool is_head[KPL];
#pragma unroll
    for (int i = 0; i < KPL; i++) {
        const int p = glane * KPL + i;
        is_head[i] = p < Ts && (p == 0 || (s_keys[grp][p] >> 32) != (s_keys[grp][p - 1] >> 32));
        heads += is_head[i];
    }
    int incl = heads;
#pragma unroll
    for (int d = 1; d < G; d <<= 1) {
        const int v = __shfl_up_sync(0xFFFFFFFFu, incl, d, G);
        if (glane >= d) incl += v;
    }
    int u = __shfl_sync(0xFFFFFFFFu, incl, G - 1, G);
    int k = incl - heads;
#pragma unroll
    for (int i = 0; i < KPL; i++)
        if (is_head[i]) s_head[grp][k++] = (short)(glane * KPL + i);
    if (long_row) u = long_row_count<DPN, G>(L, n, T, glane, gmask);
    if (glane == 0) {
        s_head[grp][u < NK ? u : NK] = (short)Ts;
        s_u[grp] = valid ? u : 0;
        s_T[grp] = valid ? T : 0;
    }
    __syncthreads();
    // 4. tile scan + decoupled look-back
    if (tid < 32) {
        int v = tid < NPT ? s_u[tid] : 0;
        int t = tid < NPT ? s_T[tid] : 0;
        int inc = v;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int o = __shfl_up_sync(0xFFFFFFFFu, inc, d);
            if (tid >= d) inc += o;
        }
        if (tid < NPT) s_ex[tid] = inc - v;
        int tmax = t, tsum = t;
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) {
            tmax = max(tmax, __shfl_xor_sync(0xFFFFFFFFu, tmax, d));
            tsum += __shfl_xor_sync(0xFFFFFFFFu, tsum, d);
        }
        const long long agg = (long long)B * __shfl_sync(0xFFFFFFFFu, inc, 31);
        if (tid == 0) {
            atomicAdd(reinterpret_cast<unsigned long long*>(&L.info->list_entries), (unsigned long long)tsum);
            atomicMax(&L.info->max_row_entries, tmax);
            volatile unsigned long long* st = tile_state;
            long long prefix = 0;
            if (tile == 0) {
                st[0] = kFlagPrefix | (unsigned long long)agg;
            } else {
                st[tile] = kFlagAggregate | (unsigned long long)agg;
                int j = tile - 1;
                long long spins = 0;
                while (j >= 0) {
                    const unsigned long long w = st[j];
                    const unsigned long long flag = w & ~kValueMask;
                    if (flag == 0) {
                        if (++spins > kMaxSpin) {
                            raise_status(L.info, FEM_ERR_TIMEOUT);
                            break;
                        }
                        __nanosleep(64);
                        continue;
                    }
                    prefix += (long long)(w & kValueMask);
                    if (flag == kFlagPrefix) break;
                    j--;
                }
                __threadfence();
                st[tile] = kFlagPrefix | (unsigned long long)(prefix + agg);
            }
            s_prefix = prefix;
            s_total = prefix + agg;
            if (tile == num_tiles - 1) {
                row_ptr[(size_t)L.N * DPN] = (int)(prefix + agg);
                L.info->nnz = prefix + agg;
                if (prefix + agg > 0x7FFFFFFFll) raise_status(L.info, FEM_ERR_RANGE);
            }
            if (prefix + agg > capacity) raise_status(L.info, FEM_ERR_CAPACITY);
        }
    }
    __syncthreads();
    // 5. writes
    if (!valid) return;
    const long long base = s_prefix + (long long)B * s_ex[grp];
    if (glane < DPN) row_ptr[(size_t)n * DPN + glane] = (int)(base + (long long)glane * DPN * u);
    if (s_total > capacity) return;
    if (long_row) {
        long_row_write<DPN, G>(L, n, u, base, glane, gmask, col_idx, values);
        return;
    }
    const int row_len = DPN * u;
    for (int a = 0; a < DPN; a++) {
        const long long rbase = base + (long long)a * row_len;
        for (int r = glane; r < row_len; r += G) {
            const int kk = r / DPN, b = r - kk * DPN;
            const int h0 = s_head[grp][kk], h1 = s_head[grp][kk + 1];
            const unsigned long long key0 = s_keys[grp][h0];
            double sum = 0.0;
            for (int h = h0; h < h1; h++) {
                const unsigned gid = (unsigned)s_keys[grp][h];
                sum += __ldg(L.vals + (size_t)gid * B + a * DPN + b);
            }
            col_idx[rbase + r] = (int)(key0 >> 32) * DPN + b;
            values[rbase + r] = sum;
        }
    }
}

__global__ void k_info_init(DevInfo* info, int pool_chunks) {
    info->pool_chunks = pool_chunks;
}

// Clears what a consolidation pass owns, so the pass can be re-run on the same
// lists (e.g. after FEM_ERR_CAPACITY with larger output buffers).
__global__ void k_consolidate_reset(DevInfo* info) {
    constexpr int kOwned = (1 << FEM_ERR_CAPACITY) | (1 << FEM_ERR_RANGE) | (1 << FEM_ERR_ROW_TOO_LONG) |
                           (1 << FEM_ERR_TIMEOUT);
    info->status_bits &= ~kOwned;
    info->nnz = 0;
    info->list_entries = 0;
    info->max_row_entries = 0;
    info->tile_ticket = 0;
}

}  // namespace

cudaError_t launch_consolidate(const ListLayout& L, int dpn, int* row_ptr, int* col_idx, double* values,
                               long long capacity, unsigned long long* tile_state, int num_tiles, cudaStream_t s) {
    cudaError_t err = cudaMemsetAsync(tile_state, 0, (size_t)num_tiles * sizeof(unsigned long long), s);
    if (err) return err;
    k_consolidate_reset<<<1, 1, 0, s>>>(L.info);
    err = cudaGetLastError();
    if (err) return err;
    if (dpn == 3)
        k_consolidate<3, 32, 8><<<num_tiles, kBlockThreads, 0, s>>>(L, row_ptr, col_idx, values, capacity, tile_state,
                                                                    num_tiles);
    else
        k_consolidate<2, 16, 2><<<num_tiles, kBlockThreads, 0, s>>>(L, row_ptr, col_idx, values, capacity, tile_state,
                                                                    num_tiles);
    return cudaGetLastError();
}

cudaError_t launch_info_init(DevInfo* info, int pool_chunks, cudaStream_t s) {
    k_info_init<<<1, 1, 0, s>>>(info, pool_chunks);
    return cudaGetLastError();
}

}  // namespace fem
