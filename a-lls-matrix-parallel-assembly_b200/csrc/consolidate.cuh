// Device code of the list -> CSR consolidation (consolidate.cu), shared with
// the batched persistent kernel (batched.cu): tile-level scan steps and the
// sorted write of a range of row-node batches. See consolidate.cu for the
// algorithm and the reference steps it replaces.
#pragma once

#include "launch.h"
#include "scan.cuh"

namespace fem {
namespace {

constexpr unsigned long long kEmptyKey = ~0ull;

constexpr int kScanItems = kScanTile / kScanThreads;  // 16 nodes per thread

__device__ __forceinline__ unsigned long long shfl_xor_u64(unsigned long long v, int m) {
    unsigned lo = (unsigned)v, hi = (unsigned)(v >> 32);
    lo = __shfl_xor_sync(0xFFFFFFFFu, lo, m);
    hi = __shfl_xor_sync(0xFFFFFFFFu, hi, m);
    return ((unsigned long long)hi << 32) | lo;
}

// Tile sums of dpn^2 * counts: tile `tile` (kScanThreads threads).
template <int B>
__device__ __forceinline__ void scan_reduce_tile(const int* __restrict__ counts, int N, long long* __restrict__ tile_sums,
                                                 int tile, long long* s_warp) {
    const long long base = (long long)tile * kScanTile;
    long long sum = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; i++) {
        const long long n = base + (long long)i * kScanThreads + threadIdx.x;
        if (n < N) sum += FEM_LDG(counts + n);
    }
    long long total;
    block_exclusive_scan(sum, s_warp, total);
    if (threadIdx.x == 0) tile_sums[tile] = (long long)B * total;
}


// Exclusive scan of the tile sums in place (one CTA), nnz, last row_ptr entry.
__device__ __forceinline__ void scan_tiles_body(long long* __restrict__ tile_sums, int num_tiles, DevInfo* info,
                                                int* __restrict__ row_ptr_end, long long capacity, int end_div,
                                                long long* s_warp) {
    long long carry = 0;
    for (int base = 0; base < num_tiles; base += kScanThreads) {
        const int t = base + threadIdx.x;
        const long long v = t < num_tiles ? __ldcg(tile_sums + t) : 0;
        long long total;
        const long long ex = block_exclusive_scan(v, s_warp, total);
        if (t < num_tiles) tile_sums[t] = carry + ex;
        carry += total;
    }
    if (threadIdx.x == 0) {
        info->nnz = carry;
        *row_ptr_end = (int)(carry / end_div);
        if (carry > 0x7FFFFFFFll) raise_status(info, FEM_ERR_RANGE);
        if (carry > capacity) raise_status(info, FEM_ERR_CAPACITY);
    }
}


// row_ptr of every dof row: node n's rows start at dpn^2 * (exclusive count sum).
// kBsr: one block row per node, block_row_ptr[n] = exclusive count sum.
template <int DPN, bool kBsr>
__device__ __forceinline__ void row_ptr_tile(const int* __restrict__ counts, int N,
                                             const long long* __restrict__ tile_offsets, int* __restrict__ row_ptr,
                                             int tile, long long* s_warp) {
    constexpr int B = DPN * DPN;
    const long long base = (long long)tile * kScanTile + (long long)threadIdx.x * kScanItems;
    int c[kScanItems];
    long long sum = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; i++) {
        const long long n = base + i;
        c[i] = n < N ? FEM_LDG(counts + n) : 0;
        sum += c[i];
    }
    long long total;
    long long off = __ldcg(tile_offsets + tile) + (long long)B * block_exclusive_scan(sum, s_warp, total);
#pragma unroll
    for (int i = 0; i < kScanItems; i++) {
        const long long n = base + i;
        if (n < N) {
            if (kBsr) {
                row_ptr[n] = (int)(off / B);
            } else {
#pragma unroll
                for (int a = 0; a < DPN; a++) row_ptr[n * DPN + a] = (int)(off + (long long)a * DPN * c[i]);
            }
        }
        off += (long long)B * c[i];
    }
}


template <int G>
__device__ __forceinline__ unsigned group_mask(int grp_in_warp) {
    return G == 32 ? 0xFFFFFFFFu : (((1u << G) - 1u) << (grp_in_warp * G));
}

// Upper-triangle CSR: entries of node n's dof rows when u of its column nodes
// are >= n (the node itself among them): row a holds (dpn - a) entries of the
// diagonal block and dpn of each of the u - 1 later blocks.
template <int DPN>
__device__ __forceinline__ long long upper_row_len(int u, int a) {
    return u > 0 ? (long long)(u - 1) * DPN + (DPN - a) : 0;
}
template <int DPN>
__device__ __forceinline__ long long upper_node_entries(int u) {
    return u > 0 ? (long long)(u - 1) * DPN * DPN + DPN * (DPN + 1) / 2 : 0;
}

// Columns >= n in node n's list (a group of G lanes per node).
template <int G>
__global__ void __launch_bounds__(kBlockThreads) k_count_upper(ListLayout L, int* __restrict__ ucounts) {
    constexpr int NPB = kBlockThreads / G;
    const int tid = threadIdx.x, grp = tid / G, glane = tid % G;
    const unsigned gmask = group_mask<G>((tid & 31) / G);
    for (long long nb = (long long)blockIdx.x * NPB; nb < L.N; nb += (long long)gridDim.x * NPB) {
        const int n = (int)(nb + grp);
        int cnt = 0;
        if (n < L.N) {
            int c = n;
            for (int step = 0; step < kMaxChainSteps; step++) {
                const int* meta = chunk_meta(L, c);
                const int cap = chunk_cap(L, c);
                const int next = FEM_LDG(meta + 1);
                for (int s = glane; s < cap; s += G) {
                    const int col = (FEM_LDG(meta + 2 + s) & kColMask) - 1;
                    cnt += col >= n;
                }
                if (next == 0) break;
                c = next - 1;
            }
        }
#pragma unroll
        for (int d = G / 2; d > 0; d >>= 1) cnt += __shfl_xor_sync(gmask, cnt, d);
        if (n < L.N && glane == 0) ucounts[n] = cnt;
    }
}

template <int DPN>
__global__ void __launch_bounds__(kScanThreads) k_scan_reduce_upper(const int* __restrict__ ucounts, int N,
                                                                    long long* __restrict__ tile_sums) {
    __shared__ long long s_warp[kScanThreads / 32 + 1];
    const long long base = (long long)blockIdx.x * kScanTile;
    long long sum = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; i++) {
        const long long n = base + (long long)i * kScanThreads + threadIdx.x;
        if (n < N) sum += upper_node_entries<DPN>(FEM_LDG(ucounts + n));
    }
    long long total;
    block_exclusive_scan(sum, s_warp, total);
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

template <int DPN>
__global__ void __launch_bounds__(kScanThreads) k_row_ptr_upper(const int* __restrict__ ucounts, int N,
                                                                const long long* __restrict__ tile_offsets,
                                                                int* __restrict__ row_ptr) {
    __shared__ long long s_warp[kScanThreads / 32 + 1];
    const long long base = (long long)blockIdx.x * kScanTile + (long long)threadIdx.x * kScanItems;
    int c[kScanItems];
    long long sum = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; i++) {
        const long long n = base + i;
        c[i] = n < N ? FEM_LDG(ucounts + n) : 0;
        sum += upper_node_entries<DPN>(c[i]);
    }
    long long total;
    long long off = tile_offsets[blockIdx.x] + block_exclusive_scan(sum, s_warp, total);
#pragma unroll
    for (int i = 0; i < kScanItems; i++) {
        const long long n = base + i;
        if (n < N) {
            long long r = off;
#pragma unroll
            for (int a = 0; a < DPN; a++) {
                row_ptr[n * DPN + a] = (int)r;
                r += upper_row_len<DPN>(c[i], a);
            }
        }
        off += upper_node_entries<DPN>(c[i]);
    }
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

// Slow path for a row with more entries than a group can sort at once (a node
// of unusually high degree): iterated minimum extraction over the row's chunk
// chain. O(u * entries / G) work, exact for any row length.
template <int G>
__device__ int long_row_next_col(const ListLayout& L, int n, int after, int glane, unsigned mask) {
    int best = 0x7FFFFFFF;
    int c = n;
    for (int step = 0; step < kMaxChainSteps; step++) {
        const int* meta = chunk_meta(L, c);
        const int cap = chunk_cap(L, c);
        const int next = FEM_LDG(meta + 1);
        for (int s = glane; s < cap; s += G) {
            const int col = (FEM_LDG(meta + 2 + s) & kColMask) - 1;
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
            const int next = FEM_LDG(meta + 1);
            for (int s = glane; s < cap; s += G) {
                if ((FEM_LDG(meta + 2 + s) & kColMask) - 1 == col) {
                    const double* p = L.vals + (size_t)slot_gid(L, c, s) * B;
#pragma unroll
                    for (int v = 0; v < B; v++) sum[v] += FEM_LDG(p + v);
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

// Long-row slow path of the block (BSR) output: block k of the node's block row.
template <int DPN, int G>
__device__ void long_row_write_bsr(const ListLayout& L, int n, int u, long long base, int glane, unsigned mask,
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
            const int next = FEM_LDG(meta + 1);
            for (int s = glane; s < cap; s += G) {
                if ((FEM_LDG(meta + 2 + s) & kColMask) - 1 == col) {
                    const double* p = L.vals + (size_t)slot_gid(L, c, s) * B;
#pragma unroll
                    for (int v = 0; v < B; v++) sum[v] += FEM_LDG(p + v);
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
            col_idx[base + k] = col;
#pragma unroll
            for (int v = 0; v < B; v++) values[(base + k) * B + v] = sum[v];
        }
    }
}

// Long-row slow path of the upper-triangle output: the node's u column nodes
// >= n in increasing order (the first is n itself).
template <int DPN, int G>
__device__ void long_row_write_upper(const ListLayout& L, int n, int u, const int* __restrict__ row_ptr, int glane,
                                     unsigned mask, int* __restrict__ col_idx, double* __restrict__ values) {
    constexpr int B = DPN * DPN;
    int last = n - 1;
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
            const int next = FEM_LDG(meta + 1);
            for (int s = glane; s < cap; s += G) {
                if ((FEM_LDG(meta + 2 + s) & kColMask) - 1 == col) {
                    const double* p = L.vals + (size_t)slot_gid(L, c, s) * B;
#pragma unroll
                    for (int v = 0; v < B; v++) sum[v] += FEM_LDG(p + v);
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
            for (int a = 0; a < DPN; a++) {
                const long long rbase = FEM_LDG(row_ptr + (size_t)n * DPN + a);
#pragma unroll
                for (int b = 0; b < DPN; b++) {
                    if (k == 0 && b < a) continue;  // below the diagonal
                    const long long pos = k == 0 ? rbase + (b - a) : rbase + (DPN - a) + (long long)(k - 1) * DPN + b;
                    col_idx[pos] = col * DPN + b;
                    values[pos] = sum[a * DPN + b];
                }
            }
        }
    }
}

enum : int { kOutCsr = 0, kOutBsr = 1, kOutUpper = 2 };

// Next link and slot words (kPre per lane of a G-lane group) of a node's first chunk.
template <int G, int kPre>
__device__ __forceinline__ void prefetch_first_chunk(const ListLayout& L, long long node, int glane, int (&w)[kPre],
                                                     int& next) {
    if (node < L.N) {
        const int* meta = chunk_meta(L, (int)node);
        next = FEM_LDG(meta + 1);
#pragma unroll
        for (int q = 0; q < kPre; q++) {
            const int s = q * G + glane;
            w[q] = s < L.S1 ? FEM_LDG(meta + 2 + s) : 0;
        }
    }
}

// Resident CTAs per SM the register budget of k_write is set for (build-time
// tuning knobs; measured on B200: 5 for the 2-D kinds, 4 for Hex20).
#ifndef FEM_WRITE_MIN_CTAS_2D
#define FEM_WRITE_MIN_CTAS_2D 5
#endif
#ifndef FEM_WRITE_MIN_CTAS_3D
#define FEM_WRITE_MIN_CTAS_3D 4
#endif

// Shared memory of the sorted write: each group's sort keys and (2-D) the
// node's sorted 2x2 blocks, loaded together before the rows are written.
template <int DPN, int G, int KPL>
struct WriteSmem {
    unsigned long long keys[kBlockThreads / G][G * KPL];
    double2 vals[DPN == 2 ? kBlockThreads / G : 1][DPN == 2 ? G * KPL : 1][2];
};

// The sorted write of the row nodes of batches nb = nb_first, nb_first +
// nb_stride, ... below nb_end (a batch: kBlockThreads / G consecutive nodes,
// one G-lane group each). Every thread of the CTA (kBlockThreads) calls it.
// kMode kOutBsr: block (BSR) output, one block row per node: block_col_idx =
// column node, block values dpn x dpn row-major; row_ptr is then the block row
// pointer. kOutUpper: the upper triangle in CSR (ucounts: columns >= n).
template <int DPN, int G, int KPL, int kMode>
__device__ __forceinline__ void write_batches(const ListLayout& L, const int* __restrict__ row_ptr,
                                              int* __restrict__ col_idx, double* __restrict__ values,
                                              long long capacity, const int* __restrict__ ucounts, long long nb_first,
                                              long long nb_stride, long long nb_end, WriteSmem<DPN, G, KPL>& sm) {
    constexpr bool kBsr = kMode == kOutBsr;
    constexpr int NK = G * KPL;             // sort capacity per node
    constexpr int B = DPN * DPN;
    // slot words of a node's first chunk per lane (2-D: 14 slots; Hex20: at most 94)
    constexpr int kPre = (DPN == 2 ? 16 : 96) / G;
    auto& s_keys = sm.keys;
    auto& s_vals = sm.vals;
    if (__ldcg(&L.info->nnz) > capacity) return;  // FEM_ERR_CAPACITY already raised; write nothing
    const int tid = threadIdx.x;
    const int grp = tid / G, glane = tid % G;
    const unsigned gmask = group_mask<G>((tid & 31) / G);
    const int gshift = G == 32 ? 0 : ((tid & 31) / G) * G;
    int t_sum = 0, t_max = 0;
    // the first chunk (next link and slot words) of the group's next node is
    // loaded while the current node is sorted and written
    int pre_w[kPre], pre_next = 0;
    prefetch_first_chunk<G, kPre>(L, nb_first + grp, glane, pre_w, pre_next);
    for (long long nb = nb_first; nb < nb_end; nb += nb_stride) {
        const int n = (int)(nb + grp);
        const bool valid = n < L.N;
        int u = 0;
        long long base = 0;
        if (valid) {
            if (kMode == kOutUpper) {
                u = FEM_LDG(ucounts + n);  // columns >= n (the full row count is in L.counts)
            } else if (kBsr) {
                base = FEM_LDG(row_ptr + n);
                u = FEM_LDG(row_ptr + n + 1) - (int)base;
            } else {
                base = FEM_LDG(row_ptr + (size_t)n * DPN);
                u = (FEM_LDG(row_ptr + (size_t)n * DPN + 1) - (int)base) / DPN;
            }
        }
        // 1. gather the non-empty slots of the node's chunk chain (the first
        // chunk from the prefetched words)
        int T = 0;
        if (valid) {
#pragma unroll
            for (int q = 0; q < kPre; q++) {
                if (q * G < L.S1) {
                    const int s = q * G + glane;
                    const int col = s < L.S1 ? (pre_w[q] & kColMask) : 0;
                    const unsigned used = (__ballot_sync(gmask, col != 0) >> gshift) & gmask >> gshift;
                    const int e = T + __popc(used & ((1u << glane) - 1u));
                    if (col != 0 && e < NK)
                        s_keys[grp][e] = ((unsigned long long)(unsigned)(col - 1) << 32) | slot_gid(L, n, s);
                    T += __popc(used);
                }
            }
            int next = pre_next;
            for (int step = 1; next != 0 && step < kMaxChainSteps; step++) {
                const int c = next - 1;
                const int* meta = chunk_meta(L, c);
                const int cap = chunk_cap(L, c);
                next = FEM_LDG(meta + 1);
                for (int s0 = 0; s0 < cap; s0 += G) {
                    const int s = s0 + glane;
                    const int col = s < cap ? (FEM_LDG(meta + 2 + s) & kColMask) : 0;
                    const unsigned used = (__ballot_sync(gmask, col != 0) >> gshift) & gmask >> gshift;
                    const int e = T + __popc(used & ((1u << glane) - 1u));
                    if (col != 0 && e < NK)
                        s_keys[grp][e] = ((unsigned long long)(unsigned)(col - 1) << 32) | slot_gid(L, c, s);
                    T += __popc(used);
                }
            }
            const int expect = kMode == kOutUpper ? FEM_LDG(L.counts + n) : u;
            if (glane == 0 && (T != expect || u > T)) raise_status(L.info, FEM_ERR_INTERNAL);
        }
        if (nb + nb_stride < nb_end) prefetch_first_chunk<G, kPre>(L, nb + nb_stride + grp, glane, pre_w, pre_next);
        t_sum += T;
        t_max = max(t_max, T);
        const bool long_row = T > NK;
        const int Ts = long_row ? 0 : min(T, kMode == kOutUpper ? T : u);
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
        if constexpr (DPN == 2) {
            // all of the node's blocks in flight at once (two 16-byte loads each)
            for (int k = glane; k < Ts; k += G) {
                const double2* p = reinterpret_cast<const double2*>(L.vals + (size_t)(unsigned)s_keys[grp][k] * B);
                s_vals[grp][k][0] = FEM_LDG(p);
                s_vals[grp][k][1] = FEM_LDG(p + 1);
            }
            __syncwarp();
        }
        // entry v of the node's k-th sorted block
        auto block_value = [&](int k, int v) -> double {
            if constexpr (DPN == 2) return reinterpret_cast<const double*>(&s_vals[grp][k][0])[v];
            return FEM_LDG(L.vals + (size_t)(unsigned)s_keys[grp][k] * B + v);
        };
        // 3. write the dpn rows of the node (or its block row, or its upper rows)
        if (valid && kMode == kOutUpper) {
            if (long_row) {
                long_row_write_upper<DPN, G>(L, n, u, row_ptr, glane, gmask, col_idx, values);
            } else if (u > 0 && u <= Ts) {
                const int k0 = Ts - u;  // the sorted row's first column >= n (n itself)
                for (int a = 0; a < DPN; a++) {
                    const long long rbase = FEM_LDG(row_ptr + (size_t)n * DPN + a);
                    const int len = (u - 1) * DPN + (DPN - a);
                    for (int r = glane; r < len; r += G) {
                        int k, b;
                        if (r < DPN - a) {
                            k = k0;
                            b = a + r;
                        } else {
                            const int q = r - (DPN - a);
                            k = k0 + 1 + q / DPN;
                            b = q - (q / DPN) * DPN;
                        }
                        const unsigned long long key = s_keys[grp][k];
                        col_idx[rbase + r] = (int)(key >> 32) * DPN + b;
                        values[rbase + r] = block_value(k, a * DPN + b);
                    }
                }
            }
        } else if (valid && kBsr) {
            if (long_row) {
                long_row_write_bsr<DPN, G>(L, n, u, base, glane, gmask, col_idx, values);
            } else {
                for (int k = glane; k < Ts; k += G) col_idx[base + k] = (int)(s_keys[grp][k] >> 32);
                for (int idx = glane; idx < Ts * B; idx += G) {
                    const int k = idx / B, v = idx - k * B;
                    values[base * B + idx] = block_value(k, v);
                }
            }
        } else if (valid) {
            if (long_row) {
                long_row_write<DPN, G>(L, n, u, base, glane, gmask, col_idx, values);
            } else {
                const int row_len = DPN * Ts;
                for (int a = 0; a < DPN; a++) {
                    const long long rbase = base + (long long)a * DPN * u;
                    for (int r = glane; r < row_len; r += G) {
                        const int k = r / DPN, b = r - k * DPN;
                        const unsigned long long key = s_keys[grp][k];
                        col_idx[rbase + r] = (int)(key >> 32) * DPN + b;
                        values[rbase + r] = block_value(k, a * DPN + b);
                    }
                }
            }
        }
        __syncwarp();
    }
    // list statistics (one atomic per warp)
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
        t_max = max(t_max, __shfl_xor_sync(0xFFFFFFFFu, t_max, d));
        t_sum += __shfl_xor_sync(0xFFFFFFFFu, t_sum, d);
    }
    if ((tid & 31) == 0) {
        // every lane of a group counted the same rows: divide by G
        atomicAdd(reinterpret_cast<unsigned long long*>(&L.info->list_entries), (unsigned long long)(t_sum / G));
        atomicMax(&L.info->max_row_entries, t_max);
    }
}

}  // namespace
}  // namespace fem
