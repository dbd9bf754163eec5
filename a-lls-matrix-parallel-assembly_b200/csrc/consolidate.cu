// List -> CSR consolidation: per-row counts -> device scan -> row_ptr, then a
// per-row sort and coalesced write of col_idx / values.
//
// Replaces both the reference's host pattern build (buildCSRStructure,
// ALLS_Quad2D_Assembly_Accuracy_Analysis.cu:605-645; buildCSRStructureHex20,
// ALLS_Hex20_3D_Assembly_Performance.cu:364-392) and its convert kernels
// (convertALLStoCSRKernel, Q4A:471-501; ...FixedArray, H20:259-278), which walk
// each row's list and binary-search the host-built col_ind.
//
// The scatter inserts every column once per row and counts the entries of each
// row node in counts[n], so the CSR layout is known before any list is read:
//   k_scan_reduce  per tile of 4096 nodes: sum of dpn^2 * counts
//   k_scan_tiles   one CTA: exclusive scan of the tile sums, nnz, capacity check
//   k_row_ptr      per tile: block scan of counts -> row_ptr of all dpn rows
//   k_write        a group of G lanes per row node: gather the node's non-empty
//                  hashed slots as 64-bit keys (col << 32 | slot), bitonic sort
//                  across the group, then write each dof row's entries
//                  (col*dpn + b, block value) with consecutive lanes on
//                  consecutive entries. Rows longer than the group's sort
//                  capacity take an exact slow path.
// Every dof row of node n holds {c*dpn + b : c in adj(n)} in increasing order,
// which is the reference's pattern. The same pass can write the node-block
// (BSR) form instead: one block row per node, the sorted column nodes and
// their dpn x dpn blocks; or the upper triangle only (columns >= row, the
// symmetric storage a Cholesky or symmetric solver reads): k_count_upper
// counts each node's columns >= the node, the scan and row pointers use those
// counts, and k_write keeps the tail of each sorted row.
#include <algorithm>

#include "consolidate.cuh"

namespace fem {
namespace {

template <int B>
__global__ void __launch_bounds__(kScanThreads) k_scan_reduce(const int* __restrict__ counts, int N,
                                                              long long* __restrict__ tile_sums) {
    __shared__ long long s_warp[kScanThreads / 32 + 1];
    scan_reduce_tile<B>(counts, N, tile_sums, blockIdx.x, s_warp);
}

__global__ void __launch_bounds__(kScanThreads) k_scan_tiles(long long* __restrict__ tile_sums, int num_tiles,
                                                             DevInfo* info, int* __restrict__ row_ptr_end,
                                                             long long capacity, int end_div) {
    __shared__ long long s_warp[kScanThreads / 32 + 1];
    scan_tiles_body(tile_sums, num_tiles, info, row_ptr_end, capacity, end_div, s_warp);
}

template <int DPN, bool kBsr>
__global__ void __launch_bounds__(kScanThreads) k_row_ptr(const int* __restrict__ counts, int N,
                                                          const long long* __restrict__ tile_offsets,
                                                          int* __restrict__ row_ptr) {
    __shared__ long long s_warp[kScanThreads / 32 + 1];
    row_ptr_tile<DPN, kBsr>(counts, N, tile_offsets, row_ptr, blockIdx.x, s_warp);
}

template <int DPN, int G, int KPL, int kMode>
__global__ void __launch_bounds__(kBlockThreads, DPN == 2 ? FEM_WRITE_MIN_CTAS_2D : FEM_WRITE_MIN_CTAS_3D)
    k_write(ListLayout L, const int* __restrict__ row_ptr, int* __restrict__ col_idx, double* __restrict__ values,
            long long capacity, const int* __restrict__ ucounts) {
    constexpr int NPB = kBlockThreads / G;  // nodes per batch
    __shared__ WriteSmem<DPN, G, KPL> sm;
    write_batches<DPN, G, KPL, kMode>(L, row_ptr, col_idx, values, capacity, ucounts, (long long)blockIdx.x * NPB,
                                      (long long)gridDim.x * NPB, L.N, sm);
}

__global__ void k_info_init(DevInfo* info, int pool_chunks) {
    info->pool_chunks = pool_chunks;
}

// Clears what a consolidation pass owns, so the pass can be re-run on the same
// lists (e.g. after FEM_ERR_CAPACITY with larger output buffers).
__global__ void k_consolidate_reset(DevInfo* info) {
    constexpr int kOwned = (1 << FEM_ERR_CAPACITY) | (1 << FEM_ERR_RANGE) | (1 << FEM_ERR_INTERNAL);
    info->status_bits &= ~kOwned;
    info->nnz = 0;
    info->list_entries = 0;
    info->max_row_entries = 0;
}

// Persistent grid of k_write: the CTAs that fit on the GPU at once.
template <int DPN, int G, int KPL, int kMode>
long long write_grid(long long batches) {
    static DeviceCache cache;
    int per_sm = 0;
    if (per_device(cache, [](int& v) {
            return cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, k_write<DPN, G, KPL, kMode>, kBlockThreads, 0);
        }, per_sm))
        per_sm = 1;
    return std::max<long long>(1, std::min<long long>(batches, (long long)per_sm * sm_count()));
}

template <int DPN, int G, int KPL, bool kBsr>
cudaError_t launch_all(const ListLayout& L, int* row_ptr, int* col_idx, double* values, long long capacity,
                       long long* tile_sums, int num_tiles, cudaStream_t s) {
    constexpr int kMode = kBsr ? kOutBsr : kOutCsr;
    // capacity is in scalar entries (BSR: blocks * dpn^2)
    k_consolidate_reset<<<1, 1, 0, s>>>(L.info);
    k_scan_reduce<DPN * DPN><<<num_tiles, kScanThreads, 0, s>>>(L.counts, L.N, tile_sums);
    k_scan_tiles<<<1, kScanThreads, 0, s>>>(tile_sums, num_tiles, L.info, row_ptr + (size_t)L.N * (kBsr ? 1 : DPN),
                                            capacity, kBsr ? DPN * DPN : 1);
    k_row_ptr<DPN, kBsr><<<num_tiles, kScanThreads, 0, s>>>(L.counts, L.N, tile_sums, row_ptr);
    if (capacity > 0) {
        constexpr int NPB = kBlockThreads / G;
        const long long batches = ((long long)L.N + NPB - 1) / NPB;
        k_write<DPN, G, KPL, kMode><<<(int)write_grid<DPN, G, KPL, kMode>(batches), kBlockThreads, 0, s>>>(
            L, row_ptr, col_idx, values, capacity, nullptr);
    }
    return cudaGetLastError();
}

template <int DPN, int G, int KPL>
cudaError_t launch_upper(const ListLayout& L, int* ucounts, int* row_ptr, int* col_idx, double* values,
                         long long capacity, long long* tile_sums, int num_tiles, cudaStream_t s) {
    constexpr int NPB = kBlockThreads / G;
    const long long batches = ((long long)L.N + NPB - 1) / NPB;
    const int grid = (int)std::max<long long>(1, std::min<long long>(batches, (long long)sm_count() * 8));
    k_consolidate_reset<<<1, 1, 0, s>>>(L.info);
    k_count_upper<G><<<grid, kBlockThreads, 0, s>>>(L, ucounts);
    k_scan_reduce_upper<DPN><<<num_tiles, kScanThreads, 0, s>>>(ucounts, L.N, tile_sums);
    k_scan_tiles<<<1, kScanThreads, 0, s>>>(tile_sums, num_tiles, L.info, row_ptr + (size_t)L.N * DPN, capacity, 1);
    k_row_ptr_upper<DPN><<<num_tiles, kScanThreads, 0, s>>>(ucounts, L.N, tile_sums, row_ptr);
    if (capacity > 0)
        k_write<DPN, G, KPL, kOutUpper><<<(int)write_grid<DPN, G, KPL, kOutUpper>(batches), kBlockThreads, 0, s>>>(
            L, row_ptr, col_idx, values, capacity, ucounts);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_consolidate(const ListLayout& L, int dpn, int* row_ptr, int* col_idx, double* values,
                               long long capacity, long long* tile_sums, int num_tiles, cudaStream_t s) {
    if (dpn == 3) return launch_all<3, 32, 4, false>(L, row_ptr, col_idx, values, capacity, tile_sums, num_tiles, s);
    return launch_all<2, 8, 2, false>(L, row_ptr, col_idx, values, capacity, tile_sums, num_tiles, s);
}

cudaError_t launch_consolidate_upper(const ListLayout& L, int dpn, int* ucounts, int* row_ptr, int* col_idx,
                                     double* values, long long capacity, long long* tile_sums, int num_tiles,
                                     cudaStream_t s) {
    if (dpn == 3) return launch_upper<3, 32, 4>(L, ucounts, row_ptr, col_idx, values, capacity, tile_sums, num_tiles, s);
    return launch_upper<2, 8, 2>(L, ucounts, row_ptr, col_idx, values, capacity, tile_sums, num_tiles, s);
}

cudaError_t launch_consolidate_bsr(const ListLayout& L, int dpn, int* block_row_ptr, int* block_col_idx,
                                   double* block_values, long long capacity_blocks, long long* tile_sums,
                                   int num_tiles, cudaStream_t s) {
    const long long cap = capacity_blocks * dpn * dpn;
    if (dpn == 3)
        return launch_all<3, 32, 4, true>(L, block_row_ptr, block_col_idx, block_values, cap, tile_sums, num_tiles, s);
    return launch_all<2, 8, 2, true>(L, block_row_ptr, block_col_idx, block_values, cap, tile_sums, num_tiles, s);
}

cudaError_t launch_info_init(DevInfo* info, int pool_chunks, cudaStream_t s) {
    k_info_init<<<1, 1, 0, s>>>(info, pool_chunks);
    return cudaGetLastError();
}

}  // namespace fem
