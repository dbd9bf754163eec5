// Host-side launchers of the assembler kernels (internal to the library).
#pragma once

#include <cuda_runtime.h>

#include "fem_internal.cuh"

namespace fem {

struct MeshView {
    const double* x;
    const double* y;
    const double* z;
    const int* conn;
    const unsigned char* types;
    const double* E;
    const double* nu;
    double E0, nu0, t;
    int N;       // nodes
    int E_count; // elements
    int stride;  // ints per connectivity row
};

// 2-D chunk rows are 16 int32 words (14 slots + fill + next).
constexpr int k2DSlots = 14;

cudaError_t launch_scatter_2d(const MeshView& m, const ListLayout& L, int npe, const int* elist,
                              const int* ecount, cudaStream_t s);
cudaError_t launch_partition_2d(const MeshView& m, int* list_q4, int* list_t3, int* counts, cudaStream_t s);
cudaError_t launch_scatter_hex20(const MeshView& m, const ListLayout& L, cudaStream_t s);
cudaError_t launch_consolidate(const ListLayout& L, int dpn, int* row_ptr, int* col_idx, double* values,
                               long long capacity, unsigned long long* tile_state, int num_tiles,
                               cudaStream_t s);
cudaError_t launch_info_init(DevInfo* info, int pool_chunks, cudaStream_t s);

// Nodes handled by one consolidation tile (one CTA).
inline int consolidate_nodes_per_tile(int dpn) { return dpn == 3 ? 8 : 16; }

}  // namespace fem
