// K1 for 2-D meshes: fused Q4 / T3 element stiffness + A-LLS row-list scatter.
//
// Replaces assembleGlobalStiffnessKernelALLS
// (ALLS_Quad2D_Assembly_Accuracy_Analysis.cu:394-468,
//  ALLS_T3_Unstructed_Elements_Assemble_Performance.cu:227-290,
//  ALLS_Q4_T3_Mixed_Elements_Assembly_Performance.cu:248-312), which runs one
// thread per element and walks a pointer list for each of its ndof^2 entries.
//
// Here one LANE serves one node block (a, b) of one element: NPE^2 lanes per
// element (T3: 9 lanes, 3 elements per warp; Q4: 16 lanes, 2 per warp).
//  * Every lane loads the element's nodes and coordinates (same addresses
//    across the element's lanes, so the loads are shared) and computes its own
//    2x2 block K_ab in FP64 (element2d.cuh).
//  * It reads row node a's 64-byte first chunk (next pointer and 14 hashed
//    slots) with four 16-byte L2 loads and looks for column node b in it. An
//    absent column is claimed with atomicCAS(empty -> col) at the first empty
//    slot of its probe sequence; a CAS that meets another column marks that
//    slot taken in the lane's view and moves on along the sequence (slots are
//    never freed, so a column is always found or placed at the first empty
//    slot of its sequence, never twice). A chunk whose probe sequence is full
//    continues in an overflow chunk (allocated from the pool with zeroed
//    values, linked by CAS).
//  * The values of every slot start at zero (the first chunks' values are
//    cleared before the launch), so the claimer and every later contributor
//    alike add their block with FP64 red.add: the claim publishes the column
//    at once, with no pending state, no fence and no waiting on another
//    thread. The warp transposes its blocks through shared memory so that each
//    red instruction covers eight whole 32-byte blocks (four consecutive lanes
//    per block) instead of 32 scattered sectors.
//  * Claims are counted per (element, row) group with one atomic per group.
// Elements are visited in the node-local order of reorder.cu, so the rows that
// a warp touches are close together and stay in L2.
// The reference's head insert can lose a contribution or insert a column
// twice (Q4A:452-463); the claim/publish protocol above does neither.
#include <algorithm>

#include "scatter2d.cuh"

namespace fem {
namespace {

template <int NPE, typename T>
__global__ void __launch_bounds__(kThreads2D, NPE == 3 ? FEM_T3_MIN_CTAS : FEM_Q4_MIN_CTAS)
    k_scatter_2d(MeshView m, ListLayout L, const int* __restrict__ perm, const int* __restrict__ range) {
    __shared__ Scatter2DWarpSmem sm[kWarps2D];
    const long long warp_id = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long num_warps = ((long long)gridDim.x * blockDim.x) >> 5;
    scatter2d_warp<NPE, T>(m, L, perm, range[0], range[1] - range[0], warp_id, num_warps, sm[threadIdx.x >> 5]);
}

}  // namespace

template <int NPE, typename T>
cudaError_t launch_scatter_2d_t(const MeshView& m, const ListLayout& L, const int* perm, const int* range,
                                int ctas_per_sm, cudaStream_t s) {
    // A persistent grid: every warp runs the pipeline over many elements.
    static DeviceCache cache;
    int per_sm = 0;
    cudaError_t err = per_device(cache, [](int& v) {
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, k_scatter_2d<NPE, T>, kThreads2D, 0);
    }, per_sm);
    if (err) return err;
    const int use = ctas_per_sm > 0 ? std::min(ctas_per_sm, per_sm) : per_sm;
    constexpr int epw = 32 / (NPE * NPE);
    const long long warps = ((long long)m.E_count + epw - 1) / epw;
    const long long want = (warps + kWarps2D - 1) / kWarps2D;
    const int grid = (int)std::min<long long>(want > 0 ? want : 1, (long long)use * sm_count());
    k_scatter_2d<NPE, T><<<grid, kThreads2D, 0, s>>>(m, L, perm, range);
    return cudaGetLastError();
}

cudaError_t launch_scatter_2d(const MeshView& m, const ListLayout& L, int npe, int precision, const int* perm,
                              const int* range, int ctas_per_sm, cudaStream_t s) {
    if (precision == FEM_PREC_FP32)
        return npe == 4 ? launch_scatter_2d_t<4, float>(m, L, perm, range, ctas_per_sm, s)
                        : launch_scatter_2d_t<3, float>(m, L, perm, range, ctas_per_sm, s);
    return npe == 4 ? launch_scatter_2d_t<4, double>(m, L, perm, range, ctas_per_sm, s)
                    : launch_scatter_2d_t<3, double>(m, L, perm, range, ctas_per_sm, s);
}

}  // namespace fem
