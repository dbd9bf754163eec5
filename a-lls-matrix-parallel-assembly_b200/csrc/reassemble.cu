// Value-only re-assembly: a mesh whose connectivity is unchanged (new
// coordinates, E or nu, as in nonlinear or time-stepping solvers) is
// re-assembled into the CSR pattern of an earlier assembly without building
// any list: a scatter map records, for every element node block (a, b), the
// CSR position of its first entry, and the element blocks are added there
// with FP64 atomics.
//
// The reference has no such path: every assembly repeats the list build
// (assembleGlobalStiffnessKernelALLS, ALLS_Quad2D_Assembly_Accuracy_Analysis.cu:394-468)
// and, on the host, the pattern (buildCSRStructure, Q4A:605-645).
//
// Map layout (int32): [E * G] block positions, G = npe^2 (Q4 and mixed 16,
// T3 9, Hex20 400), position of block (a, b) of element e at e * G + a * npe + b;
// then the element visit order [E] and its scratch (element-type ranges,
// bucket histogram, bounding box), built with the same element order as the
// A-LLS scatter. Entry (i, j) of block (a, b) lies at p + i * rowlen + j,
// rowlen being the length of the block's first CSR row (the dpn rows of a node
// have the same columns).
#include <algorithm>

#include "element2d.cuh"
#include "launch.h"

namespace fem {
namespace {

constexpr int kThreads = 256;

// Position of column col in CSR row r (sorted), or -1.
__device__ __forceinline__ int find_col(const int* __restrict__ row_ptr, const int* __restrict__ col_idx, int r,
                                        int col) {
    int lo = __ldg(row_ptr + r), hi = __ldg(row_ptr + r + 1) - 1;
    while (lo <= hi) {
        const int mid = (lo + hi) >> 1;
        const int c = __ldg(col_idx + mid);
        if (c == col) return mid;
        if (c < col) lo = mid + 1;
        else hi = mid - 1;
    }
    return -1;
}

__device__ __forceinline__ int npe_of(const MeshView& m, int e) {
    if (m.types) return __ldg(m.types + e) == FEM_Q4 ? 4 : 3;
    return m.stride == 20 ? 20 : m.stride;
}

// One thread per (element, block): binary search of the block's first column
// in its first row. Blocks past the element's nodes (T3 in a mixed mesh) get -1.
__global__ void k_build_map(MeshView m, int dpn, int npe_max, const int* __restrict__ row_ptr,
                            const int* __restrict__ col_idx, int* __restrict__ map, int* __restrict__ status) {
    const int G = npe_max * npe_max;
    const long long total = (long long)m.E_count * G;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const int e = (int)(t / G), k = (int)(t - (long long)e * G);
        const int a = k / npe_max, b = k - a * npe_max;
        const int npe = npe_of(m, e);
        int pos = -1;
        if (a < npe && b < npe) {
            const int na = __ldg(m.conn + (size_t)e * m.stride + a), nb = __ldg(m.conn + (size_t)e * m.stride + b);
            if (na < 0 || na >= m.N || nb < 0 || nb >= m.N) {
                atomicOr(status, 1 << FEM_ERR_BAD_MESH);
            } else {
                pos = find_col(row_ptr, col_idx, dpn * na, dpn * nb);
                if (pos < 0) atomicOr(status, 1 << FEM_ERR_INTERNAL);  // the pattern lacks the block
            }
        }
        map[t] = pos;
    }
}

// 2-D value-only assembly: one lane per element block (NPE^2 lanes per
// element), elements perm[range[0], range[1]), FP64 red.add into the values.
template <int NPE, typename T>
__global__ void __launch_bounds__(kThreads) k_reassemble_2d(MeshView m, const int* __restrict__ map, int G,
                                                            const int* __restrict__ perm, const int* __restrict__ range,
                                                            const int* __restrict__ row_ptr,
                                                            double* __restrict__ values, int* __restrict__ status) {
    constexpr int GL = NPE * NPE, EPW = 32 / GL;
    const int lane = threadIdx.x & 31;
    const int eslot = lane / GL, sub = lane - eslot * GL, a = sub / NPE, b = sub - (sub / NPE) * NPE;
    const int begin = range[0], count = range[1] - range[0];
    const long long warp_id = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long stride = (((long long)gridDim.x * blockDim.x) >> 5) * EPW;
    for (long long i = warp_id * EPW + eslot; i - eslot < count; i += stride) {
        if (eslot >= EPW || i >= count) continue;
        const int e = __ldg(perm + begin + i);
        const int p = __ldg(map + (size_t)e * G + a * (G == 16 ? 4 : NPE) + b);
        if (p < 0) continue;  // bad node (reported when the map was built)
        int nodes[NPE];
#pragma unroll
        for (int k = 0; k < NPE; k++) nodes[k] = __ldg(m.conn + (size_t)e * m.stride + k);
        double xe[NPE], ye[NPE];
#pragma unroll
        for (int k = 0; k < NPE; k++) {
            xe[k] = __ldg(m.x + nodes[k]);
            ye[k] = __ldg(m.y + nodes[k]);
        }
        const double E = m.E ? __ldg(m.E + e) : m.E0;
        const double nu = m.nu ? __ldg(m.nu + e) : m.nu0;
        double kv[4];
        const double det = ke_block_2d<NPE, T>(xe, ye, E, nu, m.t, a, b, kv);
        if (sub == 0 && !(det > 0.0)) atomicOr(status, 1 << FEM_ERR_DETJ);
        int row = nodes[0];
#pragma unroll
        for (int k = 1; k < NPE; k++) row = a == k ? nodes[k] : row;
        const int len = __ldg(row_ptr + 2 * row + 1) - __ldg(row_ptr + 2 * row);
        atomicAdd(values + p, kv[0]);
        atomicAdd(values + p + 1, kv[1]);
        atomicAdd(values + p + len, kv[2]);
        atomicAdd(values + p + len + 1, kv[3]);
    }
}

}  // namespace

cudaError_t launch_build_map(const MeshView& m, int kind, const int* row_ptr, const int* col_idx, int* map,
                             int* status, cudaStream_t s) {
    const int npe_max = kind == FEM_HEX20 ? 20 : (kind == FEM_T3 ? 3 : 4);
    const int dpn = kind == FEM_HEX20 ? 3 : 2;
    const long long total = (long long)m.E_count * npe_max * npe_max;
    if (total == 0) return cudaSuccess;
    const int grid = (int)std::min<long long>((total + kThreads - 1) / kThreads, (long long)sm_count() * 16);
    k_build_map<<<grid, kThreads, 0, s>>>(m, dpn, npe_max, row_ptr, col_idx, map, status);
    return cudaGetLastError();
}

template <typename T>
void reassemble_2d_t(const MeshView& m, const int* map, int G, const int* perm, const int* ranges, const int* row_ptr,
                     double* values, int* status, cudaStream_t s) {
    const bool has_q4 = m.types || m.stride == 4, has_t3 = m.types || m.stride == 3;
    const long long warps = ((long long)m.E_count + 1) / 2;
    const int grid = (int)std::min<long long>((warps * 32 + kThreads - 1) / kThreads, (long long)sm_count() * 8);
    if (has_q4)
        k_reassemble_2d<4, T><<<grid > 0 ? grid : 1, kThreads, 0, s>>>(m, map, G, perm, ranges + 0, row_ptr, values,
                                                                      status);
    if (has_t3)
        k_reassemble_2d<3, T><<<grid > 0 ? grid : 1, kThreads, 0, s>>>(m, map, G, perm, ranges + 2, row_ptr, values,
                                                                      status);
}

cudaError_t launch_reassemble_2d(const MeshView& m, int precision, const int* map, int G, const int* perm,
                                 const int* ranges, const int* row_ptr, double* values, int* status, cudaStream_t s) {
    if (precision == FEM_PREC_FP32)
        reassemble_2d_t<float>(m, map, G, perm, ranges, row_ptr, values, status, s);
    else
        reassemble_2d_t<double>(m, map, G, perm, ranges, row_ptr, values, status, s);
    return cudaGetLastError();
}

}  // namespace fem
