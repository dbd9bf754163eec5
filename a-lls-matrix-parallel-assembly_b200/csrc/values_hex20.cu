// Hex20 A-LLS scatter, pass 2 of 2: element stiffness in FP64 and the
// accumulation of its blocks into the list entries that pass 1
// (claim_hex20.cu) claimed and recorded in the groups' map records; also the
// CTA-cooperative element pass of the value-only re-assembly and of the
// colouring baseline.
//
// Replaces the value half of assembleGlobalStiffnessKernelALLSFixedArray
// (ALLS_Hex20_3D_Assembly_Performance.cu:212-256: one thread per element with
// its 60x60 FP32 Ke in 14.9 KB of local memory, atomicAdd(float) per entry)
// and its element routine computeElementStiffnessHex20 (H20:130-195).
//
// Element stiffness in direction-major form. With G_a (20 x 27) the physical
// shape-function gradients along direction a at the Gauss points and
// w_g = gauss weight * detJ_g, the nine 20 x 20 node-pair matrices
//     M^{ab} = G_a diag(w) G_b^T                    (a, b in x, y, z)
// give every 3x3 node block of the isotropic stiffness entry by entry,
//     Ke_IJ[a][b] = lambda M^{ab}_IJ + mu M^{ba}_IJ + mu delta_ab (M^{xx} + M^{yy} + M^{zz})_IJ,
// which is the reference's per-Gauss-point block formula (H20:173-191) summed
// over the Gauss points. Padded to 24 x 24 (8x8 tiles) and K = 28, the upper
// triangle of the node grid is six tile positions, each with nine M^{ab}
// tiles on the FP64 tensor cores (mma.sync.m8n8k4.f64, seven k-steps), so a
// lane holds, for its two (I, J) node pairs of a tile, all nine M^{ab}_IJ and
// forms Ke_IJ without exchanging anything with other lanes.
//
// Group value pass (k_values_group): one CTA of kGroup warps per element
// group, persistent over the wave's groups. Warp w computes the Ke of the
// group's element w alone: the lanes' gradients G_a(n, g) for the fragment
// rows n = 8 t + lane / 4 and k-columns g = 4 s + lane % 4 are the same
// values for the A and the B operands, so they stay in registers (63 per
// lane) and all six tile positions run from registers. Each of the 210 upper
// blocks is stored, already oriented as it adds to its node pair (the block,
// its transpose, or block + transpose for a repeated node), at its position
// in the group's pair-major block order (from the claim pass's record): one
// writer per position, plain shared stores. After a barrier, three threads
// per node pair sum the pair's contiguous blocks, one row each, so a pair
// that several of the group's elements share leaves the CTA once, and write
// the sum to the slot of (row u, column v) and its transpose to (row v,
// column u): a plain store for a pair only this group has (its slots were
// not zeroed), an FP64 atomic add for a shared pair (zeroed by its claimer).
// The tensor-core form computes the wave's Ke in ke_tcgen05.cu into a staging
// buffer first, and the same kernel stages those blocks instead.
//
// Element pass (k_values_hex20, kToCsrMap / kToCsrColour): one 6-warp CTA
// per element at a time, warp w owning tile position w; the shape-function
// derivatives at the 27 Gauss points (H20:95-128) are tabulated once per CTA
// and the next element's node ids and coordinates are loaded while the
// current one is computed.
#include <algorithm>

#include "values_group.cuh"

namespace fem {
namespace {

#ifndef FEM_VALUES_MIN_CTAS
#define FEM_VALUES_MIN_CTAS 3
#endif
constexpr int kThreads = kValueWarps * 32;

// kOut as values_cta (kToCsrMap: all elements in the order perm, scatter map
// row e; kToCsrColour: the elements perm[range[0], range[1]) of one colour).
template <int kOut>
__global__ void __launch_bounds__(kThreads, FEM_VALUES_MIN_CTAS)
    k_values_hex20(MeshView m, const int* __restrict__ perm, int i0, int i1, const int* __restrict__ range,
                   ValuesTarget t) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ValuesSmem& sm = *reinterpret_cast<ValuesSmem*>(smem_raw);
    if (range) {
        i0 = range[0];
        i1 = range[1];
    }
    values_init(sm);
    values_cta<kOut>(m, perm, (long long)i0 + blockIdx.x, gridDim.x, i1, t, sm);
}

template <int kOut>
cudaError_t launch_values(const MeshView& m, const int* perm, int i0, int i1, const int* range, const ValuesTarget& t,
                          int ctas_per_sm, cudaStream_t s) {
    static DeviceCache cache;
    const size_t smem = sizeof(ValuesSmem);
    int per_sm = 0;
    const cudaError_t err = per_device(cache, [&](int& v) {
        cudaError_t e =
            cudaFuncSetAttribute(k_values_hex20<kOut>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (!e) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, k_values_hex20<kOut>, kThreads, smem);
        return e;
    }, per_sm);
    if (err) return err;
    const int use = ctas_per_sm > 0 ? std::min(ctas_per_sm, per_sm) : per_sm;
    const long long count = range ? m.E_count : i1 - i0;  // a colour's size is on the device: bound by E
    const long long grid = std::max<long long>(1, std::min<long long>(count, (long long)use * sm_count()));
    k_values_hex20<kOut><<<(int)grid, kThreads, smem, s>>>(m, perm, i0, i1, range, t);
    return cudaGetLastError();
}

constexpr int kGroupThreads = kGroup * 32;

__global__ void __launch_bounds__(kGroupThreads, 1)
    k_values_group(MeshView m, int i0, int i1, const int* __restrict__ recs, const double* __restrict__ stage,
                   double* vals, DevInfo* info) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    GroupValuesSmem& sm = *reinterpret_cast<GroupValuesSmem*>(smem_raw);
    values_group_init(sm);
    values_group(m, i0, i1, recs, stage, vals, info, sm);
}

cudaError_t launch_group_values(const MeshView& m, const ListLayout& L, int i0, int i1, const int* recs,
                                const double* stage, cudaStream_t s) {
    static DeviceCache cache;
    const size_t smem = sizeof(GroupValuesSmem);
    int per_sm = 0;
    const cudaError_t err = per_device(cache, [&](int& v) {
        cudaError_t e = cudaFuncSetAttribute(k_values_group, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (!e) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, k_values_group, kGroupThreads, smem);
        return e;
    }, per_sm);
    if (err) return err;
    const long long groups = (i1 - i0 + kGroup - 1) / kGroup;
    const long long grid = std::max<long long>(1, std::min<long long>(groups, (long long)per_sm * sm_count()));
    k_values_group<<<(int)grid, kGroupThreads, smem, s>>>(m, i0, i1, recs, stage, L.vals, L.info);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_values_hex20(const MeshView& m, const ListLayout& L, int precision, const int* perm, int i0,
                                int i1, const int* map, double* stage, long long wait_ns, cudaStream_t s) {
    if (i1 <= i0) return cudaSuccess;
    if (precision == FEM_PREC_TC_F16X3) {
        cudaError_t err = launch_stage_hex20_tc(m, perm, i0, i1, stage, &L.info->status_bits, wait_ns, s);
        return err ? err : launch_group_values(m, L, i0, i1, map, stage, s);
    }
    return launch_group_values(m, L, i0, i1, map, nullptr, s);
}

cudaError_t launch_reassemble_hex20(const MeshView& m, int precision, const int* perm, const MapTarget& mt,
                                    DevInfo* info, cudaStream_t s) {
    if (m.E_count <= 0) return cudaSuccess;
    if (precision == FEM_PREC_TC_F16X3) return launch_reassemble_hex20_tc(m, perm, mt, info, s);
    ValuesTarget t{};
    t.map = mt.map;
    t.row_ptr = mt.row_ptr;
    t.csr = mt.values;
    t.info = info;
    return launch_values<kToCsrMap>(m, perm, 0, m.E_count, nullptr, t, 0, s);
}

cudaError_t launch_colour_hex20(const MeshView& m, const int* perm, const int* range, const MapTarget& mt,
                                DevInfo* info, cudaStream_t s) {
    ValuesTarget t{};
    t.row_ptr = mt.row_ptr;
    t.col_idx = mt.col_idx;
    t.csr = mt.values;
    t.info = info;
    return launch_values<kToCsrColour>(m, perm, 0, 0, range, t, 0, s);
}

}  // namespace fem
