// Hex20 A-LLS scatter, pass 2 of 2: element stiffness in FP64 and the atomic
// accumulation of its blocks into the list entries that pass 1
// (claim_hex20.cu) claimed and mapped.
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
// triangle of the node grid is six tile positions; warp w owns one and
// computes all nine M^{ab} tiles there on the FP64 tensor cores
// (mma.sync.m8n8k4.f64: 9 x 7 per warp), so each lane holds, for its two
// (I, J) node pairs, all nine M^{ab}_IJ and forms Ke_IJ without exchanging
// anything with other lanes. It then adds Ke_IJ to the list entry of (row I,
// column J) and, for I != J, its transpose to the entry of (row J, column I):
// FP64 atomics at the slot ids of the slot map, so the 210 upper blocks give
// all 400 blocks of Ke exactly symmetrically.
//
// One 6-warp CTA per element at a time, persistent over the wave's elements
// (perm[i0, i1), the spatial order); the shape-function derivatives at the 27
// Gauss points (H20:95-128) are tabulated once per CTA; the next element's
// node ids and coordinates are loaded while the current one is computed.
#include <algorithm>

#include "values_hex20.cuh"

namespace fem {
namespace {

#ifndef FEM_VALUES_MIN_CTAS
#define FEM_VALUES_MIN_CTAS 3
#endif
constexpr int kThreads = kValueWarps * 32;

// kOut as values_cta. kToSlots: positions perm[i0, i1) of one wave, slot map
// row i - i0. kToCsrMap: all elements in the order perm (scatter map row e).
// kToCsrColour: the elements perm[range[0], range[1]) of one colour.
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

}  // namespace

cudaError_t launch_values_hex20_fp64(const MeshView& m, const ListLayout& L, const int* perm, int i0, int i1,
                                     const int* map, int ctas_per_sm, cudaStream_t s) {
    if (i1 <= i0) return cudaSuccess;
    ValuesTarget t{};
    t.map = map;
    t.map_origin = i0;
    t.vals = L.vals;
    t.info = L.info;
    return launch_values<kToSlots>(m, perm, i0, i1, nullptr, t, ctas_per_sm, s);
}

cudaError_t launch_values_hex20(const MeshView& m, const ListLayout& L, int precision, const int* perm, int i0,
                                int i1, const int* map, int ctas_per_sm, long long wait_ns, cudaStream_t s) {
    return precision == FEM_PREC_TC_F16X3 ? launch_values_hex20_tc(m, L, perm, i0, i1, map, wait_ns, s)
                                          : launch_values_hex20_fp64(m, L, perm, i0, i1, map, ctas_per_sm, s);
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
