// Element stiffness matrices on their own (no assembly), in the packed
// symmetric block layout of fem_element_stiffness: for each element the upper
// node blocks (a <= b, row-major over the pairs), each dpn x dpn row-major.
//
// Replaces the reference's device element functions computeElementStiffness
// (ALLS_Quad2D_Assembly_Accuracy_Analysis.cu:178-212,
// ALLS_T3_Unstructed_Elements_Assemble_Performance.cu:136-206) and
// computeElementStiffnessHex20 (ALLS_Hex20_3D_Assembly_Performance.cu:130-195),
// which build a full Ke per thread (the Hex20 one a 60x60 FP32 array in 14.9 KB
// of local memory).
//
// 2-D (k_ke_2d): one lane per node block, as the A-LLS scatter computes it
// (FP64, or FP32 blocks with FEM_PREC_FP32).
//
// Hex20 (k_hex20_ke): one CTA (4 warps) per element at a time, persistent:
//   Jacobians at the 27 Gauss points (243 entries), their inverses and
//   w_g = weight * detJ_g (27 threads; a non-positive detJ raises
//   FEM_ERR_DETJ), physical gradients P[3n+a][g] (540 items), then
//   M = P diag(w) P^T on the FP64 tensor cores with mma.sync.m8n8k4.f64
//   (36 upper 8x8 tiles of the 64x64 padded product x 7 k-steps); each upper
//   entry of M is written to its upper 3x3 node block (so Ke is exactly
//   symmetric), and the 210 Ke blocks
//       Ke_IJ[a][b] = lambda M_IJ[a][b] + mu M_IJ[b][a] + mu delta_ab tr(M_IJ)
//   are written with coalesced stores. With FEM_PREC_FP64_SIMT the contraction
//   is plain FP64 dot products instead; FEM_PREC_TC_F16X3 runs the tcgen05
//   kernel of ke_tcgen05.cu. The Gauss-point shape derivatives
//   (H20:95-128) are tabulated once per CTA; the next element's nodes and
//   coordinates are loaded while the current one is computed.
#include <algorithm>

#include "element2d.cuh"
#include "hex20.cuh"

namespace fem {
namespace {

using namespace hex20;

constexpr int kThreads = 128;  // small CTAs: several elements' phases overlap on an SM
constexpr int kWarps = kThreads / 32;
constexpr int kTilesPerWarp = (36 + kWarps - 1) / kWarps;
constexpr int PS = 28;  // row stride of P (doubles): conflict-free m8n8k4 fragment loads

// The 36 upper 8x8 tiles (mt <= nt) of the 64x64 node-pair matrix.
__constant__ unsigned char c_tile_m[36] = {0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 1, 1, 1, 2, 2, 2,
                                           2, 2, 2, 3, 3, 3, 3, 3, 4, 4, 4, 4, 5, 5, 5, 6, 6, 7};
__constant__ unsigned char c_tile_n[36] = {0, 1, 2, 3, 4, 5, 6, 7, 1, 2, 3, 4, 5, 6, 7, 2, 3, 4,
                                           5, 6, 7, 3, 4, 5, 6, 7, 4, 5, 6, 7, 5, 6, 7, 6, 7, 7};

struct KeSmem {
    double dN[27][3][20];  // shape derivatives at the Gauss points
    union {
        double P[64][PS];          // P[3n+a][g] = G_g[n][a]; rows 60..63 and column 27 zeroed per element
        double Mb[kUpperBlocks][9];  // upper 3x3 node blocks of M
    };
    double X[20][3];  // element node coordinates
    double J[27][9];  // Jacobians, then their inverses
    double w[PS];     // Gauss weight * detJ (w[27] = 0 pads the contraction)
    double lam, mu;
    int bad;
};
static_assert(offsetof(KeSmem, Mb) % 16 == 0, "16-byte copies out of Mb");

__device__ __forceinline__ void dmma_8x8x4(double& c0, double& c1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(c0), "+d"(c1)
                 : "d"(a), "d"(b));
}

// kPrec: the node-pair contraction on the FP64 tensor cores (FEM_PREC_FP64)
// or as plain FP64 dot products on the CUDA cores (FEM_PREC_FP64_SIMT, the
// reference's arithmetic without tensor cores).
template <int kPrec>
__global__ void __launch_bounds__(kThreads, 5) k_hex20_ke(MeshView m, double* __restrict__ ke_out,
                                                          int* __restrict__ status) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    KeSmem& sm = *reinterpret_cast<KeSmem*>(smem_raw);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    for (int idx = tid; idx < 27 * 20; idx += kThreads) {
        const int g = idx / 20, n = idx % 20;
        double dx, dy, dz;
        dshape_node(n, gauss3(g / 9), gauss3((g / 3) % 3), gauss3(g % 3), dx, dy, dz);
        sm.dN[g][0][n] = dx;
        sm.dN[g][1][n] = dy;
        sm.dN[g][2][n] = dz;
    }
    if (tid < PS) sm.w[tid] = 0.0;
    // node id and coordinates of the next element, loaded a step ahead
    int pre_n = 0;
    double pre_x = 0.0, pre_y = 0.0, pre_z = 0.0;
    const int first = blockIdx.x, end = m.E_count;
    if (tid < 20 && first < end) {
        pre_n = __ldg(m.conn + (size_t)first * 20 + tid);
        if (pre_n >= 0 && pre_n < m.N) {
            pre_x = __ldg(m.x + pre_n);
            pre_y = __ldg(m.y + pre_n);
            pre_z = __ldg(m.z + pre_n);
        }
    }
    __syncthreads();

    for (int e = first; e < end; e += gridDim.x) {
        double* out = ke_out + (size_t)e * kPackedHex20;
        if (tid == 0) sm.bad = 0;
        __syncthreads();
        if (tid < 20) {
            if (pre_n < 0 || pre_n >= m.N) {
                sm.bad = 1;
            } else {
                sm.X[tid][0] = pre_x;
                sm.X[tid][1] = pre_y;
                sm.X[tid][2] = pre_z;
            }
        }
        if (tid == 32) {
            const double E = m.E ? __ldg(m.E + e) : m.E0;
            const double nu = m.nu ? __ldg(m.nu + e) : m.nu0;
            sm.lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
            sm.mu = E / (2.0 * (1.0 + nu));
        }
        __syncthreads();
        const int e_next = e + gridDim.x;
        if (tid < 20 && e_next < end) {
            pre_n = __ldg(m.conn + (size_t)e_next * 20 + tid);
            if (pre_n >= 0 && pre_n < m.N) {
                pre_x = __ldg(m.x + pre_n);
                pre_y = __ldg(m.y + pre_n);
                pre_z = __ldg(m.z + pre_n);
            }
        }
        if (sm.bad) {  // uniform: every thread reads the flag before anyone resets it
            if (tid == 0) atomicOr(status, 1 << FEM_ERR_BAD_MESH);
            for (int k = tid; k < kPackedHex20; k += kThreads) out[k] = 0.0;
            __syncthreads();
            continue;
        }
        // Jacobians: J[g][3i+j] = sum_n dN[g][i][n] X[n][j]
        for (int idx = tid; idx < 243; idx += kThreads) {
            const int g = idx / 9, r = idx % 9, i = r / 3, j = r % 3;
            double acc = 0.0;
#pragma unroll
            for (int n = 0; n < 20; n++) acc = fma(sm.dN[g][i][n], sm.X[n][j], acc);
            sm.J[g][r] = acc;
        }
        __syncthreads();
        if (tid < 27) {
            double* J = sm.J[tid];
            const double c0 = J[4] * J[8] - J[5] * J[7], c1 = J[5] * J[6] - J[3] * J[8], c2 = J[3] * J[7] - J[4] * J[6];
            const double det = J[0] * c0 + J[1] * c1 + J[2] * c2;
            if (!(det > 0.0)) atomicOr(status, 1 << FEM_ERR_DETJ);
            const double r = 1.0 / det;
            double iJ[9];
            iJ[0] = c0 * r;
            iJ[1] = (J[2] * J[7] - J[1] * J[8]) * r;
            iJ[2] = (J[1] * J[5] - J[2] * J[4]) * r;
            iJ[3] = c1 * r;
            iJ[4] = (J[0] * J[8] - J[2] * J[6]) * r;
            iJ[5] = (J[2] * J[3] - J[0] * J[5]) * r;
            iJ[6] = c2 * r;
            iJ[7] = (J[1] * J[6] - J[0] * J[7]) * r;
            iJ[8] = (J[0] * J[4] - J[1] * J[3]) * r;
#pragma unroll
            for (int k = 0; k < 9; k++) J[k] = iJ[k];
            sm.w[tid] = weight3(tid / 9) * weight3((tid / 3) % 3) * weight3(tid % 3) * det;
        }
        __syncthreads();
        // P aliases the previous element's M blocks: re-zero its padding.
        for (int idx = tid; idx < 4 * PS + 60; idx += kThreads) {
            if (idx < 4 * PS) (&sm.P[60][0])[idx] = 0.0;
            else sm.P[idx - 4 * PS][27] = 0.0;
        }
        // Physical gradients P[3n+a][g] = sum_i iJ[g][3a+i] dN[g][i][n]
        for (int idx = tid; idx < 27 * 20; idx += kThreads) {
            const int g = idx / 20, n = idx - 20 * g;
            const double* iJ = sm.J[g];
            const double d0 = sm.dN[g][0][n], d1 = sm.dN[g][1][n], d2 = sm.dN[g][2][n];
#pragma unroll
            for (int a = 0; a < 3; a++) sm.P[3 * n + a][g] = fma(iJ[3 * a], d0, fma(iJ[3 * a + 1], d1, iJ[3 * a + 2] * d2));
        }
        __syncthreads();
        if (kPrec == FEM_PREC_FP64_SIMT) {
            // every upper entry (r <= c < 60) of M as a plain FP64 dot product
            // over the 27 Gauss points; kept in registers until every thread
            // has read P, whose storage then takes the M blocks
            constexpr int kUpper = 60 * 61 / 2, kPer = (kUpper + kThreads - 1) / kThreads;
            double mv[kPer];
            int rc[kPer];
#pragma unroll
            for (int k = 0; k < kPer; k++) {
                const int idx = tid + k * kThreads;
                rc[k] = -1;
                mv[k] = 0.0;
                if (idx < kUpper) {
                    // row r of the upper triangle starts at r * 60 - r (r - 1) / 2
                    int r = (int)((121.0f - sqrtf(14641.0f - 8.0f * (float)idx)) * 0.5f);
                    while (r > 0 && r * 60 - r * (r - 1) / 2 > idx) r--;
                    while ((r + 1) * 60 - (r + 1) * r / 2 <= idx) r++;
                    const int c = r + (idx - (r * 60 - r * (r - 1) / 2));
                    double acc = 0.0;
                    for (int g = 0; g < 27; g++) acc = fma(sm.w[g] * sm.P[r][g], sm.P[c][g], acc);
                    mv[k] = acc;
                    rc[k] = r * 64 + c;
                }
            }
            __syncthreads();
#pragma unroll
            for (int k = 0; k < kPer; k++) {
                if (rc[k] < 0) continue;
                const int r = rc[k] >> 6, c = rc[k] & 63;
                const int I = r / 3, a = r - 3 * I, J = c / 3, b = c - 3 * J;
                sm.Mb[pair_index(I, J)][3 * a + b] = mv[k];
                if (I == J) sm.Mb[pair_index(I, I)][3 * b + a] = mv[k];
            }
        } else {
        // M = (P diag(w)) P^T on the FP64 tensor cores, upper 8x8 tiles only
        // (M is symmetric): the 36 tiles (mt <= nt) are dealt round-robin to the
        // warps.
        double acc[kTilesPerWarp][2];
#pragma unroll
        for (int q = 0; q < kTilesPerWarp; q++) acc[q][0] = acc[q][1] = 0.0;
        const int fr = lane >> 2, fc = lane & 3;
#pragma unroll
        for (int q = 0; q < kTilesPerWarp; q++) {
            const int t = warp + q * kWarps;
            if (t < 36) {
                const int mt = c_tile_m[t], nt = c_tile_n[t];
#pragma unroll
                for (int ks = 0; ks < 7; ks++) {
                    const int k = 4 * ks + fc;
                    dmma_8x8x4(acc[q][0], acc[q][1], sm.w[k] * sm.P[8 * mt + fr][k], sm.P[8 * nt + fr][k]);
                }
            }
        }
        __syncthreads();  // every warp has read P: its storage now takes the M blocks
#pragma unroll
        for (int q = 0; q < kTilesPerWarp; q++) {
            const int t = warp + q * kWarps;
            if (t < 36) {
                const int mt = c_tile_m[t], nt = c_tile_n[t];
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const int r = 8 * mt + fr, c = 8 * nt + 2 * fc + h;
                    // entry (r, c) stands for itself and, by symmetry, for (c, r);
                    // in a diagonal tile only r <= c writes (its mirror is in the tile)
                    if (r < 60 && c < 60 && (mt < nt || r <= c)) {
                        const int I = r / 3, a = r - 3 * I, J = c / 3, b = c - 3 * J;
                        if (I <= J) sm.Mb[pair_index(I, J)][3 * a + b] = acc[q][h];
                        if (J <= I) sm.Mb[pair_index(J, I)][3 * b + a] = acc[q][h];
                    }
                }
            }
        }
        }
        __syncthreads();
        // Ke upper blocks, consecutive threads on consecutive entries
        const double lam = sm.lam, mu = sm.mu;
        for (int k = tid; k < kPackedHex20; k += kThreads) {
            const int p = (k * 7282) >> 16;  // k / 9 for k < 1890
            const int v = k - 9 * p, a = (v * 11) >> 5, b = v - 3 * a;  // v / 3, v % 3
            const double* mb = sm.Mb[p];
            double ke = fma(lam, mb[v], mu * mb[3 * b + a]);
            if (a == b) ke = fma(mu, mb[0] + mb[4] + mb[8], ke);
            out[k] = ke;
        }
        __syncthreads();  // Mb / P storage is reused by the next element
    }
}

constexpr int kThreads2D = 256;

// One lane per upper node block (a <= b) of one 2-D element; a Q4 element
// takes 10 lanes, a T3 element 6 (its 4 block slots past the sixth are zeroed
// in a mixed mesh, whose stride is the Q4 one).
template <typename T>
__global__ void __launch_bounds__(kThreads2D) k_ke_2d(MeshView m, double* __restrict__ ke_out,
                                                      int* __restrict__ status) {
    constexpr int kLanes = 16;  // two elements per warp, up to 10 blocks each
    const int lane = threadIdx.x & 31, slot = lane / kLanes, sub = lane % kLanes;
    const int stride = m.types ? kPacked2D_Q4 : (m.stride == 4 ? kPacked2D_Q4 : kPacked2D_T3);
    const long long warp_id = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long num_warps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long base = warp_id * 2; base < m.E_count; base += num_warps * 2) {
        const long long e = base + slot;
        if (e >= m.E_count) continue;
        const bool q4 = m.types ? __ldg(m.types + e) == FEM_Q4 : m.stride == 4;
        const int npe = q4 ? 4 : 3, nblocks = q4 ? 10 : 6;
        double* out = ke_out + (size_t)e * stride + 4 * sub;
        if (sub >= nblocks) {
            if (sub < stride / 4) out[0] = out[1] = out[2] = out[3] = 0.0;
            continue;
        }
        // (a, b) of upper block index sub, row-major over a <= b
        int a = 0, r = sub;
        while (r >= npe - a) {
            r -= npe - a;
            a++;
        }
        const int b = a + r;
        int nodes[4];
        bool bad = false;
        for (int k = 0; k < npe; k++) {
            nodes[k] = __ldg(m.conn + (size_t)e * m.stride + k);
            bad |= nodes[k] < 0 || nodes[k] >= m.N;
        }
        const double E = m.E ? __ldg(m.E + e) : m.E0, nu = m.nu ? __ldg(m.nu + e) : m.nu0;
        double kv[4] = {0.0, 0.0, 0.0, 0.0};
        if (bad) {
            if (sub == 0) atomicOr(status, 1 << FEM_ERR_BAD_MESH);
        } else if (q4) {
            double xe[4], ye[4];
            for (int k = 0; k < 4; k++) {
                xe[k] = __ldg(m.x + nodes[k]);
                ye[k] = __ldg(m.y + nodes[k]);
            }
            const double det = ke_block_2d<4, T>(xe, ye, E, nu, m.t, a, b, kv);
            if (sub == 0 && !(det > 0.0)) atomicOr(status, 1 << FEM_ERR_DETJ);
        } else {
            double xe[3], ye[3];
            for (int k = 0; k < 3; k++) {
                xe[k] = __ldg(m.x + nodes[k]);
                ye[k] = __ldg(m.y + nodes[k]);
            }
            const double det = ke_block_2d<3, T>(xe, ye, E, nu, m.t, a, b, kv);
            if (sub == 0 && !(det > 0.0)) atomicOr(status, 1 << FEM_ERR_DETJ);
        }
        reinterpret_cast<double2*>(out)[0] = make_double2(kv[0], kv[1]);
        reinterpret_cast<double2*>(out)[1] = make_double2(kv[2], kv[3]);
    }
}

template <int kPrec>
cudaError_t launch_hex20_ke(const MeshView& m, double* ke_out, int* status, cudaStream_t s) {
    static DeviceCache cache;
    const size_t smem = sizeof(KeSmem);
    int blocks_per_sm = 0;
    const cudaError_t err = per_device(cache, [&](int& v) {
        cudaError_t e = cudaFuncSetAttribute(k_hex20_ke<kPrec>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (!e) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, k_hex20_ke<kPrec>, kThreads, smem);
        return e;
    }, blocks_per_sm);
    if (err) return err;
    const long long grid = std::min<long long>((long long)blocks_per_sm * sm_count(), m.E_count);
    k_hex20_ke<kPrec><<<(int)grid, kThreads, smem, s>>>(m, ke_out, status);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_element_stiffness(const MeshView& m, int kind, int precision, double* ke_out, int* status,
                                     long long wait_ns, cudaStream_t s) {
    if (m.E_count <= 0) return cudaSuccess;
    if (kind == FEM_HEX20) {
        if (precision == FEM_PREC_TC_F16X3) return launch_hex20_ke_tcgen05(m, ke_out, status, wait_ns, s);
        if (precision == FEM_PREC_FP64_SIMT) return launch_hex20_ke<FEM_PREC_FP64_SIMT>(m, ke_out, status, s);
        return launch_hex20_ke<FEM_PREC_FP64>(m, ke_out, status, s);
    } else {
        const long long warps = ((long long)m.E_count + 1) / 2;  // two elements per warp
        const int grid = (int)std::min<long long>((warps * 32 + kThreads2D - 1) / kThreads2D, (long long)sm_count() * 8);
        if (precision == FEM_PREC_FP32)
            k_ke_2d<float><<<grid > 0 ? grid : 1, kThreads2D, 0, s>>>(m, ke_out, status);
        else
            k_ke_2d<double><<<grid > 0 ? grid : 1, kThreads2D, 0, s>>>(m, ke_out, status);
    }
    return cudaGetLastError();
}

}  // namespace fem
