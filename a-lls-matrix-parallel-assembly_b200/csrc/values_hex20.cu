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

#include "hex20.cuh"

namespace fem {
namespace {

constexpr int kWarps = 6;
constexpr int kThreads = kWarps * 32;
constexpr int KS = 28;  // Gauss points padded to 7 k-steps of 4; row stride of the tables (doubles)

// The six 8x8 tile positions (ti <= tj) of the upper triangle of the 24 x 24 node grid.
__constant__ unsigned char c_ti[kWarps] = {0, 0, 0, 1, 1, 2};
__constant__ unsigned char c_tj[kWarps] = {0, 1, 2, 1, 2, 2};

struct ValuesSmem {
    double dN[3][20][KS];  // dN_n / dxi_i at Gauss point g: [i][n][g]
    double G[3][24][KS];   // physical gradients: [a][n][g]; rows 20..23 and g = 27 stay zero
    double X[20][3];
    double J[27][9];       // Jacobians, then their inverses
    double w[KS];          // gauss weight * detJ (w[27] = 0)
    int nodes[20];
    double lam, mu;
    int bad;
};

__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(c0), "+d"(c1)
                 : "d"(a), "d"(b));
}

#ifndef FEM_VALUES_MIN_CTAS
#define FEM_VALUES_MIN_CTAS 3
#endif

__global__ void __launch_bounds__(kThreads, FEM_VALUES_MIN_CTAS)
    k_values_hex20(MeshView m, ListLayout L, const int* __restrict__ perm, int i0, int i1,
                   const int* __restrict__ map) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ValuesSmem& sm = *reinterpret_cast<ValuesSmem*>(smem_raw);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    // shape-function derivative table and the zero padding of G and w
    for (int idx = tid; idx < 27 * 20; idx += kThreads) {
        const int g = idx / 20, n = idx - 20 * g;
        double dx, dy, dz;
        hex20::dshape_node(n, hex20::gauss3(g / 9), hex20::gauss3((g / 3) % 3), hex20::gauss3(g % 3), dx, dy, dz);
        sm.dN[0][n][g] = dx;
        sm.dN[1][n][g] = dy;
        sm.dN[2][n][g] = dz;
    }
    for (int idx = tid; idx < 3 * 24 * KS; idx += kThreads) (&sm.G[0][0][0])[idx] = 0.0;
    for (int idx = tid; idx < 3 * 20; idx += kThreads) sm.dN[idx / 20][idx % 20][27] = 0.0;
    if (tid < KS) sm.w[tid] = 0.0;

    const int ti = c_ti[warp], tj = c_tj[warp];
    const int fr = lane >> 2, fc = lane & 3;
    // node id and coordinates of the next element
    int pre_n = 0;
    double pre_x = 0.0, pre_y = 0.0, pre_z = 0.0;
    if (tid < 20 && i0 + (int)blockIdx.x < i1) {
        pre_n = __ldg(m.conn + (size_t)__ldg(perm + i0 + blockIdx.x) * 20 + tid);
        if (pre_n >= 0 && pre_n < m.N) {
            pre_x = __ldg(m.x + pre_n);
            pre_y = __ldg(m.y + pre_n);
            pre_z = __ldg(m.z + pre_n);
        }
    }
    __syncthreads();

    for (int i = i0 + blockIdx.x; i < i1; i += gridDim.x) {
        const int e = __ldg(perm + i);
        if (tid == 0) sm.bad = 0;
        __syncthreads();  // the previous element's G, w, lam/mu and flag are no longer read
        if (tid < 20) {
            sm.nodes[tid] = pre_n;
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
        const int i_next = i + gridDim.x;
        if (tid < 20 && i_next < i1) pre_n = __ldg(m.conn + (size_t)__ldg(perm + i_next) * 20 + tid);
        if (sm.bad) {  // reported by the claim pass; nothing to add
            if (tid < 20 && i_next < i1 && pre_n >= 0 && pre_n < m.N) {
                pre_x = __ldg(m.x + pre_n);
                pre_y = __ldg(m.y + pre_n);
                pre_z = __ldg(m.z + pre_n);
            }
            __syncthreads();  // uniform: every thread has read the flag before it is reset
            continue;
        }
        // Jacobians J[g][3i + j] = sum_n dN[i][n][g] X[n][j]
        for (int idx = tid; idx < 243; idx += kThreads) {
            const int g = idx % 27, r = idx / 27, ii = r / 3, jj = r % 3;
            double acc = 0.0;
#pragma unroll
            for (int n = 0; n < 20; n++) acc = fma(sm.dN[ii][n][g], sm.X[n][jj], acc);
            sm.J[g][r] = acc;
        }
        __syncthreads();
        if (tid < 27) {
            double* J = sm.J[tid];
            const double c0 = J[4] * J[8] - J[5] * J[7], c1 = J[5] * J[6] - J[3] * J[8], c2 = J[3] * J[7] - J[4] * J[6];
            const double det = J[0] * c0 + J[1] * c1 + J[2] * c2;
            if (!(det > 0.0)) raise_status(L.info, FEM_ERR_DETJ);
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
            sm.w[tid] = hex20::weight3(tid / 9) * hex20::weight3((tid / 3) % 3) * hex20::weight3(tid % 3) * det;
        }
        __syncthreads();
        // physical gradients G[a][n][g] = sum_i iJ[g][3a + i] dN[i][n][g]
        for (int idx = tid; idx < 20 * 27; idx += kThreads) {
            const int n = idx / 27, g = idx - 27 * n;
            const double* iJ = sm.J[g];
            const double d0 = sm.dN[0][n][g], d1 = sm.dN[1][n][g], d2 = sm.dN[2][n][g];
#pragma unroll
            for (int a = 0; a < 3; a++) sm.G[a][n][g] = fma(iJ[3 * a], d0, fma(iJ[3 * a + 1], d1, iJ[3 * a + 2] * d2));
        }
        __syncthreads();
        // the coordinates of the next element arrive during the contraction
        if (tid < 20 && i_next < i1 && pre_n >= 0 && pre_n < m.N) {
            pre_x = __ldg(m.x + pre_n);
            pre_y = __ldg(m.y + pre_n);
            pre_z = __ldg(m.z + pre_n);
        }
        // M^{ab} tiles (ti, tj): A[r][k] = w_k G[a][8 ti + r][k], B[k][c] = G[b][8 tj + c][k]
        double acc[3][3][2];
#pragma unroll
        for (int a = 0; a < 3; a++)
#pragma unroll
            for (int b = 0; b < 3; b++) acc[a][b][0] = acc[a][b][1] = 0.0;
#pragma unroll
        for (int ks = 0; ks < 7; ks++) {
            const int k = 4 * ks + fc;
            const double wk = sm.w[k];
            double A[3], B[3];
#pragma unroll
            for (int a = 0; a < 3; a++) {
                A[a] = wk * sm.G[a][8 * ti + fr][k];
                B[a] = sm.G[a][8 * tj + fr][k];
            }
#pragma unroll
            for (int a = 0; a < 3; a++)
#pragma unroll
                for (int b = 0; b < 3; b++) dmma(acc[a][b][0], acc[a][b][1], A[a], B[b]);
        }
        // Ke blocks of this lane's node pairs, added to both triangles
        const double lam = sm.lam, mu = sm.mu;
        const int* mrow = map + (size_t)(i - i0) * 400;
        const int I = 8 * ti + fr;
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int Jn = 8 * tj + 2 * fc + h;
            if (I >= 20 || Jn >= 20 || (ti == tj && Jn < I)) continue;
            const int g_ij = __ldg(mrow + I * 20 + Jn);
            const int g_ji = I != Jn ? __ldg(mrow + Jn * 20 + I) : -1;
            const double mtr = mu * (acc[0][0][h] + acc[1][1][h] + acc[2][2][h]);
            double k[3][3];
#pragma unroll
            for (int a = 0; a < 3; a++)
#pragma unroll
                for (int b = 0; b < 3; b++) k[a][b] = fma(lam, acc[a][b][h], fma(mu, acc[b][a][h], a == b ? mtr : 0.0));
            if (g_ij >= 0) {
                double* p = L.vals + (size_t)(unsigned)g_ij * 9;
#pragma unroll
                for (int a = 0; a < 3; a++)
#pragma unroll
                    for (int b = 0; b < 3; b++) atomicAdd(p + 3 * a + b, k[a][b]);
            }
            if (g_ji >= 0) {
                double* p = L.vals + (size_t)(unsigned)g_ji * 9;
#pragma unroll
                for (int a = 0; a < 3; a++)
#pragma unroll
                    for (int b = 0; b < 3; b++) atomicAdd(p + 3 * b + a, k[a][b]);
            }
        }
    }
}

}  // namespace

cudaError_t launch_values_hex20_fp64(const MeshView& m, const ListLayout& L, const int* perm, int i0, int i1,
                                     const int* map, int ctas_per_sm, cudaStream_t s) {
    if (i1 <= i0) return cudaSuccess;
    static DeviceCache cache;
    const size_t smem = sizeof(ValuesSmem);
    int per_sm = 0;
    const cudaError_t err = per_device(cache, [&](int& v) {
        cudaError_t e = cudaFuncSetAttribute(k_values_hex20, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (!e) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, k_values_hex20, kThreads, smem);
        return e;
    }, per_sm);
    if (err) return err;
    const int use = ctas_per_sm > 0 ? std::min(ctas_per_sm, per_sm) : per_sm;
    const long long grid = std::max<long long>(1, std::min<long long>(i1 - i0, (long long)use * sm_count()));
    k_values_hex20<<<(int)grid, kThreads, smem, s>>>(m, L, perm, i0, i1, map);
    return cudaGetLastError();
}

cudaError_t launch_values_hex20(const MeshView& m, const ListLayout& L, int precision, const int* perm, int i0,
                                int i1, const int* map, int ctas_per_sm, long long wait_ns, cudaStream_t s) {
    return precision == FEM_PREC_TC_F16X3 ? launch_values_hex20_tc(m, L, perm, i0, i1, map, wait_ns, s)
                                          : launch_values_hex20_fp64(m, L, perm, i0, i1, map, ctas_per_sm, s);
}

}  // namespace fem
