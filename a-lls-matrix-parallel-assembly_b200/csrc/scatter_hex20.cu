// K1 for Hex20 meshes: fused FP64 element stiffness + A-LLS row-list scatter.
//
// Replaces assembleGlobalStiffnessKernelALLSFixedArray
// (ALLS_Hex20_3D_Assembly_Performance.cu:208-257), whose 60x60 FP32 Ke lives in
// 14.9 KB of local memory per thread and whose fixed 300-entry rows silently
// drop overflow.
//
// One CTA (8 warps) per element, persistent over the element range:
//  * the 27 Gauss points' shape-function derivatives (H20:95-128) are built once
//    per CTA in shared memory;
//  * per element: J (243 dot products), det/inverse (27 threads), the
//    physical gradients G[g][node][dir] (1620 values), then the node-pair
//    matrix  M_IJ[a][b] = sum_g w_g detJ_g G[g][I][a] G[g][J][b]  for the 210
//    upper node pairs, from which the isotropic block is
//    Ke_IJ = lambda M_IJ + mu M_IJ^T + mu tr(M_IJ) I  — algebraically the
//    reference's per-Gauss-point block formula (H20:173-191) with
//    c1 = lambda + 2 mu, c2 = lambda, c3 = mu, in double;
//  * scatter: warp w serves row nodes w, w+8, w+16. The warp copies the row's
//    chunk slots into shared memory with lane-parallel L2 loads; lane j then
//    resolves column node j along its hashed probe sequence, claiming a free
//    slot with atomicCAS (empty -> col|pending) if the column is absent, and
//    following / atomicCAS-linking overflow chunks when the probe sequence is
//    full. Claimed blocks are stored, the warp fences and publishes them; found
//    blocks are accumulated with atomicAdd (after a bounded wait for slots
//    another warp is still writing).
#include "launch.h"

namespace fem {
namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kPairs = 210;
constexpr int kMaxHex20Slots = 128;  // upper bound of S1, S2 (checked on the host)

__device__ __forceinline__ int pair_index(int I, int J) { return I * 20 - I * (I - 1) / 2 + (J - I); }

// Natural coordinates of the 20 nodes in the reference order (H20:97-99).
__constant__ signed char c_xin[20] = {-1, 1, 1, -1, -1, 1, 1, -1, 0, 1, 0, -1, 0, 1, 0, -1, -1, 1, 1, -1};
__constant__ signed char c_etan[20] = {-1, -1, 1, 1, -1, -1, 1, 1, -1, 0, 1, 0, -1, 0, 1, 0, -1, -1, 1, 1};
__constant__ signed char c_zetan[20] = {-1, -1, -1, -1, 1, 1, 1, 1, -1, -1, -1, -1, 1, 1, 1, 1, 0, 0, 0, 0};

// Gauss abscissae / weights as the reference writes them (H20:45-46), in double.
__device__ __forceinline__ double gauss3(int i) { return i == 0 ? -0.774596669241483 : (i == 1 ? 0.0 : 0.774596669241483); }
__device__ __forceinline__ double weight3(int i) { return i == 1 ? 0.888888888888889 : 0.555555555555556; }

// dN_n/d(xi, eta, zeta) at one point (formulas of H20:95-128).
__device__ void hex20_dshape_node(int n, double xi, double eta, double zeta, double& dx, double& dy, double& dz) {
    const double a = c_xin[n], b = c_etan[n], c = c_zetan[n];
    if (n < 8) {
        dx = 0.125 * a * (1.0 + b * eta) * (1.0 + c * zeta) * (2.0 * a * xi + b * eta + c * zeta - 1.0);
        dy = 0.125 * b * (1.0 + a * xi) * (1.0 + c * zeta) * (a * xi + 2.0 * b * eta + c * zeta - 1.0);
        dz = 0.125 * c * (1.0 + a * xi) * (1.0 + b * eta) * (a * xi + b * eta + 2.0 * c * zeta - 1.0);
    } else if (n == 8 || n == 10 || n == 12 || n == 14) {
        dx = -0.5 * xi * (1.0 + b * eta) * (1.0 + c * zeta);
        dy = 0.25 * b * (1.0 - xi * xi) * (1.0 + c * zeta);
        dz = 0.25 * c * (1.0 - xi * xi) * (1.0 + b * eta);
    } else if (n < 16) {
        dx = 0.25 * a * (1.0 - eta * eta) * (1.0 + c * zeta);
        dy = -0.5 * eta * (1.0 + a * xi) * (1.0 + c * zeta);
        dz = 0.25 * c * (1.0 + a * xi) * (1.0 - eta * eta);
    } else {
        dx = 0.25 * a * (1.0 + b * eta) * (1.0 - zeta * zeta);
        dy = 0.25 * b * (1.0 + a * xi) * (1.0 - zeta * zeta);
        dz = -0.5 * zeta * (1.0 + a * xi) * (1.0 + b * eta);
    }
}

struct Hex20Smem {
    double dN[27][3][20];   // shape derivatives at the Gauss points
    double X[20][3];        // element node coordinates
    double J[27][9];        // Jacobians, then their inverses
    double w[27];           // Gauss weight * detJ
    double G[27][60];       // physical gradients G[g][3*node + dir]
    double K[kPairs][9];    // upper node-pair blocks of Ke
    int view[kWarps][kMaxHex20Slots];   // per-warp copy of the chunk slots being probed
    unsigned gid[kWarps][20];
    int state[kWarps][20];
    int nodes[20];
    unsigned char pI[kPairs], pJ[kPairs];
    double lam, mu;
    int bad;
};

enum SlotState : int { kUnresolved = 0, kFound = 1, kFoundPending = 2, kClaimed = 3 };

// Resolves the 20 column slots of row node I of the current element and
// scatters its 20 Ke blocks (warp-cooperative; lane j owns column node j).
__device__ __forceinline__ void scatter_row(const ListLayout& L, Hex20Smem& sm, int I, int warp, int lane,
                                            int& spare) {
    int* view = sm.view[warp];
    const int key = lane < 20 ? sm.nodes[lane] + 1 : 0;
    int state = lane < 20 ? kUnresolved : kFound;
    unsigned gid = 0;
    int* word = nullptr;
    int c = sm.nodes[I];
    for (int step = 0; step < kMaxChainSteps; step++) {
        int* meta = chunk_meta(L, c);
        const int cap = chunk_cap(L, c);
        for (int s = lane; s < cap; s += 32) view[s] = ld_cg(meta + 2 + s);
        __syncwarp();
        if (state == kUnresolved) {
            int p = probe_start(key, cap);
            for (int tries = 0; tries < cap; tries++) {
                int v = view[p];
                if (v == 0) {
                    v = atomicCAS(meta + 2 + p, 0, key | kPending);
                    if (v == 0) {
                        state = kClaimed;
                        view[p] = key | kPending;
                    } else {
                        view[p] = v;
                    }
                }
                if (state != kClaimed && (v & kColMask) == key) state = v < 0 ? kFoundPending : kFound;
                if (state != kUnresolved) {
                    gid = slot_gid(L, c, p);
                    word = meta + 2 + p;
                    break;
                }
                p = p + 1 == cap ? 0 : p + 1;
            }
        }
        __syncwarp();
        if (!__any_sync(0xFFFFFFFFu, state == kUnresolved)) break;
        int nc = 0;
        if (lane == 0) nc = next_chunk(L, c, spare);
        c = __shfl_sync(0xFFFFFFFFu, nc, 0);
        if (c < 0) break;  // pool overflow: status raised, unresolved columns dropped
    }
    if (lane < 20) {
        sm.state[warp][lane] = state;
        sm.gid[warp][lane] = gid;
    }
    __syncwarp();
    // Claimed blocks: plain stores. Found (published) blocks: atomicAdd.
    for (int idx = lane; idx < 20 * 9; idx += 32) {
        const int j = idx / 9, v = idx - j * 9;
        const int st = sm.state[warp][j];
        if (st == kUnresolved || st == kFoundPending) continue;
        const int a = v / 3, b = v - a * 3;
        const double val = I <= j ? sm.K[pair_index(I, j)][3 * a + b] : sm.K[pair_index(j, I)][3 * b + a];
        double* p = L.vals + (size_t)sm.gid[warp][j] * 9 + v;
        if (st == kClaimed)
            *p = val;
        else
            atomicAdd(p, val);
    }
    const unsigned claimed = __ballot_sync(0xFFFFFFFFu, state == kClaimed);
    if (lane == 0 && claimed) atomicAdd(L.counts + sm.nodes[I], __popc(claimed));
    if (claimed) {
        __threadfence();
        __syncwarp();
        if (state == kClaimed) atomicExch(word, key);
    }
    // Blocks of slots another warp is still writing: wait, then add.
    if (state == kFoundPending && wait_published(L, word)) {
        double* p = L.vals + (size_t)gid * 9;
        for (int v = 0; v < 9; v++) {
            const int a = v / 3, b = v - a * 3;
            atomicAdd(p + v, I <= lane ? sm.K[pair_index(I, lane)][3 * a + b] : sm.K[pair_index(lane, I)][3 * b + a]);
        }
    }
    __syncwarp();
}

__global__ void __launch_bounds__(kThreads) k_scatter_hex20(MeshView m, ListLayout L) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Hex20Smem& sm = *reinterpret_cast<Hex20Smem*>(smem_raw);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    for (int idx = tid; idx < 27 * 20; idx += kThreads) {
        const int g = idx / 20, n = idx % 20;
        double dx, dy, dz;
        hex20_dshape_node(n, gauss3(g / 9), gauss3((g / 3) % 3), gauss3(g % 3), dx, dy, dz);
        sm.dN[g][0][n] = dx;
        sm.dN[g][1][n] = dy;
        sm.dN[g][2][n] = dz;
    }
    if (tid < kPairs) {
        int I = 0, r = tid;
        while (r >= 20 - I) { r -= 20 - I; I++; }
        sm.pI[tid] = (unsigned char)I;
        sm.pJ[tid] = (unsigned char)(I + r);
    }
    int spare = -1;
    __syncthreads();

    for (int e = blockIdx.x; e < m.E_count; e += gridDim.x) {
        if (tid == 0) sm.bad = 0;
        __syncthreads();
        if (tid < 20) {
            const int n = __ldg(m.conn + (size_t)e * 20 + tid);
            sm.nodes[tid] = n;
            if (n < 0 || n >= m.N) {
                sm.bad = 1;
            } else {
                sm.X[tid][0] = __ldg(m.x + n);
                sm.X[tid][1] = __ldg(m.y + n);
                sm.X[tid][2] = __ldg(m.z + n);
            }
        }
        if (tid == 32) {
            const double E = m.E ? __ldg(m.E + e) : m.E0;
            const double nu = m.nu ? __ldg(m.nu + e) : m.nu0;
            sm.lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
            sm.mu = E / (2.0 * (1.0 + nu));
        }
        __syncthreads();
        if (sm.bad) {  // uniform: every thread reads the flag before anyone resets it
            if (tid == 0) raise_status(L.info, FEM_ERR_BAD_MESH);
            __syncthreads();
            continue;
        }
        // Jacobians: J[g][3i+j] = sum_n dN[g][i][n] X[n][j]
        if (tid < 243) {
            const int g = tid / 9, r = tid % 9, i = r / 3, j = r % 3;
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
            sm.w[tid] = weight3(tid / 9) * weight3((tid / 3) % 3) * weight3(tid % 3) * det;
        }
        __syncthreads();
        // Physical gradients G[g][3n+a] = sum_i iJ[g][3a+i] dN[g][i][n]
        for (int idx = tid; idx < 27 * 60; idx += kThreads) {
            const int g = idx / 60, r = idx % 60, n = r / 3, a = r % 3;
            const double* iJ = sm.J[g];
            sm.G[g][r] = fma(iJ[3 * a], sm.dN[g][0][n], fma(iJ[3 * a + 1], sm.dN[g][1][n], iJ[3 * a + 2] * sm.dN[g][2][n]));
        }
        __syncthreads();
        // Upper node-pair blocks.
        if (tid < kPairs) {
            const int I = sm.pI[tid], J = sm.pJ[tid];
            double acc[9];
#pragma unroll
            for (int k = 0; k < 9; k++) acc[k] = 0.0;
            for (int g = 0; g < 27; g++) {
                const double w = sm.w[g];
                const double a0 = w * sm.G[g][3 * I], a1 = w * sm.G[g][3 * I + 1], a2 = w * sm.G[g][3 * I + 2];
                const double b0 = sm.G[g][3 * J], b1 = sm.G[g][3 * J + 1], b2 = sm.G[g][3 * J + 2];
                acc[0] = fma(a0, b0, acc[0]); acc[1] = fma(a0, b1, acc[1]); acc[2] = fma(a0, b2, acc[2]);
                acc[3] = fma(a1, b0, acc[3]); acc[4] = fma(a1, b1, acc[4]); acc[5] = fma(a1, b2, acc[5]);
                acc[6] = fma(a2, b0, acc[6]); acc[7] = fma(a2, b1, acc[7]); acc[8] = fma(a2, b2, acc[8]);
            }
            const double lam = sm.lam, mu = sm.mu;
            const double tr = mu * (acc[0] + acc[4] + acc[8]);
#pragma unroll
            for (int a = 0; a < 3; a++)
#pragma unroll
                for (int b = 0; b < 3; b++)
                    sm.K[tid][3 * a + b] = fma(lam, acc[3 * a + b], mu * acc[3 * b + a]) + (a == b ? tr : 0.0);
        }
        __syncthreads();

        // Scatter: warp w serves row nodes w, w + 8, w + 16.
        for (int I = warp; I < 20; I += kWarps) scatter_row(L, sm, I, warp, lane, spare);
        __syncthreads();
    }
}

}  // namespace

cudaError_t launch_scatter_hex20(const MeshView& m, const ListLayout& L, cudaStream_t s) {
    static int blocks_per_sm = 0, sms = 0;
    const size_t smem = sizeof(Hex20Smem);
    if (!blocks_per_sm) {
        cudaError_t err = cudaFuncSetAttribute(k_scatter_hex20, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (err) return err;
        err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, k_scatter_hex20, kThreads, smem);
        if (err) return err;
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (blocks_per_sm < 1) blocks_per_sm = 1;
    }
    long long grid = (long long)blocks_per_sm * sms;
    if (grid > m.E_count) grid = m.E_count > 0 ? m.E_count : 1;
    k_scatter_hex20<<<(int)grid, kThreads, smem, s>>>(m, L);
    return cudaGetLastError();
}

}  // namespace fem
