// Device code of the Hex20 group value pass (values_hex20.cu). See
// values_hex20.cu for the method.
#pragma once

#include "group_hex20.cuh"
#include "values_hex20.cuh"

namespace fem {
namespace {

struct GroupValuesSmem {
    alignas(16) double ke[kGroup * 210 * 9];  // the group's element blocks, pair-major (record positions), each as it adds to its pair's (row u, column v) block
    double dN[3][20][KS];         // dN_n / dxi_i at Gauss point g: [i][n][g]
    double X[kGroup][20][3];      // per warp: its element's node coordinates
    double iJw[kGroup][KS][10];   // per warp: inverse Jacobian (9) and weight * detJ at each Gauss point; row 27 zero
    double lam[kGroup], mu[kGroup];
    alignas(16) int rec[2][kGroupRecWords];  // the current and the next group's record
};

__device__ __forceinline__ void cp_async16_v(void* dst, const void* src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
}

// Tables of the group value pass; every thread of the CTA calls it once.
__device__ __forceinline__ void values_group_init(GroupValuesSmem& sm) {
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int idx = tid; idx < 27 * 20; idx += nt) {
        const int g = idx / 20, n = idx - 20 * g;
        double dx, dy, dz;
        hex20::dshape_node(n, hex20::gauss3(g / 9), hex20::gauss3((g / 3) % 3), hex20::gauss3(g % 3), dx, dy, dz);
        sm.dN[0][n][g] = dx;
        sm.dN[1][n][g] = dy;
        sm.dN[2][n][g] = dz;
    }
    for (int idx = tid; idx < 3 * 20; idx += nt) sm.dN[idx / 20][idx % 20][27] = 0.0;
    for (int idx = tid; idx < kGroup * KS * 10; idx += nt) (&sm.iJw[0][0][0])[idx] = 0.0;
    __syncthreads();
}

// Stores block k (row-major 3x3, element orientation (I, J)) at its
// position in the pair-major order, as it adds to its pair's (row u, column v)
// block: k, its transpose (bit 15 of the position entry), or k + k^T (bit 14).
__device__ __forceinline__ void stage_block(double* __restrict__ ke, unsigned c, const double (&k)[9]) {
    double* d = ke + 9 * (c & kPosMask);
    const bool tr = c & kTabTransposed, both = c & kTabBoth;
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = 0; b < 3; b++) {
            const double x = k[3 * a + b], y = k[3 * b + a];
            d[3 * a + b] = both ? x + y : (tr ? y : x);
        }
}

// Ke of element w of the group (coordinates already in sm.X[w], material in
// sm.lam / sm.mu), computed by one warp; each upper block is staged at its
// position `cpos` (one writer per position, plain stores) as it adds to its
// pair: entry (a, b) is alpha M^{ab} + beta M^{ba} + gamma [a = b] mu tr M,
// with (alpha, beta, gamma) = (lam, mu, 1) for a block in its pair's
// orientation, (mu, lam, 1) transposed, (lam + mu, lam + mu, 2) for both
// orientations on one diagonal block.
__device__ __forceinline__ void group_element_fp64(int w, const unsigned short* __restrict__ cpos, DevInfo* info,
                                                   GroupValuesSmem& sm) {
    const int lane = threadIdx.x & 31, fr = lane >> 2, fc = lane & 3;
    if (lane < 27) {
        // Jacobian at Gauss point g = lane: J[3i + j] = sum_n dN[i][n][g] X[n][j]
        const int g = lane;
        double J[9];
#pragma unroll
        for (int r = 0; r < 9; r++) J[r] = 0.0;
#pragma unroll 4
        for (int n = 0; n < 20; n++) {
            const double d0 = sm.dN[0][n][g], d1 = sm.dN[1][n][g], d2 = sm.dN[2][n][g];
            const double x0 = sm.X[w][n][0], x1 = sm.X[w][n][1], x2 = sm.X[w][n][2];
            J[0] = fma(d0, x0, J[0]);
            J[1] = fma(d0, x1, J[1]);
            J[2] = fma(d0, x2, J[2]);
            J[3] = fma(d1, x0, J[3]);
            J[4] = fma(d1, x1, J[4]);
            J[5] = fma(d1, x2, J[5]);
            J[6] = fma(d2, x0, J[6]);
            J[7] = fma(d2, x1, J[7]);
            J[8] = fma(d2, x2, J[8]);
        }
        const double c0 = J[4] * J[8] - J[5] * J[7], c1 = J[5] * J[6] - J[3] * J[8], c2 = J[3] * J[7] - J[4] * J[6];
        const double det = J[0] * c0 + J[1] * c1 + J[2] * c2;
        if (!(det > 0.0)) raise_status(info, FEM_ERR_DETJ);
        const double r = 1.0 / det;
        double* o = sm.iJw[w][g];
        o[0] = c0 * r;
        o[1] = (J[2] * J[7] - J[1] * J[8]) * r;
        o[2] = (J[1] * J[5] - J[2] * J[4]) * r;
        o[3] = c1 * r;
        o[4] = (J[0] * J[8] - J[2] * J[6]) * r;
        o[5] = (J[2] * J[3] - J[0] * J[5]) * r;
        o[6] = c2 * r;
        o[7] = (J[1] * J[6] - J[0] * J[7]) * r;
        o[8] = (J[0] * J[4] - J[1] * J[3]) * r;
        o[9] = hex20::weight3(g / 9) * hex20::weight3((g / 3) % 3) * hex20::weight3(g % 3) * det;
    }
    __syncwarp();
    // physical gradients of the lane's (node, Gauss point) entries, held in
    // registers: G[t][s][a] = dN_n / dx_a at g, n = 8 t + fr, g = 4 s + fc
    // (zero in the padding n >= 20, g = 27)
    double G[3][7][3], wk[7];
#pragma unroll
    for (int s = 0; s < 7; s++) {
        const int g = 4 * s + fc;
        const double* iJ = sm.iJw[w][g];
        wk[s] = iJ[9];
#pragma unroll
        for (int t = 0; t < 3; t++) {
            const int n = 8 * t + fr;
            const bool ok = n < 20 && g < 27;
            const int nn = ok ? n : 0;
            const double d0 = sm.dN[0][nn][g], d1 = sm.dN[1][nn][g], d2 = sm.dN[2][nn][g];
#pragma unroll
            for (int a = 0; a < 3; a++)
                G[t][s][a] = ok ? fma(iJ[3 * a], d0, fma(iJ[3 * a + 1], d1, iJ[3 * a + 2] * d2)) : 0.0;
        }
    }
    const double lam = sm.lam[w], mu = sm.mu[w];
    // the six 8x8 tile positions (ti <= tj) of the upper triangle of the
    // 24 x 24 node grid; all nine M^{ab} tiles of each on the FP64 tensor cores
#pragma unroll
    for (int tile = 0; tile < 6; tile++) {
        const int ti = tile < 3 ? 0 : (tile < 5 ? 1 : 2);
        const int tj = tile == 0 ? 0 : (tile == 1 || tile == 3 ? 1 : 2);
        double c[3][3][2];
#pragma unroll
        for (int a = 0; a < 3; a++)
#pragma unroll
            for (int b = 0; b < 3; b++) c[a][b][0] = c[a][b][1] = 0.0;
#pragma unroll
        for (int s = 0; s < 7; s++) {
            double A[3];
#pragma unroll
            for (int a = 0; a < 3; a++) A[a] = wk[s] * G[ti][s][a];
#pragma unroll
            for (int a = 0; a < 3; a++)
#pragma unroll
                for (int b = 0; b < 3; b++) dmma(c[a][b][0], c[a][b][1], A[a], G[tj][s][b]);
        }
        const int I = 8 * ti + fr;
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int J = 8 * tj + 2 * fc + h;
            if (I >= 20 || J >= 20 || (ti == tj && J < I)) continue;
            const double mtr = mu * (c[0][0][h] + c[1][1][h] + c[2][2][h]);
            const unsigned e = cpos[packed_block(I, J)];
            const bool both = e & kTabBoth, tr = e & kTabTransposed;
            const double al = both ? lam + mu : (tr ? mu : lam), be = both ? lam + mu : (tr ? lam : mu);
            const double dg = both ? 2.0 * mtr : mtr;
            double* d = sm.ke + 9 * (e & kPosMask);
#pragma unroll
            for (int a = 0; a < 3; a++)
#pragma unroll
                for (int b = 0; b < 3; b++) d[3 * a + b] = fma(al, c[a][b][h], fma(be, c[b][a][h], a == b ? dg : 0.0));
        }
    }
}

// Group value pass over the groups of positions [i0, i1) of the visit order,
// group g = blockIdx.x, blockIdx.x + gridDim.x, ...; the record of group g at
// recs + g * kGroupRecWords (written by the claim pass). stage: NULL (Ke in
// FP64 here) or the packed upper Ke blocks of the wave's elements, row q - i0
// for position q (the tensor-core form). kGroup warps; every thread calls it.
__device__ void values_group(const MeshView& m, int i0, int i1, const int* __restrict__ recs,
                             const double* __restrict__ stage, double* vals, DevInfo* info, GroupValuesSmem& sm) {
    const int tid = threadIdx.x, nt = blockDim.x, warp = tid >> 5, lane = tid & 31;
    const int ngroups = (i1 - i0 + kGroup - 1) / kGroup;
    auto fetch_record = [&](int g, int buf) {
        const int* src = recs + (size_t)g * kGroupRecWords;
        for (int q = tid; q < kGroupRecWords / 4; q += nt) cp_async16_v(&sm.rec[buf][4 * q], src + 4 * q);
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    // coordinates and material of warp `warp`'s element of the group whose record is R
    double px = 0.0, py = 0.0, pz = 0.0, pE = 0.0, pnu = 0.0;
    auto fetch_element = [&](const int* R) {
        if (warp >= R[1]) return;
        if (lane < 20) {
            const int n = R[kRecOcc + 20 * warp + lane];
            px = FEM_LDG(m.x + n);
            py = FEM_LDG(m.y + n);
            pz = FEM_LDG(m.z + n);
        } else if (lane == 20) {
            const int e = R[2 + warp];
            pE = m.E ? FEM_LDG(m.E + e) : m.E0;
            pnu = m.nu ? FEM_LDG(m.nu + e) : m.nu0;
        }
    };
    int g = blockIdx.x, buf = 0;
    if (g < ngroups) {
        fetch_record(g, 0);
        asm volatile("cp.async.wait_all;" ::: "memory");
        __syncthreads();
        fetch_element(sm.rec[0]);
    }
    for (; g < ngroups; g += gridDim.x) {
        const int* R = sm.rec[buf];
        const int ne = R[1], npairs = R[0];
        const int gn = g + gridDim.x;
        if (gn < ngroups) fetch_record(gn, buf ^ 1);
        if (warp < ne) {
            const unsigned short* cpos = reinterpret_cast<const unsigned short*>(R + kRecCpos) + 210 * warp;
            if (stage) {  // the element's blocks from the stage buffer
                const long long g0 = (long long)i0 + (long long)g * kGroup;
                const double* ke = stage + (size_t)(g0 + warp - i0) * kPackedHex20;
                for (int p = lane; p < 210; p += 32) {
                    double k[9];
#pragma unroll
                    for (int q = 0; q < 9; q++) k[q] = FEM_LDG(ke + 9 * p + q);
                    stage_block(sm.ke, cpos[p], k);
                }
            } else {
                if (lane < 20) {
                    sm.X[warp][lane][0] = px;
                    sm.X[warp][lane][1] = py;
                    sm.X[warp][lane][2] = pz;
                } else if (lane == 20) {
                    sm.lam[warp] = pE * pnu / ((1.0 + pnu) * (1.0 - 2.0 * pnu));
                    sm.mu[warp] = pE / (2.0 * (1.0 + pnu));
                }
                __syncwarp();
                group_element_fp64(warp, cpos, info, sm);
            }
        }
        asm volatile("cp.async.wait_all;" ::: "memory");
        __syncthreads();  // the group's element blocks are complete; the next record is in
        if (gn < ngroups && !stage) fetch_element(sm.rec[buf ^ 1]);
        // every node pair of the group once, the sum of its staged blocks:
        // stored where the group is the pair's only contributor, added
        // atomically where other groups add too; (row u, column v) as summed,
        // (row v, column u) transposed. Three threads per pair, one row a of
        // its block each: row a of (row u, column v), column a of (row v, column u)
        const unsigned* slots = reinterpret_cast<const unsigned*>(R + kRecMap);
        const unsigned short* cofs = reinterpret_cast<const unsigned short*>(R + kRecCofs);
        for (int idx = tid; idx < npairs * 3; idx += nt) {
            const int r = idx / 3, a = idx - 3 * r;
            const unsigned w0 = slots[2 * r], w1 = slots[2 * r + 1];
            double v0 = 0.0, v1 = 0.0, v2 = 0.0;
            for (int i = cofs[r], i1 = cofs[r + 1]; i < i1; i++) {
                const double* k = sm.ke + 9 * i + 3 * a;
                v0 += k[0];
                v1 += k[1];
                v2 += k[2];
            }
            if (map_has_slot(w0)) {
                double* d = vals + (size_t)(w0 & ~kPairShared) * 9 + 3 * a;
                if (w0 & kPairShared) {
                    atomicAdd(d, v0);
                    atomicAdd(d + 1, v1);
                    atomicAdd(d + 2, v2);
                } else {
                    d[0] = v0;
                    d[1] = v1;
                    d[2] = v2;
                }
            }
            if (map_has_slot(w1)) {
                double* d = vals + (size_t)(w1 & ~kPairShared) * 9 + a;
                if (w1 & kPairShared) {
                    atomicAdd(d, v0);
                    atomicAdd(d + 3, v1);
                    atomicAdd(d + 6, v2);
                } else {
                    d[0] = v0;
                    d[3] = v1;
                    d[6] = v2;
                }
            }
        }
        __syncthreads();  // the element blocks and the record buffer are free
        buf ^= 1;
    }
}

}  // namespace
}  // namespace fem
