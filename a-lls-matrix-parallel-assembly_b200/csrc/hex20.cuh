// Hex20 element definitions shared by the element-stiffness kernels
// (element_stiffness.cu, ke_tcgen05.cu) and the A-LLS scatter (scatter_hex20.cu).
//
// Element stiffness, in double. With the physical shape-function gradients
// G_g (a 60-vector per Gauss point g, dof r = 3 node + dir) and
// w_g = gauss weight * detJ_g, the node-pair matrix
//     M = sum_g w_g G_g G_g^T          (60 x 60, contraction length 27)
// gives every 3x3 block of the isotropic stiffness as
//     Ke_IJ[a][b] = lambda M[3I+a][3J+b] + mu M[3I+b][3J+a] + mu delta_ab tr(M_IJ)
// which is algebraically the reference's per-Gauss-point block formula
// (ALLS_Hex20_3D_Assembly_Performance.cu:173-191, c1 = lambda + 2 mu,
// c2 = lambda, c3 = mu).
#pragma once

#include <cuda_fp16.h>

#include "launch.h"

namespace fem {
namespace hex20 {

constexpr int kUpperBlocks = 210;  // node pairs I <= J

// Index of node pair (I <= J) among the upper pairs, row-major.
__host__ __device__ __forceinline__ int pair_index(int I, int J) { return I * 20 - I * (I - 1) / 2 + (J - I); }

// Natural coordinates of the 20 nodes in the reference order (H20:97-99).
__device__ __forceinline__ int xi_of(int n) {
    constexpr signed char v[20] = {-1, 1, 1, -1, -1, 1, 1, -1, 0, 1, 0, -1, 0, 1, 0, -1, -1, 1, 1, -1};
    return v[n];
}
__device__ __forceinline__ int eta_of(int n) {
    constexpr signed char v[20] = {-1, -1, 1, 1, -1, -1, 1, 1, -1, 0, 1, 0, -1, 0, 1, 0, -1, -1, 1, 1};
    return v[n];
}
__device__ __forceinline__ int zeta_of(int n) {
    constexpr signed char v[20] = {-1, -1, -1, -1, 1, 1, 1, 1, -1, -1, -1, -1, 1, 1, 1, 1, 0, 0, 0, 0};
    return v[n];
}

// Gauss abscissae / weights as the reference writes them (H20:45-46), in double.
__device__ __forceinline__ double gauss3(int i) { return i == 0 ? -0.774596669241483 : (i == 1 ? 0.0 : 0.774596669241483); }
__device__ __forceinline__ double weight3(int i) { return i == 1 ? 0.888888888888889 : 0.555555555555556; }

// dN_n/d(xi, eta, zeta) at one point (formulas of H20:95-128).
__device__ __forceinline__ void dshape_node(int n, double xi, double eta, double zeta, double& dx, double& dy,
                                            double& dz) {
    const double a = xi_of(n), b = eta_of(n), c = zeta_of(n);
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

// ---------------------------------------------------------------------------
// Tensor-core form of the node-pair contraction (FEM_PREC_TC_F16X3)
// ---------------------------------------------------------------------------
//
// M = P diag(w) P^T is rewritten as M = A diag(sgn) A^T / s^2 with
// A[r][g] = s * P[r][g] * sqrt(|w_g|), sgn_g = sign(w_g) and s a power of two
// that brings a bound on max |A| into [0.5, 1) (exact scaling, per element).
// Each entry of A is rounded to FP32 and split into two FP16 numbers,
// A = A_hi + A_lo (22 significant bits; the remainder is below 2^-23 |A|), and
//     A A^T ~ A_lo A_hi^T + A_hi A_lo^T + A_hi A_hi^T
// is summed by three mma.sync.m16n8k16 FP16 products per tile with FP32
// accumulation (the dropped A_lo A_lo^T term is below 2^-22 of the scale).
// The 64 x 64 product (60 dofs padded, K = 27 Gauss points padded to 32) is
// covered by the 20 tiles of 16 x 8 that reach the upper triangle; each upper
// entry (r <= c < 60) is handed to store(r, c, value) in FP64. The Jacobian,
// its determinant and inverse, and the global accumulation stay in FP64.

constexpr int kTcLda = 40;  // halves per row of A_hi / A_lo (80 B: conflict-free fragment loads)
constexpr int kTcTiles = 20;

struct TcScratch {
    __half hi[64][kTcLda];
    __half lo[64][kTcLda];
    __half2 sgn[16];                // sign of w_g for g = 2k, 2k + 1
    double sqw[32];                 // sqrt(|w_g|)
    unsigned long long bound_bits;  // a bound on max |P sqrt|w|| (bits of a positive double)
    double inv_s2;
};

// Per Gauss point g (called by the thread that computed w_g and the inverse
// Jacobian iJ of g, after the CTA reset sc.bound_bits): sqrt(|w_g|) and the
// bound |P[r][g]| sqrt|w_g| <= sqrt|w_g| max_a sum_i |iJ[3a+i]| * dnmax, with
// dnmax the largest |dN/dxi| of the shape-function table.
__device__ __forceinline__ void tc_gauss_point(TcScratch& sc, int g, const double* iJ, double w, double dnmax) {
    const double sq = sqrt(fabs(w));
    sc.sqw[g] = sq;
    double rn = 0.0;
#pragma unroll
    for (int a = 0; a < 3; a++) rn = fmax(rn, fabs(iJ[3 * a]) + fabs(iJ[3 * a + 1]) + fabs(iJ[3 * a + 2]));
    const double b = sq * rn * dnmax;
    if (b > 0.0) atomicMax(&sc.bound_bits, (unsigned long long)__double_as_longlong(b));
}

// Builds A_hi, A_lo and the signs from P (row stride ps doubles, rows >= 60 and
// Gauss points >= 27 ignored), w and the per-point data of tc_gauss_point. The
// scale s is the power of two that brings the bound into [0.5, 1). Every
// thread of the CTA calls it; it ends with a CTA barrier.
template <int kThreads>
__device__ __forceinline__ void tc_prepare(const double* P, int ps, const double* w, TcScratch& sc, int tid) {
    const double bound = __longlong_as_double((long long)sc.bound_bits);
    int ex = 0;
    if (bound > 0.0) frexp(bound, &ex);  // bound = m * 2^ex, m in [0.5, 1)
    const double s = ldexp(1.0, -ex);
    for (int idx = tid; idx < 64 * 32; idx += kThreads) {
        const int r = idx >> 5, g = idx & 31;
        float a = 0.0f;
        if (r < 60 && g < 27) a = (float)(s * P[r * ps + g] * sc.sqw[g]);
        const __half h = __float2half_rn(a);
        sc.hi[r][g] = h;
        sc.lo[r][g] = __float2half_rn(a - __half2float(h));  // exact difference in float
    }
    if (tid < 16) {
        const int g = 2 * tid;
        const float s0 = g < 27 && w[g] < 0.0 ? -1.0f : 1.0f, s1 = g + 1 < 27 && w[g + 1] < 0.0 ? -1.0f : 1.0f;
        sc.sgn[tid] = __floats2half2_rn(s0, s1);
    }
    if (tid == 0) sc.inv_s2 = ldexp(1.0, 2 * ex);
    __syncthreads();
}

__device__ __forceinline__ void mma_16816(float (&d)[4], const unsigned (&a)[4], const unsigned (&b)[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__device__ __forceinline__ unsigned ld_h2(const __half* p) { return *reinterpret_cast<const unsigned*>(p); }

__device__ __forceinline__ unsigned mul_h2(unsigned a, __half2 s) {
    __half2 v = *reinterpret_cast<__half2*>(&a);
    v = __hmul2(v, s);
    return *reinterpret_cast<unsigned*>(&v);
}

// The 20 tiles (16-row block i, 8-column block j >= 2i) of the upper triangle,
// dealt round-robin to the kWarps warps; store(r, c, M_rc) for r <= c < 60.
template <int kWarps, typename Store>
__device__ __forceinline__ void tc_contract(const TcScratch& sc, int warp, int lane, Store store) {
    constexpr unsigned char ti[kTcTiles] = {0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 1, 1, 2, 2, 2, 2, 3, 3};
    constexpr unsigned char tj[kTcTiles] = {0, 1, 2, 3, 4, 5, 6, 7, 2, 3, 4, 5, 6, 7, 4, 5, 6, 7, 6, 7};
    const int g = lane >> 2, t = lane & 3;
    for (int tile = warp; tile < kTcTiles; tile += kWarps) {
        const int r0 = 16 * ti[tile], c0 = 8 * tj[tile];
        float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int k0 = 0; k0 < 32; k0 += 16) {
            const __half2 s0 = sc.sgn[(k0 >> 1) + t], s1 = sc.sgn[(k0 >> 1) + 4 + t];
            unsigned ah[4], al[4], bh[2], bl[2];
            ah[0] = mul_h2(ld_h2(&sc.hi[r0 + g][k0 + 2 * t]), s0);
            ah[1] = mul_h2(ld_h2(&sc.hi[r0 + g + 8][k0 + 2 * t]), s0);
            ah[2] = mul_h2(ld_h2(&sc.hi[r0 + g][k0 + 2 * t + 8]), s1);
            ah[3] = mul_h2(ld_h2(&sc.hi[r0 + g + 8][k0 + 2 * t + 8]), s1);
            al[0] = mul_h2(ld_h2(&sc.lo[r0 + g][k0 + 2 * t]), s0);
            al[1] = mul_h2(ld_h2(&sc.lo[r0 + g + 8][k0 + 2 * t]), s0);
            al[2] = mul_h2(ld_h2(&sc.lo[r0 + g][k0 + 2 * t + 8]), s1);
            al[3] = mul_h2(ld_h2(&sc.lo[r0 + g + 8][k0 + 2 * t + 8]), s1);
            bh[0] = ld_h2(&sc.hi[c0 + g][k0 + 2 * t]);
            bh[1] = ld_h2(&sc.hi[c0 + g][k0 + 2 * t + 8]);
            bl[0] = ld_h2(&sc.lo[c0 + g][k0 + 2 * t]);
            bl[1] = ld_h2(&sc.lo[c0 + g][k0 + 2 * t + 8]);
            mma_16816(acc, al, bh);
            mma_16816(acc, ah, bl);
            mma_16816(acc, ah, bh);
        }
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int r = r0 + g + (q >> 1) * 8, c = c0 + 2 * t + (q & 1);
            if (r < 60 && c < 60 && r <= c) store(r, c, (double)acc[q] * sc.inv_s2);
        }
    }
}

}  // namespace hex20
}  // namespace fem
