// Hex20 element definitions shared by the element-stiffness kernels
// (element_stiffness.cu, ke_tcgen05.cu) and the two-pass A-LLS scatter (values_hex20.cuh).
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

}  // namespace hex20
}  // namespace fem
