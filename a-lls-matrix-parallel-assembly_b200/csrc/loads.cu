// The steps after the assembled matrix: the body-force load vector and the
// Dirichlet (prescribed-displacement) boundary conditions, on the device.
// The reference stops at the assembled stiffness values; these kernels let
// the assembled system be handed to a solver without a host round trip.
//
// Body force: f_a += integral of N_a b over the element (per-element or
// uniform force per volume; 2-D kinds per area and times the thickness):
//   T3   one point: A/3 per node (A = detJ / 2);
//   Q4   2x2 Gauss with the bilinear N_a;
//   Hex20 3x3x3 Gauss with the 20-node serendipity N_a (one warp per element:
//        lane g handles Gauss point g, then each node's 27 terms are summed
//        across the lanes before one atomic per dof).
// Dirichlet: symmetric elimination in place on the CSR matrix: for every
// entry K_jc with c fixed and j free, f_j -= K_jc u_c and K_jc = 0; a fixed
// row keeps only K_ii = 1 and gets f_i = u_i. The matrix stays symmetric.
#include <algorithm>

#include "hex20.cuh"
#include "launch.h"

namespace fem {
namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ double elem_force(const double* b, double b0, const MeshView& m, int e, int dim, int d) {
    return b ? __ldg(b + (size_t)e * dim + d) : b0;
}

// 2-D kinds: one thread per element.
__global__ void k_body_force_2d(MeshView m, const double* __restrict__ b, double bx0, double by0, double* f,
                                int* status) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < m.E_count; e += gridDim.x * blockDim.x) {
        const bool q4 = m.types ? __ldg(m.types + e) == FEM_Q4 : m.stride == 4;
        const int npe = q4 ? 4 : 3;
        int n[4];
        bool bad = false;
        for (int k = 0; k < npe; k++) {
            n[k] = __ldg(m.conn + (size_t)e * m.stride + k);
            bad |= n[k] < 0 || n[k] >= m.N;
        }
        if (bad) {
            atomicOr(status, 1 << FEM_ERR_BAD_MESH);
            continue;
        }
        double x[4], y[4], wn[4] = {0.0, 0.0, 0.0, 0.0};
        for (int k = 0; k < npe; k++) {
            x[k] = __ldg(m.x + n[k]);
            y[k] = __ldg(m.y + n[k]);
        }
        if (!q4) {
            const double det = (x[1] - x[0]) * (y[2] - y[0]) - (y[1] - y[0]) * (x[2] - x[0]);
            if (!(det > 0.0)) atomicOr(status, 1 << FEM_ERR_DETJ);
            wn[0] = wn[1] = wn[2] = det / 6.0;  // (det / 2) / 3
        } else {
            constexpr double g = 0.577350269189626;
            for (int gi = 0; gi < 2; gi++)
                for (int gj = 0; gj < 2; gj++) {
                    const double xi = gi ? g : -g, eta = gj ? g : -g;
                    const double dxi[4] = {-0.25 * (1.0 - eta), 0.25 * (1.0 - eta), 0.25 * (1.0 + eta),
                                           -0.25 * (1.0 + eta)};
                    const double deta[4] = {-0.25 * (1.0 - xi), -0.25 * (1.0 + xi), 0.25 * (1.0 + xi),
                                            0.25 * (1.0 - xi)};
                    const double N[4] = {0.25 * (1.0 - xi) * (1.0 - eta), 0.25 * (1.0 + xi) * (1.0 - eta),
                                         0.25 * (1.0 + xi) * (1.0 + eta), 0.25 * (1.0 - xi) * (1.0 + eta)};
                    double j0 = 0.0, j1 = 0.0, j2 = 0.0, j3 = 0.0;
                    for (int k = 0; k < 4; k++) {
                        j0 = fma(dxi[k], x[k], j0);
                        j1 = fma(dxi[k], y[k], j1);
                        j2 = fma(deta[k], x[k], j2);
                        j3 = fma(deta[k], y[k], j3);
                    }
                    const double det = j0 * j3 - j1 * j2;
                    if (!(det > 0.0)) atomicOr(status, 1 << FEM_ERR_DETJ);
                    for (int k = 0; k < 4; k++) wn[k] = fma(N[k], det, wn[k]);
                }
        }
        const double bx = elem_force(b, bx0, m, e, 2, 0) * m.t, by = elem_force(b, by0, m, e, 2, 1) * m.t;
        for (int k = 0; k < npe; k++) {
            atomicAdd(f + 2 * n[k], wn[k] * bx);
            atomicAdd(f + 2 * n[k] + 1, wn[k] * by);
        }
    }
}

// Serendipity shape function N_n at (xi, eta, zeta) in the reference node order.
__device__ __forceinline__ double hex20_shape(int n, double xi, double eta, double zeta) {
    const double a = hex20::xi_of(n), b = hex20::eta_of(n), c = hex20::zeta_of(n);
    if (n < 8) return 0.125 * (1.0 + a * xi) * (1.0 + b * eta) * (1.0 + c * zeta) * (a * xi + b * eta + c * zeta - 2.0);
    if (n == 8 || n == 10 || n == 12 || n == 14) return 0.25 * (1.0 - xi * xi) * (1.0 + b * eta) * (1.0 + c * zeta);
    if (n < 16) return 0.25 * (1.0 + a * xi) * (1.0 - eta * eta) * (1.0 + c * zeta);
    return 0.25 * (1.0 + a * xi) * (1.0 + b * eta) * (1.0 - zeta * zeta);
}

// Hex20: one warp per element, lane g = Gauss point g.
__global__ void k_body_force_hex20(MeshView m, const double* __restrict__ b, double bx0, double by0, double bz0,
                                   double* f, int* status) {
    const int lane = threadIdx.x & 31;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long warps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long e = warp; e < m.E_count; e += warps) {
        const int nl = lane < 20 ? __ldg(m.conn + (size_t)e * 20 + lane) : 0;
        if (__any_sync(0xFFFFFFFFu, lane < 20 && (nl < 0 || nl >= m.N))) {
            if (lane == 0) atomicOr(status, 1 << FEM_ERR_BAD_MESH);
            continue;
        }
        const double xl = lane < 20 ? __ldg(m.x + nl) : 0.0, yl = lane < 20 ? __ldg(m.y + nl) : 0.0,
                     zl = lane < 20 ? __ldg(m.z + nl) : 0.0;
        double wdet = 0.0, xi = 0.0, eta = 0.0, zeta = 0.0;
        {
            const int g = lane < 27 ? lane : 0;
            xi = hex20::gauss3(g / 9);
            eta = hex20::gauss3((g / 3) % 3);
            zeta = hex20::gauss3(g % 3);
            double J[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
            for (int n = 0; n < 20; n++) {
                double d[3];
                hex20::dshape_node(n, xi, eta, zeta, d[0], d[1], d[2]);
                const double xn = __shfl_sync(0xFFFFFFFFu, xl, n), yn = __shfl_sync(0xFFFFFFFFu, yl, n),
                             zn = __shfl_sync(0xFFFFFFFFu, zl, n);
                for (int i = 0; i < 3; i++) {
                    J[3 * i] = fma(d[i], xn, J[3 * i]);
                    J[3 * i + 1] = fma(d[i], yn, J[3 * i + 1]);
                    J[3 * i + 2] = fma(d[i], zn, J[3 * i + 2]);
                }
            }
            const double det = J[0] * (J[4] * J[8] - J[5] * J[7]) + J[1] * (J[5] * J[6] - J[3] * J[8]) +
                               J[2] * (J[3] * J[7] - J[4] * J[6]);
            if (lane < 27 && !(det > 0.0)) atomicOr(status, 1 << FEM_ERR_DETJ);
            wdet = lane < 27 ? hex20::weight3(g / 9) * hex20::weight3((g / 3) % 3) * hex20::weight3(g % 3) * det : 0.0;
        }
        // node n's integral of N_n: sum over the Gauss-point lanes
        double mine = 0.0;
        for (int n = 0; n < 20; n++) {
            double v = lane < 27 ? hex20_shape(n, xi, eta, zeta) * wdet : 0.0;
#pragma unroll
            for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, d);
            if (lane == n) mine = v;
        }
        if (lane < 20) {
            const double bx = elem_force(b, bx0, m, (int)e, 3, 0), by = elem_force(b, by0, m, (int)e, 3, 1),
                         bz = elem_force(b, bz0, m, (int)e, 3, 2);
            atomicAdd(f + 3 * nl, mine * bx);
            atomicAdd(f + 3 * nl + 1, mine * by);
            atomicAdd(f + 3 * nl + 2, mine * bz);
        }
    }
}

// One warp per CSR row.
__global__ void k_dirichlet(int n_rows, const int* __restrict__ row_ptr, const int* __restrict__ col_idx,
                            double* __restrict__ values, double* __restrict__ f, const unsigned char* __restrict__ fixed,
                            const double* __restrict__ u) {
    const int lane = threadIdx.x & 31;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long warps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long r = warp; r < n_rows; r += warps) {
        const int b = __ldg(row_ptr + r), e = __ldg(row_ptr + r + 1);
        const bool row_fixed = __ldg(fixed + r) != 0;
        double df = 0.0;
        for (int k = b + lane; k < e; k += 32) {
            const int c = __ldg(col_idx + k);
            if (row_fixed) {
                values[k] = c == r ? 1.0 : 0.0;
            } else if (__ldg(fixed + c)) {
                df = fma(-values[k], __ldg(u + c), df);
                values[k] = 0.0;
            }
        }
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) df += __shfl_xor_sync(0xFFFFFFFFu, df, d);
        if (lane == 0 && f) f[r] = row_fixed ? __ldg(u + r) : f[r] + df;
    }
}

}  // namespace

cudaError_t launch_body_force(const MeshView& m, int kind, const double* b, const double* b0, double* f, int* status,
                              cudaStream_t s) {
    if (m.E_count <= 0) return cudaSuccess;
    const int sms = sm_count();
    if (kind == FEM_HEX20) {
        const long long want = ((long long)m.E_count * 32 + kThreads - 1) / kThreads;
        k_body_force_hex20<<<(int)std::min<long long>(want, (long long)sms * 16), kThreads, 0, s>>>(
            m, b, b0[0], b0[1], b0[2], f, status);
    } else {
        const long long want = ((long long)m.E_count + kThreads - 1) / kThreads;
        k_body_force_2d<<<(int)std::min<long long>(want, (long long)sms * 16), kThreads, 0, s>>>(m, b, b0[0], b0[1],
                                                                                                f, status);
    }
    return cudaGetLastError();
}

cudaError_t launch_dirichlet(int n_rows, const int* row_ptr, const int* col_idx, double* values, double* f,
                             const unsigned char* fixed, const double* u, cudaStream_t s) {
    if (n_rows <= 0) return cudaSuccess;
    const long long want = ((long long)n_rows * 32 + kThreads - 1) / kThreads;
    k_dirichlet<<<(int)std::min<long long>(want, (long long)sm_count() * 16), kThreads, 0, s>>>(
        n_rows, row_ptr, col_idx, values, f, fixed, u);
    return cudaGetLastError();
}

}  // namespace fem
