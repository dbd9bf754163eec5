// Plane-stress element stiffness of Q4 and T3 elements in FP64, node-block form.
//
// The reference computes ke[m][n] = sum_gp sum_kl B[k][m] D[k][l] B[l][n] w detJ t
// with a 3x8 (Q4, ALLS_Quad2D_Assembly_Accuracy_Analysis.cu:128-212) or 3x6 (T3,
// ALLS_T3_Unstructed_Elements_Assemble_Performance.cu:177-205) B matrix. B has
// only two nonzeros per column, so for nodes a, b with shape-function gradients
// (xa, ya), (xb, yb) and D = [[d11 d12 0][d12 d11 0][0 0 d33]] the 2x2 block is
//     K_ab = w * [ d11 xa xb + d33 ya yb    d12 xa yb + d33 ya xb ]
//                [ d12 ya xb + d33 xa yb    d11 ya yb + d33 xa xb ]
// which is what ke_block_2d accumulates (8 FMAs per block per Gauss point;
// K_ba = K_ab^T). D uses each element's own E and nu.
#pragma once

namespace fem {

__device__ __forceinline__ void plane_stress_d(double E, double nu, double& d11, double& d12, double& d33) {
    double f = E / (1.0 - nu * nu);
    d11 = f;
    d12 = f * nu;
    d33 = f * (1.0 - nu) / 2.0;
}

// One block K_ab (entries a_dof * 2 + b_dof) of a T3 or Q4 element, computed
// by the lane that scatters it. The inverse Jacobian uses one reciprocal of
// detJ per point (the reference divides four times; the results agree to the
// last bits). Returns detJ (Q4: the smallest over the Gauss points).
template <int NPE>
__device__ __forceinline__ double ke_block_2d(const double (&x)[NPE], const double (&y)[NPE], double E, double nu,
                                              double t, int a, int b, double (&kv)[4]) {
    double d11, d12, d33;
    plane_stress_d(E, nu, d11, d12, d33);
    kv[0] = kv[1] = kv[2] = kv[3] = 0.0;
    if constexpr (NPE == 3) {
        // dN/dxi = (-1, 1, 0), dN/deta = (-1, 0, 1)
        const double j0 = x[1] - x[0], j1 = y[1] - y[0], j2 = x[2] - x[0], j3 = y[2] - y[0];
        const double det = j0 * j3 - j1 * j2;
        const double r = 1.0 / det;
        const double i0 = j3 * r, i1 = -j1 * r, i2 = -j2 * r, i3 = j0 * r;
        const double xa = a == 0 ? -i0 - i1 : (a == 1 ? i0 : i1);
        const double ya = a == 0 ? -i2 - i3 : (a == 1 ? i2 : i3);
        const double xb = b == 0 ? -i0 - i1 : (b == 1 ? i0 : i1);
        const double yb = b == 0 ? -i2 - i3 : (b == 1 ? i2 : i3);
        const double w = 0.5 * det * t;
        const double wxa = w * xa, wya = w * ya;
        kv[0] = fma(d11 * wxa, xb, d33 * wya * yb);
        kv[1] = fma(d12 * wxa, yb, d33 * wya * xb);
        kv[2] = fma(d12 * wya, xb, d33 * wxa * yb);
        kv[3] = fma(d11 * wya, yb, d33 * wxa * xb);
        return det;
    } else {
        constexpr double g = 0.577350269189626;  // Q4A:85
        // natural coordinates of the four nodes
        const double sa = (a == 1 || a == 2) ? 1.0 : -1.0, ta = a >= 2 ? 1.0 : -1.0;
        const double sb = (b == 1 || b == 2) ? 1.0 : -1.0, tb = b >= 2 ? 1.0 : -1.0;
        double min_det = 1e300;
#pragma unroll
        for (int gi = 0; gi < 2; gi++) {
#pragma unroll
            for (int gj = 0; gj < 2; gj++) {
                const double xi = gi ? g : -g, eta = gj ? g : -g;
                const double dxi[4] = {-0.25 * (1.0 - eta), 0.25 * (1.0 - eta), 0.25 * (1.0 + eta), -0.25 * (1.0 + eta)};
                const double deta[4] = {-0.25 * (1.0 - xi), -0.25 * (1.0 + xi), 0.25 * (1.0 + xi), 0.25 * (1.0 - xi)};
                double j0 = 0.0, j1 = 0.0, j2 = 0.0, j3 = 0.0;
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    j0 = fma(dxi[k], x[k], j0);
                    j1 = fma(dxi[k], y[k], j1);
                    j2 = fma(deta[k], x[k], j2);
                    j3 = fma(deta[k], y[k], j3);
                }
                const double det = j0 * j3 - j1 * j2;
                min_det = fmin(min_det, det);
                const double r = 1.0 / det;
                const double i0 = j3 * r, i1 = -j1 * r, i2 = -j2 * r, i3 = j0 * r;
                const double dxa = 0.25 * sa * (1.0 + ta * eta), dea = 0.25 * ta * (1.0 + sa * xi);
                const double dxb = 0.25 * sb * (1.0 + tb * eta), deb = 0.25 * tb * (1.0 + sb * xi);
                const double xa = fma(i0, dxa, i1 * dea), ya = fma(i2, dxa, i3 * dea);
                const double xb = fma(i0, dxb, i1 * deb), yb = fma(i2, dxb, i3 * deb);
                const double w = det * t;
                const double wxa = w * xa, wya = w * ya;
                kv[0] = fma(d11 * wxa, xb, fma(d33 * wya, yb, kv[0]));
                kv[1] = fma(d12 * wxa, yb, fma(d33 * wya, xb, kv[1]));
                kv[2] = fma(d12 * wya, xb, fma(d33 * wxa, yb, kv[2]));
                kv[3] = fma(d11 * wya, yb, fma(d33 * wxa, xb, kv[3]));
            }
        }
        return min_det;
    }
}

}  // namespace fem
