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
//
// ke_block_2d<NPE, float> is the FP32 form (FEM_PREC_FP32): the node
// coordinates are taken relative to node 0 in FP64 (the Jacobian is
// translation-invariant, so no digits of the element's size are lost to its
// position), rounded to FP32, and the block is computed in FP32; it is
// returned in FP64 and accumulated in FP64 like the plain form.
#pragma once

namespace fem {

template <typename T>
__device__ __forceinline__ void plane_stress_d(T E, T nu, T& d11, T& d12, T& d33) {
    T f = E / (T(1) - nu * nu);
    d11 = f;
    d12 = f * nu;
    d33 = f * (T(1) - nu) / T(2);
}

// One block K_ab (entries a_dof * 2 + b_dof) of a T3 or Q4 element, computed
// by the lane that scatters it, in the arithmetic type T (double: the plain
// FP64 form; float: FEM_PREC_FP32). The inverse Jacobian uses one reciprocal
// of detJ per point (the reference divides four times; the results agree to
// the last bits). Returns detJ (Q4: the smallest over the Gauss points).
template <int NPE, typename T = double>
__device__ __forceinline__ double ke_block_2d(const double (&xd)[NPE], const double (&yd)[NPE], double Ed, double nud,
                                              double td, int a, int b, double (&kv)[4]) {
    T x[NPE], y[NPE];
#pragma unroll
    for (int k = 0; k < NPE; k++) {
        // FP64: the coordinates themselves (bit-identical to the reference's
        // arithmetic); FP32: relative to node 0, differenced in FP64
        x[k] = sizeof(T) == 8 ? T(xd[k]) : T(xd[k] - xd[0]);
        y[k] = sizeof(T) == 8 ? T(yd[k]) : T(yd[k] - yd[0]);
    }
    const T E = T(Ed), nu = T(nud), t = T(td);
    T d11, d12, d33;
    plane_stress_d<T>(E, nu, d11, d12, d33);
    T k0 = T(0), k1 = T(0), k2 = T(0), k3 = T(0);
    double det_out;
    if constexpr (NPE == 3) {
        // dN/dxi = (-1, 1, 0), dN/deta = (-1, 0, 1)
        const T j0 = x[1] - x[0], j1 = y[1] - y[0], j2 = x[2] - x[0], j3 = y[2] - y[0];
        const T det = j0 * j3 - j1 * j2;
        const T r = T(1) / det;
        const T i0 = j3 * r, i1 = -j1 * r, i2 = -j2 * r, i3 = j0 * r;
        const T xa = a == 0 ? -i0 - i1 : (a == 1 ? i0 : i1);
        const T ya = a == 0 ? -i2 - i3 : (a == 1 ? i2 : i3);
        const T xb = b == 0 ? -i0 - i1 : (b == 1 ? i0 : i1);
        const T yb = b == 0 ? -i2 - i3 : (b == 1 ? i2 : i3);
        const T w = T(0.5) * det * t;
        const T wxa = w * xa, wya = w * ya;
        k0 = fma(d11 * wxa, xb, d33 * wya * yb);
        k1 = fma(d12 * wxa, yb, d33 * wya * xb);
        k2 = fma(d12 * wya, xb, d33 * wxa * yb);
        k3 = fma(d11 * wya, yb, d33 * wxa * xb);
        det_out = double(det);
    } else {
        constexpr double g = 0.577350269189626;  // Q4A:85
        // natural coordinates of the four nodes
        const T sa = (a == 1 || a == 2) ? T(1) : T(-1), ta = a >= 2 ? T(1) : T(-1);
        const T sb = (b == 1 || b == 2) ? T(1) : T(-1), tb = b >= 2 ? T(1) : T(-1);
        T min_det = sizeof(T) == 8 ? T(1e300) : T(3.0e38f);
#pragma unroll
        for (int gi = 0; gi < 2; gi++) {
#pragma unroll
            for (int gj = 0; gj < 2; gj++) {
                const T xi = T(gi ? g : -g), eta = T(gj ? g : -g);
                const T q = T(0.25);
                const T dxi[4] = {-q * (T(1) - eta), q * (T(1) - eta), q * (T(1) + eta), -q * (T(1) + eta)};
                const T deta[4] = {-q * (T(1) - xi), -q * (T(1) + xi), q * (T(1) + xi), q * (T(1) - xi)};
                T j0 = T(0), j1 = T(0), j2 = T(0), j3 = T(0);
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    j0 = fma(dxi[k], x[k], j0);
                    j1 = fma(dxi[k], y[k], j1);
                    j2 = fma(deta[k], x[k], j2);
                    j3 = fma(deta[k], y[k], j3);
                }
                const T det = j0 * j3 - j1 * j2;
                min_det = fmin(min_det, det);
                const T r = T(1) / det;
                const T i0 = j3 * r, i1 = -j1 * r, i2 = -j2 * r, i3 = j0 * r;
                const T dxa = q * sa * (T(1) + ta * eta), dea = q * ta * (T(1) + sa * xi);
                const T dxb = q * sb * (T(1) + tb * eta), deb = q * tb * (T(1) + sb * xi);
                const T xa = fma(i0, dxa, i1 * dea), ya = fma(i2, dxa, i3 * dea);
                const T xb = fma(i0, dxb, i1 * deb), yb = fma(i2, dxb, i3 * deb);
                const T w = det * t;
                const T wxa = w * xa, wya = w * ya;
                k0 = fma(d11 * wxa, xb, fma(d33 * wya, yb, k0));
                k1 = fma(d12 * wxa, yb, fma(d33 * wya, xb, k1));
                k2 = fma(d12 * wya, xb, fma(d33 * wxa, yb, k2));
                k3 = fma(d11 * wya, yb, fma(d33 * wxa, xb, k3));
            }
        }
        det_out = double(min_det);
    }
    kv[0] = double(k0);
    kv[1] = double(k1);
    kv[2] = double(k2);
    kv[3] = double(k3);
    return det_out;
}

}  // namespace fem
