/*
 * CPU oracle for the FEM global-stiffness assembly path (TEST INFRASTRUCTURE).
 *
 * A plain-C restatement of the reference's serial algorithm, used only as the
 * checker of the CUDA library (tests, smoke, bench cpu_baseline). Every function
 * cites the reference lines it restates; the arithmetic follows the reference's
 * own operation order so that, compiled without FP contraction
 * (-ffp-contract=off, as the reference's host code is compiled for x86-64), the
 * Q4 results match the reference's assembleGlobalStiffnessHost bit for bit.
 *
 * Parity pins (tests/golden): pattern and Q4 values vs the reference's host code
 * built from its own sources (oracle/_ref); T3 / Q4-in-mixed / Hex20 element
 * stiffness vs the reference's device functions run on a B200.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------------------
 * Q4 plane stress (ALLS_Quad2D_Assembly_Accuracy_Analysis.cu)
 * ------------------------------------------------------------------------- */

/* Gauss abscissae and weights as the reference writes them (Q4A:47-48). */
static const double kQ4Gauss[2] = {-0.577350269189626, 0.577350269189626};
static const double kQ4Weight[2] = {1.0, 1.0};

/* Plane-stress D (Q4A:281-289), per element E and nu. */
static void d_plane_stress(double E, double nu, double D[9]) {
    double factor = E / (1.0 - nu * nu);
    D[0] = factor;      D[1] = factor * nu; D[2] = 0.0;
    D[3] = factor * nu; D[4] = factor;      D[5] = 0.0;
    D[6] = 0.0;         D[7] = 0.0;         D[8] = factor * (1.0 - nu) / 2.0;
}

/* Q4A:225-241 (shape function derivatives). */
static void q4_dshape(double xi, double eta, double dxi[4], double deta[4]) {
    dxi[0] = -0.25 * (1.0 - eta);
    dxi[1] = 0.25 * (1.0 - eta);
    dxi[2] = 0.25 * (1.0 + eta);
    dxi[3] = -0.25 * (1.0 + eta);
    deta[0] = -0.25 * (1.0 - xi);
    deta[1] = -0.25 * (1.0 + xi);
    deta[2] = 0.25 * (1.0 + xi);
    deta[3] = 0.25 * (1.0 - xi);
}

int oracle_ke_q4(const double x[4], const double y[4], double E, double nu, double t,
                 double ke[64]) {
    /* Q4A:292-326: ke = sum_gp (B^T D B) * w * detJ * t, summed B[k,m]*D[k,l]*B[l,n]. */
    int clamped = 0;
    double D[9];
    d_plane_stress(E, nu, D);
    for (int i = 0; i < 64; i++) ke[i] = 0.0;
    for (int gi = 0; gi < 2; gi++) {
        for (int gj = 0; gj < 2; gj++) {
            double xi = kQ4Gauss[gi], eta = kQ4Gauss[gj];
            double weight = kQ4Weight[gi] * kQ4Weight[gj];
            double dxi[4], deta[4];
            q4_dshape(xi, eta, dxi, deta);
            /* Q4A:243-277 (Jacobian, inverse, B). */
            double J[4] = {0.0, 0.0, 0.0, 0.0};
            for (int i = 0; i < 4; i++) {
                J[0] += dxi[i] * x[i];
                J[1] += dxi[i] * y[i];
                J[2] += deta[i] * x[i];
                J[3] += deta[i] * y[i];
            }
            double detJ = J[0] * J[3] - J[1] * J[2];
            if (fabs(detJ) < 1e-10) { detJ = 1e-10; clamped++; }
            double invJ[4] = {J[3] / detJ, -J[1] / detJ, -J[2] / detJ, J[0] / detJ};
            double B[24];
            for (int i = 0; i < 4; i++) {
                double dNdx = invJ[0] * dxi[i] + invJ[1] * deta[i];
                double dNdy = invJ[2] * dxi[i] + invJ[3] * deta[i];
                B[0 * 8 + 2 * i] = dNdx;     B[0 * 8 + 2 * i + 1] = 0.0;
                B[1 * 8 + 2 * i] = 0.0;      B[1 * 8 + 2 * i + 1] = dNdy;
                B[2 * 8 + 2 * i] = dNdy;     B[2 * 8 + 2 * i + 1] = dNdx;
            }
            double w = weight * detJ * t;
            for (int m = 0; m < 8; m++) {
                for (int n = 0; n < 8; n++) {
                    double sum = 0.0;
                    for (int k = 0; k < 3; k++)
                        for (int l = 0; l < 3; l++)
                            sum += B[k * 8 + m] * D[k * 3 + l] * B[l * 8 + n];
                    ke[m * 8 + n] += sum * w;
                }
            }
        }
    }
    return clamped;
}

/* ---------------------------------------------------------------------------
 * T3 constant-strain triangle (ALLS_T3_Unstructed_Elements_Assemble_Performance.cu)
 * ------------------------------------------------------------------------- */

int oracle_ke_t3(const double x[3], const double y[3], double E, double nu, double t,
                 double ke[36]) {
    /* T3:131-134 (constant dN/dxi), T3:177-205 (J, B 3x6, w = 0.5*detJ*t,
     * ke = sum_k B[k,r] * (sum_l D[k,l] B[l,c])). */
    static const double dxi[3] = {-1.0, 1.0, 0.0};
    static const double deta[3] = {-1.0, 0.0, 1.0};
    double D[9];
    d_plane_stress(E, nu, D);
    double J[4] = {0.0, 0.0, 0.0, 0.0};
    for (int k = 0; k < 3; k++) {
        J[0] += dxi[k] * x[k];
        J[1] += dxi[k] * y[k];
        J[2] += deta[k] * x[k];
        J[3] += deta[k] * y[k];
    }
    double detJ = J[0] * J[3] - J[1] * J[2];
    double invJ[4] = {J[3] / detJ, -J[1] / detJ, -J[2] / detJ, J[0] / detJ};
    double w = 0.5 * detJ * t;
    double B[18];
    for (int i = 0; i < 18; i++) B[i] = 0.0;
    for (int k = 0; k < 3; k++) {
        double dNdx = invJ[0] * dxi[k] + invJ[1] * deta[k];
        double dNdy = invJ[2] * dxi[k] + invJ[3] * deta[k];
        B[0 * 6 + 2 * k] = dNdx;
        B[1 * 6 + 2 * k + 1] = dNdy;
        B[2 * 6 + 2 * k] = dNdy;
        B[2 * 6 + 2 * k + 1] = dNdx;
    }
    for (int r = 0; r < 6; r++) {
        for (int c = 0; c < 6; c++) {
            double sum = 0.0;
            for (int k = 0; k < 3; k++) {
                double dval = 0.0;
                for (int l = 0; l < 3; l++) dval += D[k * 3 + l] * B[l * 6 + c];
                sum += B[k * 6 + r] * dval;
            }
            ke[r * 6 + c] = 0.0 + sum * w;
        }
    }
    return detJ <= 0.0 ? 1 : 0;
}

/* ---------------------------------------------------------------------------
 * Hex20 serendipity (ALLS_Hex20_3D_Assembly_Performance.cu), in double
 * ------------------------------------------------------------------------- */

/* Gauss abscissae and weights as the reference writes them (H20:45-46). */
static const double kH20Gauss[3] = {-0.774596669241483, 0.0, 0.774596669241483};
static const double kH20Weight[3] = {0.555555555555556, 0.888888888888889, 0.555555555555556};

/* Natural coordinates of the 20 nodes (H20:97-99). */
static const double kXiN[20] = {-1, 1, 1, -1, -1, 1, 1, -1, 0, 1, 0, -1, 0, 1, 0, -1, -1, 1, 1, -1};
static const double kEtaN[20] = {-1, -1, 1, 1, -1, -1, 1, 1, -1, 0, 1, 0, -1, 0, 1, 0, -1, -1, 1, 1};
static const double kZetaN[20] = {-1, -1, -1, -1, 1, 1, 1, 1, -1, -1, -1, -1, 1, 1, 1, 1, 0, 0, 0, 0};

/* H20:95-128: derivatives of the serendipity shape functions. */
static void hex20_dshape(double xi, double eta, double zeta, double dxi[20], double deta[20],
                         double dzeta[20]) {
    for (int i = 0; i < 8; i++) {
        double a = kXiN[i], b = kEtaN[i], c = kZetaN[i];
        dxi[i] = 0.125 * a * (1.0 + b * eta) * (1.0 + c * zeta) * (2.0 * a * xi + b * eta + c * zeta - 1.0);
        deta[i] = 0.125 * b * (1.0 + a * xi) * (1.0 + c * zeta) * (a * xi + 2.0 * b * eta + c * zeta - 1.0);
        dzeta[i] = 0.125 * c * (1.0 + a * xi) * (1.0 + b * eta) * (a * xi + b * eta + 2.0 * c * zeta - 1.0);
    }
    static const int g1[4] = {8, 10, 12, 14};
    for (int q = 0; q < 4; q++) {
        int i = g1[q];
        double b = kEtaN[i], c = kZetaN[i];
        dxi[i] = -0.5 * xi * (1.0 + b * eta) * (1.0 + c * zeta);
        deta[i] = 0.25 * b * (1.0 - xi * xi) * (1.0 + c * zeta);
        dzeta[i] = 0.25 * c * (1.0 - xi * xi) * (1.0 + b * eta);
    }
    static const int g2[4] = {9, 11, 13, 15};
    for (int q = 0; q < 4; q++) {
        int i = g2[q];
        double a = kXiN[i], c = kZetaN[i];
        dxi[i] = 0.25 * a * (1.0 - eta * eta) * (1.0 + c * zeta);
        deta[i] = -0.5 * eta * (1.0 + a * xi) * (1.0 + c * zeta);
        dzeta[i] = 0.25 * c * (1.0 + a * xi) * (1.0 - eta * eta);
    }
    for (int i = 16; i < 20; i++) {
        double a = kXiN[i], b = kEtaN[i];
        dxi[i] = 0.25 * a * (1.0 + b * eta) * (1.0 - zeta * zeta);
        deta[i] = 0.25 * b * (1.0 + a * xi) * (1.0 - zeta * zeta);
        dzeta[i] = -0.5 * zeta * (1.0 + a * xi) * (1.0 + b * eta);
    }
}

int oracle_ke_hex20(const double x[20], const double y[20], const double z[20], double E,
                    double nu, double ke[3600]) {
    /* H20:130-195 in double: isotropic node-pair block formula with
     * c1 = lambda + 2 mu, c2 = lambda, c3 = mu (H20:135-137,173-191). */
    int clamped = 0;
    double lambda = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
    double mu = E / (2.0 * (1.0 + nu));
    double c1 = lambda + 2.0 * mu, c2 = lambda, c3 = mu;
    for (int i = 0; i < 3600; i++) ke[i] = 0.0;
    for (int gi = 0; gi < 3; gi++) {
        for (int gj = 0; gj < 3; gj++) {
            for (int gk = 0; gk < 3; gk++) {
                double xi = kH20Gauss[gi], eta = kH20Gauss[gj], zeta = kH20Gauss[gk];
                double weight = kH20Weight[gi] * kH20Weight[gj] * kH20Weight[gk];
                double dxi[20], deta[20], dzeta[20];
                hex20_dshape(xi, eta, zeta, dxi, deta, dzeta);
                double J[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
                for (int m = 0; m < 20; m++) {
                    J[0] += dxi[m] * x[m];   J[1] += dxi[m] * y[m];   J[2] += dxi[m] * z[m];
                    J[3] += deta[m] * x[m];  J[4] += deta[m] * y[m];  J[5] += deta[m] * z[m];
                    J[6] += dzeta[m] * x[m]; J[7] += dzeta[m] * y[m]; J[8] += dzeta[m] * z[m];
                }
                double detJ = J[0] * (J[4] * J[8] - J[5] * J[7]) - J[1] * (J[3] * J[8] - J[5] * J[6]) +
                              J[2] * (J[3] * J[7] - J[4] * J[6]);
                if (fabs(detJ) < 1e-15) { detJ = 1e-15; clamped++; }
                double iJ[9];
                iJ[0] = (J[4] * J[8] - J[5] * J[7]) / detJ;
                iJ[1] = (J[2] * J[7] - J[1] * J[8]) / detJ;
                iJ[2] = (J[1] * J[5] - J[2] * J[4]) / detJ;
                iJ[3] = (J[5] * J[6] - J[3] * J[8]) / detJ;
                iJ[4] = (J[0] * J[8] - J[2] * J[6]) / detJ;
                iJ[5] = (J[2] * J[3] - J[0] * J[5]) / detJ;
                iJ[6] = (J[3] * J[7] - J[4] * J[6]) / detJ;
                iJ[7] = (J[1] * J[6] - J[0] * J[7]) / detJ;
                iJ[8] = (J[0] * J[4] - J[1] * J[3]) / detJ;
                double gx[20], gy[20], gz[20];
                for (int m = 0; m < 20; m++) {
                    gx[m] = iJ[0] * dxi[m] + iJ[1] * deta[m] + iJ[2] * dzeta[m];
                    gy[m] = iJ[3] * dxi[m] + iJ[4] * deta[m] + iJ[5] * dzeta[m];
                    gz[m] = iJ[6] * dxi[m] + iJ[7] * deta[m] + iJ[8] * dzeta[m];
                }
                double w = weight * detJ;
                for (int I = 0; I < 20; I++) {
                    for (int Jn = 0; Jn < 20; Jn++) {
                        int r0 = I * 3, c0 = Jn * 3;
                        double xI = gx[I], yI = gy[I], zI = gz[I];
                        double xJ = gx[Jn], yJ = gy[Jn], zJ = gz[Jn];
                        ke[(r0 + 0) * 60 + (c0 + 0)] += (c1 * xI * xJ + c3 * yI * yJ + c3 * zI * zJ) * w;
                        ke[(r0 + 0) * 60 + (c0 + 1)] += (c2 * xI * yJ + c3 * yI * xJ) * w;
                        ke[(r0 + 0) * 60 + (c0 + 2)] += (c2 * xI * zJ + c3 * zI * xJ) * w;
                        ke[(r0 + 1) * 60 + (c0 + 0)] += (c3 * xI * yJ + c2 * yI * xJ) * w;
                        ke[(r0 + 1) * 60 + (c0 + 1)] += (c3 * xI * xJ + c1 * yI * yJ + c3 * zI * zJ) * w;
                        ke[(r0 + 1) * 60 + (c0 + 2)] += (c2 * yI * zJ + c3 * zI * yJ) * w;
                        ke[(r0 + 2) * 60 + (c0 + 0)] += (c3 * xI * zJ + c2 * zI * xJ) * w;
                        ke[(r0 + 2) * 60 + (c0 + 1)] += (c3 * yI * zJ + c2 * zI * yJ) * w;
                        ke[(r0 + 2) * 60 + (c0 + 2)] += (c3 * xI * xJ + c3 * yI * yJ + c1 * zI * zJ) * w;
                    }
                }
            }
        }
    }
    return clamped;
}

/* ---------------------------------------------------------------------------
 * Pattern and serial assembly
 * ------------------------------------------------------------------------- */

static int kind_dpn(int kind) { return kind == ORACLE_HEX20 ? 3 : 2; }

static int elem_nodes(int kind, const uint8_t* types, int32_t e) {
    switch (kind) {
        case ORACLE_Q4: return 4;
        case ORACLE_T3: return 3;
        case ORACLE_HEX20: return 20;
        default: return types[e] == ORACLE_Q4 ? 4 : 3;
    }
}

static int cmp_i32(const void* a, const void* b) {
    int32_t x = *(const int32_t*)a, y = *(const int32_t*)b;
    return (x > y) - (x < y);
}

int64_t oracle_pattern(int kind, int32_t num_nodes, int32_t num_elems, int32_t stride,
                       const int32_t* conn, const uint8_t* types, int32_t* row_ptr,
                       int32_t* col_idx, int64_t col_capacity) {
    /* The reference inserts every (row dof, col dof) pair of every element into a
     * std::set per row and copies the sets out in order (Q4A:605-645; the Hex20
     * variant builds node sets and expands each node to 3 dofs, H20:364-392).
     * Every element couples all dofs of all its nodes, so the dof rows of node n
     * hold exactly {c*dpn+d : c in adj(n)}; this builds the sorted unique node
     * adjacency and expands it, which yields the same arrays. */
    const int dpn = kind_dpn(kind);
    int64_t* deg = (int64_t*)calloc((size_t)num_nodes + 1, sizeof(int64_t));
    if (!deg) return -3;
    for (int32_t e = 0; e < num_elems; e++) {
        int npe = elem_nodes(kind, types, e);
        for (int a = 0; a < npe; a++) {
            int32_t n = conn[(int64_t)e * stride + a];
            if (n < 0 || n >= num_nodes) { free(deg); return -1; }
            deg[n] += npe;
        }
    }
    int64_t* off = (int64_t*)malloc(((size_t)num_nodes + 1) * sizeof(int64_t));
    off[0] = 0;
    for (int32_t n = 0; n < num_nodes; n++) off[n + 1] = off[n] + deg[n];
    int32_t* adj = (int32_t*)malloc((size_t)(off[num_nodes] > 0 ? off[num_nodes] : 1) * sizeof(int32_t));
    int64_t* fill = deg; /* reuse as fill counters */
    memset(fill, 0, ((size_t)num_nodes + 1) * sizeof(int64_t));
    for (int32_t e = 0; e < num_elems; e++) {
        int npe = elem_nodes(kind, types, e);
        const int32_t* c = conn + (int64_t)e * stride;
        for (int a = 0; a < npe; a++)
            for (int b = 0; b < npe; b++) adj[off[c[a]] + fill[c[a]]++] = c[b];
    }
    int64_t* ucnt = fill;
    for (int32_t n = 0; n < num_nodes; n++) {
        int64_t s = off[n], cnt = off[n + 1] - off[n];
        qsort(adj + s, (size_t)cnt, sizeof(int32_t), cmp_i32);
        int64_t u = 0;
        for (int64_t k = 0; k < cnt; k++)
            if (u == 0 || adj[s + k] != adj[s + u - 1]) adj[s + u++] = adj[s + k];
        ucnt[n] = u;
    }
    int64_t nnz = 0;
    for (int32_t n = 0; n < num_nodes; n++) nnz += ucnt[n] * dpn * dpn;
    int status = 0;
    if (col_idx && nnz > col_capacity) status = -2;
    int64_t pos = 0;
    for (int32_t n = 0; n < num_nodes; n++) {
        for (int d = 0; d < dpn; d++) {
            row_ptr[(int64_t)n * dpn + d] = (int32_t)pos;
            for (int64_t k = 0; k < ucnt[n]; k++)
                for (int d2 = 0; d2 < dpn; d2++) {
                    if (col_idx && status == 0) col_idx[pos] = adj[off[n] + k] * dpn + d2;
                    pos++;
                }
        }
    }
    row_ptr[(int64_t)num_nodes * dpn] = (int32_t)pos;
    free(adj); free(off); free(deg);
    return status ? status : nnz;
}

static int64_t find_col(const int32_t* col_idx, int32_t lo, int32_t hi, int32_t target) {
    /* Q4A:346-365: binary search of target in col_idx[lo..hi]. */
    while (lo <= hi) {
        int32_t mid = lo + (hi - lo) / 2;
        if (col_idx[mid] == target) return mid;
        if (col_idx[mid] < target) lo = mid + 1; else hi = mid - 1;
    }
    return -1;
}

int64_t oracle_assemble(int kind, int32_t num_nodes, int32_t num_elems, int32_t stride,
                        const int32_t* conn, const uint8_t* types, const double* x,
                        const double* y, const double* z, const double* E, const double* nu,
                        double E0, double nu0, double thickness, const int32_t* row_ptr,
                        const int32_t* col_idx, double* values) {
    /* Q4A:329-380: zero the values, then for each element in order compute Ke
     * and add every entry at its binary-searched position. */
    (void)num_nodes;
    const int dpn = kind_dpn(kind);
    int64_t nnz = row_ptr[(int64_t)num_nodes * dpn];
    for (int64_t i = 0; i < nnz; i++) values[i] = 0.0;
    int64_t clamped = 0;
    double* ke = (double*)malloc(3600 * sizeof(double));
    for (int32_t e = 0; e < num_elems; e++) {
        const int32_t* c = conn + (int64_t)e * stride;
        int npe = elem_nodes(kind, types, e);
        double Ee = E ? E[e] : E0, nue = nu ? nu[e] : nu0;
        double xe[20], ye[20], ze[20];
        for (int a = 0; a < npe; a++) {
            xe[a] = x[c[a]];
            ye[a] = y[c[a]];
            ze[a] = z ? z[c[a]] : 0.0;
        }
        if (npe == 4) clamped += oracle_ke_q4(xe, ye, Ee, nue, thickness, ke);
        else if (npe == 3) clamped += oracle_ke_t3(xe, ye, Ee, nue, thickness, ke);
        else clamped += oracle_ke_hex20(xe, ye, ze, Ee, nue, ke);
        int nd = npe * dpn;
        int32_t dofs[60];
        for (int a = 0; a < npe; a++)
            for (int d = 0; d < dpn; d++) dofs[a * dpn + d] = c[a] * dpn + d;
        for (int i = 0; i < nd; i++) {
            int32_t r = dofs[i];
            int32_t lo = row_ptr[r], hi = row_ptr[r + 1] - 1;
            for (int j = 0; j < nd; j++) {
                int64_t pos = find_col(col_idx, lo, hi, dofs[j]);
                if (pos < 0) { free(ke); return -1; }
                values[pos] += ke[i * nd + j];
            }
        }
    }
    free(ke);
    return clamped;
}

int64_t oracle_assemble_rows(int kind, int32_t num_nodes, int32_t num_elems, int32_t stride,
                             const int32_t* conn, const uint8_t* types, const double* x,
                             const double* y, const double* z, const double* E, const double* nu,
                             double E0, double nu0, double thickness, const int32_t* row_ptr,
                             const int32_t* col_idx, const uint8_t* row_node_mask, double* values) {
    /* oracle_assemble restricted to the dof rows of the nodes marked in
     * row_node_mask: the same serial element loop and the same per-entry
     * addition order (Q4A:329-380), skipping elements that touch no marked node
     * and rows of unmarked nodes. Only the marked rows of values are written. */
    const int dpn = kind_dpn(kind);
    for (int32_t n = 0; n < num_nodes; n++) {
        if (!row_node_mask[n]) continue;
        for (int d = 0; d < dpn; d++) {
            int32_t r = n * dpn + d;
            for (int32_t k = row_ptr[r]; k < row_ptr[r + 1]; k++) values[k] = 0.0;
        }
    }
    int64_t clamped = 0;
    double* ke = (double*)malloc(3600 * sizeof(double));
    for (int32_t e = 0; e < num_elems; e++) {
        const int32_t* c = conn + (int64_t)e * stride;
        int npe = elem_nodes(kind, types, e);
        int any = 0;
        for (int a = 0; a < npe; a++) any |= row_node_mask[c[a]];
        if (!any) continue;
        double Ee = E ? E[e] : E0, nue = nu ? nu[e] : nu0;
        double xe[20], ye[20], ze[20];
        for (int a = 0; a < npe; a++) {
            xe[a] = x[c[a]];
            ye[a] = y[c[a]];
            ze[a] = z ? z[c[a]] : 0.0;
        }
        if (npe == 4) clamped += oracle_ke_q4(xe, ye, Ee, nue, thickness, ke);
        else if (npe == 3) clamped += oracle_ke_t3(xe, ye, Ee, nue, thickness, ke);
        else clamped += oracle_ke_hex20(xe, ye, ze, Ee, nue, ke);
        int nd = npe * dpn;
        int32_t dofs[60];
        for (int a = 0; a < npe; a++)
            for (int d = 0; d < dpn; d++) dofs[a * dpn + d] = c[a] * dpn + d;
        for (int i = 0; i < nd; i++) {
            if (!row_node_mask[c[i / dpn]]) continue;
            int32_t r = dofs[i];
            int32_t lo = row_ptr[r], hi = row_ptr[r + 1] - 1;
            for (int j = 0; j < nd; j++) {
                int64_t pos = find_col(col_idx, lo, hi, dofs[j]);
                if (pos < 0) { free(ke); return -1; }
                values[pos] += ke[i * nd + j];
            }
        }
    }
    free(ke);
    return clamped;
}

void oracle_precision(int64_t nnz, const double* ref, const double* test, double out[6]) {
    /* Q4A:896-960 (+ the |diff| > 1e-10 count of Q4A:1128-1168). */
    double fro_ref = 0.0, max_abs = 0.0, max_rel = 0.0, mean_abs = 0.0, mean_rel = 0.0, fro = 0.0;
    double bad = 0.0;
    for (int64_t i = 0; i < nnz; i++) fro_ref += ref[i] * ref[i];
    fro_ref = sqrt(fro_ref);
    for (int64_t i = 0; i < nnz; i++) {
        double d = fabs(test[i] - ref[i]);
        if (d > 1e-10) bad += 1.0;
        if (ref[i] != 0.0) {
            double rel = d / fabs(ref[i]);
            if (d > max_abs) max_abs = d;
            if (rel > max_rel) max_rel = rel;
            mean_abs += d;
            mean_rel += rel;
            fro += (test[i] - ref[i]) * (test[i] - ref[i]);
        }
    }
    out[0] = max_abs;
    out[1] = max_rel;
    out[2] = nnz ? mean_abs / (double)nnz : 0.0;
    out[3] = nnz ? mean_rel / (double)nnz : 0.0;
    out[4] = fro_ref > 0.0 ? sqrt(fro) / fro_ref : 0.0;
    out[5] = bad;
}
