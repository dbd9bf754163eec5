/*
 * CPU oracle for the FEM global-stiffness assembly path.
 *
 * TEST INFRASTRUCTURE ONLY. This is a plain-C restatement of the reference's
 * serial algorithm (element stiffness, host CSR pattern, serial host assembly,
 * precision analysis). It is the checker for the CUDA library: only tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline / reference legs may load
 * it, and never as the thing measured or shipped.
 *
 * Pinning: the pattern builder and the Q4 serial assembly are checked
 * bit-for-bit against the reference's own host code (built from the reference
 * sources by oracle/Makefile into oracle/_ref/), through the golden fixtures in
 * tests/golden/. The T3, mixed and Hex20 element stiffness are checked against
 * the reference's own device functions (run on a B200 through the harness).
 */
#ifndef ALLS_ORACLE_H
#define ALLS_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Element kinds, identical to the C ABI's (include/fem_alls.h). */
#define ORACLE_Q4 0
#define ORACLE_T3 1
#define ORACLE_HEX20 2
#define ORACLE_MIXED_2D 3

/* Q4 plane stress, 2x2 Gauss (restates ALLS_Quad2D_Assembly_Accuracy_Analysis.cu:225-326).
 * ke is 8x8 row-major. Returns 1 if |detJ| was clamped at a Gauss point. */
int oracle_ke_q4(const double x[4], const double y[4], double E, double nu, double t,
                 double ke[64]);

/* T3 constant-strain triangle, 1-point (restates
 * ALLS_T3_Unstructed_Elements_Assemble_Performance.cu:131-134,177-205). ke is 6x6. */
int oracle_ke_t3(const double x[3], const double y[3], double E, double nu, double t,
                 double ke[36]);

/* Hex20 serendipity, 3x3x3 Gauss, evaluated in double (restates
 * ALLS_Hex20_3D_Assembly_Performance.cu:95-195). ke is 60x60 row-major. */
int oracle_ke_hex20(const double x[20], const double y[20], const double z[20], double E,
                    double nu, double ke[3600]);

/* Sorted-unique CSR pattern (restates buildCSRStructure,
 * ALLS_Quad2D_Assembly_Accuracy_Analysis.cu:605-645, and buildCSRStructureHex20,
 * ALLS_Hex20_3D_Assembly_Performance.cu:364-392).
 * conn is [num_elems*stride]; types is NULL unless kind == ORACLE_MIXED_2D.
 * row_ptr must hold num_nodes*dpn+1 entries. col_idx may be NULL (count only) or
 * hold col_capacity entries. Returns nnz, or -1 on a bad node id, or -2 if the
 * capacity is too small. */
int64_t oracle_pattern(int kind, int32_t num_nodes, int32_t num_elems, int32_t stride,
                       const int32_t* conn, const uint8_t* types, int32_t* row_ptr,
                       int32_t* col_idx, int64_t col_capacity);

/* Serial FP64 assembly into a given pattern (restates assembleGlobalStiffnessHost,
 * ALLS_Quad2D_Assembly_Accuracy_Analysis.cu:329-380, for every element kind).
 * E/nu may be NULL (then E0/nu0). z is NULL in 2-D. Returns the number of Gauss
 * points whose |detJ| was clamped (0 for a valid mesh), or -1 if an entry was not
 * found in the pattern. */
int64_t oracle_assemble(int kind, int32_t num_nodes, int32_t num_elems, int32_t stride,
                        const int32_t* conn, const uint8_t* types, const double* x,
                        const double* y, const double* z, const double* E, const double* nu,
                        double E0, double nu0, double thickness, const int32_t* row_ptr,
                        const int32_t* col_idx, double* values);

/* oracle_assemble restricted to the dof rows of the nodes with a nonzero
 * row_node_mask[node] (num_nodes bytes): same element loop and addition order;
 * only those rows of values are written. For checking large meshes on a
 * sample of rows. */
int64_t oracle_assemble_rows(int kind, int32_t num_nodes, int32_t num_elems, int32_t stride,
                             const int32_t* conn, const uint8_t* types, const double* x,
                             const double* y, const double* z, const double* E, const double* nu,
                             double E0, double nu0, double thickness, const int32_t* row_ptr,
                             const int32_t* col_idx, const uint8_t* row_node_mask, double* values);

/* Error statistics of `test` against `ref` (restates analyzePrecision,
 * ALLS_Quad2D_Assembly_Accuracy_Analysis.cu:896-960): out[0] max abs, out[1] max
 * rel, out[2] mean abs, out[3] mean rel, out[4] Frobenius-relative error (entries
 * with ref==0 skipped, means divided by nnz as in the reference), out[5] count of
 * |diff| > 1e-10 (the reference's pass threshold, Q4A:1157). */
void oracle_precision(int64_t nnz, const double* ref, const double* test, double out[6]);

#ifdef __cplusplus
}
#endif
#endif
