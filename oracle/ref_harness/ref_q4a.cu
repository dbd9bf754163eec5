/*
 * Harness over ALLS_Quad2D_Assembly_Accuracy_Analysis.cu (TEST INFRASTRUCTURE).
 * Built by oracle/Makefile from the reference source into oracle/_ref/.
 *
 * Exposes: the reference mesh generator (Q4A:575-603), its host CSR pattern
 * builder (Q4A:605-645) and its serial FP64 host assembly (Q4A:329-380).
 */
#include "ref_common.h"

#define main alls_reference_q4a_main
#include REF_SOURCE
#undef main

static std::vector<Element> make_elements(int num_elems, const int32_t* conn, const double* x,
                                          const double* y) {
    std::vector<Element> els(num_elems);
    for (int e = 0; e < num_elems; e++) {
        for (int k = 0; k < NODES_PER_ELEMENT; k++) {
            int n = conn[e * NODES_PER_ELEMENT + k];
            els[e].nodes[k] = n;
            els[e].x[k] = x ? x[n] : 0.0;
            els[e].y[k] = y ? y[n] : 0.0;
        }
        els[e].color = -1;
    }
    return els;
}

/* Reference material constants (Q4A:44-46), for the oracle to reproduce them. */
REF_API void ref_q4a_material(double* E, double* nu, double* t) {
    *E = h_YOUNG_MODULUS;
    *nu = h_POISSON_RATIO;
    *t = h_THICKNESS;
}

/* Reference structured mesh: conn [nx*ny*4], x/y [(nx+1)*(ny+1)]. */
REF_API void ref_q4a_generate_mesh(int nx, int ny, double lx, double ly, int32_t* conn, double* x,
                                   double* y) {
    std::vector<Node> nodes;
    std::vector<Element> els;
    generateMesh(nx, ny, lx, ly, nodes, els);
    for (size_t n = 0; n < nodes.size(); n++) { x[n] = nodes[n].x; y[n] = nodes[n].y; }
    for (size_t e = 0; e < els.size(); e++)
        for (int k = 0; k < 4; k++) conn[e * 4 + k] = els[e].nodes[k];
}

REF_API int64_t ref_q4a_build_csr(int num_nodes, int num_elems, const int32_t* conn,
                                  int32_t* row_ptr, int32_t* col_ind, int64_t capacity) {
    std::vector<Element> els = make_elements(num_elems, conn, nullptr, nullptr);
    std::vector<int> rp, ci;
    buildCSRStructure(num_nodes, num_elems, els, rp, ci);
    return ref_copy_csr(rp, ci, row_ptr, col_ind, capacity);
}

/* Serial FP64 host assembly with the reference's constants into a given pattern. */
REF_API void ref_q4a_host_assemble(int num_nodes, int num_elems, const int32_t* conn,
                                   const double* x, const double* y, const int32_t* row_ptr,
                                   const int32_t* col_ind, double* values) {
    std::vector<Element> els = make_elements(num_elems, conn, x, y);
    int nrows = num_nodes * DOF_PER_NODE;
    std::vector<int> rp(row_ptr, row_ptr + nrows + 1);
    std::vector<int> ci(col_ind, col_ind + rp[nrows]);
    std::vector<double> vals(rp[nrows]);
    assembleGlobalStiffnessHost(num_elems, els, rp, ci, vals);
    std::memcpy(values, vals.data(), vals.size() * sizeof(double));
}
