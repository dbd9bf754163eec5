/*
 * Harness over ALLS_Hex20_3D_Assembly_Performance.cu (TEST INFRASTRUCTURE).
 * Built by oracle/Makefile from the reference source.
 *
 * Exposes: the reference lattice mesh generator (H20:324-362), its host CSR
 * pattern builder (H20:364-392) and, on a GPU, its FP32 device element
 * stiffness (H20:95-195) evaluated per element by a harness kernel.
 */
#include "ref_common.h"

#define main alls_reference_h20_main
#include REF_SOURCE
#undef main

static std::vector<Element> make_elements(int num_elems, const int32_t* conn, const double* x,
                                          const double* y, const double* z) {
    std::vector<Element> els(num_elems);
    for (int e = 0; e < num_elems; e++) {
        for (int k = 0; k < NODES_PER_ELEMENT; k++) {
            int n = conn[e * NODES_PER_ELEMENT + k];
            els[e].nodes[k] = n;
            els[e].x[k] = x ? (float)x[n] : 0.0f;
            els[e].y[k] = y ? (float)y[n] : 0.0f;
            els[e].z[k] = z ? (float)z[n] : 0.0f;
        }
        els[e].color = -1;
    }
    return els;
}

/* Reference lattice mesh sizes: nodes (2nx+1)(2ny+1)(2nz+1), elements nx*ny*nz. */
REF_API void ref_h20_generate_mesh(int nx, int ny, int nz, int32_t* conn, double* x, double* y,
                                   double* z) {
    std::vector<Node> nodes;
    std::vector<Element> els;
    generateMeshHex20(nx, ny, nz, 1.0f, 1.0f, 1.0f, nodes, els);
    for (size_t n = 0; n < nodes.size(); n++) { x[n] = nodes[n].x; y[n] = nodes[n].y; z[n] = nodes[n].z; }
    for (size_t e = 0; e < els.size(); e++)
        for (int k = 0; k < 20; k++) conn[e * 20 + k] = els[e].nodes[k];
}

REF_API int64_t ref_h20_build_csr(int num_nodes, int num_elems, const int32_t* conn,
                                  int32_t* row_ptr, int32_t* col_ind, int64_t capacity) {
    std::vector<Element> els = make_elements(num_elems, conn, nullptr, nullptr, nullptr);
    std::vector<int> rp, ci;
    buildCSRStructureHex20(num_nodes, els, rp, ci);
    return ref_copy_csr(rp, ci, row_ptr, col_ind, capacity);
}

static __global__ void harness_h20_ke(int n, const Element* els, float* out) {
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    float ke[ELEM_DOF * ELEM_DOF];
    computeElementStiffnessHex20(els[e], ke);
    for (int i = 0; i < ELEM_DOF * ELEM_DOF; i++) out[(size_t)e * 3600 + i] = ke[i];
}

/* Reference FP32 device Ke (60x60 per element) with (E, nu) in place of the
 * reference's __constant__ material. GPU only; returns the CUDA error code. */
REF_API int ref_h20_gpu_element_ke(int num_elems, const int32_t* conn, const double* x,
                                   const double* y, const double* z, double E, double nu,
                                   float* ke_out) {
    std::vector<Element> els = make_elements(num_elems, conn, x, y, z);
    float Ef = (float)E, nuf = (float)nu;
    cudaError_t err = cudaMemcpyToSymbol(d_YOUNG_MODULUS, &Ef, sizeof(float));
    if (!err) err = cudaMemcpyToSymbol(d_POISSON_RATIO, &nuf, sizeof(float));
    Element* d_els = nullptr;
    float* d_out = nullptr;
    if (!err) err = cudaMalloc(&d_els, els.size() * sizeof(Element));
    if (!err) err = cudaMalloc(&d_out, (size_t)num_elems * 3600 * sizeof(float));
    if (!err) err = cudaMemcpy(d_els, els.data(), els.size() * sizeof(Element), cudaMemcpyHostToDevice);
    if (!err) {
        harness_h20_ke<<<(num_elems + 31) / 32, 32>>>(num_elems, d_els, d_out);
        err = cudaGetLastError();
    }
    if (!err) err = cudaMemcpy(ke_out, d_out, (size_t)num_elems * 3600 * sizeof(float), cudaMemcpyDeviceToHost);
    cudaFree(d_els);
    cudaFree(d_out);
    return (int)err;
}
