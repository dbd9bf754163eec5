/*
 * Harness over ALLS_Q4_T3_Mixed_Elements_Assembly_Performance.cu (TEST
 * INFRASTRUCTURE). Built by oracle/Makefile from the reference source.
 *
 * Exposes: its host CSR pattern builder (MIX:488-512) and, on a GPU, its device
 * element stiffness for Q4 and T3 elements (MIX:124-227), evaluated per element
 * by a harness kernel.
 */
#include "ref_common.h"

#define main alls_reference_mix_main
#include REF_SOURCE
#undef main

static std::vector<Element> make_elements(int num_elems, int stride, const int32_t* conn,
                                          const uint8_t* types, const double* x, const double* y) {
    std::vector<Element> els(num_elems);
    for (int e = 0; e < num_elems; e++) {
        Element& el = els[e];
        int npe = types ? (types[e] == 0 ? 4 : 3) : (stride == 4 ? 4 : 3);
        el.type = npe == 4 ? ELEM_Q4 : ELEM_T3;
        el.num_nodes = npe;
        el.color = -1;
        for (int k = 0; k < MAX_NODES_PER_ELEMENT; k++) {
            int n = k < npe ? conn[e * stride + k] : -1;
            el.nodes[k] = n;
            el.x[k] = (n >= 0 && x) ? x[n] : 0.0;
            el.y[k] = (n >= 0 && y) ? y[n] : 0.0;
        }
    }
    return els;
}

REF_API int64_t ref_mix_build_csr(int num_nodes, int num_elems, int stride, const int32_t* conn,
                                  const uint8_t* types, int32_t* row_ptr, int32_t* col_ind,
                                  int64_t capacity) {
    std::vector<Element> els = make_elements(num_elems, stride, conn, types, nullptr, nullptr);
    std::vector<int> rp, ci;
    buildCSRStructure(num_nodes, els, rp, ci);
    return ref_copy_csr(rp, ci, row_ptr, col_ind, capacity);
}

static __global__ void harness_mix_ke(int n, const Element* els, double* out) {
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    double ke[MAX_ELEM_DOF * MAX_ELEM_DOF];
    computeElementStiffness(els[e], ke);
    for (int i = 0; i < MAX_ELEM_DOF * MAX_ELEM_DOF; i++) out[(size_t)e * 64 + i] = ke[i];
}

/* Reference device Ke (8x8 buffer per element) with (E, nu, t) in place of the
 * reference's __constant__ material. GPU only; returns the CUDA error code. */
REF_API int ref_mix_gpu_element_ke(int num_elems, int stride, const int32_t* conn,
                                   const uint8_t* types, const double* x, const double* y,
                                   double E, double nu, double t, double* ke_out) {
    std::vector<Element> els = make_elements(num_elems, stride, conn, types, x, y);
    cudaError_t err = cudaMemcpyToSymbol(d_YOUNG_MODULUS, &E, sizeof(double));
    if (!err) err = cudaMemcpyToSymbol(d_POISSON_RATIO, &nu, sizeof(double));
    if (!err) err = cudaMemcpyToSymbol(d_THICKNESS, &t, sizeof(double));
    Element* d_els = nullptr;
    double* d_out = nullptr;
    if (!err) err = cudaMalloc(&d_els, els.size() * sizeof(Element));
    if (!err) err = cudaMalloc(&d_out, (size_t)num_elems * 64 * sizeof(double));
    if (!err) err = cudaMemcpy(d_els, els.data(), els.size() * sizeof(Element), cudaMemcpyHostToDevice);
    if (!err) {
        harness_mix_ke<<<(num_elems + 127) / 128, 128>>>(num_elems, d_els, d_out);
        err = cudaGetLastError();
    }
    if (!err) err = cudaMemcpy(ke_out, d_out, (size_t)num_elems * 64 * sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(d_els);
    cudaFree(d_out);
    return (int)err;
}
