/*
 * Harness over ALLS_Hex20_3D_Assembly_Performance.cu (TEST INFRASTRUCTURE).
 * Built by oracle/Makefile from the reference source.
 *
 * Exposes: the reference lattice mesh generator (H20:324-362), its host CSR
 * pattern builder (H20:364-392), its host colouring (H20:394-418) and, on a
 * GPU, its FP32 device element stiffness (H20:95-195) evaluated per element by
 * a harness kernel, and its two GPU assembly methods timed by its own
 * compareAssemblyMethods (H20:421-543).
 */
#include <chrono>
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

/* One mesh through the reference's own benchmark sequence (main, H20:560-625):
 * host pattern (buildCSRStructureHex20), host colouring (colorElementsHex20),
 * elements grouped by colour, device buffers, then compareAssemblyMethods
 * (H20:421-543), which times the fixed-array A-LLS kernel + its conversion
 * kernel and the coloured kernel, 3 warm-up and 10 measured iterations each,
 * with CUDA events and the resets outside the window. The reference's
 * material is a __constant__ (E, nu here, as FP32). GPU only.
 * out[0] A-LLS ms (mean), out[1] coloured ms (mean), out[2] host pattern ms,
 * out[3] host colouring ms, out[4] colours, out[5] nnz, out[6] A-LLS atomic
 * counter, out[7] A-LLS row-array bytes. values_alls / values_colored
 * (optional, nnz floats each): the CSR values of each method's last
 * iteration, in the CSR order of the host pattern (rows sorted). Returns 0 or
 * the CUDA error code (the reference's own checks exit the process). */
REF_API int ref_h20_gpu_compare(int num_nodes, int num_elems, const int32_t* conn, const double* x,
                                const double* y, const double* z, double E, double nu, double* out,
                                float* values_alls, float* values_colored, int64_t capacity) {
    std::vector<Element> elements = make_elements(num_elems, conn, x, y, z);
    const int total_dofs = num_nodes * DOF_PER_NODE;
    std::vector<int> csr_row_ptr, csr_col_ind;
    auto t0 = std::chrono::high_resolution_clock::now();
    buildCSRStructureHex20(num_nodes, elements, csr_row_ptr, csr_col_ind);
    auto t1 = std::chrono::high_resolution_clock::now();
    const int nnz = csr_row_ptr[total_dofs];
    std::vector<std::vector<int>> color_groups;
    auto t2 = std::chrono::high_resolution_clock::now();
    const int num_colors = colorElementsHex20(elements, color_groups);
    auto t3 = std::chrono::high_resolution_clock::now();
    std::vector<int> sorted_indices, h_color_offsets(num_colors), h_color_sizes(num_colors);
    int offset = 0;
    for (int c = 0; c < num_colors; c++) {
        h_color_offsets[c] = offset;
        h_color_sizes[c] = (int)color_groups[c].size();
        sorted_indices.insert(sorted_indices.end(), color_groups[c].begin(), color_groups[c].end());
        offset += h_color_sizes[c];
    }
    std::vector<Element> sorted_elements(elements.size());
    for (size_t i = 0; i < elements.size(); i++) sorted_elements[i] = elements[sorted_indices[i]];

    float Ef = (float)E, nuf = (float)nu;
    cudaError_t err = cudaMemcpyToSymbol(d_YOUNG_MODULUS, &Ef, sizeof(float));
    if (!err) err = cudaMemcpyToSymbol(d_POISSON_RATIO, &nuf, sizeof(float));
    Element* d_elements = nullptr;
    int *d_csr_row_ptr = nullptr, *d_csr_col_ind = nullptr, *d_color_offsets = nullptr, *d_color_sizes = nullptr;
    float *d_csr_values_alls = nullptr, *d_csr_values_colored = nullptr;
    if (!err) err = cudaMalloc(&d_elements, sorted_elements.size() * sizeof(Element));
    if (!err) err = cudaMalloc(&d_csr_row_ptr, (total_dofs + 1) * sizeof(int));
    if (!err) err = cudaMalloc(&d_csr_col_ind, (size_t)nnz * sizeof(int));
    if (!err) err = cudaMalloc(&d_csr_values_alls, (size_t)nnz * sizeof(float));
    if (!err) err = cudaMalloc(&d_csr_values_colored, (size_t)nnz * sizeof(float));
    if (!err) err = cudaMalloc(&d_color_offsets, num_colors * sizeof(int));
    if (!err) err = cudaMalloc(&d_color_sizes, num_colors * sizeof(int));
    if (!err) err = cudaMemcpy(d_elements, sorted_elements.data(), sorted_elements.size() * sizeof(Element),
                               cudaMemcpyHostToDevice);
    if (!err) err = cudaMemcpy(d_csr_row_ptr, csr_row_ptr.data(), (total_dofs + 1) * sizeof(int), cudaMemcpyHostToDevice);
    if (!err) err = cudaMemcpy(d_csr_col_ind, csr_col_ind.data(), (size_t)nnz * sizeof(int), cudaMemcpyHostToDevice);
    if (!err) err = cudaMemcpy(d_color_offsets, h_color_offsets.data(), num_colors * sizeof(int), cudaMemcpyHostToDevice);
    if (!err) err = cudaMemcpy(d_color_sizes, h_color_sizes.data(), num_colors * sizeof(int), cudaMemcpyHostToDevice);
    if (!err) {
        PerformanceMetrics res = compareAssemblyMethods(num_elems, total_dofs, nnz, d_elements, d_csr_row_ptr,
                                                        d_csr_col_ind, d_csr_values_alls, d_csr_values_colored,
                                                        d_color_offsets, d_color_sizes, num_colors, h_color_sizes);
        out[0] = res.alls_time_ms;
        out[1] = res.colored_time_ms;
        out[6] = res.atomic_ops_alls;
        out[7] = (double)res.alls_mem_usage;
    }
    out[2] = std::chrono::duration<double, std::milli>(t1 - t0).count();
    out[3] = std::chrono::duration<double, std::milli>(t3 - t2).count();
    out[4] = num_colors;
    out[5] = nnz;
    if (!err && values_alls && nnz <= capacity)
        err = cudaMemcpy(values_alls, d_csr_values_alls, (size_t)nnz * sizeof(float), cudaMemcpyDeviceToHost);
    if (!err && values_colored && nnz <= capacity)
        err = cudaMemcpy(values_colored, d_csr_values_colored, (size_t)nnz * sizeof(float), cudaMemcpyDeviceToHost);
    cudaFree(d_elements);
    cudaFree(d_csr_row_ptr);
    cudaFree(d_csr_col_ind);
    cudaFree(d_csr_values_alls);
    cudaFree(d_csr_values_colored);
    cudaFree(d_color_offsets);
    cudaFree(d_color_sizes);
    return (int)err;
}
