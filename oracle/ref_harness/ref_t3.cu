/*
 * Harness over ALLS_T3_Unstructed_Elements_Assemble_Performance.cu (TEST
 * INFRASTRUCTURE). Built by oracle/Makefile from the reference source.
 *
 * Exposes: its host CSR pattern builder (T3:458-482) and, on a GPU, its device
 * element stiffness (T3:136-206) evaluated per element by a harness kernel, so
 * the oracle's T3 restatement is pinned to the reference's own arithmetic.
 */
#include "ref_common.h"

#define main alls_reference_t3_main
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

REF_API int64_t ref_t3_build_csr(int num_nodes, int num_elems, int stride, const int32_t* conn,
                                 const uint8_t* types, int32_t* row_ptr, int32_t* col_ind,
                                 int64_t capacity) {
    std::vector<Element> els = make_elements(num_elems, stride, conn, types, nullptr, nullptr);
    std::vector<int> rp, ci;
    buildCSRStructure(num_nodes, els, rp, ci);
    return ref_copy_csr(rp, ci, row_ptr, col_ind, capacity);
}

static __global__ void harness_t3_ke(int n, const Element* els, double* out) {
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    double ke[MAX_ELEM_DOF * MAX_ELEM_DOF];
    computeElementStiffness(els[e], ke);
    for (int i = 0; i < MAX_ELEM_DOF * MAX_ELEM_DOF; i++) out[(size_t)e * 64 + i] = ke[i];
}

/* Reference device Ke (8x8 buffer per element, T3 in its top-left 6x6) with
 * the reference's __constant__ material replaced by (E, nu, t). GPU only.
 * Returns 0 on success, else the CUDA error code. */
REF_API int ref_t3_gpu_element_ke(int num_elems, int stride, const int32_t* conn,
                                  const uint8_t* types, const double* x, const double* y, double E,
                                  double nu, double t, double* ke_out) {
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
        harness_t3_ke<<<(num_elems + 127) / 128, 128>>>(num_elems, d_els, d_out);
        err = cudaGetLastError();
    }
    if (!err) err = cudaMemcpy(ke_out, d_out, (size_t)num_elems * 64 * sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(d_els);
    cudaFree(d_out);
    return (int)err;
}

/* Times the reference's own GPU A-LLS assembly of this mesh on the current
 * device, as its driver runComparison does (T3:586-640): the list heads, pool
 * index and counter are reset outside the timed window, then
 * assembleGlobalStiffnessKernelALLS and convertALLStoCSRKernel (T3:227-315)
 * run between two CUDA events, `warmup` untimed and `iters` timed iterations.
 * The CSR pattern (row_ptr, col_ind: host, nnz entries) is the input the
 * driver builds on the host beforehand. The reference's material is global
 * (E, nu, t). Its pool holds one list node per element contribution, so racing
 * duplicate inserts cannot run past it (the driver allocates 2 nnz nodes).
 * ms_out: mean milliseconds of a timed iteration; values_out (nnz, may be
 * NULL): the last iteration's CSR values. Returns 0 or the CUDA error code. */
REF_API int ref_t3_gpu_alls_time(int num_nodes, int num_elems, int stride, const int32_t* conn,
                                 const uint8_t* types, const double* x, const double* y, double E, double nu,
                                 double t, const int32_t* row_ptr, const int32_t* col_ind, int64_t nnz,
                                 int warmup, int iters, double* values_out, float* ms_out) {
    std::vector<Element> els = make_elements(num_elems, stride, conn, types, x, y);
    const int total_dofs = num_nodes * DOF_PER_NODE;
    size_t contributions = 0;
    for (const Element& el : els) contributions += (size_t)(el.num_nodes * DOF_PER_NODE) * (el.num_nodes * DOF_PER_NODE);
    cudaError_t err = cudaMemcpyToSymbol(d_YOUNG_MODULUS, &E, sizeof(double));
    if (!err) err = cudaMemcpyToSymbol(d_POISSON_RATIO, &nu, sizeof(double));
    if (!err) err = cudaMemcpyToSymbol(d_THICKNESS, &t, sizeof(double));
    Element* d_elements = nullptr;
    int *d_row_ptr = nullptr, *d_col_ind = nullptr, *d_idx = nullptr, *d_counter = nullptr;
    double* d_vals = nullptr;
    ALLSNode** d_heads = nullptr;
    ALLSNode* d_pool = nullptr;
    cudaEvent_t start = nullptr, stop = nullptr;
    if (!err) err = cudaMalloc(&d_elements, els.size() * sizeof(Element));
    if (!err) err = cudaMalloc(&d_row_ptr, (total_dofs + 1) * sizeof(int));
    if (!err) err = cudaMalloc(&d_col_ind, nnz * sizeof(int));
    if (!err) err = cudaMalloc(&d_vals, nnz * sizeof(double));
    if (!err) err = cudaMalloc(&d_heads, total_dofs * sizeof(ALLSNode*));
    if (!err) err = cudaMalloc(&d_pool, (contributions + 1) * sizeof(ALLSNode));
    if (!err) err = cudaMalloc(&d_idx, sizeof(int));
    if (!err) err = cudaMalloc(&d_counter, sizeof(int));
    if (!err) err = cudaMemcpy(d_elements, els.data(), els.size() * sizeof(Element), cudaMemcpyHostToDevice);
    if (!err) err = cudaMemcpy(d_row_ptr, row_ptr, (total_dofs + 1) * sizeof(int), cudaMemcpyHostToDevice);
    if (!err) err = cudaMemcpy(d_col_ind, col_ind, nnz * sizeof(int), cudaMemcpyHostToDevice);
    if (!err) err = cudaMemcpyToSymbol(::d_alls_pool, &d_pool, sizeof(ALLSNode*));
    if (!err) err = cudaMemcpyToSymbol(::d_alls_pool_index, &d_idx, sizeof(int*));
    if (!err) err = cudaEventCreate(&start);
    if (!err) err = cudaEventCreate(&stop);
    const int grid_dim = (num_elems + BLOCK_SIZE - 1) / BLOCK_SIZE;
    const int grid_conv = (total_dofs + BLOCK_SIZE - 1) / BLOCK_SIZE;
    float total = 0.0f;
    for (int i = 0; i < warmup + iters && !err; i++) {
        err = cudaMemset(d_heads, 0, total_dofs * sizeof(ALLSNode*));
        /* the pool too: the reference links a node (atomicExch on the head)
         * before it stores the node's next pointer, with no fence, so a reader
         * on another SM can see a node whose next is still the previous
         * iteration's; cleared, such a read sees nullptr and ends the walk */
        if (!err) err = cudaMemset(d_pool, 0, (contributions + 1) * sizeof(ALLSNode));
        if (!err) err = cudaMemset(d_idx, 0, sizeof(int));
        if (!err) err = cudaMemset(d_counter, 0, sizeof(int));
        if (!err) err = cudaEventRecord(start);
        if (!err) {
            assembleGlobalStiffnessKernelALLS<<<grid_dim, BLOCK_SIZE>>>(num_elems, d_elements, d_heads, d_counter);
            convertALLStoCSRKernel<<<grid_conv, BLOCK_SIZE>>>(total_dofs, d_heads, d_vals, d_row_ptr, d_col_ind);
            err = cudaGetLastError();
        }
        if (!err) err = cudaEventRecord(stop);
        if (!err) err = cudaEventSynchronize(stop);
        float ms = 0.0f;
        if (!err) err = cudaEventElapsedTime(&ms, start, stop);
        if (i >= warmup) total += ms;
    }
    if (!err && values_out) err = cudaMemcpy(values_out, d_vals, nnz * sizeof(double), cudaMemcpyDeviceToHost);
    if (ms_out) *ms_out = iters > 0 ? total / iters : 0.0f;
    if (start) cudaEventDestroy(start);
    if (stop) cudaEventDestroy(stop);
    cudaFree(d_elements);
    cudaFree(d_row_ptr);
    cudaFree(d_col_ind);
    cudaFree(d_vals);
    cudaFree(d_heads);
    cudaFree(d_pool);
    cudaFree(d_idx);
    cudaFree(d_counter);
    return (int)err;
}
