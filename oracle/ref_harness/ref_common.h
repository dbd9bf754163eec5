/*
 * Shared helpers of the reference harness translation units (TEST INFRASTRUCTURE).
 *
 * Each harness TU includes one reference program from its own source file, with
 * its main() renamed, and exposes the reference's host functions (and, on a GPU
 * box, its device element functions) through a small extern "C" interface so
 * the tests can pin the oracle against the reference's own code. The reference
 * sources are compiled as they are; nothing here changes their algorithm.
 */
#pragma once
#include <cstdint>
#include <cstring>
#include <vector>

#define REF_API extern "C" __attribute__((visibility("default")))

/* Copies a CSR pattern into caller buffers when they are large enough.
 * Returns nnz either way, so a caller can size its buffers with a first call. */
static inline int64_t ref_copy_csr(const std::vector<int>& row_ptr, const std::vector<int>& col_ind,
                                   int32_t* row_ptr_out, int32_t* col_ind_out, int64_t capacity) {
    int64_t nnz = (int64_t)col_ind.size();
    if (row_ptr_out) std::memcpy(row_ptr_out, row_ptr.data(), row_ptr.size() * sizeof(int));
    if (col_ind_out && nnz <= capacity) std::memcpy(col_ind_out, col_ind.data(), nnz * sizeof(int));
    return nnz;
}
