/*
 * fem_alls.h - C ABI of the B200 FEM global-stiffness assembler (A-LLS method).
 *
 * A mesh (node coordinates, connectivity, element type Q4 / T3 / Hex20 / mixed
 * Q4+T3, per-element E and nu) goes in; a CSR matrix (row_ptr, col_idx sorted
 * within each row, FP64 values) comes out. Element stiffness, the atomic
 * row-list scatter and the list-to-CSR consolidation run as sm_100a CUDA
 * kernels; there is no CPU fallback.
 *
 * The reference has no library API. Its de facto assembly call is a host
 * sequence inside each benchmark driver; each entry point below names the step
 * it replaces (file:line in zhou1533/A-LLS-Matrix-Parallel-Assembly):
 *
 *   buildCSRStructure           ALLS_Quad2D_Assembly_Accuracy_Analysis.cu:605-645
 *   (host pattern)              ALLS_T3_Unstructed_Elements_Assemble_Performance.cu:458-482
 *                               ALLS_Q4_T3_Mixed_Elements_Assembly_Performance.cu:488-512
 *                               ALLS_Hex20_3D_Assembly_Performance.cu:364-392
 *   pool setup + resets         ALLS_Quad2D_Assembly_Accuracy_Analysis.cu:776-813
 *   assembleGlobalStiffness-    ALLS_Quad2D_Assembly_Accuracy_Analysis.cu:394-468
 *     KernelALLS(...)           ALLS_T3_Unstructed_Elements_Assemble_Performance.cu:227-290
 *                               ALLS_Q4_T3_Mixed_Elements_Assembly_Performance.cu:248-312
 *   ...ALLSFixedArray (Hex20)   ALLS_Hex20_3D_Assembly_Performance.cu:208-257
 *   convertALLStoCSRKernel      ALLS_Quad2D_Assembly_Accuracy_Analysis.cu:471-501
 *   ...FixedArray (Hex20)       ALLS_Hex20_3D_Assembly_Performance.cu:259-278
 *   CHECK_CUDA_ERROR -> exit(1) ALLS_Quad2D_Assembly_Accuracy_Analysis.cu:15-23
 *
 * Differences a caller of the reference must know:
 *  - the CSR pattern is built on the device (the reference builds it on the host
 *    with std::set); it is identical to the reference's pattern;
 *  - errors are returned as fem_status codes instead of exit(1);
 *  - everything is stream-ordered and re-entrant: no __device__ globals on the
 *    assembly path (the reference reaches its pool through __device__ pointers,
 *    Q4A:384-391); the one exception is fem_assemble_static, whose workspace is
 *    a static device array by design;
 *  - memory the library needs beyond inputs and outputs is a caller-provided
 *    workspace (size from fem_alls_workspace_size).
 *
 * All pointers in fem_mesh / fem_csr are DEVICE pointers unless a function says
 * otherwise. cudaStream_t is passed as void* so this header needs no CUDA header.
 */
#ifndef FEM_ALLS_H
#define FEM_ALLS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FEM_ALLS_ABI_VERSION 2

#if defined(__GNUC__)
#define FEM_API __attribute__((visibility("default")))
#else
#define FEM_API
#endif

/* ---- status codes ------------------------------------------------------- */
typedef int32_t fem_status;
#define FEM_OK 0
#define FEM_ERR_BAD_ARG 1        /* null pointer, bad size, unknown kind */
#define FEM_ERR_BAD_MESH 2       /* node id < 0 or >= num_nodes in conn */
#define FEM_ERR_POOL_OVERFLOW 3  /* list pool exhausted; retry with a larger pool_factor */
#define FEM_ERR_DETJ 4           /* non-positive Jacobian determinant at a Gauss point
                                    (the matrix is still assembled) */
#define FEM_ERR_CUDA 5           /* a CUDA call failed (fem_last_cuda_error gives the code) */
#define FEM_ERR_CAPACITY 6       /* col_idx/values capacity < nnz; info.nnz has the size */
#define FEM_ERR_WORKSPACE 7      /* workspace too small or misaligned */
#define FEM_ERR_TIMEOUT 8        /* a bounded wait inside a kernel gave up */
#define FEM_ERR_RANGE 9          /* nnz or a pool index exceeds the int32/uint32 range */
#define FEM_ERR_INTERNAL 10      /* a list failed a consistency check (entries != count) */

/* ---- element kinds -------------------------------------------------------- */
#define FEM_Q4 0        /* 4-node quadrilateral, plane stress, 2x2 Gauss, 2 dof/node */
#define FEM_T3 1        /* 3-node triangle (CST), plane stress, 1 point, 2 dof/node */
#define FEM_HEX20 2     /* 20-node serendipity hexahedron, 3x3x3 Gauss, 3 dof/node */
#define FEM_MIXED_2D 3  /* Q4 and T3 in one mesh; conn_stride 4, elem_type per element */

/* ---- precision of the element stiffness --------------------------------- */
#define FEM_PREC_FP64 0      /* plain FP64 element stiffness (the oracle path) */
#define FEM_PREC_TC_F16X3 1  /* Hex20 only: the node-pair contraction of Ke on the FP16 tensor
                                cores with split operands (A = A_hi + A_lo, three products,
                                FP32 accumulation); Jacobians, detJ, inverses and the global
                                accumulation stay FP64. Value error stated by the tests. */
#define FEM_PREC_FP64_SIMT 2 /* fem_element_stiffness only, Hex20: the contraction as plain FP64
                                dot products on the CUDA cores (the reference's arithmetic, no
                                tensor cores), for comparing the tensor-core forms against */
#define FEM_PREC_FP32 3      /* Q4, T3 and mixed meshes: each Ke block computed in FP32 from
                                node coordinates taken relative to the element's first node
                                (differenced in FP64); the global accumulation stays FP64.
                                Value error stated by the tests. */

typedef struct fem_mesh {
    int32_t kind;          /* FEM_Q4, FEM_T3, FEM_HEX20, FEM_MIXED_2D */
    int32_t num_nodes;
    int32_t num_elems;
    int32_t conn_stride;   /* ints per connectivity row: Q4 4, T3 3, HEX20 20, MIXED_2D 4 */
    const double* x;       /* [num_nodes] node coordinates (structure of arrays) */
    const double* y;       /* [num_nodes] */
    const double* z;       /* [num_nodes], HEX20 only (else NULL) */
    const int32_t* conn;   /* [num_elems * conn_stride] node ids, reference node order */
    const uint8_t* elem_type; /* MIXED_2D: [num_elems] FEM_Q4 or FEM_T3; else NULL */
    const double* E;       /* [num_elems] Young's modulus, or NULL for E0 everywhere */
    const double* nu;      /* [num_elems] Poisson ratio, or NULL for nu0 everywhere */
    double E0;
    double nu0;
    double thickness;      /* plane-stress thickness (2-D kinds) */
} fem_mesh;

typedef struct fem_opts {
    int32_t precision;     /* FEM_PREC_FP64 */
    int32_t first_slots;   /* list slots in each node's first chunk; 0 = default */
    int32_t chunk_slots;   /* list slots per overflow chunk; 0 = default */
    int32_t ctas_per_sm;   /* resident CTAs per SM of the scatter kernel's persistent grid
                              (capped at what fits); 0 = all that fit */
    double pool_factor;    /* overflow chunks per node in the pool; 0 = default */
    int32_t wait_limit_us; /* bound on a kernel's wait for its own tensor-core products
                              (FEM_PREC_TC_F16X3): 0 = the default, 200 ms; > 0 = that many
                              microseconds; < 0 = no wait at all, the wait counts as run out
                              (exercises the recovery). A wait that runs out raises FEM_ERR_TIMEOUT; the
                              kernel then waits for the products with the default bound,
                              releases its tensor memory and returns (FEM_ERR_INTERNAL too if
                              that second wait also runs out). */
    int32_t reserved;      /* 0 */
} fem_opts;

typedef struct fem_csr {
    int32_t n_rows;        /* num_nodes * dof per node */
    int32_t pad;
    int64_t nnz;           /* set by the library */
    int64_t capacity;      /* entries available in col_idx / values */
    int32_t* row_ptr;      /* [n_rows + 1] */
    int32_t* col_idx;      /* [capacity] */
    double* values;        /* [capacity] */
} fem_csr;

/* Device-side result word of the last assembly in a workspace. */
typedef struct fem_info {
    int64_t nnz;              /* CSR nonzeros */
    int64_t list_entries;     /* list slots filled by the scatter (nnz/dof^2 + duplicates) */
    int32_t status_bits;      /* OR of (1 << FEM_ERR_*) raised on the device */
    int32_t overflow_chunks;  /* overflow chunks taken from the pool */
    int32_t pool_chunks;      /* overflow chunk capacity of the pool */
    int32_t max_row_entries;  /* longest row list (node granularity, duplicates included) */
} fem_info;

/* ---- workspace ------------------------------------------------------------ */

/* Bytes of device workspace an assembly of this mesh needs (256-byte aligned).
 * Depends on num_nodes, num_elems, kind and opts only. */
FEM_API fem_status fem_alls_workspace_size(const fem_mesh* mesh, const fem_opts* opts, size_t* bytes);

/* ---- the A-LLS path -------------------------------------------------------- */

/* Resets the workspace lists and runs the fused element-stiffness + list
 * scatter kernel(s). Replaces the reference's pool resets and
 * assembleGlobalStiffnessKernelALLS / ...FixedArray launches. Asynchronous. */
FEM_API fem_status fem_alls_scatter(const fem_mesh* mesh, const fem_opts* opts, void* workspace,
                            size_t workspace_bytes, void* stream);

/* Consolidates the lists into CSR: per row sort + duplicate merge, device scan
 * for row_ptr, coalesced writes of col_idx/values. Replaces the host
 * buildCSRStructure and convertALLStoCSRKernel. row_ptr is always written; if
 * capacity < nnz nothing else is written and the device info gets
 * FEM_ERR_CAPACITY (the lists stay intact, so it can be re-run with larger
 * buffers). capacity 0 with NULL col_idx/values just counts. Asynchronous. */
FEM_API fem_status fem_alls_consolidate(const fem_mesh* mesh, const fem_opts* opts, void* workspace,
                                size_t workspace_bytes, int32_t* row_ptr, int32_t* col_idx,
                                double* values, int64_t capacity, void* stream);

/* The upper triangle of the symmetric stiffness matrix in CSR (every entry
 * with column >= row, the diagonal included): the storage a symmetric or
 * Cholesky solver reads, about half the entries of the full form (no
 * counterpart in the reference, whose output is the full CSR). Same arguments
 * as fem_alls_consolidate; row_ptr [n_rows + 1], col_idx / values of the
 * upper entries, columns sorted within each row; the info word's nnz is the
 * upper-triangle count. The entries are those of the full form's upper part,
 * bit for bit. Asynchronous. */
FEM_API fem_status fem_alls_consolidate_upper(const fem_mesh* mesh, const fem_opts* opts, void* workspace,
                                              size_t workspace_bytes, int32_t* row_ptr, int32_t* col_idx,
                                              double* values, int64_t capacity, void* stream);

/* The node-block (BSR) form of fem_alls_consolidate, for solvers that work on
 * dof_per_node^2 blocks (no counterpart in the reference, whose output is
 * scalar CSR only): one block row per node, block_row_ptr [num_nodes + 1],
 * block_col_idx [nnz / dpn^2] (column nodes, sorted within each block row),
 * block_values [nnz] (each block dpn x dpn row-major: entry (i, j) of block
 * (n, m) is K[n*dpn + i][m*dpn + j]). It holds exactly the entries of the CSR
 * form; the info word's nnz stays in scalar entries. If capacity_blocks is
 * below the block count nothing but block_row_ptr is written and the info gets
 * FEM_ERR_CAPACITY. Asynchronous. */
FEM_API fem_status fem_alls_consolidate_bsr(const fem_mesh* mesh, const fem_opts* opts, void* workspace,
                                            size_t workspace_bytes, int32_t* block_row_ptr, int32_t* block_col_idx,
                                            double* block_values, int64_t capacity_blocks, void* stream);

/* Copies the device info word of the last assembly to the host (synchronizes
 * the stream) and returns the most severe status it holds. */
FEM_API fem_status fem_alls_read_info(const void* workspace, fem_info* info, void* stream);

/* scatter + consolidate + read_info. out->nnz is set. */
FEM_API fem_status fem_assemble(const fem_mesh* mesh, const fem_opts* opts, void* workspace,
                        size_t workspace_bytes, fem_csr* out, void* stream);

/* scatter + consolidate without the host synchronization (graph capturable);
 * read the outcome later with fem_alls_read_info. */
FEM_API fem_status fem_assemble_async(const fem_mesh* mesh, const fem_opts* opts, void* workspace,
                              size_t workspace_bytes, fem_csr* out, void* stream);

/* ---- element stiffness on its own -------------------------------------------
 * Replaces the reference's device element functions computeElementStiffness
 * (ALLS_Quad2D_Assembly_Accuracy_Analysis.cu:178-212,
 * ALLS_T3_Unstructed_Elements_Assemble_Performance.cu:136-206,
 * ALLS_Q4_T3_Mixed_Elements_Assembly_Performance.cu:145-227) and
 * computeElementStiffnessHex20 (ALLS_Hex20_3D_Assembly_Performance.cu:130-195)
 * as a batched call over a whole mesh (the reference calls them inside its
 * assembly kernels only). Output, per element in natural order, the packed
 * symmetric form: the upper node blocks (a <= b, row-major over the pairs),
 * each dof_per_node^2 entries row-major, entry (i, j) of block (a, b) being
 * Ke[a*dpn + i][b*dpn + j] in the element's node order. Doubles per element:
 * Q4 40 (10 blocks), T3 24 (6), mixed 40 (a T3's last 4 blocks are zero),
 * Hex20 1890 (210 blocks). */

/* Doubles per element of fem_element_stiffness's output for this mesh. */
FEM_API fem_status fem_element_stiffness_size(const fem_mesh* mesh, int64_t* doubles_per_element);

/* ke_out: device [num_elems * doubles_per_element]. status: a device int32
 * that is zeroed and then receives (1 << FEM_ERR_*) bits (BAD_MESH: the
 * element's output is zero; DETJ). Asynchronous. opts->precision:
 * FEM_PREC_FP64; for a Hex20 mesh also FEM_PREC_TC_F16X3 or FEM_PREC_FP64_SIMT;
 * for a 2-D mesh also FEM_PREC_FP32. */
FEM_API fem_status fem_element_stiffness(const fem_mesh* mesh, const fem_opts* opts, double* ke_out,
                                         int32_t* status, void* stream);

/* ---- load vector and boundary conditions -------------------------------------
 * The steps after the assembled matrix (no counterpart in the reference, which
 * stops at the stiffness values). */

/* f[ndof] += the body-force load vector: for every element node a, the
 * integral of N_a b over the element (T3 one point, Q4 2x2, Hex20 3x3x3 Gauss;
 * 2-D kinds per area times the thickness). body_force: DEVICE [num_elems * dim]
 * force per volume (per area in 2-D), or NULL for the uniform b0 (HOST [dim]).
 * status: a device int32, zeroed, then (1 << FEM_ERR_*) bits (BAD_MESH: the
 * element is skipped; DETJ). FP64 atomics, asynchronous. */
FEM_API fem_status fem_assemble_body_force(const fem_mesh* mesh, const double* body_force, const double* b0,
                                           double* f, int32_t* status, void* stream);

/* Dirichlet conditions by symmetric elimination, in place on a CSR matrix and
 * its right-hand side (all DEVICE arrays): for every entry K_jc of a free row j
 * and a fixed column c, f_j -= K_jc u_c and K_jc = 0; a fixed row i keeps only
 * K_ii = 1 and gets f_i = u_i. fixed [n_rows] (nonzero = prescribed), u
 * [n_rows] (prescribed values, read where fixed). f may be NULL (matrix only).
 * The pattern is unchanged and the matrix stays symmetric. Asynchronous. */
FEM_API fem_status fem_apply_dirichlet(int32_t n_rows, const int32_t* row_ptr, const int32_t* col_idx,
                                       double* values, double* f, const uint8_t* fixed, const double* u,
                                       void* stream);

/* ---- batched assembly -------------------------------------------------------
 * Many independent meshes (any element kinds, uneven sizes) in one
 * stream-ordered call; the reference assembles one mesh per program run
 * (its drivers' main, e.g. ALLS_Q4_T3_Mixed_Elements_Assembly_Performance.cu:742-854).
 * One persistent kernel assembles the whole batch from a schedule of work
 * items (list resets, 2-D scatter tiles, Hex20 claim and value tiles in
 * waves, scan tiles, row pointers, sorted-write tiles, completion), which
 * its CTAs take in order and run once the items they depend on are done.
 * The meshes are dealt (largest first, to the least loaded) to `concurrency`
 * workspace slots (0 = 4, at most 256): a slot holds one mesh's lists at a
 * time, so the meshes are assembled in rounds of `concurrency`. The call is a
 * few small copy kernels and the persistent kernel on `stream`; it can be
 * captured into a CUDA graph, and calls on different streams are independent
 * (each uses only its own workspace). FP64 (opts->precision FEM_PREC_FP64). */

/* Bytes of workspace for this batch (the slots are sized for their largest mesh). */
FEM_API fem_status fem_batched_workspace_size(const fem_mesh* meshes, int32_t n, const fem_opts* opts,
                                              int32_t concurrency, size_t* bytes);

/* Assembles meshes[0..n) into outs[0..n) (caller's device buffers, as for
 * fem_alls_consolidate: a mesh whose capacity is below its nnz gets only
 * row_ptr and FEM_ERR_CAPACITY in its info). infos: DEVICE array [n] that
 * receives each mesh's fem_info (nnz, status bits, ...). stamps: optional
 * DEVICE array [n + 1] of GPU global-timer nanoseconds: stamps[0] at the start,
 * stamps[1 + i] when mesh i is done. outs[i].n_rows is set. Asynchronous.
 * A wait inside the kernel that runs out (2 s) raises FEM_ERR_TIMEOUT in the
 * info of the mesh whose item waited. */
FEM_API fem_status fem_assemble_batched(const fem_mesh* meshes, int32_t n, const fem_opts* opts,
                                        int32_t concurrency, void* workspace, size_t workspace_bytes,
                                        fem_csr* outs, fem_info* infos, unsigned long long* stamps, void* stream);

/* ---- autotuner ------------------------------------------------------------------
 * Times candidate launch and list shapes on the caller's own mesh or batch and
 * returns the fastest (no counterpart in the reference, whose launch shape is
 * fixed at 256 threads per block and one element per thread,
 * ALLS_Quad2D_Assembly_Accuracy_Analysis.cu:815-818). Each candidate runs once
 * untimed, then `repeats` times between two CUDA events on `stream`; both calls
 * synchronize the stream and must not be captured. */

/* Bytes of workspace that every candidate of fem_autotune fits in. */
FEM_API fem_status fem_autotune_workspace_size(const fem_mesh* mesh, const fem_opts* opts, size_t* bytes);

/* One mesh: the scatter grid (opts.ctas_per_sm: all that fit, 1, 2 or 3) and,
 * for Hex20, the list shape (first_slots 94, 62 or 46 with chunk_slots 30; pool
 * factor at least 1 for the smaller first chunks). The precision of opts is
 * kept. out: as for fem_assemble, with capacity >= nnz; on return it holds the
 * assembly with the chosen options (status as fem_assemble's). *best: the
 * fastest options; *best_ms (may be NULL): their mean time per assembly.
 * Candidates that overflow the pool or do not fit the workspace are skipped
 * (FEM_ERR_POOL_OVERFLOW or FEM_ERR_WORKSPACE when none is left). */
FEM_API fem_status fem_autotune(const fem_mesh* mesh, const fem_opts* opts, void* workspace, size_t workspace_bytes,
                                fem_csr* out, int32_t repeats, fem_opts* best, float* best_ms, void* stream);

/* A batch: the concurrency of fem_assemble_batched (1, 2, 4, 8, 16 slots, at
 * most n; candidates whose workspace exceeds workspace_bytes are skipped).
 * outs / infos as for fem_assemble_batched; on return they hold the batch
 * assembled with *best_concurrency. */
FEM_API fem_status fem_autotune_batched(const fem_mesh* meshes, int32_t n, const fem_opts* opts, void* workspace,
                                        size_t workspace_bytes, fem_csr* outs, fem_info* infos, int32_t repeats,
                                        int32_t* best_concurrency, float* best_ms, void* stream);

/* ---- value-only re-assembly through a scatter map ----------------------------
 * For a mesh whose connectivity is unchanged between assemblies (new
 * coordinates, E or nu: nonlinear and time-stepping solvers). The reference
 * has no such path: every assembly repeats the list build and the host pattern
 * (ALLS_Quad2D_Assembly_Accuracy_Analysis.cu:394-501,605-645). A scatter map,
 * built once from the CSR pattern of a full assembly, holds the CSR position
 * of every element node block; re-assembly then adds each element's blocks at
 * those positions with FP64 atomics, with no list, no pattern build and no
 * sort. The map buffer also holds the element visit order and a status word. */

/* Bytes of the scatter-map buffer (device, 256-byte aligned) for this mesh:
 * 4 * num_elems * npe^2 (npe 4 for Q4 and mixed, 3 for T3, 20 for Hex20) plus
 * num_elems ints and a few KB. */
FEM_API fem_status fem_scatter_map_size(const fem_mesh* mesh, size_t* bytes);

/* Builds the map from row_ptr / col_idx as fem_assemble returned them for this
 * mesh's connectivity. A block missing from the pattern raises
 * FEM_ERR_INTERNAL, a bad node id FEM_ERR_BAD_MESH (fem_scatter_map_read_info).
 * Asynchronous. */
FEM_API fem_status fem_scatter_map_build(const fem_mesh* mesh, const int32_t* row_ptr, const int32_t* col_idx,
                                         void* map, size_t map_bytes, void* stream);

/* values[0, nnz) = the assembled FP64 values of the mesh's current
 * coordinates and materials, in the pattern the map was built for (zeroed,
 * then every element block added). opts->precision as fem_alls_scatter.
 * Values are not bitwise reproducible run to run (atomic order). Asynchronous. */
FEM_API fem_status fem_reassemble_values(const fem_mesh* mesh, const fem_opts* opts, const void* map,
                                         size_t map_bytes, const int32_t* row_ptr, double* values, int64_t nnz,
                                         void* stream);

/* Most severe status of the last map build or re-assembly (synchronizes). */
FEM_API fem_status fem_scatter_map_read_info(const void* map, void* stream);

/* ---- element-colouring baseline ----------------------------------------------
 * The comparison baseline of the A-LLS path: elements are coloured so that no
 * two elements of one colour share a node, then each colour is assembled
 * without atomics into a given CSR pattern. Replaces the reference's host
 * colorElements (ALLS_Quad2D_Assembly_Accuracy_Analysis.cu:648-747,
 * ALLS_T3_Unstructed_Elements_Assemble_Performance.cu:484-523,
 * ALLS_Q4_T3_Mixed_Elements_Assembly_Performance.cu:514-553) and its coloured
 * kernels (assembleGlobalStiffnessKernelColoredNoAtomic, Q4A:504-572;
 * assembleGlobalStiffnessKernelColored, T3:316-363, MIX:341-390), whose
 * colours all run at once and so race. */

/* Bytes of device workspace the colouring path needs for this mesh. */
FEM_API fem_status fem_colour_workspace_size(const fem_mesh* mesh, size_t* bytes);

/* Colours the elements on the device (Jones-Plassmann rounds, each element
 * taking the smallest colour none of its node-sharing neighbours has; at most
 * 64 colours, else FEM_ERR_RANGE) and groups them by colour in the workspace.
 * colour_of_element: optional device int32 [num_elems] that receives each
 * element's colour. Synchronous (one host sync per colouring round). */
FEM_API fem_status fem_colour_prepare(const fem_mesh* mesh, void* workspace, size_t workspace_bytes,
                                      int32_t* num_colours, int32_t* colour_of_element, void* stream);

/* Assembles the FP64 values of the mesh (any kind) into the CSR pattern
 * row_ptr / col_idx (as fem_assemble returns it; nnz entries) after
 * fem_colour_prepare on the same workspace: values are zeroed, then one launch
 * per colour (2-D: one lane per element block; Hex20: the Hex20 element
 * kernel, one CTA per element) adds every element block at its
 * binary-searched position with plain loads and stores. Asynchronous;
 * fem_colour_read_info reports a block missing from the pattern
 * (FEM_ERR_INTERNAL) or a non-positive detJ. */
FEM_API fem_status fem_colour_assemble(const fem_mesh* mesh, const void* workspace, size_t workspace_bytes,
                                       int32_t num_colours, const int32_t* row_ptr, const int32_t* col_idx,
                                       double* values, int64_t nnz, void* stream);

/* Number of colours and the most severe status of the colouring workspace
 * (synchronizes the stream). */
FEM_API fem_status fem_colour_read_info(const void* workspace, int32_t* num_colours, void* stream);

/* ---- host-buffer entry point ------------------------------------------------ */

typedef struct fem_context fem_context;

FEM_API fem_status fem_context_create(fem_context** ctx);
FEM_API void fem_context_destroy(fem_context* ctx);

/* Same as fem_assemble, but mesh arrays and out arrays are HOST pointers (pinned
 * memory is fastest). The context keeps grow-only device buffers between calls.
 * If out->capacity < nnz, returns FEM_ERR_CAPACITY with out->nnz set and
 * row_ptr filled. Synchronous. */
FEM_API fem_status fem_assemble_host(fem_context* ctx, const fem_mesh* host_mesh, const fem_opts* opts,
                             fem_csr* host_out, void* stream);

/* ---- assembly without allocation -------------------------------------------- */

/* Size of the static device workspace of fem_assemble_static (32 MiB): enough
 * for a Q4 or T3 mesh of up to about 55,000 nodes (230x230 cells) or a Hex20
 * mesh of 9x9x9 elements, with the default options. */
#define FEM_STATIC_WORKSPACE_BYTES (32u << 20)

/* No counterpart in the reference (its drivers cudaMalloc all device memory).
 * For callers that cannot call cudaMalloc: a plug-in inside an application
 * that owns the GPU's memory through its own pool allocator, or a loop that
 * must not stall on cudaMalloc / cudaFree (they can synchronize the device).
 * Same as fem_assemble, but the workspace is a static device array of
 * FEM_STATIC_WORKSPACE_BYTES inside the library, which every GPU that loads
 * the library holds until the process exits; mesh and out are still the
 * caller's device buffers. A mesh whose fem_alls_workspace_size exceeds the
 * array is refused with FEM_ERR_WORKSPACE before any launch. The first call on
 * a device (with that device current) looks up the array's device address;
 * make that first call before any stream capture. All calls on a device share
 * the array: each call clears what must start at zero, but calls whose work
 * overlaps on the GPU (different streams or host threads) race on it.
 * Synchronous, like fem_assemble. */
FEM_API fem_status fem_assemble_static(const fem_mesh* mesh, const fem_opts* opts, fem_csr* out, void* stream);

/* ---- misc ------------------------------------------------------------------- */
FEM_API const char* fem_status_string(fem_status s);
FEM_API int32_t fem_last_cuda_error(void);   /* cudaError_t of the last FEM_ERR_CUDA (per thread) */
FEM_API int32_t fem_abi_version(void);

#ifdef __cplusplus
}
#endif
#endif /* FEM_ALLS_H */
