// C ABI of the assembler (include/fem_alls.h): workspace layout, argument
// checks, stream-ordered orchestration of the kernels, status decoding and the
// host-buffer entry point.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <new>
#include <numeric>

#include "launch.h"

using namespace fem;

namespace fem {
int sm_count() {
    static DeviceCache cache;
    int n = 0;
    per_device(cache, [](int& v) {
        int dev = 0;
        cudaError_t err = cudaGetDevice(&dev);
        if (!err) err = cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
        return err;
    }, n);
    return n > 0 ? n : 1;
}
}  // namespace fem

namespace {

thread_local int32_t g_last_cuda_error = 0;

fem_status cuda_fail(cudaError_t err) {
    g_last_cuda_error = (int32_t)err;
    return FEM_ERR_CUDA;
}

constexpr size_t kAlign = 256;
size_t align_up(size_t v) { return (v + kAlign - 1) / kAlign * kAlign; }

int kind_dpn(int kind) { return kind == FEM_HEX20 ? 3 : 2; }

fem_status check_mesh(const fem_mesh* m, bool device_pointers_needed = true) {
    (void)device_pointers_needed;
    if (!m) return FEM_ERR_BAD_ARG;
    if (m->kind < FEM_Q4 || m->kind > FEM_MIXED_2D) return FEM_ERR_BAD_ARG;
    if (m->num_nodes <= 0 || m->num_elems < 0) return FEM_ERR_BAD_ARG;
    const int need_stride = m->kind == FEM_Q4 ? 4 : m->kind == FEM_T3 ? 3 : m->kind == FEM_HEX20 ? 20 : 4;
    if (m->conn_stride != need_stride) return FEM_ERR_BAD_ARG;
    if (!m->x || !m->y || (m->num_elems > 0 && !m->conn)) return FEM_ERR_BAD_ARG;
    if (m->kind == FEM_HEX20 && !m->z) return FEM_ERR_BAD_ARG;
    if (m->kind == FEM_MIXED_2D && m->num_elems > 0 && !m->elem_type) return FEM_ERR_BAD_ARG;
    if ((long long)m->num_nodes * kind_dpn(m->kind) + 1 > 0x7FFFFFFFll) return FEM_ERR_RANGE;
    return FEM_OK;
}

// Group records of one wave (of `wave` elements) of the Hex20 scatter for a mesh of E elements.
size_t hex20_map_bytes(int E, int wave = kHex20Wave) {
    const size_t groups = ((size_t)std::min(E, wave) + kHex20GroupSize - 1) / kHex20GroupSize;
    return groups * kHex20GroupRecWords * sizeof(unsigned);
}

fem_status make_layout(const fem_mesh* m, const fem_opts* o, HostLayout& h) {
    fem_status st = check_mesh(m);
    if (st) return st;
    fem_opts d{};
    if (!o) o = &d;
    h = HostLayout{};
    h.kind = m->kind;
    h.dpn = kind_dpn(m->kind);
    h.B = h.dpn * h.dpn;
    h.N = m->num_nodes;
    h.E = m->num_elems;
    if (h.dpn == 2) {
        // 2-D chunk rows are fixed at 16 words (the scatter reads them as 4 x 16 bytes).
        if ((o->first_slots && o->first_slots != k2DSlots) || (o->chunk_slots && o->chunk_slots != k2DSlots))
            return FEM_ERR_BAD_ARG;
        h.S1 = h.S2 = k2DSlots;
    } else {
        h.S1 = o->first_slots ? o->first_slots : 94;
        h.S2 = o->chunk_slots ? o->chunk_slots : 30;
        if (h.S1 < 2 || h.S2 < 2 || (h.S1 + 2) % 4 || (h.S2 + 2) % 4 || h.S1 > 94 || h.S2 > 94)
            return FEM_ERR_BAD_ARG;
    }
    h.H1 = h.S1 + 2;
    h.H2 = h.S2 + 2;
    const double pf = o->pool_factor > 0 ? o->pool_factor : (h.dpn == 3 ? 0.5 : 0.125);
    const double cap2 = std::ceil(pf * (double)h.N) + 64;
    if (cap2 > 2e9) return FEM_ERR_RANGE;
    h.cap2 = (int)cap2;
    const double slots = (double)h.N * h.S1 + (double)h.cap2 * h.S2;
    if (slots >= 2147483648.0) return FEM_ERR_RANGE;  // slot ids carry a flag in bit 31
    h.num_tiles = (h.N + kScanTile - 1) / kScanTile;
    size_t off = 0;
    h.off_info = off;
    off += align_up(sizeof(DevInfo));
    h.off_meta1 = off;
    h.meta1_bytes = (size_t)h.N * h.H1 * sizeof(int);
    off += align_up(h.meta1_bytes);
    h.off_meta2 = off;
    off += align_up((size_t)h.cap2 * h.H2 * sizeof(int));
    h.off_vals = off;
    off += align_up((size_t)slots * h.B * sizeof(double));
    h.off_counts = off;
    off += align_up((size_t)h.N * sizeof(int));
    h.off_ucounts = off;  // upper-triangle column counts (fem_alls_consolidate_upper)
    off += align_up((size_t)h.N * sizeof(int));
    h.off_tiles = off;
    off += align_up((size_t)h.num_tiles * sizeof(long long));
    h.off_elist = off;  // visit order of the elements (perm), ranges, bucket histogram (+ bbox)
    {
        const size_t nbuckets = h.dpn == 2 ? (size_t)2 * reorder_buckets(h.N) : (size_t)1 << (3 * morton_bits(h.E));
        off += align_up((size_t)h.E * sizeof(int)) + align_up(4 * sizeof(int)) + align_up(nbuckets * sizeof(int)) +
               align_up(6 * sizeof(unsigned long long));
    }
    // Hex20: node -> element incidence (counts, offsets, lists), the map
    // records of one wave of the two-pass scatter, and (tensor-core form) the
    // staged Ke of one wave
    h.off_inc = off;
    if (h.kind == FEM_HEX20)
        off += 2 * align_up((size_t)(h.N + 1) * sizeof(int)) + align_up((size_t)h.E * 20 * sizeof(int));
    h.off_map = off;
    if (h.kind == FEM_HEX20) off += align_up(hex20_map_bytes(h.E));
    h.off_stage = off;
    if (h.kind == FEM_HEX20 && o->precision == FEM_PREC_TC_F16X3)
        off += align_up((size_t)std::min(h.E, kHex20Wave) * kPackedHex20 * sizeof(double));
    h.total = off;
    return FEM_OK;
}

ListLayout device_layout(const HostLayout& h, void* ws) {
    unsigned char* b = static_cast<unsigned char*>(ws);
    ListLayout L;
    L.N = h.N;
    L.S1 = h.S1;
    L.S2 = h.S2;
    L.H1 = h.H1;
    L.H2 = h.H2;
    L.B = h.B;
    L.cap2 = h.cap2;
    L.meta1 = reinterpret_cast<int*>(b + h.off_meta1);
    L.meta2 = reinterpret_cast<int*>(b + h.off_meta2);
    L.vals = reinterpret_cast<double*>(b + h.off_vals);
    L.counts = reinterpret_cast<int*>(b + h.off_counts);
    L.info = reinterpret_cast<DevInfo*>(b + h.off_info);
    return L;
}

MeshView mesh_view(const fem_mesh* m) {
    MeshView v;
    v.x = m->x;
    v.y = m->y;
    v.z = m->z;
    v.conn = m->conn;
    v.types = m->elem_type;
    v.E = m->E;
    v.nu = m->nu;
    v.E0 = m->E0;
    v.nu0 = m->nu0;
    v.t = m->thickness;
    v.N = m->num_nodes;
    v.E_count = m->num_elems;
    v.stride = m->conn_stride;
    return v;
}

fem_status check_ws(const HostLayout& h, const void* ws, size_t bytes) {
    if (!ws || bytes < h.total || (reinterpret_cast<uintptr_t>(ws) % kAlign)) return FEM_ERR_WORKSPACE;
    return FEM_OK;
}

// Most severe status among the device bits.
fem_status decode_bits(int bits) {
    static const int order[] = {FEM_ERR_BAD_MESH, FEM_ERR_POOL_OVERFLOW, FEM_ERR_TIMEOUT, FEM_ERR_INTERNAL,
                                FEM_ERR_RANGE,    FEM_ERR_CAPACITY,      FEM_ERR_DETJ};
    for (int code : order)
        if (bits & (1 << code)) return code;
    return FEM_OK;
}

// Precisions of the assembly entry points: FP64 for every kind; the FP16
// tensor-core contraction for Hex20; FP32 blocks for the 2-D kinds.
bool assembly_precision_ok(int precision, int kind) {
    if (precision == FEM_PREC_FP64) return true;
    if (precision == FEM_PREC_TC_F16X3) return kind == FEM_HEX20;
    if (precision == FEM_PREC_FP32) return kind == FEM_Q4 || kind == FEM_T3 || kind == FEM_MIXED_2D;
    return false;
}

}  // namespace

extern "C" {

int32_t fem_abi_version(void) { return FEM_ALLS_ABI_VERSION; }
int32_t fem_last_cuda_error(void) { return g_last_cuda_error; }

const char* fem_status_string(fem_status s) {
    switch (s) {
        case FEM_OK: return "ok";
        case FEM_ERR_BAD_ARG: return "bad argument";
        case FEM_ERR_BAD_MESH: return "bad mesh (node id out of range)";
        case FEM_ERR_POOL_OVERFLOW: return "list pool overflow (retry with a larger pool_factor)";
        case FEM_ERR_DETJ: return "non-positive Jacobian determinant";
        case FEM_ERR_CUDA: return "CUDA error";
        case FEM_ERR_CAPACITY: return "output capacity smaller than nnz";
        case FEM_ERR_WORKSPACE: return "workspace too small or misaligned";
        case FEM_ERR_TIMEOUT: return "bounded wait gave up";
        case FEM_ERR_RANGE: return "size exceeds the int32 range";
        case FEM_ERR_INTERNAL: return "list consistency check failed";
        default: return "unknown status";
    }
}

fem_status fem_alls_workspace_size(const fem_mesh* mesh, const fem_opts* opts, size_t* bytes) {
    if (!bytes) return FEM_ERR_BAD_ARG;
    HostLayout h;
    fem_status st = make_layout(mesh, opts, h);
    if (st) return st;
    *bytes = h.total;
    return FEM_OK;
}

fem_status fem_alls_scatter(const fem_mesh* mesh, const fem_opts* opts, void* workspace, size_t workspace_bytes,
                            void* stream) {
    HostLayout h;
    fem_status st = make_layout(mesh, opts, h);
    if (st) return st;
    if ((st = check_ws(h, workspace, workspace_bytes))) return st;
    const int precision = opts ? opts->precision : FEM_PREC_FP64;
    if (!assembly_precision_ok(precision, h.kind)) return FEM_ERR_BAD_ARG;
    const int ctas = opts ? opts->ctas_per_sm : 0;
    if (ctas < 0) return FEM_ERR_BAD_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    ListLayout L = device_layout(h, workspace);
    unsigned char* b = static_cast<unsigned char*>(workspace);
    cudaError_t err = cudaMemsetAsync(b + h.off_info, 0, sizeof(DevInfo), s);
    if (!err) err = launch_info_init(L.info, h.cap2, s);
    if (!err) err = cudaMemsetAsync(b + h.off_meta1, 0, h.meta1_bytes, s);
    if (!err) err = cudaMemsetAsync(b + h.off_counts, 0, (size_t)h.N * sizeof(int), s);
    // 2-D lists accumulate every contribution with atomic adds: their first
    // chunks' slot values start at zero (overflow chunks are zeroed when taken).
    if (!err && h.dpn == 2) err = cudaMemsetAsync(b + h.off_vals, 0, (size_t)h.N * h.S1 * h.B * sizeof(double), s);
    if (err) return cuda_fail(err);
    if (h.E == 0) return FEM_OK;
    MeshView m = mesh_view(mesh);
    int* perm = reinterpret_cast<int*>(b + h.off_elist);
    int* ranges = reinterpret_cast<int*>(b + h.off_elist + align_up((size_t)h.E * sizeof(int)));
    int* hist = reinterpret_cast<int*>(b + h.off_elist + align_up((size_t)h.E * sizeof(int)) + align_up(4 * sizeof(int)));
    if (h.kind == FEM_HEX20) {
        const size_t nbuckets = (size_t)1 << (3 * morton_bits(h.E));
        unsigned long long* bbox = reinterpret_cast<unsigned long long*>(
            b + h.off_elist + align_up((size_t)h.E * sizeof(int)) + align_up(4 * sizeof(int)) +
            align_up(nbuckets * sizeof(int)));
        err = launch_reorder_3d(m, hist, ranges, perm, bbox, sm_count(), s);
        // two-pass scatter in waves of the spatial order: a wave's claims
        // (entries, zeroed value blocks, map records) complete before its
        // value pass, and the blocks it touches are still in L2 when the
        // values arrive
        int* inc_cnt = reinterpret_cast<int*>(b + h.off_inc);
        int* inc_off = inc_cnt + align_up((size_t)(h.N + 1) * sizeof(int)) / sizeof(int);
        int* inc = inc_off + align_up((size_t)(h.N + 1) * sizeof(int)) / sizeof(int);
        int* map = reinterpret_cast<int*>(b + h.off_map);
        double* stage = reinterpret_cast<double*>(b + h.off_stage);
        long long* tiles = reinterpret_cast<long long*>(b + h.off_tiles);  // free until the consolidation
        const long long wait_ns = wait_ns_of(opts ? opts->wait_limit_us : 0);
        if (!err) err = launch_incidence(m, inc_cnt, inc_off, inc, tiles, &L.info->status_bits, sm_count(), s);
        for (int i0 = 0; i0 < h.E && !err; i0 += kHex20Wave) {
            const int i1 = std::min(h.E, i0 + kHex20Wave);
            err = launch_claim_hex20(m, L, perm, inc_off, inc, i0, i1, map, s);
            if (!err) err = launch_values_hex20(m, L, precision, perm, i0, i1, map, stage, wait_ns, s);
        }
    } else {
        err = launch_reorder(m, hist, ranges, perm, sm_count(), s);
        if (!err && h.kind != FEM_T3) err = launch_scatter_2d(m, L, 4, precision, perm, ranges + 0, ctas, s);
        if (!err && h.kind != FEM_Q4) err = launch_scatter_2d(m, L, 3, precision, perm, ranges + 2, ctas, s);
    }
    return err ? cuda_fail(err) : FEM_OK;
}

fem_status fem_alls_consolidate(const fem_mesh* mesh, const fem_opts* opts, void* workspace, size_t workspace_bytes,
                                int32_t* row_ptr, int32_t* col_idx, double* values, int64_t capacity, void* stream) {
    HostLayout h;
    fem_status st = make_layout(mesh, opts, h);
    if (st) return st;
    if ((st = check_ws(h, workspace, workspace_bytes))) return st;
    if (!row_ptr || capacity < 0 || (capacity > 0 && (!col_idx || !values))) return FEM_ERR_BAD_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    ListLayout L = device_layout(h, workspace);
    long long* tiles = reinterpret_cast<long long*>(static_cast<unsigned char*>(workspace) + h.off_tiles);
    cudaError_t err = launch_consolidate(L, h.dpn, row_ptr, col_idx, values, capacity, tiles, h.num_tiles, s);
    return err ? cuda_fail(err) : FEM_OK;
}

fem_status fem_alls_consolidate_bsr(const fem_mesh* mesh, const fem_opts* opts, void* workspace,
                                    size_t workspace_bytes, int32_t* block_row_ptr, int32_t* block_col_idx,
                                    double* block_values, int64_t capacity_blocks, void* stream) {
    HostLayout h;
    fem_status st = make_layout(mesh, opts, h);
    if (st) return st;
    if ((st = check_ws(h, workspace, workspace_bytes))) return st;
    if (!block_row_ptr || capacity_blocks < 0 || (capacity_blocks > 0 && (!block_col_idx || !block_values)))
        return FEM_ERR_BAD_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    ListLayout L = device_layout(h, workspace);
    long long* tiles = reinterpret_cast<long long*>(static_cast<unsigned char*>(workspace) + h.off_tiles);
    cudaError_t err = launch_consolidate_bsr(L, h.dpn, block_row_ptr, block_col_idx, block_values, capacity_blocks,
                                             tiles, h.num_tiles, s);
    return err ? cuda_fail(err) : FEM_OK;
}

fem_status fem_alls_consolidate_upper(const fem_mesh* mesh, const fem_opts* opts, void* workspace,
                                      size_t workspace_bytes, int32_t* row_ptr, int32_t* col_idx, double* values,
                                      int64_t capacity, void* stream) {
    HostLayout h;
    fem_status st = make_layout(mesh, opts, h);
    if (st) return st;
    if ((st = check_ws(h, workspace, workspace_bytes))) return st;
    if (!row_ptr || capacity < 0 || (capacity > 0 && (!col_idx || !values))) return FEM_ERR_BAD_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    ListLayout L = device_layout(h, workspace);
    unsigned char* b = static_cast<unsigned char*>(workspace);
    long long* tiles = reinterpret_cast<long long*>(b + h.off_tiles);
    int* ucounts = reinterpret_cast<int*>(b + h.off_ucounts);
    cudaError_t err =
        launch_consolidate_upper(L, h.dpn, ucounts, row_ptr, col_idx, values, capacity, tiles, h.num_tiles, s);
    return err ? cuda_fail(err) : FEM_OK;
}

fem_status fem_alls_read_info(const void* workspace, fem_info* info, void* stream) {
    if (!workspace || !info) return FEM_ERR_BAD_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t err = cudaMemcpyAsync(info, workspace, sizeof(fem_info), cudaMemcpyDeviceToHost, s);
    if (!err) err = cudaStreamSynchronize(s);
    if (err) return cuda_fail(err);
    return decode_bits(info->status_bits);
}

fem_status fem_assemble_async(const fem_mesh* mesh, const fem_opts* opts, void* workspace, size_t workspace_bytes,
                              fem_csr* out, void* stream) {
    if (!out) return FEM_ERR_BAD_ARG;
    fem_status st = fem_alls_scatter(mesh, opts, workspace, workspace_bytes, stream);
    if (st) return st;
    return fem_alls_consolidate(mesh, opts, workspace, workspace_bytes, out->row_ptr, out->col_idx, out->values,
                                out->capacity, stream);
}

fem_status fem_assemble(const fem_mesh* mesh, const fem_opts* opts, void* workspace, size_t workspace_bytes,
                        fem_csr* out, void* stream) {
    fem_status st = fem_assemble_async(mesh, opts, workspace, workspace_bytes, out, stream);
    if (st) return st;
    fem_info info;
    st = fem_alls_read_info(workspace, &info, stream);
    out->nnz = info.nnz;
    out->n_rows = mesh->num_nodes * kind_dpn(mesh->kind);
    return st;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Element stiffness on its own
// ---------------------------------------------------------------------------

extern "C" {

fem_status fem_element_stiffness_size(const fem_mesh* mesh, int64_t* doubles_per_element) {
    fem_status st = check_mesh(mesh);
    if (st) return st;
    if (!doubles_per_element) return FEM_ERR_BAD_ARG;
    *doubles_per_element = mesh->kind == FEM_HEX20 ? kPackedHex20
                           : mesh->kind == FEM_T3  ? kPacked2D_T3
                                                   : kPacked2D_Q4;
    return FEM_OK;
}

fem_status fem_element_stiffness(const fem_mesh* mesh, const fem_opts* opts, double* ke_out, int32_t* status,
                                 void* stream) {
    fem_status st = check_mesh(mesh);
    if (st) return st;
    if (!status || (mesh->num_elems > 0 && !ke_out)) return FEM_ERR_BAD_ARG;
    const int precision = opts ? opts->precision : FEM_PREC_FP64;
    if (!assembly_precision_ok(precision, mesh->kind) &&
        !(precision == FEM_PREC_FP64_SIMT && mesh->kind == FEM_HEX20))
        return FEM_ERR_BAD_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t err = cudaMemsetAsync(status, 0, sizeof(int32_t), s);
    if (!err)
        err = launch_element_stiffness(mesh_view(mesh), mesh->kind, precision, ke_out, status,
                                       wait_ns_of(opts ? opts->wait_limit_us : 0), s);
    return err ? cuda_fail(err) : FEM_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Load vector and boundary conditions
// ---------------------------------------------------------------------------

extern "C" {

fem_status fem_assemble_body_force(const fem_mesh* mesh, const double* body_force, const double* b0, double* f,
                                   int32_t* status, void* stream) {
    fem_status st = check_mesh(mesh);
    if (st) return st;
    if (!f || !status || (!body_force && !b0)) return FEM_ERR_BAD_ARG;
    const int dim = mesh->kind == FEM_HEX20 ? 3 : 2;
    double b[3] = {0.0, 0.0, 0.0};
    if (!body_force)
        for (int d = 0; d < dim; d++) b[d] = b0[d];
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t err = cudaMemsetAsync(status, 0, sizeof(int32_t), s);
    if (!err) err = launch_body_force(mesh_view(mesh), mesh->kind, body_force, b, f, status, s);
    return err ? cuda_fail(err) : FEM_OK;
}

fem_status fem_apply_dirichlet(int32_t n_rows, const int32_t* row_ptr, const int32_t* col_idx, double* values,
                               double* f, const uint8_t* fixed, const double* u, void* stream) {
    if (n_rows < 0 || (n_rows > 0 && (!row_ptr || !col_idx || !values || !fixed || !u))) return FEM_ERR_BAD_ARG;
    cudaError_t err =
        launch_dirichlet(n_rows, row_ptr, col_idx, values, f, fixed, u, static_cast<cudaStream_t>(stream));
    return err ? cuda_fail(err) : FEM_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Batched assembly
// ---------------------------------------------------------------------------

namespace {

int batch_slots(int n, int concurrency) {
    int k = concurrency > 0 ? concurrency : 4;
    k = std::min(k, kMaxBatchConcurrency);
    return std::max(1, std::min(k, n));
}

// Workspace of a batch: the control block (mesh descriptors, schedule,
// per-mesh counters, ticket) and `slots` list workspaces, each sized for the
// largest mesh dealt to it (Hex20: plus a second wave's slot map).
struct BatchLayout {
    std::vector<int> slot_of;
    std::vector<size_t> slot_off;
    size_t off_meshes, off_counters, off_ticket, off_segs, total;
};

size_t batch_mesh_bytes(const fem_mesh& m, const fem_opts* opts, fem_status& st) {
    HostLayout h;
    st = make_layout(&m, opts, h);
    if (st) return 0;
    return h.total + (h.kind == FEM_HEX20 ? align_up(hex20_map_bytes(h.E, kBatchHex20Wave)) : 0);
}

// Work items of one mesh in the batch schedule (an upper bound of the
// segments too), used to size the schedule.
int batch_segments_bound(const fem_mesh& m) {
    const int waves = m.kind == FEM_HEX20 ? (m.num_elems + kBatchHex20Wave - 1) / kBatchHex20Wave : 0;
    return 8 + 2 * waves;
}

fem_status batch_layout(const fem_mesh* meshes, int n, const fem_opts* opts, int slots, BatchLayout& bl) {
    bl.slot_of = batch_schedule(meshes, n, slots);
    std::vector<size_t> need(slots, 0);
    long long segs = 0;
    for (int i = 0; i < n; i++) {
        fem_status st;
        const size_t b = batch_mesh_bytes(meshes[i], opts, st);
        if (st) return st;
        need[bl.slot_of[i]] = std::max(need[bl.slot_of[i]], b);
        segs += batch_segments_bound(meshes[i]);
    }
    size_t off = 0;
    bl.off_meshes = off;
    off += align_up((size_t)n * sizeof(BatchMesh));
    bl.off_counters = off;
    off += align_up((size_t)n * kBatchCounters * sizeof(int));
    bl.off_ticket = off;
    off += align_up(sizeof(int));
    bl.off_segs = off;
    off += align_up((size_t)segs * sizeof(BatchSegment));
    bl.slot_off.assign(slots, 0);
    for (int k = 0; k < slots; k++) {
        bl.slot_off[k] = off;
        off += align_up(need[k]);
    }
    bl.total = off;
    return FEM_OK;
}

// Appends a segment of `count` items of one phase of mesh j.
struct ScheduleBuilder {
    std::vector<BatchSegment> segs;
    int total = 0;
    void add(int j, int phase, int count, int arg, int done, int dep0 = -1, int target0 = 0, int dep1 = -1,
             int target1 = 0) {
        if (count <= 0) return;
        BatchSegment g{};
        g.mesh = j;
        g.phase = phase;
        g.first = total;
        g.count = count;
        g.arg = arg;
        g.dep_ctr[0] = dep0;
        g.dep_target[0] = target0;
        g.dep_ctr[1] = dep1;
        g.dep_target[1] = target1;
        g.done_ctr = done;
        segs.push_back(g);
        total += count;
    }
};

}  // namespace

extern "C" {

fem_status fem_batched_workspace_size(const fem_mesh* meshes, int32_t n, const fem_opts* opts, int32_t concurrency,
                                      size_t* bytes) {
    if (!meshes || n <= 0 || !bytes) return FEM_ERR_BAD_ARG;
    BatchLayout bl;
    fem_status st = batch_layout(meshes, n, opts, batch_slots(n, concurrency), bl);
    if (!st) *bytes = bl.total;
    return st;
}

fem_status fem_assemble_batched(const fem_mesh* meshes, int32_t n, const fem_opts* opts, int32_t concurrency,
                                void* workspace, size_t workspace_bytes, fem_csr* outs, fem_info* infos,
                                unsigned long long* stamps, void* stream) {
    if (!meshes || n <= 0 || !outs || !infos) return FEM_ERR_BAD_ARG;
    if (opts && opts->precision != FEM_PREC_FP64) return FEM_ERR_BAD_ARG;  // the batch assembles in FP64
    const int slots = batch_slots(n, concurrency);
    BatchLayout bl;
    fem_status st = batch_layout(meshes, n, opts, slots, bl);
    if (st) return st;
    if (!workspace || workspace_bytes < bl.total || reinterpret_cast<uintptr_t>(workspace) % kAlign)
        return FEM_ERR_WORKSPACE;
    for (int i = 0; i < n; i++)
        if (!outs[i].row_ptr || outs[i].capacity < 0 || (outs[i].capacity > 0 && (!outs[i].col_idx || !outs[i].values)))
            return FEM_ERR_BAD_ARG;
    unsigned char* base = static_cast<unsigned char*>(workspace);
    // descriptors
    std::vector<BatchMesh> bms(n);
    std::vector<HostLayout> hl(n);
    for (int i = 0; i < n; i++) {
        if ((st = make_layout(&meshes[i], opts, hl[i]))) return st;
        const HostLayout& h = hl[i];
        unsigned char* ws = base + bl.slot_off[bl.slot_of[i]];
        BatchMesh& bm = bms[i];
        bm = BatchMesh{};
        bm.m = mesh_view(&meshes[i]);
        bm.L = device_layout(h, ws);
        bm.tiles = reinterpret_cast<long long*>(ws + h.off_tiles);
        bm.map[0] = reinterpret_cast<int*>(ws + h.off_map);
        bm.map[1] = reinterpret_cast<int*>(ws + h.total);
        bm.row_ptr = outs[i].row_ptr;
        bm.col_idx = outs[i].col_idx;
        bm.values = outs[i].values;
        bm.capacity = outs[i].capacity;
        bm.info_out = infos + i;
        bm.stamp = stamps ? stamps + 1 + i : nullptr;
        bm.zero_ptr[0] = ws;  // info word and first chunks
        bm.zero_bytes[0] = (long long)(h.off_meta1 + h.meta1_bytes);
        bm.zero_ptr[1] = ws + h.off_vals;  // 2-D: the first chunks' values (every contribution is an atomic add)
        bm.zero_bytes[1] = h.dpn == 2 ? (long long)h.N * h.S1 * h.B * (long long)sizeof(double) : 0;
        bm.zero_ptr[2] = ws + h.off_counts;
        bm.zero_bytes[2] = (long long)h.N * (long long)sizeof(int);
        bm.kind = h.kind;
        bm.dpn = h.dpn;
        bm.num_tiles = h.num_tiles;
        outs[i].n_rows = meshes[i].num_nodes * kind_dpn(meshes[i].kind);
    }
    // rounds: the r-th mesh of every slot (slots keep their meshes smallest
    // first, which brings the meshes' completions forward)
    std::vector<std::vector<int>> per_slot(slots);
    {
        std::vector<int> order(n);
        for (int i = 0; i < n; i++) order[i] = i;
        std::stable_sort(order.begin(), order.end(),
                         [&](int a, int b) { return batch_cost(meshes[a]) < batch_cost(meshes[b]); });
        for (int i : order) per_slot[bl.slot_of[i]].push_back(i);
    }
    size_t rounds = 0;
    for (auto& v : per_slot) rounds = std::max(rounds, v.size());
    ScheduleBuilder sb;
    std::vector<int> prev_in_slot(n, -1);
    for (auto& v : per_slot)
        for (size_t r = 1; r < v.size(); r++) prev_in_slot[v[r]] = v[r - 1];
    auto ctr = [](int j, int c) { return j * kBatchCounters + c; };
    for (size_t r = 0; r < rounds; r++) {
        std::vector<int> round;
        for (auto& v : per_slot)
            if (r < v.size()) round.push_back(v[r]);
        // largest first within a round, so that the long meshes start early
        std::stable_sort(round.begin(), round.end(),
                         [&](int a, int b) { return batch_cost(meshes[a]) > batch_cost(meshes[b]); });
        std::vector<int> resets(n, 0), scatter_items(n, 0), write_items(n, 0);
        for (int j : round) {
            const BatchMesh& bm = bms[j];
            const long long zb = bm.zero_bytes[0] + bm.zero_bytes[1] + bm.zero_bytes[2];
            resets[j] = (int)((zb + kBatchResetBytes - 1) / kBatchResetBytes);
            const int p = prev_in_slot[j];
            sb.add(j, kBpReset, resets[j], 0, ctr(j, kBcReset), p >= 0 ? ctr(p, kBcFinish) : -1, 1);
        }
        for (int j : round) {
            const int E = meshes[j].num_elems;
            if (E <= 0) continue;
            if (bms[j].kind == FEM_HEX20) {
                const int nw = (E + kBatchHex20Wave - 1) / kBatchHex20Wave;
                std::vector<int> claims(nw), values(nw);
                for (int w = 0; w < nw; w++) {
                    const int ew = std::min(kBatchHex20Wave, E - w * kBatchHex20Wave);
                    claims[w] = (ew + kBatchClaim - 1) / kBatchClaim;
                    values[w] = (ew + kBatchValues - 1) / kBatchValues;
                }
                std::vector<int> claims_upto(nw), values_upto(nw);
                std::partial_sum(claims.begin(), claims.end(), claims_upto.begin());
                std::partial_sum(values.begin(), values.end(), values_upto.begin());
                // C0, C1, V0, C2, V1, ...: a wave's values follow the claims of
                // the next wave; a wave's claims reuse the slot map of the wave
                // two before, once its values are in
                auto claim = [&](int w) {
                    sb.add(j, kBpClaim, claims[w], w, ctr(j, kBcScatter), ctr(j, kBcReset), resets[j],
                           w >= 2 ? ctr(j, kBcValues) : -1, w >= 2 ? values_upto[w - 2] : 0);
                };
                auto value = [&](int w) {
                    sb.add(j, kBpValues, values[w], w, ctr(j, kBcValues), ctr(j, kBcScatter),
                           claims_upto[std::min(w + 1, nw - 1)]);
                };
                claim(0);
                for (int w = 0; w < nw; w++) {
                    if (w + 1 < nw) claim(w + 1);
                    value(w);
                }
                scatter_items[j] = values_upto[nw - 1];
            } else {
                scatter_items[j] = (E + kBatchScatter2D - 1) / kBatchScatter2D;
                sb.add(j, kBpScatter2D, scatter_items[j], 0, ctr(j, kBcScatter), ctr(j, kBcReset), resets[j]);
            }
        }
        for (int j : round) {
            const int sc = bms[j].kind == FEM_HEX20 ? kBcValues : kBcScatter;
            if (meshes[j].num_elems > 0)
                sb.add(j, kBpScanReduce, bms[j].num_tiles, 0, ctr(j, kBcScanReduce), ctr(j, sc), scatter_items[j]);
            else
                sb.add(j, kBpScanReduce, bms[j].num_tiles, 0, ctr(j, kBcScanReduce), ctr(j, kBcReset), resets[j]);
        }
        for (int j : round)
            sb.add(j, kBpScanTop, 1, 0, ctr(j, kBcScanTop), ctr(j, kBcScanReduce), bms[j].num_tiles);
        for (int j : round) sb.add(j, kBpRowPtr, bms[j].num_tiles, 0, ctr(j, kBcRowPtr), ctr(j, kBcScanTop), 1);
        for (int j : round) {
            const int npb = bms[j].dpn == 3 ? kBlockThreads / 32 : kBlockThreads / 8;
            const long long per = (long long)npb * kBatchWriteBatches;
            write_items[j] = outs[j].capacity > 0 ? (int)((meshes[j].num_nodes + per - 1) / per) : 0;
            sb.add(j, kBpWrite, write_items[j], 0, ctr(j, kBcWrite), ctr(j, kBcRowPtr), bms[j].num_tiles);
        }
        for (int j : round)
            sb.add(j, kBpFinish, 1, 0, ctr(j, kBcFinish), ctr(j, kBcWrite), write_items[j],
                   ctr(j, kBcRowPtr), bms[j].num_tiles);
    }
    long long seg_bound = 0;
    for (int i = 0; i < n; i++) seg_bound += batch_segments_bound(meshes[i]);
    if ((long long)sb.segs.size() > seg_bound) return FEM_ERR_INTERNAL;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const cudaError_t err = launch_batch(
        bms.data(), n, sb.segs.data(), (int)sb.segs.size(), sb.total, reinterpret_cast<BatchMesh*>(base + bl.off_meshes),
        reinterpret_cast<BatchSegment*>(base + bl.off_segs), reinterpret_cast<int*>(base + bl.off_counters),
        reinterpret_cast<int*>(base + bl.off_ticket), stamps, 2000ll * 1000 * 1000, opts ? opts->ctas_per_sm : 0, s);
    return err ? cuda_fail(err) : FEM_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Autotuner
// ---------------------------------------------------------------------------

namespace {

// Candidate options for one mesh: the scatter grid (all resident CTAs, or
// 1..3 per SM) and, for Hex20, the list shape (first chunk 94 / 62 / 46
// slots, overflow chunks of 30; a pool of one overflow chunk per node for the
// smaller first chunks, whose corner-node rows spill).
std::vector<fem_opts> tune_candidates(const fem_mesh* m, const fem_opts* base) {
    fem_opts b{};
    if (base) b = *base;
    std::vector<fem_opts> out;
    const int ctas[] = {0, 1, 2, 3};
    if (m->kind == FEM_HEX20) {
        const int first[] = {94, 62, 46};
        for (int f : first)
            for (int c : ctas) {
                fem_opts o = b;
                o.first_slots = f;
                o.chunk_slots = 30;
                if (f < 94) o.pool_factor = std::max(o.pool_factor, 1.0);
                o.ctas_per_sm = c;
                out.push_back(o);
            }
    } else {
        for (int c : ctas) {
            fem_opts o = b;
            o.first_slots = o.chunk_slots = 0;
            o.ctas_per_sm = c;
            out.push_back(o);
        }
    }
    return out;
}

// Mean milliseconds of `repeats` calls of fn() on stream s (CUDA events).
template <typename Fn>
fem_status time_calls(cudaStream_t s, int repeats, Fn fn, float& ms) {
    cudaEvent_t a = nullptr, b = nullptr;
    cudaError_t err = cudaEventCreate(&a);
    if (!err) err = cudaEventCreate(&b);
    fem_status st = FEM_OK;
    if (!err) err = cudaEventRecord(a, s);
    for (int r = 0; r < repeats && !err && !st; r++) st = fn();
    if (!err && !st) err = cudaEventRecord(b, s);
    if (!err && !st) err = cudaEventSynchronize(b);
    if (!err && !st) err = cudaEventElapsedTime(&ms, a, b);
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    if (err) return cuda_fail(err);
    if (!st) ms /= (float)repeats;
    return st;
}

fem_status not_capturing(cudaStream_t s) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    const cudaError_t err = cudaStreamIsCapturing(s, &cs);
    if (err) return cuda_fail(err);
    return cs == cudaStreamCaptureStatusNone ? FEM_OK : FEM_ERR_BAD_ARG;
}

}  // namespace

extern "C" {

fem_status fem_autotune_workspace_size(const fem_mesh* mesh, const fem_opts* opts, size_t* bytes) {
    fem_status st = check_mesh(mesh);
    if (st) return st;
    if (!bytes) return FEM_ERR_BAD_ARG;
    *bytes = 0;
    for (const fem_opts& o : tune_candidates(mesh, opts)) {
        size_t b = 0;
        if ((st = fem_alls_workspace_size(mesh, &o, &b))) return st;
        *bytes = std::max(*bytes, b);
    }
    return FEM_OK;
}

fem_status fem_autotune(const fem_mesh* mesh, const fem_opts* opts, void* workspace, size_t workspace_bytes,
                        fem_csr* out, int32_t repeats, fem_opts* best, float* best_ms, void* stream) {
    if (!out || !best || repeats < 1) return FEM_ERR_BAD_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    fem_status st = not_capturing(s);
    if (st) return st;
    if ((st = check_mesh(mesh))) return st;
    bool found = false, overflowed = false;
    float best_t = 0.0f;
    for (const fem_opts& o : tune_candidates(mesh, opts)) {
        size_t need = 0;
        if ((st = fem_alls_workspace_size(mesh, &o, &need))) return st;
        if (need > workspace_bytes) continue;
        // one untimed run: its status decides whether the candidate counts
        fem_csr c = *out;
        st = fem_assemble(mesh, &o, workspace, workspace_bytes, &c, stream);
        if (st == FEM_ERR_POOL_OVERFLOW) {
            overflowed = true;
            continue;
        }
        if (st && st != FEM_ERR_DETJ) return st;
        float ms = 0.0f;
        st = time_calls(s, repeats, [&] { return fem_assemble_async(mesh, &o, workspace, workspace_bytes, &c, stream); },
                        ms);
        if (st) return st;
        if (!found || ms < best_t) {
            found = true;
            best_t = ms;
            *best = o;
        }
    }
    if (!found) return overflowed ? FEM_ERR_POOL_OVERFLOW : FEM_ERR_WORKSPACE;
    if (best_ms) *best_ms = best_t;
    // leave the chosen options' assembly in out
    return fem_assemble(mesh, best, workspace, workspace_bytes, out, stream);
}

fem_status fem_autotune_batched(const fem_mesh* meshes, int32_t n, const fem_opts* opts, void* workspace,
                                size_t workspace_bytes, fem_csr* outs, fem_info* infos, int32_t repeats,
                                int32_t* best_concurrency, float* best_ms, void* stream) {
    if (!meshes || n <= 0 || !outs || !infos || !best_concurrency || repeats < 1) return FEM_ERR_BAD_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    fem_status st = not_capturing(s);
    if (st) return st;
    bool found = false;
    float best_t = 0.0f;
    for (int k = 1; k <= kMaxBatchConcurrency && k <= std::max(1, (int)n); k *= 2) {
        size_t need = 0;
        if ((st = fem_batched_workspace_size(meshes, n, opts, k, &need))) return st;
        if (need > workspace_bytes) continue;
        auto run = [&] {
            return fem_assemble_batched(meshes, n, opts, k, workspace, workspace_bytes, outs, infos, nullptr, stream);
        };
        if ((st = run())) return st;  // untimed (creates the slot streams)
        float ms = 0.0f;
        if ((st = time_calls(s, repeats, run, ms))) return st;
        if (!found || ms < best_t) {
            found = true;
            best_t = ms;
            *best_concurrency = k;
        }
    }
    if (!found) return FEM_ERR_WORKSPACE;
    if (best_ms) *best_ms = best_t;
    st = fem_assemble_batched(meshes, n, opts, *best_concurrency, workspace, workspace_bytes, outs, infos, nullptr,
                              stream);
    if (st) return st;
    const cudaError_t err = cudaStreamSynchronize(s);
    return err ? cuda_fail(err) : FEM_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Value-only re-assembly through a scatter map
// ---------------------------------------------------------------------------

namespace {

struct MapHostLayout {
    int G;  // map entries per element
    size_t off_info, off_pos, off_perm, off_ranges, off_hist, off_bbox, total;
};

MapHostLayout map_layout(const fem_mesh* m) {
    MapHostLayout h{};
    const size_t E = (size_t)m->num_elems;
    const int npe = m->kind == FEM_HEX20 ? 20 : (m->kind == FEM_T3 ? 3 : 4);
    h.G = npe * npe;
    const size_t nbuckets = m->kind == FEM_HEX20 ? (size_t)1 << (3 * morton_bits(m->num_elems))
                                                 : (size_t)2 * reorder_buckets(m->num_nodes);
    size_t off = 0;
    h.off_info = off;
    off += align_up(sizeof(DevInfo));
    h.off_pos = off;
    off += align_up(E * h.G * sizeof(int));
    h.off_perm = off;
    off += align_up(E * sizeof(int));
    h.off_ranges = off;
    off += align_up(4 * sizeof(int));
    h.off_hist = off;
    off += align_up(nbuckets * sizeof(int));
    h.off_bbox = off;
    off += align_up(6 * sizeof(unsigned long long));
    h.total = off;
    return h;
}

fem_status check_map(const fem_mesh* mesh, const void* map, size_t map_bytes, MapHostLayout& h) {
    fem_status st = check_mesh(mesh);
    if (st) return st;
    h = map_layout(mesh);
    if (!map || map_bytes < h.total || reinterpret_cast<uintptr_t>(map) % kAlign) return FEM_ERR_WORKSPACE;
    return FEM_OK;
}

}  // namespace

extern "C" {

fem_status fem_scatter_map_size(const fem_mesh* mesh, size_t* bytes) {
    fem_status st = check_mesh(mesh);
    if (st) return st;
    if (!bytes) return FEM_ERR_BAD_ARG;
    *bytes = map_layout(mesh).total;
    return FEM_OK;
}

fem_status fem_scatter_map_build(const fem_mesh* mesh, const int32_t* row_ptr, const int32_t* col_idx, void* map,
                                 size_t map_bytes, void* stream) {
    MapHostLayout h;
    fem_status st = check_map(mesh, map, map_bytes, h);
    if (st) return st;
    if (!row_ptr || (mesh->num_elems > 0 && !col_idx)) return FEM_ERR_BAD_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    unsigned char* b = static_cast<unsigned char*>(map);
    DevInfo* info = reinterpret_cast<DevInfo*>(b + h.off_info);
    const MeshView m = mesh_view(mesh);
    int* perm = reinterpret_cast<int*>(b + h.off_perm);
    int* ranges = reinterpret_cast<int*>(b + h.off_ranges);
    int* hist = reinterpret_cast<int*>(b + h.off_hist);
    cudaError_t err = cudaMemsetAsync(info, 0, sizeof(DevInfo), s);
    if (!err && mesh->num_elems > 0) {
        err = launch_build_map(m, mesh->kind, row_ptr, col_idx, reinterpret_cast<int*>(b + h.off_pos),
                               &info->status_bits, s);
        // the element visit order of the A-LLS scatter, for the locality of the adds
        if (!err && mesh->kind == FEM_HEX20)
            err = launch_reorder_3d(m, hist, ranges, perm, reinterpret_cast<unsigned long long*>(b + h.off_bbox),
                                    sm_count(), s);
        else if (!err)
            err = launch_reorder(m, hist, ranges, perm, sm_count(), s);
    }
    return err ? cuda_fail(err) : FEM_OK;
}

fem_status fem_reassemble_values(const fem_mesh* mesh, const fem_opts* opts, const void* map, size_t map_bytes,
                                 const int32_t* row_ptr, double* values, int64_t nnz, void* stream) {
    MapHostLayout h;
    fem_status st = check_map(mesh, map, map_bytes, h);
    if (st) return st;
    const int precision = opts ? opts->precision : FEM_PREC_FP64;
    if (!assembly_precision_ok(precision, mesh->kind))
        return FEM_ERR_BAD_ARG;
    if (!row_ptr || nnz < 0 || (nnz > 0 && !values)) return FEM_ERR_BAD_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    unsigned char* b = static_cast<unsigned char*>(const_cast<void*>(map));
    DevInfo* info = reinterpret_cast<DevInfo*>(b + h.off_info);
    const int* pos = reinterpret_cast<const int*>(b + h.off_pos);
    const int* perm = reinterpret_cast<const int*>(b + h.off_perm);
    const int* ranges = reinterpret_cast<const int*>(b + h.off_ranges);
    cudaError_t err = cudaMemsetAsync(&info->status_bits, 0, sizeof(int), s);
    if (!err && nnz > 0) err = cudaMemsetAsync(values, 0, (size_t)nnz * sizeof(double), s);
    if (!err && mesh->num_elems > 0) {
        const MeshView m = mesh_view(mesh);
        if (mesh->kind == FEM_HEX20)
            err = launch_reassemble_hex20(m, precision, perm, MapTarget{pos, row_ptr, values, nullptr}, info, s);
        else
            err = launch_reassemble_2d(m, precision, pos, h.G, perm, ranges, row_ptr, values, &info->status_bits, s);
    }
    return err ? cuda_fail(err) : FEM_OK;
}

fem_status fem_scatter_map_read_info(const void* map, void* stream) {
    fem_info info;
    return fem_alls_read_info(map, &info, stream);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Element-colouring baseline
// ---------------------------------------------------------------------------

namespace {

struct ColourHostLayout {
    size_t off_info, off_kinfo, off_cnt, off_off, off_inc, off_colour, off_perm, off_hist, off_ranges, off_tiles, total;
};

ColourHostLayout colour_layout(const fem_mesh* m) {
    ColourHostLayout h{};
    const size_t N = (size_t)m->num_nodes, E = (size_t)m->num_elems;
    const size_t tiles = (N + kScanTile - 1) / kScanTile;
    size_t off = 0;
    h.off_info = off;
    off += align_up(sizeof(ColourInfo));
    h.off_kinfo = off;  // status of the Hex20 element kernel in the coloured assembly
    off += align_up(sizeof(DevInfo));
    h.off_cnt = off;
    off += align_up(N * sizeof(int));
    h.off_off = off;
    off += align_up((N + 1) * sizeof(int));
    h.off_inc = off;
    off += align_up(E * (size_t)m->conn_stride * sizeof(int));
    h.off_colour = off;
    off += align_up(E * sizeof(int));
    h.off_perm = off;
    off += align_up(E * sizeof(int));
    h.off_hist = off;
    off += align_up(2 * kMaxColours * sizeof(int));
    h.off_ranges = off;
    off += align_up((2 * kMaxColours + 1) * sizeof(int));
    h.off_tiles = off;
    off += align_up(tiles * sizeof(long long));
    h.total = off;
    return h;
}

ColourLayout colour_device_layout(const ColourHostLayout& h, const void* ws) {
    unsigned char* b = static_cast<unsigned char*>(const_cast<void*>(ws));
    ColourLayout C;
    C.info = reinterpret_cast<ColourInfo*>(b + h.off_info);
    C.cnt = reinterpret_cast<int*>(b + h.off_cnt);
    C.off = reinterpret_cast<int*>(b + h.off_off);
    C.inc = reinterpret_cast<int*>(b + h.off_inc);
    C.colour = reinterpret_cast<int*>(b + h.off_colour);
    C.perm = reinterpret_cast<int*>(b + h.off_perm);
    C.hist = reinterpret_cast<int*>(b + h.off_hist);
    C.ranges = reinterpret_cast<int*>(b + h.off_ranges);
    C.tiles = reinterpret_cast<long long*>(b + h.off_tiles);
    return C;
}

}  // namespace

extern "C" {

fem_status fem_colour_workspace_size(const fem_mesh* mesh, size_t* bytes) {
    if (!bytes) return FEM_ERR_BAD_ARG;
    fem_status st = check_mesh(mesh);
    if (st) return st;
    *bytes = colour_layout(mesh).total;
    return FEM_OK;
}

fem_status fem_colour_prepare(const fem_mesh* mesh, void* workspace, size_t workspace_bytes, int32_t* num_colours,
                              int32_t* colour_of_element, void* stream) {
    fem_status st = check_mesh(mesh);
    if (st) return st;
    const ColourHostLayout h = colour_layout(mesh);
    if (!workspace || workspace_bytes < h.total || reinterpret_cast<uintptr_t>(workspace) % kAlign || !num_colours)
        return !num_colours ? FEM_ERR_BAD_ARG : FEM_ERR_WORKSPACE;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const ColourLayout C = colour_device_layout(h, workspace);
    int nc = 0, bits = 0;
    cudaError_t err = cudaMemsetAsync(static_cast<unsigned char*>(workspace) + h.off_kinfo, 0, sizeof(DevInfo), s);
    if (!err) err = launch_colour_prepare(mesh_view(mesh), C, sm_count(), s, &nc, &bits);
    if (!err && colour_of_element && mesh->num_elems > 0)
        err = launch_colour_export(C, mesh->num_elems, colour_of_element, sm_count(), s);
    if (!err && colour_of_element) err = cudaStreamSynchronize(s);
    if (err) return cuda_fail(err);
    *num_colours = nc;
    return decode_bits(bits);
}

fem_status fem_colour_assemble(const fem_mesh* mesh, const void* workspace, size_t workspace_bytes,
                               int32_t num_colours, const int32_t* row_ptr, const int32_t* col_idx, double* values,
                               int64_t nnz, void* stream) {
    fem_status st = check_mesh(mesh);
    if (st) return st;
    const ColourHostLayout h = colour_layout(mesh);
    if (!workspace || workspace_bytes < h.total || reinterpret_cast<uintptr_t>(workspace) % kAlign)
        return FEM_ERR_WORKSPACE;
    if (num_colours < 0 || num_colours > kMaxColours || nnz < 0 || !row_ptr || (nnz > 0 && (!col_idx || !values)))
        return FEM_ERR_BAD_ARG;
    if (mesh->num_elems == 0 || nnz == 0) return FEM_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const ColourLayout C = colour_device_layout(h, workspace);
    cudaError_t err = cudaSuccess;
    if (mesh->kind == FEM_HEX20) {
        // the Hex20 element kernel, one launch per colour, plain adds; its
        // status bits go to the workspace's element-kernel info word
        DevInfo* info = reinterpret_cast<DevInfo*>(static_cast<unsigned char*>(const_cast<void*>(workspace)) +
                                                   h.off_kinfo);
        err = cudaMemsetAsync(info, 0, sizeof(DevInfo), s);
        if (!err) err = cudaMemsetAsync(values, 0, (size_t)nnz * sizeof(double), s);
        for (int c = 0; c < num_colours && !err; c++)
            err = launch_colour_hex20(mesh_view(mesh), C.perm, C.ranges + 2 * c,
                                      MapTarget{nullptr, row_ptr, values, col_idx}, info, s);
    } else {
        err = launch_colour_assemble(mesh_view(mesh), C, num_colours, row_ptr, col_idx, values, nnz, sm_count(), s);
    }
    return err ? cuda_fail(err) : FEM_OK;
}

fem_status fem_colour_read_info(const void* workspace, int32_t* num_colours, void* stream) {
    if (!workspace) return FEM_ERR_BAD_ARG;
    ColourInfo h{};
    DevInfo k{};
    const unsigned char* b = static_cast<const unsigned char*>(workspace);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t err = cudaMemcpyAsync(&h, b, sizeof(h), cudaMemcpyDeviceToHost, s);
    // the element-kernel info word follows the colouring one (first region, 256-byte aligned)
    if (!err) err = cudaMemcpyAsync(&k, b + align_up(sizeof(ColourInfo)), sizeof(k), cudaMemcpyDeviceToHost, s);
    if (!err) err = cudaStreamSynchronize(s);
    if (err) return cuda_fail(err);
    if (num_colours) *num_colours = h.num_colours;
    return decode_bits(h.status_bits | k.status_bits);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Host-buffer entry point
// ---------------------------------------------------------------------------

struct fem_context {
    struct Buf {
        void* p = nullptr;
        size_t n = 0;
    };
    Buf x, y, z, conn, types, E, nu, ws, row_ptr, col_idx, values;
    double pool_factor = 0.0;
    ~fem_context() {
        for (Buf* b : {&x, &y, &z, &conn, &types, &E, &nu, &ws, &row_ptr, &col_idx, &values})
            if (b->p) cudaFree(b->p);
    }
    // Grow-only device buffer.
    cudaError_t need(Buf& b, size_t bytes) {
        if (bytes <= b.n && b.p) return cudaSuccess;
        if (b.p) cudaFree(b.p);
        b.p = nullptr;
        b.n = 0;
        cudaError_t err = cudaMalloc(&b.p, bytes ? bytes : 1);
        if (!err) b.n = bytes;
        return err;
    }
};

extern "C" {

fem_status fem_context_create(fem_context** ctx) {
    if (!ctx) return FEM_ERR_BAD_ARG;
    *ctx = new (std::nothrow) fem_context();
    return *ctx ? FEM_OK : FEM_ERR_BAD_ARG;
}

void fem_context_destroy(fem_context* ctx) { delete ctx; }

fem_status fem_assemble_host(fem_context* ctx, const fem_mesh* hm, const fem_opts* opts, fem_csr* out, void* stream) {
    if (!ctx || !out || !out->row_ptr) return FEM_ERR_BAD_ARG;
    fem_status st = check_mesh(hm);
    if (st) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int dpn = kind_dpn(hm->kind);
    const size_t N = (size_t)hm->num_nodes, E = (size_t)hm->num_elems;
    cudaError_t err = cudaSuccess;
    auto up = [&](fem_context::Buf& b, const void* src, size_t bytes) {
        if (err || !src) return;
        err = ctx->need(b, bytes);
        if (!err) err = cudaMemcpyAsync(b.p, src, bytes, cudaMemcpyHostToDevice, s);
    };
    up(ctx->x, hm->x, N * sizeof(double));
    up(ctx->y, hm->y, N * sizeof(double));
    up(ctx->z, hm->z, N * sizeof(double));
    up(ctx->conn, hm->conn, E * hm->conn_stride * sizeof(int32_t));
    up(ctx->types, hm->elem_type, E);
    up(ctx->E, hm->E, E * sizeof(double));
    up(ctx->nu, hm->nu, E * sizeof(double));
    if (err) return cuda_fail(err);
    fem_mesh dm = *hm;
    dm.x = static_cast<const double*>(ctx->x.p);
    dm.y = static_cast<const double*>(ctx->y.p);
    dm.z = hm->z ? static_cast<const double*>(ctx->z.p) : nullptr;
    dm.conn = static_cast<const int32_t*>(ctx->conn.p);
    dm.elem_type = hm->elem_type ? static_cast<const uint8_t*>(ctx->types.p) : nullptr;
    dm.E = hm->E ? static_cast<const double*>(ctx->E.p) : nullptr;
    dm.nu = hm->nu ? static_cast<const double*>(ctx->nu.p) : nullptr;

    fem_opts o = opts ? *opts : fem_opts{};
    if (ctx->pool_factor > o.pool_factor) o.pool_factor = ctx->pool_factor;
    const size_t n_rows = N * dpn;
    if ((err = ctx->need(ctx->row_ptr, (n_rows + 1) * sizeof(int32_t)))) return cuda_fail(err);
    fem_info info{};
    for (int attempt = 0; attempt < 4; attempt++) {
        size_t wsb = 0;
        if ((st = fem_alls_workspace_size(&dm, &o, &wsb))) return st;
        if ((err = ctx->need(ctx->ws, wsb))) return cuda_fail(err);
        if ((st = fem_alls_scatter(&dm, &o, ctx->ws.p, ctx->ws.n, stream))) return st;
        long long cap = (long long)(ctx->values.n / sizeof(double));
        if ((st = fem_alls_consolidate(&dm, &o, ctx->ws.p, ctx->ws.n, static_cast<int32_t*>(ctx->row_ptr.p),
                                       static_cast<int32_t*>(ctx->col_idx.p), static_cast<double*>(ctx->values.p),
                                       cap, stream)))
            return st;
        st = fem_alls_read_info(ctx->ws.p, &info, stream);
        if (st == FEM_ERR_POOL_OVERFLOW) {
            // Grow the overflow pool and assemble again.
            HostLayout h;
            make_layout(&dm, &o, h);
            o.pool_factor = 2.0 * ((double)h.cap2 / (double)h.N + 0.25);
            ctx->pool_factor = o.pool_factor;
            continue;
        }
        if (st == FEM_ERR_CAPACITY) {
            if ((err = ctx->need(ctx->col_idx, (size_t)info.nnz * sizeof(int32_t)))) return cuda_fail(err);
            if ((err = ctx->need(ctx->values, (size_t)info.nnz * sizeof(double)))) return cuda_fail(err);
            if ((st = fem_alls_consolidate(&dm, &o, ctx->ws.p, ctx->ws.n, static_cast<int32_t*>(ctx->row_ptr.p),
                                           static_cast<int32_t*>(ctx->col_idx.p), static_cast<double*>(ctx->values.p),
                                           info.nnz, stream)))
                return st;
            st = fem_alls_read_info(ctx->ws.p, &info, stream);
        }
        break;
    }
    out->n_rows = (int32_t)n_rows;
    out->nnz = info.nnz;
    if (st != FEM_OK && st != FEM_ERR_DETJ) return st;
    err = cudaMemcpyAsync(out->row_ptr, ctx->row_ptr.p, (n_rows + 1) * sizeof(int32_t), cudaMemcpyDeviceToHost, s);
    if (err) return cuda_fail(err);
    if (out->capacity < info.nnz || !out->col_idx || !out->values) {
        if ((err = cudaStreamSynchronize(s))) return cuda_fail(err);
        return FEM_ERR_CAPACITY;
    }
    err = cudaMemcpyAsync(out->col_idx, ctx->col_idx.p, (size_t)info.nnz * sizeof(int32_t), cudaMemcpyDeviceToHost, s);
    if (!err)
        err = cudaMemcpyAsync(out->values, ctx->values.p, (size_t)info.nnz * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (!err) err = cudaStreamSynchronize(s);
    if (err) return cuda_fail(err);
    return st;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Assembly without allocation: the workspace in a static device array
// ---------------------------------------------------------------------------
//
// Some callers cannot call cudaMalloc. An application or solver framework that
// owns the GPU's memory through its own pool allocator does not let a plug-in
// allocate behind its back (its accounting and memory limits would be wrong),
// and a time-stepping loop that must not stall avoids cudaMalloc and cudaFree
// because they can synchronize the whole device. fem_assemble_static serves
// them: it is fem_assemble with the workspace in g_static_workspace, a
// file-scope device array of FEM_STATIC_WORKSPACE_BYTES that every GPU which
// loads this library holds until the process exits. The caller still passes
// the mesh arrays and the CSR output buffers.
//
// Set-up: the first call on a device, with that device current, looks up the
// array's device address (cudaGetSymbolAddress) and keeps it for that device;
// make that first call before any stream capture. In host code the name
// g_static_workspace is only a host-side stand-in, never a device address.
//
// All calls on a device share the one array, which keeps the last call's
// contents. Each assembly clears what must start at zero (info word, first
// chunk rows, row counters) and writes every value before reading it, so
// consecutive calls are independent; calls whose work overlaps on the GPU
// (different streams, or different host threads) race on the array and
// corrupt each other's results.

namespace {

__device__ __align__(256) unsigned char g_static_workspace[FEM_STATIC_WORKSPACE_BYTES];

constexpr int kMaxStaticDevices = 64;
std::mutex g_static_mutex;
void* g_static_ptr[kMaxStaticDevices] = {};

fem_status static_workspace(void** ptr) {
    int dev = 0;
    cudaError_t err = cudaGetDevice(&dev);
    if (err) return cuda_fail(err);
    if (dev < 0 || dev >= kMaxStaticDevices) return FEM_ERR_BAD_ARG;
    std::lock_guard<std::mutex> lock(g_static_mutex);
    if (!g_static_ptr[dev]) {
        void* p = nullptr;
        err = cudaGetSymbolAddress(&p, g_static_workspace);
        if (err) return cuda_fail(err);
        g_static_ptr[dev] = p;
    }
    *ptr = g_static_ptr[dev];
    return FEM_OK;
}

}  // namespace

extern "C" {

fem_status fem_assemble_static(const fem_mesh* mesh, const fem_opts* opts, fem_csr* out, void* stream) {
    if (!out) return FEM_ERR_BAD_ARG;
    size_t need = 0;
    fem_status st = fem_alls_workspace_size(mesh, opts, &need);
    if (st) return st;
    if (need > (size_t)FEM_STATIC_WORKSPACE_BYTES) return FEM_ERR_WORKSPACE;  // mesh too large for the array
    void* ws = nullptr;
    if ((st = static_workspace(&ws))) return st;
    return fem_assemble(mesh, opts, ws, (size_t)FEM_STATIC_WORKSPACE_BYTES, out, stream);
}

}  // extern "C"
