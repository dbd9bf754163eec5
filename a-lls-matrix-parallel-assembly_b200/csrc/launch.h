// Host-side launchers of the assembler kernels (internal to the library).
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <vector>

#include "fem_internal.cuh"

namespace fem {

// A launch-shape value (resident CTAs per SM, SM count) cached per device: it
// is computed on the first launch on each device (compute(int& v) sets v > 0),
// which also sets the kernel's per-device attributes. Devices past the table
// compute it every time.
constexpr int kMaxCachedDevices = 64;
struct DeviceCache {
    std::atomic<int> v[kMaxCachedDevices] = {};
};
template <typename F>
cudaError_t per_device(DeviceCache& cache, F&& compute, int& out) {
    int dev = 0;
    cudaError_t err = cudaGetDevice(&dev);
    if (err) return err;
    const bool cached = dev >= 0 && dev < kMaxCachedDevices;
    int v = cached ? cache.v[dev].load(std::memory_order_acquire) : 0;
    if (v <= 0) {
        if ((err = compute(v))) return err;
        if (v < 1) v = 1;
        if (cached) cache.v[dev].store(v, std::memory_order_release);
    }
    out = v;
    return cudaSuccess;
}

struct MeshView {
    const double* x;
    const double* y;
    const double* z;
    const int* conn;
    const unsigned char* types;
    const double* E;
    const double* nu;
    double E0, nu0, t;
    int N;       // nodes
    int E_count; // elements
    int stride;  // ints per connectivity row
};

// 2-D chunk rows are 16 int32 words (14 slots + fill + next).
constexpr int k2DSlots = 14;

// perm: element visit order; range: device ints {begin, end} into perm;
// precision FEM_PREC_FP64 or FEM_PREC_FP32 (the arithmetic of the Ke blocks).
// ctas_per_sm: cap on the persistent grid's resident CTAs per SM (0 = all that fit).
cudaError_t launch_scatter_2d(const MeshView& m, const ListLayout& L, int npe, int precision, const int* perm,
                              const int* range, int ctas_per_sm, cudaStream_t s);
// Node-local element order (perm) and the element ranges {q4 begin, q4 end, t3 begin, t3 end}.
int reorder_buckets(int num_nodes);
cudaError_t launch_reorder(const MeshView& m, int* hist, int* ranges, int* perm, int sms, cudaStream_t s);
int sm_count();
// Packed symmetric element stiffness (fem_element_stiffness): doubles per element.
constexpr int kPackedHex20 = 210 * 9;  // 210 upper 3x3 node blocks
constexpr int kPacked2D_Q4 = 10 * 4;   // 10 upper 2x2 node blocks (also the mixed-mesh stride)
constexpr int kPacked2D_T3 = 6 * 4;
// Element stiffness of every element, natural order; status gets 1 << FEM_ERR_* bits.
cudaError_t launch_element_stiffness(const MeshView& m, int kind, int precision, double* ke_out, int* status,
                                     long long wait_ns, cudaStream_t s);
// Hex20 element stiffness with the contraction on the tcgen05 tensor cores
// (FEM_PREC_TC_F16X3), two elements per CTA step.
// wait_ns: bound on a CTA's wait for its products (< 0: no wait), see fem_opts.wait_limit_us.
cudaError_t launch_hex20_ke_tcgen05(const MeshView& m, double* ke_out, int* status, long long wait_ns,
                                    cudaStream_t s);
// fem_opts.wait_limit_us in nanoseconds: 0 -> 200 ms, > 0 -> that bound, < 0 -> -1 (no wait).
inline long long wait_ns_of(int wait_limit_us) {
    return wait_limit_us == 0 ? 200ll * 1000 * 1000 : (wait_limit_us > 0 ? 1000ll * wait_limit_us : -1);
}
// Target of a value-only re-assembly: CSR positions of every element block.
struct MapTarget {
    const int* map;      // [E * npe^2] position of block (a, b) of element e at e * npe^2 + a * npe + b
    const int* row_ptr;  // CSR row pointers of the pattern the map was built for
    double* values;      // CSR values (zeroed by the caller)
    const int* col_idx;  // CSR columns (the colouring baseline searches them)
};

// Scatter map of a mesh into a CSR pattern; status gets 1 << FEM_ERR_* bits.
cudaError_t launch_build_map(const MeshView& m, int kind, const int* row_ptr, const int* col_idx, int* map,
                             int* status, cudaStream_t s);
// Value-only re-assembly (atomics into values): 2-D kinds over perm ranges
// {q4 begin, q4 end, t3 begin, t3 end}; Hex20 over perm (status bits in info).
cudaError_t launch_reassemble_2d(const MeshView& m, int precision, const int* map, int G, const int* perm,
                                 const int* ranges, const int* row_ptr, double* values, int* status, cudaStream_t s);
// The tensor-core form of the Hex20 value-only re-assembly (ke_tcgen05.cu).
cudaError_t launch_reassemble_hex20_tc(const MeshView& m, const int* perm, const MapTarget& t, DevInfo* info,
                                       cudaStream_t s);
cudaError_t launch_reassemble_hex20(const MeshView& m, int precision, const int* perm, const MapTarget& t,
                                    DevInfo* info, cudaStream_t s);
// Colouring baseline for Hex20: elements perm[range[0], range[1]) (one colour),
// plain adds at binary-searched CSR positions (t.map unused); status bits in info.
cudaError_t launch_colour_hex20(const MeshView& m, const int* perm, const int* range, const MapTarget& t,
                                DevInfo* info, cudaStream_t s);

// Node -> element incidence lists (incidence.cu): cnt [N] (counts), off
// [N + 1], inc [sum of nodes per element], tiles [ceil(N / kScanTile)]
// scratch; status gets 1 << FEM_ERR_* bits.
cudaError_t launch_incidence(const MeshView& m, int* cnt, int* off, int* inc, long long* tiles, int* status, int sms,
                             cudaStream_t s);
// Two-pass Hex20 list scatter over the element groups of positions
// perm[i0, i1) (one wave; i0 a multiple of the group size). inc_off / inc:
// the mesh's node -> element incidence lists (launch_incidence; NULL: every
// node pair counts as shared by several groups). Pass 1 claims the list
// entries, zeroes the value blocks of the entries several groups add to and
// writes the groups' records (claim_hex20.cu); pass 2 adds the Ke blocks
// (values_hex20.cu; in the tensor-core form the wave's Ke are computed into
// stage first, ke_tcgen05.cu). map: kHex20WaveMapWords words (the groups'
// records, group_hex20.cuh); stage:
// kHex20Wave * kPackedHex20 doubles (tensor-core form only). wait_ns: see
// wait_ns_of.
cudaError_t launch_claim_hex20(const MeshView& m, const ListLayout& L, const int* perm, const int* inc_off,
                               const int* inc, int i0, int i1, int* map, cudaStream_t s);
cudaError_t launch_values_hex20(const MeshView& m, const ListLayout& L, int precision, const int* perm, int i0,
                                int i1, const int* map, double* stage, long long wait_ns, cudaStream_t s);
// The packed Ke of the elements perm[i0, i1) on the tensor cores, row q - i0 for position q.
cudaError_t launch_stage_hex20_tc(const MeshView& m, const int* perm, int i0, int i1, double* stage, int* status,
                                  long long wait_ns, cudaStream_t s);
// Elements per wave of the two-pass scatter: a multiple of the group size,
// large enough that each pass keeps every SM busy (4,096 groups a wave);
// the batched kernel's waves are smaller (its items interleave many meshes).
constexpr int kHex20Wave = 32768;
constexpr int kBatchHex20Wave = 4096;
constexpr int kHex20GroupSize = 8;            // elements per group (group_hex20.cuh)
constexpr int kHex20GroupRecWords = 5220;     // record words per group (header, nodes, blocks by pair, slots)
constexpr size_t kHex20WaveMapWords = (size_t)kHex20Wave / kHex20GroupSize * kHex20GroupRecWords;
static_assert(kBatchHex20Wave <= kHex20Wave, "the batched ring's first map is the single-mesh one");

// Spatial (3-D Morton bucket) element order; hist needs 1 << (3 * morton_bits(E)) ints, bbox 6 words.
int morton_bits(int num_elems);
cudaError_t launch_reorder_3d(const MeshView& m, int* hist, int* ranges, int* perm, unsigned long long* bbox, int sms,
                              cudaStream_t s);
cudaError_t launch_consolidate(const ListLayout& L, int dpn, int* row_ptr, int* col_idx, double* values,
                               long long capacity, long long* tile_sums, int num_tiles, cudaStream_t s);
// Node-block (BSR) form of the consolidation; capacity in blocks.
// Upper triangle (columns >= row, diagonal included) in CSR; ucounts: N ints of scratch.
cudaError_t launch_consolidate_upper(const ListLayout& L, int dpn, int* ucounts, int* row_ptr, int* col_idx,
                                     double* values, long long capacity, long long* tile_sums, int num_tiles,
                                     cudaStream_t s);
cudaError_t launch_consolidate_bsr(const ListLayout& L, int dpn, int* block_row_ptr, int* block_col_idx,
                                   double* block_values, long long capacity_blocks, long long* tile_sums,
                                   int num_tiles, cudaStream_t s);
cudaError_t launch_info_init(DevInfo* info, int pool_chunks, cudaStream_t s);

// ---- load vector and boundary conditions (loads.cu) ----
// f += body-force load vector (b: device [E * dim] or NULL for the uniform b0[dim], host values).
cudaError_t launch_body_force(const MeshView& m, int kind, const double* b, const double* b0, double* f, int* status,
                              cudaStream_t s);
// Symmetric elimination of fixed dofs in place on a CSR matrix (and f).
cudaError_t launch_dirichlet(int n_rows, const int* row_ptr, const int* col_idx, double* values, double* f,
                             const unsigned char* fixed, const double* u, cudaStream_t s);

// ---- batched assembly (batched.cu) ----
// One persistent kernel assembles every mesh of a batch: its CTAs take work
// items from one ticket counter in a fixed order (the schedule) and wait,
// bounded, on per-mesh phase counters for the items an item depends on.
constexpr int kMaxBatchConcurrency = 256;  // meshes whose lists are live at once (workspace slots)
// Estimated work of a mesh (elements weighted by kind) and the slot of each
// mesh (largest first onto the least loaded slot).
double batch_cost(const fem_mesh& m);
std::vector<int> batch_schedule(const fem_mesh* meshes, int n, int slots);

// Everything the batched kernel needs to know about one mesh (device copy).
struct BatchMesh {
    MeshView m;
    ListLayout L;
    long long* tiles;          // scan partials
    int* map[2];               // Hex20: group records of even / odd waves
    int* row_ptr;              // the caller's CSR
    int* col_idx;
    double* values;
    long long capacity;
    fem_info* info_out;        // the caller's info array entry
    unsigned long long* stamp; // completion stamp (may be NULL)
    unsigned char* zero_ptr[3];  // what the reset clears: info + first chunks, 2-D first-chunk values, counts
    long long zero_bytes[3];
    int kind, dpn, num_tiles, pad;
};

// Phases of a mesh (work item kinds); a segment is a run of consecutive
// tickets of one phase of one mesh.
enum BatchPhase : int {
    kBpReset = 0, kBpScatter2D, kBpClaim, kBpValues, kBpScanReduce, kBpScanTop, kBpRowPtr, kBpWrite, kBpFinish
};
// Per-mesh completion counters (index within the mesh's group of kBatchCounters).
enum BatchCounter : int {
    kBcReset = 0, kBcScatter, kBcValues, kBcScanReduce, kBcScanTop, kBcRowPtr, kBcWrite, kBcFinish
};
constexpr int kBatchCounters = 8;
struct BatchSegment {
    int mesh, phase, first, count;
    int arg;                 // Hex20 claim / value items: the wave
    int dep_ctr[2];          // counter indices (-1: none) and the values they must reach first
    int dep_target[2];
    int done_ctr;            // the counter each finished item increments
};
// Work item sizes.
constexpr int kBatchResetBytes = 1 << 20;  // bytes cleared per reset item
constexpr int kBatchScatter2D = 2048;      // 2-D elements per scatter item
constexpr int kBatchClaim = 8;             // Hex20 elements per claim item (one element group)
constexpr int kBatchValues = 8;            // Hex20 elements per value item (one group, one element at a time)
constexpr int kBatchWriteBatches = 16;     // node batches per write item

// Copies the tables into the workspace and zeroes the counters and the
// ticket (with the start stamp), then launches the persistent kernel.
cudaError_t launch_batch(const BatchMesh* meshes, int n, const BatchSegment* segs, int nseg, int total_items,
                         BatchMesh* d_meshes, BatchSegment* d_segs, int* d_counters, int* d_ticket,
                         unsigned long long* stamp0, long long wait_ns, int ctas_per_sm, cudaStream_t s);

// ---- element-colouring baseline (colour.cu) ----
constexpr int kMaxColours = 64;         // colours per mesh (a 64-bit mask of neighbour colours)
constexpr int kMaxColourRounds = 4096;  // bound on Jones-Plassmann rounds

struct ColourInfo {
    int num_colours;
    int status_bits;  // 1 << FEM_ERR_*
    int uncoloured;   // elements left after the last round
    int pad[13];
};
static_assert(sizeof(ColourInfo) == 64, "ColourInfo size");

// Device buffers of the colouring path (inside the caller's workspace).
struct ColourLayout {
    ColourInfo* info;
    int* cnt;        // [N] incidence counts, then fill cursors
    int* off;        // [N + 1] node -> element offsets
    int* inc;        // [sum of nodes per element] incidence lists
    int* colour;     // [E] round << 8 | colour, -1 = uncoloured
    int* perm;       // [E] elements grouped by (colour, type)
    int* hist;       // [2 * kMaxColours] counts, then cursors
    int* ranges;     // [2 * kMaxColours + 1] offsets of each (colour, type) group in perm
    long long* tiles;  // [ceil(N / kScanTile)] scan partials
};

// Incidence, colouring rounds (host loop, one sync per round) and grouping.
cudaError_t launch_colour_prepare(const MeshView& m, const ColourLayout& C, int sms, cudaStream_t s, int* num_colours,
                                  int* status_bits);
// out[e] = colour of element e.
cudaError_t launch_colour_export(const ColourLayout& C, int E, int* out, int sms, cudaStream_t s);
// values = 0, then one launch per (colour, type) group. Asynchronous.
cudaError_t launch_colour_assemble(const MeshView& m, const ColourLayout& C, int num_colours, const int* row_ptr,
                                   const int* col_idx, double* values, long long nnz, int sms, cudaStream_t s);


}  // namespace fem
