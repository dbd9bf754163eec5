// Element-colouring assembly: the comparison baseline of the A-LLS path.
//
// The reference colours elements on the host with a greedy pass over a
// node -> element map (colorElements, ALLS_Quad2D_Assembly_Accuracy_Analysis.cu:648-747;
// ALLS_T3_Unstructed_Elements_Assemble_Performance.cu:484-523;
// ALLS_Q4_T3_Mixed_Elements_Assembly_Performance.cu:514-553) and then assembles
// with one CTA per colour, binary-searching each entry in the host CSR pattern
// and adding it without atomics (assembleGlobalStiffnessKernelColored(NoAtomic),
// Q4A:504-572, T3:316-363, MIX:341-390). All colours run at once there, so
// elements of different colours that share a node race, and the Q4 programs
// never reorder the elements by colour.
//
// Rebuilt here so that it is correct and uses the whole GPU:
//   launch_incidence                  node -> element incidence lists (CSR)
//   k_jp_round (repeated)             Jones-Plassmann colouring: in each round
//                                     an uncoloured element whose priority (a
//                                     hash of its id) beats every uncoloured
//                                     element sharing a node with it takes the
//                                     smallest colour not used by its coloured
//                                     neighbours. Elements coloured in the
//                                     current round carry the round number, so
//                                     a concurrent reader treats them as still
//                                     uncoloured: two neighbours never take a
//                                     colour in the same round.
//   k_colour_hist / k_colour_scatter  elements grouped by (colour, type)
//   k_colour_assemble_2d (per colour) one lane per node block (as the A-LLS
//                                     scatter), binary search of the block's
//                                     column in the CSR row, plain adds: no two
//                                     elements of one colour share a node, so no
//                                     two lanes of a launch touch the same row.
// Launches of consecutive colours are stream-ordered, so colours never overlap.
#include <algorithm>

#include "element2d.cuh"
#include "launch.h"

namespace fem {
namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ int elem_npe(const MeshView& m, int e) {
    if (m.types) return __ldg(m.types + e) == FEM_Q4 ? 4 : 3;
    return m.stride;
}

__device__ __forceinline__ unsigned elem_priority(int e) {
    unsigned x = (unsigned)e * 0x9E3779B1u;
    x ^= x >> 16;
    x *= 0x85EBCA6Bu;
    x ^= x >> 13;
    return x;
}

// Strict order of element priorities (ties broken by id).
__device__ __forceinline__ bool beats(int f, unsigned pf, int e, unsigned pe) {
    return pf > pe || (pf == pe && f > e);
}


// One Jones-Plassmann round. colour[e] = -1 (uncoloured) or round << 8 | c.
__global__ void k_jp_round(MeshView m, const int* __restrict__ off, const int* __restrict__ inc,
                           int* __restrict__ colour, int round, ColourInfo* info) {
    int left = 0;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < m.E_count; e += gridDim.x * blockDim.x) {
        if (__ldcg(colour + e) >= 0) continue;
        const unsigned pe = elem_priority(e);
        const int npe = elem_npe(m, e);
        unsigned long long used = 0;
        bool is_max = true;
        for (int k = 0; k < npe && is_max; k++) {
            const int n = __ldg(m.conn + (size_t)e * m.stride + k);
            if (n < 0 || n >= m.N) continue;
            const int b = __ldg(off + n), en = __ldg(off + n + 1);
            for (int q = b; q < en; q++) {
                const int f = __ldg(inc + q);
                if (f == e) continue;
                const int cf = __ldcg(colour + f);
                if (cf < 0 || (cf >> 8) == round) {  // uncoloured at the start of this round
                    if (beats(f, elem_priority(f), e, pe)) {
                        is_max = false;
                        break;
                    }
                } else {
                    used |= 1ull << (cf & 0xFF);
                }
            }
        }
        if (is_max) {
            int c = __ffsll((long long)~used) - 1;
            if (c < 0) {
                atomicOr(&info->status_bits, 1 << FEM_ERR_RANGE);  // more than kMaxColours colours needed
                c = kMaxColours - 1;
            }
            __stcg(colour + e, (round << 8) | c);
        } else {
            left++;
        }
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) left += __shfl_xor_sync(0xFFFFFFFFu, left, d);
    if ((threadIdx.x & 31) == 0 && left) atomicAdd(&info->uncoloured, left);
}

// Key of an element in the colour order: colour * 2 + (T3 in a mixed mesh).
__device__ __forceinline__ int colour_key(const MeshView& m, const int* colour, int e) {
    const int c = colour[e] & 0xFF;
    return 2 * c + ((m.types && __ldg(m.types + e) != FEM_Q4) ? 1 : 0);
}

// Per-CTA histogram of the keys, one global atomic per key per CTA.
__global__ void k_colour_hist(MeshView m, const int* __restrict__ colour, int* __restrict__ hist, ColourInfo* info) {
    __shared__ int s_hist[2 * kMaxColours];
    for (int i = threadIdx.x; i < 2 * kMaxColours; i += blockDim.x) s_hist[i] = 0;
    __syncthreads();
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < m.E_count; e += gridDim.x * blockDim.x)
        atomicAdd(s_hist + colour_key(m, colour, e), 1);
    __syncthreads();
    for (int i = threadIdx.x; i < 2 * kMaxColours; i += blockDim.x)
        if (s_hist[i]) {
            atomicAdd(hist + i, s_hist[i]);
            atomicMax(&info->num_colours, i / 2 + 1);
        }
}

// ranges[k] = exclusive prefix of hist (2 * kMaxColours + 1 entries); hist becomes a cursor.
__global__ void k_colour_ranges(int* __restrict__ hist, int* __restrict__ ranges) {
    if (threadIdx.x == 0) {
        int acc = 0;
        for (int k = 0; k < 2 * kMaxColours; k++) {
            ranges[k] = acc;
            acc += hist[k];
            hist[k] = 0;
        }
        ranges[2 * kMaxColours] = acc;
    }
}

__global__ void k_colour_scatter(MeshView m, const int* __restrict__ colour, const int* __restrict__ ranges,
                                 int* __restrict__ cursor, int* __restrict__ perm) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < m.E_count; e += gridDim.x * blockDim.x) {
        const int k = colour_key(m, colour, e);
        perm[ranges[k] + atomicAdd(cursor + k, 1)] = e;
    }
}

// Position of column col in CSR row r (sorted), or -1.
__device__ __forceinline__ int csr_find(const int* __restrict__ row_ptr, const int* __restrict__ col_idx, int r,
                                        int col) {
    int lo = __ldg(row_ptr + r), hi = __ldg(row_ptr + r + 1) - 1;
    while (lo <= hi) {
        const int mid = (lo + hi) >> 1;
        const int c = __ldg(col_idx + mid);
        if (c == col) return mid;
        if (c < col) lo = mid + 1;
        else hi = mid - 1;
    }
    return -1;
}

// Assembly of the elements perm[ranges[key] .. ranges[key+1]) (one colour, one
// element type): one lane per node block, plain read-modify-write adds.
template <int NPE>
__global__ void __launch_bounds__(kThreads) k_colour_assemble_2d(MeshView m, const int* __restrict__ perm,
                                                                 const int* __restrict__ ranges, int key,
                                                                 const int* __restrict__ row_ptr,
                                                                 const int* __restrict__ col_idx,
                                                                 double* __restrict__ values, ColourInfo* info) {
    constexpr int G = NPE * NPE, EPW = 32 / G;
    const int lane = threadIdx.x & 31;
    const int eslot = lane / G, sub = lane - eslot * G, a = sub / NPE, b = sub - (sub / NPE) * NPE;
    const int begin = ranges[key], count = ranges[key + 1] - begin;
    const long long warp_id = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long stride = (((long long)gridDim.x * blockDim.x) >> 5) * EPW;
    for (long long i = warp_id * EPW + eslot; i - eslot < count; i += stride) {
        if (eslot >= EPW || i >= count) continue;
        const int e = __ldg(perm + begin + i);
        int nodes[NPE];
        bool bad = false;
#pragma unroll
        for (int k = 0; k < NPE; k++) {
            nodes[k] = __ldg(m.conn + (size_t)e * m.stride + k);
            bad |= (nodes[k] < 0) | (nodes[k] >= m.N);
        }
        if (bad) continue;  // reported by the incidence pass
        double xe[NPE], ye[NPE];
#pragma unroll
        for (int k = 0; k < NPE; k++) {
            xe[k] = __ldg(m.x + nodes[k]);
            ye[k] = __ldg(m.y + nodes[k]);
        }
        const double E = m.E ? __ldg(m.E + e) : m.E0;
        const double nu = m.nu ? __ldg(m.nu + e) : m.nu0;
        double kv[4];
        const double det = ke_block_2d<NPE>(xe, ye, E, nu, m.t, a, b, kv);
        if (sub == 0 && !(det > 0.0)) atomicOr(&info->status_bits, 1 << FEM_ERR_DETJ);
        int row = nodes[0], col = nodes[0];
#pragma unroll
        for (int k = 1; k < NPE; k++) {
            row = a == k ? nodes[k] : row;
            col = b == k ? nodes[k] : col;
        }
        // rows 2 row and 2 row + 1 hold the same columns: one search serves both
        const int r0 = 2 * row;
        const int p0 = csr_find(row_ptr, col_idx, r0, 2 * col);
        if (p0 < 0) {
            atomicOr(&info->status_bits, 1 << FEM_ERR_INTERNAL);  // pattern lacks the entry
            continue;
        }
        const int p1 = __ldg(row_ptr + r0 + 1) + (p0 - __ldg(row_ptr + r0));
        values[p0] += kv[0];
        values[p0 + 1] += kv[1];
        values[p1] += kv[2];
        values[p1 + 1] += kv[3];
    }
}

__global__ void k_colour_export(const int* __restrict__ colour, int E, int* __restrict__ out) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < E; e += gridDim.x * blockDim.x) out[e] = colour[e] & 0xFF;
}

int grid_for(long long work, int sms) {
    const long long want = (work + kThreads - 1) / kThreads;
    return (int)std::min<long long>(want > 0 ? want : 1, (long long)sms * 8);
}

}  // namespace

cudaError_t launch_colour_prepare(const MeshView& m, const ColourLayout& C, int sms, cudaStream_t s, int* num_colours,
                                  int* status_bits) {
    cudaError_t err = cudaMemsetAsync(C.info, 0, sizeof(ColourInfo), s);
    if (!err) err = cudaMemsetAsync(C.colour, 0xFF, (size_t)m.E_count * sizeof(int), s);
    if (!err) err = cudaMemsetAsync(C.hist, 0, 2 * kMaxColours * sizeof(int), s);
    if (err) return err;
    if ((err = launch_incidence(m, C.cnt, C.off, C.inc, C.tiles, &C.info->status_bits, sms, s))) return err;
    const int ge = grid_for(m.E_count, sms);
    // Colouring rounds until every element has a colour (each round colours
    // at least the element of highest priority among the uncoloured ones).
    int left = m.E_count;
    for (int round = 0; left > 0; round++) {
        if (round >= kMaxColourRounds) {
            *status_bits |= 1 << FEM_ERR_TIMEOUT;
            return cudaSuccess;
        }
        if ((err = cudaMemsetAsync(&C.info->uncoloured, 0, sizeof(int), s))) return err;
        k_jp_round<<<ge, kThreads, 0, s>>>(m, C.off, C.inc, C.colour, round, C.info);
        if ((err = cudaMemcpyAsync(&left, &C.info->uncoloured, sizeof(int), cudaMemcpyDeviceToHost, s))) return err;
        if ((err = cudaStreamSynchronize(s))) return err;
    }
    k_colour_hist<<<ge, kThreads, 0, s>>>(m, C.colour, C.hist, C.info);
    k_colour_ranges<<<1, 32, 0, s>>>(C.hist, C.ranges);
    k_colour_scatter<<<ge, kThreads, 0, s>>>(m, C.colour, C.ranges, C.hist, C.perm);
    if ((err = cudaGetLastError())) return err;
    ColourInfo h{};
    if ((err = cudaMemcpyAsync(&h, C.info, sizeof(h), cudaMemcpyDeviceToHost, s))) return err;
    if ((err = cudaStreamSynchronize(s))) return err;
    *num_colours = h.num_colours;
    *status_bits |= h.status_bits;
    return cudaSuccess;
}

cudaError_t launch_colour_export(const ColourLayout& C, int E, int* out, int sms, cudaStream_t s) {
    k_colour_export<<<grid_for(E, sms), kThreads, 0, s>>>(C.colour, E, out);
    return cudaGetLastError();
}

cudaError_t launch_colour_assemble(const MeshView& m, const ColourLayout& C, int num_colours, const int* row_ptr,
                                   const int* col_idx, double* values, long long nnz, int sms, cudaStream_t s) {
    cudaError_t err = cudaMemsetAsync(values, 0, (size_t)nnz * sizeof(double), s);
    if (err) return err;
    // Grid: enough warps for the largest possible colour class, capped at the
    // resident size; each launch covers one (colour, type) range.
    const int epw_q4 = 2, epw_t3 = 3;
    const bool has_q4 = m.types || m.stride == 4, has_t3 = m.types || m.stride == 3;
    const int gq = grid_for(((long long)m.E_count + epw_q4 - 1) / epw_q4 * 32, sms);
    const int gt = grid_for(((long long)m.E_count + epw_t3 - 1) / epw_t3 * 32, sms);
    for (int c = 0; c < num_colours; c++) {
        if (has_q4)
            k_colour_assemble_2d<4><<<gq, kThreads, 0, s>>>(m, C.perm, C.ranges, 2 * c, row_ptr, col_idx, values,
                                                           C.info);
        if (has_t3)
            k_colour_assemble_2d<3><<<gt, kThreads, 0, s>>>(m, C.perm, C.ranges, m.types ? 2 * c + 1 : 2 * c,
                                                           row_ptr, col_idx, values, C.info);
    }
    return cudaGetLastError();
}

}  // namespace fem
