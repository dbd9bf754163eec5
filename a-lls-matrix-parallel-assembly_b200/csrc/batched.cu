// Batched assembly: many independent meshes of uneven sizes and element kinds
// in one persistent launch (graph-capturable).
//
// The reference assembles one mesh per program run (each driver's main, e.g.
// ALLS_Q4_T3_Mixed_Elements_Assembly_Performance.cu:742-854). Here the host
// turns the batch into a schedule: for each mesh its phases (list reset,
// 2-D scatter or Hex20 claim / value waves of element groups, consolidation
// scan, row pointers,
// sorted write, completion) as segments of work items, the meshes in rounds
// of `slots` (the workspace holds that many meshes' lists at once), each
// round phase by phase. One persistent kernel then runs the whole schedule:
// every CTA takes the next ticket from one counter, finds its segment, waits
// (bounded) until the mesh's phase counters say the items it depends on are
// finished, runs the item with the same device code as the single-mesh
// kernels (claim_hex20.cuh, values_hex20.cuh, scatter2d.cuh, consolidate.cuh)
// and counts it done. An item only ever depends on items with smaller
// tickets, which CTAs already running have taken, so the kernel always makes
// progress. A mesh's last item copies its info word into the caller's array
// and stamps its completion with the GPU global timer.
//
// The mesh descriptors and the schedule travel as kernel parameters of small
// copy kernels into the workspace, so a captured CUDA graph holds them; the
// counters and the ticket are zeroed by a kernel of the same sequence.
#define FEM_LDG(p) __ldcg(p)  // items read what earlier items of the launch wrote

#include <algorithm>
#include <mutex>
#include <numeric>
#include <vector>

#include "claim_hex20.cuh"
#include "consolidate.cuh"
#include "scatter2d.cuh"
#include "values_hex20.cuh"

namespace fem {
namespace {

constexpr int kBatchThreads = 256;
constexpr int kBatchWarps = kBatchThreads / 32;
static_assert(kBatchThreads == kScanThreads && kBatchThreads == kBlockThreads, "one CTA shape for every item");
static_assert(kBatchClaim % kGroup == 0 && kBatchValues == kGroup, "claim and value items of whole groups");

// A Hex20 value item: one group's topology and the element pass. Every pair
// is shared in the batch (the claim items get no node degrees), so each
// element's blocks are added atomically to slots that their claimers zeroed.
struct BatchValuesSmem {
    ValuesSmem values;
    GroupTopo topo;
};

// Shared memory of the item kinds (one at a time).
union BatchSmem {
    ClaimSmem claim;
    BatchValuesSmem gv;
    Scatter2DWarpSmem scatter[kBatchWarps];
    WriteSmem<2, 8, 2> write2;
    WriteSmem<3, 32, 4> write3;
    long long scan[kScanThreads / 32 + 1];
};

constexpr int kMeshChunk = 96;   // descriptors per copy kernel (kernel parameters stay under 32 KB)
constexpr int kSegChunk = 700;   // segments per copy kernel
struct MeshChunk {
    int first, count;
    BatchMesh m[kMeshChunk];
};
struct SegChunk {
    int first, count;
    BatchSegment s[kSegChunk];
};
static_assert(sizeof(MeshChunk) < 32000 && sizeof(SegChunk) < 32000, "kernel parameter size");

__global__ void k_copy_meshes(const MeshChunk c, BatchMesh* dst) {
    constexpr int kWords = sizeof(BatchMesh) / 8;
    static_assert(sizeof(BatchMesh) % 8 == 0, "descriptor copy in 8-byte words");
    for (int i = threadIdx.x; i < c.count * kWords; i += blockDim.x) {
        const int k = i / kWords, w = i - k * kWords;
        reinterpret_cast<unsigned long long*>(dst + c.first + k)[w] =
            reinterpret_cast<const unsigned long long*>(&c.m[k])[w];
    }
}

__global__ void k_copy_segments(const SegChunk c, BatchSegment* dst) {
    for (int i = threadIdx.x; i < c.count; i += blockDim.x) dst[c.first + i] = c.s[i];
}

__device__ __forceinline__ unsigned long long global_timer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__global__ void k_batch_start(int* counters, int n, int* ticket, unsigned long long* stamp0) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) counters[i] = 0;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        *ticket = 0;
        if (stamp0) *stamp0 = global_timer();
    }
}

// Clears bytes [lo, hi) of the concatenation of the mesh's reset ranges.
__device__ void reset_range(const BatchMesh& bm, long long lo, long long hi) {
    long long base = 0;
    for (int r = 0; r < 3; r++) {
        const long long len = bm.zero_bytes[r];
        const long long a = max(lo, base), b = min(hi, base + len);
        if (a < b) {
            unsigned char* p = bm.zero_ptr[r] + (a - base);
            const long long nb = b - a;
            // the ranges and the item bounds are 16-byte multiples except the
            // counts' tail: 16-byte stores, then bytes
            const long long n16 = nb >> 4;
            for (long long i = threadIdx.x; i < n16; i += blockDim.x)
                reinterpret_cast<int4*>(p)[i] = make_int4(0, 0, 0, 0);
            for (long long i = (n16 << 4) + threadIdx.x; i < nb; i += blockDim.x) p[i] = 0;
        }
        base += len;
    }
}

// Bounded wait of thread 0 until counters[c] >= target; false when it ran out.
__device__ bool wait_counter(const int* counters, int c, int target, long long wait_ns) {
    const volatile int* p = counters + c;
    if (*p >= target) return true;
    const unsigned long long t0 = global_timer();
    while (*p < target) {
        if ((long long)(global_timer() - t0) > wait_ns) return false;
        __nanosleep(256);
    }
    return true;
}

__global__ void __launch_bounds__(kBatchThreads, 2)
    k_batch(const BatchMesh* __restrict__ meshes, const BatchSegment* __restrict__ segs, int nseg, int total,
            int* counters, int* ticket, long long wait_ns) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    BatchSmem& sm = *reinterpret_cast<BatchSmem*>(smem_raw);
    __shared__ int s_ticket, s_seg;
    const int tid = threadIdx.x, warp = tid >> 5;
    for (;;) {
        if (tid == 0) {
            const int t = atomicAdd(ticket, 1);
            int lo = 0, hi = nseg - 1;  // the last segment whose first ticket is <= t
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (__ldg(&segs[mid].first) <= t) lo = mid;
                else hi = mid - 1;
            }
            s_ticket = t;
            s_seg = lo;
            if (t < total) {
                const BatchSegment& sg = segs[lo];
                for (int d = 0; d < 2; d++)
                    if (sg.dep_ctr[d] >= 0 && !wait_counter(counters, sg.dep_ctr[d], sg.dep_target[d], wait_ns))
                        raise_status(meshes[sg.mesh].L.info, FEM_ERR_TIMEOUT);
                __threadfence();  // what the awaited items wrote is seen after the counters
            }
        }
        __syncthreads();
        const int t = s_ticket;
        if (t >= total) break;
        const BatchSegment sg = segs[s_seg];
        const BatchMesh& bm = meshes[sg.mesh];
        const int k = t - sg.first;
        const MeshView& m = bm.m;
        const ListLayout& L = bm.L;
        switch (sg.phase) {
            case kBpReset: {
                reset_range(bm, (long long)k * kBatchResetBytes, (long long)(k + 1) * kBatchResetBytes);
                if (k == 0) {
                    __syncthreads();
                    if (tid == 0) L.info->pool_chunks = L.cap2;
                }
                break;
            }
            case kBpScatter2D: {
                const int b = k * kBatchScatter2D, cnt = min(kBatchScatter2D, m.E_count - b);
                if (bm.kind == FEM_Q4) {
                    scatter2d_warp<4, double>(m, L, nullptr, b, cnt, warp, kBatchWarps, sm.scatter[warp]);
                } else if (bm.kind == FEM_T3) {
                    scatter2d_warp<3, double>(m, L, nullptr, b, cnt, warp, kBatchWarps, sm.scatter[warp]);
                } else {
                    scatter2d_warp<4, double>(m, L, nullptr, b, cnt, warp, kBatchWarps, sm.scatter[warp], FEM_Q4);
                    scatter2d_warp<3, double>(m, L, nullptr, b, cnt, warp, kBatchWarps, sm.scatter[warp], FEM_T3);
                }
                break;
            }
            case kBpClaim: {
                const int w0 = sg.arg * kBatchHex20Wave, w1 = min(m.E_count, w0 + kBatchHex20Wave);
                const int b = w0 + k * kBatchClaim, e1 = min(w1, b + kBatchClaim);
                for (int gb = b; gb < e1; gb += kGroup)
                    claim_group(m, L, nullptr, nullptr, nullptr, gb, min(kGroup, e1 - gb),
                                bm.map[sg.arg & 1] + (size_t)((gb - w0) / kGroup) * kGroupRecWords, sm.claim);
                break;
            }
            case kBpValues: {
                const int w0 = sg.arg * kBatchHex20Wave, w1 = min(m.E_count, w0 + kBatchHex20Wave);
                const int b = w0 + k * kBatchValues, ne = min(kGroup, w1 - b);
                group_topology(m, nullptr, b, ne, sm.gv.topo);
                if (sm.gv.topo.bad) break;  // the claim item raised it
                ValuesTarget vt{};
                vt.topo = &sm.gv.topo;
                vt.rec = reinterpret_cast<const unsigned*>(bm.map[sg.arg & 1] + (size_t)((b - w0) / kGroup) * kGroupRecWords +
                                                           kRecMap);
                vt.g0 = b;
                vt.vals = L.vals;
                vt.info = L.info;
                values_init(sm.gv.values);
                values_cta<kToSlots>(m, nullptr, b, 1, b + ne, vt, sm.gv.values);
                break;
            }
            case kBpScanReduce:
                if (bm.dpn == 3) scan_reduce_tile<9>(L.counts, L.N, bm.tiles, k, sm.scan);
                else scan_reduce_tile<4>(L.counts, L.N, bm.tiles, k, sm.scan);
                break;
            case kBpScanTop:
                scan_tiles_body(bm.tiles, bm.num_tiles, L.info, bm.row_ptr + (size_t)L.N * bm.dpn, bm.capacity, 1,
                                sm.scan);
                break;
            case kBpRowPtr:
                if (bm.dpn == 3) row_ptr_tile<3, false>(L.counts, L.N, bm.tiles, bm.row_ptr, k, sm.scan);
                else row_ptr_tile<2, false>(L.counts, L.N, bm.tiles, bm.row_ptr, k, sm.scan);
                break;
            case kBpWrite:
                if (bm.dpn == 3) {
                    constexpr int NPB = kBlockThreads / 32;
                    const long long b = (long long)k * NPB * kBatchWriteBatches;
                    write_batches<3, 32, 4, kOutCsr>(L, bm.row_ptr, bm.col_idx, bm.values, bm.capacity, nullptr, b,
                                                     NPB, min((long long)L.N, b + NPB * kBatchWriteBatches),
                                                     sm.write3);
                } else {
                    constexpr int NPB = kBlockThreads / 8;
                    const long long b = (long long)k * NPB * kBatchWriteBatches;
                    write_batches<2, 8, 2, kOutCsr>(L, bm.row_ptr, bm.col_idx, bm.values, bm.capacity, nullptr, b,
                                                    NPB, min((long long)L.N, b + NPB * kBatchWriteBatches),
                                                    sm.write2);
                }
                break;
            case kBpFinish:
                if (tid < (int)(sizeof(fem_info) / 8))
                    reinterpret_cast<unsigned long long*>(bm.info_out)[tid] =
                        __ldcg(reinterpret_cast<const unsigned long long*>(L.info) + tid);
                if (tid == 0 && bm.stamp) *bm.stamp = global_timer();
                break;
            default:
                break;
        }
        __syncthreads();  // the item is finished (and the shared memory free) before it is counted
        if (tid == 0) {
            __threadfence();
            atomicAdd(counters + sg.done_ctr, 1);
        }
    }
}

}  // namespace

double batch_cost(const fem_mesh& m) {
    const double w = m.kind == FEM_HEX20 ? 60.0 : (m.kind == FEM_T3 ? 1.0 : 1.4);
    return w * (double)m.num_elems + 1e3;
}

std::vector<int> batch_schedule(const fem_mesh* meshes, int n, int slots) {
    std::vector<int> order(n), slot_of(n, 0);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return batch_cost(meshes[a]) > batch_cost(meshes[b]); });
    std::vector<double> load(slots, 0.0);
    for (int i : order) {
        const int k = (int)(std::min_element(load.begin(), load.end()) - load.begin());
        slot_of[i] = k;
        load[k] += batch_cost(meshes[i]);
    }
    return slot_of;
}

cudaError_t launch_batch(const BatchMesh* meshes, int n, const BatchSegment* segs, int nseg, int total_items,
                         BatchMesh* d_meshes, BatchSegment* d_segs, int* d_counters, int* d_ticket,
                         unsigned long long* stamp0, long long wait_ns, int ctas_per_sm, cudaStream_t s) {
    static MeshChunk mc;  // staging of the kernel parameters (copied at each launch)
    static SegChunk sc;
    static std::mutex mtx;
    std::lock_guard<std::mutex> lock(mtx);
    cudaError_t err = cudaSuccess;
    for (int f = 0; f < n && !err; f += kMeshChunk) {
        mc.first = f;
        mc.count = std::min(kMeshChunk, n - f);
        std::copy(meshes + f, meshes + f + mc.count, mc.m);
        k_copy_meshes<<<1, 256, 0, s>>>(mc, d_meshes);
        err = cudaGetLastError();
    }
    for (int f = 0; f < nseg && !err; f += kSegChunk) {
        sc.first = f;
        sc.count = std::min(kSegChunk, nseg - f);
        std::copy(segs + f, segs + f + sc.count, sc.s);
        k_copy_segments<<<1, 256, 0, s>>>(sc, d_segs);
        err = cudaGetLastError();
    }
    if (err) return err;
    k_batch_start<<<std::max(1, std::min(64, (n * kBatchCounters + 255) / 256)), 256, 0, s>>>(
        d_counters, n * kBatchCounters, d_ticket, stamp0);
    if ((err = cudaGetLastError())) return err;
    static DeviceCache cache;
    const size_t smem = sizeof(BatchSmem);
    int per_sm = 0;
    err = per_device(cache, [&](int& v) {
        cudaError_t e = cudaFuncSetAttribute(k_batch, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (!e) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, k_batch, kBatchThreads, smem);
        return e;
    }, per_sm);
    if (err) return err;
    // every CTA of the grid is resident at once: a CTA that waits never holds
    // back one that has not started
    const int use = ctas_per_sm > 0 ? std::min(ctas_per_sm, per_sm) : per_sm;
    const long long grid = std::max<long long>(1, std::min<long long>(total_items, (long long)use * sm_count()));
    k_batch<<<(int)grid, kBatchThreads, smem, s>>>(d_meshes, d_segs, nseg, total_items, d_counters, d_ticket, wait_ns);
    return cudaGetLastError();
}

}  // namespace fem
