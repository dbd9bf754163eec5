// Batched assembly: many independent meshes of uneven sizes and element kinds
// in one stream-ordered call (graph-capturable).
//
// The reference assembles one mesh per program run. Here the meshes are dealt
// to `concurrency` workspace slots; each slot has its own library stream and
// assembles its meshes one after another (scatter, consolidation, then a tiny
// kernel that copies the mesh's info word into the caller's array and stamps
// the completion time with the GPU's global timer). The slots' streams fork
// from the caller's stream and join it again through events, so the whole
// batch is ordered on the caller's stream and can be captured into a CUDA
// graph; small meshes of different slots run side by side on the GPU instead
// of one after another. Meshes are dealt largest first to the slot with the
// least estimated work (elements weighted by kind); each slot then runs its
// meshes smallest first.
#include <algorithm>
#include <mutex>
#include <numeric>
#include <vector>

#include "launch.h"

namespace fem {
namespace {

__global__ void k_stamp(unsigned long long* out) {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    *out = t;
}

// Copies a mesh's device info into the batch's info array; stamps its completion.
__global__ void k_finish(const DevInfo* info, fem_info* dst, unsigned long long* stamp) {
    static_assert(sizeof(fem_info) % 8 == 0, "fem_info copy in 8-byte words");
    const int i = threadIdx.x;
    if (i < (int)(sizeof(fem_info) / 8))
        reinterpret_cast<unsigned long long*>(dst)[i] = reinterpret_cast<const unsigned long long*>(info)[i];
    if (i == 0 && stamp) {
        unsigned long long t;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
        *stamp = t;
    }
}

// Library streams and events for the slots, per device, created on first use.
struct SlotStreams {
    cudaStream_t stream[kMaxBatchConcurrency] = {};
    cudaEvent_t fork = nullptr, join[kMaxBatchConcurrency] = {};
    bool ready = false;
};
constexpr int kMaxDevices = 64;
std::mutex g_slot_mutex;
SlotStreams g_slots[kMaxDevices];

cudaError_t slot_streams(SlotStreams*& out) {
    int dev = 0;
    cudaError_t err = cudaGetDevice(&dev);
    if (err) return err;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_slot_mutex);
    SlotStreams& s = g_slots[dev];
    if (!s.ready) {
        err = cudaEventCreateWithFlags(&s.fork, cudaEventDisableTiming);
        for (int k = 0; k < kMaxBatchConcurrency && !err; k++) {
            err = cudaStreamCreateWithFlags(&s.stream[k], cudaStreamNonBlocking);
            if (!err) err = cudaEventCreateWithFlags(&s.join[k], cudaEventDisableTiming);
        }
        if (err) return err;
        s.ready = true;
    }
    out = &s;
    return cudaSuccess;
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

cudaError_t batch_fork(int slots, cudaStream_t s, cudaStream_t* out_streams) {
    SlotStreams* ss = nullptr;
    cudaError_t err = slot_streams(ss);
    if (err) return err;
    err = cudaEventRecord(ss->fork, s);
    for (int k = 0; k < slots && !err; k++) {
        out_streams[k] = ss->stream[k];
        err = cudaStreamWaitEvent(ss->stream[k], ss->fork, 0);
    }
    return err;
}

cudaError_t batch_join(int slots, cudaStream_t s) {
    SlotStreams* ss = nullptr;
    cudaError_t err = slot_streams(ss);
    for (int k = 0; k < slots && !err; k++) {
        err = cudaEventRecord(ss->join[k], ss->stream[k]);
        if (!err) err = cudaStreamWaitEvent(s, ss->join[k], 0);
    }
    return err;
}

cudaError_t launch_stamp(unsigned long long* out, cudaStream_t s) {
    k_stamp<<<1, 1, 0, s>>>(out);
    return cudaGetLastError();
}

cudaError_t launch_finish(const DevInfo* info, fem_info* dst, unsigned long long* stamp, cudaStream_t s) {
    k_finish<<<1, 32, 0, s>>>(info, dst, stamp);
    return cudaGetLastError();
}

}  // namespace fem
