// K1 for Hex20 meshes: fused FP64 element stiffness + A-LLS row-list scatter.
//
// Replaces assembleGlobalStiffnessKernelALLSFixedArray
// (ALLS_Hex20_3D_Assembly_Performance.cu:208-257), whose 60x60 FP32 Ke lives in
// 14.9 KB of local memory per thread and whose fixed 300-entry rows silently
// drop overflow.
//
// One CTA (10 warps) per element at a time, persistent over the elements, which
// it visits in the spatial order computed by launch_reorder_3d.
//
// Element stiffness (the node-pair matrix M of hex20.cuh), in double: M is one
// symmetric 64x64x28 FP64 matrix product per element, computed on the FP64
// tensor cores with mma.sync.m8n8k4.f64 (36 upper 8x8 tiles x 7 k-steps), or
// with FEM_PREC_TC_F16X3 on the FP16 tensor cores from split operands
// (tc_prepare / tc_contract); only the 210 upper 3x3 node blocks of M are kept
// (so every Ke is exactly symmetric), in the shared memory the gradients
// occupied. Ke blocks are formed from M per scattered row. The
// Gauss-point shape derivatives (ALLS_Hex20_3D_Assembly_Performance.cu:95-128)
// are tabulated once per CTA.
//
// Scatter. Warp w serves row nodes w and w+10. It prefetches both rows' chunk
// rows (384 bytes: next pointer + 94 hashed slots) into shared memory with one
// 16-byte load per lane, matches every slot against a shared-memory hash of the
// element's 20 nodes, and builds ballot bitmaps of the empty slots. Lane j then
// claims the first empty slot on column node j's probe sequence with atomicCAS
// (empty -> col|pending) if the column is absent — re-trying past slots another
// warp has just taken — and follows / atomicCAS-links overflow chunks when the
// probe sequence is full. Each row's 20 blocks are staged once and written in
// one coalesced pass: plain stores into the slots the warp claimed, FP64
// atomicAdds into published ones. The warp then fences once and publishes its
// claims of both rows; blocks whose slot another warp was still writing are
// added after a bounded wait. The next element's nodes and coordinates are
// prefetched during the compute and the scatter.
#include "hex20.cuh"

namespace fem {
namespace {

using hex20::TcScratch;

constexpr int kThreads = 320;
constexpr int kWarps = kThreads / 32;
constexpr int kMaxHex20Words = 96;   // chunk meta rows of at most 96 words (S <= 94, checked on the host)
constexpr int PS = 28;               // row stride of P (doubles): conflict-free m8n8k4 fragment loads
constexpr int kHash = 64;            // element-node hash slots

// The 36 upper 8x8 tiles (mt <= nt) of the 64x64 node-pair matrix.
__constant__ unsigned char c_tile_m[36] = {0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 1, 1, 1, 2, 2, 2,
                                           2, 2, 2, 3, 3, 3, 3, 3, 4, 4, 4, 4, 5, 5, 5, 6, 6, 7};
__constant__ unsigned char c_tile_n[36] = {0, 1, 2, 3, 4, 5, 6, 7, 1, 2, 3, 4, 5, 6, 7, 2, 3, 4,
                                           5, 6, 7, 3, 4, 5, 6, 7, 4, 5, 6, 7, 5, 6, 7, 6, 7, 7};

enum SlotState : int { kUnresolved = 0, kFound = 1, kFoundPending = 2, kClaimed = 3 };
enum OutMode : int { kOutLists = 0, kOutMap = 1, kOutColour = 2 };

struct Hex20Smem {
    double dN[27][3][20];      // shape derivatives at the Gauss points
    union {
        double P[64][PS];      // P[3n+a][g] = G_g[n][a]; rows 60..63 and column 27 zeroed per element
        double Mb[210][9];     // upper 3x3 node blocks of M: Mb[pair(I, J)][3a + b] = M[3I+a][3J+b], I <= J
    };
    double X[20][3];           // element node coordinates
    double J[27][9];           // Jacobians, then their inverses
    double w[PS];              // Gauss weight * detJ (w[27] = 0 pads the contraction)
    alignas(16) int view[kWarps][2][kMaxHex20Words];  // per-warp copies of the two rows' chunks
    unsigned gid[kWarps][20];  // slot of each column node's entry in the row being committed
    int state[kWarps][20];
    union {
        double stage[kWarps][20 * 9];  // the row's 20 Ke blocks, entry j*9 + v
        TcScratch tc;                  // FP16 split operands while M is computed (tensor-core form)
    };
    int hkey[kHash];           // element-node hash: node + 1 -> local index
    int hval[kHash];
    int nodes[20];
    double lam, mu;
    int bad;
    unsigned long long dnmax_bits;  // largest |dN| of the table (bits of a positive double)
};

static_assert(offsetof(Hex20Smem, view) % 16 == 0, "int4 stores into view need 16-byte alignment");
static_assert(kMaxHex20Words % 32 == 0 && kMaxHex20Words <= 128, "view rows: whole ballot words");
static_assert((kMaxHex20Words * sizeof(int)) % 16 == 0, "view rows must stay 16-byte aligned");

__device__ __forceinline__ unsigned hash_slot(int key) { return ((unsigned)key * 2654435761u) >> 26; }

// Local index of node key (node + 1) in the current element, or -1.
__device__ __forceinline__ int element_lookup(const Hex20Smem& sm, int key) {
    unsigned h = hash_slot(key);
    for (int i = 0; i < kHash; i++) {
        const int k = sm.hkey[h];
        if (k == key) return sm.hval[h];
        if (k == 0) return -1;
        h = (h + 1) & (kHash - 1);
    }
    return -1;
}

__device__ __forceinline__ unsigned pick(const unsigned (&bm)[4], int k) {
    return k == 0 ? bm[0] : (k == 1 ? bm[1] : (k == 2 ? bm[2] : bm[3]));
}

// First set bit at word position >= p0, cyclically over the nw bitmap words; -1 if none.
__device__ __forceinline__ int first_empty_from(const unsigned (&bm)[4], int nw, int p0) {
    int k = p0 >> 5;
    unsigned m = pick(bm, k) & (0xFFFFFFFFu << (p0 & 31));
    for (int it = 0; it <= nw; it++) {
        if (m) return (k << 5) + __ffs(m) - 1;
        k = k + 1 == nw ? 0 : k + 1;
        m = pick(bm, k);
    }
    return -1;
}

// Block Ke_IJ into out[0..9) (row-major 3x3):
//   Ke_IJ[a][b] = lambda M[3I+a][3J+b] + mu M[3I+b][3J+a] + mu delta_ab tr(M_IJ)
__device__ __forceinline__ void ke_block(const Hex20Smem& sm, int I, int J, double* out) {
    const bool t = I > J;
    const double* m0 = sm.Mb[t ? hex20::pair_index(J, I) : hex20::pair_index(I, J)];
    const double m00 = m0[0], m11 = m0[4], m22 = m0[8];
    const double m01 = t ? m0[3] : m0[1], m02 = t ? m0[6] : m0[2];
    const double m10 = t ? m0[1] : m0[3], m12 = t ? m0[7] : m0[5];
    const double m20 = t ? m0[2] : m0[6], m21 = t ? m0[5] : m0[7];
    const double lam = sm.lam, mu = sm.mu, mtr = mu * (m00 + m11 + m22);
    out[0] = fma(lam, m00, fma(mu, m00, mtr));
    out[1] = fma(lam, m01, mu * m10);
    out[2] = fma(lam, m02, mu * m20);
    out[3] = fma(lam, m10, mu * m01);
    out[4] = fma(lam, m11, fma(mu, m11, mtr));
    out[5] = fma(lam, m12, mu * m21);
    out[6] = fma(lam, m20, mu * m02);
    out[7] = fma(lam, m21, mu * m12);
    out[8] = fma(lam, m22, fma(mu, m22, mtr));
}

// Copies the first chunk row of node n into view (one 16-byte load per lane).
__device__ __forceinline__ void load_view(const ListLayout& L, int c, int* view, int lane) {
    const int* meta = chunk_meta(L, c);
    const int H = c < L.N ? L.H1 : L.H2;
    for (int q = lane * 4; q < H; q += 128) *reinterpret_cast<int4*>(view + q) = ld_cg4(meta + q);
}

// Resolves the 20 column slots of row node I of the current element (lane j
// owns column node j). On entry `view` holds the row's first chunk. Returns the
// lane's state and slot; s_state / s_gid are per-warp scratch.
__device__ __forceinline__ void resolve_row(const ListLayout& L, const Hex20Smem& sm, int I, int lane, int* view,
                                            int* s_state, unsigned* s_gid, int& spare, int& state, unsigned& gid) {
    constexpr unsigned kFull = 0xFFFFFFFFu;
    const int key = lane < 20 ? sm.nodes[lane] + 1 : 0;
    state = lane < 20 ? kUnresolved : kFound;
    gid = 0;
    if (lane < 20) s_state[lane] = kUnresolved;
    int c = sm.nodes[I];
    for (int step = 0; step < kMaxChainSteps; step++) {
        int* meta = chunk_meta(L, c);
        const int H = c < L.N ? L.H1 : L.H2;
        if (step > 0) load_view(L, c, view, lane);
        __syncwarp();
        // columns already in this chunk
        for (int p = 2 + lane; p < H; p += 32) {
            const int v = view[p];
            if (v != 0) {
                const int j = element_lookup(sm, v & kColMask);
                if (j >= 0) {
                    s_gid[j] = slot_gid(L, c, p - 2);
                    s_state[j] = v < 0 ? kFoundPending : kFound;
                }
            }
        }
        unsigned bm[4];
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const int p = 32 * k + lane;
            bm[k] = __ballot_sync(kFull, p >= 2 && p < H && view[p] == 0);
        }
        __syncwarp();
        if (state == kUnresolved && s_state[lane] != kUnresolved) {
            state = s_state[lane];
            gid = s_gid[lane];
        }
        // claim the first empty slot on the probe sequence of each absent column
        if (state == kUnresolved) {
            int p0 = 2 + probe_start(key, H - 2);
            for (int tries = 0; tries < H; tries++) {
                const int p = first_empty_from(bm, (H + 31) >> 5, p0);
                if (p < 0) break;  // probe sequence full: continue in the next chunk
                const int old = atomicCAS(meta + p, 0, key | kPending);
                if (old == 0) {
                    state = kClaimed;
                } else if ((old & kColMask) == key) {
                    state = old < 0 ? kFoundPending : kFound;
                } else {
                    const unsigned bit = 1u << (p & 31);
                    const int k = p >> 5;
                    bm[0] &= k == 0 ? ~bit : 0xFFFFFFFFu;
                    bm[1] &= k == 1 ? ~bit : 0xFFFFFFFFu;
                    bm[2] &= k == 2 ? ~bit : 0xFFFFFFFFu;
                    bm[3] &= k == 3 ? ~bit : 0xFFFFFFFFu;
                    p0 = p;
                    continue;
                }
                gid = slot_gid(L, c, p - 2);
                break;
            }
        }
        __syncwarp();
        if (!__any_sync(kFull, state == kUnresolved)) break;
        int nc = 0;
        if (lane == 0) nc = next_chunk(L, c, spare);
        c = __shfl_sync(kFull, nc, 0);
        if (c < 0) break;  // pool overflow: status raised, unresolved columns dropped
        if (lane < 20 && state == kUnresolved) s_state[lane] = kUnresolved;
        __syncwarp();
    }
}

// Stages row I's 20 Ke blocks (lane j: column node j) with their states, then
// writes them in one pass: lane l handles entries l, l+32, ... of the 20 x 9
// values, so consecutive lanes write consecutive doubles of the same 72-byte
// slot block. Claimed slots (ours, not yet published) take plain stores,
// published ones FP64 red.add; pending ones are left for later.
__device__ __forceinline__ void write_row(const ListLayout& L, Hex20Smem& sm, int I, int warp, int lane, int state,
                                          unsigned gid) {
    if (lane < 20) {
        sm.state[warp][lane] = state;
        sm.gid[warp][lane] = gid;
        ke_block(sm, I, lane, &sm.stage[warp][lane * 9]);
    }
    __syncwarp();
#pragma unroll
    for (int k = 0; k < 6; k++) {
        const int idx = lane + 32 * k;
        if (idx < 20 * 9) {
            const int j = (idx * 57) >> 9;  // idx / 9 for idx < 180
            const int st = sm.state[warp][j];
            double* p = L.vals + (size_t)sm.gid[warp][j] * 9 + (idx - 9 * j);
            if (st == kClaimed)
                *p = sm.stage[warp][idx];
            else if (st == kFound)
                atomicAdd(p, sm.stage[warp][idx]);
        }
    }
    __syncwarp();
}

// Publishes a claimed slot: a plain store of the column after the fence that
// made its values visible.
__device__ __forceinline__ void publish(const ListLayout& L, unsigned gid, int key) {
    int cc, s;
    gid_chunk(L, gid, cc, s);
    __stcg(chunk_meta(L, cc) + 2 + s, key);
}

// A block whose slot another warp had claimed but not yet published: wait
// (bounded), then add it.
__device__ __forceinline__ void add_pending(const ListLayout& L, const Hex20Smem& sm, int I, int lane, unsigned gid) {
    int cc, s;
    gid_chunk(L, gid, cc, s);
    if (wait_published(L, chunk_meta(L, cc) + 2 + s)) {
        double v[9];
        ke_block(sm, I, lane, v);
        double* p = L.vals + (size_t)gid * 9;
#pragma unroll
        for (int k = 0; k < 9; k++) atomicAdd(p + k, v[k]);
    }
}

// Scatter of row nodes I0 and I1 (I1 < 0: none) by one warp.
__device__ __forceinline__ void scatter_rows(const ListLayout& L, Hex20Smem& sm, int I0, int I1, int warp, int lane,
                                             int& spare) {
    constexpr unsigned kFull = 0xFFFFFFFFu;
    const int key = lane < 20 ? sm.nodes[lane] + 1 : 0;
    load_view(L, sm.nodes[I0], sm.view[warp][0], lane);
    if (I1 >= 0) load_view(L, sm.nodes[I1], sm.view[warp][1], lane);
    int st0, st1 = kFound;
    unsigned g0, g1 = 0;
    resolve_row(L, sm, I0, lane, sm.view[warp][0], sm.state[warp], sm.gid[warp], spare, st0, g0);
    if (I1 >= 0) resolve_row(L, sm, I1, lane, sm.view[warp][1], sm.state[warp], sm.gid[warp], spare, st1, g1);
    const unsigned c0 = __ballot_sync(kFull, st0 == kClaimed), c1 = __ballot_sync(kFull, st1 == kClaimed);
    if (lane == 0) {
        if (c0) atomicAdd(L.counts + sm.nodes[I0], __popc(c0));
        if (c1) atomicAdd(L.counts + sm.nodes[I1], __popc(c1));
    }
    // claimed blocks stored, found blocks added; one fence, then the claims of
    // both rows are published (their slots stay pending only this long)
    write_row(L, sm, I0, warp, lane, st0, g0);
    if (I1 >= 0) write_row(L, sm, I1, warp, lane, st1, g1);
    if (c0 | c1) {
        __threadfence();
        __syncwarp();
        if (st0 == kClaimed) publish(L, g0, key);
        if (st1 == kClaimed) publish(L, g1, key);
    }
    if (st0 == kFoundPending) add_pending(L, sm, I0, lane, g0);
    if (st1 == kFoundPending) add_pending(L, sm, I1, lane, g1);
    __syncwarp();
}

// Value-only re-assembly (reassemble.cu): row nodes I0 and I1 of element e,
// lane j adds block (I, j) at the CSR positions of the scatter map.
// Colouring baseline (colour.cu): row nodes I0 and I1, lane j adds block
// (I, j) at its binary-searched CSR position with plain loads and stores (no
// two elements of a colour share a node, so no two lanes write one entry).
__device__ __forceinline__ void colour_rows(const MapTarget& t, const Hex20Smem& sm, int I0, int I1, int lane,
                                            DevInfo* info) {
    if (lane >= 20) return;
    for (int r = 0; r < 2; r++) {
        const int I = r == 0 ? I0 : I1;
        if (I < 0) continue;
        const int r0 = 3 * sm.nodes[I], col = 3 * sm.nodes[lane];
        int lo = __ldg(t.row_ptr + r0), hi = __ldg(t.row_ptr + r0 + 1) - 1, p = -1;
        const int len = hi + 1 - lo;
        while (lo <= hi) {
            const int mid = (lo + hi) >> 1;
            const int c = __ldg(t.col_idx + mid);
            if (c == col) {
                p = mid;
                break;
            }
            if (c < col) lo = mid + 1;
            else hi = mid - 1;
        }
        if (p < 0) {
            raise_status(info, FEM_ERR_INTERNAL);  // the pattern lacks the block
            continue;
        }
        double v[9];
        ke_block(sm, I, lane, v);
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) t.values[p + i * len + j] += v[3 * i + j];
    }
}

__device__ __forceinline__ void map_rows(const MapTarget& t, const Hex20Smem& sm, int e, int I0, int I1, int lane) {
    if (lane >= 20) return;
    for (int r = 0; r < 2; r++) {
        const int I = r == 0 ? I0 : I1;
        if (I < 0) continue;
        const int p = __ldg(t.map + (size_t)e * 400 + I * 20 + lane);
        if (p < 0) continue;
        const int r0 = 3 * sm.nodes[I];
        const int len = __ldg(t.row_ptr + r0 + 1) - __ldg(t.row_ptr + r0);
        double v[9];
        ke_block(sm, I, lane, v);
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) atomicAdd(t.values + p + i * len + j, v[3 * i + j]);
    }
}

__device__ __forceinline__ void dmma_8x8x4(double& c0, double& c1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(c0), "+d"(c1)
                 : "d"(a), "d"(b));
}

// Resident CTAs per SM the register budget is set for (build-time tuning knob).
#ifndef FEM_HEX20_MIN_CTAS
#define FEM_HEX20_MIN_CTAS 3
#endif

// kTc: the node-pair contraction on the FP16 tensor cores (hex20.cuh).
// kOut: kOutLists = the A-LLS list scatter; kOutMap = value-only re-assembly
// into a CSR pattern through a scatter map (atomic adds); kOutColour = the
// colouring baseline (plain adds, elements perm[range[0], range[1]) of one colour).
template <bool kTc, int kOut>
__global__ void __launch_bounds__(kThreads, FEM_HEX20_MIN_CTAS)
    k_scatter_hex20(MeshView m, ListLayout L, const int* __restrict__ perm, MapTarget target,
                    const int* __restrict__ range) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Hex20Smem& sm = *reinterpret_cast<Hex20Smem*>(smem_raw);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    if (tid == 0) sm.dnmax_bits = 0ull;
    __syncthreads();
    double dnmax = 0.0;
    for (int idx = tid; idx < 27 * 20; idx += kThreads) {
        const int g = idx / 20, n = idx % 20;
        double dx, dy, dz;
        hex20::dshape_node(n, hex20::gauss3(g / 9), hex20::gauss3((g / 3) % 3), hex20::gauss3(g % 3), dx, dy, dz);
        sm.dN[g][0][n] = dx;
        sm.dN[g][1][n] = dy;
        sm.dN[g][2][n] = dz;
        dnmax = fmax(dnmax, fmax(fabs(dx), fmax(fabs(dy), fabs(dz))));
    }
    if (kTc) atomicMax(&sm.dnmax_bits, (unsigned long long)__double_as_longlong(dnmax));
    if (tid < PS) sm.w[tid] = 0.0;
    int spare = -1;
    // node id and coordinates of the next element, loaded during the scatter
    int pre_n = 0;
    double pre_x = 0.0, pre_y = 0.0, pre_z = 0.0;
    const int i_begin = range ? range[0] : 0, i_end = range ? range[1] : m.E_count;
    if (tid < 20 && i_begin + (int)blockIdx.x < i_end) {
        pre_n = __ldg(m.conn + (size_t)__ldg(perm + i_begin + blockIdx.x) * 20 + tid);
        if (pre_n >= 0 && pre_n < m.N) {
            pre_x = __ldg(m.x + pre_n);
            pre_y = __ldg(m.y + pre_n);
            pre_z = __ldg(m.z + pre_n);
        }
    }
    __syncthreads();

    for (int i = i_begin + blockIdx.x; i < i_end; i += gridDim.x) {
        const int e = __ldg(perm + i);
        if (tid == 0) {
            sm.bad = 0;
            if (kTc) sm.tc.bound_bits = 0ull;
        }
        if (tid < kHash) sm.hkey[tid] = 0;
        __syncthreads();
        if (tid < 20) {
            const int n = pre_n;
            sm.nodes[tid] = n;
            if (n < 0 || n >= m.N) {
                sm.bad = 1;
            } else {
                sm.X[tid][0] = pre_x;
                sm.X[tid][1] = pre_y;
                sm.X[tid][2] = pre_z;
                // element-node hash (node ids of an element are distinct)
                const int key = n + 1;
                unsigned h = hash_slot(key);
                for (int i = 0; i < kHash; i++) {
                    const int old = atomicCAS(&sm.hkey[h], 0, key);
                    if (old == 0 || old == key) {
                        sm.hval[h] = tid;
                        break;
                    }
                    h = (h + 1) & (kHash - 1);
                }
            }
        }
        if (tid == 32) {
            const double E = m.E ? __ldg(m.E + e) : m.E0;
            const double nu = m.nu ? __ldg(m.nu + e) : m.nu0;
            sm.lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
            sm.mu = E / (2.0 * (1.0 + nu));
        }
        __syncthreads();
        const int i_next = i + gridDim.x;
        if (tid < 20 && i_next < i_end) pre_n = __ldg(m.conn + (size_t)__ldg(perm + i_next) * 20 + tid);
        if (sm.bad) {  // uniform: every thread reads the flag before anyone resets it
            if (tid == 0) raise_status(L.info, FEM_ERR_BAD_MESH);
            if (tid < 20 && i_next < i_end && pre_n >= 0 && pre_n < m.N) {
                pre_x = __ldg(m.x + pre_n);
                pre_y = __ldg(m.y + pre_n);
                pre_z = __ldg(m.z + pre_n);
            }
            __syncthreads();
            continue;
        }
        // Jacobians: J[g][3i+j] = sum_n dN[g][i][n] X[n][j]
        if (tid < 243) {
            const int g = tid / 9, r = tid % 9, i = r / 3, j = r % 3;
            double acc = 0.0;
#pragma unroll
            for (int n = 0; n < 20; n++) acc = fma(sm.dN[g][i][n], sm.X[n][j], acc);
            sm.J[g][r] = acc;
        }
        __syncthreads();
        if (tid < 27) {
            double* J = sm.J[tid];
            const double c0 = J[4] * J[8] - J[5] * J[7], c1 = J[5] * J[6] - J[3] * J[8], c2 = J[3] * J[7] - J[4] * J[6];
            const double det = J[0] * c0 + J[1] * c1 + J[2] * c2;
            if (!(det > 0.0)) raise_status(L.info, FEM_ERR_DETJ);
            const double r = 1.0 / det;
            double iJ[9];
            iJ[0] = c0 * r;
            iJ[1] = (J[2] * J[7] - J[1] * J[8]) * r;
            iJ[2] = (J[1] * J[5] - J[2] * J[4]) * r;
            iJ[3] = c1 * r;
            iJ[4] = (J[0] * J[8] - J[2] * J[6]) * r;
            iJ[5] = (J[2] * J[3] - J[0] * J[5]) * r;
            iJ[6] = c2 * r;
            iJ[7] = (J[1] * J[6] - J[0] * J[7]) * r;
            iJ[8] = (J[0] * J[4] - J[1] * J[3]) * r;
#pragma unroll
            for (int k = 0; k < 9; k++) J[k] = iJ[k];
            sm.w[tid] = hex20::weight3(tid / 9) * hex20::weight3((tid / 3) % 3) * hex20::weight3(tid % 3) * det;
            if (kTc)
                hex20::tc_gauss_point(sm.tc, tid, J, sm.w[tid], __longlong_as_double((long long)sm.dnmax_bits));
        }
        __syncthreads();
        // P aliases the previous element's M blocks: re-zero its padding.
        for (int idx = tid; idx < 4 * PS + 60; idx += kThreads) {
            if (idx < 4 * PS) (&sm.P[60][0])[idx] = 0.0;
            else sm.P[idx - 4 * PS][27] = 0.0;
        }
        // Physical gradients P[3n+a][g] = sum_i iJ[g][3a+i] dN[g][i][n]
        for (int idx = tid; idx < 27 * 20; idx += kThreads) {
            const int g = idx / 20, n = idx - 20 * g;
            const double* iJ = sm.J[g];
            const double d0 = sm.dN[g][0][n], d1 = sm.dN[g][1][n], d2 = sm.dN[g][2][n];
#pragma unroll
            for (int a = 0; a < 3; a++) sm.P[3 * n + a][g] = fma(iJ[3 * a], d0, fma(iJ[3 * a + 1], d1, iJ[3 * a + 2] * d2));
        }
        __syncthreads();
        if (kTc) {
            hex20::tc_prepare<kThreads>(&sm.P[0][0], PS, sm.w, sm.tc, tid);
            // P is no longer read: its storage takes M
            hex20::tc_contract<kWarps>(sm.tc, warp, lane, [&](int r, int c, double v) {
{ const int I_ = r / 3, a_ = r - 3 * I_, J_ = c / 3, b_ = c - 3 * J_;
                        if (I_ <= J_) sm.Mb[hex20::pair_index(I_, J_)][3 * a_ + b_] = v;
                        if (J_ <= I_) sm.Mb[hex20::pair_index(J_, I_)][3 * b_ + a_] = v; }
            });
        } else {
        // M = (P diag(w)) P^T on the FP64 tensor cores, upper 8x8 tiles only
        // (M is symmetric): the 36 tiles (mt <= nt) are dealt round-robin to the
        // warps, at most 4 per warp.
        double acc[4][2];
#pragma unroll
        for (int q = 0; q < 4; q++) acc[q][0] = acc[q][1] = 0.0;
        const int fr = lane >> 2, fc = lane & 3;
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int t = warp + q * kWarps;
            if (t < 36) {
                const int mt = c_tile_m[t], nt = c_tile_n[t];
#pragma unroll
                for (int ks = 0; ks < 7; ks++) {
                    const int k = 4 * ks + fc;
                    dmma_8x8x4(acc[q][0], acc[q][1], sm.w[k] * sm.P[8 * mt + fr][k], sm.P[8 * nt + fr][k]);
                }
            }
        }
        __syncthreads();  // every warp has read P: its storage now takes M
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int t = warp + q * kWarps;
            if (t < 36) {
                const int mt = c_tile_m[t], nt = c_tile_n[t];
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const int r = 8 * mt + fr, c = 8 * nt + 2 * fc + h;
                    // entry (r, c) stands for itself and, by symmetry, for (c, r);
                    // in a diagonal tile only r <= c writes (its mirror is in the tile)
                    if (r < 60 && c < 60 && (mt < nt || r <= c)) {
{ const int I_ = r / 3, a_ = r - 3 * I_, J_ = c / 3, b_ = c - 3 * J_;
                        if (I_ <= J_) sm.Mb[hex20::pair_index(I_, J_)][3 * a_ + b_] = acc[q][h];
                        if (J_ <= I_) sm.Mb[hex20::pair_index(J_, I_)][3 * b_ + a_] = acc[q][h]; }
                    }
                }
            }
        }
        }
        __syncthreads();
        // next element's coordinates: in flight during the scatter
        if (tid < 20 && i_next < i_end && pre_n >= 0 && pre_n < m.N) {
            pre_x = __ldg(m.x + pre_n);
            pre_y = __ldg(m.y + pre_n);
            pre_z = __ldg(m.z + pre_n);
        }
        // Scatter: warp w serves row nodes w and w + 10.
        if (kOut == kOutMap)
            map_rows(target, sm, e, warp, warp + kWarps < 20 ? warp + kWarps : -1, lane);
        else if (kOut == kOutColour)
            colour_rows(target, sm, warp, warp + kWarps < 20 ? warp + kWarps : -1, lane, L.info);
        else
            scatter_rows(L, sm, warp, warp + kWarps < 20 ? warp + kWarps : -1, warp, lane, spare);
        __syncthreads();
    }
}

}  // namespace

template <bool kTc, int kOut>
cudaError_t launch_scatter_hex20_t(const MeshView& m, const ListLayout& L, const int* perm, const MapTarget& t,
                                   const int* range, cudaStream_t s, int ctas_per_sm = 0) {
    static DeviceCache cache;
    const size_t smem = sizeof(Hex20Smem);
    int blocks_per_sm = 0;
    const cudaError_t err = per_device(cache, [&](int& v) {
        cudaError_t e =
            cudaFuncSetAttribute(k_scatter_hex20<kTc, kOut>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (!e) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, k_scatter_hex20<kTc, kOut>, kThreads, smem);
        return e;
    }, blocks_per_sm);
    if (err) return err;
    const int use = ctas_per_sm > 0 ? std::min(ctas_per_sm, blocks_per_sm) : blocks_per_sm;
    long long grid = (long long)use * sm_count();
    if (grid > m.E_count) grid = m.E_count > 0 ? m.E_count : 1;
    k_scatter_hex20<kTc, kOut><<<(int)grid, kThreads, smem, s>>>(m, L, perm, t, range);
    return cudaGetLastError();
}

cudaError_t launch_scatter_hex20(const MeshView& m, const ListLayout& L, int precision, const int* perm, int ctas_per_sm,
                                 cudaStream_t s) {
    const MapTarget none{};
    return precision == FEM_PREC_TC_F16X3
               ? launch_scatter_hex20_t<true, kOutLists>(m, L, perm, none, nullptr, s, ctas_per_sm)
               : launch_scatter_hex20_t<false, kOutLists>(m, L, perm, none, nullptr, s, ctas_per_sm);
}

cudaError_t launch_reassemble_hex20(const MeshView& m, int precision, const int* perm, const MapTarget& t,
                                    DevInfo* info, cudaStream_t s) {
    ListLayout L{};
    L.info = info;  // status bits (BAD_MESH, DETJ) of the element stiffness
    return precision == FEM_PREC_TC_F16X3 ? launch_scatter_hex20_t<true, kOutMap>(m, L, perm, t, nullptr, s)
                                          : launch_scatter_hex20_t<false, kOutMap>(m, L, perm, t, nullptr, s);
}

cudaError_t launch_colour_hex20(const MeshView& m, const int* perm, const int* range, const MapTarget& t,
                                DevInfo* info, cudaStream_t s) {
    ListLayout L{};
    L.info = info;
    return launch_scatter_hex20_t<false, kOutColour>(m, L, perm, t, range, s);
}

}  // namespace fem
