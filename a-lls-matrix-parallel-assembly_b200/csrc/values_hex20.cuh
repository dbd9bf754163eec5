// Device code of the CTA-cooperative Hex20 FP64 element pass: the value-only
// re-assembly and the colouring baseline (values_hex20.cu), and the value
// items of the batched persistent kernel (batched.cu). See values_hex20.cu for
// the method.
#pragma once

#include "group_hex20.cuh"
#include "hex20.cuh"

namespace fem {
namespace {

constexpr int kValueWarps = 6;  // warps that hold M tiles (one tile position each)
constexpr int KS = 28;  // Gauss points padded to 7 k-steps of 4; row stride of the tables (doubles)

// Where the value pass puts an element's Ke blocks.
enum ValueOut : int {
    kToSlots = 0,   // FP64 atomics into the list slots of a group's map record (both orientations)
    kToCsrMap = 1,  // FP64 atomics into a CSR at the positions of a scatter map (both triangles)
    kToCsrColour = 2  // plain adds into a CSR at binary-searched positions (one colour: no two
                      // elements share a node)
};

struct ValuesTarget {
    const int* map;          // kToCsrMap: CSR positions, row e
    const GroupTopo* topo;   // kToSlots: topology of the group of the elements
    const unsigned* rec;     // kToSlots: the slot words of the group's record
    long long g0;            // kToSlots: position of the group's first element
    double* vals;            // kToSlots: list values
    const int* row_ptr;   // kToCsr*: the CSR
    const int* col_idx;
    double* csr;
    DevInfo* info;        // status bits
};

// The six 8x8 tile positions (ti <= tj) of the upper triangle of the 24 x 24 node grid.
__device__ __forceinline__ int tile_ti(int w) { return w < 3 ? 0 : (w < 5 ? 1 : 2); }
__device__ __forceinline__ int tile_tj(int w) { return w == 0 ? 0 : (w == 1 || w == 3 ? 1 : 2); }

struct ValuesSmem {
    double dN[3][20][KS];  // dN_n / dxi_i at Gauss point g: [i][n][g]
    double G[3][24][KS];   // physical gradients: [a][n][g]; rows 20..23 and g = 27 stay zero
    double X[20][3];
    double J[27][9];       // Jacobians, then their inverses
    double w[KS];          // gauss weight * detJ (w[27] = 0)
    int nodes[20];
    double lam, mu;
    int bad;
    // per tile warp: its node-pair blocks, compacted, before they are added
    double stage[kValueWarps][64][9];
    int stage_gid[kValueWarps][64];
};

__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(c0), "+d"(c1)
                 : "d"(a), "d"(b));
}

// Shape-function derivative table and the zero padding of G and w; every
// thread of the CTA calls it once, before values_cta.
__device__ __forceinline__ void values_init(ValuesSmem& sm) {
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int idx = tid; idx < 27 * 20; idx += nt) {
        const int g = idx / 20, n = idx - 20 * g;
        double dx, dy, dz;
        hex20::dshape_node(n, hex20::gauss3(g / 9), hex20::gauss3((g / 3) % 3), hex20::gauss3(g % 3), dx, dy, dz);
        sm.dN[0][n][g] = dx;
        sm.dN[1][n][g] = dy;
        sm.dN[2][n][g] = dz;
    }
    for (int idx = tid; idx < 3 * 24 * KS; idx += nt) (&sm.G[0][0][0])[idx] = 0.0;
    for (int idx = tid; idx < 3 * 20; idx += nt) sm.dN[idx / 20][idx % 20][27] = 0.0;
    if (tid < KS) sm.w[tid] = 0.0;
    __syncthreads();
}

// The value pass of the elements at positions i = i_first, i_first +
// i_stride, ... below i1 of the visit order perm (perm NULL: element i) by
// one CTA of at least kValueWarps warps (warps beyond them help with the
// per-element tables only); the slot ids of position i are map row
// i - map_origin. Every thread of the CTA calls it.
template <int kOut>
__device__ __forceinline__ void values_cta(const MeshView& m, const int* __restrict__ perm, long long i_first,
                                           long long i_stride, int i1, const ValuesTarget& t, ValuesSmem& sm) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nt = blockDim.x;
    const bool tile_warp = warp < kValueWarps;
    const int ti = tile_ti(warp), tj = tile_tj(warp);
    const int fr = lane >> 2, fc = lane & 3;
    auto elem = [&](long long i) -> int { return perm ? FEM_LDG(perm + i) : (int)i; };
    // node id and coordinates of the next element
    int pre_n = 0;
    double pre_x = 0.0, pre_y = 0.0, pre_z = 0.0;
    if (tid < 20 && i_first < i1) {
        pre_n = FEM_LDG(m.conn + (size_t)elem(i_first) * 20 + tid);
        if (pre_n >= 0 && pre_n < m.N) {
            pre_x = FEM_LDG(m.x + pre_n);
            pre_y = FEM_LDG(m.y + pre_n);
            pre_z = FEM_LDG(m.z + pre_n);
        }
    }
    __syncthreads();

    for (long long i = i_first; i < i1; i += i_stride) {
        const int e = elem(i);
        if (tid == 0) sm.bad = 0;
        __syncthreads();  // the previous element's G, w, lam/mu and flag are no longer read
        if (tid < 20) {
            sm.nodes[tid] = pre_n;
            if (pre_n < 0 || pre_n >= m.N) {
                sm.bad = 1;
            } else {
                sm.X[tid][0] = pre_x;
                sm.X[tid][1] = pre_y;
                sm.X[tid][2] = pre_z;
            }
        }
        if (tid == 32) {
            const double E = m.E ? FEM_LDG(m.E + e) : m.E0;
            const double nu = m.nu ? FEM_LDG(m.nu + e) : m.nu0;
            sm.lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
            sm.mu = E / (2.0 * (1.0 + nu));
        }
        __syncthreads();
        const long long i_next = i + i_stride;
        if (tid < 20 && i_next < i1) pre_n = FEM_LDG(m.conn + (size_t)elem(i_next) * 20 + tid);
        if (sm.bad) {  // nothing to add
            if (tid == 0 && kOut != kToSlots) raise_status(t.info, FEM_ERR_BAD_MESH);  // else the claim pass did
            if (tid < 20 && i_next < i1 && pre_n >= 0 && pre_n < m.N) {
                pre_x = FEM_LDG(m.x + pre_n);
                pre_y = FEM_LDG(m.y + pre_n);
                pre_z = FEM_LDG(m.z + pre_n);
            }
            __syncthreads();  // uniform: every thread has read the flag before it is reset
            continue;
        }
        // Jacobians J[g][3i + j] = sum_n dN[i][n][g] X[n][j]
        for (int idx = tid; idx < 243; idx += nt) {
            const int g = idx % 27, r = idx / 27, ii = r / 3, jj = r % 3;
            double acc = 0.0;
#pragma unroll
            for (int n = 0; n < 20; n++) acc = fma(sm.dN[ii][n][g], sm.X[n][jj], acc);
            sm.J[g][r] = acc;
        }
        __syncthreads();
        if (tid < 27) {
            double* J = sm.J[tid];
            const double c0 = J[4] * J[8] - J[5] * J[7], c1 = J[5] * J[6] - J[3] * J[8], c2 = J[3] * J[7] - J[4] * J[6];
            const double det = J[0] * c0 + J[1] * c1 + J[2] * c2;
            if (!(det > 0.0)) raise_status(t.info, FEM_ERR_DETJ);
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
        }
        __syncthreads();
        // physical gradients G[a][n][g] = sum_i iJ[g][3a + i] dN[i][n][g]
        for (int idx = tid; idx < 20 * 27; idx += nt) {
            const int n = idx / 27, g = idx - 27 * n;
            const double* iJ = sm.J[g];
            const double d0 = sm.dN[0][n][g], d1 = sm.dN[1][n][g], d2 = sm.dN[2][n][g];
#pragma unroll
            for (int a = 0; a < 3; a++) sm.G[a][n][g] = fma(iJ[3 * a], d0, fma(iJ[3 * a + 1], d1, iJ[3 * a + 2] * d2));
        }
        __syncthreads();
        // the coordinates of the next element arrive during the contraction
        if (tid < 20 && i_next < i1 && pre_n >= 0 && pre_n < m.N) {
            pre_x = FEM_LDG(m.x + pre_n);
            pre_y = FEM_LDG(m.y + pre_n);
            pre_z = FEM_LDG(m.z + pre_n);
        }
        if (!tile_warp) continue;  // the remaining warps wait at the next element's first barrier
        // M^{ab} tiles (ti, tj): A[r][k] = w_k G[a][8 ti + r][k], B[k][c] = G[b][8 tj + c][k]
        double acc[3][3][2];
#pragma unroll
        for (int a = 0; a < 3; a++)
#pragma unroll
            for (int b = 0; b < 3; b++) acc[a][b][0] = acc[a][b][1] = 0.0;
#pragma unroll
        for (int ks = 0; ks < 7; ks++) {
            const int k = 4 * ks + fc;
            const double wk = sm.w[k];
            double A[3], B[3];
#pragma unroll
            for (int a = 0; a < 3; a++) {
                A[a] = wk * sm.G[a][8 * ti + fr][k];
                B[a] = sm.G[a][8 * tj + fr][k];
            }
#pragma unroll
            for (int a = 0; a < 3; a++)
#pragma unroll
                for (int b = 0; b < 3; b++) dmma(acc[a][b][0], acc[a][b][1], A[a], B[b]);
        }
        const double lam = sm.lam, mu = sm.mu;
        const int I = 8 * ti + fr;
        if constexpr (kOut == kToSlots) {
            // Ke block of each of this lane's node pairs {I, J}, staged for two
            // atomic passes: Ke_IJ to the slot of (row node I, column node J),
            // then its transpose to the slot of (row J, column I), the slots
            // from the group's map record
            const GroupTopo& T = *t.topo;
            const int w = (int)(i - t.g0);
            unsigned tgt[2][2];
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int Jn = 8 * tj + 2 * fc + h;
                tgt[h][0] = tgt[h][1] = kMapNone;
                if (I < 20 && Jn < 20 && (ti != tj || Jn >= I)) {
                    const int u = T.lidx[20 * w + I], v = T.lidx[20 * w + Jn];
                    if (u <= v) {
                        const int p = pair_index(T, u, v);
                        tgt[h][0] = FEM_LDG(t.rec + 2 * p);
                        // a repeated node of one element: both orientations on one block
                        tgt[h][1] = u == v ? (I != Jn ? tgt[h][0] : kMapNone) : FEM_LDG(t.rec + 2 * p + 1);
                    } else {
                        const int p = pair_index(T, v, u);
                        tgt[h][0] = FEM_LDG(t.rec + 2 * p + 1);
                        tgt[h][1] = FEM_LDG(t.rec + 2 * p);
                    }
                }
            }
#pragma unroll
            for (int o = 0; o < 2; o++) {
                int base = 0;
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const unsigned g = tgt[h][o];
                    const bool ok = map_has_slot(g);
                    const unsigned have = __ballot_sync(0xFFFFFFFFu, ok);
                    if (ok) {
                        const int slot = base + __popc(have & ((1u << lane) - 1u));
                        const double mtr = mu * (acc[0][0][h] + acc[1][1][h] + acc[2][2][h]);
#pragma unroll
                        for (int a = 0; a < 3; a++)
#pragma unroll
                            for (int b = 0; b < 3; b++) {
                                const double k = fma(lam, acc[a][b][h], fma(mu, acc[b][a][h], a == b ? mtr : 0.0));
                                sm.stage[warp][slot][o ? 3 * b + a : 3 * a + b] = k;
                            }
                        sm.stage_gid[warp][slot] = (int)(g & ~kPairShared);
                    }
                    base += __popc(have);
                }
                __syncwarp();
                // nine consecutive lanes per block, three blocks per instruction:
                // each block's 72 bytes are one atomic pass over its three sectors
                if (lane < 27) {
                    const int q = lane / 9, v = lane - 9 * q;
                    for (int blk = q; blk < base; blk += 3)
                        atomicAdd(t.vals + (size_t)(unsigned)sm.stage_gid[warp][blk] * 9 + v, sm.stage[warp][blk][v]);
                }
                __syncwarp();
            }
        } else {
            // CSR targets hold both triangles: Ke_IJ at block (I, J) and its
            // transpose at (J, I)
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int Jn = 8 * tj + 2 * fc + h;
                if (I >= 20 || Jn >= 20 || (ti == tj && Jn < I)) continue;
                const double mtr = mu * (acc[0][0][h] + acc[1][1][h] + acc[2][2][h]);
                double k[3][3];
#pragma unroll
                for (int a = 0; a < 3; a++)
#pragma unroll
                    for (int b = 0; b < 3; b++) k[a][b] = fma(lam, acc[a][b][h], fma(mu, acc[b][a][h], a == b ? mtr : 0.0));
                for (int o = 0; o < (I == Jn ? 1 : 2); o++) {
                    const int R = o ? Jn : I, Cn = o ? I : Jn;  // block (R, Cn) of the element
                    const int r0 = 3 * sm.nodes[R], c0 = 3 * sm.nodes[Cn];
                    const int lo = FEM_LDG(t.row_ptr + r0), len = FEM_LDG(t.row_ptr + r0 + 1) - lo;
                    int p = -1;
                    if constexpr (kOut == kToCsrMap) {
                        p = FEM_LDG(t.map + (size_t)e * 400 + R * 20 + Cn);
                    } else {
                        int a0 = lo, a1 = lo + len - 1;
                        while (a0 <= a1) {
                            const int mid = (a0 + a1) >> 1;
                            const int c = FEM_LDG(t.col_idx + mid);
                            if (c == c0) {
                                p = mid;
                                break;
                            }
                            if (c < c0) a0 = mid + 1;
                            else a1 = mid - 1;
                        }
                        if (p < 0) raise_status(t.info, FEM_ERR_INTERNAL);  // the pattern lacks the block
                    }
                    if (p < 0) continue;
#pragma unroll
                    for (int a = 0; a < 3; a++)
#pragma unroll
                        for (int b = 0; b < 3; b++) {
                            const double v = o ? k[b][a] : k[a][b];
                            double* d = t.csr + p + (size_t)a * len + b;
                            if constexpr (kOut == kToCsrMap) atomicAdd(d, v);
                            else *d += v;
                        }
                }
            }
        }
    }
}

}  // namespace
}  // namespace fem
