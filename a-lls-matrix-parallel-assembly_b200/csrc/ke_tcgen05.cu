// Element stiffness of Hex20 elements with the node-pair contraction on the
// 5th-generation tensor cores (tcgen05, accumulators in tensor memory): the
// FEM_PREC_TC_F16X3 form of fem_element_stiffness.
//
// Same arithmetic as the split-precision form of hex20.cuh: with the physical
// gradients P (60 x 27), w_g = weight * detJ_g and a per-element power of two
// s (from a bound on |P| sqrt|w|), A = s P sqrt|w| is rounded to FP32 and
// split into two FP16 parts A = A_hi + A_lo, and
//     M = A diag(sgn w) A^T / s^2 ~ (A_lo B_hi^T + A_hi B_lo^T + A_hi B_hi^T) / s^2
// with B = A diag(sgn w) (B = A unless some w_g < 0), summed in FP32 on the
// tensor cores. Jacobians, their inverses and determinants stay FP64; the Ke
// block formula is applied in FP32 to the FP32 products and the output is FP64. It replaces the reference's per-thread
// FP32 computeElementStiffnessHex20 (ALLS_Hex20_3D_Assembly_Performance.cu:130-195).
//
// One 4-warp CTA takes two elements at a time (persistent over element pairs):
//   rows 0..63 of the 128-row operands are element 0's dofs, rows 64..127
//   element 1's; inside an element, dof (node n, direction a) is row
//   32 (n / 10) + 3 (n % 10) + a, so each warp of the epilogue holds whole
//   node triples (rows 30, 31, 62, 63 are zero). K = 27 Gauss points padded
//   to 32. One elected thread issues six tcgen05.mma (M = 128, N = 128,
//   K = 16; FP16 inputs, FP32 accumulation) from shared-memory descriptors
//   (K-major, no swizzle: 8-row x 16-byte core matrices) into 128 columns of
//   tensor memory and commits them to an mbarrier. The two diagonal 64 x 64
//   blocks of the 128 x 128 product are the two elements' M (the off-diagonal
//   blocks are not read).
//   Epilogue: warp w reads its 32 lanes of tensor memory (tcgen05.ld, one row
//   of M per thread); the transposed entries and traces of the 3x3 blocks
//   come from the two other lanes of the node by shuffles, and each thread
//   writes its rows of the upper Ke blocks into shared memory, which one bulk
//   copy (cp.async.bulk) moves to the output.
//   The waits on the mbarrier are bounded (FEM_ERR_TIMEOUT, then the kernel
//   releases its tensor memory and returns).
#include <algorithm>
#include <cstdint>

#include <cuda_fp16.h>

#include "hex20.cuh"

namespace fem {
namespace {

using namespace hex20;

constexpr int kThreads = 128;
constexpr uint32_t kTmemCols = 128;
constexpr int kRows = 128;              // operand rows: two elements x 64
constexpr uint32_t kLBO = 128;          // bytes between the two 8-element K chunks of one MMA
constexpr uint32_t kSBO = 512;          // bytes between 8-row groups (4 K chunks of 128 B)
constexpr long long kDefaultWaitNs = 200ll * 1000 * 1000;  // the second, recovering wait of a timed-out CTA

// Instruction descriptor of tcgen05.mma kind::f16: FP32 accumulator (bits
// 4-5 = 1), FP16 A and B (bits 7-12 = 0), both K-major (bits 15, 16 = 0),
// N >> 3 in bits 17-22, M >> 4 in bits 24-28.
constexpr uint32_t kIdesc = (1u << 4) | ((128u >> 3) << 17) | ((128u >> 4) << 24);

struct KeTcSmem {
    union {
        // A_hi, A_lo, B_hi, B_lo: 16-byte core-matrix rows, index (row / 8) * 32 + chunk * 8 + row % 8
        uint4 op[4][kRows * 4];
        double ke[2][kPackedHex20];  // the pair's packed Ke, staged for the bulk copy
    };
    double dNt[20][27][4];  // dN_n / dxi_i at Gauss point g (i = 3: padding for 16-byte loads)
    double X[2][20][3];
    double iJ[2][27][12];   // Jacobian (row-major 3x3), then sqrt|w_g| times its inverse, row a at [4a, 4a + 3)
    double lam[2], mu[2];
    unsigned long long bound_bits[2];  // bound on s-free |P| sqrt|w| (bits of a positive double)
    unsigned long long dnmax_bits;
    unsigned long long mbar;
    unsigned negmask[2];    // Gauss points with w_g < 0
    unsigned tmem_base;
    int state[2];           // 0 element present, 1 bad node id, 2 no element (odd tail)
    int nodes[2][20];       // node ids of the pair (the value pass orients each block by them)
};
// more than 44.6 KB: at most four CTAs (4 x 128 tensor-memory columns) per SM
static_assert(sizeof(KeTcSmem) > 46 * 1024 && sizeof(KeTcSmem) < 56 * 1024, "four CTAs per SM");
static_assert(sizeof(double) * 2 * kPackedHex20 <= sizeof(uint4) * 4 * kRows * 4, "staging fits the operands");

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor: start address >> 4 (bits 0-13), leading
// (K) byte offset >> 4 (bits 16-29), stride (8-row group) byte offset >> 4
// (bits 32-45), descriptor version 1 (bits 46-47), no swizzle (bits 61-63 = 0).
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr) {
    return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)(kLBO >> 4) << 16) | ((uint64_t)(kSBO >> 4) << 32) |
           (1ull << 46);
}

__device__ __forceinline__ void mma_f16(uint32_t tmem, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        :
        : "r"(tmem), "l"(adesc), "l"(bdesc), "r"(kIdesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ long long global_ns() {
    long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Wait for the completion of the mbarrier phase of this parity, for at most
// limit_ns nanoseconds of the GPU's global timer; limit_ns < 0: no wait at
// all (the wait counts as run out).
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity, long long limit_ns) {
    if (limit_ns < 0) return false;
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = global_ns();
    while (!mbar_try_wait(bar, parity))
        if (global_ns() - t0 > limit_ns) return false;
    return true;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void tmem_load64(uint32_t taddr, uint32_t (&r)[64]) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x64.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, %32, %33, %34, %35, %36, %37, %38, %39, %40, %41, %42, %43, %44, %45, %46, %47, %48, %49, %50, %51, %52, %53, %54, %55, %56, %57, %58, %59, %60, %61, %62, %63}, [%64];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31]), "=r"(r[32]), "=r"(r[33]), "=r"(r[34]), "=r"(r[35]), "=r"(r[36]), "=r"(r[37]), "=r"(r[38]), "=r"(r[39]), "=r"(r[40]), "=r"(r[41]), "=r"(r[42]), "=r"(r[43]), "=r"(r[44]), "=r"(r[45]), "=r"(r[46]), "=r"(r[47]), "=r"(r[48]), "=r"(r[49]), "=r"(r[50]), "=r"(r[51]), "=r"(r[52]), "=r"(r[53]), "=r"(r[54]), "=r"(r[55]), "=r"(r[56]), "=r"(r[57]), "=r"(r[58]), "=r"(r[59]), "=r"(r[60]), "=r"(r[61]), "=r"(r[62]), "=r"(r[63])
                 : "r"(taddr));
}

__device__ __forceinline__ void tmem_wait_load() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ unsigned pack_half2(__half lo, __half hi) {
    return (unsigned)__half_as_ushort(lo) | ((unsigned)__half_as_ushort(hi) << 16);
}

// Outputs of the kernel.
enum TcOut : int {
    kTcPacked = 0,  // the packed Ke of every element to ke_out (fem_element_stiffness)
    kTcWave = 1,    // the packed Ke of a wave's elements perm[i0, i1) to ke_out, row q - i0 for
                    // position q (staging of the group value pass, values_hex20.cu)
    kTcCsrMap = 2   // value-only re-assembly: Ke_IJ and its transpose added with FP64 atomics at
                    // their CSR positions (scatter map, row e)
};

// Elements and targets of the kTcWave / kTcCsrMap modes.
struct SlotTarget {
    const int* perm;     // visit order: positions [i0, i1) (kTcWave), all elements (kTcCsrMap)
    const int* map;      // scatter map, row e (kTcCsrMap)
    const int* row_ptr;  // the CSR (kTcCsrMap)
    double* csr;
    int i0, i1;
    long long wait_ns;   // bound on the wait for the products (every mode)
};

template <int kMode>
__global__ void __launch_bounds__(kThreads, 4) k_hex20_ke_tc(MeshView m, double* __restrict__ ke_out,
                                                             int* __restrict__ status, int bulk_out, SlotTarget tgt) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    KeTcSmem& sm = *reinterpret_cast<KeTcSmem*>(smem_raw);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr bool kWave = kMode == kTcWave, kMap = kMode == kTcCsrMap;
    // elements: positions q of the wave (kTcWave), of perm (kTcCsrMap) or the mesh's elements q
    const long long count = kWave ? (long long)(tgt.i1 - tgt.i0) : (long long)m.E_count;
    const long long npairs = (count + 1) / 2;
    auto elem = [&](long long q) -> long long {
        return kWave ? (long long)__ldg(tgt.perm + tgt.i0 + q) : (kMap ? (long long)__ldg(tgt.perm + q) : q);
    };
    const uint32_t bar = smem_u32(&sm.mbar);

    if (tid == 0) {
        sm.dnmax_bits = 0ull;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&sm.tmem_base)),
                     "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    __syncthreads();
    double dnmax = 0.0;
    for (int idx = tid; idx < 27 * 20; idx += kThreads) {
        const int g = idx / 20, n = idx % 20;
        double d0, d1, d2;
        dshape_node(n, gauss3(g / 9), gauss3((g / 3) % 3), gauss3(g % 3), d0, d1, d2);
        sm.dNt[n][g][0] = d0;
        sm.dNt[n][g][1] = d1;
        sm.dNt[n][g][2] = d2;
        dnmax = fmax(dnmax, fmax(fabs(d0), fmax(fabs(d1), fabs(d2))));
    }
    atomicMax(&sm.dnmax_bits, (unsigned long long)__double_as_longlong(dnmax));
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = sm.tmem_base;
    const double dnm = __longlong_as_double((long long)sm.dnmax_bits);

    // node ids and coordinates of the next pair, loaded a step ahead
    // (threads 0..39: element tid / 20, node tid % 20)
    int pre_state = 2, pre_n = 0;
    double pre_x = 0.0, pre_y = 0.0, pre_z = 0.0;
    auto prefetch = [&](long long p) {
        if (tid >= 40) return;
        const long long q = 2 * p + tid / 20;
        pre_state = 2;
        if (p < npairs && q < count) {
            const long long e = elem(q);
            pre_n = __ldg(m.conn + (size_t)e * 20 + tid % 20);
            pre_state = (pre_n >= 0 && pre_n < m.N) ? 0 : 1;
            if (pre_state == 0) {
                pre_x = __ldg(m.x + pre_n);
                pre_y = __ldg(m.y + pre_n);
                pre_z = __ldg(m.z + pre_n);
            }
        }
    };
    prefetch(blockIdx.x);

    uint32_t parity = 0;
    bool timed_out = false;
    // per-pair flags and bounds, reset again after each pair's last reader
    // (state in step 4, bounds and signs in step 7)
    if (tid < 2) {
        sm.state[tid] = 0;
        sm.bound_bits[tid] = 0ull;
        sm.negmask[tid] = 0u;
    }
    __syncthreads();
    for (long long p = blockIdx.x; p < npairs; p += gridDim.x) {
        // 1. the pair's nodes and materials
        if (tid < 40) {
            const int e = tid / 20, k = tid % 20;
            sm.nodes[e][k] = pre_state == 0 ? pre_n : 0;
            sm.X[e][k][0] = pre_state == 0 ? pre_x : 0.0;
            sm.X[e][k][1] = pre_state == 0 ? pre_y : 0.0;
            sm.X[e][k][2] = pre_state == 0 ? pre_z : 0.0;
            if (pre_state) atomicMax(&sm.state[e], pre_state);
            if (pre_state == 1) atomicOr(status, 1 << FEM_ERR_BAD_MESH);
        } else if (tid < 42) {
            const long long q = 2 * p + (tid - 40);
            const long long e = q < count ? elem(q) : 0;
            const double E = q < count ? (m.E ? __ldg(m.E + e) : m.E0) : 0.0;
            const double nu = q < count ? (m.nu ? __ldg(m.nu + e) : m.nu0) : 0.0;
            sm.lam[tid - 40] = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
            sm.mu[tid - 40] = E / (2.0 * (1.0 + nu));
        }
        __syncthreads();
        prefetch(p + gridDim.x);
        // 2. Jacobians: J[e][g][3i + j] = sum_n dN[g][i][n] X[e][n][j]
        for (int it = tid; it < 2 * 81; it += kThreads) {
            const int e = it / 81, r = it - 81 * e, g = r / 3, i = r - 3 * g;
            double j0 = 0.0, j1 = 0.0, j2 = 0.0;
#pragma unroll
            for (int n = 0; n < 20; n++) {
                const double d = sm.dNt[n][g][i];
                j0 = fma(d, sm.X[e][n][0], j0);
                j1 = fma(d, sm.X[e][n][1], j1);
                j2 = fma(d, sm.X[e][n][2], j2);
            }
            sm.iJ[e][g][3 * i] = j0;
            sm.iJ[e][g][3 * i + 1] = j1;
            sm.iJ[e][g][3 * i + 2] = j2;
        }
        __syncthreads();
        // 3. determinants, inverses, weights and the scale bound
        if (tid < 54) {
            const int e = tid / 27, g = tid - 27 * e;
            double* Jg = sm.iJ[e][g];
            double J[9], iJ[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, w = 0.0;
#pragma unroll
            for (int k = 0; k < 9; k++) J[k] = Jg[k];
            if (sm.state[e] == 0) {
                const double c0 = J[4] * J[8] - J[5] * J[7], c1 = J[5] * J[6] - J[3] * J[8],
                             c2 = J[3] * J[7] - J[4] * J[6];
                const double det = J[0] * c0 + J[1] * c1 + J[2] * c2;
                if (!(det > 0.0)) atomicOr(status, 1 << FEM_ERR_DETJ);
                const double r = 1.0 / det;
                iJ[0] = c0 * r;
                iJ[1] = (J[2] * J[7] - J[1] * J[8]) * r;
                iJ[2] = (J[1] * J[5] - J[2] * J[4]) * r;
                iJ[3] = c1 * r;
                iJ[4] = (J[0] * J[8] - J[2] * J[6]) * r;
                iJ[5] = (J[2] * J[3] - J[0] * J[5]) * r;
                iJ[6] = c2 * r;
                iJ[7] = (J[1] * J[6] - J[0] * J[7]) * r;
                iJ[8] = (J[0] * J[4] - J[1] * J[3]) * r;
                w = weight3(g / 9) * weight3((g / 3) % 3) * weight3(g % 3) * det;
            }
            const double sq = sqrt(fabs(w));
#pragma unroll
            for (int a = 0; a < 3; a++) {
                Jg[4 * a] = iJ[3 * a] * sq;
                Jg[4 * a + 1] = iJ[3 * a + 1] * sq;
                Jg[4 * a + 2] = iJ[3 * a + 2] * sq;
            }
            double rn = 0.0;
#pragma unroll
            for (int a = 0; a < 3; a++) rn = fmax(rn, fabs(iJ[3 * a]) + fabs(iJ[3 * a + 1]) + fabs(iJ[3 * a + 2]));
            const double b = sq * rn * dnm;
            if (b > 0.0) atomicMax(&sm.bound_bits[e], (unsigned long long)__double_as_longlong(b));
            if (w < 0.0) atomicOr(&sm.negmask[e], 1u << g);
        }
        // the previous pair's bulk copy has read its staging (the operands' storage)
        if (tid == 0 && bulk_out) asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
        __syncthreads();
        // 4. operands: thread t writes row t of A (and of B when a weight is negative)
        if (tid < 2) sm.state[tid] = 0;  // last read in step 3; next written in step 1
        const bool signed_b = (sm.negmask[0] | sm.negmask[1]) != 0u;
        {
            const int e = tid >> 6, i = tid & 63, l = i & 31;
            const bool real = l < 30;
            const int n = 10 * (i >> 5) + (real ? l / 3 : 0), a = real ? l % 3 : 0;
            const double bound = __longlong_as_double((long long)sm.bound_bits[e]);
            int ex = 0;
            if (bound > 0.0) frexp(bound, &ex);  // bound = f 2^ex, f in [0.5, 1)
            const double s = ldexp(1.0, -ex);
            const unsigned neg = sm.negmask[e];
#pragma unroll
            for (int kc = 0; kc < 4; kc++) {
                unsigned hw[4], lw[4], hb[4], lb[4];
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    float v[2];
#pragma unroll
                    for (int h = 0; h < 2; h++) {
                        const int g = 8 * kc + 2 * q + h;
                        v[h] = 0.0f;
                        if (g < 27 && real) {
                            // sqrt|w_g| P[(n,a)][g] = (sqrt|w_g| iJ_g row a) . dN_g[.][n]
                            const double2 j01 = *reinterpret_cast<const double2*>(&sm.iJ[e][g][4 * a]);
                            const double2 d01 = *reinterpret_cast<const double2*>(&sm.dNt[n][g][0]);
                            const double P = fma(j01.x, d01.x, fma(j01.y, d01.y, sm.iJ[e][g][4 * a + 2] * sm.dNt[n][g][2]));
                            v[h] = (float)(s * P);
                        }
                    }
                    const __half2 hi = __float22half2_rn(make_float2(v[0], v[1]));
                    const float2 hf = __half22float2(hi);
                    const __half2 lo = __float22half2_rn(make_float2(v[0] - hf.x, v[1] - hf.y));  // exact differences
                    hw[q] = pack_half2(__low2half(hi), __high2half(hi));
                    lw[q] = pack_half2(__low2half(lo), __high2half(lo));
                    // B = A diag(sgn w): flip the sign bits of the negative-weight points
                    const int g0 = 8 * kc + 2 * q;
                    const unsigned flip = ((neg >> g0) & 1u ? 0x8000u : 0u) | ((neg >> (g0 + 1)) & 1u ? 0x80000000u : 0u);
                    hb[q] = hw[q] ^ flip;
                    lb[q] = lw[q] ^ flip;
                }
                const int idx = (tid >> 3) * 32 + kc * 8 + (tid & 7);
                sm.op[0][idx] = make_uint4(hw[0], hw[1], hw[2], hw[3]);
                sm.op[1][idx] = make_uint4(lw[0], lw[1], lw[2], lw[3]);
                if (signed_b) {
                    sm.op[2][idx] = make_uint4(hb[0], hb[1], hb[2], hb[3]);
                    sm.op[3][idx] = make_uint4(lb[0], lb[1], lb[2], lb[3]);
                }
            }
        }
        fence_async_smem();  // the operands are read by the tensor cores (async proxy)
        tc_fence_before();
        __syncthreads();
        // 5. six MMAs (lo x hi, hi x lo, hi x hi; two K steps each), one commit
        if (tid == 0) {
            tc_fence_after();
            const uint32_t a_hi = smem_u32(sm.op[0]), a_lo = smem_u32(sm.op[1]);
            const uint32_t b_hi = signed_b ? smem_u32(sm.op[2]) : a_hi, b_lo = signed_b ? smem_u32(sm.op[3]) : a_lo;
#pragma unroll
            for (int k = 0; k < 2; k++) mma_f16(tmem, smem_desc(a_lo + 256u * k), smem_desc(b_hi + 256u * k), k);
#pragma unroll
            for (int k = 0; k < 2; k++) mma_f16(tmem, smem_desc(a_hi + 256u * k), smem_desc(b_lo + 256u * k), 1u);
#pragma unroll
            for (int k = 0; k < 2; k++) mma_f16(tmem, smem_desc(a_hi + 256u * k), smem_desc(b_hi + 256u * k), 1u);
            mma_commit(bar);
        }
        const bool done = mbar_wait_bounded(bar, parity, tgt.wait_ns);
        parity ^= 1u;
        if (__syncthreads_or(!done)) {
            if (tid == 0) atomicOr(status, 1 << FEM_ERR_TIMEOUT);
            timed_out = true;
            break;
        }
        tc_fence_after();
        // 6. epilogue: thread = row (node I, direction a) of element e
        {
            const int e = warp >> 1;
            uint32_t r[64];
            tmem_load64(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(64 * e), r);
            tmem_wait_load();
            const bool real = lane < 30;
            const int I = 10 * (warp & 1) + (real ? lane / 3 : 0), a = real ? lane % 3 : 0;
            const int base = 3 * (lane / 3);
            const int src1 = base + (a + 1) % 3, src2 = base + (a + 2) % 3;
            const double bound = __longlong_as_double((long long)sm.bound_bits[e]);
            int ex = 0;
            if (bound > 0.0) frexp(bound, &ex);
            const double inv_s2 = ldexp(1.0, 2 * ex);
            const float lam = (float)sm.lam[e], mu = (float)sm.mu[e];
            double* out = sm.ke[e] + 9 * (I * 20 - I * (I - 1) / 2 - I) + 3 * a;  // + 9 J: block (I, J)
            const long long q = 2 * p + e;  // the element's position in the wave / in perm
            const long long eid = (kMap && q < count) ? elem(q) : 0;
            const int* mrow = tgt.map + (size_t)eid * 400;
            // elements with a bad node id have no map entries (-1): nothing is added
            const bool add = kMap && real && q < count;
#pragma unroll
            for (int J = 0; J < 20; J++) {
                const int c = 32 * (J / 10) + 3 * (J % 10);
                const float o0 = __uint_as_float(r[c]), o1 = __uint_as_float(r[c + 1]), o2 = __uint_as_float(r[c + 2]);
                const float dg = a == 0 ? o0 : (a == 1 ? o1 : o2);        // M[(I,a),(J,a)]
                // the lane of direction a_s sends M[(I,a_s),(J,a_s+2)] and M[(I,a_s),(J,a_s+1)]
                const float send1 = a == 0 ? o2 : (a == 1 ? o0 : o1);
                const float send2 = a == 0 ? o1 : (a == 1 ? o2 : o0);
                const float t1 = __shfl_sync(0xFFFFFFFFu, send1, src1);  // M[(I,a+1),(J,a)]
                const float t2 = __shfl_sync(0xFFFFFFFFu, send2, src2);  // M[(I,a+2),(J,a)]
                const float d1 = __shfl_sync(0xFFFFFFFFu, dg, src1), d2 = __shfl_sync(0xFFFFFFFFu, dg, src2);
                const float mtr = mu * (dg + d1 + d2);
                // M[(I,b),(J,a)] for b = 0, 1, 2
                const float T0 = a == 0 ? dg : (a == 1 ? t2 : t1);
                const float T1 = a == 0 ? t1 : (a == 1 ? dg : t2);
                const float T2 = a == 0 ? t2 : (a == 1 ? t1 : dg);
                // Ke_IJ[a][b] = lam M[(I,a),(J,b)] + mu M[(I,b),(J,a)] + mu delta_ab tr(M_IJ), FP32 on the
                // FP32 products, then scaled back by 1 / s^2 in FP64
                const float k0 = fmaf(lam, o0, fmaf(mu, T0, a == 0 ? mtr : 0.0f));
                const float k1 = fmaf(lam, o1, fmaf(mu, T1, a == 1 ? mtr : 0.0f));
                const float k2 = fmaf(lam, o2, fmaf(mu, T2, a == 2 ? mtr : 0.0f));
                if (kMap) {
                    // the CSR holds both triangles: row a of Ke_IJ at block (I, J),
                    // and, transposed, column a of block (J, I)
                    if (add && J >= I) {
                        const double v0 = (double)k0 * inv_s2, v1 = (double)k1 * inv_s2, v2 = (double)k2 * inv_s2;
                        const int rI = 3 * sm.nodes[e][I], rJ = 3 * sm.nodes[e][J];
                        const int pij = __ldg(mrow + I * 20 + J);
                        if (pij >= 0) {
                            const int len = __ldg(tgt.row_ptr + rI + 1) - __ldg(tgt.row_ptr + rI);
                            double* d = tgt.csr + pij + (size_t)a * len;
                            atomicAdd(d, v0);
                            atomicAdd(d + 1, v1);
                            atomicAdd(d + 2, v2);
                        }
                        const int pji = J != I ? __ldg(mrow + J * 20 + I) : -1;
                        if (pji >= 0) {
                            const int len = __ldg(tgt.row_ptr + rJ + 1) - __ldg(tgt.row_ptr + rJ);
                            double* d = tgt.csr + pji + a;
                            atomicAdd(d, v0);
                            atomicAdd(d + len, v1);
                            atomicAdd(d + 2 * (size_t)len, v2);
                        }
                    }
                } else if (real && J >= I) {
                    out[9 * J] = (double)k0 * inv_s2;
                    out[9 * J + 1] = (double)k1 * inv_s2;
                    out[9 * J + 2] = (double)k2 * inv_s2;
                }
            }
        }
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        // 7. copy the pair's Ke out (the bounds and signs were last read above)
        if (tid < 2) {
            sm.bound_bits[tid] = 0ull;
            sm.negmask[tid] = 0u;
        }
        if (kMap) continue;
        const int nvalid = 2 * p + 1 < count ? 2 : 1;
        double* dst = ke_out + (size_t)(2 * p) * kPackedHex20;
        if (bulk_out) {
            if (tid == 0) {
                asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst),
                             "r"(smem_u32(sm.ke[0])), "r"((uint32_t)(nvalid * kPackedHex20 * sizeof(double)))
                             : "memory");
                asm volatile("cp.async.bulk.commit_group;" ::: "memory");
            }
        } else {
            for (int k = tid; k < nvalid * kPackedHex20; k += kThreads) dst[k] = (&sm.ke[0][0])[k];
        }
    }
    // A CTA whose wait ran out still has its six products in flight: it waits
    // for them again, with the default bound, before the tensor memory they
    // write is released. If that wait runs out too, the products are presumed
    // lost; the memory is released all the same and FEM_ERR_INTERNAL tells the
    // caller to treat the device as suspect.
    if (timed_out && !mbar_wait_bounded(bar, parity ^ 1u, kDefaultWaitNs) && tid == 0)
        atomicOr(status, 1 << FEM_ERR_INTERNAL);
    if (tid == 0 && bulk_out && !kMap) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
    }
}

template <int kMode>
cudaError_t launch_tc(const MeshView& m, double* ke_out, int* status, const SlotTarget& tgt, cudaStream_t s) {
    static DeviceCache cache;
    const size_t smem = sizeof(KeTcSmem);
    int blocks_per_sm = 0;
    const cudaError_t err = per_device(cache, [&](int& v) {
        // Resident CTAs per SM from the kernel's registers, its shared memory
        // and the 512 tensor-memory columns of an SM (kTmemCols per CTA). The
        // runtime's occupancy query answers 1 for this kernel, which would
        // leave three quarters of the SM idle.
        cudaError_t e =
            cudaFuncSetAttribute(k_hex20_ke_tc<kMode>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaFuncAttributes fa;
        if (!e) e = cudaFuncGetAttributes(&fa, k_hex20_ke_tc<kMode>);
        int dev = 0, regs_sm = 0, smem_sm = 0;
        if (!e) e = cudaGetDevice(&dev);
        if (!e) e = cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev);
        if (!e) e = cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
        if (e) return e;
        const int regs_cta = ((fa.numRegs + 7) / 8) * 8 * kThreads;
        const int by_regs = regs_cta > 0 ? regs_sm / regs_cta : 1;
        const int by_smem = smem_sm / (int)(smem + 1024);  // 1 KB per CTA is reserved by the runtime
        v = std::min({by_regs, by_smem, (int)(512 / kTmemCols)});
        return cudaSuccess;
    }, blocks_per_sm);
    if (err) return err;
    const long long count = kMode == kTcWave ? (long long)(tgt.i1 - tgt.i0) : (long long)m.E_count;
    const long long npairs = (count + 1) / 2;
    const long long grid = std::max<long long>(1, std::min<long long>((long long)blocks_per_sm * sm_count(), npairs));
    const int bulk_out = kMode != kTcCsrMap && (reinterpret_cast<uintptr_t>(ke_out) & 15u) == 0;
    k_hex20_ke_tc<kMode><<<(int)grid, kThreads, smem, s>>>(m, ke_out, status, bulk_out, tgt);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_hex20_ke_tcgen05(const MeshView& m, double* ke_out, int* status, long long wait_ns,
                                    cudaStream_t s) {
    SlotTarget t{};
    t.wait_ns = wait_ns;
    return launch_tc<kTcPacked>(m, ke_out, status, t, s);
}

cudaError_t launch_stage_hex20_tc(const MeshView& m, const int* perm, int i0, int i1, double* stage, int* status,
                                  long long wait_ns, cudaStream_t s) {
    if (i1 <= i0) return cudaSuccess;
    return launch_tc<kTcWave>(m, stage, status, SlotTarget{perm, nullptr, nullptr, nullptr, i0, i1, wait_ns}, s);
}

cudaError_t launch_reassemble_hex20_tc(const MeshView& m, const int* perm, const MapTarget& mt, DevInfo* info,
                                       cudaStream_t s) {
    return launch_tc<kTcCsrMap>(m, nullptr, &info->status_bits,
                                SlotTarget{perm, mt.map, mt.row_ptr, mt.values, 0, m.E_count,
                                           wait_ns_of(0)},
                                s);
}

}  // namespace fem
