// tc_gemm.cu -- tcgen05 FP16-split tensor-core trailing update of the FP32 LU:
//     A22 -= L21 U12      (complex, FP32 storage, FP32 accumulation in TMEM)
//
// Complex -> real: with row-major interleaved storage a complex row of length
// n is a real row of length 2n, and
//     C_R[i, 2j+c] -= sum_k' L_R[i, k'] U_big[k', 2j+c],   k' = 2k + c'
//     U_big[2k, 2j] = Ur, U_big[2k+1, 2j] = -Ui, U_big[2k, 2j+1] = Ui, U_big[2k+1, 2j+1] = Ur
// so one real GEMM of M = rows, N = 2 cols, K = 2 nb does the complex update
// with no wasted products.  Both operands are staged K-major (K contiguous):
// A_s[i][k'] = L_R[i][k'] and B_s[n][k'] = U_big[k'][n], each scaled by a
// power of two and split into an FP16 high part and the FP16 rounding of the
// remainder (11 + 11 significant bits); the MMA (kind::f16, FP32
// accumulation) sums hi*hi + hi*lo + lo*hi (split_terms = 3, about FP32
// accuracy: the same 22 bits as a TF32 high part with a TF32-rounded
// remainder, at twice the tensor rate and half the operand bytes) or takes
// the high parts alone (1).  FP16 has 5 exponent bits, hence the scales:
//   L: |l| <= sqrt 2 under partial pivoting by |re| + |im|, so L is staged
//      times 2^L_SHIFT, which keeps the high part below 2^13 and moves small
//      multipliers out of the subnormal range;
//   U: each complex column j of U12 is staged times 2^s_j with s_j chosen so
//      that its largest |re| or |im| lies in [2^13, 2^14) (B_SCALE_EXP); the
//      epilogue multiplies column j of the product by 2^-(s_j + L_SHIFT),
//      kept per column in the staging buffer.
// Normwise the staged operands carry about 2^-22 of each column's (and of L's)
// largest entry, like the TF32 split's 2^-22 relative error per entry.
//
// Kernel: one CTA per 128 x 256 output tile, 6 warps.
//   warp 0       TMA producer (cp.async.bulk.tensor, SWIZZLE_128B, no multicast)
//   warp 1       TMEM allocator; one elected thread issues tcgen05.mma
//   warps 2..5   epilogue: tcgen05.ld 32x32b -> C -= D -> global
// Every mbarrier wait has an iteration budget; on expiry the CTA sets a status
// bit, drains what it issued (bounded) and frees its TMEM.
#include <cuda.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstring>

#include "internal.cuh"

namespace bb {

constexpr int TC_BM = 128, TC_BN = 256, TC_BK = 64;  // tile: rows, real cols, K per stage (fp16: 128-byte rows)
constexpr int TC_THREADS = 192;
constexpr uint32_t TC_SPIN = 1u << 24;

// ---------------------------------------------------------------------------
// PTX helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// bounded wait: false when the budget ran out (status bit set by the caller)
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
    for (uint32_t it = 0; it < TC_SPIN; ++it)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int x, int y, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ uint64_t umma_desc_sw128(const void *smem) {
    // K-major, SWIZZLE_128B: LBO = 1 (unused), SBO = 1024 B between 8-row groups
    const uint64_t addr = (smem_u32(smem) >> 4) & 0x3FFF;
    return addr | (1ull << 16) | (64ull << 32) | (1ull << 46) | (2ull << 61);
}

// kind::f16 instruction descriptor: D f32 (bits 4-5 = 1), A and B both f16
// (bits 7-9 and 10-12 = 0), both K-major, N >> 3 at bit 17, M >> 4 at bit 24;
// M = 128, N = 256
constexpr uint32_t TC_IDESC = (1u << 4) | (0u << 7) | (0u << 10) | ((uint32_t)(TC_BN >> 3) << 17) |
                              ((uint32_t)(TC_BM >> 4) << 24);

__device__ __forceinline__ void umma_f16(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(dtmem),
        "l"(adesc), "l"(bdesc), "r"(TC_IDESC), "r"(accumulate)
        : "memory");
}
__device__ __forceinline__ void umma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float *v) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// ---------------------------------------------------------------------------
// kernel: persistent over output tiles, two TMEM accumulators
// ---------------------------------------------------------------------------
struct TcArgs {
    int m;             // rows of the trailing block
    int ncr;           // real columns of the trailing block (2 x complex columns)
    int cx0, cy0;      // coordinates of the block origin in the C tensor map (real col, row)
    int brow0;         // first row of the staged B operand that this block's columns use
    int kchunks;       // K / TC_BK
    const float *bscale;  // per staged complex column: 2^-(s_j + L_SHIFT), undoing the staging's scales
    int split;         // 1 or 3
    int tiles_n;       // column tiles
    int ntiles;
    int *status;
};

__device__ __forceinline__ void tma_reduce_add_2d(const CUtensorMap *map, int x, int y, const void *src) {
    asm volatile(
        "cp.reduce.async.bulk.tensor.2d.global.shared::cta.add.tile.bulk_group [%0, {%1, %2}], [%3];" ::"l"(
            reinterpret_cast<uint64_t>(map)),
        "r"(x), "r"(y), "r"(smem_u32(src))
        : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read0() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait0() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

constexpr int TC_EPI_BYTES = 32 * 32 * 4;  // per epilogue warp: 32 rows x 32 fp32

template <int STAGES>
__global__ void __launch_bounds__(TC_THREADS, 1)
    tc_update_kernel(const __grid_constant__ CUtensorMap mA_hi, const __grid_constant__ CUtensorMap mA_lo,
                     const __grid_constant__ CUtensorMap mB_hi, const __grid_constant__ CUtensorMap mB_lo,
                     const __grid_constant__ CUtensorMap mC, TcArgs g) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char *base = reinterpret_cast<unsigned char *>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    constexpr int A_BYTES = TC_BM * TC_BK * 2, B_BYTES = TC_BN * TC_BK * 2;  // fp16 operands
    constexpr int STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;
    float *epi = reinterpret_cast<float *>(base + (size_t)STAGES * STAGE_BYTES);  // 4 x 32 x 32
    __shared__ __align__(8) uint64_t full_bar[STAGES], empty_bar[STAGES], tfull_bar[2], tempty_bar[2], drain_bar;
    __shared__ uint32_t tmem_base_slot;
    __shared__ volatile int abort_flag;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const bool split3 = g.split == 3;
    const uint32_t stage_tx = split3 ? STAGE_BYTES : (A_BYTES + B_BYTES);
    const int my_tiles = g.ntiles > (int)blockIdx.x ? (g.ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full_bar[s], 1);
            mbar_init(&empty_bar[s], 1);
        }
        for (int a = 0; a < 2; ++a) {
            mbar_init(&tfull_bar[a], 1);
            mbar_init(&tempty_bar[a], 4);
        }
        mbar_init(&drain_bar, 1);
        abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_slot)),
                     "r"(2 * TC_BN)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base_slot;

    if (warp == 0) {
        if (lane == 0) {
            int it = 0;  // running k-chunk counter over all tiles
            for (int i = 0; i < my_tiles && !abort_flag; ++i) {
                const int t = blockIdx.x + i * gridDim.x;
                const int row0 = (t / g.tiles_n) * TC_BM, col0 = (t % g.tiles_n) * TC_BN;
                for (int kc = 0; kc < g.kchunks; ++kc, ++it) {
                    const int s = it % STAGES;
                    if (it >= STAGES && !mbar_wait(&empty_bar[s], ((it / STAGES) - 1) & 1)) {
                        atomicOr(g.status, (int)DEV_BARRIER_TIMEOUT);
                        abort_flag = 1;
                        break;
                    }
                    unsigned char *st = base + (size_t)s * STAGE_BYTES;
                    mbar_expect_tx(&full_bar[s], stage_tx);
                    const int kx = kc * TC_BK;
                    tma_load_2d(st, &mA_hi, kx, row0, &full_bar[s]);
                    tma_load_2d(st + 2 * A_BYTES, &mB_hi, kx, g.brow0 + col0, &full_bar[s]);
                    if (split3) {
                        tma_load_2d(st + A_BYTES, &mA_lo, kx, row0, &full_bar[s]);
                        tma_load_2d(st + 2 * A_BYTES + B_BYTES, &mB_lo, kx, g.brow0 + col0, &full_bar[s]);
                    }
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            int it = 0;
            for (int i = 0; i < my_tiles && !abort_flag; ++i) {
                const int a = i & 1;
                const uint32_t dt = tmem + (uint32_t)(a * TC_BN);
                if (i >= 2 && !mbar_wait(&tempty_bar[a], ((i >> 1) - 1) & 1)) {
                    atomicOr(g.status, (int)DEV_BARRIER_TIMEOUT);
                    abort_flag = 1;
                    break;
                }
                tc_fence_after();
                uint32_t acc = 0;
                for (int kc = 0; kc < g.kchunks; ++kc, ++it) {
                    const int s = it % STAGES;
                    if (!mbar_wait(&full_bar[s], (it / STAGES) & 1)) {
                        atomicOr(g.status, (int)DEV_BARRIER_TIMEOUT);
                        abort_flag = 1;
                        break;
                    }
                    tc_fence_after();
                    unsigned char *st = base + (size_t)s * STAGE_BYTES;
                    const uint64_t ah = umma_desc_sw128(st), al = umma_desc_sw128(st + A_BYTES);
                    const uint64_t bh = umma_desc_sw128(st + 2 * A_BYTES),
                                   bl = umma_desc_sw128(st + 2 * A_BYTES + B_BYTES);
#pragma unroll
                    for (int kk = 0; kk < TC_BK / 16; ++kk) {
                        const uint64_t adv = (uint64_t)(kk * 32) >> 4;  // 16 f16 = 32 bytes along K
                        if (split3) {
                            umma_f16(dt, al + adv, bh + adv, acc);
                            umma_f16(dt, ah + adv, bl + adv, 1);
                            umma_f16(dt, ah + adv, bh + adv, 1);
                        } else {
                            umma_f16(dt, ah + adv, bh + adv, acc);
                        }
                        acc = 1;
                    }
                    umma_commit(&empty_bar[s]);
                }
                umma_commit(&tfull_bar[a]);
            }
            // drain: arrives once every MMA issued above has completed
            umma_commit(&drain_bar);
            if (!mbar_wait(&drain_bar, 0)) atomicOr(g.status, (int)DEV_BARRIER_TIMEOUT);
        }
    } else {
        // epilogue warps 2..5: TMEM lane quarter q = warp % 4
        const int q = warp & 3;
        float *buf = epi + (size_t)q * 32 * 32;
        for (int i = 0; i < my_tiles && !abort_flag; ++i) {
            const int a = i & 1;
            const int t = blockIdx.x + i * gridDim.x;
            const int row0 = (t / g.tiles_n) * TC_BM, col0 = (t % g.tiles_n) * TC_BN;
            if (!mbar_wait(&tfull_bar[a], (i >> 1) & 1)) {
                atomicOr(g.status, (int)DEV_BARRIER_TIMEOUT);
                abort_flag = 1;
                break;
            }
            tc_fence_after();
            const bool rows_live = row0 + q * 32 < g.m;
#pragma unroll 1
            for (int c = 0; c < TC_BN; c += 32) {
                float v[32];
                tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(a * TC_BN + c), v);
                if (!rows_live || col0 + c >= g.ncr) continue;  // nothing of this chunk is inside C
                {
                    // undo the staging's scales: lane l fetches real column c + l's factor
                    const float sl = g.bscale[(g.brow0 + col0 + c + lane) >> 1];
#pragma unroll
                    for (int i = 0; i < 32; ++i) v[i] *= __shfl_sync(0xffffffffu, sl, i);
                }
                if (lane == 0) bulk_wait_read0();  // staging buffer free again
                __syncwarp();
                // row `lane` of the 32 x 32 box, in the TMA 128-byte swizzle:
                // 16-byte chunk j of row r sits at chunk j ^ (r & 7)
#pragma unroll
                for (int j = 0; j < 8; ++j)
                    reinterpret_cast<float4 *>(buf + lane * 32)[j ^ (lane & 7)] =
                        make_float4(-v[4 * j], -v[4 * j + 1], -v[4 * j + 2], -v[4 * j + 3]);
                fence_proxy_async_smem();
                __syncwarp();
                if (lane == 0) {
                    tma_reduce_add_2d(&mC, g.cx0 + col0 + c, g.cy0 + row0 + q * 32, buf);
                    bulk_commit();
                }
            }
            // TMEM buffer a may be overwritten by the tile after next
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&tempty_bar[a]);
        }
        if (lane == 0) bulk_wait0();
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * TC_BN) : "memory");
    }
}

// ---------------------------------------------------------------------------
// operand staging: A_s[i][k'] = L_R rows, B_s[n][k'] = U_big columns, hi/lo
// FP16, scaled (see the top of this file)
// ---------------------------------------------------------------------------
__global__ void stage_a_kernel(const float2 *A, int64_t ld, int k, int nb, int m, __half *ahi, __half *alo,
                               int split) {
    // row i of L21 = A[k+nb+i][k .. k+nb), times 2^L_SHIFT
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)m * nb) return;
    const int i = (int)(idx / nb), kk = (int)(idx % nb);
    const float2 v = A[(int64_t)(k + nb + i) * ld + k + kk];
    const float sc = pow2f(L_SHIFT);
    __half hr, hi_, lr, li;
    split_f16(v.x * sc, hr, lr);
    split_f16(v.y * sc, hi_, li);
    reinterpret_cast<__half2 *>(ahi + (int64_t)i * 2 * nb)[kk] = __halves2half2(hr, hi_);
    if (split == 3) reinterpret_cast<__half2 *>(alo + (int64_t)i * 2 * nb)[kk] = __halves2half2(lr, li);
}

// One warp per complex column j of U12 (U12[kk][j] = A[k+kk][k+nb+j], j = j0 ..
// j0+ncols): the column's exponent s_j from its largest |re| or |im|, then
// rows 2j and 2j+1 of B_s get (Ur, -Ui) 2^s_j and (Ui, Ur) 2^s_j at K = 2kk,
// and bscale[j] = 2^-(s_j + L_SHIFT).
__global__ void stage_b_kernel(const float2 *A, int64_t ld, int k, int nb, int j0, int ncols, __half *bhi,
                               __half *blo, float *bscale, int split) {
    const int wi = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (wi >= ncols) return;  // whole warps
    const int j = j0 + wi;
    const float2 *col = A + (int64_t)k * ld + k + nb + j;
    float mx = 0.f;
    for (int kk = lane; kk < nb; kk += 32) {
        const float2 u = col[(int64_t)kk * ld];
        mx = fmaxf(mx, fmaxf(fabsf(u.x), fabsf(u.y)));
    }
    mx = __uint_as_float(__reduce_max_sync(0xffffffffu, __float_as_uint(mx)));  // non-negative: ordered as bits
    const int sx = stage_exp(mx);
    const float sc = pow2f(sx);
    if (lane == 0) bscale[j] = pow2f(-sx - L_SHIFT);
    __half2 *h0 = reinterpret_cast<__half2 *>(bhi + (int64_t)(2 * j) * 2 * nb);
    __half2 *h1 = reinterpret_cast<__half2 *>(bhi + (int64_t)(2 * j + 1) * 2 * nb);
    __half2 *l0 = reinterpret_cast<__half2 *>(blo + (int64_t)(2 * j) * 2 * nb);
    __half2 *l1 = reinterpret_cast<__half2 *>(blo + (int64_t)(2 * j + 1) * 2 * nb);
    for (int kk = lane; kk < nb; kk += 32) {
        const float2 u = col[(int64_t)kk * ld];
        __half er, ei, orr, oi, ler, lei, lor, loi;
        split_f16(u.x * sc, er, ler);
        split_f16(-u.y * sc, ei, lei);
        split_f16(u.y * sc, orr, lor);
        split_f16(u.x * sc, oi, loi);
        h0[kk] = __halves2half2(er, ei);
        h1[kk] = __halves2half2(orr, oi);
        if (split == 3) {
            l0[kk] = __halves2half2(ler, lei);
            l1[kk] = __halves2half2(lor, loi);
        }
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        BB_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
        BB_REQUIRE(p && q == cudaDriverEntryPointSuccess, BEAT_B200_CUDA_ERROR,
                   "cuTensorMapEncodeTiled is unavailable in this driver");
        fn = reinterpret_cast<EncodeTiledFn>(p);
    }
    return fn;
}

// rows x kdim fp16, row-major, box TC_BK (K, 128 bytes) x box_rows
static CUtensorMap make_map(const __half *ptr, int64_t rows, int kdim, int box_rows) {
    CUtensorMap m;
    std::memset(&m, 0, sizeof(m));
    cuuint64_t dims[2] = {(cuuint64_t)kdim, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)kdim * sizeof(__half)};
    cuuint32_t box[2] = {(cuuint32_t)TC_BK, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = encode_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2, (void *)ptr, dims, strides, box, estr,
                             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    BB_REQUIRE(r == CUDA_SUCCESS, BEAT_B200_CUDA_ERROR, "cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
    return m;
}

constexpr int TC_STAGES = 2;

// C: the whole matrix as fp32 rows of 2n real columns, row stride 2 ld
static CUtensorMap make_c_map(const float *ptr, int n, int64_t ld) {
    CUtensorMap m;
    std::memset(&m, 0, sizeof(m));
    cuuint64_t dims[2] = {(cuuint64_t)2 * n, (cuuint64_t)n};
    cuuint64_t strides[1] = {(cuuint64_t)ld * 8};
    cuuint32_t box[2] = {32, 32};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = encode_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, (void *)ptr, dims, strides, box, estr,
                             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                             CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    BB_REQUIRE(r == CUDA_SUCCESS, BEAT_B200_CUDA_ERROR, "cuTensorMapEncodeTiled (C) failed: " + std::to_string((int)r));
    return m;
}

// Staging of panel k's operands for the trailing update A22 -= L21 U12 (rows
// and columns k + nb .. n): A_hi/A_lo (m x 2nb fp16) and B_hi/B_lo (2m x 2nb
// fp16), m = n - k - nb, and the per-column factors bscale (m, padded), in the
// workspace's staging buffer.
struct TcStage {
    __half *ahi, *alo, *bhi, *blo;
    float *bscale;
    int m, kdim;
};

static TcStage tc_stage_buffers(beat_b200_ctx *c, int k, int nb) {
    Workspace &w = c->ws;
    const int n = c->V;
    TcStage s;
    s.m = n - k - nb;
    s.kdim = 2 * nb;
    const int64_t mpad = ((int64_t)s.m + TC_BM - 1) / TC_BM * TC_BM;
    const int64_t npad = ((int64_t)2 * s.m + TC_BN - 1) / TC_BN * TC_BN;
    // the factors: one per staged complex column, padded so that an epilogue chunk past the
    // last column still reads inside the buffer
    auto bytes = [&](int64_t mp, int64_t np) {
        return sizeof(__half) * (size_t)s.kdim * (2 * (size_t)mp + 2 * (size_t)np) +
               sizeof(float) * (size_t)(np / 2 + 64) + 1024;
    };
    if (w.stage.bytes < bytes(mpad, npad)) {
        // size for the first (largest) panel
        const int64_t m0 = n, mp0 = (m0 + TC_BM - 1) / TC_BM * TC_BM, np0 = (2 * m0 + TC_BN - 1) / TC_BN * TC_BN;
        w.stage.alloc(bytes(mp0, np0));
    }
    s.ahi = w.stage.as<__half>();
    s.alo = s.ahi + (size_t)mpad * s.kdim;
    s.bhi = s.alo + (size_t)mpad * s.kdim;
    s.blo = s.bhi + (size_t)npad * s.kdim;
    s.bscale = reinterpret_cast<float *>(s.blo + (size_t)npad * s.kdim);
    return s;
}

bool tc_update_supported(int nb) { return nb % 32 == 0; }  // K = 2 nb must be a multiple of TC_BK

// Stages L21 of panel k (every row below the panel).
void tc_stage_l(beat_b200_ctx *c, int k, int nb, int split_terms, cudaStream_t st) {
    const TcStage s = tc_stage_buffers(c, k, nb);
    if (s.m <= 0) return;
    const int64_t na = (int64_t)s.m * nb;
    stage_a_kernel<<<(unsigned)((na + 255) / 256), 256, 0, st>>>(c->ws.A.as<float2>(), c->ws.ld, k, nb, s.m, s.ahi,
                                                                 s.alo, split_terms);
    BB_CUDA(cudaGetLastError());
}

// Stages U12 of panel k for the columns [col_lo, col_hi) (absolute, >= k + nb),
// which must already hold U12 = L11^-1 A12.
void tc_stage_u(beat_b200_ctx *c, int k, int nb, int split_terms, int col_lo, int col_hi, cudaStream_t st) {
    const TcStage s = tc_stage_buffers(c, k, nb);
    const int nc = col_hi - col_lo;
    if (s.m <= 0 || nc <= 0) return;
    stage_b_kernel<<<(unsigned)(((int64_t)nc * 32 + 255) / 256), 256, 0, st>>>(
        c->ws.A.as<float2>(), c->ws.ld, k, nb, col_lo - (k + nb), nc, s.bhi, s.blo, s.bscale, split_terms);
    BB_CUDA(cudaGetLastError());
}

// The B-operand staging of panel k (rows 2 j, 2 j + 1 for column k + nb + j, K = 2 nb,
// and the column factors): the blocked U12 solve writes it directly (lu.cu).
void tc_stage_u_buffers(beat_b200_ctx *c, int k, int nb, __half **bhi, __half **blo, float **bscale) {
    const TcStage s = tc_stage_buffers(c, k, nb);
    *bhi = s.bhi;
    *blo = s.blo;
    *bscale = s.bscale;
}

// A[k+nb.., col_lo..col_hi) -= L21 U12 from the staged operands, on `st`,
// with at most max_ctas persistent CTAs (0: one per SM).
void tc_update_cols(beat_b200_ctx *c, int k, int nb, int split_terms, int col_lo, int col_hi, cudaStream_t st,
                    int max_ctas) {
    const int n = c->V;
    const TcStage s = tc_stage_buffers(c, k, nb);
    const int nc = col_hi - col_lo;
    if (s.m <= 0 || nc <= 0) return;
    const CUtensorMap mah = make_map(s.ahi, s.m, s.kdim, TC_BM), mal = make_map(s.alo, s.m, s.kdim, TC_BM);
    const CUtensorMap mbh = make_map(s.bhi, 2 * (int64_t)s.m, s.kdim, TC_BN),
                      mbl = make_map(s.blo, 2 * (int64_t)s.m, s.kdim, TC_BN);
    const CUtensorMap mc = make_c_map(c->ws.A.as<float>(), n, c->ws.ld);
    TcArgs g;
    g.m = s.m;
    g.ncr = 2 * nc;
    g.cx0 = 2 * col_lo;
    g.cy0 = k + nb;
    g.brow0 = 2 * (col_lo - (k + nb));
    g.kchunks = s.kdim / TC_BK;
    g.split = split_terms;
    g.tiles_n = (2 * nc + TC_BN - 1) / TC_BN;
    g.ntiles = g.tiles_n * ((s.m + TC_BM - 1) / TC_BM);
    g.status = c->status.as<int>();
    g.bscale = s.bscale;
    const size_t smem = (size_t)TC_STAGES * (2 * TC_BM * TC_BK * 2 + 2 * TC_BN * TC_BK * 2) + 4 * TC_EPI_BYTES + 1024;
    static std::atomic<bool> attr_done{false};  // sweep lanes call this from several threads
    if (!attr_done) {
        BB_CUDA(cudaFuncSetAttribute(tc_update_kernel<TC_STAGES>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem));
        attr_done = true;
    }
    const int cap = max_ctas > 0 ? std::min(max_ctas, c->sm_count) : c->sm_count;
    const int grid = std::min(g.ntiles, cap);
    tc_update_kernel<TC_STAGES><<<grid, TC_THREADS, smem, st>>>(mah, mal, mbh, mbl, mc, g);
    BB_CUDA(cudaGetLastError());
}

}  // namespace bb
