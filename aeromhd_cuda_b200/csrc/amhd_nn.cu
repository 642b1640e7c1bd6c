// amhd_nn.cu -- kernels of the learned coarse-grid corrector: the BF16
// tensor-core GEMMs (FP32 accumulation) that carry every convolution (im2col
// form) -- tcgen05.mma with the accumulator in tensor memory, operands by
// TMA, and mma.sync m16n8k16 for the shapes it suits better -- and the
// element-wise, pooling, loss and Adam kernels of its training and inference.
//
// Activations are FP32 in [C][B*H*W] layout (channel-major: the output of a
// GEMM W[Cout][K] x col[K][N] is the next layer's input as is); GEMM operands
// are BF16, weights keep an FP32 master copy for Adam.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <climits>
#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <string>

#include "aeromhd.h"
#include "amhd_tma.cuh"

namespace {

thread_local std::string g_nn_err;

int nn_fail(int code, const char *fmt, ...)
{
    char buf[256];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_nn_err = buf;
    return code;
}

#define NNCK(call)                                                                                   \
    do {                                                                                             \
        cudaError_t e__ = (call);                                                                    \
        if (e__ != cudaSuccess) return nn_fail(AMHD_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e__)); \
    } while (0)

inline cudaStream_t S(void *s) { return reinterpret_cast<cudaStream_t>(s); }

inline bool aligned16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

inline int blocks_for(int64_t n, int threads = 256)
{
    int64_t b = (n + threads - 1) / threads;
    if (b > 148 * 32) b = 148 * 32;
    return (int)(b < 1 ? 1 : b);
}

using bf16 = __nv_bfloat16;

// ---------------------------------------------------------------------------
// GEMM: C[M][N] = alpha * op(A) op(B) (+ beta * C), op(A) = A (row-major
// [M][K], lda) or A^T (A stored [K][M]); op(B) = B ([K][N]) or B^T (B stored
// [N][K]).  64x64x32 CTA tiles, 4 warps of 32x32, split-K over gridDim.z
// (then the partial products are added atomically into C, which the caller
// has scaled by beta beforehand).
// ---------------------------------------------------------------------------
constexpr int GBM = 64, GBN = 64, GBK = 32, GPAD = 8;

__device__ __forceinline__ void mma_bf16(float d[4], const uint32_t a[4], const uint32_t b[2])
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__global__ void __launch_bounds__(128) gemm_bf16_kernel(int transA, int transB, int M, int N, int K, const bf16 *A,
                                                        int lda, const bf16 *B, int ldb, float *C, int ldc,
                                                        float alpha, float beta, int k_per_split)
{
    __shared__ __align__(16) bf16 As[GBM][GBK + GPAD];
    __shared__ __align__(16) bf16 Bs[GBN][GBK + GPAD];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int g = lane >> 2, t4 = lane & 3;
    const int m0 = blockIdx.y * GBM, n0 = blockIdx.x * GBN;
    const int kbeg = blockIdx.z * k_per_split;
    const int kend = min(K, kbeg + k_per_split);
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
    float acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int r = 0; r < 4; ++r) acc[i][j][r] = 0.f;
    const bf16 zero = __float2bfloat16(0.f);

    for (int k0 = kbeg; k0 < kend; k0 += GBK) {
        for (int e = tid; e < GBM * GBK; e += 128) {
            int mm, kk;
            if (!transA) {
                mm = e / GBK;
                kk = e % GBK;
            } else {
                kk = e / GBM;
                mm = e % GBM;
            }
            const int gm = m0 + mm, gk = k0 + kk;
            bf16 v = zero;
            if (gm < M && gk < kend) v = transA ? A[(int64_t)gk * lda + gm] : A[(int64_t)gm * lda + gk];
            As[mm][kk] = v;
        }
        for (int e = tid; e < GBN * GBK; e += 128) {
            int nn, kk;
            if (!transB) {
                kk = e / GBN;
                nn = e % GBN;
            } else {
                nn = e / GBK;
                kk = e % GBK;
            }
            const int gn = n0 + nn, gk = k0 + kk;
            bf16 v = zero;
            if (gn < N && gk < kend) v = transB ? B[(int64_t)gn * ldb + gk] : B[(int64_t)gk * ldb + gn];
            Bs[nn][kk] = v;
        }
        __syncthreads();
#pragma unroll
        for (int ks = 0; ks < GBK; ks += 16) {
            uint32_t a[2][4], b[4][2];
#pragma unroll
            for (int mi = 0; mi < 2; ++mi) {
                const int r = wm + mi * 16 + g;
                a[mi][0] = *reinterpret_cast<const uint32_t *>(&As[r][ks + 2 * t4]);
                a[mi][1] = *reinterpret_cast<const uint32_t *>(&As[r + 8][ks + 2 * t4]);
                a[mi][2] = *reinterpret_cast<const uint32_t *>(&As[r][ks + 8 + 2 * t4]);
                a[mi][3] = *reinterpret_cast<const uint32_t *>(&As[r + 8][ks + 8 + 2 * t4]);
            }
#pragma unroll
            for (int ni = 0; ni < 4; ++ni) {
                const int c = wn + ni * 8 + g;
                b[ni][0] = *reinterpret_cast<const uint32_t *>(&Bs[c][ks + 2 * t4]);
                b[ni][1] = *reinterpret_cast<const uint32_t *>(&Bs[c][ks + 8 + 2 * t4]);
            }
#pragma unroll
            for (int mi = 0; mi < 2; ++mi)
#pragma unroll
                for (int ni = 0; ni < 4; ++ni) mma_bf16(acc[mi][ni], a[mi], b[ni]);
        }
        __syncthreads();
    }
    const bool split = gridDim.z > 1;
#pragma unroll
    for (int mi = 0; mi < 2; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const int row = m0 + wm + mi * 16 + g + (r >= 2 ? 8 : 0);
                const int col = n0 + wn + ni * 8 + 2 * t4 + (r & 1);
                if (row < M && col < N) {
                    float *p = &C[(int64_t)row * ldc + col];
                    const float v = alpha * acc[mi][ni][r];
                    if (split)
                        atomicAdd(p, v);
                    else
                        *p = (beta != 0.f) ? v + beta * (*p) : v;
                }
            }
}

// ---------------------------------------------------------------------------
// The same GEMM on the 5th-generation tensor cores: tcgen05.mma (kind::f16,
// BF16 operands, FP32 accumulation in tensor memory).  One 128 x 128 output
// tile per CTA of 4 warps, K in steps of 64: the warps stage the A and B tiles
// in shared memory, both K-major in the canonical layout without swizzle (core
// matrices of 8 rows x 8 values, 128 contiguous bytes; 128 B between core
// matrices along M / N, 2 KB between the 8-value groups along K), one thread
// issues four MMAs of K = 16 and commits them to an mbarrier, and every thread
// waits for it (bounded: after kTcWaitIters polls the CTA records an error and
// stops issuing) before the tiles are restaged.  The accumulator, 128 TMEM
// lanes x 128 columns, is read back with tcgen05.ld (each warp its 32 rows).
// The TMEM columns are freed on every path.  The CTA asks for enough shared
// memory that at most 3 are resident on an SM (3 x 128 of the 512 columns).
// Two shared-memory stages: while the MMAs of one K step run, the warps stage
// the next.
// ---------------------------------------------------------------------------
constexpr int TM = 128, TN = 128, TK = 64;
__device__ int g_tc_err;  // set when an MMA wait gave up (amhd_nn_gemm_status reads and clears it)
constexpr uint32_t kTcWaitIters = 1u << 24;
constexpr uint64_t kTcWaitNs = 1000000000ull;  // 1 s
constexpr int kTcSmemBytes = 66 * 1024;  // > 228 KB / 4: at most 3 CTAs per SM (3 x 128 TMEM columns)

// Each operand tile is stored in the layout of its source: K-major, element
// (m, k) at [k / 8][m / 8][m % 8][k % 8], when the source is contiguous along K
// (A not transposed, B transposed), MN-major, element (m, k) at
// [k / 8][m / 8][k % 8][m % 8], when it is contiguous along M / N; either way
// 8 consecutive source values are one 16-byte row of a core matrix.
struct TcSmem {
    bf16 a[2][TK / 8][TM / 8][8][8];  // two stages: the next tile is staged while the MMAs read this one
    bf16 b[2][TK / 8][TN / 8][8][8];
    uint64_t mbar[2];  // completion of the MMAs that read stage 0 / 1
    uint32_t tmem;
    int err;
};

// Stage rows x TK values of one operand: src is contiguous along K (kmajor) or
// along the rows; 8-value pieces move as 16-byte copies when aligned and in
// range, the rest value by value with zero fill.
__device__ __forceinline__ void tc_stage(bf16 (*dst)[TM / 8][8][8], const bf16 *src, int ld, bool kmajor, int r0,
                                         int rows_total, int k0, int kend, int tid)
{
    const bf16 zero = __float2bfloat16(0.f);
    constexpr int kPieces = TM * TK / 8;
#pragma unroll 2
    for (int e = tid; e < kPieces; e += 128) {
        int r, k;  // first value of the piece: tile row r, tile column k
        if (kmajor) {
            r = e / (TK / 8);
            k = (e % (TK / 8)) * 8;
        } else {
            k = e / (TM / 8);
            r = (e % (TM / 8)) * 8;
        }
        const int gr = r0 + r, gk = k0 + k;
        bf16 *d = kmajor ? &dst[k >> 3][r >> 3][r & 7][0] : &dst[k >> 3][r >> 3][k & 7][0];
        const bf16 *s = kmajor ? src + (int64_t)gr * ld + gk : src + (int64_t)gk * ld + gr;
        const bool full = kmajor ? (gr < rows_total && gk + 8 <= kend) : (gk < kend && gr + 8 <= rows_total);
        if (full && (reinterpret_cast<uintptr_t>(s) & 15) == 0) {
            *reinterpret_cast<uint4 *>(d) = *reinterpret_cast<const uint4 *>(s);
        } else {
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const int rr = kmajor ? gr : gr + i, kk = kmajor ? gk + i : gk;
                d[i] = (rr < rows_total && kk < kend) ? (kmajor ? src[(int64_t)rr * ld + kk] : src[(int64_t)kk * ld + rr])
                                                      : zero;
            }
        }
    }
}

__device__ __forceinline__ uint32_t tc_smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor: no swizzle, K-major (version 1, base offset 0)
__device__ __forceinline__ uint64_t tc_desc(const void *start, uint32_t lbo_bytes, uint32_t sbo_bytes)
{
    const uint64_t a = (tc_smem_addr(start) >> 4) & 0x3FFFu;
    return a | ((uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16) | ((uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32) |
           (1ull << 46);
}

// instruction descriptor of kind::f16: F32 accumulator, BF16 A and B, M = TM,
// N = TN; bit 15 / 16: A / B MN-major
constexpr uint32_t kTcIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TN >> 3) << 17) |
                              ((uint32_t)(TM >> 4) << 24);

// bounded wait on an mbarrier phase: 1 s, or kTcWaitIters polls
__device__ __forceinline__ bool tc_wait(uint64_t *bar, uint32_t parity)
{
    return amhd::tma::wait_for(bar, parity, kTcWaitNs, kTcWaitIters);
}

__global__ void __launch_bounds__(128) gemm_tc_kernel(int transA, int transB, int M, int N, int K, const bf16 *A,
                                                      int lda, const bf16 *B, int ldb, float *C, int ldc,
                                                      float alpha, float beta, int k_per_split, int *err_flag)
{
    extern __shared__ __align__(1024) unsigned char tc_raw[];
    TcSmem &sm = *reinterpret_cast<TcSmem *>(tc_raw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.y * TM, n0 = blockIdx.x * TN;
    const int kbeg = blockIdx.z * k_per_split;
    const int kend = min(K, kbeg + k_per_split);
    const bf16 zero = __float2bfloat16(0.f);

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc_smem_addr(&sm.tmem)),
                     "r"(TN)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        sm.err = 0;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tc_smem_addr(&sm.mbar[0])) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tc_smem_addr(&sm.mbar[1])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = sm.tmem;

    const bool a_kmajor = !transA, b_kmajor = transB != 0;
    const uint32_t idesc = kTcIdesc | (a_kmajor ? 0u : 1u << 15) | (b_kmajor ? 0u : 1u << 16);
    const int nk = kend > kbeg ? (kend - kbeg + TK - 1) / TK : 0;
    // commit i arrives on mbar[i & 1]; `done` commits have been waited for, in
    // order, so each barrier has at most one phase outstanding.  A timeout marks
    // the CTA (read by every thread only after the next barrier, so all decide
    // alike); the waits stay bounded either way.
    uint32_t ph = 0u;  // bit b: the parity awaited next on mbar[b]
    int done = 0;
    auto wait_until = [&](int n) {
        for (; done < n; ++done) {
            const int b = done & 1;
            if (!tc_wait(&sm.mbar[b], (ph >> b) & 1u)) sm.err = 1;
            ph ^= 1u << b;
        }
    };
    if (nk > 0) {
        tc_stage(sm.a[0], A, lda, a_kmajor, m0, M, kbeg, kend, tid);
        tc_stage(sm.b[0], B, ldb, b_kmajor, n0, N, kbeg, kend, tid);
    }
    int issued = 0;
    for (int it = 0; it < nk; ++it) {
        const int buf = it & 1;
        // the tensor cores read the tiles through the async proxy
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (sm.err) break;
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
            for (int j = 0; j < TK / 16; ++j) {
                const uint64_t da = tc_desc(&sm.a[buf][2 * j][0][0][0], 2048u, 128u);
                const uint64_t db = tc_desc(&sm.b[buf][2 * j][0][0][0], 2048u, 128u);
                const uint32_t acc = (it == 0 && j == 0) ? 0u : 1u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
                    "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
                    : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             tc_smem_addr(&sm.mbar[buf]))
                         : "memory");
        }
        issued = it + 1;
        if (it + 1 < nk) {
            // stage it+1 goes where the MMAs of step it-1 read: wait for them first
            wait_until(it);
            const int k1 = kbeg + (it + 1) * TK;
            tc_stage(sm.a[buf ^ 1], A, lda, a_kmajor, m0, M, k1, kend, tid);
            tc_stage(sm.b[buf ^ 1], B, ldb, b_kmajor, n0, N, k1, kend, tid);
        }
    }
    wait_until(issued);  // the MMAs still in flight (the last one or two steps)
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const bool first = issued == 0;
    if (!first && !sm.err) {
        const int row = m0 + warp * 32 + lane;
        const bool split = gridDim.z > 1;
#pragma unroll 1
        for (int c0 = 0; c0 < TN; c0 += 16) {
            uint32_t r[16];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
                "[%16];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                  "=r"(r[15])
                : "r"(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (row < M) {
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    const int col = n0 + c0 + i;
                    if (col < N) {
                        float *p = &C[(int64_t)row * ldc + col];
                        const float v = alpha * __uint_as_float(r[i]);
                        if (split)
                            atomicAdd(p, v);
                        else
                            *p = (beta != 0.f) ? v + beta * (*p) : v;
                    }
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TN) : "memory");
    }
    if (tid == 0 && sm.err) atomicOr(err_flag, 1);
}

// ---------------------------------------------------------------------------
// tcgen05 GEMM with TMA operand loads: 128 x 64 tiles (M x N), K steps of 64
// through a ring of kTmaStages shared-memory stages.  Thread 0 issues the
// loads (one TMA per operand and step, completion counted in bytes on
// full[s]); thread 32 waits for a stage, issues its four 128 x 64 x 16 MMAs
// and commits them to empty[s], which frees the stage for the next load; a
// last commit on `done` releases the epilogue (all 4 warps, one TMEM lane
// quadrant each).  Operand tiles are 128-byte swizzled (2-D tensor maps with
// SWIZZLE_128B, stage buffers 1024-byte aligned):
//   K-major (rows contiguous along K): box {64 K, tile rows} -> one 128-byte
//     row per tile row, 8-row swizzle atoms 1024 bytes apart (descriptor
//     SBO); the K step j of 16 values starts 32 j bytes into the row
//   MN-major (contiguous along the rows): box {64 rows, 64 K} per 64 rows ->
//     one 128-byte row per K index, 8-K-row atoms 1024 bytes apart (SBO),
//     the second 64 rows of A 8192 bytes on (LBO); K step j starts 2048 j
//     bytes on
// Out-of-range rows and K read as zero.  Every wait is bounded; a timeout
// marks the CTA, which still waits (bounded) for its loads and MMAs in flight
// and frees its TMEM columns.
// ---------------------------------------------------------------------------
constexpr int kTmaStages = 3, TN2 = 64;  // 74 KB per CTA: 3 CTAs per SM (4 stages, 2 per SM, ran 1.2-2.4x slower)
constexpr int kNumSMs = 148;
constexpr int kTmaABytes = TM * TK * 2, kTmaBBytes = TN2 * TK * 2;

struct TmaSmem {
    alignas(1024) unsigned char a[kTmaStages][kTmaABytes];
    alignas(1024) unsigned char b[kTmaStages][kTmaBBytes];
    uint64_t full[kTmaStages], empty[kTmaStages], done;
    uint32_t tmem;
    int err;
};
constexpr int kTmaSmemBytes = (int)sizeof(TmaSmem) + 1024;  // + alignment slack of the dynamic window

constexpr uint32_t kTmaIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TN2 >> 3) << 17) |
                               ((uint32_t)(TM >> 4) << 24);

// 2-D tiled load, coordinates innermost first; x is a multiple of 64 values (128 bytes)
__device__ __forceinline__ void tma_load(void *dst, const CUtensorMap *map, int x, int y, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
        "[%4];" ::"r"(tc_smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(tc_smem_addr(bar))
        : "memory");
}

constexpr uint64_t kSwizzle128 = 2ull << 61;  // descriptor layout type SWIZZLE_128B

// Pieces shared by the two TMA kernels below.
//
// the loads of K step k0 of the output tile (m0, n0) into one stage, counted on `bar`
__device__ __forceinline__ void tma_stage_loads(unsigned char *a, unsigned char *b, const CUtensorMap *mapA,
                                                const CUtensorMap *mapB, int a_kmajor, int b_kmajor, int a_tx,
                                                int a_two, int m0, int n0, int k0, uint64_t *bar)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(tc_smem_addr(bar)),
                 "r"(a_tx + kTmaBBytes)
                 : "memory");
    if (a_kmajor) {
        tma_load(a, mapA, k0, m0, bar);
    } else {
        tma_load(a, mapA, m0, k0, bar);
        if (a_two) tma_load(a + kTmaABytes / 2, mapA, m0 + TM / 2, k0, bar);
    }
    if (b_kmajor)
        tma_load(b, mapB, k0, n0, bar);
    else
        tma_load(b, mapB, n0, k0, bar);
}

// the four MMAs of one K step (K = 16 each) into the accumulator at TMEM address d;
// first: the tile's first K step (overwrite instead of accumulate)
__device__ __forceinline__ void mma_kstep(uint32_t d, const unsigned char *a, const unsigned char *b, int a_kmajor,
                                          int b_kmajor, uint32_t idesc, bool first)
{
#pragma unroll
    for (int j = 0; j < TK / 16; ++j) {
        // K step j: 32 bytes into each swizzled row (K-major) or two 8-row atoms on (MN-major)
        const uint64_t da = kSwizzle128 | (a_kmajor ? tc_desc(a + j * 32, 16u, 1024u)
                                                    : tc_desc(a + j * 2048, kTmaABytes / 2, 1024u));
        const uint64_t db = kSwizzle128 | (b_kmajor ? tc_desc(b + j * 32, 16u, 1024u)
                                                    : tc_desc(b + j * 2048, kTmaABytes / 2, 1024u));
        const uint32_t acc = (first && j == 0) ? 0u : 1u;
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d), "l"(da),
            "l"(db), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
            : "memory");
    }
}

// arrives on `bar` once every tcgen05 operation this thread issued so far has completed
__device__ __forceinline__ void mma_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     tc_smem_addr(bar))
                 : "memory");
}

// epilogue of one warp: its 32 accumulator rows (TMEM lanes lane0 .. lane0 + 31,
// columns col0 .. col0 + TN2 - 1) as C rows m0 + lane0 + lane, columns n0 ..;
// alpha x acc (+ beta C), or atomically added under split-K
__device__ __forceinline__ void store_tile_rows(uint32_t tmem, int lane0, int col0, int lane, int m0, int n0, int M,
                                                int N, float *C, int ldc, float alpha, float beta, bool split)
{
    const int row = m0 + lane0 + lane;
    const bool vec = !split && beta == 0.f && (ldc & 3) == 0 && (reinterpret_cast<uintptr_t>(C) & 15) == 0;
#pragma unroll 1
    for (int c0 = 0; c0 < TN2; c0 += 16) {
        uint32_t r[16];
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
            "[%16];"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
              "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
            : "r"(tmem + ((uint32_t)lane0 << 16) + (uint32_t)(col0 + c0)));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (row < M) {
            float *crow = C + (int64_t)row * ldc;
            if (vec && n0 + c0 + 16 <= N) {
#pragma unroll
                for (int i = 0; i < 16; i += 4)
                    *reinterpret_cast<float4 *>(crow + n0 + c0 + i) =
                        make_float4(alpha * __uint_as_float(r[i]), alpha * __uint_as_float(r[i + 1]),
                                    alpha * __uint_as_float(r[i + 2]), alpha * __uint_as_float(r[i + 3]));
            } else {
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    const int col = n0 + c0 + i;
                    if (col < N) {
                        float *p = crow + col;
                        const float v = alpha * __uint_as_float(r[i]);
                        if (split)
                            atomicAdd(p, v);
                        else
                            *p = (beta != 0.f) ? v + beta * (*p) : v;
                    }
                }
            }
        }
    }
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(tc_smem_addr(bar)), "r"(count) : "memory");
}

__global__ void __launch_bounds__(128) gemm_tma_kernel(const __grid_constant__ CUtensorMap mapA,
                                                       const __grid_constant__ CUtensorMap mapB, int a_kmajor,
                                                       int b_kmajor, int M, int N, int K, float *C, int ldc,
                                                       float alpha, float beta, int k_per_split, int a_tx,
                                                       int a_two, int *err_flag)
{
    extern __shared__ unsigned char tma_raw[];
    TmaSmem &sm = *reinterpret_cast<TmaSmem *>((reinterpret_cast<uintptr_t>(tma_raw) + 1023) & ~uintptr_t(1023));
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.y * TM, n0 = blockIdx.x * TN2;
    const int kbeg = blockIdx.z * k_per_split;
    const int kend = min(K, kbeg + k_per_split);
    const int nk = kend > kbeg ? (kend - kbeg + TK - 1) / TK : 0;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc_smem_addr(&sm.tmem)),
                     "r"(TN2)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        sm.err = 0;
        for (int s = 0; s < kTmaStages; ++s) {
            mbar_init(&sm.full[s], 1);
            mbar_init(&sm.empty[s], 1);
        }
        mbar_init(&sm.done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = sm.tmem;

    if (tid == 0) {
        // producer: stage s = kt % kTmaStages takes load kt once the MMAs of load kt - kTmaStages are done
        int issued = 0;
        for (int kt = 0; kt < nk; ++kt) {
            const int s = kt % kTmaStages;
            if (kt >= kTmaStages && !tc_wait(&sm.empty[s], (uint32_t)((kt / kTmaStages) - 1) & 1u)) {
                sm.err = 1;
                break;
            }
            tma_stage_loads(sm.a[s], sm.b[s], &mapA, &mapB, a_kmajor, b_kmajor, a_tx, a_two, m0, n0,
                            kbeg + kt * TK, &sm.full[s]);
            issued = kt + 1;
        }
        // the loads still in flight land before the CTA can leave: the last one of each stage
        for (int s = 0; s < kTmaStages && s < issued; ++s) {
            const int uses = (issued - 1 - s) / kTmaStages + 1;
            if (!tc_wait(&sm.full[s], (uint32_t)(uses - 1) & 1u)) sm.err = 1;
        }
    } else if (tid == 32) {
        // MMA issuer
        const uint32_t idesc = kTmaIdesc | (a_kmajor ? 0u : 1u << 15) | (b_kmajor ? 0u : 1u << 16);
        for (int kt = 0; kt < nk; ++kt) {
            const int s = kt % kTmaStages;
            if (!tc_wait(&sm.full[s], (uint32_t)(kt / kTmaStages) & 1u)) {
                sm.err = 1;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            mma_kstep(tmem, sm.a[s], sm.b[s], a_kmajor, b_kmajor, idesc, kt == 0);
            mma_commit(&sm.empty[s]);
        }
        mma_commit(&sm.done);  // arrives once every MMA issued above has completed
    }
    if (!tc_wait(&sm.done, 0u)) sm.err = 1;
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (nk > 0 && !sm.err)
        store_tile_rows(tmem, warp * 32, 0, lane, m0, n0, M, N, C, ldc, alpha, beta, gridDim.z > 1);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TN2) : "memory");
    }
    if (tid == 0 && sm.err) atomicOr(err_flag, 1);
}

// ---------------------------------------------------------------------------
// Persistent form of the same GEMM (no split-K): one CTA per SM walks the
// output tiles t = blockIdx.x, blockIdx.x + gridDim.x, ... (128 x 64 each, M
// fastest), with the roles split over its six warps so that a tile's epilogue
// overlaps the next tile's loads and MMAs:
//   warp 0 (one thread) -- TMA producer: every K step of every tile through a
//     ring of kPStages shared-memory stages (full / empty mbarriers);
//   warp 1 (one thread) -- MMA issuer: tcgen05.mma into one of two TMEM
//     accumulators (64 columns each), committed to the stage's empty barrier
//     and, after a tile's last K step, to the accumulator's full barrier;
//   warps 2..5 -- epilogue: tcgen05.ld of their 32 TMEM lanes (warp w reads
//     lanes 32 (w % 4) ..), alpha / beta, stores; then they release the
//     accumulator (its empty barrier, one arrival per warp).
// Shared memory, descriptors, boxes and the instruction descriptor are those
// of gemm_tma_kernel.  Every wait is bounded: a role that gives up marks the
// CTA and stops, the others then give up at their next wait; before the TMEM
// columns are freed the producer waits (bounded) for its loads in flight and
// every thread for the MMAs issued.
// ---------------------------------------------------------------------------
constexpr int kPStages = 8;  // 8 x 24 KB: one CTA per SM
constexpr int kPThreads = 192;

struct PersistSmem {
    alignas(1024) unsigned char a[kPStages][kTmaABytes];
    alignas(1024) unsigned char b[kPStages][kTmaBBytes];
    uint64_t full[kPStages], empty[kPStages], acc_full[2], acc_empty[2], done;
    uint32_t tmem;
    int err;
};
constexpr int kPersistSmemBytes = (int)sizeof(PersistSmem) + 1024;

__global__ void __launch_bounds__(kPThreads, 1) gemm_tma_persistent_kernel(
    const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB, int a_kmajor, int b_kmajor,
    int M, int N, int K, float *C, int ldc, float alpha, float beta, int a_tx, int a_two, int *err_flag)
{
    extern __shared__ unsigned char tma_raw[];
    PersistSmem &sm =
        *reinterpret_cast<PersistSmem *>((reinterpret_cast<uintptr_t>(tma_raw) + 1023) & ~uintptr_t(1023));
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int tiles_m = (M + TM - 1) / TM, tiles = tiles_m * ((N + TN2 - 1) / TN2);
    const int nk = (K + TK - 1) / TK;
    const int my_tiles = blockIdx.x < tiles ? (tiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc_smem_addr(&sm.tmem)),
                     "r"(2 * TN2)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        sm.err = 0;
        for (int s = 0; s < kPStages; ++s) {
            mbar_init(&sm.full[s], 1);
            mbar_init(&sm.empty[s], 1);
        }
        for (int a = 0; a < 2; ++a) {
            mbar_init(&sm.acc_full[a], 1);
            mbar_init(&sm.acc_empty[a], 4);  // one arrival per epilogue warp
        }
        mbar_init(&sm.done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = sm.tmem;

    if (tid == 0) {
        // producer: load g (g-th K step of this CTA) goes to stage g % kPStages once the
        // MMAs of load g - kPStages have released it
        int g = 0;
        bool ok = true;
        for (int i = 0; i < my_tiles && ok; ++i) {
            const int t = blockIdx.x + i * gridDim.x;
            const int m0 = (t % tiles_m) * TM, n0 = (t / tiles_m) * TN2;
            for (int kt = 0; kt < nk; ++kt, ++g) {
                const int s = g % kPStages;
                if (g >= kPStages && !tc_wait(&sm.empty[s], (uint32_t)((g / kPStages) - 1) & 1u)) {
                    sm.err = 1;
                    ok = false;
                    break;
                }
                tma_stage_loads(sm.a[s], sm.b[s], &mapA, &mapB, a_kmajor, b_kmajor, a_tx, a_two, m0, n0, kt * TK,
                                &sm.full[s]);
            }
        }
        // the loads still in flight land before the CTA can leave: the last one of each stage
        for (int s = 0; s < kPStages && s < g; ++s) {
            const int uses = (g - 1 - s) / kPStages + 1;
            if (!tc_wait(&sm.full[s], (uint32_t)(uses - 1) & 1u)) sm.err = 1;
        }
    } else if (tid == 32) {
        // MMA issuer
        int g = 0;
        bool ok = true;
        const uint32_t idesc = kTmaIdesc | (a_kmajor ? 0u : 1u << 15) | (b_kmajor ? 0u : 1u << 16);
        for (int i = 0; i < my_tiles && ok; ++i) {
            const int acc = i & 1;
            if (i >= 2 && !tc_wait(&sm.acc_empty[acc], (uint32_t)((i >> 1) - 1) & 1u)) {
                sm.err = 1;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t d = tmem + (uint32_t)(acc * TN2);
            for (int kt = 0; kt < nk; ++kt, ++g) {
                const int s = g % kPStages;
                if (!tc_wait(&sm.full[s], (uint32_t)(g / kPStages) & 1u)) {
                    sm.err = 1;
                    ok = false;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                mma_kstep(d, sm.a[s], sm.b[s], a_kmajor, b_kmajor, idesc, kt == 0);
                mma_commit(&sm.empty[s]);
            }
            if (ok) mma_commit(&sm.acc_full[acc]);
        }
        mma_commit(&sm.done);  // arrives once every MMA issued above has completed
    } else if (warp >= 2) {
        // epilogue: warp w owns TMEM lanes 32 (w % 4) .. + 31, i.e. tile rows of that quarter
        const int quarter = warp & 3;
        for (int i = 0; i < my_tiles; ++i) {
            const int acc = i & 1;
            // one decision for the warp: the TMEM loads below are warp-collective
            if (!__all_sync(0xffffffffu, tc_wait(&sm.acc_full[acc], (uint32_t)(i >> 1) & 1u))) {
                sm.err = 1;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const int t = blockIdx.x + i * gridDim.x;
            store_tile_rows(tmem, quarter * 32, acc * TN2, lane, (t % tiles_m) * TM, (t / tiles_m) * TN2, M, N, C,
                            ldc, alpha, beta, false);
            // this warp is done reading the accumulator: the MMAs of tile i + 2 may overwrite it
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0)
                asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(tc_smem_addr(&sm.acc_empty[acc]))
                             : "memory");
        }
    }
    // the role threads wait for the last MMAs; the idle lanes of warps 0 and 1 go
    // straight to the barrier (no polling beside the producer and the issuer)
    if ((tid == 0 || tid == 32 || warp >= 2) && !tc_wait(&sm.done, 0u)) sm.err = 1;
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * TN2) : "memory");
    }
    if (tid == 0 && sm.err) atomicOr(err_flag, 1);
}

__global__ void scale_kernel(float *C, int M, int N, int ldc, float beta)
{
    const int64_t n = (int64_t)M * N;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        float *p = &C[(k / N) * ldc + k % N];
        *p = beta == 0.f ? 0.f : beta * *p;
    }
}

// ---------------------------------------------------------------------------
// convolution helpers, activations [C][B][H][W] (FP32) / columns (BF16)
// ---------------------------------------------------------------------------
// grid: x over the output pixels n (256 per block), y over the rows c * 9 + tap
// of col; pixel coordinates from 32-bit divisions once per thread
__global__ void im2col3_kernel(const float *X, int C, int B, int H, int W, bf16 *col)
{
    const int N = B * H * W;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    const int row = blockIdx.y;
    const int c = row / 9, tap = row - 9 * (row / 9), dy = tap / 3 - 1, dx = tap % 3 - 1;
    const int q = n / W, w = n - q * W;
    const int b = q / H, h = q - b * H;
    const int hh = h + dy, ww = w + dx;
    float v = 0.f;
    if (hh >= 0 && hh < H && ww >= 0 && ww < W) v = X[((int64_t)c * B + b) * H * W + (int64_t)hh * W + ww];
    col[(int64_t)row * N + n] = __float2bfloat16(v);
}

// dX[c][b][h][w] = sum over taps of dcol[c*9+tap][output pixel that read (h,w) through that tap];
// grid: x over the pixels (256 per block), y over the channels
__global__ void col2im3_kernel(const float *dcol, int C, int B, int H, int W, float *dX)
{
    const int N = B * H * W;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    const int c = blockIdx.y;
    const int q = n / W, w = n - q * W;
    const int b = q / H, h = q - b * H;
    float s = 0.f;
#pragma unroll
    for (int tap = 0; tap < 9; ++tap) {
        const int dy = tap / 3 - 1, dx = tap % 3 - 1;
        const int ho = h - dy, wo = w - dx;
        if (ho >= 0 && ho < H && wo >= 0 && wo < W)
            s += dcol[(int64_t)(c * 9 + tap) * N + (b * H + ho) * W + wo];
    }
    dX[(int64_t)c * N + n] = s;
}

// The same convolution helpers, several pixels per thread (used when the image
// rows allow): identical values and summation order, 32-bit index arithmetic
// once per thread, 16-byte loads and stores.
//
// im2col, W % 8 == 0: a thread takes 8 consecutive pixels of one image row and
// writes all 9 taps of one channel (grid: x over the 8-pixel groups, y over C)
__global__ void im2col3_vec8_kernel(const float *X, int H, int W, int N, bf16 *col)
{
    const int n0 = 8 * (blockIdx.x * blockDim.x + threadIdx.x);
    if (n0 >= N) return;
    const int c = blockIdx.y;
    const int q = n0 / W, w0 = n0 - q * W, h = q % H;  // q = b H + h
    const float *xc = X + (int64_t)c * N;
#pragma unroll
    for (int dy = -1; dy <= 1; ++dy) {
        float v[10];  // source columns w0 - 1 .. w0 + 8 of image row h + dy (zero outside the image)
        if (h + dy >= 0 && h + dy < H) {
            const float *r = xc + (int64_t)(q + dy) * W;
            const float4 a = *reinterpret_cast<const float4 *>(r + w0);
            const float4 b = *reinterpret_cast<const float4 *>(r + w0 + 4);
            v[0] = w0 > 0 ? r[w0 - 1] : 0.f;
            v[1] = a.x, v[2] = a.y, v[3] = a.z, v[4] = a.w;
            v[5] = b.x, v[6] = b.y, v[7] = b.z, v[8] = b.w;
            v[9] = w0 + 8 < W ? r[w0 + 8] : 0.f;
        } else {
#pragma unroll
            for (int i = 0; i < 10; ++i) v[i] = 0.f;
        }
#pragma unroll
        for (int dx = -1; dx <= 1; ++dx) {
            const int tap = 3 * (dy + 1) + dx + 1;
            uint32_t w[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const __nv_bfloat162 t = __floats2bfloat162_rn(v[2 * i + 1 + dx], v[2 * i + 2 + dx]);
                w[i] = *reinterpret_cast<const uint32_t *>(&t);
            }
            *reinterpret_cast<uint4 *>(col + (int64_t)(c * 9 + tap) * N + n0) = make_uint4(w[0], w[1], w[2], w[3]);
        }
    }
}

// col2im, W % 4 == 0: 4 consecutive pixels of one image row per thread, taps in
// the order of col2im3_kernel (grid: x over the 4-pixel groups, y over C)
__global__ void col2im3_vec4_kernel(const float *dcol, int H, int W, int N, float *dX)
{
    const int n0 = 4 * (blockIdx.x * blockDim.x + threadIdx.x);
    if (n0 >= N) return;
    const int c = blockIdx.y;
    const int q = n0 / W, w0 = n0 - q * W, h = q % H;
    float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f;
#pragma unroll
    for (int tap = 0; tap < 9; ++tap) {
        const int dy = tap / 3 - 1, dx = tap % 3 - 1;
        if (h - dy < 0 || h - dy >= H) continue;
        const float *r = dcol + (int64_t)(c * 9 + tap) * N + (int64_t)(q - dy) * W;
        const float4 a = *reinterpret_cast<const float4 *>(r + w0);
        // pixel w0 + i reads column w0 + i - dx of the row
        if (dx == 0) {
            s0 += a.x, s1 += a.y, s2 += a.z, s3 += a.w;
        } else if (dx == 1) {
            if (w0 > 0) s0 += r[w0 - 1];
            s1 += a.x, s2 += a.y, s3 += a.z;
        } else {
            s0 += a.y, s1 += a.z, s2 += a.w;
            if (w0 + 4 < W) s3 += r[w0 + 4];
        }
    }
    *reinterpret_cast<float4 *>(dX + (int64_t)c * N + n0) = make_float4(s0, s1, s2, s3);
}

// float -> bfloat16, four values per thread (n % 4 == 0, 16-byte aligned)
__global__ void cast_bf16_vec4_kernel(const float4 *x, uint2 *y, int64_t n4)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n4; k += (int64_t)gridDim.x * blockDim.x) {
        const float4 v = x[k];
        const __nv_bfloat162 a = __floats2bfloat162_rn(v.x, v.y), b = __floats2bfloat162_rn(v.z, v.w);
        y[k] = make_uint2(*reinterpret_cast<const uint32_t *>(&a), *reinterpret_cast<const uint32_t *>(&b));
    }
}

// bias (+ ReLU), N % 4 == 0: grid y over the channels, x over the channel's float4s
__global__ void bias_act_vec4_kernel(float4 *Y, const float *bias, int64_t n4, int relu)
{
    const float b = bias[blockIdx.y];
    float4 *row = Y + (int64_t)blockIdx.y * n4;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n4; k += (int64_t)gridDim.x * blockDim.x) {
        float4 v = row[k];
        v.x += b, v.y += b, v.z += b, v.w += b;
        if (relu) v.x = fmaxf(v.x, 0.f), v.y = fmaxf(v.y, 0.f), v.z = fmaxf(v.z, 0.f), v.w = fmaxf(v.w, 0.f);
        row[k] = v;
    }
}

__global__ void relu_bwd_vec4_kernel(float4 *dY, const float4 *Y, int64_t n4)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n4; k += (int64_t)gridDim.x * blockDim.x) {
        const float4 y = Y[k];
        float4 d = dY[k];
        if (!(y.x > 0.f)) d.x = 0.f;
        if (!(y.y > 0.f)) d.y = 0.f;
        if (!(y.z > 0.f)) d.z = 0.f;
        if (!(y.w > 0.f)) d.w = 0.f;
        dY[k] = d;
    }
}

__global__ void axpy_vec4_kernel(float4 *y, const float4 *x, float a, int64_t n4)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n4; k += (int64_t)gridDim.x * blockDim.x) {
        const float4 u = x[k];
        float4 v = y[k];
        v.x += a * u.x, v.y += a * u.y, v.z += a * u.z, v.w += a * u.w;
        y[k] = v;
    }
}

// 2x2 pooling / nearest upsampling and their gradients, one plane per grid row
// (y), four input or output columns per thread (W % 4 == 0 for pooling, w % 2
// == 0 for upsampling), the sums in the scalar kernels' order
__global__ void pool2_vec_kernel(const float *X, int H, int W, float *Y)
{
    const int h2 = H / 2, w2 = W / 2;
    const int k = 2 * (blockIdx.x * blockDim.x + threadIdx.x);  // first of two outputs
    if (k >= h2 * w2) return;
    const int h = k / w2, w = k - h * w2;
    const float *x = X + (int64_t)blockIdx.y * H * W + (int64_t)(2 * h) * W + 2 * w;
    const float4 a = *reinterpret_cast<const float4 *>(x), b = *reinterpret_cast<const float4 *>(x + W);
    *reinterpret_cast<float2 *>(Y + (int64_t)blockIdx.y * h2 * w2 + k) =
        make_float2(0.25f * (a.x + a.y + b.x + b.y), 0.25f * (a.z + a.w + b.z + b.w));
}

__global__ void pool2_bwd_vec_kernel(const float *dY, int H, int W, float *dX)
{
    const int h2 = H / 2, w2 = W / 2;
    const int k = 4 * (blockIdx.x * blockDim.x + threadIdx.x);  // first of four outputs
    if (k >= H * W) return;
    const int h = k / W, w = k - h * W;
    const float *d = dY + (int64_t)blockIdx.y * h2 * w2 + (int64_t)(h / 2) * w2 + w / 2;
    const float u = 0.25f * d[0], v = 0.25f * d[1];
    *reinterpret_cast<float4 *>(dX + (int64_t)blockIdx.y * H * W + k) = make_float4(u, u, v, v);
}

__global__ void up2_vec_kernel(const float *X, int h, int w, float *Y)
{
    const int W = 2 * w, H = 2 * h;
    const int k = 4 * (blockIdx.x * blockDim.x + threadIdx.x);
    if (k >= H * W) return;
    const int y = k / W, x = k - y * W;
    const float *s = X + (int64_t)blockIdx.y * h * w + (int64_t)(y / 2) * w + x / 2;
    const float u = s[0], v = s[1];
    *reinterpret_cast<float4 *>(Y + (int64_t)blockIdx.y * H * W + k) = make_float4(u, u, v, v);
}

__global__ void up2_bwd_vec_kernel(const float *dY, int h, int w, float *dX)
{
    const int W = 2 * w;
    const int k = 2 * (blockIdx.x * blockDim.x + threadIdx.x);
    if (k >= h * w) return;
    const int y = k / w, x = k - y * w;
    const float *d = dY + (int64_t)blockIdx.y * 4 * h * w + (int64_t)(2 * y) * W + 2 * x;
    const float4 a = *reinterpret_cast<const float4 *>(d), b = *reinterpret_cast<const float4 *>(d + W);
    *reinterpret_cast<float2 *>(dX + (int64_t)blockIdx.y * h * w + k) =
        make_float2(a.x + a.y + b.x + b.y, a.z + a.w + b.z + b.w);
}

// Weights of a 3x3 convolution, w[co][ci*9 + tap] (BF16), rearranged for the
// gradient with respect to its input: wt[ci][co*9 + t] = w[co][ci*9 + 8 - t]
// (transposed, taps turned by 180 degrees: the adjoint of a zero-padded 3x3
// convolution is the convolution of dY with these weights), columns
// cout*9 .. ldo-1 zero.  One thread per output value.
__global__ void flip3_kernel(const bf16 *w, int cout, int cin, int ldo, bf16 *wt)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= cin * ldo) return;
    const int ci = k / ldo, j = k - ci * ldo;
    bf16 v = __float2bfloat16(0.f);
    if (j < cout * 9) {
        const int co = j / 9, t = j - 9 * co;
        v = w[(int64_t)co * cin * 9 + ci * 9 + 8 - t];
    }
    wt[k] = v;
}

// rows x cols BF16 values into rows x ldo (columns cols .. ldo-1 zero)
__global__ void pad_cols_kernel(const bf16 *w, int rows, int cols, int ldo, bf16 *out)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= rows * ldo) return;
    const int r = k / ldo, c = k - r * ldo;
    out[k] = c < cols ? w[(int64_t)r * cols + c] : __float2bfloat16(0.f);
}

__global__ void cast_bf16_kernel(const float *x, bf16 *y, int64_t n)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
        y[k] = __float2bfloat16(x[k]);
}

__global__ void bias_act_kernel(float *Y, const float *bias, int C, int64_t N, int relu)
{
    const int64_t total = (int64_t)C * N;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total;
         k += (int64_t)gridDim.x * blockDim.x) {
        float v = Y[k] + bias[k / N];
        Y[k] = relu ? fmaxf(v, 0.f) : v;
    }
}

__global__ void relu_bwd_kernel(float *dY, const float *Y, int64_t n)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
        if (!(Y[k] > 0.f)) dY[k] = 0.f;
}

// db[c] = sum_n dY[c][n]; one block per channel, fixed reduction order
// one block of 1024 threads per channel; four values per load where the row allows
__global__ void bias_grad_kernel(const float *dY, int64_t N, float *db)
{
    __shared__ float red[32];
    const int c = blockIdx.x;
    const float *row = dY + (int64_t)c * N;
    float s = 0.f;
    if ((N & 3) == 0 && (reinterpret_cast<uintptr_t>(row) & 15) == 0) {
        const float4 *r4 = reinterpret_cast<const float4 *>(row);
        for (int64_t n = threadIdx.x; n < N / 4; n += blockDim.x) {
            const float4 v = r4[n];
            s += (v.x + v.y) + (v.z + v.w);
        }
    } else {
        for (int64_t n = threadIdx.x; n < N; n += blockDim.x) s += row[n];
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        float t = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.f;
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
        if (threadIdx.x == 0) db[c] = t;
    }
}

// 2x2 average pooling: X [C*B][H][W] -> Y [C*B][H/2][W/2]
__global__ void pool2_kernel(const float *X, int CB, int H, int W, float *Y)
{
    const int h2 = H / 2, w2 = W / 2;
    const int64_t total = (int64_t)CB * h2 * w2;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total;
         k += (int64_t)gridDim.x * blockDim.x) {
        const int w = (int)(k % w2), h = (int)((k / w2) % h2);
        const int64_t p = k / ((int64_t)h2 * w2);
        const float *x = X + p * H * W + (int64_t)(2 * h) * W + 2 * w;
        Y[k] = 0.25f * (x[0] + x[1] + x[W] + x[W + 1]);
    }
}

__global__ void pool2_bwd_kernel(const float *dY, int CB, int H, int W, float *dX)
{
    const int64_t total = (int64_t)CB * H * W;
    const int h2 = H / 2, w2 = W / 2;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total;
         k += (int64_t)gridDim.x * blockDim.x) {
        const int w = (int)(k % W), h = (int)((k / W) % H);
        const int64_t p = k / ((int64_t)H * W);
        dX[k] = 0.25f * dY[p * h2 * w2 + (int64_t)(h / 2) * w2 + w / 2];
    }
}

// nearest 2x upsampling: X [C*B][h][w] -> Y [C*B][2h][2w]
__global__ void up2_kernel(const float *X, int CB, int h, int w, float *Y)
{
    const int H = 2 * h, W = 2 * w;
    const int64_t total = (int64_t)CB * H * W;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total;
         k += (int64_t)gridDim.x * blockDim.x) {
        const int x = (int)(k % W), y = (int)((k / W) % H);
        const int64_t p = k / ((int64_t)H * W);
        Y[k] = X[p * h * w + (int64_t)(y / 2) * w + x / 2];
    }
}

__global__ void up2_bwd_kernel(const float *dY, int CB, int h, int w, float *dX)
{
    const int64_t total = (int64_t)CB * h * w;
    const int W = 2 * w;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total;
         k += (int64_t)gridDim.x * blockDim.x) {
        const int x = (int)(k % w), y = (int)((k / w) % h);
        const int64_t p = k / ((int64_t)h * w);
        const float *d = dY + p * 4 * h * w + (int64_t)(2 * y) * W + 2 * x;
        dX[k] = d[0] + d[1] + d[W] + d[W + 1];
    }
}

__global__ void axpy_kernel(float *y, const float *x, float a, int64_t n)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
        y[k] += a * x[k];
}

// grad = 2 (pred - target) / n ; loss partials summed per block then atomically
__global__ void mse_kernel(const float *pred, const float *target, int64_t n, float *grad, float *loss)
{
    __shared__ float red[256];
    float s = 0.f;
    const float inv = 2.f / (float)n;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const float d = pred[k] - target[k];
        if (grad) grad[k] = inv * d;
        s += d * d;
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0 && loss) atomicAdd(loss, red[0] / (float)n);
}

__global__ void adam_kernel(float *w, const float *g, float *m, float *v, bf16 *wb, int64_t n, float lr, float b1,
                            float b2, float eps, float c1, float c2, float wd)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const float gk = g[k] + wd * w[k];
        const float mk = b1 * m[k] + (1.f - b1) * gk;
        const float vk = b2 * v[k] + (1.f - b2) * gk * gk;
        m[k] = mk;
        v[k] = vk;
        const float wk = w[k] - lr * (mk * c1) / (sqrtf(vk * c2) + eps);
        w[k] = wk;
        if (wb) wb[k] = __float2bfloat16(wk);
    }
}

// all tensors of a network in one launch: blockIdx.y picks the tensor, the step's
// scalars come from device memory (hyper = lr, b1, b2, eps, c1, c2)
__global__ void adam_multi_kernel(const amhd_nn_tensor *ts, const float *hyper)
{
    const amhd_nn_tensor t = ts[blockIdx.y];
    const float lr = hyper[0], b1 = hyper[1], b2 = hyper[2], eps = hyper[3], c1 = hyper[4], c2 = hyper[5];
    bf16 *wb = static_cast<bf16 *>(t.w_bf16);
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < t.n; k += (int64_t)gridDim.x * blockDim.x) {
        const float gk = t.g[k] + t.weight_decay * t.w[k];
        const float mk = b1 * t.m[k] + (1.f - b1) * gk;
        const float vk = b2 * t.v[k] + (1.f - b2) * gk * gk;
        t.m[k] = mk;
        t.v[k] = vk;
        const float wk = t.w[k] - lr * (mk * c1) / (sqrtf(vk * c2) + eps);
        t.w[k] = wk;
        if (wb) wb[k] = __float2bfloat16(wk);
    }
}

// ---------------------------------------------------------------------------
// solver <-> network data movement
// ---------------------------------------------------------------------------
// coarse interior cell (i, j) = mean of the fine interior cells [f i, f i + f) x [f j, f j + f)
template <typename R>
__global__ void restrict_kernel(const R *Uf, int pitch_f, int64_t vs_f, int nxc, int nyc, int f, float *out,
                                int64_t out_vs, int b, int B)
{
    const int64_t total = (int64_t)10 * nxc * nyc;
    const float inv = 1.f / (float)(f * f);
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total;
         k += (int64_t)gridDim.x * blockDim.x) {
        const int j = (int)(k % nyc), i = (int)((k / nyc) % nxc), v = (int)(k / ((int64_t)nxc * nyc));
        double s = 0.0;
        for (int a = 0; a < f; ++a)
            for (int c = 0; c < f; ++c)
                s += (double)Uf[v * vs_f + (int64_t)(2 + f * i + a) * pitch_f + 2 + f * j + c];
        out[(int64_t)v * out_vs + ((int64_t)b * nxc + i) * nyc + j] = (float)(s * inv);
    }
}

// pack a solver state's interior into the network input x[v][b][i][j] = (U - mean_v) / std_v
template <typename R>
__global__ void pack_kernel(const R *U, int pitch, int64_t vs, int nx, int ny, const float *mean, const float *istd,
                            float *x, int64_t x_vs, int b)
{
    const int64_t total = (int64_t)10 * nx * ny;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total;
         k += (int64_t)gridDim.x * blockDim.x) {
        const int j = (int)(k % ny), i = (int)((k / ny) % nx), v = (int)(k / ((int64_t)nx * ny));
        const float u = (float)U[v * vs + (int64_t)(i + 2) * pitch + j + 2];
        x[(int64_t)v * x_vs + ((int64_t)b * nx + i) * ny + j] = (u - mean[v]) * istd[v];
    }
}

// U_interior += scale_v * y[v][b][i][j] (the network's correction), then the caller refreshes ghosts
template <typename R>
__global__ void apply_kernel(R *U, int pitch, int64_t vs, int nx, int ny, const float *scale, const float *y,
                             int64_t y_vs, int b)
{
    const int64_t total = (int64_t)10 * nx * ny;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total;
         k += (int64_t)gridDim.x * blockDim.x) {
        const int j = (int)(k % ny), i = (int)((k / ny) % nx), v = (int)(k / ((int64_t)nx * ny));
        R *u = &U[v * vs + (int64_t)(i + 2) * pitch + j + 2];
        *u = *u + (R)(scale[v] * y[(int64_t)v * y_vs + ((int64_t)b * nx + i) * ny + j]);  // in the state's precision
    }
}

// The same, cell by cell and kept admissible: U_cell += alpha scale_v y[v] only
// when the corrected cell is finite and keeps at least min_ratio of its
// density and of its pressure p = (gamma-1)(E - |m|^2/2rho - |B|^2/2) (float64);
// otherwise the cell keeps its state and *rejected counts it.  mode: 0 the
// correction as is; 1 the passive scalar's correction scaled by 4 C (1 - C) of
// the cell (none in unmixed fluid); 2 no scalar correction; 3 every variable's
// correction scaled by 4 C (1 - C) (corrections only in the mixing layer).
template <typename R>
__global__ void apply_guarded_kernel(R *U, int pitch, int64_t vs, int nx, int ny, double gamma, const float *scale,
                                     const float *y, int64_t y_vs, int b, float alpha, float min_ratio,
                                     int scalar_mode, int *rejected)
{
    const int64_t total = (int64_t)nx * ny;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total;
         k += (int64_t)gridDim.x * blockDim.x) {
        const int j = (int)(k % ny), i = (int)(k / ny);
        const int64_t c = (int64_t)(i + 2) * pitch + j + 2;
        const int64_t yc = ((int64_t)b * nx + i) * ny + j;
        double u[10], w[10];
        bool ok = true;
        const double cc = fmin(fmax((double)U[9 * vs + c] / fmax((double)U[c], 1e-12), 0.0), 1.0);
        const float mix = float(4.0 * cc * (1.0 - cc));
        const float sfac = scalar_mode == 0 ? 1.f : (scalar_mode == 2 ? 0.f : mix);
        const float ofac = scalar_mode == 3 ? mix : 1.f;
#pragma unroll
        for (int v = 0; v < 10; ++v) {
            u[v] = (double)U[v * vs + c];
            const float a = v == 9 ? alpha * sfac : alpha * ofac;
            w[v] = (double)(R)(U[v * vs + c] + (R)(a * scale[v] * y[(int64_t)v * y_vs + yc]));
            ok = ok && isfinite(w[v]);
        }
        auto pressure = [&](const double *s) {
            const double m2 = s[1] * s[1] + s[2] * s[2] + s[3] * s[3];
            const double b2 = s[4] * s[4] + s[5] * s[5] + s[6] * s[6];
            return (gamma - 1.0) * (s[7] - 0.5 * m2 / s[0] - 0.5 * b2);
        };
        if (ok) ok = u[0] > 0.0 && w[0] >= (double)min_ratio * u[0];
        if (ok) ok = pressure(w) >= (double)min_ratio * pressure(u);
        if (ok) {
#pragma unroll
            for (int v = 0; v < 10; ++v) U[v * vs + c] = (R)w[v];
        } else if (rejected != nullptr) {
            atomicAdd(rejected, 1);
        }
    }
}

}  // namespace

namespace {

using EncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                   const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn nn_encoder()
{
    static EncodeTiledFn fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void *ptr = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(ptr);
    }
    return fn;
}

// tensor map of one GEMM operand (layouts at gemm_tma_kernel): rows = M or N,
// kmajor = the source is contiguous along K.  false: not expressible (base not
// 16-byte aligned, ld not a multiple of 8) or refused by the driver; the
// caller stages with threads instead.
bool operand_map(CUtensorMap *map, const void *base, int ld, int rows, int K, int tile_rows, bool kmajor)
{
    EncodeTiledFn fn = nn_encoder();
    if (!fn || (reinterpret_cast<uintptr_t>(base) & 15) || ld % 8 || K <= 0 || rows <= 0) return false;
    if (ld < (kmajor ? K : rows)) return false;
    const cuuint32_t estr[2] = {1, 1};
    const cuuint64_t dims[2] = {(cuuint64_t)(kmajor ? K : rows), (cuuint64_t)(kmajor ? rows : K)};
    const cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
    const cuuint32_t box[2] = {64, (cuuint32_t)(kmajor ? tile_rows : TK)};
    const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(base), dims, strides, box,
                          estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

std::atomic<long long> g_tc_tma_launches{0}, g_tc_staged_launches{0};
std::atomic<int> g_gemm_path{0};  // amhd_nn_set_gemm_path
std::atomic<int> g_persistent{1};  // amhd_nn_set_gemm_persistent

// multiprocessors of the current device (the persistent GEMM's grid)
int nn_sm_count()
{
    int dev = 0, n = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0)
        return kNumSMs;
    return n;
}

// split-K: K per split rounded up to whole K steps of `step`; returns the split count
int split_k(int K, int splits, int step, int *kps_out)
{
    if (splits < 1) splits = 1;
    int kps = (K + splits - 1) / splits;
    kps = (kps + step - 1) / step * step;
    if (kps < step) kps = step;
    *kps_out = kps;
    return K > 0 ? (K + kps - 1) / kps : 1;
}

// the TMA-fed tcgen05 GEMM, if both operands have tensor maps; *launched = false
// (and nothing enqueued) otherwise
int tma_gemm(int transA, int transB, int M, int N, int K, const void *A, int lda, const void *B, int ldb, float *C,
             int ldc, float alpha, float beta, int splits, cudaStream_t s, bool *launched)
{
    *launched = false;
    const bool a_kmajor = !transA, b_kmajor = transB != 0;
    // A boxes no taller than M needs (rounded to whole 8-row swizzle atoms; a
    // K-major box of R rows delivers R x 128 bytes, an MN-major A of M <= 64 rows
    // takes one of its two 64-row boxes): the rows past the box are whatever the
    // stage held before and only reach accumulator rows that are never stored
    const int a_rows = a_kmajor ? std::min(TM, (M + 7) / 8 * 8) : TM;
    const int a_two = a_kmajor ? 0 : (M > TM / 2 ? 1 : 0);
    const int a_tx = a_kmajor ? a_rows * TK * 2 : (a_two ? kTmaABytes : kTmaABytes / 2);
    CUtensorMap map_a, map_b;
    if (K <= 0 || !operand_map(&map_a, A, lda, M, K, a_rows, a_kmajor) ||
        !operand_map(&map_b, B, ldb, N, K, TN2, b_kmajor))
        return AMHD_OK;
    // function attributes are per device: set on every call (cheap), so that any
    // device current in this thread has the opt-in before the launch
    NNCK(cudaFuncSetAttribute(gemm_tma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kTmaSmemBytes));
    int *err = nullptr;
    NNCK(cudaGetSymbolAddress(reinterpret_cast<void **>(&err), g_tc_err));
    const int tiles = ((N + TN2 - 1) / TN2) * ((M + TM - 1) / TM);
    if (splits > 1) {
        // the caller accepted an atomic split-K: take enough splits for about
        // 2 CTAs per SM, each with at least 4 K steps
        const int want = (2 * kNumSMs + tiles - 1) / tiles, by_k = K / (4 * TK);
        splits = std::max(splits, std::min(want, by_k));
    }
    int kps;
    splits = split_k(K, splits, TK, &kps);
    if (splits == 1 && g_persistent.load()) {
        // one CTA per SM walks the tiles, each tile's epilogue under the next one's loads
        NNCK(cudaFuncSetAttribute(gemm_tma_persistent_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  kPersistSmemBytes));
        const int grid = std::min(tiles, nn_sm_count());
        gemm_tma_persistent_kernel<<<grid, kPThreads, kPersistSmemBytes, s>>>(map_a, map_b, a_kmajor, b_kmajor, M,
                                                                               N, K, C, ldc, alpha, beta, a_tx, a_two,
                                                                               err);
        NNCK(cudaGetLastError());
        ++g_tc_tma_launches;
        *launched = true;
        return AMHD_OK;
    }
    if (splits > 1) {
        scale_kernel<<<blocks_for((int64_t)M * N), 256, 0, s>>>(C, M, N, ldc, beta);
        NNCK(cudaGetLastError());
    }
    dim3 grid((N + TN2 - 1) / TN2, (M + TM - 1) / TM, splits);
    gemm_tma_kernel<<<grid, 128, kTmaSmemBytes, s>>>(map_a, map_b, a_kmajor, b_kmajor, M, N, K, C, ldc, alpha,
                                                     splits > 1 ? 0.f : beta, kps, a_tx, a_two, err);
    NNCK(cudaGetLastError());
    ++g_tc_tma_launches;
    *launched = true;
    return AMHD_OK;
}

// shapes on which the tcgen05 pipeline beats mma.sync (B200): a full 64-column
// output tile, whatever M (the rows past M are zero-filled by the TMA box and
// not stored: at M = 32 / 10, N = 262144, K = 288 tcgen05 runs 54 / 17 TFLOP/s
// against 29 / 10), or a long K (weight gradients)
bool prefer_tc(int M, int N, int K)
{
    (void)M;
    return N >= 64 || K >= 4096;
}

}  // namespace

#pragma GCC visibility push(default)
extern "C" {

const char *amhd_nn_last_error(void) { return g_nn_err.c_str(); }

int amhd_nn_gemm_tc(int32_t transA, int32_t transB, int32_t M, int32_t N, int32_t K, const void *A, int32_t lda,
                    const void *B, int32_t ldb, float *C, int32_t ldc, float alpha, float beta, int32_t splits,
                    void *stream)
{
    if (M < 0 || N < 0 || K < 0 || !A || !B || !C) return nn_fail(AMHD_ERR_ARG, "bad gemm arguments");
    if (M == 0 || N == 0) return AMHD_OK;
    // function attributes are per device: set on every call (cheap), so that any
    // device current in this thread has the opt-in before the launch
    NNCK(cudaFuncSetAttribute(gemm_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmemBytes));
    cudaStream_t s = S(stream);
    bool launched = false;
    const int rc = tma_gemm(transA, transB, M, N, K, A, lda, B, ldb, C, ldc, alpha, beta, splits, s, &launched);
    if (rc != AMHD_OK || launched) return rc;
    int *err = nullptr;
    NNCK(cudaGetSymbolAddress(reinterpret_cast<void **>(&err), g_tc_err));
    int kps;
    splits = split_k(K, splits, TK, &kps);
    if (splits > 1 || K == 0) {
        scale_kernel<<<blocks_for((int64_t)M * N), 256, 0, s>>>(C, M, N, ldc, beta);
        NNCK(cudaGetLastError());
        if (K == 0) return AMHD_OK;
    }
    ++g_tc_staged_launches;
    dim3 grid((N + TN - 1) / TN, (M + TM - 1) / TM, splits);
    gemm_tc_kernel<<<grid, 128, kTcSmemBytes, s>>>(transA, transB, M, N, K, static_cast<const bf16 *>(A), lda,
                                                   static_cast<const bf16 *>(B), ldb, C, ldc, alpha,
                                                   splits > 1 ? 0.f : beta, kps, err);
    NNCK(cudaGetLastError());
    return AMHD_OK;
}

int amhd_nn_set_gemm_persistent(int32_t on)
{
    if (on != 0 && on != 1) return nn_fail(AMHD_ERR_ARG, "persistent GEMM switch must be 0 or 1, got %d", on);
    g_persistent.store(on);
    return AMHD_OK;
}

int amhd_nn_set_gemm_path(int32_t mode)
{
    if (mode < 0 || mode > 2) return nn_fail(AMHD_ERR_ARG, "gemm path %d (0 auto, 1 mma.sync, 2 tcgen05)", mode);
    g_gemm_path.store(mode);
    return AMHD_OK;
}

int amhd_nn_gemm_tc_paths(int64_t *tma, int64_t *staged)
{
    if (!tma || !staged) return nn_fail(AMHD_ERR_ARG, "NULL output");
    *tma = g_tc_tma_launches.load();
    *staged = g_tc_staged_launches.load();
    return AMHD_OK;
}

int amhd_nn_gemm_status(int32_t *flag)
{
    if (!flag) return nn_fail(AMHD_ERR_ARG, "NULL flag");
    int v = 0, z = 0;
    NNCK(cudaMemcpyFromSymbol(&v, g_tc_err, sizeof v));
    NNCK(cudaMemcpyToSymbol(g_tc_err, &z, sizeof z));
    *flag = v;
    return AMHD_OK;
}

int amhd_nn_gemm(int32_t transA, int32_t transB, int32_t M, int32_t N, int32_t K, const void *A, int32_t lda,
                 const void *B, int32_t ldb, float *C, int32_t ldc, float alpha, float beta, int32_t splits,
                 void *stream)
{
    if (M < 0 || N < 0 || K < 0 || !A || !B || !C) return nn_fail(AMHD_ERR_ARG, "bad gemm arguments");
    if (M == 0 || N == 0) return AMHD_OK;
    cudaStream_t s = S(stream);
    const int path = g_gemm_path.load();
    if (path == 2) return amhd_nn_gemm_tc(transA, transB, M, N, K, A, lda, B, ldb, C, ldc, alpha, beta, splits, stream);
    if (path == 0 && prefer_tc(M, N, K)) {
        bool launched = false;
        const int rc = tma_gemm(transA, transB, M, N, K, A, lda, B, ldb, C, ldc, alpha, beta, splits, s, &launched);
        if (rc != AMHD_OK || launched) return rc;
    }
    int kps;
    splits = split_k(K, splits, GBK, &kps);
    if (splits > 1 || K == 0) {
        scale_kernel<<<blocks_for((int64_t)M * N), 256, 0, s>>>(C, M, N, ldc, beta);
        NNCK(cudaGetLastError());
        if (K == 0) return AMHD_OK;
    }
    dim3 grid((N + GBN - 1) / GBN, (M + GBM - 1) / GBM, splits);
    gemm_bf16_kernel<<<grid, 128, 0, s>>>(transA, transB, M, N, K, static_cast<const bf16 *>(A), lda,
                                          static_cast<const bf16 *>(B), ldb, C, ldc, alpha,
                                          splits > 1 ? 0.f : beta, kps);
    NNCK(cudaGetLastError());
    return AMHD_OK;
}

int amhd_nn_im2col3(const float *X, int32_t C, int32_t B, int32_t H, int32_t W, void *col, void *stream)
{
    if (!X || !col || C <= 0 || B <= 0 || H <= 0 || W <= 0) return nn_fail(AMHD_ERR_ARG, "bad im2col arguments");
    const int64_t n_pix = (int64_t)B * H * W;
    if (n_pix > INT32_MAX || (int64_t)C * 9 > 65535) return nn_fail(AMHD_ERR_ARG, "im2col size beyond the grid");
    if (W % 8 == 0 && aligned16(X) && aligned16(col))
        im2col3_vec8_kernel<<<dim3((unsigned)((n_pix / 8 + 255) / 256), (unsigned)C), 256, 0, S(stream)>>>(
            X, H, W, (int)n_pix, static_cast<bf16 *>(col));
    else
        im2col3_kernel<<<dim3((unsigned)((n_pix + 255) / 256), (unsigned)(C * 9)), 256, 0, S(stream)>>>(
            X, C, B, H, W, static_cast<bf16 *>(col));
    NNCK(cudaGetLastError());
    return AMHD_OK;
}

int amhd_nn_col2im3(const float *dcol, int32_t C, int32_t B, int32_t H, int32_t W, float *dX, void *stream)
{
    if (!dcol || !dX || C <= 0 || B <= 0 || H <= 0 || W <= 0) return nn_fail(AMHD_ERR_ARG, "bad col2im arguments");
    const int64_t n_pix = (int64_t)B * H * W;
    if (n_pix > INT32_MAX || C > 65535) return nn_fail(AMHD_ERR_ARG, "col2im size beyond the grid");
    if (W % 4 == 0 && aligned16(dcol) && aligned16(dX))
        col2im3_vec4_kernel<<<dim3((unsigned)((n_pix / 4 + 255) / 256), (unsigned)C), 256, 0, S(stream)>>>(
            dcol, H, W, (int)n_pix, dX);
    else
        col2im3_kernel<<<dim3((unsigned)((n_pix + 255) / 256), (unsigned)C), 256, 0, S(stream)>>>(dcol, C, B, H, W,
                                                                                                    dX);
    NNCK(cudaGetLastError());
    return AMHD_OK;
}

int amhd_nn_flip3(const void *w, int32_t cout, int32_t cin, int32_t ldo, void *wt, void *stream)
{
    if (!w || !wt || cout <= 0 || cin <= 0 || ldo < cout * 9 || (int64_t)cin * ldo > INT32_MAX)
        return nn_fail(AMHD_ERR_ARG, "bad flip3 arguments");
    const int n = cin * ldo;
    flip3_kernel<<<(n + 255) / 256, 256, 0, S(stream)>>>(static_cast<const bf16 *>(w), cout, cin, ldo,
                                                         static_cast<bf16 *>(wt));
    NNCK(cudaGetLastError());
    return AMHD_OK;
}

int amhd_nn_pad_cols(const void *w, int32_t rows, int32_t cols, int32_t ldo, void *out, void *stream)
{
    if (!w || !out || rows <= 0 || cols <= 0 || ldo < cols || (int64_t)rows * ldo > INT32_MAX)
        return nn_fail(AMHD_ERR_ARG, "bad pad_cols arguments");
    const int n = rows * ldo;
    pad_cols_kernel<<<(n + 255) / 256, 256, 0, S(stream)>>>(static_cast<const bf16 *>(w), rows, cols, ldo,
                                                            static_cast<bf16 *>(out));
    NNCK(cudaGetLastError());
    return AMHD_OK;
}

int amhd_nn_cast_bf16(const float *x, void *y, int64_t n, void *stream)
{
    if (n < 0 || (n && (!x || !y))) return nn_fail(AMHD_ERR_ARG, "bad cast arguments");
    if (n && n % 4 == 0 && aligned16(x) && aligned16(y))
        cast_bf16_vec4_kernel<<<blocks_for(n / 4), 256, 0, S(stream)>>>(reinterpret_cast<const float4 *>(x),
                                                                        static_cast<uint2 *>(y), n / 4);
    else if (n)
        cast_bf16_kernel<<<blocks_for(n), 256, 0, S(stream)>>>(x, static_cast<bf16 *>(y), n);
    NNCK(cudaGetLastError());
    return AMHD_OK;
}

int amhd_nn_bias_act(float *Y, const float *bias, int32_t C, int64_t N, int32_t relu, void *stream)
{
    if (!Y || !bias || C <= 0 || N < 0) return nn_fail(AMHD_ERR_ARG, "bad bias arguments");
    if (N % 4 == 0 && C <= 65535 && aligned16(Y)) {
        int64_t bx = (N / 4 + 255) / 256;
        if (bx > 64) bx = 64;
        if (N) bias_act_vec4_kernel<<<dim3((unsigned)bx, (unsigned)C), 256, 0, S(stream)>>>(
            reinterpret_cast<float4 *>(Y), bias, N / 4, relu);
    } else {
        bias_act_kernel<<<blocks_for((int64_t)C * N), 256, 0, S(stream)>>>(Y, bias, C, N, relu);
    }
    NNCK(cudaGetLastError());
    return AMHD_OK;
}

int amhd_nn_relu_bwd(float *dY, const float *Y, int64_t n, void *stream)
{
    if (!dY || !Y || n < 0) return nn_fail(AMHD_ERR_ARG, "bad relu arguments");
    if (n % 4 == 0 && aligned16(dY) && aligned16(Y)) {
        if (n) relu_bwd_vec4_kernel<<<blocks_for(n / 4), 256, 0, S(stream)>>>(reinterpret_cast<float4 *>(dY),
                                                                               reinterpret_cast<const float4 *>(Y), n / 4);
    } else {
        relu_bwd_kernel<<<blocks_for(n), 256, 0, S(stream)>>>(dY, Y, n);
    }
    NNCK(cudaGetLastError());
    return AMHD_OK;
}

int amhd_nn_bias_grad(const float *dY, int32_t C, int64_t N, float *db, void *stream)
{
    if (!dY || !db || C <= 0 || N <= 0) return nn_fail(AMHD_ERR_ARG, "bad bias-grad arguments");
    bias_grad_kernel<<<C, 1024, 0, S(stream)>>>(dY, N, db);
    NNCK(cudaGetLastError());
    return AMHD_OK;
}

int amhd_nn_pool2(const float *X, int32_t CB, int32_t H, int32_t W, float *Y, int32_t backward, void *stream)
{
    if (!X || !Y || CB <= 0 || H < 2 || W < 2 || (H & 1) || (W & 1)) return nn_fail(AMHD_ERR_ARG, "bad pool arguments");
    const bool vec = W % 4 == 0 && CB <= 65535 && aligned16(X) && aligned16(Y);
    if (backward && vec)
        pool2_bwd_vec_kernel<<<dim3((unsigned)((H * W / 4 + 255) / 256), (unsigned)CB), 256, 0, S(stream)>>>(X, H, W,
                                                                                                           Y);
    else if (backward)
        pool2_bwd_kernel<<<blocks_for((int64_t)CB * H * W), 256, 0, S(stream)>>>(X, CB, H, W, Y);
    else if (vec)
        pool2_vec_kernel<<<dim3((unsigned)((H * W / 8 + 255) / 256), (unsigned)CB), 256, 0, S(stream)>>>(X, H, W, Y);
    else
        pool2_kernel<<<blocks_for((int64_t)CB * H * W / 4), 256, 0, S(stream)>>>(X, CB, H, W, Y);
    NNCK(cudaGetLastError());
    return AMHD_OK;
}

int amhd_nn_up2(const float *X, int32_t CB, int32_t h, int32_t w, float *Y, int32_t backward, void *stream)
{
    if (!X || !Y || CB <= 0 || h <= 0 || w <= 0) return nn_fail(AMHD_ERR_ARG, "bad upsample arguments");
    const bool vec = w % 2 == 0 && CB <= 65535 && aligned16(X) && aligned16(Y);
    if (backward && vec)
        up2_bwd_vec_kernel<<<dim3((unsigned)((h * w / 2 + 255) / 256), (unsigned)CB), 256, 0, S(stream)>>>(X, h, w, Y);
    else if (backward)
        up2_bwd_kernel<<<blocks_for((int64_t)CB * h * w), 256, 0, S(stream)>>>(X, CB, h, w, Y);
    else if (vec)
        up2_vec_kernel<<<dim3((unsigned)((4 * h * w / 4 + 255) / 256), (unsigned)CB), 256, 0, S(stream)>>>(X, h, w, Y);
    else
        up2_kernel<<<blocks_for((int64_t)CB * 4 * h * w), 256, 0, S(stream)>>>(X, CB, h, w, Y);
    NNCK(cudaGetLastError());
    return AMHD_OK;
}

int amhd_nn_axpy(float *y, const float *x, float a, int64_t n, void *stream)
{
    if (!y || !x || n < 0) return nn_fail(AMHD_ERR_ARG, "bad axpy arguments");
    if (n && n % 4 == 0 && aligned16(y) && aligned16(x))
        axpy_vec4_kernel<<<blocks_for(n / 4), 256, 0, S(stream)>>>(reinterpret_cast<float4 *>(y),
                                                                   reinterpret_cast<const float4 *>(x), a, n / 4);
    else if (n)
        axpy_kernel<<<blocks_for(n), 256, 0, S(stream)>>>(y, x, a, n);
    NNCK(cudaGetLastError());
    return AMHD_OK;
}

int amhd_nn_mse(const float *pred, const float *target, int64_t n, float *grad, float *loss, void *stream)
{
    if (!pred || !target || n <= 0) return nn_fail(AMHD_ERR_ARG, "bad mse arguments");
    mse_kernel<<<blocks_for(n), 256, 0, S(stream)>>>(pred, target, n, grad, loss);
    NNCK(cudaGetLastError());
    return AMHD_OK;
}

int amhd_nn_adam(float *w, const float *g, float *m, float *v, void *w_bf16, int64_t n, float lr, float beta1,
                 float beta2, float eps, int32_t t, float weight_decay, void *stream)
{
    if (!w || !g || !m || !v || n < 0 || t < 1) return nn_fail(AMHD_ERR_ARG, "bad adam arguments");
    const float c1 = 1.f / (1.f - powf(beta1, (float)t)), c2 = 1.f / (1.f - powf(beta2, (float)t));
    if (n) adam_kernel<<<blocks_for(n), 256, 0, S(stream)>>>(w, g, m, v, static_cast<bf16 *>(w_bf16), n, lr, beta1,
                                                             beta2, eps, c1, c2, weight_decay);
    NNCK(cudaGetLastError());
    return AMHD_OK;
}

int amhd_nn_adam_multi(const amhd_nn_tensor *tensors_dev, int32_t n_tensors, int64_t max_n, const float *hyper_dev,
                       void *stream)
{
    if (!tensors_dev || !hyper_dev || n_tensors < 0 || n_tensors > 65535 || max_n < 0)
        return nn_fail(AMHD_ERR_ARG, "bad adam_multi arguments");
    if (n_tensors == 0 || max_n == 0) return AMHD_OK;
    int64_t bx = (max_n + 255) / 256;
    if (bx > 1024) bx = 1024;
    adam_multi_kernel<<<dim3((unsigned)bx, (unsigned)n_tensors), 256, 0, S(stream)>>>(tensors_dev, hyper_dev);
    NNCK(cudaGetLastError());
    return AMHD_OK;
}

int amhd_nn_restrict(const amhd_grid *fine, const void *Uf, int32_t factor, float *out, int64_t out_vs, int32_t b,
                     int32_t B, void *stream)
{
    if (!fine || !Uf || !out || factor < 1 || fine->nx % factor || fine->ny % factor)
        return nn_fail(AMHD_ERR_ARG, "bad restriction arguments");
    const int nxc = fine->nx / factor, nyc = fine->ny / factor;
    const int64_t n = (int64_t)10 * nxc * nyc;
    if (fine->dtype == AMHD_F64)
        restrict_kernel<double><<<blocks_for(n), 256, 0, S(stream)>>>(static_cast<const double *>(Uf), fine->pitch,
                                                                       fine->var_stride, nxc, nyc, factor, out, out_vs,
                                                                       b, B);
    else
        restrict_kernel<float><<<blocks_for(n), 256, 0, S(stream)>>>(static_cast<const float *>(Uf), fine->pitch,
                                                                      fine->var_stride, nxc, nyc, factor, out, out_vs,
                                                                      b, B);
    NNCK(cudaGetLastError());
    return AMHD_OK;
}

int amhd_nn_pack(const amhd_grid *g, const void *U, const float *mean, const float *istd, float *x, int64_t x_vs,
                 int32_t b, void *stream)
{
    if (!g || !U || !mean || !istd || !x) return nn_fail(AMHD_ERR_ARG, "bad pack arguments");
    const int64_t n = (int64_t)10 * g->nx * g->ny;
    if (g->dtype == AMHD_F64)
        pack_kernel<double><<<blocks_for(n), 256, 0, S(stream)>>>(static_cast<const double *>(U), g->pitch,
                                                                   g->var_stride, g->nx, g->ny, mean, istd, x, x_vs, b);
    else
        pack_kernel<float><<<blocks_for(n), 256, 0, S(stream)>>>(static_cast<const float *>(U), g->pitch,
                                                                  g->var_stride, g->nx, g->ny, mean, istd, x, x_vs, b);
    NNCK(cudaGetLastError());
    return AMHD_OK;
}

int amhd_nn_apply(const amhd_grid *g, void *U, const float *scale, const float *y, int64_t y_vs, int32_t b,
                  void *stream)
{
    if (!g || !U || !scale || !y) return nn_fail(AMHD_ERR_ARG, "bad apply arguments");
    const int64_t n = (int64_t)10 * g->nx * g->ny;
    if (g->dtype == AMHD_F64)
        apply_kernel<double><<<blocks_for(n), 256, 0, S(stream)>>>(static_cast<double *>(U), g->pitch, g->var_stride,
                                                                    g->nx, g->ny, scale, y, y_vs, b);
    else
        apply_kernel<float><<<blocks_for(n), 256, 0, S(stream)>>>(static_cast<float *>(U), g->pitch, g->var_stride,
                                                                   g->nx, g->ny, scale, y, y_vs, b);
    NNCK(cudaGetLastError());
    return AMHD_OK;
}

int amhd_nn_apply_guarded(const amhd_grid *g, void *U, const float *scale, const float *y, int64_t y_vs, int32_t b,
                          float alpha, float min_ratio, int32_t scalar_mode, int32_t *rejected_dev, void *stream)
{
    if (!g || !U || !scale || !y) return nn_fail(AMHD_ERR_ARG, "bad apply arguments");
    if (!(min_ratio >= 0.f && min_ratio <= 1.f)) return nn_fail(AMHD_ERR_ARG, "min_ratio must be in [0, 1]");
    if (scalar_mode < 0 || scalar_mode > 3) return nn_fail(AMHD_ERR_ARG, "mode must be 0, 1, 2 or 3");
    const int64_t n = (int64_t)g->nx * g->ny;
    if (g->dtype == AMHD_F64)
        apply_guarded_kernel<double><<<blocks_for(n), 256, 0, S(stream)>>>(
            static_cast<double *>(U), g->pitch, g->var_stride, g->nx, g->ny, g->gamma, scale, y, y_vs, b, alpha,
            min_ratio, scalar_mode, rejected_dev);
    else
        apply_guarded_kernel<float><<<blocks_for(n), 256, 0, S(stream)>>>(
            static_cast<float *>(U), g->pitch, g->var_stride, g->nx, g->ny, g->gamma, scale, y, y_vs, b, alpha,
            min_ratio, scalar_mode, rejected_dev);
    NNCK(cudaGetLastError());
    return AMHD_OK;
}

}  // extern "C"
#pragma GCC visibility pop
