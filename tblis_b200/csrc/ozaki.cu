// ozaki.cu -- Ozaki split-precision contraction on the INT8 tensor cores.
//
// C = alpha*A*B + beta*C in FP64 accuracy from INT8 products (Ozaki scheme I
// with per-row / per-column power-of-two scaling):
//
//  1. row statistics: e_r = max exponent of row r of A (of column n of B) so
//     that |x| < 2^e_r, plus the row's sum of squares for the error estimate;
//  2. slicing: x' = x*2^-e_r in (-1,1) is split into S signed digits
//     in [-127, 127] by round-to-nearest in base 254 (d_1 = rint(127 x'),
//     then d_(p+1) = rint(254 r_p)), about 8 bits per slice, so
//     x' = (sum_p d_p 254^(1-p) + r_S 254^(1-S))/127 with |r_S| <= 1/2.
//     Digits are written straight from the strided tensor (through the
//     GEMM view's scatter vectors) as tiled INT8 planes: for each row tile
//     (128 rows of A, BN rows of B) and k step (32 bytes), the S slice tiles lie
//     back to back in one block, each in the tensor core's canonical K-major
//     layout, so that a stage is one bulk copy per operand;
//  3. one fused tcgen05 kernel per 128xBN output tile (BN = 128 for S <= 4,
//     96 for S = 5, 80 for S = 6, 64 for S = 7-8 and for BF16 digits): for every k step,
//     the bulk-copy engine brings the S slice tiles of A and B into shared
//     memory and one thread
//     issues tcgen05.mma.kind::i8 for the slice pairs (p, q) with
//     p + q <= S + 1, accumulating pairs of equal p + q ("diagonal" d) in
//     their own INT32 accumulator in tensor memory (slice p of A meets
//     B slices 1..S+1-p in one wide MMA, the B tiles and the diagonals
//     being adjacent in shared and tensor memory). The sums are exact while
//     (pairs on a diagonal) * K * 127^2 < 2^31, so beyond that the kernel
//     flushes the accumulators into C after each such run of k steps and
//     restarts them; the epilogue sums the diagonals in FP64 with weights
//     254^(2-d)/127^2, applies 2^(e_m + f_n), alpha and beta, and scatters
//     into C through C's scatter vectors.
//
// FP64 arithmetic is used only for the exponent extraction and scaling, the
// digit extraction, the cross-diagonal summation and the alpha/beta update.
// The slice count S is chosen per call from an a-priori estimate of the
// normwise error (row maxima and norms of A and B) to meet the tolerance.
//
// The same kernel runs two more plane formats: BF16 planes holding base-128
// digits in [-64, 64] (tcgen05.mma.kind::f16, FP32 accumulators, exact while
// a diagonal's sum stays below 2^24, so the runs between flushes are at most
// 2^24/(S*64^2) long), and a single low-precision pass (S = 1) whose plane
// holds x' itself rounded to BF16 or TF32 (kind::f16 / kind::tf32, FP32
// accumulation over the whole K) for callers who accept that error.
#include "ozaki.hpp"
#include "mult.hpp"

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>

namespace tb
{

namespace
{

constexpr int OZ_BM = 128;           // tile rows (TMEM lanes)
// tile columns per diagonal accumulator: the S diagonals of BN columns fill
// up to the 512 TMEM columns (wider tiles reuse each A slice tile over more
// B columns, fewer shared-memory bytes per MAC). BF16 digit planes (S >= 2)
// flush every 2^24/(S*64^2) k and keep 64 columns: measured faster there.
constexpr int bn_of(int S, int kind)
{
    return kind == OZ_BF16 && S >= 2 ? 64 : S <= 4 ? 128 : S == 5 ? 96 : S == 6 ? 80 : 64;
}
constexpr int OZ_BK = 32;            // k bytes per stage (one MMA K step of any kind)
constexpr int OZ_SMAX = 8;           // 8 diagonals x 64 columns = all 512 TMEM columns
constexpr int OZ_THREADS = 192;      // warp 0 bulk copies, warp 1 MMA, warps 2-5 epilogue
constexpr int A_TILE = OZ_BM*OZ_BK;  // bytes of one A slice tile
constexpr unsigned long long WAIT_NS = 2000000000ull;   // bounded waits: 2 s by default

__device__ int g_oz_error = 0;       // set by a kernel whose bounded wait gave up
// test support: the limit of every bounded wait, and a k step (stage for the
// moduli kernel) whose operand copies the slice and moduli GEMM kernels skip
// (-1: none), so that a test can make a wait run out without any fault
__device__ unsigned long long g_oz_wait_ns = WAIT_NS;
__device__ int g_oz_skip_step = -1;

// ---------------------------------------------------------------------------------
// PTX helpers
// ---------------------------------------------------------------------------------

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long globaltimer()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, int count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" :: "r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok) : "r"(smem_u32(bar)), "r"(parity) : "memory");
    return ok != 0;
}

// waits for the phase with the given parity to complete, at most
// g_oz_wait_ns; returns false (and records the error) when the wait gave up
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* abort_flag)
{
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = globaltimer();
    for (unsigned it = 0;; it++)
    {
        if (mbar_try_wait(bar, parity)) return true;
        if ((it & 255) == 0)
        {
            if (*abort_flag) return false;
            if (globaltimer() - t0 > g_oz_wait_ns)
            {
                *abort_flag = 1;
                atomicExch(&g_oz_error, 1);
                return false;
            }
        }
    }
}

// one contiguous global -> shared copy by the bulk-copy engine (16-byte
// aligned addresses, a multiple of 16 bytes), completing on the mbarrier
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 :: "r"(smem_u32(dst)), "l"((uint64_t)src), "r"(bytes), "r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :: "r"(smem_u32(slot)), "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(taddr), "r"(ncols));
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// one tcgen05.mma of the given kind (OZ_I8: s8 x s8 -> s32, OZ_BF16:
// bf16 x bf16 -> f32, OZ_TF32: tf32 x tf32 -> f32), A and B in shared memory
template <int KIND>
__device__ __forceinline__ void mma_op(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc)
{
    if constexpr (KIND == OZ_I8)
        asm volatile("{\n\t.reg .pred p;\n\t"
                     "setp.ne.b32 p, %4, 0;\n\t"
                     "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}"
                     :: "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc));
    else if constexpr (KIND == OZ_BF16)
        asm volatile("{\n\t.reg .pred p;\n\t"
                     "setp.ne.b32 p, %4, 0;\n\t"
                     "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                     :: "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc));
    else
        asm volatile("{\n\t.reg .pred p;\n\t"
                     "setp.ne.b32 p, %4, 0;\n\t"
                     "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
                     :: "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :: "r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, int (&r)[16])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 "
                 "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Slice tiles in shared memory (and, block by block, in the planes in global
// memory) use the tensor core's canonical K-major layout without swizzle:
// core matrices of 8 rows x 16 bytes (128 contiguous bytes), the two 16-byte
// halves of a row's 32 k bytes 128 bytes apart, successive 8-row groups 256
// bytes apart. Byte (row, kb) of a tile:
__host__ __device__ constexpr int tile_byte(int row, int kb)
{
    return (row >> 3)*256 + (kb >> 4)*128 + (row & 7)*16 + (kb & 15);
}

// shared-memory matrix descriptor of such a tile: leading byte offset (the
// k direction) 128, stride byte offset (the row direction) 256, no swizzle
__device__ __forceinline__ uint64_t sdesc_kmajor(const void* p)
{
    const uint64_t addr = smem_u32(p);
    return ((addr >> 4) & 0x3FFFull)          // start address
         | ((uint64_t)(128 >> 4) << 16)        // leading byte offset: next 16 k bytes
         | ((uint64_t)(256 >> 4) << 32)        // stride byte offset: next 8 rows
         | (1ull << 46);                       // descriptor version (sm100); layout 0: no swizzle
}

// instruction descriptor, K-major A and B, M = 128, N = n (a multiple of 16
// up to 256): accumulator format at bits 4-5 (s32 = 2, f32 = 1), A and B
// formats at bits 7-9 and 10-12 (s8 = 1; bf16 = 1, tf32 = 2)
__host__ __device__ constexpr uint32_t idesc_mma(int kind, int n)
{
    return (kind == OZ_I8 ? (2u << 4) | (1u << 7) | (1u << 10)
          : kind == OZ_BF16 ? (1u << 4) | (1u << 7) | (1u << 10)
          : (1u << 4) | (2u << 7) | (2u << 10)) |
           ((uint32_t)(n >> 3) << 17) | ((uint32_t)(OZ_BM >> 4) << 24);
}
static_assert(idesc_mma(OZ_I8, 256) >> 17 == ((256u >> 3) | ((OZ_BM >> 4) << 7)), "N field is 6 bits wide");

// bytes of one element of the slice planes
__host__ __device__ constexpr int elem_bytes(int kind) { return kind == OZ_I8 ? 1 : kind == OZ_BF16 ? 2 : 4; }

struct OzGemmArgs
{
    double* C;
    const i64 *c_m, *c_n, *c_l;
    const int *eA, *eB;          // [l][m], [l][n] exponents
    const unsigned char *pA, *pB; // tiled planes: blocks [l][row tile][k step] of S slice tiles
    i64 M, N, K, L;
    i64 tiles_m, tiles_n;        // row tiles of the A and B planes
    int k_steps;                 // k steps of the planes (K rounded up)
    int kt_flush;                // k steps whose digit sums stay exact; the accumulators are
                                 // flushed into C after each such run of steps
    double alpha, beta;
    double w[OZ_SMAX];           // weight of diagonal d = p + q at w[d - 2]
};

// TMEM columns for S diagonal accumulators of bn_of(S, KIND) columns (a power of two >= 32)
template <int S, int KIND>
struct TmemCols
{
    static constexpr uint32_t need = (uint32_t)(S*bn_of(S, KIND));
    static constexpr uint32_t value = need <= 32 ? 32 : need <= 64 ? 64 : need <= 128 ? 128 : need <= 256 ? 256 : 512;
};

template <int S, int STAGES, int KIND>
__global__ void __launch_bounds__(OZ_THREADS, 1)
ozaki_gemm_kernel(const OzGemmArgs p)
{
    constexpr int BN = bn_of(S, KIND);
    constexpr int B_TILE = BN*OZ_BK;                 // bytes of one B slice tile
    constexpr int STAGE_BYTES = S*(A_TILE + B_TILE);
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    // 1024-byte aligned base for the swizzled tiles
    unsigned char* smem = reinterpret_cast<unsigned char*>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + STAGES*STAGE_BYTES);
    uint64_t* empty = full + STAGES;
    uint64_t* accum = empty + STAGES;
    uint64_t* done = accum + 1;
    uint64_t* drained = done + 1;      // the epilogue has read a flushed chunk out of TMEM
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drained + 1);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
    i64* sCm = reinterpret_cast<i64*>(tmem_slot + 4);
    i64* sCn = sCm + OZ_BM;
    double* sScaleN = reinterpret_cast<double*>(sCn + BN);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const i64 tiles_n = (p.N + BN - 1)/BN;
    const i64 tm = blockIdx.x / tiles_n, tn = blockIdx.x % tiles_n;
    const int m0 = (int)(tm*OZ_BM), n0 = (int)(tn*BN);
    const int l = blockIdx.y;
    const int kt_count = p.k_steps;
    const int kt_flush = p.kt_flush > 0 ? p.kt_flush : kt_count;
    const int nchunks = (kt_count + kt_flush - 1)/kt_flush;

    if (threadIdx.x == 0)
    {
        for (int s = 0; s < STAGES; s++) { mbar_init(&full[s], 1); mbar_init(&empty[s], 1); }
        mbar_init(accum, 1);
        mbar_init(done, 1);
        mbar_init(drained, 4);             // one arrival per epilogue warp
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 1) tmem_alloc(tmem_slot, TmemCols<S, KIND>::value);
    for (int i = threadIdx.x; i < OZ_BM; i += OZ_THREADS)
    {
        const i64 m = m0 + i;
        sCm[i] = m < p.M ? p.c_m[m] : -1;
    }
    for (int i = threadIdx.x; i < BN; i += OZ_THREADS)
    {
        const i64 n = n0 + i;
        sCn[i] = n < p.N ? p.c_n[n] : -1;
        sScaleN[i] = n < p.N ? ldexp(1.0, p.eB[(i64)l*p.N + n]) : 0.0;
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;

    if (warp == 0)
    {
        // ---- bulk-copy producer -------------------------------------------------
        if (lane == 0)
        {
            const int skip = g_oz_skip_step;
            int kt_end = 0;                              // k steps whose copies were issued
            for (int kt = 0; kt < kt_count && !*abort_flag; kt++)
            {
                const int s = kt % STAGES;
                if (kt >= STAGES && !mbar_wait(&empty[s], ((kt/STAGES) & 1) ^ 1, abort_flag)) break;
                kt_end = kt + 1;
                if (kt == skip) continue;                // test support: this stage never fills
                unsigned char* st = smem + s*STAGE_BYTES;
                mbar_expect_tx(&full[s], STAGE_BYTES);
                // the S slice tiles of A, then those of B, each one contiguous block
                bulk_load(st, p.pA + (((i64)l*p.tiles_m + tm)*p.k_steps + kt)*(S*A_TILE), S*A_TILE, &full[s]);
                bulk_load(st + S*A_TILE, p.pB + (((i64)l*p.tiles_n + tn)*p.k_steps + kt)*(S*B_TILE),
                          S*B_TILE, &full[s]);
            }
            // drain: the copies of the last stages issued must have landed
            // before exit (bounded waits, also after a wait that gave up)
            for (int kt = max(0, kt_end - STAGES); kt < kt_end; kt++)
                if (kt != skip) mbar_wait(&full[kt % STAGES], (kt/STAGES) & 1, abort_flag);
        }
    }
    else if (warp == 1)
    {
        // ---- MMA issuer ----------------------------------------------------------
        if (lane == 0)
        {
            int chunk = 0;
            for (int kt = 0; kt < kt_count; kt++)
            {
                if (kt > 0 && kt % kt_flush == 0)
                {
                    // the sums of this run of k steps are complete: hand them to
                    // the epilogue and restart once it has read them out
                    mma_commit(accum);
                    if (!mbar_wait(drained, chunk & 1, abort_flag)) break;
                    tc_fence_after();
                    chunk++;
                }
                const int s = kt % STAGES;
                if (!mbar_wait(&full[s], (kt/STAGES) & 1, abort_flag)) break;
                tc_fence_after();
                const unsigned char* st = smem + s*STAGE_BYTES;
                // slice pa of A against B slices 1..S+1-pa at once: the B
                // tiles sit back to back in shared memory and the diagonals
                // pa+1..S+1 they feed are adjacent accumulators, so one MMA
                // of N = 64*(S+1-pa) columns (split at 256) covers the row
                #pragma unroll
                for (int pa = 1; pa <= S; pa++)
                {
                    const uint64_t ad = sdesc_kmajor(st + (pa - 1)*A_TILE);
                    #pragma unroll
                    for (int n0c = 0; n0c < (S + 1 - pa)*BN; n0c += 256)
                    {
                        const int nc = min(256, (S + 1 - pa)*BN - n0c);
                        const uint64_t bd = sdesc_kmajor(st + S*A_TILE + n0c*OZ_BK);
                        const uint32_t acc_addr = tmem_base + (uint32_t)((pa - 1)*BN + n0c);
                        // the pa = 1 row spans every diagonal: it starts the sums
                        mma_op<KIND>(acc_addr, ad, bd, idesc_mma(KIND, nc),
                                     (kt % kt_flush == 0 && pa == 1) ? 0u : 1u);
                    }
                }
                mma_commit(&empty[s]);
            }
            mma_commit(accum);
            mma_commit(done);
            // the MMAs issued so far finish before the tensor memory is freed,
            // also after a wait that gave up (a separate flag: only a timeout
            // of this wait itself ends it early)
            volatile int own_timeout = 0;
            mbar_wait(done, 0, &own_timeout);
        }
    }
    else
    {
        // ---- epilogue: warps 2..5, one TMEM lane quarter each --------------------
        const int quarter = warp & 3;
        const int row = quarter*32 + lane;
        const i64 rc = sCm[row];
        const i64 m = (i64)m0 + row;
        double* C = p.C + p.c_l[l];
        // one pass per flushed chunk: the first applies beta, later ones add
        #pragma unroll 1
        for (int chunk = 0; chunk < nchunks; chunk++)
        {
            const bool ok = mbar_wait(accum, chunk & 1, abort_flag);
            tc_fence_after();
            const double rscale = (rc >= 0 && ok) ? p.alpha*ldexp(1.0, p.eA[(i64)l*p.M + m]) : 0.0;
            const double beta = chunk == 0 ? p.beta : 1.0;
            #pragma unroll 1
            for (int c = 0; c < BN/16; c++)
            {
                double v[16];
                #pragma unroll
                for (int j = 0; j < 16; j++) v[j] = 0.0;
                // smallest weights first
                #pragma unroll
                for (int d = S + 1; d >= 2; d--)
                {
                    int r[16];
                    tmem_ld16(tmem_base + ((uint32_t)(quarter*32) << 16) + (uint32_t)((d - 2)*BN + c*16), r);
                    const double w = p.w[d - 2];
                    #pragma unroll
                    for (int j = 0; j < 16; j++)
                        v[j] += (KIND == OZ_I8 ? (double)r[j] : (double)__int_as_float(r[j]))*w;
                }
                if (rc >= 0 && ok)
                {
                    #pragma unroll
                    for (int j = 0; j < 16; j++)
                    {
                        const i64 cc = sCn[c*16 + j];
                        if (cc < 0) continue;
                        double* dst = C + rc + cc;
                        const double val = rscale*sScaleN[c*16 + j]*v[j];
                        *dst = beta == 0.0 ? val : val + beta*(*dst);
                    }
                }
            }
            if (!ok) break;
            if (chunk + 1 < nchunks)
            {
                // this warp's TMEM reads are done: the MMA thread may reuse the accumulators
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(drained);
            }
        }
    }

    tc_fence_before();
    __syncthreads();
    if (warp == 1)
    {
        tc_fence_after();
        tmem_dealloc(tmem_base, TmemCols<S, KIND>::value);
    }
}

// ---------------------------------------------------------------------------------
// statistics and slicing
// ---------------------------------------------------------------------------------

// view of one operand as rows x k (rows = m for A, n for B)
struct OzOperand
{
    const double* X;
    const i64 *r_off, *k_off, *l_off;
    i64 R, K, L;
    int rmode;                     // 0: gather along rows (rows contiguous), 1: along k
    i64 r_step, k_step;            // r_off[i] == i*r_step (k alike) for every i, or -1
};

constexpr int ST_THREADS = 256;

__device__ __forceinline__ int exp_of(double x)
{
    int e = 0;
    if (x != 0.0) frexp(x, &e);
    return x != 0.0 ? e : -100000;
}

// |x| as ordered integer bits: the largest |x| of a row has the largest
// frexp exponent, so the row maximum is taken on the bits and converted once
__device__ __forceinline__ unsigned long long abs_bits(double x)
{
    return (unsigned long long)__double_as_longlong(x) & 0x7fffffffffffffffull;
}

__device__ __forceinline__ int exp_of_bits(unsigned long long b)
{
    return exp_of(__longlong_as_double((long long)b));
}

constexpr int ST_UNROLL = 8;     // independent loads in flight per thread

// rows contiguous: a thread per row, k split over blockIdx.y; partial
// (max exponent, sum of squares) per split
__global__ void __launch_bounds__(ST_THREADS)
oz_stats_rows(const OzOperand o, int ksplit, int* pexp, double* pss)
{
    const i64 r = blockIdx.x*(i64)ST_THREADS + threadIdx.x;
    const int sp = blockIdx.y;
    const int l = blockIdx.z;
    if (r >= o.R) return;
    const i64 kchunk = (o.K + ksplit - 1)/ksplit;
    const i64 k0 = sp*kchunk, k1 = min(o.K, k0 + kchunk);
    const double* X = o.X + o.l_off[l] + o.r_off[r];
    unsigned long long mb = 0;
    double ss = 0.0;
    i64 k = k0;
    const i64 ks = o.k_step;
    for (; k + ST_UNROLL <= k1; k += ST_UNROLL)
    {
        double x[ST_UNROLL];
        #pragma unroll
        for (int u = 0; u < ST_UNROLL; u++) x[u] = X[ks >= 0 ? (k + u)*ks : o.k_off[k + u]];
        #pragma unroll
        for (int u = 0; u < ST_UNROLL; u++) { mb = max(mb, abs_bits(x[u])); ss += x[u]*x[u]; }
    }
    for (; k < k1; k++)
    {
        const double x = X[o.k_off[k]];
        mb = max(mb, abs_bits(x));
        ss += x*x;
    }
    const i64 idx = ((i64)l*ksplit + sp)*o.R + r;
    pexp[idx] = exp_of_bits(mb);
    pss[idx] = ss;
}

// k contiguous: a warp per row, lanes along k
__global__ void __launch_bounds__(ST_THREADS)
oz_stats_k(const OzOperand o, int* pexp, double* pss)
{
    const i64 r = (blockIdx.x*(i64)ST_THREADS + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const int l = blockIdx.z;
    if (r >= o.R) return;
    const double* X = o.X + o.l_off[l] + o.r_off[r];
    unsigned long long mb = 0;
    double ss = 0.0;
    i64 k = lane;
    const i64 ks = o.k_step;
    for (; k + 32*(ST_UNROLL - 1) < o.K; k += 32*ST_UNROLL)
    {
        double x[ST_UNROLL];
        #pragma unroll
        for (int u = 0; u < ST_UNROLL; u++) x[u] = X[ks >= 0 ? (k + 32*u)*ks : o.k_off[k + 32*u]];
        #pragma unroll
        for (int u = 0; u < ST_UNROLL; u++) { mb = max(mb, abs_bits(x[u])); ss += x[u]*x[u]; }
    }
    for (; k < o.K; k += 32)
    {
        const double x = X[o.k_off[k]];
        mb = max(mb, abs_bits(x));
        ss += x*x;
    }
    for (int s = 16; s > 0; s >>= 1)
    {
        mb = max(mb, (unsigned long long)__shfl_xor_sync(0xffffffffu, (long long)mb, s));
        ss += __shfl_xor_sync(0xffffffffu, ss, s);
    }
    if (lane == 0) { pexp[(i64)l*o.R + r] = exp_of_bits(mb); pss[(i64)l*o.R + r] = ss; }
}

// combines the per-split partials in split order
__global__ void oz_stats_final(i64 R, i64 L, int ksplit, const int* pexp, const double* pss, int* e_out,
                               double* ss_out)
{
    const i64 i = blockIdx.x*(i64)blockDim.x + threadIdx.x;
    if (i >= R*L) return;
    const i64 l = i / R, r = i - l*R;
    int e = -100000;
    double ss = 0.0;
    for (int sp = 0; sp < ksplit; sp++)
    {
        const i64 idx = (l*ksplit + sp)*R + r;
        e = max(e, pexp[idx]);
        ss += pss[idx];
    }
    e_out[i] = e == -100000 ? 0 : e;
    ss_out[i] = ss;
}

// digits of one value x' = x*2^-e in (-1, 1). INT8 planes: base 254,
// d_1 = rint(127 x') and d_(p+1) = rint(254 r_p) with r_p the remainder in
// [-1/2, 1/2], so every digit lies in [-127, 127] and a slice carries ~8 bits:
// x' = (d_1 + d_2/254 + ... + d_S/254^(S-1) + r_S/254^(S-1))/127. BF16 planes:
// base 128, d_1 = rint(64 x'), then 7 bits per digit (products stay exact in
// FP32 over longer K). Each step is y - rint(y), exact in FP64; the scaling
// by 127 / 254 rounds at 2^-53 relative, far below any tolerance the slices
// serve.
template <int KIND>
constexpr double first_digit_scale() { return KIND == OZ_I8 ? 127.0 : 64.0; }

// digits of y = x'*first_digit_scale<KIND>()
template <int S, int KIND>
__device__ __forceinline__ void digit_words(double y, int (&d)[S])
{
    constexpr double base = KIND == OZ_I8 ? 254.0 : 128.0;
    // rounding to the nearest integer (ties to even, as rint) by adding and
    // subtracting 1.5*2^52: exact for |y| < 2^51, and the integer sits in the
    // low word of the sum, which saves the FP64 round and convert units
    constexpr double shifter = 6755399441055744.0;
    // (the _rn intrinsics keep the compiler from fusing a product into the
    // shifter add, which would round the unrounded product instead)
    #pragma unroll
    for (int p = 0; p < S; p++)
    {
        const double sh = __dadd_rn(y, shifter);
        d[p] = __double2loint(sh);      // the digit, two's complement
        if (p + 1 < S) y = __dmul_rn(__dsub_rn(y, __dsub_rn(sh, shifter)), base);
    }
}

// 2^n, directly from the exponent field where 2^n is a normal number
__device__ __forceinline__ double pow2i(int n)
{
    return (n >= -1022 && n <= 1023) ? __longlong_as_double((long long)(n + 1023) << 52) : ldexp(1.0, n);
}

// ---- Ozaki scheme II (residues modulo pairwise-coprime moduli) ------------------
//
// a = rint(x*2^s) with |a| <= 2^50 is an exact integer; its residues modulo
// the moduli m_q are INT8 planes, one INT8 GEMM per modulus gives
// sum_k a*b exactly modulo m_q (INT32 accumulation, reduced mod m_q), and
// the Chinese remainder theorem over M = prod m_q recovers the integer
// product exactly while |sum_k a*b| < M/2 (the row and column scalings are
// chosen so). The only rounding is that of a and b to integers.
constexpr int CRT_MAX = 16;
// 256 and the largest odd numbers below it that are coprime to all before
__host__ __device__ constexpr int crt_modulus(int q)
{
    constexpr int m[CRT_MAX] = {256, 255, 253, 251, 247, 241, 239, 233, 229, 227, 223, 217, 211, 199, 197, 193};
    return m[q];
}

struct CrtConsts
{
    int nm;                                  // moduli in use (the first nm)
    float m[CRT_MAX], inv[CRT_MAX];          // m_q and fl(1/m_q)
    float c16[CRT_MAX];                      // 2^16 mod m_q, in [0, m_q)
    float g[CRT_MAX][CRT_MAX];               // g[q][j] = (m_0 ... m_(j-1)) mod m_q (centred)
    float ginv[CRT_MAX];                     // (m_0 ... m_(q-1))^-1 mod m_q (centred)
    double md[CRT_MAX];                      // m_q
    double invd[CRT_MAX];                    // fl64(1/m_q)
};

constexpr float F_BIAS = 8388608.0f;         // 2^23: (0x4B000000 | u) as float is 2^23 + u
constexpr float F_SHIFT = 12582912.0f;       // 1.5*2^23: rounds to an integer when added

// r = t - m*rint(t/m), exact for |t| < 2^22 (the quotient may be off by one
// at a tie of the rounded reciprocal, so |r| <= m/2 + 1/4)
__device__ __forceinline__ float crt_reduce(float t, float m, float inv)
{
    const float q = __fsub_rn(__fmaf_rn(t, inv, F_SHIFT), F_SHIFT);
    return __fmaf_rn(-q, m, t);
}

constexpr int SL_T = 64;     // 64 rows x 64 k per block

// x' rounded to the nearest TF32 value (10 fraction bits), as FP32 bits
__device__ __forceinline__ uint32_t to_tf32_bits(double xs)
{
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(__double2float_rn(xs)));
    return r;
}

// plane element types: digits as integers (INT8, or BF16 holding the same
// integers exactly) or, for a single pass, x' itself rounded to BF16 / TF32
template <int KIND>
struct PlaneElem;
template <> struct PlaneElem<OZ_I8> { using T = signed char; };
template <> struct PlaneElem<OZ_BF16> { using T = unsigned short; };
template <> struct PlaneElem<OZ_TF32> { using T = uint32_t; };

template <int KIND>
__device__ __forceinline__ typename PlaneElem<KIND>::T digit_elem(int d)
{
    if constexpr (KIND == OZ_I8) return (signed char)d;
    else if constexpr (KIND == OZ_BF16) return __bfloat16_as_ushort(__float2bfloat16_rn((float)d));  // exact: |d| <= 64
    else return __float_as_uint((float)d);
}

template <int KIND>
__device__ __forceinline__ typename PlaneElem<KIND>::T single_elem(double xs)
{
    if constexpr (KIND == OZ_BF16) return __bfloat16_as_ushort(__double2bfloat16(xs));
    else return to_tf32_bits(xs);
}

__device__ __forceinline__ void sl_cp_async8(double* smem, const double* gmem, bool valid)
{
    const unsigned saddr = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n"
                 :: "r"(saddr), "l"(gmem), "r"(valid ? 8 : 0) : "memory");
}

// geometry of tiled planes: blocks [l][row tile][k step], each holding the S
// slice tiles (tile_rows x 32 bytes, tile_byte order) back to back
struct PlaneGeom
{
    int tile_rows;
    i64 tiles, k_steps;
    int S;
};

constexpr int SL_LD = SL_T + 1;            // padded smem row (doubles)
constexpr int SL_BLOCKS_PER_SM = 2;       // 128 registers a thread: more of the 16 elements' FP64 chains in flight
constexpr size_t SL_SMEM = 2*SL_T*SL_LD*sizeof(double);

// writes the S tiled planes (PlaneGeom) of 64x64 tiles of the operand:
// digit planes, or (SINGLE, S = 1) x' rounded to the plane type. Rows and k
// beyond the operand, up to whole tiles and k steps, get zeros.
// Persistent blocks walk the tiles; the gather of the next tile (cp.async,
// zero-filled outside the operand) runs while the current one is converted.
template <int S, int KIND, bool SINGLE, bool CRT = false>
__global__ void __launch_bounds__(256, SL_BLOCKS_PER_SM)
oz_slice(const OzOperand o, const int* e_rows, void* out_, const PlaneGeom pg, unsigned tiles_r, unsigned tiles_k,
         const CrtConsts cc)
{
    using T = typename PlaneElem<KIND>::T;
    constexpr int KE = OZ_BK/(int)sizeof(T);         // elements per k step
    unsigned char* outb = static_cast<unsigned char*>(out_);
    const i64 tile_bytes = (i64)pg.tile_rows*OZ_BK;
    extern __shared__ double sl_smem[];    // two [SL_T][SL_LD] buffers
    const unsigned per_l = tiles_r*tiles_k, ntiles = per_l*(unsigned)o.L;   // below 2^31 (host check)
    const int t = threadIdx.x;

    // each thread gathers one fixed row (rows contiguous) or one fixed k (k
    // contiguous) of the tile and 16 positions along the other index, which
    // are the same across the warp
    const bool by_rows = o.rmode == 0;
    const int fixed = t & (SL_T - 1), vary0 = t >> 6;
    const i64* fixed_off = by_rows ? o.r_off : o.k_off;
    const i64* vary_off = by_rows ? o.k_off : o.r_off;
    const i64 vary_step = by_rows ? o.k_step : o.r_step;     // -1: read the table
    const i64 fixed_n = by_rows ? o.R : o.K, vary_n = by_rows ? o.K : o.R;
    // smem position of element (fixed, vary0 + 4j): row-major [r][k] tile
    const int s_base = by_rows ? fixed*SL_LD + vary0 : vary0*SL_LD + fixed;
    const int s_step = by_rows ? 4 : 4*SL_LD;

    struct At { int l; i64 r0, k0; };
    auto where = [&](unsigned tile) {
        const unsigned l = tile/per_l, rem = tile - l*per_l;
        const unsigned tr = rem/tiles_k;
        return At{(int)l, (i64)tr*SL_T, (i64)(rem - tr*tiles_k)*SL_T};
    };
    auto load = [&](const At& w, double* buf) {
        const i64 f = (by_rows ? w.r0 : w.k0) + fixed;
        const i64 v0 = (by_rows ? w.k0 : w.r0) + vary0;
        const bool fok = f < fixed_n;
        const double* Xf = o.X + o.l_off[w.l] + (fok ? fixed_off[f] : 0);
        if (vary_step >= 0)
        {
            // a single stride: the addresses need no table reads
            const double* Xv = Xf + v0*vary_step;
            #pragma unroll
            for (int j = 0; j < SL_T*SL_T/256; j++)
            {
                const bool ok = fok && v0 + 4*j < vary_n;
                sl_cp_async8(buf + s_base + j*s_step, ok ? Xv + 4*j*vary_step : o.X, ok);
            }
        }
        else
        {
            #pragma unroll
            for (int j = 0; j < SL_T*SL_T/256; j++)
            {
                const i64 v = v0 + 4*j;
                const bool ok = fok && v < vary_n;
                sl_cp_async8(buf + s_base + j*s_step, ok ? Xf + vary_off[v] : o.X, ok);
            }
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };

    // 4 threads per row of a tile, 16 consecutive k each; a warp takes 32
    // consecutive rows of one 16-k segment, so its shared-memory reads
    // spread over the banks (the padded rows shift by two banks each) and
    // its plane stores still fill whole 128-byte lines
    const int rl = t & (SL_T - 1), seg = (t >> 6)*16;
    const i64 k_lim = pg.k_steps*KE;
    const i64 r_lim = pg.tiles*pg.tile_rows;         // rows of the planes (whole row tiles)
    unsigned tile = blockIdx.x;
    At at{0, 0, 0};
    if (tile < ntiles) { at = where(tile); load(at, sl_smem); }
    for (int it = 0; tile < ntiles; tile += gridDim.x, it++)
    {
        const double* cur = sl_smem + (it & 1)*SL_T*SL_LD;
        const unsigned nxt = tile + gridDim.x;
        At nat = at;
        if (nxt < ntiles) { nat = where(nxt); load(nat, sl_smem + ((it + 1) & 1)*SL_T*SL_LD); }
        else asm volatile("cp.async.commit_group;" ::: "memory");   // keeps the group count uniform
        asm volatile("cp.async.wait_group 1;" ::: "memory");
        __syncthreads();

        const i64 r = at.r0 + rl, kk = at.k0 + seg;
        if (kk < k_lim && r < r_lim)
        {
            // rows past the operand hold zeros: any exponent serves
            const int e = r < o.R ? e_rows[(i64)at.l*o.R + r] : 0;
            const double* src = cur + rl*SL_LD + seg;
            const i64 rt = r/pg.tile_rows;
            const int rin = (int)(r - rt*pg.tile_rows);
            // slice tile 0 of the block of row tile rt holding element k
            auto block = [&](i64 k) {
                return outb + (((i64)at.l*pg.tiles + rt)*pg.k_steps + k/KE)*S*tile_bytes +
                       tile_byte(rin, (int)(k % KE)*(int)sizeof(T));
            };
            if constexpr (CRT)
            {
                // e_rows holds the row's shift s. y = 1.5*2^52 + a with
                // a = rint(x*2^s) (one rounding, |a| <= 2^50); the low byte of
                // y is a mod 256; for odd m, y - m*rint(a/m) = 1.5*2^52 + r
                // exactly, |r| <= (m-1)/2, and its low word is r. Three FP64
                // operations per modulus; 16 k bytes per plane row.
                constexpr double SH = 6755399441055744.0;
                const int sh1 = e >> 1, sh2 = e - sh1;
                const double sc1 = pow2i(sh1), sc2 = pow2i(sh2);
                double y[16], av[16];
                #pragma unroll
                for (int u = 0; u < 16; u++)
                {
                    y[u] = __fma_rn(__dmul_rn(src[u], sc1), sc2, SH);
                    av[u] = __dsub_rn(y[u], SH);
                }
                const i64 plane_stride = tile_bytes;
                unsigned char* dst = block(kk);
                #pragma unroll
                for (int q = 0; q < S; q++)
                {
                    uint32_t w[4];
                    #pragma unroll
                    for (int g = 0; g < 4; g++)
                    {
                        uint32_t b[4];
                        #pragma unroll
                        for (int u = 0; u < 4; u++)
                        {
                            const int i = g*4 + u;
                            if (q == 0) b[u] = (uint32_t)__double2loint(y[i]);
                            else
                            {
                                const double qm = __dsub_rn(__fma_rn(av[i], cc.invd[q], SH), SH);
                                b[u] = (uint32_t)__double2loint(__fma_rn(-qm, cc.md[q], y[i]));
                            }
                        }
                        // byte 0 of each word, four to a word
                        w[g] = __byte_perm(__byte_perm(b[0], b[1], 0x0040), __byte_perm(b[2], b[3], 0x0040), 0x5410);
                    }
                    *reinterpret_cast<uint4*>(dst + q*plane_stride) = make_uint4(w[0], w[1], w[2], w[3]);
                }
            }
            else if constexpr (KIND == OZ_I8 && !SINGLE)
            {
                // 2^-e*127 is exact: x*(2^-e*127) rounds once, as x'*127 does
                const double sc = pow2i(-e)*first_digit_scale<KIND>();
                // four digits to a word: the integers sit in the low words of
                // the shifted sums, and two byte permutes interleave four of them
                uint32_t w[S][4];
                #pragma unroll
                for (int g = 0; g < 4; g++)
                {
                    int lo[4][S];
                    #pragma unroll
                    for (int u = 0; u < 4; u++) digit_words<S, KIND>(src[g*4 + u]*sc, lo[u]);
                    #pragma unroll
                    for (int q = 0; q < S; q++)
                        w[q][g] = __byte_perm(__byte_perm(lo[0][q], lo[1][q], 0x0040),
                                              __byte_perm(lo[2][q], lo[3][q], 0x0040), 0x5410);
                }
                // the 16 k bytes are one 16-byte row of a core matrix
                unsigned char* dst = block(kk);
                #pragma unroll
                for (int q = 0; q < S; q++)
                    *reinterpret_cast<uint4*>(dst + q*tile_bytes) = make_uint4(w[q][0], w[q][1], w[q][2], w[q][3]);
            }
            else
            {
                const double sc = pow2i(-e)*(SINGLE ? 1.0 : first_digit_scale<KIND>());
                alignas(16) T dg[S][16];
                #pragma unroll
                for (int j = 0; j < 16; j++)
                {
                    const double xs = src[j]*sc;
                    if constexpr (SINGLE)
                        dg[0][j] = single_elem<KIND>(xs);
                    else
                    {
                        int d[S];
                        digit_words<S, KIND>(xs, d);
                        #pragma unroll
                        for (int q = 0; q < S; q++) dg[q][j] = digit_elem<KIND>(d[q]);
                    }
                }
                // 16-byte pieces of 16/sizeof(T) elements, each one core-matrix row
                constexpr int PER = 16/(int)sizeof(T);
                #pragma unroll
                for (int v = 0; v < 16/PER; v++)
                {
                    const i64 k = kk + v*PER;
                    if (k >= k_lim) break;
                    unsigned char* dst = block(k);
                    #pragma unroll
                    for (int q = 0; q < S; q++)
                        *reinterpret_cast<uint4*>(dst + q*tile_bytes) = *reinterpret_cast<const uint4*>(&dg[q][v*PER]);
                }
            }
        }
        at = nat;
        __syncthreads();      // the buffer is refilled two tiles later
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
}

template <int S, int KIND, bool SINGLE, bool CRT = false>
void launch_slice(const OzOperand& o, const int* e, void* out, const PlaneGeom& pg, cudaStream_t st,
                  const CrtConsts* cc = nullptr)
{
    // every row of the row tiles (64-row slicing tiles may pass the last
    // one: the kernel stops at it), every k of the k steps
    const i64 tiles_r = (pg.tiles*pg.tile_rows + SL_T - 1)/SL_T;
    const i64 tiles_k = (pg.k_steps*(OZ_BK/elem_bytes(KIND)) + SL_T - 1)/SL_T;
    const i64 ntiles = tiles_r*tiles_k*o.L;
    if (ntiles == 0) return;
    TB_CHECK(ntiles < ((i64)1 << 31), TB_ERR_SIZE, "Ozaki operand above 2^31 tiles of 64x64");
    const i64 grid = std::min<i64>(ntiles, (i64)device_sm_count()*SL_BLOCKS_PER_SM);
    TB_CUDA(cudaFuncSetAttribute(oz_slice<S, KIND, SINGLE, CRT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)SL_SMEM));
    CrtConsts none = {};
    TimedLaunch t("oz_slice", st);
    oz_slice<S, KIND, SINGLE, CRT><<<(unsigned)grid, 256, SL_SMEM, st>>>(o, e, out, pg, (unsigned)tiles_r,
                                                                          (unsigned)tiles_k, cc ? *cc : none);
    check_launch("oz_slice");
}

template <int KIND>
void slice_dispatch_kind(int S, const OzOperand& o, const int* e, void* out, const PlaneGeom& pg, cudaStream_t st)
{
    switch (S)
    {
        case 1: launch_slice<1, KIND, false>(o, e, out, pg, st); break;
        case 2: launch_slice<2, KIND, false>(o, e, out, pg, st); break;
        case 3: launch_slice<3, KIND, false>(o, e, out, pg, st); break;
        case 4: launch_slice<4, KIND, false>(o, e, out, pg, st); break;
        case 5: launch_slice<5, KIND, false>(o, e, out, pg, st); break;
        case 6: launch_slice<6, KIND, false>(o, e, out, pg, st); break;
        case 7: launch_slice<7, KIND, false>(o, e, out, pg, st); break;
        default: launch_slice<8, KIND, false>(o, e, out, pg, st); break;
    }
}

void slice_dispatch(int kind, bool single, int S, const OzOperand& o, const int* e, void* out,
                    const PlaneGeom& pg, cudaStream_t st)
{
    if (single)
    {
        if (kind == OZ_BF16) launch_slice<1, OZ_BF16, true>(o, e, out, pg, st);
        else launch_slice<1, OZ_TF32, true>(o, e, out, pg, st);
        return;
    }
    if (kind == OZ_I8) slice_dispatch_kind<OZ_I8>(S, o, e, out, pg, st);
    else slice_dispatch_kind<OZ_BF16>(S, o, e, out, pg, st);
}

// ---- Ozaki scheme II: INT8 GEMM per modulus and the CRT combination -------------

constexpr int CRT_BN = 256;                    // output columns per tile (B plane row tile)
constexpr int CRT_OUT_TILE = OZ_BM*CRT_BN;     // residue bytes of one output tile and modulus
constexpr int CRT_KT_RUN = 4096;               // k steps whose INT32 sums stay exact: 4096*32*128^2 = 2^31

struct CrtGemmArgs
{
    CUtensorMap tmA, tmB;          // the planes as 4-D maps (one modulus's tiles of four blocks per copy)
    const unsigned char *pA, *pB;  // residue planes: blocks [l][row tile][k step] of nm tiles
    unsigned char* R;              // residues [l][tile][modulus][128][256], each in [0, m_q)
    i64 tiles_m, tiles_n;          // 128-row tiles of A (even), 256-column tiles of the output
    int k_steps;                   // k steps of the planes
    int kt0, kt1;                  // k steps of this launch (one exact run)
    int nm, L;
    float m[CRT_MAX], inv[CRT_MAX], c16[CRT_MAX];
};

// ---- the modulus GEMMs on CTA pairs (tcgen05 cta_group::2) ----------------------
//
// A cluster of two CTAs on one SM pair computes one 256 x 256 output tile of
// one modulus: CTA r holds rows 128r..128r+127 of A and columns
// 128r..128r+127 of B in its shared memory, and each MMA of 256 x 256 x 32
// issued by CTA 0 reads both halves of B, so each SM reads half of B per
// MAC. A stage holds two k steps (two MMAs per barrier round). Both CTAs
// copy their tiles with cta_group::2 tensor copies (no multicast) that
// complete on CTA 0's barrier, which expects the bytes of both; CTA 0's
// commits arrive on both CTAs' barriers (tcgen05.commit multicast). Each
// CTA's epilogue reduces the accumulator rows in its own SM's tensor memory.
// One work item per cluster, launched in order (modulus, batch index, row
// tile, column tile): the clusters on the GPU at any time work on
// consecutive tiles, so the nine column tiles of a row tile read its A
// rows within a short time of each other and share them through L2 (a
// persistent loop over a static share of the items drifted apart and read
// A from DRAM up to eight times); two clusters per SM pair overlap one's
// epilogue with the other's MMAs.

constexpr int CRT_KSUB = 2;                    // k steps per stage
constexpr int CRT2_STAGES = 6;                 // 16 KB per stage: 97 KB, two CTAs per SM
constexpr int CRT2_TILE = OZ_BM*OZ_BK;         // one 128-row x 32-byte tile (A, or a CTA's half of B)
constexpr int CRT2_STAGE_BYTES = 2*CRT_KSUB*CRT2_TILE;
constexpr uint32_t CRT2_TMEM_COLS = 256;       // one 128 x 256 INT32 accumulator

__device__ __forceinline__ uint32_t cluster_ctarank()
{
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}

__device__ __forceinline__ uint32_t mapa_shared(uint32_t addr, uint32_t rank)
{
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(addr), "r"(rank));
    return r;
}

__device__ __forceinline__ void cluster_sync_all()
{
    asm volatile("barrier.cluster.arrive.release.aligned;\n\t"
                 "barrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// modulus q's tiles of CRT_KSUB consecutive plane blocks from block w (one
// stage) into this CTA's shared memory, completing on CTA 0's barrier (a
// shared::cluster address)
__device__ __forceinline__ void tma_load_pair(void* dst, const CUtensorMap* map, int q, int w, uint32_t bar_cluster)
{
    asm volatile("cp.async.bulk.tensor.4d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes"
                 " [%0], [%1, {%3, %3, %4, %5}], [%2];"
                 :: "r"(smem_u32(dst)), "l"((uint64_t)map), "r"(bar_cluster), "r"(0), "r"(q), "r"(w) : "memory");
}

// arrives on the barrier at this offset in both CTAs of the pair once the
// MMAs issued so far are complete
__device__ __forceinline__ void mma_commit_pair(uint64_t* bar)
{
    asm volatile("tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;"
                 :: "r"(smem_u32(bar)), "h"((unsigned short)3) : "memory");
}

__device__ __forceinline__ void tmem_alloc_pair(uint32_t* slot, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;"
                 :: "r"(smem_u32(slot)), "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;");
}

__device__ __forceinline__ void tmem_dealloc_pair(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" :: "r"(taddr), "r"(ncols));
}

__device__ __forceinline__ void mma_i8_pair(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc)
{
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "setp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::2.kind::i8 [%0], %1, %2, %3, p;\n\t}"
                 :: "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc));
}

constexpr size_t crt_gemm2_smem()
{
    return (size_t)CRT2_STAGES*CRT2_STAGE_BYTES + 1024 + (2*CRT2_STAGES + 1)*8 + 16;
}

// work item w: modulus-major, then the batch index, then 256-row tiles, then
// 256-column tiles (consecutive items share A rows, and one modulus's B
// planes stay in L2 while its items run)
struct CrtItem { int q, l; i64 tm2, tn; };
__device__ __forceinline__ CrtItem crt_item(i64 w, int L, i64 tiles_m2, i64 tiles_n)
{
    const i64 per_q = (i64)L*tiles_m2*tiles_n;
    CrtItem it;
    it.q = (int)(w / per_q);
    i64 r = w - it.q*per_q;
    it.l = (int)(r / (tiles_m2*tiles_n));
    r -= (i64)it.l*tiles_m2*tiles_n;
    it.tm2 = r / tiles_n;
    it.tn = r - it.tm2*tiles_n;
    return it;
}

// grid.x = 2 x (work items); the planes have 128-row tiles of A and B in
// blocks [l][row tile][k step] of nm tiles (k steps a multiple of
// CRT_KSUB); residues go out as column-major 128 x 256 tiles
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(OZ_THREADS, 2)
oz_crt_gemm2(const __grid_constant__ CrtGemmArgs p)
{
    constexpr uint32_t IDESC = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(CRT_BN >> 3) << 17) |
                               ((uint32_t)(256 >> 4) << 24);      // s8 x s8 -> s32, M = 256, N = 256
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char* smem = reinterpret_cast<unsigned char*>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + CRT2_STAGES*CRT2_STAGE_BYTES);
    uint64_t* empty = full + CRT2_STAGES;
    uint64_t* tfull = empty + CRT2_STAGES;       // accumulator ready
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(tfull + 1);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t rank = cluster_ctarank();
    const i64 tiles_m2 = p.tiles_m >> 1;
    const CrtItem it = crt_item(blockIdx.x >> 1, p.L, tiles_m2, p.tiles_n);
    const i64 tm = 2*it.tm2 + rank;              // this CTA's 128-row tile of A and C
    const i64 tb = 2*it.tn + rank;               // this CTA's 128-row tile of the B plane
    const int kt0 = p.kt0, kt_count = p.kt1 - p.kt0;    // a multiple of CRT_KSUB
    const int nstage = kt_count/CRT_KSUB;

    if (threadIdx.x == 0)
    {
        for (int s = 0; s < CRT2_STAGES; s++)
        {
            mbar_init(&full[s], 1);       // CTA 0's: its producer's arrival plus both CTAs' bytes
            mbar_init(&empty[s], 1);      // CTA 0's MMA commit, multicast to both
        }
        mbar_init(tfull, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 1) tmem_alloc_pair(tmem_slot, CRT2_TMEM_COLS);
    tc_fence_before();
    // both CTAs' barriers and tensor memory exist before any remote arrival or MMA
    cluster_sync_all();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;

    if (warp == 0)
    {
        if (lane == 0)
        {
            const uint32_t full0 = mapa_shared(smem_u32(full), 0);
            // plane blocks of this CTA's A and B tiles at k step kt0
            const i64 a_blk = ((i64)it.l*p.tiles_m + tm)*p.k_steps + kt0;
            const i64 b_blk = ((i64)it.l*2*p.tiles_n + tb)*p.k_steps + kt0;
            // both CTAs issue the same stages: each stage after the first
            // CRT2_STAGES waits for the same multicast commit, and a producer
            // stops only when that wait fails (not on the other warps' abort)
            const int skip = g_oz_skip_step;
            int i_end = 0;                               // stages whose copies were issued
            volatile int own_timeout = 0;                // this producer's waits only
            for (int i = 0; i < nstage; i++)
            {
                const int s = i % CRT2_STAGES;
                if (i >= CRT2_STAGES && !mbar_wait(&empty[s], ((i/CRT2_STAGES) & 1) ^ 1, &own_timeout)) break;
                i_end = i + 1;
                // test support: neither CTA copies this stage (nor does CTA 0
                // expect it), so it never completes
                if (i == skip) continue;
                unsigned char* st = smem + s*CRT2_STAGE_BYTES;
                if (rank == 0) mbar_expect_tx(&full[s], 2*CRT2_STAGE_BYTES);
                tma_load_pair(st, &p.tmA, it.q, (int)(a_blk + i*CRT_KSUB), full0 + 8u*(uint32_t)s);
                tma_load_pair(st + CRT_KSUB*CRT2_TILE, &p.tmB, it.q, (int)(b_blk + i*CRT_KSUB),
                              full0 + 8u*(uint32_t)s);
            }
            if (rank == 0)
            {
                // the copies of both CTAs for the last stages issued have landed
                // (their bytes complete CTA 0's barriers) before either CTA
                // leaves; after a wait that gave up, each of these is bounded too
                for (int i = max(0, i_end - CRT2_STAGES); i < i_end; i++)
                    if (i != skip) mbar_wait(&full[i % CRT2_STAGES], (i/CRT2_STAGES) & 1, abort_flag);
            }
        }
    }
    else if (warp == 1)
    {
        if (lane == 0 && rank == 0)
        {
            for (int i = 0; i < nstage; i++)
            {
                const int s = i % CRT2_STAGES;
                if (!mbar_wait(&full[s], (i/CRT2_STAGES) & 1, abort_flag)) break;
                tc_fence_after();
                const unsigned char* st = smem + s*CRT2_STAGE_BYTES;
                #pragma unroll
                for (int u = 0; u < CRT_KSUB; u++)
                    mma_i8_pair(tmem_base, sdesc_kmajor(st + u*CRT2_TILE),
                                sdesc_kmajor(st + (CRT_KSUB + u)*CRT2_TILE), IDESC, (i > 0 || u > 0) ? 1u : 0u);
                mma_commit_pair(&empty[s]);
            }
            // also after a wait that gave up: the epilogues learn from this
            // commit that the MMAs issued so far are complete
            mma_commit_pair(tfull);
        }
    }
    else
    {
        // warps 2..5: TMEM lane quarter warp % 4, one output row per thread
        const int quarter = warp & 3;
        const int row = quarter*32 + lane;
        // waits for the MMAs to finish (a separate flag: another warp's
        // timeout does not end this wait early), then writes only if no wait
        // of this CTA gave up
        volatile int own_timeout = 0;
        const bool ok = mbar_wait(tfull, 0, &own_timeout) && !*abort_flag;
        tc_fence_after();
        const int q = it.q;
        const int mq = (int)p.m[q];
        const float mf = p.m[q], inv = p.inv[q], c16 = p.c16[q];
        // residue tiles are column-major (byte (col, row) at col*128 + row)
        unsigned char* out = p.R + ((((i64)it.l*p.tiles_m + tm)*p.tiles_n + it.tn)*p.nm + q)*(i64)CRT_OUT_TILE + row;
        #pragma unroll 1
        for (int c = 0; c < CRT_BN/16 && ok; c++)
        {
            int r[16];
            tmem_ld16(tmem_base + ((uint32_t)(quarter*32) << 16) + (uint32_t)(c*16), r);
            #pragma unroll
            for (int jj = 0; jj < 16; jj++)
            {
                uint32_t v;
                if (mq == 256) v = (uint32_t)r[jj] & 0xFFu;
                else
                {
                    // r = hi*2^16 + lo: hi*(2^16 mod m) + lo is below 2^23 in magnitude, exact in FP32
                    const float fh = __fsub_rn(__int_as_float(0x4B400000 + (r[jj] >> 16)), F_SHIFT);
                    const float fl = __fsub_rn(__int_as_float(0x4B000000 | (r[jj] & 0xFFFF)), F_BIAS);
                    float x = crt_reduce(__fmaf_rn(fh, c16, fl), mf, inv);
                    if (x < 0.0f) x += mf;
                    v = (uint32_t)__float_as_int(__fadd_rn(x, F_SHIFT));
                }
                out[(c*16 + jj)*OZ_BM] = (unsigned char)v;
            }
        }
    }

    tc_fence_before();
    // neither CTA leaves while the pair's MMAs, arrivals or copies may touch it
    cluster_sync_all();
    if (warp == 1)
    {
        tc_fence_after();
        tmem_dealloc_pair(tmem_base, CRT2_TMEM_COLS);
    }
}

// per-row shift s = P - e with 2^e above the row's norm (times 1 + 2^-20,
// which covers the rounding of its sum of squares), so that rint(x*2^s)
// has a norm of at most 2^P (+ sqrt(K)/2 from the rounding); 0 for a zero row
__global__ void oz_crt_shifts(const double* ss, i64 n, int P, int* s_out)
{
    const i64 i = blockIdx.x*(i64)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double v = sqrt(ss[i]);
    int s = 0;
    if (v > 0.0 && v <= 1.7e308)
    {
        int e = 0;
        frexp(v*(1.0 + 0x1p-20), &e);
        s = P - e;
    }
    s_out[i] = s;
}

struct CrtCombineArgs
{
    const unsigned char* R;        // residues of the chunks, chunk_bytes apart
    int chunks;
    i64 chunk_bytes;
    double* C;
    const i64 *c_m, *c_n, *c_l;
    const int *sA, *sB;            // shifts [l][m], [l][n]
    i64 M, N, tiles_m, tiles_n;
    double alpha, beta;
    CrtConsts cc;
};

// One block of 256 threads per (output tile, batch index, quarter of the
// tile's columns): lane t of a warp takes rows 4t..4t+3 and warp w the
// columns w, w+8, ... of the quarter; for each element
// it sums the chunk residues, recovers the balanced mixed-radix digits v_q of
// the integer product (Garner's algorithm, exact in FP32), evaluates
// sum v_q m_0...m_(q-1) by Horner in FP64, scales by 2^-(sA+sB) and applies
// alpha and beta through C's scatter vectors (beta == 0: C is not read).
template <int NM>
__global__ void __launch_bounds__(256)
oz_crt_combine(const CrtCombineArgs p)
{
    constexpr int RW = 4;                      // rows per thread (one 32-bit load per modulus)
    const i64 tile = blockIdx.x;
    const int l = blockIdx.y;
    const i64 tm = tile / p.tiles_n, tn = tile % p.tiles_n;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const i64 m0 = tm*OZ_BM + lane*RW;
    if (m0 >= p.M) return;
    double* C = p.C + p.c_l[l];
    i64 cm[RW];
    double rsc[RW];                            // 2^-sA of each row (0 past the operand)
    bool fast = true;
    int sa[RW];
    #pragma unroll
    for (int r = 0; r < RW; r++)
    {
        const bool in = m0 + r < p.M;
        cm[r] = in ? p.c_m[m0 + r] : 0;
        sa[r] = in ? p.sA[(i64)l*p.M + m0 + r] : 0;
        fast = fast && sa[r] > -500 && sa[r] < 500;
        rsc[r] = in ? pow2i(-sa[r]) : 0.0;
    }
    const unsigned char* base = p.R + ((((i64)l*p.tiles_m + tm)*p.tiles_n + tn)*NM)*(i64)CRT_OUT_TILE + lane*RW;
    const int c0 = blockIdx.z*(CRT_BN/4), c1 = c0 + CRT_BN/4;
    // the first chunk's residues of the next column are loaded while this
    // one is combined
    uint32_t wn[NM];
    auto load = [&](int col) {
        #pragma unroll
        for (int q = 0; q < NM; q++)
            wn[q] = *reinterpret_cast<const uint32_t*>(base + q*(i64)CRT_OUT_TILE + col*OZ_BM);
    };
    if (tn*CRT_BN + c0 + warp < p.N) load(c0 + warp);
    for (int col = c0 + warp; col < c1; col += 8)
    {
        const i64 n = tn*CRT_BN + col;
        if (n >= p.N) break;
        uint32_t wc[NM];
        #pragma unroll
        for (int q = 0; q < NM; q++) wc[q] = wn[q];
        if (col + 8 < c1 && n + 8 < p.N) load(col + 8);
        float v[RW][NM];
        #pragma unroll
        for (int q = 0; q < NM; q++)
        {
            uint32_t rs[RW];
            #pragma unroll
            for (int r = 0; r < RW; r++) rs[r] = (wc[q] >> (8*r)) & 0xFFu;
            for (int ch = 1; ch < p.chunks; ch++)
            {
                const uint32_t w = *reinterpret_cast<const uint32_t*>(base + ch*p.chunk_bytes +
                                                                      q*(i64)CRT_OUT_TILE + col*OZ_BM);
                #pragma unroll
                for (int r = 0; r < RW; r++) rs[r] += (w >> (8*r)) & 0xFFu;
            }
            const float mq = p.cc.m[q], inv = p.cc.inv[q], gi = p.cc.ginv[q];
            #pragma unroll
            for (int r = 0; r < RW; r++)
            {
                // r_q minus the digits found so far at their weights, times the
                // inverse weight, modulo m_q, balanced: |.| < 2^18 and 2^14, exact
                float t = __fsub_rn(__int_as_float(0x4B000000 | (int)rs[r]), F_BIAS);
                #pragma unroll
                for (int i = 0; i < q; i++) t = __fmaf_rn(-v[r][i], p.cc.g[q][i], t);
                t = crt_reduce(t, mq, inv);
                v[r][q] = crt_reduce(__fmul_rn(t, gi), mq, inv);
            }
        }
        const int sb = p.sB[(i64)l*p.N + n];
        const double csc = pow2i(-sb);
        const i64 cn = p.c_n[n];
        #pragma unroll
        for (int r = 0; r < RW; r++)
        {
            if (m0 + r >= p.M) break;
            double x = (double)v[r][NM - 1];
            #pragma unroll
            for (int q = NM - 2; q >= 0; q--) x = fma(x, p.cc.md[q], (double)v[r][q]);
            // 2^-(sA+sB) as two normal powers of two where the shifts allow
            const double val = p.alpha*((fast && sb > -500 && sb < 500) ? x*rsc[r]*csc : ldexp(x, -(sa[r] + sb)));
            double* dst = C + cm[r] + cn;
            *dst = p.beta == 0.0 ? val : val + p.beta*(*dst);
        }
    }
}

void stats(const OzOperand& o, int* e_out, double* ss_out, cudaStream_t st)
{
    TimedLaunch t("oz_stats", st);
    if (o.rmode == 0)
    {
        const int ksplit = (int)std::min<i64>(32, std::max<i64>(1, o.K/256));
        dbuf pe((size_t)o.L*ksplit*o.R*sizeof(int), st), ps((size_t)o.L*ksplit*o.R*sizeof(double), st);
        dim3 grid((unsigned)((o.R + ST_THREADS - 1)/ST_THREADS), (unsigned)ksplit, (unsigned)o.L);
        oz_stats_rows<<<grid, ST_THREADS, 0, st>>>(o, ksplit, pe.as<int>(), ps.as<double>());
        check_launch("oz_stats_rows");
        oz_stats_final<<<(unsigned)((o.R*o.L + 255)/256), 256, 0, st>>>(o.R, o.L, ksplit, pe.as<int>(),
                                                                        ps.as<double>(), e_out, ss_out);
        check_launch("oz_stats_final");
    }
    else
    {
        dbuf pe((size_t)o.L*o.R*sizeof(int), st), ps((size_t)o.L*o.R*sizeof(double), st);
        dim3 grid((unsigned)((o.R*32 + ST_THREADS - 1)/ST_THREADS), 1, (unsigned)o.L);
        oz_stats_k<<<grid, ST_THREADS, 0, st>>>(o, pe.as<int>(), ps.as<double>());
        check_launch("oz_stats_k");
        oz_stats_final<<<(unsigned)((o.R*o.L + 255)/256), 256, 0, st>>>(o.R, o.L, 1, pe.as<int>(),
                                                                        ps.as<double>(), e_out, ss_out);
        check_launch("oz_stats_final");
    }
}

// ---------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------

template <int S, int KIND>
constexpr int stages_for()
{
    return std::min(6, (200*1024)/(S*(A_TILE + bn_of(S, KIND)*OZ_BK)));
}

template <int S, int KIND>
size_t gemm_smem_bytes()
{
    constexpr int BN = bn_of(S, KIND);
    return (size_t)stages_for<S, KIND>()*S*(A_TILE + BN*OZ_BK) + 1024 /* alignment */ +
           (2*stages_for<S, KIND>() + 3)*8 + 16 + (OZ_BM + BN)*8 + BN*8;
}

template <int S, int KIND>
void launch_gemm(const OzGemmArgs& a, cudaStream_t st)
{
    constexpr int STG = stages_for<S, KIND>();
    auto kern = ozaki_gemm_kernel<S, STG, KIND>;
    const size_t bytes = gemm_smem_bytes<S, KIND>();
    TB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    const i64 tiles = ((a.M + OZ_BM - 1)/OZ_BM)*((a.N + bn_of(S, KIND) - 1)/bn_of(S, KIND));
    dim3 grid((unsigned)tiles, (unsigned)a.L, 1);
    kern<<<grid, OZ_THREADS, bytes, st>>>(a);
    check_launch("ozaki_gemm_kernel");
}

template <int KIND>
void gemm_dispatch_kind(int S, const OzGemmArgs& a, cudaStream_t st)
{
    switch (S)
    {
        case 1: launch_gemm<1, KIND>(a, st); break;
        case 2: launch_gemm<2, KIND>(a, st); break;
        case 3: launch_gemm<3, KIND>(a, st); break;
        case 4: launch_gemm<4, KIND>(a, st); break;
        case 5: launch_gemm<5, KIND>(a, st); break;
        case 6: launch_gemm<6, KIND>(a, st); break;
        case 7: launch_gemm<7, KIND>(a, st); break;
        default: launch_gemm<8, KIND>(a, st); break;
    }
}

void gemm_dispatch(int kind, int S, const OzGemmArgs& a, cudaStream_t st)
{
    TimedLaunch t("ozaki_gemm_kernel", st);
    if (kind == OZ_I8) gemm_dispatch_kind<OZ_I8>(S, a, st);
    else if (kind == OZ_BF16) gemm_dispatch_kind<OZ_BF16>(S, a, st);
    else launch_gemm<1, OZ_TF32>(a, st);
}

// a-priori normwise error estimate for S slices (rounding of both operands
// to S digits plus the dropped cross terms), from per-row maxima and norms:
// rounding row i to S digits leaves an error of about 2^(e_i - 7S) per
// element (uniform, variance 1/3), so the squared relative error of the
// operand is K/3 * sum_i 4^(e_i - 7S) / sum_i ss_i
struct ErrorModel
{
    double ra2 = 0, rb2 = 0;      // squared relative error at S = 0: mantissa ...
    int ea = 0, eb = 0;           // ... and binary exponent
    static void build(const std::vector<int>& e, const std::vector<double>& ss, i64 K, double& m, int& ex)
    {
        int emax = -100000;
        for (int v : e) emax = std::max(emax, v);
        double num = 0.0, den = 0.0;
        for (size_t i = 0; i < e.size(); i++)
        {
            num += std::ldexp(1.0, 2*(e[i] - emax));
            den += ss[i];
        }
        if (den <= 0.0 || num == 0.0) { m = 0.0; ex = 0; return; }
        m = (double)K/3.0*num/den;
        ex = 2*emax;
    }
    ErrorModel(const std::vector<int>& eA, const std::vector<double>& ssA,
               const std::vector<int>& eB, const std::vector<double>& ssB, i64 K)
    {
        build(eA, ssA, K, ra2, ea);
        build(eB, ssB, K, rb2, eb);
    }
    // residual bound of S digits relative to 2^e: base 254 (INT8):
    // 1/(2*127*254^(S-1)); base 128 (BF16): 2^-7S
    static double resolution(int kind, int S)
    {
        return kind == OZ_I8 ? 0.5/(127.0*std::pow(254.0, S - 1)) : std::ldexp(1.0, -7*S);
    }
    double operator()(int S, int kind) const
    {
        const double r = resolution(kind, S);
        const double ra = ra2 > 0 ? std::sqrt(std::ldexp(ra2, ea))*r : 0.0;
        const double rb = rb2 > 0 ? std::sqrt(std::ldexp(rb2, eb))*r : 0.0;
        // dropped pairs p + q > S + 1 are below the rounding terms by ~1/base
        return (ra + rb)*(1.0 + 2.0*S*(kind == OZ_I8 ? 1.0/127.0 : std::ldexp(1.0, -7)));
    }
};

// weight of diagonal d = p + q (p, q >= 1) in the epilogue's FP64 sum
double diagonal_weight(int kind, int d)
{
    return kind == OZ_I8 ? 1.0/(127.0*127.0*std::pow(254.0, d - 2)) : std::ldexp(1.0, 2 - 7*d);
}

// ---- scheme II host side ------------------------------------------------------

// (2 m + 1)/2 rounded: x mod m in [-(m-1)/2, (m-1)/2] ([-128, 127] for 256)
i64 centred(i64 x, i64 m)
{
    x %= m;
    if (x < 0) x += m;
    if (2*x >= m) x -= m;
    return x;
}

i64 powmod(i64 b, i64 e, i64 m)
{
    i64 r = 1 % m;
    b %= m;
    for (; e > 0; e >>= 1, b = b*b % m)
        if (e & 1) r = r*b % m;
    return r;
}

i64 invmod(i64 a, i64 m)
{
    // extended Euclid; a and m coprime
    i64 g = m, x = 0, x1 = 1, a1 = ((a % m) + m) % m;
    while (a1)
    {
        const i64 q = g/a1;
        i64 t = g - q*a1; g = a1; a1 = t;
        t = x - q*x1; x = x1; x1 = t;
    }
    return ((x % m) + m) % m;
}

// a residue plane buffer (blocks [l][row tile][k step] of nm 4 KB tiles) as
// a 4-D map: 256-byte rows, 16 rows per tile, nm tiles per block, blocks;
// a box of one modulus's tiles in four consecutive blocks (one stage's k
// steps) lands as four contiguous tiles; no swizzle
CUtensorMap plane_map(const void* base, size_t bytes, int nm)
{
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    });
    TB_CHECK(encode, TB_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
    const size_t block = (size_t)nm*CRT2_TILE;
    TB_CHECK(bytes % block == 0 && bytes/block < ((size_t)1 << 31), TB_ERR_SIZE, "Ozaki moduli planes too large");
    CUtensorMap m;
    const cuuint64_t dims[4] = {256, CRT2_TILE/256, (cuuint64_t)nm, (cuuint64_t)(bytes/block)};
    const cuuint64_t strides[3] = {256, CRT2_TILE, block};
    const cuuint32_t box[4] = {256, CRT2_TILE/256, 1, CRT_KSUB};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    const CUresult r = encode(&m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 4, const_cast<void*>(base), dims, strides, box, estr,
                              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    TB_CHECK(r == CUDA_SUCCESS, TB_ERR_CUDA, "cuTensorMapEncodeTiled failed for the Ozaki moduli planes");
    return m;
}

CrtConsts crt_consts(int nm)
{
    CrtConsts c;
    std::memset(&c, 0, sizeof(c));
    c.nm = nm;
    for (int q = 0; q < nm; q++)
    {
        const i64 m = crt_modulus(q);
        c.m[q] = (float)m;
        c.inv[q] = 1.0f/(float)m;
        c.md[q] = (double)m;
        c.invd[q] = 1.0/(double)m;
        c.c16[q] = (float)powmod(2, 16, m);
        i64 P = 1 % m;                               // m_0 ... m_(j-1) mod m_q
        for (int j = 0; j < q; j++)
        {
            c.g[q][j] = (float)centred(P, m);
            P = P*crt_modulus(j) % m;
        }
        c.ginv[q] = q == 0 ? 1.0f : (float)centred(invmod(P, m), m);
    }
    return c;
}

double crt_log2_modulus(int nm)
{
    double s = 0;
    for (int q = 0; q < nm; q++) s += std::log2((double)crt_modulus(q));
    return s;
}

// norm bound exponent P of the scaled rows and columns: |sum_k a b| <=
// ||a|| ||b|| <= (2^P + sqrt(K)/2)^2 stays below M/2; at most 50, so that
// |a| < 2^51 fits the digit extraction
int crt_norm_bits(int nm)
{
    return std::min(50, (int)std::floor((crt_log2_modulus(nm) - 1.05)/2.0));
}

// a-priori normwise error of scheme II with nm moduli: rounding x*2^s to an
// integer leaves an error below 1/2 (uniform, variance 1/12) per element, so
// ||dA||^2 ~ K/12 sum_i 4^(-s_i) with 2^-s_i ~ 2^(e_i - P)
struct CrtErrorModel
{
    double ra = 0, rb = 0;   // sqrt(K/12 sum 4^(e_i - emax)/sum ss) ...
    int ea = 0, eb = 0;      // ... and emax
    static void build(const std::vector<double>& ss, i64 K, double& r, int& emax)
    {
        std::vector<int> e(ss.size());
        emax = -100000;
        double den = 0.0;
        for (size_t i = 0; i < ss.size(); i++)
        {
            const double v = std::sqrt(ss[i]);
            int x = -100000;
            if (v > 0.0 && v <= 1.7e308) std::frexp(v*(1.0 + 0x1p-20), &x);
            e[i] = x;
            emax = std::max(emax, x);
            den += ss[i];
        }
        double num = 0.0;
        for (int x : e)
            if (x > -100000) num += std::ldexp(1.0, 2*(x - emax));
        r = den > 0.0 && num > 0.0 ? std::sqrt((double)K/12.0*num/den) : 0.0;
    }
    CrtErrorModel(const std::vector<double>& ssA, const std::vector<double>& ssB, i64 K)
    {
        build(ssA, K, ra, ea);
        build(ssB, K, rb, eb);
    }
    double operator()(int nm) const
    {
        const int P = crt_norm_bits(nm);
        return (ra > 0 ? std::ldexp(ra, ea - P) : 0.0) + (rb > 0 ? std::ldexp(rb, eb - P) : 0.0);
    }
};

// modelled device time of the two INT8 schemes, from rates measured on the
// ladder contraction (m = 25600, n = 2304, k = 25600) on one B200: the fused
// slice-pair kernel runs 2.7e15 INT8 ops/s per pair, the moduli GEMM 2.8e15
// per modulus; writing a plane costs 5.3e-13 s (digits) or 4.1e-13 s
// (residues) per operand element, and the CRT combination 1.1e-12 s per
// output element and modulus
double scheme1_seconds(int S, double m, double n, double k)
{
    return 0.5*S*(S + 1)*2.0*m*n*k/2.7e15 + S*(m + n)*k*5.3e-13;
}
double scheme2_seconds(int N, double m, double n, double k)
{
    return N*2.0*m*n*k/2.8e15 + N*(m + n)*k*4.1e-13 + N*m*n*1.1e-12;
}

template <int NM>
void launch_crt_slice(const OzOperand& o, const int* s, void* out, const PlaneGeom& pg, const CrtConsts& cc,
                      cudaStream_t st)
{
    launch_slice<NM, OZ_I8, false, true>(o, s, out, pg, st, &cc);
}

void crt_slice_dispatch(int nm, const OzOperand& o, const int* s, void* out, const PlaneGeom& pg,
                        const CrtConsts& cc, cudaStream_t st)
{
    switch (nm)
    {
        case 2: launch_crt_slice<2>(o, s, out, pg, cc, st); break;
        case 3: launch_crt_slice<3>(o, s, out, pg, cc, st); break;
        case 4: launch_crt_slice<4>(o, s, out, pg, cc, st); break;
        case 5: launch_crt_slice<5>(o, s, out, pg, cc, st); break;
        case 6: launch_crt_slice<6>(o, s, out, pg, cc, st); break;
        case 7: launch_crt_slice<7>(o, s, out, pg, cc, st); break;
        case 8: launch_crt_slice<8>(o, s, out, pg, cc, st); break;
        case 9: launch_crt_slice<9>(o, s, out, pg, cc, st); break;
        case 10: launch_crt_slice<10>(o, s, out, pg, cc, st); break;
        case 11: launch_crt_slice<11>(o, s, out, pg, cc, st); break;
        case 12: launch_crt_slice<12>(o, s, out, pg, cc, st); break;
        case 13: launch_crt_slice<13>(o, s, out, pg, cc, st); break;
        case 14: launch_crt_slice<14>(o, s, out, pg, cc, st); break;
        case 15: launch_crt_slice<15>(o, s, out, pg, cc, st); break;
        default: launch_crt_slice<16>(o, s, out, pg, cc, st); break;
    }
}

void crt_combine_dispatch(const CrtCombineArgs& a, i64 tiles, i64 L, cudaStream_t st)
{
    dim3 grid((unsigned)tiles, (unsigned)L, 4);
    switch (a.cc.nm)
    {
#define TB_CRT_CASE(n) case n: oz_crt_combine<n><<<grid, 256, 0, st>>>(a); break;
        TB_CRT_CASE(2) TB_CRT_CASE(3) TB_CRT_CASE(4) TB_CRT_CASE(5) TB_CRT_CASE(6) TB_CRT_CASE(7)
        TB_CRT_CASE(8) TB_CRT_CASE(9) TB_CRT_CASE(10) TB_CRT_CASE(11) TB_CRT_CASE(12) TB_CRT_CASE(13)
        TB_CRT_CASE(14) TB_CRT_CASE(15)
        default: oz_crt_combine<16><<<grid, 256, 0, st>>>(a); break;
#undef TB_CRT_CASE
    }
    check_launch("oz_crt_combine");
}

// scheme II on the statistics already computed: shifts, residue planes,
// one INT8 GEMM per modulus (per exact run of k), CRT combination into C
void crt_run(OzakiJob& j, int nm, cudaStream_t st)
{
    const GemmView& v = j.v;
    TB_CHECK(nm >= 2 && nm <= CRT_MAX, TB_ERR_ARG, "Ozaki moduli count must be 2..16");
    const CrtConsts cc = crt_consts(nm);
    const int P = crt_norm_bits(nm);
    dbuf shA((size_t)v.l*v.m*sizeof(int), st), shB((size_t)v.l*v.n*sizeof(int), st);
    if (v.l*v.m > 0)
    {
        oz_crt_shifts<<<(unsigned)((v.l*v.m + 255)/256), 256, 0, st>>>(j.sA.as<double>(), v.l*v.m, P, shA.as<int>());
        check_launch("oz_crt_shifts");
    }
    if (v.l*v.n > 0)
    {
        oz_crt_shifts<<<(unsigned)((v.l*v.n + 255)/256), 256, 0, st>>>(j.sB.as<double>(), v.l*v.n, P, shB.as<int>());
        check_launch("oz_crt_shifts");
    }
    OzOperand oa = {j.A, j.tab->a_m, j.tab->a_k, j.tab->a_l, v.m, v.k, v.l, v.amode,
                    j.tab->a_m_step, j.tab->a_k_step};
    OzOperand ob = {j.B, j.tab->b_n, j.tab->b_k, j.tab->b_l, v.n, v.k, v.l, v.bmode,
                    j.tab->b_n_step, j.tab->b_k_step};
    // 128-row tiles of A and B, an even number of each: a CTA pair takes
    // 256 rows of A and 256 columns (two B tiles) of the output
    const i64 k_steps = ((v.k + OZ_BK*CRT_KSUB - 1)/(OZ_BK*CRT_KSUB))*CRT_KSUB;   // a multiple of four
    const PlaneGeom ga = {OZ_BM, 2*((v.m + 255)/256), k_steps, nm};
    const PlaneGeom gb = {OZ_BM, 2*((v.n + CRT_BN - 1)/CRT_BN), k_steps, nm};
    TB_CHECK(ga.k_steps < (1ll << 31), TB_ERR_SIZE, "Ozaki contraction length above 2^31");
    dbuf pa((size_t)(v.l*ga.tiles*ga.k_steps*nm*A_TILE), st);
    dbuf pb((size_t)(v.l*gb.tiles*gb.k_steps*nm*CRT2_TILE), st);
    crt_slice_dispatch(nm, oa, shA.as<int>(), pa.ptr, ga, cc, st);
    crt_slice_dispatch(nm, ob, shB.as<int>(), pb.ptr, gb, cc, st);

    // one launch per exact run of k steps; each writes its own residues of
    // the 128 x 256 tiles
    const i64 tiles_n = gb.tiles/2;
    const i64 tiles = ga.tiles*tiles_n;
    const int chunks = (int)((ga.k_steps + CRT_KT_RUN - 1)/CRT_KT_RUN);
    const i64 chunk_bytes = v.l*tiles*nm*(i64)CRT_OUT_TILE;
    TB_CHECK(tiles < (1ll << 31) && v.l*nm < 65536, TB_ERR_SIZE, "Ozaki moduli path: grid too large");
    dbuf res((size_t)(chunks*chunk_bytes), st);
    CrtGemmArgs g;
    g.pA = pa.as<unsigned char>(); g.pB = pb.as<unsigned char>();
    g.tmA = plane_map(pa.ptr, (size_t)(v.l*ga.tiles*ga.k_steps*nm*A_TILE), nm);
    g.tmB = plane_map(pb.ptr, (size_t)(v.l*gb.tiles*gb.k_steps*nm*CRT2_TILE), nm);
    g.tiles_m = ga.tiles; g.tiles_n = tiles_n;
    g.k_steps = (int)ga.k_steps;
    g.nm = nm;
    g.L = (int)v.l;
    for (int q = 0; q < CRT_MAX; q++) { g.m[q] = cc.m[q]; g.inv[q] = cc.inv[q]; g.c16[q] = cc.c16[q]; }
    const size_t smem = crt_gemm2_smem();
    TB_CUDA(cudaFuncSetAttribute(oz_crt_gemm2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    for (int c = 0; c < chunks; c++)
    {
        g.R = res.as<unsigned char>() + c*chunk_bytes;
        g.kt0 = c*CRT_KT_RUN;
        g.kt1 = (int)std::min<i64>(ga.k_steps, (i64)(c + 1)*CRT_KT_RUN);
        TimedLaunch t("oz_crt_gemm", st);
        const i64 items = nm*v.l*tiles/2;
        TB_CHECK(2*items < ((i64)1 << 31), TB_ERR_SIZE, "Ozaki moduli path: grid too large");
        oz_crt_gemm2<<<(unsigned)(2*items), OZ_THREADS, smem, st>>>(g);
        check_launch("oz_crt_gemm");
    }

    CrtCombineArgs a;
    a.R = res.as<unsigned char>();
    a.chunks = chunks;
    a.chunk_bytes = chunk_bytes;
    a.C = j.C;
    a.c_m = j.tab->c_m; a.c_n = j.tab->c_n; a.c_l = j.tab->c_l;
    a.sA = shA.as<int>(); a.sB = shB.as<int>();
    a.M = v.m; a.N = v.n; a.tiles_m = ga.tiles; a.tiles_n = tiles_n;
    a.alpha = j.alpha; a.beta = j.beta;
    a.cc = cc;
    TimedLaunch t("oz_crt_combine", st);
    crt_combine_dispatch(a, tiles, v.l, st);
}

} // namespace

int ozaki_error_flag()
{
    int v = 0;
    cudaMemcpyFromSymbol(&v, g_oz_error, sizeof(int));
    if (v)
    {
        // reported once: the next check starts clean
        const int zero = 0;
        cudaMemcpyToSymbol(g_oz_error, &zero, sizeof(int));
    }
    return v;
}

void ozaki_inject_wait_timeout(int step, double wait_seconds)
{
    const unsigned long long ns = wait_seconds > 0.0 ? (unsigned long long)(wait_seconds*1e9) : WAIT_NS;
    TB_CUDA(cudaMemcpyToSymbol(g_oz_skip_step, &step, sizeof(int)));
    TB_CUDA(cudaMemcpyToSymbol(g_oz_wait_ns, &ns, sizeof(ns)));
}

void ozaki_begin(OzakiJob& j, cudaStream_t st)
{
    const GemmView& v = j.v;
    j.tab = gemm_tables(v, 128, 128, 16, st);
    TB_CHECK(v.m < (1ll << 31) && v.n < (1ll << 31) && v.k < (1ll << 31), TB_ERR_SIZE,
             "Ozaki path: extents beyond 2^31");
    TB_CHECK(v.l*OZ_SMAX < (1ll << 31), TB_ERR_SIZE, "Ozaki path: batch too large");
    j.eA = dbuf((size_t)v.l*v.m*sizeof(int), st);
    j.eB = dbuf((size_t)v.l*v.n*sizeof(int), st);
    j.sA = dbuf((size_t)v.l*v.m*sizeof(double), st);
    j.sB = dbuf((size_t)v.l*v.n*sizeof(double), st);
    OzOperand oa = {j.A, j.tab->a_m, j.tab->a_k, j.tab->a_l, v.m, v.k, v.l, v.amode,
                    j.tab->a_m_step, j.tab->a_k_step};
    OzOperand ob = {j.B, j.tab->b_n, j.tab->b_k, j.tab->b_l, v.n, v.k, v.l, v.bmode,
                    j.tab->b_n_step, j.tab->b_k_step};
    stats(oa, j.eA.as<int>(), j.sA.as<double>(), st);
    stats(ob, j.eB.as<int>(), j.sB.as<double>(), st);
}

void ozaki_end(OzakiJob& j, cudaStream_t st, bool stats_ready)
{
    const GemmView& v = j.v;
    const int kind = j.kind;
    TB_CHECK(kind == OZ_I8 || kind == OZ_BF16 || (kind == OZ_TF32 && j.single), TB_ERR_ARG,
             "split-precision kind must be INT8 or BF16 slices, or a single TF32/BF16 pass");
    int S = j.single ? 1 : j.slices;
    if (j.single)
    {
        // one pass in the low precision: x' rounded to 8 (BF16) or 11 (TF32)
        // significant bits in both operands, FP32 accumulation
        j.res.est_error = std::sqrt(2.0)*(kind == OZ_BF16 ? std::ldexp(1.0, -9) : std::ldexp(1.0, -11));
    }
    else
    {
        // the error model (and, without an explicit count, the slice count)
        std::vector<int> heA(v.l*v.m), heB(v.l*v.n);
        std::vector<double> hsA(v.l*v.m), hsB(v.l*v.n);
        if (stats_ready)
        {
            // the statistics are complete: copy them without queueing behind
            // the caller's stream
            TB_CUDA(cudaMemcpy(heA.data(), j.eA.ptr, heA.size()*sizeof(int), cudaMemcpyDeviceToHost));
            TB_CUDA(cudaMemcpy(heB.data(), j.eB.ptr, heB.size()*sizeof(int), cudaMemcpyDeviceToHost));
            TB_CUDA(cudaMemcpy(hsA.data(), j.sA.ptr, hsA.size()*sizeof(double), cudaMemcpyDeviceToHost));
            TB_CUDA(cudaMemcpy(hsB.data(), j.sB.ptr, hsB.size()*sizeof(double), cudaMemcpyDeviceToHost));
        }
        else
        {
            TB_CUDA(cudaMemcpyAsync(heA.data(), j.eA.ptr, heA.size()*sizeof(int), cudaMemcpyDeviceToHost, st));
            TB_CUDA(cudaMemcpyAsync(heB.data(), j.eB.ptr, heB.size()*sizeof(int), cudaMemcpyDeviceToHost, st));
            TB_CUDA(cudaMemcpyAsync(hsA.data(), j.sA.ptr, hsA.size()*sizeof(double), cudaMemcpyDeviceToHost, st));
            TB_CUDA(cudaMemcpyAsync(hsB.data(), j.sB.ptr, hsB.size()*sizeof(double), cudaMemcpyDeviceToHost, st));
            TB_CUDA(cudaStreamSynchronize(st));
        }
        const ErrorModel est(heA, hsA, heB, hsB, v.k);
        // scheme II (moduli) is an INT8 option: its count from the
        // tolerance, or the caller's when it forces the scheme
        int nm = 0;
        double nm_err = 0;
        if (kind == OZ_I8 && j.scheme != 1)
        {
            const CrtErrorModel est2(hsA, hsB, v.k);
            if (j.scheme == 2 && S > 0) nm = S;
            else
                for (int q = 2; q <= CRT_MAX; q++)
                    if (est2(q)*4.0 <= j.tol) { nm = q; break; }
            if (j.scheme == 2 && nm == 0) nm = CRT_MAX;
            if (nm > 0) nm_err = est2(nm);
        }
        bool feasible1 = S > 0;
        if (S <= 0)
        {
            S = OZ_SMAX;
            for (int s = 1; s <= OZ_SMAX; s++)
            {
                // safety factor 4 between the estimate and the target
                if (est(s, kind)*4.0 <= j.tol) { S = s; feasible1 = true; break; }
            }
        }
        // moduli when forced, or when they meet the tolerance in less
        // modelled time than the slices
        const double mm = (double)v.m*v.l, nn = (double)v.n, kk = (double)v.k;
        const bool use2 = nm > 0 && (j.scheme == 2 ||
                                     (j.scheme == 0 && (!feasible1 || scheme2_seconds(nm, mm, nn, kk) <
                                                                      scheme1_seconds(S, mm, nn, kk))));
        if (use2)
        {
            j.res.scheme = 2;
            j.res.slices = nm;
            j.res.est_error = nm_err;
            crt_run(j, nm, st);
            return;
        }
        if (S >= 1 && S <= OZ_SMAX) j.res.est_error = est(S, kind);
    }
    TB_CHECK(S >= 1 && S <= OZ_SMAX, TB_ERR_ARG, "Ozaki slice count must be 1..8");
    j.res.slices = S;

    OzOperand oa = {j.A, j.tab->a_m, j.tab->a_k, j.tab->a_l, v.m, v.k, v.l, v.amode,
                    j.tab->a_m_step, j.tab->a_k_step};
    OzOperand ob = {j.B, j.tab->b_n, j.tab->b_k, j.tab->b_l, v.n, v.k, v.l, v.bmode,
                    j.tab->b_n_step, j.tab->b_k_step};
    const int esz = elem_bytes(kind);
    const i64 ke = OZ_BK/esz;              // k elements per MMA step
    const PlaneGeom ga = {OZ_BM, (v.m + OZ_BM - 1)/OZ_BM, (v.k + ke - 1)/ke, S};
    const int bn = bn_of(S, kind);
    const PlaneGeom gb = {bn, (v.n + bn - 1)/bn, ga.k_steps, S};
    dbuf pa((size_t)(v.l*ga.tiles*ga.k_steps*S*A_TILE), st), pb((size_t)(v.l*gb.tiles*gb.k_steps*S*bn*OZ_BK), st);
    slice_dispatch(kind, j.single, S, oa, j.eA.as<int>(), pa.ptr, ga, st);
    slice_dispatch(kind, j.single, S, ob, j.eB.as<int>(), pb.ptr, gb, st);

    // exact accumulation of the digit products, (#pairs on a diagonal) *
    // (k run) * max|digit|^2 below 2^31 (INT32, digits up to 127) or 2^24
    // (FP32 holds integers exactly up to there; digits up to 64): the kernel
    // flushes the accumulators into C after each such run of k steps; a
    // single pass runs the whole K at once
    const i64 acc_limit = kind == OZ_I8 ? (i64)0x7fffffff : ((i64)1 << 24);
    const i64 dmax = kind == OZ_I8 ? 127 : 64;
    const i64 krun = j.single ? 0 : (acc_limit/((i64)S*dmax*dmax))/ke*ke;
    TB_CHECK(j.single || krun >= ke, TB_ERR_SIZE, "Ozaki exactness run below one k step");
    TB_CHECK(v.k <= (i64)0x7fffffff, TB_ERR_SIZE, "Ozaki contraction length above 2^31");
    OzGemmArgs g;
    g.C = j.C;
    g.c_m = j.tab->c_m; g.c_n = j.tab->c_n; g.c_l = j.tab->c_l;
    g.eA = j.eA.as<int>(); g.eB = j.eB.as<int>();
    g.pA = pa.as<unsigned char>(); g.pB = pb.as<unsigned char>();
    g.M = v.m; g.N = v.n; g.K = v.k; g.L = v.l;
    g.tiles_m = ga.tiles; g.tiles_n = gb.tiles;
    g.k_steps = (int)ga.k_steps;
    g.kt_flush = (int)(krun/ke);
    g.alpha = j.alpha;
    g.beta = j.beta;
    for (int d = 2; d < OZ_SMAX + 2; d++)
        g.w[d - 2] = j.single ? 1.0 : diagonal_weight(kind, d);   // a single pass: weight 1
    gemm_dispatch(kind, S, g, st);
}

OzakiResult ozaki_mult(const GemmView& v, const double* A, const double* B, double* C,
                       double alpha, double beta, double tol, int slices, cudaStream_t st,
                       int kind, bool single, int scheme)
{
    OzakiJob j;
    j.v = v; j.A = A; j.B = B; j.C = C;
    j.alpha = alpha; j.beta = beta; j.tol = tol; j.slices = slices;
    j.kind = kind; j.single = single; j.scheme = scheme;
    ozaki_begin(j, st);
    ozaki_end(j, st, false);
    return j.res;
}

} // namespace tb
