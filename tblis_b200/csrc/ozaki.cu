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
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
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
constexpr unsigned long long WAIT_NS = 2000000000ull;   // bounded waits: 2 s

__device__ int g_oz_error = 0;       // set by a kernel whose bounded wait gave up

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

// waits for the phase with the given parity to complete, at most WAIT_NS;
// returns false (and records the error) when the wait gave up
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
            if (globaltimer() - t0 > WAIT_NS)
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
            for (int kt = 0; kt < kt_count && !*abort_flag; kt++)
            {
                const int s = kt % STAGES;
                if (kt >= STAGES && !mbar_wait(&empty[s], ((kt/STAGES) & 1) ^ 1, abort_flag)) break;
                unsigned char* st = smem + s*STAGE_BYTES;
                mbar_expect_tx(&full[s], STAGE_BYTES);
                // the S slice tiles of A, then those of B, each one contiguous block
                bulk_load(st, p.pA + (((i64)l*p.tiles_m + tm)*p.k_steps + kt)*(S*A_TILE), S*A_TILE, &full[s]);
                bulk_load(st + S*A_TILE, p.pB + (((i64)l*p.tiles_n + tn)*p.k_steps + kt)*(S*B_TILE),
                          S*B_TILE, &full[s]);
            }
            // drain: the copies of the last stages must have landed before exit
            const int last = min(kt_count, STAGES);
            for (int i = 0; i < last; i++)
            {
                const int kt = kt_count - 1 - i;
                mbar_wait(&full[kt % STAGES], (kt/STAGES) & 1, abort_flag);
            }
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
            mbar_wait(done, 0, abort_flag);
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
constexpr int SL_BLOCKS_PER_SM = 3;
constexpr size_t SL_SMEM = 2*SL_T*SL_LD*sizeof(double);

// writes the S tiled planes (PlaneGeom) of 64x64 tiles of the operand:
// digit planes, or (SINGLE, S = 1) x' rounded to the plane type. Rows and k
// beyond the operand, up to whole tiles and k steps, get zeros.
// Persistent blocks walk the tiles; the gather of the next tile (cp.async,
// zero-filled outside the operand) runs while the current one is converted.
template <int S, int KIND, bool SINGLE>
__global__ void __launch_bounds__(256, SL_BLOCKS_PER_SM)
oz_slice(const OzOperand o, const int* e_rows, void* out_, const PlaneGeom pg, unsigned tiles_r, unsigned tiles_k)
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
            if constexpr (KIND == OZ_I8 && !SINGLE)
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

template <int S, int KIND, bool SINGLE>
void launch_slice(const OzOperand& o, const int* e, void* out, const PlaneGeom& pg, cudaStream_t st)
{
    // every row of the row tiles (64-row slicing tiles may pass the last
    // one: the kernel stops at it), every k of the k steps
    const i64 tiles_r = (pg.tiles*pg.tile_rows + SL_T - 1)/SL_T;
    const i64 tiles_k = (pg.k_steps*(OZ_BK/elem_bytes(KIND)) + SL_T - 1)/SL_T;
    const i64 ntiles = tiles_r*tiles_k*o.L;
    if (ntiles == 0) return;
    TB_CHECK(ntiles < ((i64)1 << 31), TB_ERR_SIZE, "Ozaki operand above 2^31 tiles of 64x64");
    const i64 grid = std::min<i64>(ntiles, (i64)device_sm_count()*SL_BLOCKS_PER_SM);
    TB_CUDA(cudaFuncSetAttribute(oz_slice<S, KIND, SINGLE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)SL_SMEM));
    TimedLaunch t("oz_slice", st);
    oz_slice<S, KIND, SINGLE><<<(unsigned)grid, 256, SL_SMEM, st>>>(o, e, out, pg, (unsigned)tiles_r,
                                                                     (unsigned)tiles_k);
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

} // namespace

int ozaki_error_flag()
{
    int v = 0;
    cudaMemcpyFromSymbol(&v, g_oz_error, sizeof(int));
    return v;
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
        if (S <= 0)
        {
            S = OZ_SMAX;
            for (int s = 1; s <= OZ_SMAX; s++)
            {
                // safety factor 4 between the estimate and the target
                if (est(s, kind)*4.0 <= j.tol) { S = s; break; }
            }
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
                       int kind, bool single)
{
    OzakiJob j;
    j.v = v; j.A = A; j.B = B; j.C = C;
    j.alpha = alpha; j.beta = beta; j.tol = tol; j.slices = slices;
    j.kind = kind; j.single = single;
    ozaki_begin(j, st);
    ozaki_end(j, st, false);
    return j.res;
}

} // namespace tb
