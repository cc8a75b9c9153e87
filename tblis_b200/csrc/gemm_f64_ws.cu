// gemm_f64_ws.cu -- packed, warp-specialised grouped FP64 DMMA path.
//
// The grouped GEMMs of one launch (a batch of independent contractions, the
// irrep GEMMs of a DPD contraction, the block products of an indexed-DPD
// contraction) read their operands through block-scatter vectors. Gathering
// those elements with per-thread cp.async inside the GEMM caps the operand
// stream at about 11 bytes per cycle per SM on B200 (the SM's outstanding
// L1 requests), while a 64x64 FP64 tile needs 16 bytes per cycle to keep the
// DMMA pipe busy. The work is therefore split in two launches:
//
//  * gemm_f64_pack_kernel gathers every row panel of A and column panel of B
//    once, through the scatter vectors (reads coalesced along whichever GEMM
//    dimension is contiguous in memory, staged through shared memory), into
//    contiguous 16-wide k steps: a P x 16 block per step, rows of 16 doubles,
//    the k index XOR-swizzled by row (k ^ 4*(row % 4)) so that the MMA
//    fragment reads are free of bank conflicts. It is bound by HBM bandwidth.
//  * gemm_f64_ws_kernel runs one continuous pipeline per CTA over all the
//    tiles it takes from the dynamic queue. One producer lane publishes each
//    tile's C row and column offsets in a ring of tile slots and streams the
//    tile's packed A and B blocks into a ring of shared-memory stages with
//    bulk copies (cp.async.bulk, completing on an mbarrier by transaction
//    bytes); four consumer warps run the m16n8k16 FP64 MMAs on each stage and,
//    after a tile's last k step, scatter alpha*AB + beta*C through the tile's
//    C offsets. The next tile's copies overlap the current tile's MMAs and C
//    update.
//
// Every group has its own tile shape (64x64, 64x32, 32x64 or 32x32, chosen by
// the plan from its M and N), so a contraction of 4..32 extents does not pad
// to 64x64 while a large irrep GEMM keeps the 64x64 tile.
//
// Every wait is bounded (wall clock, g_f64_wait_ns): a wait that gives up
// sets a flag that ends all roles of the CTA and records the error for the
// host (gemm_f64_error_flag); the producer waits for the copies it issued to
// land before it returns.
#include "gemm_f64.hpp"
#include "gemm_f64_dev.cuh"

#include <algorithm>
#include <cstdint>

namespace tb
{

namespace
{

using namespace f64dev;

constexpr int WS_STAGES = 6;
constexpr int WS_TSLOTS = 4;
constexpr int WS_CONSUMERS = 4;                                    // warps, 2 x 2 over the tile
constexpr int WS_THREADS = (WS_CONSUMERS + 1)*32;                  // + one producer warp
constexpr int WS_EDGE = 64;                                         // largest tile edge
constexpr int WS_OPER = WS_EDGE*BK;                                 // one packed operand block (doubles)
constexpr int WS_STAGE = 2*WS_OPER;
constexpr unsigned long long WS_WAIT_NS = 2000000000ull;            // 2 s

constexpr int PK_THREADS = 256;
constexpr int PK_STEPS = 4;                                         // k steps gathered per pass
constexpr int PK_K = PK_STEPS*BK;

// what the consumers need of one tile
struct WsTileMeta
{
    double* C;
    double alpha, beta;
    int nst;                  // k steps; -1 ends the CTA's work
    int shape;                // bit 1: 32 rows, bit 0: 32 columns
    i64 crow[WS_EDGE];        // C offset of each tile row, -1 past M
    i64 ccol[WS_EDGE];        // C offset of each tile column, -1 past N
};

struct WsShared
{
    WsTileMeta meta[WS_TSLOTS];
    uint64_t full[WS_STAGES], empty[WS_STAGES];
    uint64_t tfull[WS_TSLOTS], tempty[WS_TSLOTS];
    int abort;
};

constexpr size_t ws_smem_bytes() { return (size_t)WS_STAGES*WS_STAGE*sizeof(double) + sizeof(WsShared); }

__device__ int g_f64_error = 0;
__device__ unsigned long long g_f64_wait_ns = WS_WAIT_NS;
__device__ int g_f64_skip_step = -1;       // test support: a stage whose copies are never issued

__device__ __forceinline__ uint32_t su32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mb_init(uint64_t* b, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(su32(b)), "r"(count) : "memory");
}

__device__ __forceinline__ bool mb_try(uint64_t* b, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                 " selp.u32 %0, 1, 0, p;\n}" : "=r"(ok) : "r"(su32(b)), "r"(parity) : "memory");
    return ok != 0;
}

__device__ __forceinline__ void mb_arrive(uint64_t* b)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" :: "r"(su32(b)) : "memory");
}

// arrives and adds the bytes that the copies of this phase will deliver
__device__ __forceinline__ void mb_arrive_expect(uint64_t* b, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(su32(b)), "r"(bytes) : "memory");
}

// one contiguous global -> shared copy by the bulk-copy engine (16-byte
// aligned addresses, a multiple of 16 bytes), completing on the mbarrier
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cta.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 :: "r"(su32(dst)), "l"((uint64_t)src), "r"(bytes), "r"(su32(bar)) : "memory");
}

__device__ __forceinline__ unsigned long long gtimer()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// bounded wait of one thread on a phase of an mbarrier; false when the CTA
// gave up (this wait ran out of time, or another role already did). With
// drain set the wait ignores the CTA's flag (the producer's last waits for
// its own copies), and is still bounded.
__device__ __noinline__ bool mb_wait_slow(uint64_t* b, uint32_t parity, volatile int* abort_flag, bool drain)
{
    const unsigned long long t0 = gtimer();
    for (unsigned it = 0;; it++)
    {
        if (mb_try(b, parity)) return true;
        if ((it & 63) == 0)
        {
            if (!drain && *abort_flag) return false;
            if (gtimer() - t0 > g_f64_wait_ns)
            {
                *abort_flag = 1;
                atomicExch(&g_f64_error, 1);
                return false;
            }
        }
    }
}

__device__ __forceinline__ bool mb_wait(uint64_t* b, uint32_t parity, volatile int* abort_flag)
{
    return mb_try(b, parity) || mb_wait_slow(b, parity, abort_flag, false);
}

// the same for a whole warp: every lane waits (and acquires what the phase
// released), and all lanes agree on the outcome
__device__ __forceinline__ bool mb_wait_warp(uint64_t* b, uint32_t parity, volatile int* abort_flag)
{
    const bool ok = mb_wait(b, parity, abort_flag);
    return __all_sync(0xffffffffu, ok) != 0;
}

// ---- packing -------------------------------------------------------------------

// steps [s0, s0 + ns) of one panel (P rows of A, or P columns of B; the
// steps run over all segments) into their packed blocks
template <int P>
__device__ __forceinline__ void pack_panel(const GroupDesc& g, bool sideB, int panel, i64 s0, i64 ns,
                                           double* __restrict__ out, double (*T)[WS_EDGE + 1], i64* sRow, i64* sK)
{
    const int t = threadIdx.x;
    const i64 extent = sideB ? g.N : g.M;
    const i64 r0 = (i64)panel*P;
    const bool rows_contig = (sideB ? g.bmode : g.amode) == 0;
    const double* __restrict__ X = sideB ? g.B : g.A;
    const int nseg = g.nseg > 0 ? g.nseg : 1;
    i64 step = 0;                                     // first step of the segment
    for (int sg = 0; sg < nseg; sg++)
    {
        const i64 *rvec, *kvec;
        i64 K;
        if (g.nseg > 0)
        {
            const SegDesc& sd = g.segs[sg];
            rvec = sideB ? sd.b_n : sd.a_m;
            kvec = sideB ? sd.b_k : sd.a_k;
            K = sd.K;
        }
        else
        {
            rvec = sideB ? g.b_n : g.a_m;
            kvec = sideB ? g.b_k : g.a_k;
            K = g.K;
        }
        const i64 nk = (K + BK - 1)/BK;
        const i64 lo = max(s0, step), hi = min(s0 + ns, step + nk);
        if (lo < hi)
        {
            // valid k of the pass starting at step kb (a multiple of PK_STEPS past lo)
            auto valid_k = [&](i64 kb) -> int
            {
                return kb < hi - step ? (int)min(min((i64)PK_STEPS, hi - step - kb)*BK, K - kb*BK) : 0;
            };
            // this thread's share of the gather of one pass (k offsets in kofs)
            constexpr int N = P*PK_K/PK_THREADS;
            auto gather = [&](const i64* kofs, int kc, double (&v)[N])
            {
                #pragma unroll
                for (int j = 0; j < N; j++)
                {
                    const int e = t + j*PK_THREADS;
                    const int r = rows_contig ? e % P : e / PK_K;
                    const int k = rows_contig ? e / P : e % PK_K;
                    const i64 ro = sRow[r];
                    v[j] = (k < kc && ro >= 0) ? __ldg(X + ro + kofs[k]) : 0.0;
                }
            };
            static_assert(PK_K <= PK_THREADS, "one k offset per thread");
            const i64 kb0 = lo - step;
            __syncthreads();                          // the previous pass is done with sRow and sK
            for (int r = t; r < P; r += PK_THREADS) sRow[r] = r0 + r < extent ? __ldg(rvec + r0 + r) : -1;
            if (t < PK_K) sK[t] = t < valid_k(kb0) ? __ldg(kvec + kb0*BK + t) : 0;
            // the k offsets of the second pass, stored when the first one is gathered
            i64 knext = t < valid_k(kb0 + PK_STEPS) ? __ldg(kvec + (kb0 + PK_STEPS)*BK + t) : 0;
            __syncthreads();
            double v[N];
            gather(sK, valid_k(kb0), v);
            // Each iteration stores the gathered pass into T, issues the gather
            // of the next pass, and writes this pass's blocks while those loads
            // are in flight. sK holds two passes' k offsets (pass parity).
            int par = 0;
            for (i64 kb = kb0; kb < hi - step; kb += PK_STEPS, par ^= 1)
            {
                const int steps = (int)min((i64)PK_STEPS, hi - step - kb);
                #pragma unroll
                for (int j = 0; j < N; j++)
                {
                    const int e = t + j*PK_THREADS;
                    const int r = rows_contig ? e % P : e / PK_K;
                    const int k = rows_contig ? e / P : e % PK_K;
                    T[k][r] = v[j];
                }
                i64* snext = sK + (par ^ 1)*PK_K;
                if (t < PK_K) snext[t] = knext;
                __syncthreads();                      // T of this pass and the next k offsets are visible
                const i64 kn = kb + PK_STEPS;
                if (t < valid_k(kn + PK_STEPS)) knext = __ldg(kvec + (kn + PK_STEPS)*BK + t);
                if (kn < hi - step) gather(snext, valid_k(kn), v);
                // this pass's blocks, rows of 16 k, k swizzled by row
                double* __restrict__ o = out + (step + kb)*P*BK;
                const int m = steps*P*BK;
                for (int e = t; e < m; e += PK_THREADS)
                {
                    const int c = e/(P*BK), w = e % (P*BK), r = w/BK, kq = w % BK;
                    o[e] = T[c*BK + (kq ^ ((r & 3) << 2))][r];
                }
                __syncthreads();                      // T is read before the next pass stores into it
            }
        }
        step += nk;
    }
}

__global__ void __launch_bounds__(PK_THREADS, 2)
gemm_f64_pack_kernel(const GroupDesc* __restrict__ groups, const PackItem* __restrict__ items, int nitems,
                     double* __restrict__ packA, double* __restrict__ packB)
{
    __shared__ double T[PK_K][WS_EDGE + 1];
    __shared__ i64 sRow[WS_EDGE];
    __shared__ i64 sK[2*PK_K];
    for (int item = blockIdx.x; item < nitems; item += gridDim.x)
    {
        const PackItem pi = items[item];
        const GroupDesc& g = groups[pi.g];
        const bool sideB = pi.side != 0;
        const bool p32 = sideB ? (g.shape & 1) != 0 : (g.shape & 2) != 0;
        const int P = p32 ? 32 : 64;
        double* out = (sideB ? packB + g.pb : packA + g.pa) + (i64)pi.panel*g.nst*P*BK;
        if (p32) pack_panel<32>(g, sideB, pi.panel, pi.s0, pi.ns, out, T, sRow, sK);
        else pack_panel<64>(g, sideB, pi.panel, pi.s0, pi.ns, out, T, sRow, sK);
    }
}

// ---- GEMM consumers ------------------------------------------------------------

// D(16x8) += A(16x16) * B(16x8), FP64. Fragments (g = lane/4, t = lane%4):
// a[q] = A(g + 8*(q%2), t + 4*(q/2)), b[q] = B(t + 4*q, g),
// c[q] = C(g + 8*(q/2), 2*t + q%2)
__device__ __forceinline__ void dmma_k16(double* c, const double* a, const double* b)
{
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, "
                 "{%4,%5,%6,%7,%8,%9,%10,%11}, {%12,%13,%14,%15}, {%0,%1,%2,%3};\n"
                 : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
                 : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]),
                   "d"(b[0]), "d"(b[1]), "d"(b[2]), "d"(b[3]));
}

// nst k steps of one BM x BN tile (warp tile BM/2 x BN/2) into acc; the stage
// holds the packed A block (BM rows of 16) and the packed B block (BN rows of 16)
template <int BM, int BN>
__device__ __forceinline__ bool ws_consume(double (&acc)[2][4][4], int nst, const double* stages, WsShared& sh,
                                           i64& it, volatile int* abort_flag, int warp, int lane)
{
    constexpr int WM = BM/2, WN = BN/2, MS = WM/16, NS = WN/8;
    const int wm0 = (warp >> 1)*WM, wn0 = (warp & 1)*WN;
    const int fr = lane >> 2, fc = lane & 3;
    const int sw = (fr & 3) << 2;               // every fragment row of this lane is fr mod 4
    for (int k = 0; k < nst; k++)
    {
        const int s = (int)(it % WS_STAGES);
        if (!mb_wait_warp(&sh.full[s], (uint32_t)((it/WS_STAGES) & 1), abort_flag)) return false;
        const double* As = stages + (size_t)s*WS_STAGE;
        const double* Bs = As + WS_OPER;
        // the whole 16-wide step in one m16n8k16 MMA per fragment pair
        double af[MS][8], bf[NS][4];
        #pragma unroll
        for (int i = 0; i < MS; i++)
            #pragma unroll
            for (int q = 0; q < 8; q++)
                af[i][q] = As[(wm0 + i*16 + fr + 8*(q & 1))*BK + (((4*(q >> 1)) ^ sw) + fc)];
        #pragma unroll
        for (int j = 0; j < NS; j++)
            #pragma unroll
            for (int q = 0; q < 4; q++)
                bf[j][q] = Bs[(wn0 + j*8 + fr)*BK + (((4*q) ^ sw) + fc)];
        #pragma unroll
        for (int i = 0; i < MS; i++)
            #pragma unroll
            for (int j = 0; j < NS; j++)
                dmma_k16(acc[i][j], af[i], bf[j]);
        // the fragments are in registers: the stage may be refilled. The
        // refill is a bulk copy (async proxy) over what these generic loads
        // read, so each thread orders its reads before it with a proxy
        // fence; without it, refills overtook reads still in flight when
        // other kernels' blocks shared the SM, and whole warp tiles came out
        // wrong
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncwarp();
        if (lane == 0) mb_arrive(&sh.empty[s]);
        it++;
    }
    return true;
}

template <int BM, int BN>
__device__ __forceinline__ void ws_epilogue(double (&acc)[2][4][4], const WsTileMeta& tm, int warp, int lane)
{
    constexpr int WM = BM/2, WN = BN/2, MS = WM/16, NS = WN/8;
    const int wm0 = (warp >> 1)*WM, wn0 = (warp & 1)*WN;
    const int fr = lane >> 2, fc = lane & 3;
    double* C = tm.C;
    const double alpha = tm.alpha, beta = tm.beta;
    #pragma unroll
    for (int i = 0; i < MS; i++)
        #pragma unroll
        for (int hh = 0; hh < 2; hh++)
        {
            const i64 rc = tm.crow[wm0 + i*16 + 8*hh + fr];
            if (rc < 0) continue;
            #pragma unroll
            for (int j = 0; j < NS; j++)
                #pragma unroll
                for (int h = 0; h < 2; h++)
                {
                    const i64 cc = tm.ccol[wn0 + j*8 + 2*fc + h];
                    if (cc < 0) continue;
                    double* dst = C + rc + cc;
                    const double v = alpha*acc[i][j][2*hh + h];
                    *dst = beta == 0.0 ? v : v + beta*(*dst);
                }
        }
}

template <int BM, int BN>
__device__ __forceinline__ bool ws_tile(int nst, const WsTileMeta& tm, const double* stages, WsShared& sh, i64& it,
                                        volatile int* abort_flag, int warp, int lane)
{
    double acc[2][4][4];
    #pragma unroll
    for (int i = 0; i < 2; i++)
        #pragma unroll
        for (int j = 0; j < 4; j++)
            #pragma unroll
            for (int q = 0; q < 4; q++) acc[i][j][q] = 0.0;
    if (!ws_consume<BM, BN>(acc, nst, stages, sh, it, abort_flag, warp, lane)) return false;
    ws_epilogue<BM, BN>(acc, tm, warp, lane);
    return true;
}

// largest g with tile_begin[g] <= tile (tile_begin[0] == 0): a 32-way search
// by the whole warp, three rounds of one load per lane for 10^4 groups
__device__ __forceinline__ int ws_find_group(const i64* __restrict__ tile_begin, int ngroups, long long tile,
                                             int lane)
{
    int lo = 0, hi = ngroups;
    while (hi - lo > 1)
    {
        const int step = (hi - lo + 31)/32;
        const int idx = lo + lane*step;
        const bool le = idx < hi && __ldg(tile_begin + idx) <= tile;
        const unsigned b = __ballot_sync(0xffffffffu, le);
        lo += (31 - __clz(b))*step;            // lane 0 (idx = lo) always holds
        hi = min(hi, lo + step);
    }
    return lo;
}

__global__ void __launch_bounds__(WS_THREADS, 2)
gemm_f64_ws_kernel(const GroupDesc* __restrict__ groups, const i64* __restrict__ tile_begin, int ngroups,
                   i64 total_tiles, const double* __restrict__ packA, const double* __restrict__ packB,
                   unsigned long long* __restrict__ counter)
{
    extern __shared__ __align__(128) double smem[];
    double* stages = smem;
    WsShared& sh = *reinterpret_cast<WsShared*>(smem + (size_t)WS_STAGES*WS_STAGE);
    volatile int* abort_flag = &sh.abort;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    if (tid == 0)
    {
        for (int s = 0; s < WS_STAGES; s++)
        {
            mb_init(&sh.full[s], 1);                   // the producer's arrival with the stage's bytes
            mb_init(&sh.empty[s], WS_CONSUMERS);       // one arrival per consumer warp
        }
        for (int t = 0; t < WS_TSLOTS; t++)
        {
            mb_init(&sh.tfull[t], 32);                 // the producer warp's lanes
            mb_init(&sh.tempty[t], WS_CONSUMERS);      // the consumer warps, once C is written
        }
        sh.abort = 0;
        // the initialised barriers, visible to the bulk copies' completions
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();
    // from here on the roles never wait on a CTA-wide barrier

    if (warp == WS_CONSUMERS)
    {
        // ---- producer warp: takes the tiles, publishes them, streams their blocks ------
        i64 it = 0, seq = 0;
        long long next = 0;
        if (lane == 0) next = counter ? (long long)atomicAdd(counter, 1ull) : (long long)blockIdx.x;
        for (;;)
        {
            long long tile = 0;
            if (lane == 0)
            {
                tile = next;
                // the tile after this one, requested while this one streams
                if (tile < total_tiles) next = counter ? (long long)atomicAdd(counter, 1ull) : tile + gridDim.x;
            }
            tile = __shfl_sync(0xffffffffu, tile, 0);
            const bool done = tile >= total_tiles;
            const int gi = done ? 0 : ws_find_group(tile_begin, ngroups, tile, lane);
            const GroupDesc& g = groups[gi];
            const int nst = done ? -1 : g.nst;
            if (nst == 0) continue;           // nothing to contract: the plan updates such C blocks itself
            const int ts = (int)(seq % WS_TSLOTS);
            if (seq >= WS_TSLOTS &&
                !mb_wait_warp(&sh.tempty[ts], (uint32_t)(((seq/WS_TSLOTS) & 1) ^ 1), abort_flag))
                break;
            WsTileMeta& tm = sh.meta[ts];
            if (done)
            {
                if (lane == 0) tm.nst = -1;
                mb_arrive(&sh.tfull[ts]);
                break;
            }
            const int shape = g.shape;
            const int BMs = (shape & 2) ? 32 : 64, BNs = (shape & 1) ? 32 : 64;
            const i64 tiles_n = (g.N + BNs - 1)/BNs;
            const i64 local = tile - __ldg(tile_begin + gi);
            const i64 tmi = local / tiles_n, tni = local % tiles_n;
            const i64 m0 = tmi*BMs, n0 = tni*BNs;
            for (int r = lane; r < WS_EDGE; r += 32)
            {
                tm.crow[r] = r < BMs && m0 + r < g.M ? __ldg(g.c_m + m0 + r) : -1;
                tm.ccol[r] = r < BNs && n0 + r < g.N ? __ldg(g.c_n + n0 + r) : -1;
            }
            if (lane == 0)
            {
                tm.C = g.C; tm.alpha = g.alpha; tm.beta = g.beta;
                tm.nst = nst; tm.shape = shape;
            }
            // release: the slot's contents are visible to the consumers that wait on it
            mb_arrive(&sh.tfull[ts]);
            seq++;
            const double* srcA = packA + g.pa + tmi*nst*BMs*BK;
            const double* srcB = packB + g.pb + tni*nst*BNs*BK;
            const uint32_t bytesA = (uint32_t)(BMs*BK*sizeof(double)), bytesB = (uint32_t)(BNs*BK*sizeof(double));
            const int skip = g_f64_skip_step;
            bool ok = true;
            for (int st = 0; st < nst; st++)
            {
                const int s = (int)(it % WS_STAGES);
                if (it >= WS_STAGES &&
                    !mb_wait_warp(&sh.empty[s], (uint32_t)(((it/WS_STAGES) & 1) ^ 1), abort_flag))
                {
                    ok = false;
                    break;
                }
                if (lane == 0 && it != skip)
                {
                    double* As = stages + (size_t)s*WS_STAGE;
                    mb_arrive_expect(&sh.full[s], bytesA + bytesB);
                    bulk_load(As, srcA + (i64)st*BMs*BK, bytesA, &sh.full[s]);
                    bulk_load(As + WS_OPER, srcB + (i64)st*BNs*BK, bytesB, &sh.full[s]);
                }
                it++;
            }
            if (!ok) break;
        }
        // the copies of the last stages issued land before the CTA is gone
        // (bounded waits; on the normal path these phases are complete)
        if (lane == 0)
        {
            const int skip = g_f64_skip_step;
            for (i64 k = it > WS_STAGES ? it - WS_STAGES : 0; k < it; k++)
                if (k != skip && !mb_try(&sh.full[k % WS_STAGES], (uint32_t)((k/WS_STAGES) & 1)))
                    mb_wait_slow(&sh.full[k % WS_STAGES], (uint32_t)((k/WS_STAGES) & 1), abort_flag, true);
        }
        __syncwarp();
    }
    else
    {
        // ---- consumer warps --------------------------------------------------------
        i64 it = 0;
        for (i64 seq = 0;; seq++)
        {
            const int ts = (int)(seq % WS_TSLOTS);
            if (!mb_wait_warp(&sh.tfull[ts], (uint32_t)((seq/WS_TSLOTS) & 1), abort_flag)) break;
            const WsTileMeta& tm = sh.meta[ts];
            const int nst = tm.nst;
            if (nst < 0) break;
            bool ok;
            switch (tm.shape)
            {
                case 0: ok = ws_tile<64, 64>(nst, tm, stages, sh, it, abort_flag, warp, lane); break;
                case 1: ok = ws_tile<64, 32>(nst, tm, stages, sh, it, abort_flag, warp, lane); break;
                case 2: ok = ws_tile<32, 64>(nst, tm, stages, sh, it, abort_flag, warp, lane); break;
                default: ok = ws_tile<32, 32>(nst, tm, stages, sh, it, abort_flag, warp, lane); break;
            }
            if (!ok) break;
            // C of this tile is written: the slot may take another tile
            __syncwarp();
            if (lane == 0) mb_arrive(&sh.tempty[ts]);
        }
    }
}

int sm_count()
{
    int dev = 0, sms = 148;
    TB_CUDA(cudaGetDevice(&dev));
    TB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    return sms;
}

} // namespace

int gemm_f64_ws_shape(i64 M, i64 N, i64 K)
{
    // padded MMA work of each shape, the smaller tiles weighted by what their
    // lower operand reuse costs per flop
    static const double weight[4] = {1.0, 1.08, 1.08, 1.2};
    int best = 0;
    double best_cost = 0;
    for (int s = 0; s < 4; s++)
    {
        const i64 bm = (s & 2) ? 32 : 64, bn = (s & 1) ? 32 : 64;
        const double cost = weight[s]*(double)((M + bm - 1)/bm*bm)*(double)((N + bn - 1)/bn*bn)*(double)K;
        if (s == 0 || cost < best_cost) { best = s; best_cost = cost; }
    }
    return best;
}

void gemm_f64_ws_tile(int shape, int& bm, int& bn)
{
    bm = (shape & 2) ? 32 : 64;
    bn = (shape & 1) ? 32 : 64;
}

void gemm_f64_ws_pack(const GroupDesc* d_groups, const PackItem* d_items, int nitems, double* packA,
                      double* packB, cudaStream_t s)
{
    if (nitems <= 0) return;
    const int grid = (int)std::min<i64>(nitems, (i64)sm_count()*8);
    TimedLaunch t("gemm_f64_pack_kernel", s);
    gemm_f64_pack_kernel<<<grid, PK_THREADS, 0, s>>>(d_groups, d_items, nitems, packA, packB);
    check_launch("gemm_f64_pack_kernel");
}

void gemm_f64_ws_launch(const GroupDesc* d_groups, const i64* d_tile_begin, int ngroups, i64 total_tiles,
                        const double* packA, const double* packB, cudaStream_t s, unsigned long long* d_counter)
{
    if (ngroups <= 0 || total_tiles <= 0) return;
    const size_t bytes = ws_smem_bytes();
    TB_CUDA(cudaFuncSetAttribute(gemm_f64_ws_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    const i64 grid = std::min<i64>(total_tiles, (i64)sm_count()*2);
    if (d_counter) TB_CUDA(cudaMemsetAsync(d_counter, 0, sizeof(unsigned long long), s));
    TimedLaunch t("gemm_f64_ws_kernel", s);
    gemm_f64_ws_kernel<<<(unsigned)grid, WS_THREADS, bytes, s>>>(d_groups, d_tile_begin, ngroups, total_tiles,
                                                                  packA, packB, d_counter);
    check_launch("gemm_f64_ws_kernel");
}

void gemm_f64_inject_wait_timeout(int step, double wait_seconds)
{
    const unsigned long long ns = wait_seconds > 0.0 ? (unsigned long long)(wait_seconds*1e9) : WS_WAIT_NS;
    TB_CUDA(cudaMemcpyToSymbol(g_f64_skip_step, &step, sizeof(int)));
    TB_CUDA(cudaMemcpyToSymbol(g_f64_wait_ns, &ns, sizeof(ns)));
}

int gemm_f64_error_flag()
{
    int v = 0;
    cudaMemcpyFromSymbol(&v, g_f64_error, sizeof(int));
    if (v)
    {
        // reported once: the next check starts clean
        const int zero = 0;
        cudaMemcpyToSymbol(g_f64_error, &zero, sizeof(int));
    }
    return v;
}

} // namespace tb
