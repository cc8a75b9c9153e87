// gemm_f64.cu -- FP64 tensor-core (DMMA) contraction kernels with
// block-scatter gathers.
//
// Replaces TBLIS's pack + microkernel + scatter-accumulate chain
// (src/nodes/packm.hpp:79-124, src/kernels/3m/packm.hpp:292-403,
// src/nodes/gemm_ukr.hpp:16-126 and :193-364): every operand tile is gathered
// straight from the strided tensor into shared memory with cp.async, driven by
// the scatter vectors of the GEMM view (element offset of each row / column /
// k index, with per-16-block common strides that turn the k gather into
// strided arithmetic whenever the block is regular). No packed copy of A or B
// is written to HBM. The alpha/beta update of C is scattered back through C's
// scatter vectors in the epilogue; beta == 0 never reads C.
//
// A family of tile shapes shares one kernel template: CTA tile BM x BN x 16,
// warps of WM x WN built from mma.sync.m16n8k8 f64 (sm_100a has no tcgen05
// FP64 kind; DMMA is the FP64 tensor-core path), a STAGES-deep cp.async
// pipeline. Each operand is gathered along the GEMM dimension with its
// smallest stride (m or k for A, n or k for B) and laid out in shared memory
// so that both the cp.async writes and the fragment reads are free of bank
// conflicts. The first k entry and block stride of the next tile are fetched
// one iteration ahead so the gather addresses never wait on L2.
//
// Split-K partial tiles go to a workspace and are summed in a fixed order by
// gemm_f64_reduce (no atomics: results do not depend on scheduling).
#include "gemm_f64.hpp"
#include "gemm_f64_dev.cuh"

#include <algorithm>
#include <cstdlib>
#include <type_traits>

namespace tb
{

namespace
{

using namespace f64dev;

// arguments of one output tile
struct TileArgs
{
    const double* A;          // already offset to the batch entry
    const double* B;
    double* C;
    const i64 *a_m, *a_k, *b_k, *b_n, *c_m, *c_n, *a_kbs, *b_kbs;
    i64 M, N;
    i64 m0, n0;
    i64 k_begin, k_end;
    double alpha, beta;
    double* W;                // split-K partial tile output (dense, ld = N), or null
    int nseg;                 // 0: the single segment above; else segs[0..nseg)
    const SegDesc* segs;
};

template <int BM, int BN>
__host__ __device__ constexpr int tile_smem_doubles(int STAGES)
{
    // the larger of the two gather layouts, so runtime-mode kernels fit both
    return STAGES*((BK*(BM + PAD) > BM*(BK + PAD) ? BK*(BM + PAD) : BM*(BK + PAD)) +
                   (BK*(BN + PAD) > BN*(BK + PAD) ? BK*(BN + PAD) : BN*(BK + PAD)));
}

// one BM x BN output tile: gathered cp.async mainloop + DMMA + scatter epilogue
// PA / PB: gather A / B in pairs of adjacent elements (16-byte copies where
// the pair is adjacent and aligned in global memory), for operands whose
// contiguous GEMM dimension mostly is; else one 8-byte copy per element
template <int BM, int BN, int WM, int WN, int STAGES, int AMODE, int BMODE, bool PA = false, bool PB = false>
__device__ __forceinline__ void tile_body(const TileArgs& p, double* smem, i64* sAm, i64* sBn, i64* sCm, i64* sCn)
{
    constexpr int NT = (BM/WM)*(BN/WN)*32;
    // m16n8k8: MS 16-row by NS 8-column fragments per warp, 4 values each
    constexpr int MS = WM/16, NS = WN/8;
    using TA = Tile<BM, AMODE>;
    using TB = Tile<BN, BMODE>;
    constexpr int STAGE = TA::SIZE + TB::SIZE;

    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const i64 m0 = p.m0, n0 = p.n0;
    const double* __restrict__ A = p.A;
    const double* __restrict__ B = p.B;

    for (int i = tid; i < BM; i += NT)
    {
        const i64 m = m0 + i;
        sCm[i] = m < p.M ? p.c_m[m] : -1;
    }
    for (int i = tid; i < BN; i += NT)
    {
        const i64 n = n0 + i;
        sCn[i] = n < p.N ? p.c_n[n] : -1;
    }

    double acc[MS][NS][4];
    #pragma unroll
    for (int i = 0; i < MS; i++)
        #pragma unroll
        for (int j = 0; j < NS; j++)
            #pragma unroll
            for (int q = 0; q < 4; q++) acc[i][j][q] = 0.0;

    const int wm0 = (warp / (BN/WN))*WM;
    const int wn0 = (warp % (BN/WN))*WN;
    const int fr = lane >> 2, fc = lane & 3;

    const int nseg = p.nseg > 0 ? p.nseg : 1;
    for (int sg = 0; sg < nseg; sg++)
    {
        const i64 *a_m = p.a_m, *a_k = p.a_k, *b_k = p.b_k, *b_n = p.b_n, *a_kbs = p.a_kbs, *b_kbs = p.b_kbs;
        i64 k_begin = p.k_begin, k_end = p.k_end;
        if (p.nseg > 0)
        {
            const SegDesc& sd = p.segs[sg];
            a_m = sd.a_m; a_k = sd.a_k; b_k = sd.b_k; b_n = sd.b_n; a_kbs = sd.a_kbs; b_kbs = sd.b_kbs;
            k_begin = 0; k_end = sd.K;
        }
        for (int i = tid; i < BM; i += NT)
        {
            const i64 m = m0 + i;
            sAm[i] = m < p.M ? a_m[m] : -1;
        }
        for (int i = tid; i < BN; i += NT)
        {
            const i64 n = n0 + i;
            sBn[i] = n < p.N ? b_n[n] : -1;
        }
        __syncthreads();

        const i64 kt_count = (k_end - k_begin + BK - 1)/BK;

        // Per-thread gather geometry, fixed for the whole tile. In the
        // rows-contiguous layout (mode 0) a thread copies the same row (or
        // pair of rows) at k = k0 + j*KSTEP; in the k-contiguous layout (mode
        // 1) the same k (or pair of k, even and odd) of rows r0 + j*RSTEP.
        // Row offsets are read from shared memory once per tile, k offsets
        // once per stage (stride arithmetic when the 16-block of k is regular).
        auto gather = [&](auto pairs, auto mode, auto rows, const i64* sX, const double* X, double* Xs,
                          const i64* scat, const KInfo& ki, i64 k0, int kvalid, const i64* ro)
        {
            constexpr bool PR = decltype(pairs)::value;
            constexpr int MD = decltype(mode)::value, R = decltype(rows)::value;
            constexpr int W = PR ? 2 : 1;                 // elements per copy slot
            constexpr int J = BK*R/(W*NT);
            using TX = Tile<R, MD>;
            if (MD == 0)
            {
                const int r = W*(tid % (R/W)), kl0 = tid/(R/W);
                constexpr int KS = NT/(R/W);
                #pragma unroll
                for (int j = 0; j < J; j++)
                {
                    const int kl = kl0 + j*KS;
                    const bool kok = kl < kvalid;
                    const i64 ko = kok ? koff(scat, ki, k0, kl) : 0;
                    if (PR)
                        cp_pair(Xs + TX::idx(r, kl), X, ro[0] + ko, kok && ro[0] >= 0, ro[1] + ko, kok && ro[1] >= 0,
                                X);
                    else
                    {
                        const bool ok = kok && ro[0] >= 0;
                        cp_async8(Xs + TX::idx(r, kl), ok ? X + ro[0] + ko : X, ok);
                    }
                }
            }
            else
            {
                const int kl = W*(tid % (BK/W)), r0 = tid/(BK/W);
                constexpr int RS = NT/(BK/W);
                const bool k0ok = kl < kvalid, k1ok = PR && kl + 1 < kvalid;
                const i64 ko0 = k0ok ? koff(scat, ki, k0, kl) : 0;
                const i64 ko1 = k1ok ? koff(scat, ki, k0, kl + 1) : 0;
                #pragma unroll
                for (int j = 0; j < J; j++)
                {
                    const i64 o = ro[j];
                    if (PR)
                        cp_pair(Xs + TX::idx(r0 + j*RS, kl), X, o + ko0, k0ok && o >= 0, o + ko1, k1ok && o >= 0, X);
                    else
                    {
                        const bool ok = k0ok && o >= 0;
                        cp_async8(Xs + TX::idx(r0 + j*RS, kl), ok ? X + o + ko0 : X, ok);
                    }
                }
            }
        };
        // the row offsets a thread copies, per the scheme above
        auto rows_of = [&](auto pairs, auto mode, auto rows, const i64* sX, i64* ro)
        {
            constexpr bool PR = decltype(pairs)::value;
            constexpr int MD = decltype(mode)::value, R = decltype(rows)::value;
            constexpr int W = PR ? 2 : 1;
            constexpr int J = BK*R/(W*NT);
            if (MD == 0)
            {
                const int r = W*(tid % (R/W));
                ro[0] = sX[r];
                if (PR) ro[1] = sX[r + 1];
            }
            else
            {
                #pragma unroll
                for (int j = 0; j < J; j++) ro[j] = sX[tid/(BK/W) + j*(NT/(BK/W))];
            }
        };
        using PAc = std::integral_constant<bool, PA>;
        using PBc = std::integral_constant<bool, PB>;
        using AMc = std::integral_constant<int, AMODE>;
        using BMc = std::integral_constant<int, BMODE>;
        using BMr = std::integral_constant<int, BM>;
        using BNr = std::integral_constant<int, BN>;
        static_assert(NT % (BM/2) == 0 && NT % (BN/2) == 0 && NT % BM == 0 && NT % BN == 0 && NT % BK == 0 &&
                      BK*BM % (2*NT) == 0 && BK*BN % (2*NT) == 0, "gather geometry");
        constexpr int ANR = AMODE == 0 ? 2 : BK*BM/((PA ? 2 : 1)*NT);
        constexpr int BNR = BMODE == 0 ? 2 : BK*BN/((PB ? 2 : 1)*NT);
        i64 a_ro[ANR], b_ro[BNR];
        rows_of(PAc(), AMc(), BMr(), sAm, a_ro);
        rows_of(PBc(), BMc(), BNr(), sBn, b_ro);

        auto load_tile = [&](int stage, i64 kt, const KInfo& ka, const KInfo& kb)
        {
            double* As = smem + stage*STAGE;
            double* Bs = As + TA::SIZE;
            const i64 k0 = k_begin + kt*BK;
            const int kvalid = (int)min((i64)BK, k_end - k0);
            gather(PAc(), AMc(), BMr(), sAm, A, As, a_k, ka, k0, kvalid, a_ro);
            gather(PBc(), BMc(), BNr(), sBn, B, Bs, b_k, kb, k0, kvalid, b_ro);
        };

        #pragma unroll
        for (int s = 0; s < STAGES-1; s++)
        {
            if (s < kt_count)
            {
                const i64 k0 = k_begin + s*BK;
                load_tile(s, s, fetch_kinfo(a_k, a_kbs, k0, true), fetch_kinfo(b_k, b_kbs, k0, true));
            }
            cp_async_commit();
        }
        // k information of the next tile to load, one iteration ahead
        i64 nk = STAGES - 1;
        KInfo ka = fetch_kinfo(a_k, a_kbs, k_begin + nk*BK, nk < kt_count);
        KInfo kb = fetch_kinfo(b_k, b_kbs, k_begin + nk*BK, nk < kt_count);

        for (i64 kt = 0; kt < kt_count; kt++)
        {
            cp_async_wait<STAGES-2>();
            __syncthreads();

            if (nk < kt_count) load_tile((int)(nk % STAGES), nk, ka, kb);
            cp_async_commit();
            nk++;
            ka = fetch_kinfo(a_k, a_kbs, k_begin + nk*BK, nk < kt_count);
            kb = fetch_kinfo(b_k, b_kbs, k_begin + nk*BK, nk < kt_count);

            const double* As = smem + (kt % STAGES)*STAGE;
            const double* Bs = As + TA::SIZE;
            #pragma unroll
            for (int kk = 0; kk < BK; kk += 8)
            {
                double af[MS][4], bf[NS][2];
                #pragma unroll
                for (int i = 0; i < MS; i++)
                    #pragma unroll
                    for (int q = 0; q < 4; q++)
                        af[i][q] = As[TA::idx(wm0 + i*16 + fr + 8*(q & 1), kk + fc + 4*(q >> 1))];
                #pragma unroll
                for (int j = 0; j < NS; j++)
                    #pragma unroll
                    for (int q = 0; q < 2; q++)
                        bf[j][q] = Bs[TB::idx(wn0 + j*8 + fr, kk + fc + 4*q)];
                #pragma unroll
                for (int i = 0; i < MS; i++)
                    #pragma unroll
                    for (int j = 0; j < NS; j++)
                        dmma16(acc[i][j], af[i], bf[j]);
            }
        }
        cp_async_wait<0>();
        // the next segment reuses the stages and the offset arrays
        __syncthreads();
    }

    // each accumulator fragment holds rows fr and fr + 8 of a 16-row block
    if (p.W)
    {
        // raw partial sums, dense [m][n]
        #pragma unroll
        for (int i = 0; i < MS; i++)
            #pragma unroll
            for (int hh = 0; hh < 2; hh++)
            {
                const i64 m = m0 + wm0 + i*16 + 8*hh + fr;
                if (m >= p.M) continue;
                #pragma unroll
                for (int j = 0; j < NS; j++)
                    #pragma unroll
                    for (int h = 0; h < 2; h++)
                    {
                        const i64 n = n0 + wn0 + j*8 + fc*2 + h;
                        if (n < p.N) p.W[m*p.N + n] = acc[i][j][2*hh + h];
                    }
            }
    }
    else
    {
        double* C = p.C;
        const double alpha = p.alpha, beta = p.beta;
        #pragma unroll
        for (int i = 0; i < MS; i++)
            #pragma unroll
            for (int hh = 0; hh < 2; hh++)
            {
                const i64 rc = sCm[wm0 + i*16 + 8*hh + fr];
                if (rc < 0) continue;
                #pragma unroll
                for (int j = 0; j < NS; j++)
                    #pragma unroll
                    for (int h = 0; h < 2; h++)
                    {
                        const i64 cc = sCn[wn0 + j*8 + fc*2 + h];
                        if (cc < 0) continue;
                        double* dst = C + rc + cc;
                        const double v = alpha*acc[i][j][2*hh + h];
                        *dst = beta == 0.0 ? v : v + beta*(*dst);
                    }
            }
    }
    // shared memory is reused by the next tile of a persistent CTA
    __syncthreads();
}

template <int BM, int BN, int WM, int WN, int STAGES, int AMODE, int BMODE, bool PA, bool PB, int MINB>
__global__ void __launch_bounds__((BM/WM)*(BN/WN)*32, MINB)
gemm_f64_kernel(const GemmF64Args p)
{
    extern __shared__ __align__(16) double smem[];
    constexpr int SD = Tile<BM, AMODE>::SIZE + Tile<BN, BMODE>::SIZE;
    i64* sAm = reinterpret_cast<i64*>(smem + STAGES*SD);
    i64* sBn = sAm + BM;
    i64* sCm = sBn + BN;
    i64* sCn = sCm + BM;

    // rasterisation: groups of 8 m-tiles sweep the n-tiles together so
    // concurrently running CTAs share A and B panels in L2
    const i64 tiles_m = (p.M + BM - 1)/BM, tiles_n = (p.N + BN - 1)/BN;
    const i64 tile = blockIdx.x;
    const i64 group = 8;
    const i64 gid = tile/(group*tiles_n);
    const i64 first_m = gid*group;
    const i64 gsize = min(group, tiles_m - first_m);
    const i64 tm = first_m + (tile % (group*tiles_n)) % gsize;
    const i64 tn = (tile % (group*tiles_n)) / gsize;

    const i64 l = blockIdx.y;
    const int split = blockIdx.z;
    TileArgs t;
    t.A = p.A + p.a_l[l];
    t.B = p.B + p.b_l[l];
    t.C = p.C + p.c_l[l];
    t.a_m = p.a_m; t.a_k = p.a_k; t.b_k = p.b_k; t.b_n = p.b_n; t.c_m = p.c_m; t.c_n = p.c_n;
    t.a_kbs = p.a_kbs; t.b_kbs = p.b_kbs;
    t.M = p.M; t.N = p.N;
    t.m0 = tm*BM; t.n0 = tn*BN;
    t.k_begin = (i64)split*p.k_per_split;
    t.k_end = min(p.K, t.k_begin + p.k_per_split);
    t.alpha = p.alpha; t.beta = p.beta;
    t.W = p.splits > 1 ? p.partial + ((i64)split*p.L + l)*p.M*p.N : nullptr;
    t.nseg = 0;
    t.segs = nullptr;
    tile_body<BM, BN, WM, WN, STAGES, AMODE, BMODE, PA, PB>(t, smem, sAm, sBn, sCm, sCn);
}

// Persistent grouped kernel: every CTA walks the global tile list (all
// groups' tiles, in group order) with a stride of the grid size; the group of
// a tile is found by binary search in the tile prefix table. Gather modes are
// per group (runtime), so the shared-memory stage is sized for either layout.
template <int BM, int BN, int WM, int WN, int STAGES, int MINB>
__global__ void __launch_bounds__((BM/WM)*(BN/WN)*32, MINB)
gemm_f64_grouped_kernel(const GroupDesc* __restrict__ groups, const i64* __restrict__ tile_begin,
                        int ngroups, i64 total_tiles, unsigned long long* __restrict__ counter)
{
    extern __shared__ __align__(16) double smem[];
    i64* sAm = reinterpret_cast<i64*>(smem + tile_smem_doubles<BM, BN>(STAGES));
    i64* sBn = sAm + BM;
    i64* sCm = sBn + BN;
    i64* sCn = sCm + BM;
    __shared__ i64 s_next;
    // tiles come from a global counter (groups are ordered longest K first,
    // so the longest tiles start first and the short ones fill in behind);
    // without a counter, static striding by the grid size
    auto next_tile = [&](i64 cur) -> i64
    {
        if (!counter) return cur < 0 ? (i64)blockIdx.x : cur + gridDim.x;
        __syncthreads();
        if (threadIdx.x == 0) s_next = (i64)atomicAdd(counter, 1ull);
        __syncthreads();
        return s_next;
    };
    for (i64 tile = next_tile(-1); tile < total_tiles; tile = next_tile(tile))
    {
        int lo = 0, hi = ngroups - 1;
        while (lo < hi)
        {
            const int mid = (lo + hi + 1) >> 1;
            if (__ldg(tile_begin + mid) <= tile) lo = mid; else hi = mid - 1;
        }
        const GroupDesc& g = groups[lo];
        const i64 local = tile - tile_begin[lo];
        const i64 tiles_n = (g.N + BN - 1)/BN;
        TileArgs t;
        t.A = g.A; t.B = g.B; t.C = g.C;
        t.a_m = g.a_m; t.a_k = g.a_k; t.b_k = g.b_k; t.b_n = g.b_n; t.c_m = g.c_m; t.c_n = g.c_n;
        t.a_kbs = g.a_kbs; t.b_kbs = g.b_kbs;
        t.M = g.M; t.N = g.N;
        t.m0 = (local / tiles_n)*BM; t.n0 = (local % tiles_n)*BN;
        t.k_begin = 0; t.k_end = g.K;
        t.alpha = g.alpha; t.beta = g.beta;
        t.W = nullptr;
        t.nseg = g.nseg;
        t.segs = g.segs;
        if (g.K == 0 && g.nseg == 0)
        {
            // empty contraction for this group: C = beta*C (beta == 0: set)
            continue;
        }
        switch (g.amode*2 + g.bmode)
        {
            case 0: tile_body<BM, BN, WM, WN, STAGES, 0, 0>(t, smem, sAm, sBn, sCm, sCn); break;
            case 1: tile_body<BM, BN, WM, WN, STAGES, 0, 1>(t, smem, sAm, sBn, sCm, sCn); break;
            case 2: tile_body<BM, BN, WM, WN, STAGES, 1, 0>(t, smem, sAm, sBn, sCm, sCn); break;
            default: tile_body<BM, BN, WM, WN, STAGES, 1, 1>(t, smem, sAm, sBn, sCm, sCn); break;
        }
    }
}

// sums the split-K partials in split order and applies alpha/beta
__global__ void gemm_f64_reduce(const GemmF64Args p)
{
    const i64 total = p.L*p.M*p.N;
    for (i64 e = blockIdx.x*(i64)blockDim.x + threadIdx.x; e < total; e += (i64)gridDim.x*blockDim.x)
    {
        const i64 l = e/(p.M*p.N);
        const i64 mn = e - l*p.M*p.N;
        const i64 m = mn/p.N, n = mn - m*p.N;
        double s = 0.0;
        for (int sp = 0; sp < p.splits; sp++)
            s += p.partial[((i64)sp*p.L + l)*p.M*p.N + mn];
        double* dst = p.C + p.c_l[l] + p.c_m[m] + p.c_n[n];
        const double v = p.alpha*s;
        *dst = p.beta == 0.0 ? v : v + p.beta*(*dst);
    }
}

// one tile configuration
struct Variant
{
    int bm, bn;
    void (*launch)(const GemmF64Args&, dim3, cudaStream_t, int amode, int bmode);
    void (*grouped)(const GroupDesc*, const i64*, int, i64, unsigned long long*, cudaStream_t);
};

// PAIRS: the dense launch may gather in pairs (the default tile shape only,
// to bound the number of kernel instances)
template <int BM_, int BN_, int WM, int WN, int STAGES, int MINB, bool PAIRS = false>
struct Config
{
    static constexpr int NT = (BM_/WM)*(BN_/WN)*32;
    static size_t smem_bytes(int am, int bmd)
    {
        size_t a = am == 0 ? BK*(BM_ + PAD) : BM_*(BK + PAD);
        size_t b = bmd == 0 ? BK*(BN_ + PAD) : BN_*(BK + PAD);
        return (size_t)STAGES*(a + b)*sizeof(double) + (2*BM_ + 2*BN_)*sizeof(i64);
    }
    template <int AM, int BMd, bool PA, bool PB>
    static void go(const GemmF64Args& a, dim3 grid, cudaStream_t s)
    {
        auto kern = gemm_f64_kernel<BM_, BN_, WM, WN, STAGES, AM, BMd, PA, PB, MINB>;
        const size_t bytes = smem_bytes(AM, BMd);
        TB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
        TimedLaunch t("gemm_f64_kernel", s);
        kern<<<grid, NT, bytes, s>>>(a);
        check_launch("gemm_f64_kernel");
    }
    static void grouped(const GroupDesc* g, const i64* tb, int ngroups, i64 total, unsigned long long* ctr,
                        cudaStream_t s)
    {
        auto kern = gemm_f64_grouped_kernel<BM_, BN_, WM, WN, STAGES, MINB>;
        const size_t bytes = (size_t)tile_smem_doubles<BM_, BN_>(STAGES)*sizeof(double) +
                             (2*BM_ + 2*BN_)*sizeof(i64);
        TB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
        int dev = 0, sms = 148;
        TB_CUDA(cudaGetDevice(&dev));
        TB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        const i64 grid = std::min<i64>(total, (i64)sms*MINB);
        if (grid <= 0) return;
        TimedLaunch t("gemm_f64_grouped_kernel", s);
        kern<<<(unsigned)grid, NT, bytes, s>>>(g, tb, ngroups, total, ctr);
        check_launch("gemm_f64_grouped_kernel");
    }
    template <bool PA, bool PB>
    static void go_modes(const GemmF64Args& a, dim3 grid, cudaStream_t s, int am, int bmd)
    {
        switch (am*2 + bmd)
        {
            case 0: go<0, 0, PA, PB>(a, grid, s); break;
            case 1: go<0, 1, PA, PB>(a, grid, s); break;
            case 2: go<1, 0, PA, PB>(a, grid, s); break;
            default: go<1, 1, PA, PB>(a, grid, s); break;
        }
    }
    static void launch(const GemmF64Args& a, dim3 grid, cudaStream_t s, int am, int bmd)
    {
        const int pr = PAIRS ? (a.pair_a ? 2 : 0) + (a.pair_b ? 1 : 0) : 0;
        if constexpr (PAIRS)
        {
            if (pr == 3) { go_modes<true, true>(a, grid, s, am, bmd); return; }
            if (pr == 2) { go_modes<true, false>(a, grid, s, am, bmd); return; }
            if (pr == 1) { go_modes<false, true>(a, grid, s, am, bmd); return; }
        }
        go_modes<false, false>(a, grid, s, am, bmd);
    }
};

// the tile family (index = variant id - 1)
const Variant kVariants[] = {
    {128, 128, Config<128, 128, 64, 32, 4, 1>::launch, Config<128, 128, 64, 32, 4, 1>::grouped},  // 1
    {64, 128, Config<64, 128, 32, 64, 3, 2>::launch, Config<64, 128, 32, 64, 3, 2>::grouped},     // 2
    {128, 64, Config<128, 64, 64, 32, 3, 2>::launch, Config<128, 64, 64, 32, 3, 2>::grouped},     // 3
    {64, 64, Config<64, 64, 32, 32, 3, 3, true>::launch, Config<64, 64, 32, 32, 3, 3, true>::grouped},  // 4
};
constexpr int kNumVariants = sizeof(kVariants)/sizeof(kVariants[0]);

int env_variant()
{
    static int v = -1;
    if (v < 0)
    {
        const char* s = getenv("TBLIS_B200_GEMM_VARIANT");
        v = s ? atoi(s) : 0;
        if (v < 0 || v > kNumVariants) v = 0;
    }
    return v;
}

int pick_variant(const GemmF64Args& a)
{
    if (a.variant > 0 && a.variant <= kNumVariants) return a.variant;
    if (env_variant()) return env_variant();
    // 64 x 64 tiles, three CTAs per SM: fastest of the family on B200 for
    // both the large (ladder, ring, 8192^3) and the small (24^4) workloads
    return 4;
}

} // namespace

int gemm_f64_num_variants() { return kNumVariants; }
void gemm_f64_variant_tile(int variant, int& bm, int& bn)
{
    const Variant& v = kVariants[std::max(1, std::min(variant, kNumVariants)) - 1];
    bm = v.bm; bn = v.bn;
}

int gemm_f64_grouped_num_variants() { return kNumVariants + 1; }
bool gemm_f64_is_ws_variant(int variant) { return variant == kNumVariants + 1; }

void gemm_f64_grouped_launch(const GroupDesc* d_groups, const i64* d_tile_begin, int ngroups,
                             i64 total_tiles, int variant, cudaStream_t stream, unsigned long long* d_counter)
{
    if (ngroups <= 0 || total_tiles <= 0) return;
    TB_CHECK(!gemm_f64_is_ws_variant(variant), TB_ERR_ARG, "the packed variant runs through its grouped plan");
    const Variant& v = kVariants[std::max(1, std::min(variant, kNumVariants)) - 1];
    if (d_counter) TB_CUDA(cudaMemsetAsync(d_counter, 0, sizeof(unsigned long long), stream));
    v.grouped(d_groups, d_tile_begin, ngroups, total_tiles, d_counter, stream);
}

i64 gemm_f64_tile_m() { return 128; }
i64 gemm_f64_tile_n() { return 128; }
i64 gemm_f64_tile_k() { return BK; }

int gemm_f64_choose_splits(i64 M, i64 N, i64 K, i64 L, int num_sms)
{
    // tiles of the default variant (64 x 64), three resident per SM
    const i64 tiles = ((M + 63)/64)*((N + 63)/64)*L;
    const i64 kt = (K + BK - 1)/BK;
    const i64 slots = 3*(i64)num_sms;
    if (tiles >= slots || kt < 8) return 1;
    i64 s = (slots + tiles - 1)/tiles;
    s = std::min<i64>(s, kt/4);
    s = std::min<i64>(s, 32);
    return (int)std::max<i64>(1, s);
}

size_t gemm_f64_workspace_bytes(i64 M, i64 N, i64 L, int splits)
{
    return splits > 1 ? (size_t)splits*L*M*N*sizeof(double) : 0;
}

void gemm_f64_launch(GemmF64Args a, cudaStream_t stream)
{
    if (a.M == 0 || a.N == 0 || a.L == 0) return;
    const Variant& v = kVariants[pick_variant(a) - 1];
    const i64 tiles_m = (a.M + v.bm - 1)/v.bm, tiles_n = (a.N + v.bn - 1)/v.bn;
    TB_CHECK(a.L <= 65535 && a.splits <= 65535, TB_ERR_SIZE, "batch extent too large");
    TB_CHECK(tiles_m*tiles_n < (1ll << 31), TB_ERR_SIZE, "tile grid too large");
    if (a.splits < 1) a.splits = 1;
    // split boundaries on BK multiples
    const i64 kt = (a.K + BK - 1)/BK;
    const i64 kt_per = (kt + a.splits - 1)/a.splits;
    a.k_per_split = std::max<i64>(1, kt_per)*BK;
    a.splits = (int)std::max<i64>(1, (a.K + a.k_per_split - 1)/a.k_per_split);
    TB_CHECK(a.splits == 1 || a.partial, TB_ERR_ARG, "split-K needs a workspace");
    if (a.K == 0) return;
    dim3 grid((unsigned)(tiles_m*tiles_n), (unsigned)a.L, (unsigned)a.splits);
    v.launch(a, grid, stream, a.amode, a.bmode);

    if (a.splits > 1)
    {
        const i64 total = a.L*a.M*a.N;
        const int threads = 256;
        const i64 blocks = std::min<i64>((total + threads - 1)/threads, 148*16);
        gemm_f64_reduce<<<(unsigned)blocks, threads, 0, stream>>>(a);
        check_launch("gemm_f64_reduce");
    }
}

} // namespace tb
