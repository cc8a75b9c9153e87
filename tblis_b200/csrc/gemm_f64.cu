// gemm_f64.cu -- FP64 tensor-core (DMMA) contraction kernel with
// block-scatter gathers.
//
// Replaces TBLIS's pack + microkernel + scatter-accumulate chain
// (src/nodes/packm.hpp:79-124, src/kernels/3m/packm.hpp:292-403,
// src/nodes/gemm_ukr.hpp:16-126 and :193-364): every operand tile is gathered
// straight from the strided tensor into shared memory with cp.async, driven by
// the scatter vectors of the GEMM view (element offset of each row / column /
// k index, with per-BK-block common strides that turn the k gather into
// strided arithmetic whenever the block is regular). No packed copy of A or B
// is written to HBM. The alpha/beta update of C is scattered back through C's
// scatter vectors in the epilogue; beta == 0 never reads C.
//
// Tile: 128x128x16 per CTA, 8 warps as 2 (m) x 4 (n), each warp 64x32 built
// from mma.sync.m8n8k4 f64 (sm_100a has no tcgen05 FP64 kind; DMMA is the
// FP64 tensor-core path). 4-stage cp.async pipeline. Split-K partial tiles go
// to a workspace and are summed in a fixed order by gemm_f64_reduce (no
// atomics: results do not depend on scheduling).
#include "gemm_f64.hpp"

#include <algorithm>

namespace tb
{

namespace
{

constexpr int BM = 128, BN = 128, BK = 16;
constexpr int WM = 64, WN = 32;
constexpr int MS = WM/8, NS = WN/8;
constexpr int NTHREADS = 256;
constexpr int STAGES = 4;
constexpr int PADA = 4, PADB = 4;              // bank-conflict-free fragment loads
constexpr int LDA = BM + PADA, LDB = BN + PADB;
constexpr int STAGE_DOUBLES = BK*LDA + BK*LDB;
constexpr size_t SMEM_BYTES = (size_t)STAGES*STAGE_DOUBLES*sizeof(double) + (BM + BN)*sizeof(i64)*2;

__device__ __forceinline__ void cp_async8(double* smem, const double* gmem, bool valid)
{
    unsigned saddr = (unsigned)__cvta_generic_to_shared(smem);
    int src_size = valid ? 8 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n"
                 :: "r"(saddr), "l"(gmem), "r"(src_size));
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }

template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" :: "n"(N)); }

__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(c0), "+d"(c1) : "d"(a), "d"(b));
}

// offset of k index k within operand X: regular BK-blocks use strided
// arithmetic from the block's first entry, irregular ones read the vector
__device__ __forceinline__ i64 k_offset(const i64* __restrict__ scat, i64 k0, i64 bstride, int kl)
{
    return bstride != 0 ? __ldg(scat + k0) + (i64)kl*bstride : __ldg(scat + k0 + kl);
}

template <int AMODE, int BMODE>
__global__ void __launch_bounds__(NTHREADS, 1)
gemm_f64_kernel(const GemmF64Args p)
{
    extern __shared__ __align__(16) double smem[];
    double* sbase = smem;
    i64* sAm = reinterpret_cast<i64*>(smem + STAGES*STAGE_DOUBLES);
    i64* sBn = sAm + BM;
    i64* sCm = sBn + BN;
    i64* sCn = sCm + BM;

    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;

    // tile rasterisation: groups of 8 m-tiles sweep the n-tiles together so
    // concurrently running CTAs share A and B panels in L2
    const i64 tiles_m = (p.M + BM - 1)/BM, tiles_n = (p.N + BN - 1)/BN;
    i64 tile = blockIdx.x;
    const i64 group = 8;
    i64 gid = tile/(group*tiles_n);
    i64 first_m = gid*group;
    i64 gsize = min(group, tiles_m - first_m);
    i64 tm = first_m + (tile % (group*tiles_n)) % gsize;
    i64 tn = (tile % (group*tiles_n)) / gsize;
    const i64 m0 = tm*BM, n0 = tn*BN;

    const i64 l = blockIdx.y;
    const int split = blockIdx.z;
    const i64 k_begin = (i64)split*p.k_per_split;
    const i64 k_end = min(p.K, k_begin + p.k_per_split);

    const double* __restrict__ A = p.A + p.a_l[l];
    const double* __restrict__ B = p.B + p.b_l[l];

    for (int i = tid; i < BM; i += NTHREADS)
    {
        i64 m = m0 + i;
        sAm[i] = m < p.M ? p.a_m[m] : -1;
        sCm[i] = m < p.M ? p.c_m[m] : -1;
    }
    for (int i = tid; i < BN; i += NTHREADS)
    {
        i64 n = n0 + i;
        sBn[i] = n < p.N ? p.b_n[n] : -1;
        sCn[i] = n < p.N ? p.c_n[n] : -1;
    }
    __syncthreads();

    const i64 kt_count = (k_end - k_begin + BK - 1)/BK;

    auto load_tile = [&](int stage, i64 kt)
    {
        double* As = sbase + stage*STAGE_DOUBLES;
        double* Bs = As + BK*LDA;
        const i64 k0 = k_begin + kt*BK;
        const i64 kblk = k0/BK;
        const i64 abs_ = __ldg(p.a_kbs + kblk);
        const i64 bbs_ = __ldg(p.b_kbs + kblk);
        const int kvalid = (int)min((i64)BK, k_end - k0);

        if (AMODE == 0)
        {
            const int ml = tid % BM;
            const i64 ro = sAm[ml];
            #pragma unroll
            for (int j = 0; j < BK*BM/NTHREADS; j++)
            {
                const int kl = tid/BM + j*(NTHREADS/BM);
                const bool ok = ro >= 0 && kl < kvalid;
                const i64 ko = ok ? k_offset(p.a_k, k0, abs_, kl) : 0;
                cp_async8(As + kl*LDA + ml, ok ? A + ro + ko : p.A, ok);
            }
        }
        else
        {
            const int kl = tid % BK;
            const bool kok = kl < kvalid;
            const i64 ko = kok ? k_offset(p.a_k, k0, abs_, kl) : 0;
            #pragma unroll
            for (int j = 0; j < BK*BM/NTHREADS; j++)
            {
                const int ml = tid/BK + j*(NTHREADS/BK);
                const i64 ro = sAm[ml];
                const bool ok = kok && ro >= 0;
                cp_async8(As + kl*LDA + ml, ok ? A + ro + ko : p.A, ok);
            }
        }

        if (BMODE == 0)
        {
            const int nl = tid % BN;
            const i64 co = sBn[nl];
            #pragma unroll
            for (int j = 0; j < BK*BN/NTHREADS; j++)
            {
                const int kl = tid/BN + j*(NTHREADS/BN);
                const bool ok = co >= 0 && kl < kvalid;
                const i64 ko = ok ? k_offset(p.b_k, k0, bbs_, kl) : 0;
                cp_async8(Bs + kl*LDB + nl, ok ? B + co + ko : p.B, ok);
            }
        }
        else
        {
            const int kl = tid % BK;
            const bool kok = kl < kvalid;
            const i64 ko = kok ? k_offset(p.b_k, k0, bbs_, kl) : 0;
            #pragma unroll
            for (int j = 0; j < BK*BN/NTHREADS; j++)
            {
                const int nl = tid/BK + j*(NTHREADS/BK);
                const i64 co = sBn[nl];
                const bool ok = kok && co >= 0;
                cp_async8(Bs + kl*LDB + nl, ok ? B + co + ko : p.B, ok);
            }
        }
    };

    double acc[MS][NS][2];
    #pragma unroll
    for (int i = 0; i < MS; i++)
        #pragma unroll
        for (int j = 0; j < NS; j++) { acc[i][j][0] = 0.0; acc[i][j][1] = 0.0; }

    #pragma unroll
    for (int s = 0; s < STAGES-1; s++)
    {
        if (s < kt_count) load_tile(s, s);
        cp_async_commit();
    }

    const int wm0 = (warp / (BN/WN))*WM;   // 2 warps along m
    const int wn0 = (warp % (BN/WN))*WN;   // 4 warps along n
    const int fr = lane >> 2, fc = lane & 3;

    for (i64 kt = 0; kt < kt_count; kt++)
    {
        cp_async_wait<STAGES-2>();
        __syncthreads();

        const i64 nk = kt + STAGES - 1;
        if (nk < kt_count) load_tile((int)(nk % STAGES), nk);
        cp_async_commit();

        const double* As = sbase + (kt % STAGES)*STAGE_DOUBLES;
        const double* Bs = As + BK*LDA;
        #pragma unroll
        for (int kk = 0; kk < BK; kk += 4)
        {
            double af[MS], bf[NS];
            #pragma unroll
            for (int i = 0; i < MS; i++) af[i] = As[(kk + fc)*LDA + wm0 + i*8 + fr];
            #pragma unroll
            for (int j = 0; j < NS; j++) bf[j] = Bs[(kk + fc)*LDB + wn0 + j*8 + fr];
            #pragma unroll
            for (int i = 0; i < MS; i++)
                #pragma unroll
                for (int j = 0; j < NS; j++)
                    dmma(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
        }
    }
    cp_async_wait<0>();

    // epilogue
    if (p.splits > 1)
    {
        // raw partial sums into the workspace, [split][l][m][n] dense
        double* W = p.partial + ((i64)split*p.L + l)*p.M*p.N;
        #pragma unroll
        for (int i = 0; i < MS; i++)
        {
            const i64 m = m0 + wm0 + i*8 + fr;
            if (m >= p.M) continue;
            #pragma unroll
            for (int j = 0; j < NS; j++)
            {
                #pragma unroll
                for (int h = 0; h < 2; h++)
                {
                    const i64 n = n0 + wn0 + j*8 + fc*2 + h;
                    if (n < p.N) W[m*p.N + n] = acc[i][j][h];
                }
            }
        }
        return;
    }

    double* C = p.C + p.c_l[l];
    const double alpha = p.alpha, beta = p.beta;
    #pragma unroll
    for (int i = 0; i < MS; i++)
    {
        const int ml = wm0 + i*8 + fr;
        const i64 rc = sCm[ml];
        if (rc < 0) continue;
        #pragma unroll
        for (int j = 0; j < NS; j++)
        {
            #pragma unroll
            for (int h = 0; h < 2; h++)
            {
                const i64 cc = sCn[wn0 + j*8 + fc*2 + h];
                if (cc < 0) continue;
                double* dst = C + rc + cc;
                const double v = alpha*acc[i][j][h];
                *dst = beta == 0.0 ? v : v + beta*(*dst);
            }
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

template <int AM, int BMd>
void launch_one(const GemmF64Args& a, dim3 grid, cudaStream_t s)
{
    auto kern = gemm_f64_kernel<AM, BMd>;
    static bool attr_set = false;
    if (!attr_set)
    {
        TB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_BYTES));
        attr_set = true;
    }
    kern<<<grid, NTHREADS, SMEM_BYTES, s>>>(a);
    check_launch("gemm_f64_kernel");
}

} // namespace

i64 gemm_f64_tile_m() { return BM; }
i64 gemm_f64_tile_n() { return BN; }
i64 gemm_f64_tile_k() { return BK; }

int gemm_f64_choose_splits(i64 M, i64 N, i64 K, i64 L, int num_sms)
{
    const i64 tiles = ((M + BM - 1)/BM)*((N + BN - 1)/BN)*L;
    const i64 kt = (K + BK - 1)/BK;
    if (tiles >= num_sms || kt < 8) return 1;
    i64 s = (2*num_sms + tiles - 1)/tiles;
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
    const i64 tiles_m = (a.M + BM - 1)/BM, tiles_n = (a.N + BN - 1)/BN;
    TB_CHECK(a.L <= 65535 && a.splits <= 65535, TB_ERR_SIZE, "batch extent too large");
    if (a.splits < 1) a.splits = 1;
    // split boundaries on BK multiples
    const i64 kt = (a.K + BK - 1)/BK;
    const i64 kt_per = (kt + a.splits - 1)/a.splits;
    a.k_per_split = std::max<i64>(1, kt_per)*BK;
    a.splits = (int)std::max<i64>(1, (a.K + a.k_per_split - 1)/a.k_per_split);
    TB_CHECK(a.splits == 1 || a.partial, TB_ERR_ARG, "split-K needs a workspace");
    dim3 grid((unsigned)(tiles_m*tiles_n), (unsigned)a.L, (unsigned)a.splits);
    if (a.K == 0) return;

    switch (a.amode*2 + a.bmode)
    {
        case 0: launch_one<0,0>(a, grid, stream); break;
        case 1: launch_one<0,1>(a, grid, stream); break;
        case 2: launch_one<1,0>(a, grid, stream); break;
        default: launch_one<1,1>(a, grid, stream); break;
    }

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
