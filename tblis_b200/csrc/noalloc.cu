// noalloc.cu -- an allocation-free variant of the FP64 contraction.
//
// Some callers cannot let a library allocate device memory: a solver whose
// device memory is owned entirely by another allocator (a framework's caching
// allocator that reserved the GPU up front), or a latency-critical loop that
// must not hit cudaMalloc/cudaFree, which can synchronise the whole device
// and stall every other stream. tblis_b200_tensor_mult_noalloc serves them:
// it runs the same FP64 DMMA block-scatter kernel as tblis_tensor_mult, but
// every piece of scratch memory it needs -- the scatter vectors of the GEMM
// view and the split-K partial tiles -- lives in one file-scope __device__
// array of fixed size (g_noalloc_scratch below). That array is part of the
// library image: every GPU that loads libtblis_b200.so holds it until the
// process exits.
//
// Rules of use:
//  * tensors must already be in device (or managed) memory: host data would
//    need a staging buffer, which is an allocation, so host pointers are
//    rejected with TB_ERR_ARG;
//  * alpha == 0 or an empty contracted extent sets C (beta == 0) or scales it
//    by beta, as tblis_tensor_mult does; that path needs no scratch at all;
//  * scatter vectors plus split-K partials must fit in
//    TBLIS_B200_NOALLOC_SCRATCH_BYTES; when the partials do not fit the
//    split-K factor is reduced (down to no split), and a contraction whose
//    scatter vectors alone do not fit is rejected with TB_ERR_SIZE;
//  * every call shares the one array and leaves its contents behind. Nothing
//    in it has to start at zero (each call overwrites every word it reads),
//    but calls whose work overlaps on the GPU -- concurrent streams, or
//    several host threads -- race on it and must be serialised by the caller;
//  * a call that fails leaves C and its scalar untouched, as
//    tblis_tensor_mult does;
//  * the first call on a device looks up the array's device address with
//    cudaGetSymbolAddress (the array's name is only a host-side stand-in in
//    host code); make that first call before any stream capture.
#include "common.hpp"
#include "planner.hpp"
#include "gemm_f64.hpp"
#include "mult.hpp"
#include "level1.hpp"

#include <algorithm>
#include <mutex>

namespace tb
{

namespace
{

constexpr size_t kScratchBytes = TBLIS_B200_NOALLOC_SCRATCH_BYTES;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// device address of g_noalloc_scratch, looked up once per device
void* scratch_address()
{
    static std::mutex mtx;
    static void* addr[64] = {nullptr};
    int dev = 0;
    TB_CUDA(cudaGetDevice(&dev));
    TB_CHECK(dev < 64, TB_ERR_SIZE, "device ordinal beyond 63");
    std::lock_guard<std::mutex> lk(mtx);
    if (!addr[dev])
    {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            throw error(TB_ERR_CUDA, std::string("cudaGetSymbolAddress(g_noalloc_scratch): ") +
                                     cudaGetErrorString(e));
        addr[dev] = p;
    }
    return addr[dev];
}

size_t align256(size_t n) { return (n + 255) & ~size_t(255); }

void run_noalloc(const tblis_tensor* A, const label_type* idx_A,
                 const tblis_tensor* B, const label_type* idx_B,
                 tblis_tensor* C, const label_type* idx_C)
{
    TB_CHECK(A && B && C, TB_ERR_ARG, "null tensor");
    TB_CHECK(A->type == TYPE_DOUBLE && B->type == TYPE_DOUBLE && C->type == TYPE_DOUBLE, TB_ERR_TYPE,
             "noalloc mult: only double tensors");
    ensure_device();
    cudaStream_t st = current_stream();
    char* scratch = static_cast<char*>(scratch_address());

    MultGroups g = mult_groups(A, idx_A, B, idx_B, C, idx_C);
    GemmView v = gemm_view(g);
    const double alpha = A->scalar.data.d*B->scalar.data.d;
    const double beta = C->scalar.data.d;

    for (const tblis_tensor* t : {A, B, (const tblis_tensor*)C})
    {
        i64 lo, hi;
        tensor_extent(t->ndim, t->len, t->stride, lo, hi);
        if (hi >= lo && t->data)
            TB_CHECK(pointer_kind(t->data) == MEM_DEVICE, TB_ERR_ARG,
                     "noalloc mult: tensors must be in device memory (host data would need a staging allocation)");
    }

    if (v.m*v.n*v.l != 0 && (alpha == 0.0 || v.k == 0))
    {
        // no product: C = beta*C over all its dims, or C = 0 without reading
        // it (src/iface/3t/mult.cxx:133-148)
        if (beta != 1.0)
        {
            Strided s;
            ivec len, str;
            for (size_t i = 0; i < v.lenM.size(); i++) { len.push_back(v.lenM[i]); str.push_back(v.cM[i]); }
            for (size_t i = 0; i < v.lenN.size(); i++) { len.push_back(v.lenN[i]); str.push_back(v.cN[i]); }
            for (size_t i = 0; i < v.lenL.size(); i++) { len.push_back(v.lenL[i]); str.push_back(v.cL[i]); }
            TB_CHECK(len.size() <= (size_t)L1_MAX_DIM, TB_ERR_SIZE, "too many dimensions");
            s.ndim = (int)len.size();
            for (size_t i = 0; i < len.size(); i++) { s.len[i] = len[i]; s.stride[i] = str[i]; }
            if (beta == 0.0) l1_set<double>(static_cast<double*>(C->data), s, 0.0, st);
            else l1_scale<double>(static_cast<double*>(C->data), s, beta, st);
        }
    }
    else if (v.m*v.n*v.l != 0)
    {
        const i64 BM = gemm_f64_tile_m(), BN = gemm_f64_tile_n(), BK = gemm_f64_tile_k();
        const i64 nkb = (v.k + BK - 1)/BK;
        const size_t n_tab = 2*v.m + 2*v.k + 2*v.n + 3*v.l + 2*nkb;
        const size_t tab_bytes = align256(n_tab*sizeof(i64));
        TB_CHECK(tab_bytes <= kScratchBytes, TB_ERR_SIZE,
                 "noalloc mult: scatter vectors exceed the fixed scratch size");

        std::vector<i64> host(n_tab);
        i64* p = host.data();
        i64 *a_m = p; p += v.m;  i64 *c_m = p; p += v.m;
        i64 *a_k = p; p += v.k;  i64 *b_k = p; p += v.k;
        i64 *b_n = p; p += v.n;  i64 *c_n = p; p += v.n;
        i64 *a_l = p; p += v.l;  i64 *b_l = p; p += v.l;  i64 *c_l = p; p += v.l;
        i64 *a_kbs = p; p += nkb; i64 *b_kbs = p; p += nkb;
        std::vector<i64> bs(std::max({v.m, v.n, v.k, v.l}));
        fill_block_scatter(v.lenM, v.aM, BM, 0, v.m, a_m, bs.data(), v.pack_m_3d);
        fill_block_scatter(v.lenM, v.cM, BM, 0, v.m, c_m, bs.data(), v.pack_m_3d);
        fill_block_scatter(v.lenN, v.bN, BN, 0, v.n, b_n, bs.data(), v.pack_n_3d);
        fill_block_scatter(v.lenN, v.cN, BN, 0, v.n, c_n, bs.data(), v.pack_n_3d);
        fill_block_scatter(v.lenK, v.aK, BK, 0, v.k, a_k, bs.data(), v.pack_k_3d);
        for (i64 b = 0; b < nkb; b++) a_kbs[b] = bs[b*BK];
        fill_block_scatter(v.lenK, v.bK, BK, 0, v.k, b_k, bs.data(), v.pack_k_3d);
        for (i64 b = 0; b < nkb; b++) b_kbs[b] = bs[b*BK];
        fill_block_scatter(v.lenL, v.aL, 1, 0, v.l, a_l, bs.data(), false);
        fill_block_scatter(v.lenL, v.bL, 1, 0, v.l, b_l, bs.data(), false);
        fill_block_scatter(v.lenL, v.cL, 1, 0, v.l, c_l, bs.data(), false);

        // pageable source: the copy is staged by the driver before return
        TB_CUDA(cudaMemcpyAsync(scratch, host.data(), n_tab*sizeof(i64), cudaMemcpyHostToDevice, st));
        const i64* d = reinterpret_cast<const i64*>(scratch);

        GemmF64Args a = {};
        a.A = static_cast<const double*>(A->data);
        a.B = static_cast<const double*>(B->data);
        a.C = static_cast<double*>(C->data);
        a.a_m = d + (a_m - host.data()); a.c_m = d + (c_m - host.data());
        a.a_k = d + (a_k - host.data()); a.b_k = d + (b_k - host.data());
        a.b_n = d + (b_n - host.data()); a.c_n = d + (c_n - host.data());
        a.a_l = d + (a_l - host.data()); a.b_l = d + (b_l - host.data());
        a.c_l = d + (c_l - host.data());
        a.a_kbs = d + (a_kbs - host.data()); a.b_kbs = d + (b_kbs - host.data());
        a.M = v.m; a.N = v.n; a.K = v.k; a.L = v.l;
        a.alpha = alpha; a.beta = beta;
        a.amode = v.amode; a.bmode = v.bmode;
        // 16-byte pair gathers where the layout gives them, decided as for
        // tblis_tensor_mult (the kernel still checks every pair)
        bool a_pairs[2], b_pairs[2];
        gemm_pair_modes(v, a_m, a_k, b_n, b_k, a_l, b_l, a_pairs, b_pairs);
        a.pair_a = a_pairs[v.amode] && ((uintptr_t)a.A & 15) == 0;
        a.pair_b = b_pairs[v.bmode] && ((uintptr_t)a.B & 15) == 0;

        // split-K partials go after the tables; shrink the split until they fit
        int splits = gemm_f64_choose_splits(v.m, v.n, v.k, v.l, device_sm_count());
        while (splits > 1 && tab_bytes + gemm_f64_workspace_bytes(v.m, v.n, v.l, splits) > kScratchBytes)
            splits--;
        a.splits = splits;
        a.partial = splits > 1 ? reinterpret_cast<double*>(scratch + tab_bytes) : nullptr;
        gemm_f64_launch(a, st);
    }

    C->scalar.data.d = 1.0;
    C->scalar.type = TYPE_DOUBLE;
    C->conj = 0;
}

} // namespace

} // namespace tb

extern "C" {

int tblis_b200_tensor_mult_noalloc(const tblis_tensor* A, const label_type* idx_A,
                                   const tblis_tensor* B, const label_type* idx_B,
                                         tblis_tensor* C, const label_type* idx_C)
{
    return tb::guarded([&] { tb::run_noalloc(A, idx_A, B, idx_B, C, idx_C); });
}

size_t tblis_b200_noalloc_scratch_bytes(void) { return tb::kScratchBytes; }

} // extern "C"
