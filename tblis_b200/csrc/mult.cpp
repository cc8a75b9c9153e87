// mult.cpp -- contraction dispatch.
//
// Restates src/iface/3t/mult.cxx:24-165 (alpha = alpha_A*alpha_B, beta =
// C's scalar, alpha == 0 => set/scale C, C's scalar reset to 1 and conj to
// false afterwards) and src/internal/3t/dense/mult.cxx:777-1023 (empty-extent
// early outs, n_AB == 0 => set/scale C). Every non-trivial group combination
// runs through one GEMM view on the device (the reference's 16-way dispatch
// collapses because the view treats an empty group as extent 1).
#include "mult.hpp"
#include "planner.hpp"
#include "gemm_f64.hpp"
#include "level1.hpp"
#include "ozaki.hpp"

#include <cmath>

namespace tb
{

int device_sm_count()
{
    static int cached[64] = {0};
    int dev = 0;
    TB_CUDA(cudaGetDevice(&dev));
    if (dev < 64 && cached[dev]) return cached[dev];
    int n = 0;
    TB_CUDA(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
    if (dev < 64) cached[dev] = n;
    return n;
}

struct StagedOp
{
    void* dptr = nullptr;
    dbuf buf;
    void* host = nullptr;
    i64 lo = 0, n = 0;
    bool staged = false;
};

static void stage(StagedOp& o, const tblis_tensor* t, bool copy_in, cudaStream_t s)
{
    if (!t->data) return;
    if (pointer_kind(t->data) == MEM_DEVICE) { o.dptr = t->data; return; }
    i64 lo, hi;
    tensor_extent(t->ndim, t->len, t->stride, lo, hi);
    if (hi < lo) { o.dptr = t->data; return; }
    o.staged = true;
    o.host = t->data;
    o.lo = lo;
    o.n = hi - lo + 1;
    o.buf = dbuf((size_t)o.n*sizeof(double), s);
    if (copy_in)
        TB_CUDA(cudaMemcpyAsync(o.buf.ptr, static_cast<double*>(o.host) + lo, (size_t)o.n*sizeof(double),
                                cudaMemcpyHostToDevice, s));
    o.dptr = o.buf.as<double>() - lo;
}

static void unstage(StagedOp& o, cudaStream_t s)
{
    if (!o.staged) return;
    TB_CUDA(cudaMemcpyAsync(static_cast<double*>(o.host) + o.lo, o.buf.ptr, (size_t)o.n*sizeof(double),
                            cudaMemcpyDeviceToHost, s));
}

void mult_dispatch(const tblis_config* cfg,
                   const tblis_tensor* A, const label_type* idx_A,
                   const tblis_tensor* B, const label_type* idx_B,
                   tblis_tensor* C, const label_type* idx_C,
                   const tblis_b200_opts* opts, tblis_b200_report* report)
{
    TB_CHECK(A && B && C, TB_ERR_ARG, "null tensor");
    TB_CHECK(A->type == B->type && A->type == C->type, TB_ERR_TYPE, "mult: operand types differ");
    TB_CHECK(A->type == TYPE_DOUBLE, TB_ERR_TYPE,
             "mult: only double is supported on the GPU path");
    ensure_device();
    cudaStream_t st = current_stream();
    const int kernels_before = (int)g_kernel_count.load();

    MultGroups g = mult_groups(A, idx_A, B, idx_B, C, idx_C);
    GemmView v = gemm_view(g);

    const double alpha = A->scalar.data.d*B->scalar.data.d;
    const double beta = C->scalar.data.d;

    int method = cfg ? cfg->method : 1;
    double tol = cfg ? cfg->tolerance : 1e-12;
    int slices = 0;
    if (opts)
    {
        if (opts->method) method = opts->method;
        if (opts->tolerance > 0) tol = opts->tolerance;
        slices = opts->slices;
    }

    if (report)
    {
        report->method = method;
        report->slices = 0;
        report->est_error = 0;
        report->m = v.m; report->n = v.n; report->k = v.k; report->l = v.l;
        report->flops = 2.0*(double)v.m*(double)v.n*(double)v.k*(double)v.l;
        report->kernels = 0;
    }

    const bool trivial = alpha == 0.0 || v.k == 0;
    StagedOp sa, sb, sc;
    stage(sc, C, beta != 0.0, st);

    if (v.m*v.n*v.l != 0)
    {
        if (trivial)
        {
            // set or scale C over all its dims (src/iface/3t/mult.cxx:133-148)
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
                if (beta == 0.0) l1_set<double>(static_cast<double*>(sc.dptr), s, 0.0, st);
                else l1_scale<double>(static_cast<double*>(sc.dptr), s, beta, st);
            }
        }
        else
        {
            stage(sa, A, true, st);
            stage(sb, B, true, st);
            TB_CHECK(method >= 1 && method <= 5, TB_ERR_ARG, "unknown contraction method");
            if (method >= 2)
            {
                // 2: Ozaki INT8 slices, 3: Ozaki BF16 slices, 4: one TF32 pass, 5: one BF16 pass
                const int kind = method == 2 ? OZ_I8 : method == 4 ? OZ_TF32 : OZ_BF16;
                OzakiResult r = ozaki_mult(v, static_cast<const double*>(sa.dptr),
                                           static_cast<const double*>(sb.dptr),
                                           static_cast<double*>(sc.dptr), alpha, beta, tol, slices, st,
                                           kind, method >= 4);
                if (report) { report->slices = r.slices; report->est_error = r.est_error; }
            }
            else
            {
                const i64 BMt = gemm_f64_tile_m(), BNt = gemm_f64_tile_n(), BKt = gemm_f64_tile_k();
                auto tab = gemm_tables(v, BMt, BNt, BKt, st);
                GemmF64Args a = {};
                a.A = static_cast<const double*>(sa.dptr);
                a.B = static_cast<const double*>(sb.dptr);
                a.C = static_cast<double*>(sc.dptr);
                a.a_m = tab->a_m; a.a_k = tab->a_k; a.b_k = tab->b_k; a.b_n = tab->b_n;
                a.c_m = tab->c_m; a.c_n = tab->c_n; a.a_l = tab->a_l; a.b_l = tab->b_l; a.c_l = tab->c_l;
                a.a_kbs = tab->a_kbs; a.b_kbs = tab->b_kbs;
                a.M = v.m; a.N = v.n; a.K = v.k; a.L = v.l;
                a.alpha = alpha; a.beta = beta;
                a.amode = v.amode; a.bmode = v.bmode;
                a.splits = gemm_f64_choose_splits(v.m, v.n, v.k, v.l, device_sm_count());
                dbuf ws(gemm_f64_workspace_bytes(v.m, v.n, v.l, a.splits), st);
                a.partial = ws.as<double>();
                gemm_f64_launch(a, st);
                if (report) report->est_error = 1.1e-16*std::sqrt((double)v.k);
            }
        }
    }

    unstage(sc, st);
    if (sa.staged || sb.staged || sc.staged) TB_CUDA(cudaStreamSynchronize(st));

    C->scalar.data.d = 1.0;
    C->scalar.type = TYPE_DOUBLE;
    C->conj = 0;
    if (report) report->kernels = (int)(g_kernel_count.load() - kernels_before);
}

} // namespace tb
