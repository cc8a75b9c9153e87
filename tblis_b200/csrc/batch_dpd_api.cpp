// batch_dpd_api.cpp -- C ABI of the DPD contraction, the DPD block layout
// query and batched dense contractions (one grouped launch for many small
// contractions of mixed shapes).
#include "common.hpp"
#include "dpd.hpp"
#include "grouped.hpp"
#include "level1.hpp"
#include "mult.hpp"

#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>

namespace tb
{

namespace
{

void to_layout(const tblis_b200_dpd_tensor* t, DpdLayout& lay)
{
    TB_CHECK(t, TB_ERR_ARG, "null DPD tensor");
    elem_size(t->type);
    TB_CHECK(t->len, TB_ERR_ARG, "DPD: null lengths");
    std::vector<i64> lens(t->len, t->len + (size_t)t->ndim*t->nirrep);
    lay.init(t->irrep, t->nirrep, t->ndim, lens.data(), t->layout < 0 ? 5 : t->layout);
}

// device view of a DPD tensor's storage (staged when it lives on the host)
struct DpdStage
{
    dbuf buf;
    char* host = nullptr;
    char* dev = nullptr;
    size_t bytes = 0;
    void init(void* data, i64 total, size_t esz, bool copy_in, cudaStream_t st)
    {
        bytes = (size_t)total*esz;
        dev = static_cast<char*>(data);
        if (!data || total == 0 || pointer_kind(data) == MEM_DEVICE) return;
        host = static_cast<char*>(data);
        buf = dbuf(bytes, st);
        dev = buf.as<char>();
        if (copy_in) TB_CUDA(cudaMemcpyAsync(dev, host, bytes, cudaMemcpyHostToDevice, st));
    }
    void out(cudaStream_t st)
    {
        if (host) TB_CUDA(cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, st));
    }
};

void to_layout(const tblis_b200_dpd_block_table* t, DpdLayout& lay)
{
    TB_CHECK(t, TB_ERR_ARG, "null DPD tensor");
    elem_size(t->type);
    TB_CHECK(t->len, TB_ERR_ARG, "DPD: null lengths");
    std::vector<i64> lens(t->len, t->len + (size_t)t->ndim*t->nirrep);
    lay.init_explicit(t->irrep, t->nirrep, t->ndim, lens.data(), t->offset, t->stride);
}

// both descriptor kinds carry the same header fields
template <typename Desc>
void run_dpd_mult(const Desc* A, const label_type* idx_A, const Desc* B, const label_type* idx_B,
                  Desc* C, const label_type* idx_C, tblis_b200_report* report)
{
    ensure_device();
    cudaStream_t st = current_stream();
    const int k0 = (int)g_kernel_count.load();
    TB_CHECK(A && B && C, TB_ERR_ARG, "null DPD tensor");
    TB_CHECK(A->type == B->type && A->type == C->type, TB_ERR_TYPE, "DPD mult: operand types differ");
    const int type = C->type;
    const size_t esz = elem_size(type);
    DpdTensor a, b, c;
    to_layout(A, a.lay);
    to_layout(B, b.lay);
    to_layout(C, c.lay);
    const zd alpha = scalar_get(A->scalar)*scalar_get(B->scalar), beta = scalar_get(C->scalar);
    DpdStage sa, sb, sc;
    sa.init(A->data, a.lay.total(), esz, true, st);
    sb.init(B->data, b.lay.total(), esz, true, st);
    // a block table may leave gaps in the storage: those come back unchanged
    sc.init(C->data, c.lay.total(), esz, beta != 0.0 || c.lay.is_explicit(), st);
    DpdMultReport r;
    if (type == TYPE_DOUBLE)
    {
        a.data = reinterpret_cast<double*>(sa.dev); b.data = reinterpret_cast<double*>(sb.dev);
        c.data = reinterpret_cast<double*>(sc.dev);
        dpd_mult(a, idx_A, b, idx_B, c, idx_C, alpha.real(), beta.real(), st, &r);
    }
    else if (type == TYPE_DCOMPLEX)
        dpd_mult_z(a.lay, reinterpret_cast<const double*>(sa.dev), idx_A, b.lay, reinterpret_cast<const double*>(sb.dev),
                   idx_B, c.lay, reinterpret_cast<double*>(sc.dev), idx_C, alpha, beta, st, &r);
    else
    {
        // float / scomplex: contracted in double / dcomplex and rounded back
        const bool cx = type == TYPE_SCOMPLEX;
        dbuf wa = dpd_widen(sa.dev, a.lay.total(), cx, st), wb = dpd_widen(sb.dev, b.lay.total(), cx, st);
        dbuf wc;
        if (beta != 0.0) wc = dpd_widen(sc.dev, c.lay.total(), cx, st);
        else
        {
            // beta == 0: C is not read; zeros stand in for it
            wc = dbuf((size_t)std::max<i64>(c.lay.total()*(cx ? 2 : 1), 1)*sizeof(double), st);
            TB_CUDA(cudaMemsetAsync(wc.ptr, 0, wc.bytes, st));
        }
        if (cx)
            dpd_mult_z(a.lay, wa.as<double>(), idx_A, b.lay, wb.as<double>(), idx_B, c.lay, wc.as<double>(), idx_C,
                       alpha, beta, st, &r);
        else
        {
            a.data = wa.as<double>(); b.data = wb.as<double>(); c.data = wc.as<double>();
            dpd_mult(a, idx_A, b, idx_B, c, idx_C, alpha.real(), beta.real(), st, &r);
        }
        dpd_narrow_blocks(c.lay, cx, wc.as<double>(), reinterpret_cast<float*>(sc.dev), st);
    }
    sc.out(st);
    if (sa.host || sb.host || sc.host) TB_CUDA(cudaStreamSynchronize(st));
    scalar_put(C->scalar, type, 1.0);
    C->conj = 0;
    if (report)
    {
        memset(report, 0, sizeof(*report));
        report->method = 1;
        report->flops = r.flops;
        report->m = r.groups;            // number of irrep GEMMs in the grouped launch
        report->n = r.variant;           // tile configuration the autotuner picked
        report->kernels = (int)(g_kernel_count.load() - k0);
    }
}

// everything a batch plan depends on, straight from the caller's descriptors
// (lengths, strides, labels, and whether alpha is zero): a cache hit skips
// all planning
std::string batch_key(int count, const tblis_tensor* A, const label_type* const* idx_A,
                      const tblis_tensor* B, const label_type* const* idx_B,
                      const tblis_tensor* C, const label_type* const* idx_C)
{
    std::string key;
    key.reserve((size_t)count*160);
    for (int i = 0; i < count; i++)
    {
        const tblis_tensor* ts[3] = {&A[i], &B[i], &C[i]};
        const label_type* ix[3] = {idx_A[i], idx_B[i], idx_C[i]};
        for (int t = 0; t < 3; t++)
        {
            const unsigned nd = ts[t]->ndim;
            key.push_back((char)nd);
            key.append(reinterpret_cast<const char*>(ts[t]->len), nd*sizeof(len_type));
            key.append(reinterpret_cast<const char*>(ts[t]->stride), nd*sizeof(stride_type));
            if (nd) key.append(ix[t], nd);
        }
        key.push_back(A[i].scalar.data.d*B[i].scalar.data.d == 0.0 ? 'z' : 'n');
    }
    return key;
}

struct BatchPlanExtra
{
    // members that need no GEMM (alpha == 0 or an empty contracted extent)
    std::vector<std::pair<int, Strided>> trivial;
};

std::mutex g_extra_mtx;
std::map<const GroupedPlan*, BatchPlanExtra> g_extra;

void run_batch(int count, const tblis_tensor* A, const label_type* const* idx_A,
               const tblis_tensor* B, const label_type* const* idx_B,
               tblis_tensor* C, const label_type* const* idx_C, tblis_b200_report* report)
{
    ensure_device();
    cudaStream_t st = current_stream();
    const int k0 = (int)g_kernel_count.load();
    TB_CHECK(count >= 0, TB_ERR_ARG, "batch: negative count");
    std::vector<const double*> ptrs(3*(size_t)count);
    std::vector<double> alphas(count), betas(count);
    for (int i = 0; i < count; i++)
    {
        TB_CHECK(A[i].type == TYPE_DOUBLE && B[i].type == TYPE_DOUBLE && C[i].type == TYPE_DOUBLE, TB_ERR_TYPE,
                 "batch: only double tensors");
        ptrs[3*i] = static_cast<const double*>(A[i].data);
        ptrs[3*i + 1] = static_cast<const double*>(B[i].data);
        ptrs[3*i + 2] = static_cast<const double*>(C[i].data);
        alphas[i] = A[i].scalar.data.d*B[i].scalar.data.d;
        betas[i] = C[i].scalar.data.d;
    }
    const std::string key = batch_key(count, A, idx_A, B, idx_B, C, idx_C);
    auto plan = grouped_plan_cache().find(key);
    if (!plan)
    {
        auto p = std::make_shared<GroupedPlan>();
        BatchPlanExtra extra;
        double flops = 0;
        for (int i = 0; i < count; i++)
        {
            for (const tblis_tensor* t : {&A[i], &B[i], (const tblis_tensor*)&C[i]})
            {
                i64 lo, hi;
                tensor_extent(t->ndim, t->len, t->stride, lo, hi);
                TB_CHECK(hi < lo || !t->data || pointer_kind(t->data) == MEM_DEVICE, TB_ERR_ARG,
                         "batch: tensors must be in device memory");
            }
            const GemmView v = gemm_view(mult_groups(&A[i], idx_A[i], &B[i], idx_B[i], &C[i], idx_C[i]));
            const bool trivial = alphas[i] == 0.0 || v.k == 0 || v.m*v.n*v.l == 0;
            if (trivial)
            {
                if (v.m*v.n*v.l == 0) continue;
                Strided s;
                ivec len, str;
                for (size_t j = 0; j < v.lenM.size(); j++) { len.push_back(v.lenM[j]); str.push_back(v.cM[j]); }
                for (size_t j = 0; j < v.lenN.size(); j++) { len.push_back(v.lenN[j]); str.push_back(v.cN[j]); }
                for (size_t j = 0; j < v.lenL.size(); j++) { len.push_back(v.lenL[j]); str.push_back(v.cL[j]); }
                TB_CHECK(len.size() <= (size_t)L1_MAX_DIM, TB_ERR_SIZE, "too many dimensions");
                s.ndim = (int)len.size();
                for (size_t j = 0; j < len.size(); j++) { s.len[j] = len[j]; s.stride[j] = str[j]; }
                extra.trivial.push_back({i, s});
                continue;
            }
            GroupTables base;
            base.M = v.m; base.N = v.n; base.K = v.k;
            base.a_m.resize(v.m); base.c_m.resize(v.m); base.a_k.resize(v.k); base.b_k.resize(v.k);
            base.b_n.resize(v.n); base.c_n.resize(v.n);
            std::vector<i64> bs(std::max({v.m, v.n, v.k, v.l}));
            fill_block_scatter(v.lenM, v.aM, 1, 0, v.m, base.a_m.data(), bs.data(), v.pack_m_3d);
            fill_block_scatter(v.lenM, v.cM, 1, 0, v.m, base.c_m.data(), bs.data(), v.pack_m_3d);
            fill_block_scatter(v.lenN, v.bN, 1, 0, v.n, base.b_n.data(), bs.data(), v.pack_n_3d);
            fill_block_scatter(v.lenN, v.cN, 1, 0, v.n, base.c_n.data(), bs.data(), v.pack_n_3d);
            fill_block_scatter(v.lenK, v.aK, 1, 0, v.k, base.a_k.data(), bs.data(), v.pack_k_3d);
            fill_block_scatter(v.lenK, v.bK, 1, 0, v.k, base.b_k.data(), bs.data(), v.pack_k_3d);
            base.amode = v.amode; base.bmode = v.bmode;
            base.a_slot = 3*i; base.b_slot = 3*i + 1; base.c_slot = 3*i + 2;
            base.sidx = i;
            std::vector<i64> al(v.l), bl(v.l), cl(v.l);
            fill_block_scatter(v.lenL, v.aL, 1, 0, v.l, al.data(), bs.data(), false);
            fill_block_scatter(v.lenL, v.bL, 1, 0, v.l, bl.data(), bs.data(), false);
            fill_block_scatter(v.lenL, v.cL, 1, 0, v.l, cl.data(), bs.data(), false);
            for (i64 l = 0; l < v.l; l++)
            {
                GroupTables g = base;
                g.a_off = al[l]; g.b_off = bl[l]; g.c_off = cl[l];
                p->groups.push_back(std::move(g));
            }
            flops += 2.0*v.m*v.n*v.k*v.l;
        }
        p->flops = flops;
        p->nslots = 3*count;
        p->finalize(st);
        {
            std::lock_guard<std::mutex> lk(g_extra_mtx);
            g_extra[p.get()] = std::move(extra);
        }
        plan = grouped_plan_cache().insert(key, p);
    }

    // trivial members: set/scale C
    {
        std::lock_guard<std::mutex> lk(g_extra_mtx);
        for (auto& t : g_extra[plan.get()].trivial)
        {
            const int i = t.first;
            if (betas[i] == 1.0) continue;
            if (betas[i] == 0.0) l1_set<double>(static_cast<double*>(C[i].data), t.second, 0.0, st);
            else l1_scale<double>(static_cast<double*>(C[i].data), t.second, betas[i], st);
        }
    }
    grouped_run(*plan, ptrs.data(), alphas.data(), betas.data(), st);
    for (int i = 0; i < count; i++)
    {
        C[i].scalar.data.d = 1.0;
        C[i].scalar.type = TYPE_DOUBLE;
        C[i].conj = 0;
    }
    if (report)
    {
        memset(report, 0, sizeof(*report));
        report->method = 1;
        report->flops = plan->flops;
        report->m = (int64_t)plan->groups.size();
        report->n = plan->variant;
        report->kernels = (int)(g_kernel_count.load() - k0);
    }
}

} // namespace

} // namespace tb

using namespace tb;

extern "C" {

int tblis_b200_dpd_mult(const tblis_b200_dpd_tensor* A, const label_type* idx_A,
                        const tblis_b200_dpd_tensor* B, const label_type* idx_B,
                              tblis_b200_dpd_tensor* C, const label_type* idx_C,
                        tblis_b200_report* report)
{
    return guarded([&] { run_dpd_mult(A, idx_A, B, idx_B, C, idx_C, report); });
}

int tblis_b200_dpd_mult_blocks(const tblis_b200_dpd_block_table* A, const label_type* idx_A,
                               const tblis_b200_dpd_block_table* B, const label_type* idx_B,
                                     tblis_b200_dpd_block_table* C, const label_type* idx_C,
                               tblis_b200_report* report)
{
    return guarded([&] { run_dpd_mult(A, idx_A, B, idx_B, C, idx_C, report); });
}

int tblis_b200_dpd_shard_plan(const tblis_b200_dpd_tensor* A, const label_type* idx_A,
                              const tblis_b200_dpd_tensor* B, const label_type* idx_B,
                              const tblis_b200_dpd_tensor* C, const label_type* idx_C,
                              int nranks, int* owner, double* flops)
{
    return guarded([&]
    {
        TB_CHECK(owner, TB_ERR_ARG, "null owner array");
        DpdTensor a, b, c;
        to_layout(A, a.lay);
        to_layout(B, b.lay);
        to_layout(C, c.lay);
        std::vector<double> load;
        const std::vector<int> own = dpd_shard_owner(a, idx_A, b, idx_B, c, idx_C, nranks, &load);
        std::copy(own.begin(), own.end(), owner);
        if (flops) std::copy(load.begin(), load.end(), flops);
    });
}

int tblis_b200_dpd_mult_shard(const tblis_b200_dpd_tensor* A, const label_type* idx_A,
                              const tblis_b200_dpd_tensor* B, const label_type* idx_B,
                                    tblis_b200_dpd_tensor* C, const label_type* idx_C,
                              int nranks, int rank, tblis_b200_report* report)
{
    return guarded([&]
    {
        ensure_device();
        cudaStream_t st = current_stream();
        const int k0 = (int)g_kernel_count.load();
        TB_CHECK(A && B && C, TB_ERR_ARG, "null DPD tensor");
        TB_CHECK(A->type == TYPE_DOUBLE && B->type == TYPE_DOUBLE && C->type == TYPE_DOUBLE, TB_ERR_TYPE,
                 "DPD shard: double tensors only");
        DpdTensor a, b, c;
        to_layout(A, a.lay);
        to_layout(B, b.lay);
        to_layout(C, c.lay);
        const double alpha = A->scalar.data.d*B->scalar.data.d, beta = C->scalar.data.d;
        DpdStage sa, sb, sc;
        sa.init(A->data, a.lay.total(), sizeof(double), true, st);
        sb.init(B->data, b.lay.total(), sizeof(double), true, st);
        // blocks of other ranks come back unchanged: C is copied in
        sc.init(C->data, c.lay.total(), sizeof(double), true, st);
        a.data = reinterpret_cast<double*>(sa.dev);
        b.data = reinterpret_cast<double*>(sb.dev);
        c.data = reinterpret_cast<double*>(sc.dev);
        DpdMultReport r;
        dpd_mult_shard(a, idx_A, b, idx_B, c, idx_C, alpha, beta, nranks, rank, st, &r);
        sc.out(st);
        if (sa.host || sb.host || sc.host) TB_CUDA(cudaStreamSynchronize(st));
        C->scalar.data.d = 1.0;
        C->scalar.type = TYPE_DOUBLE;
        C->conj = 0;
        if (report)
        {
            memset(report, 0, sizeof(*report));
            report->method = 1;
            report->flops = r.flops;
            report->m = r.groups;
            report->kernels = (int)g_kernel_count.load() - k0;
        }
    });
}

int tblis_b200_dpd_block(const tblis_b200_dpd_tensor* A, const unsigned* irreps, len_type* len,
                         stride_type* stride, stride_type* offset)
{
    return guarded([&]
    {
        DpdLayout lay;
        to_layout(A, lay);
        std::vector<i64> l(lay.ndim), s(lay.ndim);
        i64 off;
        unsigned x = 0;
        for (unsigned i = 0; i < lay.ndim; i++)
        {
            TB_CHECK(irreps[i] < lay.nirrep, TB_ERR_ARG, "DPD: irrep out of range");
            x ^= irreps[i];
        }
        TB_CHECK(x == lay.irrep, TB_ERR_ARG, "DPD: block not allowed by symmetry");
        lay.block(irreps, l.data(), s.data(), off);
        for (unsigned i = 0; i < lay.ndim; i++) { len[i] = l[i]; stride[i] = s[i]; }
        *offset = off;
    });
}

len_type tblis_b200_dpd_size(const tblis_b200_dpd_tensor* A)
{
    len_type n = -1;
    guarded([&] { DpdLayout lay; to_layout(A, lay); n = lay.total(); });
    return n;
}

int tblis_b200_tensor_mult_batch(int count, const tblis_tensor* A, const label_type* const* idx_A,
                                 const tblis_tensor* B, const label_type* const* idx_B,
                                       tblis_tensor* C, const label_type* const* idx_C,
                                 tblis_b200_report* report)
{
    return guarded([&] { run_batch(count, A, idx_A, B, idx_B, C, idx_C, report); });
}

} // extern "C"
