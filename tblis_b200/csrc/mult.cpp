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

#include <algorithm>
#include <cmath>
#include <memory>
#include <mutex>

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
    size_t esz = sizeof(double);
    bool staged = false;
};

// t's strides count elements of esz bytes
static void stage(StagedOp& o, const tblis_tensor* t, bool copy_in, cudaStream_t s, size_t esz = sizeof(double))
{
    o.esz = esz;
    if (!t->data) return;
    if (pointer_kind(t->data) == MEM_DEVICE) { o.dptr = t->data; return; }
    i64 lo, hi;
    tensor_extent(t->ndim, t->len, t->stride, lo, hi);
    if (hi < lo) { o.dptr = t->data; return; }
    o.staged = true;
    o.host = t->data;
    o.lo = lo;
    o.n = hi - lo + 1;
    o.buf = dbuf((size_t)o.n*esz, s);
    // an extent with gaps is copied in even for an output: the copy back
    // writes the whole extent, and the gaps must come back unchanged
    i64 nelem = 1;
    for (unsigned d = 0; d < t->ndim; d++) nelem *= t->len[d];
    if (copy_in || nelem != o.n)
        TB_CUDA(cudaMemcpyAsync(o.buf.ptr, static_cast<char*>(o.host) + lo*(i64)esz, (size_t)o.n*esz,
                                cudaMemcpyHostToDevice, s));
    o.dptr = o.buf.as<char>() - lo*(i64)esz;
}

// A host-resident A is copied in slices on a copy stream while the slices
// already on the device are contracted. The cut label is A's label of
// largest stride, when that stride spans everything else A holds, so the
// slices of A are disjoint, ordered ranges of host memory. A label A shares
// with C cuts A and C (independent row slices); a label A shares with B (a
// contracted one) cuts A and B, and the slices accumulate into C (beta for
// the first, 1 after). Each slice is an ordinary contraction of sub-tensors
// (shorter extent of the label, data offset to the slice).
struct Slices
{
    int dim_A = -1, dim_C = -1, dim_B = -1;    // the cut label's dimension in A and in C or B
    std::vector<std::pair<i64, i64>> range;    // [q0, q1) of the label
    std::vector<std::pair<i64, i64>> fp;       // A footprint [lo, hi] of each slice (elements)
};

static bool plan_slices(const tblis_tensor* A, const label_type* idx_A, const tblis_tensor* B,
                        const label_type* idx_B, const tblis_tensor* C, const label_type* idx_C, Slices& sl)
{
    constexpr i64 kSliceBytes = (i64)384 << 20;
    i64 lo, hi;
    tensor_extent(A->ndim, A->len, A->stride, lo, hi);
    const i64 bytes = (hi - lo + 1)*8;
    if (bytes < 2*kSliceBytes) return false;
    for (unsigned d = 0; d < A->ndim; d++)
        if (A->stride[d] < 0) return false;
    // A's dimension of largest stride
    int q = -1;
    for (unsigned d = 0; d < A->ndim; d++)
        if (A->len[d] > 1 && (q < 0 || A->stride[d] > A->stride[q])) q = (int)d;
    if (q < 0) return false;
    const label_type c = idx_A[q];
    int nA = 0, nB = 0, nC = 0, qc = -1, qb = -1;
    for (unsigned d = 0; d < A->ndim; d++) nA += idx_A[d] == c;
    for (unsigned d = 0; d < B->ndim; d++) if (idx_B[d] == c) { nB++; qb = (int)d; }
    for (unsigned d = 0; d < C->ndim; d++) if (idx_C[d] == c) { nC++; qc = (int)d; }
    if (nA != 1 || nB + nC != 1) return false;
    // everything else of A fits below one step of the label
    i64 rest = 0;
    for (unsigned d = 0; d < A->ndim; d++)
        if ((int)d != q) rest += (A->len[d] - 1)*A->stride[d];
    const i64 s = A->stride[q], L = A->len[q];
    if (s <= rest) return false;
    const i64 n = std::min<i64>({16, L, std::max<i64>(2, bytes/kSliceBytes)});
    if (n < 2) return false;
    const i64 per = (L + n - 1)/n;
    sl.dim_A = q; sl.dim_C = qc; sl.dim_B = qb;
    for (i64 q0 = 0; q0 < L; q0 += per)
    {
        const i64 q1 = std::min(L, q0 + per);
        sl.range.push_back({q0, q1});
        sl.fp.push_back({q0*s, (q1 - 1)*s + rest});
    }
    return sl.range.size() >= 2;
}

// Row slabs of a host-resident A and C: a label of A and C (not B) whose
// lower-stride dims tile [0, stride) densely and whose higher-stride dims
// continue it as one regular pitch, in both tensors. A slab (a range of the
// label) is then a pitched block of `rows` rows of width range*stride in A
// and in C, so each slab contracts the whole K into its final part of C: its
// copy back can run while the next slab of A comes in.
struct Slabs
{
    int dim_A = -1, dim_C = -1;
    i64 s_A = 0, s_C = 0;                      // the label's strides
    i64 pitch_A = 0, pitch_C = 0;              // elements between rows
    i64 rows_A = 0, rows_C = 0;
    std::vector<std::pair<i64, i64>> range;    // [q0, q1) of the label
};

// dims below q tile [0, stride_q); dims above continue q as one pitch
static bool pitched(const tblis_tensor* X, int q, i64& pitch, i64& rows)
{
    const i64 sq = X->stride[q], lq = X->len[q];
    i64 inner = 1, span = 0;
    std::vector<std::pair<i64, i64>> outer;
    for (unsigned d = 0; d < X->ndim; d++)
    {
        if ((int)d == q || X->len[d] == 1) continue;
        if (X->stride[d] <= 0) return false;
        if (X->stride[d] < sq) { inner *= X->len[d]; span += (X->len[d] - 1)*X->stride[d]; }
        else outer.push_back({X->stride[d], X->len[d]});
    }
    if (inner != sq || span + 1 != sq) return false;
    std::sort(outer.begin(), outer.end());
    i64 expect = lq*sq;
    rows = 1;
    for (auto& o : outer)
    {
        if (o.first != expect) return false;
        expect *= o.second;
        rows *= o.second;
    }
    pitch = lq*sq;
    return true;
}

static bool plan_slabs(const tblis_tensor* A, const label_type* idx_A, const tblis_tensor* B,
                       const label_type* idx_B, const tblis_tensor* C, const label_type* idx_C, Slabs& sl)
{
    constexpr i64 kSliceBytes = (i64)384 << 20;
    constexpr i64 kMinRowBytes = 4096;         // narrower rows copy slowly
    i64 lo, hi;
    tensor_extent(A->ndim, A->len, A->stride, lo, hi);
    const i64 bytes = (hi - lo + 1)*8;
    if (bytes < 2*kSliceBytes) return false;
    i64 best_s = 0;
    for (unsigned qa = 0; qa < A->ndim; qa++)
    {
        const label_type c = idx_A[qa];
        if (A->len[qa] < 2) continue;
        int nA = 0, nB = 0, nC = 0, qc = -1;
        for (unsigned d = 0; d < A->ndim; d++) nA += idx_A[d] == c;
        for (unsigned d = 0; d < B->ndim; d++) nB += idx_B[d] == c;
        for (unsigned d = 0; d < C->ndim; d++) if (idx_C[d] == c) { nC++; qc = (int)d; }
        if (nA != 1 || nB != 0 || nC != 1) continue;
        i64 pa, ra, pc, rc;
        if (!pitched(A, (int)qa, pa, ra) || !pitched(C, qc, pc, rc)) continue;
        const i64 L = A->len[qa];
        const i64 n = std::min<i64>({16, L, std::max<i64>(2, bytes/kSliceBytes)});
        const i64 per = (L + n - 1)/n;
        if (per*std::min(A->stride[qa], C->stride[qc])*8 < kMinRowBytes) continue;
        if (A->stride[qa] <= best_s) continue;
        best_s = A->stride[qa];
        sl.dim_A = (int)qa; sl.dim_C = qc;
        sl.s_A = A->stride[qa]; sl.s_C = C->stride[qc];
        sl.pitch_A = pa; sl.pitch_C = pc; sl.rows_A = ra; sl.rows_C = rc;
        sl.range.clear();
        for (i64 q0 = 0; q0 < L; q0 += per) sl.range.push_back({q0, std::min(L, q0 + per)});
    }
    return sl.range.size() >= 2;
}

// per-device non-blocking streams for the host copies of the pipelined
// paths: 0 host-to-device, 1 device-to-host (created on first use)
static cudaStream_t aux_stream(int which)
{
    static std::mutex mtx;
    static cudaStream_t s[2][64] = {};
    int dev = 0;
    TB_CUDA(cudaGetDevice(&dev));
    TB_CHECK(dev < 64, TB_ERR_ARG, "device index");
    std::lock_guard<std::mutex> lk(mtx);
    if (!s[which][dev]) TB_CUDA(cudaStreamCreateWithFlags(&s[which][dev], cudaStreamNonBlocking));
    return s[which][dev];
}

static cudaStream_t copy_stream() { return aux_stream(0); }
static cudaStream_t copy_back_stream() { return aux_stream(1); }

static void unstage(StagedOp& o, cudaStream_t s)
{
    if (!o.staged) return;
    TB_CUDA(cudaMemcpyAsync(static_cast<char*>(o.host) + o.lo*(i64)o.esz, o.buf.ptr, (size_t)o.n*o.esz,
                            cudaMemcpyDeviceToHost, s));
}

// one contraction on device data (a GEMM view of device-resident operands)
static void contract_device(const GemmView& v, const double* A, const double* B, double* C, double alpha,
                            double beta, int method, double tol, int slices, cudaStream_t st,
                            int& used_slices, double& est_error, int* used_method = nullptr)
{
    if (used_method) *used_method = method;
    if (method >= 2)
    {
        // 2: Ozaki INT8 (slices or moduli, whichever needs less work for tol),
        // 3: Ozaki BF16 slices, 4: one TF32 pass, 5: one BF16 pass, 6: Ozaki
        // INT8 over moduli (scheme II)
        const int kind = method == 2 || method == 6 ? OZ_I8 : method == 4 ? OZ_TF32 : OZ_BF16;
        const int scheme = method == 6 ? 2 : method == 2 && slices > 0 ? 1 : 0;
        OzakiResult r = ozaki_mult(v, A, B, C, alpha, beta, tol, slices, st, kind, method == 4 || method == 5,
                                   scheme);
        used_slices = r.slices;
        est_error = r.est_error;
        if (used_method && kind == OZ_I8) *used_method = r.scheme == 2 ? 6 : 2;
        return;
    }
    const i64 BMt = gemm_f64_tile_m(), BNt = gemm_f64_tile_n(), BKt = gemm_f64_tile_k();
    auto tab = gemm_tables(v, BMt, BNt, BKt, st);
    GemmF64Args a = {};
    a.A = A; a.B = B; a.C = C;
    a.a_m = tab->a_m; a.a_k = tab->a_k; a.b_k = tab->b_k; a.b_n = tab->b_n;
    // pairs of 16-byte copies where the layout gives them (the kernel checks
    // every pair; this only picks the gather code)
    a.pair_a = tab->a_pairs[v.amode] && ((uintptr_t)A & 15) == 0;
    a.pair_b = tab->b_pairs[v.bmode] && ((uintptr_t)B & 15) == 0;
    a.c_m = tab->c_m; a.c_n = tab->c_n; a.a_l = tab->a_l; a.b_l = tab->b_l; a.c_l = tab->c_l;
    a.a_kbs = tab->a_kbs; a.b_kbs = tab->b_kbs;
    a.M = v.m; a.N = v.n; a.K = v.k; a.L = v.l;
    a.alpha = alpha; a.beta = beta;
    a.amode = v.amode; a.bmode = v.bmode;
    a.splits = gemm_f64_choose_splits(v.m, v.n, v.k, v.l, device_sm_count());
    dbuf ws(gemm_f64_workspace_bytes(v.m, v.n, v.l, a.splits), st);
    a.partial = ws.as<double>();
    gemm_f64_launch(a, st);
    used_slices = 0;
    est_error = 1.1e-16*std::sqrt((double)v.k);
}

// the double view of a dcomplex tensor: every dimension with twice the
// stride, plus the real/imaginary dimension (length 2, stride 1) last
struct ComplexParts
{
    std::vector<len_type> len, len2;
    std::vector<stride_type> stride, stride2;
    tblis_tensor whole = {}, re = {}, im = {};
    explicit ComplexParts(const tblis_tensor* X)
    {
        for (unsigned d = 0; d < X->ndim; d++) { len.push_back(X->len[d]); stride.push_back(2*X->stride[d]); }
        len2 = len; stride2 = stride;
        len2.push_back(2); stride2.push_back(1);
        whole.type = TYPE_DOUBLE;
        whole.ndim = X->ndim + 1;
        whole.len = len2.data();
        whole.stride = stride2.data();
        whole.data = X->data;
        re = whole;
        re.ndim = X->ndim;
        re.len = len.data();
        re.stride = stride.data();
        im = re;
    }
    void place(void* dptr)                      // device pointer of element 0 (real part)
    {
        re.data = dptr;
        im.data = static_cast<double*>(dptr) + 1;
    }
};

// C = alpha*op(A)*op(B) + beta*op(C) over dcomplex tensors (op = conjugate
// when the tensor's conj flag is set), as four real contractions per
// product on the FP64 (or configured) path: with A = Ar + i sa Ai and
// B = Br + i sb Bi, A*B = (Ar Br - sa sb Ai Bi) + i (sb Ar Bi + sa Ai Br).
// A complex beta first scales C in place; a complex alpha doubles the
// product terms.
static void mult_complex(const tblis_config* cfg,
                         const tblis_tensor* A, const label_type* idx_A,
                         const tblis_tensor* B, const label_type* idx_B,
                         tblis_tensor* C, const label_type* idx_C,
                         const tblis_b200_opts* opts, tblis_b200_report* report)
{
    ensure_device();
    cudaStream_t st = current_stream();
    const int kernels_before = (int)g_kernel_count.load();
    // alpha = alpha_A*alpha_B (complex), beta = C's scalar (complex)
    const double ar0 = A->scalar.data.z[0], ai0 = A->scalar.data.z[1];
    const double br0 = B->scalar.data.z[0], bi0 = B->scalar.data.z[1];
    const double alr = ar0*br0 - ai0*bi0, ali = ar0*bi0 + ai0*br0;
    const double ber = C->scalar.data.z[0], bei = C->scalar.data.z[1];
    const double sa = A->conj ? -1.0 : 1.0, sb = B->conj ? -1.0 : 1.0;

    ComplexParts pa(A), pb(B), pc(C);
    StagedOp sA, sB, sC;
    const bool read_c = ber != 0.0 || bei != 0.0;
    stage(sC, &pc.whole, read_c, st);
    stage(sA, &pa.whole, true, st);
    stage(sB, &pb.whole, true, st);
    pa.place(sA.dptr); pb.place(sB.dptr); pc.place(sC.dptr);

    auto real_add = [&](double alpha, tblis_tensor X, double beta, tblis_tensor Y)
    {
        X.scalar.type = TYPE_DOUBLE; X.scalar.data.d = alpha;
        Y.scalar.type = TYPE_DOUBLE; Y.scalar.data.d = beta;
        checked([&] { tblis_tensor_add(nullptr, cfg, &X, idx_C, &Y, idx_C); });
    };
    // beta: C <- beta*op(C); conj(C) flips the imaginary part first
    double beta_eff = 1.0;
    const double ci_sign = C->conj ? -1.0 : 1.0;
    if (!read_c)
        beta_eff = 0.0;
    else if (bei == 0.0 && ci_sign == 1.0)
        beta_eff = ber;
    else
    {
        // (ber + i bei)(Cr + i s Ci) = (ber Cr - bei s Ci) + i (ber s Ci + bei Cr)
        std::vector<len_type> dl(pc.len);
        std::vector<stride_type> ds(pc.len.size());
        i64 cnt = 1;
        for (size_t d = 0; d < dl.size(); d++) { ds[d] = cnt; cnt *= dl[d]; }
        dbuf tmp((size_t)std::max<i64>(cnt, 1)*sizeof(double), st);
        tblis_tensor T = pc.re;
        T.data = tmp.ptr;
        T.stride = ds.data();
        real_add(1.0, pc.re, 0.0, T);                         // T = Cr
        real_add(-bei*ci_sign, pc.im, ber, pc.re);            // Cr = ber Cr - bei s Ci
        real_add(bei, T, ber*ci_sign, pc.im);                 // Ci = ber s Ci + bei T
        beta_eff = 1.0;
    }

    // the real products: (X part, Y part, coefficient into Cr, coefficient into Ci)
    struct Term { const tblis_tensor* x; const tblis_tensor* y; double cr, ci; };
    const Term terms[4] = {
        {&pa.re, &pb.re, alr, ali},                       // Ar Br
        {&pa.im, &pb.im, -alr*sa*sb, -ali*sa*sb},         // Ai Bi
        {&pa.re, &pb.im, -ali*sb, alr*sb},                // Ar Bi
        {&pa.im, &pb.re, -ali*sa, alr*sa},                // Ai Br
    };
    bool first_r = true, first_i = true;
    int slices_max = 0;
    double flops = 0, est = 0;
    for (const Term& t : terms)
        for (int part = 0; part < 2; part++)
        {
            const double coef = part == 0 ? t.cr : t.ci;
            if (coef == 0.0) continue;
            bool& first = part == 0 ? first_r : first_i;
            tblis_tensor x = *t.x, y = *t.y, z = part == 0 ? pc.re : pc.im;
            x.scalar.type = y.scalar.type = z.scalar.type = TYPE_DOUBLE;
            x.scalar.data.d = coef;
            y.scalar.data.d = 1.0;
            z.scalar.data.d = first ? beta_eff : 1.0;
            x.conj = y.conj = z.conj = 0;
            tblis_b200_report r = {};
            mult_dispatch(cfg, &x, idx_A, &y, idx_B, &z, idx_C, opts, &r);
            first = false;
            slices_max = std::max(slices_max, r.slices);
            flops += r.flops;
            est += r.est_error;
        }
    // parts that received no product (alpha == 0): beta only
    for (int part = 0; part < 2; part++)
    {
        const bool untouched = part == 0 ? first_r : first_i;
        if (!untouched || beta_eff == 1.0) continue;
        tblis_tensor z = part == 0 ? pc.re : pc.im;
        z.scalar.type = TYPE_DOUBLE; z.scalar.data.d = beta_eff;
        // beta == 0 overwrites (NaN-safe), as the real path does
        tblis_scalar zero;
        zero.type = TYPE_DOUBLE;
        zero.data.d = 0.0;
        if (beta_eff == 0.0) checked([&] { tblis_tensor_set(nullptr, cfg, &zero, &z, idx_C); });
        else checked([&] { tblis_tensor_scale(nullptr, cfg, &z, idx_C); });
    }
    unstage(sC, st);
    if (sA.staged || sB.staged || sC.staged) TB_CUDA(cudaStreamSynchronize(st));
    C->scalar.type = TYPE_DCOMPLEX;
    C->scalar.data.z[0] = 1.0;
    C->scalar.data.z[1] = 0.0;
    C->conj = 0;
    if (report)
    {
        report->method = opts && opts->method ? opts->method : (cfg ? cfg->method : 1);
        report->slices = slices_max;
        report->est_error = est;
        report->flops = flops;
        report->kernels = (int)(g_kernel_count.load() - kernels_before);
    }
}

// The float view of a float or scomplex tensor (a scomplex tensor is a float
// tensor with strides x2 and an inner dim of 2), its dims merged where
// contiguous, as the strided space of the conversions.
struct RealView
{
    Strided s;
    i64 lo = 0, hi = -1;                   // extent in float units
    explicit RealView(const tblis_tensor* X)
    {
        const bool cx = X->type == TYPE_SCOMPLEX;
        std::vector<std::pair<i64, i64>> d;  // (stride, len)
        for (unsigned i = 0; i < X->ndim; i++)
            if (X->len[i] != 1) d.push_back({(cx ? 2 : 1)*X->stride[i], X->len[i]});
        if (cx) d.push_back({1, 2});
        for (auto& x : d) if (x.second == 0) { s.ndim = 1; s.len[0] = 0; s.stride[0] = 1; return; }
        std::sort(d.begin(), d.end(), [](const std::pair<i64, i64>& a, const std::pair<i64, i64>& b)
                  { return std::llabs(a.first) < std::llabs(b.first); });
        std::vector<std::pair<i64, i64>> m;
        for (auto& x : d)
        {
            if (!m.empty() && x.first == m.back().first*m.back().second && x.first > 0) m.back().second *= x.second;
            else m.push_back(x);
        }
        TB_CHECK(m.size() <= (size_t)L1_MAX_DIM, TB_ERR_SIZE, "too many dimensions");
        s.ndim = (int)std::max<size_t>(m.size(), 1);
        s.len[0] = 1; s.stride[0] = 0;
        for (size_t i = 0; i < m.size(); i++) { s.stride[i] = m[i].first; s.len[i] = m[i].second; }
        lo = 0; hi = 0;
        for (auto& x : m)
        {
            if (x.first >= 0) hi += (x.second - 1)*x.first;
            else lo += (x.second - 1)*x.first;
        }
    }
    i64 count() const { return hi - lo + 1; }
};

// float and scomplex contractions: the operands are widened to double /
// dcomplex on the device (same layout, equal offsets), the contraction runs on
// the FP64 or configured kernels, and C is rounded back to float. The result
// is at least as accurate as the reference's float arithmetic
// (src/kernels/3m/gemm.hpp:30-67 in float / scomplex).
static void mult_widened(const tblis_config* cfg,
                         const tblis_tensor* A, const label_type* idx_A,
                         const tblis_tensor* B, const label_type* idx_B,
                         tblis_tensor* C, const label_type* idx_C,
                         const tblis_b200_opts* opts, tblis_b200_report* report)
{
    ensure_device();
    cudaStream_t st = current_stream();
    const bool cx = A->type == TYPE_SCOMPLEX;
    const bool read_c = cx ? (C->scalar.data.c[0] != 0.0f || C->scalar.data.c[1] != 0.0f)
                           : C->scalar.data.s != 0.0f;
    StagedOp sa, sb, sc;
    stage(sc, C, read_c, st, cx ? 8 : 4);
    stage(sa, A, true, st, cx ? 8 : 4);
    stage(sb, B, true, st, cx ? 8 : 4);

    const tblis_tensor* src[3] = {A, B, C};
    StagedOp* sto[3] = {&sa, &sb, &sc};
    tblis_tensor wide[3];
    dbuf wbuf[3];
    RealView* rv[3] = {nullptr, nullptr, nullptr};
    std::vector<std::unique_ptr<RealView>> views;
    for (int t = 0; t < 3; t++)
    {
        const tblis_tensor* X = src[t];
        views.emplace_back(new RealView(X));
        rv[t] = views.back().get();
        wide[t] = *X;
        wide[t].type = cx ? TYPE_DCOMPLEX : TYPE_DOUBLE;
        wide[t].scalar.type = wide[t].type;
        if (cx) { wide[t].scalar.data.z[0] = X->scalar.data.c[0]; wide[t].scalar.data.z[1] = X->scalar.data.c[1]; }
        else wide[t].scalar.data.d = X->scalar.data.s;
        if (!X->data || rv[t]->s.len[0] == 0) continue;
        wbuf[t] = dbuf((size_t)rv[t]->count()*sizeof(double), st);
        double* base = wbuf[t].as<double>() - rv[t]->lo;          // element 0 of the widened tensor
        wide[t].data = base;
        if (t < 2 || read_c)
            l1_convert<float, double>(static_cast<const float*>(sto[t]->dptr), base, rv[t]->s, st);
    }
    mult_dispatch(cfg, &wide[0], idx_A, &wide[1], idx_B, &wide[2], idx_C, opts, report);
    if (C->data && rv[2]->s.len[0] != 0)
        l1_convert<double, float>(static_cast<const double*>(wide[2].data), static_cast<float*>(sc.dptr), rv[2]->s,
                                  st);
    unstage(sc, st);
    if (sa.staged || sb.staged || sc.staged) TB_CUDA(cudaStreamSynchronize(st));
    if (cx) { C->scalar.data.c[0] = 1.0f; C->scalar.data.c[1] = 0.0f; }
    else C->scalar.data.s = 1.0f;
    C->conj = 0;
}

void mult_dispatch(const tblis_config* cfg,
                   const tblis_tensor* A, const label_type* idx_A,
                   const tblis_tensor* B, const label_type* idx_B,
                   tblis_tensor* C, const label_type* idx_C,
                   const tblis_b200_opts* opts, tblis_b200_report* report)
{
    TB_CHECK(A && B && C, TB_ERR_ARG, "null tensor");
    TB_CHECK(A->type == B->type && A->type == C->type, TB_ERR_TYPE, "mult: operand types differ");
    if (A->type == TYPE_DCOMPLEX)
    {
        mult_complex(cfg, A, idx_A, B, idx_B, C, idx_C, opts, report);
        return;
    }
    if (A->type == TYPE_FLOAT || A->type == TYPE_SCOMPLEX)
    {
        mult_widened(cfg, A, idx_A, B, idx_B, C, idx_C, opts, report);
        return;
    }
    TB_CHECK(A->type == TYPE_DOUBLE, TB_ERR_TYPE, "mult: unknown element type");
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
    bool sc_back_done = false;      // C copied back slab by slab already

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
            TB_CHECK(method >= 1 && method <= 6, TB_ERR_ARG, "unknown contraction method");
            stage(sb, B, true, st);
            Slices sl;
            Slabs sb2;
            const bool host_a = A->data && pointer_kind(A->data) == MEM_HOST;
            const bool slabbed = host_a && plan_slabs(A, idx_A, B, idx_B, C, idx_C, sb2);
            const bool sliced = host_a && !slabbed && plan_slices(A, idx_A, B, idx_B, C, idx_C, sl);
            stage(sa, A, !sliced && !slabbed, st);
            int used = 0, ran = method;
            double est = 0;
            if (slabbed)
            {
                // A's slabs in on the copy stream, each slab's contraction on
                // st after its copy, and C's slab back on a second copy
                // stream as soon as it is final
                cudaStream_t cs = copy_stream(), bs = copy_back_stream();
                cudaEvent_t ready;
                TB_CUDA(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
                TB_CUDA(cudaEventRecord(ready, st));
                TB_CUDA(cudaStreamWaitEvent(cs, ready, 0));
                const size_t nsl = sb2.range.size();
                std::vector<cudaEvent_t> in(nsl), done(nsl);
                for (size_t c = 0; c < nsl; c++)
                {
                    const i64 q0 = sb2.range[c].first, nq = sb2.range[c].second - q0;
                    TB_CUDA(cudaMemcpy2DAsync(static_cast<double*>(sa.dptr) + q0*sb2.s_A, (size_t)sb2.pitch_A*8,
                                              static_cast<const double*>(A->data) + q0*sb2.s_A,
                                              (size_t)sb2.pitch_A*8, (size_t)(nq*sb2.s_A*8), (size_t)sb2.rows_A,
                                              cudaMemcpyHostToDevice, cs));
                    TB_CUDA(cudaEventCreateWithFlags(&in[c], cudaEventDisableTiming));
                    TB_CUDA(cudaEventRecord(in[c], cs));
                }
                std::vector<len_type> lenA(A->len, A->len + A->ndim), lenC(C->len, C->len + C->ndim);
                for (size_t c = 0; c < nsl; c++)
                {
                    TB_CUDA(cudaStreamWaitEvent(st, in[c], 0));
                    const i64 q0 = sb2.range[c].first, nq = sb2.range[c].second - q0;
                    tblis_tensor a = *A, b = *B, cc = *C;
                    lenA[sb2.dim_A] = nq;
                    lenC[sb2.dim_C] = nq;
                    a.len = lenA.data();
                    a.data = static_cast<double*>(sa.dptr) + q0*sb2.s_A;
                    b.data = sb.dptr;
                    cc.len = lenC.data();
                    cc.data = static_cast<double*>(sc.dptr) + q0*sb2.s_C;
                    const GemmView vs = gemm_view(mult_groups(&a, idx_A, &b, idx_B, &cc, idx_C));
                    int u = 0;
                    double e = 0;
                    contract_device(vs, static_cast<const double*>(a.data), static_cast<const double*>(b.data),
                                    static_cast<double*>(cc.data), alpha, beta, method, tol, slices, st, u, e,
                                    &ran);
                    used = std::max(used, u);
                    est = std::max(est, e);
                    if (sc.staged)
                    {
                        TB_CUDA(cudaEventCreateWithFlags(&done[c], cudaEventDisableTiming));
                        TB_CUDA(cudaEventRecord(done[c], st));
                        TB_CUDA(cudaStreamWaitEvent(bs, done[c], 0));
                        TB_CUDA(cudaMemcpy2DAsync(static_cast<double*>(C->data) + q0*sb2.s_C, (size_t)sb2.pitch_C*8,
                                                  static_cast<const double*>(sc.dptr) + q0*sb2.s_C,
                                                  (size_t)sb2.pitch_C*8, (size_t)(nq*sb2.s_C*8),
                                                  (size_t)sb2.rows_C, cudaMemcpyDeviceToHost, bs));
                        TB_CUDA(cudaEventDestroy(done[c]));
                    }
                }
                for (auto e : in) cudaEventDestroy(e);
                cudaEventDestroy(ready);
                if (sc.staged)
                {
                    // C went back slab by slab: the copy-back stream finishes it
                    TB_CUDA(cudaStreamSynchronize(bs));
                    sc.staged = false;
                    sc_back_done = true;
                }
            }
            else if (sliced)
            {
                // copies on the copy stream (once the buffer exists), each
                // slice's contraction on st after its copy
                cudaStream_t cs = copy_stream();
                cudaEvent_t ready;
                TB_CUDA(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
                TB_CUDA(cudaEventRecord(ready, st));
                TB_CUDA(cudaStreamWaitEvent(cs, ready, 0));
                std::vector<cudaEvent_t> ev(sl.range.size());
                for (size_t c = 0; c < sl.range.size(); c++)
                {
                    const i64 a = sl.fp[c].first, b = sl.fp[c].second;
                    TB_CUDA(cudaMemcpyAsync(static_cast<double*>(sa.dptr) + a, static_cast<const double*>(A->data) + a,
                                            (size_t)(b - a + 1)*sizeof(double), cudaMemcpyHostToDevice, cs));
                    TB_CUDA(cudaEventCreateWithFlags(&ev[c], cudaEventDisableTiming));
                    TB_CUDA(cudaEventRecord(ev[c], cs));
                }
                std::vector<len_type> lenA(A->len, A->len + A->ndim), lenB(B->len, B->len + B->ndim),
                                      lenC(C->len, C->len + C->ndim);
                const bool over_k = sl.dim_B >= 0;
                // slices that accumulate: each meets tol/n, so their sum meets tol
                const double tol_slice = over_k ? tol/(double)sl.range.size() : tol;
                for (size_t c = 0; c < sl.range.size(); c++)
                {
                    TB_CUDA(cudaStreamWaitEvent(st, ev[c], 0));
                    const i64 q0 = sl.range[c].first, nq = sl.range[c].second - q0;
                    tblis_tensor a = *A, b = *B, cc = *C;
                    lenA[sl.dim_A] = nq;
                    a.len = lenA.data();
                    a.data = static_cast<double*>(sa.dptr) + q0*A->stride[sl.dim_A];
                    b.data = sb.dptr;
                    cc.data = sc.dptr;
                    if (over_k)
                    {
                        lenB[sl.dim_B] = nq;
                        b.len = lenB.data();
                        b.data = static_cast<double*>(sb.dptr) + q0*B->stride[sl.dim_B];
                    }
                    else
                    {
                        lenC[sl.dim_C] = nq;
                        cc.len = lenC.data();
                        cc.data = static_cast<double*>(sc.dptr) + q0*C->stride[sl.dim_C];
                    }
                    const GemmView vs = gemm_view(mult_groups(&a, idx_A, &b, idx_B, &cc, idx_C));
                    int u = 0;
                    double e = 0;
                    contract_device(vs, static_cast<const double*>(a.data), static_cast<const double*>(b.data),
                                    static_cast<double*>(cc.data), alpha, over_k && c > 0 ? 1.0 : beta, method,
                                    tol_slice, slices, st, u, e, &ran);
                    used = std::max(used, u);
                    est = over_k ? est + e : std::max(est, e);
                }
                for (auto e : ev) cudaEventDestroy(e);
                cudaEventDestroy(ready);
            }
            else
            {
                contract_device(v, static_cast<const double*>(sa.dptr), static_cast<const double*>(sb.dptr),
                                static_cast<double*>(sc.dptr), alpha, beta, method, tol, slices, st, used, est,
                                &ran);
            }
            if (report) { report->slices = used; report->est_error = est; report->method = ran; }
        }
    }

    unstage(sc, st);
    if (sa.staged || sb.staged || sc.staged || sc_back_done) TB_CUDA(cudaStreamSynchronize(st));

    C->scalar.data.d = 1.0;
    C->scalar.type = TYPE_DOUBLE;
    C->conj = 0;
    if (report) report->kernels = (int)(g_kernel_count.load() - kernels_before);
}

} // namespace tb
