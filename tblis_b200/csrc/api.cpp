// api.cpp -- the TBLIS C ABI on the GPU.
//
// Entry points restate the reference's interface layer
// (src/iface/3t/mult.cxx:24-165, src/iface/1t/{add,dot,reduce,scale,set,shift}.cxx):
// label handling, the alpha/beta special cases and the side effects on the
// output tensor's scalar and conj fields are kept; the arithmetic goes to the
// device kernels. Paths cited are relative to the TBLIS tree.
#include "common.hpp"
#include "planner.hpp"
#include "gemm_f64.hpp"
#include "level1.hpp"
#include "mult.hpp"
#include "ozaki.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>

namespace tb
{

std::atomic<int64_t> g_kernel_count{0};
std::atomic<bool> g_ktimer_on{false};

namespace
{
struct KtRecord { std::string name; cudaEvent_t a, b; };
std::mutex g_kt_mtx;
std::vector<KtRecord> g_kt;
}

void ktimer_push(const char* name, cudaEvent_t a, cudaEvent_t b)
{
    std::lock_guard<std::mutex> lk(g_kt_mtx);
    g_kt.push_back({name, a, b});
}

namespace
{
thread_local int t_err_code = 0;
thread_local std::string t_err_msg;
thread_local cudaStream_t t_stream = 0;
unsigned g_num_threads = 1;

tblis_config_s g_cfgs[] = {
    {"b200_fp64", 1, 1e-12},
    {"b200_ozaki_i8", 2, 1e-12},
    {"b200_ozaki_bf16", 3, 1e-12},
    {"b200_tf32", 4, 1e-12},
    {"b200_bf16", 5, 1e-12},
    {"b200_ozaki_crt", 6, 1e-12},
};
}

void set_last_error(int code, const char* msg)
{
    t_err_code = code;
    t_err_msg = msg ? msg : "";
    const char* ab = getenv("TBLIS_B200_ABORT_ON_ERROR");
    if (ab && ab[0] == '1')
    {
        fprintf(stderr, "tblis_b200: %s\n", t_err_msg.c_str());
        abort();
    }
}

cudaStream_t current_stream() { return t_stream; }

void ensure_device()
{
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0)
    {
        cudaGetLastError();
        throw error(TB_ERR_NODEV, "no CUDA device: libtblis_b200 computes on the GPU only");
    }
    // keep freed workspace in this process's default pool instead of handing
    // it back to the driver at every synchronisation (a process-local
    // attribute of the pool, not a device setting)
    static std::mutex mtx;
    static bool done[64] = {false};
    int dev = 0;
    TB_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(mtx);
    if (dev < 64 && !done[dev])
    {
        cudaMemPool_t pool;
        TB_CUDA(cudaDeviceGetDefaultMemPool(&pool, dev));
        uint64_t thr = UINT64_MAX;
        TB_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
        done[dev] = true;
    }
}

mem_kind pointer_kind(const void* p)
{
    cudaPointerAttributes at;
    cudaError_t e = cudaPointerGetAttributes(&at, p);
    if (e != cudaSuccess) { cudaGetLastError(); return MEM_HOST; }
    if (at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged) return MEM_DEVICE;
    return MEM_HOST;
}

// ---- host staging -------------------------------------------------------------------------

// Device view of one operand. Host data is staged: the touched extent is
// copied in (and out for outputs) around the call.
struct Staged
{
    void* dptr = nullptr;       // device pointer to element 0 of the tensor
    dbuf buf;
    void* host = nullptr;
    i64 min_off = 0, nelem = 0;
    size_t esize = 8;
    bool staged = false;

    void init(const tblis_tensor* t, size_t es, bool copy_in, cudaStream_t s)
    {
        esize = es;
        if (!t->data) { dptr = nullptr; return; }
        if (pointer_kind(t->data) == MEM_DEVICE) { dptr = t->data; return; }
        i64 lo, hi;
        tensor_extent(t->ndim, t->len, t->stride, lo, hi);
        if (hi < lo) { dptr = t->data; return; }   // empty tensor: never dereferenced
        staged = true;
        host = t->data;
        min_off = lo;
        nelem = hi - lo + 1;
        buf = dbuf((size_t)nelem*es, s);
        char* hbase = static_cast<char*>(host) + lo*(i64)es;
        // an extent with gaps is copied in even for an output: copy_out
        // writes the whole extent back, and the gaps must come back unchanged
        i64 count = 1;
        for (unsigned d = 0; d < t->ndim; d++) count *= t->len[d];
        if (copy_in || count != nelem)
            TB_CUDA(cudaMemcpyAsync(buf.ptr, hbase, (size_t)nelem*es, cudaMemcpyHostToDevice, s));
        dptr = buf.as<char>() - lo*(i64)es;
    }

    void copy_out(cudaStream_t s)
    {
        if (!staged) return;
        char* hbase = static_cast<char*>(host) + min_off*(i64)esize;
        TB_CUDA(cudaMemcpyAsync(hbase, buf.ptr, (size_t)nelem*esize, cudaMemcpyDeviceToHost, s));
    }
};

static size_t type_size(int type)
{
    switch (type)
    {
        case TYPE_FLOAT: return 4;
        case TYPE_DOUBLE: return 8;
        case TYPE_SCOMPLEX: return 8;
        case TYPE_DCOMPLEX: return 16;
    }
    throw error(TB_ERR_TYPE, "unknown tensor type");
}

static void fill_strided(Strided& s, const ivec& len, const ivec& stride)
{
    TB_CHECK(len.size() <= (size_t)L1_MAX_DIM, TB_ERR_SIZE, "too many dimensions");
    s.ndim = (int)len.size();
    for (size_t i = 0; i < len.size(); i++) { s.len[i] = len[i]; s.stride[i] = stride[i]; }
}

// diagonal + (empty => one unit dim) + fold over one tensor (the reference's
// scale/set/shift/reduce preamble, e.g. src/iface/1t/scale.cxx:23-37)
static Strided one_tensor_dims(const tblis_tensor* A, const label_type* idx)
{
    TB_CHECK(A, TB_ERR_ARG, "null tensor");
    ivec len, stride;
    std::string lab;
    diagonal(A->ndim, A->len, A->stride, idx ? idx : "", len, stride, lab);
    if (lab.empty()) { len.push_back(1); stride.push_back(0); lab.push_back(0); }
    fold(len, lab, {&stride});
    Strided s;
    fill_strided(s, len, stride);
    return s;
}

template <typename T> static T scalar_of(const tblis_scalar& s);
template <> double scalar_of<double>(const tblis_scalar& s) { return s.data.d; }
template <> float scalar_of<float>(const tblis_scalar& s) { return s.data.s; }
template <> cplx<float> scalar_of<cplx<float>>(const tblis_scalar& s) { return {s.data.c[0], s.data.c[1]}; }
template <> cplx<double> scalar_of<cplx<double>>(const tblis_scalar& s) { return {s.data.z[0], s.data.z[1]}; }
template <typename T> static void set_scalar(tblis_scalar& s, T v);
template <> void set_scalar<double>(tblis_scalar& s, double v) { s.data.d = v; s.type = TYPE_DOUBLE; }
template <> void set_scalar<float>(tblis_scalar& s, float v) { s.data.s = v; s.type = TYPE_FLOAT; }
template <> void set_scalar<cplx<float>>(tblis_scalar& s, cplx<float> v)
{
    s.data.c[0] = v.re; s.data.c[1] = v.im; s.type = TYPE_SCOMPLEX;
}
template <> void set_scalar<cplx<double>>(tblis_scalar& s, cplx<double> v)
{
    s.data.z[0] = v.re; s.data.z[1] = v.im; s.type = TYPE_DCOMPLEX;
}

// dispatch on the element type of a level-1 call
template <typename F>
static void with_type(int type, F&& f)
{
    switch (type)
    {
        case TYPE_FLOAT: f(float()); break;
        case TYPE_DOUBLE: f(double()); break;
        case TYPE_SCOMPLEX: f(cplx<float>(0.0f)); break;
        case TYPE_DCOMPLEX: f(cplx<double>(0.0)); break;
        default: throw error(TB_ERR_TYPE, "unknown tensor type");
    }
}

// |x| of a scalar (std::abs)
template <typename T> static T abs_scalar(T x) { return x < T(0) ? -x : x; }
template <typename R> static cplx<R> abs_scalar(cplx<R> x) { return cplx<R>(std::hypot(x.re, x.im)); }

static void finish_host_call(std::vector<Staged*> outs, bool any_staged, cudaStream_t s)
{
    for (Staged* o : outs) o->copy_out(s);
    if (any_staged) TB_CUDA(cudaStreamSynchronize(s));
}

// ---- set / scale / shift ---------------------------------------------------------------------

template <typename T>
static void do_unary(int op, const tblis_scalar* val, tblis_tensor* A, const label_type* idx)
{
    ensure_device();
    cudaStream_t st = current_stream();
    Strided s = one_tensor_dims(A, idx);
    Staged sa;
    const T alpha = scalar_of<T>(A->scalar);
    const bool needs_in = !(op == 0 || (op != 0 && alpha == T(0)));
    // a conjugated complex tensor is rewritten even with a unit scalar
    const bool cj = is_cplx<T>::value && A->conj;
    sa.init(A, sizeof(T), needs_in, st);
    T* d = static_cast<T*>(sa.dptr);
    if (op == 0)                                   // set (src/iface/1t/set.cxx:39-46)
        l1_set<T>(d, s, scalar_of<T>(*val), st);
    else if (op == 1)                              // scale (src/iface/1t/scale.cxx:39-56)
    {
        if (alpha == T(0)) l1_set<T>(d, s, T(0), st);
        else if (alpha != T(1) || cj) l1_scale<T>(d, s, alpha, st, cj);
    }
    else                                           // shift (src/iface/1t/shift.cxx:39-70)
    {
        const T sh = scalar_of<T>(*val);
        if (alpha == T(0)) l1_set<T>(d, s, T(0), st);
        else if (sh == T(0)) { if (alpha != T(1) || cj) l1_scale<T>(d, s, alpha, st, cj); }
        else l1_shift<T>(d, s, sh, alpha, st, cj);
    }
    finish_host_call({&sa}, sa.staged, st);
    set_scalar<T>(A->scalar, T(1));
    A->conj = 0;
}

// ---- add ---------------------------------------------------------------------------------------

template <typename T>
static void do_add(const tblis_tensor* A, const label_type* idx_A_, tblis_tensor* B, const label_type* idx_B_)
{
    ensure_device();
    cudaStream_t st = current_stream();
    ivec lA, lB, sA, sB;
    std::string iA, iB;
    diagonal(A->ndim, A->len, A->stride, idx_A_ ? idx_A_ : "", lA, sA, iA);
    diagonal(B->ndim, B->len, B->stride, idx_B_ ? idx_B_ : "", lB, sB, iB);
    if (iA.empty() || iB.empty())
    {
        lA.push_back(1); lB.push_back(1); sA.push_back(0); sB.push_back(0);
        char f = free_idx(iA + iB);
        iA.push_back(f); iB.push_back(f);
    }
    std::string iab, iao, ibo;
    for (char c : iA) if (iB.find(c) != std::string::npos) iab.push_back(c);
    std::sort(iab.begin(), iab.end());
    for (char c : iA) if (iab.find(c) == std::string::npos) iao.push_back(c);
    for (char c : iB) if (iab.find(c) == std::string::npos) ibo.push_back(c);
    std::sort(iao.begin(), iao.end());
    std::sort(ibo.begin(), ibo.end());
    TB_CHECK(iao.empty() || ibo.empty(), TB_ERR_ARG, "add: labels only in A and only in B at once");

    auto sel = [](const ivec& v, const std::string& lab, const std::string& m)
    { ivec r; for (char c : m) r.push_back(v[lab.find(c)]); return r; };
    ivec len_ab = sel(lA, iA, iab), sa_ab = sel(sA, iA, iab), sb_ab = sel(sB, iB, iab);
    TB_CHECK(len_ab == sel(lB, iB, iab), TB_ERR_ARG, "add: mismatched lengths");
    ivec len_ao = sel(lA, iA, iao), s_ao = sel(sA, iA, iao);
    ivec len_bo = sel(lB, iB, ibo), s_bo = sel(sB, iB, ibo);
    fold(len_ab, iab, {&sa_ab, &sb_ab});
    fold(len_ao, iao, {&s_ao});
    fold(len_bo, ibo, {&s_bo});

    const T alpha = scalar_of<T>(A->scalar), beta = scalar_of<T>(B->scalar);
    const bool cja = is_cplx<T>::value && A->conj, cjb = is_cplx<T>::value && B->conj;
    Staged sta, stb;
    stb.init(B, sizeof(T), beta != T(0), st);
    if (alpha == T(0))
    {
        // src/iface/1t/add.cxx:76-90: set or scale B (conjugated B: rewritten)
        Strided s;
        ivec l = len_bo, str = s_bo;
        l.insert(l.end(), len_ab.begin(), len_ab.end());
        str.insert(str.end(), sb_ab.begin(), sb_ab.end());
        fill_strided(s, l, str);
        if (beta == T(0)) l1_set<T>(static_cast<T*>(stb.dptr), s, T(0), st);
        else if (beta != T(1) || cjb) l1_scale<T>(static_cast<T*>(stb.dptr), s, beta, st, cjb);
    }
    else
    {
        sta.init(A, sizeof(T), true, st);
        Strided2 ab;
        TB_CHECK(len_ab.size() <= (size_t)L1_MAX_DIM, TB_ERR_SIZE, "too many dimensions");
        ab.ndim = (int)len_ab.size();
        for (size_t i = 0; i < len_ab.size(); i++) { ab.len[i] = len_ab[i]; ab.sa[i] = sa_ab[i]; ab.sb[i] = sb_ab[i]; }
        Strided ao, bo;
        fill_strided(ao, len_ao, s_ao);
        fill_strided(bo, len_bo, s_bo);
        i64 n_ao = 1;
        for (i64 x : len_ao) n_ao *= x;
        if (n_ao == 0)
        {
            // src/internal/1t/dense/add.cxx:45-49: empty trace => B = beta*B
            Strided sb;
            fill_strided(sb, len_bo, s_bo);
            if (beta == T(0)) l1_set<T>(static_cast<T*>(stb.dptr), sb, T(0), st);
            else l1_scale<T>(static_cast<T*>(stb.dptr), sb, beta, st, cjb);
        }
        else
            l1_add<T>(static_cast<const T*>(sta.dptr), static_cast<T*>(stb.dptr), ab, ao, bo, alpha, beta, st,
                      cja, cjb);
    }
    finish_host_call({&stb}, sta.staged || stb.staged, st);
    set_scalar<T>(B->scalar, T(1));
    B->conj = 0;
}

// ---- dot / reduce --------------------------------------------------------------------------------

template <typename T>
static void do_dot(const tblis_tensor* A, const label_type* idx_A_, const tblis_tensor* B,
                   const label_type* idx_B_, tblis_scalar* result)
{
    ensure_device();
    cudaStream_t st = current_stream();
    ivec lA, lB, sA, sB;
    std::string iA, iB;
    diagonal(A->ndim, A->len, A->stride, idx_A_ ? idx_A_ : "", lA, sA, iA);
    diagonal(B->ndim, B->len, B->stride, idx_B_ ? idx_B_ : "", lB, sB, iB);
    if (iA.empty() || iB.empty())
    {
        lA.push_back(1); lB.push_back(1); sA.push_back(0); sB.push_back(0);
        char f = free_idx(iA + iB);
        iA.push_back(f); iB.push_back(f);
    }
    std::string iab;
    for (char c : iA) if (iB.find(c) != std::string::npos) iab.push_back(c);
    std::sort(iab.begin(), iab.end());
    TB_CHECK(iab.size() == iA.size() && iab.size() == iB.size(), TB_ERR_ARG,
             "dot: every label must appear in both tensors");
    ivec len, sa, sb;
    for (char c : iab)
    {
        len.push_back(lA[iA.find(c)]);
        TB_CHECK(len.back() == lB[iB.find(c)], TB_ERR_ARG, "dot: mismatched lengths");
        sa.push_back(sA[iA.find(c)]);
        sb.push_back(sB[iB.find(c)]);
    }
    fold(len, iab, {&sa, &sb});
    Strided2 s;
    TB_CHECK(len.size() <= (size_t)L1_MAX_DIM, TB_ERR_SIZE, "too many dimensions");
    s.ndim = (int)len.size();
    for (size_t i = 0; i < len.size(); i++) { s.len[i] = len[i]; s.sa[i] = sa[i]; s.sb[i] = sb[i]; }
    Staged sta, stb;
    sta.init(A, sizeof(T), true, st);
    stb.init(B, sizeof(T), true, st);
    dbuf out(sizeof(T), st);
    l1_dot<T>(static_cast<const T*>(sta.dptr), static_cast<const T*>(stb.dptr), s, out.as<T>(), st,
              is_cplx<T>::value && A->conj, is_cplx<T>::value && B->conj);
    T v;
    TB_CUDA(cudaMemcpyAsync(&v, out.ptr, sizeof(T), cudaMemcpyDeviceToHost, st));
    TB_CUDA(cudaStreamSynchronize(st));
    set_scalar<T>(*result, v*scalar_of<T>(A->scalar)*scalar_of<T>(B->scalar));
}

template <typename T>
static void do_reduce(int op, const tblis_tensor* A, const label_type* idx_A, tblis_scalar* result,
                      len_type* idx)
{
    ensure_device();
    cudaStream_t st = current_stream();
    Strided s = one_tensor_dims(A, idx_A);
    const T alpha = scalar_of<T>(A->scalar);
    // src/iface/1t/reduce.cxx:39-43: a negative scalar swaps MIN and MAX (a
    // complex scalar: a negative real part)
    if (alpha < T(0))
    {
        if (op == REDUCE_MIN) op = REDUCE_MAX;
        else if (op == REDUCE_MAX) op = REDUCE_MIN;
    }
    Staged sa;
    sa.init(A, sizeof(T), true, st);
    dbuf out(16 + sizeof(i64), st);
    T* dv = out.as<T>();
    i64* di = reinterpret_cast<i64*>(out.as<char>() + 16);
    l1_reduce<T>(op, static_cast<const T*>(sa.dptr), s, dv, di, st);
    T v; i64 id;
    TB_CUDA(cudaMemcpyAsync(&v, dv, sizeof(T), cudaMemcpyDeviceToHost, st));
    TB_CUDA(cudaMemcpyAsync(&id, di, sizeof(i64), cudaMemcpyDeviceToHost, st));
    TB_CUDA(cudaStreamSynchronize(st));
    // src/iface/1t/reduce.cxx:52-65: conjugate, then apply the scalar
    if (is_cplx<T>::value && A->conj) v = cj(v, true);
    if (op == REDUCE_SUM) v *= alpha;
    else if (op == REDUCE_SUM_ABS || op == REDUCE_NORM_2) v *= abs_scalar(alpha);
    set_scalar<T>(*result, v);
    if (idx) *idx = id;
}

} // namespace tb

using namespace tb;

// =====================================================================================
// C ABI
// =====================================================================================

extern "C" {

void tblis_tensor_mult(const tblis_comm*, const tblis_config* cfg,
                       const tblis_tensor* A, const label_type* idx_A,
                       const tblis_tensor* B, const label_type* idx_B,
                             tblis_tensor* C, const label_type* idx_C)
{
    guarded([&] { mult_dispatch(cfg, A, idx_A, B, idx_B, C, idx_C, nullptr, nullptr); });
}

int tblis_b200_tensor_mult_ex(const tblis_config* cfg,
                              const tblis_tensor* A, const label_type* idx_A,
                              const tblis_tensor* B, const label_type* idx_B,
                                    tblis_tensor* C, const label_type* idx_C,
                              const tblis_b200_opts* opts, tblis_b200_report* report)
{
    return guarded([&] { mult_dispatch(cfg, A, idx_A, B, idx_B, C, idx_C, opts, report); });
}

void tblis_tensor_add(const tblis_comm*, const tblis_config*,
                      const tblis_tensor* A, const label_type* idx_A,
                            tblis_tensor* B, const label_type* idx_B)
{
    guarded([&]
    {
        TB_CHECK(A && B, TB_ERR_ARG, "null tensor");
        TB_CHECK(A->type == B->type, TB_ERR_TYPE, "add: operand types differ");
        with_type(A->type, [&](auto t) { do_add<decltype(t)>(A, idx_A, B, idx_B); });
    });
}

void tblis_tensor_dot(const tblis_comm*, const tblis_config*,
                      const tblis_tensor* A, const label_type* idx_A,
                      const tblis_tensor* B, const label_type* idx_B,
                      tblis_scalar* result)
{
    guarded([&]
    {
        TB_CHECK(A && B && result, TB_ERR_ARG, "null argument");
        TB_CHECK(A->type == B->type, TB_ERR_TYPE, "dot: operand types differ");
        with_type(A->type, [&](auto t) { do_dot<decltype(t)>(A, idx_A, B, idx_B, result); });
    });
}

void tblis_tensor_reduce(const tblis_comm*, const tblis_config*, reduce_t op,
                         const tblis_tensor* A, const label_type* idx_A,
                         tblis_scalar* result, len_type* idx)
{
    guarded([&]
    {
        TB_CHECK(A && result, TB_ERR_ARG, "null argument");
        with_type(A->type, [&](auto t) { do_reduce<decltype(t)>((int)op, A, idx_A, result, idx); });
    });
}

void tblis_tensor_scale(const tblis_comm*, const tblis_config*, tblis_tensor* A, const label_type* idx_A)
{
    guarded([&]
    {
        TB_CHECK(A, TB_ERR_ARG, "null tensor");
        with_type(A->type, [&](auto t) { do_unary<decltype(t)>(1, nullptr, A, idx_A); });
    });
}

void tblis_tensor_set(const tblis_comm*, const tblis_config*, const tblis_scalar* alpha,
                      tblis_tensor* A, const label_type* idx_A)
{
    guarded([&]
    {
        TB_CHECK(A && alpha, TB_ERR_ARG, "null argument");
        TB_CHECK(alpha->type == A->type, TB_ERR_TYPE, "set: scalar and tensor types differ");
        with_type(A->type, [&](auto t) { do_unary<decltype(t)>(0, alpha, A, idx_A); });
    });
}

void tblis_tensor_shift(const tblis_comm*, const tblis_config*, const tblis_scalar* alpha,
                        tblis_tensor* A, const label_type* idx_A)
{
    guarded([&]
    {
        TB_CHECK(A && alpha, TB_ERR_ARG, "null argument");
        TB_CHECK(alpha->type == A->type, TB_ERR_TYPE, "shift: scalar and tensor types differ");
        with_type(A->type, [&](auto t) { do_unary<decltype(t)>(2, alpha, A, idx_A); });
    });
}

// src/util/basic_types.cxx:197-247
void tblis_init_scalar_s(tblis_scalar* s, float value) { s->data.s = value; s->type = TYPE_FLOAT; }
void tblis_init_scalar_d(tblis_scalar* s, double value) { s->data.d = value; s->type = TYPE_DOUBLE; }

static void init_tensor(tblis_tensor* t, type_t type, unsigned ndim, len_type* len, void* data,
                        stride_type* stride)
{
    t->type = type;
    t->conj = 0;
    t->data = data;
    t->ndim = ndim;
    t->len = len;
    t->stride = stride;
}

void tblis_init_tensor_scaled_s(tblis_tensor* t, float scalar, unsigned ndim, len_type* len,
                                float* data, stride_type* stride)
{ init_tensor(t, TYPE_FLOAT, ndim, len, data, stride); tblis_init_scalar_s(&t->scalar, scalar); }
void tblis_init_tensor_scaled_d(tblis_tensor* t, double scalar, unsigned ndim, len_type* len,
                                double* data, stride_type* stride)
{ init_tensor(t, TYPE_DOUBLE, ndim, len, data, stride); tblis_init_scalar_d(&t->scalar, scalar); }
void tblis_init_tensor_s(tblis_tensor* t, unsigned ndim, len_type* len, float* data, stride_type* stride)
{ tblis_init_tensor_scaled_s(t, 1.0f, ndim, len, data, stride); }
void tblis_init_tensor_d(tblis_tensor* t, unsigned ndim, len_type* len, double* data, stride_type* stride)
{ tblis_init_tensor_scaled_d(t, 1.0, ndim, len, data, stride); }

unsigned tblis_get_num_threads(void) { return g_num_threads; }
void tblis_set_num_threads(unsigned n) { g_num_threads = n ? n : 1; }

const tblis_config* tblis_get_config(const char* name)
{
    if (!name) return nullptr;
    for (auto& c : g_cfgs)
        if (!strcmp(name, c.name)) return &c;
    return nullptr;
}

void tblis_b200_config_set_tolerance(tblis_config* cfg, double tol)
{
    if (cfg) cfg->tolerance = tol > 0 ? tol : 1e-12;
}

double tblis_b200_config_get_tolerance(const tblis_config* cfg) { return cfg ? cfg->tolerance : 1e-12; }

int tblis_b200_last_error(void) { return t_err_code; }
const char* tblis_b200_last_error_string(void) { return t_err_msg.c_str(); }
void tblis_b200_clear_error(void) { t_err_code = 0; t_err_msg.clear(); }

void tblis_b200_set_stream(void* stream) { t_stream = static_cast<cudaStream_t>(stream); }
void* tblis_b200_get_stream(void) { return t_stream; }
void tblis_b200_synchronize(void)
{
    guarded([&]
    {
        TB_CUDA(cudaStreamSynchronize(t_stream));
        TB_CHECK(ozaki_error_flag() == 0, TB_ERR_TIMEOUT, "an Ozaki kernel gave up a bounded wait");
        TB_CHECK(gemm_f64_error_flag() == 0, TB_ERR_TIMEOUT, "a grouped FP64 kernel gave up a bounded wait");
    });
}

int tblis_b200_ozaki_inject_wait_timeout(int step, double wait_seconds)
{
    return guarded([&] { ensure_device(); ozaki_inject_wait_timeout(step, wait_seconds); });
}

int tblis_b200_grouped_inject_wait_timeout(int step, double wait_seconds)
{
    return guarded([&] { ensure_device(); gemm_f64_inject_wait_timeout(step, wait_seconds); });
}

void tblis_b200_fill_block_scatter(unsigned ndim, const len_type* len, const stride_type* stride,
                                   len_type BS, stride_type off, stride_type size,
                                   stride_type* scat, stride_type* bs, int pack_3d)
{
    guarded([&]
    {
        ivec l(len, len + ndim), s(stride, stride + ndim);
        std::vector<i64> sc(size > 0 ? size : 1), b(size > 0 ? size : 1, 0);
        for (i64 i = 0; i < size; i++) b[i] = bs[i];
        fill_block_scatter(l, s, BS, off, size, sc.data(), b.data(), pack_3d != 0);
        for (i64 i = 0; i < size; i++) { scat[i] = sc[i]; bs[i] = b[i]; }
    });
}

int tblis_b200_mult_groups(const tblis_tensor* A, const label_type* idx_A,
                           const tblis_tensor* B, const label_type* idx_B,
                           const tblis_tensor* C, const label_type* idx_C,
                           char* idx_AB, char* idx_AC, char* idx_BC, char* idx_ABC,
                           int64_t* mnkl)
{
    return guarded([&]
    {
        MultGroups g = mult_groups(A, idx_A, B, idx_B, C, idx_C);
        GemmView v = gemm_view(g);
        strcpy(idx_AB, v.idxK.c_str());
        strcpy(idx_AC, v.idxM.c_str());
        strcpy(idx_BC, v.idxN.c_str());
        strcpy(idx_ABC, v.idxL.c_str());
        mnkl[0] = v.m; mnkl[1] = v.n; mnkl[2] = v.k; mnkl[3] = v.l;
    });
}

int64_t tblis_b200_kernel_count(void) { return g_kernel_count.load(); }

int tblis_b200_kernel_timer(int enable)
{
    std::lock_guard<std::mutex> lk(g_kt_mtx);
    for (auto& r : g_kt) { cudaEventDestroy(r.a); cudaEventDestroy(r.b); }
    g_kt.clear();
    g_ktimer_on.store(enable != 0);
    return 0;
}

int tblis_b200_kernel_timer_read(const char* name, double* total_ms, int64_t* launches)
{
    return guarded([&]
    {
        TB_CHECK(name && total_ms && launches, TB_ERR_ARG, "null argument");
        std::lock_guard<std::mutex> lk(g_kt_mtx);
        double t = 0.0;
        int64_t n = 0;
        for (auto& r : g_kt)
        {
            if (r.name != name) continue;
            TB_CUDA(cudaEventSynchronize(r.b));
            float ms = 0.f;
            TB_CUDA(cudaEventElapsedTime(&ms, r.a, r.b));
            t += ms;
            n++;
        }
        *total_ms = t;
        *launches = n;
    });
}

} // extern "C"
