// dpd_level1.cpp -- add, dot, reduce, scale, set and shift over DPD tensors
// (the operations either side of a DPD contraction in a solver iteration).
//
// Each operation walks the stored blocks in the reference's block order
// (src/internal/1t/dpd/util.hpp:14-68, 204-218) and applies the dense GPU
// kernel of the same operation to each block in place: the block is a
// strided view of the DPD storage (offset and strides from the layout), so
// nothing is copied. Semantics follow src/iface/1t/{add,dot,reduce,scale,
// set,shift}.cxx for dpd_varray_view and src/internal/1t/dpd/*.cxx:
//  * add: B = alpha*A + beta*B with A-only labels traced and B-only labels
//    replicated, per stored B block over the A blocks whose irreps agree on
//    the shared labels (trace_block / replicate_block); a B block no A block
//    reaches is scaled by beta (set when beta == 0); alpha == 0 or, without
//    A-only and B-only labels, A.irrep != B.irrep scales all of B;
//  * dot: sum over blocks of the blockwise dots (0 when the irreps differ);
//  * reduce: blockwise reductions combined in block order, idx = offset of
//    the extreme element from the tensor's data (first block wins ties);
//  * scale / set / shift: every stored block.
#include "common.hpp"
#include "dpd.hpp"
#include "level1.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>

namespace tb
{

size_t elem_size(int type)
{
    switch (type)
    {
        case TYPE_FLOAT: return 4;
        case TYPE_DOUBLE: return 8;
        case TYPE_SCOMPLEX: return 8;
        case TYPE_DCOMPLEX: return 16;
    }
    throw error(TB_ERR_TYPE, "unknown element type");
}

zd scalar_get(const tblis_scalar& s)
{
    switch (s.type)
    {
        case TYPE_FLOAT: return zd(s.data.s, 0.0);
        case TYPE_DOUBLE: return zd(s.data.d, 0.0);
        case TYPE_SCOMPLEX: return zd(s.data.c[0], s.data.c[1]);
        case TYPE_DCOMPLEX: return zd(s.data.z[0], s.data.z[1]);
    }
    throw error(TB_ERR_TYPE, "unknown scalar type");
}

void scalar_put(tblis_scalar& s, int type, zd v)
{
    s.type = (type_t)type;
    switch (type)
    {
        case TYPE_FLOAT: s.data.s = (float)v.real(); return;
        case TYPE_DOUBLE: s.data.d = v.real(); return;
        case TYPE_SCOMPLEX: s.data.c[0] = (float)v.real(); s.data.c[1] = (float)v.imag(); return;
        case TYPE_DCOMPLEX: s.data.z[0] = v.real(); s.data.z[1] = v.imag(); return;
    }
    throw error(TB_ERR_TYPE, "unknown scalar type");
}

dbuf dpd_widen(const void* src, i64 total, bool cx, cudaStream_t st)
{
    const i64 n = total*(cx ? 2 : 1);
    dbuf w((size_t)std::max<i64>(n, 1)*sizeof(double), st);
    if (n > 0 && src)
    {
        Strided s;
        s.ndim = 1; s.len[0] = n; s.stride[0] = 1;
        l1_convert<float, double>(static_cast<const float*>(src), w.as<double>(), s, st);
    }
    return w;
}

void dpd_narrow_blocks(const DpdLayout& X, bool cx, const double* src, float* dst, cudaStream_t st)
{
    if (!dst) return;
    X.for_each_block([&](const std::vector<unsigned>&, const std::vector<i64>& bl, const std::vector<i64>& bs,
                         i64 off)
    {
        // a complex block in float units: strides x2 and an inner dim of 2
        TB_CHECK(X.ndim + (cx ? 1 : 0) <= (unsigned)L1_MAX_DIM, TB_ERR_SIZE, "DPD: too many dimensions");
        Strided s;
        s.ndim = 0;
        if (cx) { s.len[0] = 2; s.stride[0] = 1; s.ndim = 1; }
        for (unsigned d = 0; d < X.ndim; d++)
        {
            s.len[s.ndim] = bl[d];
            s.stride[s.ndim] = bs[d]*(cx ? 2 : 1);
            s.ndim++;
        }
        const i64 o = off*(cx ? 2 : 1);
        l1_convert<double, float>(src + o, dst + o, s, st);
    });
}

namespace
{

void to_layout(const tblis_b200_dpd_block_table* t, DpdLayout& lay)
{
    TB_CHECK(t, TB_ERR_ARG, "null DPD tensor");
    elem_size(t->type);
    TB_CHECK(t->len, TB_ERR_ARG, "DPD: null lengths");
    std::vector<i64> lens(t->len, t->len + (size_t)t->ndim*t->nirrep);
    lay.init_explicit(t->irrep, t->nirrep, t->ndim, lens.data(), t->offset, t->stride);
}

// device view of a DPD tensor's storage; host storage is staged
struct Storage
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
    void finish(cudaStream_t st)
    {
        if (host) TB_CUDA(cudaStreamSynchronize(st));
    }
};

// irrep combinations of the listed dims with a given XOR, in the order of
// assign_irreps (src/internal/1t/dpd/util.hpp:204-218): the first dim closes
// the XOR, the others run as an odometer with the second fastest
template <typename F>
void for_each_combo(const std::vector<unsigned>& dims, unsigned target, unsigned nirrep,
                    std::vector<unsigned>& irr, F&& f)
{
    if (dims.empty())
    {
        if (target == 0) f();
        return;
    }
    i64 n = 1;
    for (size_t i = 1; i < dims.size(); i++) n *= nirrep;
    for (i64 b = 0; b < n; b++)
    {
        unsigned x = target;
        i64 t = b;
        for (size_t i = 1; i < dims.size(); i++)
        {
            irr[dims[i]] = (unsigned)(t % nirrep);
            t /= nirrep;
            x ^= irr[dims[i]];
        }
        irr[dims[0]] = x;
        f();
    }
}

// the block of X at `irr` as a dense tblis_tensor over the device storage
struct BlockView
{
    std::vector<len_type> len;
    std::vector<stride_type> stride;
    tblis_tensor t = {};
    i64 offset = 0;
    bool empty = true;
    BlockView(int type, const DpdLayout& X, const void* base, const std::vector<unsigned>& irr, zd scalar,
              bool conj = false)
    {
        len.resize(X.ndim);
        stride.resize(X.ndim);
        i64 ext = 1;
        for (unsigned d = 0; d < X.ndim; d++) ext *= X.len[d][irr[d]];
        empty = ext == 0;
        if (empty) return;
        std::vector<i64> bl(X.ndim), bs(X.ndim);
        X.block(irr.data(), bl.data(), bs.data(), offset);
        for (unsigned d = 0; d < X.ndim; d++) { len[d] = bl[d]; stride[d] = bs[d]; }
        t.type = (type_t)type;
        t.conj = conj ? 1 : 0;
        scalar_put(t.scalar, type, scalar);
        t.data = const_cast<char*>(static_cast<const char*>(base)) + offset*(i64)elem_size(type);
        t.ndim = X.ndim;
        t.len = len.data();
        t.stride = stride.data();
    }
};

// B = beta*op(B) on every stored block (set when beta == 0)
void scale_all(int type, const DpdLayout& X, void* base, zd beta, bool conj, const char* idx)
{
    X.for_each_block([&](const std::vector<unsigned>& irr, const std::vector<i64>&, const std::vector<i64>&, i64)
    {
        BlockView b(type, X, base, irr, beta, conj);
        if (beta == 0.0)
        {
            tblis_scalar z;
            scalar_put(z, type, 0.0);
            checked([&] { tblis_tensor_set(nullptr, nullptr, &z, &b.t, idx); });
        }
        else if (beta != 1.0 || (conj && is_complex_type(type)))
            checked([&] { tblis_tensor_scale(nullptr, nullptr, &b.t, idx); });
    });
}

std::vector<unsigned> positions(const std::string& labels, const std::string& of)
{
    std::vector<unsigned> p;
    for (char c : labels) p.push_back((unsigned)of.find(c));
    return p;
}

} // namespace

void dpd_add_dev_t(int type, zd alpha, const DpdLayout& A, const void* a, const std::string& iA, zd beta,
                   const DpdLayout& B, void* b, const std::string& iB, bool conj_a, bool conj_b)
{
    TB_CHECK(A.nirrep == B.nirrep, TB_ERR_ARG, "DPD add: nirrep differs");
    for (const std::string* s : {&iA, &iB})
        for (size_t i = 0; i < s->size(); i++)
            for (size_t j = 0; j < i; j++)
                TB_CHECK((*s)[i] != (*s)[j], TB_ERR_ARG, "DPD add: repeated label in one tensor");
    std::string AB, Aonly, Bonly;
    for (char c : iA) (iB.find(c) != std::string::npos ? AB : Aonly).push_back(c);
    for (char c : iB) if (iA.find(c) == std::string::npos) Bonly.push_back(c);
    TB_CHECK(Aonly.empty() || Bonly.empty(), TB_ERR_ARG, "DPD add: labels only in A and only in B at once");
    TB_CHECK(!AB.empty(), TB_ERR_ARG, "DPD add: no shared label");
    for (char c : AB)
        TB_CHECK(A.len[iA.find(c)] == B.len[iB.find(c)], TB_ERR_ARG, "DPD add: per-irrep lengths differ");
    const bool cx = is_complex_type(type);
    conj_a = conj_a && cx;
    conj_b = conj_b && cx;
    if (alpha == 0.0 || (Aonly.empty() && Bonly.empty() && A.irrep != B.irrep))
    {
        scale_all(type, B, b, beta, conj_b, iB.c_str());
        return;
    }
    const auto pA_AB = positions(AB, iA), pB_AB = positions(AB, iB), pA_only = positions(Aonly, iA);
    std::vector<unsigned> irrA(A.ndim, 0);
    B.for_each_block([&](const std::vector<unsigned>& irrB, const std::vector<i64>&, const std::vector<i64>&, i64)
    {
        BlockView bb(type, B, b, irrB, beta, conj_b);
        unsigned x = A.irrep;
        for (size_t i = 0; i < AB.size(); i++) { irrA[pA_AB[i]] = irrB[pB_AB[i]]; x ^= irrB[pB_AB[i]]; }
        // beta and B's conjugation apply once, with the first A block
        zd local_beta = beta;
        bool local_conj = conj_b;
        // the A blocks reaching this B block: the A-only irreps close A's XOR
        for_each_combo(pA_only, x, A.nirrep, irrA, [&]
        {
            BlockView ab(type, A, a, irrA, alpha, conj_a);
            if (ab.empty) return;
            scalar_put(bb.t.scalar, type, local_beta);
            bb.t.conj = local_conj ? 1 : 0;
            checked([&] { tblis_tensor_add(nullptr, nullptr, &ab.t, iA.c_str(), &bb.t, iB.c_str()); });
            local_beta = 1.0;
            local_conj = false;
        });
        if (local_beta == 0.0)
        {
            tblis_scalar z;
            scalar_put(z, type, 0.0);
            checked([&] { tblis_tensor_set(nullptr, nullptr, &z, &bb.t, iB.c_str()); });
        }
        else if (local_beta != 1.0 || local_conj)
        {
            scalar_put(bb.t.scalar, type, local_beta);
            bb.t.conj = local_conj ? 1 : 0;
            checked([&] { tblis_tensor_scale(nullptr, nullptr, &bb.t, iB.c_str()); });
        }
    });
}

zd dpd_dot_dev_t(int type, const DpdLayout& A, const void* a, const std::string& iA,
                 const DpdLayout& B, const void* b, const std::string& iB, bool conj_a, bool conj_b)
{
    TB_CHECK(A.nirrep == B.nirrep && A.ndim == B.ndim, TB_ERR_ARG, "DPD dot: shapes differ");
    for (char c : iA)
    {
        const size_t p = iB.find(c);
        TB_CHECK(p != std::string::npos, TB_ERR_ARG, "DPD dot: labels must match");
        TB_CHECK(A.len[iA.find(c)] == B.len[p], TB_ERR_ARG, "DPD dot: per-irrep lengths differ");
    }
    zd sum = 0.0;
    if (A.irrep != B.irrep) return sum;
    const auto pB = positions(iA, iB);
    std::vector<unsigned> irrB(B.ndim), all(A.ndim), irrA(A.ndim, 0);
    for (unsigned d = 0; d < A.ndim; d++) all[d] = d;
    for_each_combo(all, A.irrep, A.nirrep, irrA, [&]
    {
        for (unsigned d = 0; d < A.ndim; d++) irrB[pB[d]] = irrA[d];
        BlockView ab(type, A, a, irrA, 1.0, conj_a), bb(type, B, b, irrB, 1.0, conj_b);
        if (ab.empty || bb.empty) return;
        tblis_scalar r;
        r.type = (type_t)type;
        checked([&] { tblis_tensor_dot(nullptr, nullptr, &ab.t, iA.c_str(), &bb.t, iB.c_str(), &r); });
        sum += scalar_get(r);
    });
    return sum;
}

void dpd_reduce_dev_t(int type, int op, const DpdLayout& A, const void* a, const std::string& iA, zd& result,
                      i64& idx)
{
    // reduce_init (src/util/thread.h:160-182); complex values compare by
    // their real parts, as the reference's operators do
    using lim = std::numeric_limits<double>;
    const double big = type == TYPE_FLOAT || type == TYPE_SCOMPLEX ? (double)std::numeric_limits<float>::max()
                                                                   : lim::max();
    zd acc = op == REDUCE_MAX ? zd(-big) : (op == REDUCE_MIN || op == REDUCE_MIN_ABS) ? zd(big) : zd(0.0);
    i64 at = -1;
    // blocks in the reference's order (src/internal/1t/dpd/reduce.cxx): ties
    // go to the first block reaching the extreme value
    std::vector<unsigned> all(A.ndim), irr(A.ndim, 0);
    for (unsigned d = 0; d < A.ndim; d++) all[d] = d;
    for_each_combo(all, A.irrep, A.nirrep, irr, [&]
    {
        BlockView ab(type, A, a, irr, 1.0);
        if (ab.empty) return;
        tblis_scalar r;
        r.type = (type_t)type;
        len_type bi = 0;
        checked([&] { tblis_tensor_reduce(nullptr, nullptr, (reduce_t)op, &ab.t, iA.c_str(), &r, &bi); });
        const zd v = scalar_get(r);
        const i64 gi = bi + ab.offset;
        switch (op)
        {
            case REDUCE_SUM: case REDUCE_SUM_ABS: acc += v; break;
            case REDUCE_NORM_2: acc += v.real()*v.real(); break;
            case REDUCE_MAX: if (v.real() > acc.real()) { acc = v; at = gi; } break;
            case REDUCE_MAX_ABS: if (std::fabs(v.real()) > std::fabs(acc.real())) { acc = v; at = gi; } break;
            case REDUCE_MIN: if (v.real() < acc.real()) { acc = v; at = gi; } break;
            case REDUCE_MIN_ABS: if (std::fabs(v.real()) < std::fabs(acc.real())) { acc = v; at = gi; } break;
            default: throw error(TB_ERR_ARG, "DPD reduce: unknown operation");
        }
    });
    if (op == REDUCE_NORM_2) acc = std::sqrt(acc.real());
    result = acc;
    idx = at;
}

void dpd_unary_dev_t(int type, int kind, zd alpha, zd scal, const DpdLayout& A, void* a, const std::string& iA,
                     bool conj)
{
    conj = conj && is_complex_type(type);
    A.for_each_block([&](const std::vector<unsigned>& irr, const std::vector<i64>&, const std::vector<i64>&, i64)
    {
        BlockView ab(type, A, a, irr, scal, conj);
        if (ab.empty) return;
        tblis_scalar s;
        scalar_put(s, type, alpha);
        if (kind == 0) checked([&] { tblis_tensor_scale(nullptr, nullptr, &ab.t, iA.c_str()); });
        else if (kind == 1) checked([&] { tblis_tensor_set(nullptr, nullptr, &s, &ab.t, iA.c_str()); });
        else checked([&] { tblis_tensor_shift(nullptr, nullptr, &s, &ab.t, iA.c_str()); });
    });
}

namespace
{

void dpd_add(const tblis_b200_dpd_block_table* A_, const label_type* idx_A,
             tblis_b200_dpd_block_table* B_, const label_type* idx_B)
{
    ensure_device();
    cudaStream_t st = current_stream();
    DpdLayout A, B;
    to_layout(A_, A);
    to_layout(B_, B);
    TB_CHECK(A_->type == B_->type, TB_ERR_TYPE, "DPD add: operand types differ");
    const int type = A_->type;
    const zd alpha = scalar_get(A_->scalar), beta = scalar_get(B_->scalar);
    Storage sa, sb;
    sa.init(A_->data, A.total(), elem_size(type), true, st);
    sb.init(B_->data, B.total(), elem_size(type), true, st);
    dpd_add_dev_t(type, alpha, A, sa.dev, std::string(idx_A, A.ndim), beta, B, sb.dev, std::string(idx_B, B.ndim),
                  A_->conj != 0, B_->conj != 0);
    sb.out(st);
    sb.finish(st);
    sa.finish(st);
    scalar_put(B_->scalar, type, 1.0);
    B_->conj = 0;
}

zd dpd_dot(const tblis_b200_dpd_block_table* A_, const label_type* idx_A,
           const tblis_b200_dpd_block_table* B_, const label_type* idx_B)
{
    ensure_device();
    cudaStream_t st = current_stream();
    DpdLayout A, B;
    to_layout(A_, A);
    to_layout(B_, B);
    TB_CHECK(A_->type == B_->type, TB_ERR_TYPE, "DPD dot: operand types differ");
    const int type = A_->type;
    Storage sa, sb;
    sa.init(A_->data, A.total(), elem_size(type), true, st);
    sb.init(B_->data, B.total(), elem_size(type), true, st);
    const zd sum = dpd_dot_dev_t(type, A, sa.dev, std::string(idx_A, A.ndim), B, sb.dev, std::string(idx_B, B.ndim),
                                 A_->conj != 0, B_->conj != 0);
    sa.finish(st);
    sb.finish(st);
    return scalar_get(A_->scalar)*scalar_get(B_->scalar)*sum;
}

void dpd_reduce(int op, const tblis_b200_dpd_block_table* A_, const label_type* idx_A, zd& result, i64& idx)
{
    ensure_device();
    cudaStream_t st = current_stream();
    DpdLayout A;
    to_layout(A_, A);
    Storage sa;
    sa.init(A_->data, A.total(), elem_size(A_->type), true, st);
    dpd_reduce_dev_t(A_->type, op, A, sa.dev, std::string(idx_A, A.ndim), result, idx);
    sa.finish(st);
}

// kind 0: A = scal*op(A); 1: A = alpha; 2: A = alpha + scal*op(A)
void dpd_unary(int kind, const tblis_scalar* alpha, tblis_b200_dpd_block_table* A_, const label_type* idx_A)
{
    ensure_device();
    cudaStream_t st = current_stream();
    DpdLayout A;
    to_layout(A_, A);
    const int type = A_->type;
    if (alpha) TB_CHECK(alpha->type == type, TB_ERR_TYPE, "DPD set/shift: scalar and tensor types differ");
    Storage sa;
    sa.init(A_->data, A.total(), elem_size(type), kind != 1, st);
    dpd_unary_dev_t(type, kind, alpha ? scalar_get(*alpha) : zd(0.0), scalar_get(A_->scalar), A, sa.dev,
                    std::string(idx_A, A.ndim), A_->conj != 0);
    sa.out(st);
    sa.finish(st);
    scalar_put(A_->scalar, type, 1.0);
    A_->conj = 0;
}

// The dense form of a DPD tensor and back (block_to_full / full_to_block,
// src/internal/1t/dpd/util.hpp:70-133): dimension d of the dense tensor F has
// the sum of A's lengths over the irreps, irrep x occupying
// [sum of the lengths of irreps < x, + length of x); block_to_full sets all
// of F to zero and copies every stored block of A into its region, and
// full_to_block copies every region back into A's block. Scalars and
// conjugation flags do not apply (plain copies, as in the reference).
void dpd_full_copy(tblis_b200_dpd_block_table* A_, tblis_tensor* F, bool to_full)
{
    ensure_device();
    cudaStream_t st = current_stream();
    TB_CHECK(A_ && F, TB_ERR_ARG, "null tensor");
    DpdLayout A;
    to_layout(A_, A);
    const int type = A_->type;
    TB_CHECK(F->type == type, TB_ERR_TYPE, "DPD dense form: element types differ");
    TB_CHECK(F->ndim == A.ndim, TB_ERR_ARG, "DPD dense form: dimensions differ");
    TB_CHECK(A.ndim <= 26, TB_ERR_SIZE, "DPD dense form: too many dimensions");
    std::vector<std::vector<i64>> off(A.ndim, std::vector<i64>(A.nirrep, 0));
    for (unsigned d = 0; d < A.ndim; d++)
    {
        i64 o = 0;
        for (unsigned x = 0; x < A.nirrep; x++) { off[d][x] = o; o += A.len[d][x]; }
        TB_CHECK(F->len[d] == o, TB_ERR_ARG, "DPD dense form: a dense length is not the sum of the irrep lengths");
    }
    std::string idx;
    for (unsigned d = 0; d < A.ndim; d++) idx.push_back((char)('a' + d));
    const size_t esz = elem_size(type);
    Storage sa;
    sa.init(A_->data, A.total(), esz, true, st);       // read, or kept where no block is stored
    // F is staged by the dense entry points themselves when it is on the host
    tblis_tensor f = *F;
    if (to_full)
    {
        tblis_scalar z;
        scalar_put(z, type, 0.0);
        checked([&] { tblis_tensor_set(nullptr, nullptr, &z, &f, idx.c_str()); });
    }
    std::vector<len_type> flen(A.ndim);
    A.for_each_block([&](const std::vector<unsigned>& irr, const std::vector<i64>&, const std::vector<i64>&, i64)
    {
        BlockView blk(type, A, sa.dev, irr, to_full ? zd(1.0) : zd(0.0));
        if (blk.empty) return;
        tblis_tensor sub = *F;
        char* base = static_cast<char*>(F->data);
        for (unsigned d = 0; d < A.ndim; d++) base += off[d][irr[d]]*F->stride[d]*(i64)esz;
        for (unsigned d = 0; d < A.ndim; d++) flen[d] = blk.len[d];
        sub.data = base;
        sub.len = flen.data();
        sub.conj = 0;
        scalar_put(sub.scalar, type, to_full ? 0.0 : 1.0);
        if (to_full) checked([&] { tblis_tensor_add(nullptr, nullptr, &blk.t, idx.c_str(), &sub, idx.c_str()); });
        else checked([&] { tblis_tensor_add(nullptr, nullptr, &sub, idx.c_str(), &blk.t, idx.c_str()); });
    });
    if (!to_full) sa.out(st);
    sa.finish(st);
}

} // namespace

} // namespace tb

extern "C" {

int tblis_b200_dpd_block_to_full(const tblis_b200_dpd_block_table* A, tblis_tensor* F)
{
    return tb::guarded([&] { tb::dpd_full_copy(const_cast<tblis_b200_dpd_block_table*>(A), F, true); });
}

int tblis_b200_dpd_full_to_block(const tblis_tensor* F, tblis_b200_dpd_block_table* A)
{
    return tb::guarded([&] { tb::dpd_full_copy(A, const_cast<tblis_tensor*>(F), false); });
}


int tblis_b200_dpd_add(const tblis_b200_dpd_block_table* A, const label_type* idx_A,
                       tblis_b200_dpd_block_table* B, const label_type* idx_B)
{
    return tb::guarded([&] { tb::dpd_add(A, idx_A, B, idx_B); });
}

int tblis_b200_dpd_dot(const tblis_b200_dpd_block_table* A, const label_type* idx_A,
                       const tblis_b200_dpd_block_table* B, const label_type* idx_B, tblis_scalar* result)
{
    return tb::guarded([&]
    {
        TB_CHECK(result && A, tb::TB_ERR_ARG, "null argument");
        tb::scalar_put(*result, A->type, tb::dpd_dot(A, idx_A, B, idx_B));
    });
}

int tblis_b200_dpd_reduce(reduce_t op, const tblis_b200_dpd_block_table* A, const label_type* idx_A,
                          tblis_scalar* result, len_type* idx)
{
    return tb::guarded([&]
    {
        TB_CHECK(result && idx && A, tb::TB_ERR_ARG, "null argument");
        tb::zd r = 0.0;
        tb::i64 i = -1;
        tb::dpd_reduce((int)op, A, idx_A, r, i);
        tb::scalar_put(*result, A->type, r);
        *idx = i;
    });
}

int tblis_b200_dpd_scale(tblis_b200_dpd_block_table* A, const label_type* idx_A)
{
    return tb::guarded([&] { tb::dpd_unary(0, nullptr, A, idx_A); });
}

int tblis_b200_dpd_set(const tblis_scalar* alpha, tblis_b200_dpd_block_table* A, const label_type* idx_A)
{
    return tb::guarded([&]
    {
        TB_CHECK(alpha, tb::TB_ERR_ARG, "null alpha");
        tb::dpd_unary(1, alpha, A, idx_A);
    });
}

int tblis_b200_dpd_shift(const tblis_scalar* alpha, tblis_b200_dpd_block_table* A, const label_type* idx_A)
{
    return tb::guarded([&]
    {
        TB_CHECK(alpha, tb::TB_ERR_ARG, "null alpha");
        tb::dpd_unary(2, alpha, A, idx_A);
    });
}

}
