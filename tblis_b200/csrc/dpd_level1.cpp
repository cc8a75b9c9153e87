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

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>

namespace tb
{

namespace
{

void to_layout(const tblis_b200_dpd_block_table* t, DpdLayout& lay)
{
    TB_CHECK(t, TB_ERR_ARG, "null DPD tensor");
    TB_CHECK(t->type == TYPE_DOUBLE, TB_ERR_TYPE, "DPD: only double is supported");
    TB_CHECK(t->len, TB_ERR_ARG, "DPD: null lengths");
    std::vector<i64> lens(t->len, t->len + (size_t)t->ndim*t->nirrep);
    lay.init_explicit(t->irrep, t->nirrep, t->ndim, lens.data(), t->offset, t->stride);
}

// device view of a DPD tensor's storage; host storage is staged
struct Storage
{
    dbuf buf;
    double* host = nullptr;
    double* dev = nullptr;
    i64 n = 0;
    void init(void* data, i64 total, bool copy_in, cudaStream_t st)
    {
        n = total;
        dev = static_cast<double*>(data);
        if (!data || total == 0 || pointer_kind(data) == MEM_DEVICE) return;
        host = static_cast<double*>(data);
        buf = dbuf((size_t)total*sizeof(double), st);
        dev = buf.as<double>();
        if (copy_in) TB_CUDA(cudaMemcpyAsync(dev, host, (size_t)total*sizeof(double), cudaMemcpyHostToDevice, st));
    }
    void out(cudaStream_t st)
    {
        if (host) TB_CUDA(cudaMemcpyAsync(host, dev, (size_t)n*sizeof(double), cudaMemcpyDeviceToHost, st));
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
    BlockView(const DpdLayout& X, const double* base, const std::vector<unsigned>& irr, double scalar)
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
        t.type = TYPE_DOUBLE;
        t.conj = 0;
        t.scalar.type = TYPE_DOUBLE;
        t.scalar.data.d = scalar;
        t.data = const_cast<double*>(base) + offset;
        t.ndim = X.ndim;
        t.len = len.data();
        t.stride = stride.data();
    }
};

void scale_all(const DpdLayout& X, double* base, double beta, const char* idx, cudaStream_t)
{
    X.for_each_block([&](const std::vector<unsigned>& irr, const std::vector<i64>&, const std::vector<i64>&, i64)
    {
        BlockView b(X, base, irr, beta);
        if (beta == 0.0)
        {
            tblis_scalar z;
            z.type = TYPE_DOUBLE;
            z.data.d = 0.0;
            checked([&] { tblis_tensor_set(nullptr, nullptr, &z, &b.t, idx); });
        }
        else if (beta != 1.0)
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

void dpd_add_dev(double alpha, const DpdLayout& A, const double* a, const std::string& iA, double beta,
                 const DpdLayout& B, double* b, const std::string& iB)
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
    cudaStream_t st = current_stream();
    if (alpha == 0.0 || (Aonly.empty() && Bonly.empty() && A.irrep != B.irrep))
    {
        scale_all(B, b, beta, iB.c_str(), st);
        return;
    }
    const auto pA_AB = positions(AB, iA), pB_AB = positions(AB, iB), pA_only = positions(Aonly, iA);
    std::vector<unsigned> irrA(A.ndim, 0);
    B.for_each_block([&](const std::vector<unsigned>& irrB, const std::vector<i64>&, const std::vector<i64>&, i64)
    {
        BlockView bb(B, b, irrB, beta);
        unsigned x = A.irrep;
        for (size_t i = 0; i < AB.size(); i++) { irrA[pA_AB[i]] = irrB[pB_AB[i]]; x ^= irrB[pB_AB[i]]; }
        double local_beta = beta;
        // the A blocks reaching this B block: the A-only irreps close A's XOR
        for_each_combo(pA_only, x, A.nirrep, irrA, [&]
        {
            BlockView ab(A, a, irrA, alpha);
            if (ab.empty) return;
            bb.t.scalar.data.d = local_beta;
            checked([&] { tblis_tensor_add(nullptr, nullptr, &ab.t, iA.c_str(), &bb.t, iB.c_str()); });
            local_beta = 1.0;
        });
        if (local_beta == 0.0)
        {
            tblis_scalar z;
            z.type = TYPE_DOUBLE;
            z.data.d = 0.0;
            checked([&] { tblis_tensor_set(nullptr, nullptr, &z, &bb.t, iB.c_str()); });
        }
        else if (local_beta != 1.0)
        {
            bb.t.scalar.data.d = local_beta;
            checked([&] { tblis_tensor_scale(nullptr, nullptr, &bb.t, iB.c_str()); });
        }
    });
}

void dpd_add(const tblis_b200_dpd_block_table* A_, const label_type* idx_A,
             tblis_b200_dpd_block_table* B_, const label_type* idx_B)
{
    ensure_device();
    cudaStream_t st = current_stream();
    DpdLayout A, B;
    to_layout(A_, A);
    to_layout(B_, B);
    const double alpha = A_->scalar.data.d, beta = B_->scalar.data.d;
    Storage sa, sb;
    sa.init(A_->data, A.total(), true, st);
    sb.init(B_->data, B.total(), beta != 0.0, st);
    dpd_add_dev(alpha, A, sa.dev, std::string(idx_A, A.ndim), beta, B, sb.dev, std::string(idx_B, B.ndim));
    sb.out(st);
    sb.finish(st);
    sa.finish(st);
    B_->scalar.data.d = 1.0;
    B_->scalar.type = TYPE_DOUBLE;
    B_->conj = 0;
}

double dpd_dot_dev(const DpdLayout& A, const double* a, const std::string& iA,
                   const DpdLayout& B, const double* b, const std::string& iB)
{
    TB_CHECK(A.nirrep == B.nirrep && A.ndim == B.ndim, TB_ERR_ARG, "DPD dot: shapes differ");
    for (char c : iA)
    {
        const size_t p = iB.find(c);
        TB_CHECK(p != std::string::npos, TB_ERR_ARG, "DPD dot: labels must match");
        TB_CHECK(A.len[iA.find(c)] == B.len[p], TB_ERR_ARG, "DPD dot: per-irrep lengths differ");
    }
    double sum = 0.0;
    if (A.irrep != B.irrep) return sum;
    const auto pB = positions(iA, iB);
    std::vector<unsigned> irrB(B.ndim), all(A.ndim), irrA(A.ndim, 0);
    for (unsigned d = 0; d < A.ndim; d++) all[d] = d;
    for_each_combo(all, A.irrep, A.nirrep, irrA, [&]
    {
        for (unsigned d = 0; d < A.ndim; d++) irrB[pB[d]] = irrA[d];
        BlockView ab(A, a, irrA, 1.0), bb(B, b, irrB, 1.0);
        if (ab.empty || bb.empty) return;
        tblis_scalar r;
        checked([&] { tblis_tensor_dot(nullptr, nullptr, &ab.t, iA.c_str(), &bb.t, iB.c_str(), &r); });
        sum += r.data.d;
    });
    return sum;
}

double dpd_dot(const tblis_b200_dpd_block_table* A_, const label_type* idx_A,
               const tblis_b200_dpd_block_table* B_, const label_type* idx_B)
{
    ensure_device();
    cudaStream_t st = current_stream();
    DpdLayout A, B;
    to_layout(A_, A);
    to_layout(B_, B);
    Storage sa, sb;
    sa.init(A_->data, A.total(), true, st);
    sb.init(B_->data, B.total(), true, st);
    const double sum = dpd_dot_dev(A, sa.dev, std::string(idx_A, A.ndim), B, sb.dev, std::string(idx_B, B.ndim));
    sa.finish(st);
    sb.finish(st);
    return A_->scalar.data.d*B_->scalar.data.d*sum;
}

void dpd_reduce_dev(int op, const DpdLayout& A, const double* a, const std::string& iA, double& result, i64& idx)
{
    // reduce_init (src/util/thread.h:160-182)
    using lim = std::numeric_limits<double>;
    double acc = op == REDUCE_MAX ? lim::lowest() : (op == REDUCE_MIN || op == REDUCE_MIN_ABS) ? lim::max() : 0.0;
    i64 at = -1;
    // blocks in the reference's order (src/internal/1t/dpd/reduce.cxx): ties
    // go to the first block reaching the extreme value
    std::vector<unsigned> all(A.ndim), irr(A.ndim, 0);
    for (unsigned d = 0; d < A.ndim; d++) all[d] = d;
    for_each_combo(all, A.irrep, A.nirrep, irr, [&]
    {
        BlockView ab(A, a, irr, 1.0);
        if (ab.empty) return;
        tblis_scalar r;
        len_type bi = 0;
        checked([&] { tblis_tensor_reduce(nullptr, nullptr, (reduce_t)op, &ab.t, iA.c_str(), &r, &bi); });
        const double v = r.data.d;
        const i64 gi = bi + ab.offset;
        switch (op)
        {
            case REDUCE_SUM: case REDUCE_SUM_ABS: acc += v; break;
            case REDUCE_NORM_2: acc += v*v; break;
            case REDUCE_MAX: if (v > acc) { acc = v; at = gi; } break;
            case REDUCE_MAX_ABS: if (std::fabs(v) > std::fabs(acc)) { acc = v; at = gi; } break;
            case REDUCE_MIN: if (v < acc) { acc = v; at = gi; } break;
            case REDUCE_MIN_ABS: if (std::fabs(v) < std::fabs(acc)) { acc = v; at = gi; } break;
            default: throw error(TB_ERR_ARG, "DPD reduce: unknown operation");
        }
    });
    if (op == REDUCE_NORM_2) acc = std::sqrt(acc);
    result = acc;
    idx = at;
}

void dpd_reduce(int op, const tblis_b200_dpd_block_table* A_, const label_type* idx_A, double& result, i64& idx)
{
    ensure_device();
    cudaStream_t st = current_stream();
    DpdLayout A;
    to_layout(A_, A);
    Storage sa;
    sa.init(A_->data, A.total(), true, st);
    dpd_reduce_dev(op, A, sa.dev, std::string(idx_A, A.ndim), result, idx);
    sa.finish(st);
}

// kind: 0 scale (A *= scal), 1 set (A = alpha), 2 shift (A = alpha + scal*A)
void dpd_unary_dev(int kind, double alpha, double scal, const DpdLayout& A, double* a, const std::string& iA)
{
    A.for_each_block([&](const std::vector<unsigned>& irr, const std::vector<i64>&, const std::vector<i64>&, i64)
    {
        BlockView ab(A, a, irr, scal);
        if (ab.empty) return;
        tblis_scalar s;
        s.type = TYPE_DOUBLE;
        s.data.d = alpha;
        if (kind == 0) checked([&] { tblis_tensor_scale(nullptr, nullptr, &ab.t, iA.c_str()); });
        else if (kind == 1) checked([&] { tblis_tensor_set(nullptr, nullptr, &s, &ab.t, iA.c_str()); });
        else checked([&] { tblis_tensor_shift(nullptr, nullptr, &s, &ab.t, iA.c_str()); });
    });
}

void dpd_unary(int kind, double alpha, tblis_b200_dpd_block_table* A_, const label_type* idx_A)
{
    ensure_device();
    cudaStream_t st = current_stream();
    DpdLayout A;
    to_layout(A_, A);
    Storage sa;
    sa.init(A_->data, A.total(), kind != 1, st);
    dpd_unary_dev(kind, alpha, A_->scalar.data.d, A, sa.dev, std::string(idx_A, A.ndim));
    sa.out(st);
    sa.finish(st);
    A_->scalar.data.d = 1.0;
    A_->scalar.type = TYPE_DOUBLE;
}

} // namespace tb

extern "C" {

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
        TB_CHECK(result, tb::TB_ERR_ARG, "null result");
        result->type = TYPE_DOUBLE;
        result->data.d = tb::dpd_dot(A, idx_A, B, idx_B);
    });
}

int tblis_b200_dpd_reduce(reduce_t op, const tblis_b200_dpd_block_table* A, const label_type* idx_A,
                          tblis_scalar* result, len_type* idx)
{
    return tb::guarded([&]
    {
        TB_CHECK(result && idx, tb::TB_ERR_ARG, "null result");
        double r = 0;
        tb::i64 i = -1;
        tb::dpd_reduce((int)op, A, idx_A, r, i);
        result->type = TYPE_DOUBLE;
        result->data.d = r;
        *idx = i;
    });
}

int tblis_b200_dpd_scale(tblis_b200_dpd_block_table* A, const label_type* idx_A)
{
    return tb::guarded([&] { tb::dpd_unary(0, 0.0, A, idx_A); });
}

int tblis_b200_dpd_set(const tblis_scalar* alpha, tblis_b200_dpd_block_table* A, const label_type* idx_A)
{
    return tb::guarded([&]
    {
        TB_CHECK(alpha, tb::TB_ERR_ARG, "null alpha");
        tb::dpd_unary(1, alpha->data.d, A, idx_A);
    });
}

int tblis_b200_dpd_shift(const tblis_scalar* alpha, tblis_b200_dpd_block_table* A, const label_type* idx_A)
{
    return tb::guarded([&]
    {
        TB_CHECK(alpha, tb::TB_ERR_ARG, "null alpha");
        tb::dpd_unary(2, alpha->data.d, A, idx_A);
    });
}

}
