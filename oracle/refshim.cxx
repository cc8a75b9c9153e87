/*
 * refshim.cxx -- TEST INFRASTRUCTURE ONLY.
 *
 * A thin C-linkage shim over the TBLIS reference headers, compiled by
 * oracle/Makefile into oracle/_ref/librefshim.so next to the reference
 * library. It exposes internals that the reference's C ABI does not: the
 * block-scatter vector builder (src/matrix/block_scatter_matrix.hpp:249-258),
 * the MArray DPD block layout (src/external/marray/include/dpd_marray_base.hpp)
 * and the C++ DPD and indexed-DPD contraction entry points
 * (src/iface/3t/mult.cxx:170-298, 412-541), so
 * that the tests can pin the oracle restatement and the product's planner
 * against the reference bit for bit.
 */
#include "util/basic_types.h"
#include "util/tensor.hpp"
#include "matrix/block_scatter_matrix.hpp"
#include "iface/3t/mult.h"
#include "iface/1t/add.h"
#include "iface/1t/shift.h"
#include "iface/1t/set.h"
#include "iface/1t/scale.h"
#include "iface/1t/reduce.h"
#include "iface/1t/dot.h"
#include "internal/3t/dpd/mult.hpp"
#include "internal/3t/dense/mult.hpp"

using namespace tblis;

namespace
{
struct bsm_access : block_scatter_matrix<double>
{
    using block_scatter_matrix<double>::fill_block_scatter;
};

std::vector<std::vector<len_type>> lens_of(unsigned ndim, unsigned nirrep, const len_type* lens)
{
    std::vector<std::vector<len_type>> len(ndim, std::vector<len_type>(nirrep));
    for (unsigned i = 0; i < ndim; i++)
        for (unsigned j = 0; j < nirrep; j++) len[i][j] = lens[i*nirrep+j];
    return len;
}

/*
 * The reference's C++ DPD operations for any of its element types (float,
 * double, scomplex, dcomplex: type_t codes 0-3); scalars and results are
 * passed by pointer to a value of the element type.
 */
template <typename T>
int dpd_mult_t(unsigned nirrep, const void* alpha, unsigned irrep_A, unsigned ndim_A, const len_type* lens_A,
               const void* data_A, const char* idx_A, unsigned irrep_B, unsigned ndim_B, const len_type* lens_B,
               const void* data_B, const char* idx_B, const void* beta, unsigned irrep_C, unsigned ndim_C,
               const len_type* lens_C, void* data_C, const char* idx_C)
{
    MArray::dpd_varray_view<const T> A(irrep_A, nirrep, lens_of(ndim_A, nirrep, lens_A), (const T*)data_A);
    MArray::dpd_varray_view<const T> B(irrep_B, nirrep, lens_of(ndim_B, nirrep, lens_B), (const T*)data_B);
    MArray::dpd_varray_view<T> C(irrep_C, nirrep, lens_of(ndim_C, nirrep, lens_C), (T*)data_C);
    tblis::mult<T>(*(const T*)alpha, A, idx_A, B, idx_B, *(const T*)beta, C, idx_C);
    return 0;
}

template <typename T>
int dpd_level1_t(int op, unsigned nirrep, const void* alpha, const void* beta,
                 unsigned irrep_A, unsigned ndim_A, const len_type* lens_A, const void* data_A, const char* idx_A,
                 unsigned irrep_B, unsigned ndim_B, const len_type* lens_B, void* data_B, const char* idx_B,
                 void* result, long* idx)
{
    /* op: 0 add (B = alpha*A + beta*B), 1 dot (result), 2 scale (A *= alpha),
     * 3 set (A = alpha), 4 shift (A = alpha + beta*A), 10 + r: reduce r */
    MArray::dpd_varray_view<T> A(irrep_A, nirrep, lens_of(ndim_A, nirrep, lens_A), (T*)data_A);
    if (op == 0)
    {
        MArray::dpd_varray_view<T> B(irrep_B, nirrep, lens_of(ndim_B, nirrep, lens_B), (T*)data_B);
        tblis::add<T>(*(const T*)alpha, A, idx_A, *(const T*)beta, B, idx_B);
    }
    else if (op == 1)
    {
        MArray::dpd_varray_view<const T> B(irrep_B, nirrep, lens_of(ndim_B, nirrep, lens_B), (const T*)data_B);
        *(T*)result = tblis::dot<T>(A, idx_A, B, idx_B);
    }
    else if (op == 2) tblis::scale<T>(*(const T*)alpha, A, idx_A);
    else if (op == 3) tblis::set<T>(*(const T*)alpha, A, idx_A);
    else if (op == 4) tblis::shift<T>(*(const T*)alpha, *(const T*)beta, A, idx_A);
    else
    {
        auto r = tblis::reduce<T>((tblis::reduce_t)(op - 10), MArray::dpd_varray_view<const T>(A), idx_A);
        *(T*)result = r.first;
        *idx = r.second;
    }
    return 0;
}
}

extern "C"
{

int refshim_version() { return 1; }

/* Selects the reference's dense contraction implementation
 * (src/internal/3t/dense/mult.cxx:24): 0 = BLIS_BASED (default),
 * 2 = REFERENCE (mult_ref, the one that applies conjugation flags).
 * Returns the previous value. */
int refshim_set_dense_impl(int impl)
{
    const int old = (int)tblis::internal::impl;
    tblis::internal::impl = impl == 2 ? tblis::internal::REFERENCE : tblis::internal::BLIS_BASED;
    return old;
}

/*
 * Selects the reference's DPD contraction implementation
 * (src/internal/3t/dpd/mult.cxx:26): 0 = BLIS (its default block path),
 * 1 = BLOCKED, 2 = FULL (dense round trip). Returns the previous value.
 */
int refshim_set_dpd_impl(int impl)
{
    const int old = tblis::internal::dpd_impl == tblis::internal::FULL ? 2 :
                    tblis::internal::dpd_impl == tblis::internal::BLOCKED ? 1 : 0;
    tblis::internal::dpd_impl = impl == 2 ? tblis::internal::FULL : impl == 1 ? tblis::internal::BLOCKED
                                                                            : tblis::internal::BLIS;
    return old;
}

void refshim_fill_block_scatter(unsigned ndim, const len_type* len, const stride_type* stride,
                                len_type BS, stride_type off, stride_type size,
                                stride_type* scat, stride_type* bs, int pack_3d)
{
    len_vector l(len, len+ndim);
    stride_vector s(stride, stride+ndim);
    bsm_access::fill_block_scatter(l, s, BS, off, size, scat, bs, pack_3d != 0);
}

/*
 * DPD layout of a dense-stored DPD tensor: for every block (irreps tuple with
 * XOR equal to `irrep`, enumerated with the first dimension's irrep fastest),
 * writes the block's data offset from the tensor base and its strides.
 * lens is [ndim][nirrep]. layout: MArray dpd_layout enum value.
 * Returns the total number of elements, or -1.
 */
long refshim_dpd_layout(unsigned irrep, unsigned nirrep, unsigned ndim, const len_type* lens,
                        int layout, long* block_offsets, long* block_strides, long max_blocks)
{
    std::vector<std::vector<len_type>> len(ndim, std::vector<len_type>(nirrep));
    for (unsigned i = 0; i < ndim; i++)
        for (unsigned j = 0; j < nirrep; j++)
            len[i][j] = lens[i*nirrep+j];

    MArray::dpd_varray<double> A(irrep, nirrep, len, 0.0, (MArray::dpd_layout)layout);

    long nblock = 0;
    MArray::irrep_vector irreps(ndim);
    long total = 1;
    for (unsigned i = 0; i+1 < ndim; i++) total *= nirrep;
    for (long b = 0; b < total && nblock < max_blocks; b++)
    {
        long t = b;
        unsigned x = irrep;
        for (unsigned i = 1; i < ndim; i++)
        {
            irreps[i] = t % nirrep;
            t /= nirrep;
            x ^= irreps[i];
        }
        irreps[0] = x;
        auto v = A(irreps);
        block_offsets[nblock] = v.data() - A.data();
        for (unsigned i = 0; i < ndim; i++) block_strides[nblock*ndim+i] = v.stride(i);
        nblock++;
    }
    return (long)A.size();
}

/*
 * C = alpha*A*B + beta*C through the reference's own C++ DPD entry point
 * (tblis::mult over dpd_varray_view, src/iface/3t/mult.cxx:170-298). The three
 * tensors are given by their lens ([ndim][nirrep]), irrep and dense storage
 * (default MArray layout). Returns 0 on success.
 */
int refshim_dpd_mult(unsigned nirrep,
                     double alpha, unsigned irrep_A, unsigned ndim_A, const len_type* lens_A,
                     const double* data_A, const char* idx_A,
                     unsigned irrep_B, unsigned ndim_B, const len_type* lens_B,
                     const double* data_B, const char* idx_B,
                     double beta, unsigned irrep_C, unsigned ndim_C, const len_type* lens_C,
                     double* data_C, const char* idx_C)
{
    auto mk = [&](unsigned ndim, const len_type* lens)
    {
        std::vector<std::vector<len_type>> len(ndim, std::vector<len_type>(nirrep));
        for (unsigned i = 0; i < ndim; i++)
            for (unsigned j = 0; j < nirrep; j++)
                len[i][j] = lens[i*nirrep+j];
        return len;
    };

    MArray::dpd_varray_view<const double> A(irrep_A, nirrep, mk(ndim_A, lens_A), data_A);
    MArray::dpd_varray_view<const double> B(irrep_B, nirrep, mk(ndim_B, lens_B), data_B);
    MArray::dpd_varray_view<double> C(irrep_C, nirrep, mk(ndim_C, lens_C), data_C);

    tblis::mult<double>(alpha, A, idx_A, B, idx_B, beta, C, idx_C);
    return 0;
}

/*
 * The reference's DPD level-1 operations (tblis::add / dot / reduce / scale /
 * set / shift over dpd_varray_view, src/iface/1t/*.cxx) on default-layout
 * storage. kind for the unary entry: 0 scale (A *= alpha), 1 set (A = alpha),
 * 2 shift (A = alpha + beta*A). Return 0 on success.
 */
static std::vector<std::vector<len_type>> dpd_lens(unsigned ndim, unsigned nirrep, const len_type* lens)
{
    std::vector<std::vector<len_type>> len(ndim, std::vector<len_type>(nirrep));
    for (unsigned i = 0; i < ndim; i++)
        for (unsigned j = 0; j < nirrep; j++) len[i][j] = lens[i*nirrep+j];
    return len;
}

int refshim_dpd_add(unsigned nirrep, double alpha, unsigned irrep_A, unsigned ndim_A, const len_type* lens_A,
                    const double* data_A, const char* idx_A, double beta, unsigned irrep_B, unsigned ndim_B,
                    const len_type* lens_B, double* data_B, const char* idx_B)
{
    MArray::dpd_varray_view<const double> A(irrep_A, nirrep, dpd_lens(ndim_A, nirrep, lens_A), data_A);
    MArray::dpd_varray_view<double> B(irrep_B, nirrep, dpd_lens(ndim_B, nirrep, lens_B), data_B);
    tblis::add<double>(alpha, A, idx_A, beta, B, idx_B);
    return 0;
}

double refshim_dpd_dot(unsigned nirrep, unsigned irrep_A, unsigned ndim_A, const len_type* lens_A,
                       const double* data_A, const char* idx_A, unsigned irrep_B, unsigned ndim_B,
                       const len_type* lens_B, const double* data_B, const char* idx_B)
{
    MArray::dpd_varray_view<const double> A(irrep_A, nirrep, dpd_lens(ndim_A, nirrep, lens_A), data_A);
    MArray::dpd_varray_view<const double> B(irrep_B, nirrep, dpd_lens(ndim_B, nirrep, lens_B), data_B);
    return tblis::dot<double>(A, idx_A, B, idx_B);
}

int refshim_dpd_reduce(int op, unsigned nirrep, unsigned irrep_A, unsigned ndim_A, const len_type* lens_A,
                       const double* data_A, const char* idx_A, double* result, long* idx)
{
    MArray::dpd_varray_view<const double> A(irrep_A, nirrep, dpd_lens(ndim_A, nirrep, lens_A), data_A);
    auto r = tblis::reduce<double>((tblis::reduce_t)op, A, idx_A);
    *result = r.first;
    *idx = r.second;
    return 0;
}

int refshim_dpd_unary(int kind, double alpha, double beta, unsigned nirrep, unsigned irrep_A, unsigned ndim_A,
                      const len_type* lens_A, double* data_A, const char* idx_A)
{
    MArray::dpd_varray_view<double> A(irrep_A, nirrep, dpd_lens(ndim_A, nirrep, lens_A), data_A);
    if (kind == 0) tblis::scale<double>(alpha, A, idx_A);
    else if (kind == 1) tblis::set<double>(alpha, A, idx_A);
    else tblis::shift<double>(alpha, beta, A, idx_A);
    return 0;
}

/*
 * An owning MArray indexed DPD tensor filled from flat storage (entries back
 * to back, default layout) and factors; and its storage copied back.
 */
static void fill_indexed(MArray::indexed_dpd_varray<double>& T, unsigned nirrep, unsigned irrep, unsigned ndim,
                         const len_type* lens, unsigned nidim, const unsigned* irr, long nidx,
                         const len_type* idx, const double* data, const double* f)
{
    MArray::matrix<len_type> len({ndim, nirrep}, MArray::ROW_MAJOR);
    for (unsigned i = 0; i < ndim; i++)
        for (unsigned j = 0; j < nirrep; j++) len[i][j] = lens[i*nirrep+j];
    std::vector<unsigned> ir(irr, irr + nidim);
    MArray::matrix<len_type> ix({(len_type)nidx, (len_type)nidim}, MArray::ROW_MAJOR);
    for (long e = 0; e < nidx; e++)
        for (unsigned d = 0; d < nidim; d++) ix[e][d] = idx[e*nidim+d];
    T.reset(irrep, nirrep, len, ir, ix);
    const len_type n = T.dense_size();
    for (long e = 0; e < nidx; e++)
    {
        std::copy_n(data + e*n, n, T.data(e));
        T.factor(e) = f[e];
    }
}

static void copy_out(const MArray::indexed_dpd_varray<double>& T, long nidx, double* data)
{
    const len_type n = T.dense_size();
    for (long e = 0; e < nidx; e++) std::copy_n(T.data(e), n, data + e*n);
}

#define IDX_ARGS(X) unsigned irrep_##X, unsigned ndim_##X, const len_type* lens_##X, unsigned nidim_##X, \
                    const unsigned* irr_##X, long nidx_##X, const len_type* idx_##X, double* data_##X, \
                    const double* f_##X, const char* lab_##X
#define IDX_FILL(T, X) fill_indexed(T, nirrep, irrep_##X, ndim_##X, lens_##X, nidim_##X, irr_##X, nidx_##X, \
                                    idx_##X, data_##X, f_##X)

/*
 * The reference's indexed-DPD level-1 operations (tblis::add / dot / reduce /
 * scale / set / shift over indexed_dpd_varray_view). unary kind: 0 scale
 * (A *= alpha), 1 set (A = alpha), 2 shift (A = alpha + beta*A).
 */
int refshim_indexed_dpd_add(unsigned nirrep, double alpha, IDX_ARGS(A), double beta, IDX_ARGS(B))
{
    MArray::indexed_dpd_varray<double> A, B;
    IDX_FILL(A, A);
    IDX_FILL(B, B);
    tblis::add<double>(alpha, A, lab_A, beta, B, lab_B);
    copy_out(B, nidx_B, data_B);
    return 0;
}

double refshim_indexed_dpd_dot(unsigned nirrep, IDX_ARGS(A), IDX_ARGS(B))
{
    MArray::indexed_dpd_varray<double> A, B;
    IDX_FILL(A, A);
    IDX_FILL(B, B);
    return tblis::dot<double>(A, lab_A, B, lab_B);
}

int refshim_indexed_dpd_reduce(int op, unsigned nirrep, IDX_ARGS(A), double* result, long* idx)
{
    MArray::indexed_dpd_varray<double> A;
    IDX_FILL(A, A);
    auto r = tblis::reduce<double>((tblis::reduce_t)op, A, lab_A);
    *result = r.first;
    // offsets are counted from entry 0's data, which is where the flat copy starts too
    *idx = r.second;
    return 0;
}

int refshim_indexed_dpd_unary(int kind, double alpha, double beta, unsigned nirrep, IDX_ARGS(A))
{
    MArray::indexed_dpd_varray<double> A;
    IDX_FILL(A, A);
    if (kind == 0) tblis::scale<double>(alpha, A, lab_A);
    else if (kind == 1) tblis::set<double>(alpha, A, lab_A);
    else tblis::shift<double>(alpha, beta, A, lab_A);
    copy_out(A, nidx_A, data_A);
    return 0;
}

/*
 * The reference's indexed-DPD contraction (tblis::mult over
 * indexed_dpd_varray_view, src/iface/3t/mult.cxx:412-541). Each tensor is
 * given by its overall irrep, ndim, lens [ndim][nirrep], the irreps of its
 * last nidx_dim (indexed) dimensions, nidx index tuples [nidx][nidx_dim], the
 * storage of its entries back to back (nidx x dense size, MArray's default
 * layout, as indexed_dpd_varray allocates it) and the entry factors. C's
 * storage is updated in place. impl selects the reference's implementation
 * (0 default, 1 BLOCKED, 2 FULL). Returns 0 on success.
 */
int refshim_indexed_dpd_mult(unsigned nirrep, double alpha,
                             unsigned irrep_A, unsigned ndim_A, const len_type* lens_A, unsigned nidim_A,
                             const unsigned* irr_A, long nidx_A, const len_type* idx_A_, const double* data_A,
                             const double* f_A, const char* lab_A,
                             unsigned irrep_B, unsigned ndim_B, const len_type* lens_B, unsigned nidim_B,
                             const unsigned* irr_B, long nidx_B, const len_type* idx_B_, const double* data_B,
                             const double* f_B, const char* lab_B,
                             double beta,
                             unsigned irrep_C, unsigned ndim_C, const len_type* lens_C, unsigned nidim_C,
                             const unsigned* irr_C, long nidx_C, const len_type* idx_C_, double* data_C,
                             const double* f_C, const char* lab_C, int impl)
{
    // filled in place (MArray's owning containers are not returned by value)
    auto fill = [&](MArray::indexed_dpd_varray<double>& T, unsigned irrep, unsigned ndim, const len_type* lens,
                    unsigned nidim, const unsigned* irr, long nidx, const len_type* idx, const double* data,
                    const double* f)
    {
        MArray::matrix<len_type> len({ndim, nirrep}, MArray::ROW_MAJOR);
        for (unsigned i = 0; i < ndim; i++)
            for (unsigned j = 0; j < nirrep; j++) len[i][j] = lens[i*nirrep+j];
        std::vector<unsigned> ir(irr, irr + nidim);
        MArray::matrix<len_type> ix({(len_type)nidx, (len_type)nidim}, MArray::ROW_MAJOR);
        for (long e = 0; e < nidx; e++)
            for (unsigned d = 0; d < nidim; d++) ix[e][d] = idx[e*nidim+d];
        T.reset(irrep, nirrep, len, ir, ix);
        const len_type n = T.dense_size();
        for (long e = 0; e < nidx; e++)
        {
            std::copy_n(data + e*n, n, T.data(e));
            T.factor(e) = f[e];
        }
    };
    MArray::indexed_dpd_varray<double> A, B, C;
    fill(A, irrep_A, ndim_A, lens_A, nidim_A, irr_A, nidx_A, idx_A_, data_A, f_A);
    fill(B, irrep_B, ndim_B, lens_B, nidim_B, irr_B, nidx_B, idx_B_, data_B, f_B);
    fill(C, irrep_C, ndim_C, lens_C, nidim_C, irr_C, nidx_C, idx_C_, data_C, f_C);
    // impl: 0 = the default block path, 1 = BLOCKED, 2 = FULL (dense round
    // trip, src/internal/3t/indexed_dpd/mult.cxx:68-114)
    const auto saved = tblis::internal::dpd_impl;
    tblis::internal::dpd_impl = impl == 2 ? tblis::internal::FULL : impl == 1 ? tblis::internal::BLOCKED
                                                                            : tblis::internal::BLIS;
    tblis::mult<double>(alpha, A, lab_A, B, lab_B, beta, C, lab_C);
    tblis::internal::dpd_impl = saved;
    const len_type n = C.dense_size();
    for (long e = 0; e < nidx_C; e++) std::copy_n(C.data(e), n, data_C + e*n);
    return 0;
}


int refshim_dpd_mult_t(int type, unsigned nirrep, const void* alpha, unsigned irrep_A, unsigned ndim_A,
                       const len_type* lens_A, const void* data_A, const char* idx_A, unsigned irrep_B,
                       unsigned ndim_B, const len_type* lens_B, const void* data_B, const char* idx_B,
                       const void* beta, unsigned irrep_C, unsigned ndim_C, const len_type* lens_C, void* data_C,
                       const char* idx_C)
{
#define REFSHIM_ARGS nirrep, alpha, irrep_A, ndim_A, lens_A, data_A, idx_A, irrep_B, ndim_B, lens_B, data_B, \
                     idx_B, beta, irrep_C, ndim_C, lens_C, data_C, idx_C
    switch (type)
    {
        case 0: return dpd_mult_t<float>(REFSHIM_ARGS);
        case 1: return dpd_mult_t<double>(REFSHIM_ARGS);
        case 2: return dpd_mult_t<scomplex>(REFSHIM_ARGS);
        case 3: return dpd_mult_t<dcomplex>(REFSHIM_ARGS);
    }
#undef REFSHIM_ARGS
    return 1;
}

int refshim_dpd_level1_t(int type, int op, unsigned nirrep, const void* alpha, const void* beta,
                         unsigned irrep_A, unsigned ndim_A, const len_type* lens_A, const void* data_A,
                         const char* idx_A, unsigned irrep_B, unsigned ndim_B, const len_type* lens_B,
                         void* data_B, const char* idx_B, void* result, long* idx)
{
#define REFSHIM_ARGS op, nirrep, alpha, beta, irrep_A, ndim_A, lens_A, data_A, idx_A, irrep_B, ndim_B, lens_B, \
                     data_B, idx_B, result, idx
    switch (type)
    {
        case 0: return dpd_level1_t<float>(REFSHIM_ARGS);
        case 1: return dpd_level1_t<double>(REFSHIM_ARGS);
        case 2: return dpd_level1_t<scomplex>(REFSHIM_ARGS);
        case 3: return dpd_level1_t<dcomplex>(REFSHIM_ARGS);
    }
#undef REFSHIM_ARGS
    return 1;
}

}
