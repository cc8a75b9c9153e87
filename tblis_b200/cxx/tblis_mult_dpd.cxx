// tblis_mult_dpd.cxx -- TBLIS's compiled C++ overloads of tblis::mult over
// MArray's DPD views, reaching the GPU library through its C ABI.
//
// TBLIS declares these overloads in src/iface/3t/mult.h:56-60 and 92-96 (and
// the level-1 ones in src/iface/1t/*.h) and instantiates them in its library
// (src/iface/3t/mult.cxx:292-298, 535-541; src/iface/1t/*.cxx) for float,
// double, scomplex and dcomplex, so a C++ program links
// against their mangled names. This file defines the same templates with the
// same instantiations; compiled against the caller's MArray headers (the
// views' layout must match the caller's, so the same MARRAY_* configuration
// is used: ptrdiff_t lengths and strides, the default short-vector size), it
// goes into libtblis_b200_cxx.so, which depends on libtblis_b200.so.
//
// Each view is described to the C ABI by the geometry of its stored blocks as
// the view itself reports it (operator()(irreps), dpd_varray_base.hpp:482-508),
// so permuted views work as well as the six storage layouts. Every
// instantiated type computes on the GPU: double directly, dcomplex as four
// real contractions, float and scomplex widened to double on the device and
// rounded back.
//
// Threading follows TCI's contract (src/util/thread.h:333-352): every thread
// of the communicator enters; the master thread issues the GPU work and the
// others wait at the communicator's barrier.
#include "dpd_varray_view.hpp"
#include "indexed_dpd_varray_view.hpp"

#include "../../include/tblis_b200.h"

#include <complex>
#include <cstring>
#include <vector>

namespace tci { class communicator; }

// TCI's barrier, resolved from the caller's libtci when it is loaded (a
// communicator of more than one thread exists only then)
extern "C" int tci_comm_barrier(void* comm) __attribute__((weak));

namespace tblis
{

using MArray::dpd_varray_view;
using MArray::indexed_dpd_varray_view;

namespace
{

// the data of tci::communicator: one tci_comm (tci/communicator.h:8-15)
struct comm_data
{
    void* context;
    unsigned ngang, gid, nthread, tid;
};

template <typename T> type_t type_of();
template <> type_t type_of<float>() { return TYPE_FLOAT; }
template <> type_t type_of<double>() { return TYPE_DOUBLE; }
template <> type_t type_of<std::complex<float>>() { return TYPE_SCOMPLEX; }
template <> type_t type_of<std::complex<double>>() { return TYPE_DCOMPLEX; }

// a value of T into / out of tblis_scalar's union (float, double,
// complex<float> and complex<double> share its leading bytes)
template <typename T> void set_scalar(tblis_scalar& s, T v)
{
    s.type = type_of<T>();
    std::memset(&s.data, 0, sizeof(s.data));
    std::memcpy(&s.data, &v, sizeof(T));
}

template <typename T> T get_scalar(const tblis_scalar& s)
{
    T v;
    std::memcpy(&v, &s.data, sizeof(T));
    return v;
}

// lengths and the per-block geometry of one DPD view
struct Table
{
    std::vector<len_type> len;
    std::vector<stride_type> off, stride;
    tblis_b200_dpd_block_table t;

    template <typename T, typename S>
    Table(const dpd_varray_view<T>& V, S scalar)
    {
        const unsigned nd = V.dimension(), nirrep = V.num_irreps();
        len.resize((size_t)nd*nirrep);
        for (unsigned d = 0; d < nd; d++)
            for (unsigned r = 0; r < nirrep; r++) len[(size_t)d*nirrep + r] = V.length(d, r);
        size_t nt = 1;
        for (unsigned d = 0; d < nd; d++) nt *= nirrep;
        off.assign(nt, -1);
        stride.assign(nt*nd, 0);
        std::vector<unsigned> irr(nd, 0);
        for (size_t tpl = 0; tpl < nt; tpl++)
        {
            unsigned x = 0;
            len_type ext = 1;
            for (unsigned d = 0; d < nd; d++) { x ^= irr[d]; ext *= V.length(d, irr[d]); }
            if (x == V.irrep() && ext > 0)
            {
                auto blk = V(irr);
                off[tpl] = blk.data() - V.data();
                for (unsigned d = 0; d < nd; d++) stride[tpl*nd + d] = blk.stride(d);
            }
            unsigned d = 0;
            while (d < nd && ++irr[d] == nirrep) { irr[d] = 0; d++; }
        }
        t.type = type_of<typename std::remove_const<T>::type>();
        t.conj = 0;
        set_scalar(t.scalar, scalar);
        t.data = const_cast<void*>(static_cast<const void*>(V.data()));
        t.ndim = nd;
        t.nirrep = nirrep;
        t.irrep = V.irrep();
        t.len = len.data();
        t.offset = off.data();
        t.stride = stride.data();
    }
};

// an indexed DPD view: its entries, and the block table of one entry
struct IdxTable
{
    std::vector<len_type> len, indices;
    std::vector<unsigned> idx_irrep;
    std::vector<void*> data;
    std::vector<unsigned char> factor;        // the entries' factors, elements of the view's type
    Table dense;
    tblis_b200_indexed_dpd_tensor t;

    template <typename T, typename S>
    IdxTable(const indexed_dpd_varray_view<T>& V, S scalar) : dense(V[0], scalar)
    {
        using U = typename std::remove_const<T>::type;
        const unsigned nd = V.dimension(), nirrep = V.num_irreps(), ni = V.indexed_dimension();
        len.resize((size_t)nd*nirrep);
        for (unsigned d = 0; d < nd; d++)
            for (unsigned r = 0; r < nirrep; r++) len[(size_t)d*nirrep + r] = V.length(d, r);
        for (unsigned d = 0; d < ni; d++) idx_irrep.push_back(V.indexed_irrep(d));
        const len_type n = V.num_indices();
        for (len_type e = 0; e < n; e++)
        {
            for (unsigned d = 0; d < ni; d++) indices.push_back(ni ? V.indices(e)[d] : 0);
            data.push_back(const_cast<U*>(V.data(e)));
            const U f = V.factor(e);
            const unsigned char* fb = reinterpret_cast<const unsigned char*>(&f);
            factor.insert(factor.end(), fb, fb + sizeof(U));
        }
        t.type = type_of<U>();
        set_scalar(t.scalar, scalar);
        t.ndim = nd;
        t.dense_ndim = V.dense_dimension();
        t.nirrep = nirrep;
        t.dense_irrep = V.dense_irrep();
        t.len = len.data();
        t.idx_irrep = idx_irrep.empty() ? nullptr : idx_irrep.data();
        t.nidx = n;
        t.indices = indices.empty() ? nullptr : indices.data();
        t.data = data.data();
        t.factor = factor.data();
        t.offset = dense.off.data();
        t.stride = dense.stride.data();
    }
};

void wait_all(const tci::communicator& comm)
{
    const comm_data* c = reinterpret_cast<const comm_data*>(&comm);
    if (c->nthread > 1 && tci_comm_barrier) tci_comm_barrier(const_cast<comm_data*>(c));
}

bool is_master(const tci::communicator& comm)
{
    return reinterpret_cast<const comm_data*>(&comm)->tid == 0;
}

} // namespace

template <typename T>
void mult(const tci::communicator& comm,
          T alpha, dpd_varray_view<const T> A, const label_type* idx_A,
                   dpd_varray_view<const T> B, const label_type* idx_B,
          T  beta, dpd_varray_view<      T> C, const label_type* idx_C)
{
    if (is_master(comm))
    {
        Table a(A, alpha), b(B, T(1)), c(C, beta);
        // host data is staged and the call returns with the result in place;
        // device data is computed in order on the library's stream
        tblis_b200_dpd_mult_blocks(&a.t, idx_A, &b.t, idx_B, &c.t, idx_C, nullptr);
    }
    wait_all(comm);
}

template <typename T>
void mult(const tci::communicator& comm,
          T alpha, indexed_dpd_varray_view<const T> A, const label_type* idx_A,
                   indexed_dpd_varray_view<const T> B, const label_type* idx_B,
          T  beta, indexed_dpd_varray_view<      T> C, const label_type* idx_C)
{
    if (is_master(comm))
    {
        IdxTable a(A, alpha), b(B, T(1)), c(C, beta);
        tblis_b200_indexed_dpd_mult(&a.t, idx_A, &b.t, idx_B, &c.t, idx_C, nullptr);
    }
    wait_all(comm);
}

// the reference's reduce_t lives in namespace tblis (src/util/basic_types.h:53-64)
typedef enum
{
    REDUCE_SUM_ = 0, REDUCE_SUM_ABS_ = 1, REDUCE_MAX_ = 2, REDUCE_MAX_ABS_ = 3,
    REDUCE_MIN_ = 4, REDUCE_MIN_ABS_ = 5, REDUCE_NORM_2_ = 6
} reduce_t;

// level-1 operations over DPD views (src/iface/1t/{add,dot,reduce,scale,set,
// shift}.cxx, instantiated there for the same four types)
template <typename T>
void add(const tci::communicator& comm,
         T alpha, dpd_varray_view<const T> A, const label_type* idx_A,
         T  beta, dpd_varray_view<      T> B, const label_type* idx_B)
{
    if (is_master(comm))
    {
        Table a(A, alpha), b(B, beta);
        tblis_b200_dpd_add(&a.t, idx_A, &b.t, idx_B);
    }
    wait_all(comm);
}

template <typename T>
void dot(const tci::communicator& comm,
         dpd_varray_view<const T> A, const label_type* idx_A,
         dpd_varray_view<const T> B, const label_type* idx_B, T& result)
{
    if (is_master(comm))
    {
        Table a(A, T(1)), b(B, T(1));
        tblis_scalar r;
        if (tblis_b200_dpd_dot(&a.t, idx_A, &b.t, idx_B, &r) == 0) result = get_scalar<T>(r);
    }
    wait_all(comm);
}

template <typename T>
void reduce(const tci::communicator& comm, reduce_t op,
            dpd_varray_view<const T> A, const label_type* idx_A, T& result, len_type& idx)
{
    if (is_master(comm))
    {
        Table a(A, T(1));
        tblis_scalar r;
        len_type i = -1;
        if (tblis_b200_dpd_reduce((::reduce_t)op, &a.t, idx_A, &r, &i) == 0)
        {
            result = get_scalar<T>(r);
            idx = i;
        }
    }
    wait_all(comm);
}

template <typename T>
void scale(const tci::communicator& comm, T alpha, dpd_varray_view<T> A, const label_type* idx_A)
{
    if (is_master(comm))
    {
        Table a(A, alpha);
        tblis_b200_dpd_scale(&a.t, idx_A);
    }
    wait_all(comm);
}

template <typename T>
void set(const tci::communicator& comm, T alpha, dpd_varray_view<T> A, const label_type* idx_A)
{
    if (is_master(comm))
    {
        Table a(A, T(1));
        tblis_scalar s;
        set_scalar(s, alpha);
        tblis_b200_dpd_set(&s, &a.t, idx_A);
    }
    wait_all(comm);
}

template <typename T>
void shift(const tci::communicator& comm, T alpha, T beta, dpd_varray_view<T> A, const label_type* idx_A)
{
    if (is_master(comm))
    {
        Table a(A, beta);
        tblis_scalar s;
        set_scalar(s, alpha);
        tblis_b200_dpd_shift(&s, &a.t, idx_A);
    }
    wait_all(comm);
}

#define TBLIS_B200_DPD_LEVEL1(T) \
template void add(const tci::communicator&, T, dpd_varray_view<const T>, const label_type*, \
                  T, dpd_varray_view<T>, const label_type*); \
template void dot(const tci::communicator&, dpd_varray_view<const T>, const label_type*, \
                  dpd_varray_view<const T>, const label_type*, T&); \
template void reduce(const tci::communicator&, reduce_t, dpd_varray_view<const T>, const label_type*, \
                     T&, len_type&); \
template void scale(const tci::communicator&, T, dpd_varray_view<T>, const label_type*); \
template void set(const tci::communicator&, T, dpd_varray_view<T>, const label_type*); \
template void shift(const tci::communicator&, T, T, dpd_varray_view<T>, const label_type*);
TBLIS_B200_DPD_LEVEL1(float)
TBLIS_B200_DPD_LEVEL1(double)
TBLIS_B200_DPD_LEVEL1(std::complex<float>)
TBLIS_B200_DPD_LEVEL1(std::complex<double>)

// the same over indexed DPD views (instantiated in src/iface/1t/*.cxx)
template <typename T>
void add(const tci::communicator& comm,
         T alpha, indexed_dpd_varray_view<const T> A, const label_type* idx_A,
         T  beta, indexed_dpd_varray_view<      T> B, const label_type* idx_B)
{
    if (is_master(comm))
    {
        IdxTable a(A, alpha), b(B, beta);
        tblis_b200_indexed_dpd_add(&a.t, idx_A, &b.t, idx_B);
    }
    wait_all(comm);
}

template <typename T>
void dot(const tci::communicator& comm,
         indexed_dpd_varray_view<const T> A, const label_type* idx_A,
         indexed_dpd_varray_view<const T> B, const label_type* idx_B, T& result)
{
    if (is_master(comm))
    {
        IdxTable a(A, T(1)), b(B, T(1));
        tblis_scalar r;
        if (tblis_b200_indexed_dpd_dot(&a.t, idx_A, &b.t, idx_B, &r) == 0) result = get_scalar<T>(r);
    }
    wait_all(comm);
}

template <typename T>
void reduce(const tci::communicator& comm, reduce_t op,
            indexed_dpd_varray_view<const T> A, const label_type* idx_A, T& result, len_type& idx)
{
    if (is_master(comm))
    {
        IdxTable a(A, T(1));
        tblis_scalar r;
        len_type i = -1;
        if (tblis_b200_indexed_dpd_reduce((::reduce_t)op, &a.t, idx_A, &r, &i) == 0)
        {
            result = get_scalar<T>(r);
            idx = i;
        }
    }
    wait_all(comm);
}

template <typename T>
void scale(const tci::communicator& comm, T alpha, indexed_dpd_varray_view<T> A, const label_type* idx_A)
{
    if (is_master(comm))
    {
        IdxTable a(A, alpha);
        tblis_b200_indexed_dpd_scale(&a.t, idx_A);
    }
    wait_all(comm);
}

template <typename T>
void set(const tci::communicator& comm, T alpha, indexed_dpd_varray_view<T> A, const label_type* idx_A)
{
    if (is_master(comm))
    {
        IdxTable a(A, T(1));
        tblis_scalar s;
        set_scalar(s, alpha);
        tblis_b200_indexed_dpd_set(&s, &a.t, idx_A);
    }
    wait_all(comm);
}

template <typename T>
void shift(const tci::communicator& comm, T alpha, T beta, indexed_dpd_varray_view<T> A, const label_type* idx_A)
{
    if (is_master(comm))
    {
        IdxTable a(A, beta);
        tblis_scalar s;
        set_scalar(s, alpha);
        tblis_b200_indexed_dpd_shift(&s, &a.t, idx_A);
    }
    wait_all(comm);
}

#define TBLIS_B200_INDEXED_DPD_LEVEL1(T) \
template void add(const tci::communicator&, T, indexed_dpd_varray_view<const T>, const label_type*, \
                  T, indexed_dpd_varray_view<T>, const label_type*); \
template void dot(const tci::communicator&, indexed_dpd_varray_view<const T>, const label_type*, \
                  indexed_dpd_varray_view<const T>, const label_type*, T&); \
template void reduce(const tci::communicator&, reduce_t, indexed_dpd_varray_view<const T>, const label_type*, \
                     T&, len_type&); \
template void scale(const tci::communicator&, T, indexed_dpd_varray_view<T>, const label_type*); \
template void set(const tci::communicator&, T, indexed_dpd_varray_view<T>, const label_type*); \
template void shift(const tci::communicator&, T, T, indexed_dpd_varray_view<T>, const label_type*);
TBLIS_B200_INDEXED_DPD_LEVEL1(float)
TBLIS_B200_INDEXED_DPD_LEVEL1(double)
TBLIS_B200_INDEXED_DPD_LEVEL1(std::complex<float>)
TBLIS_B200_INDEXED_DPD_LEVEL1(std::complex<double>)

#define TBLIS_B200_DPD_MULT(T) \
template void mult(const tci::communicator& comm, \
                   T alpha, dpd_varray_view<const T> A, const label_type* idx_A, \
                            dpd_varray_view<const T> B, const label_type* idx_B, \
                   T  beta, dpd_varray_view<      T> C, const label_type* idx_C);
#define TBLIS_B200_INDEXED_DPD_MULT(T) \
template void mult(const tci::communicator& comm, \
                   T alpha, indexed_dpd_varray_view<const T> A, const label_type* idx_A, \
                            indexed_dpd_varray_view<const T> B, const label_type* idx_B, \
                   T  beta, indexed_dpd_varray_view<      T> C, const label_type* idx_C);
TBLIS_B200_DPD_MULT(float)
TBLIS_B200_DPD_MULT(double)
TBLIS_B200_DPD_MULT(std::complex<float>)
TBLIS_B200_DPD_MULT(std::complex<double>)
TBLIS_B200_INDEXED_DPD_MULT(float)
TBLIS_B200_INDEXED_DPD_MULT(double)
TBLIS_B200_INDEXED_DPD_MULT(std::complex<float>)
TBLIS_B200_INDEXED_DPD_MULT(std::complex<double>)

} // namespace tblis
