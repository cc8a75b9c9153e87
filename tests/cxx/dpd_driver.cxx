// dpd_driver.cxx -- test driver for libtblis_b200_cxx.so: a C++ caller
// written against TBLIS's own headers (src/tblis.h, which declares the
// tblis::mult overloads over MArray DPD and indexed-DPD views,
// src/iface/3t/mult.h:56-60 and 92-96) with TCI's own communicator. It links
// against libtblis_b200_cxx.so, libtblis_b200.so and TCI's library (the one a
// TBLIS caller links beside libtblis), so the tests reach the library's
// mangled C++ entry points exactly as such a program does.
#include "tblis.h"
#include "indexed_dpd_varray.hpp"

#include <vector>

// the library's extension entry points this driver uses (no counterpart in
// TBLIS's headers; the rest of include/tblis_b200.h restates TBLIS's types,
// which tblis.h already declares)
extern "C" {
int tblis_b200_last_error(void);
void tblis_b200_clear_error(void);
void tblis_b200_synchronize(void);
}

using tblis::len_type;

namespace
{
std::vector<std::vector<len_type>> lens_of(unsigned ndim, unsigned nirrep, const len_type* lens)
{
    std::vector<std::vector<len_type>> len(ndim, std::vector<len_type>(nirrep));
    for (unsigned i = 0; i < ndim; i++)
        for (unsigned j = 0; j < nirrep; j++) len[i][j] = lens[i*nirrep + j];
    return len;
}

std::vector<unsigned> perm_of(unsigned ndim, const unsigned* perm)
{
    std::vector<unsigned> p(ndim);
    for (unsigned i = 0; i < ndim; i++) p[i] = perm ? perm[i] : i;
    return p;
}
}

namespace
{
// an owning indexed DPD tensor filled from flat storage (entries back to back)
void fill_indexed(MArray::indexed_dpd_varray<double>& T, unsigned nirrep, unsigned irrep, unsigned ndim,
                  const len_type* lens, unsigned nidim, const unsigned* irr, long nidx, const len_type* idx,
                  const double* data, const double* f)
{
    MArray::matrix<len_type> len({ndim, nirrep}, MArray::ROW_MAJOR);
    for (unsigned i = 0; i < ndim; i++)
        for (unsigned j = 0; j < nirrep; j++) len[i][j] = lens[i*nirrep + j];
    std::vector<unsigned> ir(irr, irr + nidim);
    MArray::matrix<len_type> ix({(len_type)nidx, (len_type)nidim}, MArray::ROW_MAJOR);
    for (long e = 0; e < nidx; e++)
        for (unsigned d = 0; d < nidim; d++) ix[e][d] = idx[e*nidim + d];
    T.reset(irrep, nirrep, len, ir, ix);
    const len_type n = T.dense_size();
    for (long e = 0; e < nidx; e++)
    {
        std::copy_n(data + e*n, n, T.data(e));
        T.factor(e) = f[e];
    }
}
}

extern "C" {

// Indexed DPD tensors given as the oracle's indexed-DPD entry takes them;
// C's storage is updated in place. Returns the library's last error code.
int driver_indexed_dpd_mult(unsigned nirrep, double alpha,
                            unsigned irrep_A, unsigned ndim_A, const len_type* lens_A, unsigned nidim_A,
                            const unsigned* irr_A, long nidx_A, const len_type* idx_A, const double* data_A,
                            const double* f_A, const char* lab_A,
                            unsigned irrep_B, unsigned ndim_B, const len_type* lens_B, unsigned nidim_B,
                            const unsigned* irr_B, long nidx_B, const len_type* idx_B, const double* data_B,
                            const double* f_B, const char* lab_B,
                            double beta,
                            unsigned irrep_C, unsigned ndim_C, const len_type* lens_C, unsigned nidim_C,
                            const unsigned* irr_C, long nidx_C, const len_type* idx_C, double* data_C,
                            const double* f_C, const char* lab_C)
{
    tblis_b200_clear_error();
    MArray::indexed_dpd_varray<double> A, B, C;
    fill_indexed(A, nirrep, irrep_A, ndim_A, lens_A, nidim_A, irr_A, nidx_A, idx_A, data_A, f_A);
    fill_indexed(B, nirrep, irrep_B, ndim_B, lens_B, nidim_B, irr_B, nidx_B, idx_B, data_B, f_B);
    fill_indexed(C, nirrep, irrep_C, ndim_C, lens_C, nidim_C, irr_C, nidx_C, idx_C, data_C, f_C);
    tci::communicator comm;
    tblis::mult<double>(comm, alpha, A, lab_A, B, lab_B, beta, C, lab_C);
    tblis_b200_synchronize();
    const len_type n = C.dense_size();
    for (long e = 0; e < nidx_C; e++) std::copy_n(C.data(e), n, data_C + e*n);
    return tblis_b200_last_error();
}

// Each tensor: irrep, ndim, lens [ndim][nirrep], MArray layout code, an
// optional permutation of the view's dimensions (NULL = none), storage and
// labels (in the permuted order). Returns the library's last error code.
int driver_dpd_mult(unsigned nirrep, double alpha,
                    unsigned irrep_A, unsigned ndim_A, const len_type* lens_A, int layout_A,
                    const unsigned* perm_A, const double* data_A, const char* idx_A,
                    unsigned irrep_B, unsigned ndim_B, const len_type* lens_B, int layout_B,
                    const unsigned* perm_B, const double* data_B, const char* idx_B,
                    double beta,
                    unsigned irrep_C, unsigned ndim_C, const len_type* lens_C, int layout_C,
                    const unsigned* perm_C, double* data_C, const char* idx_C)
{
    tblis_b200_clear_error();
    MArray::dpd_varray_view<const double> A(irrep_A, nirrep, lens_of(ndim_A, nirrep, lens_A), data_A,
                                            MArray::dpd_layout(layout_A));
    MArray::dpd_varray_view<const double> B(irrep_B, nirrep, lens_of(ndim_B, nirrep, lens_B), data_B,
                                            MArray::dpd_layout(layout_B));
    MArray::dpd_varray_view<double> C(irrep_C, nirrep, lens_of(ndim_C, nirrep, lens_C), data_C,
                                      MArray::dpd_layout(layout_C));
    if (perm_A) A.permute(perm_of(ndim_A, perm_A));
    if (perm_B) B.permute(perm_of(ndim_B, perm_B));
    if (perm_C) C.permute(perm_of(ndim_C, perm_C));
    tci::communicator comm;
    tblis::mult<double>(comm, alpha, A, idx_A, B, idx_B, beta, C, idx_C);
    tblis_b200_synchronize();
    return tblis_b200_last_error();
}

}
