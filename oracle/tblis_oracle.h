/*
 * tblis_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C, single-threaded restatement of the TBLIS reference algorithms on
 * the tensor-contraction hot path. Only the tests, the smoke check and the
 * CPU-baseline leg of the benchmark load it, and only as the checker; the
 * product library never links or calls it.
 *
 * Parity of this restatement is pinned against the reference itself, compiled
 * from its own sources by oracle/Makefile into oracle/_ref/ (tests compare the
 * two on seeded inputs), and against the golden DPD layout vectors of the
 * reference's MArray test suite (tests/golden/).
 *
 * Every function cites the reference file:line it restates (paths relative to
 * the TBLIS source tree).
 */
#ifndef TBLIS_ORACLE_H
#define TBLIS_ORACLE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef ptrdiff_t orc_len;
typedef ptrdiff_t orc_stride;

#define ORC_MAX_DIM 16

/* src/util/tensor.hpp:375-412 (diagonal): sort dims by label, drop length-1
 * dims, merge repeated labels by summing strides. Returns the new ndim. */
unsigned orc_diagonal(unsigned ndim, const orc_len* len, const orc_stride* stride,
                      const char* idx, orc_len* len_out, orc_stride* stride_out,
                      char* idx_out);

/* src/util/tensor.hpp:341-373 (fold): sort the group by the first stride
 * vector, merge adjacent dims contiguous in every stride vector. nstr stride
 * vectors are updated in place; returns the new number of dims. */
unsigned orc_fold(unsigned ndim, orc_len* len, char* idx, unsigned nstr,
                  orc_stride** strides);

/* src/util/tensor.hpp:95-148 (sort_by_stride): permutation that orders dims by
 * (min over the nstr stride vectors, then each vector in turn). */
void orc_sort_by_stride(unsigned ndim, unsigned nstr, const orc_stride* const* strides,
                        unsigned* perm);

/* src/matrix/block_scatter_matrix.hpp:68-258 (fill_scatter, fill_block_stride,
 * fill_block_scatter): scatter offsets of rows [off, off+size) of a group of
 * dims and the common stride of each BS-block (0 if irregular). */
void orc_fill_block_scatter(unsigned ndim, const orc_len* len, const orc_stride* stride,
                            orc_len BS, orc_stride off, orc_stride size,
                            orc_stride* scat, orc_stride* bs, int pack_3d);

/* Index-group split of a contraction, as src/iface/3t/mult.cxx:30-116 does it
 * (diagonal, fake unit dims, AB/AC/BC/ABC split, fold of every group). */
typedef struct orc_mult_groups
{
    unsigned n_AB, n_AC, n_BC, n_ABC;
    char idx_AB[ORC_MAX_DIM], idx_AC[ORC_MAX_DIM], idx_BC[ORC_MAX_DIM], idx_ABC[ORC_MAX_DIM];
    orc_len len_AB[ORC_MAX_DIM], len_AC[ORC_MAX_DIM], len_BC[ORC_MAX_DIM], len_ABC[ORC_MAX_DIM];
    orc_stride sA_AB[ORC_MAX_DIM], sB_AB[ORC_MAX_DIM];
    orc_stride sA_AC[ORC_MAX_DIM], sC_AC[ORC_MAX_DIM];
    orc_stride sB_BC[ORC_MAX_DIM], sC_BC[ORC_MAX_DIM];
    orc_stride sA_ABC[ORC_MAX_DIM], sB_ABC[ORC_MAX_DIM], sC_ABC[ORC_MAX_DIM];
} orc_mult_groups;

int orc_mult_groups_build(unsigned ndim_A, const orc_len* len_A, const orc_stride* stride_A, const char* idx_A,
                          unsigned ndim_B, const orc_len* len_B, const orc_stride* stride_B, const char* idx_B,
                          unsigned ndim_C, const orc_len* len_C, const orc_stride* stride_C, const char* idx_C,
                          orc_mult_groups* g);

/* C = alpha*sum_AB A*B + beta*C over strided double tensors; the loop nest of
 * src/internal/3t/dense/mult.cxx:653-720 (mult_ref), beta==0 never reads C.
 * Returns 0 on success. */
int orc_tensor_mult_d(double alpha, unsigned ndim_A, const orc_len* len_A, const orc_stride* stride_A,
                      const double* A, const char* idx_A,
                      unsigned ndim_B, const orc_len* len_B, const orc_stride* stride_B,
                      const double* B, const char* idx_B,
                      double beta, unsigned ndim_C, const orc_len* len_C, const orc_stride* stride_C,
                      double* C, const char* idx_C);

/* Same contraction, evaluated only at nsample entries of C given by their
 * multi-indices in C's label order (row-major [nsample][ndim_C]); writes the
 * values alpha*sum + beta*C_old into out. Used to check full-size results. */
int orc_tensor_mult_sample_d(double alpha, unsigned ndim_A, const orc_len* len_A, const orc_stride* stride_A,
                             const double* A, const char* idx_A,
                             unsigned ndim_B, const orc_len* len_B, const orc_stride* stride_B,
                             const double* B, const char* idx_B,
                             double beta, unsigned ndim_C, const orc_len* len_C, const orc_stride* stride_C,
                             const double* C, const char* idx_C,
                             orc_len nsample, const orc_len* sample_idx, double* out);

/* B = alpha*A (+trace over A-only, replicate over B-only) + beta*B;
 * src/iface/1t/add.cxx:24-110 and src/internal/1t/dense/add.cxx:15-261. */
int orc_tensor_add_d(double alpha, unsigned ndim_A, const orc_len* len_A, const orc_stride* stride_A,
                     const double* A, const char* idx_A,
                     double beta, unsigned ndim_B, const orc_len* len_B, const orc_stride* stride_B,
                     double* B, const char* idx_B);

/* sum A*B over matching labels; src/iface/1t/dot.cxx:16-74. */
int orc_tensor_dot_d(double alpha_A, unsigned ndim_A, const orc_len* len_A, const orc_stride* stride_A,
                     const double* A, const char* idx_A,
                     double alpha_B, unsigned ndim_B, const orc_len* len_B, const orc_stride* stride_B,
                     const double* B, const char* idx_B, double* result);

/* src/iface/1t/reduce.cxx:16-68, src/internal/1t/dense/reduce.cxx:12-67,
 * src/kernels/1v/reduce.hpp:16-106: op codes as reduce_t. */
int orc_tensor_reduce_d(int op, double alpha, unsigned ndim_A, const orc_len* len_A,
                        const orc_stride* stride_A, const double* A, const char* idx_A,
                        double* result, orc_len* idx);

/* src/iface/1t/scale.cxx:20-60, set.cxx, shift.cxx */
int orc_tensor_scale_d(double alpha, unsigned ndim, const orc_len* len, const orc_stride* stride, double* A);
int orc_tensor_set_d(double alpha, unsigned ndim, const orc_len* len, const orc_stride* stride, double* A);
int orc_tensor_shift_d(double shift, double alpha, unsigned ndim, const orc_len* len,
                       const orc_stride* stride, double* A);

/* src/external/marray/include/dpd_marray_base.hpp:34-228: offset, lengths
 * and strides of one block of a dense-stored DPD tensor (layout: MArray
 * dpd_layout type 0..5), and the total number of stored elements. */
int orc_dpd_block(unsigned irrep, unsigned nirrep, unsigned ndim, const orc_len* lens, int layout,
                  const unsigned* irreps, orc_len* blen, orc_stride* bstride, orc_stride* offset);
orc_len orc_dpd_size(unsigned irrep, unsigned nirrep, unsigned ndim, const orc_len* lens, int layout);

#ifdef __cplusplus
}
#endif

#endif
