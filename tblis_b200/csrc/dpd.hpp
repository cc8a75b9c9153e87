// dpd.hpp -- DPD (direct-product-decomposition, irrep block-sparse) tensors:
// the storage layout of MArray's dpd_varray and the block-sparse contraction
// built on it.
#pragma once

#include "planner.hpp"

namespace tb
{

// Storage description of a dense-stored DPD tensor and its layout tree
// (src/external/marray/include/dpd_marray_base.hpp:34-228).
struct DpdLayout
{
    unsigned ndim = 0, nirrep = 1, irrep = 0;
    int layout = 5;                               // MArray dpd_layout type, 5 = PREFIX_ROW_MAJOR (default)
    std::vector<std::vector<i64>> len;            // [ndim][nirrep] as given
    std::vector<std::vector<i64>> size;           // [2*ndim-1][nirrep] subtree sizes
    std::vector<unsigned> leaf, parent, perm;

    // explicit block table (layout = -1): the geometry of every stored block
    // as the caller's view reports it, for views that are not one of the six
    // MArray storage layouts (permuted or sliced views)
    std::vector<i64> xoff;                        // [nirrep^ndim] offset per irrep tuple (dim 0 fastest), -1 = none
    std::vector<i64> xstride;                     // [nirrep^ndim][ndim]
    i64 xextent = 0;                              // elements from the data base past the last stored element

    void init(unsigned irrep, unsigned nirrep, unsigned ndim, const i64* lens, int layout);
    void init_explicit(unsigned irrep, unsigned nirrep, unsigned ndim, const i64* lens, const i64* offsets,
                       const i64* strides);
    bool is_explicit() const { return !xoff.empty(); }
    // block (one irrep per dimension): lengths, strides, offset from the data base
    void block(const unsigned* irreps, i64* blen, i64* bstride, i64& offset) const;
    i64 total() const { return is_explicit() ? xextent : size.empty() ? 0 : size[2*ndim - 2][irrep]; }
    // every stored block with a non-zero extent: irreps, lengths, strides, offset
    template <typename F> void for_each_block(F&& f) const
    {
        std::vector<unsigned> irr(ndim, 0);
        std::vector<i64> bl(ndim), bs(ndim);
        while (true)
        {
            unsigned x = 0;
            i64 ext = 1;
            for (unsigned d = 0; d < ndim; d++) { x ^= irr[d]; ext *= len[d][irr[d]]; }
            if (x == irrep && ext > 0)
            {
                i64 off;
                block(irr.data(), bl.data(), bs.data(), off);
                f(irr, bl, bs, off);
            }
            unsigned d = 0;
            while (d < ndim && ++irr[d] == nirrep) { irr[d] = 0; d++; }
            if (d == ndim) break;
        }
    }
};

// src/external/marray/include/dpd_marray_base.hpp:34-67
std::vector<unsigned> dpd_default_depth(int layout, unsigned ndim);

struct DpdTensor
{
    DpdLayout lay;
    double* data = nullptr;
    double alpha = 1.0;
};

struct DpdMultReport
{
    int groups = 0;               // irrep GEMMs launched (non-empty)
    double flops = 0;             // sum over symmetry-allowed blocks of 2*m*n*k
    int variant = 0;              // tile configuration picked by the tuner
};

// reference_irrep_check: skip the contraction as src/iface/3t/mult.cxx:270
// does (its operator precedence included); false: skip only when
// irrep(A) ^ irrep(B) != irrep(C), as the internal block loops of the
// indexed-DPD contraction see it
void dpd_mult(const DpdTensor& A, const char* idx_A, const DpdTensor& B, const char* idx_B,
              DpdTensor& C, const char* idx_C, double alpha, double beta, cudaStream_t st,
              DpdMultReport* rep, bool reference_irrep_check = true);

// level-1 operations on device-resident DPD storage (dpd_level1.cpp):
// B = alpha*A + beta*B (trace / replicate per block), sum A*B, a reduction
// with the offset of its extreme element, and the unary updates (kind 0:
// A *= scal, 1: A = alpha, 2: A = alpha + scal*A)
void dpd_add_dev(double alpha, const DpdLayout& A, const double* a, const std::string& iA, double beta,
                 const DpdLayout& B, double* b, const std::string& iB);
double dpd_dot_dev(const DpdLayout& A, const double* a, const std::string& iA,
                   const DpdLayout& B, const double* b, const std::string& iB);
void dpd_reduce_dev(int op, const DpdLayout& A, const double* a, const std::string& iA, double& result, i64& idx);
void dpd_unary_dev(int kind, double alpha, double scal, const DpdLayout& A, double* a, const std::string& iA);

} // namespace tb
