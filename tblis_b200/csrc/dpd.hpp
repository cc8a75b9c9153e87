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

    void init(unsigned irrep, unsigned nirrep, unsigned ndim, const i64* lens, int layout);
    // block (one irrep per dimension): lengths, strides, offset from the data base
    void block(const unsigned* irreps, i64* blen, i64* bstride, i64& offset) const;
    i64 total() const { return size.empty() ? 0 : size[2*ndim - 2][irrep]; }
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

void dpd_mult(const DpdTensor& A, const char* idx_A, const DpdTensor& B, const char* idx_B,
              DpdTensor& C, const char* idx_C, double alpha, double beta, cudaStream_t st,
              DpdMultReport* rep);

} // namespace tb
