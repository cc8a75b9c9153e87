// dpd.hpp -- DPD (direct-product-decomposition, irrep block-sparse) tensors:
// the storage layout of MArray's dpd_varray and the block-sparse contraction
// built on it.
#pragma once

#include "planner.hpp"

#include <complex>
#include <deque>
#include <string>

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
// owned (optional) marks the units of work whose C blocks are computed, for a
// rank's share of a sharded contraction (dpd_shard_owner's units); the other
// blocks of C are left untouched
void dpd_mult(const DpdTensor& A, const char* idx_A, const DpdTensor& B, const char* idx_B,
              DpdTensor& C, const char* idx_C, double alpha, double beta, cudaStream_t st,
              DpdMultReport* rep, bool reference_irrep_check = true, const std::vector<char>* owned = nullptr);

// A DPD contraction split across ranks with no collective on the data path.
// The unit of work is a row band of one irrep GEMM
// (src/internal/3t/dpd/mult.cxx:308): the C blocks that share their AC (and
// batch) irreps. Units go to ranks largest first onto the least loaded one,
// by FLOPs computed from the lengths alone, so every rank derives the same
// split without a device. Returns the owner of every irrep tuple of C
// (dimension 0 fastest, -1 where no block is stored) and, when asked, each
// rank's FLOPs and each unit's rank.
std::vector<int> dpd_shard_owner(const DpdTensor& A, const char* idx_A, const DpdTensor& B, const char* idx_B,
                                 const DpdTensor& C, const char* idx_C, int nranks, std::vector<double>* load,
                                 std::vector<int>* unit_rank = nullptr);
// rank's blocks of C = alpha*A*B + beta*C; the others stay as they are
void dpd_mult_shard(const DpdTensor& A, const char* idx_A, const DpdTensor& B, const char* idx_B,
                    DpdTensor& C, const char* idx_C, double alpha, double beta, int nranks, int rank,
                    cudaStream_t st, DpdMultReport* rep);

// One real term C += alpha*A*B (beta = 1) of a sequence of DPD contractions.
// Terms whose C storage may overlap carry the same c_key.
struct DpdTerm
{
    const DpdTensor* a = nullptr;
    const char* ia = nullptr;
    const DpdTensor* b = nullptr;
    const char* ib = nullptr;
    const DpdTensor* c = nullptr;
    const char* ic = nullptr;
    double alpha = 1.0;
    i64 c_key = 0;
};

// Runs the terms with the result of running them one after another: the k-th
// contributing term on each c_key goes into the k-th grouped launch, so terms
// on distinct C storage share a launch and terms on the same storage keep
// their order. rep (if given) sums groups and flops; returns the launches.
int dpd_mult_terms(const std::vector<DpdTerm>& terms, cudaStream_t st, DpdMultReport* rep,
                   bool reference_irrep_check = true);

// Element types of the DPD operations: float, double, scomplex, dcomplex
// (type_t); scalars of any type travel as complex<double>.
using zd = std::complex<double>;
size_t elem_size(int type);
inline bool is_complex_type(int type) { return type == TYPE_SCOMPLEX || type == TYPE_DCOMPLEX; }
zd scalar_get(const tblis_scalar& s);
void scalar_put(tblis_scalar& s, int type, zd v);

// float / scomplex DPD storage of `total` elements widened to double /
// dcomplex at equal offsets (a new device buffer), and the stored blocks of
// such a widened copy rounded back into the float storage (gaps untouched)
dbuf dpd_widen(const void* src, i64 total, bool cx, cudaStream_t st);
void dpd_narrow_blocks(const DpdLayout& X, bool cx, const double* src, float* dst, cudaStream_t st);

// the same blocks with every offset and stride multiplied by `scale` and the
// offsets shifted by `shift`: the real (shift 0) or imaginary (shift 1) part
// of a complex DPD tensor, seen as doubles
DpdLayout scaled_layout(const DpdLayout& X, i64 scale, i64 shift);

// complex DPD contraction on dcomplex device storage (double pointers to the
// storage base): C = beta*C, then the four real products of the parts, each
// a real DPD contraction (src/internal/3t/dense/mult.cxx:653-720 as 4M)
void dpd_mult_z(const DpdLayout& la, const double* a, const char* idx_A, const DpdLayout& lb, const double* b,
                const char* idx_B, const DpdLayout& lc, double* c, const char* idx_C, zd alpha, zd beta,
                cudaStream_t st, DpdMultReport* rep, bool reference_irrep_check = true);

// the real terms of the complex contraction C += alpha*A*B on dcomplex
// storage (4M, beta = 1), appended to `terms` with the real and imaginary
// parts of C under the keys 2*c_key and 2*c_key + 1; `store` holds the part
// tensors the terms point to
void dpd_terms_z(const DpdLayout& la, const double* a, const char* idx_A, const DpdLayout& lb, const double* b,
                 const char* idx_B, const DpdLayout& lc, double* c, const char* idx_C, zd alpha, i64 c_key,
                 std::deque<DpdTensor>& store, std::vector<DpdTerm>& terms);

// level-1 operations on device-resident DPD storage of element type `type`
// (dpd_level1.cpp): B = alpha*op(A) + beta*op(B) (trace / replicate per
// block), sum op(A)*op(B), a reduction with the offset of its extreme
// element, and the unary updates (kind 0: A = scal*op(A), 1: A = alpha,
// 2: A = alpha + scal*op(A)); op conjugates a complex operand whose flag is set
void dpd_add_dev_t(int type, zd alpha, const DpdLayout& A, const void* a, const std::string& iA, zd beta,
                   const DpdLayout& B, void* b, const std::string& iB, bool conj_a = false, bool conj_b = false);
zd dpd_dot_dev_t(int type, const DpdLayout& A, const void* a, const std::string& iA,
                 const DpdLayout& B, const void* b, const std::string& iB, bool conj_a = false,
                 bool conj_b = false);
void dpd_reduce_dev_t(int type, int op, const DpdLayout& A, const void* a, const std::string& iA, zd& result,
                      i64& idx);
void dpd_unary_dev_t(int type, int kind, zd alpha, zd scal, const DpdLayout& A, void* a, const std::string& iA,
                     bool conj = false);

// the same on double storage
inline void dpd_add_dev(double alpha, const DpdLayout& A, const double* a, const std::string& iA, double beta,
                        const DpdLayout& B, double* b, const std::string& iB)
{
    dpd_add_dev_t(TYPE_DOUBLE, alpha, A, a, iA, beta, B, b, iB);
}
inline double dpd_dot_dev(const DpdLayout& A, const double* a, const std::string& iA,
                          const DpdLayout& B, const double* b, const std::string& iB)
{
    return dpd_dot_dev_t(TYPE_DOUBLE, A, a, iA, B, b, iB).real();
}
inline void dpd_reduce_dev(int op, const DpdLayout& A, const double* a, const std::string& iA, double& result,
                           i64& idx)
{
    zd r;
    dpd_reduce_dev_t(TYPE_DOUBLE, op, A, a, iA, r, idx);
    result = r.real();
}
inline void dpd_unary_dev(int kind, double alpha, double scal, const DpdLayout& A, double* a, const std::string& iA)
{
    dpd_unary_dev_t(TYPE_DOUBLE, kind, alpha, scal, A, a, iA);
}

} // namespace tb
