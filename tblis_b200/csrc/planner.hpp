// planner.hpp -- host-side contraction planner.
//
// Restates TBLIS's index-label algebra (diagonal, fold, sort_by_stride, the
// AB/AC/BC/ABC group split) and its block-scatter vector builder, and turns a
// contraction into a "GEMM view": m/n/k/l extents plus per-operand scatter
// vectors (element offset of every row, column and k index) that the device
// kernels gather through. Nothing here touches tensor data.
#pragma once

#include "common.hpp"

#include <memory>
#include <string>

namespace tb
{

typedef std::vector<i64> ivec;

// src/util/tensor.hpp:375-412
void diagonal(unsigned ndim, const len_type* len, const stride_type* stride, const char* idx,
              ivec& len_out, ivec& stride_out, std::string& idx_out);

// src/util/tensor.hpp:95-148: permutation ordering dims by (min stride over the
// given vectors, then each vector in turn); std::sort as in the reference.
std::vector<unsigned> sort_by_stride(const std::vector<const ivec*>& strides);

// src/util/tensor.hpp:341-373
void fold(ivec& len, std::string& idx, const std::vector<ivec*>& strides);

// src/util/tensor.hpp:33-60
char free_idx(std::string labels);

// src/matrix/block_scatter_matrix.hpp:68-258 (element type double)
void fill_block_scatter(const ivec& len, const ivec& stride, i64 BS, i64 off, i64 size,
                        i64* scat, i64* bs, bool pack_3d);

// Index groups of a contraction after diagonal/fold (src/iface/3t/mult.cxx:30-116)
struct MultGroups
{
    std::string AB, AC, BC, ABC;
    ivec len_AB, len_AC, len_BC, len_ABC;
    ivec sA_AB, sB_AB, sA_AC, sC_AC, sB_BC, sC_BC, sA_ABC, sB_ABC, sC_ABC;
};

MultGroups mult_groups(const tblis_tensor* A, const char* idx_A,
                       const tblis_tensor* B, const char* idx_B,
                       const tblis_tensor* C, const char* idx_C);

// GEMM view: the groups reordered as src/internal/3t/dense/mult.cxx:460-571
// reorders them (stride sort, unit-stride dimension, 3-D packing rotation).
struct GemmView
{
    i64 m = 1, n = 1, k = 1, l = 1;
    std::string idxM, idxN, idxK, idxL;
    ivec lenM, lenN, lenK, lenL;
    ivec aM, cM, aK, bK, bN, cN, aL, bL, cL;   // strides in GEMM order
    bool pack_m_3d = false, pack_n_3d = false, pack_k_3d = false;
    int amode = 0;   // 0: A gathered along m (m-contiguous), 1: along k
    int bmode = 0;   // 0: B gathered along n, 1: along k
};

GemmView gemm_view(const MultGroups& g);

// Device-resident scatter tables of one GEMM view for given tile sizes.
struct GemmTables
{
    i64* dev = nullptr;      // one allocation holding every vector below
    i64 *a_m, *c_m, *a_k, *b_k, *b_n, *c_n, *a_l, *b_l, *c_l, *a_kbs, *b_kbs;
    // s where the table is i*s for every i (a single stride), else -1
    i64 a_m_step = -1, a_k_step = -1, b_n_step = -1, b_k_step = -1;
    // per gather mode (0: rows contiguous, 1: k contiguous): whether nearly
    // all pairs of adjacent elements of the contiguous dimension are adjacent
    // and 16-byte aligned in memory (offsets even), so that the FP64 kernel
    // gathers A / B in pairs
    bool a_pairs[2] = {false, false}, b_pairs[2] = {false, false};
    size_t bytes = 0;
    ~GemmTables();
};

// Decides, from a view's host scatter vectors, whether the FP64 kernel may
// gather A and B in 16-byte pairs in each gather mode (GemmTables::a_pairs).
void gemm_pair_modes(const GemmView& v, const i64* a_m, const i64* a_k, const i64* b_n, const i64* b_k,
                     const i64* a_l, const i64* b_l, bool a_pairs[2], bool b_pairs[2]);

// Builds (or fetches from the plan cache) the device tables for a view.
std::shared_ptr<GemmTables> gemm_tables(const GemmView& v, i64 BM, i64 BN, i64 BK,
                                        cudaStream_t stream);

// Total extent in elements [min_off, max_off] touched by a strided tensor.
void tensor_extent(unsigned ndim, const len_type* len, const stride_type* stride,
                   i64& min_off, i64& max_off);

} // namespace tb
