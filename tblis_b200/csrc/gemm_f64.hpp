// gemm_f64.hpp -- FP64 DMMA block-scatter contraction kernel (see gemm_f64.cu)
#pragma once

#include "common.hpp"

namespace tb
{

struct GemmF64Args
{
    const double* A;
    const double* B;
    double* C;
    // scatter vectors (device): element offsets per GEMM index
    const i64 *a_m, *a_k, *b_k, *b_n, *c_m, *c_n, *a_l, *b_l, *c_l;
    // per-BK-block common k strides of A and B (0 = irregular block)
    const i64 *a_kbs, *b_kbs;
    i64 M, N, K, L;
    double alpha, beta;
    int amode, bmode;        // gather directions (see GemmView)
    int splits;              // split-K factor
    i64 k_per_split;         // set by the launcher
    double* partial;         // split-K workspace (splits*L*M*N doubles)
    int variant;             // tile configuration, 0 = automatic
    int pair_a, pair_b;      // gather the operand's contiguous dimension in pairs (16-byte copies)
};

// one K segment of a grouped GEMM: the rows of A / columns of B it reads
// and its k range (all segments of a group accumulate into the same C tile)
struct SegDesc
{
    const i64 *a_m, *a_k, *b_k, *b_n, *a_kbs, *b_kbs;
    i64 K;
};

// one GEMM of a grouped launch (no batch dimension: one entry per batch index).
// With nseg == 0 the group has a single segment given by the inline fields;
// otherwise segs[0..nseg) replace them (A and B offsets per segment).
struct GroupDesc
{
    const double* A;
    const double* B;
    double* C;
    const i64 *a_m, *a_k, *b_k, *b_n, *c_m, *c_n, *a_kbs, *b_kbs;
    i64 M, N, K;
    double alpha, beta;
    int amode, bmode;
    int nseg;
    const SegDesc* segs;
};

int gemm_f64_num_variants();
void gemm_f64_variant_tile(int variant, int& bm, int& bn);
// tile_begin[g] = first global tile of group g (tiles of BM x BN of the variant).
// d_counter (optional, one 64-bit word of device memory, zeroed by the launch)
// turns the static tile striding into a dynamic queue.
void gemm_f64_grouped_launch(const GroupDesc* d_groups, const i64* d_tile_begin, int ngroups,
                             i64 total_tiles, int variant, cudaStream_t stream,
                             unsigned long long* d_counter = nullptr);

i64 gemm_f64_tile_m();
i64 gemm_f64_tile_n();
i64 gemm_f64_tile_k();
int gemm_f64_choose_splits(i64 M, i64 N, i64 K, i64 L, int num_sms);
size_t gemm_f64_workspace_bytes(i64 M, i64 N, i64 L, int splits);
void gemm_f64_launch(GemmF64Args a, cudaStream_t stream);

} // namespace tb
