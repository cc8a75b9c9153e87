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
    // packed path (gemm_f64_ws.cu): tile shape (gemm_f64_ws_shape), k steps
    // over all segments, and the offsets (in doubles) of the group's packed A
    // panels and B panels
    int shape;
    int nst;
    i64 pa, pb;
};

// one piece of a panel to pack: k steps [s0, s0 + ns) of rows
// [panel*BM, ...) of group g's A (side 0), or of columns [panel*BN, ...) of
// its B (side 1); steps are counted over all segments of the group
struct PackItem
{
    int g, side, panel, s0, ns, pad;
};

int gemm_f64_num_variants();
void gemm_f64_variant_tile(int variant, int& bm, int& bn);
// variants of a grouped launch: the tile family above, then the packed path
// (variant gemm_f64_num_variants() + 1, tiles of each group's own shape; run
// by the grouped plan, not by gemm_f64_grouped_launch)
int gemm_f64_grouped_num_variants();
bool gemm_f64_is_ws_variant(int variant);

// The packed grouped path (gemm_f64_ws.cu): gemm_f64_ws_pack gathers the A
// row panels and B column panels of every group into contiguous, swizzled
// 16-wide k steps (panel p of group g at pa / pb + p*nst*P*16, P the panel
// width of the group's shape); gemm_f64_ws_launch then runs the groups' tiles
// on them, one producer lane streaming the blocks with bulk copies and four
// consumer warps running the MMAs, consecutive tiles overlapping.
// shape: bit 1 = 32 rows (else 64), bit 0 = 32 columns (else 64)
int gemm_f64_ws_shape(i64 M, i64 N, i64 K);
void gemm_f64_ws_tile(int shape, int& bm, int& bn);
void gemm_f64_ws_pack(const GroupDesc* d_groups, const PackItem* d_items, int nitems, double* packA,
                      double* packB, cudaStream_t stream);
// tile_begin[g] = first tile of group g in tiles of its own shape; d_counter
// as for gemm_f64_grouped_launch
void gemm_f64_ws_launch(const GroupDesc* d_groups, const i64* d_tile_begin, int ngroups, i64 total_tiles,
                        const double* packA, const double* packB, cudaStream_t stream,
                        unsigned long long* d_counter);
// 1 when a kernel of gemm_f64_ws.cu gave up a bounded wait since the last
// call (the flag is cleared by reading it)
int gemm_f64_error_flag();
// test support: the packed GEMM's producer issues no copy for the CTA's
// stage number `step` (-1: none) and every bounded wait gives up after
// wait_seconds (<= 0: the default 2 s)
void gemm_f64_inject_wait_timeout(int step, double wait_seconds);
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
