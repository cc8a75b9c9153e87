// grouped.hpp -- many GEMM views in one persistent launch: plans, the
// tile-shape autotuner and CUDA-graph replay.
#pragma once

#include "planner.hpp"
#include "gemm_f64.hpp"

#include <map>
#include <memory>
#include <mutex>

namespace tb
{

// host scatter vectors of one K segment of a segmented group
struct SegTables
{
    ivec a_m, a_k, b_k, b_n;
};

// host scatter vectors of one group (one GEMM view, one batch index). A
// segmented group (segs non-empty) takes A's rows, B's columns and the k range
// from each segment in turn and ignores a_m, a_k, b_k, b_n, K.
struct GroupTables
{
    std::vector<SegTables> segs;
    ivec a_m, a_k, b_k, b_n, c_m, c_n;
    i64 M = 0, N = 0, K = 0;
    int amode = 0, bmode = 0;
    int a_slot = 0, b_slot = 1, c_slot = 2;   // indices into the run's pointer array
    i64 a_off = 0, b_off = 0, c_off = 0;      // element offsets added to those pointers
    int sidx = 0;                             // index into the run's alpha/beta arrays
    int ws_shape = 0;                         // tile shape of the packed path (finalize)
    int nst = 0;                              // k steps over all segments (finalize)
    i64 pa = 0, pb = 0;                       // offsets of the packed A / B panels (finalize)
};

struct GroupedPlan
{
    std::vector<GroupTables> groups;
    std::vector<std::pair<ivec, ivec>> empty_patches;   // C patches scaled by beta only
    double flops = 0;
    int nslots = 3;

    // device state (finalize)
    i64* d_tables = nullptr;
    std::vector<const i64*> d_ptr;            // per group: a_m, a_k, b_k, b_n, c_m, c_n, a_kbs, b_kbs
    SegDesc* d_segs = nullptr;                // all segments of all groups
    std::vector<i64> seg_begin;               // per group: first entry in d_segs
    std::vector<std::vector<i64>> tile_begin; // per variant (index variant-1)
    std::vector<i64> total_tiles;
    i64* d_tile_begin = nullptr;              // all variants, concatenated
    GroupDesc* d_descs = nullptr;
    unsigned long long* d_counter = nullptr;  // dynamic tile queue
    GroupDesc* h_descs = nullptr;             // pinned
    int variant = 0;                          // tuned tile configuration
    cudaGraphExec_t graph = nullptr;
    bool graph_failed = false;
    cudaEvent_t last_use = nullptr;
    // the pointers and scalars the pinned descriptors were last built from
    std::vector<const double*> last_ptrs;
    std::vector<double> last_scalars;         // alphas, then betas
    bool descs_valid = false;
    i64 c_lo = 0, c_hi = -1;                  // extent of C offsets (for the tuner's scratch)
    // packed path: the panels to pack, the packed sizes (doubles) and the
    // buffer (allocated on first use; A panels, then B panels)
    std::vector<PackItem> pack_items;
    PackItem* d_pack_items = nullptr;
    i64 pack_a = 0, pack_b = 0;
    double* d_pack = nullptr;
    size_t pack_held = 0;                     // bytes of d_pack counted against the cap
    bool pack_failed = false;
    std::string histogram;
    std::vector<std::shared_ptr<GroupedPlan>> parts;   // plans whose groups this one merges (kept alive)

    void finalize(cudaStream_t st);
    ~GroupedPlan();
};

// plan cache keyed by a shape string (LRU)
struct GroupedPlanCache
{
    std::shared_ptr<GroupedPlan> find(const std::string& key);
    std::shared_ptr<GroupedPlan> insert(const std::string& key, std::shared_ptr<GroupedPlan> p);
    std::mutex mtx;
    std::map<std::string, std::shared_ptr<GroupedPlan>> map;
};
GroupedPlanCache& grouped_plan_cache();

// runs every group of the plan: C_g = alphas[sidx_g]*A_g*B_g + betas[sidx_g]*C_g,
// with A_g = ptrs[a_slot] + a_off etc. One launch, graph-replayed.
void grouped_run(GroupedPlan& plan, const double* const* ptrs, const double* alphas, const double* betas,
                 cudaStream_t st);

// C[c_m[i] + c_n[j]] = beta*C[...] (beta == 0: set) for a patch without contracted blocks
void scale_patch(double* C, const ivec& c_m, const ivec& c_n, double beta, cudaStream_t st);

// disables graph capture (debug / environments without graph support)
bool grouped_use_graphs();

} // namespace tb
