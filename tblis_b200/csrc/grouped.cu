// grouped.cu -- grouped GEMM plans: device tables, tile-shape autotuner and
// CUDA-graph replay of the single persistent launch.
//
// Autotuner: the first time a plan with a new group-size histogram (count of
// groups per (log2 M, log2 N, log2 K) bucket) runs, every tile configuration
// of the FP64 DMMA family is timed once on the plan with C redirected to a
// scratch buffer; the fastest is cached under the histogram and reused by
// every plan with the same histogram.
#include "grouped.hpp"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <list>

namespace tb
{

namespace
{

std::mutex g_tune_mtx;
std::map<std::string, int> g_tuned;         // histogram -> variant

std::string histogram_key(const std::vector<GroupTables>& gs)
{
    std::map<std::string, int> h;
    auto b = [](i64 x) { return x <= 1 ? 0 : (int)std::ceil(std::log2((double)x)); };
    for (auto& g : gs) h[std::to_string(b(g.M)) + "," + std::to_string(b(g.N)) + "," + std::to_string(b(g.K))]++;
    std::string k;
    for (auto& kv : h) k += kv.first + ":" + std::to_string(kv.second) + ";";
    return k;
}

__global__ void k_scale_patch(double* C, const i64* cm, const i64* cn, i64 M, i64 N, double beta)
{
    for (i64 e = blockIdx.x*(i64)blockDim.x + threadIdx.x; e < M*N; e += (i64)gridDim.x*blockDim.x)
    {
        const i64 i = e / N, j = e - i*N;
        double* p = C + cm[i] + cn[j];
        *p = beta == 0.0 ? 0.0 : beta*(*p);
    }
}

void block_strides(const ivec& v, ivec& bs, i64 BK)
{
    const i64 n = (i64)v.size();
    const i64 nb = (n + BK - 1)/BK;
    bs.assign(nb, 0);
    for (i64 b = 0; b < nb; b++)
    {
        const i64 i = b*BK;
        const i64 bl = std::min(n - i, BK);
        i64 s = bl > 1 ? v[i + 1] - v[i] : 1;
        for (i64 j = i + 1; j + 1 < i + bl; j++)
            if (v[j + 1] - v[j] != s) s = 0;
        bs[b] = s;
    }
}

} // namespace

bool grouped_use_graphs()
{
    static int v = -1;
    if (v < 0)
    {
        const char* s = getenv("TBLIS_B200_NO_GRAPHS");
        v = (s && s[0] == '1') ? 0 : 1;
    }
    return v == 1;
}

void GroupedPlan::finalize(cudaStream_t st)
{
    const i64 BK = gemm_f64_tile_k();
    for (auto& g : groups)
    {
        i64 K = g.K;
        if (!g.segs.empty())
        {
            K = 0;
            for (auto& sg : g.segs) K += (i64)sg.a_k.size();
        }
        g.ws_shape = gemm_f64_ws_shape(g.M, g.N, K);
    }
    // groups that run the same code (tile shape and gather layouts) together,
    // so a CTA's consecutive tiles stay in the instruction cache; within each
    // such class longest K first: with the dynamic tile queue the longest
    // tiles start first
    auto code_class = [](const GroupTables& g) { return g.ws_shape*4 + g.amode*2 + g.bmode; };
    std::stable_sort(groups.begin(), groups.end(), [&](const GroupTables& a, const GroupTables& b)
    {
        const int ca = code_class(a), cb = code_class(b);
        return ca != cb ? ca < cb : a.K > b.K;
    });
    // device tables: for each group a_m, a_k, b_k, b_n, c_m, c_n, a_kbs, b_kbs,
    // then for each segment a_m, a_k, b_k, b_n, a_kbs, b_kbs
    std::vector<i64> host;
    std::vector<size_t> offs, seg_offs;
    auto put = [&](const ivec& v, std::vector<size_t>& o)
    {
        o.push_back(host.size());
        host.insert(host.end(), v.begin(), v.end());
        if (v.empty()) host.push_back(0);
    };
    for (auto& g : groups)
    {
        ivec akbs, bkbs;
        block_strides(g.a_k, akbs, BK);
        block_strides(g.b_k, bkbs, BK);
        const ivec* vecs[8] = {&g.a_m, &g.a_k, &g.b_k, &g.b_n, &g.c_m, &g.c_n, &akbs, &bkbs};
        for (const ivec* v : vecs) put(*v, offs);
        for (auto& sg : g.segs)
        {
            ivec sa, sb;
            block_strides(sg.a_k, sa, BK);
            block_strides(sg.b_k, sb, BK);
            const ivec* sv[6] = {&sg.a_m, &sg.a_k, &sg.b_k, &sg.b_n, &sa, &sb};
            for (const ivec* v : sv) put(*v, seg_offs);
        }
    }
    // the C extent is the sum of the extreme row and column offsets
    {
        i64 lo = 0, hi = 0;
        for (auto& g : groups)
        {
            i64 mlo = 0, mhi = 0, nlo = 0, nhi = 0;
            if (!g.c_m.empty()) { mlo = *std::min_element(g.c_m.begin(), g.c_m.end()); mhi = *std::max_element(g.c_m.begin(), g.c_m.end()); }
            if (!g.c_n.empty()) { nlo = *std::min_element(g.c_n.begin(), g.c_n.end()); nhi = *std::max_element(g.c_n.begin(), g.c_n.end()); }
            lo = std::min(lo, g.c_off + mlo + nlo);
            hi = std::max(hi, g.c_off + mhi + nhi);
        }
        c_lo = lo; c_hi = hi;
    }
    if (!host.empty())
    {
        TB_CUDA(cudaMalloc(&d_tables, host.size()*sizeof(i64)));
        TB_CUDA(cudaMemcpy(d_tables, host.data(), host.size()*sizeof(i64), cudaMemcpyHostToDevice));
    }
    d_ptr.resize(offs.size());
    for (size_t i = 0; i < offs.size(); i++) d_ptr[i] = d_tables + offs[i];
    // segment descriptors
    std::vector<SegDesc> hs;
    size_t so = 0;
    for (auto& g : groups)
    {
        seg_begin.push_back((i64)hs.size());
        for (auto& sg : g.segs)
        {
            SegDesc d;
            d.a_m = d_tables + seg_offs[so + 0]; d.a_k = d_tables + seg_offs[so + 1];
            d.b_k = d_tables + seg_offs[so + 2]; d.b_n = d_tables + seg_offs[so + 3];
            d.a_kbs = d_tables + seg_offs[so + 4]; d.b_kbs = d_tables + seg_offs[so + 5];
            d.K = (i64)sg.a_k.size();
            so += 6;
            hs.push_back(d);
        }
    }
    if (!hs.empty())
    {
        TB_CUDA(cudaMalloc(&d_segs, hs.size()*sizeof(SegDesc)));
        TB_CUDA(cudaMemcpy(d_segs, hs.data(), hs.size()*sizeof(SegDesc), cudaMemcpyHostToDevice));
    }

    const int nv = gemm_f64_grouped_num_variants();
    tile_begin.assign(nv, {});
    total_tiles.assign(nv, 0);
    std::vector<i64> all;
    for (int v = 1; v <= nv; v++)
    {
        const bool ws = gemm_f64_is_ws_variant(v);
        int bm = 0, bn = 0;
        if (!ws) gemm_f64_variant_tile(v, bm, bn);
        i64 t = 0;
        for (auto& g : groups)
        {
            if (ws) gemm_f64_ws_tile(g.ws_shape, bm, bn);
            tile_begin[v - 1].push_back(t);
            t += ((g.M + bm - 1)/bm)*((g.N + bn - 1)/bn);
        }
        total_tiles[v - 1] = t;
        all.insert(all.end(), tile_begin[v - 1].begin(), tile_begin[v - 1].end());
    }
    if (!all.empty())
    {
        TB_CUDA(cudaMalloc(&d_tile_begin, all.size()*sizeof(i64)));
        TB_CUDA(cudaMemcpy(d_tile_begin, all.data(), all.size()*sizeof(i64), cudaMemcpyHostToDevice));
    }
    // packed path: each group's k steps, its packed panel offsets, and the
    // panels to pack in pieces of at most kPackSteps k steps (so that the few
    // long panels of a large GEMM spread over the whole GPU)
    {
        constexpr i64 kPackSteps = 64;
        pack_a = pack_b = 0;
        pack_items.clear();
        for (size_t gi = 0; gi < groups.size(); gi++)
        {
            GroupTables& g = groups[gi];
            i64 nst = 0;
            if (g.segs.empty()) nst = (g.K + BK - 1)/BK;
            else for (auto& sg : g.segs) nst += ((i64)sg.a_k.size() + BK - 1)/BK;
            TB_CHECK(nst < (1ll << 31), TB_ERR_SIZE, "contracted extent too large");
            g.nst = (int)nst;
            int bm, bn;
            gemm_f64_ws_tile(g.ws_shape, bm, bn);
            const i64 pan_a = (g.M + bm - 1)/bm, pan_b = (g.N + bn - 1)/bn;
            g.pa = pack_a;
            g.pb = pack_b;
            pack_a += pan_a*bm*nst*BK;
            pack_b += pan_b*bn*nst*BK;
            if (nst == 0) continue;
            for (int side = 0; side < 2; side++)
                for (i64 p = 0, np = side ? pan_b : pan_a; p < np; p++)
                    for (i64 s0 = 0; s0 < nst; s0 += kPackSteps)
                        pack_items.push_back({(int)gi, side, (int)p, (int)s0, (int)std::min(kPackSteps, nst - s0), 0});
        }
        TB_CHECK(pack_items.size() < (1ull << 31), TB_ERR_SIZE, "too many panels");
        if (!pack_items.empty())
        {
            TB_CUDA(cudaMalloc(&d_pack_items, pack_items.size()*sizeof(PackItem)));
            TB_CUDA(cudaMemcpy(d_pack_items, pack_items.data(), pack_items.size()*sizeof(PackItem),
                               cudaMemcpyHostToDevice));
        }
    }
    TB_CUDA(cudaMalloc(&d_counter, sizeof(unsigned long long)));
    if (!groups.empty())
    {
        TB_CUDA(cudaMalloc(&d_descs, groups.size()*sizeof(GroupDesc)));
        TB_CUDA(cudaMallocHost(&h_descs, groups.size()*sizeof(GroupDesc)));
    }
    TB_CUDA(cudaEventCreateWithFlags(&last_use, cudaEventDisableTiming));
    histogram = histogram_key(groups);
    (void)st;
}

static void release_pack(GroupedPlan& plan);

GroupedPlan::~GroupedPlan()
{
    if (graph) cudaGraphExecDestroy(graph);
    if (last_use) { cudaEventSynchronize(last_use); cudaEventDestroy(last_use); }
    if (d_tables) cudaFree(d_tables);
    if (d_segs) cudaFree(d_segs);
    if (d_tile_begin) cudaFree(d_tile_begin);
    if (d_descs) cudaFree(d_descs);
    if (d_counter) cudaFree(d_counter);
    if (h_descs) cudaFreeHost(h_descs);
    if (d_pack_items) cudaFree(d_pack_items);
    release_pack(*this);
}

GroupedPlanCache& grouped_plan_cache()
{
    static GroupedPlanCache* c = new GroupedPlanCache();
    return *c;
}

std::shared_ptr<GroupedPlan> GroupedPlanCache::find(const std::string& key)
{
    std::lock_guard<std::mutex> lk(mtx);
    auto it = map.find(key);
    return it == map.end() ? nullptr : it->second;
}

std::shared_ptr<GroupedPlan> GroupedPlanCache::insert(const std::string& key, std::shared_ptr<GroupedPlan> p)
{
    std::lock_guard<std::mutex> lk(mtx);
    if (map.size() >= 256)
    {
        cudaDeviceSynchronize();
        map.clear();
    }
    map[key] = p;
    return p;
}

static void fill_descs(GroupedPlan& plan, GroupDesc* out, const double* const* ptrs, const double* alphas,
                       const double* betas, double* c_override)
{
    for (size_t i = 0; i < plan.groups.size(); i++)
    {
        const GroupTables& g = plan.groups[i];
        GroupDesc& d = out[i];
        d.A = ptrs[g.a_slot] + g.a_off;
        d.B = ptrs[g.b_slot] + g.b_off;
        d.C = c_override ? c_override : const_cast<double*>(ptrs[g.c_slot]) + g.c_off;
        d.a_m = plan.d_ptr[8*i + 0]; d.a_k = plan.d_ptr[8*i + 1];
        d.b_k = plan.d_ptr[8*i + 2]; d.b_n = plan.d_ptr[8*i + 3];
        d.c_m = plan.d_ptr[8*i + 4]; d.c_n = plan.d_ptr[8*i + 5];
        d.a_kbs = plan.d_ptr[8*i + 6]; d.b_kbs = plan.d_ptr[8*i + 7];
        d.M = g.M; d.N = g.N; d.K = g.K;
        d.alpha = alphas[g.sidx]; d.beta = betas[g.sidx];
        d.amode = g.amode; d.bmode = g.bmode;
        d.nseg = (int)g.segs.size();
        d.segs = g.segs.empty() ? nullptr : plan.d_segs + plan.seg_begin[i];
        d.shape = g.ws_shape;
        d.nst = g.nst;
        d.pa = g.pa;
        d.pb = g.pb;
    }
}

static const i64* variant_tile_begin(GroupedPlan& plan, int v)
{
    return plan.d_tile_begin + (size_t)(v - 1)*plan.groups.size();
}

// device memory held by the packed-panel buffers of all live plans, and its
// cap: 40% of the device's memory, so that cached plans never crowd out the
// caller's own allocations
static std::atomic<size_t> g_pack_held{0};

static size_t pack_cap()
{
    static size_t cap = 0;
    if (!cap)
    {
        size_t freeb = 0, total = 0;
        cap = cudaMemGetInfo(&freeb, &total) == cudaSuccess ? total/10*4 : ((size_t)8 << 30);
    }
    return cap;
}

static void release_pack(GroupedPlan& plan)
{
    if (!plan.d_pack) return;
    cudaFree(plan.d_pack);
    plan.d_pack = nullptr;
    g_pack_held -= plan.pack_held;
    plan.pack_held = 0;
}

// the packed panels' buffer, allocated on the packed path's first use; false
// (and the path is not used for this plan) when it would pass the cap or the
// device has no room
static bool ensure_pack(GroupedPlan& plan)
{
    if (plan.d_pack) return true;
    if (plan.pack_failed) return false;
    const size_t bytes = (size_t)std::max<i64>(plan.pack_a + plan.pack_b, 1)*sizeof(double);
    if (g_pack_held.load() + bytes > pack_cap() || cudaMalloc(&plan.d_pack, bytes) != cudaSuccess)
    {
        cudaGetLastError();
        plan.d_pack = nullptr;
        plan.pack_failed = true;
        return false;
    }
    plan.pack_held = bytes;
    g_pack_held += bytes;
    return true;
}

// one run of variant v of the plan on the descriptors descs
static void launch_variant(GroupedPlan& plan, const GroupDesc* descs, int v, cudaStream_t st)
{
    const int ng = (int)plan.groups.size();
    if (gemm_f64_is_ws_variant(v))
    {
        TB_CHECK(plan.d_pack, TB_ERR_ARG, "packed path without its buffer");
        gemm_f64_ws_pack(descs, plan.d_pack_items, (int)plan.pack_items.size(), plan.d_pack,
                         plan.d_pack + plan.pack_a, st);
        gemm_f64_ws_launch(descs, variant_tile_begin(plan, v), ng, plan.total_tiles[v - 1], plan.d_pack,
                           plan.d_pack + plan.pack_a, st, plan.d_counter);
    }
    else
        gemm_f64_grouped_launch(descs, variant_tile_begin(plan, v), ng, plan.total_tiles[v - 1], v, st,
                                plan.d_counter);
}

static int autotune(GroupedPlan& plan, const double* const* ptrs, const double* alphas, const double* betas,
                    cudaStream_t st)
{
    {
        std::lock_guard<std::mutex> lk(g_tune_mtx);
        auto it = g_tuned.find(plan.histogram);
        if (it != g_tuned.end()) return it->second;
    }
    const char* env = getenv("TBLIS_B200_GEMM_VARIANT");
    if (env && atoi(env) >= 1 && atoi(env) <= gemm_f64_grouped_num_variants() &&
        (!gemm_f64_is_ws_variant(atoi(env)) || ensure_pack(plan)))
        return atoi(env);

    // scratch C covering the offsets of every group: candidates write there
    const i64 span = plan.c_hi - plan.c_lo + 1;
    dbuf scratch((size_t)std::max<i64>(span, 1)*sizeof(double), st);
    TB_CUDA(cudaMemsetAsync(scratch.ptr, 0, (size_t)std::max<i64>(span, 1)*sizeof(double), st));
    std::vector<GroupDesc> hd(plan.groups.size());
    fill_descs(plan, hd.data(), ptrs, alphas, betas, scratch.as<double>() - plan.c_lo);
    for (size_t i = 0; i < hd.size(); i++) hd[i].C = scratch.as<double>() - plan.c_lo + plan.groups[i].c_off;
    dbuf dd(hd.size()*sizeof(GroupDesc), st);
    TB_CUDA(cudaMemcpyAsync(dd.ptr, hd.data(), hd.size()*sizeof(GroupDesc), cudaMemcpyHostToDevice, st));
    cudaEvent_t e0, e1;
    TB_CUDA(cudaEventCreate(&e0));
    TB_CUDA(cudaEventCreate(&e1));
    int best = 1;
    float best_ms = 1e30f;
    for (int v = 1; v <= gemm_f64_grouped_num_variants(); v++)
    {
        if (gemm_f64_is_ws_variant(v) && !ensure_pack(plan)) continue;
        launch_variant(plan, dd.as<GroupDesc>(), v, st);     // warm-up
        TB_CUDA(cudaEventRecord(e0, st));
        launch_variant(plan, dd.as<GroupDesc>(), v, st);
        TB_CUDA(cudaEventRecord(e1, st));
        TB_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        TB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        if (ms < best_ms) { best_ms = ms; best = v; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    // the timed launches are complete (event synchronised): give the room back
    if (!gemm_f64_is_ws_variant(best)) release_pack(plan);
    std::lock_guard<std::mutex> lk(g_tune_mtx);
    g_tuned[plan.histogram] = best;
    return best;
}

void grouped_run(GroupedPlan& plan, const double* const* ptrs, const double* alphas, const double* betas,
                 cudaStream_t st)
{
    if (plan.groups.empty()) return;
    if (plan.variant == 0)
    {
        plan.variant = autotune(plan, ptrs, alphas, betas, st);
        // a variant tuned on another plan of the same shape histogram: the
        // packed path needs this plan's buffer too
        if (gemm_f64_is_ws_variant(plan.variant) && !ensure_pack(plan)) plan.variant = 4;
    }
    const int v = plan.variant;

    // The descriptors depend only on the run's pointers and scalars. A run
    // with the same ones as the last (an iterative solver's repeated step)
    // reuses them as they are, without waiting for the previous launch.
    // Otherwise the pinned descriptor buffer is read by the previous launch:
    // wait for it, then rebuild.
    int nsc = 0;
    for (auto& g : plan.groups) nsc = std::max(nsc, g.sidx + 1);
    const bool same = plan.descs_valid && (int)plan.last_ptrs.size() == plan.nslots &&
                      (int)plan.last_scalars.size() == 2*nsc &&
                      std::equal(ptrs, ptrs + plan.nslots, plan.last_ptrs.begin()) &&
                      std::equal(alphas, alphas + nsc, plan.last_scalars.begin()) &&
                      std::equal(betas, betas + nsc, plan.last_scalars.begin() + nsc);
    if (!same)
    {
        TB_CUDA(cudaEventSynchronize(plan.last_use));
        fill_descs(plan, plan.h_descs, ptrs, alphas, betas, nullptr);
        plan.last_ptrs.assign(ptrs, ptrs + plan.nslots);
        plan.last_scalars.assign(alphas, alphas + nsc);
        plan.last_scalars.insert(plan.last_scalars.end(), betas, betas + nsc);
        plan.descs_valid = true;
    }

    if (grouped_use_graphs() && !plan.graph_failed)
    {
        if (!plan.graph)
        {
            cudaStream_t cs;
            TB_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
            cudaGraph_t g;
            TB_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
            cudaError_t e1 = cudaMemcpyAsync(plan.d_descs, plan.h_descs, plan.groups.size()*sizeof(GroupDesc),
                                             cudaMemcpyHostToDevice, cs);
            bool ok = e1 == cudaSuccess;
            if (ok)
            {
                try
                {
                    launch_variant(plan, plan.d_descs, v, cs);
                }
                catch (const error&) { ok = false; }
            }
            cudaError_t e2 = cudaStreamEndCapture(cs, &g);
            cudaStreamDestroy(cs);
            if (ok && e2 == cudaSuccess && cudaGraphInstantiate(&plan.graph, g, 0) == cudaSuccess)
                cudaGraphDestroy(g);
            else
            {
                // capture unavailable here: run the launch directly from now on
                if (e2 == cudaSuccess) cudaGraphDestroy(g);
                cudaGetLastError();
                plan.graph = nullptr;
                plan.graph_failed = true;
            }
        }
    }
    if (plan.graph)
    {
        const bool ws = gemm_f64_is_ws_variant(v);
        TimedLaunch t(ws ? "gemm_f64_pack_kernel+gemm_f64_ws_kernel" : "gemm_f64_grouped_kernel", st);
        TB_CUDA(cudaGraphLaunch(plan.graph, st));
        count_launch();
        if (ws) count_launch();             // the pack kernel and the GEMM kernel
    }
    else
    {
        TB_CUDA(cudaMemcpyAsync(plan.d_descs, plan.h_descs, plan.groups.size()*sizeof(GroupDesc),
                                cudaMemcpyHostToDevice, st));
        launch_variant(plan, plan.d_descs, v, st);
    }
    TB_CUDA(cudaEventRecord(plan.last_use, st));
}

void scale_patch(double* C, const ivec& c_m, const ivec& c_n, double beta, cudaStream_t st)
{
    if (beta == 1.0 || c_m.empty() || c_n.empty()) return;
    dbuf d((c_m.size() + c_n.size())*sizeof(i64), st);
    std::vector<i64> h(c_m.begin(), c_m.end());
    h.insert(h.end(), c_n.begin(), c_n.end());
    TB_CUDA(cudaMemcpyAsync(d.ptr, h.data(), h.size()*sizeof(i64), cudaMemcpyHostToDevice, st));
    TB_CUDA(cudaStreamSynchronize(st));     // h dies at return
    const i64 M = (i64)c_m.size(), N = (i64)c_n.size();
    const int blocks = (int)std::min<i64>((M*N + 255)/256, 148*8);
    k_scale_patch<<<blocks, 256, 0, st>>>(C, d.as<i64>(), d.as<i64>() + M, M, N, beta);
    check_launch("k_scale_patch");
}

} // namespace tb
