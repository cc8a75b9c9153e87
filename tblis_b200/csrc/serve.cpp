// serve.cpp -- a continuous-batching contraction server.
//
// Requests (tblis_tensor_mult calls on device-resident operands) are queued
// by tblis_b200_server_submit from any host thread. One scheduler thread
// admits queued requests in arrival order while their operand footprint fits
// the HBM budget, folds every admitted request into one grouped launch of the
// FP64 DMMA kernel and launches it on the next free slot. Each request shape
// (lengths, strides and labels of A, B and C) gets its GEMM view and device
// scatter vectors once; a batch then packs only its descriptors and tile
// prefix table into one pinned buffer, copied with a single transfer. Large
// requests whose tolerance allows it run as Ozaki jobs beside the grouped
// launch, and large FP64 ones as their own launch. Each slot owns a stream,
// so up to `slots` batches run on the GPU at once, and requests that arrive
// while others run are admitted as soon as a slot and budget free up.
// Completion is detected with events; each request records its latency
// (submit to completion).
//
// Each request's result does not depend on the batch it lands in: every
// output tile is computed by one CTA with a fixed k order and a fixed tile
// shape, whatever else runs.
#include "common.hpp"
#include "planner.hpp"
#include "gemm_f64.hpp"
#include "level1.hpp"
#include "mult.hpp"
#include "ozaki.hpp"

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <memory>

namespace tb
{

namespace
{

using clk = std::chrono::steady_clock;

struct Request
{
    int64_t id;
    tblis_tensor A, B, C;
    std::vector<len_type> len[3];
    std::vector<stride_type> stride[3];
    std::string idx[3];
    double tol;
    i64 footprint;                   // bytes of A, B and C counted against the budget
    clk::time_point t_submit, t_done;
    int state = 0;                   // 0 queued, 1 running, 2 done, 3 failed
    int err = 0;
    std::string msg;
};

// The GEMM view of one request shape (lengths, strides and labels of A, B
// and C) and, for the FP64 kernel, its scatter vectors in device memory:
// built once per shape and reused by every later request of that shape.
struct ShapeEntry
{
    GemmView v;
    bool has_tables = false;
    std::vector<i64> host;           // a_l, b_l, c_l (descriptor offsets), kept on the host
    i64 *dev = nullptr;              // a_m, c_m, b_n, c_n, a_k, b_k, a_kbs, b_kbs, a_l, b_l, c_l
    cudaStream_t owner = nullptr;    // stream the device block was allocated on
    const i64 *a_m = nullptr, *c_m = nullptr, *b_n = nullptr, *c_n = nullptr;
    const i64 *a_k = nullptr, *b_k = nullptr, *a_kbs = nullptr, *b_kbs = nullptr;
    const i64 *a_l = nullptr, *b_l = nullptr, *c_l = nullptr;      // into host
    const i64* dev_l[3] = {nullptr, nullptr, nullptr};              // a_l, b_l, c_l on the device
    ~ShapeEntry()
    {
        // the last holder is a finished batch or the server's teardown: no
        // queued kernel reads the block any more
        if (dev) cudaFreeAsync(dev, owner);
    }
};

struct Slot
{
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    cudaEvent_t stats = nullptr;     // Ozaki statistics of the current batch done
    char* hbuf = nullptr;            // pinned staging
    size_t hcap = 0;
    std::vector<char*> old_hbufs;    // outgrown staging, freed with the server (freeing syncs the device)
    char* dbuf_ = nullptr;           // device copy
    size_t dcap = 0;
    std::vector<int64_t> reqs;
    std::vector<std::shared_ptr<ShapeEntry>> shapes;   // held until the batch completes
    bool busy = false;
    i64 footprint = 0;
    unsigned long long* counter = nullptr;   // dynamic tile queue of the grouped launch
};

constexpr int kVariant = 4;          // 64 x 64 tiles: every batch uses the same tile shape
constexpr i64 kDenseTiles = 2*148;   // requests with this many 64x64 tiles run as their own launch

// large contractions whose requested tolerance allows it run on the INT8
// tensor cores (Ozaki slices, slice count chosen from the tolerance)
bool use_ozaki(const GemmView& v, double tol)
{
    return tol >= 1e-13 && v.m >= 256 && v.n >= 256 && v.k >= 512 &&
           2.0*(double)v.m*(double)v.n*(double)v.k*(double)v.l >= 4e9;
}

size_t align_up(size_t x) { return (x + 255) & ~size_t(255); }

} // namespace

struct Server
{
    std::mutex mtx;
    std::condition_variable cv, done_cv;
    std::deque<int64_t> queue;
    std::map<int64_t, std::unique_ptr<Request>> reqs;
    std::vector<Slot> slots;
    std::thread worker;
    bool stop = false;
    int64_t next_id = 1;
    i64 budget = 0, in_use = 0;
    int device = 0;
    int max_batch = 256;
    // request shapes seen so far (scheduler thread only)
    std::unordered_map<std::string, std::shared_ptr<ShapeEntry>> shape_cache;
    static constexpr size_t kShapeCap = 4096;
    // statistics
    int64_t n_done = 0, n_failed = 0, n_batches = 0, batched_requests = 0, n_ozaki = 0;
    int64_t shape_hits = 0, shape_misses = 0;
    int max_running = 0;
    std::vector<double> latencies;
    std::string fatal;

    Server(size_t budget_bytes, int nslots)
    {
        budget = (i64)budget_bytes;
        TB_CUDA(cudaGetDevice(&device));
        slots.resize(std::max(1, nslots));
        for (auto& s : slots)
        {
            TB_CUDA(cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking));
            TB_CUDA(cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming));
            TB_CUDA(cudaMalloc(&s.counter, sizeof(unsigned long long)));
            TB_CUDA(cudaEventCreateWithFlags(&s.stats, cudaEventDisableTiming));
        }
        worker = std::thread([this] { loop(); });
    }

    ~Server()
    {
        {
            std::lock_guard<std::mutex> lk(mtx);
            stop = true;
        }
        cv.notify_all();
        if (worker.joinable()) worker.join();
        for (auto& s : slots)
            if (s.stream) cudaStreamSynchronize(s.stream);
        // shapes free their device blocks in their streams' order
        for (auto& s : slots) s.shapes.clear();
        shape_cache.clear();
        for (auto& s : slots)
        {
            if (s.stream) cudaStreamSynchronize(s.stream);
            if (s.hbuf) cudaFreeHost(s.hbuf);
            for (char* h : s.old_hbufs) cudaFreeHost(h);
            if (s.dbuf_) cudaFreeAsync(s.dbuf_, s.stream);
            if (s.stream) cudaStreamSynchronize(s.stream);
            if (s.done) cudaEventDestroy(s.done);
            if (s.counter) cudaFree(s.counter);
            if (s.stats) cudaEventDestroy(s.stats);
            if (s.stream) cudaStreamDestroy(s.stream);
        }
    }

    int64_t submit(const tblis_tensor* A, const char* ia, const tblis_tensor* B, const char* ib,
                   const tblis_tensor* C, const char* ic, double tol)
    {
        auto r = std::make_unique<Request>();
        const tblis_tensor* in[3] = {A, B, C};
        const char* ix[3] = {ia, ib, ic};
        r->footprint = 0;
        for (int t = 0; t < 3; t++)
        {
            TB_CHECK(in[t] && in[t]->type == TYPE_DOUBLE, TB_ERR_TYPE, "server: double tensors only");
            const unsigned nd = in[t]->ndim;
            r->len[t].assign(in[t]->len, in[t]->len + nd);
            r->stride[t].assign(in[t]->stride, in[t]->stride + nd);
            r->idx[t] = ix[t] ? std::string(ix[t], nd) : std::string();
            i64 lo, hi;
            tensor_extent(nd, in[t]->len, in[t]->stride, lo, hi);
            if (hi >= lo)
            {
                TB_CHECK(pointer_kind(in[t]->data) == MEM_DEVICE, TB_ERR_ARG,
                         "server: operands must be device-resident");
                r->footprint += (hi - lo + 1)*(i64)sizeof(double);
            }
        }
        TB_CHECK(r->footprint <= budget, TB_ERR_BUDGET, "server: request larger than the HBM budget");
        r->A = *A; r->B = *B; r->C = *C;
        r->A.len = r->len[0].data(); r->A.stride = r->stride[0].data();
        r->B.len = r->len[1].data(); r->B.stride = r->stride[1].data();
        r->C.len = r->len[2].data(); r->C.stride = r->stride[2].data();
        r->tol = tol;
        r->t_submit = clk::now();
        std::lock_guard<std::mutex> lk(mtx);
        TB_CHECK(fatal.empty(), TB_ERR_CUDA, "server stopped: " + fatal);
        const int64_t id = next_id++;
        r->id = id;
        reqs[id] = std::move(r);
        queue.push_back(id);
        cv.notify_all();
        return id;
    }

    // 0 done, 1 pending, else the request's error code
    int status(int64_t id, double* latency_ms, bool wait)
    {
        std::unique_lock<std::mutex> lk(mtx);
        auto it = reqs.find(id);
        TB_CHECK(it != reqs.end(), TB_ERR_ARG, "server: unknown request id");
        if (wait)
            done_cv.wait(lk, [&] { return it->second->state >= 2 || !fatal.empty(); });
        Request& r = *it->second;
        if (r.state < 2)
        {
            TB_CHECK(fatal.empty(), TB_ERR_CUDA, "server stopped: " + fatal);
            return 1;
        }
        if (latency_ms)
            *latency_ms = std::chrono::duration<double, std::milli>(r.t_done - r.t_submit).count();
        const int e = r.state == 3 ? (r.err ? r.err : TB_ERR_ARG) : 0;
        if (e) set_last_error(e, r.msg.c_str());
        reqs.erase(it);
        return e;
    }

    // builds one batch into a slot's staging buffer and launches it: requests
    // large enough to fill the GPU run as their own dense launch (with split-K
    // where it pays), the rest are folded into one grouped launch whose tiles
    // are handed out longest-K first
    // the view of a request's shape, from the cache or built now
    std::shared_ptr<ShapeEntry> shape_of(const Request& r)
    {
        std::string key;
        for (int t = 0; t < 3; t++)
        {
            key.append(reinterpret_cast<const char*>(r.len[t].data()), r.len[t].size()*sizeof(len_type));
            key.append(reinterpret_cast<const char*>(r.stride[t].data()), r.stride[t].size()*sizeof(stride_type));
            key += r.idx[t];
            key.push_back('|');
        }
        auto it = shape_cache.find(key);
        if (it != shape_cache.end())
        {
            shape_hits++;
            return it->second;
        }
        shape_misses++;
        auto e = std::make_shared<ShapeEntry>();
        e->v = gemm_view(mult_groups(&r.A, r.idx[0].c_str(), &r.B, r.idx[1].c_str(), &r.C, r.idx[2].c_str()));
        // entries still used by running batches stay alive through the slots
        if (shape_cache.size() >= kShapeCap) shape_cache.clear();
        shape_cache.emplace(std::move(key), e);
        return e;
    }

    // the shape's scatter vectors on the device (built once per shape)
    static void tables_of(ShapeEntry& e, i64 BK, cudaStream_t st)
    {
        if (e.has_tables) return;
        const GemmView& v = e.v;
        const i64 nkb = (v.k + BK - 1)/BK;
        const i64 n = 2*v.m + 2*v.n + 2*v.k + 2*nkb + 3*v.l;
        std::vector<i64> h((size_t)std::max<i64>(n, 1)), bs((size_t)std::max({v.m, v.n, v.k, v.l, (i64)1}) + 1);
        i64* q = h.data();
        i64 *a_m = q; q += v.m;  i64 *c_m = q; q += v.m;
        i64 *b_n = q; q += v.n;  i64 *c_n = q; q += v.n;
        i64 *a_k = q; q += v.k;  i64 *b_k = q; q += v.k;
        i64 *a_kbs = q; q += nkb; i64 *b_kbs = q; q += nkb;
        i64 *a_l = q; q += v.l;  i64 *b_l = q; q += v.l;  i64 *c_l = q;
        fill_block_scatter(v.lenM, v.aM, 1, 0, v.m, a_m, bs.data(), v.pack_m_3d);
        fill_block_scatter(v.lenM, v.cM, 1, 0, v.m, c_m, bs.data(), v.pack_m_3d);
        fill_block_scatter(v.lenN, v.bN, 1, 0, v.n, b_n, bs.data(), v.pack_n_3d);
        fill_block_scatter(v.lenN, v.cN, 1, 0, v.n, c_n, bs.data(), v.pack_n_3d);
        fill_block_scatter(v.lenK, v.aK, 1, 0, v.k, a_k, bs.data(), v.pack_k_3d);
        fill_block_scatter(v.lenK, v.bK, 1, 0, v.k, b_k, bs.data(), v.pack_k_3d);
        // per k block of BK: its common stride, or 0 when the offsets are not affine
        auto kbs = [&](const i64* k, i64* out)
        {
            for (i64 b = 0; b < nkb; b++)
            {
                const i64 i0 = b*BK, bl = std::min(v.k - i0, BK);
                i64 sv = bl > 1 ? k[i0 + 1] - k[i0] : 1;
                for (i64 j = i0 + 1; j + 1 < i0 + bl; j++) if (k[j + 1] - k[j] != sv) sv = 0;
                out[b] = sv;
            }
        };
        kbs(a_k, a_kbs);
        kbs(b_k, b_kbs);
        fill_block_scatter(v.lenL, v.aL, 1, 0, v.l, a_l, bs.data(), false);
        fill_block_scatter(v.lenL, v.bL, 1, 0, v.l, b_l, bs.data(), false);
        fill_block_scatter(v.lenL, v.cL, 1, 0, v.l, c_l, bs.data(), false);
        // the slot's stream is idle here (its previous batch is complete): the
        // copy from pageable memory has the source staged when it returns
        TB_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&e.dev), (size_t)h.size()*sizeof(i64), st));
        e.owner = st;
        TB_CUDA(cudaMemcpyAsync(e.dev, h.data(), h.size()*sizeof(i64), cudaMemcpyHostToDevice, st));
        const i64* d = e.dev;
        auto at = [&](const i64* hp) { return d + (hp - h.data()); };
        e.a_m = at(a_m); e.c_m = at(c_m); e.b_n = at(b_n); e.c_n = at(c_n);
        e.a_k = at(a_k); e.b_k = at(b_k); e.a_kbs = at(a_kbs); e.b_kbs = at(b_kbs);
        e.dev_l[0] = at(a_l); e.dev_l[1] = at(b_l); e.dev_l[2] = at(c_l);
        e.host.assign(a_l, a_l + 3*v.l);
        e.a_l = e.host.data(); e.b_l = e.host.data() + v.l; e.c_l = e.host.data() + 2*v.l;
        e.has_tables = true;
    }

    void launch(Slot& s, std::vector<Request*>& batch)
    {
        cudaStream_t st = s.stream;
        struct Prep
        {
            Request* r;
            GemmView v;
            std::shared_ptr<ShapeEntry> e;
            bool trivial, dense, ozaki;
            double alpha, beta;
        };
        std::vector<Prep> prep;
        size_t ngroups = 0;
        const i64 BK = gemm_f64_tile_k();
        int bm, bn;
        gemm_f64_variant_tile(kVariant, bm, bn);
        for (Request* r : batch)
        {
            try
            {
                std::shared_ptr<ShapeEntry> e = shape_of(*r);
                const GemmView& v = e->v;
                const double alpha = r->A.scalar.data.d*r->B.scalar.data.d, beta = r->C.scalar.data.d;
                const bool trivial = alpha == 0.0 || v.k == 0 || v.m*v.n*v.l == 0;
                const bool ozaki = !trivial && use_ozaki(v, r->tol);
                const bool dense = !trivial && !ozaki &&
                                   ((v.m + bm - 1)/bm)*((v.n + bn - 1)/bn)*v.l >= kDenseTiles;
                if (!trivial && !ozaki)
                {
                    tables_of(*e, BK, st);
                    if (!dense) ngroups += v.l;
                }
                s.shapes.push_back(e);
                prep.push_back({r, v, e, trivial, dense, ozaki, alpha, beta});
            }
            catch (const error& e)
            {
                r->state = 3; r->err = e.code; r->msg = e.what();
            }
        }
        // longest K first in the grouped launch
        std::stable_sort(prep.begin(), prep.end(), [](const Prep& a, const Prep& b) { return a.v.k > b.v.k; });

        // only the descriptors and the tile prefix travel per batch: the
        // scatter vectors of every shape are already on the device
        const size_t desc_bytes = align_up(ngroups*sizeof(GroupDesc));
        const size_t tb_bytes = align_up((ngroups + 1)*sizeof(i64));
        const size_t need = desc_bytes + tb_bytes;
        // growth without a device-wide synchronisation, which would wait for
        // the batches running on the other slots: the outgrown pinned buffer
        // is kept until the server closes, the device buffer is freed and
        // reallocated in this slot's stream order
        if (need > s.hcap)
        {
            if (s.hbuf) s.old_hbufs.push_back(s.hbuf);
            s.hbuf = nullptr;
            s.hcap = std::max(need, 2*s.hcap);
            TB_CUDA(cudaMallocHost(&s.hbuf, s.hcap));
        }
        if (need > s.dcap)
        {
            if (s.dbuf_) TB_CUDA(cudaFreeAsync(s.dbuf_, st));
            s.dbuf_ = nullptr;
            s.dcap = std::max(need, 2*s.dcap);
            TB_CUDA(cudaMallocAsync(&s.dbuf_, s.dcap, st));
        }
        GroupDesc* hdesc = reinterpret_cast<GroupDesc*>(s.hbuf);
        i64* htb = reinterpret_cast<i64*>(s.hbuf + desc_bytes);
        GroupDesc* ddesc = reinterpret_cast<GroupDesc*>(s.dbuf_);
        const i64* dtb = reinterpret_cast<const i64*>(s.dbuf_ + desc_bytes);

        size_t g = 0;
        i64 tiles = 0;
        std::vector<GemmF64Args> dense;
        for (Prep& p : prep)
        {
            const GemmView& v = p.v;
            if (p.r->state == 3) continue;
            if (p.ozaki) continue;
            if (p.trivial)
            {
                if (v.m*v.n*v.l == 0 || p.beta == 1.0) continue;
                Strided sc;
                ivec len, str;
                for (size_t j = 0; j < v.lenM.size(); j++) { len.push_back(v.lenM[j]); str.push_back(v.cM[j]); }
                for (size_t j = 0; j < v.lenN.size(); j++) { len.push_back(v.lenN[j]); str.push_back(v.cN[j]); }
                for (size_t j = 0; j < v.lenL.size(); j++) { len.push_back(v.lenL[j]); str.push_back(v.cL[j]); }
                sc.ndim = (int)len.size();
                for (size_t j = 0; j < len.size(); j++) { sc.len[j] = len[j]; sc.stride[j] = str[j]; }
                if (p.beta == 0.0) l1_set<double>(static_cast<double*>(p.r->C.data), sc, 0.0, st);
                else l1_scale<double>(static_cast<double*>(p.r->C.data), sc, p.beta, st);
                continue;
            }
            const ShapeEntry& e = *p.e;
            if (p.dense)
            {
                GemmF64Args a = {};
                a.A = static_cast<const double*>(p.r->A.data);
                a.B = static_cast<const double*>(p.r->B.data);
                a.C = static_cast<double*>(p.r->C.data);
                a.a_m = e.a_m; a.a_k = e.a_k; a.b_k = e.b_k; a.b_n = e.b_n; a.c_m = e.c_m; a.c_n = e.c_n;
                a.a_l = e.dev_l[0]; a.b_l = e.dev_l[1]; a.c_l = e.dev_l[2];
                a.a_kbs = e.a_kbs; a.b_kbs = e.b_kbs;
                a.M = v.m; a.N = v.n; a.K = v.k; a.L = v.l;
                a.alpha = p.alpha; a.beta = p.beta;
                a.amode = v.amode; a.bmode = v.bmode;
                a.variant = kVariant;
                dense.push_back(a);
                continue;
            }
            for (i64 l = 0; l < v.l; l++)
            {
                GroupDesc& d = hdesc[g];
                d.A = static_cast<const double*>(p.r->A.data) + e.a_l[l];
                d.B = static_cast<const double*>(p.r->B.data) + e.b_l[l];
                d.C = static_cast<double*>(p.r->C.data) + e.c_l[l];
                d.a_m = e.a_m; d.a_k = e.a_k; d.b_k = e.b_k; d.b_n = e.b_n; d.c_m = e.c_m; d.c_n = e.c_n;
                d.a_kbs = e.a_kbs; d.b_kbs = e.b_kbs;
                d.M = v.m; d.N = v.n; d.K = v.k;
                d.alpha = p.alpha; d.beta = p.beta;
                d.amode = v.amode; d.bmode = v.bmode;
                d.nseg = 0; d.segs = nullptr; d.shape = 0; d.nst = 0; d.pa = 0; d.pb = 0;
                htb[g] = tiles;
                tiles += ((v.m + bm - 1)/bm)*((v.n + bn - 1)/bn);
                g++;
            }
        }
        // Ozaki members: statistics first, so the wait below covers only them
        std::vector<std::unique_ptr<OzakiJob>> jobs;
        for (Prep& p : prep)
        {
            if (!p.ozaki || p.r->state == 3) continue;
            auto j = std::make_unique<OzakiJob>();
            j->v = p.v;
            j->A = static_cast<const double*>(p.r->A.data);
            j->B = static_cast<const double*>(p.r->B.data);
            j->C = static_cast<double*>(p.r->C.data);
            j->alpha = p.alpha; j->beta = p.beta; j->tol = p.r->tol;
            ozaki_begin(*j, st);
            jobs.push_back(std::move(j));
        }
        if (!jobs.empty()) TB_CUDA(cudaEventRecord(s.stats, st));
        if (g > 0)
        {
            htb[g] = tiles;
            TB_CUDA(cudaMemcpyAsync(s.dbuf_, s.hbuf, need, cudaMemcpyHostToDevice, st));
        }
        if (g > 0)
            gemm_f64_grouped_launch(ddesc, dtb, (int)g, tiles, kVariant, st, s.counter);
        for (GemmF64Args& a : dense)
        {
            a.splits = gemm_f64_choose_splits(a.M, a.N, a.K, a.L, device_sm_count());
            dbuf ws(gemm_f64_workspace_bytes(a.M, a.N, a.L, a.splits), st);
            a.partial = ws.as<double>();
            gemm_f64_launch(a, st);
        }
        if (!jobs.empty())
        {
            TB_CUDA(cudaEventSynchronize(s.stats));
            for (auto& j : jobs) ozaki_end(*j, st, true);
            std::lock_guard<std::mutex> lk(mtx);
            n_ozaki += (int64_t)jobs.size();
        }
        TB_CUDA(cudaEventRecord(s.done, st));
    }

    void loop()
    {
        cudaSetDevice(device);
        while (true)
        {
            std::vector<Request*> batch;
            Slot* slot = nullptr;
            {
                std::unique_lock<std::mutex> lk(mtx);
                // completions
                for (auto& s : slots)
                {
                    if (!s.busy) continue;
                    cudaError_t q = cudaEventQuery(s.done);
                    if (q == cudaErrorNotReady) continue;
                    const auto now = clk::now();
                    for (int64_t id : s.reqs)
                    {
                        auto it = reqs.find(id);
                        if (it == reqs.end()) continue;
                        Request& r = *it->second;
                        if (r.state == 1)
                        {
                            if (q == cudaSuccess) { r.state = 2; n_done++; }
                            else { r.state = 3; r.err = TB_ERR_CUDA; r.msg = cudaGetErrorString(q); n_failed++; }
                            r.t_done = now;
                            latencies.push_back(std::chrono::duration<double, std::milli>(now - r.t_submit).count());
                        }
                        else if (r.state == 3) { r.t_done = now; n_failed++; }
                    }
                    s.reqs.clear();
                    s.shapes.clear();
                    s.busy = false;
                    in_use -= s.footprint;
                    s.footprint = 0;
                    done_cv.notify_all();
                }
                int running = 0;
                for (auto& s : slots) running += s.busy;
                max_running = std::max(max_running, running);
                if (stop && queue.empty() && running == 0) break;
                // admission: arrival order, while the budget allows
                for (auto& s : slots) if (!s.busy) { slot = &s; break; }
                if (slot && !queue.empty())
                {
                    while (!queue.empty() && (int)batch.size() < max_batch)
                    {
                        Request& r = *reqs[queue.front()];
                        if (in_use + r.footprint > budget) break;
                        in_use += r.footprint;
                        slot->footprint += r.footprint;
                        r.state = 1;
                        batch.push_back(&r);
                        slot->reqs.push_back(r.id);
                        queue.pop_front();
                    }
                }
                if (batch.empty())
                {
                    if (running == 0) cv.wait_for(lk, std::chrono::milliseconds(1));
                    else
                    {
                        lk.unlock();
                        std::this_thread::sleep_for(std::chrono::microseconds(20));
                    }
                    continue;
                }
                slot->busy = true;
            }
            try
            {
                launch(*slot, batch);
                std::lock_guard<std::mutex> lk(mtx);
                n_batches++;
                batched_requests += (int64_t)batch.size();
            }
            catch (const std::exception& e)
            {
                std::lock_guard<std::mutex> lk(mtx);
                fatal = e.what();
                for (Request* r : batch) { r->state = 3; r->err = TB_ERR_CUDA; r->msg = e.what(); }
                cudaEventRecord(slot->done, slot->stream);
                done_cv.notify_all();
            }
        }
    }
};

} // namespace tb

using namespace tb;

extern "C" {

struct tblis_b200_server { Server* s; };

tblis_b200_server* tblis_b200_server_create(size_t hbm_budget_bytes, int slots)
{
    tblis_b200_server* out = nullptr;
    guarded([&]
    {
        ensure_device();
        out = new tblis_b200_server{new Server(hbm_budget_bytes, slots)};
    });
    return out;
}

void tblis_b200_server_destroy(tblis_b200_server* srv)
{
    if (!srv) return;
    delete srv->s;
    delete srv;
}

int64_t tblis_b200_server_submit(tblis_b200_server* srv, const tblis_tensor* A, const label_type* idx_A,
                                 const tblis_tensor* B, const label_type* idx_B,
                                 const tblis_tensor* C, const label_type* idx_C, double tolerance)
{
    int64_t id = -1;
    guarded([&]
    {
        TB_CHECK(srv, TB_ERR_ARG, "null server");
        id = srv->s->submit(A, idx_A, B, idx_B, C, idx_C, tolerance);
    });
    return id;
}

int tblis_b200_server_poll(tblis_b200_server* srv, int64_t id, double* latency_ms)
{
    int r = -1;
    int e = guarded([&] { TB_CHECK(srv, TB_ERR_ARG, "null server"); r = srv->s->status(id, latency_ms, false); });
    return e ? e : r;
}

int tblis_b200_server_wait(tblis_b200_server* srv, int64_t id, double* latency_ms)
{
    int r = -1;
    int e = guarded([&] { TB_CHECK(srv, TB_ERR_ARG, "null server"); r = srv->s->status(id, latency_ms, true); });
    return e ? e : r;
}

int tblis_b200_server_get_stats(tblis_b200_server* srv, tblis_b200_server_stats* out)
{
    return guarded([&]
    {
        TB_CHECK(srv && out, TB_ERR_ARG, "null argument");
        Server& s = *srv->s;
        std::lock_guard<std::mutex> lk(s.mtx);
        memset(out, 0, sizeof(*out));
        out->completed = s.n_done;
        out->failed = s.n_failed;
        out->batches = s.n_batches;
        out->mean_batch = s.n_batches ? (double)s.batched_requests/s.n_batches : 0.0;
        out->max_concurrent_batches = s.max_running;
        out->queued = (int64_t)s.queue.size();
        out->ozaki = s.n_ozaki;
        out->shape_hits = s.shape_hits;
        out->shape_misses = s.shape_misses;
        std::vector<double> l = s.latencies;
        if (!l.empty())
        {
            std::sort(l.begin(), l.end());
            auto pct = [&](double q) { return l[std::min(l.size() - 1, (size_t)(q*(l.size() - 1) + 0.5))]; };
            out->p50_ms = pct(0.50);
            out->p99_ms = pct(0.99);
            out->max_ms = l.back();
        }
    });
}

} // extern "C"
