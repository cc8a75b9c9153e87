// planner.cpp -- see planner.hpp. Paths cited are relative to the TBLIS tree.
#include "planner.hpp"

#include <algorithm>
#include <cstring>
#include <list>
#include <mutex>
#include <numeric>
#include <unordered_map>

namespace tb
{

void diagonal(unsigned ndim, const len_type* len, const stride_type* stride, const char* idx,
              ivec& len_out, ivec& stride_out, std::string& idx_out)
{
    len_out.clear(); stride_out.clear(); idx_out.clear();
    std::vector<unsigned> inds(ndim);
    std::iota(inds.begin(), inds.end(), 0u);
    std::sort(inds.begin(), inds.end(), [&](unsigned i, unsigned j) { return idx[i] < idx[j]; });

    for (unsigned i = 0; i < ndim; i++)
    {
        if (i == 0 || idx[inds[i]] != idx[inds[i-1]])
        {
            if (len[inds[i]] != 1)
            {
                len_out.push_back(len[inds[i]]);
                stride_out.push_back(stride[inds[i]]);
                idx_out.push_back(idx[inds[i]]);
            }
        }
        else if (len[inds[i]] != 1)
        {
            TB_CHECK(!len_out.empty() && len_out.back() == len[inds[i]], TB_ERR_ARG,
                     "repeated label with different lengths");
            stride_out.back() += stride[inds[i]];
        }
    }
}

std::vector<unsigned> sort_by_stride(const std::vector<const ivec*>& strides)
{
    size_t n = strides.empty() ? 0 : strides[0]->size();
    std::vector<unsigned> perm(n);
    std::iota(perm.begin(), perm.end(), 0u);
    std::sort(perm.begin(), perm.end(), [&](unsigned i, unsigned j)
    {
        i64 mi = (*strides[0])[i], mj = (*strides[0])[j];
        for (size_t k = 1; k < strides.size(); k++)
        {
            mi = std::min(mi, (*strides[k])[i]);
            mj = std::min(mj, (*strides[k])[j]);
        }
        if (mi < mj) return true;
        if (mi > mj) return false;
        for (size_t k = 0; k < strides.size(); k++)
        {
            i64 si = (*strides[k])[i], sj = (*strides[k])[j];
            if (si < sj) return true;
            if (si > sj) return false;
        }
        return false;
    });
    return perm;
}

void fold(ivec& len, std::string& idx, const std::vector<ivec*>& strides)
{
    size_t ndim = len.size();
    auto inds = sort_by_stride({strides[0]});
    ivec oldlen; oldlen.swap(len);
    std::string oldidx; oldidx.swap(idx);
    std::vector<ivec> olds(strides.size());
    for (size_t k = 0; k < strides.size(); k++) { olds[k].swap(*strides[k]); }

    for (size_t i = 0; i < ndim; i++)
    {
        bool contig = i != 0;
        for (size_t k = 0; contig && k < strides.size(); k++)
            if (olds[k][inds[i]] != olds[k][inds[i-1]]*oldlen[inds[i-1]]) contig = false;
        if (contig)
        {
            len.back() *= oldlen[inds[i]];
        }
        else
        {
            idx.push_back(oldidx[inds[i]]);
            len.push_back(oldlen[inds[i]]);
            for (size_t k = 0; k < strides.size(); k++) strides[k]->push_back(olds[k][inds[i]]);
        }
    }
}

char free_idx(std::string s)
{
    if (s.empty()) return 0;
    std::sort(s.begin(), s.end());
    if (s[0] > 0) return 0;
    for (size_t i = 1; i < s.size(); i++)
        if (s[i] > s[i-1]+1) return (char)(s[i-1]+1);
    return (char)(s.back()+1);
}

static i64 gcd64(i64 a, i64 b)
{
    a = a < 0 ? -a : a; b = b < 0 ? -b : b;
    while (b) { i64 t = a % b; a = b; b = t; }
    return a;
}

// offset of linear position p over (len, stride), first dim fastest
static i64 offset_at(const i64* len, const i64* stride, size_t n, i64 p)
{
    i64 off = 0;
    for (size_t i = 0; i < n; i++) { off += (p % len[i])*stride[i]; p /= len[i]; }
    return off;
}

void fill_block_scatter(const ivec& len, const ivec& stride, i64 BS, i64 off, i64 size,
                        i64* scat, i64* bs, bool pack_3d)
{
    if (size == 0) return;
    const i64 CL = 64/sizeof(double);

    if (len.empty())
    {
        *scat = 0;
    }
    else if (!pack_3d)
    {
        i64 m0 = len[0], s0 = stride[0];
        size_t n1 = len.size()-1;
        i64 nouter = 1;
        for (size_t i = 1; i < len.size(); i++) nouter *= len[i];
        i64 p0 = off % m0, b = off / m0, idx = 0;
        for (; idx < size && b < nouter; b++)
        {
            i64 pos = offset_at(len.data()+1, stride.data()+1, n1, b) + p0*s0;
            i64 imax = std::min(m0-p0, size-idx);
            for (i64 i = 0; i < imax; i++) { scat[idx++] = pos; pos += s0; }
            p0 = 0;
        }
    }
    else
    {
        TB_CHECK(len.size() >= 2, TB_ERR_ARG, "3-D scatter needs two dimensions");
        i64 m0 = len[0], s0 = stride[0], m1 = len[1], s1 = stride[1];
        i64 BS0 = std::min(BS*CL/gcd64(BS, CL), std::max(BS, m0 - m0%BS));
        i64 BS1 = std::min(CL, std::max(BS, m1 - m1%BS));
        size_t n2 = len.size()-2;
        i64 nouter = 1;
        for (size_t i = 2; i < len.size(); i++) nouter *= len[i];

        i64 p01 = off % (m0*m1), p0 = p01 % m0, p1 = p01 / m0;
        i64 q01 = (off+size-1) % (m0*m1), q0 = q01 % m0, q1 = q01 / m0;
        i64 r0 = q0 - q0 % BS0;
        i64 b_min = off/(m0*m1), b_max = (off+size-1)/(m0*m1)+1;
        if (p0 == 0) p1--;
        if (q0 == m0-1) q1++;

        i64 idx = 0;
        if (r0 > 0)
        {
            for (i64 b = b_min; b < b_max && b < nouter; b++)
            {
                i64 pos = offset_at(len.data()+2, stride.data()+2, n2, b);
                i64 min1 = b == b_min ? p1+1 : 0;
                i64 max1 = b == b_max-1 ? q1 : m1;
                for (i64 i1 = min1; i1 < max1; i1 += BS1)
                for (i64 i0 = 0; i0 < r0; i0 += BS0)
                for (i64 j1 = 0; j1 < std::min(BS1, max1-i1); j1++)
                for (i64 j0 = 0; j0 < BS0; j0++)
                    scat[idx++] = pos + (i0+j0)*s0 + (i1+j1)*s1;
            }
        }
        for (i64 b = b_min; b < b_max && b < nouter; b++)
        {
            i64 pos = offset_at(len.data()+2, stride.data()+2, n2, b);
            i64 min1 = b == b_min ? p1+1 : 0;
            i64 max1 = b == b_max-1 ? q1 : m1;
            for (i64 j1 = min1; j1 < max1; j1++)
            for (i64 j0 = r0; j0 < m0; j0++)
                scat[idx++] = pos + j0*s0 + j1*s1;
            bool do_p = b == b_min && p0 > 0;
            bool do_q = b == b_max-1 && q0 < m0-1;
            if (do_p && do_q && p1 == q1)
            {
                for (i64 j0 = p0; j0 <= q0; j0++) scat[idx++] = pos + j0*s0 + p1*s1;
            }
            else
            {
                if (do_p) for (i64 j0 = p0; j0 < m0; j0++) scat[idx++] = pos + j0*s0 + p1*s1;
                if (do_q) for (i64 j0 = 0; j0 <= q0; j0++) scat[idx++] = pos + j0*s0 + q1*s1;
            }
        }
        TB_CHECK(idx == size, TB_ERR_ARG, "3-D scatter size mismatch");
    }

    // block strides (src/matrix/block_scatter_matrix.hpp:232-247)
    for (i64 i = 0; i < size; i += BS)
    {
        i64 bl = std::min(size-i, BS);
        i64 s = bl > 1 ? scat[i+1]-scat[i] : 1;
        for (i64 j = i+1; j+1 < i+bl; j++)
            if (scat[j+1]-scat[j] != s) s = 0;
        bs[i] = s;
    }
}

// ---- group split -----------------------------------------------------------

static std::string sorted_unique(std::string s)
{
    std::sort(s.begin(), s.end());
    s.erase(std::unique(s.begin(), s.end()), s.end());
    return s;
}

static std::string intersect(const std::string& a, const std::string& b)
{
    std::string r;
    for (char c : sorted_unique(a)) if (b.find(c) != std::string::npos) r.push_back(c);
    return r;
}

static std::string exclude(const std::string& a, const std::string& b)
{
    std::string r;
    for (char c : sorted_unique(a)) if (b.find(c) == std::string::npos) r.push_back(c);
    return r;
}

static ivec select_from(const ivec& v, const std::string& lab, const std::string& match)
{
    ivec r;
    for (char c : match) r.push_back(v[lab.find(c)]);
    return r;
}

MultGroups mult_groups(const tblis_tensor* A, const char* idx_A,
                       const tblis_tensor* B, const char* idx_B,
                       const tblis_tensor* C, const char* idx_C)
{
    TB_CHECK(A && B && C, TB_ERR_ARG, "null tensor");
    TB_CHECK(A->ndim == 0 || idx_A, TB_ERR_ARG, "null label string");
    TB_CHECK(B->ndim == 0 || idx_B, TB_ERR_ARG, "null label string");
    TB_CHECK(C->ndim == 0 || idx_C, TB_ERR_ARG, "null label string");
    ivec lA, lB, lC, sA, sB, sC;
    std::string iA, iB, iC;
    diagonal(A->ndim, A->len, A->stride, idx_A, lA, sA, iA);
    diagonal(B->ndim, B->len, B->stride, idx_B, lB, sB, iB);
    diagonal(C->ndim, C->len, C->stride, idx_C, lC, sC, iC);

    size_t nabc = intersect(intersect(iA, iB), iC).size();
    if (iA.size() == nabc || iB.size() == nabc || iC.size() == nabc)
    {
        lA.push_back(1); lB.push_back(1); lC.push_back(1); lC.push_back(1);
        sA.push_back(0); sB.push_back(0); sC.push_back(0); sC.push_back(0);
        char f = free_idx(iA + iB + iC);
        iA.push_back(f); iC.push_back(f);
        f = free_idx(iA + iB + iC);
        iB.push_back(f); iC.push_back(f);
    }

    MultGroups g;
    g.ABC = intersect(intersect(iA, iB), iC);
    g.AB = exclude(intersect(iA, iB), g.ABC);
    g.AC = exclude(intersect(iA, iC), g.ABC);
    g.BC = exclude(intersect(iB, iC), g.ABC);

    TB_CHECK(exclude(exclude(exclude(iA, g.AB), g.AC), g.ABC).empty(), TB_ERR_ARG,
             "label appears only in A");
    TB_CHECK(exclude(exclude(exclude(iB, g.AB), g.BC), g.ABC).empty(), TB_ERR_ARG,
             "label appears only in B");
    TB_CHECK(exclude(exclude(exclude(iC, g.AC), g.BC), g.ABC).empty(), TB_ERR_ARG,
             "label appears only in C");

    g.len_ABC = select_from(lA, iA, g.ABC);
    TB_CHECK(g.len_ABC == select_from(lB, iB, g.ABC) && g.len_ABC == select_from(lC, iC, g.ABC),
             TB_ERR_ARG, "mismatched lengths of a batch label");
    g.sA_ABC = select_from(sA, iA, g.ABC);
    g.sB_ABC = select_from(sB, iB, g.ABC);
    g.sC_ABC = select_from(sC, iC, g.ABC);

    g.len_AB = select_from(lA, iA, g.AB);
    TB_CHECK(g.len_AB == select_from(lB, iB, g.AB), TB_ERR_ARG, "mismatched contracted lengths");
    g.sA_AB = select_from(sA, iA, g.AB);
    g.sB_AB = select_from(sB, iB, g.AB);

    g.len_AC = select_from(lA, iA, g.AC);
    TB_CHECK(g.len_AC == select_from(lC, iC, g.AC), TB_ERR_ARG, "mismatched row lengths");
    g.sA_AC = select_from(sA, iA, g.AC);
    g.sC_AC = select_from(sC, iC, g.AC);

    g.len_BC = select_from(lB, iB, g.BC);
    TB_CHECK(g.len_BC == select_from(lC, iC, g.BC), TB_ERR_ARG, "mismatched column lengths");
    g.sB_BC = select_from(sB, iB, g.BC);
    g.sC_BC = select_from(sC, iC, g.BC);

    fold(g.len_ABC, g.ABC, {&g.sA_ABC, &g.sB_ABC, &g.sC_ABC});
    fold(g.len_AB, g.AB, {&g.sA_AB, &g.sB_AB});
    fold(g.len_AC, g.AC, {&g.sA_AC, &g.sC_AC});
    fold(g.len_BC, g.BC, {&g.sB_BC, &g.sC_BC});
    return g;
}

// src/util/tensor.hpp:484-491
static unsigned unit_dim(const ivec& stride, const std::vector<unsigned>& reorder)
{
    for (unsigned i = 0; i < reorder.size(); i++)
        if (stride[reorder[i]] == 1) return i;
    return (unsigned)reorder.size();
}

template <typename V>
static V permuted(const V& v, const std::vector<unsigned>& p)
{
    V r;
    for (unsigned i : p) r.push_back(v[i]);
    return r;
}

GemmView gemm_view(const MultGroups& g)
{
    auto reorder_AC = sort_by_stride({&g.sC_AC, &g.sA_AC});
    auto reorder_BC = sort_by_stride({&g.sC_BC, &g.sB_BC});
    auto reorder_AB = sort_by_stride({&g.sA_AB, &g.sB_AB});
    auto reorder_ABC = sort_by_stride({&g.sC_ABC, &g.sA_ABC, &g.sB_ABC});

    unsigned unit_A_AC = unit_dim(g.sA_AC, reorder_AC);
    unsigned unit_B_BC = unit_dim(g.sB_BC, reorder_BC);
    unsigned unit_A_AB = unit_dim(g.sA_AB, reorder_AB);
    unsigned unit_B_AB = unit_dim(g.sB_AB, reorder_AB);

    GemmView v;
    v.pack_m_3d = unit_A_AC > 0 && unit_A_AC < g.AC.size();
    v.pack_n_3d = unit_B_BC > 0 && unit_B_BC < g.BC.size();
    v.pack_k_3d = (unit_A_AB > 0 && unit_A_AB < g.AB.size()) ||
                  (unit_B_AB > 0 && unit_B_AB < g.AB.size());

    if (v.pack_m_3d)
        std::rotate(reorder_AC.begin()+1, reorder_AC.begin()+unit_A_AC, reorder_AC.end());
    if (v.pack_n_3d)
        std::rotate(reorder_BC.begin()+1, reorder_BC.begin()+unit_B_BC, reorder_BC.end());
    if (v.pack_k_3d)
        std::rotate(reorder_AB.begin()+1, reorder_AB.begin()+std::max(unit_A_AB, unit_B_AB),
                    reorder_AB.end());

    v.idxM = permuted(g.AC, reorder_AC); v.lenM = permuted(g.len_AC, reorder_AC);
    v.aM = permuted(g.sA_AC, reorder_AC); v.cM = permuted(g.sC_AC, reorder_AC);
    v.idxN = permuted(g.BC, reorder_BC); v.lenN = permuted(g.len_BC, reorder_BC);
    v.bN = permuted(g.sB_BC, reorder_BC); v.cN = permuted(g.sC_BC, reorder_BC);
    v.idxK = permuted(g.AB, reorder_AB); v.lenK = permuted(g.len_AB, reorder_AB);
    v.aK = permuted(g.sA_AB, reorder_AB); v.bK = permuted(g.sB_AB, reorder_AB);
    v.idxL = permuted(g.ABC, reorder_ABC); v.lenL = permuted(g.len_ABC, reorder_ABC);
    v.aL = permuted(g.sA_ABC, reorder_ABC); v.bL = permuted(g.sB_ABC, reorder_ABC);
    v.cL = permuted(g.sC_ABC, reorder_ABC);

    v.m = v.n = v.k = v.l = 1;
    for (i64 x : v.lenM) v.m *= x;
    for (i64 x : v.lenN) v.n *= x;
    for (i64 x : v.lenK) v.k *= x;
    for (i64 x : v.lenL) v.l *= x;

    // gather direction: along whichever GEMM dimension has the smaller
    // leading stride in the operand (ties prefer k, which is the inner loop)
    auto lead = [](const ivec& s) { return s.empty() ? (i64)1 << 62 : std::llabs(s[0]); };
    v.amode = lead(v.aM) < lead(v.aK) ? 0 : 1;
    v.bmode = lead(v.bN) < lead(v.bK) ? 0 : 1;
    return v;
}

// ---- device tables and plan cache ---------------------------------------------

GemmTables::~GemmTables()
{
    if (dev) cudaFree(dev);
}

namespace
{
struct TableCache
{
    std::mutex mtx;
    std::list<std::string> lru;
    std::unordered_map<std::string, std::pair<std::shared_ptr<GemmTables>,
                                              std::list<std::string>::iterator>> map;
    size_t capacity = 512;
    // evicted tables: kernels queued before their last holder let go of them
    // may still read them, so they are freed in batches after a device
    // synchronisation, never one synchronisation per eviction (which would
    // stall every other stream's caller, e.g. a server's other slots)
    std::vector<std::shared_ptr<GemmTables>> retired;
    size_t retired_bytes = 0;
};

TableCache& table_cache()
{
    static TableCache* c = new TableCache();   // never destroyed: outlives CUDA teardown
    return *c;
}

void append_key(std::string& key, const ivec& v)
{
    key.append(reinterpret_cast<const char*>(v.data()), v.size()*sizeof(i64));
    key.push_back('|');
}
}

// s when t[i] == i*s for every i < n, else -1
static i64 affine_step(const i64* t, i64 n)
{
    if (n == 0) return 0;
    const i64 s = n > 1 ? t[1] : 0;
    for (i64 i = 0; i < n; i++)
        if (t[i] != i*s) return -1;
    return s;
}

// fraction of index pairs (2i, 2i+1) adjacent in memory with an even first
// offset, and fraction of even offsets
static void pair_stats(const i64* t, i64 n, double& adj, double& even)
{
    i64 a = 0, e = 0;
    for (i64 i = 0; i + 1 < n; i += 2) a += t[i + 1] == t[i] + 1 && (t[i] & 1) == 0;
    for (i64 i = 0; i < n; i++) e += (t[i] & 1) == 0;
    adj = n > 1 ? (double)a/(double)(n/2) : 0.0;
    even = n > 0 ? (double)e/(double)n : 0.0;
}

void gemm_pair_modes(const GemmView& v, const i64* a_m, const i64* a_k, const i64* b_n, const i64* b_k,
                     const i64* a_l, const i64* b_l, bool a_pairs[2], bool b_pairs[2])
{
    double am_adj, am_even, ak_adj, ak_even, bn_adj, bn_even, bk_adj, bk_even, l_adj, l_even_a, l_even_b;
    pair_stats(a_m, v.m, am_adj, am_even); pair_stats(a_k, v.k, ak_adj, ak_even);
    pair_stats(b_n, v.n, bn_adj, bn_even); pair_stats(b_k, v.k, bk_adj, bk_even);
    pair_stats(a_l, v.l, l_adj, l_even_a); pair_stats(b_l, v.l, l_adj, l_even_b);
    const double q = 0.9;
    const bool la = l_even_a == 1.0, lb = l_even_b == 1.0;
    a_pairs[0] = la && am_adj >= q && ak_even >= q;
    a_pairs[1] = la && ak_adj >= q && am_even >= q;
    b_pairs[0] = lb && bn_adj >= q && bk_even >= q;
    b_pairs[1] = lb && bk_adj >= q && bn_even >= q;
}

std::shared_ptr<GemmTables> gemm_tables(const GemmView& v, i64 BM, i64 BN, i64 BK,
                                        cudaStream_t stream)
{
    int dev = 0;
    TB_CUDA(cudaGetDevice(&dev));
    std::string key;
    ivec head = {dev, BM, BN, BK, v.pack_m_3d, v.pack_n_3d, v.pack_k_3d};
    for (const ivec* p : std::initializer_list<const ivec*>{&head, &v.lenM, &v.lenN, &v.lenK, &v.lenL, &v.aM, &v.cM, &v.aK,
                          &v.bK, &v.bN, &v.cN, &v.aL, &v.bL, &v.cL})
        append_key(key, *p);

    auto& cache = table_cache();
    {
        std::lock_guard<std::mutex> lk(cache.mtx);
        auto it = cache.map.find(key);
        if (it != cache.map.end())
        {
            cache.lru.splice(cache.lru.begin(), cache.lru, it->second.second);
            return it->second.first;
        }
    }

    i64 nkb = (v.k + BK - 1)/BK;
    size_t n_total = 2*v.m + 2*v.k + 2*v.n + 3*v.l + 2*nkb;
    std::vector<i64> host(n_total);
    i64* p = host.data();
    i64 *a_m = p; p += v.m;  i64 *c_m = p; p += v.m;
    i64 *a_k = p; p += v.k;  i64 *b_k = p; p += v.k;
    i64 *b_n = p; p += v.n;  i64 *c_n = p; p += v.n;
    i64 *a_l = p; p += v.l;  i64 *b_l = p; p += v.l;  i64 *c_l = p; p += v.l;
    i64 *a_kbs = p; p += nkb; i64 *b_kbs = p; p += nkb;

    std::vector<i64> bs(std::max({v.m, v.n, v.k, v.l}));
    fill_block_scatter(v.lenM, v.aM, BM, 0, v.m, a_m, bs.data(), v.pack_m_3d);
    fill_block_scatter(v.lenM, v.cM, BM, 0, v.m, c_m, bs.data(), v.pack_m_3d);
    fill_block_scatter(v.lenN, v.bN, BN, 0, v.n, b_n, bs.data(), v.pack_n_3d);
    fill_block_scatter(v.lenN, v.cN, BN, 0, v.n, c_n, bs.data(), v.pack_n_3d);
    fill_block_scatter(v.lenK, v.aK, BK, 0, v.k, a_k, bs.data(), v.pack_k_3d);
    for (i64 b = 0; b < nkb; b++) a_kbs[b] = bs[b*BK];
    fill_block_scatter(v.lenK, v.bK, BK, 0, v.k, b_k, bs.data(), v.pack_k_3d);
    for (i64 b = 0; b < nkb; b++) b_kbs[b] = bs[b*BK];
    fill_block_scatter(v.lenL, v.aL, 1, 0, v.l, a_l, bs.data(), false);
    fill_block_scatter(v.lenL, v.bL, 1, 0, v.l, b_l, bs.data(), false);
    fill_block_scatter(v.lenL, v.cL, 1, 0, v.l, c_l, bs.data(), false);

    auto t = std::make_shared<GemmTables>();
    t->a_m_step = affine_step(a_m, v.m); t->a_k_step = affine_step(a_k, v.k);
    t->b_n_step = affine_step(b_n, v.n); t->b_k_step = affine_step(b_k, v.k);
    gemm_pair_modes(v, a_m, a_k, b_n, b_k, a_l, b_l, t->a_pairs, t->b_pairs);
    t->bytes = n_total*sizeof(i64);
    TB_CUDA(cudaMalloc(&t->dev, t->bytes));
    TB_CUDA(cudaMemcpyAsync(t->dev, host.data(), t->bytes, cudaMemcpyHostToDevice, stream));
    // the host vector dies at return: make the copy complete first
    TB_CUDA(cudaStreamSynchronize(stream));
    i64* d = t->dev;
    t->a_m = d + (a_m - host.data()); t->c_m = d + (c_m - host.data());
    t->a_k = d + (a_k - host.data()); t->b_k = d + (b_k - host.data());
    t->b_n = d + (b_n - host.data()); t->c_n = d + (c_n - host.data());
    t->a_l = d + (a_l - host.data()); t->b_l = d + (b_l - host.data());
    t->c_l = d + (c_l - host.data());
    t->a_kbs = d + (a_kbs - host.data()); t->b_kbs = d + (b_kbs - host.data());

    std::vector<std::shared_ptr<GemmTables>> drop;
    {
        std::lock_guard<std::mutex> lk(cache.mtx);
        cache.lru.push_front(key);
        cache.map[key] = {t, cache.lru.begin()};
        while (cache.map.size() > cache.capacity)
        {
            auto it = cache.map.find(cache.lru.back());
            cache.retired_bytes += it->second.first->bytes;
            cache.retired.push_back(std::move(it->second.first));
            cache.map.erase(it);
            cache.lru.pop_back();
        }
        if (cache.retired.size() >= 256 || cache.retired_bytes >= ((size_t)64 << 20))
        {
            // tables no caller holds any more: nobody can fetch them again, and
            // every kernel that reads them was queued before the synchronisation
            // below
            std::vector<std::shared_ptr<GemmTables>> keep;
            for (auto& r : cache.retired)
            {
                if (r.use_count() == 1)
                {
                    cache.retired_bytes -= r->bytes;
                    drop.push_back(std::move(r));
                }
                else keep.push_back(std::move(r));
            }
            cache.retired.swap(keep);
        }
    }
    if (!drop.empty())
    {
        cudaDeviceSynchronize();
        drop.clear();
    }
    return t;
}

void tensor_extent(unsigned ndim, const len_type* len, const stride_type* stride,
                   i64& min_off, i64& max_off)
{
    min_off = 0; max_off = 0;
    for (unsigned i = 0; i < ndim; i++)
    {
        if (len[i] == 0) { min_off = 0; max_off = -1; return; }
        i64 span = (len[i]-1)*stride[i];
        if (span < 0) min_off += span; else max_off += span;
    }
}

} // namespace tb
