// indexed_dpd.cpp -- contraction of indexed DPD tensors (MArray's
// indexed_dpd_varray: a list of DPD tensors over the "dense" dimensions, one
// per index tuple of the "indexed" dimensions, each with a scalar factor).
//
// Semantics (src/iface/3t/mult.cxx:412-533 and the FULL form of
// src/internal/3t/indexed_dpd/mult.cxx:68-114 with
// src/internal/1t/indexed_dpd/util.hpp:14-113): every entry i of C is first
// scaled by f^C_i*beta (beta == 1: untouched; beta == 0 or f^C_i == 0: set
// to zero), then
//     C_i += alpha * f^C_i * sum_{j,k} f^A_j f^B_k (A_j . B_k)
// over the entries j of A and k of B whose index values agree with C_i's and
// with each other on every shared indexed label. A label indexed in one tensor
// and dense in another selects one slice (the indexed irrep, the index value)
// of the dense dimension.
//
// GPU form: each consistent (i, j, k) triple is a DPD contraction over the
// labels that are dense everywhere. Its operands are the entries' storage
// with the selected slices folded into per-block offsets (an explicit block
// table), so no dense copy of any tensor is made; every triple runs through
// the grouped persistent FP64 kernel with the factor-weighted alpha and
// beta = 1 on top of the initial scaling. Triples on distinct entries of C
// share one grouped launch: the k-th triple of every entry of C runs in the
// k-th launch, so each entry accumulates its triples in the sequential order.
// Element types: double; dcomplex as four real contractions of the parts
// (dpd_terms_z); float and scomplex
// widened to double / dcomplex for the contraction and rounded back; the
// level-1 operations run on every type directly.
#include "common.hpp"
#include "dpd.hpp"
#include "level1.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <map>
#include <string>

namespace tb
{

namespace
{

struct IdxTensor
{
    unsigned ndim = 0, dense_ndim = 0, nirrep = 1, dense_irrep = 0;
    std::vector<std::vector<i64>> len;          // [ndim][nirrep]
    std::vector<unsigned> idx_irrep;            // [ndim - dense_ndim]
    i64 nidx = 0;
    std::vector<i64> indices;                   // [nidx][ndim - dense_ndim]
    int type = TYPE_DOUBLE;
    size_t esz = sizeof(double);
    std::vector<char*> data;                    // per entry (device after staging)
    std::vector<zd> factor;
    DpdLayout dense;                            // block table of one entry, relative to its data
    unsigned irrep() const
    {
        unsigned x = dense_irrep;
        for (unsigned r : idx_irrep) x ^= r;
        return x;
    }
    unsigned nindexed() const { return ndim - dense_ndim; }
    i64 index(i64 entry, unsigned d) const { return indices[(size_t)entry*nindexed() + d]; }
};

void parse(const tblis_b200_indexed_dpd_tensor* t, IdxTensor& x)
{
    TB_CHECK(t, TB_ERR_ARG, "null indexed DPD tensor");
    x.type = t->type;
    x.esz = elem_size(t->type);
    TB_CHECK(t->dense_ndim >= 1 && t->dense_ndim <= t->ndim, TB_ERR_ARG, "indexed DPD: needs 1..ndim dense dimensions");
    TB_CHECK(t->nidx >= 1, TB_ERR_ARG, "indexed DPD: needs at least one index entry");
    TB_CHECK(t->len && t->data && t->offset && t->stride, TB_ERR_ARG, "indexed DPD: null array");
    x.ndim = t->ndim; x.dense_ndim = t->dense_ndim; x.nirrep = t->nirrep; x.dense_irrep = t->dense_irrep;
    const unsigned ni = t->ndim - t->dense_ndim;
    TB_CHECK(ni == 0 || (t->idx_irrep && t->indices), TB_ERR_ARG, "indexed DPD: null index arrays");
    TB_CHECK(ni > 0 || t->nidx == 1, TB_ERR_ARG, "indexed DPD: several entries need indexed dimensions");
    x.len.assign(x.ndim, std::vector<i64>(x.nirrep));
    for (unsigned d = 0; d < x.ndim; d++)
        for (unsigned r = 0; r < x.nirrep; r++) x.len[d][r] = t->len[(size_t)d*x.nirrep + r];
    x.idx_irrep.assign(t->idx_irrep, t->idx_irrep + ni);
    for (unsigned d = 0; d < ni; d++) TB_CHECK(x.idx_irrep[d] < x.nirrep, TB_ERR_ARG, "indexed DPD: bad indexed irrep");
    x.nidx = t->nidx;
    x.indices.assign(t->indices, t->indices + (size_t)t->nidx*ni);
    for (i64 e = 0; e < x.nidx; e++)
        for (unsigned d = 0; d < ni; d++)
        {
            const i64 v = x.index(e, d);
            TB_CHECK(v >= 0 && v < x.len[t->dense_ndim + d][x.idx_irrep[d]], TB_ERR_ARG,
                     "indexed DPD: index value out of range");
        }
    x.data.resize(t->nidx);
    for (i64 e = 0; e < t->nidx; e++) x.data[e] = static_cast<char*>(t->data[e]);
    x.factor.assign(t->nidx, 1.0);
    if (t->factor)
        for (i64 e = 0; e < t->nidx; e++)
        {
            tblis_scalar f;
            f.type = t->type;
            std::memcpy(&f.data, static_cast<const char*>(t->factor) + e*(i64)x.esz, x.esz);
            x.factor[e] = scalar_get(f);
        }
    std::vector<i64> dl((size_t)x.dense_ndim*x.nirrep);
    for (unsigned d = 0; d < x.dense_ndim; d++)
        for (unsigned r = 0; r < x.nirrep; r++) dl[(size_t)d*x.nirrep + r] = x.len[d][r];
    x.dense.init_explicit(x.dense_irrep, x.nirrep, x.dense_ndim, dl.data(), t->offset, t->stride);
}

// device copies of host-resident entries
struct EntryStage
{
    std::vector<dbuf> bufs;
    std::vector<std::pair<char*, char*>> back;          // (host, device) to copy out
    size_t bytes = 0;
    void init(IdxTensor& x, bool copy_in, bool copy_out, cudaStream_t st)
    {
        bytes = (size_t)x.dense.total()*x.esz;
        for (auto& p : x.data)
        {
            if (!p || bytes == 0 || pointer_kind(p) == MEM_DEVICE) continue;
            bufs.emplace_back(bytes, st);
            char* d = bufs.back().as<char>();
            if (copy_in) TB_CUDA(cudaMemcpyAsync(d, p, bytes, cudaMemcpyHostToDevice, st));
            if (copy_out) back.push_back({p, d});
            p = d;
        }
    }
    void out(cudaStream_t st)
    {
        for (auto& hd : back)
            TB_CUDA(cudaMemcpyAsync(hd.first, hd.second, bytes, cudaMemcpyDeviceToHost, st));
    }
    bool staged() const { return !bufs.empty(); }
};

// float / scomplex entries widened to double / dcomplex device copies for a
// contraction; narrow() rounds the stored blocks back into the entries
struct EntryWiden
{
    std::vector<dbuf> bufs;
    std::vector<char*> orig;
    bool cx = false;
    void init(IdxTensor& x, bool read, cudaStream_t st)
    {
        cx = x.type == TYPE_SCOMPLEX;
        orig = x.data;
        const i64 n = x.dense.total();
        for (auto& p : x.data)
        {
            if (read) bufs.push_back(dpd_widen(p, n, cx, st));
            else
            {
                bufs.emplace_back((size_t)std::max<i64>(n*(cx ? 2 : 1), 1)*sizeof(double), st);
                TB_CUDA(cudaMemsetAsync(bufs.back().ptr, 0, bufs.back().bytes, st));
            }
            p = bufs.back().as<char>();
        }
        x.type = cx ? TYPE_DCOMPLEX : TYPE_DOUBLE;
        x.esz = elem_size(x.type);
    }
    void narrow(const IdxTensor& x, cudaStream_t st)
    {
        for (size_t e = 0; e < orig.size(); e++)
            dpd_narrow_blocks(x.dense, cx, bufs[e].as<double>(), reinterpret_cast<float*>(orig[e]), st);
    }
};

// one operand of a triple: which dense dims stay, which are sliced
struct Slicing
{
    std::vector<unsigned> keep;                     // dense dims that stay (in order)
    std::vector<unsigned> cut;                      // dense dims fixed to one (irrep, value)
    std::vector<unsigned> cut_irrep;
    std::vector<int> cut_label;                     // label of each cut dim
    std::string labels;                             // labels of the kept dims
};

// the DPD tensor of entry `e` of x with the cut dims fixed to `values`
// (parallel to s.cut); false when a cut value lies outside its block
bool slice_entry(const IdxTensor& x, i64 e, const Slicing& s, const std::vector<i64>& values,
                 unsigned ndummy, DpdTensor& out)
{
    const unsigned nk = (unsigned)s.keep.size();
    const unsigned nd = nk + ndummy;
    const unsigned nirrep = x.nirrep;
    unsigned irrep = x.dense_irrep;
    for (size_t c = 0; c < s.cut.size(); c++)
    {
        irrep ^= s.cut_irrep[c];
        if (values[c] < 0 || values[c] >= x.len[s.cut[c]][s.cut_irrep[c]]) return false;
    }
    std::vector<i64> lens((size_t)nd*nirrep, 0);
    for (unsigned k = 0; k < nk; k++)
        for (unsigned r = 0; r < nirrep; r++) lens[(size_t)k*nirrep + r] = x.len[s.keep[k]][r];
    for (unsigned u = 0; u < ndummy; u++) lens[(size_t)(nk + u)*nirrep + 0] = 1;     // one element, irrep 0
    size_t nt = 1;
    for (unsigned d = 0; d < nd; d++) nt *= nirrep;
    std::vector<i64> off(nt, -1), str(nt*nd, 0);
    std::vector<unsigned> sub(nd, 0), full(x.dense_ndim, 0);
    std::vector<i64> bl(x.dense_ndim), bs(x.dense_ndim);
    for (size_t t = 0; t < nt; t++)
    {
        unsigned xr = 0;
        i64 ext = 1;
        for (unsigned d = 0; d < nd; d++)
        {
            xr ^= sub[d];
            ext *= lens[(size_t)d*nirrep + sub[d]];
        }
        if (xr == irrep && ext > 0)
        {
            for (unsigned k = 0; k < nk; k++) full[s.keep[k]] = sub[k];
            for (size_t c = 0; c < s.cut.size(); c++) full[s.cut[c]] = s.cut_irrep[c];
            i64 o;
            x.dense.block(full.data(), bl.data(), bs.data(), o);
            for (size_t c = 0; c < s.cut.size(); c++) o += values[c]*bs[s.cut[c]];
            off[t] = o;
            for (unsigned k = 0; k < nk; k++) str[t*nd + k] = bs[s.keep[k]];
            for (unsigned u = 0; u < ndummy; u++) str[t*nd + nk + u] = 1;
        }
        unsigned d = 0;
        while (d < nd && ++sub[d] == nirrep) { sub[d] = 0; d++; }
    }
    out.lay = DpdLayout();
    out.lay.init_explicit(irrep, nirrep, nd, lens.data(), off.data(), str.data());
    out.data = reinterpret_cast<double*>(x.data[e]);     // storage of x.type elements
    return true;
}

} // namespace

void indexed_dpd_mult(const tblis_b200_indexed_dpd_tensor* A_, const label_type* idx_A,
                      const tblis_b200_indexed_dpd_tensor* B_, const label_type* idx_B,
                      tblis_b200_indexed_dpd_tensor* C_, const label_type* idx_C,
                      tblis_b200_report* report)
{
    ensure_device();
    cudaStream_t st = current_stream();
    const int k0 = (int)g_kernel_count.load();
    IdxTensor A, B, C;
    parse(A_, A); parse(B_, B); parse(C_, C);
    TB_CHECK(B.nirrep == A.nirrep && C.nirrep == A.nirrep, TB_ERR_ARG, "indexed DPD: nirrep differs");
    const std::string iA(idx_A, A.ndim), iB(idx_B, B.ndim), iC(idx_C, C.ndim);
    for (const std::string* s : {&iA, &iB, &iC})
        for (size_t i = 0; i < s->size(); i++)
            for (size_t j = 0; j < i; j++)
                TB_CHECK((*s)[i] != (*s)[j], TB_ERR_ARG, "indexed DPD: repeated label in one tensor");
    // every label in exactly two or three tensors, equal per-irrep lengths
    const IdxTensor* T[3] = {&A, &B, &C};
    const std::string* I[3] = {&iA, &iB, &iC};
    for (int t = 0; t < 3; t++)
        for (size_t p = 0; p < I[t]->size(); p++)
        {
            const char c = (*I[t])[p];
            int n = 0;
            for (int u = 0; u < 3; u++)
            {
                const size_t q = I[u]->find(c);
                if (q == std::string::npos) continue;
                n++;
                TB_CHECK(T[u]->len[q] == T[t]->len[p], TB_ERR_ARG, "indexed DPD: per-irrep lengths differ");
            }
            TB_CHECK(n >= 2, TB_ERR_ARG, "indexed DPD: a label appears in one tensor only");
        }

    TB_CHECK(A.type == B.type && A.type == C.type, TB_ERR_TYPE, "indexed DPD: operand types differ");
    const int type = C.type;
    const zd alpha = scalar_get(A_->scalar)*scalar_get(B_->scalar), beta = scalar_get(C_->scalar);

    EntryStage sa, sb, sc;
    sa.init(A, true, false, st);
    sb.init(B, true, false, st);
    sc.init(C, beta != 0.0, true, st);
    // float / scomplex: contracted in double / dcomplex
    EntryWiden wa, wb, wc;
    const bool widened = type == TYPE_FLOAT || type == TYPE_SCOMPLEX;
    if (widened)
    {
        wa.init(A, true, st);
        wb.init(B, true, st);
        wc.init(C, beta != 0.0, st);
    }
    const int wtype = C.type;

    // beta through the entries' factors (src/internal/3t/indexed_dpd/mult.cxx:1217-1224
    // with src/internal/1t/indexed_dpd/scale.cxx and set.cxx): beta == 1
    // leaves C, beta == 0 or a zero factor sets the entry to 0, otherwise
    // entry e is scaled by f_e*beta
    if (beta != 1.0)
    {
        const std::string dl = iC.substr(0, C.dense_ndim);
        for (i64 e = 0; e < C.nidx; e++)
        {
            if (beta == 0.0 || C.factor[e] == 0.0) dpd_unary_dev_t(wtype, 1, 0.0, 1.0, C.dense, C.data[e], dl);
            else dpd_unary_dev_t(wtype, 0, 0.0, C.factor[e]*beta, C.dense, C.data[e], dl);
        }
    }

    // labels shared by all three tensors and dense in all of them are batch
    // labels of each entry triple's DPD contraction
    auto indexed_in = [&](int t, char c, unsigned& slot)
    {
        const size_t p = I[t]->find(c);
        if (p == std::string::npos || p < T[t]->dense_ndim) return false;
        slot = (unsigned)(p - T[t]->dense_ndim);
        return true;
    };

    // src/iface/3t/mult.cxx:514 (with its operator precedence) and the
    // indexed-irrep agreement of src/internal/3t/indexed_dpd/mult.cxx:1226-1280
    bool has_abc = false;
    for (char c : iA) if (iB.find(c) != std::string::npos && iC.find(c) != std::string::npos) has_abc = true;
    bool skip = alpha == 0.0 || (!has_abc && (A.irrep() ^ (unsigned)(B.irrep() != C.irrep())) != 0);
    // fixed (irrep) of every label indexed somewhere; they must agree
    std::map<char, unsigned> fixed_irrep;
    for (int t = 0; t < 3 && !skip; t++)
        for (unsigned d = 0; d < T[t]->nindexed(); d++)
        {
            const char c = (*I[t])[T[t]->dense_ndim + d];
            auto it = fixed_irrep.find(c);
            if (it == fixed_irrep.end()) fixed_irrep[c] = T[t]->idx_irrep[d];
            else if (it->second != T[t]->idx_irrep[d]) skip = true;
        }

    int launches = 0;
    double flops = 0;
    if (!skip)
    {
        // per tensor: dense dims kept (label dense everywhere) or cut (label indexed elsewhere)
        Slicing S[3];
        for (int t = 0; t < 3; t++)
            for (unsigned d = 0; d < T[t]->dense_ndim; d++)
            {
                const char c = (*I[t])[d];
                auto it = fixed_irrep.find(c);
                if (it == fixed_irrep.end()) { S[t].keep.push_back(d); S[t].labels.push_back(c); }
                else { S[t].cut.push_back(d); S[t].cut_irrep.push_back(it->second); S[t].cut_label.push_back(c); }
            }
        // labels for tensors left without dims: a length-1 dimension shared
        // with a partner (AB for A or B, AC for C)
        std::string used = iA + iB + iC;
        auto fresh = [&]()
        {
            for (int c = 33; c < 127; c++)
                if (used.find((char)c) == std::string::npos) { used.push_back((char)c); return (char)c; }
            throw error(TB_ERR_ARG, "indexed DPD: no free label");
        };
        unsigned dumA = 0, dumB = 0, dumC = 0;
        std::string lA = S[0].labels, lB = S[1].labels, lC = S[2].labels;
        if (lA.empty() || lB.empty())
        {
            const char k = fresh();               // contracted, length 1
            lA.push_back(k); lB.push_back(k); dumA++; dumB++;
        }
        if (lC.empty())
        {
            const char m = fresh();               // A and C, length 1
            lA.push_back(m); lC.push_back(m); dumA++; dumC++;
        }

        // value of every fixed label for a given entry of a tensor
        auto value_of = [&](int t, i64 e, char c, i64& v)
        {
            unsigned slot;
            if (!indexed_in(t, c, slot)) return false;
            v = T[t]->index(e, slot);
            return true;
        };
        // terms on distinct entries of C share launches unless entries overlap
        bool c_overlap = false;
        {
            std::vector<std::pair<const char*, const char*>> span;
            const i64 bytes = C.dense.total()*(i64)C.esz;
            for (i64 e = 0; e < C.nidx; e++)
                if (bytes > 0) span.push_back({C.data[e], C.data[e] + bytes});
            std::sort(span.begin(), span.end());
            for (size_t i = 1; i < span.size(); i++)
                if (span[i].first < span[i - 1].second) c_overlap = true;
        }
        std::deque<DpdTensor> store;
        std::vector<DpdTerm> terms;
        // entries of A and B keyed by the values of the fixed labels they index
        for (i64 ec = 0; ec < C.nidx; ec++)
        {
            for (i64 ea = 0; ea < A.nidx; ea++)
            {
                // A and C agree on labels indexed in both
                bool ok = true;
                for (unsigned d = 0; d < A.nindexed() && ok; d++)
                {
                    const char c = iA[A.dense_ndim + d];
                    i64 v;
                    if (value_of(2, ec, c, v) && v != A.index(ea, d)) ok = false;
                }
                if (!ok) continue;
                for (i64 eb = 0; eb < B.nidx; eb++)
                {
                    bool okb = true;
                    for (unsigned d = 0; d < B.nindexed() && okb; d++)
                    {
                        const char c = iB[B.dense_ndim + d];
                        i64 v;
                        if (value_of(0, ea, c, v) && v != B.index(eb, d)) okb = false;
                        if (value_of(2, ec, c, v) && v != B.index(eb, d)) okb = false;
                    }
                    if (!okb) continue;
                    // the value of every cut label, from whichever tensor indexes it
                    auto cut_values = [&](int t, std::vector<i64>& vals)
                    {
                        vals.clear();
                        for (char c : S[t].cut_label)
                        {
                            i64 v = -1;
                            if (!value_of(0, ea, c, v) && !value_of(1, eb, c, v)) value_of(2, ec, c, v);
                            vals.push_back(v);
                        }
                    };
                    std::vector<i64> vA, vB, vC;
                    cut_values(0, vA); cut_values(1, vB); cut_values(2, vC);
                    DpdTensor a, b, c;
                    if (!slice_entry(A, ea, S[0], vA, dumA, a) || !slice_entry(B, eb, S[1], vB, dumB, b) ||
                        !slice_entry(C, ec, S[2], vC, dumC, c))
                        continue;
                    const zd w = alpha*A.factor[ea]*B.factor[eb]*C.factor[ec];
                    if (w == 0.0) continue;
                    const i64 key = c_overlap ? 0 : ec;
                    if (wtype == TYPE_DOUBLE)
                    {
                        store.push_back(std::move(a)); const DpdTensor* pa = &store.back();
                        store.push_back(std::move(b)); const DpdTensor* pb = &store.back();
                        store.push_back(std::move(c)); const DpdTensor* pc = &store.back();
                        DpdTerm t;
                        t.a = pa; t.ia = lA.c_str();
                        t.b = pb; t.ib = lB.c_str();
                        t.c = pc; t.ic = lC.c_str();
                        t.alpha = w.real();
                        t.c_key = key;
                        terms.push_back(t);
                    }
                    else
                        dpd_terms_z(a.lay, a.data, lA.c_str(), b.lay, b.data, lB.c_str(), c.lay, c.data, lC.c_str(),
                                    w, key, store, terms);
                }
            }
        }
        // every term with beta = 1 on top of the initial scaling; the k-th
        // term on each entry of C goes into the k-th grouped launch
        DpdMultReport r;
        launches = dpd_mult_terms(terms, st, &r, false);
        flops = r.flops;
    }

    if (widened) wc.narrow(C, st);
    sc.out(st);
    if (sa.staged() || sb.staged() || sc.staged() || widened) TB_CUDA(cudaStreamSynchronize(st));
    scalar_put(C_->scalar, type, 1.0);
    if (report)
    {
        memset(report, 0, sizeof(*report));
        report->method = 1;
        report->flops = flops;
        report->m = launches;            // grouped launches of the contraction terms
        report->kernels = (int)(g_kernel_count.load() - k0);
    }
}

namespace
{

// scales every entry's blocks by f_e*beta (set when beta == 0 or f_e == 0),
// as src/internal/1t/indexed_dpd/scale.cxx and set.cxx do
void scale_entries(const IdxTensor& X, zd beta, const std::string& labels)
{
    const std::string dl = labels.substr(0, X.dense_ndim);
    for (i64 e = 0; e < X.nidx; e++)
    {
        if (beta == 0.0 || X.factor[e] == 0.0) dpd_unary_dev_t(X.type, 1, 0.0, 1.0, X.dense, X.data[e], dl);
        else dpd_unary_dev_t(X.type, 0, 0.0, X.factor[e]*beta, X.dense, X.data[e], dl);
    }
}

// the pairs (entry of X, entry of Y) that agree on the labels both index, as
// DPD tensors over the labels dense in both with the other labels fixed
// (slices); a shared length-1 label stands in when none is left
template <typename F>
void for_each_pair(const IdxTensor& X, const std::string& iX, const IdxTensor& Y, const std::string& iY, F&& f)
{
    const IdxTensor* T[2] = {&X, &Y};
    const std::string* I[2] = {&iX, &iY};
    std::map<char, unsigned> fixed;
    for (int t = 0; t < 2; t++)
        for (unsigned d = 0; d < T[t]->nindexed(); d++) fixed[(*I[t])[T[t]->dense_ndim + d]] = T[t]->idx_irrep[d];
    Slicing S[2];
    for (int t = 0; t < 2; t++)
        for (unsigned d = 0; d < T[t]->dense_ndim; d++)
        {
            const char c = (*I[t])[d];
            auto it = fixed.find(c);
            if (it == fixed.end()) { S[t].keep.push_back(d); S[t].labels.push_back(c); }
            else { S[t].cut.push_back(d); S[t].cut_irrep.push_back(it->second); S[t].cut_label.push_back(c); }
        }
    bool shared = false;
    for (char c : S[0].labels) if (S[1].labels.find(c) != std::string::npos) shared = true;
    std::string lX = S[0].labels, lY = S[1].labels;
    unsigned dum = 0;
    if (!shared)
    {
        std::string used = iX + iY;
        for (int c = 33; c < 127 && !dum; c++)
            if (used.find((char)c) == std::string::npos) { lX.push_back((char)c); lY.push_back((char)c); dum = 1; }
        TB_CHECK(dum, TB_ERR_ARG, "indexed DPD: no free label");
    }
    auto value_of = [&](int t, i64 e, char c, i64& v)
    {
        const size_t p = I[t]->find(c);
        if (p == std::string::npos || p < T[t]->dense_ndim) return false;
        v = T[t]->index(e, (unsigned)(p - T[t]->dense_ndim));
        return true;
    };
    for (i64 ex = 0; ex < X.nidx; ex++)
        for (i64 ey = 0; ey < Y.nidx; ey++)
        {
            bool ok = true;
            for (unsigned d = 0; d < Y.nindexed() && ok; d++)
            {
                i64 v;
                if (value_of(0, ex, iY[Y.dense_ndim + d], v) && v != Y.index(ey, d)) ok = false;
            }
            if (!ok) continue;
            std::vector<i64> vals[2];
            for (int t = 0; t < 2; t++)
                for (char c : S[t].cut_label)
                {
                    i64 v = -1;
                    if (!value_of(0, ex, c, v)) value_of(1, ey, c, v);
                    vals[t].push_back(v);
                }
            DpdTensor x, y;
            if (!slice_entry(X, ex, S[0], vals[0], dum, x) || !slice_entry(Y, ey, S[1], vals[1], dum, y)) continue;
            f(ex, ey, x, lX, y, lY);
        }
}

bool indexed_irreps_agree(const IdxTensor& X, const std::string& iX, const IdxTensor& Y, const std::string& iY)
{
    for (unsigned d = 0; d < X.nindexed(); d++)
    {
        const size_t p = iY.find(iX[X.dense_ndim + d]);
        if (p != std::string::npos && p >= Y.dense_ndim && Y.idx_irrep[p - Y.dense_ndim] != X.idx_irrep[d])
            return false;
    }
    return true;
}

struct IdxCall
{
    IdxTensor A, B;
    EntryStage sa, sb;
};

} // namespace

void indexed_dpd_add(const tblis_b200_indexed_dpd_tensor* A_, const label_type* idx_A,
                     tblis_b200_indexed_dpd_tensor* B_, const label_type* idx_B)
{
    ensure_device();
    cudaStream_t st = current_stream();
    IdxTensor A, B;
    parse(A_, A); parse(B_, B);
    TB_CHECK(A.nirrep == B.nirrep, TB_ERR_ARG, "indexed DPD add: nirrep differs");
    const std::string iA(idx_A, A.ndim), iB(idx_B, B.ndim);
    std::string Aonly, Bonly;
    for (char c : iA) if (iB.find(c) == std::string::npos) Aonly.push_back(c);
    for (char c : iB) if (iA.find(c) == std::string::npos) Bonly.push_back(c);
    TB_CHECK(A.type == B.type, TB_ERR_TYPE, "indexed DPD add: operand types differ");
    const zd alpha = scalar_get(A_->scalar), beta = scalar_get(B_->scalar);
    EntryStage sa, sb;
    sa.init(A, true, false, st);
    sb.init(B, beta != 0.0, true, st);
    // src/iface/1t/add.cxx:312-325: alpha == 0 or an irrep mismatch only
    // scales (through the factors, beta == 1 included)
    if (alpha == 0.0 || (Aonly.empty() && Bonly.empty() && A.irrep() != B.irrep()))
    {
        for (i64 e = 0; e < B.nidx; e++)
        {
            const std::string dl = iB.substr(0, B.dense_ndim);
            if (beta == 0.0 || B.factor[e] == 0.0) dpd_unary_dev_t(B.type, 1, 0.0, 1.0, B.dense, B.data[e], dl);
            else dpd_unary_dev_t(B.type, 0, 0.0, B.factor[e]*beta, B.dense, B.data[e], dl);
        }
    }
    else
    {
        if (beta != 1.0) scale_entries(B, beta, iB);
        if (indexed_irreps_agree(A, iA, B, iB))
            for_each_pair(A, iA, B, iB, [&](i64 ea, i64 eb, const DpdTensor& a, const std::string& la,
                                            const DpdTensor& b, const std::string& lb)
            {
                const zd w = alpha*A.factor[ea]*B.factor[eb];
                if (w == 0.0) return;
                dpd_add_dev_t(A.type, w, a.lay, a.data, la, 1.0, b.lay, b.data, lb);
            });
    }
    sb.out(st);
    if (sa.staged() || sb.staged()) TB_CUDA(cudaStreamSynchronize(st));
    scalar_put(B_->scalar, B.type, 1.0);
}

zd indexed_dpd_dot(const tblis_b200_indexed_dpd_tensor* A_, const label_type* idx_A,
                   const tblis_b200_indexed_dpd_tensor* B_, const label_type* idx_B)
{
    ensure_device();
    cudaStream_t st = current_stream();
    IdxTensor A, B;
    parse(A_, A); parse(B_, B);
    TB_CHECK(A.nirrep == B.nirrep && A.ndim == B.ndim, TB_ERR_ARG, "indexed DPD dot: shapes differ");
    const std::string iA(idx_A, A.ndim), iB(idx_B, B.ndim);
    for (char c : iA) TB_CHECK(iB.find(c) != std::string::npos, TB_ERR_ARG, "indexed DPD dot: labels must match");
    TB_CHECK(A.type == B.type, TB_ERR_TYPE, "indexed DPD dot: operand types differ");
    EntryStage sa, sb;
    sa.init(A, true, false, st);
    sb.init(B, true, false, st);
    zd sum = 0.0;
    if (indexed_irreps_agree(A, iA, B, iB))
        for_each_pair(A, iA, B, iB, [&](i64 ea, i64 eb, const DpdTensor& a, const std::string& la,
                                        const DpdTensor& b, const std::string& lb)
        {
            const zd w = A.factor[ea]*B.factor[eb];
            if (w == 0.0) return;
            sum += w*dpd_dot_dev_t(A.type, a.lay, a.data, la, b.lay, b.data, lb);
        });
    if (sa.staged() || sb.staged()) TB_CUDA(cudaStreamSynchronize(st));
    return scalar_get(A_->scalar)*scalar_get(B_->scalar)*sum;
}

// src/internal/1t/indexed_dpd/reduce.cxx: each entry's reduction scaled by
// its factor, combined in entry order; idx counts from entry 0's data
void indexed_dpd_reduce(int op, const tblis_b200_indexed_dpd_tensor* A_, const label_type* idx_A,
                        zd& result, i64& idx)
{
    ensure_device();
    cudaStream_t st = current_stream();
    IdxTensor A;
    parse(A_, A);
    const std::vector<char*> orig = A.data;
    EntryStage sa;
    sa.init(A, true, false, st);
    const std::string dl(idx_A, A.dense_ndim);
    // complex values compare by their real parts, as the reference's operators do
    using lim = std::numeric_limits<double>;
    const double big = A.type == TYPE_FLOAT || A.type == TYPE_SCOMPLEX ? (double)std::numeric_limits<float>::max()
                                                                       : lim::max();
    zd acc = op == REDUCE_MAX ? zd(-big) : (op == REDUCE_MIN || op == REDUCE_MIN_ABS) ? zd(big) : zd(0.0);
    i64 at = -1;
    for (i64 e = 0; e < A.nidx; e++)
    {
        zd v;
        i64 bi;
        dpd_reduce_dev_t(A.type, op, A.dense, A.data[e], dl, v, bi);
        const zd fv = A.factor[e]*v;
        const i64 gi = bi + (i64)((orig[e] - orig[0])/(i64)A.esz);
        switch (op)
        {
            case REDUCE_SUM: case REDUCE_SUM_ABS: acc += fv; break;
            case REDUCE_NORM_2: acc += std::norm(fv); break;
            case REDUCE_MAX: if (fv.real() > acc.real()) { acc = fv; at = gi; } break;
            case REDUCE_MAX_ABS: if (std::abs(fv) > acc.real()) { acc = std::abs(fv); at = gi; } break;
            case REDUCE_MIN: if (fv.real() < acc.real()) { acc = fv; at = gi; } break;
            case REDUCE_MIN_ABS: if (std::abs(fv) < acc.real()) { acc = std::abs(fv); at = gi; } break;
            default: throw error(TB_ERR_ARG, "indexed DPD reduce: unknown operation");
        }
    }
    if (sa.staged()) TB_CUDA(cudaStreamSynchronize(st));
    if (op == REDUCE_NORM_2) acc = std::sqrt(acc.real());
    result = acc;
    idx = at;
}

// kind 0: scale by A.scalar, 1: set to alpha, 2: shift (alpha + A.scalar*A),
// each entry through its factor (src/internal/1t/indexed_dpd/{scale,set,shift}.cxx)
void indexed_dpd_unary(int kind, const tblis_scalar* alpha_, tblis_b200_indexed_dpd_tensor* A_,
                       const label_type* idx_A)
{
    ensure_device();
    cudaStream_t st = current_stream();
    IdxTensor A;
    parse(A_, A);
    if (alpha_) TB_CHECK(alpha_->type == A.type, TB_ERR_TYPE, "indexed DPD set/shift: scalar and tensor types differ");
    const zd alpha = alpha_ ? scalar_get(*alpha_) : zd(0.0);
    EntryStage sa;
    sa.init(A, kind != 1, true, st);
    const std::string dl(idx_A, A.dense_ndim);
    const zd scal = scalar_get(A_->scalar);
    const int ty = A.type;
    for (i64 e = 0; e < A.nidx; e++)
    {
        const zd f = A.factor[e];
        if (kind == 0)
        {
            if (scal == 0.0 || f == 0.0) dpd_unary_dev_t(ty, 1, 0.0, 1.0, A.dense, A.data[e], dl);
            else dpd_unary_dev_t(ty, 0, 0.0, f*scal, A.dense, A.data[e], dl);
        }
        else if (kind == 1)
            dpd_unary_dev_t(ty, 1, f*alpha, 1.0, A.dense, A.data[e], dl);
        else if (f == 0.0)
        {
            if (scal == 0.0) dpd_unary_dev_t(ty, 1, 0.0, 1.0, A.dense, A.data[e], dl);
            else if (scal != 1.0) dpd_unary_dev_t(ty, 0, 0.0, scal, A.dense, A.data[e], dl);
        }
        else
            dpd_unary_dev_t(ty, 2, f*alpha, scal, A.dense, A.data[e], dl);
    }
    sa.out(st);
    if (sa.staged()) TB_CUDA(cudaStreamSynchronize(st));
    scalar_put(A_->scalar, ty, 1.0);
}

} // namespace tb

extern "C" {

int tblis_b200_indexed_dpd_add(const tblis_b200_indexed_dpd_tensor* A, const label_type* idx_A,
                               tblis_b200_indexed_dpd_tensor* B, const label_type* idx_B)
{
    return tb::guarded([&] { tb::indexed_dpd_add(A, idx_A, B, idx_B); });
}

int tblis_b200_indexed_dpd_dot(const tblis_b200_indexed_dpd_tensor* A, const label_type* idx_A,
                               const tblis_b200_indexed_dpd_tensor* B, const label_type* idx_B,
                               tblis_scalar* result)
{
    return tb::guarded([&]
    {
        TB_CHECK(result && A, tb::TB_ERR_ARG, "null argument");
        tb::scalar_put(*result, A->type, tb::indexed_dpd_dot(A, idx_A, B, idx_B));
    });
}

int tblis_b200_indexed_dpd_reduce(reduce_t op, const tblis_b200_indexed_dpd_tensor* A, const label_type* idx_A,
                                  tblis_scalar* result, len_type* idx)
{
    return tb::guarded([&]
    {
        TB_CHECK(result && idx && A, tb::TB_ERR_ARG, "null argument");
        tb::zd r = 0.0;
        tb::i64 i = -1;
        tb::indexed_dpd_reduce((int)op, A, idx_A, r, i);
        tb::scalar_put(*result, A->type, r);
        *idx = i;
    });
}

int tblis_b200_indexed_dpd_scale(tblis_b200_indexed_dpd_tensor* A, const label_type* idx_A)
{
    return tb::guarded([&] { tb::indexed_dpd_unary(0, nullptr, A, idx_A); });
}

int tblis_b200_indexed_dpd_set(const tblis_scalar* alpha, tblis_b200_indexed_dpd_tensor* A,
                               const label_type* idx_A)
{
    return tb::guarded([&]
    {
        TB_CHECK(alpha, tb::TB_ERR_ARG, "null alpha");
        tb::indexed_dpd_unary(1, alpha, A, idx_A);
    });
}

int tblis_b200_indexed_dpd_shift(const tblis_scalar* alpha, tblis_b200_indexed_dpd_tensor* A,
                                 const label_type* idx_A)
{
    return tb::guarded([&]
    {
        TB_CHECK(alpha, tb::TB_ERR_ARG, "null alpha");
        tb::indexed_dpd_unary(2, alpha, A, idx_A);
    });
}


int tblis_b200_indexed_dpd_mult(const tblis_b200_indexed_dpd_tensor* A, const label_type* idx_A,
                                const tblis_b200_indexed_dpd_tensor* B, const label_type* idx_B,
                                      tblis_b200_indexed_dpd_tensor* C, const label_type* idx_C,
                                tblis_b200_report* report)
{
    return tb::guarded([&] { tb::indexed_dpd_mult(A, idx_A, B, idx_B, C, idx_C, report); });
}

}
