// dpd.cpp -- DPD tensors: MArray's block layout and the block-sparse
// contraction on the GPU.
//
// Layout: restates the binary layout tree of MArray's dpd_varray
// (src/external/marray/include/dpd_marray_base.hpp:34-228: default_depth,
// set_tree, set_size, get_block) so block offsets and strides are bit-exact.
//
// Contraction: as in src/internal/3t/dpd/mult.cxx:223-356, one GEMM per irrep
// h of the contracted index group: rows are all AC irrep combinations with
// XOR = irrep(A)^h, columns all BC combinations with XOR = irrep(B)^h, k all
// AB combinations with XOR = h, each combination contributing its dense block
// extent. For the layout trees MArray builds, the offset of element (row, k) of
// such a "patch matrix" is row_part + k_part (checked for every block pair);
// the patches then become ordinary GEMM views with scatter vectors, and all of
// them run in ONE persistent grouped launch of the FP64 DMMA kernel. The tile
// shape of that launch is chosen by a small autotuner keyed on the histogram of
// group sizes, and the launch (descriptor upload + kernel) is captured once in
// a CUDA graph and replayed.
#include "dpd.hpp"
#include "gemm_f64.hpp"
#include "level1.hpp"
#include "grouped.hpp"

#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>

namespace tb
{

std::vector<unsigned> dpd_default_depth(int layout, unsigned ndim)
{
    std::vector<unsigned> depth(ndim);
    if (layout == 0 || layout == 1)            // BALANCED_{COLUMN,ROW}_MAJOR
    {
        unsigned dl = sizeof(unsigned)*8 - __builtin_clz(ndim) - 1;
        unsigned du = dl + ((ndim & (ndim - 1)) ? 1 : 0);
        unsigned o = ndim - (1u << dl);
        unsigned k = 2*((o + 1)/2);
        unsigned l = 2*(o/2);
        unsigned h = (ndim + 1)/2;
        for (unsigned i = 0; i < k; i++) depth[i] = du;
        for (unsigned i = k; i < h; i++) depth[i] = dl;
        for (unsigned i = h; i < h + l; i++) depth[i] = du;
        for (unsigned i = h + l; i < ndim; i++) depth[i] = dl;
    }
    else if (layout == 4 || layout == 5)       // PREFIX_{COLUMN,ROW}_MAJOR
    {
        depth[0] = ndim - 1;
        for (unsigned i = 1; i < ndim; i++) depth[i] = ndim - i;
    }
    else                                       // BLOCKED_{COLUMN,ROW}_MAJOR
    {
        for (unsigned i = 0; i + 1 < ndim; i++) depth[i] = i + 1;
        depth[ndim - 1] = ndim - 1;
    }
    return depth;
}

void DpdLayout::init(unsigned irrep_, unsigned nirrep_, unsigned ndim_, const i64* lens, int layout_)
{
    TB_CHECK(nirrep_ == 1 || nirrep_ == 2 || nirrep_ == 4 || nirrep_ == 8, TB_ERR_ARG,
             "DPD: nirrep must be 1, 2, 4 or 8");
    TB_CHECK(ndim_ > 0 && ndim_ <= 16, TB_ERR_ARG, "DPD: 1..16 dimensions");
    TB_CHECK(layout_ >= 0 && layout_ <= 5, TB_ERR_ARG, "DPD: unknown layout");
    TB_CHECK(irrep_ < nirrep_, TB_ERR_ARG, "DPD: irrep out of range");
    ndim = ndim_; nirrep = nirrep_; irrep = irrep_; layout = layout_;
    len.assign(ndim, std::vector<i64>(nirrep));
    for (unsigned i = 0; i < ndim; i++)
        for (unsigned j = 0; j < nirrep; j++)
        {
            len[i][j] = lens[i*nirrep + j];
            TB_CHECK(len[i][j] >= 0, TB_ERR_ARG, "DPD: negative length");
        }

    // set_tree (dpd_marray_base.hpp:69-119)
    leaf.assign(ndim, 0);
    parent.assign(2*ndim - 1, 0);
    std::vector<unsigned> depth = dpd_default_depth(layout, ndim);
    std::vector<unsigned> node(ndim);
    std::vector<long> leaf_idx(ndim);
    for (unsigned i = 0; i < ndim; i++) leaf_idx[i] = i;
    unsigned pos = 0;
    for (unsigned d = ndim; d-- > 0;)
    {
        for (unsigned i = 0; i < depth.size(); i++)
        {
            if (depth[i] == d + 1)
            {
                TB_CHECK(i + 1 < depth.size() && depth[i + 1] == d + 1, TB_ERR_ARG, "DPD: bad layout tree");
                parent[node[i]] = parent[node[i + 1]] = pos;
                depth.erase(depth.begin() + i + 1);
                depth[i]--;
                node.erase(node.begin() + i + 1);
                node[i] = pos++;
                leaf_idx.erase(leaf_idx.begin() + i + 1);
                leaf_idx[i] = -1;
            }
            else if (depth[i] == d)
            {
                node[i] = pos++;
                if (leaf_idx[i] != -1) leaf[leaf_idx[i]] = node[i];
            }
        }
    }
    TB_CHECK(pos == 2*ndim - 1, TB_ERR_ARG, "DPD: bad layout tree");

    // set_size (dpd_marray_base.hpp:121-169)
    size.assign(2*ndim - 1, std::vector<i64>(nirrep, 0));
    perm.assign(ndim, 0);
    const bool column_major = layout == 0 || layout == 2 || layout == 4;
    for (unsigned i = 0; i < ndim; i++)
    {
        if (column_major)
        {
            size[leaf[i]] = len[i];
            perm[i] = i;
        }
        else
        {
            size[leaf[ndim - 1 - i]] = len[i];
            perm[i] = ndim - 1 - i;
        }
    }
    for (unsigned i = 0; i + 1 < ndim; i++)
    {
        unsigned next = parent[2*i];
        for (unsigned irr1 = 0; irr1 < nirrep; irr1++)
        {
            size[next][irr1] = 0;
            for (unsigned irr2 = 0; irr2 < nirrep; irr2++)
                size[next][irr1] += size[2*i][irr1 ^ irr2]*size[2*i + 1][irr2];
        }
    }
}

void DpdLayout::init_explicit(unsigned irrep_, unsigned nirrep_, unsigned ndim_, const i64* lens,
                              const i64* offsets, const i64* strides)
{
    TB_CHECK(ndim_ >= 1 && ndim_ <= 16, TB_ERR_ARG, "DPD: 1..16 dimensions");
    TB_CHECK(nirrep_ == 1 || nirrep_ == 2 || nirrep_ == 4 || nirrep_ == 8, TB_ERR_ARG, "DPD: nirrep must be 1, 2, 4 or 8");
    TB_CHECK(irrep_ < nirrep_, TB_ERR_ARG, "DPD: irrep out of range");
    TB_CHECK(offsets && strides, TB_ERR_ARG, "DPD: null block table");
    ndim = ndim_; nirrep = nirrep_; irrep = irrep_; layout = -1;
    len.assign(ndim, std::vector<i64>(nirrep));
    for (unsigned d = 0; d < ndim; d++)
        for (unsigned r = 0; r < nirrep; r++)
        {
            len[d][r] = lens[(size_t)d*nirrep + r];
            TB_CHECK(len[d][r] >= 0, TB_ERR_ARG, "DPD: negative length");
        }
    size_t nt = 1;
    for (unsigned d = 0; d < ndim; d++) nt *= nirrep;
    TB_CHECK(nt <= ((size_t)1 << 24), TB_ERR_SIZE, "DPD: block table too large");
    xoff.assign(offsets, offsets + nt);
    xstride.assign(strides, strides + nt*ndim);
    xextent = 0;
    // every stored block must be given, with non-negative geometry
    std::vector<unsigned> irr(ndim, 0);
    for (size_t t = 0; t < nt; t++)
    {
        unsigned x = 0;
        i64 ext = 1, last = 0;
        for (unsigned d = 0; d < ndim; d++) { x ^= irr[d]; ext *= len[d][irr[d]]; }
        if (x == irrep && ext > 0)
        {
            TB_CHECK(xoff[t] >= 0, TB_ERR_ARG, "DPD: block table lacks a stored block");
            for (unsigned d = 0; d < ndim; d++)
            {
                TB_CHECK(xstride[t*ndim + d] >= 0, TB_ERR_ARG, "DPD: negative block stride");
                last += (len[d][irr[d]] - 1)*xstride[t*ndim + d];
            }
            xextent = std::max(xextent, xoff[t] + last + 1);
        }
        unsigned d = 0;
        while (d < ndim && ++irr[d] == nirrep) { irr[d] = 0; d++; }
    }
}

// get_block (dpd_marray_base.hpp:171-228) for a full (unsliced) tensor
DpdLayout scaled_layout(const DpdLayout& X, i64 scale, i64 shift)
{
    size_t nt = 1;
    for (unsigned d = 0; d < X.ndim; d++) nt *= X.nirrep;
    std::vector<i64> lens((size_t)X.ndim*X.nirrep), offs(nt, -1), strides(nt*X.ndim, 0);
    for (unsigned d = 0; d < X.ndim; d++)
        for (unsigned r = 0; r < X.nirrep; r++) lens[(size_t)d*X.nirrep + r] = X.len[d][r];
    X.for_each_block([&](const std::vector<unsigned>& irr, const std::vector<i64>&, const std::vector<i64>& bs,
                         i64 off)
    {
        size_t t = 0;
        for (unsigned d = X.ndim; d-- > 0;) t = t*X.nirrep + irr[d];
        offs[t] = off*scale + shift;
        for (unsigned d = 0; d < X.ndim; d++) strides[t*X.ndim + d] = bs[d]*scale;
    });
    DpdLayout out;
    out.init_explicit(X.irrep, X.nirrep, X.ndim, lens.data(), offs.data(), strides.data());
    return out;
}

void DpdLayout::block(const unsigned* irreps, i64* blen, i64* bstride, i64& offset) const
{
    if (is_explicit())
    {
        size_t t = 0;
        for (unsigned d = ndim; d-- > 0;) t = t*nirrep + irreps[d];
        offset = xoff[t];
        for (unsigned d = 0; d < ndim; d++)
        {
            blen[d] = len[d][irreps[d]];
            bstride[d] = xstride[t*ndim + d];
        }
        return;
    }
    std::vector<unsigned> dirrep(2*ndim - 1, 0);
    std::vector<i64> dstride(2*ndim - 1, 0);
    dstride[2*ndim - 2] = 1;
    // stored lengths are reversed for row-major layouts; perm maps them back
    for (unsigned i = 0; i < ndim; i++) dirrep[leaf[perm[i]]] = irreps[i];
    for (unsigned i = 0; i + 1 < ndim; i++) dirrep[parent[2*i]] = dirrep[2*i] ^ dirrep[2*i + 1];
    offset = 0;
    for (unsigned i = ndim - 1; i-- > 0;)
    {
        const unsigned irr = dirrep[parent[2*i]];
        dstride[2*i] = dstride[parent[2*i]];
        dstride[2*i + 1] = dstride[2*i]*size[2*i][dirrep[2*i]];
        i64 off = 0;
        for (unsigned irr1 = 0; irr1 < dirrep[2*i + 1]; irr1++)
            off += size[2*i][irr1 ^ irr]*size[2*i + 1][irr1];
        offset += off*dstride[2*i];
    }
    for (unsigned i = 0; i < ndim; i++)
    {
        bstride[i] = dstride[leaf[perm[i]]];
        blen[i] = len[i][irreps[i]];
    }
}

namespace
{

// irrep combinations of n labels with XOR == target, in the order of
// src/internal/1t/dpd/util.hpp:14-68 (irrep_iterator: the last n-1 labels run
// as an odometer with the second label fastest, the first label closes the XOR)
std::vector<std::vector<unsigned>> combos(unsigned n, unsigned target, unsigned nirrep)
{
    std::vector<std::vector<unsigned>> out;
    if (n == 0)
    {
        if (target == 0) out.push_back({});
        return out;
    }
    std::vector<unsigned> pos(n - 1, 0);
    while (true)
    {
        std::vector<unsigned> c(n);
        unsigned x = target;
        for (unsigned i = 1; i < n; i++) { c[i] = pos[i - 1]; x ^= pos[i - 1]; }
        c[0] = x;
        out.push_back(c);
        unsigned d = 0;
        while (d < n - 1 && ++pos[d] == nirrep) { pos[d] = 0; d++; }
        if (d == n - 1) break;
    }
    return out;
}

// One operand's patch matrix for a (row group, column group) pair: offset of
// element (r, c) = row[r] + col[c]. Returns false when the layout does not
// split that way (checked on every block pair).
bool patch_view(const DpdLayout& X, const std::vector<unsigned>& rdims,
                const std::vector<std::vector<unsigned>>& rcombos,
                const std::vector<unsigned>& cdims, const std::vector<std::vector<unsigned>>& ccombos,
                ivec& row, ivec& col)
{
    row.clear(); col.clear();
    const unsigned nd = X.ndim;
    std::vector<unsigned> irr(nd);
    std::vector<i64> bl(nd), bs(nd);
    auto blk = [&](const std::vector<unsigned>& rc, const std::vector<unsigned>& cc, i64& off)
    {
        for (size_t i = 0; i < rdims.size(); i++) irr[rdims[i]] = rc[i];
        for (size_t i = 0; i < cdims.size(); i++) irr[cdims[i]] = cc[i];
        X.block(irr.data(), bl.data(), bs.data(), off);
    };
    auto extent = [&](const std::vector<unsigned>& dims, const std::vector<unsigned>& c)
    {
        i64 e = 1;
        for (size_t i = 0; i < dims.size(); i++) e *= X.len[dims[i]][c[i]];
        return e;
    };
    // reference combinations: the first non-empty ones
    size_t r0 = rcombos.size(), c0 = ccombos.size();
    for (size_t i = 0; i < rcombos.size(); i++) if (extent(rdims, rcombos[i]) > 0) { r0 = i; break; }
    for (size_t i = 0; i < ccombos.size(); i++) if (extent(cdims, ccombos[i]) > 0) { c0 = i; break; }
    if (r0 == rcombos.size() || c0 == ccombos.size()) return true;   // empty patch

    i64 base00;
    blk(rcombos[r0], ccombos[c0], base00);
    std::vector<i64> rstr0, cstr0;
    // rows
    for (size_t ri = 0; ri < rcombos.size(); ri++)
    {
        const i64 ext = extent(rdims, rcombos[ri]);
        if (ext == 0) continue;
        i64 baseR;
        blk(rcombos[ri], ccombos[c0], baseR);
        ivec lens, strs;
        for (unsigned d : rdims) { lens.push_back(bl[d]); strs.push_back(bs[d]); }
        const i64 shift = baseR - base00;
        std::vector<i64> sc(ext), tmp(ext);
        fill_block_scatter(lens, strs, 1, 0, ext, sc.data(), tmp.data(), false);
        for (i64 v : sc) row.push_back(v + shift);
        // every column combination must see the same row strides
        for (size_t ci = 0; ci < ccombos.size(); ci++)
        {
            if (extent(cdims, ccombos[ci]) == 0) continue;
            i64 b;
            blk(rcombos[ri], ccombos[ci], b);
            for (size_t i = 0; i < rdims.size(); i++) if (bs[rdims[i]] != strs[i]) return false;
            i64 b0c, bR0;
            blk(rcombos[r0], ccombos[ci], b0c);
            blk(rcombos[ri], ccombos[c0], bR0);
            if (b - bR0 - b0c + base00 != 0) return false;
        }
    }
    // columns
    for (size_t ci = 0; ci < ccombos.size(); ci++)
    {
        const i64 ext = extent(cdims, ccombos[ci]);
        if (ext == 0) continue;
        i64 baseC;
        blk(rcombos[r0], ccombos[ci], baseC);
        ivec lens, strs;
        for (unsigned d : cdims) { lens.push_back(bl[d]); strs.push_back(bs[d]); }
        for (size_t ri = 0; ri < rcombos.size(); ri++)
        {
            if (extent(rdims, rcombos[ri]) == 0) continue;
            i64 b;
            blk(rcombos[ri], ccombos[ci], b);
            for (size_t i = 0; i < cdims.size(); i++) if (bs[cdims[i]] != strs[i]) return false;
        }
        std::vector<i64> sc(ext), tmp(ext);
        fill_block_scatter(lens, strs, 1, 0, ext, sc.data(), tmp.data(), false);
        for (i64 v : sc) col.push_back(v + baseC);
    }
    return true;
}

// offsets inside the block `irr` of X over the dims `dims` (first fastest),
// plus the block's base offset
ivec block_part(const DpdLayout& X, const std::vector<unsigned>& irr, const std::vector<unsigned>& dims, i64& base)
{
    std::vector<i64> bl(X.ndim), bs(X.ndim);
    X.block(irr.data(), bl.data(), bs.data(), base);
    ivec lens, strs;
    i64 ext = 1;
    for (unsigned d : dims) { lens.push_back(bl[d]); strs.push_back(bs[d]); ext *= bl[d]; }
    ivec out(ext), tmp(std::max<i64>(ext, 1));
    if (ext > 0) fill_block_scatter(lens, strs, 1, 0, ext, out.data(), tmp.data(), false);
    return out;
}

int gather_mode(const ivec& mvec, const ivec& kvec)
{
    auto lead = [](const ivec& v) { return v.size() > 1 ? std::llabs(v[1] - v[0]) : (i64)1 << 60; };
    return lead(mvec) < lead(kvec) ? 0 : 1;
}

} // namespace

// key of everything a DPD plan depends on except the data pointers
static std::string dpd_key(const DpdTensor& A, const char* ia, const DpdTensor& B, const char* ib,
                           const DpdTensor& C, const char* ic)
{
    std::string k;
    for (const DpdTensor* t : {&A, &B, &C})
    {
        const DpdLayout& l = t->lay;
        k += std::to_string(l.ndim) + "," + std::to_string(l.nirrep) + "," + std::to_string(l.irrep) + "," +
             std::to_string(l.layout) + ":";
        for (auto& r : l.len) for (i64 x : r) k += std::to_string(x) + ",";
        if (l.is_explicit())
        {
            k.append(reinterpret_cast<const char*>(l.xoff.data()), l.xoff.size()*sizeof(i64));
            k.append(reinterpret_cast<const char*>(l.xstride.data()), l.xstride.size()*sizeof(i64));
        }
        k += "|";
    }
    k += std::string(ia) + "|" + ib + "|" + ic;
    return k;
}

namespace
{

// the label groups of a DPD contraction and whether its irreps rule it out
struct DpdLabels
{
    std::string ABC, AB, AC, BC;
    bool mismatch = false;
};

DpdLabels dpd_labels(const DpdTensor& A, const char* idx_A, const DpdTensor& B, const char* idx_B,
                     const DpdTensor& C, const char* idx_C, bool reference_irrep_check)
{
    const unsigned nirrep = A.lay.nirrep;
    TB_CHECK(B.lay.nirrep == nirrep && C.lay.nirrep == nirrep, TB_ERR_ARG, "DPD: nirrep differs");
    const std::string iA(idx_A, A.lay.ndim), iB(idx_B, B.lay.ndim), iC(idx_C, C.lay.ndim);
    for (const std::string* s : {&iA, &iB, &iC})
        for (size_t i = 0; i < s->size(); i++)
            for (size_t j = 0; j < i; j++)
                TB_CHECK((*s)[i] != (*s)[j], TB_ERR_ARG, "DPD: repeated label in one tensor");

    std::string ABC, AB, AC, BC;
    for (char c : iA)
    {
        bool b = iB.find(c) != std::string::npos, cc = iC.find(c) != std::string::npos;
        if (b && cc) ABC.push_back(c);
        else if (b) AB.push_back(c);
        else if (cc) AC.push_back(c);
        else throw error(TB_ERR_ARG, "DPD: label appears only in A");
    }
    for (char c : iB)
        if (iA.find(c) == std::string::npos)
        {
            if (iC.find(c) != std::string::npos) BC.push_back(c);
            else throw error(TB_ERR_ARG, "DPD: label appears only in B");
        }
    for (char c : iC)
        TB_CHECK(iA.find(c) != std::string::npos || iB.find(c) != std::string::npos, TB_ERR_ARG,
                 "DPD: label appears only in C");
    auto pos = [](const std::string& s, char c) { return (unsigned)s.find(c); };
    auto same_len = [&](const DpdTensor& X, const std::string& ix, const DpdTensor& Y, const std::string& iy,
                        const std::string& labs)
    {
        for (char c : labs)
            TB_CHECK(X.lay.len[pos(ix, c)] == Y.lay.len[pos(iy, c)], TB_ERR_ARG, "DPD: per-irrep lengths differ");
    };
    same_len(A, iA, B, iB, AB); same_len(A, iA, C, iC, AC); same_len(B, iB, C, iC, BC);
    same_len(A, iA, B, iB, ABC); same_len(A, iA, C, iC, ABC);

    // src/iface/3t/mult.cxx:270: "A.irrep()^B.irrep() != C.irrep()" parses as
    // A.irrep() ^ (B.irrep() != C.irrep()); kept as is
    const unsigned irrA = A.lay.irrep, irrB = B.lay.irrep, irrC = C.lay.irrep;
    const bool mismatch = reference_irrep_check ? (irrA ^ (unsigned)(irrB != irrC)) != 0
                                                : (irrA ^ irrB) != irrC;
    DpdLabels r;
    r.ABC = ABC; r.AB = AB; r.AC = AC; r.BC = BC;
    r.mismatch = mismatch;
    return r;
}

// the cached grouped plan of a DPD contraction
// the unit of work a stored C block belongs to: its AC and batch irreps, a
// row band of one irrep GEMM (src/internal/3t/dpd/mult.cxx:308; the irrep of
// the contracted labels follows from them), numbered over those dims of C in
// C's dimension order
size_t dpd_block_unit(const DpdLabels& lab, const std::string& iC, unsigned nirrep,
                      const std::vector<unsigned>& irrC)
{
    size_t u = 0;
    for (size_t d = iC.size(); d-- > 0;)
        if (lab.AC.find(iC[d]) != std::string::npos || lab.ABC.find(iC[d]) != std::string::npos)
            u = u*nirrep + irrC[d];
    return u;
}

// the C blocks a plan covers: every block (owned == nullptr) or those whose
// unit is marked in *owned
struct DpdShare
{
    const std::vector<char>* owned = nullptr;
    const DpdLabels* lab = nullptr;
    std::string iC;
    unsigned nirrep = 1;
    bool covers(const std::vector<unsigned>& irrC) const
    {
        return !owned || (*owned)[dpd_block_unit(*lab, iC, nirrep, irrC)];
    }
};

std::shared_ptr<GroupedPlan> dpd_plan(const DpdTensor& A, const char* idx_A, const DpdTensor& B, const char* idx_B,
                                      const DpdTensor& C, const char* idx_C, const DpdLabels& lab, cudaStream_t st,
                                      const DpdShare& share = DpdShare())
{
    const unsigned nirrep = A.lay.nirrep;
    const std::string iA(idx_A, A.lay.ndim), iB(idx_B, B.lay.ndim), iC(idx_C, C.lay.ndim);
    auto pos = [](const std::string& s, char c) { return (unsigned)s.find(c); };
    const unsigned irrA = A.lay.irrep, irrB = B.lay.irrep;
    std::string AB = lab.AB, AC = lab.AC, BC = lab.BC;

    // label order inside each group: stride order of the dense-equivalent
    // layout (src/internal/3t/dpd/mult.cxx:256-270), C then A (AC), C then B
    // (BC), A then B (AB)
    auto dense_stride = [](const DpdTensor& X, unsigned d)
    {
        if (X.lay.is_explicit())
        {
            // a view's own strides, taken from its first stored block
            i64 s = 0;
            bool found = false;
            X.lay.for_each_block([&](const std::vector<unsigned>&, const std::vector<i64>&,
                                     const std::vector<i64>& bs, i64)
            {
                if (!found) { s = bs[d]; found = true; }
            });
            return s;
        }
        // row-major layouts: last dimension fastest
        const bool cm = X.lay.layout == 0 || X.lay.layout == 2 || X.lay.layout == 4;
        i64 s = 1;
        if (cm) { for (unsigned j = 0; j < d; j++) { i64 t = 0; for (i64 x : X.lay.len[j]) t += x; s *= t; } }
        else { for (unsigned j = X.lay.ndim - 1; j > d; j--) { i64 t = 0; for (i64 x : X.lay.len[j]) t += x; s *= t; } }
        return s;
    };
    auto order = [&](std::string labs, const DpdTensor& X, const std::string& ix, const DpdTensor& Y,
                     const std::string& iy)
    {
        ivec sx, sy;
        for (char c : labs) { sx.push_back(dense_stride(X, pos(ix, c))); sy.push_back(dense_stride(Y, pos(iy, c))); }
        auto p = sort_by_stride({&sx, &sy});
        std::string r;
        for (unsigned i : p) r.push_back(labs[i]);
        return r;
    };
    AC = order(AC, C, iC, A, iA);
    BC = order(BC, C, iC, B, iB);
    AB = order(AB, A, iA, B, iB);
    auto dims = [&](const std::string& labs, const std::string& ix)
    {
        std::vector<unsigned> d;
        for (char c : labs) d.push_back(pos(ix, c));
        return d;
    };

    std::string key = dpd_key(A, idx_A, B, idx_B, C, idx_C);
    if (share.owned)
    {
        key += "|units:";
        for (char o : *share.owned) key.push_back(o ? '1' : '0');
    }
    auto plan = grouped_plan_cache().find(key);
    if (!plan && !lab.ABC.empty())
    {
        // batch labels (in A, B and C): C = alpha*A*B + beta*C element-wise
        // along them, as the reference's FULL and BLOCKED paths compute it
        // (src/internal/3t/dpd/mult.cxx:28-74, 670-847). For every stored C
        // block, split its irreps into AC (r), BC (c) and batch (t) parts.
        // Only blocks with XOR(t) = irrep(A)^irrep(B)^irrep(C) receive
        // products (A and B blocks exist for both only then); each batch
        // element z of such a block is one group of the grouped launch
        // (rows AC, columns BC, one K segment per AB irrep combination, every
        // offset shifted by z through that block's own batch strides). Other
        // blocks, and groups without contracted blocks, are beta-only patches.
        auto p = std::make_shared<GroupedPlan>();
        double flops = 0;
        const std::string ABC = lab.ABC;
        const unsigned x_need = A.lay.irrep ^ B.lay.irrep ^ C.lay.irrep;
        const auto dAC = dims(AC, iA), dAB = dims(AB, iA), dBAB = dims(AB, iB), dBBC = dims(BC, iB);
        const auto dCAC = dims(AC, iC), dCBC = dims(BC, iC);
        const auto zA = dims(ABC, iA), zB = dims(ABC, iB), zC = dims(ABC, iC);
        std::vector<unsigned> dCACZ = dCAC;
        dCACZ.insert(dCACZ.end(), zC.begin(), zC.end());
        C.lay.for_each_block([&](const std::vector<unsigned>& irrC, const std::vector<i64>& cl,
                                 const std::vector<i64>& cs, i64 baseC)
        {
            unsigned xr = 0, xt = 0;
            std::vector<unsigned> r(AC.size()), c(BC.size()), t(ABC.size());
            for (size_t i = 0; i < AC.size(); i++) { r[i] = irrC[dCAC[i]]; xr ^= r[i]; }
            for (size_t i = 0; i < BC.size(); i++) c[i] = irrC[dCBC[i]];
            for (size_t i = 0; i < ABC.size(); i++) { t[i] = irrC[zC[i]]; xt ^= t[i]; }
            if (!share.covers(irrC)) return;                              // another rank's unit
            i64 dummy;
            if (xt != x_need)
            {
                // no A and B blocks meet here: beta only, over the whole block
                ivec pm = block_part(C.lay, irrC, dCACZ, dummy), pn = block_part(C.lay, irrC, dCBC, dummy);
                for (i64& x : pm) x += baseC;
                if (!pm.empty() && !pn.empty()) p->empty_patches.push_back({std::move(pm), std::move(pn)});
                return;
            }
            // the A and B blocks of each AB irrep combination k
            const auto kc = combos((unsigned)AB.size(), A.lay.irrep ^ xr ^ xt, nirrep);
            struct Pair { std::vector<unsigned> ia, ib; };
            std::vector<Pair> pairs;
            for (auto& k : kc)
            {
                Pair q;
                q.ia.assign(A.lay.ndim, 0);
                q.ib.assign(B.lay.ndim, 0);
                for (size_t i = 0; i < AC.size(); i++) q.ia[dAC[i]] = r[i];
                for (size_t i = 0; i < AB.size(); i++) { q.ia[dAB[i]] = k[i]; q.ib[dBAB[i]] = k[i]; }
                for (size_t i = 0; i < BC.size(); i++) q.ib[dBBC[i]] = c[i];
                for (size_t i = 0; i < ABC.size(); i++) { q.ia[zA[i]] = t[i]; q.ib[zB[i]] = t[i]; }
                pairs.push_back(std::move(q));
            }
            ivec cm0 = block_part(C.lay, irrC, dCAC, dummy), cn = block_part(C.lay, irrC, dCBC, dummy);
            if (cm0.empty() || cn.empty()) return;
            // batch elements of this block (odometer over the batch dims, first fastest)
            std::vector<i64> zl(ABC.size());
            i64 nz = 1;
            for (size_t i = 0; i < ABC.size(); i++) { zl[i] = cl[zC[i]]; nz *= zl[i]; }
            std::vector<i64> z(ABC.size(), 0);
            for (i64 e = 0; e < nz; e++)
            {
                i64 offC = baseC;
                for (size_t i = 0; i < ABC.size(); i++) offC += z[i]*cs[zC[i]];
                GroupTables gb;
                gb.c_m = cm0;
                for (i64& x : gb.c_m) x += offC;
                gb.c_n = cn;
                gb.M = (i64)gb.c_m.size(); gb.N = (i64)gb.c_n.size(); gb.K = 0;
                for (const Pair& q : pairs)
                {
                    std::vector<i64> al(A.lay.ndim), as(A.lay.ndim), bl(B.lay.ndim), bs(B.lay.ndim);
                    i64 baseA, baseB;
                    A.lay.block(q.ia.data(), al.data(), as.data(), baseA);
                    B.lay.block(q.ib.data(), bl.data(), bs.data(), baseB);
                    SegTables sg;
                    sg.a_k = block_part(A.lay, q.ia, dAB, dummy);
                    if (sg.a_k.empty()) continue;
                    for (size_t i = 0; i < ABC.size(); i++) { baseA += z[i]*as[zA[i]]; baseB += z[i]*bs[zB[i]]; }
                    sg.a_m = block_part(A.lay, q.ia, dAC, dummy);
                    sg.b_k = block_part(B.lay, q.ib, dBAB, dummy);
                    sg.b_n = block_part(B.lay, q.ib, dBBC, dummy);
                    for (i64& x : sg.a_m) x += baseA;
                    for (i64& x : sg.b_k) x += baseB;
                    gb.K += (i64)sg.a_k.size();
                    gb.segs.push_back(std::move(sg));
                }
                if (gb.segs.empty()) p->empty_patches.push_back({gb.c_m, gb.c_n});
                else
                {
                    gb.amode = gather_mode(gb.segs[0].a_m, gb.segs[0].a_k);
                    gb.bmode = gather_mode(gb.segs[0].b_n, gb.segs[0].b_k);
                    gb.a_slot = 0; gb.b_slot = 1; gb.c_slot = 2;
                    flops += 2.0*gb.M*gb.N*gb.K;
                    p->groups.push_back(std::move(gb));
                }
                for (size_t i = 0; i < ABC.size() && ++z[i] == zl[i]; i++) z[i] = 0;
            }
        });
        p->flops = flops;
        p->finalize(st);
        plan = grouped_plan_cache().insert(key, p);
    }
    if (!plan)
    {
        auto p = std::make_shared<GroupedPlan>();
        double flops = 0;
        for (unsigned h = 0; h < nirrep; h++)
        {
            const unsigned irr_AC = irrA ^ h, irr_BC = irrB ^ h;
            auto rc = combos((unsigned)AC.size(), irr_AC, nirrep);
            auto cc = combos((unsigned)BC.size(), irr_BC, nirrep);
            if (share.owned && !cc.empty())
            {
                // this rank's row bands only (every block of a band shares its unit)
                std::vector<std::vector<unsigned>> mine;
                const auto dCAC0 = dims(AC, iC), dCBC0 = dims(BC, iC);
                for (auto& r : rc)
                {
                    std::vector<unsigned> irrC(C.lay.ndim, 0);
                    for (size_t i = 0; i < AC.size(); i++) irrC[dCAC0[i]] = r[i];
                    for (size_t i = 0; i < BC.size(); i++) irrC[dCBC0[i]] = cc[0][i];
                    if (share.covers(irrC)) mine.push_back(r);
                }
                rc.swap(mine);
            }
            if (rc.empty()) continue;
            auto kc = combos((unsigned)AB.size(), h, nirrep);
            GroupTables g;
            bool ok = patch_view(A.lay, dims(AC, iA), rc, dims(AB, iA), kc, g.a_m, g.a_k) &&
                      patch_view(B.lay, dims(AB, iB), kc, dims(BC, iB), cc, g.b_k, g.b_n) &&
                      patch_view(C.lay, dims(AC, iC), rc, dims(BC, iC), cc, g.c_m, g.c_n);
            if (ok)
            {
                const i64 M = (i64)g.c_m.size(), N = (i64)g.c_n.size(), K = (i64)g.a_k.size();
                if (M == 0 || N == 0) continue;
                if (K == 0)
                {
                    // no contracted blocks for this irrep: C patch = beta*C patch
                    p->empty_patches.push_back({g.c_m, g.c_n});
                    continue;
                }
                g.M = M; g.N = N; g.K = K;
                g.amode = gather_mode(g.a_m, g.a_k);
                g.bmode = gather_mode(g.b_n, g.b_k);
                g.a_slot = 0; g.b_slot = 1; g.c_slot = 2;
                flops += 2.0*M*N*K;
                p->groups.push_back(std::move(g));
                continue;
            }
            // the labels of a group interleave in the layout tree: one group per
            // C block, one K segment per contributing (A block, B block) pair
            const auto dAC = dims(AC, iA), dAB = dims(AB, iA), dBAB = dims(AB, iB), dBBC = dims(BC, iB);
            const auto dCAC = dims(AC, iC), dCBC = dims(BC, iC);
            for (auto& r : rc)
                for (auto& c : cc)
                {
                    std::vector<unsigned> irrC(C.lay.ndim);
                    for (size_t i = 0; i < AC.size(); i++) irrC[dCAC[i]] = r[i];
                    for (size_t i = 0; i < BC.size(); i++) irrC[dCBC[i]] = c[i];
                    i64 baseC;
                    GroupTables gb;
                    ivec cm = block_part(C.lay, irrC, dCAC, baseC);
                    i64 dummy;
                    gb.c_n = block_part(C.lay, irrC, dCBC, dummy);
                    if (cm.empty() || gb.c_n.empty()) continue;
                    for (i64& x : cm) x += baseC;
                    gb.c_m = std::move(cm);
                    gb.M = (i64)gb.c_m.size(); gb.N = (i64)gb.c_n.size(); gb.K = 0;
                    for (auto& k : kc)
                    {
                        std::vector<unsigned> irrA(A.lay.ndim), irrB(B.lay.ndim);
                        for (size_t i = 0; i < AC.size(); i++) irrA[dAC[i]] = r[i];
                        for (size_t i = 0; i < AB.size(); i++) { irrA[dAB[i]] = k[i]; irrB[dBAB[i]] = k[i]; }
                        for (size_t i = 0; i < BC.size(); i++) irrB[dBBC[i]] = c[i];
                        SegTables sg;
                        i64 baseA, baseB, d2;
                        sg.a_m = block_part(A.lay, irrA, dAC, baseA);
                        sg.a_k = block_part(A.lay, irrA, dAB, d2);
                        sg.b_k = block_part(B.lay, irrB, dBAB, baseB);
                        sg.b_n = block_part(B.lay, irrB, dBBC, d2);
                        if (sg.a_k.empty()) continue;
                        for (i64& x : sg.a_m) x += baseA;
                        for (i64& x : sg.b_k) x += baseB;
                        gb.K += (i64)sg.a_k.size();
                        gb.segs.push_back(std::move(sg));
                    }
                    if (gb.segs.empty())
                    {
                        p->empty_patches.push_back({gb.c_m, gb.c_n});
                        continue;
                    }
                    gb.amode = gather_mode(gb.segs[0].a_m, gb.segs[0].a_k);
                    gb.bmode = gather_mode(gb.segs[0].b_n, gb.segs[0].b_k);
                    gb.a_slot = 0; gb.b_slot = 1; gb.c_slot = 2;
                    flops += 2.0*gb.M*gb.N*gb.K;
                    p->groups.push_back(std::move(gb));
                }
        }
        p->flops = flops;
        p->finalize(st);
        plan = grouped_plan_cache().insert(key, p);
    }
    return plan;
}

} // namespace

void dpd_mult(const DpdTensor& A, const char* idx_A, const DpdTensor& B, const char* idx_B,
              DpdTensor& C, const char* idx_C, double alpha, double beta, cudaStream_t st,
              DpdMultReport* rep, bool reference_irrep_check, const std::vector<char>* owned)
{
    const DpdLabels lab = dpd_labels(A, idx_A, B, idx_B, C, idx_C, reference_irrep_check);
    const i64 ctotal = C.lay.total();
    DpdShare share;
    share.owned = owned;
    share.lab = &lab;
    share.iC.assign(idx_C, C.lay.ndim);
    share.nirrep = C.lay.nirrep;
    if (alpha == 0.0 || (lab.ABC.empty() && lab.mismatch))
    {
        if (beta == 1.0 || ctotal == 0) return;
        if (C.lay.is_explicit() || owned)
        {
            // a view's blocks need not fill [0, extent), and a rank's share is
            // a set of blocks: scale block by block
            C.lay.for_each_block([&](const std::vector<unsigned>& irrC, const std::vector<i64>& bl,
                                     const std::vector<i64>& bs, i64 off)
            {
                if (!share.covers(irrC)) return;
                TB_CHECK(C.lay.ndim <= (unsigned)L1_MAX_DIM, TB_ERR_SIZE, "DPD: too many dimensions");
                Strided s;
                s.ndim = (int)C.lay.ndim;
                for (unsigned d = 0; d < C.lay.ndim; d++) { s.len[d] = bl[d]; s.stride[d] = bs[d]; }
                if (beta == 0.0) l1_set<double>(C.data + off, s, 0.0, st);
                else l1_scale<double>(C.data + off, s, beta, st);
            });
            return;
        }
        Strided s; s.ndim = 1; s.len[0] = ctotal; s.stride[0] = 1;
        if (beta == 0.0) l1_set<double>(C.data, s, 0.0, st);
        else l1_scale<double>(C.data, s, beta, st);
        return;
    }
    const std::shared_ptr<GroupedPlan> plan = dpd_plan(A, idx_A, B, idx_B, C, idx_C, lab, st, share);

    const double* ptrs[3] = {A.data, B.data, C.data};
    // C patches without contracted blocks: beta scaling (rare; irreps with K_h == 0)
    for (auto& ep : plan->empty_patches)
        scale_patch(C.data, ep.first, ep.second, beta, st);
    grouped_run(*plan, ptrs, &alpha, &beta, st);
    if (rep)
    {
        rep->groups = (int)plan->groups.size();
        rep->flops = plan->flops;
        rep->variant = plan->variant;
    }
}

std::vector<int> dpd_shard_owner(const DpdTensor& A, const char* idx_A, const DpdTensor& B, const char* idx_B,
                                 const DpdTensor& C, const char* idx_C, int nranks, std::vector<double>* load,
                                 std::vector<int>* unit_rank_out)
{
    TB_CHECK(nranks >= 1, TB_ERR_ARG, "DPD shard: nranks must be at least 1");
    const DpdLabels lab = dpd_labels(A, idx_A, B, idx_B, C, idx_C, true);
    const unsigned nirrep = C.lay.nirrep;
    const std::string iA(idx_A, A.lay.ndim), iC(idx_C, C.lay.ndim);
    size_t nunits = 1;
    for (char c : iC)
        if (lab.AC.find(c) != std::string::npos || lab.ABC.find(c) != std::string::npos) nunits *= nirrep;
    // flops of each unit from the lengths alone: every C block of the band
    // times the K extent of the AB irrep combinations that reach it
    std::vector<double> flops(nunits, 0.0);
    std::vector<unsigned> ab;
    for (char c : lab.AB) ab.push_back((unsigned)iA.find(c));
    C.lay.for_each_block([&](const std::vector<unsigned>& irrC, const std::vector<i64>& bl,
                             const std::vector<i64>&, i64)
    {
        unsigned h = A.lay.irrep;
        for (char c : lab.AC) h ^= irrC[iC.find(c)];
        for (char c : lab.ABC) h ^= irrC[iC.find(c)];
        double mnz = 1.0;
        for (i64 x : bl) mnz *= (double)x;
        double k = 0.0;
        for (auto& kc : combos((unsigned)ab.size(), h, nirrep))
        {
            double e = 1.0;
            for (size_t i = 0; i < ab.size(); i++) e *= (double)A.lay.len[ab[i]][kc[i]];
            k += e;
        }
        flops[dpd_block_unit(lab, iC, nirrep, irrC)] += 2.0*mnz*std::max(k, 1.0);
    });
    // largest unit first onto the least loaded rank (ties: lower unit, lower rank)
    std::vector<size_t> order(nunits);
    for (size_t u = 0; u < nunits; u++) order[u] = u;
    std::stable_sort(order.begin(), order.end(), [&](size_t x, size_t y) { return flops[x] > flops[y]; });
    std::vector<int> unit_rank(nunits, 0);
    std::vector<double> rl(nranks, 0.0);
    for (size_t u : order)
    {
        if (flops[u] == 0.0) continue;
        int best = 0;
        for (int r = 1; r < nranks; r++) if (rl[r] < rl[best]) best = r;
        unit_rank[u] = best;
        rl[best] += flops[u];
    }
    if (load) *load = rl;
    if (unit_rank_out) *unit_rank_out = unit_rank;
    // the owner of every irrep tuple of C (dimension 0 fastest); -1 where no
    // block is stored
    size_t nt = 1;
    for (unsigned d = 0; d < C.lay.ndim; d++) nt *= nirrep;
    std::vector<int> owner(nt, -1);
    C.lay.for_each_block([&](const std::vector<unsigned>& irrC, const std::vector<i64>&, const std::vector<i64>&, i64)
    {
        size_t t = 0;
        for (unsigned d = C.lay.ndim; d-- > 0;) t = t*nirrep + irrC[d];
        owner[t] = unit_rank[dpd_block_unit(lab, iC, nirrep, irrC)];
    });
    return owner;
}

void dpd_mult_shard(const DpdTensor& A, const char* idx_A, const DpdTensor& B, const char* idx_B,
                    DpdTensor& C, const char* idx_C, double alpha, double beta, int nranks, int rank,
                    cudaStream_t st, DpdMultReport* rep)
{
    TB_CHECK(rank >= 0 && rank < nranks, TB_ERR_ARG, "DPD shard: rank out of range");
    std::vector<int> unit_rank;
    dpd_shard_owner(A, idx_A, B, idx_B, C, idx_C, nranks, nullptr, &unit_rank);
    std::vector<char> owned(unit_rank.size());
    bool any = false;
    for (size_t u = 0; u < unit_rank.size(); u++) { owned[u] = unit_rank[u] == rank; any = any || owned[u]; }
    if (!any) { if (rep) *rep = DpdMultReport(); return; }
    dpd_mult(A, idx_A, B, idx_B, C, idx_C, alpha, beta, st, rep, true, &owned);
}

int dpd_mult_terms(const std::vector<DpdTerm>& terms, cudaStream_t st, DpdMultReport* rep,
                   bool reference_irrep_check)
{
    if (rep) *rep = DpdMultReport();
    std::vector<std::shared_ptr<GroupedPlan>> plans(terms.size());
    std::vector<int> wave(terms.size(), -1);
    std::map<i64, int> seen;
    int nwave = 0;
    for (size_t t = 0; t < terms.size(); t++)
    {
        const DpdTerm& x = terms[t];
        const DpdLabels lab = dpd_labels(*x.a, x.ia, *x.b, x.ib, *x.c, x.ic, reference_irrep_check);
        if (x.alpha == 0.0 || (lab.ABC.empty() && lab.mismatch)) continue;
        plans[t] = dpd_plan(*x.a, x.ia, *x.b, x.ib, *x.c, x.ic, lab, st);
        // beta = 1: C patches without contracted blocks stay as they are
        if (plans[t]->groups.empty()) continue;
        wave[t] = seen[x.c_key]++;
        nwave = std::max(nwave, wave[t] + 1);
        if (rep)
        {
            rep->groups += (int)plans[t]->groups.size();
            rep->flops += plans[t]->flops;
        }
    }
    for (int w = 0; w < nwave; w++)
    {
        std::vector<size_t> mem;
        for (size_t t = 0; t < terms.size(); t++)
            if (wave[t] == w) mem.push_back(t);
        std::vector<const double*> ptrs;
        std::vector<double> alphas, betas(mem.size(), 1.0);
        for (size_t t : mem)
        {
            ptrs.push_back(terms[t].a->data);
            ptrs.push_back(terms[t].b->data);
            ptrs.push_back(terms[t].c->data);
            alphas.push_back(terms[t].alpha);
        }
        std::shared_ptr<GroupedPlan> plan;
        if (mem.size() == 1) plan = plans[mem[0]];
        else
        {
            // the merged plan is keyed by its members' plans, which it keeps
            // alive, so a key never names a freed and reused plan
            std::string key = "dpd-terms:";
            for (size_t t : mem)
            {
                const GroupedPlan* q = plans[t].get();
                key.append(reinterpret_cast<const char*>(&q), sizeof(q));
            }
            plan = grouped_plan_cache().find(key);
            if (!plan)
            {
                auto p = std::make_shared<GroupedPlan>();
                for (size_t i = 0; i < mem.size(); i++)
                {
                    const std::shared_ptr<GroupedPlan>& q = plans[mem[i]];
                    p->parts.push_back(q);
                    for (const GroupTables& g : q->groups)
                    {
                        GroupTables h = g;
                        h.a_slot = 3*(int)i + g.a_slot;
                        h.b_slot = 3*(int)i + g.b_slot;
                        h.c_slot = 3*(int)i + g.c_slot;
                        h.sidx = (int)i;
                        p->groups.push_back(std::move(h));
                    }
                    p->flops += q->flops;
                }
                p->nslots = 3*(int)mem.size();
                p->finalize(st);
                plan = grouped_plan_cache().insert(key, p);
            }
        }
        grouped_run(*plan, ptrs.data(), alphas.data(), betas.data(), st);
        if (rep) rep->variant = plan->variant;
    }
    return nwave;
}

void dpd_terms_z(const DpdLayout& la, const double* a, const char* idx_A, const DpdLayout& lb, const double* b,
                 const char* idx_B, const DpdLayout& lc, double* c, const char* idx_C, zd alpha, i64 c_key,
                 std::deque<DpdTensor>& store, std::vector<DpdTerm>& terms)
{
    if (alpha == 0.0) return;
    auto part = [&](const DpdLayout& l, const double* x, i64 shift)
    {
        store.emplace_back();
        store.back().lay = scaled_layout(l, 2, shift);
        store.back().data = const_cast<double*>(x);
        return &store.back();
    };
    const DpdTensor *ar = part(la, a, 0), *ai = part(la, a, 1), *br = part(lb, b, 0), *bi = part(lb, b, 1);
    const DpdTensor *cr = part(lc, c, 0), *ci = part(lc, c, 1);
    const double alr = alpha.real(), ali = alpha.imag();
    // (A part, B part, coefficient into Re C, coefficient into Im C)
    struct Term { const DpdTensor* x; const DpdTensor* y; double cr, ci; };
    const Term four[4] = {
        {ar, br, alr, ali},         // Ar Br
        {ai, bi, -alr, -ali},       // Ai Bi
        {ar, bi, -ali, alr},        // Ar Bi
        {ai, br, -ali, alr},        // Ai Br
    };
    for (const Term& t : four)
        for (int p = 0; p < 2; p++)
        {
            DpdTerm d;
            d.a = t.x; d.ia = idx_A;
            d.b = t.y; d.ib = idx_B;
            d.c = p == 0 ? cr : ci; d.ic = idx_C;
            d.alpha = p == 0 ? t.cr : t.ci;
            d.c_key = 2*c_key + p;
            if (d.alpha != 0.0) terms.push_back(d);
        }
}

void dpd_mult_z(const DpdLayout& la, const double* a, const char* idx_A, const DpdLayout& lb, const double* b,
                const char* idx_B, const DpdLayout& lc, double* c, const char* idx_C, zd alpha, zd beta,
                cudaStream_t st, DpdMultReport* rep, bool reference_irrep_check)
{
    const std::string iC(idx_C, lc.ndim);
    // beta first (set when zero: beta == 0 never reads C), on the complex layout
    if (beta == 0.0) dpd_unary_dev_t(TYPE_DCOMPLEX, 1, 0.0, 1.0, lc, c, iC);
    else if (beta != 1.0) dpd_unary_dev_t(TYPE_DCOMPLEX, 0, 0.0, beta, lc, c, iC);
    if (rep) *rep = DpdMultReport();
    if (alpha == 0.0) return;
    // the real and imaginary parts of C are disjoint, so each pair of terms
    // that write them shares a launch
    std::deque<DpdTensor> store;
    std::vector<DpdTerm> terms;
    dpd_terms_z(la, a, idx_A, lb, b, idx_B, lc, c, idx_C, alpha, 0, store, terms);
    dpd_mult_terms(terms, st, rep, reference_irrep_check);
}

} // namespace tb
