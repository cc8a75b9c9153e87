// shard.cpp -- a contraction split across ranks (one process per GPU) with no
// collective on the data path: C is partitioned along one of its labels that
// is not contracted, and each rank computes its slab of C from the matching
// slice of A (label in A and C) or of B (label in B and C). The slabs are
// disjoint and cover C, so an optional all-gather of C is the only exchange.
//
// The label is chosen the same way on every rank from the tensors' shapes
// alone: the longest label of C that appears in C and exactly one of A and B,
// ties to the first in C's label order. Rank r of n owns the range
// [len*r/n, len*(r+1)/n) of it. A label repeated in one tensor (a diagonal) is
// cut in every one of its dimensions alike.
#include "common.hpp"
#include "mult.hpp"

#include <cstring>
#include <string>
#include <vector>

namespace tb
{

namespace
{

size_t elem_bytes_of(int type)
{
    switch (type)
    {
        case TYPE_FLOAT: return 4;
        case TYPE_DOUBLE: return 8;
        case TYPE_SCOMPLEX: return 8;
        case TYPE_DCOMPLEX: return 16;
    }
    throw error(TB_ERR_TYPE, "unknown tensor type");
}

std::string labels_of(const tblis_tensor* t, const label_type* idx)
{
    return std::string(idx ? idx : "", t->ndim);
}

// the extent of `label` in tensor t (0 when t lacks it)
i64 extent_of(const tblis_tensor* t, const std::string& lab, char label)
{
    for (unsigned d = 0; d < t->ndim; d++)
        if (lab[d] == label) return t->len[d];
    return 0;
}

struct Plan
{
    char label = 0;        // 0: no label to cut (rank 0 computes everything)
    i64 begin = 0, end = 0;
    int where = -1;        // 0: the label is in A and C, 1: in B and C
};

Plan make_plan(const tblis_tensor* A, const label_type* idx_A, const tblis_tensor* B, const label_type* idx_B,
               const tblis_tensor* C, const label_type* idx_C, int nranks, int rank)
{
    TB_CHECK(A && B && C, TB_ERR_ARG, "null tensor");
    TB_CHECK(nranks >= 1 && rank >= 0 && rank < nranks, TB_ERR_ARG, "shard: rank outside 0..nranks-1");
    const std::string iA = labels_of(A, idx_A), iB = labels_of(B, idx_B), iC = labels_of(C, idx_C);
    Plan p;
    i64 best = 0;
    for (unsigned d = 0; d < C->ndim; d++)
    {
        const char c = iC[d];
        const bool inA = iA.find(c) != std::string::npos, inB = iB.find(c) != std::string::npos;
        if (inA == inB) continue;                 // contracted-free labels only: AC or BC
        if (C->len[d] > best)
        {
            best = C->len[d];
            p.label = c;
            p.where = inA ? 0 : 1;
        }
    }
    if (!p.label)
    {
        p.begin = 0;
        p.end = rank == 0 ? 1 : 0;                // no cut: rank 0 owns the whole contraction
        return p;
    }
    p.begin = best*rank/nranks;
    p.end = best*(rank + 1)/nranks;
    return p;
}

// t restricted to label in [b, e): shorter extent, data moved to the start
struct SubTensor
{
    std::vector<len_type> len;
    tblis_tensor t;
    SubTensor(const tblis_tensor* x, const std::string& lab, char label, i64 b, i64 e)
    {
        t = *x;
        len.assign(x->len, x->len + x->ndim);
        i64 off = 0;
        for (unsigned d = 0; d < x->ndim; d++)
            if (lab[d] == label)
            {
                len[d] = e - b;
                off += b*x->stride[d];
            }
        t.len = len.data();
        if (x->data) t.data = static_cast<char*>(x->data) + off*(i64)elem_bytes_of(x->type);
    }
};

} // namespace

} // namespace tb

using namespace tb;

extern "C" {

int tblis_b200_shard_plan(const tblis_tensor* A, const label_type* idx_A,
                          const tblis_tensor* B, const label_type* idx_B,
                          const tblis_tensor* C, const label_type* idx_C,
                          int nranks, int rank, char* label, len_type* begin, len_type* end)
{
    return guarded([&]
    {
        TB_CHECK(label && begin && end, TB_ERR_ARG, "null output");
        const Plan p = make_plan(A, idx_A, B, idx_B, C, idx_C, nranks, rank);
        *label = p.label;
        *begin = p.begin;
        *end = p.end;
    });
}

int tblis_b200_tensor_mult_shard(const tblis_config* cfg,
                                 const tblis_tensor* A, const label_type* idx_A,
                                 const tblis_tensor* B, const label_type* idx_B,
                                       tblis_tensor* C, const label_type* idx_C,
                                 int nranks, int rank, tblis_b200_report* report)
{
    return guarded([&]
    {
        const Plan p = make_plan(A, idx_A, B, idx_B, C, idx_C, nranks, rank);
        if (report) std::memset(report, 0, sizeof(*report));
        if (p.end > p.begin)
        {
            if (!p.label)
                mult_dispatch(cfg, A, idx_A, B, idx_B, C, idx_C, nullptr, report);
            else
            {
                const std::string iA = labels_of(A, idx_A), iB = labels_of(B, idx_B), iC = labels_of(C, idx_C);
                SubTensor sc(C, iC, p.label, p.begin, p.end);
                SubTensor sa(A, iA, p.where == 0 ? p.label : 0, p.begin, p.end);
                SubTensor sb(B, iB, p.where == 1 ? p.label : 0, p.begin, p.end);
                mult_dispatch(cfg, &sa.t, idx_A, &sb.t, idx_B, &sc.t, idx_C, nullptr, report);
            }
        }
        // as after any contraction call, C's scalar and conj are reset
        std::memset(&C->scalar.data, 0, sizeof(C->scalar.data));
        if (C->type == TYPE_FLOAT) C->scalar.data.s = 1.0f;
        else if (C->type == TYPE_DOUBLE) C->scalar.data.d = 1.0;
        else if (C->type == TYPE_SCOMPLEX) C->scalar.data.c[0] = 1.0f;
        else C->scalar.data.z[0] = 1.0;
        C->conj = 0;
    });
}

}
