/*
 * tblis_oracle.c -- TEST INFRASTRUCTURE ONLY (see tblis_oracle.h).
 *
 * Plain-C, single-threaded restatement of the TBLIS reference algorithms on
 * the contraction hot path. It is the checker of the tests, the smoke check
 * and the CPU-baseline leg of the benchmark; the product never uses it.
 * Paths cited are relative to the TBLIS source tree.
 */
#include "tblis_oracle.h"

#include <math.h>
#include <float.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------- */
/* small helpers                                                              */
/* ------------------------------------------------------------------------- */

/* odometer over ndim dims with up to 3 stride vectors; mirrors MArray's
 * viterator (first dim fastest) */
typedef struct it3
{
    unsigned ndim;
    orc_len len[ORC_MAX_DIM];
    orc_len pos[ORC_MAX_DIM];
    orc_stride s[3][ORC_MAX_DIM];
    orc_stride off[3];
    int started, done;
} it3;

static void it3_init(it3* it, unsigned ndim, const orc_len* len,
                     const orc_stride* s0, const orc_stride* s1, const orc_stride* s2)
{
    memset(it, 0, sizeof(*it));
    it->ndim = ndim;
    for (unsigned i = 0; i < ndim; i++)
    {
        it->len[i] = len[i];
        it->s[0][i] = s0 ? s0[i] : 0;
        it->s[1][i] = s1 ? s1[i] : 0;
        it->s[2][i] = s2 ? s2[i] : 0;
        if (len[i] == 0) it->done = 1;
    }
}

/* advances; returns 0 when exhausted. First call yields the origin. */
static int it3_next(it3* it)
{
    if (it->done) return 0;
    if (!it->started) { it->started = 1; return 1; }
    for (unsigned i = 0; i < it->ndim; i++)
    {
        if (++it->pos[i] < it->len[i])
        {
            for (int k = 0; k < 3; k++) it->off[k] += it->s[k][i];
            return 1;
        }
        for (int k = 0; k < 3; k++) it->off[k] -= it->s[k][i]*(it->len[i]-1);
        it->pos[i] = 0;
    }
    it->done = 1;
    return 0;
}

static orc_len prod(unsigned n, const orc_len* l)
{
    orc_len p = 1;
    for (unsigned i = 0; i < n; i++) p *= l[i];
    return p;
}

static int find_label(unsigned n, const char* idx, char c)
{
    for (unsigned i = 0; i < n; i++) if (idx[i] == c) return (int)i;
    return -1;
}

static void sort_chars(unsigned n, char* c)
{
    for (unsigned i = 1; i < n; i++)
        for (unsigned j = i; j > 0 && c[j-1] > c[j]; j--)
        { char t = c[j]; c[j] = c[j-1]; c[j-1] = t; }
}

/* ------------------------------------------------------------------------- */
/* label / stride algebra                                                     */
/* ------------------------------------------------------------------------- */

/* src/util/tensor.hpp:375-412 */
unsigned orc_diagonal(unsigned ndim, const orc_len* len, const orc_stride* stride,
                      const char* idx, orc_len* len_out, orc_stride* stride_out,
                      char* idx_out)
{
    unsigned inds[ORC_MAX_DIM];
    for (unsigned i = 0; i < ndim; i++) inds[i] = i;
    /* order by label (stable insertion sort; equal labels are merged below) */
    for (unsigned i = 1; i < ndim; i++)
        for (unsigned j = i; j > 0 && idx[inds[j-1]] > idx[inds[j]]; j--)
        { unsigned t = inds[j]; inds[j] = inds[j-1]; inds[j-1] = t; }

    unsigned n = 0;
    for (unsigned i = 0; i < ndim; i++)
    {
        if (i == 0 || idx[inds[i]] != idx[inds[i-1]])
        {
            if (len[inds[i]] != 1)
            {
                len_out[n] = len[inds[i]];
                stride_out[n] = stride[inds[i]];
                idx_out[n] = idx[inds[i]];
                n++;
            }
        }
        else if (len[inds[i]] != 1)
        {
            stride_out[n-1] += stride[inds[i]];
        }
    }
    return n;
}

/* src/util/tensor.hpp:95-148 (sort_by_stride_helper ordering) */
void orc_sort_by_stride(unsigned ndim, unsigned nstr, const orc_stride* const* strides,
                        unsigned* perm)
{
    for (unsigned i = 0; i < ndim; i++) perm[i] = i;
    for (unsigned a = 1; a < ndim; a++)
    {
        for (unsigned b = a; b > 0; b--)
        {
            unsigned i = perm[b], j = perm[b-1];
            /* is i < j ? */
            orc_stride mi = strides[0][i], mj = strides[0][j];
            for (unsigned k = 1; k < nstr; k++)
            {
                if (strides[k][i] < mi) mi = strides[k][i];
                if (strides[k][j] < mj) mj = strides[k][j];
            }
            int less = 0, decided = 0;
            if (mi < mj) { less = 1; decided = 1; }
            else if (mi > mj) { less = 0; decided = 1; }
            for (unsigned k = 0; !decided && k < nstr; k++)
            {
                if (strides[k][i] < strides[k][j]) { less = 1; decided = 1; }
                else if (strides[k][i] > strides[k][j]) { less = 0; decided = 1; }
            }
            if (!less) break;
            perm[b] = j; perm[b-1] = i;
        }
    }
}

/* src/util/tensor.hpp:341-373 */
unsigned orc_fold(unsigned ndim, orc_len* len, char* idx, unsigned nstr, orc_stride** strides)
{
    unsigned inds[ORC_MAX_DIM];
    const orc_stride* s0[1] = { strides[0] };
    orc_sort_by_stride(ndim, 1, s0, inds);

    orc_len oldlen[ORC_MAX_DIM];
    char oldidx[ORC_MAX_DIM];
    orc_stride olds[4][ORC_MAX_DIM];
    memcpy(oldlen, len, ndim*sizeof(orc_len));
    memcpy(oldidx, idx, ndim);
    for (unsigned k = 0; k < nstr; k++) memcpy(olds[k], strides[k], ndim*sizeof(orc_stride));

    unsigned n = 0;
    for (unsigned i = 0; i < ndim; i++)
    {
        int contig = i != 0;
        for (unsigned k = 0; contig && k < nstr; k++)
            if (olds[k][inds[i]] != olds[k][inds[i-1]]*oldlen[inds[i-1]]) contig = 0;
        if (contig)
        {
            len[n-1] *= oldlen[inds[i]];
        }
        else
        {
            idx[n] = oldidx[inds[i]];
            len[n] = oldlen[inds[i]];
            for (unsigned k = 0; k < nstr; k++) strides[k][n] = olds[k][inds[i]];
            n++;
        }
    }
    return n;
}

/* src/util/tensor.hpp:33-60 (free_idx over the union of labels) */
static char free_idx(unsigned n, const char* labels)
{
    char s[3*ORC_MAX_DIM];
    memcpy(s, labels, n);
    sort_chars(n, s);
    if (n == 0) return 0;
    if (s[0] > 0) return 0;
    for (unsigned i = 1; i < n; i++) if (s[i] > s[i-1]+1) return (char)(s[i-1]+1);
    return (char)(s[n-1]+1);
}

/* ------------------------------------------------------------------------- */
/* block scatter vectors                                                      */
/* ------------------------------------------------------------------------- */

static orc_len gcd_(orc_len a, orc_len b)
{
    a = a < 0 ? -a : a; b = b < 0 ? -b : b;
    while (b) { orc_len t = a % b; a = b; b = t; }
    return a;
}
static orc_len lcm_(orc_len a, orc_len b) { return a*b/gcd_(a, b); }
static orc_len minl(orc_len a, orc_len b) { return a < b ? a : b; }
static orc_len maxl(orc_len a, orc_len b) { return a > b ? a : b; }

/* position an odometer over (len, stride) at linear index p (first dim fastest) */
static orc_stride offset_of(unsigned ndim, const orc_len* len, const orc_stride* stride, orc_len p)
{
    orc_stride off = 0;
    for (unsigned i = 0; i < ndim; i++) { off += (p % len[i])*stride[i]; p /= len[i]; }
    return off;
}

/* src/matrix/block_scatter_matrix.hpp:68-230 for double (cache line = 8 elements) */
static void fill_scatter(unsigned ndim, const orc_len* len, const orc_stride* stride,
                         orc_len BS, orc_stride off, orc_stride size, orc_stride* scat, int pack_3d)
{
    if (size == 0) return;
    const orc_len CL = 64/8;
    if (ndim == 0) { *scat = 0; return; }

    orc_len m0 = len[0];
    orc_stride s0 = stride[0];

    if (!pack_3d)
    {
        const orc_len* l1 = len+1; const orc_stride* st1 = stride+1; unsigned n1 = ndim-1;
        orc_len nouter = prod(n1, l1);
        orc_len p0 = off % m0;
        orc_len b = off / m0;
        orc_len idx = 0;
        for (; idx < size && b < nouter; b++)
        {
            orc_stride pos = offset_of(n1, l1, st1, b);
            orc_stride pos2 = pos + p0*s0;
            orc_len imax = minl(m0-p0, size-idx);
            for (orc_len i = 0; i < imax; i++) { scat[idx++] = pos2; pos2 += s0; }
            p0 = 0;
        }
        return;
    }

    orc_len m1 = len[1];
    orc_stride s1 = stride[1];
    orc_len BS0 = minl(lcm_(BS, CL), maxl(BS, m0 - m0%BS));
    orc_len BS1 = minl(CL, maxl(BS, m1 - m1%BS));
    const orc_len* l2 = len+2; const orc_stride* st2 = stride+2; unsigned n2 = ndim-2;
    orc_len nouter = prod(n2, l2);

    orc_len p01 = off % (m0*m1);
    orc_len p0 = p01 % m0;
    orc_len p1 = p01 / m0;
    orc_len q01 = (off+size-1) % (m0*m1);
    orc_len q0 = q01 % m0;
    orc_len q1 = q01 / m0;
    orc_len r0 = q0 - q0 % BS0;
    orc_len b_min = off/(m0*m1);
    orc_len b_max = (off+size-1)/(m0*m1)+1;
    if (p0 == 0) p1--;
    if (q0 == m0-1) q1++;

    orc_len idx = 0;
    if (r0 > 0)
    {
        for (orc_len b = b_min; b < b_max && b < nouter; b++)
        {
            orc_stride pos = offset_of(n2, l2, st2, b);
            orc_len min1 = b == b_min ? p1+1 : 0;
            orc_len max1 = b == b_max-1 ? q1 : m1;
            for (orc_len i1 = min1; i1 < max1; i1 += BS1)
            for (orc_len i0 = 0; i0 < r0; i0 += BS0)
            for (orc_len j1 = 0; j1 < minl(BS1, max1-i1); j1++)
            for (orc_len j0 = 0; j0 < BS0; j0++)
                scat[idx++] = pos + (i0+j0)*s0 + (i1+j1)*s1;
        }
    }
    for (orc_len b = b_min; b < b_max && b < nouter; b++)
    {
        orc_stride pos = offset_of(n2, l2, st2, b);
        orc_len min1 = b == b_min ? p1+1 : 0;
        orc_len max1 = b == b_max-1 ? q1 : m1;
        for (orc_len j1 = min1; j1 < max1; j1++)
        for (orc_len j0 = r0; j0 < m0; j0++)
            scat[idx++] = pos + j0*s0 + j1*s1;

        int do_p = b == b_min && p0 > 0;
        int do_q = b == b_max-1 && q0 < m0-1;
        if (do_p && do_q && p1 == q1)
        {
            for (orc_len j0 = p0; j0 <= q0; j0++) scat[idx++] = pos + j0*s0 + p1*s1;
        }
        else
        {
            if (do_p) for (orc_len j0 = p0; j0 < m0; j0++) scat[idx++] = pos + j0*s0 + p1*s1;
            if (do_q) for (orc_len j0 = 0; j0 <= q0; j0++) scat[idx++] = pos + j0*s0 + q1*s1;
        }
    }
}

/* src/matrix/block_scatter_matrix.hpp:232-247 */
static void fill_block_stride(orc_len BS, orc_stride size, const orc_stride* scat, orc_stride* bs)
{
    for (orc_len i = 0; i < size; i += BS)
    {
        orc_len bl = minl(size-i, BS);
        orc_stride s = bl > 1 ? scat[i+1]-scat[i] : 1;
        for (orc_len j = i+1; j+1 < i+bl; j++)
            if (scat[j+1]-scat[j] != s) s = 0;
        bs[i] = s;
    }
}

/* src/matrix/block_scatter_matrix.hpp:249-258 */
void orc_fill_block_scatter(unsigned ndim, const orc_len* len, const orc_stride* stride,
                            orc_len BS, orc_stride off, orc_stride size,
                            orc_stride* scat, orc_stride* bs, int pack_3d)
{
    if (size == 0) return;
    fill_scatter(ndim, len, stride, BS, off, size, scat, pack_3d);
    fill_block_stride(BS, size, scat, bs);
}

/* ------------------------------------------------------------------------- */
/* contraction                                                                */
/* ------------------------------------------------------------------------- */

/* set of labels helpers (sorted, unique) */
static unsigned lab_intersect(unsigned na, const char* a, unsigned nb, const char* b, char* out)
{
    unsigned n = 0;
    for (unsigned i = 0; i < na; i++) if (find_label(nb, b, a[i]) >= 0) out[n++] = a[i];
    sort_chars(n, out);
    return n;
}
static unsigned lab_exclude(unsigned na, const char* a, unsigned nb, const char* b, char* out)
{
    unsigned n = 0;
    for (unsigned i = 0; i < na; i++) if (find_label(nb, b, a[i]) < 0) out[n++] = a[i];
    sort_chars(n, out);
    return n;
}
static void select_from(unsigned nm, const char* match, unsigned n, const char* lab,
                        const orc_len* v, orc_len* out)
{
    for (unsigned i = 0; i < nm; i++) { int j = find_label(n, lab, match[i]); out[i] = v[j]; }
}

/* src/iface/3t/mult.cxx:30-116 */
int orc_mult_groups_build(unsigned ndim_A_, const orc_len* len_A_, const orc_stride* stride_A_, const char* idx_A_,
                          unsigned ndim_B_, const orc_len* len_B_, const orc_stride* stride_B_, const char* idx_B_,
                          unsigned ndim_C_, const orc_len* len_C_, const orc_stride* stride_C_, const char* idx_C_,
                          orc_mult_groups* g)
{
    orc_len lA[ORC_MAX_DIM+2], lB[ORC_MAX_DIM+2], lC[ORC_MAX_DIM+2];
    orc_stride sA[ORC_MAX_DIM+2], sB[ORC_MAX_DIM+2], sC[ORC_MAX_DIM+2];
    char iA[ORC_MAX_DIM+2], iB[ORC_MAX_DIM+2], iC[ORC_MAX_DIM+2];
    if (ndim_A_ > ORC_MAX_DIM || ndim_B_ > ORC_MAX_DIM || ndim_C_ > ORC_MAX_DIM) return -1;
    unsigned nA = orc_diagonal(ndim_A_, len_A_, stride_A_, idx_A_, lA, sA, iA);
    unsigned nB = orc_diagonal(ndim_B_, len_B_, stride_B_, idx_B_, lB, sB, iB);
    unsigned nC = orc_diagonal(ndim_C_, len_C_, stride_C_, idx_C_, lC, sC, iC);

    char t1[ORC_MAX_DIM+2], abc[ORC_MAX_DIM+2];
    unsigned n1 = lab_intersect(nA, iA, nB, iB, t1);
    unsigned nabc = lab_intersect(n1, t1, nC, iC, abc);

    if (nA == nabc || nB == nabc || nC == nabc)
    {
        char all[3*ORC_MAX_DIM+4];
        unsigned na = 0;
        memcpy(all+na, iA, nA); na += nA; memcpy(all+na, iB, nB); na += nB; memcpy(all+na, iC, nC); na += nC;
        char f = free_idx(na, all);
        lA[nA] = 1; sA[nA] = 0; iA[nA++] = f;
        lC[nC] = 1; sC[nC] = 0; iC[nC++] = f;
        na = 0;
        memcpy(all+na, iA, nA); na += nA; memcpy(all+na, iB, nB); na += nB; memcpy(all+na, iC, nC); na += nC;
        f = free_idx(na, all);
        lB[nB] = 1; sB[nB] = 0; iB[nB++] = f;
        lC[nC] = 1; sC[nC] = 0; iC[nC++] = f;
        n1 = lab_intersect(nA, iA, nB, iB, t1);
        nabc = lab_intersect(n1, t1, nC, iC, abc);
    }

    memset(g, 0, sizeof(*g));
    /* ABC */
    g->n_ABC = nabc; memcpy(g->idx_ABC, abc, nabc);
    select_from(nabc, abc, nA, iA, lA, g->len_ABC);
    select_from(nabc, abc, nA, iA, sA, g->sA_ABC);
    select_from(nabc, abc, nB, iB, sB, g->sB_ABC);
    select_from(nabc, abc, nC, iC, sC, g->sC_ABC);
    /* AB */
    char tmp[ORC_MAX_DIM+2];
    unsigned nt = lab_intersect(nA, iA, nB, iB, tmp);
    g->n_AB = lab_exclude(nt, tmp, nabc, abc, g->idx_AB);
    select_from(g->n_AB, g->idx_AB, nA, iA, lA, g->len_AB);
    select_from(g->n_AB, g->idx_AB, nA, iA, sA, g->sA_AB);
    select_from(g->n_AB, g->idx_AB, nB, iB, sB, g->sB_AB);
    /* AC */
    nt = lab_intersect(nA, iA, nC, iC, tmp);
    g->n_AC = lab_exclude(nt, tmp, nabc, abc, g->idx_AC);
    select_from(g->n_AC, g->idx_AC, nA, iA, lA, g->len_AC);
    select_from(g->n_AC, g->idx_AC, nA, iA, sA, g->sA_AC);
    select_from(g->n_AC, g->idx_AC, nC, iC, sC, g->sC_AC);
    /* BC */
    nt = lab_intersect(nB, iB, nC, iC, tmp);
    g->n_BC = lab_exclude(nt, tmp, nabc, abc, g->idx_BC);
    select_from(g->n_BC, g->idx_BC, nB, iB, lB, g->len_BC);
    select_from(g->n_BC, g->idx_BC, nB, iB, sB, g->sB_BC);
    select_from(g->n_BC, g->idx_BC, nC, iC, sC, g->sC_BC);

    /* single-operand labels are not allowed (mult.cxx:98-104) */
    if (g->n_AB + g->n_AC + g->n_ABC != nA) return -2;
    if (g->n_AB + g->n_BC + g->n_ABC != nB) return -2;
    if (g->n_AC + g->n_BC + g->n_ABC != nC) return -2;

    orc_stride* s3[3];
    s3[0] = g->sA_ABC; s3[1] = g->sB_ABC; s3[2] = g->sC_ABC;
    g->n_ABC = orc_fold(g->n_ABC, g->len_ABC, g->idx_ABC, 3, s3);
    s3[0] = g->sA_AB; s3[1] = g->sB_AB;
    g->n_AB = orc_fold(g->n_AB, g->len_AB, g->idx_AB, 2, s3);
    s3[0] = g->sA_AC; s3[1] = g->sC_AC;
    g->n_AC = orc_fold(g->n_AC, g->len_AC, g->idx_AC, 2, s3);
    s3[0] = g->sB_BC; s3[1] = g->sC_BC;
    g->n_BC = orc_fold(g->n_BC, g->len_BC, g->idx_BC, 2, s3);
    return 0;
}

/* src/internal/3t/dense/mult.cxx:653-720 (mult_ref), with the empty-extent
 * early outs of :795-816 and the alpha==0 handling of
 * src/iface/3t/mult.cxx:133-148 */
int orc_tensor_mult_d(double alpha, unsigned ndim_A, const orc_len* len_A, const orc_stride* stride_A,
                      const double* A, const char* idx_A,
                      unsigned ndim_B, const orc_len* len_B, const orc_stride* stride_B,
                      const double* B, const char* idx_B,
                      double beta, unsigned ndim_C, const orc_len* len_C, const orc_stride* stride_C,
                      double* C, const char* idx_C)
{
    orc_mult_groups g;
    int rc = orc_mult_groups_build(ndim_A, len_A, stride_A, idx_A, ndim_B, len_B, stride_B, idx_B,
                                   ndim_C, len_C, stride_C, idx_C, &g);
    if (rc) return rc;

    orc_len n_AB = prod(g.n_AB, g.len_AB), n_AC = prod(g.n_AC, g.len_AC);
    orc_len n_BC = prod(g.n_BC, g.len_BC), n_ABC = prod(g.n_ABC, g.len_ABC);

    /* C's full dim list for set/scale */
    orc_len lc[3*ORC_MAX_DIM]; orc_stride sc[3*ORC_MAX_DIM]; unsigned nc = 0;
    for (unsigned i = 0; i < g.n_AC; i++) { lc[nc] = g.len_AC[i]; sc[nc++] = g.sC_AC[i]; }
    for (unsigned i = 0; i < g.n_BC; i++) { lc[nc] = g.len_BC[i]; sc[nc++] = g.sC_BC[i]; }
    for (unsigned i = 0; i < g.n_ABC; i++) { lc[nc] = g.len_ABC[i]; sc[nc++] = g.sC_ABC[i]; }

    if (alpha == 0.0 || n_AB == 0)
    {
        if (n_AC == 0 || n_BC == 0 || n_ABC == 0) return 0;
        if (beta == 0.0) return orc_tensor_set_d(0.0, nc, lc, sc, C);
        if (beta != 1.0) return orc_tensor_scale_d(beta, nc, lc, sc, C);
        return 0;
    }
    if (n_AC == 0 || n_BC == 0 || n_ABC == 0) return 0;

    it3 iabc; it3_init(&iabc, g.n_ABC, g.len_ABC, g.sA_ABC, g.sB_ABC, g.sC_ABC);
    while (it3_next(&iabc))
    {
        it3 iac; it3_init(&iac, g.n_AC, g.len_AC, g.sA_AC, g.sC_AC, NULL);
        while (it3_next(&iac))
        {
            it3 ibc; it3_init(&ibc, g.n_BC, g.len_BC, g.sB_BC, g.sC_BC, NULL);
            while (it3_next(&ibc))
            {
                const double* A1 = A + iabc.off[0] + iac.off[0];
                const double* B1 = B + iabc.off[1] + ibc.off[0];
                double* C1 = C + iabc.off[2] + iac.off[1] + ibc.off[1];
                double temp = 0.0;
                it3 iab; it3_init(&iab, g.n_AB, g.len_AB, g.sA_AB, g.sB_AB, NULL);
                while (it3_next(&iab)) temp += A1[iab.off[0]]*B1[iab.off[1]];
                temp *= alpha;
                if (beta == 0.0) *C1 = temp;
                else *C1 = temp + beta*(*C1);
            }
        }
    }
    return 0;
}

int orc_tensor_mult_sample_d(double alpha, unsigned ndim_A, const orc_len* len_A, const orc_stride* stride_A,
                             const double* A, const char* idx_A,
                             unsigned ndim_B, const orc_len* len_B, const orc_stride* stride_B,
                             const double* B, const char* idx_B,
                             double beta, unsigned ndim_C, const orc_len* len_C, const orc_stride* stride_C,
                             const double* C, const char* idx_C,
                             orc_len nsample, const orc_len* sample_idx, double* out)
{
    (void)len_C;
    /* contracted labels: in A and B but not C */
    char ab[ORC_MAX_DIM]; orc_len lab[ORC_MAX_DIM]; orc_stride sa[ORC_MAX_DIM], sb[ORC_MAX_DIM];
    unsigned nab = 0;
    for (unsigned i = 0; i < ndim_A; i++)
    {
        char c = idx_A[i];
        if (find_label(ndim_C, idx_C, c) >= 0 || find_label(nab, ab, c) >= 0) continue;
        int jb = find_label(ndim_B, idx_B, c);
        if (jb < 0) return -2;
        ab[nab] = c; lab[nab] = len_A[i];
        sa[nab] = 0; sb[nab] = 0;
        for (unsigned k = 0; k < ndim_A; k++) if (idx_A[k] == c) sa[nab] += stride_A[k];
        for (unsigned k = 0; k < ndim_B; k++) if (idx_B[k] == c) sb[nab] += stride_B[k];
        nab++;
    }
    for (orc_len s = 0; s < nsample; s++)
    {
        const orc_len* ci = sample_idx + s*ndim_C;
        orc_stride oa = 0, ob = 0, oc = 0;
        for (unsigned k = 0; k < ndim_C; k++) oc += ci[k]*stride_C[k];
        for (unsigned k = 0; k < ndim_A; k++)
        {
            int j = find_label(ndim_C, idx_C, idx_A[k]);
            if (j >= 0) oa += ci[j]*stride_A[k];
        }
        for (unsigned k = 0; k < ndim_B; k++)
        {
            int j = find_label(ndim_C, idx_C, idx_B[k]);
            if (j >= 0) ob += ci[j]*stride_B[k];
        }
        double temp = 0.0;
        it3 iab; it3_init(&iab, nab, lab, sa, sb, NULL);
        while (it3_next(&iab)) temp += A[oa + iab.off[0]]*B[ob + iab.off[1]];
        temp *= alpha;
        out[s] = beta == 0.0 ? temp : temp + beta*C[oc];
    }
    return 0;
}

/* ------------------------------------------------------------------------- */
/* level-1                                                                    */
/* ------------------------------------------------------------------------- */

/* src/iface/1t/add.cxx:24-110 + src/internal/1t/dense/add.cxx:15-261 */
int orc_tensor_add_d(double alpha, unsigned ndim_A_, const orc_len* len_A_, const orc_stride* stride_A_,
                     const double* A, const char* idx_A_,
                     double beta, unsigned ndim_B_, const orc_len* len_B_, const orc_stride* stride_B_,
                     double* B, const char* idx_B_)
{
    orc_len lA[ORC_MAX_DIM+1], lB[ORC_MAX_DIM+1];
    orc_stride sA[ORC_MAX_DIM+1], sB[ORC_MAX_DIM+1];
    char iA[ORC_MAX_DIM+1], iB[ORC_MAX_DIM+1];
    unsigned nA = orc_diagonal(ndim_A_, len_A_, stride_A_, idx_A_, lA, sA, iA);
    unsigned nB = orc_diagonal(ndim_B_, len_B_, stride_B_, idx_B_, lB, sB, iB);
    if (nA == 0 || nB == 0)
    {
        char all[2*ORC_MAX_DIM+2]; memcpy(all, iA, nA); memcpy(all+nA, iB, nB);
        char f = free_idx(nA+nB, all);
        lA[nA] = 1; sA[nA] = 0; iA[nA++] = f;
        lB[nB] = 1; sB[nB] = 0; iB[nB++] = f;
    }
    char iab[ORC_MAX_DIM], iao[ORC_MAX_DIM], ibo[ORC_MAX_DIM];
    unsigned nab = lab_intersect(nA, iA, nB, iB, iab);
    unsigned nao = lab_exclude(nA, iA, nab, iab, iao);
    unsigned nbo = lab_exclude(nB, iB, nab, iab, ibo);
    if (nao && nbo) return -2;
    orc_len lab[ORC_MAX_DIM], lao[ORC_MAX_DIM], lbo[ORC_MAX_DIM];
    orc_stride saab[ORC_MAX_DIM], sbab[ORC_MAX_DIM], sao[ORC_MAX_DIM], sbo[ORC_MAX_DIM];
    select_from(nab, iab, nA, iA, lA, lab);
    select_from(nab, iab, nA, iA, sA, saab);
    select_from(nab, iab, nB, iB, sB, sbab);
    select_from(nao, iao, nA, iA, lA, lao);
    select_from(nao, iao, nA, iA, sA, sao);
    select_from(nbo, ibo, nB, iB, lB, lbo);
    select_from(nbo, ibo, nB, iB, sB, sbo);

    orc_len n_AB = prod(nab, lab), n_A = prod(nao, lao), n_B = prod(nbo, lbo);

    if (alpha == 0.0)
    {
        orc_len lb[2*ORC_MAX_DIM]; orc_stride sb[2*ORC_MAX_DIM]; unsigned n = 0;
        for (unsigned i = 0; i < nbo; i++) { lb[n] = lbo[i]; sb[n++] = sbo[i]; }
        for (unsigned i = 0; i < nab; i++) { lb[n] = lab[i]; sb[n++] = sbab[i]; }
        if (beta == 0.0) return orc_tensor_set_d(0.0, n, lb, sb, B);
        if (beta != 1.0) return orc_tensor_scale_d(beta, n, lb, sb, B);
        return 0;
    }
    if (n_AB == 0 || n_B == 0) return 0;
    if (n_A == 0)
    {
        /* internal add: scale B (beta == 0 included) over the B-only dims */
        it3 ib; it3_init(&ib, nbo, lbo, sbo, NULL, NULL);
        while (it3_next(&ib)) B[ib.off[0]] *= beta;
        return 0;
    }

    it3 iabit; it3_init(&iabit, nab, lab, saab, sbab, NULL);
    while (it3_next(&iabit))
    {
        const double* A1 = A + iabit.off[0];
        double* B1 = B + iabit.off[1];
        double sum = 0.0;
        it3 ia; it3_init(&ia, nao, lao, sao, NULL, NULL);
        while (it3_next(&ia)) sum += A1[ia.off[0]];
        sum *= alpha;
        it3 ib; it3_init(&ib, nbo, lbo, sbo, NULL, NULL);
        while (it3_next(&ib))
        {
            double* p = B1 + ib.off[0];
            *p = beta == 0.0 ? sum : sum + beta*(*p);
        }
    }
    return 0;
}

/* src/iface/1t/dot.cxx:16-74, src/internal/1t/dense/dot.cxx:10-50 */
int orc_tensor_dot_d(double alpha_A, unsigned ndim_A, const orc_len* len_A, const orc_stride* stride_A,
                     const double* A, const char* idx_A,
                     double alpha_B, unsigned ndim_B, const orc_len* len_B, const orc_stride* stride_B,
                     const double* B, const char* idx_B, double* result)
{
    orc_len lA[ORC_MAX_DIM], lB[ORC_MAX_DIM];
    orc_stride sA[ORC_MAX_DIM], sB[ORC_MAX_DIM];
    char iA[ORC_MAX_DIM], iB[ORC_MAX_DIM];
    unsigned nA = orc_diagonal(ndim_A, len_A, stride_A, idx_A, lA, sA, iA);
    unsigned nB = orc_diagonal(ndim_B, len_B, stride_B, idx_B, lB, sB, iB);
    char iab[ORC_MAX_DIM];
    unsigned nab = lab_intersect(nA, iA, nB, iB, iab);
    if (nab != nA || nab != nB) return -2;
    orc_len l[ORC_MAX_DIM]; orc_stride sa[ORC_MAX_DIM], sb[ORC_MAX_DIM];
    select_from(nab, iab, nA, iA, lA, l);
    select_from(nab, iab, nA, iA, sA, sa);
    select_from(nab, iab, nB, iB, sB, sb);
    double sum = 0.0;
    it3 it; it3_init(&it, nab, l, sa, sb, NULL);
    while (it3_next(&it)) sum += A[it.off[0]]*B[it.off[1]];
    *result = sum*(alpha_A*alpha_B);
    return 0;
}

/* src/iface/1t/reduce.cxx:16-68 and src/kernels/1v/reduce.hpp:16-106.
 * For MAX/MIN-type ops the first extreme element in memory-offset order of
 * the folded iteration wins ties (strict comparisons), and idx is its offset
 * from A. */
int orc_tensor_reduce_d(int op, double alpha, unsigned ndim_A, const orc_len* len_A,
                        const orc_stride* stride_A, const double* A, const char* idx_A,
                        double* result, orc_len* idx)
{
    orc_len l[ORC_MAX_DIM+1]; orc_stride s[ORC_MAX_DIM+1]; char ii[ORC_MAX_DIM+1];
    unsigned n = orc_diagonal(ndim_A, len_A, stride_A, idx_A, l, s, ii);
    if (n == 0) { l[0] = 1; s[0] = 0; ii[0] = 0; n = 1; }
    orc_stride* sv[1] = { s };
    n = orc_fold(n, l, ii, 1, sv);

    if (alpha < 0.0) { if (op == 4) op = 2; else if (op == 2) op = 4; }

    double val;
    orc_len id = -1;
    switch (op)
    {
        case 2: val = -DBL_MAX; break;
        case 4: case 5: val = DBL_MAX; break;
        default: val = 0.0;
    }
    it3 it; it3_init(&it, n, l, s, NULL, NULL);
    while (it3_next(&it))
    {
        double a = A[it.off[0]];
        switch (op)
        {
            case 0: val += a; break;
            case 1: val += fabs(a); break;
            case 2: if (a > val) { val = a; id = it.off[0]; } break;
            case 3: if (fabs(a) > val) { val = fabs(a); id = it.off[0]; } break;
            case 4: if (a < val) { val = a; id = it.off[0]; } break;
            case 5: if (fabs(a) < val) { val = fabs(a); id = it.off[0]; } break;
            case 6: val += a*a; break;
            default: return -3;
        }
    }
    if (op == 6) val = sqrt(val);
    if (op == 0) val *= alpha;
    else if (op == 1 || op == 6) val *= fabs(alpha);
    *result = val;
    *idx = id;
    return 0;
}

int orc_tensor_scale_d(double alpha, unsigned ndim, const orc_len* len, const orc_stride* stride, double* A)
{
    it3 it; it3_init(&it, ndim, len, stride, NULL, NULL);
    if (alpha == 0.0) { while (it3_next(&it)) A[it.off[0]] = 0.0; return 0; }
    while (it3_next(&it)) A[it.off[0]] *= alpha;
    return 0;
}

int orc_tensor_set_d(double alpha, unsigned ndim, const orc_len* len, const orc_stride* stride, double* A)
{
    it3 it; it3_init(&it, ndim, len, stride, NULL, NULL);
    while (it3_next(&it)) A[it.off[0]] = alpha;
    return 0;
}

/* src/iface/1t/shift.cxx:14-75, src/kernels/1v/shift.hpp:17-40:
 * A = shift + alpha*A (alpha==0 sets zero) */
int orc_tensor_shift_d(double shift, double alpha, unsigned ndim, const orc_len* len,
                       const orc_stride* stride, double* A)
{
    it3 it; it3_init(&it, ndim, len, stride, NULL, NULL);
    if (alpha == 0.0) { while (it3_next(&it)) A[it.off[0]] = 0.0; return 0; }
    if (shift == 0.0) { if (alpha != 1.0) while (it3_next(&it)) A[it.off[0]] *= alpha; return 0; }
    while (it3_next(&it)) A[it.off[0]] = shift + alpha*A[it.off[0]];
    return 0;
}

/* ------------------------------------------------------------------------- */
/* DPD layout (src/external/marray/include/dpd_marray_base.hpp:34-228)       */
/* ------------------------------------------------------------------------- */

#define ORC_DPD_MAXN (2*ORC_MAX_DIM)

typedef struct orc_dpd
{
    unsigned ndim, nirrep, irrep;
    orc_len len[ORC_MAX_DIM][8];
    orc_len size[ORC_DPD_MAXN][8];
    unsigned leaf[ORC_MAX_DIM], parent[ORC_DPD_MAXN], perm[ORC_MAX_DIM];
} orc_dpd;

/* default_depth, :34-67 */
static void dpd_depth(int layout, unsigned ndim, unsigned* depth)
{
    if (layout == 0 || layout == 1)
    {
        unsigned dl = 31 - __builtin_clz(ndim);
        unsigned du = dl + ((ndim & (ndim - 1)) ? 1 : 0);
        unsigned o = ndim - (1u << dl), k = 2*((o + 1)/2), l = 2*(o/2), h = (ndim + 1)/2;
        for (unsigned i = 0; i < ndim; i++)
            depth[i] = i < k ? du : i < h ? dl : i < h + l ? du : dl;
    }
    else if (layout == 4 || layout == 5)
    {
        depth[0] = ndim - 1;
        for (unsigned i = 1; i < ndim; i++) depth[i] = ndim - i;
    }
    else
    {
        for (unsigned i = 0; i + 1 < ndim; i++) depth[i] = i + 1;
        depth[ndim - 1] = ndim - 1;
    }
}

/* set_tree :69-119 and set_size :121-169 */
static int dpd_init(orc_dpd* t, unsigned irrep, unsigned nirrep, unsigned ndim, const orc_len* lens, int layout)
{
    if (ndim == 0 || ndim > ORC_MAX_DIM || nirrep > 8) return -1;
    memset(t, 0, sizeof(*t));
    t->ndim = ndim; t->nirrep = nirrep; t->irrep = irrep;
    for (unsigned i = 0; i < ndim; i++)
        for (unsigned j = 0; j < nirrep; j++) t->len[i][j] = lens[i*nirrep + j];

    unsigned depth[ORC_MAX_DIM], node[ORC_MAX_DIM];
    long leaf_idx[ORC_MAX_DIM];
    unsigned n = ndim;
    dpd_depth(layout, ndim, depth);
    for (unsigned i = 0; i < ndim; i++) leaf_idx[i] = i;
    unsigned pos = 0;
    for (unsigned d = ndim; d-- > 0;)
    {
        for (unsigned i = 0; i < n; i++)
        {
            if (depth[i] == d + 1)
            {
                if (i + 1 >= n || depth[i + 1] != d + 1) return -2;
                t->parent[node[i]] = t->parent[node[i + 1]] = pos;
                for (unsigned j = i + 1; j + 1 < n; j++)
                {
                    depth[j] = depth[j + 1]; node[j] = node[j + 1]; leaf_idx[j] = leaf_idx[j + 1];
                }
                n--;
                depth[i]--;
                node[i] = pos++;
                leaf_idx[i] = -1;
            }
            else if (depth[i] == d)
            {
                node[i] = pos++;
                if (leaf_idx[i] != -1) t->leaf[leaf_idx[i]] = node[i];
            }
        }
    }
    if (pos != 2*ndim - 1) return -3;

    int colmajor = layout == 0 || layout == 2 || layout == 4;
    for (unsigned i = 0; i < ndim; i++)
    {
        unsigned target = colmajor ? t->leaf[i] : t->leaf[ndim - 1 - i];
        for (unsigned j = 0; j < nirrep; j++) t->size[target][j] = t->len[i][j];
        t->perm[i] = colmajor ? i : ndim - 1 - i;
    }
    for (unsigned i = 0; i + 1 < ndim; i++)
    {
        unsigned next = t->parent[2*i];
        for (unsigned a = 0; a < nirrep; a++)
        {
            orc_len s = 0;
            for (unsigned b = 0; b < nirrep; b++) s += t->size[2*i][a ^ b]*t->size[2*i + 1][b];
            t->size[next][a] = s;
        }
    }
    return 0;
}

/* get_block :171-228 (unsliced tensor: off = 0, leap = 1) */
int orc_dpd_block(unsigned irrep, unsigned nirrep, unsigned ndim, const orc_len* lens, int layout,
                  const unsigned* irreps, orc_len* blen, orc_stride* bstride, orc_stride* offset)
{
    orc_dpd t;
    int rc = dpd_init(&t, irrep, nirrep, ndim, lens, layout);
    if (rc) return rc;
    unsigned dirrep[ORC_DPD_MAXN] = {0};
    orc_stride dstride[ORC_DPD_MAXN] = {0};
    dstride[2*ndim - 2] = 1;
    for (unsigned i = 0; i < ndim; i++) dirrep[t.leaf[t.perm[i]]] = irreps[i];
    for (unsigned i = 0; i + 1 < ndim; i++) dirrep[t.parent[2*i]] = dirrep[2*i] ^ dirrep[2*i + 1];
    orc_stride off = 0;
    for (unsigned i = ndim - 1; i-- > 0;)
    {
        unsigned irr = dirrep[t.parent[2*i]];
        dstride[2*i] = dstride[t.parent[2*i]];
        dstride[2*i + 1] = dstride[2*i]*t.size[2*i][dirrep[2*i]];
        orc_stride o = 0;
        for (unsigned a = 0; a < dirrep[2*i + 1]; a++) o += t.size[2*i][a ^ irr]*t.size[2*i + 1][a];
        off += o*dstride[2*i];
    }
    for (unsigned i = 0; i < ndim; i++)
    {
        bstride[i] = dstride[t.leaf[t.perm[i]]];
        blen[i] = t.len[i][irreps[i]];
    }
    *offset = off;
    return 0;
}

orc_len orc_dpd_size(unsigned irrep, unsigned nirrep, unsigned ndim, const orc_len* lens, int layout)
{
    orc_dpd t;
    if (dpd_init(&t, irrep, nirrep, ndim, lens, layout)) return -1;
    return t.size[2*ndim - 2][irrep];
}
