/* dropin_c.c -- a C program written against TBLIS's own header (src/tblis.h
 * of the TBLIS tree, with its MArray and TCI headers) and linked against
 * libtblis_b200.so alone: it shows that a TBLIS C caller re-links unchanged.
 * It calls tblis_init_tensor[_scaled]_d, tblis_get_config, tblis_tensor_mult
 * (default and an Ozaki config), tblis_tensor_add (a transpose),
 * tblis_tensor_dot, tblis_tensor_reduce and tblis_tensor_scale on host
 * buffers, and writes inputs and results to the file named by argv[1] for
 * the test to check against the oracle. Exit status 0 on success. */
#include <stddef.h>
#include <stdio.h>
#include <stdlib.h>

#include "tblis.h"

#include "abi_layout.h"
#include "dropin_io.h"

ABI_CHECK_LAYOUT(tblis_scalar, tblis_tensor);

int main(int argc, char** argv)
{
    if (argc < 2) return 2;
    FILE* f = fopen(argv[1], "wb");
    if (!f) return 3;

    /* A[abef] with a padded, permuted layout; B[efij] and C[abij] column-major */
    len_type lenA[4] = {7, 6, 5, 4}, lenB[4] = {5, 4, 3, 6}, lenC[4] = {7, 6, 3, 6};
    stride_type strA[4] = {6*21, 21, 4, 1}, strB[4] = {1, 5, 20, 60}, strC[4] = {1, 7, 42, 126};
    const long nA = 7*6*21, nB = 5*4*3*6, nC = 7*6*3*6;
    double *a = malloc(nA*sizeof(double)), *b = malloc(nB*sizeof(double));
    double *c = malloc(nC*sizeof(double)), *c2 = malloc(nC*sizeof(double)), *d = malloc(nC*sizeof(double));
    dropin_fill(a, nA, 11);
    dropin_fill(b, nB, 12);
    dropin_fill(c, nC, 13);
    for (long i = 0; i < nC; i++) c2[i] = c[i];
    dropin_record(f, "A", a, nA);
    dropin_record(f, "B", b, nB);
    dropin_record(f, "C0", c, nC);

    tblis_tensor A, B, C, C2, D;
    tblis_init_tensor_scaled_d(&A, 0.5, 4, lenA, a, strA);
    tblis_init_tensor_d(&B, 4, lenB, b, strB);
    tblis_init_tensor_scaled_d(&C, 2.0, 4, lenC, c, strC);
    /* C = 0.5*A*B + 2*C through the default configuration */
    tblis_tensor_mult(NULL, NULL, &A, "abef", &B, "efij", &C, "abij");
    double scal[2] = {C.scalar.data.d, (double)C.conj};
    dropin_record(f, "C", c, nC);
    dropin_record(f, "Cscalar", scal, 2);

    /* the same through a named configuration (Ozaki INT8, 1e-12) */
    const tblis_config* cfg = tblis_get_config("b200_ozaki_i8");
    tblis_init_tensor_scaled_d(&A, 0.5, 4, lenA, a, strA);
    tblis_init_tensor_scaled_d(&C2, 2.0, 4, lenC, c2, strC);
    tblis_tensor_mult(NULL, cfg, &A, "abef", &B, "efij", &C2, "abij");
    double has_cfg = cfg != NULL;
    dropin_record(f, "C_ozaki", c2, nC);
    dropin_record(f, "has_cfg", &has_cfg, 1);

    /* D[ijab] = 1.5*C[abij] (beta 0: D is not read) */
    len_type lenD[4] = {3, 6, 7, 6};
    stride_type strD[4] = {1, 3, 18, 126};
    for (long i = 0; i < nC; i++) d[i] = 1e300;
    tblis_init_tensor_scaled_d(&C, 1.5, 4, lenC, c, strC);
    tblis_init_tensor_scaled_d(&D, 0.0, 4, lenD, d, strD);
    tblis_tensor_add(NULL, NULL, &C, "abij", &D, "ijab");
    dropin_record(f, "D", d, nC);

    /* dot of A with itself, NORM_2 and MAX_ABS of C */
    tblis_init_tensor_d(&A, 4, lenA, a, strA);
    tblis_scalar r;
    tblis_init_scalar_d(&r, 0.0);
    tblis_tensor_dot(NULL, NULL, &A, "abef", &A, "abef", &r);
    double dot = r.data.d;
    dropin_record(f, "dot", &dot, 1);
    tblis_init_tensor_d(&C, 4, lenC, c, strC);
    len_type idx = -1;
    tblis_tensor_reduce(NULL, NULL, REDUCE_NORM_2, &C, "abij", &r, &idx);
    double nrm = r.data.d;
    dropin_record(f, "norm2", &nrm, 1);
    tblis_tensor_reduce(NULL, NULL, REDUCE_MAX_ABS, &C, "abij", &r, &idx);
    double mx[2] = {r.data.d, (double)idx};
    dropin_record(f, "maxabs", mx, 2);

    /* C *= -0.25 */
    tblis_init_tensor_scaled_d(&C, -0.25, 4, lenC, c, strC);
    tblis_tensor_scale(NULL, NULL, &C, "abij");
    dropin_record(f, "Cscaled", c, nC);

    fclose(f);
    free(a); free(b); free(c); free(c2); free(d);
    return 0;
}
