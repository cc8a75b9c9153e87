// dropin_cxx.cxx -- a C++ program written against TBLIS's own header
// (src/tblis.h) and its inline templates over MArray views
// (tblis::mult/add/dot/reduce/scale, src/iface/3t/mult.h:28-38,
// src/iface/1t/{add,dot,reduce,scale}.h), linked against libtblis_b200.so
// alone: it shows that a TBLIS C++ caller of those templates re-links
// unchanged. Inputs and results go to the file named by argv[1] for the test
// to check against the oracle. Exit status 0 on success.
#include <cstddef>
#include <cstdio>
#include <vector>

#include "tblis.h"

#include "abi_layout.h"
#include "dropin_io.h"

static_assert(sizeof(tblis::tblis_scalar) == ABI_SCALAR_SIZE, "tblis_scalar size");
static_assert(sizeof(tblis::tblis_tensor) == ABI_TENSOR_SIZE, "tblis_tensor size");
static_assert(offsetof(tblis::tblis_tensor, data) == ABI_TENSOR_OFF_DATA, "tblis_tensor.data");
static_assert(offsetof(tblis::tblis_tensor, len) == ABI_TENSOR_OFF_LEN, "tblis_tensor.len");
static_assert(offsetof(tblis::tblis_tensor, stride) == ABI_TENSOR_OFF_STRIDE, "tblis_tensor.stride");

// elements of a dense varray
template <typename V> long count(const V& x)
{
    long n = 1;
    for (auto l : x.lengths()) n *= (long)l;
    return n;
}

int main(int argc, char** argv)
{
    if (argc < 2) return 2;
    FILE* f = std::fopen(argv[1], "wb");
    if (!f) return 3;

    // MArray's default layout is row-major (utility.hpp:67-68)
    MArray::varray<double> A({6, 7, 5, 4}), B({7, 4, 5, 3}), C({6, 5, 5, 3});
    dropin_fill(A.data(), count(A), 21);
    dropin_fill(B.data(), count(B), 22);
    dropin_fill(C.data(), count(C), 23);
    dropin_record(f, "A", A.data(), count(A));
    dropin_record(f, "B", B.data(), count(B));
    dropin_record(f, "C0", C.data(), count(C));

    // C[abij] = 0.75*A[aebf]*B[efij] - 0.5*C[abij]
    tblis::mult<double>(0.75, A, "aebf", B, "efij", -0.5, C, "abij");
    dropin_record(f, "C", C.data(), count(C));

    // D[jiba] = 2*C[abij]
    MArray::varray<double> D({3, 5, 5, 6});
    tblis::add<double>(2.0, C, "abij", 0.0, D, "jiba");
    dropin_record(f, "D", D.data(), count(D));

    // a view of C with a permuted dimension order (strides, not a copy)
    MArray::varray_view<double> Cv = C.view();
    Cv.permute({3, 1, 0, 2});
    double dot = tblis::dot<double>(Cv, "jbai", C, "abij");
    dropin_record(f, "dot", &dot, 1);
    auto mx = tblis::reduce<double>(tblis::REDUCE_MAX, C, "abij");
    double mxv[2] = {mx.first, (double)mx.second};
    dropin_record(f, "max", mxv, 2);

    tblis::scale<double>(3.0, C, "abij");
    dropin_record(f, "Cscaled", C.data(), count(C));

    std::fclose(f);
    return 0;
}
