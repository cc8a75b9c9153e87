// level1.hpp -- strided level-1 tensor kernels: set, scale, shift, add
// (permute / trace / replicate), dot and reduce. See level1.cu.
#pragma once

#include "common.hpp"
#include "cplx.hpp"

namespace tb
{

constexpr int L1_MAX_DIM = 12;

// a strided iteration space: dims[0] is the inner (fastest) dimension
struct Strided
{
    int ndim = 0;
    i64 len[L1_MAX_DIM];
    i64 stride[L1_MAX_DIM];
};

// iteration space shared by two operands (same lengths, two stride sets)
struct Strided2
{
    int ndim = 0;
    i64 len[L1_MAX_DIM];
    i64 sa[L1_MAX_DIM];
    i64 sb[L1_MAX_DIM];
};

// T: float, double, cplx<float>, cplx<double>; conj flags act on complex
// elements only (A <- alpha*conj(A) for scale, shift + alpha*conj(A) for shift)
template <typename T> void l1_set(T* A, const Strided& s, T value, cudaStream_t st);
template <typename T> void l1_scale(T* A, const Strided& s, T alpha, cudaStream_t st, bool conj = false);
template <typename T> void l1_shift(T* A, const Strided& s, T shift, T alpha, cudaStream_t st, bool conj = false);

// B[ab, bo] = alpha * op(sum_ao A[ab, ao]) + beta * op(B[ab, bo])  (beta == 0:
// no read; op conjugates when the operand's flag is set)
template <typename T>
void l1_add(const T* A, T* B, const Strided2& ab, const Strided& ao, const Strided& bo,
            T alpha, T beta, cudaStream_t st, bool conj_a = false, bool conj_b = false);

// sum_ab op(A)*op(B) into a device scalar (deterministic two-pass)
template <typename T>
void l1_dot(const T* A, const T* B, const Strided2& ab, T* d_result, cudaStream_t st, bool conj_a = false,
            bool conj_b = false);

// dst[o] = (D)src[o] for every offset o of the strided space (widening and
// rounding copies between float and double storage of the same layout)
template <typename S, typename D>
void l1_convert(const S* src, D* dst, const Strided& s, cudaStream_t st);

// reduction of A with op (reduce_t); writes value and offset to device memory
template <typename T>
void l1_reduce(int op, const T* A, const Strided& s, T* d_value, i64* d_idx, cudaStream_t st);

} // namespace tb
