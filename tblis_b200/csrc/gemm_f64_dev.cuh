// gemm_f64_dev.cuh -- device building blocks shared by the FP64 DMMA
// kernels: cp.async gathers, the m16n8k8 FP64 MMA, the shared-memory layouts
// of an operand tile and the per-16-block k offsets of a scatter vector.
#pragma once

#include "common.hpp"

namespace tb
{
namespace f64dev
{

constexpr int BK = 16;
constexpr int PAD = 4;                         // doubles of padding per smem row

__device__ __forceinline__ void cp_async8(double* smem, const double* gmem, bool valid)
{
    unsigned saddr = (unsigned)__cvta_generic_to_shared(smem);
    int src_size = valid ? 8 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n"
                 :: "r"(saddr), "l"(gmem), "r"(src_size));
}

__device__ __forceinline__ void cp_async16(double* smem, const double* gmem)
{
    unsigned saddr = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" :: "r"(saddr), "l"(gmem));
}

// two adjacent tile elements (smem 16-byte aligned): one 16-byte copy when both
// are valid and adjacent, 16-byte aligned, in global memory; else two 8-byte
// copies (zero-filled where not valid)
__device__ __forceinline__ void cp_pair(double* smem, const double* X, i64 off0, bool ok0, i64 off1, bool ok1,
                                        const double* dummy)
{
    if (ok0 && ok1 && off1 == off0 + 1 && (((uintptr_t)(X + off0)) & 15) == 0)
    {
        cp_async16(smem, X + off0);
        return;
    }
    cp_async8(smem, ok0 ? X + off0 : dummy, ok0);
    cp_async8(smem + 1, ok1 ? X + off1 : dummy, ok1);
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }

template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" :: "n"(N)); }

// D(16x8) += A(16x8) * B(8x8), FP64. Fragments (g = lane/4, t = lane%4):
// a[q] = A(g + 8*(q%2), t + 4*(q/2)), b[q] = B(t + 4*q, g),
// c[q] = C(g + 8*(q/2), 2*t + q%2)
__device__ __forceinline__ void dmma16(double* c, const double* a, const double* b)
{
    asm volatile("mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                 "{%0,%1,%2,%3};\n"
                 : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
                 : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

// shared-memory geometry of one operand tile (ROWS = BM or BN)
template <int ROWS, int MODE>
struct Tile
{
    // MODE 0: [BK][ROWS+PAD] (rows contiguous); MODE 1: [ROWS][BK+PAD] (k contiguous)
    static constexpr int SIZE = MODE == 0 ? BK*(ROWS + PAD) : ROWS*(BK + PAD);
    __device__ static __forceinline__ int idx(int r, int k)
    {
        return MODE == 0 ? k*(ROWS + PAD) + r : r*(BK + PAD) + k;
    }
};

// k-offset information of one BK block of one operand
struct KInfo
{
    i64 first;     // offset of the block's first k
    i64 stride;    // common stride inside the block, 0 if irregular
};

__device__ __forceinline__ KInfo fetch_kinfo(const i64* __restrict__ scat, const i64* __restrict__ bstr,
                                             i64 k0, bool valid)
{
    KInfo r = {0, 1};
    if (valid)
    {
        r.first = __ldg(scat + k0);
        r.stride = __ldg(bstr + k0/BK);
    }
    return r;
}

__device__ __forceinline__ i64 koff(const i64* __restrict__ scat, const KInfo& ki, i64 k0, int kl)
{
    return ki.stride != 0 ? ki.first + (i64)kl*ki.stride : __ldg(scat + k0 + kl);
}

} // namespace f64dev
} // namespace tb
