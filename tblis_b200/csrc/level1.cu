// level1.cu -- strided level-1 tensor kernels.
//
// GPU counterparts of TBLIS's level-1 tensor operations
// (src/internal/1t/dense/{add,dot,reduce,scale,set,shift}.cxx and their
// microkernels src/kernels/1v/*.hpp, src/kernels/1m/trans.hpp). The host folds
// each operand's dims first (the reference's fold), so most tensors arrive as
// one or two long dims; the kernels then walk "segments" (a run of the inner
// dimension of one outer row) with a warp per segment, 128-bit vector
// accesses where the inner dim is unit-stride and 16-byte aligned, and
// shared-memory tiles for transposes (the inner dims of A and B differ).
// Reductions are two-pass and deterministic (fixed grid, fixed combine
// order, no atomics). The element type is float, double or their complex
// counterparts (cplx.hpp); conj flags apply to complex operands as the
// reference's microkernels apply them (src/kernels/1v/{add,scale,shift,dot}.hpp).
#include "level1.hpp"
#include "cplx.hpp"
#include "mult.hpp"

#include <algorithm>
#include <cfloat>
#include <cmath>

namespace tb
{

namespace
{

constexpr int SEG = 1024;          // inner elements per segment
constexpr int L1_THREADS = 256;
constexpr int RED_BLOCKS = 148*4;  // fixed grid of the reductions

template <typename T>
__device__ __forceinline__ T shfl_down(T v, int o) { return __shfl_down_sync(0xffffffffu, v, o); }
template <typename R>
__device__ __forceinline__ cplx<R> shfl_down(cplx<R> v, int o)
{
    return {__shfl_down_sync(0xffffffffu, v.re, o), __shfl_down_sync(0xffffffffu, v.im, o)};
}

int l1_grid(i64 work_items, int per_block)
{
    i64 b = (work_items + per_block - 1)/per_block;
    return (int)std::max<i64>(1, std::min<i64>(b, 148*32));
}

// one full wave of a grid-stride kernel: every SM holds as many blocks as
// fit, and no partial last wave leaves SMs idle at the end
template <typename K>
int resident_grid(K kernel, i64 work_items, int threads)
{
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0) != cudaSuccess || per_sm < 1)
    {
        cudaGetLastError();
        per_sm = 1;
    }
    return (int)std::max<i64>(1, std::min<i64>(work_items, (i64)per_sm*device_sm_count()));
}

__device__ __forceinline__ i64 row_offset(const i64* len, const i64* stride, int ndim, i64 r)
{
    i64 off = 0;
    for (int d = 1; d < ndim; d++)
    {
        i64 q = r / len[d];
        off += (r - q*len[d])*stride[d];
        r = q;
    }
    return off;
}

__device__ __forceinline__ void row_offset2(const Strided2& s, i64 r, i64& oa, i64& ob)
{
    oa = 0; ob = 0;
    for (int d = 1; d < s.ndim; d++)
    {
        i64 q = r / s.len[d];
        i64 i = r - q*s.len[d];
        oa += i*s.sa[d];
        ob += i*s.sb[d];
        r = q;
    }
}

// ---- set / scale / shift ------------------------------------------------------

// op: 0 = set(value), 1 = scale(alpha), 2 = shift: shift + alpha*A
// (A conjugated first when conj)
template <typename T, int OP>
__global__ void __launch_bounds__(L1_THREADS) k_unary(T* A, const Strided s, T v0, T v1, bool conj)
{
    const i64 n0 = s.ndim ? s.len[0] : 1;
    const i64 st0 = s.ndim ? s.stride[0] : 0;
    i64 rows = 1;
    for (int d = 1; d < s.ndim; d++) rows *= s.len[d];
    const i64 nchunk = (n0 + SEG - 1)/SEG;
    const i64 nseg = rows*nchunk;
    const int lane = threadIdx.x & 31;
    const i64 warp0 = (blockIdx.x*(i64)blockDim.x + threadIdx.x) >> 5;
    const i64 nwarps = ((i64)gridDim.x*blockDim.x) >> 5;
    for (i64 sg = warp0; sg < nseg; sg += nwarps)
    {
        const i64 r = rows == 1 ? 0 : sg / nchunk, c = sg - r*nchunk;   // one row: no division
        T* base = A + row_offset(s.len, s.stride, s.ndim, r);
        const i64 i0 = c*SEG, i1 = min(n0, i0 + SEG);
        for (i64 i = i0 + lane; i < i1; i += 32)
        {
            T* p = base + i*st0;
            if (OP == 0) *p = v0;
            else if (OP == 1) *p = v0*cj(*p, conj);
            else *p = v0 + v1*cj(*p, conj);
        }
    }
}

// ---- element-type conversion at equal offsets -------------------------------------

template <typename S, typename D>
__global__ void __launch_bounds__(L1_THREADS) k_convert(const S* __restrict__ src, D* __restrict__ dst, const Strided s)
{
    const i64 n0 = s.ndim ? s.len[0] : 1;
    const i64 st0 = s.ndim ? s.stride[0] : 0;
    i64 rows = 1;
    for (int d = 1; d < s.ndim; d++) rows *= s.len[d];
    const i64 nchunk = (n0 + SEG - 1)/SEG;
    const i64 nseg = rows*nchunk;
    const int lane = threadIdx.x & 31;
    const i64 warp0 = (blockIdx.x*(i64)blockDim.x + threadIdx.x) >> 5;
    const i64 nwarps = ((i64)gridDim.x*blockDim.x) >> 5;
    for (i64 sg = warp0; sg < nseg; sg += nwarps)
    {
        const i64 r = rows == 1 ? 0 : sg / nchunk, c = sg - r*nchunk;   // one row: no division
        const i64 ro = row_offset(s.len, s.stride, s.ndim, r);
        const i64 i0 = c*SEG, i1 = min(n0, i0 + SEG);
        for (i64 i = i0 + lane; i < i1; i += 32) dst[ro + i*st0] = (D)src[ro + i*st0];
    }
}

// ---- add: permute / trace / replicate ------------------------------------------

template <typename T, bool BETA0>
__global__ void __launch_bounds__(L1_THREADS)
k_add_general(const T* __restrict__ A, T* __restrict__ B, const Strided2 ab, const Strided ao,
              const Strided bo, T alpha, T beta, bool conj_a, bool conj_b)
{
    const i64 n0 = ab.len[0];
    i64 rows = 1;
    for (int d = 1; d < ab.ndim; d++) rows *= ab.len[d];
    i64 nao = 1, nbo = 1;
    for (int d = 0; d < ao.ndim; d++) nao *= ao.len[d];
    for (int d = 0; d < bo.ndim; d++) nbo *= bo.len[d];
    const i64 total = rows*n0;
    for (i64 e = blockIdx.x*(i64)blockDim.x + threadIdx.x; e < total; e += (i64)gridDim.x*blockDim.x)
    {
        const i64 r = e / n0, i = e - r*n0;
        i64 oa, ob;
        row_offset2(ab, r, oa, ob);
        oa += i*ab.sa[0];
        ob += i*ab.sb[0];
        T sum = T(0);
        for (i64 t = 0; t < nao; t++)
        {
            i64 x = t, o = 0;
            for (int d = 0; d < ao.ndim; d++) { i64 q = x/ao.len[d]; o += (x - q*ao.len[d])*ao.stride[d]; x = q; }
            sum += A[oa + o];
        }
        const T v = alpha*cj(sum, conj_a);
        for (i64 t = 0; t < nbo; t++)
        {
            i64 x = t, o = 0;
            for (int d = 0; d < bo.ndim; d++) { i64 q = x/bo.len[d]; o += (x - q*bo.len[d])*bo.stride[d]; x = q; }
            T* p = B + ob + o;
            *p = BETA0 ? v : v + beta*cj(*p, conj_b);
        }
    }
}

// same unit-stride dimension in A and B: warp per segment of the inner dim,
// 16-byte vectors when both inner strides are 1 and the rows are aligned
template <typename T, bool BETA0>
__global__ void __launch_bounds__(L1_THREADS)
k_add_rows(const T* __restrict__ A, T* __restrict__ B, const Strided2 s, T alpha, T beta, bool conj_a,
           bool conj_b)
{
    const i64 n0 = s.len[0];
    i64 rows = 1;
    for (int d = 1; d < s.ndim; d++) rows *= s.len[d];
    const i64 nchunk = (n0 + SEG - 1)/SEG;
    const i64 nseg = rows*nchunk;
    const int lane = threadIdx.x & 31;
    const i64 warp0 = (blockIdx.x*(i64)blockDim.x + threadIdx.x) >> 5;
    const i64 nwarps = ((i64)gridDim.x*blockDim.x) >> 5;
    const bool unit = s.sa[0] == 1 && s.sb[0] == 1;
    constexpr int VW = 16/sizeof(T);
    for (i64 sg = warp0; sg < nseg; sg += nwarps)
    {
        const i64 r = rows == 1 ? 0 : sg / nchunk, c = sg - r*nchunk;   // one row: no division
        i64 oa, ob;
        row_offset2(s, r, oa, ob);
        const i64 i0 = c*SEG, i1 = min(n0, i0 + SEG);
        const T* a = A + oa;
        T* b = B + ob;
        const bool vec = unit && ((((uintptr_t)(a + i0)) | ((uintptr_t)(b + i0))) & 15) == 0;
        if (vec)
        {
            const i64 nv = (i1 - i0)/VW;
            typedef typename std::conditional<sizeof(T) == 8, double2, float4>::type V;
            const V* av = reinterpret_cast<const V*>(a + i0);
            V* bv = reinterpret_cast<V*>(b + i0);
            for (i64 v = lane; v < nv; v += 32)
            {
                V x = av[v];
                T* xs = reinterpret_cast<T*>(&x);
                V y;
                T* ys = reinterpret_cast<T*>(&y);
                if (!BETA0) y = bv[v];
                #pragma unroll
                for (int q = 0; q < VW; q++)
                    ys[q] = BETA0 ? alpha*cj(xs[q], conj_a) : alpha*cj(xs[q], conj_a) + beta*cj(ys[q], conj_b);
                bv[v] = y;
            }
            for (i64 i = i0 + nv*VW + lane; i < i1; i += 32)
                b[i] = BETA0 ? alpha*cj(a[i], conj_a) : alpha*cj(a[i], conj_a) + beta*cj(b[i], conj_b);
        }
        else
        {
            for (i64 i = i0 + lane; i < i1; i += 32)
            {
                const T x = cj(a[i*s.sa[0]], conj_a);
                T* p = b + i*s.sb[0];
                *p = BETA0 ? alpha*x : alpha*x + beta*cj(*p, conj_b);
            }
        }
    }
}

// transpose: dim p is A's unit dim, dim q is B's unit dim, the rest are outer.
// Square tile through shared memory (64 wide, 32 for 16-byte elements so the
// tile stays below 48 KB); reads coalesced along p, writes along q. VW = 2
// moves pairs of elements (16 bytes for 8-byte types) on both sides when the
// host has checked that both unit strides are 1, both extents and every other
// stride are even and both bases are aligned to a pair, so every pair is
// contiguous and aligned.
template <typename T>
constexpr int tile_of() { return sizeof(T) >= 16 ? 32 : 64; }

template <int BYTES> struct RawVec;
template <> struct RawVec<8> { typedef uint2 type; };
template <> struct RawVec<16> { typedef uint4 type; };

template <typename T, bool BETA0, int VW>
__global__ void __launch_bounds__(L1_THREADS, 3)
k_transpose(const T* __restrict__ A, T* __restrict__ B, const Strided2 s, int p, int q,
            i64 tiles_p, i64 tiles_q, i64 outer, T alpha, T beta, bool conj_a, bool conj_b)
{
    constexpr int TT = tile_of<T>();
    typedef typename RawVec<(VW == 1 || sizeof(T)*VW < 8) ? 8 : sizeof(T)*VW>::type Raw;
    static_assert(VW == 1 || sizeof(Raw) == sizeof(T)*VW, "pair width");
    __shared__ T tile[TT][TT + 1];
    const i64 np = s.len[p], nq = s.len[q];
    // tile indices in 32 bits (the host checks the tile count), so each tile
    // costs a few 32-bit divisions instead of 64-bit ones
    const unsigned ntiles = (unsigned)(tiles_p*tiles_q*outer);
    const unsigned tpn = (unsigned)tiles_p, tpq = (unsigned)(tiles_p*tiles_q);
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;   // 32 x 8
    for (unsigned t = blockIdx.x; t < ntiles; t += gridDim.x)
    {
        unsigned o = t / tpq;
        const unsigned pq = t - o*tpq;
        const unsigned tq = pq / tpn, tp = pq - tq*tpn;
        // outer offsets: decompose o over dims other than p and q
        i64 oa = 0, ob = 0;
        for (int d = 0; d < s.ndim; d++)
        {
            if (d == p || d == q) continue;
            const unsigned ld = (unsigned)s.len[d];
            const unsigned qq = o / ld;
            const unsigned i = o - qq*ld;
            oa += (i64)i*s.sa[d]; ob += (i64)i*s.sb[d];
            o = qq;
        }
        const i64 p0 = (i64)tp*TT, q0 = (i64)tq*TT;
        // load: lanes along p (A contiguous), VW consecutive p per lane. All
        // of a thread's loads are issued into registers before the first
        // shared-memory store, so they are in flight together.
        constexpr int NJ = TT/8, NH = TT/(32*VW);
        typedef typename std::conditional<VW == 1, T, Raw>::type Item;
        Item in[NJ][NH];
        #pragma unroll
        for (int j = 0; j < NJ; j++)
        {
            #pragma unroll
            for (int h = 0; h < NH; h++)
            {
                const i64 pi = p0 + (tx + 32*h)*VW, qi = q0 + ty + 8*j;
                if (pi < np && qi < nq)
                    in[j][h] = *reinterpret_cast<const Item*>(A + oa + pi*s.sa[p] + qi*s.sa[q]);
            }
        }
        #pragma unroll
        for (int j = 0; j < NJ; j++)
        {
            const int ql = ty + 8*j;
            #pragma unroll
            for (int h = 0; h < NH; h++)
            {
                const int pl = (tx + 32*h)*VW;
                if (p0 + pl < np && q0 + ql < nq)
                {
                    const T* e = reinterpret_cast<const T*>(&in[j][h]);
                    #pragma unroll
                    for (int u = 0; u < VW; u++) tile[ql][pl + u] = e[u];
                }
            }
        }
        __syncthreads();
        // store: lanes along q (B contiguous), VW consecutive q per lane
        #pragma unroll
        for (int j = 0; j < TT/8; j++)
        {
            const int pl = ty + 8*j;
            #pragma unroll
            for (int h = 0; h < TT/(32*VW); h++)
            {
                const int ql = (tx + 32*h)*VW;
                const i64 pi = p0 + pl, qi = q0 + ql;
                if (pi < np && qi < nq)
                {
                    T* dst = B + ob + pi*s.sb[p] + qi*s.sb[q];
                    if (VW == 1)
                    {
                        const T v = alpha*cj(tile[ql][pl], conj_a);
                        *dst = BETA0 ? v : v + beta*cj(*dst, conj_b);
                    }
                    else
                    {
                        Raw r;
                        if (!BETA0) r = *reinterpret_cast<const Raw*>(dst);
                        T* e = reinterpret_cast<T*>(&r);
                        #pragma unroll
                        for (int u = 0; u < VW; u++)
                        {
                            const T v = alpha*cj(tile[ql + u][pl], conj_a);
                            e[u] = BETA0 ? v : v + beta*cj(e[u], conj_b);
                        }
                        *reinterpret_cast<Raw*>(dst) = r;
                    }
                }
            }
        }
        __syncthreads();
    }
}

// ---- dot / reduce -----------------------------------------------------------------

// Loads a lane keeps in flight per inner step of the reductions. The segment
// loops issue U loads before the first add, in the order of the plain loop,
// so the sums are the same bit for bit.
template <typename T> constexpr int red_unroll(int operands) { return sizeof(T) >= 16 ? 4/operands : 8/operands; }

template <typename T>
__global__ void __launch_bounds__(L1_THREADS, RED_BLOCKS/148)
k_dot_partial(const T* __restrict__ A, const T* __restrict__ B, const Strided2 s, T* partial, bool conj_a,
              bool conj_b)
{
    const i64 n0 = s.ndim ? s.len[0] : 1;
    i64 rows = 1;
    for (int d = 1; d < s.ndim; d++) rows *= s.len[d];
    const i64 nchunk = (n0 + SEG - 1)/SEG;
    const i64 nseg = rows*nchunk;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const i64 warp0 = (blockIdx.x*(i64)blockDim.x + threadIdx.x) >> 5;
    const i64 nwarps = ((i64)gridDim.x*blockDim.x) >> 5;
    const i64 sa0 = s.ndim ? s.sa[0] : 0, sb0 = s.ndim ? s.sb[0] : 0;
    T acc = T(0);
    for (i64 sg = warp0; sg < nseg; sg += nwarps)
    {
        const i64 r = rows == 1 ? 0 : sg / nchunk, c = sg - r*nchunk;   // one row: no division
        i64 oa, ob;
        row_offset2(s, r, oa, ob);
        const i64 i0 = c*SEG, i1 = min(n0, i0 + SEG);
        constexpr int U = red_unroll<T>(2);
        i64 i = i0 + lane;
        for (; i + 32*(U - 1) < i1; i += 32*U)
        {
            T x[U], y[U];
#pragma unroll
            for (int u = 0; u < U; u++) { x[u] = A[oa + (i + 32*u)*sa0]; y[u] = B[ob + (i + 32*u)*sb0]; }
#pragma unroll
            for (int u = 0; u < U; u++) acc += cj(x[u], conj_a)*cj(y[u], conj_b);
        }
        for (; i < i1; i += 32) acc += cj(A[oa + i*sa0], conj_a)*cj(B[ob + i*sb0], conj_b);
    }
    for (int o = 16; o > 0; o >>= 1) acc += shfl_down(acc, o);
    __shared__ T ws[L1_THREADS/32];
    if (lane == 0) ws[wib] = acc;
    __syncthreads();
    if (threadIdx.x == 0)
    {
        T t = T(0);
        for (int w = 0; w < L1_THREADS/32; w++) t += ws[w];
        partial[blockIdx.x] = t;
    }
}

template <typename T>
__global__ void k_sum_partials(const T* partial, int n, T* out)
{
    // one warp, fixed order
    const int lane = threadIdx.x;
    T acc = T(0);
    for (int i = lane; i < n; i += 32) acc += partial[i];
    for (int o = 16; o > 0; o >>= 1) acc += shfl_down(acc, o);
    if (lane == 0) *out = acc;
}

// candidate of a MAX/MIN-type reduction: value, linear position, offset
template <typename T>
struct Cand { T v; i64 lin; i64 off; };

template <typename T>
__device__ __forceinline__ bool better(int op, const Cand<T>& a, const Cand<T>& b)
{
    // is a preferred over b? strict comparison; ties go to the earlier
    // position in iteration order (the reference's sequential result)
    if (a.lin < 0) return false;
    if (b.lin < 0) return true;
    // complex values order by their real parts, as the reference's operators do
    const auto ka = order_key(a.v), kb = order_key(b.v);
    bool gt = ka > kb, lt = ka < kb;
    bool maxop = op == REDUCE_MAX || op == REDUCE_MAX_ABS;
    if (maxop ? gt : lt) return true;
    if (ka == kb) return a.lin < b.lin;
    return false;
}

template <typename T>
__device__ __forceinline__ T red_val(int op, T x)
{
    switch (op)
    {
        case REDUCE_SUM_ABS: case REDUCE_MAX_ABS: case REDUCE_MIN_ABS: return abs_elem(x);
        case REDUCE_NORM_2: return norm2_elem(x);
        default: return x;
    }
}

template <typename T>
__global__ void __launch_bounds__(L1_THREADS, RED_BLOCKS/148)
k_reduce_partial(int op, const T* __restrict__ A, const Strided s, T* pv, i64* plin, i64* poff)
{
    const i64 n0 = s.ndim ? s.len[0] : 1;
    i64 rows = 1;
    for (int d = 1; d < s.ndim; d++) rows *= s.len[d];
    const i64 nchunk = (n0 + SEG - 1)/SEG;
    const i64 nseg = rows*nchunk;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const i64 warp0 = (blockIdx.x*(i64)blockDim.x + threadIdx.x) >> 5;
    const i64 nwarps = ((i64)gridDim.x*blockDim.x) >> 5;
    const i64 st0 = s.ndim ? s.stride[0] : 0;
    const bool is_sum = op == REDUCE_SUM || op == REDUCE_SUM_ABS || op == REDUCE_NORM_2;
    T acc = T(0);
    Cand<T> best = {T(0), -1, -1};
    for (i64 sg = warp0; sg < nseg; sg += nwarps)
    {
        const i64 r = rows == 1 ? 0 : sg / nchunk, c = sg - r*nchunk;   // one row: no division
        const i64 ro = row_offset(s.len, s.stride, s.ndim, r);
        const i64 i0 = c*SEG, i1 = min(n0, i0 + SEG);
        if (is_sum)
        {
            constexpr int U = red_unroll<T>(1);
            i64 i = i0 + lane;
            for (; i + 32*(U - 1) < i1; i += 32*U)
            {
                T x[U];
#pragma unroll
                for (int u = 0; u < U; u++) x[u] = A[ro + (i + 32*u)*st0];
#pragma unroll
                for (int u = 0; u < U; u++) acc += red_val(op, x[u]);
            }
            for (; i < i1; i += 32) acc += red_val(op, A[ro + i*st0]);
            continue;
        }
        for (i64 i = i0 + lane; i < i1; i += 32)
        {
            const i64 off = ro + i*st0;
            const T x = red_val(op, A[off]);
            if (is_sum) acc += x;
            else
            {
                Cand<T> cnd = {x, r*n0 + i, off};
                if (better(op, cnd, best)) best = cnd;
            }
        }
    }
    __shared__ T sv[L1_THREADS];
    __shared__ i64 sl[L1_THREADS], so[L1_THREADS];
    if (is_sum)
    {
        for (int o = 16; o > 0; o >>= 1) acc += shfl_down(acc, o);
        if (lane == 0) sv[wib] = acc;
        __syncthreads();
        if (threadIdx.x == 0)
        {
            T t = T(0);
            for (int w = 0; w < L1_THREADS/32; w++) t += sv[w];
            pv[blockIdx.x] = t; plin[blockIdx.x] = -1; poff[blockIdx.x] = -1;
        }
    }
    else
    {
        sv[threadIdx.x] = best.v; sl[threadIdx.x] = best.lin; so[threadIdx.x] = best.off;
        __syncthreads();
        if (threadIdx.x == 0)
        {
            Cand<T> b = {sv[0], sl[0], so[0]};
            for (int t = 1; t < L1_THREADS; t++)
            {
                Cand<T> c = {sv[t], sl[t], so[t]};
                if (better(op, c, b)) b = c;
            }
            pv[blockIdx.x] = b.v; plin[blockIdx.x] = b.lin; poff[blockIdx.x] = b.off;
        }
    }
}

template <typename T>
__global__ void k_reduce_final(int op, const T* pv, const i64* plin, const i64* poff, int n,
                               T* out_v, i64* out_idx)
{
    if (threadIdx.x != 0) return;
    const bool is_sum = op == REDUCE_SUM || op == REDUCE_SUM_ABS || op == REDUCE_NORM_2;
    if (is_sum)
    {
        T t = T(0);
        for (int i = 0; i < n; i++) t += pv[i];
        if (op == REDUCE_NORM_2) t = sqrt_elem(t);
        *out_v = t; *out_idx = -1;
        return;
    }
    Cand<T> b = {pv[0], plin[0], poff[0]};
    for (int i = 1; i < n; i++)
    {
        Cand<T> c = {pv[i], plin[i], poff[i]};
        if (better(op, c, b)) b = c;
    }
    if (b.lin < 0)
    {
        // empty tensor: the reference's initial values
        using R = typename real_of<T>::type;
        const R big = sizeof(R) == 8 ? (R)DBL_MAX : (R)FLT_MAX;
        switch (op)
        {
            case REDUCE_MAX: b.v = T(-big); break;
            case REDUCE_MIN: case REDUCE_MIN_ABS: b.v = T(big); break;
            default: b.v = T(0);
        }
    }
    *out_v = b.v; *out_idx = b.off;
}

} // namespace

// ---- host launchers -------------------------------------------------------------------

static i64 total_of(const Strided& s) { i64 t = 1; for (int d = 0; d < s.ndim; d++) t *= s.len[d]; return t; }
static i64 total_of(const Strided2& s) { i64 t = 1; for (int d = 0; d < s.ndim; d++) t *= s.len[d]; return t; }

template <typename T>
static void unary_launch(int op, T* A, const Strided& s, T v0, T v1, bool conj, cudaStream_t st)
{
    i64 total = total_of(s);
    if (total == 0) return;
    i64 n0 = s.ndim ? s.len[0] : 1;
    i64 segs = (total/n0)*((n0 + SEG - 1)/SEG);
    int grid = l1_grid(segs, L1_THREADS/32);
    if (op == 0) k_unary<T, 0><<<grid, L1_THREADS, 0, st>>>(A, s, v0, v1, conj);
    else if (op == 1) k_unary<T, 1><<<grid, L1_THREADS, 0, st>>>(A, s, v0, v1, conj);
    else k_unary<T, 2><<<grid, L1_THREADS, 0, st>>>(A, s, v0, v1, conj);
    check_launch("k_unary");
}

template <typename T> void l1_set(T* A, const Strided& s, T value, cudaStream_t st) { unary_launch<T>(0, A, s, value, T(0), false, st); }
template <typename T> void l1_scale(T* A, const Strided& s, T alpha, cudaStream_t st, bool conj)
{
    unary_launch<T>(1, A, s, alpha, T(0), conj, st);
}
template <typename T> void l1_shift(T* A, const Strided& s, T shift, T alpha, cudaStream_t st, bool conj)
{
    unary_launch<T>(2, A, s, shift, alpha, conj, st);
}

template <typename S, typename D>
void l1_convert(const S* src, D* dst, const Strided& s, cudaStream_t st)
{
    i64 total = total_of(s);
    if (total == 0) return;
    i64 n0 = s.ndim ? s.len[0] : 1;
    i64 segs = (total/n0)*((n0 + SEG - 1)/SEG);
    int grid = l1_grid(segs, L1_THREADS/32);
    k_convert<S, D><<<grid, L1_THREADS, 0, st>>>(src, dst, s);
    check_launch("k_convert");
}

template void l1_convert<float, double>(const float*, double*, const Strided&, cudaStream_t);
template void l1_convert<double, float>(const double*, float*, const Strided&, cudaStream_t);

template <typename T>
void l1_add(const T* A, T* B, const Strided2& ab, const Strided& ao, const Strided& bo,
            T alpha, T beta, cudaStream_t st, bool conj_a, bool conj_b)
{
    i64 nab = total_of(ab);
    if (nab == 0 || total_of(bo) == 0) return;
    const bool b0 = beta == T(0);

    if (ao.ndim == 0 && bo.ndim == 0 && ab.ndim > 0)
    {
        // find the unit-stride dims of A and B (smallest |stride| otherwise)
        int pa = 0, pb = 0;
        for (int d = 1; d < ab.ndim; d++)
        {
            if (std::llabs(ab.sa[d]) < std::llabs(ab.sa[pa])) pa = d;
            if (std::llabs(ab.sb[d]) < std::llabs(ab.sb[pb])) pb = d;
        }
        if (pa == pb || ab.len[pa] == 1 || ab.len[pb] == 1)
        {
            // rows along the common fastest dim
            Strided2 s = ab;
            std::swap(s.len[0], s.len[pa]); std::swap(s.sa[0], s.sa[pa]); std::swap(s.sb[0], s.sb[pa]);
            i64 n0 = s.len[0];
            i64 segs = (nab/n0)*((n0 + SEG - 1)/SEG);
            int grid = l1_grid(segs, L1_THREADS/32);
            TimedLaunch t("k_add_rows", st);
            if (b0) k_add_rows<T, true><<<grid, L1_THREADS, 0, st>>>(A, B, s, alpha, beta, conj_a, conj_b);
            else k_add_rows<T, false><<<grid, L1_THREADS, 0, st>>>(A, B, s, alpha, beta, conj_a, conj_b);
            check_launch("k_add_rows");
            return;
        }
        constexpr int TT = tile_of<T>();
        i64 tp = (ab.len[pa] + TT - 1)/TT, tq = (ab.len[pb] + TT - 1)/TT;
        i64 outer = nab/(ab.len[pa]*ab.len[pb]);
        i64 ntiles = tp*tq*outer;
        TB_CHECK(ntiles < ((i64)1 << 32), TB_ERR_SIZE, "transpose: too many tiles");
        // pairs: every pair (2i, 2i+1) along p in A and along q in B is
        // contiguous and aligned to twice the element size
        bool pairs = sizeof(T) <= 8 && ab.sa[pa] == 1 && ab.sb[pb] == 1 && ab.len[pa] % 2 == 0 &&
                     ab.len[pb] % 2 == 0 && ((uintptr_t)A % (2*sizeof(T))) == 0 &&
                     ((uintptr_t)B % (2*sizeof(T))) == 0;
        for (int d = 0; d < ab.ndim && pairs; d++)
        {
            if (d != pa && ab.sa[d] % 2 != 0) pairs = false;
            if (d != pb && ab.sb[d] % 2 != 0) pairs = false;
        }
        TimedLaunch t("k_transpose", st);
        if constexpr (sizeof(T) <= 8)
        {
            if (pairs)
            {
                const int grid = resident_grid(k_transpose<T, true, 2>, ntiles, L1_THREADS);
                if (b0) k_transpose<T, true, 2><<<grid, L1_THREADS, 0, st>>>(A, B, ab, pa, pb, tp, tq, outer,
                                                                             alpha, beta, conj_a, conj_b);
                else k_transpose<T, false, 2><<<grid, L1_THREADS, 0, st>>>(A, B, ab, pa, pb, tp, tq, outer,
                                                                            alpha, beta, conj_a, conj_b);
                check_launch("k_transpose");
                return;
            }
        }
        const int grid = resident_grid(k_transpose<T, true, 1>, ntiles, L1_THREADS);
        if (b0) k_transpose<T, true, 1><<<grid, L1_THREADS, 0, st>>>(A, B, ab, pa, pb, tp, tq, outer, alpha, beta,
                                                                     conj_a, conj_b);
        else k_transpose<T, false, 1><<<grid, L1_THREADS, 0, st>>>(A, B, ab, pa, pb, tp, tq, outer, alpha, beta,
                                                                    conj_a, conj_b);
        check_launch("k_transpose");
        return;
    }

    Strided2 s = ab;
    if (s.ndim == 0) { s.ndim = 1; s.len[0] = 1; s.sa[0] = 0; s.sb[0] = 0; }
    int grid = l1_grid(nab, L1_THREADS);
    if (b0) k_add_general<T, true><<<grid, L1_THREADS, 0, st>>>(A, B, s, ao, bo, alpha, beta, conj_a, conj_b);
    else k_add_general<T, false><<<grid, L1_THREADS, 0, st>>>(A, B, s, ao, bo, alpha, beta, conj_a, conj_b);
    check_launch("k_add_general");
}

template <typename T>
void l1_dot(const T* A, const T* B, const Strided2& ab, T* d_result, cudaStream_t st, bool conj_a, bool conj_b)
{
    dbuf part(RED_BLOCKS*sizeof(T), st);
    k_dot_partial<T><<<RED_BLOCKS, L1_THREADS, 0, st>>>(A, B, ab, part.as<T>(), conj_a, conj_b);
    check_launch("k_dot_partial");
    k_sum_partials<T><<<1, 32, 0, st>>>(part.as<T>(), RED_BLOCKS, d_result);
    check_launch("k_sum_partials");
}

template <typename T>
void l1_reduce(int op, const T* A, const Strided& s, T* d_value, i64* d_idx, cudaStream_t st)
{
    TB_CHECK(op >= 0 && op <= 6, TB_ERR_ARG, "unknown reduce op");
    dbuf part(RED_BLOCKS*(sizeof(T) + 2*sizeof(i64)), st);
    T* pv = part.as<T>();
    i64* pl = reinterpret_cast<i64*>(part.as<char>() + RED_BLOCKS*sizeof(T));   // 8-byte aligned
    i64* po = pl + RED_BLOCKS;
    k_reduce_partial<T><<<RED_BLOCKS, L1_THREADS, 0, st>>>(op, A, s, pv, pl, po);
    check_launch("k_reduce_partial");
    k_reduce_final<T><<<1, 32, 0, st>>>(op, pv, pl, po, RED_BLOCKS, d_value, d_idx);
    check_launch("k_reduce_final");
}

#define TB_L1_INST(T) \
    template void l1_set<T>(T*, const Strided&, T, cudaStream_t); \
    template void l1_scale<T>(T*, const Strided&, T, cudaStream_t, bool); \
    template void l1_shift<T>(T*, const Strided&, T, T, cudaStream_t, bool); \
    template void l1_add<T>(const T*, T*, const Strided2&, const Strided&, const Strided&, T, T, cudaStream_t, \
                            bool, bool); \
    template void l1_dot<T>(const T*, const T*, const Strided2&, T*, cudaStream_t, bool, bool); \
    template void l1_reduce<T>(int, const T*, const Strided&, T*, i64*, cudaStream_t);

TB_L1_INST(float)
TB_L1_INST(double)
TB_L1_INST(cplx<float>)
TB_L1_INST(cplx<double>)

} // namespace tb
