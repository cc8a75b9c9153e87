// cplx.hpp -- complex element type for the level-1 kernels and the
// conversions of the complex contraction path.
//
// The storage is TBLIS's scomplex / dcomplex (std::complex<float/double>,
// src/util/basic_types.h:97-98): real part then imaginary part, aligned to
// the full element so that 16-byte vector accesses stay legal. Ordering
// follows the reference's stl_ext operators
// (src/external/stl_ext/include/complex.hpp:187-240): a < b compares the
// real parts only, which is what MAX / MIN reductions and the sign test of a
// reduce's scalar use.
#pragma once

#include <cmath>
#include <type_traits>

#ifdef __CUDACC__
#define TB_HD __host__ __device__
#else
#define TB_HD
#endif

namespace tb
{

template <typename R>
struct alignas(2*sizeof(R)) cplx
{
    R re, im;
    cplx() = default;
    TB_HD constexpr cplx(R r) : re(r), im(R(0)) {}
    TB_HD constexpr cplx(R r, R i) : re(r), im(i) {}
};

template <typename R> TB_HD inline cplx<R> operator+(cplx<R> a, cplx<R> b) { return {a.re + b.re, a.im + b.im}; }
template <typename R> TB_HD inline cplx<R> operator-(cplx<R> a, cplx<R> b) { return {a.re - b.re, a.im - b.im}; }
template <typename R> TB_HD inline cplx<R> operator-(cplx<R> a) { return {-a.re, -a.im}; }
template <typename R> TB_HD inline cplx<R> operator*(cplx<R> a, cplx<R> b)
{
    return {a.re*b.re - a.im*b.im, a.re*b.im + a.im*b.re};
}
template <typename R> TB_HD inline cplx<R>& operator+=(cplx<R>& a, cplx<R> b) { a = a + b; return a; }
template <typename R> TB_HD inline cplx<R>& operator*=(cplx<R>& a, cplx<R> b) { a = a*b; return a; }
template <typename R> TB_HD inline bool operator==(cplx<R> a, cplx<R> b) { return a.re == b.re && a.im == b.im; }
template <typename R> TB_HD inline bool operator!=(cplx<R> a, cplx<R> b) { return !(a == b); }
template <typename R> TB_HD inline bool operator<(cplx<R> a, cplx<R> b) { return a.re < b.re; }
template <typename R> TB_HD inline bool operator>(cplx<R> a, cplx<R> b) { return b.re < a.re; }

template <typename T> struct is_cplx : std::false_type {};
template <typename R> struct is_cplx<cplx<R>> : std::true_type {};

template <typename T> struct real_of { using type = T; };
template <typename R> struct real_of<cplx<R>> { using type = R; };

// conj(x) when c, else x (identity for real types)
template <typename T> TB_HD inline T cj(T x, bool) { return x; }
template <typename R> TB_HD inline cplx<R> cj(cplx<R> x, bool c) { return c ? cplx<R>{x.re, -x.im} : x; }

// the ordering key of the reference's comparisons (real part for complex)
template <typename T> TB_HD inline T order_key(T x) { return x; }
template <typename R> TB_HD inline R order_key(cplx<R> x) { return x.re; }

// |x| as an element (std::abs; a complex result has zero imaginary part)
template <typename T> TB_HD inline T abs_elem(T x) { return x < T(0) ? -x : x; }
template <typename R> TB_HD inline cplx<R> abs_elem(cplx<R> x) { return cplx<R>(hypot(x.re, x.im)); }

// |x|^2 as an element (stl_ext::norm2)
template <typename T> TB_HD inline T norm2_elem(T x) { return x*x; }
template <typename R> TB_HD inline cplx<R> norm2_elem(cplx<R> x) { return cplx<R>(x.re*x.re + x.im*x.im); }

// sqrt of a real (or real-valued complex) element
template <typename T> TB_HD inline T sqrt_elem(T x) { return sqrt(x); }
template <typename R> TB_HD inline cplx<R> sqrt_elem(cplx<R> x) { return cplx<R>(sqrt(x.re)); }

} // namespace tb
