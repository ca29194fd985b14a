// cl_shim.hpp -- TEST INFRASTRUCTURE ONLY (part of the parity oracle).
//
// Lets the reference's OpenCL 1.2 C kernels (opencl/*.cl of atthecodeface/slm)
// compile as C++17 with g++ so that they can be executed on host cores as the
// pinned "reference" arm of the oracle.  Nothing in the product links this.
//
// The reference's kernel sources are never copied into this repository: the
// recipe in oracle/build_ref.py reads them from the reference checkout at build
// time, applies three syntactic rewrites (vector literals -> braced init,
// `(char)(` -> slm_cvt_char(`, the connect_channels private buffer size) and
// writes the generated translation units into oracle/_ref/ (git-ignored).
//
// Floating-point contract (shared with the C restatement and the CUDA kernels):
//   * every float operation is a separately rounded IEEE-754 binary32 op
//     (compile with -ffp-contract=off -fno-fast-math; x86-64 SSE, no x87);
//   * fast_length(v)    = sqrtf(v.x*v.x + v.y*v.y)            (IEEE sqrt)
//     fast_normalize(v) = (v.x/len, v.y/len), len = fast_length(v)
//     OpenCL leaves the precision of both implementation-defined
//     (reference opencl/essentials.cl:44, opencl/computestep.cl:98);
//   * float -> char conversion = truncate to int32 the x86 way (out-of-range
//     and NaN give INT32_MIN) then keep the low byte.  OpenCL leaves
//     out-of-range casts undefined; the reference's Euler tail step
//     (opencl/rungekutta.cl:109-112) relies on one;
//   * vector literal components are evaluated left to right (OpenCL C leaves
//     this unspecified; it matters for (float2)(rand(),rand()) in
//     opencl/rng.cl:62-67).
#pragma once
#include <cmath>
#include <cfloat>
#include <cstdint>
#include <cstdlib>
#include <cstdio>

typedef unsigned int uint;
typedef unsigned short ushort;
typedef unsigned char uchar;
typedef unsigned long ulong;

#define __kernel extern "C"
#define __global
#define __private
#define __local
#define __constant const
#ifndef MAXFLOAT
#define MAXFLOAT FLT_MAX
#endif

// ---------------------------------------------------------------- conversions
static inline signed char slm_cvt_char(float v) {
    int32_t i;
    if (!(v >= -2147483648.0f && v < 2147483648.0f)) i = INT32_MIN;
    else i = (int32_t)v;
    return (signed char)(uint8_t)(i & 0xff);
}
static inline signed char slm_cvt_char(double v) {
    int32_t i;
    if (!(v >= -2147483648.0 && v < 2147483648.0)) i = INT32_MIN;
    else i = (int32_t)v;
    return (signed char)(uint8_t)(i & 0xff);
}
static inline signed char slm_cvt_char(int v) { return (signed char)(uint8_t)(v & 0xff); }
static inline signed char slm_cvt_char(unsigned v) { return (signed char)(uint8_t)(v & 0xffu); }
static inline signed char slm_cvt_char(long v) { return (signed char)(uint8_t)(v & 0xff); }
static inline signed char slm_cvt_char(unsigned long v) { return (signed char)(uint8_t)(v & 0xff); }

// ---------------------------------------------------------------- float2
struct float2 {
    float s[2];
    float2() : s{0.0f, 0.0f} {}
    template <class A, class B>
    float2(A a, B b) : s{(float)a, (float)b} {}
    float& operator[](int i) { return s[i]; }
    const float& operator[](int i) const { return s[i]; }
    float2& operator+=(const float2& o) { s[0] = s[0] + o.s[0]; s[1] = s[1] + o.s[1]; return *this; }
    float2& operator-=(const float2& o) { s[0] = s[0] - o.s[0]; s[1] = s[1] - o.s[1]; return *this; }
    float2& operator*=(float f) { s[0] = s[0] * f; s[1] = s[1] * f; return *this; }
    float2& operator/=(float f) { s[0] = s[0] / f; s[1] = s[1] / f; return *this; }
};
static inline float2 operator+(const float2& a, const float2& b) { return float2(a.s[0] + b.s[0], a.s[1] + b.s[1]); }
static inline float2 operator-(const float2& a, const float2& b) { return float2(a.s[0] - b.s[0], a.s[1] - b.s[1]); }
static inline float2 operator-(const float2& a) { return float2(-a.s[0], -a.s[1]); }
static inline float2 operator*(const float2& a, const float2& b) { return float2(a.s[0] * b.s[0], a.s[1] * b.s[1]); }
static inline float2 operator/(const float2& a, const float2& b) { return float2(a.s[0] / b.s[0], a.s[1] / b.s[1]); }
// Scalar operands of any arithmetic type are first converted to float, as
// OpenCL does for a scalar widened to a float vector.
template <class T> static inline float2 operator*(const float2& a, T f) { float g = (float)f; return float2(a.s[0] * g, a.s[1] * g); }
template <class T> static inline float2 operator*(T f, const float2& a) { float g = (float)f; return float2(g * a.s[0], g * a.s[1]); }
template <class T> static inline float2 operator/(const float2& a, T f) { float g = (float)f; return float2(a.s[0] / g, a.s[1] / g); }
template <class T> static inline float2 operator+(const float2& a, T f) { float g = (float)f; return float2(a.s[0] + g, a.s[1] + g); }
template <class T> static inline float2 operator-(const float2& a, T f) { float g = (float)f; return float2(a.s[0] - g, a.s[1] - g); }

// ---------------------------------------------------------------- char2
struct char2 {
    signed char s[2];
    char2() : s{0, 0} {}
    char2(int v) : s{(signed char)v, (signed char)v} {}
    template <class A, class B>
    char2(A a, B b) : s{slm_cvt_char(a), slm_cvt_char(b)} {}
    signed char& operator[](int i) { return s[i]; }
    const signed char& operator[](int i) const { return s[i]; }
};

// ---------------------------------------------------------------- builtins
static inline float fast_length(const float2& v) { return sqrtf(v.s[0] * v.s[0] + v.s[1] * v.s[1]); }
static inline float2 fast_normalize(const float2& v) {
    const float len = fast_length(v);
    return float2(v.s[0] / len, v.s[1] / len);
}
// OpenCL integer/float min, max, clamp: "y if y<x else x" (min),
// "y if x<y else x" (max).  Names get an slm_cl_ prefix and a macro alias so
// that they never collide with the C library's abs/select/isless.
template <class A, class B> static inline auto slm_cl_min(A a, B b) -> decltype(a + b) {
    typedef decltype(a + b) T; return ((T)b < (T)a) ? (T)b : (T)a;
}
template <class A, class B> static inline auto slm_cl_max(A a, B b) -> decltype(a + b) {
    typedef decltype(a + b) T; return ((T)a < (T)b) ? (T)b : (T)a;
}
template <class A, class B, class C> static inline A slm_cl_clamp(A x, B lo, C hi) {
    return (A)slm_cl_min(slm_cl_max(x, (A)lo), (A)hi);
}
static inline uint slm_cl_abs(int x) { return x < 0 ? 0u - (uint)x : (uint)x; }
static inline float slm_cl_minmag(float x, float y) {
    if (fabsf(x) < fabsf(y)) return x;
    if (fabsf(y) < fabsf(x)) return y;
    return fminf(x, y);
}
template <class A, class B, class C> static inline A slm_cl_select(A a, B b, C c) { return c ? (A)b : a; }
template <class A, class B> static inline int slm_cl_isequal(A a, B b) { return a == b; }
template <class A, class B> static inline int slm_cl_isnotequal(A a, B b) { return a != b; }
template <class A, class B> static inline int slm_cl_isless(A a, B b) { return a < b; }
template <class A, class B> static inline int slm_cl_isgreater(A a, B b) { return a > b; }
template <class A, class B> static inline int slm_cl_isgreaterequal(A a, B b) { return a >= b; }
template <class A, class B> static inline int slm_cl_islessequal(A a, B b) { return a <= b; }
#define min slm_cl_min
#define max slm_cl_max
#define clamp slm_cl_clamp
#define abs slm_cl_abs
#define minmag slm_cl_minmag
#define select slm_cl_select
#define isequal slm_cl_isequal
#define isnotequal slm_cl_isnotequal
#define isless slm_cl_isless
#define isgreater slm_cl_isgreater
#define isgreaterequal slm_cl_isgreaterequal
#define islessequal slm_cl_islessequal

// Atomics are relaxed host atomics; in the sequential schedule they are plain
// read-modify-writes in ascending work-item order.
static inline uint atomic_add(volatile uint* p, uint v) { return __atomic_fetch_add((uint*)p, v, __ATOMIC_RELAXED); }
static inline uint atomic_inc(volatile uint* p) { return __atomic_fetch_add((uint*)p, 1u, __ATOMIC_RELAXED); }
static inline uint atomic_or(volatile uint* p, uint v) { return __atomic_fetch_or((uint*)p, v, __ATOMIC_RELAXED); }
static inline uint atomic_and(volatile uint* p, uint v) { return __atomic_fetch_and((uint*)p, v, __ATOMIC_RELAXED); }
static inline uint atomic_xchg(volatile uint* p, uint v) { return __atomic_exchange_n((uint*)p, v, __ATOMIC_RELAXED); }
static inline int atomic_xchg(volatile int* p, int v) { return __atomic_exchange_n((int*)p, v, __ATOMIC_RELAXED); }
static inline int atomic_or(volatile int* p, int v) { return __atomic_fetch_or((int*)p, v, __ATOMIC_RELAXED); }

// ---------------------------------------------------------------- work-items
static thread_local uint slmref_gid = 0;
static uint slmref_gsize = 0;
static uint slmref_goffset = 0;
static inline uint get_global_id(uint d) { return d == 0 ? slmref_gid : 0u; }
static inline uint get_global_size(uint d) { return d == 0 ? slmref_gsize : 1u; }
static inline uint get_global_offset(uint d) { return d == 0 ? slmref_goffset : 0u; }
static inline uint get_local_size(uint d) { (void)d; return 32u; }
static inline uint get_num_groups(uint d) { return d == 0 ? (slmref_gsize + 31u) / 32u : 1u; }

// ---------------------------------------------------------------- parameters
// Every -D macro of the reference's pocl.set_compile_options() is #defined by
// the generated translation unit as a field of a run-time struct (slmref_P,
// same layout as slm_params), so one library serves every parameter set.
