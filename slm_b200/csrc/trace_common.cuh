// trace_common.cuh -- device arithmetic shared by every tracing kernel.
//
// Bit-exact restatement of the reference's per-step arithmetic on sm_100a.
// The translation units that include this are compiled with --fmad=false and
// IEEE division / square root (no fast-math), so each expression below is a
// sequence of separately rounded binary32 operations in the order written,
// the same order as the reference's OpenCL C:
//   speed_interpolator   opencl/essentials.cl:24-45
//   get_array_idx        opencl/essentials.cl:56-59
//   approximate          opencl/essentials.cl:104-109
//   lehmer_rand_*        opencl/rng.cl:37-67
//   compute_step_vec[_jittered]  opencl/computestep.cl:42-57, 86-106
// Conventions fixed where OpenCL leaves them open (shared with the oracle):
//   fast_length = IEEE sqrt(x*x+y*y); fast_normalize divides by it;
//   float->char = x86 truncation (out of range / NaN -> INT32_MIN) low byte;
//   the two variates of lehmer_rand_vec are drawn x first, then y.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "slm_b200.h"

namespace slm {

typedef unsigned long long u64;

struct Vec2 { float x, y; };

// float -> char the way x86 converts (cvttss2si, keep the low byte): x86
// gives INT32_MIN for NaN and out-of-range values.  The device conversion
// saturates (NaN -> 0, below -2^31 -> INT32_MIN, from 2^31 up -> INT32_MAX),
// which has the same low byte (0) except from 2^31 up, the one case tested.
__device__ __forceinline__ int8_t cvt_i8(float v) {
    const int32_t i = (v < 2147483648.0f) ? __float2int_rz(v) : (int32_t)0x80000000;
    return (int8_t)(i & 0xff);
}

// clamped axis index: min(n-1, (uint)max(0, c + pad + 0.5))
__device__ __forceinline__ uint32_t axis_index(float c, float pp5, uint32_t n) {
    const float v = c + pp5;
    const float m = (0.0f < v) ? v : 0.0f;
    const uint32_t i = __float2uint_rz(m);
    return (i < n - 1u) ? i : n - 1u;
}

// The values of the step arithmetic that belong to one grid (one DTM tile):
// padded size and the macros the reference derives from it (pocl.py:231-277:
// GRID_SCALE = sqrt(nx*ny), COMBO_FACTOR = GRID_SCALE * step factor * sign,
// DT_MAX = min(1/nx, 1/ny, 0.1)).  Single-grid kernels take them from the
// parameter block; the batched kernel holds one per lane.
struct Geo {
    uint32_t nxp, nyp;
    float cf, dt_max, gs;
    float gs_inv;  // 1/gs when gs is a power of two (x/gs == x*gs_inv exactly), else 0
};

__device__ __forceinline__ float pow2_reciprocal(float v) {
    const uint32_t b = __float_as_uint(v);
    const uint32_t e = (b >> 23) & 0xffu;
    const bool pow2 = (b >> 31) == 0u && (b & 0x7fffffu) == 0u && e >= 1u && e <= 253u;
    return pow2 ? __fdiv_rn(1.0f, v) : 0.0f;
}

__device__ __forceinline__ Geo make_geo(uint32_t nxp, uint32_t nyp, float cf, float dt_max, float gs) {
    return Geo{nxp, nyp, cf, dt_max, gs, pow2_reciprocal(gs)};
}

__device__ __forceinline__ Geo geo_of(const slm_params& p) {
    return make_geo(p.nx_padded, p.ny_padded, p.combo_factor, p.dt_max, p.grid_scale);
}

// x / GRID_SCALE: a multiplication when GRID_SCALE is a power of two (both
// are the correctly rounded value of the same quotient).  P2: the caller has
// checked that it is (slm_pow2_steps), so the test is left out.
template <bool P2 = false>
__device__ __forceinline__ float div_gs(float x, const Geo& g) {
    if (P2) return x * g.gs_inv;
    return g.gs_inv != 0.0f ? x * g.gs_inv : __fdiv_rn(x, g.gs);
}

__device__ __forceinline__ uint32_t pixel_of(Vec2 a, const slm_params& p, const Geo& g) {
    return axis_index(a.y, p.pad_width_pp5, g.nyp)
         + g.nyp * axis_index(a.x, p.pad_width_pp5, g.nxp);
}

__device__ __forceinline__ uint32_t pixel_of(Vec2 a, const slm_params& p) {
    return pixel_of(a, p, geo_of(p));
}

// Bilinear, renormalised flow vector at a (essentials.cl:24-45).
__device__ __forceinline__ Vec2 sample_uv(Vec2 a, const float2* __restrict__ uv,
                                          const slm_params& p, const Geo& g) {
    const uint32_t nyp = g.nyp;
    const uint32_t xl = axis_index(a.x, p.pad_width_pp5, g.nxp);
    const uint32_t yd = axis_index(a.y, p.pad_width_pp5, nyp);
    const uint32_t xr = (xl + 1u < g.nxp - 1u) ? xl + 1u : g.nxp - 1u;
    const uint32_t yu = (yd + 1u < nyp - 1u) ? yd + 1u : nyp - 1u;
    const float wr = a.x - (float)xl + (float)p.pad_width;
    const float wl = 1.0f - wr;
    const float wu = a.y - (float)yd + (float)p.pad_width;
    const float wd = 1.0f - wu;
    const float2 q00 = __ldg(uv + (nyp * xl + yd));
    const float2 q10 = __ldg(uv + (nyp * xr + yd));
    const float2 q01 = __ldg(uv + (nyp * xl + yu));
    const float2 q11 = __ldg(uv + (nyp * xr + yu));
    const float bx = q00.x * wl + q10.x * wr, by = q00.y * wl + q10.y * wr;
    const float tx = q01.x * wl + q11.x * wr, ty = q01.y * wl + q11.y * wr;
    const float vx = bx * wd + tx * wu, vy = by * wd + ty * wu;
    const float len = __fsqrt_rn(vx * vx + vy * vy);
    return Vec2{__fdiv_rn(vx, len), __fdiv_rn(vy, len)};
}

__device__ __forceinline__ Vec2 sample_uv(Vec2 a, const float2* __restrict__ uv,
                                          const slm_params& p) {
    return sample_uv(a, uv, p, geo_of(p));
}

// Quantisation scale.  When trajectory_resolution is a power of two (128 by
// default) dividing by it is exactly a multiplication by its reciprocal.
// P2: the caller has checked that it is, so the test is left out.
template <bool P2 = false>
struct Quant {
    float res, inv;
    bool pow2;
    __device__ __forceinline__ float operator()(float v) const {
        const float c = (float)cvt_i8(v * res);
        if (P2) return c * inv;
        return pow2 ? c * inv : __fdiv_rn(c, res);
    }
};

template <bool P2 = false>
__device__ __forceinline__ Quant<P2> make_quant(uint32_t r) {
    Quant<P2> q;
    q.res = (float)r;
    q.inv = __fdiv_rn(1.0f, (float)r);
    q.pow2 = r != 0u && (r & (r - 1u)) == 0u;
    return q;
}

// x / 6 correctly rounded, for finite |x| >= 2^-120 without a division: the
// product by the constant 1/6 held as two floats, C_h = RN(1/6) and
// C_l = RN(1/6 - C_h), formed as RN(C_h x + RN(C_l x)) with one fused
// multiply-add -- Brisebarre and Muller's correctly rounded multiplication
// by a constant ("Correctly rounded multiplication by arbitrary precision
// constants", IEEE Transactions on Computers 57(2), 2008).  For 1/6 in
// binary32 it equals the IEEE quotient x / 6.0f for every finite x with
// |x| >= 2^-121 (checked over all 2^32 bit patterns: it differs only below
// that, where C_l x underflows, and at +-infinity).  Those inputs, and NaN,
// take the IEEE division; the RK4 step's sums are far inside the range.
// slm_selftest_div6 repeats the exhaustive check on the device.
__device__ __forceinline__ float div6(float x) {
    const float c_hi = 0x1.555556p-3f, c_lo = -0x1.555556p-28f;
    const float ax = fabsf(x);
    if (__builtin_expect(ax >= 0x1p-120f && ax <= 0x1.fffffep+127f, 1))
        return __fmaf_rn(c_hi, x, __fmul_rn(c_lo, x));
    return __fdiv_rn(x, 6.0f);
}

__device__ __forceinline__ float quant(float v, float res) {
    return __fdiv_rn((float)cvt_i8(v * res), res);
}

// Lehmer step s <- ((u64)(s+1) * 279470273) mod (2^32 - 5) (rng.cl:37-45),
// reduced with 2^32 == 5 (mod 2^32-5): two folds and one conditional subtract.
// With x = hi*2^32 + lo (hi < 2^28.1): lo + 5*hi < 2^32 + 2^31, so one carry
// c folds it to (lo + 5*hi mod 2^32) + 5c < 2^32, then one conditional subtract.
__device__ __forceinline__ uint32_t lehmer_next(uint32_t s) {
    const uint32_t t = s + 1u;
    const uint32_t lo = t * 279470273u;
    const uint32_t hi = __umulhi(t, 279470273u);
    const uint32_t h5 = hi * 5u;
    const uint32_t y = lo + h5;
    const uint32_t z = y + ((y < lo) ? 5u : 0u);
    return z >= 0xfffffffbu ? z - 0xfffffffbu : z;
}

// initial_rng_state of a seed: byte-reverse, one Lehmer step, byte-reverse
// (integratefields.cl:24-28, 96-99)
__device__ __forceinline__ uint32_t seed_rng(uint32_t seed_idx) {
    return __byte_perm(lehmer_next(__byte_perm(seed_idx, 0, 0x0123)), 0, 0x0123);
}

__device__ __forceinline__ Vec2 jitter(Vec2 u, uint32_t& rng, float mag) {
    // (float)r / (float)0xfffffffb: the divisor rounds to 2^32, and dividing
    // by a power of two is exactly a multiplication by 2^-32.
    rng = lehmer_next(rng);
    const float rx = __uint2float_rn(rng) * 2.3283064365386963e-10f - 0.5f;
    rng = lehmer_next(rng);
    const float ry = __uint2float_rn(rng) * 2.3283064365386963e-10f - 0.5f;
    u.x = u.x + rx * mag;
    u.y = u.y + ry * mag;
    const float len = __fsqrt_rn(u.x * u.x + u.y * u.y);
    u.x = __fdiv_rn(u.x, len);
    u.y = __fdiv_rn(u.y, len);
    return u;
}

struct Step {
    Vec2 d1, d2;   // first-order and final quantised steps
    Vec2 u1;       // flow vector at the start point
    Vec2 next;     // start + d2
    uint32_t idx;  // pixel of next
};

// RK2 (computestep.cl:42-57 / 86-106), or the RK4 extension (same
// quantisation; d1 = approx(h k1) for the error estimate).  P2: the
// trajectory resolution is a power of two (checked by the caller).
template <int ORDER, bool JITTER, bool P2 = false>
__device__ __forceinline__ Step rk_step(Vec2 a, float dt, uint32_t& rng,
                                        const float2* __restrict__ uv, const slm_params& p,
                                        const Geo& g) {
    Step s;
    const float cf = g.cf;
    const Quant<P2> quant = make_quant<P2>(p.trajectory_resolution);
    Vec2 k1 = sample_uv(a, uv, p, g);
    if (JITTER) k1 = jitter(k1, rng, p.jitter_magnitude);
    s.u1 = k1;
    if (ORDER == 2) {
        s.d1.x = quant(k1.x * cf * dt);
        s.d1.y = quant(k1.y * cf * dt);
        const Vec2 b{a.x + s.d1.x, a.y + s.d1.y};
        Vec2 k2 = sample_uv(b, uv, p, g);
        if (JITTER) k2 = jitter(k2, rng, p.jitter_magnitude);
        s.d2.x = quant(0.5f * (s.d1.x + k2.x * cf * dt));
        s.d2.y = quant(0.5f * (s.d1.y + k2.y * cf * dt));
    } else {
        const float h1x = k1.x * cf * dt, h1y = k1.y * cf * dt;
        s.d1.x = quant(h1x);
        s.d1.y = quant(h1y);
        const Vec2 b{a.x + 0.5f * h1x, a.y + 0.5f * h1y};
        Vec2 k2 = sample_uv(b, uv, p, g);
        if (JITTER) k2 = jitter(k2, rng, p.jitter_magnitude);
        const float h2x = k2.x * cf * dt, h2y = k2.y * cf * dt;
        const Vec2 c{a.x + 0.5f * h2x, a.y + 0.5f * h2y};
        Vec2 k3 = sample_uv(c, uv, p, g);
        if (JITTER) k3 = jitter(k3, rng, p.jitter_magnitude);
        const float h3x = k3.x * cf * dt, h3y = k3.y * cf * dt;
        const Vec2 d{a.x + h3x, a.y + h3y};
        Vec2 k4 = sample_uv(d, uv, p, g);
        if (JITTER) k4 = jitter(k4, rng, p.jitter_magnitude);
        const float h4x = k4.x * cf * dt, h4y = k4.y * cf * dt;
        s.d2.x = quant(div6(h1x + 2.0f * h2x + 2.0f * h3x + h4x));
        s.d2.y = quant(div6(h1y + 2.0f * h2y + 2.0f * h3y + h4y));
    }
    s.next.x = a.x + s.d2.x;
    s.next.y = a.y + s.d2.y;
    s.idx = pixel_of(s.next, p, g);
    return s;
}

template <int ORDER, bool JITTER>
__device__ __forceinline__ Step rk_step(Vec2 a, float dt, uint32_t& rng,
                                        const float2* __restrict__ uv, const slm_params& p) {
    return rk_step<ORDER, JITTER>(a, dt, rng, uv, p, geo_of(p));
}

__device__ __forceinline__ float vlen(float x, float y) { return __fsqrt_rn(x * x + y * y); }

// adaptive dt (rungekutta.cl:70-71): DT_MAX when the error is 0, else
// fmin(DT_MAX, ADJUSTED_MAX_ERROR*dt/err)
__device__ __forceinline__ float next_dt(float dt, float err, const slm_params& p, const Geo& g) {
    const float cand = fminf(g.dt_max, __fdiv_rn(p.adjusted_max_error * dt, err));
    return (err == 0.0f) ? g.dt_max : cand;
}

__device__ __forceinline__ float next_dt(float dt, float err, const slm_params& p) {
    return next_dt(dt, err, p, geo_of(p));
}

}  // namespace slm
