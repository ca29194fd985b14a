/* slm_oracle_trace.c -- TEST INFRASTRUCTURE ONLY: CPU restatement of the
 * reference's streamline tracer, used as the parity oracle and as the CPU
 * baseline.  It is never linked into, or called by, the product library.
 *
 * Follows, operation for operation, the OpenCL C of atthecodeface/slm:
 *   speed_interpolator       opencl/essentials.cl:24-45
 *   get_array_idx            opencl/essentials.cl:56-59
 *   compress / approximate   opencl/essentials.cl:71-74, 104-109
 *   dt_to_nearest_edge       opencl/essentials.cl:121-129
 *   lehmer_rand_uint/vec     opencl/rng.cl:37-67
 *   BYTE_REVERSAL, seeding   opencl/integratefields.cl:24-28, 96-99
 *   compute_step_vec[_jittered] opencl/computestep.cl:42-57, 86-106
 *   runge_kutta_step_record / euler_step_record  opencl/rungekutta.cl:49-120
 *   runge_kutta_step_write_sl_data               opencl/rungekutta.cl:163-186
 *   jittered_trajectory      opencl/jittertrajectory.cl:42-88
 *   integrate_fields         opencl/integratefields.cl:60-114
 *   trajectory_record        opencl/trajectory.cl:41-80
 * The RK4 integrator is this project's extension (no counterpart in the
 * reference, so its parity is pinned only by this restatement).
 *
 * Compile with -O2 -ffp-contract=off -fno-fast-math: every float operation is
 * a separately rounded IEEE binary32 op in the order written.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>
#include "slm_b200.h"

typedef struct { float x, y; } v2;

/* x86 float->char conversion (see cl_shim.hpp). */
static inline int8_t cvt_i8(float v) {
    int32_t i = (v >= -2147483648.0f && v < 2147483648.0f) ? (int32_t)v : INT32_MIN;
    return (int8_t)(uint8_t)(i & 0xff);
}

static inline uint32_t axis_index(float c, float pp5, uint32_t n) {
    float v = c + pp5;
    float m = (0.0f < v) ? v : 0.0f;
    uint32_t i = (uint32_t)m;
    return (i < n - 1u) ? i : n - 1u;
}

static inline uint32_t pixel_of(v2 a, const slm_params* p) {
    return axis_index(a.y, p->pad_width_pp5, p->ny_padded)
         + p->ny_padded * axis_index(a.x, p->pad_width_pp5, p->nx_padded);
}

static v2 sample_uv(v2 a, const float* uv, const slm_params* p) {
    const uint32_t nyp = p->ny_padded;
    const uint32_t xl = axis_index(a.x, p->pad_width_pp5, p->nx_padded);
    const uint32_t yd = axis_index(a.y, p->pad_width_pp5, p->ny_padded);
    const uint32_t xr = (xl + 1u < p->nx_padded - 1u) ? xl + 1u : p->nx_padded - 1u;
    const uint32_t yu = (yd + 1u < p->ny_padded - 1u) ? yd + 1u : p->ny_padded - 1u;
    const float wr = a.x - (float)xl + (float)p->pad_width;
    const float wl = 1.0f - wr;
    const float wu = a.y - (float)yd + (float)p->pad_width;
    const float wd = 1.0f - wu;
    const float* q00 = uv + 2u * (nyp * xl + yd);
    const float* q10 = uv + 2u * (nyp * xr + yd);
    const float* q01 = uv + 2u * (nyp * xl + yu);
    const float* q11 = uv + 2u * (nyp * xr + yu);
    const float bx = q00[0] * wl + q10[0] * wr, by = q00[1] * wl + q10[1] * wr;
    const float tx = q01[0] * wl + q11[0] * wr, ty = q01[1] * wl + q11[1] * wr;
    const float vx = bx * wd + tx * wu, vy = by * wd + ty * wu;
    const float len = sqrtf(vx * vx + vy * vy);
    v2 r = {vx / len, vy / len};
    return r;
}

static inline float quant(float v, uint32_t res) {
    const float r = (float)res;
    return (float)cvt_i8(v * r) / r;
}

static inline uint32_t lehmer(uint32_t* s) {
    *s = (uint32_t)(((uint64_t)(uint32_t)(*s + 1u) * 279470273u) % 0xfffffffbu);
    return *s;
}

static inline uint32_t byte_swap(uint32_t s) {
    return (s >> 24 & 0xffu) | (s >> 8 & 0xff00u) | (s << 8 & 0xff0000u) | (s << 24 & 0xff000000u);
}

/* initial_rng_state of a seed (integratefields.cl:96-99) */
static inline uint32_t seed_rng(uint32_t seed_idx) {
    uint32_t s = byte_swap(seed_idx);
    lehmer(&s);
    return byte_swap(s);
}

/* one jitter-and-renormalise of a sampled flow vector (computestep.cl:96-98) */
static inline v2 jitter(v2 u, uint32_t* rng, float mag) {
    const float rx = (float)lehmer(rng) / (float)0xfffffffbu - 0.5f;
    const float ry = (float)lehmer(rng) / (float)0xfffffffbu - 0.5f;
    u.x = u.x + rx * mag;
    u.y = u.y + ry * mag;
    const float len = sqrtf(u.x * u.x + u.y * u.y);
    u.x = u.x / len;
    u.y = u.y / len;
    return u;
}

typedef struct {
    v2 d1, d2;   /* first-order and final (quantised) step */
    v2 u1;       /* flow vector at the start point */
    v2 next;     /* start + d2 */
    uint32_t idx;
} step_t;

/* RK2 step, plain (rng==NULL) or jittered (computestep.cl:42-57, 86-106) */
static step_t rk2_step(v2 a, float dt, uint32_t* rng, const float* uv, const slm_params* p) {
    step_t s;
    const float cf = p->combo_factor;
    const uint32_t res = p->trajectory_resolution;
    v2 u1 = sample_uv(a, uv, p);
    if (rng) u1 = jitter(u1, rng, p->jitter_magnitude);
    s.u1 = u1;
    s.d1.x = quant(u1.x * cf * dt, res);
    s.d1.y = quant(u1.y * cf * dt, res);
    v2 b = {a.x + s.d1.x, a.y + s.d1.y};
    v2 u2 = sample_uv(b, uv, p);
    if (rng) u2 = jitter(u2, rng, p->jitter_magnitude);
    s.d2.x = quant(0.5f * (s.d1.x + u2.x * cf * dt), res);
    s.d2.y = quant(0.5f * (s.d1.y + u2.y * cf * dt), res);
    s.next.x = a.x + s.d2.x;
    s.next.y = a.y + s.d2.y;
    s.idx = pixel_of(s.next, p);
    return s;
}

/* RK4 step (extension): k1..k4 at a, a+h/2 k1, a+h/2 k2, a+h k3 with h = cf*dt;
 * d1 = approx(h k1) is the first-order step used for the error estimate and
 * d2 = approx((h k1 + 2 h k2 + 2 h k3 + h k4) / 6).  Jitter, when on, is
 * applied to each k as in the RK2 jittered step (2 draws per sample). */
static step_t rk4_step(v2 a, float dt, uint32_t* rng, const float* uv, const slm_params* p) {
    step_t s;
    const float cf = p->combo_factor;
    const uint32_t res = p->trajectory_resolution;
    v2 k1 = sample_uv(a, uv, p);
    if (rng) k1 = jitter(k1, rng, p->jitter_magnitude);
    s.u1 = k1;
    const float h1x = k1.x * cf * dt, h1y = k1.y * cf * dt;
    s.d1.x = quant(h1x, res);
    s.d1.y = quant(h1y, res);
    v2 b = {a.x + 0.5f * h1x, a.y + 0.5f * h1y};
    v2 k2 = sample_uv(b, uv, p);
    if (rng) k2 = jitter(k2, rng, p->jitter_magnitude);
    const float h2x = k2.x * cf * dt, h2y = k2.y * cf * dt;
    v2 c = {a.x + 0.5f * h2x, a.y + 0.5f * h2y};
    v2 k3 = sample_uv(c, uv, p);
    if (rng) k3 = jitter(k3, rng, p->jitter_magnitude);
    const float h3x = k3.x * cf * dt, h3y = k3.y * cf * dt;
    v2 d = {a.x + h3x, a.y + h3y};
    v2 k4 = sample_uv(d, uv, p);
    if (rng) k4 = jitter(k4, rng, p->jitter_magnitude);
    const float h4x = k4.x * cf * dt, h4y = k4.y * cf * dt;
    s.d2.x = quant((h1x + 2.0f * h2x + 2.0f * h3x + h4x) / 6.0f, res);
    s.d2.y = quant((h1y + 2.0f * h2y + 2.0f * h3y + h4y) / 6.0f, res);
    s.next.x = a.x + s.d2.x;
    s.next.y = a.y + s.d2.y;
    s.idx = pixel_of(s.next, p);
    return s;
}

static inline step_t take_step(int rk4, v2 a, float dt, uint32_t* rng, const float* uv,
                               const slm_params* p) {
    return rk4 ? rk4_step(a, dt, rng, uv, p) : rk2_step(a, dt, rng, uv, p);
}

static inline float vlen(float x, float y) { return sqrtf(x * x + y * y); }

/* adaptive dt of every RK step function (rungekutta.cl:70-71) */
static inline float next_dt(float dt, float err, const slm_params* p) {
    const float cand = fminf(p->dt_max, (p->adjusted_max_error * dt) / err);
    return (err == 0.0f) ? p->dt_max : cand;
}

static inline void visit(uint64_t* slt, uint64_t* slc, uint32_t idx, float l, int atomic) {
    const uint64_t v = (uint32_t)(l + 0.5f);
    if (atomic) {
        __atomic_fetch_add(&slt[idx], v, __ATOMIC_RELAXED);
        __atomic_fetch_add(&slc[idx], (uint64_t)1, __ATOMIC_RELAXED);
    } else {
        slt[idx] += v;
        slc[idx] += 1;
    }
}

/* jittered_trajectory (jittertrajectory.cl:42-88); returns the number of RK steps */
static uint64_t field_trajectory(v2 start, uint32_t rng0, int rk4, const uint8_t* mask,
                                 const float* uv, uint64_t* slc, uint64_t* slt,
                                 const slm_params* p, int atomic) {
    uint32_t rng = rng0, n = 0, idx;
    float l = 0.0f, dl, dt = p->dt_max;
    v2 a = start;
    uint64_t steps = 0;
    idx = pixel_of(a, p);
    if (!mask[idx]) visit(slt, slc, idx, l, atomic);
    while (idx < p->nxy_padded && !mask[idx] && (l < p->max_length && n < p->max_n_steps)) {
        const step_t s = take_step(rk4, a, dt, &rng, uv, p);
        steps++;
        idx = s.idx;
        /* idx never reaches nxy_padded (pixel_of clamps), so the reference's
         * Euler branch (jittertrajectory.cl:79-84) cannot run. */
        if (mask[idx]) continue;           /* loop condition then ends the trajectory */
        const float err = vlen((s.d2.x - s.d1.x) / p->grid_scale, (s.d2.y - s.d1.y) / p->grid_scale);
        dl = vlen(s.d2.x, s.d2.y);
        a = s.next;
        if (dl < p->integration_halt_threshold) {
            l += dl; n++;
            idx = pixel_of(a, p);
            if (idx < p->nxy_padded && !mask[idx]) visit(slt, slc, idx, l, atomic);
            break;
        }
        dt = next_dt(dt, err, p);
        l += dl; n++;
        idx = pixel_of(a, p);
        if (idx < p->nxy_padded && !mask[idx]) visit(slt, slc, idx, l, atomic);
    }
    return steps;
}

/* Fields: every seed in [seed_begin, seed_end) with stride, d*d sub-pixel
 * trajectories each (integratefields.cl:83-113).  slc/slt are uint64 and
 * accumulate.  Returns the number of RK steps taken; *n_traj gets the number
 * of trajectories. */
uint64_t oracle_integrate_fields(const slm_params* p, int integrator,
                                 const float* seed_point, uint32_t seed_begin,
                                 uint32_t seed_end, uint32_t seed_stride,
                                 const uint8_t* mask, const float* uv,
                                 uint64_t* slc, uint64_t* slt, uint64_t* n_traj,
                                 int n_threads) {
    const int rk4 = integrator == SLM_RK4;
    const uint32_t d = p->subpixel_seed_point_density;
    uint64_t steps = 0, ntraj = 0;
    if (seed_end > p->n_seed_points) seed_end = p->n_seed_points;
    if (seed_stride == 0) seed_stride = 1;
    const long n_iter = seed_end > seed_begin ? (long)((seed_end - seed_begin + seed_stride - 1) / seed_stride) : 0;
    const int atomic = n_threads > 1;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : steps, ntraj) num_threads(n_threads > 1 ? n_threads : 1)
    for (long it = 0; it < n_iter; ++it) {
        const uint32_t seed_idx = seed_begin + (uint32_t)it * seed_stride;
        const uint32_t rng0 = seed_rng(seed_idx);
        const v2 c = {seed_point[2 * (size_t)seed_idx], seed_point[2 * (size_t)seed_idx + 1]};
        for (uint32_t j = 0; j < d; ++j) {
            for (uint32_t i = 0; i < d; ++i) {
                v2 s0;
                s0.x = c.x + ((float)i * p->subpixel_seed_step - p->subpixel_seed_halfspan);
                s0.y = c.y + ((float)j * p->subpixel_seed_step - p->subpixel_seed_halfspan);
                steps += field_trajectory(s0, rng0, rk4, mask, uv, slc, slt, p, atomic);
                ntraj++;
            }
        }
    }
    if (n_traj) *n_traj = ntraj;
    return steps;
}

/* Per-seed RK step counts of a field pass (the sum over the seed's d*d
 * trajectories) -- the per-seed load a seed shard carries; slc/slt receive
 * the pass's sums as in oracle_integrate_fields. */
void oracle_field_seed_steps(const slm_params* p, int integrator, const float* seed_point,
                             const uint8_t* mask, const float* uv, uint64_t* slc, uint64_t* slt,
                             uint32_t* seed_steps, int n_threads) {
    const int rk4 = integrator == SLM_RK4;
    const uint32_t d = p->subpixel_seed_point_density;
    const long n = (long)p->n_seed_points;
    const int atomic = n_threads > 1;
#pragma omp parallel for schedule(dynamic, 64) num_threads(n_threads > 1 ? n_threads : 1)
    for (long it = 0; it < n; ++it) {
        const uint32_t seed_idx = (uint32_t)it;
        const uint32_t rng0 = seed_rng(seed_idx);
        const v2 c = {seed_point[2 * (size_t)seed_idx], seed_point[2 * (size_t)seed_idx + 1]};
        uint64_t steps = 0;
        for (uint32_t j = 0; j < d; ++j) {
            for (uint32_t i = 0; i < d; ++i) {
                v2 s0;
                s0.x = c.x + ((float)i * p->subpixel_seed_step - p->subpixel_seed_halfspan);
                s0.y = c.y + ((float)j * p->subpixel_seed_step - p->subpixel_seed_halfspan);
                steps += field_trajectory(s0, rng0, rk4, mask, uv, slc, slt, p, atomic);
            }
        }
        seed_steps[seed_idx] = (uint32_t)steps;
    }
}

static inline float edge_dt(float x, float u) {
    float dt = 0.0f;
    const float right = ((float)(int32_t)(x + 1.5f) - (x + 0.5f)) / u;
    const float left = -((x + 0.5f) - (float)(int32_t)(x + 0.5f)) / u;
    if (u > 0.0f) dt = right;
    if (u < 0.0f) dt = left;
    return dt;
}

static inline float min_mag(float x, float y) {
    if (fabsf(x) < fabsf(y)) return x;
    if (fabsf(y) < fabsf(x)) return y;
    return fminf(x, y);
}

/* trajectory_record (trajectory.cl:41-80) for chunk-local seed g */
static uint64_t record_trajectory(v2 a, int rk4, const uint8_t* mask, const float* uv,
                                  const slm_params* p, int8_t* rec, uint16_t* nsteps_out,
                                  float* length_out) {
    uint32_t n = 0, idx;
    float l = 0.0f, dl, dt = p->dt_max;
    v2 prev = a;
    uint64_t steps = 0;
    const float res = (float)p->trajectory_resolution;
    idx = pixel_of(a, p);
    while (!mask[idx] && (l < p->max_length && n < p->max_n_steps)) {
        const step_t s = take_step(rk4, a, dt, NULL, uv, p);
        steps++;
        idx = s.idx;
        if (!mask[idx]) {
            const float err = vlen((s.d2.x - s.d1.x) / p->grid_scale, (s.d2.y - s.d1.y) / p->grid_scale);
            v2 next = s.next;
            dl = vlen(s.d2.x, s.d2.y);
            if (dl < p->integration_halt_threshold) {
                next.x = a.x + s.d1.x;
                next.y = a.y + s.d1.y;
                dl = vlen(s.d1.x, s.d1.y);
            }
            a = next;
            idx = pixel_of(next, p);
            const int stuck = dl < p->integration_halt_threshold;
            if (!stuck) dt = next_dt(dt, err, p);
            l += dl;
            rec[2 * (size_t)n] = cvt_i8((a.x - prev.x) * res);
            rec[2 * (size_t)n + 1] = cvt_i8((a.y - prev.y) * res);
            n++;
            if (stuck) break;
            prev = a;
        } else {
            /* euler_step_record (rungekutta.cl:96-120): DOWNUP_SIGN is an
             * unsigned literal, so upstream it widens to 4294967296.0f. */
            const float sg = (float)p->downup_sign;
            const float sx = s.u1.x * sg, sy = s.u1.y * sg;
            const float dtx = edge_dt(a.x, sx), dty = edge_dt(a.y, sy);
            dt = min_mag(dtx, dty);
            a.x = a.x + sx * dt;
            a.y = a.y + sy * dt;
            a.x = quant(a.x, p->trajectory_resolution);
            a.y = quant(a.y, p->trajectory_resolution);
            a.x = fminf(fmaxf(a.x, -0.5f), p->nxf_mp5);
            a.y = fminf(fmaxf(a.y, -0.5f), p->nyf_mp5);
            dl = vlen(a.x - prev.x, a.y - prev.y);
            l += dl;
            rec[2 * (size_t)n] = cvt_i8((a.x - prev.x) * res);
            rec[2 * (size_t)n + 1] = cvt_i8((a.y - prev.y) * res);
            n++;
            break;
        }
    }
    *nsteps_out = (uint16_t)n;
    *length_out = l;
    return steps;
}

/* Trajectories of the chunk seeds_chunk_offset .. +n_chunk (clipped to
 * n_seed_points); buffers are chunk-local.  Returns RK steps taken. */
uint64_t oracle_integrate_trajectory(const slm_params* p, int integrator, uint32_t n_chunk,
                                     const float* seed_point, const uint8_t* mask,
                                     const float* uv, int8_t* trajectories,
                                     uint16_t* nsteps, float* length, int n_threads) {
    const int rk4 = integrator == SLM_RK4;
    uint64_t steps = 0;
#pragma omp parallel for schedule(dynamic, 4) reduction(+ : steps) num_threads(n_threads > 1 ? n_threads : 1)
    for (long g = 0; g < (long)n_chunk; ++g) {
        const uint32_t seed_idx = p->seeds_chunk_offset + (uint32_t)g;
        if (seed_idx >= p->n_seed_points) continue;
        const v2 a = {seed_point[2 * (size_t)seed_idx], seed_point[2 * (size_t)seed_idx + 1]};
        steps += record_trajectory(a, rk4, mask, uv, p,
                                   trajectories + 2 * (size_t)g * p->max_n_steps,
                                   &nsteps[g], &length[g]);
    }
    return steps;
}
