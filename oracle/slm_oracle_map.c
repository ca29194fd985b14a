/* slm_oracle_map.c -- TEST INFRASTRUCTURE ONLY: CPU restatement of the
 * reference's channel/segment mapping kernels, run as one pinned schedule:
 * work-items one after another in ascending global id.  Used as the parity
 * oracle; never linked into the product library.
 *
 *   connect_channels           opencl/connect.cl:26-108
 *   map_channel_heads          opencl/channelheads.cl:32-93
 *   prune_channel_heads        opencl/channelheads.cl:143-199
 *   count_downchannels         opencl/countlink.cl:34-114
 *   flag_downchannels          opencl/countlink.cl:134-210
 *   label_confluences          opencl/label.cl:49-134
 *   segment_downchannels       opencl/segment.cl:38-107
 *   segment_hillslopes         opencl/segment.cl:133-188
 *   subsegment_channel_edges   opencl/segment.cl:195-334
 *   subsegment_flanks          opencl/segment.cl:360-414
 *   fix_right_flanks           opencl/segment.cl:441-504
 *   fix_left_flanks            opencl/segment.cl:530-594
 *   hillslopes                 opencl/hillslopes.cl:31-91
 *   hillslope_lengths          opencl/lengths.cl:37-116
 * with the step functions of opencl/rungekutta.cl:280-516 and
 * compute_step_vec (opencl/computestep.cl:42-57).
 *
 * Where the reference can run without bound or read outside the grid, this
 * restatement caps the loop or skips the access and reports it through the
 * returned status word (bit 0: a loop cap was hit, bit 1: an out-of-grid
 * index was skipped); on the inputs the tests use neither happens.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include "slm_b200.h"

#define ST_CAP 1u
#define ST_OOB 2u
#define LOOP_CAP (1u << 26)

typedef struct { float x, y; } v2;

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
static inline float vlen(float x, float y) { return sqrtf(x * x + y * y); }

/* compute_step_vec: RK2 with quantised steps; returns next pixel via *idx */
typedef struct { v2 d1, d2, next; } rk_t;
static rk_t rk_compute(v2 a, float dt, const float* uv, const slm_params* p, uint32_t* idx) {
    rk_t s;
    const float cf = p->combo_factor;
    const uint32_t res = p->trajectory_resolution;
    v2 u1 = sample_uv(a, uv, p);
    s.d1.x = quant(u1.x * cf * dt, res);
    s.d1.y = quant(u1.y * cf * dt, res);
    v2 b = {a.x + s.d1.x, a.y + s.d1.y};
    v2 u2 = sample_uv(b, uv, p);
    s.d2.x = quant(0.5f * (s.d1.x + u2.x * cf * dt), res);
    s.d2.y = quant(0.5f * (s.d1.y + u2.y * cf * dt), res);
    s.next.x = a.x + s.d2.x;
    s.next.y = a.y + s.d2.y;
    *idx = pixel_of(s.next, p);
    return s;
}

/* the part every *_runge_kutta_step shares (rungekutta.cl:289-296 etc.):
 * error estimate, step length, first-order fallback when stuck, move */
typedef struct { float err, dl; int stuck; } rkmove_t;
static rkmove_t rk_move(const rk_t* s, v2* vec, uint32_t* idx, const slm_params* p) {
    rkmove_t m;
    m.err = vlen((s->d2.x - s->d1.x) / p->grid_scale, (s->d2.y - s->d1.y) / p->grid_scale);
    v2 next = s->next;
    m.dl = vlen(s->d2.x, s->d2.y);
    if (m.dl < p->integration_halt_threshold) {
        next.x = vec->x + s->d1.x;
        next.y = vec->y + s->d1.y;
        m.dl = vlen(s->d1.x, s->d1.y);
    }
    *vec = next;
    *idx = pixel_of(next, p);
    m.stuck = m.dl < p->integration_halt_threshold;
    return m;
}
static inline float next_dt(float dt, float err, const slm_params* p) {
    const float cand = fminf(p->dt_max, (p->adjusted_max_error * dt) / err);
    return (err == 0.0f) ? p->dt_max : cand;
}
static inline v2 seed_at(const float* seeds, uint32_t g) {
    v2 a = {seeds[2 * (size_t)g], seeds[2 * (size_t)g + 1]};
    return a;
}

/* ------------------------------------------------------------- connect */
uint32_t oracle_connect_channels(const slm_params* p, const float* seeds, uint32_t n,
                                 const uint8_t* mask, const float* uv, uint32_t* mapping) {
    uint32_t status = 0;
    /* only entries below interchannel_max_n_steps are ever read back */
    const uint32_t cap_rec = p->interchannel_max_n_steps;
    int8_t* rec = (int8_t*)malloc(2 * (size_t)(cap_rec + 1));
    for (uint32_t g = 0; g < n; ++g) {
        const v2 start = seed_at(seeds, g);
        uint32_t idx, prev_idx, n_steps = 0, step;
        float l = 0.0f, dt = p->dt_max;
        v2 vec = start, prev = start;
        (void)l;
        idx = pixel_of(vec, p);
        prev_idx = idx;
        uint32_t guard = 0;
        /* integrate downstream one pixel (connect.cl:60-68) */
        while (prev_idx == idx && !mask[idx] && n_steps != p->max_n_steps) {
            if (++guard > LOOP_CAP) { status |= ST_CAP; break; }
            rk_t s = rk_compute(vec, dt, uv, p, &idx);
            if (!mask[idx]) {
                rkmove_t m = rk_move(&s, &vec, &idx, p);
                if (!m.stuck) dt = next_dt(dt, m.err, p);
                l += m.dl;
                if (n_steps < cap_rec) {
                    rec[2 * n_steps] = cvt_i8((vec.x - prev.x) * (float)p->trajectory_resolution);
                    rec[2 * n_steps + 1] = cvt_i8((vec.y - prev.y) * (float)p->trajectory_resolution);
                }
                n_steps++;
                if (!m.stuck) prev = vec;
            }
        }
        /* until back on a channel pixel or masked (connect.cl:70-79).  Every
         * pass that does not exit adds a step, so the loop ends at
         * n_steps == INTERCHANNEL_MAX_N_STEPS; when the first loop already
         * went past that count, the reference's loop writes nothing and ends
         * with n_steps >= the count (at a channel, a masked pixel or the
         * 32-bit wrap), so the flagging below does not run either way. */
        guard = 0;
        while (n_steps <= p->interchannel_max_n_steps && (mapping[idx] & p->is_channel) == 0
               && !mask[idx] && n_steps != p->interchannel_max_n_steps) {
            if (++guard > LOOP_CAP) { status |= ST_CAP; break; }
            rk_t s = rk_compute(vec, dt, uv, p, &idx);
            if (!mask[idx]) {
                rkmove_t m = rk_move(&s, &vec, &idx, p);
                if (!m.stuck) dt = next_dt(dt, m.err, p);
                l += m.dl;
                if (n_steps < cap_rec) {
                    rec[2 * n_steps] = cvt_i8((vec.x - prev.x) * (float)p->trajectory_resolution);
                    rec[2 * n_steps + 1] = cvt_i8((vec.y - prev.y) * (float)p->trajectory_resolution);
                }
                n_steps++;
                if (!m.stuck) prev = vec;
            }
        }
        if (n_steps > 2 && n_steps < p->interchannel_max_n_steps) {
            /* flag the pixels between channels (connect.cl:80-97) */
            vec = start;
            idx = pixel_of(vec, p);
            step = 0;
            while (!mask[idx] && step < n_steps - 1) {
                if (mapping[idx] == 0u) mapping[idx] |= p->is_interchannel;
                vec.x = vec.x + (float)rec[2 * step] / (float)p->trajectory_resolution;
                vec.y = vec.y + (float)rec[2 * step + 1] / (float)p->trajectory_resolution;
                idx = pixel_of(vec, p);
                step++;
            }
        }
    }
    free(rec);
    return status;
}

/* ------------------------------------------------------------- channel heads */
uint32_t oracle_map_channel_heads(const slm_params* p, const float* seeds, uint32_t n,
                                  const uint8_t* mask, const float* uv, uint32_t* mapping) {
    uint32_t status = 0;
    for (uint32_t g = 0; g < n; ++g) {
        uint32_t idx, prev_idx, n_steps = 0;
        float dt = p->dt_max;
        v2 vec = seed_at(seeds, g);
        idx = pixel_of(vec, p);
        prev_idx = idx;
        while (prev_idx == idx && !mask[idx] && n_steps < p->max_n_steps) {
            rk_t s = rk_compute(vec, dt, uv, p, &idx);
            rkmove_t m = rk_move(&s, &vec, &idx, p);
            n_steps++;
            dt = next_dt(dt, m.err, p);   /* channelheads step updates dt unconditionally */
        }
        if (n_steps >= p->max_n_steps) continue;
        if (!mask[idx]) {
            idx = pixel_of(vec, p);
            if (((~mapping[idx]) & p->is_thinchannel) || (mapping[prev_idx] & p->is_thinchannel))
                mapping[idx] &= ~p->is_channelhead;
        }
    }
    return status;
}

uint32_t oracle_prune_channel_heads(const slm_params* p, const float* seeds, uint32_t n,
                                    const uint8_t* mask, const float* uv, uint32_t* mapping) {
    (void)mask; (void)uv;
    /* neighbour order N, S, E, W, NE, SE, NW, SW (channelheads.cl:181-188) */
    static const float off[8][2] = {{0, 1}, {0, -1}, {1, 0}, {-1, 0}, {1, 1}, {1, -1}, {-1, 1}, {-1, -1}};
    for (uint32_t g = 0; g < n; ++g) {
        const v2 vec = seed_at(seeds, g);
        uint32_t flag = 0;
        for (int k = 0; k < 8; ++k) {
            v2 nb = {vec.x + off[k][0], vec.y + off[k][1]};
            flag += (mapping[pixel_of(nb, p)] & p->is_thinchannel) != 0;
        }
        if (flag != 1u) {
            const uint32_t idx = pixel_of(vec, p);
            mapping[idx] &= ~p->is_channelhead;
            if (flag == 0) mapping[idx] &= ~(p->is_thinchannel | p->is_channel);
        }
    }
    return 0;
}

/* ------------------------------------------------------------- count / flag */
uint32_t oracle_count_downchannels(const slm_params* p, const float* seeds, uint32_t n,
                                   const uint8_t* mask, const float* uv, uint32_t* mapping,
                                   uint32_t* count, uint32_t* link) {
    for (uint32_t g = 0; g < n; ++g) {
        uint32_t idx, prev_idx, n_steps = 0, counter = 1;
        float dt = p->dt_max;
        v2 vec = seed_at(seeds, g);
        idx = pixel_of(vec, p);
        prev_idx = idx;
        count[idx] = counter++;
        while (!mask[idx] && n_steps < 1000u * p->max_n_steps) {
            rk_t s = rk_compute(vec, dt, uv, p, &idx);
            rkmove_t m = rk_move(&s, &vec, &idx, p);
            if (m.stuck) break;
            dt = next_dt(dt, m.err, p);
            n_steps++;
            if (prev_idx != idx) {
                mapping[idx] &= ~p->is_channelhead;
                mapping[idx] |= p->is_thinchannel;
                link[prev_idx] = idx;
                if (++counter < count[idx]) break;
                count[idx] = counter;
                prev_idx = idx;
            }
        }
        link[prev_idx] = idx;
    }
    return 0;
}

uint32_t oracle_flag_downchannels(const slm_params* p, const float* seeds, uint32_t n,
                                  const uint8_t* mask, const float* uv, uint32_t* mapping,
                                  uint32_t* count, const uint32_t* link) {
    (void)uv;
    const uint32_t lim = 1000u * p->max_n_steps;
    for (uint32_t g = 0; g < n; ++g) {
        const v2 vec = seed_at(seeds, g);
        const uint32_t head = pixel_of(vec, p);
        uint32_t idx = head, prev_idx = idx + 1u, counter = 1;
        count[idx] = counter;
        mapping[idx] |= p->is_thinchannel;
        while (!mask[idx] && prev_idx != idx && counter < lim) {
            prev_idx = idx;
            idx = link[idx];
            counter++;
            if (!mask[idx]) {
                if (((mapping[idx] & p->is_minorinflow) > 0 || (counter == 2u && count[idx] > 2u))
                    && counter < 20u)
                    mapping[head] &= ~p->is_channelhead;
                mapping[idx] |= p->is_thinchannel;
                if (counter >= count[idx]) count[idx] = counter;
            } else {
                break;
            }
        }
        if (!mask[prev_idx] && counter < lim) mapping[prev_idx] |= p->is_channeltail;
    }
    return 0;
}

/* ------------------------------------------------------------- label */
uint32_t oracle_label_confluences(const slm_params* p, const float* seeds, uint32_t n,
                                  const uint8_t* mask, const float* uv, const float* slt,
                                  uint32_t* mapping, const uint32_t* count, const uint32_t* link) {
    (void)uv;
    static const float off[8][2] = {{0, 1}, {0, -1}, {1, 0}, {-1, 0}, {1, 1}, {1, -1}, {-1, 1}, {-1, -1}};
    for (uint32_t g = 0; g < n; ++g) {
        const v2 vec = seed_at(seeds, g);
        const uint32_t idx = pixel_of(vec, p);
        uint32_t inflows[8], equal_dom[8], n_in = 0, n_eq = 0, dom_idx = 0;
        float dom_slt = -3.40282347e+38f;
        for (int k = 0; k < 8; ++k) {
            v2 nb = {vec.x + off[k][0], vec.y + off[k][1]};
            const uint32_t ni = pixel_of(nb, p);
            if (!mask[ni] && (mapping[ni] & p->is_thinchannel) && link[ni] == idx)
                inflows[n_in++] = ni;
        }
        if (n_in > 1) {
            mapping[idx] |= p->is_majorconfluence;
            for (uint32_t i = 0; i < n_in; ++i) {
                if (count[idx] != count[inflows[i]] + 1u) {
                    mapping[inflows[i]] |= p->is_minorinflow;
                } else {
                    equal_dom[n_eq++] = inflows[i];
                    if (slt[inflows[i]] > dom_slt) {
                        dom_idx = inflows[i];
                        dom_slt = slt[dom_idx];
                    }
                }
            }
            for (uint32_t i = 0; i < n_eq; ++i) {
                if (equal_dom[i] == dom_idx) mapping[equal_dom[i]] |= p->is_majorinflow;
                else mapping[equal_dom[i]] |= p->is_minorinflow;
            }
        }
    }
    return 0;
}

/* ------------------------------------------------------------- segments */
uint32_t oracle_segment_downchannels(const slm_params* p, const float* seeds, uint32_t n,
                                     const uint8_t* mask, const float* uv, uint32_t* mapping,
                                     const uint32_t* count, const uint32_t* link, uint32_t* label) {
    (void)uv;
    uint32_t status = 0;
    for (uint32_t g = 0; g < n; ++g) {
        const v2 vec = seed_at(seeds, g);
        uint32_t prev_idx = pixel_of(vec, p), idx, seg_counter = 0, seg_label;
        seg_label = prev_idx;
        label[prev_idx] = seg_label;
        mapping[prev_idx] |= p->is_subsegmenthead;
        idx = link[prev_idx];
        uint32_t guard = 0;
        while (!mask[idx] && prev_idx != idx && (mapping[idx] & p->is_subsegmenthead) == 0) {
            if (++guard > LOOP_CAP) { status |= ST_CAP; break; }
            if (count[idx] >= seg_counter + p->segmentation_threshold / 2u) {
                seg_label = idx;
                seg_counter = count[idx] + p->segmentation_threshold;
                mapping[idx] |= p->is_subsegmenthead;
            }
            label[idx] = seg_label;
            prev_idx = idx;
            idx = link[idx];
        }
    }
    return status;
}

/* segment_runge_kutta_step: n_steps++ always; stuck ends the walk */
static inline int seg_step(v2* vec, uint32_t* idx, float* dt, uint32_t* n_steps, const float* uv,
                           const slm_params* p, int do_compute, rk_t* pre) {
    rk_t s = do_compute ? rk_compute(*vec, *dt, uv, p, idx) : *pre;
    rkmove_t m = rk_move(&s, vec, idx, p);
    (*n_steps)++;
    if (m.stuck) return 1;
    *dt = next_dt(*dt, m.err, p);
    return 0;
}

uint32_t oracle_segment_hillslopes(const slm_params* p, const float* seeds, uint32_t n,
                                   const uint8_t* mask, const float* uv, const uint32_t* mapping,
                                   const uint32_t* count, const uint32_t* link, uint32_t* label) {
    (void)count; (void)link;
    for (uint32_t g = 0; g < n; ++g) {
        v2 vec = seed_at(seeds, g);
        uint32_t idx = pixel_of(vec, p), n_steps = 0;
        const uint32_t h = idx;
        float dt = p->dt_max;
        while (!mask[idx] && ((~mapping[idx]) & p->is_thinchannel) && n_steps < p->max_n_steps) {
            if (seg_step(&vec, &idx, &dt, &n_steps, uv, p, 1, NULL)) break;
        }
        if (mapping[idx] & p->is_thinchannel) label[h] = label[idx];
    }
    return 0;
}

static inline uint32_t rotate_left(uint32_t px, uint32_t py, int8_t* dx, int8_t* dy, uint32_t nyp) {
    const int8_t rdx = (int8_t)(*dx - *dy), rdy = (int8_t)(*dx + *dy);
    const int adx = rdx < 0 ? -rdx : rdx, ady = rdy < 0 ? -rdy : rdy;
    const int8_t cx = (int8_t)(adx < 1 ? 1 : (adx > 2 ? 2 : adx));
    const int8_t cy = (int8_t)(ady < 1 ? 1 : (ady > 2 ? 2 : ady));
    *dx = (int8_t)(rdx / cx);
    *dy = (int8_t)(rdy / cy);
    return (px + (uint32_t)(int32_t)*dx) * nyp + (py + (uint32_t)(int32_t)*dy);
}

uint32_t oracle_subsegment_channel_edges(const slm_params* p, const float* seeds, uint32_t n,
                                         const uint8_t* mask, const float* uv, uint32_t* mapping,
                                         const uint32_t* channel_label, const uint32_t* link,
                                         uint32_t* label) {
    (void)uv; (void)channel_label;
    uint32_t status = 0;
    const uint32_t nyp = p->ny_padded, nxy = p->nxy_padded;
    for (uint32_t g = 0; g < n; ++g) {
        const v2 vec = seed_at(seeds, g);
        uint32_t prev_idx = pixel_of(vec, p), idx, n_steps = 0;
        idx = link[prev_idx];
        while (prev_idx != idx && n_steps++ < p->max_n_steps) {
            const uint32_t px = prev_idx / nyp, py = prev_idx % nyp;
            const uint32_t x = idx / nyp, y = idx % nyp;
            uint32_t n_turns = 0, left_idx = idx;
            int8_t dx = (int8_t)(uint8_t)((x - px) & 0xffu), dy = (int8_t)(uint8_t)((y - py) & 0xffu);
            int do_left = 1;
            while (left_idx != prev_idx && ++n_turns <= 7u) {
                left_idx = rotate_left(px, py, &dx, &dy, nyp);
                if (left_idx >= nxy) { status |= ST_OOB; continue; }
                if (n_turns >= 2u && !mask[left_idx] && (mapping[left_idx] & p->is_thinchannel)) {
                    if (left_idx == link[idx]) do_left = 0;
                    break;
                }
            }
            if (do_left) {
                n_turns = 0;
                left_idx = idx;
                dx = (int8_t)(uint8_t)((x - px) & 0xffu);
                dy = (int8_t)(uint8_t)((y - py) & 0xffu);
                while (left_idx != prev_idx && ++n_turns <= 4u) {
                    left_idx = rotate_left(px, py, &dx, &dy, nyp);
                    if (left_idx >= nxy) { status |= ST_OOB; continue; }
                    if (n_turns >= 2u && !mask[left_idx]) {
                        if (mapping[left_idx] & p->is_thinchannel) break;
                        mapping[left_idx] |= p->is_leftflank;
                        label[left_idx] |= p->left_flank_addition;
                    }
                }
            }
            prev_idx = idx;
            idx = link[idx];
            if (mask[idx] || (mapping[prev_idx] & p->is_subsegmenthead)) break;
        }
    }
    return status;
}

uint32_t oracle_subsegment_flanks(const slm_params* p, const float* seeds, uint32_t n,
                                  const uint8_t* mask, const float* uv, uint32_t* mapping,
                                  const uint32_t* count, const uint32_t* link, uint32_t* label) {
    (void)count; (void)link;
    for (uint32_t g = 0; g < n; ++g) {
        v2 vec = seed_at(seeds, g);
        uint32_t idx = pixel_of(vec, p), n_steps = 0;
        const uint32_t h = idx;
        float dt = p->dt_max;
        while (!mask[idx] && ((~mapping[idx]) & p->is_leftflank)
               && ((~mapping[idx]) & p->is_thinchannel) && n_steps < p->max_n_steps) {
            if (seg_step(&vec, &idx, &dt, &n_steps, uv, p, 1, NULL)) break;
        }
        if (mapping[idx] & p->is_leftflank) label[h] |= p->left_flank_addition;
    }
    return 0;
}

static uint32_t fix_flanks(const slm_params* p, const float* seeds, uint32_t n,
                           const uint8_t* mask, const float* uv, const uint32_t* mapping,
                           uint32_t* label, int left) {
    const uint32_t lfa = p->left_flank_addition;
    for (uint32_t g = 0; g < n; ++g) {
        v2 vec = seed_at(seeds, g);
        uint32_t idx = pixel_of(vec, p), n_steps = 0;
        const uint32_t h = idx;
        float dt = p->dt_max;
        for (;;) {
            const int flank_ok = left ? (label[idx] & lfa) != 0 : ((~label[idx]) & lfa) != 0;
            if (!(!mask[idx] && flank_ok && ((~mapping[idx]) & p->is_thinchannel)
                  && n_steps < p->max_n_steps))
                break;
            rk_t s = rk_compute(vec, dt, uv, p, &idx);
            if ((label[h] & ~lfa) != (label[idx] & ~lfa)) label[h] = label[idx];
            if (seg_step(&vec, &idx, &dt, &n_steps, uv, p, 0, &s)) break;
        }
        if ((label[h] & ~lfa) != (label[idx] & ~lfa)) label[h] = label[idx];
        if (left) {
            if (((~label[idx]) & lfa) && ((~mapping[idx]) & p->is_thinchannel)) label[h] &= ~lfa;
        } else {
            if (label[idx] & lfa) label[h] |= lfa;
        }
    }
    return 0;
}

uint32_t oracle_fix_right_flanks(const slm_params* p, const float* seeds, uint32_t n,
                                 const uint8_t* mask, const float* uv, uint32_t* mapping,
                                 const uint32_t* count, const uint32_t* link, uint32_t* label) {
    (void)count; (void)link;
    return fix_flanks(p, seeds, n, mask, uv, mapping, label, 0);
}

uint32_t oracle_fix_left_flanks(const slm_params* p, const float* seeds, uint32_t n,
                                const uint8_t* mask, const float* uv, uint32_t* mapping,
                                const uint32_t* count, const uint32_t* link, uint32_t* label) {
    (void)count; (void)link;
    return fix_flanks(p, seeds, n, mask, uv, mapping, label, 1);
}

/* ------------------------------------------------------------- hillslopes */
uint32_t oracle_hillslopes(const slm_params* p, const float* seeds, uint32_t n,
                           const uint8_t* mask, const float* uv, uint32_t* mapping,
                           const uint32_t* count, uint32_t* link) {
    (void)mapping; (void)count;
    for (uint32_t g = 0; g < n; ++g) {
        v2 vec = seed_at(seeds, g);
        uint32_t idx = pixel_of(vec, p), prev_idx = idx, n_steps = 0;
        float dt = p->dt_max;
        while (prev_idx == idx && !mask[idx] && n_steps < 100u * p->max_n_steps) {
            prev_idx = idx;
            rk_t s = rk_compute(vec, dt, uv, p, &idx);
            rkmove_t m = rk_move(&s, &vec, &idx, p);
            if (m.stuck) break;
            dt = next_dt(dt, m.err, p);
            n_steps++;
        }
        if (prev_idx != idx && !mask[idx]) link[prev_idx] = idx;
    }
    return 0;
}

uint32_t oracle_hillslope_lengths(const slm_params* p, const float* seeds, uint32_t n,
                                  const uint8_t* mask, const float* uv, const uint32_t* mapping,
                                  const uint32_t* label, float* traj_length) {
    (void)label;
    const uint32_t from_flag = p->do_measure_hsl_from_ridges ? p->is_ridge : p->is_midslope;
    for (uint32_t g = 0; g < n; ++g) {
        v2 vec = seed_at(seeds, g);
        uint32_t idx = pixel_of(vec, p), n_steps = 0;
        float dt = p->dt_max, l = 0.0f;
        int moved_off = 0, done = 0;
        while (((~mapping[idx]) & p->is_thinchannel) && n_steps < p->max_n_steps) {
            rk_t s = rk_compute(vec, dt, uv, p, &idx);
            if (mask[idx]) { done = 1; break; }
            if (!moved_off && ((~mapping[idx]) & from_flag)) {
                moved_off = 1;
            } else if (moved_off && (mapping[idx] & from_flag)) {
                done = 1;
                break;
            }
            rkmove_t m = rk_move(&s, &vec, &idx, p);
            if (m.stuck) {
                l += m.dl;
                n_steps++;
                done = 1;
                break;
            }
            dt = next_dt(dt, m.err, p);
            l += m.dl;
            n_steps++;
        }
        if (done) continue;
        if (mapping[idx] & p->is_thinchannel) traj_length[g] = l * p->pixel_size;
    }
    return 0;
}

/* Per-item flank walk steps up to the label-independent end, as (compute
 * pixel, moved-to pixel) pairs with consecutive duplicates merged; used by
 * tests to check the dependency-round formulation of fix_*_flanks.  Writes at
 * most cap pairs per item; returns the total number of pairs. */
uint64_t oracle_flank_paths(const slm_params* p, const float* seeds, uint32_t n,
                            const uint8_t* mask, const float* uv, const uint32_t* mapping,
                            uint32_t cap, uint32_t* counts, uint32_t* pairs) {
    uint64_t total = 0;
    for (uint32_t g = 0; g < n; ++g) {
        v2 vec = seed_at(seeds, g);
        uint32_t idx = pixel_of(vec, p), n_steps = 0, k = 0, lq = 0xffffffffu, lr = 0xffffffffu;
        float dt = p->dt_max;
        while (!mask[idx] && ((~mapping[idx]) & p->is_thinchannel) && n_steps < p->max_n_steps) {
            rk_t s = rk_compute(vec, dt, uv, p, &idx);
            const uint32_t q = idx;
            const int stuck = seg_step(&vec, &idx, &dt, &n_steps, uv, p, 0, &s);
            if (q != lq || idx != lr) {
                lq = q; lr = idx;
                if (k < cap) { pairs[2 * ((size_t)g * cap + k)] = q; pairs[2 * ((size_t)g * cap + k) + 1] = idx; }
                k++;
            }
            if (stuck) break;
        }
        counts[g] = k;
        total += k;
    }
    return total;
}
