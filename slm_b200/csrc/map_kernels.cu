// map_kernels.cu -- channel, segment and hillslope mapping kernels.
//
// Each reference mapping kernel (opencl/connect.cl, channelheads.cl,
// countlink.cl, label.cl, segment.cl, hillslopes.cl, lengths.cl) becomes one
// entry point computing the same result as the reference's work-items run one
// after another in ascending global id -- the pinned schedule, since several
// reference kernels race (atomic_xchg last-writer-wins, reads of values other
// work-items write) and have no other defined result.
//
// Order-independent kernels (every cross-item read is of bits the kernel never
// writes, or every write is an idempotent atomic OR/AND) run one thread per
// seed: connect_channels, map_channel_heads, label_confluences, hillslopes,
// segment_hillslopes, subsegment_channel_edges, subsegment_flanks,
// hillslope_lengths.
//
// Order-dependent kernels:
//   count_downchannels  the RK walk from each head is independent of the
//       shared state except for where it stops, so every head's sequence of
//       newly entered pixels is traced in parallel (k_count_paths), then one
//       thread replays the integer updates (count, link, flags) head by head
//       with the reference's early stop (k_count_replay);
//   flag_downchannels, segment_downchannels, prune_channel_heads  link walks
//       and neighbour checks with no RK arithmetic, replayed in seed order by
//       one thread;
//   fix_right_flanks, fix_left_flanks  every work-item writes only its own
//       pixel's label and reads labels along its RK path, so its result depends
//       only on the final labels of lower-index items owning pixels on that
//       path.  One persistent launch (k_flank_resolve) takes items in
//       ascending order and walks each once, waiting for the final label of a
//       lower-index owner it reads.  Fallback (a bounded wait ran out): paths
//       are traced in parallel (k_flank_paths, compressed to the steps whose
//       (compute pixel, moved-to pixel) pair changes), then items are
//       resolved in rounds (k_flank_round): an item resolves once every
//       lower-index owner it reads has resolved in an earlier round.  The
//       lowest unresolved item always can, so both forms end.
//
// Every loop is bounded; a cap that the reference would exceed (it would loop
// on) or a neighbour index outside the grid sets a bit in the caller's status
// word instead of trapping.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <type_traits>
#include <vector>
#include "capi_util.cuh"
#include "trace_common.cuh"

#define MAP_ST_CAP 1u
#define MAP_ST_OOB 2u
#define MAP_LOOP_CAP (1u << 26)
#define CONNECT_REC_MAX 256
#define CNT_PREFETCH 16u
#define NO_OWNER 0xffffffffu
#define FLANK_PERIOD 0x80000000u

namespace slm {

__device__ __forceinline__ Vec2 seed_vec(const float2* __restrict__ seeds, uint32_t g) {
    const float2 s = seeds[g];
    return Vec2{s.x, s.y};
}

struct Move { float err, dl; bool stuck; };

// the shared tail of every *_runge_kutta_step (rungekutta.cl:289-296 ...):
// error, length, first-order fallback when stuck, move to the new point
__device__ __forceinline__ Move rk_move(const Step& s, Vec2& vec, uint32_t& idx, const slm_params& p) {
    Move m;
    m.err = vlen(__fdiv_rn(s.d2.x - s.d1.x, p.grid_scale), __fdiv_rn(s.d2.y - s.d1.y, p.grid_scale));
    Vec2 next = s.next;
    m.dl = vlen(s.d2.x, s.d2.y);
    if (m.dl < p.integration_halt_threshold) {
        next.x = vec.x + s.d1.x;
        next.y = vec.y + s.d1.y;
        m.dl = vlen(s.d1.x, s.d1.y);
    }
    vec = next;
    idx = pixel_of(next, p);
    m.stuck = m.dl < p.integration_halt_threshold;
    return m;
}

__device__ __forceinline__ Step rk_plain(Vec2 a, float dt, const float2* __restrict__ uv,
                                         const slm_params& p) {
    uint32_t rng = 0;
    return rk_step<2, false>(a, dt, rng, uv, p);
}

// Brent's cycle detection on a walk's (vec, dt) state, which determines the
// rest of the walk: true once the state equals the one at the last
// power-of-two checkpoint.  A walk whose loop test held at every state of the
// cycle repeats it until its step bound.
struct StateCycle {
    Vec2 tv;
    float tdt;
    uint32_t power, lam;
    __device__ void init(Vec2 v, float dt) { tv = v; tdt = dt; power = 1; lam = 0; }
    __device__ bool repeated(Vec2 v, float dt) {
        if (__float_as_uint(v.x) == __float_as_uint(tv.x) && __float_as_uint(v.y) == __float_as_uint(tv.y)
            && __float_as_uint(dt) == __float_as_uint(tdt))
            return true;
        if (++lam == power) { tv = v; tdt = dt; power <<= 1; lam = 0; }
        return false;
    }
};

// ------------------------------------------------------------------ connect
__global__ void k_connect_channels(const slm_params p, uint32_t n, const float2* __restrict__ seeds,
                                   const uint8_t* __restrict__ mask, const float2* __restrict__ uv,
                                   uint32_t* mapping, uint32_t* status) {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    int8_t rec[2 * CONNECT_REC_MAX];
    const uint32_t cap_rec = p.interchannel_max_n_steps;
    const float res = (float)p.trajectory_resolution;
    const Vec2 start = seed_vec(seeds, g);
    Vec2 vec = start, prev = start;
    float dt = p.dt_max;
    uint32_t idx = pixel_of(vec, p), prev_idx = idx, n_steps = 0, guard = 0;
    while (prev_idx == idx && !mask[idx] && n_steps != p.max_n_steps) {
        if (++guard > MAP_LOOP_CAP) { atomicOr(status, MAP_ST_CAP); break; }
        const Step s = rk_plain(vec, dt, uv, p);
        idx = s.idx;
        if (!mask[idx]) {
            const Move m = rk_move(s, vec, idx, p);
            if (!m.stuck) dt = next_dt(dt, m.err, p);
            if (n_steps < cap_rec) {
                rec[2 * n_steps] = cvt_i8((vec.x - prev.x) * res);
                rec[2 * n_steps + 1] = cvt_i8((vec.y - prev.y) * res);
            }
            n_steps++;
            if (!m.stuck) prev = vec;
        }
    }
    // The second loop ends at n_steps == INTERCHANNEL_MAX_N_STEPS (every pass
    // that does not exit adds a step).  If the first loop already went past
    // that count, the reference's loop runs until a channel, a masked pixel
    // or the 32-bit wrap of n_steps, writes nothing, and leaves n_steps >=
    // INTERCHANNEL_MAX_N_STEPS, so the flagging below does not run: skipping
    // it gives the same flags, and bounds the kernel.
    guard = 0;
    while (n_steps <= p.interchannel_max_n_steps && (mapping[idx] & p.is_channel) == 0 && !mask[idx]
           && n_steps != p.interchannel_max_n_steps) {
        if (++guard > MAP_LOOP_CAP) { atomicOr(status, MAP_ST_CAP); break; }
        const Step s = rk_plain(vec, dt, uv, p);
        idx = s.idx;
        if (!mask[idx]) {
            const Move m = rk_move(s, vec, idx, p);
            if (!m.stuck) dt = next_dt(dt, m.err, p);
            if (n_steps < cap_rec) {
                rec[2 * n_steps] = cvt_i8((vec.x - prev.x) * res);
                rec[2 * n_steps + 1] = cvt_i8((vec.y - prev.y) * res);
            }
            n_steps++;
            if (!m.stuck) prev = vec;
        }
    }
    if (n_steps > 2 && n_steps < p.interchannel_max_n_steps) {
        vec = start;
        idx = pixel_of(vec, p);
        uint32_t step = 0;
        while (!mask[idx] && step < n_steps - 1) {
            if (*(volatile uint32_t*)(mapping + idx) == 0u) atomicOr(mapping + idx, p.is_interchannel);
            vec.x = vec.x + __fdiv_rn((float)rec[2 * step], res);
            vec.y = vec.y + __fdiv_rn((float)rec[2 * step + 1], res);
            idx = pixel_of(vec, p);
            step++;
        }
    }
}

// ------------------------------------------------------------------ channel heads
__global__ void k_map_channel_heads(const slm_params p, uint32_t n, const float2* __restrict__ seeds,
                                    const uint8_t* __restrict__ mask, const float2* __restrict__ uv,
                                    uint32_t* mapping) {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    Vec2 vec = seed_vec(seeds, g);
    float dt = p.dt_max;
    uint32_t idx = pixel_of(vec, p), prev_idx = idx, n_steps = 0;
    // Every state the loop continues from lies in the start pixel, and
    // (vec, dt) determines the rest of the walk: once that state repeats
    // (Brent) the walk circles inside the pixel until the step bound, where
    // it returns without a change.  Walks stuck on flats and in pits end here
    // instead of running max_n_steps steps.
    StateCycle cyc;
    cyc.init(vec, dt);
    while (prev_idx == idx && !mask[idx] && n_steps < p.max_n_steps) {
        const Step s = rk_plain(vec, dt, uv, p);
        idx = s.idx;
        const Move m = rk_move(s, vec, idx, p);
        n_steps++;
        dt = next_dt(dt, m.err, p);
        if (prev_idx == idx && cyc.repeated(vec, dt)) return;
    }
    if (n_steps >= p.max_n_steps) return;
    if (!mask[idx]) {
        idx = pixel_of(vec, p);
        const uint32_t here = *(volatile uint32_t*)(mapping + idx);
        const uint32_t before = *(volatile uint32_t*)(mapping + prev_idx);
        if (((~here) & p.is_thinchannel) || (before & p.is_thinchannel))
            atomicAnd(mapping + idx, ~p.is_channelhead);
    }
}

// neighbour offsets in the reference's check order N, S, E, W, NE, SE, NW, SW
__constant__ float c_nbr[8][2] = {{0, 1}, {0, -1}, {1, 0}, {-1, 0}, {1, 1}, {1, -1}, {-1, 1}, {-1, -1}};

// One head of prune_channel_heads (channelheads.cl:143-199): count the thin
// channel pixels among the 8 neighbours; not exactly one clears the head's
// IS_CHANNELHEAD, none also its IS_THINCHANNEL | IS_CHANNEL.
__device__ __forceinline__ void prune_head(uint32_t g, const slm_params& p, const float2* __restrict__ seeds,
                                           uint32_t* mapping) {
    const Vec2 vec = seed_vec(seeds, g);
    uint32_t flag = 0;
    for (int k = 0; k < 8; ++k) {
        const Vec2 nb{vec.x + c_nbr[k][0], vec.y + c_nbr[k][1]};
        flag += (*(volatile uint32_t*)(mapping + pixel_of(nb, p)) & p.is_thinchannel) != 0u;
    }
    if (flag != 1u) {
        const uint32_t idx = pixel_of(vec, p);
        atomicAnd(mapping + idx, ~p.is_channelhead);
        if (flag == 0u) atomicAnd(mapping + idx, ~(p.is_thinchannel | p.is_channel));
    }
}

// prune_channel_heads with the result of the reference's sequential schedule
// (ascending global id).  A head reads its neighbours' IS_THINCHANNEL bits
// and changes bits of its own pixel only.  When every head is itself a thin
// channel pixel -- as the mapping sequence leaves them -- no count can change
// while the heads run: a head that clears its thin bit has no thin
// neighbour, so no head is its neighbour.  The heads then run in parallel.
// Otherwise a head that is not thin may count an isolated thin head that
// runs before it, and the heads run one after another.  One block decides
// and runs either case, so no scratch word is needed.
__global__ void __launch_bounds__(1024) k_prune_channel_heads(const slm_params p, uint32_t n,
                                                              const float2* __restrict__ seeds,
                                                              uint32_t* mapping) {
    int all_thin = 1;
    for (uint32_t g = threadIdx.x; g < n; g += blockDim.x)
        if ((mapping[pixel_of(seed_vec(seeds, g), p)] & p.is_thinchannel) == 0u) all_thin = 0;
    all_thin = __syncthreads_and(all_thin);
    if (all_thin) {
        for (uint32_t g = threadIdx.x; g < n; g += blockDim.x) prune_head(g, p, seeds, mapping);
    } else if (threadIdx.x == 0) {
        for (uint32_t g = 0; g < n; ++g) prune_head(g, p, seeds, mapping);
    }
}

// ------------------------------------------------------------------ count / flag
// Phase A of count_downchannels: the pixels each head's walk enters, in order,
// up to the walk's state-independent end; with events == nullptr only counts.
// Event stream of one count_downchannels walk: the pixels it enters, in
// order.  Walks that oscillate (e.g. across a valley floor) run to the
// 1000*MAX_N_STEPS bound and enter millions of pixels in a short repeating
// pattern, so the stream is compressed losslessly: literal events are pixel
// indices (< 2^31); a repeat record (two words: 0x80000000|P, n) stands for
// the next n events continuing the pattern of the last P decoded events.
constexpr uint32_t CNT_PMAX = 8;
constexpr uint32_t CNT_REPEAT = 0x80000000u;
// A period record (words 0xC0000000|E, the E pattern pixels, n) stands for the
// walk's remaining n events: the E-event pattern repeated (last lap partial).
constexpr uint32_t CNT_PERIOD = 0xC0000000u;
constexpr uint32_t CNT_KIND = 0xC0000000u;

struct EventWriter {
    uint32_t* out;  // null: count words only
    u64 k;          // words written
    uint32_t ring[2 * CNT_PMAX];
    uint32_t nlit;  // literals in the ring (capped at 2*CNT_PMAX)
    uint32_t P, pos;
    uint32_t pat[CNT_PMAX];
    uint32_t reps;  // events matched by the open repeat record
    __device__ void put(uint32_t w) {
        if (out) out[k] = w;
        k++;
    }
    __device__ void close_repeat() {
        if (P && reps) {
            put(CNT_REPEAT | P);
            put(reps);
        }
        P = 0;
        reps = 0;
        nlit = 0;
    }
    __device__ void literal(uint32_t e) {
        put(e);
        if (nlit == 2 * CNT_PMAX) {
#pragma unroll
            for (uint32_t q = 0; q + 1 < 2 * CNT_PMAX; ++q) ring[q] = ring[q + 1];
            ring[2 * CNT_PMAX - 1] = e;
        } else {
            ring[nlit++] = e;
        }
        // the literal tail periodic over two periods -> open a repeat record
        for (uint32_t q = 1; q <= CNT_PMAX && 2 * q <= nlit; ++q) {
            bool same = true;
            for (uint32_t t = 0; t < q && same; ++t) same = ring[nlit - 1 - t] == ring[nlit - 1 - q - t];
            if (same) {
                P = q;
                pos = 0;
                reps = 0;
                for (uint32_t t = 0; t < q; ++t) pat[t] = ring[nlit - q + t];
                return;
            }
        }
    }
    __device__ void event(uint32_t e) {
        if (P) {
            if (e == pat[pos]) {
                reps++;
                pos = pos + 1 == P ? 0 : pos + 1;
                return;
            }
            close_repeat();
        }
        literal(e);
    }
};

__global__ void k_count_paths(const slm_params p, uint32_t n, const float2* __restrict__ seeds,
                              const uint8_t* __restrict__ mask, const float2* __restrict__ uv,
                              u64* __restrict__ n_events, const u64* __restrict__ offsets,
                              uint32_t* __restrict__ events, uint32_t* __restrict__ tail_idx) {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    Vec2 vec = seed_vec(seeds, g);
    float dt = p.dt_max;
    uint32_t idx = pixel_of(vec, p), prev_idx = idx, n_steps = 0;
    const uint32_t lim = 1000u * p.max_n_steps;
    EventWriter w;
    w.out = events ? events + offsets[g] : nullptr;
    w.k = 0;
    w.nlit = 0;
    w.P = 0;
    w.reps = 0;
    // The walk's dynamics depend only on (vec, dt): once that state repeats
    // bit for bit (Brent's cycle detection), every later step repeats the
    // period, up to the 1000*MAX_N_STEPS bound.  The period is then walked
    // again from the repeated state -- once to count its events and find the
    // pixel the walk ends on, once to write them -- and the remaining events
    // go out as one period record instead of being traced.
    Vec2 tv = vec;
    float tdt = dt;
    uint32_t power = 1, lam = 0;
    while (!mask[idx] && n_steps < lim) {
        const Step s = rk_plain(vec, dt, uv, p);
        idx = s.idx;
        const Move m = rk_move(s, vec, idx, p);
        if (m.stuck) break;
        dt = next_dt(dt, m.err, p);
        n_steps++;
        if (prev_idx != idx) {
            w.event(idx);
            prev_idx = idx;
        }
        lam++;
        if (__float_as_uint(vec.x) == __float_as_uint(tv.x) && __float_as_uint(vec.y) == __float_as_uint(tv.y)
            && __float_as_uint(dt) == __float_as_uint(tdt)) {
            const uint32_t L = lam, R = lim - n_steps, Rm = R % L;
            uint32_t E = 0, partial = 0, end_idx = idx;
            for (int pass = 0; pass < 2; ++pass) {
                Vec2 v2 = vec;
                float d2 = dt;
                uint32_t i2 = idx, prev2 = idx;
                if (pass == 1) {
                    const uint32_t nfut = (R / L) * E + partial;
                    if (nfut == 0) break;
                    w.close_repeat();
                    w.put(CNT_PERIOD | E);
                    E = nfut;  // written after the pattern
                }
                for (uint32_t t = 1; t <= L; ++t) {
                    const Step s2 = rk_plain(v2, d2, uv, p);
                    i2 = s2.idx;
                    const Move m2 = rk_move(s2, v2, i2, p);
                    d2 = next_dt(d2, m2.err, p);
                    if (prev2 != i2) {
                        if (pass == 0) {
                            E++;
                            if (t <= Rm) partial++;
                        } else {
                            w.put(i2);
                        }
                        prev2 = i2;
                    }
                    if (pass == 0 && t == Rm) end_idx = i2;
                }
                if (pass == 1) w.put(E);
            }
            idx = end_idx;  // the pixel after the walk's last step
            break;
        }
        if (lam == power) {
            tv = vec;
            tdt = dt;
            power <<= 1;
            lam = 0;
        }
    }
    w.close_repeat();
    if (events) tail_idx[g] = idx;
    else n_events[g] = w.k;
}

// The reference's per-event update of count_downchannels (countlink.cl:
// 104-118); false = the walk stops (it joined a longer path)
__device__ __forceinline__ bool count_event(const slm_params& p, uint32_t e, uint32_t& counter,
                                            uint32_t& prev, uint32_t* mapping, uint32_t* count,
                                            uint32_t* link) {
    mapping[e] &= ~p.is_channelhead;
    mapping[e] |= p.is_thinchannel;
    link[prev] = e;
    if (++counter < count[e]) return false;
    count[e] = counter;
    prev = e;
    return true;
}

// One thread replays the walks head by head (the pinned sequential order).
// A repeat record is replayed event by event for its first lap; after a lap
// every pattern pixel holds a count this walk wrote at most one lap ago,
// below the running counter, so no later event can stop the walk.  The laps
// in between only rewrite the same links, flags and growing counts, so they
// are skipped and the final lap is replayed with its own counter values.
__global__ void k_count_replay(const slm_params p, uint32_t n, const float2* __restrict__ seeds,
                               const u64* __restrict__ offsets, const uint32_t* __restrict__ events,
                               const uint32_t* __restrict__ tail_idx, uint32_t* mapping,
                               uint32_t* count, uint32_t* link) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    uint32_t last8[CNT_PMAX];
    for (uint32_t g = 0; g < n; ++g) {
        const uint32_t head = pixel_of(seed_vec(seeds, g), p);
        uint32_t counter = 1, prev = head, last = tail_idx[g];
        uint32_t nd = 0;  // decoded events (for the pattern ring)
        count[head] = counter++;
        bool stopped = false;
        const u64 k_end = offsets[g + 1];
        for (u64 k = offsets[g]; k < k_end && !stopped; ++k) {
            const uint32_t wd = events[k];
            // one thread walks the events: bring the pixels of the event
            // CNT_PREFETCH ahead into L2 so their loads do not wait on DRAM
            if (k + CNT_PREFETCH < k_end) {
                const uint32_t ahead = events[k + CNT_PREFETCH];
                if (ahead < p.nxy_padded) {  // a pixel, or a count word that is still in the grid
                    asm volatile("prefetch.global.L2 [%0];" ::"l"(count + ahead));
                    asm volatile("prefetch.global.L2 [%0];" ::"l"(mapping + ahead));
                    asm volatile("prefetch.global.L2 [%0];" ::"l"(link + ahead));
                }
            }
            if ((wd & CNT_REPEAT) == 0u) {
                if (!count_event(p, wd, counter, prev, mapping, count, link)) { last = wd; stopped = true; break; }
                last8[nd % CNT_PMAX] = wd;
                nd++;
                continue;
            }
            uint32_t pat_ring[CNT_PMAX];
            const uint32_t* pat;
            uint32_t P, reps;
            if ((wd & CNT_KIND) == CNT_PERIOD) {
                P = wd & ~CNT_KIND;
                pat = events + k + 1;
                k += P;
                reps = events[++k];
            } else {
                P = wd & ~CNT_REPEAT;
                reps = events[++k];
                for (uint32_t t = 0; t < P; ++t) pat_ring[t] = last8[(nd - P + t) % CNT_PMAX];
                pat = pat_ring;
            }
            const uint32_t lap = reps < P ? reps : P;
            for (uint32_t t = 0; t < lap; ++t) {
                const uint32_t e = pat[t];
                if (!count_event(p, e, counter, prev, mapping, count, link)) { last = e; stopped = true; break; }
                last8[nd % CNT_PMAX] = e;
                nd++;
            }
            if (stopped) break;
            const uint32_t r = reps - lap;  // events after the first lap, from pattern position 0
            if (r > 0) {
                // skip to the final lap (events start..r-1) and replay it in order:
                // every pattern pixel's last link and count assignments fall in
                // it; flags were set by the first lap
                const uint32_t c0 = counter;
                const uint32_t start = r > P ? r - P : 0u;
                prev = pat[(start + P - 1) % P];
                for (uint32_t i = start; i < r; ++i) {
                    const uint32_t e = pat[i % P];
                    link[prev] = e;
                    count[e] = c0 + 1 + i;
                    prev = e;
                    last8[nd % CNT_PMAX] = e;
                    nd++;
                }
                counter = c0 + r;
            }
        }
        link[prev] = last;
    }
}


// The same replay with one warp: runs of plain events (up to 32) are
// decided together.  Event i of a run takes counter c + i + 1; the count it
// compares with is the one an earlier event of the run wrote to the same
// pixel (c + j + 1, always lower) or else the count loaded before the run,
// so the first stopping event is a ballot.  Flags (an idempotent update),
// links (the last writer per pixel wins: the highest lane of a match group
// writes) and counts are then written in parallel, in the order the single
// thread would leave them.  Repeat records are replayed by lane 0 as above.
// __syncwarp orders each run's writes before the next run's loads.
__global__ void __launch_bounds__(32) k_count_replay_warp(const slm_params p, uint32_t n,
                                                          const float2* __restrict__ seeds,
                                                          const u64* __restrict__ offsets,
                                                          const uint32_t* __restrict__ events,
                                                          const uint32_t* __restrict__ tail_idx, uint32_t* mapping,
                                                          uint32_t* count, uint32_t* link) {
    if (blockIdx.x != 0) return;
    const unsigned FULL = 0xffffffffu;
    const unsigned lane = threadIdx.x;
    const uint32_t dummy = 0xFFFFFFE0u + lane;  // matches no pixel (nxy_padded < 2^32 - 32)
    __shared__ uint32_t ring[CNT_PMAX];
    for (uint32_t g = 0; g < n; ++g) {
        const uint32_t head = pixel_of(seed_vec(seeds, g), p);
        uint32_t counter = 1, prev = head, last = tail_idx[g], nd = 0;
        if (lane == 0) count[head] = counter;
        counter++;
        bool stopped = false;
        u64 k = offsets[g];
        const u64 k_end = offsets[g + 1];
        __syncwarp();
        while (k < k_end && !stopped) {
            const uint32_t wd0 = events[k];
            if (wd0 & CNT_REPEAT) {
                // a repeat record, by lane 0 as the single-thread replay does
                if (lane == 0) {
                    uint32_t pat_ring[CNT_PMAX];
                    const uint32_t* pat;
                    uint32_t P, reps;
                    if ((wd0 & CNT_KIND) == CNT_PERIOD) {
                        P = wd0 & ~CNT_KIND;
                        pat = events + k + 1;
                        k += P;
                        reps = events[++k];
                    } else {
                        P = wd0 & ~CNT_REPEAT;
                        reps = events[++k];
                        for (uint32_t t = 0; t < P; ++t) pat_ring[t] = ring[(nd - P + t) % CNT_PMAX];
                        pat = pat_ring;
                    }
                    ++k;
                    const uint32_t lap = reps < P ? reps : P;
                    for (uint32_t t = 0; t < lap; ++t) {
                        const uint32_t e = pat[t];
                        if (!count_event(p, e, counter, prev, mapping, count, link)) {
                            last = e;
                            stopped = true;
                            break;
                        }
                        ring[nd % CNT_PMAX] = e;
                        nd++;
                    }
                    const uint32_t r = reps - lap;
                    if (!stopped && r > 0) {
                        const uint32_t c0 = counter;
                        const uint32_t start = r > P ? r - P : 0u;
                        prev = pat[(start + P - 1) % P];
                        for (uint32_t i = start; i < r; ++i) {
                            const uint32_t e = pat[i % P];
                            link[prev] = e;
                            count[e] = c0 + 1 + i;
                            prev = e;
                            ring[nd % CNT_PMAX] = e;
                            nd++;
                        }
                        counter = c0 + r;
                    }
                }
                counter = __shfl_sync(FULL, counter, 0);
                prev = __shfl_sync(FULL, prev, 0);
                last = __shfl_sync(FULL, last, 0);
                nd = __shfl_sync(FULL, nd, 0);
                k = __shfl_sync(FULL, k, 0);
                stopped = __shfl_sync(FULL, stopped ? 1 : 0, 0) != 0;
                __syncwarp();
                continue;
            }
            // a run of plain events: the prefix of events[k ..] up to a record
            uint32_t e = dummy;
            bool plain = false;
            if (k + lane < k_end) {
                const uint32_t w = events[k + lane];
                plain = (w & CNT_REPEAT) == 0u;
                if (plain) e = w;
            }
            const unsigned pm = __ballot_sync(FULL, plain);
            const uint32_t m = (~pm == 0u) ? 32u : (uint32_t)(__ffs(~pm) - 1);
            const bool in = lane < m;
            if (!in) e = dummy;
            const uint32_t c_loaded = in ? count[e] : 0u;
            const unsigned same = __match_any_sync(FULL, e);
            const unsigned earlier = same & ((1u << lane) - 1u);
            const uint32_t mine = counter + lane + 1u;
            const uint32_t seen = earlier ? counter + (uint32_t)(31 - __clz(earlier)) + 1u : c_loaded;
            const unsigned stops = __ballot_sync(FULL, in && mine < seen);
            const uint32_t s_at = stops ? (uint32_t)(__ffs(stops) - 1) : m;
            const uint32_t n_proc = stops ? s_at + 1u : m;  // flags and links
            const uint32_t n_pass = s_at;                   // counts, prev, ring
            uint32_t prev_i = __shfl_up_sync(FULL, e, 1);
            if (lane == 0) prev_i = prev;
            if (lane < n_proc) mapping[e] = (mapping[e] & ~p.is_channelhead) | p.is_thinchannel;
            const unsigned lm = __match_any_sync(FULL, lane < n_proc ? prev_i : dummy);
            if (lane < n_proc && (uint32_t)(31 - __clz(lm)) == lane) link[prev_i] = e;
            const unsigned cm = __match_any_sync(FULL, lane < n_pass ? e : dummy);
            if (lane < n_pass && (uint32_t)(31 - __clz(cm)) == lane) count[e] = mine;
            if (lane < n_pass && lane + CNT_PMAX >= n_pass) ring[(nd + lane) % CNT_PMAX] = e;
            const uint32_t e_last_pass = __shfl_sync(FULL, e, n_pass > 0 ? n_pass - 1 : 0);
            if (n_pass > 0) prev = e_last_pass;
            nd += n_pass;
            counter += n_pass;
            if (stops) {
                last = __shfl_sync(FULL, e, s_at);
                stopped = true;
            }
            k += n_proc;
            __syncwarp();
        }
        if (lane == 0) link[prev] = last;
        __syncwarp();
    }
}

// ------------------------------------------------------------------ label
__global__ void k_label_confluences(const slm_params p, uint32_t n, const float2* __restrict__ seeds,
                                    const uint8_t* __restrict__ mask, const float* __restrict__ slt,
                                    uint32_t* mapping, const uint32_t* __restrict__ count,
                                    const uint32_t* __restrict__ link) {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    const Vec2 vec = seed_vec(seeds, g);
    const uint32_t idx = pixel_of(vec, p);
    uint32_t inflows[8], equal_dom[8], n_in = 0, n_eq = 0, dom_idx = 0;
    float dom_slt = -3.40282347e+38f;
    for (int k = 0; k < 8; ++k) {
        const Vec2 nb{vec.x + c_nbr[k][0], vec.y + c_nbr[k][1]};
        const uint32_t ni = pixel_of(nb, p);
        if (!mask[ni] && (*(volatile uint32_t*)(mapping + ni) & p.is_thinchannel) && link[ni] == idx)
            inflows[n_in++] = ni;
    }
    if (n_in > 1) {
        atomicOr(mapping + idx, p.is_majorconfluence);
        for (uint32_t i = 0; i < n_in; ++i) {
            if (count[idx] != count[inflows[i]] + 1u) {
                atomicOr(mapping + inflows[i], p.is_minorinflow);
            } else {
                equal_dom[n_eq++] = inflows[i];
                if (slt[inflows[i]] > dom_slt) {
                    dom_idx = inflows[i];
                    dom_slt = slt[dom_idx];
                }
            }
        }
        for (uint32_t i = 0; i < n_eq; ++i)
            atomicOr(mapping + equal_dom[i], equal_dom[i] == dom_idx ? p.is_majorinflow : p.is_minorinflow);
    }
}

// ------------------------------------------------------------------ segments
__global__ void k_segment_downchannels(const slm_params p, uint32_t n, const float2* __restrict__ seeds,
                                       const uint8_t* __restrict__ mask, uint32_t* mapping,
                                       const uint32_t* __restrict__ count,
                                       const uint32_t* __restrict__ link, uint32_t* label,
                                       uint32_t* status) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    for (uint32_t g = 0; g < n; ++g) {
        uint32_t prev_idx = pixel_of(seed_vec(seeds, g), p), seg_counter = 0;
        uint32_t seg_label = prev_idx;
        label[prev_idx] = seg_label;
        mapping[prev_idx] |= p.is_subsegmenthead;
        uint32_t idx = link[prev_idx], guard = 0;
        while (!mask[idx] && prev_idx != idx && (mapping[idx] & p.is_subsegmenthead) == 0u) {
            if (++guard > MAP_LOOP_CAP) { *status |= MAP_ST_CAP; break; }
            if (count[idx] >= seg_counter + p.segmentation_threshold / 2u) {
                seg_label = idx;
                seg_counter = count[idx] + p.segmentation_threshold;
                mapping[idx] |= p.is_subsegmenthead;
            }
            label[idx] = seg_label;
            prev_idx = idx;
            idx = link[idx];
        }
    }
}

// segment_runge_kutta_step (rungekutta.cl:435-459): n_steps++ always, stuck ends
__device__ __forceinline__ bool seg_move(const Step& s, Vec2& vec, uint32_t& idx, float& dt,
                                         uint32_t& n_steps, const slm_params& p) {
    const Move m = rk_move(s, vec, idx, p);
    n_steps++;
    if (m.stuck) return true;
    dt = next_dt(dt, m.err, p);
    return false;
}

// Per-pixel walks with warp-local refill: warp w owns items
// [w * WALK_PER_WARP, (w + 1) * WALK_PER_WARP); a lane whose walk ends takes
// the warp's next item at once (a ballot, no global counter), so a warp's
// lanes stay busy however uneven their walks are.  Each item's walk is the
// one-thread-per-item walk, so results are unchanged.
constexpr uint32_t WALK_PER_WARP = 256;

template <class W>
__global__ void __launch_bounds__(256) k_walks(W w, uint32_t n) {
    const unsigned FULL = 0xffffffffu;
    const unsigned lane = threadIdx.x & 31u;
    const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t lo = warp * WALK_PER_WARP;
    const uint64_t hi = lo + WALK_PER_WARP < n ? lo + WALK_PER_WARP : n;
    uint64_t next = lo;
    bool alive = false;
    while (true) {
        const unsigned idle = __ballot_sync(FULL, !alive);
        if (idle && next < hi) {
            const uint64_t mine = next + __popc(idle & ((1u << lane) - 1u));
            next += __popc(idle);
            if (!alive && mine < hi) alive = w.start((uint32_t)mine);
        }
        if (!__any_sync(FULL, alive)) {
            if (next >= hi) break;
            continue;
        }
        if (alive) alive = w.step();
    }
}

static unsigned walk_grid(uint32_t n) {
    const uint64_t warps = ((uint64_t)n + WALK_PER_WARP - 1) / WALK_PER_WARP;
    return (unsigned)((warps + 7) / 8);  // 8 warps per block of 256
}

// segment_hillslopes (segment.cl): from each hillslope pixel down to a thin
// channel, whose label it takes
struct SegHillWalk {
    slm_params p;
    const float2* seeds;
    const uint8_t* mask;
    const float2* uv;
    const uint32_t* mapping;
    uint32_t* label;
    Vec2 vec;
    float dt;
    uint32_t idx, h, n_steps;
    StateCycle cyc;
    __device__ bool start(uint32_t g) {
        vec = seed_vec(seeds, g);
        idx = pixel_of(vec, p);
        h = idx;
        n_steps = 0;
        dt = p.dt_max;
        cyc.init(vec, dt);
        return step_test();
    }
    // the loop test; false ends the walk (and writes its label)
    __device__ bool step_test() {
        if (!mask[idx] && ((~mapping[idx]) & p.is_thinchannel) && n_steps < p.max_n_steps) return true;
        finish();
        return false;
    }
    __device__ void finish() {
        if (mapping[idx] & p.is_thinchannel) label[h] = label[idx];
    }
    __device__ bool step() {
        const Step s = rk_plain(vec, dt, uv, p);
        idx = s.idx;
        if (seg_move(s, vec, idx, dt, n_steps, p)) {
            finish();
            return false;
        }
        // a cycle of states that all continue the loop ends at the bound on a
        // pixel that is not a thin channel: no label
        if (cyc.repeated(vec, dt)) return false;
        return step_test();
    }
};

__device__ __forceinline__ uint32_t rotate_left(uint32_t px, uint32_t py, int8_t& dx, int8_t& dy,
                                                uint32_t nyp) {
    const int8_t rdx = (int8_t)(dx - dy), rdy = (int8_t)(dx + dy);
    const int adx = rdx < 0 ? -rdx : rdx, ady = rdy < 0 ? -rdy : rdy;
    const int8_t cx = (int8_t)(adx < 1 ? 1 : (adx > 2 ? 2 : adx));
    const int8_t cy = (int8_t)(ady < 1 ? 1 : (ady > 2 ? 2 : ady));
    dx = (int8_t)(rdx / cx);
    dy = (int8_t)(rdy / cy);
    return (px + (uint32_t)(int32_t)dx) * nyp + (py + (uint32_t)(int32_t)dy);
}

__global__ void k_subsegment_channel_edges(const slm_params p, uint32_t n,
                                           const float2* __restrict__ seeds,
                                           const uint8_t* __restrict__ mask, uint32_t* mapping,
                                           const uint32_t* __restrict__ link, uint32_t* label,
                                           uint32_t* status) {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    const uint32_t nyp = p.ny_padded, nxy = p.nxy_padded;
    uint32_t prev_idx = pixel_of(seed_vec(seeds, g), p), n_steps = 0;
    uint32_t idx = link[prev_idx];
    while (prev_idx != idx && n_steps++ < p.max_n_steps) {
        if (idx >= nxy) { atomicOr(status, MAP_ST_OOB); break; }
        const uint32_t px = prev_idx / nyp, py = prev_idx % nyp;
        const uint32_t x = idx / nyp, y = idx % nyp;
        uint32_t n_turns = 0, left_idx = idx;
        int8_t dx = (int8_t)(uint8_t)((x - px) & 0xffu), dy = (int8_t)(uint8_t)((y - py) & 0xffu);
        bool do_left = true;
        while (left_idx != prev_idx && ++n_turns <= 7u) {
            left_idx = rotate_left(px, py, dx, dy, nyp);
            if (left_idx >= nxy) { atomicOr(status, MAP_ST_OOB); continue; }
            // THINCHANNEL bits are never written by this kernel
            if (n_turns >= 2u && !mask[left_idx] && (*(volatile uint32_t*)(mapping + left_idx) & p.is_thinchannel)) {
                if (left_idx == link[idx]) do_left = false;
                break;
            }
        }
        if (do_left) {
            n_turns = 0;
            left_idx = idx;
            dx = (int8_t)(uint8_t)((x - px) & 0xffu);
            dy = (int8_t)(uint8_t)((y - py) & 0xffu);
            while (left_idx != prev_idx && ++n_turns <= 4u) {
                left_idx = rotate_left(px, py, dx, dy, nyp);
                if (left_idx >= nxy) { atomicOr(status, MAP_ST_OOB); continue; }
                if (n_turns >= 2u && !mask[left_idx]) {
                    if (*(volatile uint32_t*)(mapping + left_idx) & p.is_thinchannel) break;
                    atomicOr(mapping + left_idx, p.is_leftflank);
                    atomicOr(label + left_idx, p.left_flank_addition);
                }
            }
        }
        prev_idx = idx;
        idx = link[idx];
        if (idx >= nxy) { atomicOr(status, MAP_ST_OOB); break; }
        if (mask[idx] || (*(volatile uint32_t*)(mapping + prev_idx) & p.is_subsegmenthead)) break;
    }
}

// subsegment_flanks (segment.cl:360-414): from each pixel down to a left
// flank or thin channel; the left-flank bit when a left flank is reached
struct SubsegFlankWalk {
    slm_params p;
    const float2* seeds;
    const uint8_t* mask;
    const float2* uv;
    const uint32_t* mapping;
    uint32_t* label;
    Vec2 vec;
    float dt;
    uint32_t idx, h, n_steps;
    StateCycle cyc;
    __device__ bool start(uint32_t g) {
        vec = seed_vec(seeds, g);
        idx = pixel_of(vec, p);
        h = idx;
        n_steps = 0;
        dt = p.dt_max;
        cyc.init(vec, dt);
        return step_test();
    }
    __device__ bool step_test() {
        if (!mask[idx] && ((~mapping[idx]) & p.is_leftflank) && ((~mapping[idx]) & p.is_thinchannel)
            && n_steps < p.max_n_steps)
            return true;
        finish();
        return false;
    }
    __device__ void finish() {
        if (mapping[idx] & p.is_leftflank) label[h] |= p.left_flank_addition;
    }
    __device__ bool step() {
        const Step s = rk_plain(vec, dt, uv, p);
        idx = s.idx;
        if (seg_move(s, vec, idx, dt, n_steps, p)) {
            finish();
            return false;
        }
        // a cycle of states that all continue the loop ends at the bound on a
        // pixel that is not left flank: no flank bit
        if (cyc.repeated(vec, dt)) return false;
        return step_test();
    }
};

// ------------------------------------------------------------------ fix flanks
__global__ void k_owner_map(const slm_params p, uint32_t n, const float2* __restrict__ seeds,
                            uint32_t* __restrict__ owner, uint32_t* __restrict__ hpix) {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    const uint32_t h = pixel_of(seed_vec(seeds, g), p);
    hpix[g] = h;
    owner[h] = g;
}

// Stored flank paths: linked blocks of FLANK_BLOCK entries, FLANK_BLOCK - 1
// pairs and the index of the next block.
constexpr uint32_t FLANK_BLOCK = 32;
constexpr uint32_t NO_BLOCK = 0xffffffffu;

// A block index for each calling lane of the warp (one atomic per call site
// and warp); NO_BLOCK when the pool of cap blocks is used up.
__device__ __forceinline__ uint32_t take_block(uint32_t* taken, uint32_t cap) {
    const unsigned m = __activemask();
    const unsigned lane = threadIdx.x & 31u;
    const int leader = __ffs(m) - 1;
    uint32_t b = 0;
    if ((int)lane == leader) b = atomicAdd(taken, (uint32_t)__popc(m));
    b = __shfl_sync(m, b, leader) + __popc(m & ((1u << lane) - 1u));
    return b < cap ? b : NO_BLOCK;
}

// Where a flank walk's pairs go: counted only (out == NULL), a contiguous
// range, or linked blocks taken from a pool as needed (counting goes on
// after the pool runs out; *overflow is then set).
struct ContigSink {
    uint2* out;
    u64 k;
    __device__ void put(uint2 e) {
        if (out) out[k] = e;
        ++k;
    }
};

struct LinkedSink {
    uint2* pool;
    uint32_t* taken;
    uint32_t* overflow;
    uint32_t cap, cur, f;
    uint32_t* head;
    u64 k;
    bool ok;
    __device__ void put(uint2 e) {
        ++k;
        if (!ok) return;
        if (cur == NO_BLOCK || f == FLANK_BLOCK - 1) {
            const uint32_t b = take_block(taken, cap);
            if (b == NO_BLOCK) {
                ok = false;
                atomicOr(overflow, 1u);
                return;
            }
            if (cur == NO_BLOCK) *head = b;
            else pool[(u64)cur * FLANK_BLOCK + (FLANK_BLOCK - 1)] = make_uint2(b, 0u);
            cur = b;
            f = 0;
        }
        pool[(u64)cur * FLANK_BLOCK + f++] = e;
    }
};

// Steps of a flank walk up to its label-independent end (mask, thin channel,
// step cap, stuck), as (compute pixel, moved-to pixel) pairs; consecutive
// equal pairs are stored once.  With pairs == nullptr only counts.
// Items g0 .. g0+n-1; paths are stored at pairs[offsets[g] - base] (a chunk
// of the item range at a time, so the stored paths fit the workspace).
// The walk of item g into `sink`; returns its pair count.
template <class Sink>
__device__ u64 flank_walk(const slm_params& p, uint32_t g, const float2* __restrict__ seeds,
                          const uint8_t* __restrict__ stop, const float2* __restrict__ uv, Sink& sink) {
    Vec2 vec = seed_vec(seeds, g);
    uint32_t idx = pixel_of(vec, p), n_steps = 0;
    float dt = p.dt_max;
    uint2 last = make_uint2(NO_OWNER, NO_OWNER);
    // As in count_downchannels: once (vec, dt) repeats bit for bit the
    // per-step pairs repeat with the period, so the rest of the walk is
    // stored as one period record {0x80000000|E, n} + the E pairs of a lap
    // (after every step `last` is that step's pair, so each lap merges alike).
    Vec2 tv = vec;
    float tdt = dt;
    uint32_t power = 1, lam = 0;
    while (!stop[idx] && n_steps < p.max_n_steps) {
        const Step s = rk_plain(vec, dt, uv, p);
        const uint32_t q = s.idx;
        idx = q;
        const bool stuck = seg_move(s, vec, idx, dt, n_steps, p);
        if (q != last.x || idx != last.y) {
            last = make_uint2(q, idx);
            sink.put(last);
        }
        if (stuck) break;
        lam++;
        if (__float_as_uint(vec.x) == __float_as_uint(tv.x) && __float_as_uint(vec.y) == __float_as_uint(tv.y)
            && __float_as_uint(dt) == __float_as_uint(tdt) && n_steps < p.max_n_steps) {
            const uint32_t L = lam, R = p.max_n_steps - n_steps, Rm = R % L;
            uint32_t E = 0, partial = 0;
            for (int pass = 0; pass < 2; ++pass) {
                Vec2 v2 = vec;
                float d2 = dt;
                uint32_t i2 = idx, ns2 = 0;
                uint2 l2 = last;
                if (pass == 1) {
                    const uint32_t nfut = (R / L) * E + partial;
                    if (nfut == 0) break;
                    sink.put(make_uint2(FLANK_PERIOD | E, nfut));
                }
                for (uint32_t t2 = 1; t2 <= L; ++t2) {
                    const Step s2 = rk_plain(v2, d2, uv, p);
                    const uint32_t q2 = s2.idx;
                    i2 = q2;
                    seg_move(s2, v2, i2, d2, ns2, p);
                    if (q2 != l2.x || i2 != l2.y) {
                        l2 = make_uint2(q2, i2);
                        if (pass == 0) {
                            E++;
                            if (t2 <= Rm) partial++;
                        } else {
                            sink.put(l2);
                        }
                    }
                }
            }
            break;
        }
        if (lam == power) {
            tv = vec;
            tdt = dt;
            power <<= 1;
            lam = 0;
        }
    }
    return sink.k;
}

// Items g0 .. g0+n-1: with pairs == NULL the pair counts into n_pairs[g],
// else the pairs into pairs[offsets[g] - base ..].
__global__ void k_flank_paths(const slm_params p, uint32_t g0, uint32_t n, const float2* __restrict__ seeds,
                              const uint8_t* __restrict__ stop, const float2* __restrict__ uv,
                              u64* __restrict__ n_pairs, const u64* __restrict__ offsets, u64 base,
                              uint2* __restrict__ pairs) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const uint32_t g = g0 + t;
    ContigSink sink{pairs ? pairs + (offsets[g] - base) : nullptr, 0};
    const u64 k = flank_walk(p, g, seeds, stop, uv, sink);
    if (!pairs) n_pairs[g] = k;
}

// Items 0 .. n-1 in one pass: each path into linked blocks from the pool
// (head block heads[g], NO_BLOCK for an empty path), its count into
// n_pairs[g]; pool_ctr[0] counts the blocks taken, pool_ctr[1] is set when
// the pool ran out (the counts are still exact).
__global__ void k_flank_paths_linked(const slm_params p, uint32_t n, const float2* __restrict__ seeds,
                                     const uint8_t* __restrict__ stop, const float2* __restrict__ uv,
                                     u64* __restrict__ n_pairs, uint32_t* __restrict__ heads,
                                     uint2* __restrict__ pool, uint32_t cap_blocks, uint32_t* pool_ctr) {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    heads[g] = NO_BLOCK;
    LinkedSink sink{pool, pool_ctr, pool_ctr + 1, cap_blocks, NO_BLOCK, 0, heads + g, 0, true};
    n_pairs[g] = flank_walk(p, g, seeds, stop, uv, sink);
}

// The label of pixel q as flank item g sees it: item g's own running value if
// q is g's pixel; the initial label if q has no owner or a higher-index owner;
// the resolved label if its owner has a lower index and resolved in an
// earlier round.  Returns false when that owner has not resolved yet.
// Kept out of line: the inlined form gave wrong labels on sm_100a for a few
// items of the 96x80 test case (tests/test_mapping_gpu.py), the out-of-line
// form matches the oracle on every case.
__device__ __noinline__ bool flank_read(uint32_t q, uint32_t g, uint32_t h, uint32_t lab_h,
                                           uint32_t cur_round, const uint32_t* __restrict__ owner,
                                           const uint32_t* __restrict__ label_init,
                                           const uint32_t* label,
                                           const uint32_t* resolved_round, uint32_t& out) {
    if (q == h) { out = lab_h; return true; }
    const uint32_t o = owner[q];
    if (o == NO_OWNER || o > g) { out = label_init[q]; return true; }
    const uint32_t r = ((volatile const uint32_t*)resolved_round)[o];
    if (r == 0u || r >= cur_round) return false;
    out = ((volatile const uint32_t*)label)[q];
    return true;
}

// One resolution round of fix_right_flanks (side 0) or fix_left_flanks
// (side 1) (segment.cl:441-504, 530-594).
__global__ void k_flank_round(const slm_params p, uint32_t g0, uint32_t n, uint32_t side, uint32_t cur_round,
                              const u64* __restrict__ offsets, u64 base, const uint2* __restrict__ pairs,
                              const uint32_t* __restrict__ hpix, const uint8_t* __restrict__ mask,
                              const uint32_t* __restrict__ mapping, const uint32_t* __restrict__ owner,
                              const uint32_t* __restrict__ label_init, uint32_t* label,
                              uint32_t* resolved_round, uint32_t* n_resolved) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const uint32_t g = g0 + t;
    if (resolved_round[g] != 0u) return;
    const uint32_t lfa = p.left_flank_addition;
    const uint32_t thin = p.is_thinchannel;
    const uint32_t h = hpix[g];
    uint32_t lab_h = label_init[h];
    uint32_t at = h, v = 0u;
    const u64 k_end = offsets[g + 1];
    // one step of the walk's label scan: 0 go on, 1 the walk stops, 2 wait
    // (a lower-index owner on the path is not resolved yet)
    auto scan = [&](uint2 e) -> int {
        if (!flank_read(at, g, h, lab_h, cur_round, owner, label_init, label, resolved_round, v)) return 2;
        const bool flank_ok = side ? (v & lfa) != 0u : ((~v) & lfa) != 0u;
        if (mask[at] || !flank_ok || (mapping[at] & thin)) return 1;
        if (!flank_read(e.x, g, h, lab_h, cur_round, owner, label_init, label, resolved_round, v)) return 2;
        if ((lab_h & ~lfa) != (v & ~lfa)) lab_h = v;
        at = e.y;
        return 0;
    };
    int st = 0;
    for (u64 k = offsets[g]; k < k_end && st == 0; ++k) {
        const uint2 e = pairs[k - base];
        if ((e.x & FLANK_PERIOD) == 0u) {
            st = scan(e);
            continue;
        }
        // period record: n pairs cycling through the next E.  Every read but
        // that of the item's own pixel gives the same value each lap and `at`
        // starts each lap at the lap's last pair, so a lap is a function of
        // lab_h at its start: once a lap-start lab_h repeats, whole multiples
        // of that lap period change nothing and are skipped.
        const uint32_t E = e.x & ~FLANK_PERIOD;
        const uint32_t nfut = e.y;
        const uint2* pat = pairs + (k + 1 - base);
        k += E;
        const uint32_t full = nfut / E, rem = nfut % E;
        uint32_t seen[8];
        bool skipped = false;
        for (uint32_t lap = 0; lap < full && st == 0; ++lap) {
            if (!skipped && lap < 8) {
                for (uint32_t j = 0; j < lap; ++j)
                    if (seen[j] == lab_h) {
                        const uint32_t per = lap - j;
                        lap += ((full - lap) / per) * per;
                        skipped = true;
                        break;
                    }
                if (!skipped) seen[lap] = lab_h;
                if (lap >= full) break;
            }
            for (uint32_t i = 0; i < E && st == 0; ++i) st = scan(pat[i]);
        }
        for (uint32_t i = 0; i < rem && st == 0; ++i) st = scan(pat[i]);
    }
    if (st == 2) return;
    if (!flank_read(at, g, h, lab_h, cur_round, owner, label_init, label, resolved_round, v)) return;
    if ((lab_h & ~lfa) != (v & ~lfa)) lab_h = v;
    flank_read(at, g, h, lab_h, cur_round, owner, label_init, label, resolved_round, v);
    if (side) {
        if (((~v) & lfa) && !(mapping[at] & thin)) lab_h &= ~lfa;
    } else {
        if (v & lfa) lab_h |= lfa;
    }
    label[h] = lab_h;
    resolved_round[g] = cur_round;
    atomicAdd(n_resolved, 1u);
}

// ------------------------------------------------------------------ fix flanks, settled in one launch
// The stored paths of a chunk of flank items resolved in one persistent
// launch instead of rounds.  Warps take items in ascending index from a
// queue (warp-aggregated atomicAdd), so every item below one a lane holds
// has been taken.  A lane scans its item's stored path as k_flank_round does;
// at a read of a lower-index owner that has not resolved it stops, notes that
// owner and its place in the path (the start of a period record when inside
// one, with the running label there), and on later passes only polls the
// owner's flag until it can go on.  The lowest unresolved item taken waits on
// nothing unresolved, so some lane always advances.  A label is published
// by a release store of its resolved flag, read with acquire.  The RK walks are traced in parallel
// beforehand (k_flank_paths), so only the path scans lie on a chain of waits.
//
// Every wait is bounded: a lane that polls FLANK_WAIT_LIMIT times in a row
// sets bit 0 of *status, and every warp stops; the caller then resolves the
// items in rounds (k_flank_round) from the initial labels.
#define FLANK_WAIT_LIMIT (1u << 24)

// the label of pixel q as item g reads it (flank_read's rules, with the
// owner's flag, read with acquire, instead of its round); false and *wait_o
// when the owner has not resolved.  Out of line, as flank_read.
// a flag read that orders the loads after it (acquire), and the flag write
// that publishes the stores before it (release), at GPU scope
__device__ __forceinline__ uint32_t load_acquire(const uint32_t* a) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(a) : "memory");
    return v;
}
__device__ __forceinline__ void store_release(uint32_t* a, uint32_t v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(a), "r"(v) : "memory");
}

__device__ __noinline__ bool settle_read(uint32_t q, uint32_t g, uint32_t h, uint32_t lab_h,
                                        const uint2* __restrict__ pix, const uint32_t* label,
                                        const uint32_t* resolved, uint32_t& out, uint32_t& wait_o) {
    if (q == h) { out = lab_h; return true; }
    const uint2 oi = pix[q];  // (owner, initial label) in one load
    const uint32_t o = oi.x;
    if (o == NO_OWNER || o > g) { out = oi.y; return true; }
    if (load_acquire(resolved + o) == 0u) { wait_o = o; return false; }
    out = ((volatile const uint32_t*)label)[q];
    return true;
}

// A stored path read pair by pair: a contiguous range (pairs[k], k <
// k_end), or linked blocks of FLANK_BLOCK entries, FLANK_BLOCK - 1 pairs and
// the index of the next block, with `left` pairs still to read.
struct ContigPath {
    const uint2* pairs;  // the chunk's store, indexed from the chunk's base
    u64 k, k_end;
    __device__ bool more() const { return k < k_end; }
    __device__ uint2 get() { return pairs[k]; }
    __device__ void next() { ++k; }
    __device__ void end() { k = k_end; }
};

struct LinkedPath {
    const uint2* pool;
    uint32_t blk, off;
    u64 left;
    __device__ bool more() const { return left > 0; }
    __device__ void follow() {
        if (off == FLANK_BLOCK - 1) {
            blk = pool[(u64)blk * FLANK_BLOCK + off].x;
            off = 0;
        }
    }
    __device__ uint2 get() {
        follow();
        return pool[(u64)blk * FLANK_BLOCK + off];
    }
    __device__ void next() {
        follow();
        ++off;
        --left;
    }
    __device__ void end() { left = 0; }
};

template <class P>
struct SettleLane {
    P path;
    uint32_t g, h, at, lab_h, wait_o, waited;
    bool alive, waiting;
};

// Scan item state `w` on from its place in its path; 0: resolved (label
// written), 2: blocked (w.path, w.at, w.lab_h at the place to resume,
// w.wait_o set).
template <class P>
__device__ int settle_scan(SettleLane<P>& w, uint32_t side, const slm_params& p,
                           const uint8_t* __restrict__ stop, const uint32_t* __restrict__ mapping,
                           const uint2* __restrict__ pix, uint32_t* label, uint32_t* resolved) {
    const uint32_t lfa = p.left_flank_addition, thin = p.is_thinchannel;
    uint32_t v = 0;
    // one pair of the walk's label scan: 0 go on, 1 the walk stops, 2 wait
    // (stop[q]: mask or thin channel at q; when the compute pixel is the
    // current one its label is the one just read)
    // The stop byte and both pixels' (owner, initial label) words are loaded
    // together; each label is then settled as settle_read does.
    auto scan = [&](uint2 e) -> int {
        const uint32_t a = w.at, c = e.x;
        const bool own_a = a == w.h, own_c = c == w.h, same = c == a;
        const uint8_t st_a = stop[a];
        const uint2 oa = own_a ? make_uint2(NO_OWNER, 0u) : pix[a];
        const uint2 oc = (own_c || same) ? make_uint2(NO_OWNER, 0u) : pix[c];
        if (st_a) return 1;
        if (own_a) {
            v = w.lab_h;
        } else if (oa.x == NO_OWNER || oa.x > w.g) {
            v = oa.y;
        } else if (load_acquire(resolved + oa.x) == 0u) {
            w.wait_o = oa.x;
            return 2;
        } else {
            v = ((volatile const uint32_t*)label)[a];
        }
        const bool flank_ok = side ? (v & lfa) != 0u : ((~v) & lfa) != 0u;
        if (!flank_ok) return 1;
        if (!same) {
            if (own_c) {
                v = w.lab_h;
            } else if (oc.x == NO_OWNER || oc.x > w.g) {
                v = oc.y;
            } else if (load_acquire(resolved + oc.x) == 0u) {
                w.wait_o = oc.x;
                return 2;
            } else {
                v = ((volatile const uint32_t*)label)[c];
            }
        }
        if ((w.lab_h & ~lfa) != (v & ~lfa)) w.lab_h = v;
        w.at = e.y;
        return 0;
    };
    while (w.path.more()) {
        const uint2 e = w.path.get();
        if ((e.x & FLANK_PERIOD) == 0u) {
            const int st = scan(e);
            if (st == 2) return 2;
            if (st == 1) { w.path.end(); break; }
            w.path.next();
            continue;
        }
        // a period record, as k_flank_round runs it (n pairs cycling through
        // the next E); a wait inside it restarts the record
        const uint32_t E = e.x & ~FLANK_PERIOD, nfut = e.y;
        P pat = w.path;
        pat.next();
        const uint32_t at0 = w.at, lab0 = w.lab_h;
        const uint32_t full = nfut / E, rem = nfut % E;
        uint32_t seen[8];
        bool skipped = false;
        int st = 0;
        for (uint32_t lap = 0; lap < full && st == 0; ++lap) {
            if (!skipped && lap < 8) {
                for (uint32_t j = 0; j < lap; ++j)
                    if (seen[j] == w.lab_h) {
                        const uint32_t per = lap - j;
                        lap += ((full - lap) / per) * per;
                        skipped = true;
                        break;
                    }
                if (!skipped) seen[lap] = w.lab_h;
                if (lap >= full) break;
            }
            P it = pat;
            for (uint32_t i = 0; i < E && st == 0; ++i) {
                st = scan(it.get());
                it.next();
            }
        }
        P it = pat;
        for (uint32_t i = 0; i < rem && st == 0; ++i) {
            st = scan(it.get());
            it.next();
        }
        if (st == 2) {
            w.at = at0;
            w.lab_h = lab0;
            return 2;
        }
        if (st == 1) { w.path.end(); break; }
        w.path = pat;
        for (uint32_t i = 0; i < E; ++i) w.path.next();
    }
    // after the walk: the label at the last pixel, then the flank bit
    if (!settle_read(w.at, w.g, w.h, w.lab_h, pix, label, resolved, v, w.wait_o)) return 2;
    if ((w.lab_h & ~lfa) != (v & ~lfa)) w.lab_h = v;
    settle_read(w.at, w.g, w.h, w.lab_h, pix, label, resolved, v, w.wait_o);
    if (side) {
        if (((~v) & lfa) && !(mapping[w.at] & thin)) w.lab_h &= ~lfa;
    } else {
        if (v & lfa) w.lab_h |= lfa;
    }
    label[w.h] = w.lab_h;
    store_release(resolved + w.g, 1u);
    return 0;
}

// pix[q] = (owner[q], label_init[q]), read together by the settle scan
__global__ void k_flank_pix(uint32_t nxy, const uint32_t* __restrict__ owner,
                            const uint32_t* __restrict__ label_init, uint2* __restrict__ pix) {
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < nxy; q += gridDim.x * blockDim.x)
        pix[q] = make_uint2(owner[q], label_init[q]);
}

// stop[q] = 1 where a flank walk's loop test ends regardless of labels
__global__ void k_flank_stop(uint32_t nxy, const uint8_t* __restrict__ mask, const uint32_t* __restrict__ mapping,
                             uint32_t thin, uint8_t* __restrict__ stop) {
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < nxy; q += gridDim.x * blockDim.x)
        stop[q] = (mask[q] || (mapping[q] & thin)) ? 1 : 0;
}

// Items g0 .. g0+n-1: with LinkedPath, item g's path starts at block
// heads[g] and holds n_pairs[g] pairs in `store`; with ContigPath it is
// store[offsets[g] - base .. offsets[g + 1] - base).
template <class P>
__global__ void __launch_bounds__(256)
k_flank_settle(const slm_params p, uint32_t g0, uint32_t n, uint32_t side, const u64* __restrict__ offsets,
               u64 base, const uint32_t* __restrict__ heads, const u64* __restrict__ n_pairs,
               const uint2* __restrict__ store, const uint32_t* __restrict__ hpix,
               const uint8_t* __restrict__ stop, const uint32_t* __restrict__ mapping,
               const uint2* __restrict__ pix, uint32_t* label, uint32_t* resolved, uint32_t* queue_head,
               uint32_t* status) {
    const unsigned FULL = 0xffffffffu;
    const unsigned lane = threadIdx.x & 31u;
    SettleLane<P> w;
    w.alive = false;
    bool drained = false;
    for (uint32_t pass = 0;; ++pass) {
        // a lane that gave up stops every warp (the caller falls back)
        if ((pass & 63u) == 0u) {
            uint32_t stop_all = 0;
            if (lane == 0) stop_all = *(volatile const uint32_t*)status;
            if (__shfl_sync(FULL, stop_all, 0)) break;
        }
        if (!drained) {
            const unsigned idle = __ballot_sync(FULL, !w.alive);
            if (idle) {
                const int leader = __ffs(idle) - 1;
                uint32_t head = 0;
                if ((int)lane == leader) head = atomicAdd(queue_head, (uint32_t)__popc(idle));
                head = __shfl_sync(FULL, head, leader);
                if ((u64)head + __popc(idle) >= n) drained = true;
                if (!w.alive) {
                    const uint32_t t = head + __popc(idle & ((1u << lane) - 1u));
                    if (t < n) {
                        w.g = g0 + t;
                        if constexpr (std::is_same<P, LinkedPath>::value) {
                            w.path.pool = store;
                            w.path.blk = heads[w.g];
                            w.path.off = 0;
                            w.path.left = n_pairs[w.g];
                        } else {
                            w.path.pairs = store;
                            w.path.k = offsets[w.g] - base;
                            w.path.k_end = offsets[w.g + 1] - base;
                        }
                        w.h = hpix[w.g];
                        w.at = w.h;
                        w.lab_h = pix[w.h].y;
                        w.waited = 0;
                        w.waiting = false;
                        w.alive = true;
                    }
                }
            }
        }
        if (!__any_sync(FULL, w.alive)) {
            if (drained) break;
            continue;
        }
        bool idle_pass = true;  // this lane did nothing but wait this pass
        if (w.alive) {
            bool go = true;
            if (w.waiting) {
                if (load_acquire(resolved + w.wait_o) == 0u) {
                    go = false;
                    if (++w.waited >= FLANK_WAIT_LIMIT) {
                        atomicOr(status, 1u);
                        w.alive = false;
                    }
                } else {
                    w.waiting = false;
                    w.waited = 0;
                }
            }
            if (go) {
                idle_pass = false;
                if (settle_scan(w, side, p, stop, mapping, pix, label, resolved) == 2)
                    w.waiting = true;
                else
                    w.alive = false;
            }
        }
        // a warp whose every lane only waited backs off, leaving the issue
        // slots to warps that scan
        if (__all_sync(FULL, idle_pass)) __nanosleep(256);
    }
}

// ------------------------------------------------------------------ hillslopes
__global__ void k_hillslopes(const slm_params p, uint32_t n, const float2* __restrict__ seeds,
                             const uint8_t* __restrict__ mask, const float2* __restrict__ uv,
                             uint32_t* link) {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    Vec2 vec = seed_vec(seeds, g);
    float dt = p.dt_max;
    uint32_t idx = pixel_of(vec, p), prev_idx = idx, n_steps = 0;
    // a (vec, dt) state repeating inside the start pixel (Brent) means the
    // walk circles there until the step bound and writes no link
    Vec2 tv = vec;
    float tdt = dt;
    uint32_t power = 1, lam = 0;
    while (prev_idx == idx && !mask[idx] && n_steps < 100u * p.max_n_steps) {
        prev_idx = idx;
        const Step s = rk_plain(vec, dt, uv, p);
        idx = s.idx;
        const Move m = rk_move(s, vec, idx, p);
        if (m.stuck) break;
        dt = next_dt(dt, m.err, p);
        n_steps++;
        if (idx == prev_idx && __float_as_uint(vec.x) == __float_as_uint(tv.x)
            && __float_as_uint(vec.y) == __float_as_uint(tv.y) && __float_as_uint(dt) == __float_as_uint(tdt))
            return;
        if (++lam == power) {
            tv = vec;
            tdt = dt;
            power <<= 1;
            lam = 0;
        }
    }
    if (prev_idx != idx && !mask[idx]) link[prev_idx] = idx;
}

__global__ void k_hillslope_lengths(const slm_params p, uint32_t n, const float2* __restrict__ seeds,
                                    const uint8_t* __restrict__ mask, const float2* __restrict__ uv,
                                    const uint32_t* __restrict__ mapping, float* traj_length) {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    const uint32_t from_flag = p.do_measure_hsl_from_ridges ? p.is_ridge : p.is_midslope;
    Vec2 vec = seed_vec(seeds, g);
    uint32_t idx = pixel_of(vec, p), n_steps = 0;
    float dt = p.dt_max, l = 0.0f;
    bool moved_off = false;
    // (vec, dt, moved_off) determines the rest of the walk (l only
    // accumulates).  Once it repeats (Brent; the checkpoint restarts when
    // moved_off turns), every lap passes the same tests, so the walk circles
    // to its step bound on a pixel that is not a thin channel and writes
    // nothing: it returns now.
    StateCycle cyc;
    cyc.init(vec, dt);
    while (((~mapping[idx]) & p.is_thinchannel) && n_steps < p.max_n_steps) {
        const Step s = rk_plain(vec, dt, uv, p);
        idx = s.idx;
        if (mask[idx]) return;
        bool turned = false;
        if (!moved_off && ((~mapping[idx]) & from_flag)) {
            moved_off = true;
            turned = true;
        } else if (moved_off && (mapping[idx] & from_flag)) {
            return;
        }
        const Move m = rk_move(s, vec, idx, p);
        l = l + m.dl;
        n_steps++;
        if (m.stuck) return;
        dt = next_dt(dt, m.err, p);
        if (turned) cyc.init(vec, dt);
        else if (cyc.repeated(vec, dt)) return;
    }
    if (mapping[idx] & p.is_thinchannel) traj_length[g] = l * p.pixel_size;
}

// ------------------------------------------------------------------ scan
// exclusive prefix sum of n uint64 counts into out[0..n] (out[n] = total);
// one block walks the array in chunks of its size.
__global__ void k_exclusive_scan(const u64* __restrict__ in, uint32_t n, u64* __restrict__ out) {
    __shared__ u64 buf[1024];
    u64 carry = 0;
    for (uint32_t base = 0; base < n; base += blockDim.x) {
        const uint32_t i = base + threadIdx.x;
        const u64 v = i < n ? in[i] : 0ull;
        buf[threadIdx.x] = v;
        __syncthreads();
        for (uint32_t off = 1; off < blockDim.x; off <<= 1) {
            const u64 t = threadIdx.x >= off ? buf[threadIdx.x - off] : 0ull;
            __syncthreads();
            buf[threadIdx.x] += t;
            __syncthreads();
        }
        if (i < n) out[i] = carry + buf[threadIdx.x] - v;
        const u64 tot = buf[blockDim.x - 1];
        __syncthreads();
        carry += tot;
    }
    if (threadIdx.x == 0) out[n] = carry;
}

// Exclusive scan of n u64 for large n, in tiles of SCAN_TILE: per-tile sums,
// an exclusive scan of those (k_exclusive_scan), then each tile rescanned
// with its offset.  out[n] = the total.
constexpr uint32_t SCAN_PER = 8;
constexpr uint32_t SCAN_TILE = 1024 * SCAN_PER;

__global__ void __launch_bounds__(1024) k_tile_sums(const u64* __restrict__ in, uint32_t n, u64* __restrict__ sums) {
    __shared__ u64 warp_sum[32];
    const u64 t0 = (u64)blockIdx.x * SCAN_TILE + (u64)threadIdx.x * SCAN_PER;
    u64 v = 0;
#pragma unroll
    for (uint32_t k = 0; k < SCAN_PER; ++k)
        if (t0 + k < n) v += in[t0 + k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) warp_sum[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        u64 w = warp_sum[threadIdx.x];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
        if (threadIdx.x == 0) sums[blockIdx.x] = w;
    }
}

__global__ void __launch_bounds__(1024) k_tile_scan(const u64* __restrict__ in, uint32_t n,
                                                    const u64* __restrict__ tile_off, uint32_t n_tiles,
                                                    u64* __restrict__ out) {
    __shared__ u64 warp_off[32];
    const unsigned lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
    const u64 t0 = (u64)blockIdx.x * SCAN_TILE + (u64)threadIdx.x * SCAN_PER;
    u64 x[SCAN_PER];
    u64 tot = 0;
#pragma unroll
    for (uint32_t k = 0; k < SCAN_PER; ++k) {
        x[k] = t0 + k < n ? in[t0 + k] : 0ull;
        tot += x[k];
    }
    // inclusive scan of the thread totals within the warp, then across warps
    u64 inc = tot;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const u64 y = __shfl_up_sync(0xffffffffu, inc, o);
        if ((int)lane >= o) inc += y;
    }
    if (lane == 31) warp_off[wid] = inc;
    __syncthreads();
    if (wid == 0) {
        u64 w = warp_off[lane];
        u64 wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const u64 y = __shfl_up_sync(0xffffffffu, wi, o);
            if ((int)lane >= o) wi += y;
        }
        warp_off[lane] = wi - w;  // exclusive
    }
    __syncthreads();
    u64 run = tile_off[blockIdx.x] + warp_off[wid] + (inc - tot);
#pragma unroll
    for (uint32_t k = 0; k < SCAN_PER; ++k) {
        if (t0 + k < n) out[t0 + k] = run;
        run += x[k];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) out[n] = tile_off[n_tiles];
}

// scratch words exclusive_scan needs for n elements
static inline size_t scan_scratch_words(uint32_t n) { return 2 * ((size_t)(n + SCAN_TILE - 1) / SCAN_TILE + 1); }

static int exclusive_scan(const u64* in, uint32_t n, u64* out, u64* scratch, cudaStream_t s) {
    const uint32_t n_tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    if (n_tiles <= 8) {
        k_exclusive_scan<<<1, 1024, 0, s>>>(in, n, out);
        SLM_LAUNCHED("k_exclusive_scan");
        return SLM_OK;
    }
    u64* sums = scratch;
    u64* off = scratch + n_tiles + 1;
    k_tile_sums<<<n_tiles, 1024, 0, s>>>(in, n, sums);
    SLM_LAUNCHED("k_tile_sums");
    k_exclusive_scan<<<1, 1024, 0, s>>>(sums, n_tiles, off);
    SLM_LAUNCHED("k_exclusive_scan");
    k_tile_scan<<<n_tiles, 1024, 0, s>>>(in, n, off, n_tiles, out);
    SLM_LAUNCHED("k_tile_scan");
    return SLM_OK;
}

// ------------------------------------------------------------------ parallel flag_downchannels
// The pinned sequential flag_downchannels (countlink.cl:124-210, heads in
// index order) computed by all heads at once.  link is not written, so each
// head's walk is fixed; its effects are flag ORs (order-free), the head-flag
// clear, the tail flag, and count writes, which are "count = counter if
// counter >= count" (a max) after the unconditional count[head] = 1 of each
// head.  Per pixel x (g_x = the head whose head pixel is x, if any):
//   final count[x] = g_x ? max(1, visits by heads g >= g_x)
//                        : max(initial count[x], all visits)
// The only order-dependent read is count[x2] > 2 at a head's second pixel
// (counter 2), i.e. whether an earlier head visited x2 with a counter > 2
// since x2's reset: F1[x] = first head >= g_x, F0[x] = first head at all,
// visiting x with a counter > 2.
constexpr uint32_t NO_HEAD = 0xffffffffu;

__global__ void k_flag_head_index(const slm_params p, uint32_t n, const float2* __restrict__ seeds,
                                  uint32_t* __restrict__ head_of, uint32_t* __restrict__ head_pix) {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    const uint32_t hp = pixel_of(seed_vec(seeds, g), p);
    head_pix[g] = hp;
    atomicMin(head_of + hp, g);  // seeds are distinct pixels; min keeps it exact regardless
}

__device__ __forceinline__ void flag_visit(uint32_t x, uint32_t g, uint32_t c, const uint32_t* __restrict__ head_of,
                                           uint32_t* cmax, uint32_t* f0, uint32_t* f1) {
    const uint32_t gx = head_of[x];
    if (gx == NO_HEAD || g >= gx) atomicMax(cmax + x, c);
    if (c > 2u) {
        atomicMin(f0 + x, g);
        if (gx != NO_HEAD && g >= gx) atomicMin(f1 + x, g);
    }
}

__global__ void k_flag_walks(const slm_params p, uint32_t n, const uint8_t* __restrict__ mask,
                             uint32_t* mapping, const uint32_t* __restrict__ link,
                             const uint32_t* __restrict__ head_pix, const uint32_t* __restrict__ head_of,
                             uint32_t* cmax, uint32_t* f0, uint32_t* f1, uint8_t* __restrict__ clear_head,
                             uint32_t* __restrict__ second) {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    const uint32_t lim = 1000u * p.max_n_steps;
    const uint32_t head = head_pix[g];
    uint32_t idx = head, prev_idx = idx + 1u, counter = 1;
    atomicOr(mapping + idx, p.is_thinchannel);
    uint8_t clr = 0;
    uint32_t x2 = NO_HEAD;
    uint32_t tort = idx, power = 1, lam = 0;
    while (!mask[idx] && prev_idx != idx && counter < lim) {
        prev_idx = idx;
        idx = link[idx];
        counter++;
        if (mask[idx]) break;
        if (counter == 2u) x2 = idx;
        if (counter < 20u && (mapping[idx] & p.is_minorinflow)) clr = 1;
        atomicOr(mapping + idx, p.is_thinchannel);
        flag_visit(idx, g, counter, head_of, cmax, f0, f1);
        lam++;
        if (idx == tort && counter >= 20u && prev_idx != idx && counter < lim) {
            // a cycle of lam pixels walked once since tort (and the counter <
            // 20 window of the minor-inflow test already walked): the walk
            // circles until counter == lim; each pixel's last visit counts
            const uint32_t r = lim - counter;
            uint32_t q = idx;
            for (uint32_t o = 1; o <= lam && o <= r; ++o) {
                q = link[q];
                flag_visit(q, g, counter + o + lam * ((r - o) / lam), head_of, cmax, f0, f1);
            }
            counter = lim;
            break;
        }
        if (lam == power) {
            tort = idx;
            power <<= 1;
            lam = 0;
        }
    }
    if (!mask[prev_idx] && counter < lim) atomicOr(mapping + prev_idx, p.is_channeltail);
    clear_head[g] = clr;
    second[g] = x2;
}

__global__ void k_flag_heads(uint32_t n, uint32_t is_channelhead, const uint32_t* __restrict__ head_pix,
                             const uint32_t* __restrict__ head_of, const uint32_t* __restrict__ count_init,
                             const uint32_t* __restrict__ f0, const uint32_t* __restrict__ f1,
                             const uint8_t* __restrict__ clear_head, const uint32_t* __restrict__ second,
                             uint32_t* mapping) {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    bool clr = clear_head[g] != 0;
    const uint32_t x2 = second[g], hp = head_pix[g];
    if (!clr && x2 != NO_HEAD && x2 != hp) {
        const uint32_t gx = head_of[x2];
        if (gx != NO_HEAD && gx < g) clr = f1[x2] < g;  // x2 was reset by an earlier head
        else clr = count_init[x2] > 2u || f0[x2] < g;
    }
    if (clr) atomicAnd(mapping + hp, ~is_channelhead);
}

__global__ void k_flag_counts(uint32_t nxy, const uint32_t* __restrict__ head_of,
                              const uint32_t* __restrict__ cmax, uint32_t* count) {
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= nxy) return;
    const uint32_t c = cmax[x];
    if (head_of[x] != NO_HEAD) count[x] = c > 1u ? c : 1u;
    else if (c > count[x]) count[x] = c;
}

// ------------------------------------------------------------------ thinning
// One sub-iteration of Zhang-Suen thinning (T. Y. Zhang, C. Y. Suen, CACM
// 27(3), 1984) on a 0/1 image [nx][ny] (x-major, outside = 0): dst = src with
// every removable pixel cleared; *changed set when one was.  Neighbours P2..P9
// run clockwise from (x-1, y): (x-1,y) (x-1,y+1) (x,y+1) (x+1,y+1) (x+1,y)
// (x+1,y-1) (x,y-1) (x-1,y-1).
__global__ void k_zhang_suen(const uint8_t* __restrict__ src, uint8_t* __restrict__ dst, uint32_t nx,
                             uint32_t ny, int step, uint32_t* changed) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nx * ny) return;
    const uint32_t x = i / ny, y = i % ny;
    const uint8_t c = src[i];
    uint8_t out = c;
    if (c) {
        auto at = [&](int dx, int dy) -> uint32_t {
            const int xx = (int)x + dx, yy = (int)y + dy;
            if (xx < 0 || yy < 0 || xx >= (int)nx || yy >= (int)ny) return 0u;
            return src[(size_t)xx * ny + yy] ? 1u : 0u;
        };
        const uint32_t n[8] = {at(-1, 0), at(-1, 1), at(0, 1), at(1, 1), at(1, 0), at(1, -1), at(0, -1), at(-1, -1)};
        uint32_t b = 0, a = 0;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            b += n[k];
            a += (n[k] == 0u && n[(k + 1) & 7] == 1u) ? 1u : 0u;
        }
        const uint32_t p2 = n[0], p4 = n[2], p6 = n[4], p8 = n[6];
        const bool c1 = step == 0 ? (p2 * p4 * p6) == 0u : (p2 * p4 * p8) == 0u;
        const bool c2 = step == 0 ? (p4 * p6 * p8) == 0u : (p2 * p6 * p8) == 0u;
        if (b >= 2u && b <= 6u && a == 1u && c1 && c2) {
            out = 0;
            *changed = 1u;
        }
    }
    dst[i] = out;
}

}  // namespace slm

using namespace slm;

static int map_checks(const slm_params* p, uint32_t n, const void* seeds) {
    SLM_REQUIRE(p != nullptr, "params is NULL");
    SLM_REQUIRE(p->nx_padded >= 2 && p->ny_padded >= 2 &&
                (u64)p->nx_padded * p->ny_padded == p->nxy_padded, "bad grid size");
    SLM_REQUIRE(p->trajectory_resolution > 0, "trajectory_resolution is 0");
    SLM_REQUIRE(n == 0 || (seeds && aligned(seeds, 8)), "seed_point NULL or misaligned");
    return SLM_OK;
}

static inline unsigned blocks_for(uint32_t n, unsigned b) { return (n + b - 1) / b; }
#define F2(x) reinterpret_cast<const float2*>(x)
#define SS (cudaStream_t) stream

extern "C" {

int slm_connect_channels(const slm_params* p, uint32_t n, const float* seed_point, const uint8_t* mask,
                         const float* uv, uint32_t* mapping, uint32_t* status, void* stream) {
    clear_error();
    int rc = map_checks(p, n, seed_point);
    if (rc) return rc;
    SLM_REQUIRE(p->interchannel_max_n_steps <= CONNECT_REC_MAX,
                "interchannel_max_n_steps %u above the supported %d", p->interchannel_max_n_steps,
                CONNECT_REC_MAX);
    SLM_REQUIRE(status, "status word is NULL");
    SLM_CUDA(cudaMemsetAsync(status, 0, sizeof(uint32_t), SS));
    if (n == 0) return SLM_OK;
    k_connect_channels<<<blocks_for(n, 128), 128, 0, SS>>>(*p, n, F2(seed_point), mask, F2(uv), mapping, status);
    SLM_LAUNCHED("k_connect_channels");
    return SLM_OK;
}

int slm_map_channel_heads(const slm_params* p, uint32_t n, const float* seed_point, const uint8_t* mask,
                          const float* uv, uint32_t* mapping, void* stream) {
    clear_error();
    int rc = map_checks(p, n, seed_point);
    if (rc) return rc;
    if (n == 0) return SLM_OK;
    k_map_channel_heads<<<blocks_for(n, 128), 128, 0, SS>>>(*p, n, F2(seed_point), mask, F2(uv), mapping);
    SLM_LAUNCHED("k_map_channel_heads");
    return SLM_OK;
}

int slm_prune_channel_heads(const slm_params* p, uint32_t n, const float* seed_point, const uint8_t* mask,
                            const float* uv, uint32_t* mapping, void* stream) {
    (void)mask; (void)uv;
    clear_error();
    int rc = map_checks(p, n, seed_point);
    if (rc) return rc;
    if (n == 0) return SLM_OK;
    k_prune_channel_heads<<<1, 1024, 0, SS>>>(*p, n, F2(seed_point), mapping);
    SLM_LAUNCHED("k_prune_channel_heads");
    return SLM_OK;
}

size_t slm_count_downchannels_workspace(uint32_t n_seeds, uint64_t n_events) {
    return (size_t)(2 * (size_t)n_seeds + 1) * sizeof(u64) + (size_t)n_seeds * sizeof(uint32_t)
         + (size_t)n_events * sizeof(uint32_t) + 256;
}

int slm_count_downchannels(const slm_params* p, uint32_t n, const float* seed_point, const uint8_t* mask,
                           const float* uv, uint32_t* mapping, uint32_t* count, uint32_t* link,
                           void* workspace, size_t workspace_bytes, uint64_t* required_bytes,
                           void* stream) {
    clear_error();
    int rc = map_checks(p, n, seed_point);
    if (rc) return rc;
    if (n == 0) return SLM_OK;
    SLM_REQUIRE(workspace && workspace_bytes >= slm_count_downchannels_workspace(n, 0),
                "workspace below the minimum %zu bytes", slm_count_downchannels_workspace(n, 0));
    u64* n_events = reinterpret_cast<u64*>(workspace);
    u64* offsets = n_events + n;
    uint32_t* tails = reinterpret_cast<uint32_t*>(offsets + n + 1);
    uint32_t* events = tails + n;
    k_count_paths<<<blocks_for(n, 128), 128, 0, SS>>>(*p, n, F2(seed_point), mask, F2(uv), n_events,
                                                     nullptr, nullptr, nullptr);
    SLM_LAUNCHED("k_count_paths");
    k_exclusive_scan<<<1, 1024, 0, SS>>>(n_events, n, offsets);
    SLM_LAUNCHED("k_exclusive_scan");
    u64 total = 0;
    SLM_CUDA(cudaMemcpyAsync(&total, offsets + n, sizeof(u64), cudaMemcpyDeviceToHost, SS));
    SLM_CUDA(cudaStreamSynchronize(SS));
    const size_t need = slm_count_downchannels_workspace(n, total);
    if (required_bytes) *required_bytes = need;
    if (need > workspace_bytes) {
        set_error("count_downchannels needs %zu workspace bytes (%llu path events)", need,
                  (unsigned long long)total);
        return SLM_ERR_CAPACITY;
    }
    k_count_paths<<<blocks_for(n, 128), 128, 0, SS>>>(*p, n, F2(seed_point), mask, F2(uv), nullptr,
                                                     offsets, events, tails);
    SLM_LAUNCHED("k_count_paths");
    SLM_REQUIRE(p->nxy_padded < 0xFFFFFFE0u, "grid too large for the count replay");
    k_count_replay_warp<<<1, 32, 0, SS>>>(*p, n, F2(seed_point), offsets, events, tails, mapping, count, link);
    SLM_LAUNCHED("k_count_replay_warp");
    return SLM_OK;
}

size_t slm_flag_downchannels_workspace(uint32_t n_seeds, uint32_t nxy_padded) {
    return (size_t)nxy_padded * 4 * sizeof(uint32_t) + (size_t)n_seeds * (2 * sizeof(uint32_t) + 1) + 256;
}

int slm_flag_downchannels(const slm_params* p, uint32_t n, const float* seed_point, const uint8_t* mask,
                          const float* uv, uint32_t* mapping, uint32_t* count, const uint32_t* link,
                          void* workspace, size_t workspace_bytes, uint64_t* required_bytes, void* stream) {
    (void)uv;
    clear_error();
    int rc = map_checks(p, n, seed_point);
    if (rc) return rc;
    const uint32_t nxy = p->nxy_padded;
    const size_t need = slm_flag_downchannels_workspace(n, nxy);
    if (required_bytes) *required_bytes = need;
    if (n == 0) return SLM_OK;
    if (!workspace || workspace_bytes < need) {
        set_error("flag_downchannels needs %zu workspace bytes", need);
        return SLM_ERR_CAPACITY;
    }
    uint32_t* head_of = reinterpret_cast<uint32_t*>(workspace);
    uint32_t* cmax = head_of + nxy;
    uint32_t* f0 = cmax + nxy;
    uint32_t* f1 = f0 + nxy;
    uint32_t* head_pix = f1 + nxy;
    uint32_t* second = head_pix + n;
    uint8_t* clear_head = reinterpret_cast<uint8_t*>(second + n);
    SLM_CUDA(cudaMemsetAsync(head_of, 0xff, (size_t)nxy * sizeof(uint32_t), SS));
    SLM_CUDA(cudaMemsetAsync(cmax, 0, (size_t)nxy * sizeof(uint32_t), SS));
    SLM_CUDA(cudaMemsetAsync(f0, 0xff, (size_t)2 * nxy * sizeof(uint32_t), SS));
    k_flag_head_index<<<blocks_for(n, 256), 256, 0, SS>>>(*p, n, F2(seed_point), head_of, head_pix);
    SLM_LAUNCHED("k_flag_head_index");
    k_flag_walks<<<blocks_for(n, 128), 128, 0, SS>>>(*p, n, mask, mapping, link, head_pix, head_of, cmax, f0, f1,
                                                     clear_head, second);
    SLM_LAUNCHED("k_flag_walks");
    k_flag_heads<<<blocks_for(n, 256), 256, 0, SS>>>(n, p->is_channelhead, head_pix, head_of, count, f0, f1,
                                                     clear_head, second, mapping);
    SLM_LAUNCHED("k_flag_heads");
    k_flag_counts<<<blocks_for(nxy, 256), 256, 0, SS>>>(nxy, head_of, cmax, count);
    SLM_LAUNCHED("k_flag_counts");
    return SLM_OK;
}

int slm_label_confluences(const slm_params* p, uint32_t n, const float* seed_point, const uint8_t* mask,
                          const float* uv, const float* slt, uint32_t* mapping, const uint32_t* count,
                          const uint32_t* link, void* stream) {
    (void)uv;
    clear_error();
    int rc = map_checks(p, n, seed_point);
    if (rc) return rc;
    if (n == 0) return SLM_OK;
    k_label_confluences<<<blocks_for(n, 128), 128, 0, SS>>>(*p, n, F2(seed_point), mask, slt, mapping,
                                                           count, link);
    SLM_LAUNCHED("k_label_confluences");
    return SLM_OK;
}

int slm_segment_downchannels(const slm_params* p, uint32_t n, const float* seed_point,
                             const uint8_t* mask, const float* uv, uint32_t* mapping,
                             const uint32_t* count, const uint32_t* link, uint32_t* label,
                             uint32_t* status, void* stream) {
    (void)uv;
    clear_error();
    int rc = map_checks(p, n, seed_point);
    if (rc) return rc;
    SLM_REQUIRE(status, "status word is NULL");
    SLM_CUDA(cudaMemsetAsync(status, 0, sizeof(uint32_t), SS));
    if (n == 0) return SLM_OK;
    k_segment_downchannels<<<1, 1, 0, SS>>>(*p, n, F2(seed_point), mask, mapping, count, link, label,
                                            status);
    SLM_LAUNCHED("k_segment_downchannels");
    return SLM_OK;
}

int slm_segment_hillslopes(const slm_params* p, uint32_t n, const float* seed_point, const uint8_t* mask,
                           const float* uv, const uint32_t* mapping, const uint32_t* count,
                           const uint32_t* link, uint32_t* label, void* stream) {
    (void)count; (void)link;
    clear_error();
    int rc = map_checks(p, n, seed_point);
    if (rc) return rc;
    if (n == 0) return SLM_OK;
    SegHillWalk w{*p, F2(seed_point), mask, F2(uv), mapping, label};
    k_walks<SegHillWalk><<<walk_grid(n), 256, 0, SS>>>(w, n);
    SLM_LAUNCHED("k_walks<SegHillWalk>");
    return SLM_OK;
}

int slm_subsegment_channel_edges(const slm_params* p, uint32_t n, const float* seed_point,
                                 const uint8_t* mask, const float* uv, uint32_t* mapping,
                                 const uint32_t* channel_label, const uint32_t* link, uint32_t* label,
                                 uint32_t* status, void* stream) {
    (void)uv; (void)channel_label;
    clear_error();
    int rc = map_checks(p, n, seed_point);
    if (rc) return rc;
    SLM_REQUIRE(status, "status word is NULL");
    SLM_CUDA(cudaMemsetAsync(status, 0, sizeof(uint32_t), SS));
    if (n == 0) return SLM_OK;
    k_subsegment_channel_edges<<<blocks_for(n, 128), 128, 0, SS>>>(*p, n, F2(seed_point), mask, mapping,
                                                                  link, label, status);
    SLM_LAUNCHED("k_subsegment_channel_edges");
    return SLM_OK;
}

int slm_subsegment_flanks(const slm_params* p, uint32_t n, const float* seed_point, const uint8_t* mask,
                          const float* uv, const uint32_t* mapping, const uint32_t* channel_label,
                          const uint32_t* link, uint32_t* label, void* stream) {
    (void)channel_label; (void)link;
    clear_error();
    int rc = map_checks(p, n, seed_point);
    if (rc) return rc;
    if (n == 0) return SLM_OK;
    SubsegFlankWalk w{*p, F2(seed_point), mask, F2(uv), mapping, label};
    k_walks<SubsegFlankWalk><<<walk_grid(n), 256, 0, SS>>>(w, n);
    SLM_LAUNCHED("k_walks<SubsegFlankWalk>");
    return SLM_OK;
}

size_t slm_exclusive_scan_u64_scratch(uint32_t n) { return scan_scratch_words(n) * sizeof(u64); }

int slm_exclusive_scan_u64(const uint64_t* in, uint32_t n, uint64_t* out, void* scratch, size_t scratch_bytes,
                           void* stream) {
    clear_error();
    SLM_REQUIRE(in && out && scratch, "NULL buffer");
    SLM_REQUIRE(aligned(in, 8) && aligned(out, 8) && aligned(scratch, 8), "buffers must be 8-byte aligned");
    SLM_REQUIRE(scratch_bytes >= slm_exclusive_scan_u64_scratch(n), "scratch holds %zu bytes, needs %zu",
                scratch_bytes, slm_exclusive_scan_u64_scratch(n));
    return exclusive_scan(reinterpret_cast<const u64*>(in), n, reinterpret_cast<u64*>(out),
                          reinterpret_cast<u64*>(scratch), SS);
}

size_t slm_fix_flanks_workspace(uint32_t n_seeds, uint32_t nxy_padded, uint64_t n_pairs) {
    return (size_t)(2 * (size_t)n_seeds + 1) * sizeof(u64) + (size_t)n_seeds * 3 * sizeof(uint32_t)
         + (size_t)nxy_padded * 2 * sizeof(uint32_t) + 8 * sizeof(uint32_t) + 256
         + scan_scratch_words(n_seeds) * sizeof(u64) + ((size_t)nxy_padded + 16)
         + ((size_t)nxy_padded * sizeof(uint2) + 16) + (size_t)n_pairs * sizeof(uint2);
}

// restore the labels and flags before the rounds start over
static int flank_restart(uint32_t* label, const uint32_t* label_init, uint32_t* resolved, uint32_t n,
                         uint32_t nxy, cudaStream_t s) {
    SLM_CUDA(cudaMemcpyAsync(label, label_init, (size_t)nxy * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
    SLM_CUDA(cudaMemsetAsync(resolved, 0, (size_t)n * sizeof(uint32_t), s));
    return SLM_OK;
}

static int fix_flanks(const slm_params* p, uint32_t n, const float* seed_point, const uint8_t* mask,
                      const float* uv, const uint32_t* mapping, uint32_t* label, void* workspace,
                      size_t workspace_bytes, uint64_t* required_bytes, void* stream, bool left) {
    clear_error();
    int rc = map_checks(p, n, seed_point);
    if (rc) return rc;
    if (n == 0) return SLM_OK;
    const uint32_t nxy = p->nxy_padded;
    const size_t fixed = slm_fix_flanks_workspace(n, nxy, 0);
    SLM_REQUIRE(workspace && workspace_bytes >= fixed, "workspace below the minimum %zu bytes", fixed);
    u64* n_pairs = reinterpret_cast<u64*>(workspace);
    u64* offsets = n_pairs + n;
    uint32_t* hpix = reinterpret_cast<uint32_t*>(offsets + n + 1);
    uint32_t* resolved = hpix + n;
    uint32_t* heads = resolved + n;
    uint32_t* owner = heads + n;
    uint32_t* label_init = owner + nxy;
    // [0] rounds: resolved count; [1] queue head; [2] status; [3] pool blocks
    // taken; [4] pool ran out
    uint32_t* words = label_init + nxy;
    uintptr_t pa = reinterpret_cast<uintptr_t>(words + 8);
    pa = (pa + 15) & ~(uintptr_t)15;
    u64* scan_scratch = reinterpret_cast<u64*>(pa);
    uint8_t* stop = reinterpret_cast<uint8_t*>(scan_scratch + scan_scratch_words(n));
    pa = reinterpret_cast<uintptr_t>(stop + nxy);
    pa = (pa + 15) & ~(uintptr_t)15;
    uint2* pix = reinterpret_cast<uint2*>(pa);
    uint2* pairs = pix + nxy;  // the path store
    const u64 cap_pairs = (workspace_bytes - fixed) / sizeof(uint2);
    SLM_CUDA(cudaMemsetAsync(owner, 0xff, (size_t)nxy * sizeof(uint32_t), SS));
    SLM_CUDA(cudaMemsetAsync(resolved, 0, (size_t)n * sizeof(uint32_t), SS));
    SLM_CUDA(cudaMemsetAsync(words, 0, 8 * sizeof(uint32_t), SS));
    SLM_CUDA(cudaMemcpyAsync(label_init, label, (size_t)nxy * sizeof(uint32_t), cudaMemcpyDeviceToDevice, SS));
    k_owner_map<<<blocks_for(n, 256), 256, 0, SS>>>(*p, n, F2(seed_point), owner, hpix);
    SLM_LAUNCHED("k_owner_map");
    k_flank_stop<<<(unsigned)(num_sms() * 8), 256, 0, SS>>>(nxy, mask, mapping, p->is_thinchannel, stop);
    SLM_LAUNCHED("k_flank_stop");
    k_flank_pix<<<(unsigned)(num_sms() * 8), 256, 0, SS>>>(nxy, owner, label_init, pix);
    SLM_LAUNCHED("k_flank_pix");
    if (required_bytes) *required_bytes = fixed;

    // 1. Every walk traced once into linked blocks, then settled in one
    //    persistent launch.  The rounds (k_flank_round) run instead when the
    //    environment variable SLM_FLANK_ROUNDS is nonzero (for tests), and
    //    from the initial labels if a settle wait ran out.
    const char* force = std::getenv("SLM_FLANK_ROUNDS");
    const bool rounds_only = force && force[0] && force[0] != '0';
    const unsigned side = left ? 1u : 0u;
    bool counted = false, settle = !rounds_only;
    unsigned settle_grid = 0;
    if (settle) {
        int occ = 0;
        SLM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_flank_settle<LinkedPath>, 256, 0));
        settle_grid = (unsigned)(num_sms() * (occ > 0 ? occ : 1));
        const u64 cap_blocks = cap_pairs / FLANK_BLOCK;
        k_flank_paths_linked<<<blocks_for(n, 128), 128, 0, SS>>>(
            *p, n, F2(seed_point), stop, F2(uv), n_pairs, heads, pairs,
            (uint32_t)(cap_blocks < 0xfffffffeull ? cap_blocks : 0xfffffffeull), words + 3);
        SLM_LAUNCHED("k_flank_paths_linked");
        counted = true;
        uint32_t ran_out = 0;
        SLM_CUDA(cudaMemcpyAsync(&ran_out, words + 4, sizeof(uint32_t), cudaMemcpyDeviceToHost, SS));
        SLM_CUDA(cudaStreamSynchronize(SS));
        if (!ran_out) {
            k_flank_settle<LinkedPath><<<settle_grid, 256, 0, SS>>>(
                *p, 0u, n, side, nullptr, 0ull, heads, n_pairs, pairs, hpix, stop, mapping, pix, label, resolved,
                words + 1, words + 2);
            SLM_LAUNCHED("k_flank_settle");
            uint32_t st = 0;
            SLM_CUDA(cudaMemcpyAsync(&st, words + 2, sizeof(uint32_t), cudaMemcpyDeviceToHost, SS));
            SLM_CUDA(cudaStreamSynchronize(SS));
            if (st == 0u) return SLM_OK;
            rc = flank_restart(label, label_init, resolved, n, nxy, SS);
            if (rc) return rc;
            settle = false;
        }
    }

    // 2. The paths did not fit the pool (or the rounds run): stored
    //    contiguously, in index-ordered chunks when they do not all fit.  An
    //    item reads only initial labels and the final labels of lower-index
    //    owners, which earlier chunks have resolved.
    if (!counted) {
        k_flank_paths<<<blocks_for(n, 128), 128, 0, SS>>>(*p, 0u, n, F2(seed_point), stop, F2(uv), n_pairs,
                                                         nullptr, 0ull, nullptr);
        SLM_LAUNCHED("k_flank_paths");
    }
    rc = exclusive_scan(n_pairs, n, offsets, scan_scratch, SS);
    if (rc) return rc;
    u64 total = 0;
    SLM_CUDA(cudaMemcpyAsync(&total, offsets + n, sizeof(u64), cudaMemcpyDeviceToHost, SS));
    SLM_CUDA(cudaStreamSynchronize(SS));
    if (required_bytes) *required_bytes = slm_fix_flanks_workspace(n, nxy, total);
    std::vector<std::pair<uint32_t, uint32_t>> chunks;
    if (total <= cap_pairs) {
        chunks.emplace_back(0u, n);
    } else {
        std::vector<u64> off((size_t)n + 1);
        SLM_CUDA(cudaMemcpyAsync(off.data(), offsets, ((size_t)n + 1) * sizeof(u64), cudaMemcpyDeviceToHost, SS));
        SLM_CUDA(cudaStreamSynchronize(SS));
        u64 biggest = 0;
        for (uint32_t g = 0; g < n; ++g) biggest = std::max<u64>(biggest, off[g + 1] - off[g]);
        if (biggest > cap_pairs) {
            if (required_bytes) *required_bytes = slm_fix_flanks_workspace(n, nxy, biggest);
            set_error("fix flanks: one path has %llu steps; the workspace holds %llu",
                      (unsigned long long)biggest, (unsigned long long)cap_pairs);
            return SLM_ERR_CAPACITY;
        }
        uint32_t a = 0;
        while (a < n) {
            uint32_t b = a + 1;
            while (b < n && off[b + 1] - off[a] <= cap_pairs) ++b;
            chunks.emplace_back(a, b);
            a = b;
        }
    }
    if (settle) {
        int occ = 0;
        SLM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_flank_settle<ContigPath>, 256, 0));
        const unsigned grid = (unsigned)(num_sms() * (occ > 0 ? occ : 1));
        for (const auto& c : chunks) {
            const uint32_t a = c.first, m = c.second - c.first;
            u64 base = 0;
            SLM_CUDA(cudaMemcpyAsync(&base, offsets + a, sizeof(u64), cudaMemcpyDeviceToHost, SS));
            SLM_CUDA(cudaStreamSynchronize(SS));
            k_flank_paths<<<blocks_for(m, 128), 128, 0, SS>>>(*p, a, m, F2(seed_point), stop, F2(uv), nullptr,
                                                             offsets, base, pairs);
            SLM_LAUNCHED("k_flank_paths");
            SLM_CUDA(cudaMemsetAsync(words + 1, 0, sizeof(uint32_t), SS));
            k_flank_settle<ContigPath><<<grid, 256, 0, SS>>>(*p, a, m, side, offsets, base, nullptr, nullptr,
                                                             pairs, hpix, stop, mapping, pix, label, resolved,
                                                             words + 1, words + 2);
            SLM_LAUNCHED("k_flank_settle");
        }
        uint32_t st = 0;
        SLM_CUDA(cudaMemcpyAsync(&st, words + 2, sizeof(uint32_t), cudaMemcpyDeviceToHost, SS));
        SLM_CUDA(cudaStreamSynchronize(SS));
        if (st == 0u) return SLM_OK;
        rc = flank_restart(label, label_init, resolved, n, nxy, SS);
        if (rc) return rc;
    }
    // 3. Rounds; they keep counting across chunks, so owners of earlier
    //    chunks count as resolved before.
    uint32_t round = 1;
    for (const auto& c : chunks) {
        const uint32_t a = c.first, m = c.second - c.first;
        u64 base = 0;
        SLM_CUDA(cudaMemcpyAsync(&base, offsets + a, sizeof(u64), cudaMemcpyDeviceToHost, SS));
        SLM_CUDA(cudaStreamSynchronize(SS));
        k_flank_paths<<<blocks_for(m, 128), 128, 0, SS>>>(*p, a, m, F2(seed_point), stop, F2(uv), nullptr,
                                                         offsets, base, pairs);
        SLM_LAUNCHED("k_flank_paths");
        uint32_t done = 0;
        for (uint32_t r0 = round; done < m; ++round) {
            if (round - r0 > m + 1) {
                set_error("fix flanks did not resolve within %u rounds", m + 1);
                return SLM_ERR_ITERATION_CAP;
            }
            SLM_CUDA(cudaMemsetAsync(words, 0, sizeof(uint32_t), SS));
            k_flank_round<<<blocks_for(m, 256), 256, 0, SS>>>(*p, a, m, side, round, offsets, base, pairs, hpix,
                                                             mask, mapping, owner, label_init, label, resolved,
                                                             words);
            SLM_LAUNCHED("k_flank_round");
            uint32_t newly = 0;
            SLM_CUDA(cudaMemcpyAsync(&newly, words, sizeof(uint32_t), cudaMemcpyDeviceToHost, SS));
            SLM_CUDA(cudaStreamSynchronize(SS));
            if (newly == 0) {
                set_error("fix flanks round %u resolved nothing", round);
                return SLM_ERR_ITERATION_CAP;
            }
            done += newly;
        }
    }
    return SLM_OK;
}

int slm_fix_right_flanks(const slm_params* p, uint32_t n, const float* seed_point, const uint8_t* mask,
                         const float* uv, const uint32_t* mapping, const uint32_t* channel_label,
                         const uint32_t* link, uint32_t* label, void* workspace, size_t workspace_bytes,
                         uint64_t* required_bytes, void* stream) {
    (void)channel_label; (void)link;
    return fix_flanks(p, n, seed_point, mask, uv, mapping, label, workspace, workspace_bytes,
                      required_bytes, stream, false);
}

int slm_fix_left_flanks(const slm_params* p, uint32_t n, const float* seed_point, const uint8_t* mask,
                        const float* uv, const uint32_t* mapping, const uint32_t* channel_label,
                        const uint32_t* link, uint32_t* label, void* workspace, size_t workspace_bytes,
                        uint64_t* required_bytes, void* stream) {
    (void)channel_label; (void)link;
    return fix_flanks(p, n, seed_point, mask, uv, mapping, label, workspace, workspace_bytes,
                      required_bytes, stream, true);
}

int slm_hillslopes(const slm_params* p, uint32_t n, const float* seed_point, const uint8_t* mask,
                   const float* uv, const uint32_t* mapping, const uint32_t* count, uint32_t* link,
                   void* stream) {
    (void)mapping; (void)count;
    clear_error();
    int rc = map_checks(p, n, seed_point);
    if (rc) return rc;
    if (n == 0) return SLM_OK;
    k_hillslopes<<<blocks_for(n, 128), 128, 0, SS>>>(*p, n, F2(seed_point), mask, F2(uv), link);
    SLM_LAUNCHED("k_hillslopes");
    return SLM_OK;
}

int slm_thin(uint8_t* image, uint8_t* scratch, uint32_t nx, uint32_t ny, uint32_t max_iter,
             uint32_t* flag, uint32_t* iterations, void* stream) {
    clear_error();
    SLM_REQUIRE(image && scratch && flag, "NULL buffer");
    SLM_REQUIRE((uint64_t)nx * ny < (1ull << 32), "image too large");
    if (iterations) *iterations = 0;
    const uint32_t np_ = nx * ny;
    if (np_ == 0) return SLM_OK;
    uint32_t it = 0;
    for (; it < max_iter; ++it) {
        SLM_CUDA(cudaMemsetAsync(flag, 0, sizeof(uint32_t), SS));
        k_zhang_suen<<<blocks_for(np_, 256), 256, 0, SS>>>(image, scratch, nx, ny, 0, flag);
        SLM_LAUNCHED("k_zhang_suen");
        k_zhang_suen<<<blocks_for(np_, 256), 256, 0, SS>>>(scratch, image, nx, ny, 1, flag);
        SLM_LAUNCHED("k_zhang_suen");
        uint32_t changed = 0;
        SLM_CUDA(cudaMemcpyAsync(&changed, flag, sizeof(uint32_t), cudaMemcpyDeviceToHost, SS));
        SLM_CUDA(cudaStreamSynchronize(SS));
        if (!changed) { ++it; break; }
    }
    if (iterations) *iterations = it;
    return SLM_OK;
}

int slm_hillslope_lengths(const slm_params* p, uint32_t n, const float* seed_point, const uint8_t* mask,
                          const float* uv, const uint32_t* mapping, const uint32_t* label,
                          float* traj_length, void* stream) {
    (void)label;
    clear_error();
    int rc = map_checks(p, n, seed_point);
    if (rc) return rc;
    if (n == 0) return SLM_OK;
    k_hillslope_lengths<<<blocks_for(n, 128), 128, 0, SS>>>(*p, n, F2(seed_point), mask, F2(uv), mapping,
                                                           traj_length);
    SLM_LAUNCHED("k_hillslope_lengths");
    return SLM_OK;
}

}  // extern "C"
