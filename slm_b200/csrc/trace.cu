// trace.cu -- streamline tracing kernels and their C ABI.
//
//   k_fields_plain       one thread per (seed, sub-pixel) trajectory
//   k_fields_persistent  persistent warps; a lane whose trajectory ends takes
//                        the next one from a global work queue, so warps stay
//                        full however uneven the trajectory lengths are
//   k_trajectory         one thread per seed, records char2 steps
//
// Both field kernels produce identical slc/slt: every trajectory is computed
// bit-exactly as the reference's jittered_trajectory
// (opencl/jittertrajectory.cl:42-88) and the per-pixel sums are integer sums,
// independent of order.  Each lane merges consecutive visits to the same pixel
// (a step is at most integrator_step_factor px, so a trajectory usually visits
// a pixel several times in a row) and adds the merged count and length sum
// with one 64-bit atomic each when it moves to another pixel.
#include <cstring>
#include "capi_util.cuh"
#include "trace_common.cuh"


static_assert(sizeof(slm_tile) == 40, "slm_tile layout is part of the ABI");

namespace slm {

// Run-length merge of pixel visits for one lane.
struct Acc {
    uint32_t idx, cnt;
    u64 sum;
};

__device__ __forceinline__ void acc_flush(Acc& a, u64* __restrict__ slc, u64* __restrict__ slt) {
    if (a.cnt) {
        atomicAdd(slt + a.idx, a.sum);
        atomicAdd(slc + a.idx, (u64)a.cnt);
        a.cnt = 0;
    }
}

// writearray.cl:31-40: slt += (uint)(l+0.5), slc += 1
__device__ __forceinline__ void acc_visit(Acc& a, uint32_t idx, float l, u64* __restrict__ slc,
                                          u64* __restrict__ slt) {
    const u64 v = __float2uint_rz(l + 0.5f);
    // only the two atomics of a finished run branch; the bookkeeping is
    // selects, so a warp whose lanes change pixel at different steps runs it
    // once with every lane active
    const bool same = (idx == a.idx) && a.cnt;
    if (!same && a.cnt) {
        atomicAdd(slt + a.idx, a.sum);
        atomicAdd(slc + a.idx, (u64)a.cnt);
    }
    a.cnt = same ? a.cnt + 1u : 1u;
    a.sum = same ? a.sum + v : v;
    a.idx = idx;
}

// State of one jittered field trajectory between steps.
struct FieldLane {
    Vec2 a;
    float l, dt;
    uint32_t n, rng;
    uint32_t item, k;  // queue position and RK steps so far (kept only when recording)
    bool alive;
};

// Begin the trajectory of sub-pixel `sub` (= j*d + i) of the seed at `c`,
// whose RNG stream is that of seed index `rng_idx`
// (integratefields.cl:83-113; jittertrajectory.cl:56-62).  `mask` is the
// grid's own; pixel indices are offset by `base` into slc/slt.
__device__ __forceinline__ void field_init(FieldLane& s, float2 c, uint32_t rng_idx, uint32_t sub,
                                           uint32_t item, const uint8_t* __restrict__ mask,
                                           const slm_params& p, const Geo& g, uint32_t base,
                                           Acc& acc, u64* __restrict__ slc, u64* __restrict__ slt) {
    const uint32_t d = p.subpixel_seed_point_density;
    const uint32_t j = sub / d, i = sub % d;
    s.a.x = c.x + ((float)i * p.subpixel_seed_step - p.subpixel_seed_halfspan);
    s.a.y = c.y + ((float)j * p.subpixel_seed_step - p.subpixel_seed_halfspan);
    s.rng = seed_rng(rng_idx);
    s.l = 0.0f;
    s.dt = g.dt_max;
    s.n = 0;
    s.item = item;
    s.k = 0;
    const uint32_t idx = pixel_of(s.a, p, g);
    const bool masked = __ldg(mask + idx) != 0;
    if (!masked) acc_visit(acc, base + idx, 0.0f, slc, slt);
    s.alive = !masked && (0.0f < p.max_length) && (0u < p.max_n_steps);
}

// queue item -> (queue position, sub-pixel index)
__device__ __forceinline__ void split_item(u64 item, uint32_t dd, uint32_t& pos, uint32_t& sub) {
    if (item < 0x100000000ull) {  // 32-bit division unless the queue is huge
        const uint32_t it = (uint32_t)item;
        pos = it / dd;
        sub = it - pos * dd;
    } else {
        pos = (uint32_t)(item / dd);
        sub = (uint32_t)(item - (u64)pos * dd);
    }
}

// Start trajectory `item` = (seed - seed_begin) * d*d + j*d + i of one grid.
//
// `order` (optional) maps queue positions to seed indices, so trajectories can
// be traced in any order; the RNG stream still follows the seed index, so no
// trajectory changes.
__device__ __forceinline__ void field_start(FieldLane& s, u64 item, uint32_t seed_begin,
                                            const float2* __restrict__ seeds,
                                            const uint32_t* __restrict__ order,
                                            const uint8_t* __restrict__ mask, const slm_params& p,
                                            const Geo& g, Acc& acc, u64* __restrict__ slc,
                                            u64* __restrict__ slt) {
    const uint32_t d = p.subpixel_seed_point_density;
    uint32_t seed_off, sub;
    split_item(item, d * d, seed_off, sub);
    const uint32_t seed_idx = order ? __ldg(order + seed_begin + seed_off) : seed_begin + seed_off;
    field_init(s, __ldg(seeds + seed_idx), seed_idx, sub, (uint32_t)item, mask, p, g, 0u, acc, slc, slt);
}

// One pass of the while loop of jittered_trajectory with
// runge_kutta_step_write_sl_data (rungekutta.cl:163-186).  The Euler branch
// of that loop is unreachable (get_array_idx clamps into the grid).  P2:
// trajectory_resolution and GRID_SCALE are powers of two (slm_pow2_steps).
template <int ORDER, bool P2 = false>
__device__ __forceinline__ void field_step(FieldLane& s, const uint8_t* __restrict__ mask,
                                           const float2* __restrict__ uv, const slm_params& p,
                                           const Geo& g, uint32_t base, Acc& acc,
                                           u64* __restrict__ slc, u64* __restrict__ slt) {
    const Step st = rk_step<ORDER, true, P2>(s.a, s.dt, s.rng, uv, p, g);
    if (__ldg(mask + st.idx)) {
        s.alive = false;
        return;
    }
    const float err = vlen(div_gs<P2>(st.d2.x - st.d1.x, g), div_gs<P2>(st.d2.y - st.d1.y, g));
    const float dl = vlen(st.d2.x, st.d2.y);
    s.a = st.next;
    if (dl < p.integration_halt_threshold) {
        s.l = s.l + dl;
        s.n += 1;
        acc_visit(acc, base + st.idx, s.l, slc, slt);
        s.alive = false;
        return;
    }
    s.dt = next_dt(s.dt, err, p, g);
    s.l = s.l + dl;
    s.n += 1;
    acc_visit(acc, base + st.idx, s.l, slc, slt);
    s.alive = (s.l < p.max_length) && (s.n < p.max_n_steps);
}


// per-trajectory RK step count, saturated to 16 bits, indexed by queue position
template <bool RECORD>
__device__ __forceinline__ void record_end(const FieldLane& s, uint16_t* __restrict__ item_steps) {
    if (RECORD) item_steps[s.item] = (uint16_t)(s.k < 65535u ? s.k : 65535u);
}

__device__ __forceinline__ void warp_add_counters(u64 steps, u64 ntraj, u64* work) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        steps += __shfl_xor_sync(0xffffffffu, steps, o);
        ntraj += __shfl_xor_sync(0xffffffffu, ntraj, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(work + 1, steps);
        atomicAdd(work + 2, ntraj);
    }
}

template <int ORDER, bool RECORD>
__global__ void __launch_bounds__(256)
k_fields_plain(const slm_params p, const float2* __restrict__ seeds, uint32_t seed_begin,
               u64 n_items, const uint8_t* __restrict__ mask, const float2* __restrict__ uv,
               u64* __restrict__ slc, u64* __restrict__ slt, u64* __restrict__ work,
               const uint32_t* __restrict__ order, uint16_t* __restrict__ item_steps) {
    const u64 item = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    u64 steps = 0, ntraj = 0;
    Acc acc{0u, 0u, 0ull};
    const Geo g = geo_of(p);
    if (item < n_items) {
        FieldLane s;
        field_start(s, item, seed_begin, seeds, order, mask, p, g, acc, slc, slt);
        ntraj = 1;
        while (s.alive) {
            field_step<ORDER>(s, mask, uv, p, g, 0u, acc, slc, slt);
            steps++;
            if (RECORD) s.k++;
        }
        record_end<RECORD>(s, item_steps);
        acc_flush(acc, slc, slt);
    }
    warp_add_counters(steps, ntraj, work);
}

// Persistent form: the queue head work[0] must be 0 at launch.  Every loop
// pass either hands queue items to idle lanes or advances every live
// trajectory by one step, and each trajectory ends within max_n_steps steps,
// so the loop ends; the exit test is warp-uniform.
template <int ORDER, bool RECORD>
__global__ void __launch_bounds__(256)
k_fields_persistent(const slm_params p, const float2* __restrict__ seeds, uint32_t seed_begin,
                    u64 n_items, const uint8_t* __restrict__ mask, const float2* __restrict__ uv,
                    u64* __restrict__ slc, u64* __restrict__ slt, u64* __restrict__ work,
                    const uint32_t* __restrict__ order, uint16_t* __restrict__ item_steps,
                    uint32_t refill_min) {
    const unsigned FULL = 0xffffffffu;
    const unsigned lane = threadIdx.x & 31u;
    const Geo g = geo_of(p);
    FieldLane s;
    s.alive = false;
    Acc acc{0u, 0u, 0ull};
    u64 steps = 0, ntraj = 0;
    bool drained = false;
    while (true) {
        if (!drained) {
            const unsigned idle = __ballot_sync(FULL, !s.alive);
            if (idle && (idle == FULL || (uint32_t)__popc(idle) >= refill_min)) {
                const int leader = __ffs(idle) - 1;
                const unsigned n_idle = __popc(idle);
                u64 base = 0;
                if ((int)lane == leader) base = atomicAdd(work, (u64)n_idle);
                base = __shfl_sync(FULL, base, leader);
                if (base + n_idle >= n_items) drained = true;
                if (!s.alive) {
                    const u64 item = base + __popc(idle & ((1u << lane) - 1u));
                    if (item < n_items) {
                        field_start(s, item, seed_begin, seeds, order, mask, p, g, acc, slc, slt);
                        ntraj++;
                        if (!s.alive) record_end<RECORD>(s, item_steps);
                    }
                }
            }
        }
        if (!__any_sync(FULL, s.alive)) {
            if (drained) break;
            continue;
        }
        if (s.alive) {
            field_step<ORDER>(s, mask, uv, p, g, 0u, acc, slc, slt);
            steps++;
            if (RECORD) {
                s.k++;
                if (!s.alive) record_end<RECORD>(s, item_steps);
            }
        }
    }
    acc_flush(acc, slc, slt);
    warp_add_counters(steps, ntraj, work);
}

// ------------------------------------------------------------------ both directions
// Both directions of one grid in one persistent launch: queue items
// [0, n) trace downstream, [n, 2n) upstream, so the long trajectories that end
// one direction run alongside the other direction's bulk instead of as its
// own tail.  A lane keeps its trajectory's COMBO_FACTOR (the only per-
// direction value of the step) and its accumulator offset (0, or up_stride
// for the upstream slc/slt); every trajectory is the single-direction
// kernels'.
template <int ORDER, bool P2>
__global__ void __launch_bounds__(256)
k_fields_pair(const slm_params p, float cf_up, const float2* __restrict__ seeds, uint32_t seed_begin,
              u64 n_items, const uint8_t* __restrict__ mask, const float2* __restrict__ uv,
              u64* __restrict__ slc, u64* __restrict__ slt, uint32_t up_stride, u64* __restrict__ work,
              const uint32_t* __restrict__ order, const uint32_t* __restrict__ order_up,
              uint32_t refill_min) {
    const unsigned FULL = 0xffffffffu;
    const unsigned lane = threadIdx.x & 31u;
    const uint32_t dd = p.subpixel_seed_point_density * p.subpixel_seed_point_density;
    const Geo g_down = geo_of(p);
    Geo g_up = g_down;
    g_up.cf = cf_up;
    const u64 n_total = 2 * n_items;
    FieldLane s;
    s.alive = false;
    bool up = false;
    uint32_t base = 0;
    Acc acc{0u, 0u, 0ull};
    u64 steps = 0, ntraj = 0, steps_up = 0;
    bool drained = false;
    while (true) {
        if (!drained) {
            const unsigned idle = __ballot_sync(FULL, !s.alive);
            if (idle && (idle == FULL || (uint32_t)__popc(idle) >= refill_min)) {
                const int leader = __ffs(idle) - 1;
                const unsigned n_idle = __popc(idle);
                u64 head = 0;
                if ((int)lane == leader) head = atomicAdd(work, (u64)n_idle);
                head = __shfl_sync(FULL, head, leader);
                if (head + n_idle >= n_total) drained = true;
                if (!s.alive) {
                    u64 item = head + __popc(idle & ((1u << lane) - 1u));
                    if (item < n_total) {
                        up = item >= n_items;
                        if (up) item -= n_items;
                        base = up ? up_stride : 0u;
                        uint32_t pos, sub;
                        split_item(item, dd, pos, sub);
                        const uint32_t* o = up ? order_up : order;
                        const uint32_t seed_idx = o ? __ldg(o + seed_begin + pos) : seed_begin + pos;
                        field_init(s, __ldg(seeds + seed_idx), seed_idx, sub, (uint32_t)item, mask, p,
                                   up ? g_up : g_down, base, acc, slc, slt);
                        ntraj++;
                    }
                }
            }
        }
        if (!__any_sync(FULL, s.alive)) {
            if (drained) break;
            continue;
        }
        if (s.alive) {
            field_step<ORDER, P2>(s, mask, uv, p, up ? g_up : g_down, base, acc, slc, slt);
            steps++;
            steps_up += up;
        }
    }
    acc_flush(acc, slc, slt);
    warp_add_counters(steps, ntraj, work);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) steps_up += __shfl_xor_sync(FULL, steps_up, o);
    if (lane == 0) atomicAdd(work + 3, steps_up);
}

// ------------------------------------------------------------------ batched tiles
// Last tile whose first seed is <= x (tiles sorted by seed_begin; the host
// checks the table), found by binary search over the L1-cached table.
__device__ __forceinline__ uint32_t find_tile(const slm_tile* __restrict__ tiles, uint32_t n_tiles,
                                              uint32_t x) {
    uint32_t lo = 0, hi = n_tiles;
    while (hi - lo > 1u) {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldg(&tiles[mid].seed_begin) <= x) lo = mid;
        else hi = mid;
    }
    return lo;
}

// Many grids (DTM tiles of any sizes) in one persistent launch.  The queue
// runs over every trajectory of every tile; a lane that takes an item looks up
// its tile and keeps the tile's geometry (Geo) and pixel base with its
// trajectory, so lanes of one warp may trace different tiles.  Each
// trajectory is computed exactly as a single-grid launch on its tile computes
// it (RNG stream of the tile-local seed index).  work[3] receives 1 if a seed
// falls outside its tile's range (an inconsistent table).
template <int ORDER, bool RECORD>
__global__ void __launch_bounds__(256, 5)
k_fields_batched(const slm_params p, const slm_tile* __restrict__ tiles, uint32_t n_tiles,
                 const float2* __restrict__ seeds, u64 n_items, const uint8_t* __restrict__ mask,
                 const float2* __restrict__ uv, u64* __restrict__ slc, u64* __restrict__ slt,
                 u64* __restrict__ work, const uint32_t* __restrict__ order,
                 uint16_t* __restrict__ item_steps, uint32_t refill_min) {
    const unsigned FULL = 0xffffffffu;
    const unsigned lane = threadIdx.x & 31u;
    const uint32_t dd = p.subpixel_seed_point_density * p.subpixel_seed_point_density;
    FieldLane s;
    s.alive = false;
    Geo g = make_geo(2u, 2u, 0.0f, 0.0f, 1.0f);
    uint32_t base = 0;
    Acc acc{0u, 0u, 0ull};
    u64 steps = 0, ntraj = 0;
    bool drained = false;
    while (true) {
        if (!drained) {
            const unsigned idle = __ballot_sync(FULL, !s.alive);
            if (idle && (idle == FULL || (uint32_t)__popc(idle) >= refill_min)) {
                const int leader = __ffs(idle) - 1;
                const unsigned n_idle = __popc(idle);
                u64 head = 0;
                if ((int)lane == leader) head = atomicAdd(work, (u64)n_idle);
                head = __shfl_sync(FULL, head, leader);
                if (head + n_idle >= n_items) drained = true;
                if (!s.alive) {
                    const u64 item = head + __popc(idle & ((1u << lane) - 1u));
                    if (item < n_items) {
                        uint32_t pos, sub;
                        split_item(item, dd, pos, sub);
                        const uint32_t seed = order ? __ldg(order + pos) : pos;
                        const uint32_t t = find_tile(tiles, n_tiles, seed);
                        const slm_tile& T = tiles[t];
                        const uint32_t local = seed - __ldg(&T.seed_begin);
                        ntraj++;
                        if (local < __ldg(&T.n_seeds)) {
                            g = make_geo(__ldg(&T.nx_padded), __ldg(&T.ny_padded), __ldg(&T.combo_factor),
                                         __ldg(&T.dt_max), __ldg(&T.grid_scale));
                            base = (uint32_t)__ldg(&T.grid_offset);
                            field_init(s, __ldg(seeds + seed), local, sub, (uint32_t)item, mask + base, p,
                                       g, base, acc, slc, slt);
                        } else {
                            atomicOr(reinterpret_cast<unsigned long long*>(work + 3), 1ull);
                            s.alive = false;
                            s.item = (uint32_t)item;
                            s.k = 0;
                        }
                        if (!s.alive) record_end<RECORD>(s, item_steps);
                    }
                }
            }
        }
        if (!__any_sync(FULL, s.alive)) {
            if (drained) break;
            continue;
        }
        if (s.alive) {
            field_step<ORDER>(s, mask + base, uv + base, p, g, base, acc, slc, slt);
            steps++;
            if (RECORD) {
                s.k++;
                if (!s.alive) record_end<RECORD>(s, item_steps);
            }
        }
    }
    acc_flush(acc, slc, slt);
    warp_add_counters(steps, ntraj, work);
}

// ------------------------------------------------------------------ trajectories
__device__ __forceinline__ float edge_dt(float x, float u) {
    float dt = 0.0f;
    const float right = __fdiv_rn((float)__float2int_rz(x + 1.5f) - (x + 0.5f), u);
    const float left = __fdiv_rn(-((x + 0.5f) - (float)__float2int_rz(x + 0.5f)), u);
    if (u > 0.0f) dt = right;
    if (u < 0.0f) dt = left;
    return dt;
}

__device__ __forceinline__ float min_mag(float x, float y) {
    if (fabsf(x) < fabsf(y)) return x;
    if (fabsf(y) < fabsf(x)) return y;
    return fminf(x, y);
}

__device__ __forceinline__ void put_step(int8_t* rec, uint32_t n, float dx, float dy, float res) {
    const uint32_t lo = (uint8_t)cvt_i8(dx * res), hi = (uint8_t)cvt_i8(dy * res);
    reinterpret_cast<uint16_t*>(rec)[n] = (uint16_t)(lo | (hi << 8));
}

// trajectory_record (trajectory.cl:41-80) with runge_kutta_step_record and
// euler_step_record (rungekutta.cl:49-120)
template <int ORDER>
__global__ void __launch_bounds__(128)
k_trajectory(const slm_params p, uint32_t n_chunk, const float2* __restrict__ seeds,
             const uint8_t* __restrict__ mask, const float2* __restrict__ uv,
             int8_t* __restrict__ traj, uint16_t* __restrict__ nsteps_out,
             float* __restrict__ length_out) {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n_chunk) return;
    const uint32_t seed_idx = p.seeds_chunk_offset + g;
    if (seed_idx >= p.n_seed_points) return;
    int8_t* rec = traj + 2ull * g * p.max_n_steps;
    const float res = (float)p.trajectory_resolution;
    const float2 c = __ldg(seeds + seed_idx);
    Vec2 a{c.x, c.y}, prev = a;
    uint32_t n = 0, rng = 0;
    float l = 0.0f, dt = p.dt_max;
    const Geo geo = geo_of(p);
    uint32_t idx = pixel_of(a, p, geo);
    while (!__ldg(mask + idx) && (l < p.max_length && n < p.max_n_steps)) {
        const Step st = rk_step<ORDER, false>(a, dt, rng, uv, p, geo);
        idx = st.idx;
        if (!__ldg(mask + idx)) {
            const float err = vlen(div_gs(st.d2.x - st.d1.x, geo), div_gs(st.d2.y - st.d1.y, geo));
            Vec2 next = st.next;
            float dl = vlen(st.d2.x, st.d2.y);
            if (dl < p.integration_halt_threshold) {
                next.x = a.x + st.d1.x;
                next.y = a.y + st.d1.y;
                dl = vlen(st.d1.x, st.d1.y);
            }
            a = next;
            idx = pixel_of(next, p, geo);
            const bool stuck = dl < p.integration_halt_threshold;
            if (!stuck) dt = next_dt(dt, err, p, geo);
            l = l + dl;
            put_step(rec, n, a.x - prev.x, a.y - prev.y, res);
            n++;
            if (stuck) break;
            prev = a;
        } else {
            // DOWNUP_SIGN is an unsigned literal: upstream it widens to 4294967296.0f
            const float sg = __uint2float_rn(p.downup_sign);
            const float sx = st.u1.x * sg, sy = st.u1.y * sg;
            const float dtx = edge_dt(a.x, sx), dty = edge_dt(a.y, sy);
            dt = min_mag(dtx, dty);
            a.x = a.x + sx * dt;
            a.y = a.y + sy * dt;
            a.x = quant(a.x, res);
            a.y = quant(a.y, res);
            a.x = fminf(fmaxf(a.x, -0.5f), p.nxf_mp5);
            a.y = fminf(fmaxf(a.y, -0.5f), p.nyf_mp5);
            const float dl = vlen(a.x - prev.x, a.y - prev.y);
            l = l + dl;
            put_step(rec, n, a.x - prev.x, a.y - prev.y, res);
            n++;
            break;
        }
    }
    nsteps_out[g] = (uint16_t)n;
    length_out[g] = l;
}

// ------------------------------------------------------------------ finish
// Fields.integrate's host arithmetic on the raw sums (fields.py:146-167 and
// :293-310), in NumPy's promotion order: per pixel and direction
//   slc  (uint32 wrap of the sum, or float64 of it when exact)
//   slt  float32(slt)                    (exact: float32(float64(sum)))
//   sla  float32(float64(sqrt 2) * slt / slc)       where slc > 0, else 0
//   slt  float32(float64(slt) / d^2)                where slc > 0
//   slt  float32(slt * ds_scale[dir]),  slt = sqrt(slt)
//   slc  sqrt 2 * pow(slc / d^2, 2/3)   (float64; table[slc] when given)
// Outputs are [nxy][2] (direction innermost), as the (nxp, nyp, 2) arrays.
__global__ void k_fields_finish(const u64* __restrict__ acc, uint32_t nxy, uint32_t dd, double ds0,
                                double ds1, int exact, const double* __restrict__ table,
                                uint32_t table_len, double* __restrict__ slc_out,
                                float* __restrict__ slt_out, float* __restrict__ sla_out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nxy) return;
    const double sqrt2 = 1.4142135623730951;  // np.sqrt(2.0), correctly rounded
#pragma unroll
    for (int d = 0; d < 2; ++d) {
        const u64 c64 = acc[(size_t)(2 * d) * nxy + i];
        const u64 t64 = acc[(size_t)(2 * d + 1) * nxy + i];
        double c;
        float t;
        if (exact) {
            c = (double)c64;
            t = (float)(double)t64;
        } else {
            c = (double)(uint32_t)c64;
            t = (float)(uint32_t)t64;
        }
        float a = 0.0f;
        if (c > 0.0) {
            a = (float)((sqrt2 * (double)t) / c);
            t = (float)((double)t / (double)dd);  // d^2 is a uint32 scalar: float64 division
        }
        t = (float)((double)t * (d == 0 ? ds0 : ds1));
        t = sqrtf(t);
        double f;
        if (table && c < (double)table_len) f = table[(uint32_t)c];
        else f = sqrt2 * pow(c / (double)dd, 2.0 / 3.0);
        slc_out[2 * (size_t)i + d] = f;
        slt_out[2 * (size_t)i + d] = t;
        sla_out[2 * (size_t)i + d] = a;
    }
}

}  // namespace slm

using namespace slm;

// True when the step's two power-of-two shortcuts hold for the whole launch:
// trajectory_resolution is a power of two (Quant) and GRID_SCALE is one whose
// reciprocal is a normal float (pow2_reciprocal), the same tests the device
// makes per step; the pair launch then runs the form without them.
static bool pow2_steps(const slm_params& p) {
    const uint32_t r = p.trajectory_resolution;
    uint32_t b;
    std::memcpy(&b, &p.grid_scale, sizeof b);
    const uint32_t e = (b >> 23) & 0xffu;
    const bool gs_pow2 = (b >> 31) == 0u && (b & 0x7fffffu) == 0u && e >= 1u && e <= 253u;
    return r != 0u && (r & (r - 1u)) == 0u && gs_pow2;
}

static int check_grid(const slm_params* p) {
    SLM_REQUIRE(p != nullptr, "params is NULL");
    SLM_REQUIRE(p->nx_padded >= 2 && p->ny_padded >= 2, "grid too small: %u x %u",
                p->nx_padded, p->ny_padded);
    SLM_REQUIRE((u64)p->nx_padded * p->ny_padded == p->nxy_padded,
                "nxy_padded %u != nx_padded*ny_padded", p->nxy_padded);
    SLM_REQUIRE(p->trajectory_resolution > 0, "trajectory_resolution is 0");
    return SLM_OK;
}

// slm_launch.chunk: a warp takes queue items once at least this many of its
// lanes are idle (or all are); 0 selects 4, which measured best on the 2048^2
// and 8192^2 RK4 workloads (fewer refill passes run by one or two lanes).
static uint32_t refill_min(const slm_launch& L) {
    if (L.chunk == 0) return 4u;
    return L.chunk <= 1 ? 1u : (L.chunk >= 32 ? 32u : (uint32_t)L.chunk);
}

template <int ORDER, bool RECORD>
static int launch_fields(const slm_params* p, const slm_launch& L, int block, const float2* sp,
                         uint32_t begin, u64 n_items, const uint8_t* mask, const float2* u2, u64* slc,
                         u64* slt, u64* work, const uint32_t* order, uint16_t* rec, cudaStream_t s) {
    if (L.schedule == SLM_SCHED_PLAIN) {
        const u64 grid = (n_items + block - 1) / block;
        SLM_REQUIRE(grid < (1ull << 31), "too many trajectories for one launch");
        k_fields_plain<ORDER, RECORD><<<(unsigned)grid, block, 0, s>>>(*p, sp, begin, n_items, mask, u2,
                                                                      slc, slt, work, order, rec);
        SLM_LAUNCHED("k_fields_plain");
    } else if (L.schedule == SLM_SCHED_PERSISTENT) {
        int per_sm = L.blocks_per_sm;
        if (per_sm <= 0) {
            int occ = 0;
            SLM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_fields_persistent<ORDER, RECORD>, block, 0));
            per_sm = occ > 0 ? occ : 1;
        }
        const unsigned grid = (unsigned)(num_sms() * per_sm);
        k_fields_persistent<ORDER, RECORD><<<grid, block, 0, s>>>(*p, sp, begin, n_items, mask, u2, slc, slt,
                                                                  work, order, rec, refill_min(L));
        SLM_LAUNCHED("k_fields_persistent");
    } else {
        set_error("unknown schedule %d", L.schedule);
        return SLM_ERR_ARGS;
    }
    return SLM_OK;
}

template <int ORDER, bool RECORD>
static int launch_batched(const slm_params* p, const slm_launch& L, int block, const slm_tile* tiles,
                          uint32_t n_tiles, const float2* sp, u64 n_items, const uint8_t* mask,
                          const float2* u2, u64* slc, u64* slt, u64* work, const uint32_t* order,
                          uint16_t* rec, cudaStream_t s) {
    int per_sm = L.blocks_per_sm;
    if (per_sm <= 0) {
        int occ = 0;
        SLM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_fields_batched<ORDER, RECORD>, block, 0));
        per_sm = occ > 0 ? occ : 1;
    }
    const unsigned grid = (unsigned)(num_sms() * per_sm);
    k_fields_batched<ORDER, RECORD><<<grid, block, 0, s>>>(*p, tiles, n_tiles, sp, n_items, mask, u2, slc, slt,
                                                          work, order, rec, refill_min(L));
    SLM_LAUNCHED("k_fields_batched");
    return SLM_OK;
}

extern "C" {

size_t slm_fields_workspace_words(void) { return 4; }

int slm_integrate_fields(const slm_params* p, const slm_launch* launch, const float* seed_point,
                         const uint8_t* mask, const float* uv, uint32_t* mapping, uint64_t* slc,
                         uint64_t* slt, uint64_t* workspace, void* stream) {
    return slm_integrate_fields_scheduled(p, launch, seed_point, mask, uv, mapping, slc, slt,
                                          workspace, nullptr, nullptr, stream);
}

int slm_integrate_fields_scheduled(const slm_params* p, const slm_launch* launch,
                                   const float* seed_point, const uint8_t* mask, const float* uv,
                                   uint32_t* mapping, uint64_t* slc, uint64_t* slt,
                                   uint64_t* workspace, const uint32_t* seed_order,
                                   uint16_t* item_steps, void* stream) {
    (void)mapping;
    clear_error();
    int rc = check_grid(p);
    if (rc) return rc;
    SLM_REQUIRE(seed_point && mask && uv && slc && slt && workspace, "NULL buffer");
    SLM_REQUIRE(aligned(uv, 8) && aligned(seed_point, 8), "uv/seed_point must be 8-byte aligned");
    SLM_REQUIRE(aligned(slc, 8) && aligned(slt, 8) && aligned(workspace, 8),
                "slc/slt/workspace must be 8-byte aligned");
    SLM_REQUIRE(p->subpixel_seed_point_density >= 1, "subpixel_seed_point_density is 0");
    slm_launch def{SLM_SCHED_PERSISTENT, SLM_RK2, 256, 0, 0, {0, 0, 0}};
    const slm_launch& L = launch ? *launch : def;
    SLM_REQUIRE(L.integrator == SLM_RK2 || L.integrator == SLM_RK4, "integrator must be 2 or 4");
    const int block = L.block_threads > 0 ? L.block_threads : 256;
    SLM_REQUIRE(block % 32 == 0 && block <= 256, "block_threads must be a multiple of 32, <= 256");
    cudaStream_t s = (cudaStream_t)stream;
    SLM_CUDA(cudaMemsetAsync(workspace, 0, slm_fields_workspace_words() * sizeof(uint64_t), s));
    const uint32_t begin = p->seeds_chunk_offset;
    if (begin >= p->n_seed_points) return SLM_OK;
    const u64 dd = (u64)p->subpixel_seed_point_density * p->subpixel_seed_point_density;
    const u64 n_items = (u64)(p->n_seed_points - begin) * dd;
    SLM_REQUIRE(!item_steps || n_items < (1ull << 32), "step recording needs fewer than 2^32 trajectories");
    const float2* sp = reinterpret_cast<const float2*>(seed_point);
    const float2* u2 = reinterpret_cast<const float2*>(uv);
    u64* w = (u64*)workspace;
    if (L.integrator == SLM_RK4)
        return item_steps ? launch_fields<4, true>(p, L, block, sp, begin, n_items, mask, u2, (u64*)slc, (u64*)slt, w, seed_order, item_steps, s)
                          : launch_fields<4, false>(p, L, block, sp, begin, n_items, mask, u2, (u64*)slc, (u64*)slt, w, seed_order, nullptr, s);
    return item_steps ? launch_fields<2, true>(p, L, block, sp, begin, n_items, mask, u2, (u64*)slc, (u64*)slt, w, seed_order, item_steps, s)
                      : launch_fields<2, false>(p, L, block, sp, begin, n_items, mask, u2, (u64*)slc, (u64*)slt, w, seed_order, nullptr, s);
}

int slm_integrate_fields_pair(const slm_params* p_down, const slm_params* p_up, const slm_launch* launch,
                              const float* seed_point, const uint8_t* mask, const float* uv, uint64_t* slc,
                              uint64_t* slt, uint64_t up_stride, uint64_t* workspace, const uint32_t* seed_order,
                              const uint32_t* seed_order_up, void* stream) {
    clear_error();
    int rc = check_grid(p_down);
    if (rc) return rc;
    SLM_REQUIRE(p_up != nullptr, "params is NULL");
    // the two parameter blocks may differ only in the direction
    SLM_REQUIRE(p_up->nxy_padded == p_down->nxy_padded && p_up->nx_padded == p_down->nx_padded &&
                p_up->n_seed_points == p_down->n_seed_points &&
                p_up->seeds_chunk_offset == p_down->seeds_chunk_offset &&
                p_up->subpixel_seed_point_density == p_down->subpixel_seed_point_density &&
                p_up->max_n_steps == p_down->max_n_steps && p_up->max_length == p_down->max_length &&
                p_up->dt_max == p_down->dt_max && p_up->grid_scale == p_down->grid_scale &&
                p_up->combo_factor == -p_down->combo_factor,
                "downstream and upstream parameters differ in more than the direction");
    SLM_REQUIRE(seed_point && mask && uv && slc && slt && workspace, "NULL buffer");
    SLM_REQUIRE(aligned(uv, 8) && aligned(seed_point, 8), "uv/seed_point must be 8-byte aligned");
    SLM_REQUIRE(aligned(slc, 8) && aligned(slt, 8) && aligned(workspace, 8),
                "slc/slt/workspace must be 8-byte aligned");
    SLM_REQUIRE(up_stride >= p_down->nxy_padded && up_stride + p_down->nxy_padded < (1ull << 32),
                "up_stride must be >= nxy_padded and leave the upstream arrays below 2^32 elements");
    SLM_REQUIRE(p_down->subpixel_seed_point_density >= 1, "subpixel_seed_point_density is 0");
    slm_launch def{SLM_SCHED_PERSISTENT, SLM_RK2, 256, 0, 0, {0, 0, 0}};
    const slm_launch& L = launch ? *launch : def;
    SLM_REQUIRE(L.schedule == SLM_SCHED_PERSISTENT, "the pair form runs the persistent schedule");
    SLM_REQUIRE(L.integrator == SLM_RK2 || L.integrator == SLM_RK4, "integrator must be 2 or 4");
    const int block = L.block_threads > 0 ? L.block_threads : 256;
    SLM_REQUIRE(block % 32 == 0 && block <= 256, "block_threads must be a multiple of 32, <= 256");
    cudaStream_t s = (cudaStream_t)stream;
    SLM_CUDA(cudaMemsetAsync(workspace, 0, slm_fields_workspace_words() * sizeof(uint64_t), s));
    const uint32_t begin = p_down->seeds_chunk_offset;
    if (begin >= p_down->n_seed_points) return SLM_OK;
    const u64 dd = (u64)p_down->subpixel_seed_point_density * p_down->subpixel_seed_point_density;
    const u64 n_items = (u64)(p_down->n_seed_points - begin) * dd;
    const float2* sp = reinterpret_cast<const float2*>(seed_point);
    const float2* u2 = reinterpret_cast<const float2*>(uv);
    const bool p2 = pow2_steps(*p_down);
    int per_sm = L.blocks_per_sm;
    if (per_sm <= 0) {
        int occ = 0;
        const void* fn = L.integrator == SLM_RK4 ? (p2 ? (const void*)k_fields_pair<4, true>
                                                       : (const void*)k_fields_pair<4, false>)
                                                 : (p2 ? (const void*)k_fields_pair<2, true>
                                                       : (const void*)k_fields_pair<2, false>);
        SLM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, block, 0));
        per_sm = occ > 0 ? occ : 1;
    }
    const unsigned grid = (unsigned)(num_sms() * per_sm);
    const uint32_t* o_up = seed_order_up ? seed_order_up : seed_order;
#define SLM_PAIR_LAUNCH(ORD, P2)                                                                          \
    k_fields_pair<ORD, P2><<<grid, block, 0, s>>>(*p_down, p_up->combo_factor, sp, begin, n_items, mask, u2, \
                                                  (u64*)slc, (u64*)slt, (uint32_t)up_stride,              \
                                                  (u64*)workspace, seed_order, o_up, refill_min(L))
    if (L.integrator == SLM_RK4) {
        if (p2) SLM_PAIR_LAUNCH(4, true);
        else SLM_PAIR_LAUNCH(4, false);
    } else {
        if (p2) SLM_PAIR_LAUNCH(2, true);
        else SLM_PAIR_LAUNCH(2, false);
    }
#undef SLM_PAIR_LAUNCH
    SLM_LAUNCHED("k_fields_pair");
    return SLM_OK;
}

int slm_integrate_fields_batched(const slm_params* p, const slm_launch* launch, const slm_tile* tiles,
                                 uint32_t n_tiles, uint32_t n_seeds, const float* seed_point,
                                 const uint8_t* mask, const float* uv, uint64_t* slc, uint64_t* slt,
                                 uint64_t* workspace, const uint32_t* seed_order, uint16_t* item_steps,
                                 void* stream) {
    clear_error();
    SLM_REQUIRE(p != nullptr, "params is NULL");
    SLM_REQUIRE(tiles && n_tiles >= 1, "no tiles");
    SLM_REQUIRE(seed_point && mask && uv && slc && slt && workspace, "NULL buffer");
    SLM_REQUIRE(aligned(uv, 8) && aligned(seed_point, 8) && aligned(tiles, 8),
                "uv/seed_point/tiles must be 8-byte aligned");
    SLM_REQUIRE(aligned(slc, 8) && aligned(slt, 8) && aligned(workspace, 8),
                "slc/slt/workspace must be 8-byte aligned");
    SLM_REQUIRE(p->subpixel_seed_point_density >= 1, "subpixel_seed_point_density is 0");
    SLM_REQUIRE(p->trajectory_resolution > 0, "trajectory_resolution is 0");
    slm_launch def{SLM_SCHED_PERSISTENT, SLM_RK2, 256, 0, 0, {0, 0, 0}};
    const slm_launch& L = launch ? *launch : def;
    SLM_REQUIRE(L.schedule == SLM_SCHED_PERSISTENT, "batched tracing runs the persistent schedule");
    SLM_REQUIRE(L.integrator == SLM_RK2 || L.integrator == SLM_RK4, "integrator must be 2 or 4");
    const int block = L.block_threads > 0 ? L.block_threads : 256;
    SLM_REQUIRE(block % 32 == 0 && block <= 256, "block_threads must be a multiple of 32, <= 256");
    cudaStream_t s = (cudaStream_t)stream;
    SLM_CUDA(cudaMemsetAsync(workspace, 0, slm_fields_workspace_words() * sizeof(uint64_t), s));
    if (n_seeds == 0) return SLM_OK;
    const u64 dd = (u64)p->subpixel_seed_point_density * p->subpixel_seed_point_density;
    const u64 n_items = (u64)n_seeds * dd;
    SLM_REQUIRE(!item_steps || n_items < (1ull << 32), "step recording needs fewer than 2^32 trajectories");
    const float2* sp = reinterpret_cast<const float2*>(seed_point);
    const float2* u2 = reinterpret_cast<const float2*>(uv);
    u64* w = (u64*)workspace;
    if (L.integrator == SLM_RK4)
        return item_steps ? launch_batched<4, true>(p, L, block, tiles, n_tiles, sp, n_items, mask, u2, (u64*)slc, (u64*)slt, w, seed_order, item_steps, s)
                          : launch_batched<4, false>(p, L, block, tiles, n_tiles, sp, n_items, mask, u2, (u64*)slc, (u64*)slt, w, seed_order, nullptr, s);
    return item_steps ? launch_batched<2, true>(p, L, block, tiles, n_tiles, sp, n_items, mask, u2, (u64*)slc, (u64*)slt, w, seed_order, item_steps, s)
                      : launch_batched<2, false>(p, L, block, tiles, n_tiles, sp, n_items, mask, u2, (u64*)slc, (u64*)slt, w, seed_order, nullptr, s);
}

int slm_fields_finish(const uint64_t* acc, uint32_t nxy_padded, uint32_t density, double ds_scale_down,
                      double ds_scale_up, int exact, const double* slc_table, uint32_t table_len,
                      double* slc_out, float* slt_out, float* sla_out, void* stream) {
    clear_error();
    if (nxy_padded == 0) return SLM_OK;
    SLM_REQUIRE(acc && slc_out && slt_out && sla_out, "NULL buffer");
    SLM_REQUIRE(density >= 1, "density is 0");
    SLM_REQUIRE(aligned(acc, 8) && aligned(slc_out, 8) && aligned(slt_out, 4) && aligned(sla_out, 4),
                "misaligned buffer");
    k_fields_finish<<<(nxy_padded + 255) / 256, 256, 0, (cudaStream_t)stream>>>(
        (const u64*)acc, nxy_padded, density * density, ds_scale_down, ds_scale_up, exact, slc_table,
        slc_table ? table_len : 0u, slc_out, slt_out, sla_out);
    SLM_LAUNCHED("k_fields_finish");
    return SLM_OK;
}

int slm_integrate_trajectory(const slm_params* p, int32_t integrator, uint32_t n_chunk,
                             const float* seed_point, const uint8_t* mask, const float* uv,
                             uint32_t* mapping, int8_t* trajectories, uint16_t* nsteps,
                             float* length, void* stream) {
    (void)mapping;
    clear_error();
    int rc = check_grid(p);
    if (rc) return rc;
    SLM_REQUIRE(integrator == SLM_RK2 || integrator == SLM_RK4, "integrator must be 2 or 4");
    if (n_chunk == 0) return SLM_OK;
    SLM_REQUIRE(seed_point && mask && uv && trajectories && nsteps && length, "NULL buffer");
    SLM_REQUIRE(aligned(uv, 8) && aligned(seed_point, 8), "uv/seed_point must be 8-byte aligned");
    SLM_REQUIRE(aligned(trajectories, 2) && aligned(nsteps, 2) && aligned(length, 4),
                "trajectory buffers misaligned");
    cudaStream_t s = (cudaStream_t)stream;
    const unsigned block = 128, grid = (n_chunk + block - 1) / block;
    const float2* sp = reinterpret_cast<const float2*>(seed_point);
    const float2* u2 = reinterpret_cast<const float2*>(uv);
    if (integrator == SLM_RK4)
        k_trajectory<4><<<grid, block, 0, s>>>(*p, n_chunk, sp, mask, u2, trajectories, nsteps, length);
    else
        k_trajectory<2><<<grid, block, 0, s>>>(*p, n_chunk, sp, mask, u2, trajectories, nsteps, length);
    SLM_LAUNCHED("k_trajectory");
    return SLM_OK;
}

}  // extern "C"

// ------------------------------------------------------------------ no-alloc variant
// Some callers cannot call cudaMalloc: a host application that hands a plugin
// only its own pre-allocated buffers, or a binding of the reference's
// six-buffer integrate_fields signature, which has no workspace argument.
// For them, slm_integrate_fields_noalloc keeps the field tracer's scratch (the
// work-queue head and the step/trajectory counters) in the file-scope device
// array below instead of a caller-allocated workspace.  The array is modest
// (SLM_NOALLOC_SCRATCH_WORDS 64-bit words, 512 bytes) and every GPU that loads
// this library holds it until the process exits.
namespace slm {

static __device__ __align__(256) unsigned long long g_noalloc_scratch[SLM_NOALLOC_SCRATCH_WORDS];

// Device address of g_noalloc_scratch in the current context.  In host code
// the array's name is only a host-side stand-in, so the address comes from
// cudaGetSymbolAddress.  It is looked up on every call (a cheap query) rather
// than cached: an address belongs to the context the module was loaded in, and
// a cached one would go stale after cudaDeviceReset or in a caller's own
// context.
static int noalloc_scratch(u64** out) {
    void* ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess) {
        int dev = -1;
        cudaGetDevice(&dev);
        set_error("cudaGetSymbolAddress(scratch) failed on device %d: %s", dev, cudaGetErrorString(e));
        return SLM_ERR_CUDA;
    }
    *out = static_cast<u64*>(ptr);
    return SLM_OK;
}

}  // namespace slm

extern "C" int slm_integrate_fields_noalloc(const slm_params* p, const slm_launch* launch,
                                            const float* seed_point, const uint8_t* mask,
                                            const float* uv, uint32_t* mapping, uint64_t* slc,
                                            uint64_t* slt, void* stream) {
    clear_error();
    const size_t need = slm_fields_workspace_words();
    if (need > SLM_NOALLOC_SCRATCH_WORDS) {
        set_error("field tracer needs %zu scratch words, the static array holds %d",
                  need, SLM_NOALLOC_SCRATCH_WORDS);
        return SLM_ERR_CAPACITY;
    }
    u64* scratch = nullptr;
    int rc = noalloc_scratch(&scratch);
    if (rc) return rc;
    // slm_integrate_fields clears the scratch words it uses (queue head and
    // counters) on the stream before its launch, so a previous call's contents
    // never leak into this one.
    return slm_integrate_fields(p, launch, seed_point, mask, uv, mapping, slc, slt,
                                reinterpret_cast<uint64_t*>(scratch), stream);
}

// ------------------------------------------------------------------ self-test
namespace slm {
// counts[0] += inputs whose div6 differs from the IEEE quotient (NaN equals
// NaN); counts[1] = the largest such input bit pattern + 1 (0: none)
__global__ void k_selftest_div6(u64* counts) {
    u64 bad = 0, last = 0;
    for (u64 b = (u64)blockIdx.x * blockDim.x + threadIdx.x; b < (1ull << 32); b += (u64)gridDim.x * blockDim.x) {
        const float x = __uint_as_float((uint32_t)b);
        const float want = __fdiv_rn(x, 6.0f), got = div6(x);
        const bool same = __float_as_uint(want) == __float_as_uint(got) || (want != want && got != got);
        if (!same) {
            bad++;
            last = b + 1;
        }
    }
    if (bad) {
        atomicAdd(counts, bad);
        atomicMax(counts + 1, last);
    }
}
}  // namespace slm

// counts[0] += inputs whose cvt_i8 differs from the x86 conversion the
// reference's float -> char follows (cvttss2si: truncation in range, INT32_MIN
// for NaN and out of range; the low byte kept); counts[1] as for div6
__global__ void k_selftest_cvt_i8(u64* counts) {
    u64 bad = 0, last = 0;
    for (u64 b = (u64)blockIdx.x * blockDim.x + threadIdx.x; b < (1ull << 32); b += (u64)gridDim.x * blockDim.x) {
        const float x = __uint_as_float((uint32_t)b);
        int32_t w = (int32_t)0x80000000;
        if (x >= -2147483648.0f && x < 2147483648.0f) w = __float2int_rz(x);
        if ((int8_t)(w & 0xff) != cvt_i8(x)) {
            bad++;
            last = b + 1;
        }
    }
    if (bad) {
        atomicAdd(counts, bad);
        atomicMax(counts + 1, last);
    }
}

extern "C" int slm_selftest_div6(uint64_t* counts, void* stream) {
    clear_error();
    SLM_REQUIRE(counts && aligned(counts, 8), "counts must be two 8-byte aligned device words");
    cudaStream_t s = (cudaStream_t)stream;
    SLM_CUDA(cudaMemsetAsync(counts, 0, 2 * sizeof(uint64_t), s));
    k_selftest_div6<<<(unsigned)(num_sms() * 8), 256, 0, s>>>((u64*)counts);
    SLM_LAUNCHED("k_selftest_div6");
    return SLM_OK;
}

extern "C" int slm_selftest_cvt_i8(uint64_t* counts, void* stream) {
    clear_error();
    SLM_REQUIRE(counts && aligned(counts, 8), "counts must be two 8-byte aligned device words");
    cudaStream_t s = (cudaStream_t)stream;
    SLM_CUDA(cudaMemsetAsync(counts, 0, 2 * sizeof(uint64_t), s));
    k_selftest_cvt_i8<<<(unsigned)(num_sms() * 8), 256, 0, s>>>((u64*)counts);
    SLM_LAUNCHED("k_selftest_cvt_i8");
    return SLM_OK;
}
