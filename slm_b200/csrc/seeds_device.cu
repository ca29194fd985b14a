// seeds_device.cu -- create_seeds' seed list built in device memory.
//
// The same rows in the same order as slm_create_seeds (argwhere(~mask) - pad,
// then NumPy's legacy np.random.shuffle after np.random.seed(rng_seed);
// useful.py:470-517), without the host's random-access pass over the rows:
//
//   1. argwhere: slm_pick_seeds' order-preserving compaction of the mask;
//   2. the swap partners j(i), i = n-1 .. 1: drawn on the host with the
//      generator of slm_create_seeds (mt19937.hpp) by a drawing thread,
//      and copied to the device in chunks of SWAP_CHUNK as they become final;
//   3. the swaps, chunk by chunk while the next chunk is drawn.  A chunk holds
//      the next swaps in sequential order (i from high to low), and every
//      earlier chunk's swaps are done before it starts.  Within a chunk:  Fisher-Yates applies swap(i, j(i)) for i = n-1 down to 1,
//      and the value a row ends with depends only on the swaps that touch it,
//      taken in that order.  So the swaps run in rounds: every pending swap
//      reserves its two rows with atomicMax of (round, i); a swap that holds
//      the reservation of both rows is the earliest pending swap on each, so
//      every earlier swap on those rows is done and it runs now; the others
//      wait for the next round.  Each row sees its swaps in the sequential
//      order, so the rows end as the sequential shuffle leaves them (the
//      reservation schedule of Shun, Gu, Blelloch, Fineman and Gibbons,
//      "Sequential random permutation, list contraction and tree contraction
//      are highly parallel", SODA 2015, who show that O(log n) rounds suffice
//      with high probability).  The latest pending swap always runs, so the
//      rounds end within n.
#include <atomic>
#include <chrono>
#include <thread>
#include <vector>

#include "capi_util.cuh"
#include "mt19937.hpp"

namespace slm {

typedef unsigned long long u64;

// swaps per chunk of the pipelined shuffle
constexpr uint32_t SWAP_CHUNK = 1u << 22;

// every pending swap i (list[k], or first + k in a chunk's first round, when
// list is NULL) reserves rows i and j(i) with (round << 32) | i; rounds are
// numbered across chunks, so a reservation left by an earlier chunk is
// always below the current round's
__global__ void k_fy_reserve(const uint32_t* __restrict__ js, const uint32_t* __restrict__ list, uint32_t first,
                             uint32_t count, u64 tag, u64* __restrict__ res) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x) {
        const uint32_t i = list ? list[k] : first + k;
        const u64 v = tag | i;
        atomicMax(res + i, v);
        atomicMax(res + js[i], v);
    }
}

// a swap holding both reservations runs; the others go to the next list
__global__ void k_fy_commit(const uint32_t* __restrict__ js, const uint32_t* __restrict__ list, uint32_t first,
                            uint32_t count, u64 tag, const u64* __restrict__ res, float2* __restrict__ rows,
                            uint32_t* __restrict__ next, uint32_t* __restrict__ n_next) {
    const unsigned FULL = 0xffffffffu;
    const unsigned lane = threadIdx.x & 31u;
    // the loop bound is uniform over the block, so whole warps iterate together
    for (uint32_t k0 = blockIdx.x * blockDim.x; k0 < count; k0 += gridDim.x * blockDim.x) {
        const uint32_t k = k0 + threadIdx.x;
        bool wait = false;
        uint32_t i = 0;
        if (k < count) {
            i = list ? list[k] : first + k;
            const uint32_t j = js[i];
            const u64 v = tag | i;
            if (res[i] == v && res[j] == v) {
                if (i != j) {
                    const float2 a = rows[i], b = rows[j];
                    rows[i] = b;
                    rows[j] = a;
                }
            } else {
                wait = true;
            }
        }
        const unsigned m = __ballot_sync(FULL, wait);
        if (m) {
            const int leader = __ffs(m) - 1;
            uint32_t base = 0;
            if ((int)lane == leader) base = atomicAdd(n_next, (uint32_t)__popc(m));
            base = __shfl_sync(FULL, base, leader);
            if (wait) next[base + __popc(m & ((1u << lane) - 1u))] = i;
        }
    }
}

static size_t up256(size_t b) { return (b + 255) & ~(size_t)255; }

// The swaps i = hi .. lo (js already on the device) in reservation rounds,
// numbered on from *round.
static int run_swaps(const uint32_t* js_d, u64* res, float2* rows, uint32_t* list_a, uint32_t* list_b,
                     uint32_t* n_next, uint32_t lo, uint32_t hi, u64* round, u64 round_cap, cudaStream_t s) {
    const uint32_t* list = nullptr;  // first round: every swap lo .. hi
    uint32_t* next = list_a;
    uint32_t count = hi - lo + 1u;
    const uint32_t max_grid = (uint32_t)num_sms() * 8u;
    while (count > 0) {
        const u64 r = ++*round;
        if (r > round_cap) {
            set_error("shuffle rounds exceeded %llu", (unsigned long long)round_cap);
            return SLM_ERR_ITERATION_CAP;
        }
        const u64 tag = r << 32;
        const uint32_t want = (count + 255u) / 256u;
        const unsigned grid = want < max_grid ? want : max_grid;
        SLM_CUDA(cudaMemsetAsync(n_next, 0, sizeof(uint32_t), s));
        k_fy_reserve<<<grid, 256, 0, s>>>(js_d, list, lo, count, tag, res);
        SLM_LAUNCHED("k_fy_reserve");
        k_fy_commit<<<grid, 256, 0, s>>>(js_d, list, lo, count, tag, res, rows, next, n_next);
        SLM_LAUNCHED("k_fy_commit");
        uint32_t pending = 0;
        SLM_CUDA(cudaMemcpyAsync(&pending, n_next, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        SLM_CUDA(cudaStreamSynchronize(s));
        if (pending >= count) {
            set_error("shuffle round %llu ran no swap", (unsigned long long)r);
            return SLM_ERR_ITERATION_CAP;
        }
        count = pending;
        list = next;
        next = (next == list_a) ? list_b : list_a;
    }
    return SLM_OK;
}

// Joins the drawing thread on every way out of slm_create_seeds_device.
struct Joiner {
    std::thread t;
    ~Joiner() {
        if (t.joinable()) t.join();
    }
};

}  // namespace slm

using namespace slm;

extern "C" {

size_t slm_create_seeds_device_workspace(uint64_t n_pixels) {
    if (n_pixels == 0 || n_pixels >= (1ull << 32)) return 0;
    const size_t n = (size_t)n_pixels;
    return up256(slm_pick_seeds_workspace((uint32_t)n_pixels)) + up256(4 * n) + up256(8 * n) + 2 * up256(4 * n) +
           256;
}

int slm_create_seeds_device(const uint8_t* mask, uint32_t nx_padded, uint32_t ny_padded, uint32_t pad,
                            int do_shuffle, uint32_t rng_seed, float* seed_point, uint64_t capacity,
                            uint64_t* n_seeds, uint32_t* generator_state, void* workspace, size_t workspace_bytes,
                            void* stream) {
    clear_error();
    SLM_REQUIRE(mask && seed_point && n_seeds && workspace, "NULL buffer");
    const uint64_t n_px = (uint64_t)nx_padded * ny_padded;
    SLM_REQUIRE(n_px > 0 && n_px < (1ull << 32), "grid size");
    const size_t need = slm_create_seeds_device_workspace(n_px);
    SLM_REQUIRE(workspace_bytes >= need, "workspace holds %zu bytes, needs %zu", workspace_bytes, need);
    SLM_REQUIRE(aligned(seed_point, 8) && aligned(workspace, 256), "seed_point must be 8-byte and workspace "
                "256-byte aligned");
    cudaStream_t s = (cudaStream_t)stream;
    const size_t n_all = (size_t)n_px;
    char* w = static_cast<char*>(workspace);
    const size_t pick_bytes = up256(slm_pick_seeds_workspace((uint32_t)n_px));
    void* pick_ws = w;
    uint32_t* js_d = reinterpret_cast<uint32_t*>(w + pick_bytes);
    u64* res = reinterpret_cast<u64*>(w + pick_bytes + up256(4 * n_all));
    uint32_t* list_a = reinterpret_cast<uint32_t*>(w + pick_bytes + up256(4 * n_all) + up256(8 * n_all));
    uint32_t* list_b = reinterpret_cast<uint32_t*>(reinterpret_cast<char*>(list_a) + up256(4 * n_all));
    uint32_t* n_next = reinterpret_cast<uint32_t*>(reinterpret_cast<char*>(list_b) + up256(4 * n_all));

    // 1. argwhere(~mask) - pad, row-major, as float32 rows
    uint32_t n = 0;
    const uint32_t cap32 = capacity < 0xffffffffull ? (uint32_t)capacity : 0xffffffffu;
    const int rc = slm_pick_seeds(mask, nullptr, 0u, 0, nx_padded, ny_padded, pad, seed_point, cap32, &n, pick_ws,
                                  pick_bytes, stream);
    *n_seeds = n;
    if (rc != SLM_OK) return rc;

    slm_mt::Mt19937 mt;
    mt.seed(rng_seed);
    if (do_shuffle && n > 1) {
        // 2. the swap partners, drawn as slm_create_seeds draws them, by a
        // drawing thread (inline if no thread can be started) ...
        std::vector<uint32_t> js;
        try {
            js.resize(n);
        } catch (...) {  // no exception crosses the C ABI
            set_error("no host memory for %u swap partners", n);
            return SLM_ERR_CAPACITY;
        }
        js[0] = 0u;
        std::atomic<uint64_t> final_above{n};  // js[i] is final for every i >= final_above
        SLM_CUDA(cudaMemsetAsync(res, 0, (size_t)n * 8u, s));
        Joiner drawer;
        try {
            drawer.t = std::thread([&] { mt.intervals_down(n - 1u, js.data(), &final_above); });
        } catch (...) {
            mt.intervals_down(n - 1u, js.data(), &final_above);
        }
        // 3. ... while this thread copies each chunk of final partners to the
        // device and runs its swaps
        float2* rows = reinterpret_cast<float2*>(seed_point);
        uint32_t todo = n - 1u;  // swaps todo .. 1 remain
        u64 round = 0;
        const u64 round_cap = (u64)n + (u64)n / SWAP_CHUNK + 1u;
        while (todo >= 1u) {
            const uint64_t ready = final_above.load(std::memory_order_acquire);
            const uint32_t lo_ready = ready > 1u ? (uint32_t)ready : 1u;
            if (lo_ready > todo || (lo_ready > 1u && todo - lo_ready + 1u < SWAP_CHUNK)) {
                std::this_thread::sleep_for(std::chrono::microseconds(50));
                continue;
            }
            const uint32_t lo = (todo - lo_ready + 1u > SWAP_CHUNK) ? todo - SWAP_CHUNK + 1u : lo_ready;
            SLM_CUDA(cudaMemcpyAsync(js_d + lo, js.data() + lo, (size_t)(todo - lo + 1u) * 4u,
                                     cudaMemcpyHostToDevice, s));
            const int rc2 = run_swaps(js_d, res, rows, list_a, list_b, n_next, lo, todo, &round, round_cap, s);
            if (rc2 != SLM_OK) return rc2;
            todo = lo - 1u;
        }
    }
    if (generator_state) {
        for (int k = 0; k < 624; ++k) generator_state[k] = mt.key[k];
        generator_state[624] = (uint32_t)mt.pos;
    }
    return SLM_OK;
}

}  // extern "C"
