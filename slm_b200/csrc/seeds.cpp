// seeds.cpp -- create_seeds' seed list on the host, in native code.
//
// The reference builds the field seeds as argwhere(~mask) - pad and shuffles
// the rows with NumPy's global legacy generator (useful.py:470-517:
// np.random.seed(rng_seed); np.random.shuffle(seed_point_array)).  The
// shuffle fixes each seed's index, and with it the seed's jitter RNG stream,
// so it must be NumPy's exactly.  That is:
//   - MT19937 (Matsumoto and Nishimura, 1998) seeded by the classic
//     init_genrand recurrence, which is what legacy RandomState.seed(int)
//     does; 32-bit outputs with the standard tempering;
//   - Fisher-Yates from the last row down: for i = n-1 .. 1, j is drawn in
//     [0, i] by masked rejection (the smallest all-ones mask >= i applied to
//     32-bit draws until the value is <= i), then rows i and j swap.
// NumPy does this one random-access swap at a time; here all j are drawn
// first (branch-free over tempered blocks of the generator's output), then
// the swaps run with the rows they touch prefetched ahead.  The
// final generator state is handed back so that the caller can leave NumPy's
// global generator where the reference's shuffle leaves it.
#include <atomic>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include "slm_b200.h"
#include "mt19937.hpp"

using slm_mt::Mt19937;

extern "C" {

int slm_create_seeds(const uint8_t* mask, uint32_t nx_padded, uint32_t ny_padded, uint32_t pad, int do_shuffle,
                     uint32_t rng_seed, float* seed_point, uint64_t capacity, uint64_t* n_seeds,
                     uint32_t* generator_state) {
    if (!mask || !n_seeds) return SLM_ERR_ARGS;
    const uint64_t n_px = (uint64_t)nx_padded * ny_padded;
    uint64_t n = 0;
    for (uint64_t i = 0; i < n_px; ++i) n += mask[i] ? 0u : 1u;
    *n_seeds = n;
    if (!seed_point) return SLM_OK;  // size query
    if (n > capacity) return SLM_ERR_CAPACITY;
    if (n >= (1ull << 32)) return SLM_ERR_ARGS;
    // argwhere(~mask) in row-major order, as float32, minus the pad
    uint64_t k = 0;
    const float fpad = (float)pad;
    for (uint32_t x = 0; x < nx_padded; ++x) {
        const uint8_t* row = mask + (uint64_t)x * ny_padded;
        for (uint32_t y = 0; y < ny_padded; ++y) {
            if (!row[y]) {
                seed_point[2 * k] = (float)x - fpad;
                seed_point[2 * k + 1] = (float)y - fpad;
                ++k;
            }
        }
    }
    Mt19937 mt;
    mt.seed(rng_seed);
    if (do_shuffle && n > 1) {
        // the swap partners j(i), i = n-1 .. 1, in draw order
        // one thread draws the swap partners j(i), i = n-1 .. 1; this one
        // swaps row i with row j(i) as soon as j(i) is final
        std::vector<uint32_t> js;
        try {
            js.resize(n);
        } catch (...) {
            return SLM_ERR_CAPACITY;  // no exception crosses the C ABI
        }
        std::atomic<uint64_t> final_above{n};  // js[i] is final for every i >= final_above
        std::thread drawer;
        bool threaded = true;
        try {
            drawer = std::thread([&] { mt.intervals_down(n - 1, js.data(), &final_above); });
        } catch (...) {  // no thread to be had: draw everything first, then swap
            threaded = false;
            mt.intervals_down(n - 1, js.data(), &final_above);
        }
        char* rows = reinterpret_cast<char*>(seed_point);  // 8-byte (x, y) rows
        const uint64_t ahead = 32;
        uint64_t ready = n;  // js[i] final for i >= ready
        for (uint64_t i = n - 1; i >= 1; --i) {
            while (i < ready) {
                ready = final_above.load(std::memory_order_acquire);
                if (i < ready) std::this_thread::yield();
            }
            if (i > ahead && i - ahead >= ready) __builtin_prefetch(rows + 8 * (uint64_t)js[i - ahead], 1, 0);
            char* a = rows + 8 * (uint64_t)js[i];
            char* b = rows + 8 * i;
            uint64_t ta, tb;
            std::memcpy(&ta, a, 8);
            std::memcpy(&tb, b, 8);
            std::memcpy(a, &tb, 8);
            std::memcpy(b, &ta, 8);
        }
        if (threaded) drawer.join();
    }
    if (generator_state) {
        std::memcpy(generator_state, mt.key, sizeof(mt.key));
        generator_state[624] = (uint32_t)mt.pos;
    }
    return SLM_OK;
}

}  // extern "C"
