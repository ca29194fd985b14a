// mt19937.hpp -- host-side MT19937 as NumPy's legacy RandomState draws it.
//
// MT19937 (Matsumoto and Nishimura, 1998) seeded by the classic init_genrand
// recurrence, which is what legacy RandomState.seed(int) does; 32-bit outputs
// with the standard tempering; bounded draws by masked rejection (the
// smallest all-ones mask >= the bound, 32-bit draws until the value fits).
// Shared by the host seed list (seeds.cpp) and the device one
// (seeds_device.cu), which draw the same swap partners.
#pragma once
#include <atomic>
#include <cstdint>

namespace slm_mt {

struct Mt19937 {
    uint32_t key[624];
    int pos;

    void seed(uint32_t s) {
        for (int i = 0; i < 624; ++i) {
            key[i] = s;
            s = 1812433253u * (s ^ (s >> 30)) + (uint32_t)(i + 1);
        }
        pos = 624;
    }

    void regenerate() {
        const uint32_t upper = 0x80000000u, lower = 0x7fffffffu, matrix = 0x9908b0dfu;
        int k = 0;
        for (; k < 624 - 397; ++k) {
            const uint32_t y = (key[k] & upper) | (key[k + 1] & lower);
            key[k] = key[k + 397] ^ (y >> 1) ^ ((y & 1u) ? matrix : 0u);
        }
        for (; k < 623; ++k) {
            const uint32_t y = (key[k] & upper) | (key[k + 1] & lower);
            key[k] = key[k + 397 - 624] ^ (y >> 1) ^ ((y & 1u) ? matrix : 0u);
        }
        const uint32_t y = (key[623] & upper) | (key[0] & lower);
        key[623] = key[396] ^ (y >> 1) ^ ((y & 1u) ? matrix : 0u);
        pos = 0;
    }

    uint32_t next() {
        if (pos == 624) regenerate();
        uint32_t y = key[pos++];
        y ^= y >> 11;
        y ^= (y << 7) & 0x9d2c5680u;
        y ^= (y << 15) & 0xefc60000u;
        y ^= y >> 18;
        return y;
    }

    // uniform in [0, max] by masked rejection on 32-bit draws (max < 2^32)
    uint32_t interval(uint32_t max) {
        if (max == 0) return 0;
        uint32_t mask = max;
        mask |= mask >> 1;
        mask |= mask >> 2;
        mask |= mask >> 4;
        mask |= mask >> 8;
        mask |= mask >> 16;
        uint32_t v;
        while ((v = (next() & mask)) > max) {
        }
        return v;
    }

    // js[i] = interval(i) for i = top .. 1, in that order: the same draws as
    // calling interval() in a loop, consumed a tempered 624-word block at a
    // time without a data-dependent branch (a rejected draw's value is
    // written and then overwritten by the next draw for the same i).  The
    // mask only changes when i drops below a power of two, so the inner loop
    // runs with it fixed while i > mask/2: a compare and a subtract per draw
    // on the loop-carried path.  After each block, *final_above (if given) is
    // set to the lowest index whose js is final (release order): the index
    // still being drawn is not.  top < 2^32.
    void intervals_down(uint64_t top, uint32_t* js, std::atomic<uint64_t>* final_above = nullptr) {
        uint32_t block[624];
        uint32_t i = (uint32_t)top;
        while (i >= 1u) {
            if (pos == 624) regenerate();
            for (int k = pos; k < 624; ++k) {
                uint32_t y = key[k];
                y ^= y >> 11;
                y ^= (y << 7) & 0x9d2c5680u;
                y ^= (y << 15) & 0xefc60000u;
                y ^= y >> 18;
                block[k] = y;
            }
            int k = pos;
            while (k < 624 && i >= 1u) {
                const uint32_t mask = 0xffffffffu >> __builtin_clz(i);
                const uint32_t low = mask >> 1;  // the mask holds while i > low
                for (; k < 624 && i > low; ++k) {
                    const uint32_t v = block[k] & mask;
                    js[i] = v;
                    i -= (uint32_t)(v <= i);
                }
            }
            pos = k;
            if (final_above) final_above->store((uint64_t)i + 1, std::memory_order_release);
        }
    }
};

}  // namespace slm_mt
