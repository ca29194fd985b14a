// map_device.cu -- the host steps between the mapping kernels, on the device,
// so map_channels_segments can keep every grid on the GPU from the fields to
// the labels (the reference runs them in NumPy between its kernels,
// mapping.py:627-775, useful.py:519-538, segment.py:83-88).  Each restates
// one NumPy expression of the host wrappers element for element.
#include "capi_util.cuh"

namespace slm {

constexpr uint32_t PICK_ITEMS = 16;  // pixels per thread in the compaction
constexpr uint32_t PICK_BLOCK = 256;

// pick_seeds predicate (useful.py:519-538): unmasked (when a mask is given)
// and (map & flag) > 0 (when a map is given; ~map when invert)
__device__ __forceinline__ bool picked(uint32_t i, const uint8_t* __restrict__ mask,
                                       const uint32_t* __restrict__ map, uint32_t flag, int invert) {
    if (mask && mask[i]) return false;
    if (map) {
        const uint32_t m = invert ? ~map[i] : map[i];
        if ((m & flag) == 0u) return false;
    }
    return true;
}

__global__ void k_pick_count(const uint8_t* __restrict__ mask, const uint32_t* __restrict__ map,
                             uint32_t flag, int invert, uint32_t n, uint32_t* __restrict__ block_count) {
    __shared__ uint32_t warp_sum[PICK_BLOCK / 32];
    const uint32_t base = blockIdx.x * PICK_BLOCK * PICK_ITEMS + threadIdx.x * PICK_ITEMS;
    uint32_t c = 0;
    for (uint32_t k = 0; k < PICK_ITEMS; ++k) {
        const uint32_t i = base + k;
        if (i < n && picked(i, mask, map, flag, invert)) c++;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0) warp_sum[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (uint32_t w = 0; w < PICK_BLOCK / 32; ++w) t += warp_sum[w];
        block_count[blockIdx.x] = t;
    }
}

// writes the picked pixels of this block in index order, at block_off[block]
__global__ void k_pick_write(const uint8_t* __restrict__ mask, const uint32_t* __restrict__ map,
                             uint32_t flag, int invert, uint32_t n, uint32_t ny, float pad,
                             const uint32_t* __restrict__ block_off, float2* __restrict__ seeds) {
    __shared__ uint32_t warp_off[PICK_BLOCK / 32 + 1];
    const uint32_t base = blockIdx.x * PICK_BLOCK * PICK_ITEMS + threadIdx.x * PICK_ITEMS;
    uint32_t c = 0;
    for (uint32_t k = 0; k < PICK_ITEMS; ++k) {
        const uint32_t i = base + k;
        if (i < n && picked(i, mask, map, flag, invert)) c++;
    }
    // exclusive prefix of c over the block (threads hold consecutive pixel runs)
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if ((int)lane >= o) x += y;
    }
    if (lane == 31) warp_off[warp] = x;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t run = 0;
        for (uint32_t w = 0; w < PICK_BLOCK / 32; ++w) {
            const uint32_t t = warp_off[w];
            warp_off[w] = run;
            run += t;
        }
    }
    __syncthreads();
    uint32_t pos = block_off[blockIdx.x] + warp_off[warp] + x - c;
    for (uint32_t k = 0; k < PICK_ITEMS; ++k) {
        const uint32_t i = base + k;
        if (i < n && picked(i, mask, map, flag, invert)) {
            // argwhere(...).astype(float32) - pad: exact integers
            seeds[pos++] = make_float2((float)(i / ny) - pad, (float)(i % ny) - pad);
        }
    }
}

// exclusive scan of uint32 a[0..n) into out (total in out[n]), multi-block:
// per-block sums, one block scanning them, then each block adds its offset
constexpr uint32_t SCAN_BLOCK = 1024;
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* sh, uint32_t& total) {
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if ((int)lane >= o) x += y;
    }
    if (lane == 31) sh[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < (blockDim.x >> 5) ? sh[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if ((int)lane >= o) w += y;
        }
        sh[lane] = w;
    }
    __syncthreads();
    const uint32_t excl = (warp ? sh[warp - 1] : 0u) + x - v;
    total = sh[(blockDim.x >> 5) - 1];
    __syncthreads();
    return excl;
}

__global__ void k_scan_blocks(const uint32_t* __restrict__ a, uint32_t n, uint32_t* __restrict__ out,
                              uint32_t* __restrict__ sums) {
    __shared__ uint32_t sh[32];
    const uint32_t i = blockIdx.x * SCAN_BLOCK + threadIdx.x;
    const uint32_t v = i < n ? a[i] : 0u;
    uint32_t total;
    const uint32_t e = block_excl_scan(v, sh, total);
    if (i < n) out[i] = e;
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

__global__ void k_scan_sums(uint32_t* __restrict__ sums, uint32_t nb, uint32_t* __restrict__ total_out) {
    __shared__ uint32_t sh[32];
    uint32_t carry = 0;
    for (uint32_t base = 0; base < nb; base += SCAN_BLOCK) {
        const uint32_t i = base + threadIdx.x;
        const uint32_t v = i < nb ? sums[i] : 0u;
        uint32_t total;
        const uint32_t e = block_excl_scan(v, sh, total);
        if (i < nb) sums[i] = carry + e;
        carry += total;
    }
    if (threadIdx.x == 0) *total_out = carry;
}

__global__ void k_scan_add(uint32_t* __restrict__ out, uint32_t n, const uint32_t* __restrict__ sums) {
    const uint32_t i = blockIdx.x * SCAN_BLOCK + threadIdx.x;
    if (i < n) out[i] += sums[blockIdx.x];
}

static int scan_u32(const uint32_t* a, uint32_t n, uint32_t* out, uint32_t* sums, uint32_t* total,
                    cudaStream_t s) {
    const uint32_t nb = (n + SCAN_BLOCK - 1) / SCAN_BLOCK;
    k_scan_blocks<<<nb, SCAN_BLOCK, 0, s>>>(a, n, out, sums);
    SLM_LAUNCHED("k_scan_blocks");
    k_scan_sums<<<1, SCAN_BLOCK, 0, s>>>(sums, nb, total);
    SLM_LAUNCHED("k_scan_sums");
    k_scan_add<<<nb, SCAN_BLOCK, 0, s>>>(out, n, sums);
    SLM_LAUNCHED("k_scan_add");
    return SLM_OK;
}

// mapping[cond] = IS_CHANNEL with cond = (slt >= thr) & (slt * 2 >= slc):
// slt float32 * 2 stays float32, the comparison with float64 slc is float64
// (mapping.py:695-702 under NumPy promotion)
__global__ void k_map_channels(const float* __restrict__ slt, const double* __restrict__ slc, float thr,
                               uint32_t n, uint32_t is_channel, uint32_t* __restrict__ mapping) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float t = slt[i];
    if (t >= thr && (double)(t * 2.0f) >= slc[i]) mapping[i] = is_channel;
}

// op 0: m[(m & a) == a] |= b;  op 1: m[(m & a) != 0] ^= a;
// op 2: m[sel != 0] |= b (sel a byte grid);  op 3: sel = ((m & a) == a) | ((m & b) == b)
__global__ void k_flag_op(uint32_t* __restrict__ m, uint8_t* __restrict__ sel, uint32_t n, int op,
                          uint32_t a, uint32_t b) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t v = m[i];
    if (op == 0) {
        if ((v & a) == a) m[i] = v | b;
    } else if (op == 1) {
        if (v & a) m[i] = v ^ a;
    } else if (op == 2) {
        if (sel[i]) m[i] = v | b;
    } else {
        sel[i] = ((v & a) == a) || ((v & b) == b) ? 1 : 0;
    }
}

__global__ void k_mark_labels(const uint32_t* __restrict__ label, uint32_t n, uint32_t* __restrict__ present) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int32_t l = (int32_t)label[i];
    if (l > 0 && (uint32_t)l < n) present[l] = 1u;
}

__global__ void k_apply_ranks(uint32_t* __restrict__ label, uint32_t n, const uint32_t* __restrict__ rank,
                              uint32_t* __restrict__ bad) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int32_t l = (int32_t)label[i];
    if (l > 0) {
        if ((uint32_t)l < n) label[i] = rank[l] + 1u;
        else *bad = 1u;
    }
}

// lab[lab < 0] = -(int64(lab) + LEFT_FLANK_ADDITION) as int32 (mapping.py:772-773)
__global__ void k_signed_labels(uint32_t* __restrict__ label, uint32_t n, uint32_t lfa) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int32_t l = (int32_t)label[i];
    if (l < 0) label[i] = (uint32_t)(int32_t)(-((long long)l + (long long)lfa));
}

}  // namespace slm

using namespace slm;

static unsigned blocks(uint32_t n, uint32_t b) { return (n + b - 1) / b; }

extern "C" {

size_t slm_pick_seeds_workspace(uint32_t n_pixels) {
    const uint32_t nb = blocks(n_pixels, PICK_BLOCK * PICK_ITEMS);
    return ((size_t)2 * nb + blocks(nb, SCAN_BLOCK) + 2) * sizeof(uint32_t) + 256;
}

int slm_pick_seeds(const uint8_t* mask, const uint32_t* map, uint32_t flag, int invert_map,
                   uint32_t nx_padded, uint32_t ny_padded, uint32_t pad, float* seed_point,
                   uint32_t capacity, uint32_t* n_picked, void* workspace, size_t workspace_bytes,
                   void* stream) {
    clear_error();
    SLM_REQUIRE(seed_point && n_picked && workspace, "NULL buffer");
    const uint64_t n64 = (uint64_t)nx_padded * ny_padded;
    SLM_REQUIRE(n64 > 0 && n64 < (1ull << 32), "grid size");
    const uint32_t n = (uint32_t)n64;
    SLM_REQUIRE(workspace_bytes >= slm_pick_seeds_workspace(n), "workspace below %zu bytes",
                slm_pick_seeds_workspace(n));
    cudaStream_t s = (cudaStream_t)stream;
    const uint32_t nb = blocks(n, PICK_BLOCK * PICK_ITEMS);
    uint32_t* cnt = reinterpret_cast<uint32_t*>(workspace);
    uint32_t* off = cnt + nb;
    uint32_t* sums = off + nb;
    uint32_t* total = sums + blocks(nb, SCAN_BLOCK);
    k_pick_count<<<nb, PICK_BLOCK, 0, s>>>(mask, map, flag, invert_map, n, cnt);
    SLM_LAUNCHED("k_pick_count");
    scan_u32(cnt, nb, off, sums, total, s);
    uint32_t got = 0;
    SLM_CUDA(cudaMemcpyAsync(&got, total, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    SLM_CUDA(cudaStreamSynchronize(s));
    *n_picked = got;
    if (got > capacity) {
        set_error("%u seeds picked, capacity %u", got, capacity);
        return SLM_ERR_CAPACITY;
    }
    if (got == 0) return SLM_OK;
    k_pick_write<<<nb, PICK_BLOCK, 0, s>>>(mask, map, flag, invert_map, n, ny_padded, (float)pad, off,
                                          reinterpret_cast<float2*>(seed_point));
    SLM_LAUNCHED("k_pick_write");
    return SLM_OK;
}

int slm_map_channels(const float* slt_down, const double* slc_down, float channel_threshold,
                     uint32_t n_pixels, uint32_t is_channel, uint32_t* mapping, void* stream) {
    clear_error();
    if (n_pixels == 0) return SLM_OK;
    SLM_REQUIRE(slt_down && slc_down && mapping, "NULL buffer");
    k_map_channels<<<blocks(n_pixels, 256), 256, 0, (cudaStream_t)stream>>>(slt_down, slc_down,
                                                                          channel_threshold, n_pixels,
                                                                          is_channel, mapping);
    SLM_LAUNCHED("k_map_channels");
    return SLM_OK;
}

int slm_flag_op(uint32_t* mapping, uint8_t* select, uint32_t n_pixels, int op, uint32_t a, uint32_t b,
                void* stream) {
    clear_error();
    if (n_pixels == 0) return SLM_OK;
    SLM_REQUIRE(mapping && (op < 2 || select) && op >= 0 && op <= 3, "bad flag op");
    k_flag_op<<<blocks(n_pixels, 256), 256, 0, (cudaStream_t)stream>>>(mapping, select, n_pixels, op, a, b);
    SLM_LAUNCHED("k_flag_op");
    return SLM_OK;
}

size_t slm_relabel_workspace(uint32_t n_pixels) {
    return ((size_t)2 * n_pixels + blocks(n_pixels, SCAN_BLOCK) + 4) * sizeof(uint32_t) + 256;
}

int slm_relabel(uint32_t* label, uint32_t n_pixels, void* workspace, size_t workspace_bytes,
                uint32_t* n_labels, void* stream) {
    clear_error();
    SLM_REQUIRE(label && workspace && n_labels, "NULL buffer");
    SLM_REQUIRE(workspace_bytes >= slm_relabel_workspace(n_pixels), "workspace below %zu bytes",
                slm_relabel_workspace(n_pixels));
    *n_labels = 0;
    if (n_pixels == 0) return SLM_OK;
    cudaStream_t s = (cudaStream_t)stream;
    uint32_t* present = reinterpret_cast<uint32_t*>(workspace);
    uint32_t* rank = present + n_pixels;
    uint32_t* sums = rank + n_pixels;
    uint32_t* total = sums + blocks(n_pixels, SCAN_BLOCK);
    uint32_t* bad = total + 1;
    SLM_CUDA(cudaMemsetAsync(present, 0, (size_t)n_pixels * sizeof(uint32_t), s));
    SLM_CUDA(cudaMemsetAsync(bad, 0, sizeof(uint32_t), s));
    k_mark_labels<<<blocks(n_pixels, 256), 256, 0, s>>>(label, n_pixels, present);
    SLM_LAUNCHED("k_mark_labels");
    scan_u32(present, n_pixels, rank, sums, total, s);
    k_apply_ranks<<<blocks(n_pixels, 256), 256, 0, s>>>(label, n_pixels, rank, bad);
    SLM_LAUNCHED("k_apply_ranks");
    uint32_t out[2] = {0, 0};
    SLM_CUDA(cudaMemcpyAsync(out, total, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    SLM_CUDA(cudaStreamSynchronize(s));
    SLM_REQUIRE(out[1] == 0u, "a label exceeds the grid size");
    *n_labels = out[0];
    return SLM_OK;
}

int slm_signed_labels(uint32_t* label, uint32_t n_pixels, uint32_t left_flank_addition, void* stream) {
    clear_error();
    if (n_pixels == 0) return SLM_OK;
    SLM_REQUIRE(label, "NULL buffer");
    k_signed_labels<<<blocks(n_pixels, 256), 256, 0, (cudaStream_t)stream>>>(label, n_pixels,
                                                                           left_flank_addition);
    SLM_LAUNCHED("k_signed_labels");
    return SLM_OK;
}

}  // extern "C"
