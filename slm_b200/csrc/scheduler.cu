// scheduler.cu -- learned trajectory-length scheduler: a small BF16 CNN that
// reads a 16x16x2 patch of the flow field around a seed pixel and predicts
// log(1 + RK steps) of the seed's downstream and upstream trajectories, its
// training kernels, and the counting sort that turns predictions into the
// order the field tracer issues seeds in.  Ordering never changes a result:
// the tracer's per-pixel sums are integer and every trajectory's RNG stream
// follows its seed index.
//
// Network (all operands rounded to bfloat16, fp32 accumulation):
//   conv1  4x4 stride 4, 2 -> 32 channels, ReLU   (16 tiles x 32 features)
//   conv2  2x2 stride 2, 32 -> 64 channels, ReLU  (4 positions x 128 features)
//   dense  256 -> 2
// Feature orders: X1[t][f], t = 4*ti + tj, f = 2*(4*di + dj) + c, pixel
// (cx-8+4ti+di, cy-8+4tj+dj) clamped to the padded grid; X2[u][g], u = 2*ui+uj,
// g = 32*(2*ei+ej) + o reads A1[4*(2ui+ei) + (2uj+ej)][o]; X3[h] = A2[h/64][h%64].
//
// Training runs as batched GEMMs on the tensor cores (slm_gemm, gemm_tc.cu:
// tcgen05 with bf16 operands and fp32 accumulators in tensor memory, split-K
// for the weight gradients); inference is one fused kernel per warp of 16
// seeds (mma.sync m16n8k16 bf16 -> fp32).
#include <cuda_bf16.h>
#include "capi_util.cuh"

namespace slm {

constexpr int CNN_F1 = 32, CNN_C1 = 32, CNN_T1 = 16;
constexpr int CNN_F2 = 128, CNN_C2 = 64, CNN_U2 = 4;
constexpr int CNN_F3 = 256, CNN_OUT = 2;

__device__ __forceinline__ float bf16r(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

// ------------------------------------------------------------------ gather
// X1 rows for sample s: X1[(s*16 + t)*32 + f]
__global__ void k_patch_gather(const float2* __restrict__ uv, uint32_t nxp, uint32_t nyp, uint32_t pad,
                               const float2* __restrict__ seeds, const uint32_t* __restrict__ index,
                               uint32_t n, float* __restrict__ x1) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;  // one thread per (sample, tile, cell)
    if (tid >= n * 256u) return;
    const uint32_t s = tid >> 8, t = (tid >> 4) & 15u, m = tid & 15u;
    const uint32_t seed = index ? index[s] : s;
    const float2 sp = seeds[seed];
    const int cx = (int)sp.x + (int)pad, cy = (int)sp.y + (int)pad;
    const int ti = t >> 2, tj = t & 3, di = m >> 2, dj = m & 3;
    int x = cx - 8 + 4 * ti + di, y = cy - 8 + 4 * tj + dj;
    x = x < 0 ? 0 : (x >= (int)nxp ? (int)nxp - 1 : x);
    y = y < 0 ? 0 : (y >= (int)nyp ? (int)nyp - 1 : y);
    const float2 v = uv[(size_t)x * nyp + y];
    float* row = x1 + ((size_t)s * 16 + t) * 32 + 2 * m;
    row[0] = bf16r(v.x);
    row[1] = bf16r(v.y);
}

// A1 [n*16][32] -> X2 [n*4][128]
__global__ void k_a1_to_x2(const float* __restrict__ a1, uint32_t n, float* __restrict__ x2) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= n * 512u) return;
    const uint32_t s = tid >> 9, u = (tid >> 7) & 3u, g = tid & 127u;
    const uint32_t e = g >> 5, o = g & 31u;
    const uint32_t ui = u >> 1, uj = u & 1u, ei = e >> 1, ej = e & 1u;
    const uint32_t t = 4u * (2u * ui + ei) + (2u * uj + ej);
    x2[tid] = a1[((size_t)s * 16 + t) * 32 + o];
}

// dX2 [n*4][128] -> dA1 [n*16][32] (each A1 element feeds exactly one X2 element)
__global__ void k_dx2_to_da1(const float* __restrict__ dx2, uint32_t n, float* __restrict__ da1) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= n * 512u) return;
    const uint32_t s = tid >> 9, u = (tid >> 7) & 3u, g = tid & 127u;
    const uint32_t e = g >> 5, o = g & 31u;
    const uint32_t ui = u >> 1, uj = u & 1u, ei = e >> 1, ej = e & 1u;
    const uint32_t t = 4u * (2u * ui + ei) + (2u * uj + ej);
    da1[((size_t)s * 16 + t) * 32 + o] = dx2[tid];
}

// dZ = dA * (Z > 0)
__global__ void k_relu_backward(const float* __restrict__ da, const float* __restrict__ z, size_t n,
                                float* __restrict__ dz) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dz[i] = z[i] > 0.0f ? da[i] : 0.0f;
}

// column sums of dZ [rows][cols] added into db[cols]
__global__ void k_bias_grad(const float* __restrict__ dz, size_t rows, int cols, float* __restrict__ db) {
    const int c = blockIdx.x;
    float s = 0.0f;
    for (size_t r = threadIdx.x; r < rows; r += blockDim.x) s += dz[r * cols + c];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    __shared__ float part[32];
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        float t = threadIdx.x < (blockDim.x >> 5) ? part[threadIdx.x] : 0.0f;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
        if (threadIdx.x == 0) atomicAdd(db + c, t);
    }
}

// dY = 2 W (Y - T) inv_n, loss += sum W (Y - T)^2 inv_n (W = 1 without weights)
__global__ void k_mse(const float* __restrict__ y, const float* __restrict__ t, const float* __restrict__ w,
                      size_t n_el, float inv_n, float* __restrict__ dy, float* __restrict__ loss) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    float l = 0.0f;
    if (i < n_el) {
        const float d = y[i] - t[i];
        const float wi = (w ? w[i] : 1.0f) * inv_n;
        dy[i] = 2.0f * d * wi;
        l = d * d * wi;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, l);
}

// Adam on fp32 master weights; also writes the bf16-rounded working copy.
__global__ void k_adam(float* __restrict__ w, float* __restrict__ wq, const float* __restrict__ g,
                       float* __restrict__ m, float* __restrict__ v, size_t n, float lr, float b1,
                       float b2, float eps, float c1, float c2, int round_w) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = wi;
    wq[i] = round_w ? bf16r(wi) : wi;
}

// ------------------------------------------------------------------ inference
__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    const __nv_bfloat162 p = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&p);
}

__device__ __forceinline__ void mma_bf16(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
                 "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
                 : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Shared-memory layout of the inference kernel (bf16 pairs as uint32):
//   W1t [32 n][16 kpairs], W2t [64 n][64 kpairs], W3t [8 n][128 kpairs] (n-major,
//   so a B fragment (k pair, n) is one 32-bit word); biases fp32; per warp an
//   A1 stage [4 seeds][16 t][16 pairs] and an A2/X3 stage [16 seeds][128 pairs].
constexpr int INF_WARPS = 4;
struct InferSmem {
    uint32_t w1[32][16 + 1];
    uint32_t w2[64][64 + 1];
    uint32_t w3[8][128 + 1];
    float b1[32], b2[64], b3[8];
    uint32_t a1[INF_WARPS][4][16][16 + 1];
    uint32_t x3[INF_WARPS][16][128 + 1];
};

__global__ void __launch_bounds__(INF_WARPS * 32)
k_cnn_infer(const float2* __restrict__ uv, uint32_t nxp, uint32_t nyp, uint32_t pad,
            const float2* __restrict__ seeds, const uint32_t* __restrict__ index, uint32_t n,
            const float* __restrict__ w1,
            const float* __restrict__ b1, const float* __restrict__ w2, const float* __restrict__ b2,
            const float* __restrict__ w3, const float* __restrict__ b3, float* __restrict__ out) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    InferSmem& S = *reinterpret_cast<InferSmem*>(smem_raw);
    for (int i = threadIdx.x; i < 32 * 16; i += blockDim.x) {
        const int nn = i / 16, kp = i % 16;
        S.w1[nn][kp] = pack_bf16(w1[(2 * kp) * CNN_C1 + nn], w1[(2 * kp + 1) * CNN_C1 + nn]);
    }
    for (int i = threadIdx.x; i < 64 * 64; i += blockDim.x) {
        const int nn = i / 64, kp = i % 64;
        S.w2[nn][kp] = pack_bf16(w2[(2 * kp) * CNN_C2 + nn], w2[(2 * kp + 1) * CNN_C2 + nn]);
    }
    for (int i = threadIdx.x; i < 8 * 128; i += blockDim.x) {
        const int nn = i / 128, kp = i % 128;
        S.w3[nn][kp] = nn < CNN_OUT ? pack_bf16(w3[(2 * kp) * CNN_OUT + nn], w3[(2 * kp + 1) * CNN_OUT + nn]) : 0u;
    }
    for (int i = threadIdx.x; i < 32; i += blockDim.x) S.b1[i] = b1[i];
    for (int i = threadIdx.x; i < 64; i += blockDim.x) S.b2[i] = b2[i];
    for (int i = threadIdx.x; i < 8; i += blockDim.x) S.b3[i] = i < CNN_OUT ? b3[i] : 0.0f;
    __syncthreads();

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int gid = lane >> 2, tig = lane & 3;
    const uint32_t groups = (n + 15) / 16;
    for (uint32_t grp = blockIdx.x * INF_WARPS + warp; grp < groups; grp += gridDim.x * INF_WARPS) {
        // 16 seeds per warp pass; conv1 + conv2 in 4 quarters of 4 seeds
        for (int q = 0; q < 4; ++q) {
            for (int sl = 0; sl < 4; ++sl) {
                const uint32_t s = grp * 16 + q * 4 + sl;
                const uint32_t sc = s < n ? s : n - 1;
                const float2 sp = seeds[index ? __ldg(index + sc) : sc];
                const int cx = (int)sp.x + (int)pad, cy = (int)sp.y + (int)pad;
                // conv1: M = 16 tiles, K = 32, N = 32
                float c[4][4] = {};
#pragma unroll
                for (int ks = 0; ks < 2; ++ks) {
                    uint32_t a[4];
#pragma unroll
                    for (int r = 0; r < 4; ++r) {
                        const int t = gid + ((r & 1) ? 8 : 0);
                        const int m = ks * 8 + tig + ((r & 2) ? 4 : 0);
                        const int ti = t >> 2, tj = t & 3, di = m >> 2, dj = m & 3;
                        int x = cx - 8 + 4 * ti + di, y = cy - 8 + 4 * tj + dj;
                        x = x < 0 ? 0 : (x >= (int)nxp ? (int)nxp - 1 : x);
                        y = y < 0 ? 0 : (y >= (int)nyp ? (int)nyp - 1 : y);
                        const float2 v = uv[(size_t)x * nyp + y];
                        a[r] = pack_bf16(v.x, v.y);
                    }
#pragma unroll
                    for (int nt = 0; nt < 4; ++nt) {
                        const int nn = nt * 8 + gid;
                        mma_bf16(c[nt], a, S.w1[nn][ks * 8 + tig], S.w1[nn][ks * 8 + tig + 4]);
                    }
                }
#pragma unroll
                for (int nt = 0; nt < 4; ++nt) {
                    const int o = nt * 8 + tig * 2;
                    const float v0 = fmaxf(c[nt][0] + S.b1[o], 0.0f), v1 = fmaxf(c[nt][1] + S.b1[o + 1], 0.0f);
                    const float v2 = fmaxf(c[nt][2] + S.b1[o], 0.0f), v3 = fmaxf(c[nt][3] + S.b1[o + 1], 0.0f);
                    S.a1[warp][sl][gid][o / 2] = pack_bf16(v0, v1);
                    S.a1[warp][sl][gid + 8][o / 2] = pack_bf16(v2, v3);
                }
            }
            __syncwarp();
            // conv2: M = 16 rows (4 seeds x 4 positions), K = 128, N = 64
            float c2[8][4] = {};
#pragma unroll
            for (int ks = 0; ks < 8; ++ks) {
                uint32_t a[4];
#pragma unroll
                for (int r = 0; r < 4; ++r) {
                    const int row = gid + ((r & 1) ? 8 : 0);
                    const int sl = row >> 2, u = row & 3;
                    const int kp = ks * 8 + tig + ((r & 2) ? 4 : 0);   // k pair index (0..63)
                    const int g = 2 * kp, e = g >> 5, o = g & 31;
                    const int ui = u >> 1, uj = u & 1, ei = e >> 1, ej = e & 1;
                    const int t = 4 * (2 * ui + ei) + (2 * uj + ej);
                    a[r] = S.a1[warp][sl][t][o / 2];
                }
#pragma unroll
                for (int nt = 0; nt < 8; ++nt) {
                    const int nn = nt * 8 + gid;
                    mma_bf16(c2[nt], a, S.w2[nn][ks * 8 + tig], S.w2[nn][ks * 8 + tig + 4]);
                }
            }
#pragma unroll
            for (int nt = 0; nt < 8; ++nt) {
                const int o2 = nt * 8 + tig * 2;
#pragma unroll
                for (int hh = 0; hh < 2; ++hh) {
                    const int row = gid + hh * 8;
                    const int sl = row >> 2, u = row & 3;
                    const float v0 = fmaxf(c2[nt][2 * hh] + S.b2[o2], 0.0f);
                    const float v1 = fmaxf(c2[nt][2 * hh + 1] + S.b2[o2 + 1], 0.0f);
                    S.x3[warp][q * 4 + sl][(u * 64 + o2) / 2] = pack_bf16(v0, v1);
                }
            }
            __syncwarp();
        }
        // dense: M = 16 seeds, K = 256, N = 8 (2 used)
        float c3[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
        for (int ks = 0; ks < 16; ++ks) {
            uint32_t a[4];
            a[0] = S.x3[warp][gid][ks * 8 + tig];
            a[1] = S.x3[warp][gid + 8][ks * 8 + tig];
            a[2] = S.x3[warp][gid][ks * 8 + tig + 4];
            a[3] = S.x3[warp][gid + 8][ks * 8 + tig + 4];
            mma_bf16(c3, a, S.w3[gid][ks * 8 + tig], S.w3[gid][ks * 8 + tig + 4]);
        }
        if (tig == 0) {
            const uint32_t s0 = grp * 16 + gid, s1 = s0 + 8;
            if (s0 < n) {
                const size_t o = index ? __ldg(index + s0) : s0;
                out[2 * o] = c3[0] + S.b3[0];
                out[2 * o + 1] = c3[1] + S.b3[1];
            }
            if (s1 < n) {
                const size_t o = index ? __ldg(index + s1) : s1;
                out[2 * o] = c3[2] + S.b3[0];
                out[2 * o + 1] = c3[3] + S.b3[1];
            }
        }
        __syncwarp();
    }
}

// ------------------------------------------------------------------ ordering
// Seed orders are counting sorts of the seed indices by a small integer key
// (a bin); seeds within one bin keep no particular order, which is harmless:
// the traced fields do not depend on the order.

// bin of a predicted log length: higher prediction -> lower bin (issued first)
__device__ __forceinline__ uint32_t pred_bin(float v, float lo, float hi, uint32_t nb) {
    const float t = fminf(fmaxf((v - lo) / (hi - lo), 0.0f), 1.0f);  // NaN -> 0
    const uint32_t b = (uint32_t)(t * (float)(nb - 1) + 0.5f);
    return nb - 1u - b;
}

struct PredKey {
    const float* __restrict__ pred;
    uint32_t stride, col;
    float lo, hi;
    uint32_t nb;
    __device__ __forceinline__ uint32_t operator()(uint32_t i) const {
        return pred_bin(pred[(size_t)i * stride + col], lo, hi, nb);
    }
};

// Spatial key: the block_px x block_px block of the seed's pixel, blocks in
// x-major order (the grids' own layout), so seeds traced together lie close
// together and their uv / mask / slc / slt lines stay in L2.  With a
// prediction, seeds predicted at or above `thr` come first (class 0).
struct SpatialKey {
    const float2* __restrict__ seeds;
    uint32_t nx, ny, bs, nby, nblocks;
    const float* __restrict__ pred;
    uint32_t stride, col;
    float thr;
    __device__ __forceinline__ uint32_t operator()(uint32_t i) const {
        const float2 c = seeds[i];
        const float fx = fminf(fmaxf(c.x + 0.5f, 0.0f), (float)(nx - 1u));  // NaN -> 0
        const float fy = fminf(fmaxf(c.y + 0.5f, 0.0f), (float)(ny - 1u));
        const uint32_t xi = (uint32_t)fx, yi = (uint32_t)fy;
        const uint32_t cls = (pred && !(pred[(size_t)i * stride + col] >= thr)) ? 1u : 0u;
        return cls * nblocks + (xi / bs) * nby + yi / bs;
    }
};

constexpr uint32_t SMEM_BINS = 4096;  // bins counted in shared memory per block

template <class K>
__global__ void k_key_hist(K key, uint32_t n, uint32_t nb, uint32_t* __restrict__ hist) {
    extern __shared__ uint32_t sh[];
    const bool local = nb <= SMEM_BINS;
    if (local) {
        for (uint32_t b = threadIdx.x; b < nb; b += blockDim.x) sh[b] = 0;
        __syncthreads();
    }
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t b = key(i);
        if (local) atomicAdd(sh + b, 1u);
        else atomicAdd(hist + b, 1u);
    }
    if (local) {
        __syncthreads();
        for (uint32_t b = threadIdx.x; b < nb; b += blockDim.x)
            if (sh[b]) atomicAdd(hist + b, sh[b]);
    }
}

// Exclusive prefix sum of a[0..n) in place, one block of 1024 threads.
__global__ void __launch_bounds__(1024) k_scan_u32(uint32_t* __restrict__ a, uint32_t n) {
    __shared__ uint32_t wsum[32];
    __shared__ uint32_t carry;
    const unsigned FULL = 0xffffffffu;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (uint32_t base = 0; base < n; base += blockDim.x) {
        const uint32_t i = base + threadIdx.x;
        const uint32_t v = i < n ? a[i] : 0u;
        uint32_t x = v;
#pragma unroll
        for (uint32_t o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(FULL, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) wsum[warp] = x;
        __syncthreads();
        if (warp == 0) {
            uint32_t w = lane < nw ? wsum[lane] : 0u;
#pragma unroll
            for (uint32_t o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(FULL, w, o);
                if (lane >= o) w += y;
            }
            wsum[lane] = w;
        }
        __syncthreads();
        const uint32_t excl = carry + (warp ? wsum[warp - 1] : 0u) + x - v;
        if (i < n) a[i] = excl;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = excl + v;
        __syncthreads();
    }
}

// Each block places a contiguous range of seeds: per-bin counts in shared
// memory, one global reservation per (block, bin), then local slots.
template <class K>
__global__ void k_key_scatter(K key, uint32_t n, uint32_t nb, uint32_t* __restrict__ cursor,
                              uint32_t* __restrict__ order) {
    extern __shared__ uint32_t sh[];
    const uint32_t chunk = (n + gridDim.x - 1) / gridDim.x;
    const uint32_t b0 = blockIdx.x * chunk;
    const uint32_t b1 = min(n, b0 + chunk);
    if (nb > SMEM_BINS) {
        for (uint32_t i = b0 + threadIdx.x; i < b1; i += blockDim.x) order[atomicAdd(cursor + key(i), 1u)] = i;
        return;
    }
    for (uint32_t b = threadIdx.x; b < nb; b += blockDim.x) sh[b] = 0;
    __syncthreads();
    for (uint32_t i = b0 + threadIdx.x; i < b1; i += blockDim.x) atomicAdd(sh + key(i), 1u);
    __syncthreads();
    for (uint32_t b = threadIdx.x; b < nb; b += blockDim.x) {
        const uint32_t c = sh[b];
        sh[b] = c ? atomicAdd(cursor + b, c) : 0u;
    }
    __syncthreads();
    for (uint32_t i = b0 + threadIdx.x; i < b1; i += blockDim.x) order[atomicAdd(sh + key(i), 1u)] = i;
}

template <class K>
static int counting_order(const K& key, uint32_t n, uint32_t nb, uint32_t* bins, uint32_t* order,
                          cudaStream_t s) {
    SLM_CUDA(cudaMemsetAsync(bins, 0, (size_t)nb * sizeof(uint32_t), s));
    const size_t smem = nb <= SMEM_BINS ? (size_t)nb * sizeof(uint32_t) : 0;
    unsigned grid = (n + 255) / 256;
    const unsigned cap = (unsigned)num_sms() * 4u;
    if (grid > cap) grid = cap;
    k_key_hist<K><<<grid, 256, smem, s>>>(key, n, nb, bins);
    SLM_LAUNCHED("k_key_hist");
    k_scan_u32<<<1, 1024, 0, s>>>(bins, nb);
    SLM_LAUNCHED("k_scan_u32");
    k_key_scatter<K><<<grid, 256, smem, s>>>(key, n, nb, bins, order);
    SLM_LAUNCHED("k_key_scatter");
    return SLM_OK;
}

}  // namespace slm

using namespace slm;

extern "C" {

int slm_cnn_gather(const float* uv, uint32_t nx_padded, uint32_t ny_padded, uint32_t pad,
                   const float* seed_point, const uint32_t* index, uint32_t n, float* x1, void* stream) {
    clear_error();
    if (n == 0) return SLM_OK;
    SLM_REQUIRE(uv && seed_point && x1, "NULL buffer");
    const uint64_t threads = (uint64_t)n * 256u;
    SLM_REQUIRE(threads < (1ull << 32), "too many samples");
    k_patch_gather<<<(unsigned)((threads + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
        reinterpret_cast<const float2*>(uv), nx_padded, ny_padded, pad,
        reinterpret_cast<const float2*>(seed_point), index, n, x1);
    SLM_LAUNCHED("k_patch_gather");
    return SLM_OK;
}

int slm_cnn_rearrange(const float* src, uint32_t n, float* dst, int backward, void* stream) {
    clear_error();
    if (n == 0) return SLM_OK;
    const uint64_t threads = (uint64_t)n * 512u;
    SLM_REQUIRE(threads < (1ull << 32), "too many samples");
    const unsigned grid = (unsigned)((threads + 255) / 256);
    if (backward) k_dx2_to_da1<<<grid, 256, 0, (cudaStream_t)stream>>>(src, n, dst);
    else k_a1_to_x2<<<grid, 256, 0, (cudaStream_t)stream>>>(src, n, dst);
    SLM_LAUNCHED("k_a1_to_x2/k_dx2_to_da1");
    return SLM_OK;
}

int slm_relu_backward(const float* da, const float* z, uint64_t n, float* dz, void* stream) {
    clear_error();
    if (n == 0) return SLM_OK;
    k_relu_backward<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(da, z, n, dz);
    SLM_LAUNCHED("k_relu_backward");
    return SLM_OK;
}

int slm_bias_grad(const float* dz, uint64_t rows, int cols, float* db, void* stream) {
    clear_error();
    SLM_REQUIRE(cols > 0, "cols must be > 0");
    k_bias_grad<<<cols, 256, 0, (cudaStream_t)stream>>>(dz, rows, cols, db);
    SLM_LAUNCHED("k_bias_grad");
    return SLM_OK;
}

int slm_mse(const float* y, const float* t, const float* w, uint64_t n_el, float inv_n, float* dy, float* loss,
            void* stream) {
    clear_error();
    if (n_el == 0) return SLM_OK;
    k_mse<<<(unsigned)((n_el + 255) / 256), 256, 0, (cudaStream_t)stream>>>(y, t, w, n_el, inv_n, dy, loss);
    SLM_LAUNCHED("k_mse");
    return SLM_OK;
}

int slm_adam(float* w, float* wq, const float* g, float* m, float* v, uint64_t n, float lr, float b1,
             float b2, float eps, int step, int round_w, void* stream) {
    clear_error();
    if (n == 0) return SLM_OK;
    const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
    k_adam<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(w, wq, g, m, v, n, lr, b1, b2, eps,
                                                                         c1, c2, round_w);
    SLM_LAUNCHED("k_adam");
    return SLM_OK;
}

int slm_cnn_infer(const float* uv, uint32_t nx_padded, uint32_t ny_padded, uint32_t pad,
                  const float* seed_point, const uint32_t* index, uint32_t n, const float* w1,
                  const float* b1,
                  const float* w2, const float* b2, const float* w3, const float* b3, float* out,
                  void* stream) {
    clear_error();
    if (n == 0) return SLM_OK;
    SLM_REQUIRE(uv && seed_point && w1 && b1 && w2 && b2 && w3 && b3 && out, "NULL buffer");
    const size_t smem = sizeof(InferSmem);
    SLM_CUDA(cudaFuncSetAttribute(k_cnn_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const uint32_t groups = (n + 15) / 16;
    unsigned grid = (groups + INF_WARPS - 1) / INF_WARPS;
    const unsigned cap = (unsigned)num_sms() * 8u;
    if (grid > cap) grid = cap;
    k_cnn_infer<<<grid, INF_WARPS * 32, smem, (cudaStream_t)stream>>>(
        reinterpret_cast<const float2*>(uv), nx_padded, ny_padded, pad,
        reinterpret_cast<const float2*>(seed_point), index, n, w1, b1, w2, b2, w3, b3, out);
    SLM_LAUNCHED("k_cnn_infer");
    return SLM_OK;
}

int slm_order_by_prediction(const float* pred, uint32_t stride, uint32_t col, uint32_t n, float lo,
                            float hi, uint32_t n_bins, uint32_t* bins, uint32_t* order, void* stream) {
    clear_error();
    if (n == 0) return SLM_OK;
    SLM_REQUIRE(pred && bins && order && n_bins >= 2 && hi > lo, "bad ordering arguments");
    return counting_order(PredKey{pred, stride, col, lo, hi, n_bins}, n, n_bins, bins, order,
                          (cudaStream_t)stream);
}

uint32_t slm_order_spatial_bins(uint32_t nx, uint32_t ny, uint32_t block_px, int with_prediction) {
    if (nx == 0 || ny == 0 || block_px == 0) return 0;
    const uint64_t nbl = (uint64_t)((nx + block_px - 1) / block_px) * ((ny + block_px - 1) / block_px);
    const uint64_t nb = nbl * (with_prediction ? 2u : 1u);
    return nb < (1ull << 32) ? (uint32_t)nb : 0u;
}

int slm_order_spatial(const float* seed_point, uint32_t n, uint32_t nx, uint32_t ny, uint32_t block_px,
                      const float* pred, uint32_t stride, uint32_t col, float threshold, uint32_t* bins,
                      uint32_t n_bins_capacity, uint32_t* order, void* stream) {
    clear_error();
    if (n == 0) return SLM_OK;
    SLM_REQUIRE(seed_point && bins && order, "NULL buffer");
    SLM_REQUIRE(nx > 0 && ny > 0 && block_px > 0, "bad grid or block size");
    const uint32_t nb = slm_order_spatial_bins(nx, ny, block_px, pred != nullptr);
    SLM_REQUIRE(nb > 0 && nb <= n_bins_capacity, "bins holds %u entries, needs %u", n_bins_capacity, nb);
    const uint32_t nby = (ny + block_px - 1) / block_px;
    const uint32_t nblocks = pred ? nb / 2u : nb;
    SpatialKey key{reinterpret_cast<const float2*>(seed_point), nx, ny, block_px, nby, nblocks, pred,
                   stride, col, threshold};
    return counting_order(key, n, nb, bins, order, (cudaStream_t)stream);
}

}  // extern "C"
