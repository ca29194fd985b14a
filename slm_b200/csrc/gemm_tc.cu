// gemm_tc.cu -- the learned scheduler's training GEMMs on the 5th-generation
// tensor cores (tcgen05), with the accumulators in tensor memory.
//
//   C[M][N] = op(A)[M][K] op(B)[K][N]   (+ bias[N], ReLU, pre-activation into Z,
//                                        bf16 rounding of the output)
//   op(A) = A [M][K] or A^T with A [K][M];  op(B) = B [K][N] or B^T with B [N][K]
//
// One CTA of 128 threads owns a 128-row tile of C and every one of its N
// (<= 256) columns.  Per 64-element K stage the CTA converts its A and B
// tiles to bfloat16 (round to nearest even) into shared memory in the
// canonical K-major, no-swizzle layout: 8-row x 16-byte core matrices, 128 B
// apart along M / N (SBO) and rows x 16 B apart along K (LBO).  One thread
// issues four tcgen05.mma (M=128, K=16, N padded to a multiple of 16) that
// accumulate in fp32 in tensor memory, and commits them to an mbarrier the
// CTA waits on before the next stage overwrites the tiles.  The epilogue
// reads the accumulators with tcgen05.ld: warp w owns tensor-memory lanes
// (= rows) 32w..32w+31.
//
// Split-K (the weight gradients, K up to 65536): gridDim.z slices of K, each
// writing its tile to partial[z][M][N]; k_split_sum adds them
// in slice order, so results do not depend on the order blocks run in.
//
// Every wait is bounded.  A wait that runs out sets bit 0 of *status, waits
// (bounded again) for the MMAs in flight, frees the tensor memory and
// returns.  Tensor-memory columns per CTA times resident CTAs per SM stay
// within the SM's 512 columns: the launch asks for enough shared memory to
// cap the CTAs an SM holds.
#include <cuda_bf16.h>
#include "capi_util.cuh"

namespace slm {
namespace tc {

constexpr int BM = 128;       // rows per CTA (one tensor-memory lane each)
constexpr int BK = 64;        // K per shared-memory stage (bf16)
constexpr int THREADS = 128;  // four warps
constexpr uint32_t WAIT_LIMIT = 1u << 22;
constexpr uint32_t ST_TIMEOUT = 1u;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// byte offset of element (row, k) of a rows x BK tile in the canonical layout
__device__ __forceinline__ uint32_t core_offset(int row, int k, int rows) {
    return (uint32_t)((k >> 3) * (rows * 16) + (row >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

// shared-memory matrix descriptor: start address, LBO and SBO in 16-byte
// units, the Blackwell descriptor version (bit 46), no swizzle, base offset 0
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// instruction descriptor of kind::f16: fp32 accumulator, bf16 A and B, both
// K-major, N = npad, M = 128
__device__ __forceinline__ uint32_t instr_desc(int npad) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(npad >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (uint32_t i = 0; i < WAIT_LIMIT; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

template <bool TA, bool TB>
__global__ void __launch_bounds__(THREADS)
k_gemm_tc(const float* __restrict__ A, const float* __restrict__ B, float* __restrict__ C,
          float* __restrict__ Z, const float* __restrict__ bias, int M, int N, int K, int relu,
          int round_out, float* __restrict__ partial, int npad, uint32_t tmem_cols,
          uint32_t* __restrict__ status) {
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ __align__(8) unsigned long long bar;
    __shared__ uint32_t tmem_base;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    __nv_bfloat16* sa = reinterpret_cast<__nv_bfloat16*>(smem);
    __nv_bfloat16* sb = reinterpret_cast<__nv_bfloat16*>(smem + BM * BK * 2);
    const int m0 = blockIdx.y * BM;
    const int kchunk = (K + gridDim.z - 1) / gridDim.z;
    const int kb = blockIdx.z * kchunk, ke = min(K, kb + kchunk);
    const uint32_t bar_a = smem_u32(&bar);

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_u32(&tmem_base)), "r"(tmem_cols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(bar_a));
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmem_base;
    const uint32_t idesc = instr_desc(npad);
    const uint32_t a_lbo = BM * 16, b_lbo = (uint32_t)npad * 16;
    uint32_t phase = 0;
    bool ok = true, any = false;

    for (int k0 = kb; k0 < ke && ok; k0 += BK) {
        // op(A) rows m0.. and op(B) columns as bf16 tiles (zero outside the
        // matrix and outside this slice's K range)
        for (int i = tid; i < BM * BK; i += THREADS) {
            const int r = TA ? (i % BM) : (i / BK), k = TA ? (i / BM) : (i % BK);
            const int m = m0 + r, kk = k0 + k;
            float v = 0.0f;
            if (m < M && kk < ke) v = TA ? A[(size_t)kk * M + m] : A[(size_t)m * K + kk];
            sa[core_offset(r, k, BM) >> 1] = __float2bfloat16_rn(v);
        }
        for (int i = tid; i < npad * BK; i += THREADS) {
            const int n = TB ? (i / BK) : (i % npad), k = TB ? (i % BK) : (i / npad);
            const int kk = k0 + k;
            float v = 0.0f;
            if (n < N && kk < ke) v = TB ? B[(size_t)n * K + kk] : B[(size_t)kk * N + n];
            sb[core_offset(n, k, npad) >> 1] = __float2bfloat16_rn(v);
        }
        // the tensor cores read shared memory through the async proxy
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;");
            const uint32_t a0 = smem_u32(sa), b0 = smem_u32(sb);
#pragma unroll
            for (int s = 0; s < BK / 16; ++s) {
                const uint64_t ad = smem_desc(a0 + 2 * s * a_lbo, a_lbo, 128);
                const uint64_t bd = smem_desc(b0 + 2 * s * b_lbo, b_lbo, 128);
                const uint32_t acc = (any || s > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
                    :
                    : "r"(tmem), "l"(ad), "l"(bd), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                         :: "r"(bar_a) : "memory");
        }
        any = true;
        // every thread sees the stage's MMAs complete (or the CTA gives up
        // together) before the tiles are overwritten
        const bool done = __syncthreads_and(mbar_wait(bar_a, phase) ? 1 : 0) != 0;
        if (!done) {
            ok = false;
            if (tid == 0) atomicOr(status, ST_TIMEOUT);
            mbar_wait(bar_a, phase);  // let the MMAs in flight finish before the tiles or TMEM go
        }
        phase ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;");
    }

    if (ok) {
        const int m = m0 + warp * 32 + lane;
        const uint32_t row_addr = tmem + ((uint32_t)(warp * 32) << 16);
        for (int c = 0; c < npad; c += 8) {
            uint32_t v[8];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];\n"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
                : "r"(row_addr + (uint32_t)c));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (m < M) {
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const int n = c + j;
                    if (n >= N) continue;
                    const float acc = any ? __uint_as_float(v[j]) : 0.0f;
                    const size_t o = (size_t)m * N + n;
                    if (partial) {
                        partial[(size_t)blockIdx.z * M * N + o] = acc;
                    } else {
                        float x = acc + (bias ? bias[n] : 0.0f);
                        if (Z) Z[o] = x;
                        if (relu) x = fmaxf(x, 0.0f);
                        if (round_out) x = __bfloat162float(__float2bfloat16_rn(x));
                        C[o] = x;
                    }
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(tmem_cols));
}

}  // namespace tc

// C[o] += partial[0][o] + partial[1][o] + ... in slice order
__global__ void k_split_sum(const float* __restrict__ partial, int slices, size_t mn, float* __restrict__ C) {
    const size_t o = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= mn) return;
    float v = C[o];
    for (int z = 0; z < slices; ++z) v += partial[(size_t)z * mn + o];
    C[o] = v;
}

}  // namespace slm

using namespace slm;

extern "C" int slm_gemm(int trans_a, int trans_b, int M, int N, int K, const float* A, const float* B, float* C,
                        float* Z, const float* bias, int relu, int round_out, int split_k, float* partial,
                        uint32_t* status, void* stream) {
    clear_error();
    SLM_REQUIRE(M > 0 && N > 0 && K > 0 && A && B && C && status, "bad GEMM arguments");
    SLM_REQUIRE(N <= 256, "N = %d: the tensor-core GEMM keeps every column of a tile, N <= 256", N);
    SLM_REQUIRE(split_k <= 0 || partial, "split_k needs a partial buffer of split_k*M*N floats");
    float* part = split_k > 0 ? partial : nullptr;
    const int npad = ((N + 15) / 16) * 16;
    uint32_t cols = 32;
    while (cols < (uint32_t)npad) cols <<= 1;
    // shared memory: the two tiles, raised so that an SM holds at most
    // 512 / cols CTAs (each holds cols tensor-memory columns)
    const size_t tiles = (size_t)tc::BM * tc::BK * 2 + (size_t)npad * tc::BK * 2;
    const size_t per_sm = 227 * 1024;
    const size_t cap = per_sm / (512 / cols) + 1024;
    const size_t smem = tiles > cap ? tiles : cap;
    dim3 grid(1, (M + tc::BM - 1) / tc::BM, split_k > 0 ? split_k : 1);
    cudaStream_t s = (cudaStream_t)stream;
#define SLM_GEMM_TC(TA, TB)                                                                                     \
    do {                                                                                                        \
        SLM_CUDA(cudaFuncSetAttribute(tc::k_gemm_tc<TA, TB>, cudaFuncAttributeMaxDynamicSharedMemorySize,       \
                                      (int)smem));                                                              \
        tc::k_gemm_tc<TA, TB><<<grid, tc::THREADS, smem, s>>>(A, B, C, Z, bias, M, N, K, relu, round_out, part, \
                                                              npad, cols, status);                              \
    } while (0)
    if (trans_a && trans_b) SLM_GEMM_TC(true, true);
    else if (trans_a) SLM_GEMM_TC(true, false);
    else if (trans_b) SLM_GEMM_TC(false, true);
    else SLM_GEMM_TC(false, false);
#undef SLM_GEMM_TC
    SLM_LAUNCHED("k_gemm_tc");
    if (part) {
        const size_t mn = (size_t)M * N;
        k_split_sum<<<(unsigned)((mn + 255) / 256), 256, 0, s>>>(part, split_k, mn, C);
        SLM_LAUNCHED("k_split_sum");
    }
    return SLM_OK;
}
