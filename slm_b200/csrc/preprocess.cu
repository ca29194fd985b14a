// preprocess.cu -- the conditioned gradient vector field of a DTM region
// (python/streamlines/preprocess.py:531-621) in one tiled kernel.
//
// The reference runs it on the host: two scipy generic_filter passes with
// Python callbacks (find_blockages, :647-699), np.gradient, then numba loops
// over every cell (find_and_fix_loops, :302-349) and over the blockages
// (fix_blockages, :351-387), normalisation, edge padding and the NaN mask.
// Every value of a pixel depends only on the ROI within two pixels of it, so
// one kernel does it all: a CTA stages a 16 x 32 tile of the ROI with a
// two-pixel halo in shared memory, derives velocities, blockage codes and
// looped cells for the tile plus a one-pixel halo, and writes each pixel's
// final uv (with its edge-padding replicas), slope, masks and codes.
//
// Arithmetic follows the reference operation for operation (IEEE float32,
// --fmad=false):
//   gradient   np.gradient of the float32 ROI, one-sided at the edges, then
//              / pixel_size in float32;
//   hypot      float32 np.hypot: the double sum of the exact squares,
//              square-rooted in double and rounded once to float32;
//   loops      check_has_loop as numba compiles it: velocity sums in float32,
//              its speed in double rounded to float32, divergence and curl in
//              float32 (2-term dot products round once), compared with the
//              double thresholds (a float32 against a float64 parameter);
//   fixes      break_out_of_loop: component / hypotf of the int8 vector;
//              fix_blockages: (dx, dy) / sqrt(2) in double, stored as float32.
#include "capi_util.cuh"

namespace slm {

constexpr int PP_TX = 16;   // tile rows (x)
constexpr int PP_TY = 32;   // tile columns (y, the contiguous axis)
constexpr int PP_THREADS = 256;  // each thread finishes PP_TX * PP_TY / PP_THREADS pixels
constexpr int PP_HX = PP_TX + 4, PP_HY = PP_TY + 4;  // ROI tile with a 2-pixel halo
constexpr int PP_VX = PP_TX + 2, PP_VY = PP_TY + 2;  // velocities / codes, 1-pixel halo
constexpr int PP_CX = PP_TX + 1, PP_CY = PP_TY + 1;  // cells x0-1 .. x0+TX-1

// flow-vector bits (get_flow_vector, preprocess.py:195-226)
enum : uint32_t { FV_W = 1, FV_E = 2, FV_S = 4, FV_N = 8, FV_SW = 16, FV_SE = 32, FV_NW = 64, FV_NE = 128 };

__device__ __forceinline__ int clampi(int i, int n) { return i < 0 ? 0 : (i >= n ? n - 1 : i); }

__device__ __forceinline__ float hypot_f32(float a, float b) {
    if (isinf(a) || isinf(b)) return __int_as_float(0x7f800000);
    const double s = __dadd_rn(__dmul_rn((double)a, (double)a), __dmul_rn((double)b, (double)b));
    return __double2float_rn(__dsqrt_rn(s));
}

// set_speed_field (preprocess.py:118-136)
__device__ __forceinline__ float speed_of(float u, float v) {
    const float s = hypot_f32(u, v);
    return (!isfinite(s) || s == 0.0f) ? 1.0f : s;
}

// get_flow_vector's priority: SW, SE, NW, NE, W, E, S, N
__device__ __forceinline__ void flow_vector(uint32_t nn, int& dx, int& dy) {
    dx = 0; dy = 0;
    if (nn & FV_SW) { dx = -1; dy = -1; }
    else if (nn & FV_SE) { dx = +1; dy = -1; }
    else if (nn & FV_NW) { dx = -1; dy = +1; }
    else if (nn & FV_NE) { dx = +1; dy = +1; }
    else if (nn & FV_W) { dx = -1; }
    else if (nn & FV_E) { dx = +1; }
    else if (nn & FV_S) { dy = -1; }
    else if (nn & FV_N) { dy = +1; }
}

struct PreOut {
    float2* uv;            // [nxp][nyp]
    float* slope;          // [nxp][nyp] or null
    uint8_t* uv_mask;      // [nxp][nyp] or null
    uint8_t* mask;         // [nxp][nyp] or null: pad frame | NaN ROI | NaN uv
    uint8_t* blockages;    // [nx][ny] or null
    uint8_t* blocked;      // [nx][ny] or null
    uint8_t* loop_cells;   // [nx][ny] or null
    float* gradx;          // [nx][ny] or null
    float* grady;          // [nx][ny] or null
    uint32_t* n_cells;     // 1 word or null
};

template <typename T>
__global__ void __launch_bounds__(PP_THREADS)
k_preprocess(const T* __restrict__ roi, int nx, int ny, float pixel_size, int pad, double vecsum_threshold,
             double divergence_threshold, double curl_threshold, int normalize, PreOut out) {
    __shared__ T h[PP_HX][PP_HY];
    __shared__ float su[PP_VX][PP_VY], sv[PP_VX][PP_VY], sr[PP_VX][PP_VY];  // unit velocity, raw speed
    __shared__ uint8_t code[PP_VX][PP_VY];
    __shared__ uint8_t cell[PP_CX][PP_CY];
    __shared__ uint32_t n_tile_cells;
    const int tid = threadIdx.x;
    const int x0 = blockIdx.y * PP_TX, y0 = blockIdx.x * PP_TY;
    if (tid == 0) n_tile_cells = 0;

    // A: the ROI tile, clamped (scipy's 'reflect' of a 3-wide window repeats
    // the edge pixel; the gradient and the loop fixes never read the halo
    // outside the grid)
    for (int i = tid; i < PP_HX * PP_HY; i += PP_THREADS) {
        const int a = i / PP_HY, b = i % PP_HY;
        const int gx = clampi(x0 - 2 + a, nx), gy = clampi(y0 - 2 + b, ny);
        h[a][b] = roi[(size_t)gx * ny + gy];
    }
    __syncthreads();

    // B: velocities and blockage codes on the tile plus a 1-pixel halo.
    // Halo positions outside the grid take the code of their clamped pixel
    // (the second generic_filter's 'reflect'); their velocities are unused.
    for (int i = tid; i < PP_VX * PP_VY; i += PP_THREADS) {
        const int a = i / PP_VY, b = i % PP_VY;
        const int px = x0 - 1 + a, py = y0 - 1 + b;
        // code of the clamped pixel: its 3x3 window in h (clamped loads)
        {
            const int qa = clampi(px, nx) - (x0 - 2), qb = clampi(py, ny) - (y0 - 2);
            const T c = h[qa][qb];
            uint32_t nn = 0;
            if (h[qa - 1][qb - 1] < c) nn |= FV_SW;
            if (h[qa][qb - 1] < c) nn |= FV_S;
            if (h[qa + 1][qb - 1] < c) nn |= FV_SE;
            if (h[qa - 1][qb] < c) nn |= FV_W;
            if (h[qa + 1][qb] < c) nn |= FV_E;
            if (h[qa - 1][qb + 1] < c) nn |= FV_NW;
            if (h[qa][qb + 1] < c) nn |= FV_N;
            if (h[qa + 1][qb + 1] < c) nn |= FV_NE;
            code[a][b] = (uint8_t)(((nn & 0xF0u) == nn) ? nn : 0u);
        }
        float u = 0.0f, v = 0.0f, raw = 1.0f;
        if (px >= 0 && px < nx && py >= 0 && py < ny) {
            const int ha = a + 1, hb = b + 1;  // position in h
            float gxv, gyv;
            // np.gradient, edge_order 1 (shapes below 2 are refused on the host)
            if (px == 0) gxv = (float)h[ha + 1][hb] - (float)h[ha][hb];
            else if (px == nx - 1) gxv = (float)h[ha][hb] - (float)h[ha - 1][hb];
            else gxv = ((float)h[ha + 1][hb] - (float)h[ha - 1][hb]) / 2.0f;
            if (py == 0) gyv = (float)h[ha][hb + 1] - (float)h[ha][hb];
            else if (py == ny - 1) gyv = (float)h[ha][hb] - (float)h[ha][hb - 1];
            else gyv = ((float)h[ha][hb + 1] - (float)h[ha][hb - 1]) / 2.0f;
            gxv = gxv / pixel_size;
            gyv = gyv / pixel_size;
            if (a >= 1 && a <= PP_TX && b >= 1 && b <= PP_TY) {
                const size_t gi = (size_t)px * ny + py;
                if (out.gradx) out.gradx[gi] = gxv;
                if (out.grady) out.grady[gi] = gyv;
            }
            u = -gxv;
            v = -gyv;
            raw = speed_of(u, v);
            u = u / raw;
            v = v / raw;
        }
        su[a][b] = u;
        sv[a][b] = v;
        sr[a][b] = raw;
    }
    __syncthreads();

    // C: looped cells x0-1 .. x0+TX-1 (check_has_loop on the normalised
    // velocities; cells need pixels cx+1, cy+1 inside the grid)
    for (int i = tid; i < PP_CX * PP_CY; i += PP_THREADS) {
        const int a = i / PP_CY, b = i % PP_CY;
        const int cx = x0 - 1 + a, cy = y0 - 1 + b;
        uint8_t hit = 0;
        if (cx >= 0 && cx <= nx - 2 && cy >= 0 && cy <= ny - 2) {
            const float u00 = su[a][b], v00 = sv[a][b];
            const float u10 = su[a + 1][b], v10 = sv[a + 1][b];
            const float u11 = su[a + 1][b + 1], v11 = sv[a + 1][b + 1];
            const float u01 = su[a][b + 1], v01 = sv[a][b + 1];
            const float vx = (((u00 + u10) + u11) + u01) / 4.0f;
            const float vy = (((v00 + v10) + v11) + v01) / 4.0f;
            const float speed = hypot_f32(vx, vy);  // numba: double dot product and sqrt
            const float div = (((-u00 - v00) + (u10 - v10)) + (u11 + v11)) + (-u01 + v01);
            const float curl = (((u00 - v00) + (u10 + v10)) + (-u11 + v11)) + (-u01 - v01);
            hit = ((double)speed < vecsum_threshold && (double)div <= divergence_threshold &&
                   (double)fabsf(curl) >= curl_threshold) ? 1 : 0;
            if (a >= 1 && b >= 1) {  // this tile's own cells
                if (out.loop_cells) out.loop_cells[(size_t)cx * ny + cy] = hit;
                if (hit) atomicAdd(&n_tile_cells, 1u);
            }
        } else if (a >= 1 && b >= 1 && cx < nx && cy < ny && out.loop_cells) {
            out.loop_cells[(size_t)cx * ny + cy] = 0;
        }
        cell[a][b] = hit;
    }
    __syncthreads();
    if (tid == 0 && n_tile_cells && out.n_cells) atomicAdd(out.n_cells, n_tile_cells);

    // D: PP_TX * PP_TY / PP_THREADS pixels per thread, rows PP_THREADS / PP_TY apart
    const float inv_sqrt2 = __double2float_rn(__ddiv_rn(1.0, __dsqrt_rn(2.0)));
    const int nyp = ny + 2 * pad;
#pragma unroll 1
    for (int k = tid; k < PP_TX * PP_TY; k += PP_THREADS) {
        const int a = k / PP_TY + 1, b = k % PP_TY + 1;  // position in the 1-halo arrays
        const int x = x0 + a - 1, y = y0 + b - 1;
        if (x >= nx || y >= ny) continue;
        float u = su[a][b], v = sv[a][b];
        const float raw = sr[a][b];  // speed of the unfixed gradient
        const int ha = a + 1, hb = b + 1;
        // break_out_of_loop for a pixel marked by any of its four cells
        const bool marked = cell[a][b] | cell[a - 1][b] | cell[a][b - 1] | cell[a - 1][b - 1];
        if (marked && x >= 1 && x <= nx - 2 && y >= 1 && y <= ny - 2) {
            // break_out_of_loop's vectors: W, E, S, N, SW, SE, NW, NE
            T h_min = (T)3.402823466e38f;
            int bdx = -1, bdy = 0;
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const int dx = q < 2 ? (q == 0 ? -1 : 1) : (q < 4 ? 0 : ((q & 1) ? 1 : -1));
                const int dy = q < 2 ? 0 : (q < 4 ? (q == 2 ? -1 : 1) : (q < 6 ? -1 : 1));
                const T hv = h[ha + dx][hb + dy];
                if (h_min > hv) { h_min = hv; bdx = dx; bdy = dy; }
            }
            const float len = hypot_f32((float)bdx, (float)bdy);
            u = (float)bdx / len;
            v = (float)bdy / len;
        }
        // fix_blockages: blockages, then blocked neighbours
        const uint32_t c0 = code[a][b];
        uint32_t c1 = 0;
        {
            const uint8_t sw = code[a - 1][b - 1], s = code[a][b - 1], se = code[a + 1][b - 1];
            const uint8_t w = code[a - 1][b], e = code[a + 1][b];
            const uint8_t nw = code[a - 1][b + 1], n = code[a][b + 1], ne = code[a + 1][b + 1];
            if (sw == FV_SW) c1 |= FV_SW;
            if (s == FV_SW || s == FV_SE) c1 |= FV_S;
            if (se == FV_SE) c1 |= FV_SE;
            if (w == FV_SW || w == FV_NW) c1 |= FV_W;
            if (e == FV_NE || e == FV_SE) c1 |= FV_E;
            if (nw == FV_NW) c1 |= FV_NW;
            if (n == FV_NW || n == FV_NE) c1 |= FV_N;
            if (ne == FV_NE) c1 |= FV_NE;
        }
        if (c0) {
            int dx, dy;
            flow_vector(c0, dx, dy);
            u = dx ? (float)dx * inv_sqrt2 : 0.0f;
            v = dy ? (float)dy * inv_sqrt2 : 0.0f;
        }
        if (c1) {
            int dx, dy;
            flow_vector(c1, dx, dy);
            u = dx ? (float)dx * inv_sqrt2 : 0.0f;
            v = dy ? (float)dy * inv_sqrt2 : 0.0f;
        }
        if (normalize) {
            const float sp = speed_of(u, v);
            u = u / sp;
            v = v / sp;
        } else {
            u = u * raw;
            v = v * raw;
        }
        const bool bad = isnan(u) || isnan(v);
        if (bad) { u = 0.0f; v = 0.0f; }
        const float slope = atanf(raw) * (180.0f / 3.14159265358979323846f);
        const bool roi_nan = isnan((float)h[ha][hb]);
        const size_t gi = (size_t)x * ny + y;
        if (out.blockages) out.blockages[gi] = (uint8_t)c0;
        if (out.blocked) out.blocked[gi] = (uint8_t)c1;
        // the pixel and its edge-padding replicas
        const int xa = (x == 0) ? 0 : x + pad, xb = (x == nx - 1) ? nx + 2 * pad - 1 : x + pad;
        const int ya = (y == 0) ? 0 : y + pad, yb = (y == ny - 1) ? nyp - 1 : y + pad;
        for (int qx = xa; qx <= xb; ++qx) {
            for (int qy = ya; qy <= yb; ++qy) {
                const size_t pi = (size_t)qx * nyp + qy;
                out.uv[pi] = make_float2(u, v);
                if (out.slope) out.slope[pi] = slope;
                if (out.uv_mask) out.uv_mask[pi] = bad ? 1 : 0;
                if (out.mask) {
                    const bool frame = qx < pad || qx >= nx + pad || qy < pad || qy >= ny + pad;
                    out.mask[pi] = (frame || roi_nan || bad) ? 1 : 0;
                }
            }
        }
    }
}

}  // namespace slm

using namespace slm;

extern "C" {

int slm_preprocess(const void* roi, int roi_dtype, uint32_t nx, uint32_t ny, const slm_preprocess_params* prm,
                   float* uv, float* slope, uint8_t* uv_mask, uint8_t* mask, uint8_t* blockages,
                   uint8_t* blocked_neighbors, uint8_t* loop_cells, float* gradx, float* grady,
                   uint32_t* n_loop_cells, void* stream) {
    clear_error();
    SLM_REQUIRE(roi && uv && prm, "NULL roi, uv or params");
    SLM_REQUIRE(roi_dtype == SLM_F32 || roi_dtype == SLM_F64, "roi_dtype must be SLM_F32 or SLM_F64");
    SLM_REQUIRE(nx >= 2 && ny >= 2, "the gradient needs at least 2 pixels along each axis (got %u x %u)", nx, ny);
    SLM_REQUIRE(prm->pad_width < 65536, "pad_width too large");
    const uint64_t nxp = (uint64_t)nx + 2ull * prm->pad_width, nyp = (uint64_t)ny + 2ull * prm->pad_width;
    SLM_REQUIRE(nxp < (1ull << 31) && nyp < (1ull << 31) && nxp * nyp < (1ull << 40), "grid too large");
    SLM_REQUIRE(aligned(uv, 8), "uv must be 8-byte aligned");
    SLM_REQUIRE(aligned(roi, roi_dtype == SLM_F64 ? 8 : 4), "roi misaligned");
    cudaStream_t s = (cudaStream_t)stream;
    PreOut o{(float2*)uv, slope, uv_mask, mask, blockages, blocked_neighbors, loop_cells, gradx, grady,
             n_loop_cells};
    if (n_loop_cells) SLM_CUDA(cudaMemsetAsync(n_loop_cells, 0, sizeof(uint32_t), s));
    const dim3 grid((ny + PP_TY - 1) / PP_TY, (nx + PP_TX - 1) / PP_TX);
    static_assert(PP_THREADS % PP_TY == 0 && (PP_TX * PP_TY) % PP_THREADS == 0, "tile / block shape");
    SLM_REQUIRE(grid.y < 65536, "nx too large for the tile grid");
    const float ps = (float)prm->pixel_size;
    if (roi_dtype == SLM_F64)
        k_preprocess<double><<<grid, PP_THREADS, 0, s>>>((const double*)roi, (int)nx, (int)ny, ps,
                                                             (int)prm->pad_width, prm->vecsum_threshold,
                                                             prm->divergence_threshold, prm->curl_threshold,
                                                             prm->do_normalize_speed ? 1 : 0, o);
    else
        k_preprocess<float><<<grid, PP_THREADS, 0, s>>>((const float*)roi, (int)nx, (int)ny, ps,
                                                           (int)prm->pad_width, prm->vecsum_threshold,
                                                           prm->divergence_threshold, prm->curl_threshold,
                                                           prm->do_normalize_speed ? 1 : 0, o);
    SLM_LAUNCHED("k_preprocess");
    return SLM_OK;
}

}  // extern "C"
