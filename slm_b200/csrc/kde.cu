// kde.cu -- kernel-density estimation of log-distributions (histogram + fp64
// half-kernel smoothing), uni- and bivariate.
//
// Same arithmetic as the reference's opencl/kde.cl (k_sample :20-92,
// histogram_bivariate :109-123, pdf_bivariate_rows :144-228,
// pdf_bivariate_cols :249-361, histogram_univariate :383-394, pdf_univariate
// :426-526), including its mix of signed/unsigned 32-bit index arithmetic and
// the binary32 macros widened to double.  Histogram counts are exact (integer
// atomics).  The smoothing sums are fp64 in the reference's order; exp() and
// cos() are CUDA's, so smoothed values can differ from a host libm in the last
// bits of the double before the final rounding to float.
//
// Layout: histograms uint32 [n_hist_bins] or [n_hist_bins^2] (row = x bin),
// partial pdf float [n_hist_bins^2], pdf float [n_pdf_points] or
// [n_pdf_points^2].  The rows and cols passes take the kernel weights they
// reuse from a per-block shared-memory table.
#include <cmath>
#include "capi_util.cuh"

namespace slm {

__device__ __forceinline__ double k_sample(uint32_t kind, double x, double w) {
    switch (kind) {
    case 0: return fabs(x) < w ? 1.0 : 0.0;
    case 1: return fmax((double)1.0f - fabs(x / w), 0.0);
    case 2: return fmax((double)1.0f - (x / w) * (x / w), 0.0);
    case 3: return fmax(cos(1.57079632679489661923 * x), 0.0);
    default: {
        const double s = w * (double)0.4f;
        return exp((double)-0.5f * (x / s) * (x / s));
    }
    }
}

// float -> uint as C's truncation through a 64-bit integer
__device__ __forceinline__ uint32_t f2u(float v) { return (uint32_t)__float2ll_rz(v); }

__global__ void k_histogram_univariate(const slm_params p, const float* __restrict__ data,
                                       uint32_t n, uint32_t* __restrict__ hist) {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    const float bin_x = __fdiv_rn(data[g] - p.logx_min, p.logx_range);
    uint32_t idx = f2u(bin_x * (float)p.n_hist_bins);
    idx = idx < p.n_hist_bins - 1u ? idx : p.n_hist_bins - 1u;
    atomicAdd(hist + idx, 1u);
}

__global__ void k_histogram_bivariate(const slm_params p, const float2* __restrict__ data,
                                      uint32_t n, uint32_t* __restrict__ hist) {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    const uint32_t nb = p.n_hist_bins;
    const float2 v = data[g];
    const float bx = __fdiv_rn(v.x - p.logx_min, p.logx_range);
    const float by = __fdiv_rn(v.y - p.logy_min, p.logy_range);
    uint32_t ix = f2u(bx * (float)(nb - 1u));
    uint32_t iy = f2u(by * (float)(nb - 1u));
    ix = ix < nb - 1u ? ix : nb - 1u;
    iy = iy < nb - 1u ? iy : nb - 1u;
    atomicAdd(hist + (iy + nb * ix), 1u);
}

// one thread per pdf point (kde.cl:426-526)
__global__ void k_pdf_univariate(const slm_params p, const uint32_t* __restrict__ hist,
                                 float* __restrict__ pdf) {
    const uint32_t pdf_idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (pdf_idx >= p.n_pdf_points) return;
    const uint32_t nbpp = p.n_hist_bins / p.n_pdf_points;
    const double half_dx = (double)__fdiv_rn(p.pdf_dx, 2.0f);
    double acc = 0.0, kw = 0.0;
    for (uint32_t k = 0; k <= p.n_kdf_part_points_x; ++k) {
        const double edge = (double)k * (double)p.pdf_dx - half_dx;
        const int32_t col_r = (int32_t)(pdf_idx + k);
        const int32_t col_l = (int32_t)(pdf_idx - k + 1u);
        const bool ok_r = col_r < (int32_t)p.n_pdf_points;
        const bool ok_l = (k != 0u) && (col_l > 0);
        for (uint32_t h = 0; h < nbpp; ++h) {
            const double x = edge + (double)p.bin_dx * ((double)h + 0.5);
            const double kv = k_sample(p.kdf_kind, x, (double)p.kdf_width_x);
            const uint32_t hr = (uint32_t)col_r * nbpp + h;
            const uint32_t hl = (uint32_t)col_l * nbpp - h - 1u;
            if (ok_r) acc += (double)hist[hr] * kv;
            if (ok_l) acc += (double)hist[hl] * kv;
            if (ok_r) kw += kv;
            if (ok_l) kw += kv;
        }
    }
    pdf[pdf_idx] = (float)((double)(float)acc / kw);
}

// one thread per histogram bin; weights k_sample(k, n_y + 0.5), k = 0..n_y,
// shared per block (kde.cl:144-228)
__global__ void k_pdf_bivariate_rows(const slm_params p, const uint32_t* __restrict__ hist,
                                     float* __restrict__ partial) {
    extern __shared__ double wtab[];
    const uint32_t nk = p.n_kdf_part_points_y + 1u;
    const double k_width = (double)p.n_kdf_part_points_y + 0.5;
    for (uint32_t k = threadIdx.x; k < nk; k += blockDim.x)
        wtab[k] = k_sample(p.kdf_kind, (double)k, k_width);
    __syncthreads();
    const uint32_t nb = p.n_hist_bins;
    const uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= nb * nb) return;
    const int32_t col = (int32_t)(gid % nb);
    const int32_t row = (int32_t)(gid / nb);
    double acc = 0.0, kw = 1.0;
    for (uint32_t k = 0; k < nk; ++k) {
        const int32_t col_r = col + (int32_t)k;
        const int32_t col_l = col - (int32_t)k + 1;
        const double kv = wtab[k];
        const bool ok_r = col_r < (int32_t)nb;
        const bool ok_l = (k != 0u) && (col_l >= 0);
        const uint32_t hr = (uint32_t)row * nb + (uint32_t)col_r;
        const uint32_t hl = (uint32_t)row * nb + (uint32_t)col_l;
        if (ok_r) acc += kv * (double)hist[hr];
        if (ok_l) acc += kv * (double)hist[hl];
        if (ok_r) kw += kv;
        if (ok_l) kw += kv;
    }
    partial[gid] = (float)(acc / kw);
}

// one thread per pdf point; weights k_sample(hrow + k*nbpp, n_x + 0.5) shared
// per block (kde.cl:249-361)
__global__ void k_pdf_bivariate_cols(const slm_params p, const float* __restrict__ partial,
                                     float* __restrict__ pdf) {
    extern __shared__ double wtab[];
    const uint32_t nb = p.n_hist_bins, np = p.n_pdf_points;
    const uint32_t nbpp = nb / np;
    const uint32_t nk = p.n_kdf_part_points_x + 1u;
    const double k_width = (double)p.n_kdf_part_points_x + 0.5;
    for (uint32_t t = threadIdx.x; t < nk * nbpp; t += blockDim.x) {
        const uint32_t k = t / nbpp, hrow = t % nbpp;
        wtab[t] = k_sample(p.kdf_kind, (double)(int32_t)hrow + ((double)k) * (double)nbpp, k_width);
    }
    __syncthreads();
    const uint32_t pdf_idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (pdf_idx >= np * np) return;
    const int32_t pcol = (int32_t)(pdf_idx % np);
    const int32_t prow = (int32_t)(pdf_idx / np);
    double acc = 0.0, kw = 1.0;
    for (uint32_t k = 0; k < nk; ++k) {
        const int32_t row_dn = prow + (int32_t)k;
        const int32_t row_up = prow - (int32_t)k;
        const int32_t off_dn = (int32_t)(((uint32_t)pcol + (uint32_t)row_dn * nb) * nbpp);
        const int32_t off_up = (int32_t)(((uint32_t)pcol + (uint32_t)row_up * nb) * nbpp);
        for (int32_t hrow = 0; hrow < (int32_t)nbpp; ++hrow) {
            const double kv = wtab[k * nbpp + (uint32_t)hrow];
            for (int32_t hcol = 0; hcol < (int32_t)nbpp; ++hcol) {
                const int32_t i_dn = (int32_t)((uint32_t)off_dn + (uint32_t)hrow * nb + (uint32_t)hcol);
                const int32_t i_up = (int32_t)((uint32_t)off_up + (nbpp - 1u - (uint32_t)hrow) * nb
                                               + (uint32_t)hcol);
                const bool ok_dn = i_dn < (int32_t)(nb * nb);
                const bool ok_up = (k != 0u) && (i_up >= 0);
                if (ok_dn) acc += kv * (double)partial[(uint32_t)i_dn];
                if (ok_up) acc += kv * (double)partial[(uint32_t)i_up];
                if (ok_dn) kw += kv;
                if (ok_up) kw += kv;
            }
        }
    }
    pdf[pdf_idx] = (float)(acc / kw);
}

}  // namespace slm

using namespace slm;

static int check_kde(const slm_params* p, bool bivariate) {
    SLM_REQUIRE(p != nullptr, "params is NULL");
    SLM_REQUIRE(p->n_hist_bins > 0 && p->n_pdf_points > 0, "n_hist_bins and n_pdf_points must be > 0");
    SLM_REQUIRE(p->n_hist_bins % p->n_pdf_points == 0,
                "n_hist_bins (%u) must be a multiple of n_pdf_points (%u)", p->n_hist_bins,
                p->n_pdf_points);
    SLM_REQUIRE(p->kdf_kind <= 4, "kdf_kind %u unknown", p->kdf_kind);
    if (bivariate)
        SLM_REQUIRE((uint64_t)p->n_hist_bins * p->n_hist_bins < (1ull << 31),
                    "n_hist_bins^2 must fit a signed 32-bit index");
    return SLM_OK;
}

extern "C" {

int slm_histogram_univariate(const slm_params* p, const float* sl, uint32_t n_data, uint32_t* hist,
                             void* stream) {
    clear_error();
    int rc = check_kde(p, false);
    if (rc) return rc;
    if (n_data == 0) return SLM_OK;
    SLM_REQUIRE(sl && hist, "NULL buffer");
    const unsigned block = 256, grid = (n_data + block - 1) / block;
    k_histogram_univariate<<<grid, block, 0, (cudaStream_t)stream>>>(*p, sl, n_data, hist);
    SLM_LAUNCHED("k_histogram_univariate");
    return SLM_OK;
}

int slm_histogram_bivariate(const slm_params* p, const float* sl, uint32_t n_data, uint32_t* hist,
                            void* stream) {
    clear_error();
    int rc = check_kde(p, true);
    if (rc) return rc;
    if (n_data == 0) return SLM_OK;
    SLM_REQUIRE(sl && hist && aligned(sl, 8), "NULL or misaligned buffer");
    const unsigned block = 256, grid = (n_data + block - 1) / block;
    k_histogram_bivariate<<<grid, block, 0, (cudaStream_t)stream>>>(
        *p, reinterpret_cast<const float2*>(sl), n_data, hist);
    SLM_LAUNCHED("k_histogram_bivariate");
    return SLM_OK;
}

int slm_pdf_univariate(const slm_params* p, const uint32_t* hist, float* pdf, void* stream) {
    clear_error();
    int rc = check_kde(p, false);
    if (rc) return rc;
    SLM_REQUIRE(hist && pdf, "NULL buffer");
    const unsigned block = 128, grid = (p->n_pdf_points + block - 1) / block;
    k_pdf_univariate<<<grid, block, 0, (cudaStream_t)stream>>>(*p, hist, pdf);
    SLM_LAUNCHED("k_pdf_univariate");
    return SLM_OK;
}

int slm_pdf_bivariate_rows(const slm_params* p, const uint32_t* hist, float* partial, void* stream) {
    clear_error();
    int rc = check_kde(p, true);
    if (rc) return rc;
    SLM_REQUIRE(hist && partial, "NULL buffer");
    const size_t smem = (size_t)(p->n_kdf_part_points_y + 1u) * sizeof(double);
    SLM_REQUIRE(smem <= 160 * 1024, "n_kdf_part_points_y %u too large", p->n_kdf_part_points_y);
    if (smem > 48 * 1024)
        SLM_CUDA(cudaFuncSetAttribute(k_pdf_bivariate_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const uint64_t n = (uint64_t)p->n_hist_bins * p->n_hist_bins;
    const unsigned block = 256, grid = (unsigned)((n + block - 1) / block);
    k_pdf_bivariate_rows<<<grid, block, smem, (cudaStream_t)stream>>>(*p, hist, partial);
    SLM_LAUNCHED("k_pdf_bivariate_rows");
    return SLM_OK;
}

int slm_pdf_bivariate_cols(const slm_params* p, const float* partial, float* pdf, void* stream) {
    clear_error();
    int rc = check_kde(p, true);
    if (rc) return rc;
    SLM_REQUIRE(partial && pdf, "NULL buffer");
    const uint32_t nbpp = p->n_hist_bins / p->n_pdf_points;
    const size_t smem = (size_t)(p->n_kdf_part_points_x + 1u) * nbpp * sizeof(double);
    SLM_REQUIRE(smem <= 160 * 1024, "n_kdf_part_points_x %u too large", p->n_kdf_part_points_x);
    if (smem > 48 * 1024)
        SLM_CUDA(cudaFuncSetAttribute(k_pdf_bivariate_cols, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const uint64_t n = (uint64_t)p->n_pdf_points * p->n_pdf_points;
    const unsigned block = 128, grid = (unsigned)((n + block - 1) / block);
    k_pdf_bivariate_cols<<<grid, block, smem, (cudaStream_t)stream>>>(*p, partial, pdf);
    SLM_LAUNCHED("k_pdf_bivariate_cols");
    return SLM_OK;
}

}  // extern "C"
