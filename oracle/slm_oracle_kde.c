/* slm_oracle_kde.c -- TEST INFRASTRUCTURE ONLY: CPU restatement of the
 * reference's kernel-density estimation kernels (opencl/kde.cl of
 * atthecodeface/slm), used as the parity oracle.  Never linked into the
 * product library.
 *
 *   k_sample (5 shapes)      kde.cl:20-92
 *   histogram_bivariate      kde.cl:109-123
 *   filter_along_rows        kde.cl:144-199, pdf_bivariate_rows kde.cl:202-228
 *   filter_along_cols        kde.cl:249-330, pdf_bivariate_cols kde.cl:333-361
 *   histogram_univariate     kde.cl:383-394
 *   filter                   kde.cl:426-484, pdf_univariate kde.cl:500-526
 *
 * Integer arithmetic keeps the reference's mix of signed and unsigned 32-bit
 * types (int*uint is unsigned, converted back to int on assignment), and
 * float macros (PDF_DX, BIN_DX, KDF_WIDTH_X, ...) are binary32 values widened
 * to double where the reference widens them.  float->uint conversion is C's
 * truncation through a 64-bit integer (what x86-64 compilers emit).
 */
#include <math.h>
#include <stdint.h>
#include "slm_b200.h"

double oracle_k_sample(uint32_t kind, double x, double w) {
    switch (kind) {
    case 0: return fabs(x) < w ? 1.0 : 0.0;                            /* tophat */
    case 1: return fmax((double)1.0f - fabs(x / w), 0.0);               /* triangle */
    case 2: return fmax((double)1.0f - (x / w) * (x / w), 0.0);         /* epanechnikov */
    case 3: return fmax(cos(M_PI_2 * x), 0.0);                          /* cosine */
    default: {                                                          /* gaussian */
        const double s = w * (double)0.4f;
        return exp((double)-0.5f * (x / s) * (x / s));
    }
    }
}

static inline uint32_t f2u(float v) { return (uint32_t)(int64_t)v; }

/* histogram_univariate over data[0..n) */
void oracle_histogram_univariate(const slm_params* p, const float* data, uint32_t n,
                                 uint32_t* hist) {
    for (uint32_t g = 0; g < n; ++g) {
        const float bin_x = (data[g] - p->logx_min) / p->logx_range;
        uint32_t idx = f2u(bin_x * (float)p->n_hist_bins);
        idx = idx < p->n_hist_bins - 1u ? idx : p->n_hist_bins - 1u;
        hist[idx] += 1u;
    }
}

/* histogram_bivariate over data[0..n) (x,y pairs) */
void oracle_histogram_bivariate(const slm_params* p, const float* data, uint32_t n,
                                uint32_t* hist) {
    const uint32_t nb = p->n_hist_bins;
    for (uint32_t g = 0; g < n; ++g) {
        const float bin_x = (data[2 * (size_t)g] - p->logx_min) / p->logx_range;
        const float bin_y = (data[2 * (size_t)g + 1] - p->logy_min) / p->logy_range;
        uint32_t ix = f2u(bin_x * (float)(nb - 1u));
        uint32_t iy = f2u(bin_y * (float)(nb - 1u));
        ix = ix < nb - 1u ? ix : nb - 1u;
        iy = iy < nb - 1u ? iy : nb - 1u;
        hist[iy + nb * ix] += 1u;
    }
}

/* pdf_univariate: pdf[0..n_pdf_points) from hist[0..n_hist_bins) */
void oracle_pdf_univariate(const slm_params* p, const uint32_t* hist, float* pdf) {
    const uint32_t nbpp = p->n_hist_bins / p->n_pdf_points;
    const double half_dx = (double)(p->pdf_dx / 2.0f);
    for (uint32_t pdf_idx = 0; pdf_idx < p->n_pdf_points; ++pdf_idx) {
        double acc = 0.0, kw = 0.0;
        for (uint32_t k = 0; k <= p->n_kdf_part_points_x; ++k) {
            const double k_bin_point = (double)k * (double)p->pdf_dx;
            const double k_bin_edge = k_bin_point - half_dx;
            const int32_t col_r = (int32_t)(pdf_idx + k);
            const int32_t col_l = (int32_t)(pdf_idx - k + 1u);
            const int ok_r = col_r < (int32_t)p->n_pdf_points;
            const int ok_l = (k != 0u) & (col_l > 0);
            for (uint32_t h = 0; h < nbpp; ++h) {
                const double x = k_bin_edge + (double)p->bin_dx * ((double)h + 0.5);
                const double kv = oracle_k_sample(p->kdf_kind, x, (double)p->kdf_width_x);
                uint32_t hr = (uint32_t)col_r * nbpp + h;
                uint32_t hl = (uint32_t)col_l * nbpp - h - 1u;
                hr = ok_r ? hr : 0u;
                hl = ok_l ? hl : 0u;
                if (ok_r) acc += (double)hist[hr] * kv;
                if (ok_l) acc += (double)hist[hl] * kv;
                if (ok_r) kw += kv;
                if (ok_l) kw += kv;
            }
        }
        pdf[pdf_idx] = (float)((double)(float)acc / kw);
    }
}

/* pdf_bivariate_rows: partial[0..nb*nb) from hist[0..nb*nb) */
void oracle_pdf_bivariate_rows(const slm_params* p, const uint32_t* hist, float* partial) {
    const uint32_t nb = p->n_hist_bins;
    const double k_width = (double)p->n_kdf_part_points_y + 0.5;
    for (uint32_t gid = 0; gid < nb * nb; ++gid) {
        double acc = 0.0, kw = 1.0;
        const int32_t col = (int32_t)(gid % nb);
        const int32_t row = (int32_t)(gid / nb);
        for (uint32_t k = 0; k <= p->n_kdf_part_points_y; ++k) {
            const int32_t col_r = col + (int32_t)k;
            const int32_t col_l = col - (int32_t)k + 1;
            const double kv = oracle_k_sample(p->kdf_kind, (double)k, k_width);
            const int ok_r = col_r < (int32_t)nb;
            const int ok_l = (k != 0u) & (col_l >= 0);
            int32_t hr = (int32_t)((uint32_t)row * nb + (uint32_t)col_r);
            int32_t hl = (int32_t)((uint32_t)row * nb + (uint32_t)col_l);
            hr = ok_r ? hr : 0;
            hl = ok_l ? hl : 0;
            if (ok_r) acc += kv * (double)hist[(uint32_t)hr];
            if (ok_l) acc += kv * (double)hist[(uint32_t)hl];
            if (ok_r) kw += kv;
            if (ok_l) kw += kv;
        }
        partial[gid] = (float)(acc / kw);
    }
}

/* pdf_bivariate_cols: pdf[0..np*np) from partial[0..nb*nb) */
void oracle_pdf_bivariate_cols(const slm_params* p, const float* partial, float* pdf) {
    const uint32_t nb = p->n_hist_bins, np = p->n_pdf_points;
    const uint32_t nbpp = nb / np;
    const double k_width = (double)p->n_kdf_part_points_x + 0.5;
    for (uint32_t pdf_idx = 0; pdf_idx < np * np; ++pdf_idx) {
        double acc = 0.0, kw = 1.0;
        const int32_t pcol = (int32_t)(pdf_idx % np);
        const int32_t prow = (int32_t)(pdf_idx / np);
        for (uint32_t k = 0; k <= p->n_kdf_part_points_x; ++k) {
            const int32_t row_dn = prow + (int32_t)k;
            const int32_t row_up = prow - (int32_t)k;
            const int32_t off_dn = (int32_t)(((uint32_t)pcol + (uint32_t)row_dn * nb) * nbpp);
            const int32_t off_up = (int32_t)(((uint32_t)pcol + (uint32_t)row_up * nb) * nbpp);
            for (int32_t hrow = 0; hrow < (int32_t)nbpp; ++hrow) {
                const double kx = (double)hrow + ((double)k) * (double)nbpp;
                const double kv = oracle_k_sample(p->kdf_kind, kx, k_width);
                for (int32_t hcol = 0; hcol < (int32_t)nbpp; ++hcol) {
                    int32_t i_dn = (int32_t)((uint32_t)off_dn + (uint32_t)hrow * nb + (uint32_t)hcol);
                    int32_t i_up = (int32_t)((uint32_t)off_up + (nbpp - 1u - (uint32_t)hrow) * nb
                                             + (uint32_t)hcol);
                    const int ok_dn = i_dn < (int32_t)(nb * nb);
                    const int ok_up = (k != 0u) & (i_up >= 0);
                    i_dn = ok_dn ? i_dn : 0;
                    i_up = ok_up ? i_up : 0;
                    if (ok_dn) acc += kv * (double)partial[(uint32_t)i_dn];
                    if (ok_up) acc += kv * (double)partial[(uint32_t)i_up];
                    if (ok_dn) kw += kv;
                    if (ok_up) kw += kv;
                }
            }
        }
        pdf[pdf_idx] = (float)(acc / kw);
    }
}
