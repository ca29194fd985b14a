// Fast-marching hillslope lengths of the Mapping stage's pass 2
// (python/streamlines/mapping.py:841-900, fmm_lengths, which calls
// scikit-fmm's skfmm.distance once per fine subsegment).
//
// One problem per fine subsegment s of a window: the pixels with |label| ==
// |s| are grown by one pixel (4-neighbour dilation, the reference's
// generate_binary_structure(2, 1)); that grown region is the unmasked
// domain; its thin-channel pixels with |label| == |s| take phi = -1, the
// rest phi = +1.  The signed distance from phi's zero contour is marched over
// the domain, and the problem returns the sum and count of the reached
// distances (the masked array's mean is sum / count) beside the pixel counts
// the reference's ratio test uses.
//
// The method (J. A. Sethian, "Level Set Methods and Fast Marching Methods",
// 1999, ch. 8), on a unit grid, distances times dx at the end:
//   - interface points: per axis the nearest sign change along it,
//     |phi_p| / |phi_p - phi_q|; a point with crossings on both axes takes
//     1 / sqrt(1/d0^2 + 1/d1^2).  They are frozen first.
//   - update of |distance| from frozen neighbours: per axis the smaller
//     neighbour a (minus side on a tie), second order (3u - 4a + b) / 2 when
//     the next point b on that side is frozen with b <= a, else first order;
//     a frozen value across the contour enters negated.  The two-axis
//     quadratic is used when its root is >= both a, else the smaller axis
//     alone.
//   - points freeze in increasing (|distance|, row-major index) order: a
//     binary heap with stale entries skipped, so ties resolve as any other
//     store of the narrow band would.
// Every step is an IEEE double operation in a fixed order (--fmad=false), so
// the results equal the oracle's restatement of the method bit for bit.
//
// One thread runs one problem: a problem is a sequential march over a few
// hundred to a few thousand pixels, and a window's problems are independent.
// Each problem's workspace (|distance|, state, heap) is the box of its grown
// region, so it stays in L1/L2 while the thread works on it.

#include "capi_util.cuh"

namespace slm {
namespace fmm {

enum : uint8_t { FAR = 0, BAND = 1, FROZEN = 2, MASKED = 3, STATE = 3, NEG = 4 };

struct Box {
    int x0, y0, h, w;  // first row / column in the window, rows, columns
};

struct Problem {
    const Box b;
    double* val;    // |distance| in pixels; at the end signed distance x dx
    uint8_t* st;    // state | NEG
    double* hkey;   // heap keys
    int32_t* hidx;  // heap entries' local indices
    int64_t cap;    // heap capacity
    int64_t n;      // heap size
};

__device__ __forceinline__ bool heap_less(const Problem& P, int64_t i, int64_t j) {
    const double a = P.hkey[i], b = P.hkey[j];
    return a < b || (a == b && P.hidx[i] < P.hidx[j]);
}

__device__ __forceinline__ void heap_swap(Problem& P, int64_t i, int64_t j) {
    const double k = P.hkey[i];
    P.hkey[i] = P.hkey[j];
    P.hkey[j] = k;
    const int32_t x = P.hidx[i];
    P.hidx[i] = P.hidx[j];
    P.hidx[j] = x;
}

__device__ __forceinline__ bool heap_push(Problem& P, double key, int32_t idx) {
    if (P.n >= P.cap) return false;
    int64_t i = P.n++;
    P.hkey[i] = key;
    P.hidx[i] = idx;
    while (i > 0) {
        const int64_t parent = (i - 1) >> 1;
        if (!heap_less(P, i, parent)) break;
        heap_swap(P, i, parent);
        i = parent;
    }
    return true;
}

__device__ __forceinline__ void heap_pop(Problem& P, double& key, int32_t& idx) {
    key = P.hkey[0];
    idx = P.hidx[0];
    P.n -= 1;
    if (P.n == 0) return;
    P.hkey[0] = P.hkey[P.n];
    P.hidx[0] = P.hidx[P.n];
    int64_t i = 0;
    while (true) {
        const int64_t l = 2 * i + 1, r = l + 1;
        int64_t m = i;
        if (l < P.n && heap_less(P, l, m)) m = l;
        if (r < P.n && heap_less(P, r, m)) m = r;
        if (m == i) break;
        heap_swap(P, i, m);
        i = m;
    }
}

__device__ __forceinline__ bool inside(const Box& b, int x, int y) {
    return x >= 0 && x < b.h && y >= 0 && y < b.w;
}

__device__ __forceinline__ bool frozen_at(const Problem& P, int x, int y) {
    return inside(P.b, x, y) && (P.st[x * P.b.w + y] & STATE) == FROZEN;
}

// the frozen |distance| at q seen from p's side of the contour
__device__ __forceinline__ double rel(const Problem& P, int p, int q) {
    const double v = P.val[q];
    return ((P.st[p] ^ P.st[q]) & NEG) ? -v : v;
}

struct Term {
    bool ok;
    double a, alpha, beta;
};

__device__ __forceinline__ Term axis_term(const Problem& P, int x, int y, int dx, int dy, int order) {
    const int p = x * P.b.w + y;
    Term t{false, 0.0, 0.0, 0.0};
    int side = 0;
    for (int s = -1; s <= 1; s += 2) {
        const int qx = x + s * dx, qy = y + s * dy;
        if (frozen_at(P, qx, qy)) {
            const double a = rel(P, p, qx * P.b.w + qy);
            if (!t.ok || a < t.a) {
                t.ok = true;
                t.a = a;
                side = s;
            }
        }
    }
    if (!t.ok) return t;
    if (order == 2) {
        const int rx = x + 2 * side * dx, ry = y + 2 * side * dy;
        if (frozen_at(P, rx, ry)) {
            const double b = rel(P, p, rx * P.b.w + ry);
            if (b <= t.a) {
                t.alpha = 1.5;
                t.beta = (4.0 * t.a - b) / 2.0;
                return t;
            }
        }
    }
    t.alpha = 1.0;
    t.beta = t.a;
    return t;
}

// tentative |distance| at (x, y); false without a frozen neighbour
__device__ __forceinline__ bool update(const Problem& P, int x, int y, int order, double& u) {
    const Term t0 = axis_term(P, x, y, 1, 0, order);
    const Term t1 = axis_term(P, x, y, 0, 1, order);
    if (!t0.ok && !t1.ok) return false;
    Term one;
    if (t0.ok && t1.ok) {
        const bool first = t0.a <= t1.a;
        const Term lo = first ? t0 : t1, hi = first ? t1 : t0;
        const double A = lo.alpha * lo.alpha + hi.alpha * hi.alpha;
        const double B = lo.alpha * lo.beta + hi.alpha * hi.beta;
        const double C = (lo.beta * lo.beta + hi.beta * hi.beta) - 1.0;
        const double disc = B * B - A * C;
        if (disc >= 0.0) {
            const double r = (B + sqrt(disc)) / A;
            if (r >= hi.a) {
                u = r;
                return true;
            }
        }
        one = lo;
    } else {
        one = t0.ok ? t0 : t1;
    }
    u = (one.beta + 1.0) / one.alpha;
    return true;
}

// status words of one problem
enum : int32_t { OK = 0, NO_CHANNEL = 1, NO_CONTOUR = 2, HEAP_FULL = 3, BAD_BOX = 4 };

__global__ void __launch_bounds__(64)
k_fmm_lengths(const int32_t* __restrict__ label, const uint32_t* __restrict__ flags, int nx, int ny,
              uint32_t thin_bit, const int32_t* __restrict__ subsegment, const int32_t* __restrict__ box,
              const int64_t* __restrict__ offset, int n, int64_t total, int order, double dx,
              double* __restrict__ val_ws, uint8_t* __restrict__ st_ws, double* __restrict__ hkey_ws,
              int32_t* __restrict__ hidx_ws, double* __restrict__ sum, int64_t* __restrict__ count,
              int64_t* __restrict__ n_phi, int64_t* __restrict__ n_channel, int32_t* __restrict__ status) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    sum[i] = 0.0;
    count[i] = 0;
    n_phi[i] = 0;
    n_channel[i] = 0;
    const int x0 = box[4 * i], x1 = box[4 * i + 1], y0 = box[4 * i + 2], y1 = box[4 * i + 3];
    const int64_t off = offset[i];
    // the box must lie in the window and its workspace in the buffers
    if (x0 < 0 || y0 < 0 || x1 < x0 || y1 < y0 || x1 >= nx || y1 >= ny || off < 0 ||
        off + (int64_t)(x1 - x0 + 1) * (y1 - y0 + 1) > total) {
        status[i] = BAD_BOX;
        return;
    }
    const int h = x1 - x0 + 1, w = y1 - y0 + 1;
    const int64_t area = (int64_t)h * w;
    Problem P{Box{x0, y0, h, w}, val_ws + off, st_ws + off, hkey_ws + 4 * off, hidx_ws + 4 * off, 4 * area, 0};
    const int32_t s = subsegment[i];
    auto in_phi = [&](int gx, int gy) {
        if (gx < 0 || gx >= nx || gy < 0 || gy >= ny) return false;
        const int32_t v = label[(int64_t)gx * ny + gy];
        return (v < 0 ? -v : v) == s;
    };
    // the domain: |label| == |s| grown by one pixel; phi -1 on its channel
    int64_t nphi = 0, nchan = 0;
    for (int x = 0; x < h; ++x) {
        for (int y = 0; y < w; ++y) {
            const int gx = x0 + x, gy = y0 + y;
            const bool own = in_phi(gx, gy);
            const bool dil = own || in_phi(gx - 1, gy) || in_phi(gx + 1, gy) || in_phi(gx, gy - 1) ||
                             in_phi(gx, gy + 1);
            const int p = x * w + y;
            P.val[p] = 0.0;
            if (!dil) {
                P.st[p] = MASKED;
                continue;
            }
            const bool chan = own && (flags[(int64_t)gx * ny + gy] & thin_bit) == thin_bit;
            nphi += own;
            nchan += chan;
            P.st[p] = chan ? (uint8_t)(FAR | NEG) : (uint8_t)FAR;
        }
    }
    n_phi[i] = nphi;
    n_channel[i] = nchan;
    if (nchan == 0) {
        status[i] = NO_CHANNEL;
        return;
    }
    // interface points (phi is +-1 here, never 0)
    int64_t nfrozen = 0;
    for (int x = 0; x < h; ++x) {
        for (int y = 0; y < w; ++y) {
            const int p = x * w + y;
            if ((P.st[p] & STATE) == MASKED) continue;
            const double pp = (P.st[p] & NEG) ? -1.0 : 1.0;
            double inv = 0.0;
            bool crossed = false;
            for (int axis = 0; axis < 2; ++axis) {
                const int dx_ = axis == 0 ? 1 : 0, dy_ = axis == 0 ? 0 : 1;
                bool have = false;
                double dmin = 0.0;
                for (int sd = -1; sd <= 1; sd += 2) {
                    const int qx = x + sd * dx_, qy = y + sd * dy_;
                    if (!inside(P.b, qx, qy)) continue;
                    const int q = qx * w + qy;
                    if ((P.st[q] & STATE) == MASKED) continue;
                    const double pq = (P.st[q] & NEG) ? -1.0 : 1.0;
                    if ((pp > 0.0 && pq < 0.0) || (pp < 0.0 && pq > 0.0)) {
                        const double d = fabs(pp) / fabs(pp - pq);
                        if (!have || d < dmin) {
                            have = true;
                            dmin = d;
                        }
                    }
                }
                if (have) {
                    inv = inv + 1.0 / (dmin * dmin);
                    crossed = true;
                }
            }
            if (crossed) {
                P.st[p] = (uint8_t)((P.st[p] & NEG) | FROZEN);
                P.val[p] = 1.0 / sqrt(inv);
                ++nfrozen;
            }
        }
    }
    if (nfrozen == 0) {
        status[i] = NO_CONTOUR;
        return;
    }
    // the narrow band around the frozen interface
    int32_t st_code = OK;
    for (int x = 0; x < h && st_code == OK; ++x) {
        for (int y = 0; y < w; ++y) {
            const int p = x * w + y;
            if ((P.st[p] & STATE) != FAR) continue;
            double u;
            if (update(P, x, y, order, u)) {
                P.val[p] = u;
                P.st[p] = (uint8_t)((P.st[p] & NEG) | BAND);
                if (!heap_push(P, u, p)) {
                    st_code = HEAP_FULL;
                    break;
                }
            }
        }
    }
    // march: at most 4 pushes per pixel, so the loop ends
    while (st_code == OK && P.n > 0) {
        double u;
        int32_t p;
        heap_pop(P, u, p);
        if ((P.st[p] & STATE) == FROZEN || u != P.val[p]) continue;
        P.st[p] = (uint8_t)((P.st[p] & NEG) | FROZEN);
        const int x = p / w, y = p - (p / w) * w;
        const int nb[4][2] = {{x - 1, y}, {x + 1, y}, {x, y - 1}, {x, y + 1}};
        for (int k = 0; k < 4; ++k) {
            const int qx = nb[k][0], qy = nb[k][1];
            if (!inside(P.b, qx, qy)) continue;
            const int q = qx * w + qy;
            const uint8_t sq = P.st[q] & STATE;
            if (sq == MASKED || sq == FROZEN) continue;
            double v;
            update(P, qx, qy, order, v);  // p is a frozen neighbour
            if (sq == FAR || v != P.val[q]) {
                P.val[q] = v;
                P.st[q] = (uint8_t)((P.st[q] & NEG) | BAND);
                if (!heap_push(P, v, q)) {
                    st_code = HEAP_FULL;
                    break;
                }
            }
        }
    }
    if (st_code != OK) {
        status[i] = st_code;
        return;
    }
    // signed distance x dx on the reached points; their sum and count
    double acc = 0.0;
    int64_t c = 0;
    for (int64_t p = 0; p < area; ++p) {
        if ((P.st[p] & STATE) == FROZEN) {
            const double d = ((P.st[p] & NEG) ? -P.val[p] : P.val[p]) * dx;
            P.val[p] = d;
            acc = acc + d;
            ++c;
        } else {
            P.val[p] = 0.0;
        }
    }
    sum[i] = acc;
    count[i] = c;
    status[i] = OK;
}

}  // namespace fmm
}  // namespace slm

extern "C" int slm_fmm_lengths(const int32_t* label, const uint32_t* flags, int nx, int ny, uint32_t thin_bit,
                               const int32_t* subsegment, const int32_t* box, const int64_t* offset, int n,
                               int64_t total, int order, double dx, double* val_ws, uint8_t* st_ws,
                               double* hkey_ws, int32_t* hidx_ws, double* sum, int64_t* count, int64_t* n_phi,
                               int64_t* n_channel, int32_t* status, void* stream) {
    using namespace slm;
    clear_error();
    SLM_REQUIRE(nx > 0 && ny > 0, "window %d x %d", nx, ny);
    SLM_REQUIRE(n >= 0, "n %d", n);
    SLM_REQUIRE(order == 1 || order == 2, "order %d (1 or 2)", order);
    SLM_REQUIRE(total >= 0 && total < (int64_t)1 << 40, "workspace pixels %lld", (long long)total);
    SLM_REQUIRE((int64_t)nx * ny < ((int64_t)1 << 31), "window of %lld pixels", (long long)nx * ny);
    if (n == 0) return SLM_OK;
    SLM_REQUIRE(label && flags && subsegment && box && offset && val_ws && st_ws && hkey_ws && hidx_ws && sum &&
                    count && n_phi && n_channel && status,
                "null pointer");
    const int block = 64;
    fmm::k_fmm_lengths<<<(n + block - 1) / block, block, 0, (cudaStream_t)stream>>>(
        label, flags, nx, ny, thin_bit, subsegment, box, offset, n, total, order, dx, val_ws, st_ws, hkey_ws,
        hidx_ws, sum, count, n_phi, n_channel, status);
    SLM_LAUNCHED("k_fmm_lengths");
    return SLM_OK;
}
