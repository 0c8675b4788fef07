// nfor.cu — the NFOR denoiser (Denoise::applyNFOR, src/core/Denoise/NFOR.cpp)
// on the GPU, in FP64, one thread per pixel per pass.
//
// Passes, as applyNFOR runs them (NFOR.cpp:977-1102):
//   firefly suppression of colour A, colour B and their average   (:145-214)
//   feature prefilter of A guided by B and of B guided by A         (:398-465)
//   two-bandwidth regression of A with B's features and vice versa  (:740-831)
//   MSE estimates and bandwidth selection, each cross-filtered      (:833-950)
//   blend, then a last regression on the blended image              (:1072-1088)
// Every pixel's arithmetic follows the reference statement by statement
// (same neighbour order, same clamped coordinates, same 12 x 12 normal
// equations and Gauss-Jordan elimination with partial pivoting), so the result
// differs from the CPU's only where CUDA's exp differs from the host libm's in
// the last bit.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "luz_gpu.h"
#include "nfor.h"

namespace luz_nfor {

constexpr int kF = LUZ_NFOR_FEATURES;   // NFOR_FEATURE_COUNT
constexpr int kR = kF + 1;              // REGRESSION_SIZE
constexpr double kDblEps = 2.220446049250313e-16;   // std::numeric_limits<double>::epsilon()

struct Img {
    int w, h;
};

__device__ __forceinline__ int clampc(int v, int lim) { return v < 0 ? 0 : (v >= lim ? lim - 1 : v); }

__device__ __forceinline__ double lum(const double* c)   // colorLuminance (NFOR.cpp:92-101)
{
    const double l = c[0] * 0.2722287168 + c[1] * 0.6740817658 + c[2] * 0.0536895174;
    return (!isfinite(l) || l <= 0.0) ? 0.0 : l;
}
__device__ __forceinline__ double cdist2(const double* a, const double* b)   // colorDistanceSquared
{
    const double r = a[0] - b[0], g = a[1] - b[1], bl = a[2] - b[2];
    return ((r * r) + (g * g) + (bl * bl)) / 3.0;
}

// suppressDenoiseFireflies (NFOR.cpp:116-214); avg != 0 first averages in and in2.
__global__ void k_firefly(Img I, const double* in, const double* in2, double* out)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= I.w || y >= I.h) return;
    auto px = [&](int xx, int yy, double* c) {
        const int i = 3 * (yy * I.w + xx);
        for (int k = 0; k < 3; k++) c[k] = in2 ? (in[i + k] + in2[i + k]) * 0.5 : in[i + k];
    };
    double center[3];
    px(x, y, center);
    double* o = out + 3 * (y * I.w + x);
    for (int k = 0; k < 3; k++) o[k] = center[k];
    if (I.w < 3 || I.h < 3) return;
    const double l = lum(center);
    double nl[24], cand[24][3], cl[24];
    int nn = 0, nc = 0;
    unsigned similar = 0;
    for (int oy = -2; oy <= 2; oy++)
        for (int ox = -2; ox <= 2; ox++) {
            if (ox == 0 && oy == 0) continue;
            const int sx = x + ox, sy = y + oy;
            if (sx < 0 || sy < 0 || sx >= I.w || sy >= I.h) continue;
            double c[3];
            px(sx, sy, c);
            const double cl0 = lum(c);
            nl[nn++] = cl0;
            if (cl0 >= l * 0.65) {
                similar++;
            } else {
                for (int k = 0; k < 3; k++) cand[nc][k] = c[k];
                cl[nc] = cl0;
                nc++;
            }
        }
    if (nc == 0 || l < 0.30 || nn == 0 || similar >= 2) return;   // isDenoiseFirefly
    for (int i = 1; i < nn; i++) {   // median of the neighbour luminances
        const double v = nl[i];
        int j = i - 1;
        while (j >= 0 && nl[j] > v) {
            nl[j + 1] = nl[j];
            j--;
        }
        nl[j + 1] = v;
    }
    const double med = nl[nn / 2];
    if (!(l >= med * 2.5 && l >= med + 0.18)) return;
    // medianColorByLuminance: the candidate of rank nc / 2 by luminance
    int order[24];
    for (int i = 0; i < nc; i++) order[i] = i;
    for (int i = 1; i < nc; i++) {
        const int v = order[i];
        int j = i - 1;
        while (j >= 0 && cl[order[j]] > cl[v]) {
            order[j + 1] = order[j];
            j--;
        }
        order[j + 1] = v;
    }
    const int m = order[nc / 2];
    for (int k = 0; k < 3; k++) o[k] = cand[m][k];
}

// prefilterFeatures (NFOR.cpp:398-465); fvar = per-pixel feature variance (11 values).
__global__ void k_prefilter(Img I, const double* image, const double* guide, const double* fvar, int radius,
                            double minvar, double* out)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= I.w || y >= I.h) return;
    auto favg = [&](int i) {   // averageFeatureVariance
        double v = 0.0;
        for (int f = 0; f < kF; f++) v += fvar[(size_t)kF * i + f];
        return v / (double)kF;
    };
    const int center = y * I.w + x;
    const double cv = favg(center);
    double sum[kF];
    for (int f = 0; f < kF; f++) sum[f] = 0.0;
    double total = 0.0;
    const double sig = fmax(1.0, (double)radius);
    for (int oy = -radius; oy <= radius; oy++)
        for (int ox = -radius; ox <= radius; ox++) {
            const int s = clampc(y + oy, I.h) * I.w + clampc(x + ox, I.w);
            const double lv = cv + favg(s) + minvar;
            double d = 0.0;   // featureDistanceSquared
            for (int f = 0; f < kF; f++) {
                const double df = guide[(size_t)kF * center + f] - guide[(size_t)kF * s + f];
                d += df * df;
            }
            d = d / (double)kF;
            const double dist = d / lv;
            const double sd = (double)((ox * ox) + (oy * oy));
            const double wgt = exp(-dist / 0.25) * exp(-sd / (2.0 * sig * sig));
            for (int f = 0; f < kF; f++) sum[f] += image[(size_t)kF * s + f] * wgt;
            total += wgt;
        }
    double* o = out + (size_t)kF * center;
    if (total <= kDblEps) {
        for (int f = 0; f < kF; f++) o[f] = image[(size_t)kF * center + f];
    } else {
        for (int f = 0; f < kF; f++) o[f] = sum[f] / total;
    }
}

// patchDistance (NFOR.cpp:240-310): the clamped loop (equal to the unclamped one inside the image).
__device__ double patch_distance(Img I, const double* guide, const double* var, double vscale, int x1, int y1, int x2,
                                 int y2, int r, double minvar)
{
    if (x1 == x2 && y1 == y2) return 0.0;
    double dist = 0.0;
    unsigned n = 0;
    for (int oy = -r; oy <= r; oy++)
        for (int ox = -r; ox <= r; ox++) {
            const int a = clampc(y1 + oy, I.h) * I.w + clampc(x1 + ox, I.w);
            const int b = clampc(y2 + oy, I.h) * I.w + clampc(x2 + ox, I.w);
            const double lv = (var[a] * vscale) + (var[b] * vscale) + minvar;
            dist += cdist2(guide + 3 * a, guide + 3 * b) / lv;
            n++;
        }
    return dist / (double)n;
}
__device__ __forceinline__ double weight_from_distance(double d, double bw, double minvar)
{
    return exp(-d / fmax(minvar, bw * bw));
}

// weightedAverageFallback (NFOR.cpp:519-556)
__device__ void fallback(Img I, const double* image, const double* var, double vscale, int x, int y, int radius,
                         double minvar, double* o)
{
    double r[3] = {0.0, 0.0, 0.0}, total = 0.0;
    for (int oy = -radius; oy <= radius; oy++)
        for (int ox = -radius; ox <= radius; ox++) {
            const int s = clampc(y + oy, I.h) * I.w + clampc(x + ox, I.w);
            const double sd = (double)((ox * ox) + (oy * oy));
            const double vw = 1.0 / ((var[s] * vscale) + minvar);
            const double wgt = vw * exp(-sd / 8.0);
            for (int k = 0; k < 3; k++) r[k] += image[3 * s + k] * wgt;
            total += wgt;
        }
    if (total <= kDblEps) {
        for (int k = 0; k < 3; k++) o[k] = image[3 * (y * I.w + x) + k];
        return;
    }
    for (int k = 0; k < 3; k++) o[k] = r[k] / total;   // Color / double divides each channel
}

struct RegArgs {
    Img I;
    const double* image;     // colour (3 per pixel)
    const double* features;  // 11 per pixel
    const double* var;       // variance for the patch distance and the fallback
    double vscale;           // 2 for the doubled colour variance of the pair passes, else 1
    int radius, patch;
    double minvar;
    double bw1, bw2;         // bandwidths; bw2 < 0: single regression (regressionPass)
    double* out1;
    double* out2;
    const double* dist;      // patch distances: (2 radius + 1)^2 rows of one double per pixel (k_patch_dist)
};

// patchDistance (NFOR.cpp:482-517) of every pixel to each neighbour of its
// regression window, row k = (oy + radius) (2 radius + 1) + (ox + radius): the
// terms summed in patch order, then divided by the patch size; 0 where the
// clamped neighbour is the pixel itself. One thread per (neighbour, pixel).
__global__ void k_patch_dist(RegArgs A, double* D)
{
    const Img I = A.I;
    const long long npix = (long long)I.w * I.h;
    const int side = 2 * A.radius + 1;
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= npix * side * side) return;
    const int k = (int)(idx / npix);
    const long long pix = idx % npix;
    const int x = (int)(pix % I.w), y = (int)(pix / I.w);
    const int sx = clampc(x + (k % side - A.radius), I.w), sy = clampc(y + (k / side - A.radius), I.h);
    double d = 0.0;
    if (!(sx == x && sy == y)) {
        const int pw = 2 * A.patch + 1, P = pw * pw;
        for (int t = 0; t < P; t++) {
            const int py = t / pw - A.patch, px = t % pw - A.patch;
            const int a = clampc(y + py, I.h) * I.w + clampc(x + px, I.w);
            const int b = clampc(sy + py, I.h) * I.w + clampc(sx + px, I.w);
            const double lv = (A.var[a] * A.vscale) + (A.var[b] * A.vscale) + A.minvar;
            d += cdist2(A.image + 3 * a, A.image + 3 * b) / lv;
        }
        d = d / (double)P;
    }
    D[idx] = d;
}

// regressionPass (NFOR.cpp:674-738) / regressionPairPass (:740-831) with one
// half-warp per (pixel, bandwidth): lane c of the
// half holds column c of the 12 x 12 normal equations (c < 12) or one colour
// channel of the right-hand side (c = 12..14), in registers. Every entry is
// accumulated over the neighbours in the reference's order with the
// reference's products, the lower triangle is mirrored from the upper one
// (completeRegressionMatrix), and Gauss-Jordan elimination with partial
// pivoting (solveLinearSystemRGB) runs with the pivot column's lane choosing the
// pivot row: the reference's arithmetic, spread over the lanes instead of a
// 1.4 KB per-thread array in local memory.
// The neighbours' weights come from the precomputed patch distances, 16 at a
// time with one neighbour per lane, and reach the other lanes by shuffle.
// Pair mode (bw2 >= 0): one pixel per warp, half 0 with bw1, half 1 with bw2.
// Single mode: two pixels per warp, both with bw1.
__global__ void __launch_bounds__(128) k_regression_warp(RegArgs A)
{
    const Img I = A.I;
    const unsigned lane = threadIdx.x & 31u, half = lane >> 4, j = lane & 15u;
    const unsigned hmask = half ? 0xffff0000u : 0x0000ffffu;
    const bool pair = A.bw2 >= 0.0;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long pix = pair ? warp : 2 * warp + half;
    const long long npix = (long long)I.w * I.h;
    if (pix >= npix) return;   // both halves of a warp leave together except the last odd pixel's half
    const int x = (int)(pix % I.w), y = (int)(pix / I.w);
    const int center = y * I.w + x;
    const double bw = (pair && half) ? A.bw2 : A.bw1;
    double* out = (pair && half) ? A.out2 : A.out1;
    double M[kR];
#pragma unroll
    for (int r = 0; r < kR; r++) M[r] = (j < (unsigned)kR && r == (int)j) ? 1e-4 : 0.0;   // ridge on the diagonal
    const int side = 2 * A.radius + 1, K = side * side;
    double wreg = 0.0;
    for (int k = 0; k < K; k++) {
            if ((k & 15) == 0) {   // weights of neighbours k .. k + 15, one per lane
                const int kk = k + (int)j;
                wreg = kk < K ? weight_from_distance(A.dist[(size_t)kk * npix + pix], bw, A.minvar) : 0.0;
            }
            const double wgt = __shfl_sync(hmask, wreg, k & 15, 16);
            const int sx = clampc(x + (k % side - A.radius), I.w), sy = clampc(y + (k / side - A.radius), I.h);
            const int s = sy * I.w + sx;
            double basis[kR];
            basis[0] = 1.0;
#pragma unroll
            for (int f = 0; f < kF; f++)
                basis[f + 1] = A.features[(size_t)kF * s + f] - A.features[(size_t)kF * center + f];
            if (j < (unsigned)kR) {   // matrix column j: rows 0..j
                const double bj = j == 0 ? 1.0 : A.features[(size_t)kF * s + j - 1] - A.features[(size_t)kF * center + j - 1];
#pragma unroll
                for (int r = 0; r < kR; r++)
                    if (r <= (int)j) M[r] += (wgt * basis[r]) * bj;
            } else if (j < (unsigned)kR + 3) {   // right-hand side, channel j - 12
                const double c = A.image[3 * s + (j - kR)];
#pragma unroll
                for (int r = 0; r < kR; r++) M[r] += (wgt * basis[r]) * c;
            }
        }
    // completeRegressionMatrix: m[r][i] = m[i][r] for r > i (column i takes row i of column r)
#pragma unroll
    for (int r = 1; r < kR; r++)
#pragma unroll
        for (int i = 0; i < r; i++) {
            const double t = __shfl_sync(hmask, M[i], r, 16);
            if ((int)j == i) M[r] = t;
        }
    // Gauss-Jordan with partial pivoting (solveLinearSystemRGB)
    bool ok = true;
#pragma unroll
    for (int pv = 0; pv < kR; pv++) {
        int best = pv;
        double bv = fabs(M[pv]);
#pragma unroll
        for (int r = pv + 1; r < kR; r++) {
            const double v = fabs(M[r]);
            if (v > bv) {
                bv = v;
                best = r;
            }
        }
        best = __shfl_sync(hmask, best, pv, 16);
        bv = __shfl_sync(hmask, bv, pv, 16);
        if (bv < 1e-10) {
            ok = false;
            break;
        }
        if (best != pv) {
#pragma unroll
            for (int r = pv + 1; r < kR; r++)
                if (r == best) {
                    const double t = M[r];
                    M[r] = M[pv];
                    M[pv] = t;
                }
        }
        const double p = __shfl_sync(hmask, M[pv], pv, 16);
        const bool mine = (int)j >= pv && j < (unsigned)kR + 3;   // columns pivot.. and the right-hand side
        if (mine) M[pv] /= p;
        double f[kR];
#pragma unroll
        for (int r = 0; r < kR; r++) f[r] = __shfl_sync(hmask, M[r], pv, 16);
        if (mine) {
            const double mp = M[pv];
#pragma unroll
            for (int r = 0; r < kR; r++)
                if (r != pv) M[r] -= f[r] * mp;
        }
    }
    if (ok) {
        if (j >= (unsigned)kR && j < (unsigned)kR + 3) out[3 * center + (j - kR)] = M[0];
    } else if (j == 0) {
        fallback(I, A.image, A.var, A.vscale, x, y, A.radius, A.minvar, out + 3 * center);
    }
}

// estimateMSE (NFOR.cpp:903-922) for both bandwidths, with the doubled colour
// variance applyNFOR passes it (regressionVariance).
__global__ void k_mse(Img I, const double* ca, const double* cb, const double* fa1, const double* fb1,
                      const double* fa2, const double* fb2, const double* cvar, double* mse1, double* mse2)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= I.w || y >= I.h) return;
    const int i = y * I.w + x;
    const double var = cvar[i] * 2.0;
    auto mse = [&](const double* fa, const double* fb) {
        const double a = cdist2(cb + 3 * i, fa + 3 * i) - 2.0 * var;
        const double b = cdist2(ca + 3 * i, fb + 3 * i) - 2.0 * var;
        const double rv = cdist2(fa + 3 * i, fb + 3 * i) * 0.25;
        const double v = ((a + b) * 0.5) - rv;
        return 0.0 < v ? v : 0.0;   // std::max(0.0, v)
    };
    mse1[i] = mse(fa1, fb1);
    mse2[i] = mse(fa2, fb2);
}

// filterScalarMapPair (NFOR.cpp:833-901): patch radius 1, bandwidth 1. select != 0
// filters the bandwidth-selection maps of a and b instead of a and b.
__global__ void k_filter_pair(Img I, const double* a, const double* b, int select, const double* guide,
                              const double* gvar, int radius, double minvar, double* oa, double* ob)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= I.w || y >= I.h) return;
    auto va = [&](int s) { return select ? (a[s] <= b[s] ? 1.0 : 0.0) : a[s]; };   // bandwidthSelectionMap
    auto vb = [&](int s) { return select ? (b[s] <= a[s] ? 1.0 : 0.0) : b[s]; };
    double fa = 0.0, fb = 0.0, total = 0.0;
    const int center = y * I.w + x;
    for (int oy = -radius; oy <= radius; oy++)
        for (int ox = -radius; ox <= radius; ox++) {
            const int sx = clampc(x + ox, I.w), sy = clampc(y + oy, I.h);
            const int s = sy * I.w + sx;
            const double d = patch_distance(I, guide, gvar, 1.0, x, y, sx, sy, 1, minvar);
            const double wgt = weight_from_distance(d, 1.0, minvar);
            fa += va(s) * wgt;
            fb += vb(s) * wgt;
            total += wgt;
        }
    if (total > kDblEps) {
        oa[center] = fa / total;
        ob[center] = fb / total;
    } else {
        oa[center] = va(center);
        ob[center] = vb(center);
    }
}

// The blend of applyNFOR (NFOR.cpp:1072-1088) and combinedResultVariance (:924-936).
__global__ void k_combine(Img I, const double* sel1, const double* sel2, const double* mse1, const double* mse2,
                          const double* fa1, const double* fa2, const double* fb1, const double* fb2,
                          const double* feata, const double* featb, double minvar, double* color, double* feat,
                          double* var)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= I.w || y >= I.h) return;
    const int i = y * I.w + x;
    const double st = sel1[i] + sel2[i];
    const double w0 = st > minvar ? sel1[i] / st : (mse1[i] <= mse2[i] ? 1.0 : 0.0);
    for (int k = 0; k < 3; k++) {
        const double ra = fa1[3 * i + k] * w0 + fa2[3 * i + k] * (1.0 - w0);
        const double rb = fb1[3 * i + k] * w0 + fb2[3 * i + k] * (1.0 - w0);
        color[3 * i + k] = (ra + rb) * 0.5;
    }
    for (int f = 0; f < kF; f++)   // featureBlend(A, B, 0.5)
        feat[(size_t)kF * i + f] = feata[(size_t)kF * i + f] * 0.5 + featb[(size_t)kF * i + f] * (1.0 - 0.5);
    var[i] = cdist2(fa2 + 3 * i, fb2 + 3 * i) * 0.25;
}

}  // namespace luz_nfor

// ---------------------------------------------------------------------------- host

using namespace luz_nfor;

namespace {

thread_local std::string g_nfor_err;

struct NforError {
    int code;
    std::string msg;
};

#define NCK(x)                                                                                \
    do {                                                                                      \
        cudaError_t e_ = (x);                                                                 \
        if (e_ != cudaSuccess) throw NforError{LUZ_E_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)}; \
    } while (0)

struct Buffers {
    std::vector<void*> p;
    double* get(size_t n)
    {
        void* q = nullptr;
        NCK(cudaMalloc(&q, sizeof(double) * (n ? n : 1)));
        p.push_back(q);
        return static_cast<double*>(q);
    }
    ~Buffers()
    {
        for (void* q : p) cudaFree(q);
    }
};

LuzNforSettings checked_settings(const LuzNforSettings* st)
{
    LuzNforSettings s{1, 2, 1, 0, 1e-5};   // NFORSettings defaults (include/luz/Denoise/NFOR.hpp:39-47)
    if (st) s = *st;
    if (s.regression_radius <= 0 || s.patch_radius <= 0 || s.feature_prefilter_radius < 0)
        throw NforError{LUZ_E_INVALID, "NFOR radii must be positive."};
    return s;
}

void run_device(const double* ca, const double* cb, const double* cv, const double* ga, const double* gb,
                const double* gv, int32_t width, int32_t height, const LuzNforSettings& s, double* d_out,
                cudaStream_t st)
{
    const size_t n = (size_t)width * height;
    Buffers B;
    const Img I{width, height};
    const dim3 blk(64), grd((unsigned)((width + 63) / 64), (unsigned)height);
    // firefly suppression of A, B and of their average (applyNFOR :989-996)
    double* fa = B.get(3 * n);
    double* fb = B.get(3 * n);
    double* col = B.get(3 * n);
    k_firefly<<<grd, blk, 0, st>>>(I, ca, nullptr, fa);
    k_firefly<<<grd, blk, 0, st>>>(I, cb, nullptr, fb);
    k_firefly<<<grd, blk, 0, st>>>(I, fa, fb, col);
    // features prefiltered with the other half as the guide
    double* pfa = B.get(kF * n);
    double* pfb = B.get(kF * n);
    k_prefilter<<<grd, blk, 0, st>>>(I, ga, gb, gv, s.feature_prefilter_radius, s.min_variance, pfa);
    k_prefilter<<<grd, blk, 0, st>>>(I, gb, ga, gv, s.feature_prefilter_radius, s.min_variance, pfb);
    // two-bandwidth regressions (variance doubled)
    double* ra1 = B.get(3 * n);
    double* ra2 = B.get(3 * n);
    double* rb1 = B.get(3 * n);
    double* rb2 = B.get(3 * n);
    const unsigned rgrid_pair = (unsigned)((n * 32 + 127) / 128), rgrid_single = (unsigned)((((n + 1) / 2) * 32 + 127) / 128);
    const size_t K = (size_t)(2 * s.regression_radius + 1) * (2 * s.regression_radius + 1);
    double* dist = B.get(K * n);
    const unsigned dgrid = (unsigned)((K * n + 255) / 256);
    RegArgs A{I, fa, pfb, cv, 2.0, s.regression_radius, s.patch_radius, s.min_variance, 0.5, 1.0, ra1, ra2, dist};
    k_patch_dist<<<dgrid, 256, 0, st>>>(A, dist);
    k_regression_warp<<<rgrid_pair, 128, 0, st>>>(A);
    RegArgs Bb{I, fb, pfa, cv, 2.0, s.regression_radius, s.patch_radius, s.min_variance, 0.5, 1.0, rb1, rb2, dist};
    k_patch_dist<<<dgrid, 256, 0, st>>>(Bb, dist);
    k_regression_warp<<<rgrid_pair, 128, 0, st>>>(Bb);
    // MSE, filtered; selection, filtered (guide: the averaged colour, undoubled variance)
    double* m1 = B.get(n);
    double* m2 = B.get(n);
    double* fm1 = B.get(n);
    double* fm2 = B.get(n);
    double* s1 = B.get(n);
    double* s2 = B.get(n);
    k_mse<<<grd, blk, 0, st>>>(I, fa, fb, ra1, rb1, ra2, rb2, cv, m1, m2);
    k_filter_pair<<<grd, blk, 0, st>>>(I, m1, m2, 0, col, cv, 3, s.min_variance, fm1, fm2);
    k_filter_pair<<<grd, blk, 0, st>>>(I, fm1, fm2, 1, col, cv, 3, s.min_variance, s1, s2);
    // blend, final features and variance, last regression
    double* comb = B.get(3 * n);
    double* ff = B.get(kF * n);
    double* fv = B.get(n);
    k_combine<<<grd, blk, 0, st>>>(I, s1, s2, fm1, fm2, ra1, ra2, rb1, rb2, pfa, pfb, s.min_variance, comb, ff, fv);
    RegArgs C{I, comb, ff, fv, 1.0, s.regression_radius, s.patch_radius, s.min_variance, 1.0, -1.0, d_out, nullptr, dist};
    k_patch_dist<<<dgrid, 256, 0, st>>>(C, dist);
    k_regression_warp<<<rgrid_single, 128, 0, st>>>(C);
    NCK(cudaGetLastError());
    NCK(cudaStreamSynchronize(st));   // the scratch buffers are freed on return
}

int do_nfor(int32_t device, const LuzNforBuffers* in, int32_t width, int32_t height, const LuzNforSettings* st,
            double* rgb_out)
{
    if (!in || !rgb_out) throw NforError{LUZ_E_INVALID, "NULL argument."};
    if (width < 0 || height < 0) throw NforError{LUZ_E_INVALID, "Image size must be non-negative."};
    const LuzNforSettings s = checked_settings(st);
    if (width == 0 || height == 0) return LUZ_OK;   // empty buffers: empty image
    if (!in->color_a || !in->color_b || !in->color_variance || !in->features_a || !in->features_b || !in->feature_variance)
        throw NforError{LUZ_E_INVALID, "NFOR needs every buffer."};
    NCK(cudaSetDevice(device));
    const size_t n = (size_t)width * height;
    Buffers B;
    double* ca = B.get(3 * n);
    double* cb = B.get(3 * n);
    double* cv = B.get(n);
    double* ga = B.get(kF * n);
    double* gb = B.get(kF * n);
    double* gv = B.get(kF * n);
    double* out = B.get(3 * n);
    NCK(cudaMemcpy(ca, in->color_a, sizeof(double) * 3 * n, cudaMemcpyHostToDevice));
    NCK(cudaMemcpy(cb, in->color_b, sizeof(double) * 3 * n, cudaMemcpyHostToDevice));
    NCK(cudaMemcpy(cv, in->color_variance, sizeof(double) * n, cudaMemcpyHostToDevice));
    NCK(cudaMemcpy(ga, in->features_a, sizeof(double) * kF * n, cudaMemcpyHostToDevice));
    NCK(cudaMemcpy(gb, in->features_b, sizeof(double) * kF * n, cudaMemcpyHostToDevice));
    NCK(cudaMemcpy(gv, in->feature_variance, sizeof(double) * kF * n, cudaMemcpyHostToDevice));
    run_device(ca, cb, cv, ga, gb, gv, width, height, s, out, 0);
    NCK(cudaMemcpy(rgb_out, out, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost));
    return LUZ_OK;
}

}  // namespace

int luz_nfor_on_device(const double* ca, const double* cb, const double* cv, const double* ga, const double* gb,
                       const double* gv, int32_t width, int32_t height, const LuzNforSettings* settings,
                       double* d_out, void* stream, std::string& msg)
{
    try {
        const LuzNforSettings s = checked_settings(settings);
        if (width > 0 && height > 0)
            run_device(ca, cb, cv, ga, gb, gv, width, height, s, d_out, (cudaStream_t)stream);
        return LUZ_OK;
    } catch (const NforError& e) {
        msg = e.msg;
        return e.code;
    }
}

extern "C" int luz_gpu_nfor_error(char* buf, size_t len)
{
    if (buf && len) {
        std::strncpy(buf, g_nfor_err.c_str(), len - 1);
        buf[len - 1] = 0;
    }
    return 0;
}

extern "C" int luz_gpu_nfor_denoise(int32_t device, const LuzNforBuffers* buffers, int32_t width, int32_t height,
                                    const LuzNforSettings* settings, double* rgb_out)
{
    try {
        return do_nfor(device, buffers, width, height, settings, rgb_out);
    } catch (const NforError& e) {
        g_nfor_err = e.msg;
        return e.code;
    } catch (const std::exception& e) {
        g_nfor_err = e.what();
        return LUZ_E_CUDA;
    }
}
