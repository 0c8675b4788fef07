// Learned radiance cache: a small MLP (FP16 weights and activations, FP32
// accumulation on the tensor cores with mma.sync m16n8k16) that predicts the
// radiance leaving a path vertex toward the previous one, trained online on
// the integrator's own path suffixes (relative L2 loss, Adam). The reference
// renderer has no counterpart.
//
// Network: 10 inputs (position normalised to the scene box, outgoing
// direction, shading normal, roughness), each encoded as sin/cos(2^k pi x),
// k = 0..5 (120 columns) plus a constant 1 (column 120, the first layer's
// bias) padded to 128; four hidden layers of 64 with ReLU; a linear output of
// 16 columns of which the first 3 are RGB radiance. Layer l maps K_l inputs
// to N_l outputs with W_l[k][n] (FP32 master copy, row-major).
//
// One warp runs 16 rows through every layer with the activations in
// registers: the accumulator fragments of two adjacent 8-column output tiles
// are exactly the A fragment of one 16-column k-chunk of the next layer.
#pragma once

#include <cuda_fp16.h>
#include <cstdint>

namespace luz {

constexpr int kCacheIn = 10;             // raw inputs per row
constexpr int kCacheFreq = 6;            // frequencies per input
constexpr int kCacheEnc = 128;           // encoded width (120 + bias + padding)
constexpr int kCacheHidden = 64;
constexpr int kCacheOut = 16;            // padded output width (3 used)
constexpr int kCacheLayers = 5;
constexpr int kCacheRowsPerBlock = 128;  // training: 8 warps x 16 rows
constexpr int kCacheGradThreads = 2 * kCacheRowsPerBlock;

// Layer l: K inputs, N outputs, offsets of W (floats), of the forward FP16
// copy [n][K + 8] and of the backward FP16 copy [k][N + 8] (halves).
struct CacheLayer {
    int K, N, w, f, b;
};
__host__ __device__ constexpr CacheLayer cache_layer(int l)
{
    return l == 0 ? CacheLayer{128, 64, 0, 0, 0}
         : l == 1 ? CacheLayer{64, 64, 8192, 8704, 9216}
         : l == 2 ? CacheLayer{64, 64, 12288, 13312, 13824}
         : l == 3 ? CacheLayer{64, 64, 16384, 17920, 18432}
                  : CacheLayer{64, 16, 20480, 22528, 23040};
}
constexpr int kCacheParams = 21504;      // floats in W0..W4
constexpr int kCacheHalfF = 23680;       // halves in the forward copies
constexpr int kCacheHalfB = 24576;       // halves in the backward copies

// Training / query record: 10 inputs, then 3 target (or throughput) values,
// then the path slot (as float bits) and padding: 64 bytes.
struct alignas(16) CacheRecord {
    float in[kCacheIn];
    float v[3];
    uint32_t path;
    float pad[2];
};

__device__ __forceinline__ void mma16816(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1)
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}
__device__ __forceinline__ uint32_t pack_h2(float lo, float hi)
{
    const __half2 h = __floats2half2_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&h);
}
__device__ __forceinline__ float2 unpack_h2(uint32_t v)
{
    return __half22float2(*reinterpret_cast<const __half2*>(&v));
}

// Encoded column c of a row with raw inputs x: c = 12 f + 2 k + (0 sin, 1 cos).
__device__ __forceinline__ float cache_encode(const float* x, int c)
{
    if (c >= 12 * kCacheIn) return c == 12 * kCacheIn ? 1.0f : 0.0f;
    const int f = c / 12, k = (c % 12) >> 1;
    const float a = x[f] * (float)(1 << k);
    return (c & 1) ? cospif(a) : sinpif(a);
}

// A fragments of the encoded input for rows g and g + 8 of a 16-row tile.
__device__ __forceinline__ void cache_input_frags(const float* x0, const float* x1, uint32_t (&a)[8][4])
{
    const int t = threadIdx.x & 3;
#pragma unroll
    for (int kc = 0; kc < 8; kc++) {
        const int c = 16 * kc + 2 * t;
        a[kc][0] = pack_h2(cache_encode(x0, c), cache_encode(x0, c + 1));
        a[kc][1] = pack_h2(cache_encode(x1, c), cache_encode(x1, c + 1));
        a[kc][2] = pack_h2(cache_encode(x0, c + 8), cache_encode(x0, c + 9));
        a[kc][3] = pack_h2(cache_encode(x1, c + 8), cache_encode(x1, c + 9));
    }
}

// C (16 x 8 NT) = A (16 x 16 KC) x B, with B(k, n) = Ws[n * ldw + k] (pairs along k).
template <int KC, int NT>
__device__ __forceinline__ void cache_mm(const uint32_t (&a)[KC][4], const __half* Ws, int ldw, float (&c)[NT][4])
{
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int nt = 0; nt < NT; nt++) c[nt][0] = c[nt][1] = c[nt][2] = c[nt][3] = 0.0f;
#pragma unroll
    for (int kc = 0; kc < KC; kc++)
#pragma unroll
        for (int nt = 0; nt < NT; nt++) {
            const __half* row = Ws + (8 * nt + g) * ldw + 16 * kc + 2 * t;
            mma16816(c[nt], a[kc], *reinterpret_cast<const uint32_t*>(row), *reinterpret_cast<const uint32_t*>(row + 8));
        }
}

// Accumulator tiles -> A fragments of the next layer, optionally through ReLU.
template <int NT, bool RELU>
__device__ __forceinline__ void cache_chain(const float (&c)[NT][4], uint32_t (&a)[NT / 2][4])
{
#pragma unroll
    for (int kc = 0; kc < NT / 2; kc++) {
        auto r = [](float v) { return RELU ? fmaxf(v, 0.0f) : v; };
        a[kc][0] = pack_h2(r(c[2 * kc][0]), r(c[2 * kc][1]));
        a[kc][1] = pack_h2(r(c[2 * kc][2]), r(c[2 * kc][3]));
        a[kc][2] = pack_h2(r(c[2 * kc + 1][0]), r(c[2 * kc + 1][1]));
        a[kc][3] = pack_h2(r(c[2 * kc + 1][2]), r(c[2 * kc + 1][3]));
    }
}

// Forward pass of one 16-row tile; h[l] keeps the post-ReLU activations of
// hidden layer l (A-fragment layout) for the backward pass.
__device__ __forceinline__ void cache_forward(const __half* Wf, const uint32_t (&in)[8][4], uint32_t (&h)[4][4][4],
                                              float (&y)[2][4])
{
    float c[8][4];
    cache_mm<8, 8>(in, Wf + cache_layer(0).f, 128 + 8, c);
    cache_chain<8, true>(c, h[0]);
#pragma unroll
    for (int l = 1; l < 4; l++) {
        cache_mm<4, 8>(h[l - 1], Wf + cache_layer(l).f, 64 + 8, c);
        cache_chain<8, true>(c, h[l]);
    }
    cache_mm<4, 2>(h[3], Wf + cache_layer(4).f, 64 + 8, y);
}

}  // namespace luz

// The cache kernels are defined in the unit that launches them (integrator.cu);
// the shade unit (shade_kernels.cu) only needs the device-side inference above.
#ifndef LUZ_NO_CACHE_KERNELS
namespace luz {

// FP16 copies of W: forward Wf[n][K + 8] and backward Wb[k][N + 8] per layer.
__global__ void k_cache_pack(const float* W, __half* Wf, __half* Wb)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kCacheParams) return;
    int l = 0;
    while (l + 1 < kCacheLayers && i >= cache_layer(l + 1).w) l++;
    const CacheLayer L = cache_layer(l);
    const int k = (i - L.w) / L.N, n = (i - L.w) % L.N;
    const __half h = __float2half_rn(W[i]);
    Wf[L.f + n * (L.K + 8) + k] = h;
    Wb[L.b + k * (L.N + 8) + n] = h;
}

__device__ __forceinline__ void cache_load_smem(__half* dst, const __half* src, int halves)
{
    const int4* s = reinterpret_cast<const int4*>(src);
    int4* d = reinterpret_cast<int4*>(dst);
    for (int i = threadIdx.x; i < halves / 8; i += blockDim.x) d[i] = s[i];
}

// Radiance predictions for n records: out (3 floats per record) when given,
// else each record's path gets rad += throughput (record v) * max(prediction, 0).
__global__ void __launch_bounds__(128) k_cache_infer(const CacheRecord* rec, const uint32_t* count, int n_fixed,
                                                     const __half* Wf_g, float* out, float4* rad)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __half* Wf = reinterpret_cast<__half*>(smem_raw);
    cache_load_smem(Wf, Wf_g, kCacheHalfF);
    __syncthreads();
    const int n = count ? (int)*count : n_fixed;
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int tile = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; tile * 16 < n; tile += warps) {
        const int r0 = tile * 16 + g, r1 = r0 + 8;
        float x0[kCacheIn], x1[kCacheIn];
#pragma unroll
        for (int f = 0; f < kCacheIn; f++) {
            x0[f] = r0 < n ? rec[r0].in[f] : 0.0f;
            x1[f] = r1 < n ? rec[r1].in[f] : 0.0f;
        }
        uint32_t in[8][4], h[4][4][4];
        float y[2][4];
        cache_input_frags(x0, x1, in);
        cache_forward(Wf, in, h, y);
        // columns 0, 1 live in lane t = 0, column 2 in lane t = 1
        const float b0 = __shfl_down_sync(0xffffffffu, y[0][0], 1), b1 = __shfl_down_sync(0xffffffffu, y[0][2], 1);
        if (t == 0) {
            const float p0[3] = {y[0][0], y[0][1], b0}, p1[3] = {y[0][2], y[0][3], b1};
            for (int s = 0; s < 2; s++) {
                const int r = s ? r1 : r0;
                if (r >= n) continue;
                const float* p = s ? p1 : p0;
                if (out) {
                    for (int c = 0; c < 3; c++) out[3 * (size_t)r + c] = p[c];
                } else {
                    const CacheRecord& q = rec[r];
                    float4 v = rad[q.path];
                    v.x += q.v[0] * fmaxf(p[0], 0.0f);
                    v.y += q.v[1] * fmaxf(p[1], 0.0f);
                    v.z += q.v[2] * fmaxf(p[2], 0.0f);
                    rad[q.path] = v;
                }
            }
        }
    }
}

// Loss gradient of the relative L2 loss sum_c (y - t)^2 / (y^2 + 0.01) (the
// denominator held constant), clamped to +-2000, times the loss scale (|value| <= 16000, inside FP16).
constexpr float kCacheLossScale = 8.0f;
constexpr float kCacheGradClamp = 2000.0f;

// Stages a 16-row tile of A fragments (KC chunks) into shared memory rows [row][ld].
template <int KC>
__device__ __forceinline__ void cache_stage(const uint32_t (&a)[KC][4], __half* S, int ld, int row0)
{
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int kc = 0; kc < KC; kc++) {
        const int c = 16 * kc + 2 * t;
        *reinterpret_cast<uint32_t*>(S + (row0 + g) * ld + c) = a[kc][0];
        *reinterpret_cast<uint32_t*>(S + (row0 + g + 8) * ld + c) = a[kc][1];
        *reinterpret_cast<uint32_t*>(S + (row0 + g) * ld + c + 8) = a[kc][2];
        *reinterpret_cast<uint32_t*>(S + (row0 + g + 8) * ld + c + 8) = a[kc][3];
    }
}

// delta (accumulator tiles) times relu'(h) (the post-ReLU activations in A-fragment layout).
template <int NT>
__device__ __forceinline__ void cache_relu_mask(float (&c)[NT][4], const uint32_t (&h)[NT / 2][4])
{
#pragma unroll
    for (int nt = 0; nt < NT; nt++) {
        const float2 lo = unpack_h2(h[nt >> 1][(nt & 1) ? 2 : 0]);
        const float2 hi = unpack_h2(h[nt >> 1][(nt & 1) ? 3 : 1]);
        if (!(lo.x > 0.0f)) c[nt][0] = 0.0f;
        if (!(lo.y > 0.0f)) c[nt][1] = 0.0f;
        if (!(hi.x > 0.0f)) c[nt][2] = 0.0f;
        if (!(hi.y > 0.0f)) c[nt][3] = 0.0f;
    }
}

// Shared-memory layout of k_cache_grad (halves): first the forward and backward
// weight copies; once every warp has finished its backward pass, the same memory
// holds per layer the block's input rows X_l [R][K_l + 8] and output gradients
// D_l [R][N_l + 8] (R = kCacheRowsPerBlock).
constexpr int kGR = kCacheRowsPerBlock;
__host__ __device__ constexpr int cache_x_off(int l) { return l == 0 ? 0 : kGR * 136 + (l - 1) * kGR * 72; }
__host__ __device__ constexpr int cache_d_off(int l) { return cache_x_off(4) + kGR * 72 + l * kGR * 72; }
constexpr int kCacheGradStageHalves = cache_d_off(4) + kGR * 24;
constexpr int kCacheGradSmemHalves =
    kCacheGradStageHalves > kCacheHalfF + kCacheHalfB ? kCacheGradStageHalves : kCacheHalfF + kCacheHalfB;

// Rows of one training step: records [offset, offset + n) with n = min(*count -
// offset, n_max), at least 0 (count NULL: n_max).
__device__ __forceinline__ int cache_step_rows(const uint32_t* count, int offset, int n_max)
{
    return count ? max(0, min((int)*count - offset, n_max)) : n_max;
}

// Gradient of the summed loss over the step's rows (in: inputs, v: targets)
// with respect to W, times the loss scale, added into G; the summed loss into
// *loss. Launch with ceil(n_max / kCacheRowsPerBlock) blocks of kCacheGradThreads.
__global__ void __launch_bounds__(kCacheGradThreads) k_cache_grad(const CacheRecord* rec, const uint32_t* count, int offset,
                                                    int n_max, const __half* Wf_g, const __half* Wb_g, float* G,
                                                    float* loss)
{
    const int n = cache_step_rows(count, offset, n_max);
    rec += offset;
    if ((int)blockIdx.x * kCacheRowsPerBlock >= n) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __half* sm = reinterpret_cast<__half*>(smem_raw);
    __half* Wf = sm;
    __half* Wb = sm + kCacheHalfF;
    cache_load_smem(Wf, Wf_g, kCacheHalfF);
    cache_load_smem(Wb, Wb_g, kCacheHalfB);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const int row0 = warp * 16;                           // rows of this warp within the block
    const int base = blockIdx.x * kCacheRowsPerBlock + row0;
    const int r0 = base + g, r1 = r0 + 8;
    float x0[kCacheIn], x1[kCacheIn], t0[3], t1[3];
#pragma unroll
    for (int f = 0; f < kCacheIn; f++) {
        x0[f] = r0 < n ? rec[r0].in[f] : 0.0f;
        x1[f] = r1 < n ? rec[r1].in[f] : 0.0f;
    }
#pragma unroll
    for (int c = 0; c < 3; c++) {
        t0[c] = r0 < n ? rec[r0].v[c] : 0.0f;
        t1[c] = r1 < n ? rec[r1].v[c] : 0.0f;
    }
    uint32_t in[8][4], h[4][4][4];
    float y[2][4];
    cache_input_frags(x0, x1, in);
    cache_forward(Wf, in, h, y);
    // output gradient (columns 0..2)
    float dy[2][4];
    float lsum = 0.0f;
#pragma unroll
    for (int nt = 0; nt < 2; nt++)
#pragma unroll
        for (int e = 0; e < 4; e++) {
            const int col = 8 * nt + 2 * t + (e & 1);
            const bool lower = e >= 2;
            const int r = lower ? r1 : r0;
            float gsum = 0.0f;
            if (col < 3 && r < n) {
                const float yy = y[nt][e], tt = lower ? t1[col] : t0[col];
                const float den = (yy * yy) + 0.01f;
                lsum += ((yy - tt) * (yy - tt)) / den;
                gsum = fminf(kCacheGradClamp, fmaxf(-kCacheGradClamp, (2.0f * (yy - tt)) / den)) * kCacheLossScale;
            }
            dy[nt][e] = gsum;
        }
    for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
    if (lane == 0) atomicAdd(loss, lsum);
    uint32_t d[5][4][4];   // FP16 output gradients: d[0..3] hidden layers 1..4, d[4] the output (1 chunk)
    {
        uint32_t dyf[1][4];
        cache_chain<2, false>(dy, dyf);
        d[4][0][0] = dyf[0][0];
        d[4][0][1] = dyf[0][1];
        d[4][0][2] = dyf[0][2];
        d[4][0][3] = dyf[0][3];
        float c[8][4];
        cache_mm<1, 8>(dyf, Wb + cache_layer(4).b, 16 + 8, c);
        cache_relu_mask<8>(c, h[3]);
        cache_chain<8, false>(c, d[3]);
#pragma unroll
        for (int l = 3; l >= 1; l--) {
            cache_mm<4, 8>(d[l], Wb + cache_layer(l).b, 64 + 8, c);
            cache_relu_mask<8>(c, h[l - 1]);
            cache_chain<8, false>(c, d[l - 1]);
        }
    }
    // stage inputs and output gradients of every layer for the block's rows, over
    // the weight copies once every warp is done reading them
    __syncthreads();
    cache_stage<8>(in, sm + cache_x_off(0), 136, row0);
#pragma unroll
    for (int l = 1; l < 5; l++) cache_stage<4>(h[l - 1], sm + cache_x_off(l), 72, row0);
#pragma unroll
    for (int l = 0; l < 4; l++) cache_stage<4>(d[l], sm + cache_d_off(l), 72, row0);
    {
        uint32_t dl[1][4] = {{d[4][0][0], d[4][0][1], d[4][0][2], d[4][0][3]}};
        cache_stage<1>(dl, sm + cache_d_off(4), 24, row0);
    }
    __syncthreads();
    // dW_l (K x N) = X_l^T D_l over the block's rows: tiles of 16 k x 8 n, 16-row steps
    int tile = 0;
    for (int l = 0; l < kCacheLayers; l++) {
        const CacheLayer L = cache_layer(l);
        const __half* X = sm + cache_x_off(l);
        const __half* D = sm + cache_d_off(l);
        const int ldx = L.K + 8, ldd = L.N + 8;
        for (int mk = 0; mk < L.K / 16; mk++)
            for (int nj = 0; nj < L.N / 8; nj++, tile++) {
                if (tile % (kCacheGradThreads / 32) != warp) continue;
                float c[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
                for (int kb = 0; kb < kCacheRowsPerBlock / 16; kb++) {
                    const int b = 16 * kb + 2 * t, k = 16 * mk + g, j = 8 * nj + g;
                    auto hx = [&](int bb, int kk) { return X[bb * ldx + kk]; };
                    auto hd = [&](int bb, int jj) { return D[bb * ldd + jj]; };
                    auto pk = [](__half lo, __half hi) {
                        const __half2 v = __halves2half2(lo, hi);
                        return *reinterpret_cast<const uint32_t*>(&v);
                    };
                    const uint32_t a[4] = {pk(hx(b, k), hx(b + 1, k)), pk(hx(b, k + 8), hx(b + 1, k + 8)),
                                           pk(hx(b + 8, k), hx(b + 9, k)), pk(hx(b + 8, k + 8), hx(b + 9, k + 8))};
                    mma16816(c, a, pk(hd(b, j), hd(b + 1, j)), pk(hd(b + 8, j), hd(b + 9, j)));
                }
                const int k = 16 * mk + g, j = 8 * nj + 2 * t;
                atomicAdd(G + L.w + k * L.N + j, c[0]);
                atomicAdd(G + L.w + k * L.N + j + 1, c[1]);
                atomicAdd(G + L.w + (k + 8) * L.N + j, c[2]);
                atomicAdd(G + L.w + (k + 8) * L.N + j + 1, c[3]);
            }
    }
}

// Adam step (Kingma & Ba 2015) on the master weights; G holds the summed,
// loss-scaled gradient of the step's rows. Clears G for the next step.
__global__ void k_cache_adam(float* W, float* G, float* m, float* v, float lr, float b1, float b2, float eps,
                             float b1t, float b2t, const uint32_t* count, int offset, int n_max)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kCacheParams) return;
    const int n = cache_step_rows(count, offset, n_max);
    const float gr = G[i] / (kCacheLossScale * (float)max(n, 1));
    G[i] = 0.0f;
    if (n == 0 || !isfinite(gr)) return;
    const float mi = b1 * m[i] + (1.0f - b1) * gr;
    const float vi = b2 * v[i] + (1.0f - b2) * gr * gr;
    m[i] = mi;
    v[i] = vi;
    W[i] -= lr * (mi / (1.0f - b1t)) / (sqrtf(vi / (1.0f - b2t)) + eps);
}

}  // namespace luz
#endif  // LUZ_NO_CACHE_KERNELS
