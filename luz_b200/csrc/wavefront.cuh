// wavefront.cuh — per-path device logic of the wavefront integrator (state
// layout, camera rays, the shade step); kernels live in integrator.cu.
#pragma once
#include "cache.cuh"
#include "caustics.cuh"
#include "shade.cuh"

namespace luz {

constexpr int kMaxBounceSlots = 256;
constexpr int kBlock = 128;
constexpr int kShadeClasses = 10;           // 0 = miss, 1..9 = material type of the hit

struct Ctrl {
    uint32_t count[kMaxBounceSlots + 2];    // extension queue size entering bounce b
    uint32_t shadow[kMaxBounceSlots + 2];   // shadow rays emitted at bounce b
    uint32_t fetch_ext[kMaxBounceSlots + 2];
    uint32_t fetch_sh[kMaxBounceSlots + 2];
    uint32_t bin[kMaxBounceSlots + 2][kShadeClasses];   // paths of bounce b per shade class
};

struct PathBuf {
    float4* ray_o;
    float4* ray_d;
    float4* thr;       // xyz throughput, w previous scatter pdf
    float4* rad;       // xyz radiance, w flags
    float4* pend0;     // pending light-NEE contribution
    float4* pend1;     // pending environment-NEE contribution
    uint32_t* pixel;
    uint32_t* sample;
    float4* hit;       // t, u, v, object (bits)
    int32_t* hit_prim;
    uint32_t* queue0;
    uint32_t* queue1;
    float4* sh_o;      // xyz origin, w tmax
    float4* sh_d;      // xyz direction, w path | slot << 31 (bits)
    int2* sh_x;        // source primitive excluded from the shadow ray
    float4* color;     // per-path final colour
    float4* feat;      // NFOR primary-vertex features 2..10, 3 float4 per path (NULL unless requested)
    uint32_t* bins;    // kShadeClasses segments of bin_stride paths, filled by extend in hit-class order
                       // (NULL: shade reads the extension queue as it is)
    uint32_t bin_stride;
    uint32_t* seg;     // multi-scene waves: the wave segment (scene) of each path; NULL otherwise
    uint32_t* sort_keys;   // coherence sort of the extension queue (tuning): key per queue entry,
    uint32_t* qsort;       // the sorted queue,
    uint32_t* sort_hist;   // and the per-key counts / offsets (kSortBins)
};

// Training snapshot of a path at its cache vertex: inputs, throughput and the
// radiance gathered before the vertex's own light (emission excepted).
struct CacheSnap {
    float in[kCacheIn];
    float thr[3];
    float rad[3];
};

// Path-replay state of a Metal vertex whose roughness texture is differentiated
// (luz_gpu_adjoint_backward on a roughness texture): d ln f / d roughness per
// channel for the light-sample direction, the environment-sample direction and
// the continuation, and where the texture was read.
struct AdjRough {
    float dn0[3], dn1[3], dc[3];
    float u, v;
    uint32_t active;
};

struct WaveArgs {
    int32_t width, height;
    uint32_t seed, stream;
    int32_t pix_begin, pix_count;
    int32_t s_begin, s_count;
    int32_t sample_offset;
    int32_t max_bounces;
    int64_t n;                    // paths in this wave
    const int32_t* list_x;        // list mode (trace_paths): explicit (x, y, s)
    const int32_t* list_y;
    const int32_t* list_s;
    int32_t list_mode;
    const uint32_t* pix_list;     // pixel of each pixel slot (adaptive rounds); NULL = pix_begin + slot
    int32_t half_streams;         // NFOR: sample s runs on sampler stream 1 + s % 2
    int32_t nfor;                 // store primary features in PathBuf.feat
    int32_t adjoint;              // replay pass of luz_gpu_adjoint_backward
    int32_t grad_texture;         // texture whose texel gradient is accumulated
    int32_t grad_kind;            // 0: Lambertian albedo texture; 1: Metal roughness texture (red channel)
    AdjRough* adj_rough;          // grad_kind 1: one record per path
    int32_t grad_emission;        // replay: gradient with respect to each light's emitted radiance
    double* grad_light;           // kEmissionReplicas copies of light_count * 3 (summed on the host)
    int32_t* pend_light;          // per path: light of the pending light sample, -1 = none
    int32_t grad_volume;          // replay: GObject index of the volume whose density is differentiated, -1 = none
    double* grad_density;         // kEmissionReplicas partial sums of dLoss/d(density)
    float2* dens_score;           // per path: score of the path so far, score of its pending light samples
    const float* adj_rgb;         // dLoss/dPixel, W*H*3
    double* grad;                 // dLoss/dTexel, texture W*H*3
    double inv_spp;
    GCamera cam;
    // radiance-cache render (luz_gpu_render_cached)
    int32_t cache_prefix;         // first bounce whose surface vertex queries the cache
    uint32_t cache_train_every;   // one training path in this many
    uint32_t cache_wave;          // wave counter: varies the training paths
    CacheRecord* cache_q;         // queries of the paths that end at the cache
    CacheSnap* cache_s;           // training snapshots, one slot per path
    uint8_t* cache_flag;          // 1 where the path left a training snapshot
    uint32_t* cache_count;        // [0] queries
    float cache_lo[3], cache_inv[3];   // position input = (p - lo) * inv
    float cache_min_rough;        // vertices rougher than this (cache_roughness) query the cache
    uint32_t cache_self_train;    // 1: a training path queries the cache at its next eligible vertex
    const uint32_t* sorted_queue;   // extension queue in coherence order for bounces >= 1 (NULL: as shaded)
    // multi-scene waves (luz_gpu_batch_render): one WaveArgs per segment of a wave, the
    // segment's scene and the first wave slot it covers
    int32_t batch_scene;
    int32_t batch_pad;
    int64_t batch_offset;
};


enum PathFlags : uint32_t { PF_PREV_SPECULAR = 1u, PF_PREV_SVIL = 2u, PF_CACHE_DONE = 4u };

// Pixel of slot `i` of a width x height image walked in 8x8 tiles: tiles row
// by row, Z-order inside a full tile, row-major inside the partial tiles of the
// right and bottom edges. A bijection of [0, width*height); the 16 or 32
// consecutive pixels of a warp form a 4x4 or 8x4 block, so its rays start
// close together and traverse the same BVH nodes more often than a row strip.
__device__ __forceinline__ void tiled_pixel(uint32_t i, uint32_t width, uint32_t height, uint32_t& x, uint32_t& y)
{
    const uint32_t ty = i / (8u * width);
    const uint32_t r = i - ty * (8u * width);
    const uint32_t th = min(8u, height - 8u * ty);
    const uint32_t tx = r / (8u * th);
    const uint32_t q = r - tx * (8u * th);
    const uint32_t tw = min(8u, width - 8u * tx);
    uint32_t lx, ly;
    if (tw == 8u && th == 8u) {
        lx = (q & 1u) | ((q >> 1) & 2u) | ((q >> 2) & 4u);
        ly = ((q >> 1) & 1u) | ((q >> 2) & 2u) | ((q >> 3) & 4u);
    } else {
        ly = q / tw;
        lx = q - ly * tw;
    }
    x = 8u * tx + lx;
    y = 8u * ty + ly;
}

// (x, y, sample) of path p. The result of a path depends on these alone (the
// sampler keys on them), not on which slot of a wave carries it.
__device__ __forceinline__ void path_coords(const WaveArgs& w, uint32_t p, uint32_t& x, uint32_t& y, uint32_t& s)
{
    if (w.list_mode) {
        x = (uint32_t)w.list_x[p];
        y = (uint32_t)w.list_y[p];
        s = (uint32_t)w.list_s[p];
        return;
    }
    const uint32_t slot = (uint32_t)w.pix_begin + p / (uint32_t)w.s_count;
    s = (uint32_t)(w.s_begin + w.sample_offset) + p % (uint32_t)w.s_count;
    if (w.pix_list) {
        const uint32_t pix = w.pix_list[slot];
        x = pix % (uint32_t)w.width;
        y = pix / (uint32_t)w.width;
    } else {
        tiled_pixel(slot, (uint32_t)w.width, (uint32_t)w.height, x, y);
    }
}

__device__ __forceinline__ Key path_key(const WaveArgs& w, uint32_t x, uint32_t y, uint32_t s, uint32_t bounce)
{
    // _threadRender with denoise buffers: beginPixelSample(x, y, s, s % 2 + 1) (Threads.cpp:593-598).
    const uint32_t stream = w.half_streams ? 1u + (s & 1u) : w.stream;
    return Key{base_key(w.seed, x, y, stream), s, bounce};
}

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

// Warp-aggregated queue append: one atomicAdd per warp (ballot + popc).
__device__ __forceinline__ uint32_t warp_append(uint32_t* counter, bool pred)
{
    const unsigned mask = __ballot_sync(0xffffffffu, pred);
    if (!mask) return 0;
    const uint32_t lane = lane_id();
    const int leader = __ffs(mask) - 1;
    uint32_t base = 0;
    if ((int)lane == leader) base = atomicAdd(counter, (uint32_t)__popc(mask));
    base = __shfl_sync(0xffffffffu, base, leader);
    return base + (uint32_t)__popc(mask & ((1u << lane) - 1u));
}

// _generateRay (src/renderer/RayHelper.cpp:85-106) in FP64, rounded to FP32.
static __device__ void camera_ray(const WaveArgs& w, uint32_t x, uint32_t y, uint32_t s, double* o, double* d)
{
    const Key k = path_key(w, x, y, s, 0);
    const GCamera& c = w.cam;
    const S2 cs = sample2d(k, DIM_CAMERA);
    const double xu = ((double)x + (double)cs.x) * c.inv_w1;
    const double yv = ((double)y + (double)cs.y) * c.inv_h1;
    double off[3] = {0.0, 0.0, 0.0};
    if (c.lens_radius > 0.0) {
        float dx, dy;
        unit_disk(k, DIM_LENS, dx, dy);
        const double rx = (double)dx * c.lens_radius, ry = (double)dy * c.lens_radius;
        for (int a = 0; a < 3; a++) off[a] = c.u[a] * rx + c.v[a] * ry;
    }
    for (int a = 0; a < 3; a++) {
        o[a] = c.position[a] + off[a];
        d[a] = (((c.lower_left[a] - (c.horizontal[a] * xu)) - (c.vertical[a] * yv)) - c.position[a]) - off[a];
    }
    const double len = sqrt((d[0] * d[0]) + (d[1] * d[1]) + (d[2] * d[2]));
    if (!isfinite(len) || len <= 0.0) {
        d[0] = d[1] = d[2] = 0.0;
    } else {
        const double il = 1.0 / len;
        for (int a = 0; a < 3; a++) d[a] = il * d[a];
    }
}

// ---------------------------------------------------------------------------- shade

__device__ __forceinline__ F3 clamp_ray_color(F3 c)   // clampRayColor (ColorHelper.cpp:259-274)
{
    const float l = luminance(c);
    if (!isfinite(l)) return F3{0.f, 0.f, 0.f};
    if (l > 1.0e12f) c = c * (1.0e12f / l);
    return c;
}
__device__ __forceinline__ F3 clamp_color_lum(F3 c, float maxl)
{
    const float l = luminance(c);
    if (!isfinite(l)) return F3{0.f, 0.f, 0.f};
    if (maxl > 0.0f && l > maxl) c = c * (maxl / l);
    return c;
}
__device__ __forceinline__ F3 clamp_bg_miss(const DScene& S, F3 c)   // clampConstantBackgroundMiss
{
    const float bl = S.k.background_luminance;
    if (!isfinite(bl) || bl <= 0.0f) return c;
    return clamp_color_lum(c, bl * 4.0f);
}
__device__ __forceinline__ float power_heuristic(float a, float b)
{
    const float f = a * a, s = b * b, sum = f + s;
    if (sum <= 0.0f || !isfinite(sum)) return 0.0f;
    return f / sum;
}
__device__ __forceinline__ bool terminated(F3 t)
{
    const float m = maxc(t);
    return !isfinite(m) || m <= 1e-6f;
}
__device__ __forceinline__ bool russian_roulette(F3& thr, int bounce, const Key& k)
{
    if (bounce < 3) return true;
    float surv = maxc(thr);
    surv = fmaxf(0.05f, fminf(0.95f, surv));
    if (sample1d(k, DIM_RUSSIAN_ROULETTE) > (double)surv) return false;
    thr = cdiv(thr, surv);
    return true;
}
__device__ __forceinline__ bool leaves_opaque(const GMaterial& m, const Hit& h, F3 dir)
{
    if (m.flags & MF_CAN_TRANSMIT) return true;
    F3 g = h.gn;
    if (len2(g) <= 1e-12f) g = h.n;
    if (len2(g) <= 1e-12f) return true;
    return dot(g, dir) > 1e-7f;
}
__device__ __forceinline__ float direct_prob(int bounce) { return bounce < 2 ? 1.0f : 0.5f; }

// relocateSubsurfaceExit (ColorHelper.cpp:428-504)
static __device__ __noinline__ void relocate_subsurface(const DScene& S, const GMaterial& m, Hit& h, Scatter& sr, F3 ray_d, const Key& k)
{
    if (!sr.subsurface || sr.thin) return;
    const float dl = maxc(sr.ss_radius_m);
    if (!isfinite(dl) || dl <= 0.0f) return;
    const double comp = sample1d(k, DIM_SUBSURFACE_PROFILE_COMPONENT);
    const S2 rs = sample2d(k, DIM_SUBSURFACE_SPATIAL);
    const float u = fmaxf(1e-12f, fminf(1.0f - 1e-12f, rs.y));
    const float scale = comp < 0.25 ? dl : 3.0f * dl;
    const float radius_m = -scale * logf(1.0f - u);
    const float mpu = (float)S.k.meters_per_unit;
    if (radius_m <= 0.0f || !isfinite(radius_m) || mpu <= 0.0f) return;
    const float radius = radius_m / mpu;
    if (radius <= kTMin) return;
    F3 n = h.n;
    if (len2(n) <= 1e-12f) n = h.gn;
    if (len2(n) <= 1e-12f) return;
    n = normalize(n);
    const Onb b = make_onb(n);
    const float ang = 2.0f * kPiF * rs.x;
    const F3 off = onb_local(b, cosf(ang) * radius, sinf(ang) * radius, 0.0f);
    const F3 cand = h.p + off;
    const float probe = fmaxf(radius + (4.0f * dl / mpu), 16.0f * kTMin);
    const TRay pr = make_ray(cand + n * probe, ray_dir_normalized(n * -1.0f));
    VolSample vs{&k, 0.0, false};
    LocalStack<true> st;
    const THit th = closest_hit<TF_ALL>(S, pr, kTMin, kInf, vs, st);
    if (th.obj < 0) return;
    const Hit eh = make_hit(S, pr, th);
    if (eh.material != h.material || eh.t <= kTMin || eh.t > (2.0f * probe + kTMin)) return;
    // refreshSubsurfaceScatterAtExit (ColorHelper.cpp:395-426)
    const F3 dir = onb_local(make_onb(eh.n), cosine_hemisphere(k, DIM_BSDF_DIRECTION));
    const float pdf = bsdf_pdf(S, m, eh, ray_d, dir);
    const F3 bc = bsdf_eval(S, m, eh, ray_d, dir);
    if (pdf <= 0.0f || !isfinite(pdf) || maxc(bc) <= 0.0f) return;
    h = eh;
    sr.dir = dir;
    sr.spdf = pdf;
    sr.att = cdiv(bc, pdf);
}

struct ShadeOut {
    int32_t xobj, xprim;   // source primitive of the next ray and the shadow rays
    bool cont;
    F3 next_o, next_d;
    bool sh[2];
    F3 sh_o[2], sh_d[2];
    float sh_t[2];
};

// NFOR primary-vertex features (primaryMissFeatures / primaryHitFeatures,
// src/renderer/ColorHelper.cpp:725-799), entries 2..10; entries 0 and 1 (the
// pixel coordinates) are formed in FP64 when the samples are accumulated.
__device__ __forceinline__ float nfor_channel(float v)
{
    if (!isfinite(v) || v <= 0.0f) return 0.0f;
    return (float)fmin(1.0, log1p((double)v) / log1p(1.0e12));   // D_MAX_RAY_COLOR_LUMINANCE
}
static __device__ __noinline__ void store_miss_features(const PathBuf& P, uint32_t p, F3 sky)
{
    P.feat[3 * p] = make_float4(0.0f, 1.0f, 0.5f, 0.5f);
    P.feat[3 * p + 1] = make_float4(0.5f, nfor_channel(sky.x), nfor_channel(sky.y), nfor_channel(sky.z));
    P.feat[3 * p + 2] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
}
static __device__ __noinline__ void store_hit_features(const DScene& S, const PathBuf& P, uint32_t p, const Hit& h,
                                                const GMaterial& m)
{
    double nx = h.n.x, ny = h.n.y, nz = h.n.z;
    const double l2 = nx * nx + ny * ny + nz * nz;
    if (l2 > 0.0) {
        const double l = sqrt(l2);
        nx /= l;
        ny /= l;
        nz /= l;
    }
    const double t = h.t;
    const F3 albedo = color_at(S, m, h);
    P.feat[3 * p] = make_float4(1.0f, t > 0.0 ? (float)(t / (1.0 + t)) : 0.0f, (float)(nx * 0.5 + 0.5),
                                (float)(ny * 0.5 + 0.5));
    P.feat[3 * p + 1] = make_float4((float)(nz * 0.5 + 0.5), nfor_channel(albedo.x), nfor_channel(albedo.y),
                                    nfor_channel(albedo.z));
    P.feat[3 * p + 2] = make_float4((float)((double)m.type / (double)MT_PRINCIPLED), 0.0f, 0.0f, 0.0f);
}

// Adds g * (bilinear weight) to channel ch of the four texels a lookup at (u, v)
// of the differentiated texture reads (texture_sample's footprint).
__device__ __forceinline__ void scatter_texel_grad(const DScene& S, const WaveArgs& w, float u0, float v0, int ch, double g)
{
    if (g == 0.0 || !isfinite(g)) return;
    const GTexture T = S.textures[w.grad_texture];
    const float u = wrap01f(u0), v = wrap01f(v0);
    const float x = u * (float)(T.width - 1);
    const float y = (1.0f - v) * (float)(T.height - 1);
    const int x0 = (int)floorf(x), y0 = (int)floorf(y);
    const int x1 = min(x0 + 1, T.width - 1), y1 = min(y0 + 1, T.height - 1);
    const float tx = x - (float)x0, ty = y - (float)y0;
    const double wt[4] = {(double)((1.0f - tx) * (1.0f - ty)), (double)(tx * (1.0f - ty)), (double)((1.0f - tx) * ty),
                          (double)(tx * ty)};
    const int idx[4] = {y0 * T.width + x0, y0 * T.width + x1, y1 * T.width + x0, y1 * T.width + x1};
    for (int q = 0; q < 4; q++)
        if (wt[q] != 0.0) atomicAdd(&w.grad[3 * (int64_t)idx[q] + ch], g * wt[q]);
}

// d ln f / d roughness of a rough Metal lobe toward dir, per channel, by a central
// difference of the BSDF in roughness (alpha = roughness^2 >= 1e-4); 0 where f is 0.
static __device__ __noinline__ F3 dlnf_rough(const DScene& S, const GMaterial& m, const Hit& h, F3 ray_d, F3 dir)
{
    const F3 f = bsdf_eval(S, m, h, ray_d, dir);
    const float r = m.roughness, r1 = fminf(1.0f, r + 1e-3f), r0 = fmaxf(0.0f, r - 1e-3f);
    GMaterial a = m, b = m;
    a.alpha = fmaxf(1e-4f, r1 * r1);
    b.alpha = fmaxf(1e-4f, r0 * r0);
    const F3 fa = bsdf_eval(S, a, h, ray_d, dir), fb = bsdf_eval(S, b, h, ray_d, dir);
    const float inv = 1.0f / (r1 - r0);
    auto q = [&](float x, float y, float z) { return (z > 0.0f && isfinite(z)) ? ((x - y) * inv) / z : 0.0f; };
    return F3{q(fa.x, fb.x, f.x), q(fa.y, fb.y, f.y), q(fa.z, fb.z, f.z)};
}

// Roughness gradient of the vertex recorded in ar, once its light (a) and
// environment (b) samples are known after the shadow test: each contribution
// times its d ln f, the continuation (final path radiance L minus the radiance
// gathered up to this vertex's samples, rad) times d ln f of its direction
// (sampling densities held fixed: each sample's f / pdf is differentiated in f).
static __device__ __noinline__ void adjoint_rough_resolve(const DScene& S, const WaveArgs& w, const PathBuf& P, uint32_t p,
                                                   F3 a, F3 b, F3 rad, bool continued, AdjRough& ar)
{
    const float4 L = P.color[p];
    const uint32_t pix = P.pixel[p];
    const float la[3] = {a.x, a.y, a.z}, lb[3] = {b.x, b.y, b.z}, lr[3] = {rad.x, rad.y, rad.z};
    const float Lc[3] = {L.x, L.y, L.z};
    double g = 0.0;
    for (int ch = 0; ch < 3; ch++) {
        const double cont = continued ? (double)Lc[ch] - (double)lr[ch] : 0.0;
        const double term = (double)la[ch] * ar.dn0[ch] + (double)lb[ch] * ar.dn1[ch] + cont * ar.dc[ch];
        if (isfinite(term)) g += (double)w.adj_rgb[3 * (int64_t)pix + ch] * term;
    }
    scatter_texel_grad(S, w, ar.u, ar.v, 0, g * w.inv_spp);
    ar.active = 0;
}

// Emission gradient of light `light` for a contribution c of its emitted
// radiance E reaching pixel pix: adj * c / E per channel (contributions are
// linear in E; light selection weights are held fixed).
// Warps add into one of kEmissionReplicas copies, so that a scene with one light
// does not serialise every path on three addresses.
constexpr int kEmissionReplicas = 256;
__device__ __forceinline__ void adjoint_emission_add(const DScene& S, const WaveArgs& w, uint32_t pix, int32_t light, F3 c)
{
    if (light < 0 || light >= S.k.light_count) return;
    const int64_t rep = (int64_t)((blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) & (kEmissionReplicas - 1));
    double* gl = w.grad_light + rep * 3 * (int64_t)S.k.light_count;
    const float* E = S.lights[light].emitted;
    const float cc[3] = {c.x, c.y, c.z};
    for (int ch = 0; ch < 3; ch++) {
        if (!(E[ch] > 0.0f) || !isfinite(cc[ch]) || cc[ch] == 0.0f) continue;
        const double g = (double)w.adj_rgb[3 * (int64_t)pix + ch] * (double)cc[ch] / (double)E[ch] * w.inv_spp;
        atomicAdd(&gl[3 * (int64_t)light + ch], g);
    }
}

// Density gradient (luz_gpu_adjoint_density): a score-function estimate. The
// distance a bounce's rays sample in the differentiated medium is hd = -ln(u) /
// density (ConstantVolume.cpp:62-121), density p(hd) = density e^(-density hd),
// score d ln p / d density = 1 / density - hd; one u per bounce serves every
// ray of the bounce (the extension ray that reaches the vertex and the light
// samples leaving it), so the score is counted once for them. Every
// contribution is multiplied by the summed scores of the draws it depends on.
__device__ __forceinline__ float density_score(const DScene& S, const WaveArgs& w, const Key& k)
{
    const GObject& O = S.objects[w.grad_volume];
    const double sigma = -1.0 / (double)O.f[6];
    const double hd = (double)O.f[6] * log(fmax(sample1d(k, DIM_VOLUME_DISTANCE), 1e-12));
    return (float)(1.0 / sigma - hd);
}
__device__ __forceinline__ void density_add(const DScene& S, const WaveArgs& w, uint32_t pix, F3 c, float score)
{
    const double g = ((double)w.adj_rgb[3 * (int64_t)pix] * c.x + (double)w.adj_rgb[3 * (int64_t)pix + 1] * c.y
                      + (double)w.adj_rgb[3 * (int64_t)pix + 2] * c.z) * (double)score * w.inv_spp;
    if (g == 0.0 || !isfinite(g)) return;
    const int64_t rep = (int64_t)((blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) & (kEmissionReplicas - 1));
    atomicAdd(&w.grad_density[rep], g);
}

// Path replay gradient of a Lambertian albedo texture (luz_gpu_adjoint_backward).
// Everything the path gathers from this vertex on (its NEE and every later
// vertex) carries the vertex's albedo = colour * clamp01(bilinear(texels)) as
// one factor per channel, so with L the path's final radiance (stored by the
// first pass) and `before` what it had gathered before this vertex:
//   dL/dtexel = (L - before) / bilinear(u, v) * (bilinear weight of the texel)
// per channel, zero where the clamp is active. The pixel's film is the mean of
// cleanColor(L) over its samples, so each path adds adj(pixel) / spp times that.
// Russian roulette's survival probability is held fixed (not differentiated).
static __device__ __noinline__ void adjoint_texture(const DScene& S, const WaveArgs& w, const PathBuf& P, uint32_t p,
                                             const Hit& h, F3 before)
{
    const float4 L = P.color[p];
    const uint32_t pix = P.pixel[p];
    const GTexture T = S.textures[w.grad_texture];
    const float u = wrap01f(h.u), v = wrap01f(h.v);
    const float x = u * (float)(T.width - 1);
    const float y = (1.0f - v) * (float)(T.height - 1);
    const int x0 = (int)floorf(x), y0 = (int)floorf(y);
    const int x1 = min(x0 + 1, T.width - 1), y1 = min(y0 + 1, T.height - 1);
    const float tx = x - (float)x0, ty = y - (float)y0;
    const float4 c00 = __ldg(S.texels + T.offset + y0 * T.width + x0);
    const float4 c10 = __ldg(S.texels + T.offset + y0 * T.width + x1);
    const float4 c01 = __ldg(S.texels + T.offset + y1 * T.width + x0);
    const float4 c11 = __ldg(S.texels + T.offset + y1 * T.width + x1);
    const F3 top = (F3{c00.x, c00.y, c00.z} * (1.0f - tx)) + (F3{c10.x, c10.y, c10.z} * tx);
    const F3 bot = (F3{c01.x, c01.y, c01.z} * (1.0f - tx)) + (F3{c11.x, c11.y, c11.z} * tx);
    const F3 raw = (top * (1.0f - ty)) + (bot * ty);
    const double wt[4] = {(double)((1.0f - tx) * (1.0f - ty)), (double)(tx * (1.0f - ty)), (double)((1.0f - tx) * ty),
                          (double)(tx * ty)};
    const int idx[4] = {y0 * T.width + x0, y0 * T.width + x1, y1 * T.width + x0, y1 * T.width + x1};
    const float Lc[3] = {L.x, L.y, L.z}, bc[3] = {before.x, before.y, before.z}, rc[3] = {raw.x, raw.y, raw.z};
    for (int ch = 0; ch < 3; ch++) {
        if (!(rc[ch] > 0.0f && rc[ch] < 1.0f) || !isfinite(Lc[ch])) continue;
        const double g = (double)w.adj_rgb[3 * (int64_t)pix + ch] * w.inv_spp * ((double)Lc[ch] - (double)bc[ch])
                       / (double)rc[ch];
        if (g == 0.0 || !isfinite(g)) continue;
        for (int q = 0; q < 4; q++)
            if (wt[q] != 0.0) atomicAdd(&w.grad[3 * (int64_t)idx[q] + ch], g * wt[q]);
    }
}

// The ray the atmosphere integrates along, in FP64: at bounce 0 the camera ray
// is regenerated in FP64 (a planet-scale origin loses metres in FP32), later
// rays are the FP32 ray widened.
static __device__ __noinline__ void atmos_ray(const WaveArgs& w, const PathBuf& P, uint32_t p, int bounce, const TRay& ray,
                                       double* o, double* d)
{
    if (bounce == 0) {
        const uint32_t pix = P.pixel[p];
        camera_ray(w, pix % (uint32_t)w.width, pix / (uint32_t)w.width, P.sample[p], o, d);
        return;
    }
    o[0] = ray.o.x; o[1] = ray.o.y; o[2] = ray.o.z;
    d[0] = ray.d.x; d[1] = ray.d.y; d[2] = ray.d.z;
}

// CAUSTICS: the scene has a caustic photon map (a separate instantiation, so
// that scenes without one keep the leaner kernel).
// Roughness the radiance cache sees: 1 for diffuse and volume phase materials.
__device__ __forceinline__ float cache_roughness(const GMaterial& m)
{
    const bool diffuse = m.type == MT_LAMBERTIAN || m.type == MT_ISOTROPIC || m.type == MT_HG || m.type == MT_EMISSIVE;
    return diffuse ? 1.0f : m.roughness;
}

// Radiance-cache inputs at a surface hit: position in the scene box, outgoing
// direction, shading normal, roughness (1 for diffuse and volume phase materials).
__device__ __forceinline__ void cache_inputs(const WaveArgs& w, const Hit& h, const GMaterial& m, F3 ray_d, float* in)
{
    in[0] = (h.p.x - w.cache_lo[0]) * w.cache_inv[0];
    in[1] = (h.p.y - w.cache_lo[1]) * w.cache_inv[1];
    in[2] = (h.p.z - w.cache_lo[2]) * w.cache_inv[2];
    const F3 wo = safe_normalize(ray_d * -1.0f, h.n);
    in[3] = wo.x;
    in[4] = wo.y;
    in[5] = wo.z;
    in[6] = h.n.x;
    in[7] = h.n.y;
    in[8] = h.n.z;
    in[9] = cache_roughness(m);
}

// MODE 0: plain; 1: with the caustic photon map; 2: radiance-cache render;
// 3: adjoint (gradient) passes.
template <int MODE>
static __device__ void shade_path(const DScene& S, const WaveArgs& w, const PathBuf& P, uint32_t p, int bounce, ShadeOut& out)
{
    out.cont = false;
    out.sh[0] = out.sh[1] = false;
    out.xobj = -1;
    out.xprim = -1;
    const float4 t4 = P.thr[p], r4 = P.rad[p];
    F3 thr{t4.x, t4.y, t4.z};
    F3 rad{r4.x, r4.y, r4.z};
    uint32_t flags = __float_as_uint(r4.w);
    const float prev_pdf = t4.w;
    F3 pend_in{0.f, 0.f, 0.f};   // the previous vertex's light samples, as the shadow test left them

    {
        const float4 a = P.pend0[p], b = P.pend1[p];
        pend_in = F3{a.x, a.y, a.z} + F3{b.x, b.y, b.z};
        rad = (rad + F3{a.x, a.y, a.z}) + F3{b.x, b.y, b.z};
        if (MODE == 3 && w.adjoint && w.grad_kind == 1 && w.adj_rough[p].active)
            adjoint_rough_resolve(S, w, P, p, F3{a.x, a.y, a.z}, F3{b.x, b.y, b.z}, rad, true, w.adj_rough[p]);
        if (MODE == 3 && w.adjoint && w.grad_emission && w.pend_light[p] >= 0) {   // the last vertex's light sample
            adjoint_emission_add(S, w, P.pixel[p], w.pend_light[p], F3{a.x, a.y, a.z});
            w.pend_light[p] = -1;
        }
    }
    if constexpr (MODE == 2) {   // a training snapshot taken at the previous vertex: radiance up to its NEE
        if (w.cache_flag[p] == 2) {
            CacheSnap& sn = w.cache_s[p];
            sn.rad[0] = rad.x;
            sn.rad[1] = rad.y;
            sn.rad[2] = rad.z;
            w.cache_flag[p] = 1;
        }
    }
    F3 pend0{0.f, 0.f, 0.f}, pend1{0.f, 0.f, 0.f};
    const float4 ro = P.ray_o[p], rd = P.ray_d[p];
    const TRay ray = make_ray_x(F3{ro.x, ro.y, ro.z}, F3{rd.x, rd.y, rd.z}, __float_as_int(ro.w), __float_as_int(rd.w));
    const float4 h4 = P.hit[p];
    const int32_t obj = __float_as_int(h4.w);
    const uint32_t pix = P.pixel[p];
    const Key k = path_key(w, pix % (uint32_t)w.width, pix / (uint32_t)w.width, P.sample[p], (uint32_t)bounce);
    const bool prev_spec = (flags & PF_PREV_SPECULAR) != 0;
    // density gradient: scores of the draws this vertex's contributions depend on
    float dscore = 0.0f, dscore_b = 0.0f;
    bool dext = false;
    F3 rad_start = rad;
    if constexpr (MODE == 3) {
        if (w.adjoint && w.grad_volume >= 0) {
            const float2 ds = w.dens_score[p];
            density_add(S, w, pix, pend_in, ds.y);
            const float t_hit = obj < 0 ? kInf : h4.x;
            dscore_b = density_score(S, w, k);
            dext = volume_overlap(S.objects[w.grad_volume], ray.o, ray.d, kTMin, t_hit) > 0.0f;
            dscore = ds.x + (dext ? dscore_b : 0.0f);
        }
    }

    if (obj < 0) {   // miss (ColorHelper.cpp:1169-1210)
        float env_mis = 1.0f;
        const bool need_pdf = bounce > 0 && !prev_spec && (flags & PF_PREV_SVIL);
        const bool need_rad = (S.k.sky == 3 || S.k.sky == 2) && S.k.env.present;
        F3 env_rad{0.f, 0.f, 0.f};
        float env_p = 0.0f;
        if ((need_pdf && S.k.env.lighting) || need_rad) env_query(S, ray.d, need_rad, need_pdf && S.k.env.lighting, env_rad, env_p);
        if (need_pdf) {
            float ipdf = 0.0f;
            if (S.k.env.lighting) ipdf = env_p;
            else if (S.k.has_constant_background_light) ipdf = 1.0f / (4.0f * kPiF);
            env_mis = power_heuristic(prev_pdf, ipdf);
        }
        F3 sky;
        if (S.k.sky == 1) {   // SKY_LINEAR: _calculateSkyInterpolation (Atmospherics.cpp:44-53), skyline 0.5
            const float tl = 0.5f * ((ray.d.y / sqrtf(len2(ray.d))) + 1.0f);
            sky = (F3{1.0f, 1.0f, 1.0f} * (1.0f - tl)) + (F3{0.5f, 0.7f, 1.0f} * tl);
        } else if (S.k.sky == 2) {   // sampleAtmosphereSky (ColorHelper.cpp:590-605)
            double ao[3], ad[3];
            atmos_ray(w, P, p, bounce, ray, ao, ad);
            const AtmosSample a = atmos_segment(S, ao, ad, kDblMax);
            double bg[3];
            if (need_rad) {
                const F3 e = (env_rad * S.k.env.strength) * env_mis;
                bg[0] = e.x; bg[1] = e.y; bg[2] = e.z;
            } else {
                bg[0] = bg[1] = bg[2] = atmos_stars(S, k, a.in);
            }
            sky = F3{(float)(a.in[0] + a.tr[0] * bg[0]), (float)(a.in[1] + a.tr[1] * bg[1]),
                     (float)(a.in[2] + a.tr[2] * bg[2])};
        } else if (need_rad) {
            sky = (env_rad * S.k.env.strength) * env_mis;
        } else {
            sky = f3(S.k.background) * env_mis;
        }
        if (bounce == 0 && w.nfor) store_miss_features(P, p, sky);   // env_mis is 1 at bounce 0
        F3 contrib = thr * sky;
        if (bounce > 0 && S.k.has_constant_background_light) contrib = clamp_bg_miss(S, contrib);
        rad = rad + clamp_ray_color(contrib);
        goto done;
    }
    {
        THit th{h4.x, obj, P.hit_prim[p], h4.y, h4.z};
        Hit h = make_hit(S, ray, th);
        // The material is read where it lies (L1-cached global memory); only a Metal whose
        // roughness comes from a texture gets a resolved copy.
        const GMaterial* mp = S.materials + h.material;
        GMaterial m_res;
        if (mp->rtexture >= 0) {
            m_res = *mp;
            resolve_material(S, m_res, h);
            mp = &m_res;
        }
        const GMaterial& m = *mp;
        if (bounce == 0 && w.nfor) store_hit_features(S, P, p, h, m);
        if (bounce == 0 && S.k.sky == 2) {   // compositePrimaryAtmosphereSegment (ColorHelper.cpp:645-659)
            double ao[3], ad[3];
            atmos_ray(w, P, p, bounce, ray, ao, ad);
            const AtmosSample a = atmos_segment(S, ao, ad, primary_atmos_tmax(S, ao, ad, (double)h.t));
            rad = rad + clamp_ray_color(thr * F3{(float)a.in[0], (float)a.in[1], (float)a.in[2]});
            thr = clamp_ray_color(thr * F3{(float)a.tr[0], (float)a.tr[1], (float)a.tr[2]});
            if (terminated(thr)) goto done;
        }
        const F3 emitted = m.type == MT_EMISSIVE ? f3(m.color) : F3{0.f, 0.f, 0.f};
        Scatter sr;
        if (!scatter(S, m, h, ray.d, k, sr)) {
            // previousScatterOrigin: read only after a non-specular scatter, whose hit point is this ray's origin
            const float plp = (!prev_spec && S.k.light_count > 0) ? lights_pdf(S, ray.o, ray.d) : 0.0f;
            const float wgt = prev_spec ? 1.0f : power_heuristic(prev_pdf, plp);
            rad = rad + clamp_ray_color((thr * emitted) * wgt);
            if (MODE == 3 && w.adjoint && w.grad_emission && m.type == MT_EMISSIVE) {   // an emitter hit
                for (int32_t li = 0; li < S.k.light_count; li++)
                    if (S.lights[li].object == h.obj) {
                        adjoint_emission_add(S, w, pix, li, clamp_ray_color((thr * emitted) * wgt));
                        break;
                    }
            }
            goto done;
        }
        relocate_subsurface(S, m, h, sr, ray.d, k);
        if (!h.volume) {
            out.xobj = h.obj;
            out.xprim = h.prim;
        }
        F3 att = sr.att;
        if (!h.front && sr.absorb) {   // effectiveScatterAttenuation + mediumTransmittance
            const float dm = h.t * (float)S.k.meters_per_unit;
            if (isfinite(dm) && dm > 0.0f)
                att = att * F3{expf(-sr.absorption.x * dm), expf(-sr.absorption.y * dm), expf(-sr.absorption.z * dm)};
        }
        if (sr.specular) {
            if (!leaves_opaque(m, h, sr.dir)) goto done;
            thr = clamp_ray_color(thr * att);
            if (terminated(thr) || !russian_roulette(thr, bounce, k)) goto done;
            out.cont = true;
            out.next_o = h.p;
            out.next_d = sr.dir;
            flags = PF_PREV_SPECULAR | (flags & PF_CACHE_DONE);
            P.thr[p] = make_float4(thr.x, thr.y, thr.z, 0.0f);
            goto done;
        }
        rad = rad + thr * emitted;
        // Radiance cache: at the path's first surface vertex at or after the prefix
        // bounce, the vertex's own light (emission here, NEE below) stays explicit and
        // the cache answers for the continuation; one path in cache_train_every runs
        // on and records what the continuation gathered, itself ended in the cache at
        // the path's next eligible vertex (after the first wave).
        bool cache_query = false;
        if constexpr (MODE == 2) {
            if (bounce >= w.cache_prefix && !h.volume && (flags & PF_CACHE_DONE) && w.cache_self_train &&
                w.cache_flag[p] == 1 && cache_roughness(m) >= w.cache_min_rough) {
                cache_query = true;   // a training path's next eligible vertex: its target ends in the cache
            } else if (bounce >= w.cache_prefix && !h.volume && !(flags & PF_CACHE_DONE) &&
                cache_roughness(m) >= w.cache_min_rough) {
                const uint64_t key = ((uint64_t)pix << 24) ^ (uint64_t)P.sample[p] ^ ((uint64_t)w.cache_wave << 48);
                if (splitmix64(key) % w.cache_train_every == 0) {
                    CacheSnap& sn = w.cache_s[p];
                    cache_inputs(w, h, m, ray.d, sn.in);
                    sn.thr[0] = thr.x;
                    sn.thr[1] = thr.y;
                    sn.thr[2] = thr.z;
                    w.cache_flag[p] = 2;   // radiance up to this vertex's NEE: taken at the next vertex
                    flags |= PF_CACHE_DONE;
                } else {
                    cache_query = true;
                }
            }
        }
        if (MODE == 3 && w.adjoint && w.grad_kind == 0 && m.type == MT_LAMBERTIAN && m.texture == w.grad_texture)
            adjoint_texture(S, w, P, p, h, rad);
        const bool rough_grad =
            MODE == 3 && w.adjoint && w.grad_kind == 1 && m.type == MT_METAL && m.rtexture == w.grad_texture;
        if (rough_grad) {
            AdjRough& ar = w.adj_rough[p];
            for (int c = 0; c < 3; c++) ar.dn0[c] = ar.dn1[c] = ar.dc[c] = 0.0f;
            ar.u = h.u;
            ar.v = h.v;
            ar.active = 1;
        }
        if (terminated(thr * att)) goto done;
        if constexpr (MODE == 1)
            if (S.cm.count) rad = rad + clamp_ray_color(thr * caustic_estimate(S, h, sr, m, ray.d));
        if (S.k.light_count > 0) {   // estimateDirectLighting (ColorHelper.cpp:973-1033)
            const float prob = direct_prob(bounce);
            bool go = true;
            if (prob < 1.0f && sample1d(k, DIM_LIGHT_STRATEGY) >= (double)prob) go = false;
            LightSample ls;
            if (go && sample_light(S, h.p, k, ls) && leaves_opaque(m, h, ls.dir)) {
                const float sp = scatter_pdf(S, sr, m, h, ray.d, ls.dir);
                const F3 bc = scatter_bsdfcos(S, sr, m, h, ray.d, ls.dir);
                if (!(sp <= 0.0f || !isfinite(sp) || maxc(bc) <= 0.0f)) {
                    const float mis = power_heuristic(ls.pdf, sp);
                    const F3 c = (bc * ls.emitted) * (mis / (ls.pdf * prob));
                    pend0 = clamp_ray_color(thr * c);
                    out.sh[0] = true;
                    if (MODE == 3 && w.adjoint && w.grad_emission) w.pend_light[p] = ls.light;
                    if (rough_grad) {
                        const F3 dl = dlnf_rough(S, m, h, ray.d, ls.dir);
                        w.adj_rough[p].dn0[0] = dl.x;
                        w.adj_rough[p].dn0[1] = dl.y;
                        w.adj_rough[p].dn0[2] = dl.z;
                    }
                    out.sh_o[0] = h.p;
                    out.sh_d[0] = ls.dir;
                    out.sh_t[0] = ls.tmax - kTMin;
                }
            }
        }
        if (S.k.sampled_infinite_light) {   // estimateEnvironmentLighting (ColorHelper.cpp:1035-1098)
            const bool cbg = S.k.has_constant_background_light != 0;
            bool go = !(cbg && sr.pdf == PDF_BSDF);
            const float prob = direct_prob(bounce);
            if (go && prob < 1.0f && sample1d(k, DIM_ENVIRONMENT_STRATEGY) >= (double)prob) go = false;
            LightSample ls;
            ls.valid = false;
            if (go) {
                if (S.k.env.lighting) {
                    F3 rdn;
                    float pdf;
                    if (env_sample(S, k, ls.dir, rdn, pdf)) {
                        ls.emitted = rdn * S.k.env.strength;
                        ls.pdf = pdf;
                        ls.valid = maxc(ls.emitted) > 0.0f;
                    }
                } else if (cbg) {
                    ls.dir = sphere_direction(k, DIM_ENVIRONMENT_POINT);
                    ls.emitted = f3(S.k.background);
                    ls.pdf = 1.0f / (4.0f * kPiF);
                    ls.valid = maxc(ls.emitted) > 0.0f;
                }
            }
            if (ls.valid && leaves_opaque(m, h, ls.dir)) {
                const float sp = scatter_pdf(S, sr, m, h, ray.d, ls.dir);
                const F3 bc = scatter_bsdfcos(S, sr, m, h, ray.d, ls.dir);
                if (!(sp <= 0.0f || !isfinite(sp) || maxc(bc) <= 0.0f)) {
                    const float mis = power_heuristic(ls.pdf, sp);
                    F3 c = (bc * ls.emitted) * (mis / (ls.pdf * prob));
                    if (cbg) c = clamp_bg_miss(S, c);
                    pend1 = clamp_ray_color(thr * c);
                    out.sh[1] = true;
                    if (rough_grad) {
                        const F3 dl = dlnf_rough(S, m, h, ray.d, ls.dir);
                        w.adj_rough[p].dn1[0] = dl.x;
                        w.adj_rough[p].dn1[1] = dl.y;
                        w.adj_rough[p].dn1[2] = dl.z;
                    }
                    out.sh_o[1] = h.p;
                    out.sh_d[1] = ls.dir;
                    out.sh_t[1] = kInf;
                }
            }
        }
        if constexpr (MODE == 2) {
            if (cache_query) {
                CacheRecord q;
                cache_inputs(w, h, m, ray.d, q.in);
                q.v[0] = thr.x;
                q.v[1] = thr.y;
                q.v[2] = thr.z;
                q.path = p;
                q.pad[0] = q.pad[1] = 0.0f;
                w.cache_q[atomicAdd(w.cache_count, 1u)] = q;
                goto done;
            }
        }
        const F3 dir = scatter_generate(sr, k);
        if (!leaves_opaque(m, h, dir)) goto done;
        // For a BSDF record this is scatteringPDF of the sampled direction with the same
        // inputs that produced sr.spdf, so the stored value is reused.
        const float pdf = sr.pdf == PDF_BSDF ? sr.spdf : scatter_pdf(S, sr, m, h, ray.d, dir);
        if (pdf <= 0.0f || !isfinite(pdf)) goto done;
        thr = clamp_ray_color(thr * att);
        if (terminated(thr) || !russian_roulette(thr, bounce, k)) goto done;
        out.cont = true;
        out.next_o = h.p;
        out.next_d = dir;
        if (rough_grad) {
            // A GGX sample whose half vector faces away or whose reflection falls below the
            // surface is replaced by the mirror direction (ggx_reflection_sample, as the
            // reference does): that direction is not drawn from the density the throughput
            // divides by, so the sample carries no roughness derivative.
            const F3 view = safe_normalize(ray.d * -1.0f, h.n);
            const F3 hv = sample_ggx_half(h.n, m.alpha, sample2d(k, DIM_BSDF_DIRECTION));
            const bool fallback = dot(view, hv) <= 0.0f || dot(reflect(ray.d, hv), h.n) <= 0.0f;
            const F3 dl = fallback ? F3{0.f, 0.f, 0.f} : dlnf_rough(S, m, h, ray.d, dir);
            w.adj_rough[p].dc[0] = dl.x;
            w.adj_rough[p].dc[1] = dl.y;
            w.adj_rough[p].dc[2] = dl.z;
        }
        const bool svil = ((S.k.sky == 3 || S.k.sky == 2) && S.k.env.lighting)
                       || (S.k.has_constant_background_light && sr.pdf != PDF_BSDF);
        flags = (svil ? PF_PREV_SVIL : 0u) | (flags & PF_CACHE_DONE);
        P.thr[p] = make_float4(thr.x, thr.y, thr.z, pdf);
    }
done:
    if constexpr (MODE == 3) {
        if (w.adjoint && w.grad_volume >= 0) {
            density_add(S, w, pix, rad - rad_start, dscore);
            bool sh_used = false;
            for (int q = 0; q < 2; q++)
                if (out.sh[q] && volume_overlap(S.objects[w.grad_volume], out.sh_o[q], out.sh_d[q], kTMin, out.sh_t[q]) > 0.0f)
                    sh_used = true;
            w.dens_score[p] = make_float2(dscore, (!dext && sh_used) ? dscore + dscore_b : dscore);
        }
    }
    if (bounce >= w.max_bounces) out.cont = false;
    P.rad[p] = make_float4(rad.x, rad.y, rad.z, __uint_as_float(flags));
    P.pend0[p] = make_float4(pend0.x, pend0.y, pend0.z, 0.f);
    P.pend1[p] = make_float4(pend1.x, pend1.y, pend1.z, 0.f);
    if (out.cont) {
        P.ray_o[p] = make_float4(out.next_o.x, out.next_o.y, out.next_o.z, __int_as_float(out.xobj));
        P.ray_d[p] = make_float4(out.next_d.x, out.next_d.y, out.next_d.z, __int_as_float(out.xprim));
    }
}

// ---------------------------------------------------------------------------- film

__device__ __forceinline__ F3 clean(F3 c)   // cleanColor (Threads.cpp:122-137)
{
    return F3{isfinite(c.x) ? c.x : 0.f, isfinite(c.y) ? c.y : 0.f, isfinite(c.z) ? c.z : 0.f};
}

// Shade-stage kernels k_shade<mode> (shade_kernels.cu): 0 plain, 1 with the
// caustic estimate, 2 radiance-cache render, 3 adjoint replay.
using ShadeKernel = void (*)(const DScene*, WaveArgs, PathBuf, Ctrl*, int);
ShadeKernel shade_kernel(int mode);
ShadeKernel shade_kernel_cached();   // k_shade<2>, in its own translation unit

// Multi-scene waves: every path finds its segment in P.seg, the segment's WaveArgs
// in segs and its scene in scenes[segs[seg].batch_scene]. Modes 0 and 1 as above.
using BatchShadeKernel = void (*)(const DScene*, const WaveArgs*, PathBuf, Ctrl*, int);
BatchShadeKernel batch_shade_kernel(int mode);

}  // namespace luz
