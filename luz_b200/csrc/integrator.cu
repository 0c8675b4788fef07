// integrator.cu — wavefront path tracer for B200 (sm_100a) behind the C ABI.
//
// One render = waves of (pixel block x sample block) paths. Each wave runs
//   raygen  -> [extend -> shade -> shadow] x (max_bounces + 1) -> accumulate
// over SoA path state. Queues are compacted with warp ballots (one atomic per
// warp); extend/shadow are persistent kernels whose warps fetch 32-ray batches
// from a global counter, so warps that finish early steal the remaining work.
// Per-bounce counters live on the device; the host never waits inside a wave.
//
// The per-path arithmetic follows calculateLightRaysColor
// (src/renderer/ColorHelper.cpp:1136-1326) step for step; NEE shadow tests are
// deferred to the shadow kernel: shade stores each candidate contribution in a
// per-path "pending" slot and the shadow kernel clears the slot when the ray is
// occluded, which gives the same sum as the reference's inline test.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "luz_gpu.h"
#include "pack.h"
#include "wavefront.cuh"

namespace luz {

// ---------------------------------------------------------------------------- raygen

__global__ void __launch_bounds__(kBlock) k_raygen(WaveArgs w, PathBuf P, Ctrl* C)
{
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p == 0) C->count[0] = (uint32_t)w.n;
    if (p >= w.n) return;
    uint32_t x, y, s;
    path_coords(w, (uint32_t)p, x, y, s);
    double o[3], d[3];
    camera_ray(w, x, y, s, o, d);
    P.ray_o[p] = make_float4((float)o[0], (float)o[1], (float)o[2], __int_as_float(-1));
    P.ray_d[p] = make_float4((float)d[0], (float)d[1], (float)d[2], __int_as_float(-1));
    P.thr[p] = make_float4(1.f, 1.f, 1.f, 0.f);
    P.rad[p] = make_float4(0.f, 0.f, 0.f, __uint_as_float(PF_PREV_SPECULAR));
    P.prev_o[p] = make_float4(0.f, 0.f, 0.f, 0.f);
    P.pend0[p] = make_float4(0.f, 0.f, 0.f, 0.f);
    P.pend1[p] = make_float4(0.f, 0.f, 0.f, 0.f);
    P.pixel[p] = y * (uint32_t)w.width + x;
    P.sample[p] = s;
    P.queue0[p] = (uint32_t)p;
}

// ---------------------------------------------------------------------------- extend (closest hit)

// Resident blocks per SM the register allocator is asked to allow (measured on
// B200: more resident warps beat the few spills this costs in the traversal).
#ifndef LUZ_EXTEND_MIN_BLOCKS
#define LUZ_EXTEND_MIN_BLOCKS 6
#endif
#ifndef LUZ_SHADE_MIN_BLOCKS
#define LUZ_SHADE_MIN_BLOCKS 4
#endif
#ifndef LUZ_SHADOW_MIN_BLOCKS
#define LUZ_SHADOW_MIN_BLOCKS 8
#endif

__global__ void __launch_bounds__(kBlock, LUZ_EXTEND_MIN_BLOCKS) k_extend(DScene S, WaveArgs w, PathBuf P, Ctrl* C, int bounce)
{
    const uint32_t count = C->count[bounce];
    const uint32_t* q = (bounce & 1) ? P.queue1 : P.queue0;
    while (true) {
        uint32_t base = 0;
        if (lane_id() == 0) base = atomicAdd(&C->fetch_ext[bounce], 32u);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= count) break;
        const uint32_t i = base + lane_id();
        if (i >= count) continue;
        const uint32_t p = q[i];
        const float4 o = P.ray_o[p], d = P.ray_d[p];
        const TRay r = make_ray_x(F3{o.x, o.y, o.z}, F3{d.x, d.y, d.z}, __float_as_int(o.w), __float_as_int(d.w));
        const uint32_t pix = P.pixel[p];
        const Key k = path_key(w, pix % (uint32_t)w.width, pix / (uint32_t)w.width, P.sample[p], (uint32_t)bounce);
        VolSample vs{&k, 0.0, false};
        const THit h = closest_hit(S, r, kTMin, kInf, vs);
        P.hit[p] = make_float4(h.t, h.u, h.v, __int_as_float(h.obj));
        P.hit_prim[p] = h.prim;
        if (S.counters) {
            atomicAdd(&S.counters[0], (unsigned long long)vs.nodes);
            atomicAdd(&S.counters[1], (unsigned long long)vs.tris);
            atomicAdd(&S.counters[2], (unsigned long long)vs.top);
        }
    }
}

// ---------------------------------------------------------------------------- shadow (any hit)

__global__ void __launch_bounds__(kBlock, LUZ_SHADOW_MIN_BLOCKS) k_shadow(DScene S, WaveArgs w, PathBuf P, Ctrl* C, int bounce)
{
    const uint32_t count = C->shadow[bounce];
    while (true) {
        uint32_t base = 0;
        if (lane_id() == 0) base = atomicAdd(&C->fetch_sh[bounce], 32u);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= count) break;
        const uint32_t i = base + lane_id();
        if (i >= count) continue;
        const float4 o = P.sh_o[i], d = P.sh_d[i];
        const uint32_t tag = __float_as_uint(d.w);
        const uint32_t p = tag & 0x7fffffffu;
        const int2 x = P.sh_x[i];
        const TRay r = make_ray_x(F3{o.x, o.y, o.z}, F3{d.x, d.y, d.z}, x.x, x.y);
        const uint32_t pix = P.pixel[p];
        const Key k = path_key(w, pix % (uint32_t)w.width, pix / (uint32_t)w.width, P.sample[p], (uint32_t)bounce);
        VolSample vs{&k, 0.0, false};
        if (any_hit(S, r, kTMin, o.w, vs)) {
            if (tag & 0x80000000u) P.pend1[p] = make_float4(0.f, 0.f, 0.f, 0.f);
            else P.pend0[p] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
        if (S.counters) {
            atomicAdd(&S.counters[3], (unsigned long long)vs.nodes);
            atomicAdd(&S.counters[4], (unsigned long long)vs.tris);
            atomicAdd(&S.counters[5], (unsigned long long)vs.top);
        }
    }
}

__global__ void __launch_bounds__(kBlock, LUZ_SHADE_MIN_BLOCKS) k_shade(const DScene* __restrict__ Sp, WaveArgs w, PathBuf P, Ctrl* C, int bounce)
{
    const DScene& S = *Sp;
    const uint32_t count = C->count[bounce];
    const uint32_t* q = (bounce & 1) ? P.queue1 : P.queue0;
    uint32_t* nq = (bounce & 1) ? P.queue0 : P.queue1;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    for (uint32_t base = wid * 32u; base < count; base += warps * 32u) {
        const uint32_t i = base + lane_id();
        const bool valid = i < count;
        ShadeOut o;
        o.cont = false;
        o.sh[0] = o.sh[1] = false;
        uint32_t p = 0;
        if (valid) {
            p = q[i];
            shade_path(S, w, P, p, bounce, o);
        }
        __syncwarp();
        const uint32_t qi = warp_append(&C->count[bounce + 1], o.cont);
        if (o.cont) nq[qi] = p;
        for (int slot = 0; slot < 2; slot++) {
            const uint32_t si = warp_append(&C->shadow[bounce], o.sh[slot]);
            if (o.sh[slot]) {
                P.sh_o[si] = make_float4(o.sh_o[slot].x, o.sh_o[slot].y, o.sh_o[slot].z, o.sh_t[slot]);
                P.sh_d[si] = make_float4(o.sh_d[slot].x, o.sh_d[slot].y, o.sh_d[slot].z,
                                         __uint_as_float(p | ((uint32_t)slot << 31)));
                P.sh_x[si] = make_int2(o.xobj, o.xprim);
            }
        }
    }
}

// Adds one wave's per-bounce queue sizes to the render totals (no host wait per wave).
__global__ void k_tally(const Ctrl* C, int max_b, unsigned long long* totals)
{
    unsigned long long e = 0, s = 0;
    for (int b = 0; b <= max_b; b++) {
        e += C->count[b];
        s += C->shadow[b];
    }
    totals[0] += e;
    totals[1] += s;
}

__global__ void k_path_color(WaveArgs w, PathBuf P)
{
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= w.n) return;
    const float4 r = P.rad[p], a = P.pend0[p], b = P.pend1[p];
    const F3 c = (F3{r.x, r.y, r.z} + F3{a.x, a.y, a.z}) + F3{b.x, b.y, b.z};
    P.color[p] = make_float4(c.x, c.y, c.z, 0.f);
}

// Sums the wave's samples of each pixel in sample order into the FP64 film.
__global__ void k_accumulate(WaveArgs w, PathBuf P, double* film)
{
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= w.pix_count) return;
    double sx = 0.0, sy = 0.0, sz = 0.0;
    const int64_t b = j * w.s_count;
    for (int s = 0; s < w.s_count; s++) {
        const float4 r = P.rad[b + s], a = P.pend0[b + s], c2 = P.pend1[b + s];
        const F3 c = clean((F3{r.x, r.y, r.z} + F3{a.x, a.y, a.z}) + F3{c2.x, c2.y, c2.z});
        sx += (double)c.x;
        sy += (double)c.y;
        sz += (double)c.z;
    }
    double* f = film + 3 * (int64_t)(w.pix_begin + j);
    f[0] += sx;
    f[1] += sy;
    f[2] += sz;
}

__global__ void k_resolve(const double* film, int64_t npix, double spp, float* out)
{
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= npix) return;
    for (int a = 0; a < 3; a++) {
        const double v = film[3 * j + a] / spp;
        out[3 * j + a] = isfinite(v) ? (float)v : 0.f;
    }
}

// ---------------------------------------------------------------------------- ray batches

__global__ void k_trace_rays(DScene S, const float* rays, int64_t n, int any, uint32_t seed, const int32_t* vkey,
                             LuzHit* out)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* r = rays + 8 * i;
    const TRay ray = make_ray(F3{r[0], r[1], r[2]}, F3{r[4], r[5], r[6]});
    Key k;
    if (vkey) k = Key{base_key(seed, (uint32_t)vkey[4 * i], (uint32_t)vkey[4 * i + 1], 0), (uint32_t)vkey[4 * i + 2],
                      (uint32_t)vkey[4 * i + 3]};
    else k = Key{base_key(seed, 0, 0, 0), 0, 0};
    VolSample vs{&k, 0.0, false};
    LuzHit o;
    if (any) {
        const bool occ = any_hit(S, ray, r[3], r[7], vs);
        o = LuzHit{0.f, occ ? 0 : -1, 0, 0.f, 0.f};
    } else {
        const THit h = closest_hit(S, ray, r[3], r[7], vs);
        if (h.obj < 0) {
            o = LuzHit{kInf, -1, -1, 0.f, 0.f};
        } else {
            const GObject O = S.objects[h.obj];
            int32_t prim = h.prim;
            if (O.kind == OK_MESH || O.kind == OK_INSTANCE) prim = (int32_t)load_tri(S.tris, (uint32_t)h.prim).orig;
            o = LuzHit{h.t, O.id, prim, h.u, h.v};
        }
    }
    out[i] = o;
}

}  // namespace luz

// =============================================================================== host side

using namespace luz;

namespace {

thread_local std::string g_err;

#define CK(x)                                                                               \
    do {                                                                                    \
        cudaError_t e_ = (x);                                                               \
        if (e_ != cudaSuccess) throw Status(LUZ_E_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
    } while (0)

template <class T> T* dalloc(std::size_t n)
{
    void* p = nullptr;
    if (n == 0) n = 1;
    CK(cudaMalloc(&p, n * sizeof(T)));
    return static_cast<T*>(p);
}
template <class T> T* dupload(const std::vector<T>& v)
{
    T* p = dalloc<T>(v.size());
    if (!v.empty()) CK(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    return p;
}

int guard(const std::function<int()>& f)
{
    try {
        return f();
    } catch (const Status& s) {
        set_error(s.what());
        return s.code;
    } catch (const std::exception& e) {
        set_error(e.what());
        return LUZ_E_INVALID;
    }
}

}  // namespace

struct luz_gpu_scene {
    int device = 0;
    std::unique_ptr<ScenePack> pack;
    DScene ds{};
    DScene* dds = nullptr;           // device copy of ds: k_shade reads it through a pointer so that
                                     // its out-of-line calls pass a reference, not a stack copy
    std::vector<void*> allocs;
    cudaStream_t stream = nullptr;
    // path buffers (grown on demand)
    int64_t cap = 0;
    PathBuf pb{};
    std::vector<void*> pallocs;
    Ctrl* ctrl = nullptr;
    Ctrl* ctrl_host = nullptr;
    unsigned long long* totals = nullptr;   // device: extension / shadow rays of the current render
    double* film = nullptr;
    int64_t film_pix = 0;
    int sms = 0;
    int occ_ext = 1, occ_shade = 1, occ_sh = 1;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;

    template <class T> T* up(const std::vector<T>& v)
    {
        T* p = dupload(v);
        allocs.push_back(p);
        return p;
    }
    template <class T> T* palloc(int64_t n)
    {
        T* p = dalloc<T>((std::size_t)n);
        pallocs.push_back(p);
        return p;
    }
    void free_paths()
    {
        for (void* p : pallocs) cudaFree(p);
        pallocs.clear();
        cap = 0;
    }
    void ensure_paths(int64_t n)
    {
        if (n <= cap) return;
        free_paths();
        pb.ray_o = palloc<float4>(n);
        pb.ray_d = palloc<float4>(n);
        pb.thr = palloc<float4>(n);
        pb.rad = palloc<float4>(n);
        pb.prev_o = palloc<float4>(n);
        pb.pend0 = palloc<float4>(n);
        pb.pend1 = palloc<float4>(n);
        pb.pixel = palloc<uint32_t>(n);
        pb.sample = palloc<uint32_t>(n);
        pb.hit = palloc<float4>(n);
        pb.hit_prim = palloc<int32_t>(n);
        pb.queue0 = palloc<uint32_t>(n);
        pb.queue1 = palloc<uint32_t>(n);
        pb.sh_o = palloc<float4>(2 * n);
        pb.sh_d = palloc<float4>(2 * n);
        pb.sh_x = palloc<int2>(2 * n);
        pb.color = palloc<float4>(n);
        cap = n;
    }
    ~luz_gpu_scene()
    {
        cudaSetDevice(device);
        free_paths();
        for (void* p : allocs) cudaFree(p);
        if (ctrl) cudaFree(ctrl);
        if (ctrl_host) cudaFreeHost(ctrl_host);
        if (film) cudaFree(film);
        if (dds) cudaFree(dds);
        if (totals) cudaFree(totals);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

constexpr int64_t kWaveTarget = int64_t(1) << 22;   // ~4M paths in flight per wave

// Stage timing (LUZ_RENDER_PROFILE): one event pair per stage launch, summed per wave.
struct StageTimer {
    bool on = false;
    std::vector<cudaEvent_t> ev;
    std::vector<int> stage;
    double ms[3] = {0, 0, 0};
    void mark(cudaStream_t st, int which, bool begin)
    {
        if (!on) return;
        cudaEvent_t e;
        CK(cudaEventCreate(&e));
        CK(cudaEventRecord(e, st));
        ev.push_back(e);
        if (begin) stage.push_back(which);
    }
    void collect()
    {
        for (std::size_t i = 0; i + 1 < ev.size(); i += 2) {
            float m = 0.f;
            CK(cudaEventElapsedTime(&m, ev[i], ev[i + 1]));
            ms[stage[i / 2]] += m;
        }
        for (cudaEvent_t e : ev) cudaEventDestroy(e);
        ev.clear();
        stage.clear();
    }
};

void launch_bounces(luz_gpu_scene* s, const WaveArgs& w, cudaStream_t st, int64_t& launches, StageTimer& T)
{
    const int g_ext = s->sms * s->occ_ext, g_sh = s->sms * s->occ_sh, g_shade = s->sms * s->occ_shade;
    for (int b = 0; b <= w.max_bounces; b++) {
        T.mark(st, 0, true);
        k_extend<<<g_ext, kBlock, 0, st>>>(s->ds, w, s->pb, s->ctrl, b);
        T.mark(st, 0, false);
        T.mark(st, 1, true);
        k_shade<<<g_shade, kBlock, 0, st>>>(s->dds, w, s->pb, s->ctrl, b);
        T.mark(st, 1, false);
        T.mark(st, 2, true);
        k_shadow<<<g_sh, kBlock, 0, st>>>(s->ds, w, s->pb, s->ctrl, b);
        T.mark(st, 2, false);
        launches += 3;
    }
    CK(cudaGetLastError());
}

void check_params(const LuzRenderParams* p)
{
    if (!p) throw Status(LUZ_E_INVALID, "Render parameters are NULL.");
    if (p->width <= 0) throw Status(LUZ_E_INVALID, "Image width must be positive.");
    if (p->height <= 0) throw Status(LUZ_E_INVALID, "Image height must be positive.");
    if (p->spp <= 0) throw Status(LUZ_E_INVALID, "Sample count must be positive.");
    if (p->max_bounces < 0 || p->max_bounces >= kMaxBounceSlots)
        throw Status(LUZ_E_INVALID, "Max light bounces must be in [0, 255).");
    if (p->flags & ~(LUZ_RENDER_PROFILE | LUZ_RENDER_COUNT))
        throw Status(LUZ_E_UNSUPPORTED, "Adaptive sampling and NFOR buffers are not on the GPU path.");
    if (p->sample_offset < 0) throw Status(LUZ_E_INVALID, "Sample offset must be non-negative.");
}

WaveArgs base_args(luz_gpu_scene* s, const LuzRenderParams* p)
{
    WaveArgs w{};
    w.width = p->width;
    w.height = p->height;
    w.seed = p->seed;
    w.stream = p->stream;
    w.sample_offset = p->sample_offset;
    w.max_bounces = p->max_bounces;
    w.cam = prepare_camera(s->pack->camera, s->pack->consts.meters_per_unit, p->width, p->height);
    return w;
}

void finish_wave(luz_gpu_scene* s, cudaStream_t st, LuzRenderStats* acc, int max_b)
{
    CK(cudaMemcpyAsync(s->ctrl_host, s->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (acc) {
        for (int b = 0; b <= max_b; b++) {
            acc->extension_rays += s->ctrl_host->count[b];
            acc->shadow_rays += s->ctrl_host->shadow[b];
        }
    }
    uint32_t err = 0;
    CK(cudaMemcpy(&err, s->ds.error, sizeof(uint32_t), cudaMemcpyDeviceToHost));
    if (err) throw Status(LUZ_E_DEVICE, "Traversal stack overflow reported by the device (flags " + std::to_string(err) + ").");
}

int do_render(luz_gpu_scene* s, const LuzRenderParams* p, float* d_out, cudaStream_t st, LuzRenderStats* stats)
{
    check_params(p);
    CK(cudaSetDevice(s->device));
    WaveArgs w = base_args(s, p);
    const int64_t npix = (int64_t)p->width * p->height;
    const int s_wave = (int)std::min<int64_t>(p->spp, std::max<int64_t>(1, kWaveTarget / 1));
    const int64_t pix_wave = std::max<int64_t>(1, std::min<int64_t>(npix, kWaveTarget / s_wave));
    const int64_t n_wave = pix_wave * s_wave;
    s->ensure_paths(n_wave);
    if (s->film_pix < npix) {
        if (s->film) cudaFree(s->film);
        s->film = dalloc<double>((std::size_t)(3 * npix));
        s->film_pix = npix;
    }
    LuzRenderStats acc{};
    StageTimer T;
    T.on = (p->flags & LUZ_RENDER_PROFILE) != 0;
    unsigned long long* counters = nullptr;
    if (p->flags & LUZ_RENDER_COUNT) {
        counters = dalloc<unsigned long long>(8);
        CK(cudaMemsetAsync(counters, 0, 8 * sizeof(unsigned long long), st));
    }
    s->ds.counters = counters;
    CK(cudaMemcpyAsync(s->dds, &s->ds, sizeof(DScene), cudaMemcpyHostToDevice, st));
    CK(cudaMemsetAsync(s->film, 0, sizeof(double) * 3 * npix, st));
    CK(cudaMemsetAsync(s->totals, 0, 2 * sizeof(unsigned long long), st));
    CK(cudaEventRecord(s->ev0, st));
    int64_t launches = 0, waves = 0;
    for (int sb = 0; sb < p->spp; sb += s_wave) {
        const int sc = std::min(s_wave, p->spp - sb);
        for (int64_t pb = 0; pb < npix; pb += pix_wave) {
            const int64_t pc = std::min<int64_t>(pix_wave, npix - pb);
            w.pix_begin = (int32_t)pb;
            w.pix_count = (int32_t)pc;
            w.s_begin = sb;
            w.s_count = sc;
            w.n = pc * sc;
            w.list_mode = 0;
            CK(cudaMemsetAsync(s->ctrl, 0, sizeof(Ctrl), st));
            k_raygen<<<(unsigned)((w.n + kBlock - 1) / kBlock), kBlock, 0, st>>>(w, s->pb, s->ctrl);
            launch_bounces(s, w, st, launches, T);
            k_accumulate<<<(unsigned)((pc + 127) / 128), 128, 0, st>>>(w, s->pb, s->film);
            k_tally<<<1, 1, 0, st>>>(s->ctrl, w.max_bounces, s->totals);
            launches += 3;
            waves++;
            if (T.on) {
                CK(cudaStreamSynchronize(st));
                T.collect();
            }
        }
    }
    k_resolve<<<(unsigned)((npix + 255) / 256), 256, 0, st>>>(s->film, npix, (double)p->spp, d_out);
    launches++;
    CK(cudaEventRecord(s->ev1, st));
    CK(cudaEventSynchronize(s->ev1));
    CK(cudaGetLastError());
    {
        unsigned long long tot[2] = {0, 0};
        uint32_t err = 0;
        CK(cudaMemcpy(tot, s->totals, sizeof(tot), cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(&err, s->ds.error, sizeof(uint32_t), cudaMemcpyDeviceToHost));
        if (err) throw Status(LUZ_E_DEVICE, "Traversal stack overflow reported by the device (flags " + std::to_string(err) + ").");
        acc.extension_rays = (double)tot[0];
        acc.shadow_rays = (double)tot[1];
    }
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, s->ev0, s->ev1));
    s->ds.counters = nullptr;
    unsigned long long cnt[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (counters) {
        CK(cudaMemcpy(cnt, counters, sizeof(cnt), cudaMemcpyDeviceToHost));
        cudaFree(counters);
        CK(cudaMemcpy(s->dds, &s->ds, sizeof(DScene), cudaMemcpyHostToDevice));
    }
    if (stats) {
        *stats = acc;
        stats->render_ms = ms;
        stats->samples = (double)npix * p->spp;
        stats->kernel_launches = launches;
        stats->waves = waves;
        stats->extend_ms = T.ms[0];
        stats->shade_ms = T.ms[1];
        stats->shadow_ms = T.ms[2];
        stats->extend_launches = waves * (p->max_bounces + 1);
        stats->shadow_launches = waves * (p->max_bounces + 1);
        stats->ext_nodes = (double)cnt[0];
        stats->ext_tris = (double)cnt[1];
        stats->ext_top = (double)cnt[2];
        stats->sh_nodes = (double)cnt[3];
        stats->sh_tris = (double)cnt[4];
        stats->sh_top = (double)cnt[5];
    }
    return LUZ_OK;
}

}  // namespace

// ---------------------------------------------------------------------------- no-allocation render
//
// One file-scope device array holds the path state, queues and film of
// luz_gpu_render_device_noalloc, so that entry point never allocates. Its
// layout (256-B aligned sub-arrays) is carved on the host from the array's
// device address, resolved once per device with cudaGetSymbolAddress.

static __device__ __align__(256) unsigned char g_static_scratch[LUZ_STATIC_SCRATCH_BYTES];

namespace {

struct StaticArena {
    PathBuf pb{};
    Ctrl* ctrl = nullptr;
    unsigned long long* totals = nullptr;
    double* film = nullptr;
    int64_t film_pixels = 0;
};

constexpr std::size_t align256(std::size_t b) { return (b + 255) & ~std::size_t(255); }

StaticArena carve_static(unsigned char* base)
{
    const int64_t n = LUZ_STATIC_WAVE_PATHS;
    std::size_t off = 0;
    auto take = [&](std::size_t bytes) {
        unsigned char* p = base + off;
        off += align256(bytes);
        return p;
    };
    StaticArena A;
    PathBuf& P = A.pb;
    P.ray_o = reinterpret_cast<float4*>(take(n * sizeof(float4)));
    P.ray_d = reinterpret_cast<float4*>(take(n * sizeof(float4)));
    P.thr = reinterpret_cast<float4*>(take(n * sizeof(float4)));
    P.rad = reinterpret_cast<float4*>(take(n * sizeof(float4)));
    P.prev_o = reinterpret_cast<float4*>(take(n * sizeof(float4)));
    P.pend0 = reinterpret_cast<float4*>(take(n * sizeof(float4)));
    P.pend1 = reinterpret_cast<float4*>(take(n * sizeof(float4)));
    P.hit = reinterpret_cast<float4*>(take(n * sizeof(float4)));
    P.pixel = reinterpret_cast<uint32_t*>(take(n * sizeof(uint32_t)));
    P.sample = reinterpret_cast<uint32_t*>(take(n * sizeof(uint32_t)));
    P.hit_prim = reinterpret_cast<int32_t*>(take(n * sizeof(int32_t)));
    P.queue0 = reinterpret_cast<uint32_t*>(take(n * sizeof(uint32_t)));
    P.queue1 = reinterpret_cast<uint32_t*>(take(n * sizeof(uint32_t)));
    P.sh_o = reinterpret_cast<float4*>(take(2 * n * sizeof(float4)));
    P.sh_d = reinterpret_cast<float4*>(take(2 * n * sizeof(float4)));
    P.sh_x = reinterpret_cast<int2*>(take(2 * n * sizeof(int2)));
    P.color = nullptr;   // used by trace_paths only
    A.ctrl = reinterpret_cast<Ctrl*>(take(sizeof(Ctrl)));
    A.totals = reinterpret_cast<unsigned long long*>(take(2 * sizeof(unsigned long long)));
    A.film = reinterpret_cast<double*>(base + off);
    A.film_pixels = (int64_t)((LUZ_STATIC_SCRATCH_BYTES - off) / (3 * sizeof(double)));
    return A;
}

// Device address of g_static_scratch, per device, resolved on first use with
// that device current.
unsigned char* static_scratch_address(int device)
{
    static std::mutex mu;
    static std::vector<unsigned char*> addr;
    std::lock_guard<std::mutex> lock(mu);
    if ((int)addr.size() <= device) addr.resize(device + 1, nullptr);
    if (!addr[device]) {
        void* p = nullptr;
        CK(cudaGetSymbolAddress(&p, g_static_scratch));
        addr[device] = static_cast<unsigned char*>(p);
    }
    return addr[device];
}

int do_render_noalloc(luz_gpu_scene* s, const LuzRenderParams* p, float* d_out, cudaStream_t st, LuzRenderStats* stats)
{
    check_params(p);
    if (p->flags != 0) throw Status(LUZ_E_UNSUPPORTED, "luz_gpu_render_device_noalloc takes no render flags.");
    CK(cudaSetDevice(s->device));
    const StaticArena A = carve_static(static_scratch_address(s->device));
    const int64_t npix = (int64_t)p->width * p->height;
    if (npix > LUZ_STATIC_MAX_PIXELS || npix > A.film_pixels)
        throw Status(LUZ_E_LIMIT, "Image of " + std::to_string(npix) + " pixels exceeds the static film of " +
                                      std::to_string((long long)LUZ_STATIC_MAX_PIXELS) + " pixels.");
    WaveArgs w = base_args(s, p);
    const int64_t target = LUZ_STATIC_WAVE_PATHS;
    const int s_wave = (int)std::min<int64_t>(p->spp, target);
    const int64_t pix_wave = std::max<int64_t>(1, std::min<int64_t>(npix, target / s_wave));
    CK(cudaMemsetAsync(A.film, 0, sizeof(double) * 3 * npix, st));
    CK(cudaMemsetAsync(A.totals, 0, 2 * sizeof(unsigned long long), st));
    CK(cudaEventRecord(s->ev0, st));
    int64_t launches = 0, waves = 0;
    StageTimer T;
    for (int sb = 0; sb < p->spp; sb += s_wave) {
        const int sc = std::min(s_wave, p->spp - sb);
        for (int64_t pb = 0; pb < npix; pb += pix_wave) {
            const int64_t pc = std::min<int64_t>(pix_wave, npix - pb);
            w.pix_begin = (int32_t)pb;
            w.pix_count = (int32_t)pc;
            w.s_begin = sb;
            w.s_count = sc;
            w.n = pc * sc;
            w.list_mode = 0;
            CK(cudaMemsetAsync(A.ctrl, 0, sizeof(Ctrl), st));
            k_raygen<<<(unsigned)((w.n + kBlock - 1) / kBlock), kBlock, 0, st>>>(w, A.pb, A.ctrl);
            const int g_ext = s->sms * s->occ_ext, g_sh = s->sms * s->occ_sh, g_shade = s->sms * s->occ_shade;
            for (int b = 0; b <= w.max_bounces; b++) {
                k_extend<<<g_ext, kBlock, 0, st>>>(s->ds, w, A.pb, A.ctrl, b);
                k_shade<<<g_shade, kBlock, 0, st>>>(s->dds, w, A.pb, A.ctrl, b);
                k_shadow<<<g_sh, kBlock, 0, st>>>(s->ds, w, A.pb, A.ctrl, b);
                launches += 3;
            }
            k_accumulate<<<(unsigned)((pc + 127) / 128), 128, 0, st>>>(w, A.pb, A.film);
            k_tally<<<1, 1, 0, st>>>(A.ctrl, w.max_bounces, A.totals);
            launches += 3;
            waves++;
        }
    }
    k_resolve<<<(unsigned)((npix + 255) / 256), 256, 0, st>>>(A.film, npix, (double)p->spp, d_out);
    launches++;
    CK(cudaGetLastError());
    CK(cudaEventRecord(s->ev1, st));
    CK(cudaEventSynchronize(s->ev1));
    unsigned long long tot[2] = {0, 0};
    uint32_t err = 0;
    CK(cudaMemcpy(tot, A.totals, sizeof(tot), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(&err, s->ds.error, sizeof(uint32_t), cudaMemcpyDeviceToHost));
    if (err) throw Status(LUZ_E_DEVICE, "Traversal stack overflow reported by the device (flags " + std::to_string(err) + ").");
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, s->ev0, s->ev1));
    if (stats) {
        *stats = LuzRenderStats{};
        stats->render_ms = ms;
        stats->samples = (double)npix * p->spp;
        stats->extension_rays = (double)tot[0];
        stats->shadow_rays = (double)tot[1];
        stats->kernel_launches = launches;
        stats->waves = waves;
    }
    return LUZ_OK;
}

}  // namespace

extern "C" {

int luz_gpu_render_device_noalloc(luz_gpu_scene* s, const LuzRenderParams* p, float* d_out, void* stream,
                                  LuzRenderStats* stats)
{
    return guard([&] {
        if (!s || !d_out) throw Status(LUZ_E_INVALID, "NULL argument.");
        return do_render_noalloc(s, p, d_out, stream ? (cudaStream_t)stream : s->stream, stats);
    });
}

int luz_gpu_last_error(char* buffer, size_t length)
{
    if (buffer && length) {
        std::strncpy(buffer, get_error().c_str(), length - 1);
        buffer[length - 1] = 0;
    }
    return LUZ_OK;
}

int luz_gpu_device_count(int32_t* count)
{
    return guard([&] {
        int n = 0;
        const cudaError_t e = cudaGetDeviceCount(&n);
        if (e != cudaSuccess) n = 0;
        *count = n;
        return LUZ_OK;
    });
}

int luz_gpu_scene_create(const LuzSceneDesc* desc, int32_t device, luz_gpu_scene** out)
{
    return guard([&] {
        if (!out) throw Status(LUZ_E_INVALID, "Output handle pointer is NULL.");
        *out = nullptr;
        auto s = std::make_unique<luz_gpu_scene>();
        s->pack.reset(pack_scene(desc));
        s->device = device;
        CK(cudaSetDevice(device));
        CK(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
        CK(cudaEventCreate(&s->ev0));
        CK(cudaEventCreate(&s->ev1));
        const ScenePack& P = *s->pack;
        DScene& d = s->ds;
        d.rects = s->up(P.rects);
        d.objects = s->up(P.objects);
        d.top_nodes = s->up(P.top_nodes);
        d.top_children = s->up(P.top_children);
        d.nodes = s->up(P.nodes);
        d.tris = s->up(P.tris);
        d.tri_shade = s->up(P.tri_shade);
        d.vnormals = s->up(P.vnormals);
        d.vuvs = s->up(P.vuvs);
        d.meshes = s->up(P.meshes);
        d.materials = s->up(P.materials);
        d.textures = s->up(P.textures);
        d.texels = reinterpret_cast<const float4*>(s->up(P.texels));
        d.lights = s->up(P.lights);
        d.cdf = s->up(P.cdf);
        d.index_pool = s->up(P.index_pool);
        d.env_texels = reinterpret_cast<const float4*>(s->up(P.env_texels));
        uint32_t* err = dalloc<uint32_t>(1);
        CK(cudaMemset(err, 0, sizeof(uint32_t)));
        s->allocs.push_back(err);
        d.error = err;
        d.counters = nullptr;
        d.k = P.consts;
        s->dds = dalloc<DScene>(1);
        CK(cudaMemcpy(s->dds, &s->ds, sizeof(DScene), cudaMemcpyHostToDevice));
        s->ctrl = dalloc<Ctrl>(1);
        s->totals = dalloc<unsigned long long>(2);
        CK(cudaMallocHost(&s->ctrl_host, sizeof(Ctrl)));
        cudaDeviceProp prop;
        CK(cudaGetDeviceProperties(&prop, device));
        s->sms = prop.multiProcessorCount;
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&s->occ_ext, k_extend, kBlock, 0));
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&s->occ_shade, k_shade, kBlock, 0));
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&s->occ_sh, k_shadow, kBlock, 0));
        s->occ_ext = std::max(1, s->occ_ext);
        s->occ_shade = std::max(1, s->occ_shade);
        s->occ_sh = std::max(1, s->occ_sh);
        *out = s.release();
        return LUZ_OK;
    });
}

int luz_gpu_scene_destroy(luz_gpu_scene* scene)
{
    delete scene;
    return LUZ_OK;
}

int luz_gpu_scene_info(const luz_gpu_scene* s, LuzSceneInfo* info)
{
    return guard([&] {
        if (!s || !info) throw Status(LUZ_E_INVALID, "NULL argument.");
        const ScenePack& P = *s->pack;
        info->top_nodes = (int64_t)P.top_nodes.size();
        info->top_leaf_objects = (int64_t)P.objects.size();
        info->mesh_nodes = (int64_t)P.nodes.size();
        info->mesh_triangles = (int64_t)P.tris.size();
        info->device_bytes = P.device_bytes();
        info->max_mesh_depth = P.max_mesh_depth;
        info->light_count = P.consts.light_count;
        return LUZ_OK;
    });
}

int luz_gpu_render_device(luz_gpu_scene* s, const LuzRenderParams* p, float* d_out, void* stream, LuzRenderStats* stats)
{
    return guard([&] {
        if (!s || !d_out) throw Status(LUZ_E_INVALID, "NULL argument.");
        return do_render(s, p, d_out, stream ? (cudaStream_t)stream : s->stream, stats);
    });
}

int luz_gpu_render(luz_gpu_scene* s, const LuzRenderParams* p, float* rgb_out, LuzRenderStats* stats)
{
    return guard([&] {
        if (!s || !rgb_out) throw Status(LUZ_E_INVALID, "NULL argument.");
        check_params(p);
        CK(cudaSetDevice(s->device));
        const int64_t npix = (int64_t)p->width * p->height;
        float* d = dalloc<float>((std::size_t)(3 * npix));
        int rc = LUZ_OK;
        try {
            rc = do_render(s, p, d, s->stream, stats);
            CK(cudaMemcpy(rgb_out, d, sizeof(float) * 3 * npix, cudaMemcpyDeviceToHost));
        } catch (...) {
            cudaFree(d);
            throw;
        }
        cudaFree(d);
        return rc;
    });
}

int luz_gpu_trace_paths(luz_gpu_scene* s, const LuzRenderParams* p, const int32_t* x, const int32_t* y,
                        const int32_t* sample, int64_t count, float* rgb_out)
{
    return guard([&] {
        if (!s || !x || !y || !sample || !rgb_out) throw Status(LUZ_E_INVALID, "NULL argument.");
        check_params(p);
        if (count <= 0) return LUZ_OK;
        for (int64_t i = 0; i < count; i++)
            if (x[i] < 0 || x[i] >= p->width || y[i] < 0 || y[i] >= p->height || sample[i] < 0)
                throw Status(LUZ_E_INVALID, "Path coordinates out of range.");
        CK(cudaSetDevice(s->device));
        cudaStream_t st = s->stream;
        const int64_t chunk = std::min<int64_t>(count, kWaveTarget);
        s->ensure_paths(chunk);
        int32_t* dx = dalloc<int32_t>(chunk);
        int32_t* dy = dalloc<int32_t>(chunk);
        int32_t* dsm = dalloc<int32_t>(chunk);
        std::vector<float4> host((std::size_t)chunk);
        int64_t launches = 0;
        try {
            WaveArgs w = base_args(s, p);
            for (int64_t b = 0; b < count; b += chunk) {
                const int64_t n = std::min(chunk, count - b);
                CK(cudaMemcpyAsync(dx, x + b, n * 4, cudaMemcpyHostToDevice, st));
                CK(cudaMemcpyAsync(dy, y + b, n * 4, cudaMemcpyHostToDevice, st));
                CK(cudaMemcpyAsync(dsm, sample + b, n * 4, cudaMemcpyHostToDevice, st));
                w.list_mode = 1;
                w.list_x = dx;
                w.list_y = dy;
                w.list_s = dsm;
                w.n = n;
                w.s_count = 1;
                w.pix_count = (int32_t)n;
                CK(cudaMemsetAsync(s->ctrl, 0, sizeof(Ctrl), st));
                k_raygen<<<(unsigned)((n + kBlock - 1) / kBlock), kBlock, 0, st>>>(w, s->pb, s->ctrl);
                StageTimer T;
                launch_bounces(s, w, st, launches, T);
                k_path_color<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(w, s->pb);
                CK(cudaMemcpyAsync(host.data(), s->pb.color, n * sizeof(float4), cudaMemcpyDeviceToHost, st));
                finish_wave(s, st, nullptr, w.max_bounces);
                for (int64_t i = 0; i < n; i++) {
                    rgb_out[3 * (b + i)] = host[i].x;
                    rgb_out[3 * (b + i) + 1] = host[i].y;
                    rgb_out[3 * (b + i) + 2] = host[i].z;
                }
            }
        } catch (...) {
            cudaFree(dx);
            cudaFree(dy);
            cudaFree(dsm);
            throw;
        }
        cudaFree(dx);
        cudaFree(dy);
        cudaFree(dsm);
        return LUZ_OK;
    });
}

int luz_gpu_trace_rays(luz_gpu_scene* s, const float* rays, int64_t count, int32_t any_hit, uint32_t seed,
                       const int32_t* volume_key, LuzHit* out)
{
    return guard([&] {
        if (!s || !rays || !out) throw Status(LUZ_E_INVALID, "NULL argument.");
        if (count <= 0) return LUZ_OK;
        CK(cudaSetDevice(s->device));
        cudaStream_t st = s->stream;
        float* dr = dalloc<float>((std::size_t)(8 * count));
        LuzHit* dh = dalloc<LuzHit>((std::size_t)count);
        int32_t* dk = volume_key ? dalloc<int32_t>((std::size_t)(4 * count)) : nullptr;
        try {
            CK(cudaMemcpyAsync(dr, rays, sizeof(float) * 8 * count, cudaMemcpyHostToDevice, st));
            if (dk) CK(cudaMemcpyAsync(dk, volume_key, sizeof(int32_t) * 4 * count, cudaMemcpyHostToDevice, st));
            k_trace_rays<<<(unsigned)((count + 127) / 128), 128, 0, st>>>(s->ds, dr, count, any_hit, seed, dk, dh);
            CK(cudaGetLastError());
            CK(cudaMemcpyAsync(out, dh, sizeof(LuzHit) * count, cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            uint32_t err = 0;
            CK(cudaMemcpy(&err, s->ds.error, sizeof(uint32_t), cudaMemcpyDeviceToHost));
            if (err) throw Status(LUZ_E_DEVICE, "Traversal stack overflow reported by the device.");
        } catch (...) {
            cudaFree(dr);
            cudaFree(dh);
            if (dk) cudaFree(dk);
            throw;
        }
        cudaFree(dr);
        cudaFree(dh);
        if (dk) cudaFree(dk);
        return LUZ_OK;
    });
}

}  // extern "C"
