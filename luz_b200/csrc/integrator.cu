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
#include <cub/device/device_radix_sort.cuh>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <map>
#include <cstdio>
#include <cstring>
#include <functional>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "luz_gpu.h"
#include "nfor.h"
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
    P.pend0[p] = make_float4(0.f, 0.f, 0.f, 0.f);
    P.pend1[p] = make_float4(0.f, 0.f, 0.f, 0.f);
    P.pixel[p] = y * (uint32_t)w.width + x;
    P.sample[p] = s;
    P.queue0[p] = (uint32_t)p;
}

// ---------------------------------------------------------------------------- extend (closest hit)

// Resident blocks per SM the register allocator is asked to allow, measured on
// B200 (1080p glossy frame at 16 spp, extend / shadow stage): extend 7 blocks (72
// registers) 35.8-35.9 ms, 8 (64) 36.8 ms, 6 (80) 37.1 ms, 5 (96, almost no spills)
// 38.0 ms (on an earlier build with more local-memory traffic 5 blocks had led 6 and
// 7); shadow 8 blocks 16.0 ms, 10 16.7 ms, 12 18.4 ms (shade: shade_kernels.cu).
#ifndef LUZ_EXTEND_MIN_BLOCKS
#define LUZ_EXTEND_MIN_BLOCKS 7
#endif
#ifndef LUZ_SHADOW_MIN_BLOCKS
#define LUZ_SHADOW_MIN_BLOCKS 8
#endif
// The instantiations for scenes with instances (instance transform, two nested walks),
// measured at 4-6 blocks (5 again on the final build: 85.5 against 72.0 ms):
// 4 blocks (128 registers, a few hundred bytes of spills instead of 1-2 KB at 96) took
// the 1e5-instance frame's extend stage from 85.1 to 71.8 ms at 4 spp (6 blocks: 85.8).
#ifndef LUZ_EXTEND_MIN_BLOCKS_INST
#define LUZ_EXTEND_MIN_BLOCKS_INST 4
#endif

// Radiance-cache training steps: on the warm-up wave (the first sample of every pixel,
// every path a training row) when LuzCacheParams.warm_steps is 0, and at most per later
// wave. Cornell box 300x300, time to the plain 256-spp error: 16 warm-up steps 1.5-2.1x,
// 32 2.81-2.88x, 48 2.91-3.09x, 64 3.06-3.17x; two warm-up samples per pixel with 64 or
// 96 steps 2.86-3.01x. Four steps per later wave instead of 16: 2.81-2.83x (no change).
#ifndef LUZ_CACHE_WARM_STEPS
#define LUZ_CACHE_WARM_STEPS 64
#endif
#ifndef LUZ_CACHE_WAVE_STEPS
#define LUZ_CACHE_WAVE_STEPS 16
#endif

// Appends path p to the segment of its shade class; the lanes of vmask with the
// same class share one atomic (match.any).
__device__ __forceinline__ void bin_append(uint32_t* bin_count, const PathBuf& P, unsigned vmask, uint32_t cls,
                                           uint32_t p)
{
    const unsigned peers = __match_any_sync(vmask, cls);
    const int leader = __ffs(peers) - 1;
    const uint32_t lane = lane_id();
    uint32_t base = 0;
    if ((int)lane == leader) base = atomicAdd(&bin_count[cls], (uint32_t)__popc(peers));
    base = __shfl_sync(peers, base, leader);
    P.bins[cls * P.bin_stride + base + (uint32_t)__popc(peers & ((1u << lane) - 1u))] = p;
}

// Extend and shadow are instantiated per scene feature set (TF_* bits:
// instances, volumes); a scene without them runs traversal code without the
// instance transform or the volume sampler, and skips the per-ray sampler key.
// COUNT instantiations add the record counts of LUZ_RENDER_COUNT; the others
// carry no counting code (the shadow kernel counts under a runtime branch).
template <uint32_t F, bool COUNT>
__global__ void __launch_bounds__(kBlock, (F & TF_INSTANCE) ? LUZ_EXTEND_MIN_BLOCKS_INST : LUZ_EXTEND_MIN_BLOCKS)
    k_extend(DScene S, WaveArgs w, PathBuf P, Ctrl* C, int bounce)
{
    if constexpr ((F & TF_STAGED) != 0) stage_top_nodes(S);
    LocalStack<true> st;
    const uint32_t count = C->count[bounce];
    const uint32_t* q = (w.sorted_queue && bounce >= 1) ? w.sorted_queue : ((bounce & 1) ? P.queue1 : P.queue0);
    while (true) {
        uint32_t base = 0;
        if (lane_id() == 0) base = atomicAdd(&C->fetch_ext[bounce], 32u);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= count) break;
        const uint32_t i = base + lane_id();
        const unsigned vmask = __ballot_sync(0xffffffffu, i < count);
        if (i >= count) continue;
        const uint32_t p = q[i];
        const float4 o = P.ray_o[p], d = P.ray_d[p];
        const TRay r = make_ray_x(F3{o.x, o.y, o.z}, F3{d.x, d.y, d.z}, __float_as_int(o.w), __float_as_int(d.w));
        Key k{};
        if constexpr ((F & TF_VOLUME) != 0) {
            const uint32_t pix = P.pixel[p];
            k = path_key(w, pix % (uint32_t)w.width, pix / (uint32_t)w.width, P.sample[p], (uint32_t)bounce);
        }
        VolSample vs{&k, 0.0, false};
        const THit h = closest_hit<F>(S, r, kTMin, kInf, vs, st);
        P.hit[p] = make_float4(h.t, h.u, h.v, __int_as_float(h.obj));
        P.hit_prim[p] = h.prim;
        if (P.bins) bin_append(C->bin[bounce], P, vmask, h.obj < 0 ? 0u : (uint32_t)S.obj_class[h.obj], p);
        if constexpr (COUNT) {
            atomicAdd(&S.counters[0], (unsigned long long)vs.nodes);
            atomicAdd(&S.counters[1], (unsigned long long)vs.tris);
            atomicAdd(&S.counters[2], (unsigned long long)vs.top);
            atomicAdd(&S.counters[6], (unsigned long long)vs.bnodes);
        }
    }
}

// ---------------------------------------------------------------------------- shadow (any hit)

// (The record counts stay a runtime branch here: an instantiation without them
// measured 2.6x slower on B200, at 2.3 instead of 7.0 active threads per warp
// instruction for the same rays, a reconvergence effect of the smaller loop body.)
template <uint32_t F>
__global__ void __launch_bounds__(kBlock, LUZ_SHADOW_MIN_BLOCKS) k_shadow(DScene S, WaveArgs w, PathBuf P, Ctrl* C, int bounce)
{
    if constexpr ((F & TF_STAGED) != 0) stage_top_nodes(S);
    LocalStack<false> st;
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
        Key k{};
        if constexpr ((F & TF_VOLUME) != 0) {
            const uint32_t pix = P.pixel[p];
            k = path_key(w, pix % (uint32_t)w.width, pix / (uint32_t)w.width, P.sample[p], (uint32_t)bounce);
        }
        VolSample vs{&k, 0.0, false};
        if (any_hit<F>(S, r, kTMin, o.w, vs, st)) {
            if (tag & 0x80000000u) P.pend1[p] = make_float4(0.f, 0.f, 0.f, 0.f);
            else P.pend0[p] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
        if (S.counters) {
            atomicAdd(&S.counters[3], (unsigned long long)vs.nodes);
            atomicAdd(&S.counters[4], (unsigned long long)vs.tris);
            atomicAdd(&S.counters[5], (unsigned long long)vs.top);
            atomicAdd(&S.counters[7], (unsigned long long)vs.bnodes);
        }
    }
}

using TraceKernel = void (*)(DScene, WaveArgs, PathBuf, Ctrl*, int);
// Indexed [count][features | staged]: TF_STAGED variants read the scene's top
// collapsed nodes from shared memory (a tuning choice, off by default: on the
// 1080p glossy frame they measured 2.5% slower, the nodes being L1-resident).
const TraceKernel kExtendKernels[2][8] = {
    {k_extend<0, false>, k_extend<1, false>, k_extend<2, false>, k_extend<3, false>,
     k_extend<4, false>, k_extend<5, false>, k_extend<6, false>, k_extend<7, false>},
    {k_extend<0, true>, k_extend<1, true>, k_extend<2, true>, k_extend<3, true>,
     k_extend<4, true>, k_extend<5, true>, k_extend<6, true>, k_extend<7, true>}};
const TraceKernel kShadowKernels[8] = {k_shadow<0>, k_shadow<1>, k_shadow<2>, k_shadow<3>,
                                       k_shadow<4>, k_shadow<5>, k_shadow<6>, k_shadow<7>};


// ---------------------------------------------------------------------------- coherence sort
//
// A counting sort of an extension queue by (direction octant, cell of the ray
// origin in a 16^3 grid over the scene box, Morton order): rays of a warp then start
// close together and head the same way. Keys and counts stay on the device (the
// queue length is C->count[bounce]); the order inside a key is arbitrary, and the
// image does not depend on the order rays are traced in.
constexpr int kSortCellBits = 4;
constexpr int kSortBins = 8 << (3 * kSortCellBits);

__device__ __forceinline__ uint32_t spread3_4(uint32_t v)   // 4 bits -> bits 0, 3, 6, 9
{
    return (v & 1u) | ((v & 2u) << 2) | ((v & 4u) << 4) | ((v & 8u) << 6);
}

__global__ void k_sort_keys(const Ctrl* C, int bounce, const uint32_t* q, PathBuf P, GSceneConst K)
{
    const uint32_t count = C->count[bounce];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const uint32_t p = q[i];
        const float4 o = P.ray_o[p], d = P.ray_d[p];
        const float fo[3] = {o.x, o.y, o.z};
        uint32_t cell = 0;
#pragma unroll
        for (int a = 0; a < 3; a++) {
            const float c = (fo[a] - K.box_lo[a]) * K.box_inv[a] * (float)(1 << kSortCellBits);
            const uint32_t ci = (uint32_t)fminf(fmaxf(c, 0.0f), (float)((1 << kSortCellBits) - 1));
            cell |= spread3_4(ci) << a;
        }
        const uint32_t oct = (d.x < 0.0f ? 1u : 0u) | (d.y < 0.0f ? 2u : 0u) | (d.z < 0.0f ? 4u : 0u);
        const uint32_t key = (oct << (3 * kSortCellBits)) | cell;
        P.sort_keys[i] = key;
        const unsigned m = __activemask();
        const unsigned peers = __match_any_sync(m, key);
        if ((int)lane_id() == __ffs(peers) - 1) atomicAdd(&P.sort_hist[key], (uint32_t)__popc(peers));
    }
}

// Exclusive scan of the kSortBins counts in place (one block of 1024 threads).
__global__ void __launch_bounds__(1024) k_sort_scan(uint32_t* hist)
{
    constexpr int per = kSortBins / 1024;
    __shared__ uint32_t part[1024];
    uint32_t v[per], sum = 0;
#pragma unroll
    for (int k = 0; k < per; k++) {
        v[k] = hist[threadIdx.x * per + k];
        sum += v[k];
    }
    part[threadIdx.x] = sum;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
        const uint32_t add = threadIdx.x >= (unsigned)off ? part[threadIdx.x - off] : 0u;
        __syncthreads();
        part[threadIdx.x] += add;
        __syncthreads();
    }
    uint32_t run = part[threadIdx.x] - sum;
#pragma unroll
    for (int k = 0; k < per; k++) {
        hist[threadIdx.x * per + k] = run;
        run += v[k];
    }
}

__global__ void k_sort_scatter(const Ctrl* C, int bounce, const uint32_t* q, PathBuf P)
{
    const uint32_t count = C->count[bounce];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const uint32_t key = P.sort_keys[i];
        const unsigned m = __activemask();
        const unsigned peers = __match_any_sync(m, key);
        const int leader = __ffs(peers) - 1;
        uint32_t base = 0;
        if ((int)lane_id() == leader) base = atomicAdd(&P.sort_hist[key], (uint32_t)__popc(peers));
        base = __shfl_sync(peers, base, leader);
        P.qsort[base + (uint32_t)__popc(peers & ((1u << lane_id()) - 1u))] = q[i];
    }
}

// ---------------------------------------------------------------------------- multi-scene waves
//
// luz_gpu_batch_render packs the paths of many scenes into one wave: the wave is a
// list of segments (WaveArgs with batch_scene / batch_offset), each covering every
// sample of a run of pixels of one scene, and every path records its segment in
// P.seg. One launch per stage and bounce then serves all scenes: the persistent
// trace kernels fetch rays of any scene from the shared queues, look up the ray's
// scene in the table of DScene records (all of them pointing into one geometry
// arena) and traverse it; the shade kernel does the same. Rays traced per scene
// are counted for the per-scene statistics.

// Segment of wave slot p: the last segment starting at or before p.
__device__ __forceinline__ uint32_t find_segment(const WaveArgs* segs, uint32_t nseg, int64_t p)
{
    uint32_t lo = 0, hi = nseg;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (segs[mid].batch_offset <= p) lo = mid;
        else hi = mid;
    }
    return lo;
}

// The size of a multi-scene wave, read by the kernels of the wave's replayed graph.
struct BatchWaveHeader {
    int64_t n;
    uint32_t nseg;
    uint32_t pad;
};

__global__ void __launch_bounds__(kBlock) k_raygen_batch(const WaveArgs* segs, const BatchWaveHeader* hdr, PathBuf P,
                                                         Ctrl* C)
{
    const int64_t n = hdr->n;
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p == 0) C->count[0] = (uint32_t)n;
    if (p >= n) return;
    const uint32_t sg = find_segment(segs, hdr->nseg, p);
    const WaveArgs& w = segs[sg];
    uint32_t x, y, s;
    path_coords(w, (uint32_t)(p - w.batch_offset), x, y, s);
    double o[3], d[3];
    camera_ray(w, x, y, s, o, d);
    P.ray_o[p] = make_float4((float)o[0], (float)o[1], (float)o[2], __int_as_float(-1));
    P.ray_d[p] = make_float4((float)d[0], (float)d[1], (float)d[2], __int_as_float(-1));
    P.thr[p] = make_float4(1.f, 1.f, 1.f, 0.f);
    P.rad[p] = make_float4(0.f, 0.f, 0.f, __uint_as_float(PF_PREV_SPECULAR));
    P.pend0[p] = make_float4(0.f, 0.f, 0.f, 0.f);
    P.pend1[p] = make_float4(0.f, 0.f, 0.f, 0.f);
    P.pixel[p] = y * (uint32_t)w.width + x;
    P.sample[p] = s;
    P.seg[p] = sg;
    P.queue0[p] = (uint32_t)p;
}

// One per-scene counter add per group of lanes with the same scene.
__device__ __forceinline__ void count_by_scene(unsigned mask, uint32_t sid, unsigned long long* counts)
{
    const unsigned peers = __match_any_sync(mask, sid);
    if ((int)lane_id() == __ffs(peers) - 1) atomicAdd(&counts[sid], (unsigned long long)__popc(peers));
}

__global__ void __launch_bounds__(kBlock, LUZ_EXTEND_MIN_BLOCKS) k_extend_batch(const DScene* __restrict__ scenes,
                                                                               const WaveArgs* __restrict__ segs,
                                                                               PathBuf P, Ctrl* C, int bounce,
                                                                               unsigned long long* ext_rays)
{
    LocalStack<true> st;
    const uint32_t count = C->count[bounce];
    const uint32_t* q = (bounce & 1) ? P.queue1 : P.queue0;
    while (true) {
        uint32_t base = 0;
        if (lane_id() == 0) base = atomicAdd(&C->fetch_ext[bounce], 32u);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= count) break;
        const uint32_t i = base + lane_id();
        const unsigned vmask = __ballot_sync(0xffffffffu, i < count);
        if (i >= count) continue;
        const uint32_t p = q[i];
        const WaveArgs& w = segs[P.seg[p]];
        const DScene& S = scenes[w.batch_scene];
        const float4 o = P.ray_o[p], d = P.ray_d[p];
        const TRay r = make_ray_x(F3{o.x, o.y, o.z}, F3{d.x, d.y, d.z}, __float_as_int(o.w), __float_as_int(d.w));
        const uint32_t pix = P.pixel[p];
        Key k = path_key(w, pix % (uint32_t)w.width, pix / (uint32_t)w.width, P.sample[p], (uint32_t)bounce);
        VolSample vs{&k, 0.0, false};
        const THit h = closest_hit<TF_ALL>(S, r, kTMin, kInf, vs, st);
        P.hit[p] = make_float4(h.t, h.u, h.v, __int_as_float(h.obj));
        P.hit_prim[p] = h.prim;
        bin_append(C->bin[bounce], P, vmask, h.obj < 0 ? 0u : (uint32_t)S.obj_class[h.obj], p);
        count_by_scene(vmask, (uint32_t)w.batch_scene, ext_rays);
    }
}

__global__ void __launch_bounds__(kBlock, LUZ_SHADOW_MIN_BLOCKS) k_shadow_batch(const DScene* __restrict__ scenes,
                                                                               const WaveArgs* __restrict__ segs,
                                                                               PathBuf P, Ctrl* C, int bounce,
                                                                               unsigned long long* sh_rays)
{
    LocalStack<false> st;
    const uint32_t count = C->shadow[bounce];
    while (true) {
        uint32_t base = 0;
        if (lane_id() == 0) base = atomicAdd(&C->fetch_sh[bounce], 32u);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= count) break;
        const uint32_t i = base + lane_id();
        const unsigned vmask = __ballot_sync(0xffffffffu, i < count);
        if (i >= count) continue;
        const float4 o = P.sh_o[i], d = P.sh_d[i];
        const uint32_t tag = __float_as_uint(d.w);
        const uint32_t p = tag & 0x7fffffffu;
        const WaveArgs& w = segs[P.seg[p]];
        const DScene& S = scenes[w.batch_scene];
        const int2 x = P.sh_x[i];
        const TRay r = make_ray_x(F3{o.x, o.y, o.z}, F3{d.x, d.y, d.z}, x.x, x.y);
        const uint32_t pix = P.pixel[p];
        Key k = path_key(w, pix % (uint32_t)w.width, pix / (uint32_t)w.width, P.sample[p], (uint32_t)bounce);
        VolSample vs{&k, 0.0, false};
        if (any_hit<TF_ALL>(S, r, kTMin, o.w, vs, st)) {
            if (tag & 0x80000000u) P.pend1[p] = make_float4(0.f, 0.f, 0.f, 0.f);
            else P.pend0[p] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
        count_by_scene(vmask, (uint32_t)w.batch_scene, sh_rays);
    }
}

// k_accumulate over the segments of a multi-scene wave (blockIdx.y = segment): each
// pixel's samples, in sample order, into its scene's FP64 film.
__global__ void k_accumulate_batch(const WaveArgs* segs, const BatchWaveHeader* hdr, PathBuf P, double* const* films)
{
    if (blockIdx.y >= hdr->nseg) return;
    const WaveArgs& w = segs[blockIdx.y];
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= w.pix_count) return;
    double sx = 0.0, sy = 0.0, sz = 0.0;
    const int64_t b = w.batch_offset + j * w.s_count;
    for (int s = 0; s < w.s_count; s++) {
        const float4 r = P.rad[b + s], a = P.pend0[b + s], c2 = P.pend1[b + s];
        const F3 c = clean((F3{r.x, r.y, r.z} + F3{a.x, a.y, a.z}) + F3{c2.x, c2.y, c2.z});
        sx += (double)c.x;
        sy += (double)c.y;
        sz += (double)c.z;
    }
    double* f = films[w.batch_scene] + 3 * (int64_t)P.pixel[b];
    f[0] += sx;
    f[1] += sy;
    f[2] += sz;
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
    double* f = film + 3 * (int64_t)P.pixel[b];   // the slot's pixel (path_coords)
    f[0] += sx;
    f[1] += sy;
    f[2] += sz;
}

// Training rows of a radiance-cache wave: for every path with a snapshot, the
// cache's inputs at the vertex and the radiance its continuation gathered (final
// path radiance, as k_accumulate adds it, minus the radiance up to the vertex's
// NEE) over its throughput there; 0 when the path ended at the vertex.
__global__ void k_cache_targets(WaveArgs w, PathBuf P, CacheRecord* rows, uint32_t* count)
{
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= w.n || !w.cache_flag[p]) return;
    const float4 r = P.rad[p], a = P.pend0[p], b = P.pend1[p];
    const F3 fin = clean((F3{r.x, r.y, r.z} + F3{a.x, a.y, a.z}) + F3{b.x, b.y, b.z});
    const CacheSnap& sn = w.cache_s[p];
    const bool ended = w.cache_flag[p] == 2;
    CacheRecord q;
    for (int f = 0; f < kCacheIn; f++) q.in[f] = sn.in[f];
    const float fc[3] = {fin.x, fin.y, fin.z};
    for (int c = 0; c < 3; c++) {
        const float v = (!ended && sn.thr[c] > 1e-20f) ? (fc[c] - sn.rad[c]) / sn.thr[c] : 0.0f;
        q.v[c] = isfinite(v) ? v : 0.0f;
    }
    q.path = (uint32_t)p;
    q.pad[0] = q.pad[1] = 0.0f;
    rows[atomicAdd(count, 1u)] = q;
}

// Roughness-gradient records still open after a replay wave (their path ended at
// the vertex): the final light and environment samples, no continuation.
__global__ void k_adjoint_rough_finish(DScene S, WaveArgs w, PathBuf P)
{
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= w.n || !w.adj_rough[p].active) return;
    const float4 a = P.pend0[p], b = P.pend1[p];
    adjoint_rough_resolve(S, w, P, (uint32_t)p, F3{a.x, a.y, a.z}, F3{b.x, b.y, b.z}, F3{0.f, 0.f, 0.f}, false,
                          w.adj_rough[p]);
}

// Light samples still pending after a replay wave (their path ended at the
// vertex): the final, shadow-tested contribution of each.
__global__ void k_adjoint_emission_finish(DScene S, WaveArgs w, PathBuf P)
{
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= w.n || w.pend_light[p] < 0) return;
    const float4 a = P.pend0[p];
    adjoint_emission_add(S, w, P.pixel[p], w.pend_light[p], F3{a.x, a.y, a.z});
    w.pend_light[p] = -1;
}

// Light samples still pending after a density-replay wave, with their scores.
__global__ void k_adjoint_density_finish(DScene S, WaveArgs w, PathBuf P)
{
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= w.n) return;
    const float4 a = P.pend0[p], b = P.pend1[p];
    density_add(S, w, P.pixel[p], F3{a.x + b.x, a.y + b.y, a.z + b.z}, w.dens_score[p].y);
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

// ---------------------------------------------------------------------------- adaptive sampling / NFOR

// Per-pixel running sums of _threadRender (Threads.cpp:551-641): the colour sum
// and square sum (pixelColor / pixelColorSquare, equal to the adaptive
// accumulator's colorSum / colorSquareSum) and AdaptiveAccumulator's luminance
// statistics (Threads.cpp:31-53). Samples are added one at a time in sample
// order, as the reference does, so every sum is the same FP64 sequence.
struct PixAcc {
    double c[3], c2[3];
    double lum, lum2, lmax;
};
// DenoiseHalfAccumulator A/B and the feature sums (Threads.cpp:274-290).
struct PixNfor {
    double ca[3], cb[3];
    double fa[LUZ_NFOR_FEATURES], fb[LUZ_NFOR_FEATURES], fs[LUZ_NFOR_FEATURES], fq[LUZ_NFOR_FEATURES];
    uint32_t na, nb;
};
// Finished NFOR buffers on the device, laid out as LuzNforBuffers.
struct NforOut {
    double* color_a;
    double* color_b;
    double* color_variance;
    double* features_a;
    double* features_b;
    double* feature_variance;
};

// Adds the wave's samples of each pixel slot, in sample order, to its sums.
__global__ void k_accumulate_px(WaveArgs w, PathBuf P, PixAcc* acc, PixNfor* nf)
{
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= w.pix_count) return;
    const uint32_t pix = w.pix_list[w.pix_begin + j];
    PixAcc a = acc[pix];
    double f[LUZ_NFOR_FEATURES];
    if (nf) {   // setPrimaryCoordinates (ColorHelper.cpp:734-743)
        const uint32_t x = pix % (uint32_t)w.width, y = pix / (uint32_t)w.width;
        f[0] = w.width > 1 ? (double)x / ((double)w.width - 1.0) : 0.0;
        f[1] = w.height > 1 ? (double)y / ((double)w.height - 1.0) : 0.0;
    }
    const int64_t b = j * w.s_count;
    for (int s = 0; s < w.s_count; s++) {
        const float4 r = P.rad[b + s], pa = P.pend0[b + s], pb = P.pend1[b + s];
        const F3 cf = clean((F3{r.x, r.y, r.z} + F3{pa.x, pa.y, pa.z}) + F3{pb.x, pb.y, pb.z});
        const double c[3] = {(double)cf.x, (double)cf.y, (double)cf.z};
        if (nf) {
            const float4 g0 = P.feat[3 * (b + s)], g1 = P.feat[3 * (b + s) + 1], g2 = P.feat[3 * (b + s) + 2];
            f[2] = g0.x; f[3] = g0.y; f[4] = g0.z; f[5] = g0.w;
            f[6] = g1.x; f[7] = g1.y; f[8] = g1.z; f[9] = g1.w;
            f[10] = g2.x;
            PixNfor& n = nf[pix];
            const bool half_a = ((uint32_t)(w.s_begin + w.sample_offset + s) & 1u) == 0u;
            double* hc = half_a ? n.ca : n.cb;
            double* hf = half_a ? n.fa : n.fb;
            for (int k = 0; k < 3; k++) hc[k] += c[k];
            if (half_a) n.na++;
            else n.nb++;
            for (int k = 0; k < LUZ_NFOR_FEATURES; k++) {   // addDenoiseFeatureSample (Threads.cpp:274-290)
                hf[k] += f[k];
                n.fs[k] += f[k];
                n.fq[k] += f[k] * f[k];
            }
        }
        for (int k = 0; k < 3; k++) {
            a.c[k] += c[k];
            a.c2[k] += c[k] * c[k];
        }
        // sampleLuminance: ACEScg luminance in FP64 (ColorManagement.cpp:313-320), 0 if not finite.
        double l = c[0] * 0.2722287168 + c[1] * 0.6740817658 + c[2] * 0.0536895174;
        if (!isfinite(l)) l = 0.0;
        a.lum += l;
        a.lum2 += l * l;
        a.lmax = a.lmax < l ? l : a.lmax;
    }
    acc[pix] = a;
}

struct AdaptiveRule {
    uint32_t max_samples;   // scene sample count
    uint32_t min_samples;   // min(adaptive minimum, sample count)
    uint32_t interval;
    uint32_t dark_min;      // darkMinimumSamples (Threads.cpp:182-192)
    double threshold;
    int32_t can_stop;       // adaptiveSamplingCanStop (Threads.cpp:267-273)
};

// sampleMeanVariance (Threads.cpp:150-161); std::max(0, NaN) is 0.
__device__ __forceinline__ double mean_variance(double sum, double sq, uint32_t count)
{
    if (count <= 1) return 0.0;
    const double n = (double)count;
    const double var = (sq - (sum * sum / n)) / (n - 1.0);
    const double v = var / n;
    return 0.0 < v ? v : 0.0;
}
// confidenceInterval95 (Threads.cpp:163-172)
__device__ __forceinline__ double ci95(double sum, double sq, uint32_t count)
{
    const double mv = mean_variance(sum, sq, count);
    if (!isfinite(mv)) return __longlong_as_double(0x7ff0000000000000ll);
    return 1.96 * sqrt(mv);
}
// channelConverged (Threads.cpp:174-180)
__device__ __forceinline__ bool channel_converged(double mean, double ci, double threshold)
{
    const double am = fabs(mean);
    const double target = threshold * (am < 0.02 ? 0.02 : am);
    return ci <= target;
}
// adaptiveSampleConverged (Threads.cpp:194-265)
__device__ bool adaptive_converged(const AdaptiveRule& R, uint32_t used, const PixAcc& a)
{
    if (used >= R.max_samples) return true;
    if (!R.can_stop) return false;
    if (used < R.min_samples) return false;
    if ((used - R.min_samples) % R.interval != 0) return false;
    if (used <= 1) return false;
    const double n = (double)used;
    const double lum_mean = a.lum / n;
    if (a.lmax < 0.02 && used < R.dark_min) return false;
    const double lci = ci95(a.lum, a.lum2, used);
    const double rci = ci95(a.c[0], a.c2[0], used);
    const double gci = ci95(a.c[1], a.c2[1], used);
    const double bci = ci95(a.c[2], a.c2[2], used);
    return channel_converged(lum_mean, lci, R.threshold) && channel_converged(a.c[0] / n, rci, R.threshold)
        && channel_converged(a.c[1] / n, gci, R.threshold) && channel_converged(a.c[2] / n, bci, R.threshold);
}

// After a round of `used` samples: finished pixels get their mean colour,
// sample count and NFOR buffers (storeDenoisePixel, Threads.cpp:343-372); the
// others go to the next active list.
__global__ void k_converge(AdaptiveRule R, uint32_t used, const uint32_t* act, uint32_t n_act, uint32_t* next,
                           uint32_t* next_count, const PixAcc* acc, const PixNfor* nf, NforOut out_nf, float* rgb,
                           int32_t* used_out)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < n_act;
    const uint32_t pix = valid ? act[i] : 0u;
    bool done = true;
    if (valid) {
        const PixAcc a = acc[pix];
        done = adaptive_converged(R, used, a);
        if (done) {
            const double n = (double)used;
            for (int k = 0; k < 3; k++) {
                const double m = a.c[k] / n;
                rgb[3 * (int64_t)pix + k] = isfinite(m) ? (float)m : 0.0f;   // cleanColor(pixelColor / samplesUsed)
            }
            used_out[pix] = (int32_t)used;
            if (nf) {
                const PixNfor& f = nf[pix];
                const int64_t p3 = 3 * (int64_t)pix, pf = (int64_t)LUZ_NFOR_FEATURES * pix;
                for (int k = 0; k < 3; k++) {   // meanColor with the whole-pixel mean as fallback
                    out_nf.color_a[p3 + k] = f.na ? f.ca[k] / (double)f.na : a.c[k] / n;
                    out_nf.color_b[p3 + k] = f.nb ? f.cb[k] / (double)f.nb : a.c[k] / n;
                }
                out_nf.color_variance[pix] = (mean_variance(a.c[0], a.c2[0], used) + mean_variance(a.c[1], a.c2[1], used)
                                              + mean_variance(a.c[2], a.c2[2], used)) / 3.0;
                for (int k = 0; k < LUZ_NFOR_FEATURES; k++) {
                    const double fb = f.fs[k] / n;
                    out_nf.features_a[pf + k] = f.na ? f.fa[k] / (double)f.na : fb;
                    out_nf.features_b[pf + k] = f.nb ? f.fb[k] / (double)f.nb : fb;
                    out_nf.feature_variance[pf + k] = mean_variance(f.fs[k], f.fq[k], used);
                }
            }
        }
    }
    const uint32_t slot = warp_append(next_count, valid && !done);
    if (valid && !done) next[slot] = pix;
}

// ---------------------------------------------------------------------------- ray batches

// luz_gpu_trace_rays: one ray per thread through the traversal instantiation
// the extend / shadow kernels use for this scene.
template <uint32_t F>
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
    LocalStack<true> st;
    if (any) {
        const bool occ = any_hit<F>(S, ray, r[3], r[7], vs, st);
        o = LuzHit{0.f, occ ? 0 : -1, 0, 0.f, 0.f};
    } else {
        const THit h = closest_hit<F>(S, ray, r[3], r[7], vs, st);
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

using RayKernel = void (*)(DScene, const float*, int64_t, int, uint32_t, const int32_t*, LuzHit*);
const RayKernel kTraceRayKernels[4] = {k_trace_rays<0>, k_trace_rays<1>, k_trace_rays<2>, k_trace_rays<3>};

// ----------------------------------------------------------------------------- caustic photon map

// CausticPhotonMap::build photon loop (src/renderer/CausticPhotonMap.cpp:452-549),
// one thread per photon index: photon i of pass p (passStart = target * p / passes)
// samples with key (i, p, i - passStart, CAUSTIC_STREAM) under seed ^ CAUSTIC_SEED_SCRAMBLE.
// A stored photon is written to slot i with its packed cell key; other slots keep
// the empty key, so a stable sort by key gives cells in order and, inside a cell,
// photons in index order (the reference's storePhoton order).
template <uint32_t F>
__global__ void __launch_bounds__(128) k_photons(DScene S, uint32_t seed, int max_bounces, float4* ph,
                                                 unsigned long long* keys, uint32_t* order, uint32_t* stored)
{
    const GCaustics& G = S.k.caustics;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= G.photons) return;
    keys[i] = kEmptyCell;
    order[i] = (uint32_t)i;
    const int64_t target = G.photons, passes = G.passes;
    int64_t pass = i * passes / target;
    while (pass + 1 < passes && target * (pass + 1) / passes <= i) pass++;
    while (pass > 0 && target * pass / passes > i) pass--;
    const int64_t start = target * pass / passes;
    Key k{base_key(seed ^ kCausticSeedScramble, (uint32_t)i, (uint32_t)pass, kCausticStream), (uint32_t)(i - start), 0u};
    Emission e;
    double sel = 0.0;
    if (!photon_emission(S, k, e, sel)) return;
    const double scale = e.power * G.m2_per_area, den = (double)target * sel;
    F3 thr{(float)((double)e.emitted.x * scale / den), (float)((double)e.emitted.y * scale / den),
           (float)((double)e.emitted.z * scale / den)};
    if (!valid_positive(thr)) return;
    TRay ray = make_ray(e.pos + e.dir * (2.0f * kTMin), e.dir);
    bool caustic = false;
    LocalStack<true> st;
    for (int b = 0; b <= max_bounces; b++) {
        k.bounce = (uint32_t)b;
        VolSample vs{&k, 0.0, false};
        const THit th = closest_hit<F>(S, ray, kTMin, kInf, vs, st);
        if (th.obj < 0) break;
        const Hit h = make_hit(S, ray, th);
        GMaterial m = S.materials[h.material];
        resolve_material(S, m, h);
        if (m.type == MT_EMISSIVE) break;
        if (caustic && receives_caustics(m)) {
            const double r = G.radius_su;
            unsigned long long key;
            if (!pack_cell(floor((double)h.p.x / r), floor((double)h.p.y / r), floor((double)h.p.z / r), key)) {
                atomicOr(S.error, ERR_CAUSTIC_GRID);
                break;
            }
            ph[3 * i] = make_float4(h.p.x, h.p.y, h.p.z, thr.x);
            ph[3 * i + 1] = make_float4(h.n.x, h.n.y, h.n.z, thr.y);
            ph[3 * i + 2] = make_float4(ray.d.x, ray.d.y, ray.d.z, thr.z);
            keys[i] = key;
            atomicAdd(stored, 1u);
            break;
        }
        Scatter sr;
        if (!scatter(S, m, h, ray.d, k, sr)) break;
        F3 att = sr.att;
        if (!h.front && sr.absorb) {   // effectiveScatterAttenuation (:135-149)
            const float dm = h.t * (float)S.k.meters_per_unit;
            if (isfinite(dm) && dm > 0.0f)
                att = att * F3{expf(-sr.absorption.x * dm), expf(-sr.absorption.y * dm), expf(-sr.absorption.z * dm)};
        }
        if (!valid_positive(att)) break;
        if (!sr.specular && !(m.flags & MF_TRANSPORT)) break;
        thr = thr * att;
        if (!valid_positive(thr) || !photon_roulette(thr, b, k)) break;
        ray = make_ray_x(h.p, sr.dir, h.volume ? -1 : h.obj, h.volume ? -1 : h.prim);
        caustic = true;
    }
}

using PhotonKernel = void (*)(DScene, uint32_t, int, float4*, unsigned long long*, uint32_t*, uint32_t*);
const PhotonKernel kPhotonKernels[4] = {k_photons<0>, k_photons<1>, k_photons<2>, k_photons<3>};

// Sorted photon j <- unsorted photon order[j].
__global__ void k_photon_gather(const float4* raw, const uint32_t* order, uint32_t n, float4* out)
{
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const uint32_t i = order[j];
    out[3 * (size_t)j] = raw[3 * (size_t)i];
    out[3 * (size_t)j + 1] = raw[3 * (size_t)i + 1];
    out[3 * (size_t)j + 2] = raw[3 * (size_t)i + 2];
}
// The first photon of each cell inserts the cell key with its begin index.
// The table holds at least twice as many slots as photons, so a free slot exists.
__global__ void k_cell_starts(const unsigned long long* keys, uint32_t n, unsigned long long* tkeys, uint2* ranges,
                              uint32_t mask)
{
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const unsigned long long key = keys[j];
    if (j > 0 && keys[j - 1] == key) return;
    uint32_t slot = cell_slot(key, mask);
    for (uint32_t probe = 0; probe <= mask; probe++) {
        const unsigned long long prev = atomicCAS(tkeys + slot, kEmptyCell, key);
        if (prev == kEmptyCell || prev == key) {
            ranges[slot].x = j;
            return;
        }
        slot = (slot + 1) & mask;
    }
}
// The last photon of each cell writes the end of the cell's range.
__global__ void k_cell_ends(const unsigned long long* keys, uint32_t n, const unsigned long long* tkeys, uint2* ranges,
                            uint32_t mask)
{
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const unsigned long long key = keys[j];
    if (j + 1 < n && keys[j + 1] == key) return;
    uint32_t slot = cell_slot(key, mask);
    for (uint32_t probe = 0; probe <= mask; probe++) {
        if (tkeys[slot] == key) {
            ranges[slot].y = j + 1;
            return;
        }
        slot = (slot + 1) & mask;
    }
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

uint64_t next_scene_uid()
{
    static std::atomic<uint64_t> n{0};
    return ++n;
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
    // second wave lane (render_enqueue): its counters, stream and the events that order
    // the lanes (setup before lane 1; each wave's film accumulation after the previous
    // wave's; lane 1 done before the resolve); created by the first two-lane render
    Ctrl* ctrl2 = nullptr;
    cudaStream_t stream2 = nullptr;
    cudaEvent_t lane_setup = nullptr, lane_done = nullptr, lane_acc[2] = {nullptr, nullptr};
    unsigned long long* status_host = nullptr;   // pinned: ray totals [0..1] and error word [2] of a call
    unsigned long long* totals = nullptr;   // device: extension / shadow rays of the current render
    double* film = nullptr;
    int64_t film_pix = 0;
    float* out_dev = nullptr;        // luz_gpu_render: device film of per-pixel means
    int64_t out_cap = 0;
    int sms = 0;
    int occ_ext = 1, occ_shade = 1, occ_sh = 1;
    LuzTuneParams tune{};            // luz_gpu_scene_set_tuning / luz_gpu_autotune; zeros = defaults
    // multi-scene batches copy the scene arrays into their geometry arena: byte offset of
    // each array pointer inside DScene and the array's size; uid / version name the
    // content (version changes with texels or the caustic map)
    std::vector<std::pair<std::size_t, std::size_t>> arena_fields;
    uint64_t uid = 0, version = 0;
    TraceKernel extend = nullptr, shadow = nullptr;   // instantiations for this scene's features
    ShadeKernel shade = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // caustic photon map: buffers grown on demand; the map is kept while the
    // render seed and bounce limit stay the same (textures unchanged)
    struct PhotonMap {
        std::vector<void*> bufs, tbufs;
        int64_t cap = 0, tcap = 0;
        float4 *raw = nullptr, *ph = nullptr;
        unsigned long long *kin = nullptr, *kout = nullptr, *tkeys = nullptr;
        uint32_t *vin = nullptr, *vout = nullptr, *count = nullptr;
        uint2* ranges = nullptr;
        void* tmp = nullptr;
        size_t tmp_bytes = 0;
        bool valid = false;
        uint32_t seed = 0;
        int bounces = -1;
        uint32_t stored = 0;
        float last_ms = 0.f;   // build time of the last call that built the map (0 when reused)
    } cm;

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
    // Bytes of path state per path: the PathBuf arrays a wave allocates (NFOR
    // features add 3 float4).
    static constexpr int64_t kPathBytes = 8 * 16 + 5 * 4 + 2 * (16 + 16 + 8) + kShadeClasses * 4 + 2 * 4;
    static constexpr int64_t kFeatBytes = 3 * 16;
    // Smallest wave a render falls back to when cudaMalloc refuses a larger one.
    static constexpr int64_t kMinWavePaths = int64_t(1) << 20;
    int64_t path_budget = -1;        // bytes of path state this handle may hold; -1 = a quarter of
                                     // the device memory free (plus what the handle holds) at the time
    void alloc_paths(int64_t n, bool feat)
    {
        pb.ray_o = palloc<float4>(n);
        pb.ray_d = palloc<float4>(n);
        pb.thr = palloc<float4>(n);
        pb.rad = palloc<float4>(n);
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
        pb.feat = feat ? palloc<float4>(3 * n) : nullptr;
        pb.bins = palloc<uint32_t>(kShadeClasses * n);
        pb.bin_stride = (uint32_t)n;
        pb.sort_keys = palloc<uint32_t>(n);
        pb.qsort = palloc<uint32_t>(n);
        pb.sort_hist = palloc<uint32_t>(2 * kSortBins);   // one histogram per wave lane
        cap = n;
    }
    // Paths a wave of up to `want` paths may use: the buffers held when they are
    // large enough, else new ones of min(want, budget) paths. When cudaMalloc
    // refuses them (memory held by other work on the device) the request is
    // halved, down to kMinWavePaths, so the render runs in more, smaller waves
    // (the image does not depend on the wave size). Returns the paths available.
    int64_t reserve_paths(int64_t want, bool feat = false)
    {
        want = std::max<int64_t>(1, want);
        // buffers already held serve without asking the driver for its free memory
        // (cudaMemGetInfo costs host time on every render otherwise)
        if (want <= cap && (!feat || pb.feat) && (path_budget < 0 || want * (kPathBytes + (feat ? kFeatBytes : 0)) <= path_budget))
            return want;
        const int64_t per = kPathBytes + (feat ? kFeatBytes : 0);
        int64_t budget = path_budget;
        if (budget < 0) {
            size_t free_b = 0, total_b = 0;
            CK(cudaMemGetInfo(&free_b, &total_b));
            const int64_t held = cap * (kPathBytes + (pb.feat ? kFeatBytes : 0));
            budget = ((int64_t)free_b + held) / 4;
        }
        int64_t n = std::min(want, std::max<int64_t>(1, budget / per));
        if (n <= cap && (!feat || pb.feat)) return n;
        const int64_t floor_n = std::min(n, kMinWavePaths);
        n = std::max(n, std::min(cap, want));
        free_paths();
        while (true) {
            try {
                alloc_paths(n, feat);
                return n;
            } catch (const Status& e) {
                free_paths();
                (void)cudaGetLastError();   // clears the allocation error
                if (e.code != LUZ_E_CUDA || n <= floor_n) throw;
                n = std::max(floor_n, n / 2);
            }
        }
    }
    ~luz_gpu_scene()
    {
        cudaSetDevice(device);
        free_paths();
        for (void* p : cm.bufs) cudaFree(p);
        for (void* p : cm.tbufs) cudaFree(p);
        if (out_dev) cudaFree(out_dev);
        for (void* p : allocs) cudaFree(p);
        if (ctrl) cudaFree(ctrl);
        if (ctrl_host) cudaFreeHost(ctrl_host);
        if (status_host) cudaFreeHost(status_host);
        if (film) cudaFree(film);
        if (dds) cudaFree(dds);
        if (totals) cudaFree(totals);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (stream) cudaStreamDestroy(stream);
        if (ctrl2) cudaFree(ctrl2);
        for (cudaEvent_t e : {lane_setup, lane_done, lane_acc[0], lane_acc[1]})
            if (e) cudaEventDestroy(e);
        if (stream2) cudaStreamDestroy(stream2);
    }
    void ensure_lanes()
    {
        if (stream2) return;
        ctrl2 = dalloc<Ctrl>(1);
        CK(cudaEventCreateWithFlags(&lane_setup, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&lane_done, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&lane_acc[0], cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&lane_acc[1], cudaEventDisableTiming));
        CK(cudaStreamCreateWithFlags(&stream2, cudaStreamNonBlocking));
    }
};

namespace {

// Lane 1's view of a path buffer: the upper half of every per-path array, from
// path `off` on (shadow records 2 per path, features 3; the class segments keep
// their stride, so lane 1 uses the upper half of each), and the second sort histogram.
PathBuf lane_view(const PathBuf& b, int64_t off)
{
    PathBuf v = b;
    v.ray_o += off;
    v.ray_d += off;
    v.thr += off;
    v.rad += off;
    v.pend0 += off;
    v.pend1 += off;
    v.pixel += off;
    v.sample += off;
    v.hit += off;
    v.hit_prim += off;
    v.queue0 += off;
    v.queue1 += off;
    v.sh_o += 2 * off;
    v.sh_d += 2 * off;
    v.sh_x += 2 * off;
    v.color += off;
    if (v.feat) v.feat += 3 * off;
    v.bins += off;
    if (v.seg) v.seg += off;
    v.sort_keys += off;
    v.qsort += off;
    v.sort_hist += kSortBins;
    return v;
}

}  // namespace

namespace {

// Smallest lane of a two-lane render (render_prepare).
constexpr int64_t kMinLanePaths = int64_t(1) << 22;

// Paths in flight per wave. A launch of the persistent trace kernels lasts at
// least as long as its slowest warp's traversal, a tail of the order of half a
// millisecond per bounce on incoherent rays; larger waves pay it fewer times per
// frame (1080p glossy frame, 64 spp: 4 Mi paths 231.5, 8 Mi 305.6, 16 Mi 363.5,
// 32 Mi 395.4-400.0, 64 Mi 414.5 Msamples/s, the image the same bit for bit).
// Path state is 268 B per path (18 GB at 64 Mi, a tenth of the B200's HBM) and
// stays allocated with the scene handle.
constexpr int64_t kWaveTarget = int64_t(1) << 26;
// The cached render updates its cache once per wave; its default wave is 4 Mi
// paths (a handle's tuned wave_paths replaces it).
constexpr int64_t kCacheWaveTarget = int64_t(1) << 22;

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

// shade: the shade instantiation to run (NULL: the scene's own).
void launch_bounces(luz_gpu_scene* s, const WaveArgs& w, cudaStream_t st, int64_t& launches, StageTimer& T,
                    ShadeKernel shade, const PathBuf& pb, Ctrl* ctrl)
{
    auto blocks = [](int tuned, int occ) { return tuned > 0 ? std::min(tuned, occ) : occ; };
    const int g_ext = s->sms * blocks(s->tune.extend_blocks_per_sm, s->occ_ext);
    const int g_sh = s->sms * blocks(s->tune.shadow_blocks_per_sm, s->occ_sh);
    const int g_shade = s->sms * blocks(s->tune.shade_blocks_per_sm, s->occ_shade);
    if (!shade) shade = s->shade;
    const int count = s->ds.counters ? 1 : 0;   // LUZ_RENDER_COUNT renders run the counting instantiations
    const uint32_t kv = (s->ds.k.features & TF_ALL) | (s->tune.staged_top_nodes && s->ds.top4_count ? TF_STAGED : 0u);
    const TraceKernel extend = kExtendKernels[count][kv];
    const TraceKernel shadow = kShadowKernels[kv];
    WaveArgs ws = w;
    const bool sort = s->tune.sort_rays != 0 && pb.qsort;
    if (sort) ws.sorted_queue = pb.qsort;
    for (int b = 0; b <= w.max_bounces; b++) {
        if (sort && b >= 1) {
            const uint32_t* q = (b & 1) ? pb.queue1 : pb.queue0;
            CK(cudaMemsetAsync(pb.sort_hist, 0, sizeof(uint32_t) * kSortBins, st));
            k_sort_keys<<<s->sms * 8, 256, 0, st>>>(ctrl, b, q, pb, s->ds.k);
            k_sort_scan<<<1, 1024, 0, st>>>(pb.sort_hist);
            k_sort_scatter<<<s->sms * 8, 256, 0, st>>>(ctrl, b, q, pb);
            launches += 3;
        }
        T.mark(st, 0, true);
        extend<<<g_ext, kBlock, 0, st>>>(s->ds, ws, pb, ctrl, b);
        T.mark(st, 0, false);
        T.mark(st, 1, true);
        shade<<<g_shade, kBlock, 0, st>>>(s->dds, w, pb, ctrl, b);
        T.mark(st, 1, false);
        T.mark(st, 2, true);
        shadow<<<g_sh, kBlock, 0, st>>>(s->ds, w, pb, ctrl, b);
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
        throw Status(LUZ_E_UNSUPPORTED, "Unknown render flags.");
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

// CausticPhotonMap::build for this render's seed and bounce limit (Renderer.cpp:40-48
// builds it before every render): photon kernel, stable radix sort of the photon
// slots by cell key, gather, and the cell table. Synchronous on st.
void prepare_caustics(luz_gpu_scene* s, const LuzRenderParams* p, cudaStream_t st)
{
    const GCaustics& G = s->pack->consts.caustics;
    auto& M = s->cm;
    M.last_ms = 0.f;
    if (!G.enabled) return;
    if (M.valid && M.seed == p->seed && M.bounces == p->max_bounces) return;
    M.valid = false;
    s->ds.cm = DCaustics{};
    const int64_t n = G.photons;
    if (n > M.cap) {
        for (void* q : M.bufs) cudaFree(q);
        M.bufs.clear();
        M.cap = 0;
        auto get = [&](std::size_t bytes) {
            void* q = dalloc<uint8_t>(bytes);
            M.bufs.push_back(q);
            return q;
        };
        M.raw = static_cast<float4*>(get(sizeof(float4) * 3 * (std::size_t)n));
        M.ph = static_cast<float4*>(get(sizeof(float4) * 3 * (std::size_t)n));
        M.kin = static_cast<unsigned long long*>(get(sizeof(unsigned long long) * (std::size_t)n));
        M.kout = static_cast<unsigned long long*>(get(sizeof(unsigned long long) * (std::size_t)n));
        M.vin = static_cast<uint32_t*>(get(sizeof(uint32_t) * (std::size_t)n));
        M.vout = static_cast<uint32_t*>(get(sizeof(uint32_t) * (std::size_t)n));
        M.count = static_cast<uint32_t*>(get(sizeof(uint32_t)));
        M.tmp_bytes = 0;
        CK(cub::DeviceRadixSort::SortPairs(nullptr, M.tmp_bytes, M.kin, M.kout, M.vin, M.vout, (int)n, 0, 64, st));
        M.tmp = get(std::max<size_t>(M.tmp_bytes, 16));
        M.cap = n;
    }
    CK(cudaEventRecord(s->ev0, st));
    CK(cudaMemsetAsync(M.count, 0, sizeof(uint32_t), st));
    kPhotonKernels[s->ds.k.features & TF_ALL]<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(
        s->ds, p->seed, p->max_bounces, M.raw, M.kin, M.vin, M.count);
    CK(cudaGetLastError());
    size_t tb = M.tmp_bytes;
    CK(cub::DeviceRadixSort::SortPairs(M.tmp, tb, M.kin, M.kout, M.vin, M.vout, (int)n, 0, 64, st));
    uint32_t stored = 0, err = 0;
    CK(cudaMemcpyAsync(&stored, M.count, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(&err, s->ds.error, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (err & ERR_CAUSTIC_GRID) {
        CK(cudaMemsetAsync(s->ds.error, 0, sizeof(uint32_t), st));
        CK(cudaStreamSynchronize(st));
        throw Status(LUZ_E_LIMIT, "Caustic photons lie outside the photon grid (2^21 cells per axis).");
    }
    int64_t T = 64;
    while (T < 2 * (int64_t)stored) T *= 2;
    if (T > M.tcap) {
        for (void* q : M.tbufs) cudaFree(q);
        M.tbufs.clear();
        M.tcap = 0;
        M.tkeys = dalloc<unsigned long long>((std::size_t)T);
        M.tbufs.push_back(M.tkeys);
        M.ranges = dalloc<uint2>((std::size_t)T);
        M.tbufs.push_back(M.ranges);
        M.tcap = T;
    }
    const uint32_t mask = (uint32_t)(T - 1);
    CK(cudaMemsetAsync(M.tkeys, 0xff, sizeof(unsigned long long) * (std::size_t)T, st));
    CK(cudaMemsetAsync(M.ranges, 0, sizeof(uint2) * (std::size_t)T, st));
    if (stored > 0) {
        const unsigned g = (stored + 127) / 128;
        k_photon_gather<<<g, 128, 0, st>>>(M.raw, M.vout, stored, M.ph);
        k_cell_starts<<<g, 128, 0, st>>>(M.kout, stored, M.tkeys, M.ranges, mask);
        k_cell_ends<<<g, 128, 0, st>>>(M.kout, stored, M.tkeys, M.ranges, mask);
        CK(cudaGetLastError());
    }
    CK(cudaEventRecord(s->ev1, st));
    CK(cudaEventSynchronize(s->ev1));
    CK(cudaEventElapsedTime(&M.last_ms, s->ev0, s->ev1));
    s->ds.cm = DCaustics{M.ph, M.tkeys, M.ranges, mask, stored};
    s->version++;
    CK(cudaMemcpy(s->dds, &s->ds, sizeof(DScene), cudaMemcpyHostToDevice));
    M.stored = stored;
    M.seed = p->seed;
    M.bounces = p->max_bounces;
    M.valid = true;
}

void caustic_stats(const luz_gpu_scene* s, LuzRenderStats* stats)
{
    if (!stats || !s->pack->consts.caustics.enabled) return;
    stats->caustic_photons = (double)s->cm.stored;
    stats->caustic_ms = s->cm.last_ms;
}

// Every call clears the scene's device error word on its stream before it
// enqueues work, and reads it back (finish_status) after the work: a flag set by
// one call is reported by that call alone and leaves the handle usable.
void clear_error(luz_gpu_scene* s, cudaStream_t st)
{
    CK(cudaMemsetAsync(s->ds.error, 0, sizeof(uint32_t), st));
}

// After a call's work on st: copies the ray totals (when `totals` is given) and
// the error word into the handle's pinned status buffer, clears the word, waits
// for st and throws LUZ_E_DEVICE when a kernel set a flag.
void finish_status(luz_gpu_scene* s, cudaStream_t st, const unsigned long long* totals = nullptr,
                   unsigned long long* tot_out = nullptr)
{
    unsigned long long* h = s->status_host;
    h[0] = h[1] = h[2] = 0;
    if (totals) CK(cudaMemcpyAsync(h, totals, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(h + 2, s->ds.error, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    CK(cudaMemsetAsync(s->ds.error, 0, sizeof(uint32_t), st));
    CK(cudaStreamSynchronize(st));
    if (tot_out) {
        tot_out[0] = h[0];
        tot_out[1] = h[1];
    }
    const uint32_t err = (uint32_t)h[2];
    if (err)
        throw Status(LUZ_E_DEVICE, "Traversal stack overflow reported by the device (flags " + std::to_string(err) + ").");
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
    finish_status(s, st);
}

// One render split in three phases so that a batch can allocate for every
// scene first (cudaFree synchronises the device), then enqueue every scene on
// its own stream, then wait: render_prepare / render_enqueue / render_finish.
struct RenderJob {
    luz_gpu_scene* s = nullptr;
    const LuzRenderParams* p = nullptr;
    float* d_out = nullptr;
    cudaStream_t st = nullptr;
    WaveArgs w{};
    int64_t npix = 0, pix_wave = 0;
    int64_t wave_target = kWaveTarget;
    int s_wave = 0;
    int lanes = 1;                 // 2: waves alternate between two halves of the path state
    int64_t lane_paths = 0;        // paths per lane
    StageTimer T;
    unsigned long long* counters = nullptr;
    int64_t launches = 0, waves = 0;
};

void render_prepare(RenderJob& J)
{
    const LuzRenderParams* p = J.p;
    luz_gpu_scene* s = J.s;
    check_params(p);
    CK(cudaSetDevice(s->device));
    clear_error(s, J.st);
    prepare_caustics(s, p, J.st);
    J.w = base_args(s, p);
    J.npix = (int64_t)p->width * p->height;
    const int64_t target = s->tune.wave_paths > 0 ? s->tune.wave_paths : J.wave_target;   // the budget caps both
    const int64_t n = s->reserve_paths(std::min<int64_t>(target, J.npix * (int64_t)p->spp));
    // Two lanes when the frame takes more than one wave: the path state is split in
    // halves and consecutive waves run on two streams, so that the last bounces of
    // one wave (few rays, each launch as long as its slowest warp) overlap the first
    // bounces of the next. Stage-timed renders keep one lane.
    J.T.on = (p->flags & LUZ_RENDER_PROFILE) != 0;
    J.lanes = (!J.T.on && s->tune.lanes != 1 && J.npix * (int64_t)p->spp > n && n >= 2 * kMinLanePaths) ? 2 : 1;
    J.lane_paths = n / J.lanes;
    if (J.lanes == 2) s->ensure_lanes();
    J.s_wave = (int)std::min<int64_t>(p->spp, J.lane_paths);
    J.pix_wave = std::max<int64_t>(1, std::min<int64_t>(J.npix, J.lane_paths / J.s_wave));
    if (s->film_pix < J.npix) {
        if (s->film) cudaFree(s->film);
        s->film = nullptr;
        s->film_pix = 0;
        s->film = dalloc<double>((std::size_t)(3 * J.npix));
        s->film_pix = J.npix;
    }
    if (p->flags & LUZ_RENDER_COUNT) J.counters = dalloc<unsigned long long>(8);
}

void render_enqueue(RenderJob& J)
{
    luz_gpu_scene* s = J.s;
    const LuzRenderParams* p = J.p;
    const cudaStream_t st = J.st;
    WaveArgs& w = J.w;
    CK(cudaSetDevice(s->device));
    CK(cudaEventRecord(s->ev0, st));   // render_ms spans all of the render's work on the stream
    clear_error(s, st);
    if (J.counters) CK(cudaMemsetAsync(J.counters, 0, 8 * sizeof(unsigned long long), st));
    s->ds.counters = J.counters;
    CK(cudaMemcpyAsync(s->dds, &s->ds, sizeof(DScene), cudaMemcpyHostToDevice, st));
    CK(cudaMemsetAsync(s->film, 0, sizeof(double) * 3 * J.npix, st));
    CK(cudaMemsetAsync(s->totals, 0, 2 * sizeof(unsigned long long), st));
    const bool two = J.lanes == 2;
    const cudaStream_t lane_st[2] = {st, two ? s->stream2 : st};
    Ctrl* const lane_ctrl[2] = {s->ctrl, two ? s->ctrl2 : s->ctrl};
    const PathBuf lane_pb[2] = {s->pb, two ? lane_view(s->pb, J.lane_paths) : s->pb};
    if (two) {   // lane 1 starts after the film, totals and scene copy are set
        CK(cudaEventRecord(s->lane_setup, st));
        CK(cudaStreamWaitEvent(s->stream2, s->lane_setup, 0));
    }
    int64_t k = 0;
    for (int sb = 0; sb < p->spp; sb += J.s_wave) {
        const int sc = std::min(J.s_wave, p->spp - sb);
        for (int64_t pb = 0; pb < J.npix; pb += J.pix_wave) {
            const int64_t pc = std::min<int64_t>(J.pix_wave, J.npix - pb);
            const int L = two ? (int)(k & 1) : 0;
            const cudaStream_t ls = lane_st[L];
            w.pix_begin = (int32_t)pb;
            w.pix_count = (int32_t)pc;
            w.s_begin = sb;
            w.s_count = sc;
            w.n = pc * sc;
            w.list_mode = 0;
            CK(cudaMemsetAsync(lane_ctrl[L], 0, sizeof(Ctrl), ls));
            k_raygen<<<(unsigned)((w.n + kBlock - 1) / kBlock), kBlock, 0, ls>>>(w, lane_pb[L], lane_ctrl[L]);
            launch_bounces(s, w, ls, J.launches, J.T, nullptr, lane_pb[L], lane_ctrl[L]);
            // the film adds waves in order (samples of a pixel in sample order), the totals one at a time
            if (two && k > 0) CK(cudaStreamWaitEvent(ls, s->lane_acc[1 - L], 0));
            k_accumulate<<<(unsigned)((pc + 127) / 128), 128, 0, ls>>>(w, lane_pb[L], s->film);
            k_tally<<<1, 1, 0, ls>>>(lane_ctrl[L], w.max_bounces, s->totals);
            if (two) CK(cudaEventRecord(s->lane_acc[L], ls));
            J.launches += 3;
            J.waves++;
            k++;
            if (J.T.on) {
                CK(cudaStreamSynchronize(st));
                J.T.collect();
            }
        }
    }
    if (two) {
        CK(cudaEventRecord(s->lane_done, s->stream2));
        CK(cudaStreamWaitEvent(st, s->lane_done, 0));
    }
    k_resolve<<<(unsigned)((J.npix + 255) / 256), 256, 0, st>>>(s->film, J.npix, (double)p->spp, J.d_out);
    J.launches++;
    CK(cudaGetLastError());
    CK(cudaEventRecord(s->ev1, st));
}

void render_finish(RenderJob& J, LuzRenderStats* stats)
{
    luz_gpu_scene* s = J.s;
    const LuzRenderParams* p = J.p;
    CK(cudaSetDevice(s->device));
    CK(cudaEventSynchronize(s->ev1));
    CK(cudaGetLastError());
    LuzRenderStats acc{};
    {
        unsigned long long tot[2] = {0, 0};
        finish_status(s, J.st, s->totals, tot);
        acc.extension_rays = (double)tot[0];
        acc.shadow_rays = (double)tot[1];
    }
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, s->ev0, s->ev1));
    s->ds.counters = nullptr;
    unsigned long long cnt[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (J.counters) {
        CK(cudaMemcpy(cnt, J.counters, sizeof(cnt), cudaMemcpyDeviceToHost));
        cudaFree(J.counters);
        J.counters = nullptr;
        CK(cudaMemcpy(s->dds, &s->ds, sizeof(DScene), cudaMemcpyHostToDevice));
    }
    if (stats) {
        *stats = acc;
        stats->render_ms = ms;
        stats->samples = (double)J.npix * p->spp;
        stats->kernel_launches = J.launches;
        stats->waves = J.waves;
        stats->extend_ms = J.T.ms[0];
        stats->shade_ms = J.T.ms[1];
        stats->shadow_ms = J.T.ms[2];
        stats->extend_launches = J.waves * (p->max_bounces + 1);
        stats->shadow_launches = J.waves * (p->max_bounces + 1);
        stats->ext_nodes = (double)cnt[0];
        stats->ext_tris = (double)cnt[1];
        stats->ext_top = (double)cnt[2];
        stats->sh_nodes = (double)cnt[3];
        stats->sh_tris = (double)cnt[4];
        stats->sh_top = (double)cnt[5];
        stats->ext_bnodes = (double)cnt[6];
        stats->sh_bnodes = (double)cnt[7];
        caustic_stats(s, stats);
    }
}

int do_render(luz_gpu_scene* s, const LuzRenderParams* p, float* d_out, cudaStream_t st, LuzRenderStats* stats)
{
    RenderJob J;
    J.s = s;
    J.p = p;
    J.d_out = d_out;
    J.st = st;
    try {
        render_prepare(J);
        render_enqueue(J);
        render_finish(J, stats);
    } catch (...) {
        if (J.counters) {
            cudaFree(J.counters);
            s->ds.counters = nullptr;
        }
        throw;
    }
    return LUZ_OK;
}

// Device buffers of one luz_gpu_render_ex call, freed on every exit path.
struct DeviceScratch {
    std::vector<void*> ptrs;
    template <class T> T* get(int64_t n, cudaStream_t st)
    {
        T* p = dalloc<T>((std::size_t)n);
        ptrs.push_back(p);
        CK(cudaMemsetAsync(p, 0, sizeof(T) * (std::size_t)std::max<int64_t>(n, 1), st));
        return p;
    }
    ~DeviceScratch()
    {
        for (void* p : ptrs) cudaFree(p);
    }
};

// Scene::setAdaptive* validation (src/scene/Scene.cpp:193-222).
void check_adaptive(const LuzAdaptiveParams* a)
{
    if (!a || !a->enabled) return;
    if (a->min_samples <= 0) throw Status(LUZ_E_INVALID, "Adaptive minimum samples must be positive.");
    if (a->check_interval <= 0) throw Status(LUZ_E_INVALID, "Adaptive check interval must be positive.");
    if (!std::isfinite(a->threshold) || a->threshold <= 0.0)
        throw Status(LUZ_E_INVALID, "Adaptive threshold must be positive.");
}

// The sample counts after which some pixel may stop: every check point
// adaptiveSampleConverged can pass (min, min + interval, ... > 1) and spp.
std::vector<uint32_t> round_ends(const AdaptiveRule& R)
{
    std::vector<uint32_t> e;
    if (R.can_stop)
        for (uint64_t m = R.min_samples; m < R.max_samples; m += R.interval)
            if (m > 1) e.push_back((uint32_t)m);
    e.push_back(R.max_samples);
    return e;
}

// pixels / pixel_count: render only these pixels (y * width + x, distinct); rgb_out then
// holds pixel_count means in list order.
int do_render_ex(luz_gpu_scene* s, const LuzRenderParams* p, const LuzAdaptiveParams* ad, float* rgb_out,
                 const LuzNforBuffers* nfor, int32_t* samples_out, LuzRenderStats* stats,
                 const LuzNforSettings* denoise = nullptr, double* denoised_out = nullptr,
                 const int32_t* pixels = nullptr, int64_t pixel_count = 0)
{
    check_params(p);
    check_adaptive(ad);
    if (denoised_out && denoise &&
        (denoise->regression_radius <= 0 || denoise->patch_radius <= 0 || denoise->feature_prefilter_radius < 0))
        throw Status(LUZ_E_INVALID, "NFOR radii must be positive.");
    if (p->flags) throw Status(LUZ_E_UNSUPPORTED, "Render flags are not supported with adaptive sampling or NFOR buffers.");
    CK(cudaSetDevice(s->device));
    const cudaStream_t st = s->stream;
    const int64_t npix = (int64_t)p->width * p->height;
    if (npix > (int64_t)UINT32_MAX) throw Status(LUZ_E_LIMIT, "Image has too many pixels.");
    clear_error(s, st);
    prepare_caustics(s, p, st);

    AdaptiveRule R{};
    R.max_samples = (uint32_t)p->spp;
    const bool enabled = ad && ad->enabled;
    R.can_stop = enabled && ad->min_samples < p->spp;
    if (R.can_stop) {
        R.min_samples = (uint32_t)std::min(ad->min_samples, p->spp);
        R.interval = (uint32_t)ad->check_interval;
        R.threshold = ad->threshold;
        const uint64_t dark = std::max<uint64_t>(256u, (uint64_t)R.min_samples + 3ull * R.interval);
        R.dark_min = (uint32_t)std::min<uint64_t>(R.max_samples, std::max<uint64_t>(R.min_samples, dark));
    } else {
        R.min_samples = R.max_samples;
        R.interval = 1;
        R.dark_min = R.max_samples;
    }
    const std::vector<uint32_t> ends = round_ends(R);
    const bool want_nfor = nfor != nullptr || denoised_out != nullptr;

    DeviceScratch D;
    PixAcc* acc = D.get<PixAcc>(npix, st);
    PixNfor* nf = want_nfor ? D.get<PixNfor>(npix, st) : nullptr;
    NforOut nout{};
    if (want_nfor) {
        nout.color_a = D.get<double>(3 * npix, st);
        nout.color_b = D.get<double>(3 * npix, st);
        nout.color_variance = D.get<double>(npix, st);
        nout.features_a = D.get<double>(LUZ_NFOR_FEATURES * npix, st);
        nout.features_b = D.get<double>(LUZ_NFOR_FEATURES * npix, st);
        nout.feature_variance = D.get<double>(LUZ_NFOR_FEATURES * npix, st);
    }
    uint32_t* act[2] = {D.get<uint32_t>(npix, st), D.get<uint32_t>(npix, st)};
    uint32_t* act_count = D.get<uint32_t>(2, st);
    float* d_rgb = D.get<float>(3 * npix, st);
    int32_t* d_used = D.get<int32_t>(npix, st);
    const int64_t n_start = pixels ? pixel_count : npix;
    {
        std::vector<uint32_t> all((std::size_t)n_start);
        if (pixels) {
            std::vector<char> seen((std::size_t)npix, 0);
            for (int64_t i = 0; i < pixel_count; i++) {
                if (pixels[i] < 0 || pixels[i] >= npix || seen[(std::size_t)pixels[i]])
                    throw Status(LUZ_E_INVALID, "Pixel list entries must be distinct and inside the image.");
                seen[(std::size_t)pixels[i]] = 1;
                all[(std::size_t)i] = (uint32_t)pixels[i];
            }
        } else {
            for (int64_t i = 0; i < npix; i++) all[(std::size_t)i] = (uint32_t)i;
        }
        if (n_start > 0)
            CK(cudaMemcpyAsync(act[0], all.data(), sizeof(uint32_t) * (std::size_t)n_start, cudaMemcpyHostToDevice,
                               st));
        CK(cudaStreamSynchronize(st));
    }

    WaveArgs w = base_args(s, p);
    w.half_streams = want_nfor ? 1 : 0;
    w.nfor = want_nfor ? 1 : 0;
    uint32_t max_round = 0, prev = 0;
    for (uint32_t e : ends) {
        max_round = std::max(max_round, e - prev);
        prev = e;
    }
    const int64_t n_wave =
        s->reserve_paths(std::min<int64_t>(kWaveTarget, npix * (int64_t)std::max<uint32_t>(1u, max_round)), want_nfor);
    const int s_wave = (int)std::min<int64_t>(max_round, n_wave);
    CK(cudaMemsetAsync(s->totals, 0, 2 * sizeof(unsigned long long), st));
    CK(cudaEventRecord(s->ev0, st));

    StageTimer T;
    int64_t launches = 0, waves = 0;
    double samples = 0.0;
    uint32_t n_act = (uint32_t)n_start, done_to = 0;
    int cur = 0;
    for (uint32_t e : ends) {
        if (n_act == 0) break;
        const int round = (int)(e - done_to);
        const int sc_max = std::min(round, s_wave);
        const int64_t pix_wave = std::max<int64_t>(1, std::min<int64_t>(n_act, n_wave / sc_max));
        w.pix_list = act[cur];
        for (int sb = 0; sb < round; sb += sc_max) {          // sample chunks in order: sums stay sequential
            const int sc = std::min(sc_max, round - sb);
            for (int64_t pb = 0; pb < n_act; pb += pix_wave) {
                const int64_t pc = std::min<int64_t>(pix_wave, n_act - pb);
                w.pix_begin = (int32_t)pb;
                w.pix_count = (int32_t)pc;
                w.s_begin = (int32_t)done_to + sb;
                w.s_count = sc;
                w.n = pc * sc;
                w.list_mode = 0;
                CK(cudaMemsetAsync(s->ctrl, 0, sizeof(Ctrl), st));
                k_raygen<<<(unsigned)((w.n + kBlock - 1) / kBlock), kBlock, 0, st>>>(w, s->pb, s->ctrl);
                launch_bounces(s, w, st, launches, T, nullptr, s->pb, s->ctrl);
                k_accumulate_px<<<(unsigned)((pc + 127) / 128), 128, 0, st>>>(w, s->pb, acc, nf);
                k_tally<<<1, 1, 0, st>>>(s->ctrl, w.max_bounces, s->totals);
                launches += 3;
                waves++;
            }
        }
        samples += (double)n_act * round;
        CK(cudaMemsetAsync(act_count, 0, sizeof(uint32_t), st));
        k_converge<<<(unsigned)((n_act + 127) / 128), 128, 0, st>>>(R, e, act[cur], n_act, act[cur ^ 1], act_count, acc,
                                                                  nf, nout, d_rgb, d_used);
        launches++;
        CK(cudaMemcpyAsync(&n_act, act_count, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        cur ^= 1;
        done_to = e;
    }
    if (n_act != 0) throw Status(LUZ_E_DEVICE, "Adaptive sampling left pixels unfinished.");
    CK(cudaEventRecord(s->ev1, st));
    CK(cudaEventSynchronize(s->ev1));
    CK(cudaGetLastError());
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, s->ev0, s->ev1));
    unsigned long long tot[2] = {0, 0};
    finish_status(s, st, s->totals, tot);
    if (pixels) {
        std::vector<float> full((std::size_t)(3 * npix));
        CK(cudaMemcpy(full.data(), d_rgb, sizeof(float) * full.size(), cudaMemcpyDeviceToHost));
        for (int64_t i = 0; i < pixel_count; i++)
            for (int k = 0; k < 3; k++) rgb_out[3 * i + k] = full[(std::size_t)(3 * (int64_t)pixels[i] + k)];
    } else {
        CK(cudaMemcpy(rgb_out, d_rgb, sizeof(float) * 3 * (std::size_t)npix, cudaMemcpyDeviceToHost));
    }
    if (samples_out) CK(cudaMemcpy(samples_out, d_used, sizeof(int32_t) * (std::size_t)npix, cudaMemcpyDeviceToHost));
    if (nfor) {
        auto down = [&](double* host, const double* dev, int64_t n) {
            if (host) CK(cudaMemcpy(host, dev, sizeof(double) * (std::size_t)n, cudaMemcpyDeviceToHost));
        };
        down(nfor->color_a, nout.color_a, 3 * npix);
        down(nfor->color_b, nout.color_b, 3 * npix);
        down(nfor->color_variance, nout.color_variance, npix);
        down(nfor->features_a, nout.features_a, LUZ_NFOR_FEATURES * npix);
        down(nfor->features_b, nout.features_b, LUZ_NFOR_FEATURES * npix);
        down(nfor->feature_variance, nout.feature_variance, LUZ_NFOR_FEATURES * npix);
    }
    float denoise_ms = 0.f;
    if (denoised_out) {
        // Denoise::applyNFOR on the device-resident buffers (Threads.cpp:514-536)
        double* d_den = D.get<double>(3 * npix, st);
        std::string msg;
        CK(cudaEventRecord(s->ev0, st));
        const int rc = luz_nfor_on_device(nout.color_a, nout.color_b, nout.color_variance, nout.features_a,
                                          nout.features_b, nout.feature_variance, p->width, p->height, denoise, d_den,
                                          (void*)st, msg);
        if (rc != LUZ_OK) throw Status(rc, msg);
        CK(cudaEventRecord(s->ev1, st));
        CK(cudaEventSynchronize(s->ev1));
        CK(cudaEventElapsedTime(&denoise_ms, s->ev0, s->ev1));
        CK(cudaMemcpy(denoised_out, d_den, sizeof(double) * 3 * (std::size_t)npix, cudaMemcpyDeviceToHost));
    }
    if (stats) {
        *stats = LuzRenderStats{};
        stats->render_ms = ms;
        stats->denoise_ms = denoise_ms;
        caustic_stats(s, stats);
        stats->samples = samples;
        stats->extension_rays = (double)tot[0];
        stats->shadow_rays = (double)tot[1];
        stats->kernel_launches = launches;
        stats->waves = waves;
        stats->extend_launches = waves * (p->max_bounces + 1);
        stats->shadow_launches = waves * (p->max_bounces + 1);
    }
    return LUZ_OK;
}

// Replaces the texels of one texture on the device (same size).
void set_texture(luz_gpu_scene* s, int32_t texture, const double* rgb)
{
    const ScenePack& P = *s->pack;
    if (texture < 0 || (std::size_t)texture >= P.textures.size()) throw Status(LUZ_E_INVALID, "Texture index out of range.");
    if (!rgb) throw Status(LUZ_E_INVALID, "NULL argument.");
    const GTexture& T = P.textures[(std::size_t)texture];
    const int64_t n = (int64_t)T.width * T.height;
    std::vector<float4> tx((std::size_t)n);
    for (int64_t k = 0; k < n; k++)
        tx[(std::size_t)k] = make_float4((float)rgb[3 * k], (float)rgb[3 * k + 1], (float)rgb[3 * k + 2], 0.f);
    CK(cudaSetDevice(s->device));
    CK(cudaMemcpy(const_cast<float4*>(s->ds.texels) + T.offset, tx.data(), sizeof(float4) * (std::size_t)n,
                  cudaMemcpyHostToDevice));
    s->version++;
    if (s->cm.valid) {   // photon throughput may depend on the texels: rebuild on the next render
        s->cm.valid = false;
        s->ds.cm = DCaustics{};
        CK(cudaMemcpy(s->dds, &s->ds, sizeof(DScene), cudaMemcpyHostToDevice));
    }
}

int do_adjoint_backward(luz_gpu_scene* s, const LuzRenderParams* p, int32_t texture, const float* adj_rgb,
                        double* grad_out, LuzRenderStats* stats)
{
    check_params(p);
    if (p->flags) throw Status(LUZ_E_UNSUPPORTED, "Render flags are not supported in the adjoint pass.");
    if (s->pack->consts.caustics.enabled)
        throw Status(LUZ_E_UNSUPPORTED, "The adjoint pass does not differentiate caustic photon maps.");
    const ScenePack& PK = *s->pack;
    if (texture < 0 || (std::size_t)texture >= PK.textures.size()) throw Status(LUZ_E_INVALID, "Texture index out of range.");
    bool albedo = false, rough = false;
    for (const GMaterial& m : PK.materials) {
        if (m.texture == texture) {
            if (m.type != MT_LAMBERTIAN)
                throw Status(LUZ_E_UNSUPPORTED,
                             "Texture gradients are defined for Lambertian albedo and Metal roughness textures only.");
            albedo = true;
        }
        if (m.rtexture == texture) rough = true;
    }
    if (albedo && rough)
        throw Status(LUZ_E_UNSUPPORTED, "A texture differentiated as both albedo and roughness is not supported.");
    CK(cudaSetDevice(s->device));
    const cudaStream_t st = s->stream;
    clear_error(s, st);
    const GTexture& T = PK.textures[(std::size_t)texture];
    const int64_t npix = (int64_t)p->width * p->height, ntex = (int64_t)T.width * T.height;
    DeviceScratch D;
    float* d_adj = D.get<float>(3 * npix, st);
    double* d_grad = D.get<double>(3 * ntex, st);
    CK(cudaMemcpyAsync(d_adj, adj_rgb, sizeof(float) * 3 * (std::size_t)npix, cudaMemcpyHostToDevice, st));
    WaveArgs w = base_args(s, p);
    w.grad_texture = texture;
    w.grad_kind = rough ? 1 : 0;
    w.grad_emission = 0;
    w.grad_volume = -1;
    w.adj_rgb = d_adj;
    w.grad = d_grad;
    w.inv_spp = 1.0 / (double)p->spp;
    const int64_t n_wave = s->reserve_paths(std::min<int64_t>(kWaveTarget, npix * (int64_t)p->spp));
    const int s_wave = (int)std::min<int64_t>(p->spp, n_wave);
    const int64_t pix_wave = std::max<int64_t>(1, std::min<int64_t>(npix, n_wave / s_wave));
    w.adj_rough = rough ? D.get<AdjRough>(pix_wave * s_wave, st) : nullptr;
    CK(cudaMemcpyAsync(s->dds, &s->ds, sizeof(DScene), cudaMemcpyHostToDevice, st));
    CK(cudaEventRecord(s->ev0, st));
    StageTimer T0;
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
            const unsigned grid = (unsigned)((w.n + kBlock - 1) / kBlock);
            for (int pass = 0; pass < 2; pass++) {   // 0: radiance of every path; 1: replay with gradients
                w.adjoint = pass;
                CK(cudaMemsetAsync(s->ctrl, 0, sizeof(Ctrl), st));
                if (pass == 1 && rough) CK(cudaMemsetAsync(w.adj_rough, 0, sizeof(AdjRough) * (std::size_t)w.n, st));
                k_raygen<<<grid, kBlock, 0, st>>>(w, s->pb, s->ctrl);
                launch_bounces(s, w, st, launches, T0, shade_kernel(3), s->pb, s->ctrl);
                launches++;
                if (pass == 0) {
                    k_path_color<<<grid, kBlock, 0, st>>>(w, s->pb);
                    launches++;
                } else if (rough) {
                    k_adjoint_rough_finish<<<grid, kBlock, 0, st>>>(s->ds, w, s->pb);
                    launches++;
                }
            }
            waves++;
        }
    }
    CK(cudaGetLastError());
    CK(cudaEventRecord(s->ev1, st));
    CK(cudaEventSynchronize(s->ev1));
    finish_status(s, st);
    CK(cudaMemcpy(grad_out, d_grad, sizeof(double) * 3 * (std::size_t)ntex, cudaMemcpyDeviceToHost));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, s->ev0, s->ev1));
    if (stats) {
        *stats = LuzRenderStats{};
        stats->render_ms = ms;
        stats->samples = (double)npix * p->spp;
        stats->kernel_launches = launches;
        stats->waves = waves;
    }
    return LUZ_OK;
}

// dLoss/d(emitted radiance) of every light by path replay: emitter hits and light
// samples add adj * contribution / E (both linear in E); light selection held fixed.
int do_adjoint_emission(luz_gpu_scene* s, const LuzRenderParams* p, const float* adj_rgb, double* grad_out,
                        LuzRenderStats* stats)
{
    check_params(p);
    if (p->flags) throw Status(LUZ_E_UNSUPPORTED, "Render flags are not supported in the adjoint pass.");
    if (s->pack->consts.caustics.enabled)
        throw Status(LUZ_E_UNSUPPORTED, "The adjoint pass does not differentiate caustic photon maps.");
    const int64_t nl = s->pack->consts.light_count;
    CK(cudaSetDevice(s->device));
    const cudaStream_t st = s->stream;
    clear_error(s, st);
    const int64_t npix = (int64_t)p->width * p->height;
    DeviceScratch D;
    float* d_adj = D.get<float>(3 * npix, st);
    double* d_grad = D.get<double>(kEmissionReplicas * 3 * std::max<int64_t>(nl, 1), st);
    CK(cudaMemcpyAsync(d_adj, adj_rgb, sizeof(float) * 3 * (std::size_t)npix, cudaMemcpyHostToDevice, st));
    WaveArgs w = base_args(s, p);
    w.grad_texture = -1;
    w.grad_kind = 2;   // no texture hook
    w.grad_emission = 1;
    w.grad_volume = -1;
    w.grad_light = d_grad;
    w.adj_rgb = d_adj;
    w.inv_spp = 1.0 / (double)p->spp;
    const int64_t n_wave = s->reserve_paths(std::min<int64_t>(kWaveTarget, npix * (int64_t)p->spp));
    const int s_wave = (int)std::min<int64_t>(p->spp, n_wave);
    const int64_t pix_wave = std::max<int64_t>(1, std::min<int64_t>(npix, n_wave / s_wave));
    w.pend_light = D.get<int32_t>(pix_wave * s_wave, st);
    CK(cudaMemcpyAsync(s->dds, &s->ds, sizeof(DScene), cudaMemcpyHostToDevice, st));
    CK(cudaEventRecord(s->ev0, st));
    StageTimer T0;
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
            const unsigned grid = (unsigned)((w.n + kBlock - 1) / kBlock);
            w.adjoint = 1;   // one replay: the contributions themselves carry the gradient
            CK(cudaMemsetAsync(s->ctrl, 0, sizeof(Ctrl), st));
            CK(cudaMemsetAsync(w.pend_light, 0xff, sizeof(int32_t) * (std::size_t)w.n, st));
            k_raygen<<<grid, kBlock, 0, st>>>(w, s->pb, s->ctrl);
            launch_bounces(s, w, st, launches, T0, shade_kernel(3), s->pb, s->ctrl);
            k_adjoint_emission_finish<<<grid, kBlock, 0, st>>>(s->ds, w, s->pb);
            launches += 2;
            waves++;
        }
    }
    CK(cudaGetLastError());
    CK(cudaEventRecord(s->ev1, st));
    CK(cudaEventSynchronize(s->ev1));
    finish_status(s, st);
    if (nl > 0) {
        std::vector<double> rep((std::size_t)(kEmissionReplicas * 3 * nl));
        CK(cudaMemcpy(rep.data(), d_grad, sizeof(double) * rep.size(), cudaMemcpyDeviceToHost));
        for (int64_t i = 0; i < 3 * nl; i++) {
            double acc = 0.0;
            for (int r = 0; r < kEmissionReplicas; r++) acc += rep[(std::size_t)(r * 3 * nl + i)];
            grad_out[i] = acc;
        }
    }
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, s->ev0, s->ev1));
    if (stats) {
        *stats = LuzRenderStats{};
        stats->render_ms = ms;
        stats->samples = (double)npix * p->spp;
        stats->kernel_launches = launches;
        stats->waves = waves;
    }
    return LUZ_OK;
}

// dLoss/d(density) of one volume by a score-function replay (density_score).
int do_adjoint_density(luz_gpu_scene* s, const LuzRenderParams* p, int32_t object, const float* adj_rgb,
                       double* grad_out, LuzRenderStats* stats)
{
    check_params(p);
    if (p->flags) throw Status(LUZ_E_UNSUPPORTED, "Render flags are not supported in the adjoint pass.");
    if (s->pack->consts.caustics.enabled)
        throw Status(LUZ_E_UNSUPPORTED, "The adjoint pass does not differentiate caustic photon maps.");
    const ScenePack& PK = *s->pack;
    if (object < 0 || (std::size_t)object >= PK.object_of_desc.size() || PK.object_of_desc[(std::size_t)object] < 0)
        throw Status(LUZ_E_INVALID, "Object index out of range.");
    const int32_t gi = PK.object_of_desc[(std::size_t)object];
    if (PK.objects[(std::size_t)gi].kind != OK_VOLUME) throw Status(LUZ_E_INVALID, "The object is not a volume.");
    CK(cudaSetDevice(s->device));
    const cudaStream_t st = s->stream;
    clear_error(s, st);
    const int64_t npix = (int64_t)p->width * p->height;
    DeviceScratch D;
    float* d_adj = D.get<float>(3 * npix, st);
    double* d_grad = D.get<double>(kEmissionReplicas, st);
    CK(cudaMemcpyAsync(d_adj, adj_rgb, sizeof(float) * 3 * (std::size_t)npix, cudaMemcpyHostToDevice, st));
    WaveArgs w = base_args(s, p);
    w.grad_texture = -1;
    w.grad_kind = 2;
    w.grad_emission = 0;
    w.grad_volume = gi;
    w.grad_density = d_grad;
    w.adj_rgb = d_adj;
    w.inv_spp = 1.0 / (double)p->spp;
    const int64_t n_wave = s->reserve_paths(std::min<int64_t>(kWaveTarget, npix * (int64_t)p->spp));
    const int s_wave = (int)std::min<int64_t>(p->spp, n_wave);
    const int64_t pix_wave = std::max<int64_t>(1, std::min<int64_t>(npix, n_wave / s_wave));
    w.dens_score = D.get<float2>(pix_wave * s_wave, st);
    CK(cudaMemcpyAsync(s->dds, &s->ds, sizeof(DScene), cudaMemcpyHostToDevice, st));
    CK(cudaEventRecord(s->ev0, st));
    StageTimer T0;
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
            const unsigned grid = (unsigned)((w.n + kBlock - 1) / kBlock);
            w.adjoint = 1;
            CK(cudaMemsetAsync(s->ctrl, 0, sizeof(Ctrl), st));
            CK(cudaMemsetAsync(w.dens_score, 0, sizeof(float2) * (std::size_t)w.n, st));
            k_raygen<<<grid, kBlock, 0, st>>>(w, s->pb, s->ctrl);
            launch_bounces(s, w, st, launches, T0, shade_kernel(3), s->pb, s->ctrl);
            k_adjoint_density_finish<<<grid, kBlock, 0, st>>>(s->ds, w, s->pb);
            launches += 2;
            waves++;
        }
    }
    CK(cudaGetLastError());
    CK(cudaEventRecord(s->ev1, st));
    CK(cudaEventSynchronize(s->ev1));
    finish_status(s, st);
    std::vector<double> rep(kEmissionReplicas);
    CK(cudaMemcpy(rep.data(), d_grad, sizeof(double) * rep.size(), cudaMemcpyDeviceToHost));
    double acc = 0.0;
    for (double v : rep) acc += v;
    *grad_out = acc;
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, s->ev0, s->ev1));
    if (stats) {
        *stats = LuzRenderStats{};
        stats->render_ms = ms;
        stats->samples = (double)npix * p->spp;
        stats->kernel_launches = launches;
        stats->waves = waves;
    }
    return LUZ_OK;
}

// ---------------------------------------------------------------------------- multi-scene batches
//
// One batch context per device holds the geometry arena (a copy of every scene's
// arrays in one allocation, reused while the same scene contents come back), the
// table of DScene records pointing into it, the shared path state, the segment
// tables and the CUDA graph of one wave. A wave is recorded once per batch call
// (raygen, every bounce's extend / shade / shadow, accumulate) and replayed for
// every wave with that wave's segment table copied to a fixed device address.

constexpr int64_t kBatchWaveDefault = int64_t(1) << 24;
constexpr int kBatchMaxSegments = 4096;   // segments per wave (scenes split across waves)

struct BatchContext {
    std::mutex mu;
    int device = -1;
    cudaStream_t st = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    unsigned char* arena = nullptr;
    std::size_t arena_bytes = 0;
    std::vector<uint64_t> arena_key;         // (uid, version) of the scenes in the arena, in order
    DScene* d_scenes = nullptr;
    std::vector<DScene> h_scenes;
    int64_t cap = 0;
    PathBuf pb{};
    std::vector<void*> pallocs;
    Ctrl* ctrl = nullptr;
    WaveArgs* d_segs = nullptr;              // kBatchMaxSegments entries
    WaveArgs* h_segs = nullptr;              // pinned, one region per wave of the call
    int64_t h_seg_cap = 0;
    std::map<std::vector<uint64_t>, int64_t> tuned_wave;   // autotuned wave size per scene set
    LuzBatchReport last_report{};
    ~BatchContext()
    {
        if (device < 0) return;
        cudaSetDevice(device);
        for (void* p : pallocs) cudaFree(p);
        if (arena) cudaFree(arena);
        if (d_scenes) cudaFree(d_scenes);
        if (ctrl) cudaFree(ctrl);
        if (d_segs) cudaFree(d_segs);
        if (h_segs) cudaFreeHost(h_segs);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (st) cudaStreamDestroy(st);
    }
    void ensure_paths(int64_t n)
    {
        if (n <= cap) return;
        for (void* p : pallocs) cudaFree(p);
        pallocs.clear();
        cap = 0;
        auto get = [&](std::size_t bytes) {
            void* p = dalloc<uint8_t>(bytes);
            pallocs.push_back(p);
            return p;
        };
        pb = PathBuf{};
        pb.ray_o = static_cast<float4*>(get(16 * n));
        pb.ray_d = static_cast<float4*>(get(16 * n));
        pb.thr = static_cast<float4*>(get(16 * n));
        pb.rad = static_cast<float4*>(get(16 * n));
        pb.pend0 = static_cast<float4*>(get(16 * n));
        pb.pend1 = static_cast<float4*>(get(16 * n));
        pb.pixel = static_cast<uint32_t*>(get(4 * n));
        pb.sample = static_cast<uint32_t*>(get(4 * n));
        pb.hit = static_cast<float4*>(get(16 * n));
        pb.hit_prim = static_cast<int32_t*>(get(4 * n));
        pb.queue0 = static_cast<uint32_t*>(get(4 * n));
        pb.queue1 = static_cast<uint32_t*>(get(4 * n));
        pb.sh_o = static_cast<float4*>(get(32 * n));
        pb.sh_d = static_cast<float4*>(get(32 * n));
        pb.sh_x = static_cast<int2*>(get(16 * n));
        pb.bins = static_cast<uint32_t*>(get(4 * kShadeClasses * n));
        pb.bin_stride = (uint32_t)n;
        pb.seg = static_cast<uint32_t*>(get(4 * n));
        cap = n;
    }
};

BatchContext& batch_context(int device)
{
    static std::mutex mu;
    static std::vector<std::unique_ptr<BatchContext>> ctx;
    std::lock_guard<std::mutex> lock(mu);
    if ((int)ctx.size() <= device) ctx.resize(device + 1);
    if (!ctx[device]) {
        ctx[device] = std::make_unique<BatchContext>();
        BatchContext& c = *ctx[device];
        CK(cudaSetDevice(device));
        CK(cudaStreamCreateWithFlags(&c.st, cudaStreamNonBlocking));
        CK(cudaEventCreate(&c.ev0));
        CK(cudaEventCreate(&c.ev1));
        c.ctrl = dalloc<Ctrl>(1);
        c.d_segs = dalloc<WaveArgs>(kBatchMaxSegments);
        c.device = device;
    }
    return *ctx[device];
}

// The geometry arena for these scenes (rebuilt when the set or a scene's content changed).
void batch_arena(BatchContext& C, luz_gpu_scene* const* scenes, int32_t count)
{
    std::vector<uint64_t> key;
    for (int32_t i = 0; i < count; i++) {
        key.push_back(scenes[i]->uid);
        key.push_back(scenes[i]->version);
    }
    if (key == C.arena_key && C.arena) return;
    struct Copy {
        const void* src;
        std::size_t off, bytes;
    };
    std::vector<Copy> copies;
    std::vector<DScene> hs((std::size_t)count);
    std::size_t total = 0;
    auto place = [&](const void* src, std::size_t bytes) {
        const std::size_t off = total;
        total += (std::max<std::size_t>(bytes, 16) + 255) & ~std::size_t(255);
        if (src && bytes) copies.push_back(Copy{src, off, bytes});
        return off;
    };
    std::vector<std::vector<std::pair<std::size_t, std::size_t>>> offs((std::size_t)count);   // (field, arena offset)
    std::vector<std::size_t> err_off((std::size_t)count), cm_off((std::size_t)count * 3);
    for (int32_t i = 0; i < count; i++) {
        const luz_gpu_scene* sc = scenes[i];
        for (const auto& f : sc->arena_fields) {
            const void* src = *reinterpret_cast<const void* const*>((const char*)&sc->ds + f.first);
            offs[(std::size_t)i].push_back({f.first, place(src, f.second)});
        }
        err_off[(std::size_t)i] = place(nullptr, sizeof(uint32_t));
        const DCaustics& cm = sc->ds.cm;
        cm_off[3 * i] = place(cm.photons, cm.count ? sizeof(float4) * 3 * (std::size_t)cm.count : 0);
        cm_off[3 * i + 1] = place(cm.cell_keys, cm.count ? sizeof(unsigned long long) * ((std::size_t)cm.mask + 1) : 0);
        cm_off[3 * i + 2] = place(cm.cell_ranges, cm.count ? sizeof(uint2) * ((std::size_t)cm.mask + 1) : 0);
    }
    if (C.arena) cudaFree(C.arena);
    C.arena = nullptr;
    C.arena_key.clear();
    C.arena = dalloc<unsigned char>(total);
    C.arena_bytes = total;
    CK(cudaMemsetAsync(C.arena, 0, total, C.st));
    for (const Copy& c : copies) CK(cudaMemcpyAsync(C.arena + c.off, c.src, c.bytes, cudaMemcpyDeviceToDevice, C.st));
    for (int32_t i = 0; i < count; i++) {
        DScene d = scenes[i]->ds;
        for (const auto& f : offs[(std::size_t)i])
            *reinterpret_cast<const void**>((char*)&d + f.first) = C.arena + f.second;
        d.error = reinterpret_cast<uint32_t*>(C.arena + err_off[(std::size_t)i]);
        d.counters = nullptr;
        if (d.cm.count) {
            d.cm.photons = reinterpret_cast<const float4*>(C.arena + cm_off[3 * i]);
            d.cm.cell_keys = reinterpret_cast<const unsigned long long*>(C.arena + cm_off[3 * i + 1]);
            d.cm.cell_ranges = reinterpret_cast<const uint2*>(C.arena + cm_off[3 * i + 2]);
        }
        hs[(std::size_t)i] = d;
    }
    if ((int)C.h_scenes.size() < count || !C.d_scenes) {
        if (C.d_scenes) cudaFree(C.d_scenes);
        C.d_scenes = nullptr;
        C.d_scenes = dalloc<DScene>((std::size_t)count);
    }
    C.h_scenes = hs;
    CK(cudaMemcpyAsync(C.d_scenes, hs.data(), sizeof(DScene) * (std::size_t)count, cudaMemcpyHostToDevice, C.st));
    CK(cudaStreamSynchronize(C.st));
    C.arena_key = key;
}

// Pixel runs of every scene packed into waves of at most `cap` paths; a run always takes
// every sample of its pixels, so each pixel's FP64 sum is the same sequence as in a
// single render (films equal bit for bit).
std::vector<std::vector<WaveArgs>> batch_waves(luz_gpu_scene* const* scenes, const LuzRenderParams* params, int32_t count,
                                               int64_t cap)
{
    std::vector<std::vector<WaveArgs>> waves(1);
    int64_t used = 0;
    for (int32_t i = 0; i < count; i++) {
        const LuzRenderParams& p = params[i];
        const int64_t npix = (int64_t)p.width * p.height;
        const int64_t spp = p.spp;
        if (spp > cap) throw Status(LUZ_E_LIMIT, "A batched scene's sample count exceeds the wave size.");
        for (int64_t pb = 0; pb < npix;) {
            int64_t fit = (cap - used) / spp;
            if (fit <= 0 || (int64_t)waves.back().size() >= kBatchMaxSegments) {
                waves.emplace_back();
                used = 0;
                continue;
            }
            const int64_t pc = std::min(fit, npix - pb);
            WaveArgs w = base_args(scenes[i], &p);
            w.pix_begin = (int32_t)pb;
            w.pix_count = (int32_t)pc;
            w.s_begin = 0;
            w.s_count = (int32_t)spp;
            w.n = pc * spp;
            w.list_mode = 0;
            w.batch_scene = i;
            w.batch_offset = used;
            waves.back().push_back(w);
            used += pc * spp;
            pb += pc;
        }
    }
    if (waves.back().empty()) waves.pop_back();
    return waves;
}

// Records the launches of one wave (the segment table at C.d_segs, its header at hdr)
// into a graph: every kernel reads the wave's size from device memory.
cudaGraphExec_t batch_graph(BatchContext& C, const BatchWaveHeader* hdr, int max_b, int64_t cap_paths,
                            int64_t max_pix, int64_t max_segs, double* const* d_films, unsigned long long* d_rays,
                            int32_t count, bool caustics, int sms, int occ_ext, int occ_sh, int occ_shade,
                            int64_t& launches)
{
    (void)hdr;
    (void)count;
    const BatchShadeKernel shade = batch_shade_kernel(caustics ? 1 : 0);
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(C.st, cudaStreamCaptureModeThreadLocal));
    try {
        CK(cudaMemsetAsync(C.ctrl, 0, sizeof(Ctrl), C.st));
        k_raygen_batch<<<(unsigned)((cap_paths + kBlock - 1) / kBlock), kBlock, 0, C.st>>>(C.d_segs, hdr, C.pb, C.ctrl);
        launches++;
        for (int b = 0; b <= max_b; b++) {
            k_extend_batch<<<sms * occ_ext, kBlock, 0, C.st>>>(C.d_scenes, C.d_segs, C.pb, C.ctrl, b, d_rays);
            shade<<<sms * occ_shade, kBlock, 0, C.st>>>(C.d_scenes, C.d_segs, C.pb, C.ctrl, b);
            k_shadow_batch<<<sms * occ_sh, kBlock, 0, C.st>>>(C.d_scenes, C.d_segs, C.pb, C.ctrl, b, d_rays + count);
            launches += 3;
        }
        dim3 ag((unsigned)((max_pix + 127) / 128), (unsigned)max_segs);
        k_accumulate_batch<<<ag, 128, 0, C.st>>>(C.d_segs, hdr, C.pb, d_films);
        launches++;
        CK(cudaGetLastError());
    } catch (...) {
        cudaStreamEndCapture(C.st, &g);
        if (g) cudaGraphDestroy(g);
        throw;
    }
    CK(cudaStreamEndCapture(C.st, &g));
    cudaGraphExec_t ex = nullptr;
    const cudaError_t e = cudaGraphInstantiate(&ex, g, 0);
    cudaGraphDestroy(g);
    CK(e);
    return ex;
}

int batch_render(luz_gpu_scene* const* scenes, const LuzRenderParams* params, int32_t count, float* const* rgb_out,
                 LuzRenderStats* stats, LuzBatchReport* report)
{
    const int device = scenes[0]->device;
    BatchContext& C = batch_context(device);
    std::lock_guard<std::mutex> lock(C.mu);
    CK(cudaSetDevice(device));
    bool caustics = false;
    int max_b = 0;
    int64_t max_pix = 0, max_spp = 0;
    for (int32_t i = 0; i < count; i++) {   // photon maps are built per scene before the arena copy
        clear_error(scenes[i], scenes[i]->stream);
        prepare_caustics(scenes[i], &params[i], scenes[i]->stream);
        CK(cudaStreamSynchronize(scenes[i]->stream));
        caustics |= scenes[i]->pack->consts.caustics.enabled != 0;
        max_b = std::max(max_b, params[i].max_bounces);
        max_pix = std::max<int64_t>(max_pix, (int64_t)params[i].width * params[i].height);
        max_spp = std::max<int64_t>(max_spp, params[i].spp);
    }
    batch_arena(C, scenes, count);
    const cudaStream_t st = C.st;
    // wave size: the autotuned choice for this scene set, else the default
    std::vector<uint64_t> key;
    for (int32_t i = 0; i < count; i++) {
        key.push_back(scenes[i]->uid);
        key.push_back((uint64_t)params[i].width << 40 ^ (uint64_t)params[i].height << 20 ^ (uint64_t)params[i].spp);
    }
    const auto it = C.tuned_wave.find(key);
    int64_t cap = it != C.tuned_wave.end() ? it->second : kBatchWaveDefault;
    cap = std::max<int64_t>(cap, max_spp);
    // per-scene FP64 films and device output films, ray counters, the wave header
    std::vector<int64_t> film_off((std::size_t)count), out_off((std::size_t)count);
    int64_t film_doubles = 0, out_floats = 0;
    for (int32_t i = 0; i < count; i++) {
        const int64_t npix = (int64_t)params[i].width * params[i].height;
        film_off[(std::size_t)i] = film_doubles;
        out_off[(std::size_t)i] = out_floats;
        film_doubles += 3 * npix;
        out_floats += 3 * npix;
    }
    DeviceScratch D;
    double* films = D.get<double>(film_doubles, st);
    float* outs = D.get<float>(out_floats, st);
    double** d_films = D.get<double*>(count, st);
    unsigned long long* d_rays = D.get<unsigned long long>(2 * (int64_t)count, st);
    BatchWaveHeader* hdr = D.get<BatchWaveHeader>(1, st);
    {
        std::vector<double*> hf((std::size_t)count);
        for (int32_t i = 0; i < count; i++) hf[(std::size_t)i] = films + film_off[(std::size_t)i];
        CK(cudaMemcpyAsync(d_films, hf.data(), sizeof(double*) * (std::size_t)count, cudaMemcpyHostToDevice, st));
        CK(cudaStreamSynchronize(st));
    }
    int occ_ext = 1, occ_sh = 1, occ_shade = 1;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_ext, k_extend_batch, kBlock, 0));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_sh, k_shadow_batch, kBlock, 0));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_shade, batch_shade_kernel(caustics ? 1 : 0), kBlock, 0));
    occ_ext = std::max(1, occ_ext);
    occ_sh = std::max(1, occ_sh);
    occ_shade = std::max(1, occ_shade);
    const int sms = scenes[0]->sms;

    // autotuner: on the first call for a scene set, time one wave at each candidate size
    // (the first wave's pixels, every candidate processing the same work) and keep the
    // fastest paths per millisecond; the trial waves' films are discarded
    std::vector<LuzBatchTrial> trials;
    auto run = [&](int64_t wave_cap, bool first_only, int64_t& launches, int64_t& nwaves, float& ms) {
        const auto waves = batch_waves(scenes, params, count, wave_cap);
        int64_t total_segs = 0;
        for (const auto& wv : waves) total_segs += (int64_t)wv.size();
        if (total_segs > C.h_seg_cap) {
            if (C.h_segs) cudaFreeHost(C.h_segs);
            C.h_segs = nullptr;
            C.h_seg_cap = 0;
            CK(cudaMallocHost(&C.h_segs, sizeof(WaveArgs) * (std::size_t)total_segs));
            C.h_seg_cap = total_segs;
        }
        int64_t wave_max = 0;
        for (const auto& wv : waves) {
            int64_t n = 0;
            for (const WaveArgs& w : wv) n += w.n;
            wave_max = std::max(wave_max, n);
        }
        C.ensure_paths(wave_max);
        int64_t pix_max = 0, segs_max = 0;
        for (const auto& wv : waves) {
            segs_max = std::max<int64_t>(segs_max, (int64_t)wv.size());
            for (const WaveArgs& w : wv) pix_max = std::max<int64_t>(pix_max, w.pix_count);
        }
        cudaGraphExec_t ex = batch_graph(C, hdr, max_b, wave_max, pix_max, segs_max, d_films, d_rays, count, caustics,
                                         sms, occ_ext, occ_sh, occ_shade, launches);
        CK(cudaMemsetAsync(films, 0, sizeof(double) * (std::size_t)film_doubles, st));
        CK(cudaMemsetAsync(d_rays, 0, sizeof(unsigned long long) * 2 * (std::size_t)count, st));
        CK(cudaEventRecord(C.ev0, st));
        int64_t seg_at = 0;
        std::vector<BatchWaveHeader> hh(waves.size());
        for (std::size_t k = 0; k < waves.size(); k++) {
            const auto& wv = waves[k];
            std::memcpy(C.h_segs + seg_at, wv.data(), sizeof(WaveArgs) * wv.size());
            int64_t n = 0;
            for (const WaveArgs& w : wv) n += w.n;
            hh[k] = BatchWaveHeader{n, (uint32_t)wv.size(), 0u};
            CK(cudaMemcpyAsync(C.d_segs, C.h_segs + seg_at, sizeof(WaveArgs) * wv.size(), cudaMemcpyHostToDevice, st));
            CK(cudaMemcpyAsync(hdr, &hh[k], sizeof(BatchWaveHeader), cudaMemcpyHostToDevice, st));
            CK(cudaGraphLaunch(ex, st));
            seg_at += (int64_t)wv.size();
            nwaves++;
            if (first_only) break;
        }
        CK(cudaEventRecord(C.ev1, st));
        CK(cudaEventSynchronize(C.ev1));
        cudaGraphExecDestroy(ex);
        CK(cudaEventElapsedTime(&ms, C.ev0, C.ev1));
        return first_only ? hh[0].n : (int64_t)0;
    };
    if (it == C.tuned_wave.end()) {
        double best = -1.0;
        int64_t best_cap = cap;
        for (int64_t c : {int64_t(1) << 22, int64_t(1) << 24, int64_t(1) << 26}) {
            if (c < max_spp) continue;
            int64_t l = 0, nw = 0;
            float ms = 0.f;
            const int64_t n = run(c, true, l, nw, ms);
            const double rate = (double)n / std::max(1e-3, (double)ms);
            trials.push_back(LuzBatchTrial{c, (double)n, (double)ms});
            if (rate > best) {
                best = rate;
                best_cap = c;
            }
        }
        cap = best_cap;
        C.tuned_wave[key] = cap;
    }
    int64_t launches = 0, nwaves = 0;
    float ms = 0.f;
    run(cap, false, launches, nwaves, ms);
    // films: means per scene, each scene's error word, ray counts
    for (int32_t i = 0; i < count; i++) {
        const int64_t npix = (int64_t)params[i].width * params[i].height;
        k_resolve<<<(unsigned)((npix + 255) / 256), 256, 0, st>>>(films + film_off[(std::size_t)i], npix,
                                                                 (double)params[i].spp, outs + out_off[(std::size_t)i]);
        launches++;
    }
    CK(cudaGetLastError());
    for (int32_t i = 0; i < count; i++)
        CK(cudaMemcpyAsync(rgb_out[i], outs + out_off[(std::size_t)i],
                           sizeof(float) * 3 * (std::size_t)params[i].width * params[i].height, cudaMemcpyDeviceToHost,
                           st));
    std::vector<unsigned long long> rays(2 * (std::size_t)count);
    std::vector<uint32_t> errs((std::size_t)count);
    CK(cudaMemcpyAsync(rays.data(), d_rays, sizeof(unsigned long long) * rays.size(), cudaMemcpyDeviceToHost, st));
    for (int32_t i = 0; i < count; i++)
        CK(cudaMemcpyAsync(&errs[(std::size_t)i], C.h_scenes[(std::size_t)i].error, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                           st));
    CK(cudaStreamSynchronize(st));
    for (int32_t i = 0; i < count; i++)
        if (errs[(std::size_t)i])
            throw Status(LUZ_E_DEVICE, "Traversal stack overflow reported by the device (scene " + std::to_string(i) +
                                           ", flags " + std::to_string(errs[(std::size_t)i]) + ").");
    if (stats)
        for (int32_t i = 0; i < count; i++) {
            LuzRenderStats& o = stats[i];
            o = LuzRenderStats{};
            o.render_ms = ms;
            o.samples = (double)params[i].width * params[i].height * params[i].spp;
            o.extension_rays = (double)rays[(std::size_t)i];
            o.shadow_rays = (double)rays[(std::size_t)(count + i)];
            o.kernel_launches = launches;
            o.waves = nwaves;
            caustic_stats(scenes[i], &o);
        }
    LuzBatchReport r{};
    r.wave_paths = cap;
    r.waves = nwaves;
    r.render_ms = ms;
    r.kernel_launches = launches;
    r.trial_count = (int32_t)trials.size();
    for (std::size_t k = 0; k < trials.size() && k < 8; k++) r.trials[k] = trials[k];
    C.last_report = r;
    if (report) *report = r;
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
    P.feat = nullptr;
    P.bins = reinterpret_cast<uint32_t*>(take((std::size_t)kShadeClasses * n * sizeof(uint32_t)));
    P.bin_stride = (uint32_t)n;
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
    if (s->pack->consts.caustics.enabled && !(s->cm.valid && s->cm.seed == p->seed && s->cm.bounces == p->max_bounces))
        throw Status(LUZ_E_UNSUPPORTED, "luz_gpu_render_device_noalloc needs the caustic photon map of this seed and "
                                        "bounce limit built by an earlier render.");
    CK(cudaSetDevice(s->device));
    const StaticArena A = carve_static(static_scratch_address(s->device));
    const int64_t npix = (int64_t)p->width * p->height;
    if (npix > LUZ_STATIC_MAX_PIXELS || npix > A.film_pixels)
        throw Status(LUZ_E_LIMIT, "Image of " + std::to_string(npix) + " pixels exceeds the static film of " +
                                      std::to_string((long long)LUZ_STATIC_MAX_PIXELS) + " pixels.");
    clear_error(s, st);
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
                s->extend<<<g_ext, kBlock, 0, st>>>(s->ds, w, A.pb, A.ctrl, b);
                s->shade<<<g_shade, kBlock, 0, st>>>(s->dds, w, A.pb, A.ctrl, b);
                s->shadow<<<g_sh, kBlock, 0, st>>>(s->ds, w, A.pb, A.ctrl, b);
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
    finish_status(s, st, A.totals, tot);
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
        luz_gpu_scene* sp = s.get();
        auto field = [&](auto& dst, const auto& v) {
            using T = typename std::decay_t<decltype(v)>::value_type;
            dst = reinterpret_cast<std::decay_t<decltype(dst)>>(sp->up(v));
            sp->arena_fields.push_back({(std::size_t)((const char*)&dst - (const char*)&sp->ds), v.size() * sizeof(T)});
        };
        field(d.rects, P.rects);
        field(d.objects, P.objects);
        field(d.top_nodes, P.top_nodes);
        field(d.top_children, P.top_children);
        field(d.nodes4, P.nodes4);
        field(d.tris, P.tris);
        field(d.tri_shade, P.tri_shade);
        field(d.vnormals, P.vnormals);
        field(d.vuvs, P.vuvs);
        field(d.meshes, P.meshes);
        field(d.materials, P.materials);
        field(d.textures, P.textures);
        field(d.texels, P.texels);
        field(d.lights, P.lights);
        field(d.ies, P.ies);
        field(d.cdf, P.cdf);
        field(d.index_pool, P.index_pool);
        field(d.env_texels, P.env_texels);
        field(d.obj_class, P.obj_class);
        s->uid = next_scene_uid();
        uint32_t* err = dalloc<uint32_t>(1);
        CK(cudaMemset(err, 0, sizeof(uint32_t)));
        s->allocs.push_back(err);
        d.error = err;
        d.counters = nullptr;
        d.mesh_stack_limit = kMeshStack4;
        d.top_stack_limit = kTopStack;
        // the breadth-first top of the largest mesh's collapsed BVH, staged by the trace kernels
        d.top4_base = 0;
        d.top4_count = 0;
        int64_t best = -1;
        for (std::size_t m = 0; m < P.meshes.size(); m++) {
            const GMesh& M = P.meshes[m];
            if (M.node4_offset < 0 || (int64_t)M.tri_count <= best) continue;
            int64_t end = (int64_t)P.nodes4.size();
            for (const GMesh& o : P.meshes)
                if (o.node4_offset > M.node4_offset) end = std::min<int64_t>(end, o.node4_offset);
            best = M.tri_count;
            d.top4_base = (uint32_t)M.node4_offset;
            d.top4_count = (uint32_t)std::min<int64_t>(kTopNodes4, end - M.node4_offset);
        }
        d.k = P.consts;
        s->dds = dalloc<DScene>(1);
        CK(cudaMemcpy(s->dds, &s->ds, sizeof(DScene), cudaMemcpyHostToDevice));
        s->ctrl = dalloc<Ctrl>(1);
        s->totals = dalloc<unsigned long long>(2);
        CK(cudaMallocHost(&s->ctrl_host, sizeof(Ctrl)));
        CK(cudaMallocHost(&s->status_host, 4 * sizeof(unsigned long long)));
        cudaDeviceProp prop;
        CK(cudaGetDeviceProperties(&prop, device));
        s->sms = prop.multiProcessorCount;
        const int feat = P.consts.features & TF_ALL;
        s->extend = kExtendKernels[0][feat];
        s->shadow = kShadowKernels[feat];
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&s->occ_ext, s->extend, kBlock, 0));
        s->shade = shade_kernel(P.consts.caustics.enabled ? 1 : 0);
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&s->occ_shade, s->shade, kBlock, 0));
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&s->occ_sh, s->shadow, kBlock, 0));
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

int luz_gpu_scene_set_path_budget(luz_gpu_scene* s, int64_t bytes)
{
    return guard([&] {
        if (!s) throw Status(LUZ_E_INVALID, "NULL argument.");
        if (bytes < -1) throw Status(LUZ_E_INVALID, "Path budget must be -1 (default) or non-negative.");
        s->path_budget = bytes;
        const int64_t held = s->cap * (luz_gpu_scene::kPathBytes + (s->pb.feat ? luz_gpu_scene::kFeatBytes : 0));
        if (bytes >= 0 && held > bytes) {   // release path state above the new budget
            CK(cudaSetDevice(s->device));
            CK(cudaStreamSynchronize(s->stream));
            s->free_paths();
        }
        return LUZ_OK;
    });
}

static void check_tune(const LuzTuneParams& t)
{
    if (t.wave_paths < 0 || t.staged_top_nodes < 0 || t.staged_top_nodes > 1 || t.sort_rays < 0 || t.sort_rays > 1
        || t.lanes < 0 || t.lanes > 1 || t.extend_blocks_per_sm < 0
        || t.shadow_blocks_per_sm < 0 || t.shade_blocks_per_sm < 0)
        throw Status(LUZ_E_INVALID, "Tuning parameters out of range.");
}

int luz_gpu_scene_set_tuning(luz_gpu_scene* s, const LuzTuneParams* tune)
{
    return guard([&] {
        if (!s) throw Status(LUZ_E_INVALID, "NULL argument.");
        LuzTuneParams t{};
        if (tune) t = *tune;
        check_tune(t);
        s->tune = t;
        return LUZ_OK;
    });
}

int luz_gpu_scene_get_tuning(const luz_gpu_scene* s, LuzTuneParams* tune)
{
    return guard([&] {
        if (!s || !tune) throw Status(LUZ_E_INVALID, "NULL argument.");
        *tune = s->tune;
        return LUZ_OK;
    });
}

int luz_gpu_autotune(luz_gpu_scene* s, const LuzRenderParams* p, LuzTuneParams* chosen, LuzTuneTrial* trials,
                     int32_t trial_capacity, int32_t* trial_count)
{
    return guard([&] {
        if (!s) throw Status(LUZ_E_INVALID, "NULL argument.");
        check_params(p);
        if (p->flags) throw Status(LUZ_E_UNSUPPORTED, "Render flags are not supported by the autotuner.");
        CK(cudaSetDevice(s->device));
        const int64_t npix = (int64_t)p->width * p->height;
        float* d_out = dalloc<float>((std::size_t)(3 * npix));
        std::vector<LuzTuneTrial> log;
        try {
            // coordinate descent over the knobs, each trial one timed render of the frame
            LuzTuneParams best = s->tune;
            auto time_of = [&](const LuzTuneParams& t) {
                s->tune = t;
                LuzRenderStats st{};
                do_render(s, p, d_out, s->stream, &st);   // warm: the first render of a shape allocates
                do_render(s, p, d_out, s->stream, &st);
                LuzTuneTrial r{};
                r.params = t;
                r.render_ms = st.render_ms;
                log.push_back(r);
                return st.render_ms;
            };
            double best_ms = time_of(best);
            auto consider = [&](LuzTuneParams t) {
                const double ms = time_of(t);
                if (ms < best_ms) {
                    best_ms = ms;
                    best = t;
                }
            };
            {
                LuzTuneParams t = best;
                t.staged_top_nodes = best.staged_top_nodes ? 0 : 1;
                consider(t);
            }
            {
                LuzTuneParams t = best;
                t.sort_rays = best.sort_rays ? 0 : 1;
                consider(t);
            }
            {
                LuzTuneParams t = best;
                t.lanes = best.lanes ? 0 : 1;
                consider(t);
            }
            for (int64_t wave : {int64_t(1) << 22, int64_t(1) << 24, int64_t(0)}) {
                if (wave == best.wave_paths) continue;
                LuzTuneParams t = best;
                t.wave_paths = wave;
                consider(t);
            }
            for (int b : {s->occ_ext - 1, s->occ_ext}) {
                if (b < 1 || b == (best.extend_blocks_per_sm ? best.extend_blocks_per_sm : s->occ_ext)) continue;
                LuzTuneParams t = best;
                t.extend_blocks_per_sm = b == s->occ_ext ? 0 : b;
                consider(t);
            }
            for (int b : {s->occ_sh / 2, s->occ_sh}) {
                if (b < 1 || b == (best.shadow_blocks_per_sm ? best.shadow_blocks_per_sm : s->occ_sh)) continue;
                LuzTuneParams t = best;
                t.shadow_blocks_per_sm = b == s->occ_sh ? 0 : b;
                consider(t);
            }
            s->tune = best;
            if (chosen) *chosen = best;
        } catch (...) {
            cudaFree(d_out);
            throw;
        }
        cudaFree(d_out);
        if (trial_count) *trial_count = (int32_t)log.size();
        if (trials)
            for (int32_t i = 0; i < std::min<int32_t>(trial_capacity, (int32_t)log.size()); i++) trials[i] = log[(std::size_t)i];
        return LUZ_OK;
    });
}

int luz_gpu_scene_set_traversal_limits(luz_gpu_scene* s, int32_t mesh_entries, int32_t top_entries)
{
    return guard([&] {
        if (!s) throw Status(LUZ_E_INVALID, "NULL argument.");
        if (mesh_entries < 0 || mesh_entries > kMeshStack4 || top_entries < 0 || top_entries > kTopStack)
            throw Status(LUZ_E_INVALID, "Traversal limits must lie in [0, the compiled stack sizes].");
        CK(cudaSetDevice(s->device));
        CK(cudaStreamSynchronize(s->stream));
        s->ds.mesh_stack_limit = mesh_entries ? mesh_entries : kMeshStack4;
        s->ds.top_stack_limit = top_entries ? top_entries : kTopStack;
        CK(cudaMemcpy(s->dds, &s->ds, sizeof(DScene), cudaMemcpyHostToDevice));
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
        if (s->out_cap < npix) {   // device copy of the film, kept between calls
            if (s->out_dev) cudaFree(s->out_dev);
            s->out_dev = nullptr;
            s->out_cap = 0;
            s->out_dev = dalloc<float>((std::size_t)(3 * npix));
            s->out_cap = npix;
        }
        const int rc = do_render(s, p, s->out_dev, s->stream, stats);
        CK(cudaMemcpyAsync(rgb_out, s->out_dev, sizeof(float) * 3 * npix, cudaMemcpyDeviceToHost, s->stream));
        CK(cudaStreamSynchronize(s->stream));
        return rc;
    });
}

int luz_gpu_batch_render(luz_gpu_scene* const* scenes, const LuzRenderParams* params, int32_t count,
                         float* const* rgb_out, LuzRenderStats* stats)
{
    return guard([&] {
        if (count < 0) throw Status(LUZ_E_INVALID, "Batch size must be non-negative.");
        if (count == 0) return LUZ_OK;
        if (!scenes || !params || !rgb_out) throw Status(LUZ_E_INVALID, "NULL argument.");
        for (int32_t i = 0; i < count; i++) {
            if (!scenes[i] || !rgb_out[i]) throw Status(LUZ_E_INVALID, "NULL argument.");
            if (params[i].flags) throw Status(LUZ_E_UNSUPPORTED, "Render flags are not supported in a batch.");
            check_params(&params[i]);
            if (scenes[i]->device != scenes[0]->device)
                throw Status(LUZ_E_INVALID, "The scenes of a batch must be on one device.");
            for (int32_t j = 0; j < i; j++)
                if (scenes[j] == scenes[i])
                    throw Status(LUZ_E_INVALID, "A scene handle appears twice in one batch.");
        }
        return batch_render(scenes, params, count, rgb_out, stats, nullptr);
    });
}

int luz_gpu_batch_render_ex(luz_gpu_scene* const* scenes, const LuzRenderParams* params, int32_t count,
                            float* const* rgb_out, LuzRenderStats* stats, LuzBatchReport* report)
{
    if (report) *report = LuzBatchReport{};
    const int rc = luz_gpu_batch_render(scenes, params, count, rgb_out, stats);
    if (rc != LUZ_OK || !report || count == 0) return rc;
    return guard([&] {
        BatchContext& C = batch_context(scenes[0]->device);
        std::lock_guard<std::mutex> lock(C.mu);
        *report = C.last_report;
        return LUZ_OK;
    });
}

int luz_gpu_scene_set_texture(luz_gpu_scene* s, int32_t texture, const double* rgb)
{
    return guard([&] {
        if (!s) throw Status(LUZ_E_INVALID, "NULL argument.");
        set_texture(s, texture, rgb);
        return LUZ_OK;
    });
}

int luz_gpu_adjoint_forward(luz_gpu_scene* s, const LuzRenderParams* p, int32_t texture, const double* texels,
                            float* rgb_out, LuzRenderStats* stats)
{
    if (!s || !texels) {
        set_error("NULL argument.");
        return LUZ_E_INVALID;
    }
    const int rc = luz_gpu_scene_set_texture(s, texture, texels);
    if (rc != LUZ_OK) return rc;
    return luz_gpu_render(s, p, rgb_out, stats);
}

int luz_gpu_adjoint_backward(luz_gpu_scene* s, const LuzRenderParams* p, int32_t texture, const float* adjoint_rgb,
                             double* grad_out, LuzRenderStats* stats)
{
    return guard([&] {
        if (!s || !adjoint_rgb || !grad_out) throw Status(LUZ_E_INVALID, "NULL argument.");
        return do_adjoint_backward(s, p, texture, adjoint_rgb, grad_out, stats);
    });
}

int luz_gpu_adjoint_density(luz_gpu_scene* s, const LuzRenderParams* p, int32_t object, const float* adjoint_rgb,
                            double* grad_out, LuzRenderStats* stats)
{
    return guard([&] {
        if (!s || !adjoint_rgb || !grad_out) throw Status(LUZ_E_INVALID, "NULL argument.");
        return do_adjoint_density(s, p, object, adjoint_rgb, grad_out, stats);
    });
}

int luz_gpu_adjoint_emission(luz_gpu_scene* s, const LuzRenderParams* p, const float* adjoint_rgb, double* grad_out,
                             LuzRenderStats* stats)
{
    return guard([&] {
        if (!s || !adjoint_rgb || (!grad_out && s->pack->consts.light_count > 0))
            throw Status(LUZ_E_INVALID, "NULL argument.");
        return do_adjoint_emission(s, p, adjoint_rgb, grad_out, stats);
    });
}

int luz_gpu_render_ex(luz_gpu_scene* s, const LuzRenderParams* p, const LuzAdaptiveParams* adaptive, float* rgb_out,
                      const LuzNforBuffers* nfor, int32_t* samples_out, LuzRenderStats* stats)
{
    return guard([&] {
        if (!s || !rgb_out) throw Status(LUZ_E_INVALID, "NULL argument.");
        return do_render_ex(s, p, adaptive, rgb_out, nfor, samples_out, stats);
    });
}

int luz_gpu_render_pixels(luz_gpu_scene* s, const LuzRenderParams* p, const int32_t* pixels, int64_t count,
                          float* rgb_out, LuzRenderStats* stats)
{
    return guard([&] {
        if (!s || (count > 0 && (!pixels || !rgb_out))) throw Status(LUZ_E_INVALID, "NULL argument.");
        if (count < 0) throw Status(LUZ_E_INVALID, "Pixel count must be non-negative.");
        if (count == 0) return LUZ_OK;
        return do_render_ex(s, p, nullptr, rgb_out, nullptr, nullptr, stats, nullptr, nullptr, pixels, count);
    });
}

int luz_gpu_render_denoised(luz_gpu_scene* s, const LuzRenderParams* p, const LuzAdaptiveParams* adaptive,
                            const LuzNforSettings* settings, float* rgb_out, double* denoised_out,
                            int32_t* samples_out, LuzRenderStats* stats)
{
    return guard([&] {
        if (!s || !rgb_out || !denoised_out) throw Status(LUZ_E_INVALID, "NULL argument.");
        return do_render_ex(s, p, adaptive, rgb_out, nullptr, samples_out, stats, settings, denoised_out);
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
        clear_error(s, st);
        prepare_caustics(s, p, st);
        const int64_t chunk = s->reserve_paths(std::min<int64_t>(count, kWaveTarget));
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
                launch_bounces(s, w, st, launches, T, nullptr, s->pb, s->ctrl);
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
            clear_error(s, st);
            CK(cudaMemcpyAsync(dr, rays, sizeof(float) * 8 * count, cudaMemcpyHostToDevice, st));
            if (dk) CK(cudaMemcpyAsync(dk, volume_key, sizeof(int32_t) * 4 * count, cudaMemcpyHostToDevice, st));
            kTraceRayKernels[s->ds.k.features & TF_ALL]<<<(unsigned)((count + 127) / 128), 128, 0, st>>>(
                s->ds, dr, count, any_hit, seed, dk, dh);
            CK(cudaGetLastError());
            CK(cudaMemcpyAsync(out, dh, sizeof(LuzHit) * count, cudaMemcpyDeviceToHost, st));
            finish_status(s, st);
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

// ---------------------------------------------------------------------------- learned radiance cache

struct luz_gpu_cache {
    int device = 0;
    LuzCacheParams prm{};
    float *W = nullptr, *G = nullptr, *m = nullptr, *v = nullptr, *loss = nullptr;
    __half *Wf = nullptr, *Wb = nullptr;
    int64_t step = 0;   // Adam steps taken (bias correction)
    ~luz_gpu_cache()
    {
        cudaSetDevice(device);
        for (void* p : {(void*)W, (void*)G, (void*)m, (void*)v, (void*)loss, (void*)Wf, (void*)Wb})
            if (p) cudaFree(p);
    }
};

namespace {

constexpr int kCacheGradSmem = kCacheGradSmemHalves * 2;
constexpr int kCacheInferSmem = kCacheHalfF * 2;

void cache_pack(luz_gpu_cache* c, cudaStream_t st)
{
    k_cache_pack<<<(kCacheParams + 255) / 256, 256, 0, st>>>(c->W, c->Wf, c->Wb);
    CK(cudaGetLastError());
}

// Uniform +-sqrt(6 / fan_in) weights from a splitmix64 stream.
std::vector<float> cache_init(uint32_t seed)
{
    std::vector<float> w(kCacheParams);
    for (int l = 0; l < kCacheLayers; l++) {
        const CacheLayer L = cache_layer(l);
        const double a = std::sqrt(6.0 / (double)L.K);
        for (int i = 0; i < L.K * L.N; i++) {
            const uint64_t h = splitmix64(((uint64_t)seed << 32) ^ (uint64_t)(L.w + i));
            const double u = (double)(h >> 11) * (1.0 / 9007199254740992.0);
            w[(std::size_t)(L.w + i)] = (float)((2.0 * u - 1.0) * a);
        }
    }
    return w;
}

void cache_set(luz_gpu_cache* c, const float* w)
{
    CK(cudaMemcpy(c->W, w, sizeof(float) * kCacheParams, cudaMemcpyHostToDevice));
    CK(cudaMemset(c->m, 0, sizeof(float) * kCacheParams));
    CK(cudaMemset(c->v, 0, sizeof(float) * kCacheParams));
    CK(cudaMemset(c->G, 0, sizeof(float) * kCacheParams));
    c->step = 0;
    cache_pack(c, 0);
    CK(cudaDeviceSynchronize());
}

// One Adam step on rows [offset, offset + n_max) of the device rows (count:
// device row count, or NULL for exactly n_max rows).
void cache_step(luz_gpu_cache* c, const CacheRecord* rows, const uint32_t* count, int offset, int n_max,
                cudaStream_t st)
{
    k_cache_grad<<<(unsigned)((n_max + kCacheRowsPerBlock - 1) / kCacheRowsPerBlock), kCacheGradThreads, kCacheGradSmem, st>>>(
        rows, count, offset, n_max, c->Wf, c->Wb, c->G, c->loss);
    c->step++;
    const float b1 = 0.9f, b2 = 0.99f;
    k_cache_adam<<<(kCacheParams + 255) / 256, 256, 0, st>>>(c->W, c->G, c->m, c->v, c->prm.learning_rate, b1, b2, 1e-8f,
                                                             (float)std::pow((double)b1, (double)c->step),
                                                             (float)std::pow((double)b2, (double)c->step), count, offset,
                                                             n_max);
    cache_pack(c, st);
}

std::vector<CacheRecord> cache_rows(const float* inputs, const float* targets, int64_t n)
{
    std::vector<CacheRecord> r((std::size_t)n);
    for (int64_t i = 0; i < n; i++) {
        CacheRecord& q = r[(std::size_t)i];
        std::memset(&q, 0, sizeof(q));
        for (int f = 0; f < kCacheIn; f++) q.in[f] = inputs[kCacheIn * i + f];
        if (targets)
            for (int k = 0; k < 3; k++) q.v[k] = targets[3 * i + k];
    }
    return r;
}

void cache_check_rows(const luz_gpu_cache* c, const float* inputs, int64_t n)
{
    if (!c || (!inputs && n > 0)) throw Status(LUZ_E_INVALID, "NULL argument.");
    if (n < 0 || n > (int64_t)INT32_MAX / 2) throw Status(LUZ_E_INVALID, "Row count out of range.");
}

int do_render_cached(luz_gpu_scene* s, luz_gpu_cache* c, const LuzRenderParams* p, float* rgb_out, LuzRenderStats* stats)
{
    check_params(p);
    if (p->flags) throw Status(LUZ_E_UNSUPPORTED, "Render flags are not supported with the radiance cache.");
    if (s->pack->consts.caustics.enabled)
        throw Status(LUZ_E_UNSUPPORTED, "The radiance cache is not combined with caustic photon maps.");
    if (c->device != s->device) throw Status(LUZ_E_INVALID, "The cache and the scene are on different devices.");
    CK(cudaSetDevice(s->device));
    const cudaStream_t st = s->stream;
    clear_error(s, st);
    const int64_t npix = (int64_t)p->width * p->height;
    // waves as the plain render makes them (samples inner), one cache update per wave
    const int64_t target = s->tune.wave_paths > 0 ? s->tune.wave_paths : kCacheWaveTarget;
    const int64_t n_cap = s->reserve_paths(std::min<int64_t>(target, npix * (int64_t)p->spp));
    const int s_wave = (int)std::min<int64_t>(p->spp, std::max<int64_t>(1, n_cap / npix));
    const int64_t pix_wave = std::max<int64_t>(1, std::min<int64_t>(npix, n_cap / s_wave));
    const int64_t n_wave = pix_wave * s_wave;
    DeviceScratch D;
    CacheRecord* q = D.get<CacheRecord>(n_wave, st);
    CacheRecord* rows = D.get<CacheRecord>(n_wave, st);
    CacheSnap* snaps = D.get<CacheSnap>(n_wave, st);
    uint8_t* tflag = D.get<uint8_t>(n_wave, st);
    uint32_t* counts = D.get<uint32_t>(2, st);
    double* film = D.get<double>(3 * npix, st);
    float* d_out = D.get<float>(3 * npix, st);
    const ShadeKernel shade_cached = shade_kernel(2);
    int occ = 1;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, shade_cached, kBlock, 0));
    occ = std::max(1, occ);

    WaveArgs w = base_args(s, p);
    const GSceneConst& K = s->pack->consts;
    w.cache_prefix = c->prm.prefix;
    w.cache_train_every = (uint32_t)c->prm.train_every;
    w.cache_min_rough = c->prm.min_roughness;
    w.cache_q = q;
    w.cache_s = snaps;
    w.cache_flag = tflag;
    w.cache_count = counts;
    for (int a = 0; a < 3; a++) {
        w.cache_lo[a] = K.box_lo[a];
        w.cache_inv[a] = K.box_inv[a];
    }
    CK(cudaMemcpyAsync(s->dds, &s->ds, sizeof(DScene), cudaMemcpyHostToDevice, st));
    CK(cudaMemsetAsync(s->totals, 0, 2 * sizeof(unsigned long long), st));
    CK(cudaEventRecord(s->ev0, st));
    const int g_ext = s->sms * s->occ_ext, g_sh = s->sms * s->occ_sh, g_shade = s->sms * occ;
    const int batch = c->prm.batch;
    int64_t launches = 0, waves = 0;
    // The first sample of every pixel is rendered plain, every path training the
    // cache (warm_steps steps over its rows); later waves use the cache and
    // train at most kCacheWaveSteps steps each.
    const int warm_steps = c->prm.warm_steps > 0 ? c->prm.warm_steps : LUZ_CACHE_WARM_STEPS;
    constexpr int64_t kCacheWaveSteps = LUZ_CACHE_WAVE_STEPS;
    for (int sb = 0; sb < p->spp;) {
        const bool warm = sb == 0;
        const int sc = warm ? 1 : std::min(s_wave, p->spp - sb);
        for (int64_t pb = 0; pb < npix; pb += pix_wave) {
            const int64_t pc = std::min<int64_t>(pix_wave, npix - pb);
            w.pix_begin = (int32_t)pb;
            w.pix_count = (int32_t)pc;
            w.s_begin = sb;
            w.s_count = sc;
            w.n = pc * sc;
            w.list_mode = 0;
            w.cache_wave = (uint32_t)waves;
            w.cache_train_every = warm ? 1u : (uint32_t)c->prm.train_every;
            // after the warm-up wave, training paths end at their next eligible vertex in the cache
            w.cache_self_train = warm ? 0u : 1u;
            CK(cudaMemsetAsync(s->ctrl, 0, sizeof(Ctrl), st));
            CK(cudaMemsetAsync(counts, 0, 2 * sizeof(uint32_t), st));
            CK(cudaMemsetAsync(tflag, 0, (std::size_t)w.n, st));
            CK(cudaMemsetAsync(c->loss, 0, sizeof(float), st));
            k_raygen<<<(unsigned)((w.n + kBlock - 1) / kBlock), kBlock, 0, st>>>(w, s->pb, s->ctrl);
            for (int b = 0; b <= w.max_bounces; b++) {
                s->extend<<<g_ext, kBlock, 0, st>>>(s->ds, w, s->pb, s->ctrl, b);
                shade_cached<<<g_shade, kBlock, 0, st>>>(s->dds, w, s->pb, s->ctrl, b);
                s->shadow<<<g_sh, kBlock, 0, st>>>(s->ds, w, s->pb, s->ctrl, b);
            }
            k_cache_infer<<<(unsigned)(2 * s->sms), 128, kCacheInferSmem, st>>>(q, counts, 0, c->Wf, nullptr, s->pb.rad);
            k_cache_targets<<<(unsigned)((w.n + 255) / 256), 256, 0, st>>>(w, s->pb, rows, counts + 1);
            // about n / train_every rows: one step per batch of them (at most kCacheWaveSteps);
            // the warm-up wave cycles warm_steps steps over its rows
            const int64_t expect = (w.n + w.cache_train_every - 1) / w.cache_train_every;
            const int64_t chunks = std::max<int64_t>(1, (expect + batch - 1) / batch);
            const int steps = warm ? warm_steps : (int)std::min<int64_t>(kCacheWaveSteps, chunks);
            for (int i = 0; i < steps; i++)
                cache_step(c, rows, counts + 1, (int)((i % chunks) * batch), (int)std::min<int64_t>(batch, w.n), st);
            k_accumulate<<<(unsigned)((pc + 127) / 128), 128, 0, st>>>(w, s->pb, film);
            k_tally<<<1, 1, 0, st>>>(s->ctrl, w.max_bounces, s->totals);
            CK(cudaGetLastError());
            launches += 3 * (w.max_bounces + 1) + 6 + 3 * steps;
            waves++;
        }
        sb += sc;
    }
    k_resolve<<<(unsigned)((npix + 255) / 256), 256, 0, st>>>(film, npix, (double)p->spp, d_out);
    CK(cudaEventRecord(s->ev1, st));
    CK(cudaEventSynchronize(s->ev1));
    CK(cudaGetLastError());
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, s->ev0, s->ev1));
    unsigned long long tot[2] = {0, 0};
    finish_status(s, st, s->totals, tot);
    CK(cudaMemcpy(rgb_out, d_out, sizeof(float) * 3 * (std::size_t)npix, cudaMemcpyDeviceToHost));
    if (stats) {
        *stats = LuzRenderStats{};
        stats->render_ms = ms;
        stats->samples = (double)npix * p->spp;
        stats->extension_rays = (double)tot[0];
        stats->shadow_rays = (double)tot[1];
        stats->kernel_launches = launches + 1;
        stats->waves = waves;
    }
    return LUZ_OK;
}

}  // namespace

extern "C" {

int luz_gpu_cache_create(int32_t device, const LuzCacheParams* prm, luz_gpu_cache** out)
{
    return guard([&] {
        if (!prm || !out) throw Status(LUZ_E_INVALID, "NULL argument.");
        *out = nullptr;
        if (prm->batch <= 0) throw Status(LUZ_E_INVALID, "Cache batch must be positive.");
        if (!(prm->learning_rate > 0.0f) || !std::isfinite(prm->learning_rate))
            throw Status(LUZ_E_INVALID, "Cache learning rate must be finite and positive.");
        if (prm->prefix < 0) throw Status(LUZ_E_INVALID, "Cache prefix must be non-negative.");
        if (prm->train_every < 1) throw Status(LUZ_E_INVALID, "Cache training interval must be at least 1.");
        if (!(prm->min_roughness >= 0.0f && prm->min_roughness <= 1.0f))
            throw Status(LUZ_E_INVALID, "Cache minimum roughness must lie in [0, 1].");
        if (prm->warm_steps < 0 || prm->warm_steps > 4096)
            throw Status(LUZ_E_INVALID, "Cache warm-up steps must lie in [0, 4096].");
        CK(cudaSetDevice(device));
        std::unique_ptr<luz_gpu_cache> c(new luz_gpu_cache);
        c->device = device;
        c->prm = *prm;
        c->W = dalloc<float>(kCacheParams);
        c->G = dalloc<float>(kCacheParams);
        c->m = dalloc<float>(kCacheParams);
        c->v = dalloc<float>(kCacheParams);
        c->loss = dalloc<float>(1);
        c->Wf = dalloc<__half>(kCacheHalfF);
        c->Wb = dalloc<__half>(kCacheHalfB);
        CK(cudaMemset(c->Wf, 0, sizeof(__half) * kCacheHalfF));
        CK(cudaMemset(c->Wb, 0, sizeof(__half) * kCacheHalfB));
        CK(cudaFuncSetAttribute(k_cache_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, kCacheGradSmem));
        CK(cudaFuncSetAttribute(k_cache_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, kCacheInferSmem));
        const std::vector<float> w0 = cache_init(prm->seed);
        cache_set(c.get(), w0.data());
        *out = c.release();
        return LUZ_OK;
    });
}

int luz_gpu_cache_destroy(luz_gpu_cache* c)
{
    delete c;
    return LUZ_OK;
}

int luz_gpu_cache_weights(luz_gpu_cache* c, float* get, const float* set)
{
    return guard([&] {
        if (!c) throw Status(LUZ_E_INVALID, "NULL argument.");
        CK(cudaSetDevice(c->device));
        if (get) CK(cudaMemcpy(get, c->W, sizeof(float) * kCacheParams, cudaMemcpyDeviceToHost));
        if (set) cache_set(c, set);
        return LUZ_OK;
    });
}

int luz_gpu_cache_predict(luz_gpu_cache* c, const float* inputs, int64_t n, float* rgb_out)
{
    return guard([&] {
        cache_check_rows(c, inputs, n);
        if (!rgb_out && n > 0) throw Status(LUZ_E_INVALID, "NULL argument.");
        if (n == 0) return LUZ_OK;
        CK(cudaSetDevice(c->device));
        const std::vector<CacheRecord> r = cache_rows(inputs, nullptr, n);
        CacheRecord* d = dupload(r);
        float* o = nullptr;
        try {
            o = dalloc<float>((std::size_t)(3 * n));
            const int tiles = (int)((n + 15) / 16);
            k_cache_infer<<<(unsigned)std::max(1, std::min(tiles / 4 + 1, 1184)), 128, kCacheInferSmem>>>(
                d, nullptr, (int)n, c->Wf, o, nullptr);
            CK(cudaGetLastError());
            CK(cudaMemcpy(rgb_out, o, sizeof(float) * 3 * (std::size_t)n, cudaMemcpyDeviceToHost));
        } catch (...) {
            cudaFree(d);
            if (o) cudaFree(o);
            throw;
        }
        cudaFree(d);
        cudaFree(o);
        return LUZ_OK;
    });
}

int luz_gpu_cache_gradient(luz_gpu_cache* c, const float* inputs, const float* targets, int64_t n, float* grad_out,
                           double* loss_out)
{
    return guard([&] {
        cache_check_rows(c, inputs, n);
        if (!targets || n <= 0) throw Status(LUZ_E_INVALID, "Gradient needs rows and targets.");
        CK(cudaSetDevice(c->device));
        const std::vector<CacheRecord> r = cache_rows(inputs, targets, n);
        CacheRecord* d = dupload(r);
        try {
            CK(cudaMemset(c->G, 0, sizeof(float) * kCacheParams));
            CK(cudaMemset(c->loss, 0, sizeof(float)));
            k_cache_grad<<<(unsigned)((n + kCacheRowsPerBlock - 1) / kCacheRowsPerBlock), kCacheGradThreads, kCacheGradSmem>>>(
                d, nullptr, 0, (int)n, c->Wf, c->Wb, c->G, c->loss);
            CK(cudaGetLastError());
            std::vector<float> g(kCacheParams);
            float l = 0.f;
            CK(cudaMemcpy(g.data(), c->G, sizeof(float) * kCacheParams, cudaMemcpyDeviceToHost));
            CK(cudaMemcpy(&l, c->loss, sizeof(float), cudaMemcpyDeviceToHost));
            CK(cudaMemset(c->G, 0, sizeof(float) * kCacheParams));
            if (grad_out)
                for (int i = 0; i < kCacheParams; i++) grad_out[i] = g[(std::size_t)i] / (kCacheLossScale * (float)n);
            if (loss_out) *loss_out = (double)l / (double)n;
        } catch (...) {
            cudaFree(d);
            throw;
        }
        cudaFree(d);
        return LUZ_OK;
    });
}

int luz_gpu_cache_train(luz_gpu_cache* c, const float* inputs, const float* targets, int64_t n, int32_t steps,
                        double* loss_out)
{
    return guard([&] {
        cache_check_rows(c, inputs, n);
        if (!targets || n <= 0) throw Status(LUZ_E_INVALID, "Training needs rows and targets.");
        if (n > c->prm.batch) throw Status(LUZ_E_INVALID, "More rows than the cache batch.");
        if (steps < 0) throw Status(LUZ_E_INVALID, "Step count must be non-negative.");
        CK(cudaSetDevice(c->device));
        const std::vector<CacheRecord> r = cache_rows(inputs, targets, n);
        CacheRecord* d = dupload(r);
        try {
            for (int i = 0; i < steps; i++) {
                CK(cudaMemset(c->loss, 0, sizeof(float)));
                cache_step(c, d, nullptr, 0, (int)n, 0);
                CK(cudaGetLastError());
                float l = 0.f;
                CK(cudaMemcpy(&l, c->loss, sizeof(float), cudaMemcpyDeviceToHost));
                if (loss_out) loss_out[i] = (double)l / (double)n;
            }
        } catch (...) {
            cudaFree(d);
            throw;
        }
        cudaFree(d);
        return LUZ_OK;
    });
}

int luz_gpu_render_cached(luz_gpu_scene* s, luz_gpu_cache* c, const LuzRenderParams* p, float* rgb_out,
                          LuzRenderStats* stats)
{
    return guard([&] {
        if (!s || !c || !rgb_out) throw Status(LUZ_E_INVALID, "NULL argument.");
        return do_render_cached(s, c, p, rgb_out, stats);
    });
}

}  // extern "C"
