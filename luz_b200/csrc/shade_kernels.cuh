// shade_kernels.cuh — the shade-stage kernels (k_shade, k_shade_batch), included by
// the translation units that instantiate them: shade_kernels.cu (with the sampler,
// light sampling and hit record inlined) and shade_cache_kernels.cu (the radiance-cache
// instantiation, with them out of line). Internal linkage: each unit emits only the
// instantiations it uses.
#pragma once
#include "wavefront.cuh"

namespace luz {
namespace {


// Resident blocks per SM the register allocator is asked to allow, measured on the
// 1080p glossy frame (16 spp, shade stage; the kernel is latency-bound, and more warps
// hide more of it despite spills): 6 blocks (80 registers) 20.3 ms, 7 (72) 20.1 ms,
// 8 (64) 20.7 ms, 5 (96) 22.1-22.4 ms, 4 (128) 22.6 ms, 3 (168) 25.2 ms.
#ifndef LUZ_SHADE_MIN_BLOCKS
#define LUZ_SHADE_MIN_BLOCKS 6
#endif

// Path of shade slot i: slots run through the class segments in class order.
__device__ __forceinline__ uint32_t binned_path(const PathBuf& P, const uint32_t* bin, uint32_t i)
{
    uint32_t k = 0, start = 0;
    while (k < kShadeClasses - 1 && i >= start + bin[k]) {
        start += bin[k];
        k++;
    }
    return P.bins[k * P.bin_stride + (i - start)];
}

template <int MODE>
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
            p = P.bins ? binned_path(P, C->bin[bounce], i) : q[i];
            shade_path<MODE>(S, w, P, p, bounce, o);
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


// k_shade over a multi-scene wave: the scene and wave arguments are the path's segment's.
template <int MODE>
__global__ void __launch_bounds__(kBlock, LUZ_SHADE_MIN_BLOCKS) k_shade_batch(const DScene* __restrict__ scenes,
                                                                             const WaveArgs* __restrict__ segs,
                                                                             PathBuf P, Ctrl* C, int bounce)
{
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
            p = P.bins ? binned_path(P, C->bin[bounce], i) : q[i];
            const WaveArgs& w = segs[P.seg[p]];
            shade_path<MODE>(scenes[w.batch_scene], w, P, p, bounce, o);
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

}  // namespace
}  // namespace luz
