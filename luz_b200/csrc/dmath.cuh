// dmath.cuh — device vector helpers and the Luz sampler stream.
//
// Traversal and ray generation are compiled with -fmad=false (integrator.cu),
// so the FP32 traversal matches its C restatement bit for bit; the shade stage
// (shade_kernels.cu) is compiled with FMA contraction. The sampler's FP64
// lattice arithmetic is written with explicit round-to-nearest intrinsics, so
// it reproduces the reference bit for bit in either unit.
#pragma once
// Out of line by default; the shade kernels' translation unit inlines the sampler.
#ifndef LUZ_SAMPLER_ATTR
#define LUZ_SAMPLER_ATTR __noinline__
#endif
#include <cuda_runtime.h>
#include <stdint.h>

#include "layout.h"

namespace luz {

constexpr double kPiD = 3.14159265358979323846;
constexpr float kInf = __builtin_huge_valf();

struct F3 {
    float x, y, z;
};
__device__ __forceinline__ F3 f3(float x, float y, float z) { return F3{x, y, z}; }
__device__ __forceinline__ F3 f3(const float* p) { return F3{p[0], p[1], p[2]}; }
__device__ __forceinline__ F3 operator+(F3 a, F3 b) { return F3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ F3 operator-(F3 a, F3 b) { return F3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ F3 operator*(F3 a, F3 b) { return F3{a.x * b.x, a.y * b.y, a.z * b.z}; }
__device__ __forceinline__ F3 operator*(float f, F3 v) { return F3{f * v.x, f * v.y, f * v.z}; }
__device__ __forceinline__ F3 operator*(F3 v, float f) { return F3{f * v.x, f * v.y, f * v.z}; }
__device__ __forceinline__ F3 operator-(F3 a) { return F3{-a.x, -a.y, -a.z}; }
// Vector3 / f is (1 / f) * v (include/luz/Vector3.hpp); Color / f divides per channel.
__device__ __forceinline__ F3 vdiv(F3 v, float f) { return (1.0f / f) * v; }
__device__ __forceinline__ F3 cdiv(F3 c, float f) { return F3{c.x / f, c.y / f, c.z / f}; }
__device__ __forceinline__ float dot(F3 a, F3 b) { return (a.x * b.x) + (a.y * b.y) + (a.z * b.z); }
__device__ __forceinline__ F3 cross(F3 a, F3 b)
{
    return F3{(a.y * b.z) - (a.z * b.y), (a.z * b.x) - (a.x * b.z), (a.x * b.y) - (a.y * b.x)};
}
__device__ __forceinline__ float len2(F3 v) { return (v.x * v.x) + (v.y * v.y) + (v.z * v.z); }
__device__ __forceinline__ F3 normalize(F3 v) { return vdiv(v, sqrtf(len2(v))); }
__device__ __forceinline__ float maxc(F3 c) { return fmaxf(c.x, fmaxf(c.y, c.z)); }
__device__ __forceinline__ bool finitef(float v) { return isfinite(v); }
__device__ __forceinline__ F3 reflect(F3 v, F3 n) { return v - (2.0f * dot(v, n)) * n; }
// ACEScg luminance (src/core/ColorManagement.cpp:313-320).
__device__ __forceinline__ float luminance(F3 c)
{
    return c.x * 0.2722287168f + c.y * 0.6740817658f + c.z * 0.0536895174f;
}
__device__ __forceinline__ float4 ld4(const float4* p) { return __ldg(p); }

// ----------------------------------------------------------------------------- sampler
// Sampler (src/core/Sampler.cpp:31-237): stateless splitmix64 keyed on
// (render seed, x, y, stream, sample, bounce, dimension, component), with a
// rank-1 lattice + Cranley-Patterson shift for the "progressive" dimensions.
enum Dim : uint32_t {
    DIM_CAMERA = 0, DIM_LENS = 1, DIM_LIGHT_STRATEGY = 2, DIM_LIGHT_SELECTION = 3, DIM_LIGHT_SURFACE_SELECTION = 4,
    DIM_LIGHT_SURFACE_POINT = 5, DIM_BSDF_DIRECTION = 6, DIM_MATERIAL_DECISION = 7, DIM_MATERIAL_FUZZ = 8,
    DIM_RUSSIAN_ROULETTE = 9, DIM_VOLUME_DISTANCE = 10, DIM_ATMOSPHERE = 11, DIM_ENVIRONMENT_SELECTION = 12,
    DIM_ENVIRONMENT_POINT = 13, DIM_ENVIRONMENT_STRATEGY = 14, DIM_LIGHT_EMISSION_SIDE = 15,
    DIM_LIGHT_EMISSION_DIRECTION = 16, DIM_SUBSURFACE_SPATIAL = 17, DIM_SUBSURFACE_PROFILE_COMPONENT = 18,
    DIM_SUBSURFACE_THIN_SIDE = 19
};

struct Key {
    uint64_t base;
    uint32_t sample;
    uint32_t bounce;
};

__host__ __device__ __forceinline__ uint64_t splitmix64(uint64_t v)
{
    v += 0x9e3779b97f4a7c15ull;
    v = (v ^ (v >> 30)) * 0xbf58476d1ce4e5b9ull;
    v = (v ^ (v >> 27)) * 0x94d049bb133111ebull;
    return v ^ (v >> 31);
}
__device__ __forceinline__ double unit24(uint64_t v)   // unitFromHash(hash32(v))
{
    return (double)((uint32_t)(splitmix64(v) >> 32) >> 8) * (1.0 / 16777216.0);
}
__device__ __forceinline__ double unit53(uint64_t h) { return (double)(h >> 11) * (1.0 / 9007199254740992.0); }
__device__ __forceinline__ double fract(double x) { return x - floor(x); }

__host__ __device__ __forceinline__ uint64_t base_key(uint32_t seed, uint32_t x, uint32_t y, uint32_t stream)
{
    uint64_t k = seed;
    k ^= ((uint64_t)x + 1ull) * 0xbf58476d1ce4e5b9ull;
    k ^= ((uint64_t)y + 1ull) * 0x94d049bb133111ebull;
    k ^= ((uint64_t)stream + 1ull) * 0xda942042e4dd58b5ull;
    return k;
}

__device__ __forceinline__ double dim_step(uint32_t dim, uint32_t comp)
{
    const uint64_t key = ((uint64_t)dim + 1ull) * 0x9e3779b97f4a7c15ull ^ ((uint64_t)comp + 1ull) * 0xda942042e4dd58b5ull;
    double s = unit24(key);
    if (s < 0.05 || s > 0.95) s = fract(s + 0.6180339887498948);
    return s;
}
__device__ __forceinline__ bool progressive(uint32_t dim)
{
    const uint32_t b = dim % 32u;
    return b == DIM_CAMERA || b == DIM_LENS || b == DIM_LIGHT_SURFACE_SELECTION || b == DIM_LIGHT_SURFACE_POINT
           || b == DIM_ENVIRONMENT_SELECTION || b == DIM_ENVIRONMENT_POINT || b == DIM_LIGHT_EMISSION_DIRECTION;
}
__device__ __forceinline__ uint64_t ctx_key(const Key& k, uint32_t dk)
{
    return k.base ^ (((uint64_t)dk + 1ull) * 0x9e3779b97f4a7c15ull);
}
__device__ __forceinline__ double hashed(const Key& k, uint32_t dk, uint32_t comp)
{
    uint64_t key = ctx_key(k, dk);
    key ^= ((uint64_t)k.sample + 1ull) * 0x94d049bb133111ebull;
    key ^= ((uint64_t)comp + 1ull) * 0xbf58476d1ce4e5b9ull;
    return unit53(splitmix64(key));
}
static __device__ LUZ_SAMPLER_ATTR double sample1d(const Key& k, uint32_t dim)
{
    const uint32_t dk = dim + k.bounce * 32u;
    if (!progressive(dim)) return hashed(k, dk, 0);
    const double shift = unit24(ctx_key(k, dk));
    const double step = dim_step(dk, 0);
    // fract(0.5 + (s + 1) * step + shift), each operation rounded on its own as the reference computes it
    return fract(__dadd_rn(__dadd_rn(0.5, __dmul_rn((double)k.sample + 1.0, step)), shift));
}
struct S2 {
    float x, y;
};
static __device__ LUZ_SAMPLER_ATTR S2 sample2d(const Key& k, uint32_t dim)
{
    const uint32_t dk = dim + k.bounce * 32u;
    if (!progressive(dim)) return S2{(float)hashed(k, dk, 0), (float)hashed(k, dk, 1)};
    const uint64_t key = ctx_key(k, dk);
    const double sx = unit24(key);
    const double sy = unit24(key ^ 0xda942042e4dd58b5ull);
    const double s = (double)k.sample + 1.0;
    return S2{(float)fract(__dadd_rn(__dadd_rn(0.5, __dmul_rn(s, dim_step(dk, 0))), sx)),
              (float)fract(__dadd_rn(__dadd_rn(0.5, __dmul_rn(s, dim_step(dk, 1))), sy))};
}

constexpr float kTwoPiF = 6.28318530717958647692f;   // static_cast<float>(2.0 * D_PI)
constexpr float kPiF = 3.14159265358979323846f;

__device__ __forceinline__ F3 cosine_hemisphere(const Key& k, uint32_t dim)
{
    const S2 s = sample2d(k, dim);
    const float phi = kTwoPiF * s.x;
    const float r = sqrtf(s.y);
    const float z = sqrtf(fmaxf(0.0f, 1.0f - s.y));
    return F3{r * cosf(phi), r * sinf(phi), z};
}
__device__ __forceinline__ F3 sphere_direction(const Key& k, uint32_t dim)
{
    const S2 s = sample2d(k, dim);
    const float z = 1.0f - (2.0f * s.y);
    const float r = sqrtf(fmaxf(0.0f, 1.0f - z * z));
    const float phi = kTwoPiF * s.x;
    return F3{r * cosf(phi), r * sinf(phi), z};
}
__device__ __forceinline__ void unit_disk(const Key& k, uint32_t dim, float& ox, float& oy)
{
    const S2 s = sample2d(k, dim);
    const float sx = (2.0f * s.x) - 1.0f;
    const float sy = (2.0f * s.y) - 1.0f;
    if (sx == 0.0f && sy == 0.0f) {
        ox = 0.f;
        oy = 0.f;
        return;
    }
    float radius, theta;
    if (fabsf(sx) > fabsf(sy)) {
        radius = sx;
        theta = (kPiF / 4.0f) * (sy / sx);
    } else {
        radius = sy;
        theta = (kPiF / 2.0f) - ((kPiF / 4.0f) * (sx / sy));
    }
    ox = radius * cosf(theta);
    oy = radius * sinf(theta);
}

// ONB (src/core/ONB.cpp:5-15).
struct Onb {
    F3 u, v, w;
};
__device__ __forceinline__ Onb make_onb(F3 n)
{
    Onb b;
    b.w = normalize(n);
    const F3 a = (fabsf(b.w.x) > 0.9f) ? F3{0.f, 1.f, 0.f} : F3{1.f, 0.f, 0.f};
    b.v = normalize(cross(b.w, a));
    b.u = cross(b.w, b.v);
    return b;
}
__device__ __forceinline__ F3 onb_local(const Onb& b, float a, float c1, float c2)
{
    return ((a * b.u) + (c1 * b.v)) + (c2 * b.w);
}
__device__ __forceinline__ F3 onb_local(const Onb& b, F3 v) { return onb_local(b, v.x, v.y, v.z); }

}  // namespace luz
