// shade.cuh — hit records, BSDFs, lights and the environment on the device.
//
// FP32 restatements of:
//   HitRecord construction          Triangle.cpp:196-270, Rectangle.cpp:212-261,
//                                   Sphere.cpp:227-270, Plane.cpp, MeshInstance.cpp:274-301,
//                                   ConstantVolume.cpp:106-121
//   BSDF helpers                    src/core/Materials/BSDF.cpp:47-458
//   Lambertian / Metal / Dielectric / Isotropic / HenyeyGreenstein / Principled
//                                   src/core/Materials/*.cpp (scatter, evaluateBSDFCos, scatteringPDF)
//   scatterPDFValue / scatterBSDFCos / scatterPDFGenerate / HG sampling
//                                   src/renderer/ColorHelper.cpp:38-165
//   lights: sampleLight + pdfValue  Rectangle.cpp:345-419, Sphere.cpp:359-466,
//                                   Mesh.cpp:844-936, Triangle.cpp:307-420,
//                                   MeshInstance.cpp:393-547, DirectionalLight.cpp:68-91
//   EnvironmentMap sample/pdf/lookup src/core/EnvironmentMap.cpp:457-623 (index math in FP64)
#pragma once
// Out of line by default (small code for the trace and adjoint kernels); the shade
// kernels' translation unit defines these as __forceinline__.
#ifndef LUZ_HIT_ATTR
#define LUZ_HIT_ATTR __noinline__
#endif
#ifndef LUZ_LIGHT_ATTR
#define LUZ_LIGHT_ATTR __noinline__
#endif
#include "trace.cuh"

namespace luz {

struct Hit {
    F3 p, n, gn;
    bool front;
    float u, v;
    float t;
    int32_t material;
    int32_t obj;
    int32_t prim;
    bool volume;
};

__device__ __forceinline__ float clamp01f(float v) { return isfinite(v) ? fmaxf(0.0f, fminf(1.0f, v)) : 0.0f; }
__device__ __forceinline__ F3 clamp_color01(F3 c) { return F3{clamp01f(c.x), clamp01f(c.y), clamp01f(c.z)}; }
__device__ __forceinline__ F3 safe_normalize(F3 v, F3 fb)
{
    const float l2 = len2(v);
    if (!isfinite(l2) || l2 <= 0.0f) return fb;
    return vdiv(v, sqrtf(l2));
}
__device__ __forceinline__ void set_face(const F3& d, F3 outward, Hit& h)
{
    h.front = ((d.x * outward.x) + (d.y * outward.y) + (d.z * outward.z)) < 0.0f;
    h.n = h.front ? outward : outward * -1.0f;
    h.gn = h.n;
}
__device__ __forceinline__ F3 face_toward(const F3& d, F3 n) { return dot(d, n) > 0.0f ? n * -1.0f : n; }

// Sphere UVs in a 4x3 cube-cross atlas (setCubeCrossUV, Sphere.cpp:22-83): the
// dominant axis of the outward normal picks the face (ties go to x, then y),
// the face coordinates are inset by 0.02 on each side.
__device__ __forceinline__ void sphere_cube_cross_uv(const F3& n, float& u, float& v)
{
    const float ax = fabsf(n.x), ay = fabsf(n.y), az = fabsf(n.z);
    int column, row;
    float s, t;
    if (ax >= ay && ax >= az) {
        column = n.x >= 0.0f ? 2 : 0;
        row = 1;
        s = n.x >= 0.0f ? 0.5f - (n.z / (2.0f * ax)) : 0.5f + (n.z / (2.0f * ax));
        t = 0.5f + (n.y / (2.0f * ax));
    } else if (ay >= ax && ay >= az) {
        column = n.y >= 0.0f ? 2 : 0;
        row = n.y >= 0.0f ? 2 : 0;
        s = n.y >= 0.0f ? 0.5f - (n.z / (2.0f * ay)) : 0.5f + (n.z / (2.0f * ay));
        t = 0.5f - (n.x / (2.0f * ay));
    } else {
        column = n.z >= 0.0f ? 1 : 3;
        row = 1;
        s = n.z >= 0.0f ? 0.5f + (n.x / (2.0f * az)) : 0.5f - (n.x / (2.0f * az));
        t = 0.5f + (n.y / (2.0f * az));
    }
    const float inset = 0.02f;
    s = inset + (fminf(fmaxf(s, 0.0f), 1.0f) * (1.0f - (2.0f * inset)));
    t = inset + (fminf(fmaxf(t, 0.0f), 1.0f) * (1.0f - (2.0f * inset)));
    u = ((float)column + s) / 4.0f;
    v = ((float)row + t) / 3.0f;
}

// Triangle::hit shading (Triangle.cpp:234-269) in the frame of ray r.
static __device__ void triangle_shading(const DScene& S, const GMesh& M, int32_t slot, float bu, float bv, const F3& d,
                                 F3& n, F3& gn, bool& front, float& u, float& v)
{
    const float4 fs = __ldg(reinterpret_cast<const float4*>(S.tri_shade + slot));
    const F3 fn = F3{fs.x, fs.y, fs.z};
    F3 sn = fn;
    const float w0 = (1.0f - bu - bv);
    if (M.normal_offset >= 0 && fs.w != 0.0f) {
        const float* vn = S.vnormals + (size_t)9 * (size_t)(M.normal_offset + (slot - M.tri_offset));
        const F3 in = ((f3(vn) * w0) + (f3(vn + 3) * bu)) + (f3(vn + 6) * bv);
        sn = len2(in) <= 1e-24f ? fn : normalize(in);
    }
    u = 0.f;
    v = 0.f;
    if (M.uv_offset >= 0) {
        const float* uv = S.vuvs + (size_t)6 * (size_t)(M.uv_offset + (slot - M.tri_offset));
        u = ((uv[0] * w0) + (uv[2] * bu)) + (uv[4] * bv);
        v = ((uv[1] * w0) + (uv[3] * bu)) + (uv[5] * bv);
    }
    front = ((d.x * sn.x) + (d.y * sn.y) + (d.z * sn.z)) < 0.0f;
    n = front ? sn : sn * -1.0f;
    gn = face_toward(d, fn);
    if (dot(d, fn) == 0.0f) gn = fn * -1.0f;   // setFaceNormal: frontFace false -> negated
}

__device__ __forceinline__ F3 transform_normal(const GObject& O, F3 n)
{
    const F3 is = F3{n.x / O.f[3], n.y / O.f[4], n.z / O.f[5]};
    const F3 r = fwd_rotate(O, is);
    const float l2 = len2(r);
    if (!isfinite(l2) || l2 <= 1e-24f) return F3{0.f, 0.f, 0.f};
    return vdiv(r, sqrtf(l2));
}

// Builds the HitRecord the reference's hit() would fill for THit h on ray r.
// XUV: the scene has cube-cross spheres (a separate instantiation: the branch
// alone enlarges this out-of-line function's frame and slowed the shade stage
// by 3.5% on scenes without such spheres).
template <bool XUV>
static __device__ LUZ_HIT_ATTR Hit make_hit_t(const DScene& S, const TRay& r, const THit& th)
{
    Hit h;
    const GObject O = S.objects[th.obj];
    h.t = th.t;
    h.obj = th.obj;
    h.prim = th.prim;
    h.volume = O.kind == OK_VOLUME;
    h.p = r.o + (th.t * r.d);
    h.material = O.material;
    h.u = 0.f;
    h.v = 0.f;
    switch (O.kind) {
    case OK_RECT:
    case OK_CUBE: {
        const GRect R = S.rects[O.aux + (O.kind == OK_CUBE ? th.prim : 0)];
        set_face(r.d, f3(R.n), h);
        const F3 dd = h.p - f3(R.p);
        h.u = (dot(dd, f3(R.wa)) / R.w) + 0.5f;
        h.v = (dot(dd, f3(R.ha)) / R.h) + 0.5f;
        if (O.kind == OK_RECT && O.f[8] != 0.0f) {   // Rectangle::_uvAt: bilinear corners (Rectangle.cpp:64-70, 154-161)
            const float u = h.u, v = h.v;
            const float bu = (O.f[0] * (1.0f - u)) + (O.f[2] * u), bv = (O.f[1] * (1.0f - u)) + (O.f[3] * u);
            const float tu = (O.f[6] * (1.0f - u)) + (O.f[4] * u), tv = (O.f[7] * (1.0f - u)) + (O.f[5] * u);
            h.u = (bu * (1.0f - v)) + (tu * v);
            h.v = (bv * (1.0f - v)) + (tv * v);
        }
        break;
    }
    case OK_SPHERE: {
        const F3 outward = vdiv(h.p - f3(O.f), O.f[3]);
        if (XUV && O.f[5] != 0.0f) {
            sphere_cube_cross_uv(outward, h.u, h.v);
        } else {
            const float phi = atan2f(outward.z, outward.x);
            const float theta = acosf(fminf(fmaxf(outward.y, -1.0f), 1.0f));
            h.u = 0.5f + phi / (2.0f * kPiF);
            h.v = 1.0f - theta / kPiF;
        }
        set_face(r.d, outward, h);
        break;
    }
    case OK_PLANE:
        set_face(r.d, f3(O.f + 1), h);
        break;
    case OK_MESH: {
        const GMesh M = S.meshes[O.aux];
        triangle_shading(S, M, th.prim, th.u, th.v, r.d, h.n, h.gn, h.front, h.u, h.v);
        h.material = M.material;
        break;
    }
    case OK_INSTANCE: {
        const GMesh M = S.meshes[O.aux];
        F3 ln, lgn;
        bool lf;
        triangle_shading(S, M, th.prim, th.u, th.v, r.d /* facing fixed below */, ln, lgn, lf, h.u, h.v);
        F3 wn = transform_normal(O, ln);
        F3 wg = transform_normal(O, lgn);
        if (dot(r.d, wn) > 0.0f) wn = wn * -1.0f;
        if (dot(r.d, wg) > 0.0f) wg = wg * -1.0f;
        h.n = wn;
        h.gn = wg;
        h.front = dot(r.d, wn) < 0.0f;
        break;
    }
    case OK_VOLUME:
    default:
        h.n = F3{1.f, 0.f, 0.f};
        h.gn = h.n;
        h.front = true;
        break;
    }
    return h;
}

__device__ __forceinline__ Hit make_hit(const DScene& S, const TRay& r, const THit& th)
{
    return S.k.cube_cross_spheres ? make_hit_t<true>(S, r, th) : make_hit_t<false>(S, r, th);
}

// ----------------------------------------------------------------------------- textures / colour

__device__ __forceinline__ float wrap01f(float v)
{
    v = v - floorf(v);
    if (v < 0.0f) v += 1.0f;
    return v;
}
static __device__ __noinline__ F3 texture_sample(const DScene& S, int32_t ti, float u, float v)
{
    const GTexture T = S.textures[ti];
    u = wrap01f(u);
    v = wrap01f(v);
    const float x = u * (float)(T.width - 1);
    const float y = (1.0f - v) * (float)(T.height - 1);
    const int x0 = (int)floorf(x), y0 = (int)floorf(y);
    const int x1 = min(x0 + 1, T.width - 1), y1 = min(y0 + 1, T.height - 1);
    const float tx = x - (float)x0, ty = y - (float)y0;
    auto px = [&](int xx, int yy) {
        const float4 c = __ldg(S.texels + T.offset + yy * T.width + xx);
        return F3{c.x, c.y, c.z};
    };
    const F3 top = (px(x0, y0) * (1.0f - tx)) + (px(x1, y0) * tx);
    const F3 bot = (px(x0, y1) * (1.0f - tx)) + (px(x1, y1) * tx);
    const F3 c = (top * (1.0f - ty)) + (bot * ty);
    return F3{fmaxf(0.f, fminf(1.f, c.x)), fmaxf(0.f, fminf(1.f, c.y)), fmaxf(0.f, fminf(1.f, c.z))};
}
__device__ __forceinline__ F3 color_at(const DScene& S, const GMaterial& m, const Hit& h)
{
    const F3 c = f3(m.color);
    if (m.texture >= 0) return c * texture_sample(S, m.texture, h.u, h.v);
    return c;
}

// Metal roughness from a texture (red channel, bilinear, clamped to [0, 1]) when
// the material has one: the per-hit copy gets roughness and alpha =
// roughnessToAlpha(roughness) (BSDF.cpp:53-57).
__device__ __forceinline__ void resolve_material(const DScene& S, GMaterial& m, const Hit& h)
{
    if (m.rtexture >= 0) {
        const float r = texture_sample(S, m.rtexture, h.u, h.v).x;
        m.roughness = r;
        m.alpha = fmaxf(1e-4f, r * r);
    }
}

// ----------------------------------------------------------------------------- BSDF helpers

__device__ __forceinline__ F3 schlick(F3 f0, float cosT)
{
    cosT = clamp01f(cosT);
    const float factor = powf(1.0f - cosT, 5.0f);
    f0 = clamp_color01(f0);
    return F3{f0.x + (1.0f - f0.x) * factor, f0.y + (1.0f - f0.y) * factor, f0.z + (1.0f - f0.z) * factor};
}
static __device__ float dielectric_fresnel(float c, float ei, float et)
{
    c = clamp01f(fabsf(c));
    if (!isfinite(ei) || !isfinite(et) || ei <= 0.0f || et <= 0.0f) return 1.0f;
    const float si = sqrtf(fmaxf(0.0f, (1.0f - c) * (1.0f + c)));
    const float st = ei / et * si;
    if (st >= 1.0f) return 1.0f;
    const float ct = sqrtf(fmaxf(0.0f, (1.0f - st) * (1.0f + st)));
    const float rpa = ((et * c) - (ei * ct)) / ((et * c) + (ei * ct));
    const float rpe = ((ei * c) - (et * ct)) / ((ei * c) + (et * ct));
    return clamp01f(0.5f * (rpa * rpa + rpe * rpe));
}
static __device__ float conductor_channel(float e, float k, float c)
{
    if (!isfinite(e) || !isfinite(k) || e <= 0.0f || k < 0.0f) return 0.0f;
    const float c2 = c * c, e2 = e * e, k2 = k * k;
    const float ek = e2 + k2;
    const float tec = 2.0f * e * c;
    const float pd = ek * c2 + tec + 1.0f;
    const float sd = ek + tec + c2;
    if (fabsf(pd) <= 1e-10f || fabsf(sd) <= 1e-10f) return 0.0f;
    const float rpa = (ek * c2 - tec + 1.0f) / pd;
    const float rpe = (ek - tec + c2) / sd;
    return clamp01f(0.5f * (rpa + rpe));
}
__device__ __forceinline__ F3 conductor_fresnel(F3 eta, F3 k, float c)
{
    c = clamp01f(c);
    return F3{conductor_channel(eta.x, k.x, c), conductor_channel(eta.y, k.y, c), conductor_channel(eta.z, k.z, c)};
}
static __device__ F3 sample_ggx_half(F3 n, float alpha, S2 s)
{
    alpha = fmaxf(1e-4f, alpha);
    const float a2 = alpha * alpha;
    const float phi = kTwoPiF * clamp01f(s.x);
    const float u = fminf(1.0f - 1e-7f, clamp01f(s.y));
    // cos^2 = (1-u) / (1 + (a2-1) u) and sin^2 = 1 - cos^2 = a2 u / ((1-u) + a2 u), each from its
    // own quotient: the same values in exact arithmetic, and sin stays accurate where cos is
    // within FP32 rounding of 1 (narrow lobes: 1 - ct would carry ~1e-3 relative error there).
    const float omu = 1.0f - u;
    const float q = omu + a2 * u;
    const float ct = sqrtf(omu / q);
    const float st = sqrtf((a2 * u) / q);
    return onb_local(make_onb(n), st * cosf(phi), st * sinf(phi), ct);
}
// GGX D of the half vector h about the normal n (both unit): noh^2 (a2 - 1) + 1 is
// written as sin^2 + a2 cos^2 with sin^2 = |n x h|^2, which keeps its relative
// accuracy where noh is within FP32 rounding of 1 (narrow lobes), unlike (1 - noh)(1 + noh).
__device__ __forceinline__ float ggx_d(F3 n, F3 h, float alpha)
{
    const float noh = clamp01f(dot(n, h));
    alpha = fmaxf(1e-4f, alpha);
    const float a2 = alpha * alpha;
    const float s2 = noh > 0.0f ? fminf(len2(cross(n, h)), 1.0f) : 1.0f;
    const float den = s2 + a2 * (noh * noh);
    const float val = a2 / (kPiF * den * den);
    return isfinite(val) ? val : 0.0f;
}
__device__ __forceinline__ float ggx_g1(float now, float alpha)
{
    now = clamp01f(now);
    alpha = fmaxf(1e-4f, alpha);
    if (now <= 0.0f) return 0.0f;
    const float a2 = alpha * alpha;
    const float den = now + sqrtf(a2 + (1.0f - a2) * now * now);
    if (den <= 1e-10f || !isfinite(den)) return 0.0f;
    return 2.0f * now / den;
}
__device__ __forceinline__ float ggx_g(float nov, float nol, float a) { return ggx_g1(nov, a) * ggx_g1(nol, a); }
static __device__ float ggx_reflection_pdf(F3 n, F3 view, F3 dir, float alpha)
{
    const float nov = dot(n, view), nol = dot(n, dir);
    if (nov <= 0.0f || nol <= 0.0f) return 0.0f;
    const F3 h = safe_normalize(view + dir, n);
    const float voh = dot(view, h), noh = dot(n, h);
    if (voh <= 1e-10f || noh <= 0.0f) return 0.0f;
    const float pdf = ggx_d(n, h, alpha) * noh / (4.0f * voh);
    return (isfinite(pdf) && pdf > 0.0f) ? pdf : 0.0f;
}
__device__ __forceinline__ F3 color_from_scale(F3 c, float s)
{
    if (!isfinite(s) || s <= 0.0f) return F3{0.f, 0.f, 0.f};
    return c * s;
}
static __device__ F3 ggx_reflection_bsdfcos(F3 fres, F3 n, F3 view, F3 dir, float alpha)
{
    const float nov = dot(n, view), nol = dot(n, dir);
    if (nov <= 0.0f || nol <= 0.0f) return F3{0.f, 0.f, 0.f};
    const F3 h = safe_normalize(view + dir, n);
    const float scale = ggx_d(n, h, alpha) * ggx_g(nov, nol, alpha) / (4.0f * nov);
    return color_from_scale(clamp_color01(fres), scale);
}
__device__ __forceinline__ F3 ggx_schlick_bsdfcos(F3 f0, F3 n, F3 view, F3 dir, float alpha)
{
    const F3 h = safe_normalize(view + dir, n);
    const float voh = fmaxf(0.0f, dot(view, h));
    return ggx_reflection_bsdfcos(schlick(f0, voh), n, view, dir, alpha);
}
__device__ __forceinline__ F3 ggx_conductor_bsdfcos(F3 eta, F3 k, F3 n, F3 view, F3 dir, float alpha)
{
    const F3 h = safe_normalize(view + dir, n);
    const float voh = fmaxf(0.0f, dot(view, h));
    return ggx_reflection_bsdfcos(conductor_fresnel(eta, k, voh), n, view, dir, alpha);
}
static __device__ bool refract_dir(F3 inc, F3 m, float eta, F3& out)
{
    const float ct = fminf(1.0f, dot(inc * -1.0f, m));
    const F3 perp = eta * (inc + ct * m);
    const float pl2 = len2(perp);
    if (pl2 > 1.0f) return false;
    const F3 par = (-sqrtf(fmaxf(0.0f, 1.0f - pl2))) * m;
    out = safe_normalize(perp + par, reflect(inc, m));
    return len2(out) > 0.0f;
}
// Utilities::refract (include/luz/Utilities.hpp:55-62)
__device__ __forceinline__ F3 refract_smooth(F3 v, F3 n, float ratio)
{
    const float ct = fminf(dot(v * -1.0f, n), 1.0f);
    const F3 perp = ratio * (v + ct * n);
    const F3 par = (-sqrtf(fabsf(1.0f - len2(perp)))) * n;
    return perp + par;
}
__device__ __forceinline__ F3 oriented_half(F3 n, F3 h) { return dot(n, h) < 0.0f ? h * -1.0f : h; }
static __device__ float ggx_dielectric_pdf(F3 n, F3 view, F3 dir, float alpha, float ei, float et)
{
    const float nov = dot(n, view), nol = dot(n, dir);
    if (nov <= 0.0f || nol == 0.0f || ei <= 0.0f || et <= 0.0f) return 0.0f;
    if (nol > 0.0f) {
        const F3 h = safe_normalize(view + dir, n);
        const float F = dielectric_fresnel(dot(view, h), ei, et);
        return F * ggx_reflection_pdf(n, view, dir, alpha);
    }
    const float eta = ei / et;
    F3 h = safe_normalize(view + dir * eta, n);
    h = oriented_half(n, h);
    const float noh = dot(n, h), voh = dot(view, h), loh = dot(dir, h);
    if (noh <= 0.0f || voh <= 0.0f || loh >= 0.0f) return 0.0f;
    const float den = voh + eta * loh;
    if (fabsf(den) <= 1e-10f) return 0.0f;
    const float F = dielectric_fresnel(voh, ei, et);
    const float dh = fabsf((eta * eta * loh) / (den * den));
    const float pdf = (1.0f - F) * ggx_d(n, h, alpha) * noh * dh;
    return (isfinite(pdf) && pdf > 0.0f) ? pdf : 0.0f;
}
static __device__ F3 ggx_dielectric_bsdfcos(F3 color, F3 n, F3 view, F3 dir, float alpha, float ei, float et)
{
    const float nov = dot(n, view), nol = dot(n, dir);
    const F3 zero{0.f, 0.f, 0.f};
    if (nov <= 0.0f || nol == 0.0f || ei <= 0.0f || et <= 0.0f) return zero;
    color = clamp_color01(color);
    if (nol > 0.0f) {
        const F3 h = safe_normalize(view + dir, n);
        const float F = dielectric_fresnel(dot(view, h), ei, et);
        return ggx_reflection_bsdfcos(F3{F, F, F}, n, view, dir, alpha);
    }
    const float eta = ei / et;
    F3 h = safe_normalize(view + dir * eta, n);
    h = oriented_half(n, h);
    const float noh = dot(n, h), voh = dot(view, h), loh = dot(dir, h);
    if (noh <= 0.0f || voh <= 0.0f || loh >= 0.0f) return zero;
    const float den = voh + eta * loh;
    if (fabsf(den) <= 1e-10f) return zero;
    const float F = dielectric_fresnel(voh, ei, et);
    const float scale = (1.0f - F) * ggx_d(n, h, alpha) * ggx_g(nov, fabsf(nol), alpha) * eta * eta * fabsf(voh * loh)
                        / (nov * den * den);
    return color_from_scale(color, scale);
}

// ----------------------------------------------------------------------------- principled

struct PWeights {
    float w[7];
    float total;
};
__device__ __forceinline__ float lum_weight(F3 c)
{
    const float l = luminance(c);
    return (!isfinite(l) || l <= 0.0f) ? 0.0f : l;
}
__device__ __forceinline__ float principled_diffuse_scale(const GMaterial& m)
{
    return (1.0f - m.metallic) * (1.0f - m.transmission) * (1.0f - m.f0_diel) * (1.0f - 0.25f * m.clearcoat);
}
// componentWeights (Principled.cpp:159-205)
static __device__ PWeights principled_weights(const GMaterial& m, F3 base)
{
    PWeights r;
    const float bl = fmaxf(0.05f, lum_weight(base));
    const float diffuse = principled_diffuse_scale(m);
    const float dspec = (1.0f - m.metallic) * fmaxf(0.03f, m.f0_diel);
    const float ssw = diffuse * m.subsurface;
    const float sdiff = diffuse * (1.0f - m.subsurface);
    r.w[0] = sdiff * bl;
    r.w[1] = ssw * fmaxf(0.05f, lum_weight(base * f3(m.ss_color)));
    r.w[2] = diffuse * m.sheen * 0.35f;
    r.w[3] = dspec * (1.0f - 0.5f * m.transmission);
    r.w[4] = m.metallic * fmaxf(0.05f, bl);
    r.w[5] = (1.0f - m.metallic) * m.transmission;
    r.w[6] = m.clearcoat * 0.25f * (1.0f - 0.5f * m.roughness);
    r.total = 0.0f;
    for (int i = 0; i < 7; i++)
        if (isfinite(r.w[i]) && r.w[i] > 0.0f) r.total += r.w[i];
    if (r.total <= 0.0f) {
        r.w[0] = 1.0f;
        r.total = 1.0f;
    }
    return r;
}
static __device__ __noinline__ F3 principled_eval(const DScene& S, const GMaterial& m, const Hit& h, F3 ray_d, F3 dir)
{
    const F3 base = clamp_color01(color_at(S, m, h));
    const F3 view = safe_normalize(ray_d * -1.0f, h.n);
    const F3 n = h.n;
    const float transmission = m.transmission * (1.0f - m.metallic);
    const float diffuse = principled_diffuse_scale(m);
    F3 res{0.f, 0.f, 0.f};
    const float nol = dot(n, dir);
    {  // diffuse
        const float sc = diffuse * (1.0f - m.subsurface);
        if (!(nol <= 0.0f || sc <= 0.0f)) res = base * (sc * nol / kPiF);
    }
    {  // subsurface
        float nl = nol;
        if (m.flags & MF_THIN) nl = fabsf(nl);
        const float sc = diffuse * m.subsurface;
        if (!(nl <= 0.0f || sc <= 0.0f)) res = res + (base * f3(m.ss_color)) * (sc * nl / kPiF);
    }
    {  // sheen
        const float sc = diffuse * m.sheen;
        if (!(nol <= 0.0f || sc <= 0.0f)) {
            const F3 hv = safe_normalize(view + dir, n);
            const float fall = powf(1.0f - clamp01f(dot(dir, hv)), 5.0f);
            const F3 sheen = (F3{1.f, 1.f, 1.f} * (1.0f - 0.5f)) + (base * 0.5f);
            res = res + sheen * (sc * fall * nol / kPiF);
        }
    }
    {  // dielectric specular
        F3 c{0.f, 0.f, 0.f};
        if (!(nol <= 0.0f)) {
            const F3 hv = safe_normalize(view + dir, n);
            const float F = dielectric_fresnel(dot(view, hv), 1.0f, m.ior);
            c = ggx_reflection_bsdfcos(F3{F, F, F}, n, view, dir, m.alpha);
        }
        res = res + color_from_scale(c, 1.0f - m.metallic);
    }
    res = res + color_from_scale(ggx_schlick_bsdfcos(base, n, view, dir, m.alpha), m.metallic);
    if (nol < 0.0f && transmission > 0.0f) {
        const float ei = h.front ? 1.0f : m.ior, et = h.front ? m.ior : 1.0f;
        res = res + color_from_scale(ggx_dielectric_bsdfcos(base, n, view, dir, m.alpha, ei, et), transmission);
    }
    res = res + color_from_scale(ggx_schlick_bsdfcos(F3{0.04f, 0.04f, 0.04f}, n, view, dir, m.clearcoat_alpha),
                                 m.clearcoat * 0.25f);
    return res;
}
static __device__ __noinline__ float principled_pdf(const DScene& S, const GMaterial& m, const Hit& h, F3 ray_d, F3 dir)
{
    const F3 base = clamp_color01(color_at(S, m, h));
    const PWeights W = principled_weights(m, base);
    const F3 view = safe_normalize(ray_d * -1.0f, h.n);
    const F3 n = h.n;
    const float ei = h.front ? 1.0f : m.ior, et = h.front ? m.ior : 1.0f;
    float p[7];
    const float c = dot(n, dir);
    p[0] = c <= 0.0f ? 0.0f : c / kPiF;
    p[1] = (m.flags & MF_THIN) ? fabsf(c) / (2.0f * kPiF) : p[0];
    p[2] = p[0];
    p[3] = ggx_reflection_pdf(n, view, dir, m.alpha);
    p[4] = p[3];
    p[5] = c < 0.0f ? ggx_dielectric_pdf(n, view, dir, m.alpha, ei, et) : 0.0f;
    p[6] = ggx_reflection_pdf(n, view, dir, m.clearcoat_alpha);
    float pdf = 0.0f;
    for (int i = 0; i < 7; i++)
        if (W.w[i] > 0.0f && p[i] > 0.0f) pdf += (W.w[i] / W.total) * p[i];
    return (isfinite(pdf) && pdf > 0.0f) ? pdf : 0.0f;
}

// ----------------------------------------------------------------------------- scatter record

enum PdfType : int32_t { PDF_NONE = 0, PDF_COSINE = 1, PDF_SPHERE = 2, PDF_HG = 3, PDF_BSDF = 4 };

struct Scatter {
    bool specular;
    int32_t pdf;
    F3 att;
    F3 dir;            // specular ray direction, or BSDF sampled direction
    float spdf;
    F3 cos_w;          // cosine basis normal
    F3 phase;          // HG phase direction
    float g;
    bool absorb;
    F3 absorption;
    bool subsurface;
    bool thin;
    F3 ss_radius_m;
};

__device__ __forceinline__ F3 ray_dir_normalized(F3 d)   // Ray::_normalize (include/luz/Ray/Ray.hpp:60-73)
{
    const float l = sqrtf((d.x * d.x) + (d.y * d.y) + (d.z * d.z));
    if (!isfinite(l) || l <= 0.0f) return F3{0.f, 0.f, 0.f};
    return vdiv(d, l);
}

// Material::evaluateBSDFCos / scatteringPDF for the BSDF-typed materials.
static __device__ __noinline__ F3 bsdf_eval(const DScene& S, const GMaterial& m, const Hit& h, F3 ray_d, F3 dir)
{
    const F3 view = safe_normalize(ray_d * -1.0f, h.n);
    switch (m.type) {
    case MT_METAL:
        if (m.flags & MF_CONDUCTOR) return ggx_conductor_bsdfcos(f3(m.eta), f3(m.k), h.n, view, dir, m.alpha);
        return ggx_schlick_bsdfcos(clamp_color01(color_at(S, m, h)), h.n, view, dir, m.alpha);
    case MT_DIELECTRIC: {
        const float ei = h.front ? 1.0f : m.ior, et = h.front ? m.ior : 1.0f;
        return ggx_dielectric_bsdfcos(color_at(S, m, h), h.n, view, dir, m.alpha, ei, et);
    }
    case MT_PRINCIPLED:
        return principled_eval(S, m, h, ray_d, dir);
    case MT_GLOSSY:   // Glossy::evaluateBSDFCos (Glossy.cpp:86-100): GGX lobe tinted by the colour, no Fresnel
        return ggx_reflection_bsdfcos(clamp_color01(color_at(S, m, h)), h.n, view, dir, m.alpha);
    case MT_DIFFUSE_GLOSSY: {   // DiffuseGlossy::evaluateBSDFCos (DiffuseGlossy.cpp:144-160)
        const float nol = dot(h.n, dir);
        const F3 diffuse = nol <= 0.0f ? F3{0.f, 0.f, 0.f} : clamp_color01(color_at(S, m, h)) * (nol / kPiF);
        const F3 glossy = ggx_reflection_bsdfcos(clamp_color01(f3(m.gcolor)), h.n, view, dir, m.alpha);
        return (diffuse * (1.0f - m.gweight)) + (glossy * m.gweight);
    }
    default:
        return F3{0.f, 0.f, 0.f};
    }
}
static __device__ __noinline__ float bsdf_pdf(const DScene& S, const GMaterial& m, const Hit& h, F3 ray_d, F3 dir)
{
    const F3 view = safe_normalize(ray_d * -1.0f, h.n);
    switch (m.type) {
    case MT_METAL:
        return ggx_reflection_pdf(h.n, view, dir, m.alpha);
    case MT_DIELECTRIC: {
        const float ei = h.front ? 1.0f : m.ior, et = h.front ? m.ior : 1.0f;
        return ggx_dielectric_pdf(h.n, view, dir, m.alpha, ei, et);
    }
    case MT_PRINCIPLED:
        return principled_pdf(S, m, h, ray_d, dir);
    case MT_GLOSSY:
        return ggx_reflection_pdf(h.n, view, dir, m.alpha);
    case MT_DIFFUSE_GLOSSY: {   // DiffuseGlossy::scatteringPDF (DiffuseGlossy.cpp:162-176)
        const float c = dot(h.n, dir);
        const float dp = c <= 0.0f ? 0.0f : c / kPiF;
        return (dp * (1.0f - m.gweight)) + (ggx_reflection_pdf(h.n, view, dir, m.alpha) * m.gweight);
    }
    case MT_LAMBERTIAN: {
        const float c = dot(h.n, dir);
        return c < 0.0f ? 0.0f : c / kPiF;
    }
    case MT_ISOTROPIC:
    case MT_HG:
        return 1.0f / (4.0f * kPiF);
    default:
        return 0.0f;
    }
}

__device__ __forceinline__ F3 ggx_reflection_sample(F3 d, F3 n, float alpha, const Key& k)
{
    const F3 view = safe_normalize(d * -1.0f, n);
    F3 hv = sample_ggx_half(n, alpha, sample2d(k, DIM_BSDF_DIRECTION));
    if (dot(view, hv) <= 0.0f) hv = n;
    F3 dir = reflect(d, hv);
    if (dot(dir, n) <= 0.0f) dir = reflect(d, n);
    return dir;
}

__device__ __forceinline__ bool finish_bsdf(const DScene& S, const GMaterial& m, const Hit& h, F3 d, F3 dir, Scatter& sr)
{
    const float pdf = bsdf_pdf(S, m, h, d, dir);
    const F3 bc = bsdf_eval(S, m, h, d, dir);
    if (pdf <= 0.0f || !isfinite(pdf) || maxc(bc) <= 0.0f) return false;
    sr.dir = dir;
    sr.spdf = pdf;
    sr.att = cdiv(bc, pdf);
    sr.specular = false;
    sr.pdf = PDF_BSDF;
    return true;
}

// Material::scatter for every type on the path; false = no scatter (emitter or failed sample).
static __device__ __noinline__ bool scatter(const DScene& S, const GMaterial& m, const Hit& h, F3 d, const Key& k, Scatter& sr)
{
    sr.specular = false;
    sr.pdf = PDF_NONE;
    sr.absorb = false;
    sr.subsurface = false;
    sr.thin = false;
    switch (m.type) {
    case MT_LAMBERTIAN:
        sr.att = color_at(S, m, h);
        sr.pdf = PDF_COSINE;
        sr.cos_w = h.n;
        return true;
    case MT_ISOTROPIC:
        sr.att = color_at(S, m, h);
        sr.pdf = PDF_SPHERE;
        return true;
    case MT_HG:
        sr.att = color_at(S, m, h);
        sr.pdf = PDF_HG;
        sr.phase = len2(d) <= 0.0f ? F3{0.f, 0.f, 1.f} : normalize(d);
        sr.g = m.anisotropy;
        return true;
    case MT_METAL: {
        const F3 view = safe_normalize(d * -1.0f, h.n);
        const float ct = fminf(1.0f, fmaxf(0.0f, dot(view, h.n)));
        if (m.roughness <= 1e-4f) {
            sr.dir = ray_dir_normalized(reflect(d, h.n));
            sr.att = (m.flags & MF_CONDUCTOR) ? conductor_fresnel(f3(m.eta), f3(m.k), ct)
                                              : schlick(clamp_color01(color_at(S, m, h)), ct);
            sr.specular = true;
            return true;
        }
        return finish_bsdf(S, m, h, d, ggx_reflection_sample(d, h.n, m.alpha, k), sr);
    }
    case MT_DIELECTRIC: {
        sr.absorb = (m.flags & MF_ABSORPTION) != 0;
        sr.absorption = f3(m.absorption);
        const F3 view = safe_normalize(d * -1.0f, h.n);
        const float ei = h.front ? 1.0f : m.ior, et = h.front ? m.ior : 1.0f;
        const float ratio = ei / et;
        if (m.roughness <= 1e-4f) {
            const float ct = fminf(dot(view, h.n), 1.0f);
            const float st = sqrtf(1.0f - ct * ct);
            const bool cannot = ratio * st > 1.0f;
            F3 dir;
            if (cannot || (double)dielectric_fresnel(ct, ei, et) > sample1d(k, DIM_MATERIAL_DECISION)) {
                dir = reflect(d, h.n);
                sr.att = F3{1.f, 1.f, 1.f};
            } else {
                dir = refract_smooth(d, h.n, ratio);
                sr.att = color_at(S, m, h);
            }
            sr.specular = true;
            sr.dir = ray_dir_normalized(dir);
            return true;
        }
        F3 hv = sample_ggx_half(h.n, m.alpha, sample2d(k, DIM_BSDF_DIRECTION));
        if (dot(view, hv) <= 0.0f) hv = h.n;
        const float F = dielectric_fresnel(dot(view, hv), ei, et);
        F3 refr;
        const bool can = refract_dir(d, hv, ratio, refr);
        F3 dir;
        if (!can || sample1d(k, DIM_MATERIAL_DECISION) < (double)F) dir = reflect(d, hv);
        else dir = refr;
        return finish_bsdf(S, m, h, d, dir, sr);
    }
    case MT_GLOSSY:   // Glossy::scatter (Glossy.cpp:68-84)
        return finish_bsdf(S, m, h, d, ggx_reflection_sample(d, h.n, m.alpha, k), sr);
    case MT_DIFFUSE_GLOSSY: {   // DiffuseGlossy::scatter (DiffuseGlossy.cpp:118-142)
        F3 dir;
        if (sample1d(k, DIM_MATERIAL_DECISION) < (double)m.gweight) dir = ggx_reflection_sample(d, h.n, m.alpha, k);
        else dir = onb_local(make_onb(h.n), cosine_hemisphere(k, DIM_BSDF_DIRECTION));
        return finish_bsdf(S, m, h, d, dir, sr);
    }
    case MT_PRINCIPLED: {
        const F3 base = clamp_color01(color_at(S, m, h));
        sr.absorb = m.transmission > 0.0f && (m.flags & MF_ABSORPTION);
        sr.absorption = f3(m.absorption);
        if (m.flags & MF_SMOOTH_FULL_TRANSMISSION) {   // scatterSmoothTransmission
            const F3 view = safe_normalize(d * -1.0f, h.n);
            const float ei = h.front ? 1.0f : m.ior, et = h.front ? m.ior : 1.0f;
            const float ratio = ei / et;
            const float ct = fminf(1.0f, dot(view, h.n));
            const float st = sqrtf(fmaxf(0.0f, 1.0f - ct * ct));
            F3 dir;
            if (ratio * st > 1.0f || (double)dielectric_fresnel(ct, ei, et) > sample1d(k, DIM_MATERIAL_DECISION)) {
                dir = reflect(d, h.n);
                sr.att = F3{1.f, 1.f, 1.f};
            } else {
                dir = refract_smooth(d, h.n, ratio);
                sr.att = base;
            }
            sr.specular = true;
            sr.dir = ray_dir_normalized(dir);
            return true;
        }
        const PWeights W = principled_weights(m, base);
        double target = sample1d(k, DIM_MATERIAL_DECISION) * (double)W.total;
        int comp = 0;
        {
            bool found = false;
            for (int i = 0; i < 7; i++) {
                target -= (double)W.w[i];
                if (target <= 0.0) {
                    comp = i;
                    found = true;
                    break;
                }
            }
            if (!found) comp = 0;
        }
        F3 dir;
        if (comp == 0 || comp == 2 || comp == 1) {
            const Onb b = make_onb(h.n);
            F3 l = cosine_hemisphere(k, DIM_BSDF_DIRECTION);
            if (comp == 1 && (m.flags & MF_THIN) && sample1d(k, DIM_SUBSURFACE_THIN_SIDE) < 0.5) l.z = -l.z;
            dir = onb_local(b, l);
        } else if (comp == 5) {
            const F3 view = safe_normalize(d * -1.0f, h.n);
            const float ei = h.front ? 1.0f : m.ior, et = h.front ? m.ior : 1.0f;
            F3 hv = sample_ggx_half(h.n, m.alpha, sample2d(k, DIM_BSDF_DIRECTION));
            if (dot(view, hv) <= 0.0f) hv = h.n;
            F3 refr;
            dir = refract_dir(d, hv, ei / et, refr) ? refr : reflect(d, hv);
        } else if (comp == 6) {
            dir = ggx_reflection_sample(d, h.n, m.clearcoat_alpha, k);
        } else {
            dir = ggx_reflection_sample(d, h.n, m.alpha, k);
        }
        if (!finish_bsdf(S, m, h, d, dir, sr)) return false;
        sr.subsurface = comp == 1;
        sr.thin = sr.subsurface && (m.flags & MF_THIN);
        sr.ss_radius_m = f3(m.ss_radius_m);
        return true;
    }
    default:
        return false;   // Emissive and BASIC do not scatter
    }
}

// scatterPDFValue (ColorHelper.cpp:38-86)
static __device__ float scatter_pdf(const DScene& S, const Scatter& sr, const GMaterial& m, const Hit& h, F3 ray_d, F3 dir)
{
    switch (sr.pdf) {
    case PDF_COSINE: {
        const float c = dot(dir, normalize(sr.cos_w));
        return c <= 0.0f ? 0.0f : c / kPiF;
    }
    case PDF_SPHERE:
        return 1.0f / (4.0f * kPiF);
    case PDF_HG: {
        const float dl = len2(dir), pl = len2(sr.phase);
        if (dl <= 0.0f || pl <= 0.0f || !isfinite(dl) || !isfinite(pl)) return 0.0f;
        const F3 nd = vdiv(dir, sqrtf(dl));
        const F3 pd = vdiv(sr.phase, sqrtf(pl));
        const float ct = fmaxf(-1.0f, fminf(1.0f, dot(nd, pd)));
        const float g = fmaxf(-0.99f, fminf(0.99f, sr.g));
        const float g2 = g * g;
        const float den = fmaxf(1e-12f, 1.0f + g2 - (2.0f * g * ct));
        return (1.0f - g2) / (4.0f * kPiF * den * sqrtf(den));
    }
    case PDF_BSDF:
        return bsdf_pdf(S, m, h, ray_d, dir);
    default:
        return 0.0f;
    }
}
// scatterBSDFCos (ColorHelper.cpp:88-106)
static __device__ F3 scatter_bsdfcos(const DScene& S, const Scatter& sr, const GMaterial& m, const Hit& h, F3 ray_d, F3 dir)
{
    if (sr.pdf == PDF_BSDF) return bsdf_eval(S, m, h, ray_d, dir);
    return sr.att * scatter_pdf(S, sr, m, h, ray_d, dir);
}
// henyeyGreensteinDirection (ColorHelper.cpp:108-140)
static __device__ __noinline__ F3 hg_direction(const Scatter& sr, const Key& k)
{
    const float pl = len2(sr.phase);
    if (pl <= 0.0f || !isfinite(pl)) return sphere_direction(k, DIM_BSDF_DIRECTION);
    const F3 pd = vdiv(sr.phase, sqrtf(pl));
    const float g = fmaxf(-0.99f, fminf(0.99f, sr.g));
    const S2 s = sample2d(k, DIM_BSDF_DIRECTION);
    const float phi = 2.0f * kPiF * s.x;
    float ct;
    if (fabsf(g) < 1e-3f) {
        ct = 1.0f - (2.0f * s.y);
    } else {
        const float rm = (1.0f - (g * g)) / (1.0f - g + (2.0f * g * s.y));
        ct = (1.0f + (g * g) - (rm * rm)) / (2.0f * g);
        ct = fmaxf(-1.0f, fminf(1.0f, ct));
    }
    const float st = sqrtf(fmaxf(0.0f, 1.0f - (ct * ct)));
    return onb_local(make_onb(pd), st * cosf(phi), st * sinf(phi), ct);
}
// scatterPDFGenerate (ColorHelper.cpp:142-158)
static __device__ F3 scatter_generate(const Scatter& sr, const Key& k)
{
    switch (sr.pdf) {
    case PDF_COSINE:
        return onb_local(make_onb(sr.cos_w), cosine_hemisphere(k, DIM_BSDF_DIRECTION));
    case PDF_SPHERE:
        return sphere_direction(k, DIM_BSDF_DIRECTION);
    case PDF_HG:
        return hg_direction(sr, k);
    case PDF_BSDF:
        return sr.dir;
    default:
        return F3{0.f, 0.f, 0.f};
    }
}

// ----------------------------------------------------------------------------- atmosphere (FP64)

// planetaryHit (Atmosphere.cpp:310-341): both roots of a sphere at the origin.
__device__ __forceinline__ bool planet_hit(double radius, const double* o, const double* d, double& t0, double& t1)
{
    if (!isfinite(radius) || radius <= 0.0) return false;
    const double a = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
    if (!isfinite(a) || a <= 0.0) return false;
    const double hb = o[0] * d[0] + o[1] * d[1] + o[2] * d[2];
    const double c = (o[0] * o[0] + o[1] * o[1] + o[2] * o[2]) - radius * radius;
    const double disc = hb * hb - a * c;
    if (!isfinite(disc) || disc < 0.0) return false;
    const double sq = sqrt(fmax(0.0, disc));
    t0 = (-hb - sq) / a;
    t1 = (-hb + sq) / a;
    if (t0 > t1) {
        const double x = t0;
        t0 = t1;
        t1 = x;
    }
    return true;
}
__device__ __forceinline__ double atmos_density(double height, double inv_h)
{
    if (height < 0.0 || !isfinite(height)) return 0.0;
    return exp(-height * inv_h);
}
constexpr double kDblMax = 1.7976931348623157e308;   // T_MAX (Defaults.hpp:19)
// Atmosphere::sceneUnitsToMeters (Atmosphere.cpp:156-172)
__device__ __forceinline__ double to_meters(double su, double mpu)
{
    if (!isfinite(su)) return su;
    const double mx = kDblMax / mpu;
    if (su >= mx) return kDblMax;
    if (su <= -mx) return -kDblMax;
    return su * mpu;
}

struct AtmosSample {
    double in[3];   // in-scattering
    double tr[3];   // view transmittance
};

// Atmosphere::sampleSegment (Atmosphere.cpp:344-471): single-scattering
// Rayleigh + Mie along the ray up to t_max (scene units), midpoint samples on
// the view segment and on each sample's path to the sun.
static __device__ __noinline__ AtmosSample atmos_segment(const DScene& S, const double* ro, const double* d, double t_max)
{
    const GAtmos& A = S.k.atmos;
    AtmosSample out{{0.0, 0.0, 0.0}, {1.0, 1.0, 1.0}};
    const double mpu = S.k.meters_per_unit;
    if (!isfinite(t_max) || t_max <= 0.001) return out;
    const double tmax_m = to_meters(t_max, mpu), tmin_m = to_meters(0.001, mpu);
    if (!isfinite(tmax_m) || tmax_m <= tmin_m) return out;
    const double o[3] = {ro[0] * mpu, ro[1] * mpu, ro[2] * mpu};
    double a0, a1;
    if (!planet_hit(A.atmos_r, o, d, a0, a1) || a1 <= tmin_m) return out;
    double tmax = tmax_m, e0, e1;
    if (planet_hit(A.earth_r, o, d, e0, e1) && e1 > tmin_m) tmax = fmin(tmax, fmax(0.0, e0));
    const double tmin = fmax(tmin_m, a0);
    tmax = fmin(tmax, a1);
    if (!isfinite(tmin) || !isfinite(tmax) || tmax <= tmin) return out;
    const double seg = (tmax - tmin) / A.samples;
    if (!isfinite(seg) || seg <= 0.0) return out;
    const double bR[3] = {3.8e-6, 13.5e-6, 33.1e-6}, bM = 21e-6;   // Atmosphere::betaR / betaM
    const double g = 0.76;                                          // kMieG
    double sumR[3] = {0.0, 0.0, 0.0}, sumM[3] = {0.0, 0.0, 0.0};
    double odR = 0.0, odM = 0.0;
    const double mu = fmin(1.0, fmax(-1.0, d[0] * A.sun_dir[0] + d[1] * A.sun_dir[1] + d[2] * A.sun_dir[2]));
    const double mu2 = mu * mu;
    const double phR = (3.0 / (16.0 * kPiD)) * (1.0 + mu2);
    const double mb = fmax(1.0 + g * g - 2.0 * g * mu, 1.0e-6);
    const double md = mb * sqrt(mb);
    const double phM = (3.0 / (8.0 * kPiD)) * ((1.0 - g * g) * (1.0 + mu2) / ((2.0 + g * g) * md));
    for (int i = 0; i < A.samples; i++) {
        const double vt = tmin + ((double)i + 0.5) * seg;
        const double p[3] = {o[0] + vt * d[0], o[1] + vt * d[1], o[2] + vt * d[2]};
        const double h = sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]) - A.earth_r;
        const double dR = atmos_density(h, A.inv_hr), dM = atmos_density(h, A.inv_hm);
        if (dR == 0.0 && dM == 0.0) continue;
        const double sR = dR * seg, sM = dM * seg;
        odR += sR;
        odM += sM;
        double l0, l1;
        if (!planet_hit(A.atmos_r, p, A.sun_dir, l0, l1) || l1 <= 0.0) continue;
        const double segL = l1 / A.light_samples;
        if (!isfinite(segL) || segL <= 0.0) continue;
        double oLR = 0.0, oLM = 0.0;
        bool reaches = true;
        for (int j = 0; j < A.light_samples; j++) {
            const double lt = ((double)j + 0.5) * segL;
            const double q[3] = {p[0] + lt * A.sun_dir[0], p[1] + lt * A.sun_dir[1], p[2] + lt * A.sun_dir[2]};
            const double hl = sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]) - A.earth_r;
            if (hl < 0.0) {
                reaches = false;
                break;
            }
            oLR += atmos_density(hl, A.inv_hr) * segL;
            oLM += atmos_density(hl, A.inv_hm) * segL;
        }
        if (!reaches) continue;
        for (int c = 0; c < 3; c++) {
            const double tau = bR[c] * (odR + oLR) + (bM * 1.1) * (odM + oLM);   // kMieAbsorptionScale
            const double att = exp(-tau);
            sumR[c] += att * sR;
            sumM[c] += att * sM;
        }
    }
    for (int c = 0; c < 3; c++) {
        out.tr[c] = exp(-(bR[c] * odR + (bM * 1.1) * odM));
        out.in[c] = ((sumR[c] * bR[c]) * phR + (sumM[c] * bM) * phM) * A.sun_rad[c];
    }
    return out;
}

// primaryAtmosphereTMax (ColorHelper.cpp:624-643): a camera ray that hits the
// scene inside the planet still sees the atmosphere up to the ground.
__device__ __forceinline__ double primary_atmos_tmax(const DScene& S, const double* o, const double* d, double surface_t)
{
    if (!isfinite(surface_t) || surface_t <= 0.001) return surface_t;
    double t0, t1;
    if (!planet_hit(S.k.atmos.earth_r / S.k.meters_per_unit, o, d, t0, t1) || t1 <= 0.001) return surface_t;
    const double ground = fmax(0.0, t0);
    if (!isfinite(ground) || ground <= 0.001) return surface_t;
    return fmax(surface_t, ground);
}

// sampleProceduralStars (ColorHelper.cpp:568-589)
__device__ __forceinline__ float atmos_stars(const DScene& S, const Key& k, const double* in)
{
    if (sample1d(k, DIM_ATMOSPHERE) < 0.9996) return 0.0f;
    double diff = (S.k.atmos.stars - 0.2 + (0.4 * sample1d(k, DIM_ATMOSPHERE + 1))) - ((in[0] + in[1] + in[2]) / 3.0);
    diff = diff < 0.0 ? 0.0 : (diff > 1.0 ? 1.0 : diff);
    return (float)diff;
}

// ----------------------------------------------------------------------------- environment (FP64 index math)

__device__ __forceinline__ double wrap01d(double v)
{
    v = v - floor(v);
    if (v < 0.0) v += 1.0;
    return v;
}
__device__ __forceinline__ double clamp01d(double v) { return fmax(0.0, fmin(1.0, v)); }
__device__ __forceinline__ void env_dir_to_uv(const GEnv& E, F3 dir, double& u, double& v)
{
    const double dx = dir.x, dy = dir.y, dz = dir.z;
    const double l2 = (dx * dx) + (dy * dy) + (dz * dz);
    if (!isfinite(l2) || l2 <= 0.0) {
        u = 0.0;
        v = 0.5;
        return;
    }
    const double il = 1.0 / sqrt(l2);
    const double nx = il * dx, ny = il * dy, nz = il * dz;
    const double phi = atan2(nz, nx);
    const double y = fmin(fmax(ny, -1.0), 1.0);
    u = wrap01d(0.5 + (phi / (2.0 * kPiD)) + (E.rotation / 360.0));
    v = clamp01d(0.5 + (asin(y) / kPiD));
}
static __device__ LUZ_LIGHT_ATTR F3 env_lookup_uv(const DScene& S, double u, double v)
{
    const GEnv& E = S.k.env;
    u = wrap01d(u);
    v = clamp01d(v);
    const double x = (u * (double)E.width) - 0.5;
    const double y = ((1.0 - v) * (double)E.height) - 0.5;
    const long long xf = (long long)floor(x), yf = (long long)floor(y);
    auto wrap = [&](long long i) {
        i %= (long long)E.width;
        if (i < 0) i += E.width;
        return (int)i;
    };
    const int x0 = wrap(xf), x1 = wrap(xf + 1);
    const int y0 = (int)min(max(yf, 0ll), (long long)E.height - 1);
    const int y1 = (int)min(max(yf + 1, 0ll), (long long)E.height - 1);
    const float tx = (float)(x - floor(x)), ty = (float)(y - floor(y));
    auto px = [&](int xx, int yy) {
        const float4 c = __ldg(S.env_texels + (size_t)yy * E.width + xx);
        return F3{c.x, c.y, c.z};
    };
    const F3 top = (px(x0, y0) * (1.0f - tx)) + (px(x1, y0) * tx);
    const F3 bot = (px(x0, y1) * (1.0f - tx)) + (px(x1, y1) * tx);
    const F3 c = (top * (1.0f - ty)) + (bot * ty);
    return F3{isfinite(c.x) ? fmaxf(0.f, c.x) : 0.f, isfinite(c.y) ? fmaxf(0.f, c.y) : 0.f,
              isfinite(c.z) ? fmaxf(0.f, c.z) : 0.f};
}
static __device__ LUZ_LIGHT_ATTR F3 env_radiance(const DScene& S, F3 dir)   // sampleDirection
{
    double u, v;
    env_dir_to_uv(S.k.env, dir, u, v);
    return env_lookup_uv(S, u, v);
}
__device__ __forceinline__ float env_pdf_uv(const DScene& S, double u, double v)
{
    const GEnv& E = S.k.env;
    if (E.total_weight <= 0.0 || E.pdf_offset < 0) return 1.0f / (4.0f * kPiF);
    const long long x = min((long long)floor(wrap01d(u) * (double)E.width), (long long)E.width - 1);
    const long long y = min((long long)floor((1.0 - clamp01d(v)) * (double)E.height), (long long)E.height - 1);
    return (float)S.cdf[E.pdf_offset + y * E.width + x];
}
// EnvironmentMap::sampleDirection and ::pdf of one direction: both start from the same
// directionToUV(direction), so it is evaluated once.
static __device__ LUZ_LIGHT_ATTR void env_query(const DScene& S, F3 dir, bool want_rad, bool want_pdf, F3& rad, float& pdf)
{
    double u, v;
    env_dir_to_uv(S.k.env, dir, u, v);
    if (want_rad) rad = env_lookup_uv(S, u, v);
    if (want_pdf) pdf = env_pdf_uv(S, u, v);
}
static __device__ LUZ_LIGHT_ATTR float env_pdf(const DScene& S, F3 dir)
{
    const GEnv& E = S.k.env;
    if (E.total_weight <= 0.0 || E.pdf_offset < 0) return 1.0f / (4.0f * kPiF);
    double u, v;
    env_dir_to_uv(E, dir, u, v);
    const long long x = min((long long)floor(wrap01d(u) * (double)E.width), (long long)E.width - 1);
    const long long y = min((long long)floor((1.0 - clamp01d(v)) * (double)E.height), (long long)E.height - 1);
    return (float)S.cdf[E.pdf_offset + y * E.width + x];
}
struct LightSample {
    F3 dir;
    F3 emitted;
    float pdf;
    float tmax;
    bool valid;
    float scale;   // IES relative intensity of a sphere light sample (1 otherwise)
    int32_t light; // index of the sampled light (sample_light)
};

// IESProfile::candelaAt (IESProfile.cpp:231-299), FP64.
static __device__ double ies_candela(const DScene& S, const GIes& I, double vdeg, double hdeg)
{
    const double* va = S.cdf + I.offset;
    const double* ha = va + I.nv;
    const double* cd = ha + I.nh;
    const int nv = I.nv, nh = I.nh;
    if (!isfinite(vdeg) || vdeg < va[0] || vdeg > va[nv - 1]) return 0.0;
    int v0 = 0;
    while (v0 + 1 < nv && va[v0 + 1] < vdeg) v0++;
    const int v1 = min(v0 + 1, nv - 1);
    const double vspan = va[v1] - va[v0];
    const double vt = vspan > 0.0 ? (vdeg - va[v0]) / vspan : 0.0;
    int h0 = 0, h1 = 0;
    double ht = 0.0;
    if (nh > 1) {
        double hz = isfinite(hdeg) ? fmod(hdeg, 360.0) : 0.0;
        if (hz < 0.0) hz += 360.0;
        const double first = ha[0], last = ha[nh - 1];
        if (hz < first) hz += 360.0;
        if (hz > last && last >= 360.0) hz = fmin(hz, last);
        while (h0 + 1 < nh && ha[h0 + 1] < hz) h0++;
        if (h0 + 1 < nh) {
            h1 = h0 + 1;
            const double hspan = ha[h1] - ha[h0];
            ht = hspan > 0.0 ? (hz - ha[h0]) / hspan : 0.0;
        } else {
            h1 = 0;
            const double hspan = (first + 360.0) - ha[h0];
            ht = hspan > 0.0 ? (hz - ha[h0]) / hspan : 0.0;
        }
    }
    const double a = cd[h0 * nv + v0] * (1.0 - vt) + cd[h0 * nv + v1] * vt;
    const double b = cd[h1 * nv + v0] * (1.0 - vt) + cd[h1 * nv + v1] * vt;
    return a * (1.0 - ht) + b * ht;
}

// IESProfile::relativeIntensity (IESProfile.cpp:301-323) for emission direction e (FP64).
static __device__ __noinline__ float ies_relative(const DScene& S, const GLight& L, F3 e)
{
    const GIes I = S.ies[L.ies];
    if (!(I.mean_candela > 0.0) || !isfinite(I.mean_candela)) return 0.0f;
    auto norm_or = [](double x, double y, double z, double fx, double fy, double fz, double* o) {
        const double l2 = x * x + y * y + z * z;
        if (!isfinite(l2) || l2 <= 0.0) {
            o[0] = fx; o[1] = fy; o[2] = fz;
            return;
        }
        const double il = 1.0 / sqrt(l2);   // Vector3 / double is (1 / d) * v
        o[0] = il * x; o[1] = il * y; o[2] = il * z;
    };
    double ax[3], dr[3], tg[3];
    norm_or(L.ies_axis[0], L.ies_axis[1], L.ies_axis[2], 0.0, -1.0, 0.0, ax);
    norm_or((double)e.x, (double)e.y, (double)e.z, ax[0], ax[1], ax[2], dr);
    const double ct = fmin(1.0, fmax(-1.0, dr[0] * ax[0] + dr[1] * ax[1] + dr[2] * ax[2]));
    const double vdeg = acos(ct) * (180.0 / kPiD);
    const double hp[3] = {fabs(ax[1]) < 0.95 ? 0.0 : 1.0, fabs(ax[1]) < 0.95 ? 1.0 : 0.0, 0.0};
    norm_or(hp[1] * ax[2] - hp[2] * ax[1], hp[2] * ax[0] - hp[0] * ax[2], hp[0] * ax[1] - hp[1] * ax[0], 1.0, 0.0, 0.0, tg);
    const double bt[3] = {ax[1] * tg[2] - ax[2] * tg[1], ax[2] * tg[0] - ax[0] * tg[2], ax[0] * tg[1] - ax[1] * tg[0]};
    double hdeg = atan2(dr[0] * bt[0] + dr[1] * bt[1] + dr[2] * bt[2], dr[0] * tg[0] + dr[1] * tg[1] + dr[2] * tg[2])
                * (180.0 / kPiD) + L.ies_rotation;
    if (!isfinite(hdeg)) hdeg = 0.0;
    hdeg = fmod(hdeg, 360.0);
    if (hdeg < 0.0) hdeg += 360.0;
    return (float)(ies_candela(S, I, vdeg, hdeg) / I.mean_candela);
}
__device__ __forceinline__ double clamp_sample(double v)
{
    if (!isfinite(v) || v <= 0.0) return 0.0;
    if (v >= 1.0) return 0.99999999999999989;   // std::nextafter(1.0, 0.0)
    return v;
}
// EnvironmentMap::sample (EnvironmentMap.cpp:468-513)
static __device__ LUZ_LIGHT_ATTR bool env_sample(const DScene& S, const Key& k, F3& dir, F3& radiance, float& pdf)
{
    const GEnv& E = S.k.env;
    const double sel0 = sample1d(k, DIM_ENVIRONMENT_SELECTION);
    S2 j = sample2d(k, DIM_ENVIRONMENT_POINT);
    j.x = (float)clamp_sample((double)j.x);
    j.y = (float)clamp_sample((double)j.y);
    if (E.total_weight <= 0.0 || E.pdf_offset < 0) {
        const double z = 1.0 - (2.0 * (double)j.y);
        const double rr = sqrt(fmax(0.0, 1.0 - z * z));
        const double phi = 2.0 * kPiD * (double)j.x;
        dir = F3{(float)(rr * cos(phi)), (float)z, (float)(rr * sin(phi))};
        radiance = env_radiance(S, dir);
        pdf = 1.0f / (4.0f * kPiF);
        return true;
    }
    const double target = clamp_sample(sel0) * E.total_weight;
    const int64_t n = (int64_t)E.width * E.height;
    const double* cdf = S.cdf + E.cdf_offset;
    // std::lower_bound over the CDF, narrowed to the guide-table range of the
    // target's bucket (the answer provably lies inside it; same result, few loads).
    int64_t lo = 0, hi = n;
    if (E.guide_offset >= 0) {
        const int32_t* g = S.index_pool + E.guide_offset;
        const double fb = (target / E.total_weight) * (double)E.guide_count;
        const int64_t b = min(max((int64_t)floor(fb), (int64_t)0), (int64_t)E.guide_count - 1);
        lo = g[b];
        hi = g[E.guide_count + b];
    }
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (cdf[mid] < target) lo = mid + 1;
        else hi = mid;
    }
    if (lo >= n) lo = n - 1;
    const int64_t y = lo / E.width, x = lo % E.width;
    const double u = ((double)x + (double)j.x) / (double)E.width;
    const double v = 1.0 - (((double)y + (double)j.y) / (double)E.height);
    const double phi = (wrap01d(u - (E.rotation / 360.0)) - 0.5) * 2.0 * kPiD;
    const double yy = sin((clamp01d(v) - 0.5) * kPiD);
    const double rr = sqrt(fmax(0.0, 1.0 - yy * yy));
    dir = F3{(float)(rr * cos(phi)), (float)yy, (float)(rr * sin(phi))};
    env_query(S, dir, true, true, radiance, pdf);
    return pdf > 0.0f && isfinite(pdf);
}

// ----------------------------------------------------------------------------- lights

__device__ __forceinline__ int64_t lower_bound_d(const double* a, int64_t n, double target)
{
    int64_t lo = 0, hi = n;
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (a[mid] < target) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}
__device__ __forceinline__ int64_t upper_bound_d(const double* a, int64_t n, double target)
{
    int64_t lo = 0, hi = n;
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (!(target < a[mid])) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// Triangle::sampleSurface position (Triangle.cpp:288-305), leaf slot.
__device__ __forceinline__ F3 tri_point(const DScene& S, int32_t slot, const Key& k)
{
    const GTri T = load_tri(S.tris, (uint32_t)slot);
    const S2 s = sample2d(k, DIM_LIGHT_SURFACE_POINT);
    float u = s.x, v = s.y;
    if (u + v > 1.0f) {
        u = 1.0f - u;
        v = 1.0f - v;
    }
    return (f3(T.v0) + (f3(T.e1) * u)) + (f3(T.e2) * v);
}
// Mesh area CDF pick; returns leaf slot or -1 (Mesh.cpp:844-885).
static __device__ int32_t mesh_pick(const DScene& S, const GMesh& M, const Key& k, double& selected)
{
    if (M.tri_count <= 0 || M.total_area <= 0.0) return -1;
    const double* c = S.cdf + M.cdf_offset;
    const double target = sample1d(k, DIM_LIGHT_SURFACE_SELECTION) * M.total_area;
    int64_t idx = lower_bound_d(c, M.tri_count, target);
    if (idx > M.tri_count - 1) idx = M.tri_count - 1;
    const double prev = idx == 0 ? 0.0 : c[idx - 1];
    selected = c[idx] - prev;
    if (selected <= 0.0) return -1;
    return S.index_pool[M.slot_offset + idx];
}

static __device__ __noinline__ bool light_surface_sample(const DScene& S, const GLight& L, F3 origin, const Key& k, LightSample& ls)
{
    ls.valid = false;
    switch (L.kind) {
    case LK_RECT: {
        const GObject O = S.objects[L.object];
        const GRect R = S.rects[O.aux];
        const S2 s = sample2d(k, DIM_LIGHT_SURFACE_POINT);
        const F3 pt = (f3(R.p) + (f3(R.wa) * ((s.x - 0.5f) * R.w))) + (f3(R.ha) * ((s.y - 0.5f) * R.h));
        const F3 dir = pt - origin;
        const float d2 = len2(dir);
        if (!isfinite(d2) || d2 <= 0.0f) return false;
        const float dist = sqrtf(d2);
        ls.dir = vdiv(dir, dist);
        const float area = R.h * R.w;
        const float c = fabsf(dot(ls.dir, f3(R.n)));
        if (area <= 0.0f || c <= 0.0f) return false;
        ls.pdf = d2 / (c * area);
        ls.tmax = dist;
        return isfinite(ls.pdf) && ls.pdf > 0.0f;
    }
    case LK_SPHERE: {
        const GObject O = S.objects[L.object];
        const F3 c = f3(O.f);
        const float r = O.f[3];
        const F3 toc = c - origin;
        const float d2 = len2(toc);
        if (r <= 0.0f || !isfinite(d2) || d2 <= r * r) return false;
        const S2 s = sample2d(k, DIM_LIGHT_SURFACE_POINT);
        const float rr2 = (r * r) / d2;
        const float z = 1.0f + s.y * (sqrtf(fmaxf(0.0f, 1.0f - rr2)) - 1.0f);
        const float phi = kTwoPiF * s.x;
        const float rad = sqrtf(fmaxf(0.0f, 1.0f - z * z));
        F3 dir = onb_local(make_onb(toc), F3{cosf(phi) * rad, sinf(phi) * rad, z});
        const float dl2 = len2(dir);
        if (!isfinite(dl2) || dl2 <= 0.0f) return false;
        const float dl = sqrtf(dl2);
        dir = F3{dir.x / dl, dir.y / dl, dir.z / dl};
        const F3 oc = origin - c;
        const float a = len2(dir);
        const float b = dot(oc, dir);
        const F3 fq = oc - (b / a) * dir;   // b^2 - a(|oc|^2 - r^2) = a (r^2 - |oc - (b/a) dir|^2)
        const float disc = a * ((r * r) - len2(fq));
        if (disc < 0.0f) return false;
        const float sq = sqrtf(disc);
        float root = (-b - sq) / a;
        if (root < kTMin || root > kInf) root = (-b + sq) / a;
        if (root < kTMin || root > kInf) return false;
        const float ctm = sqrtf(1.0f - rr2);
        const float sa = 2.0f * kPiF * (rr2 / (1.0f + ctm));   // 2 pi (1 - cos theta_max), cancellation-free
        if (sa <= 0.0f || !isfinite(sa)) return false;
        ls.dir = dir;
        ls.pdf = 1.0f / sa;
        ls.tmax = root;
        if (L.ies >= 0) ls.scale = ies_relative(S, L, dir * -1.0f);
        return isfinite(ls.pdf) && ls.pdf > 0.0f && ls.tmax > kTMin;
    }
    case LK_MESH: {
        const GMesh M = S.meshes[L.mesh];
        double selected;
        const int32_t slot = mesh_pick(S, M, k, selected);
        if (slot < 0) return false;
        const GTri T = load_tri(S.tris, (uint32_t)slot);
        const F3 pt = tri_point(S, slot, k);
        const F3 dir = pt - origin;
        const float d2 = len2(dir);
        if (!isfinite(d2) || d2 <= 0.0f) return false;
        const float dist = sqrtf(d2);
        ls.dir = vdiv(dir, dist);
        const float4 fs = __ldg(reinterpret_cast<const float4*>(S.tri_shade + slot));
        const float c = fabsf(dot(ls.dir, F3{fs.x, fs.y, fs.z}));
        if (c <= 0.0f) return false;
        float pdf = d2 / (c * T.area);
        if (!(isfinite(pdf) && pdf > 0.0f)) return false;
        pdf = (float)((double)pdf * (selected / M.total_area));
        ls.pdf = pdf;
        ls.tmax = dist;
        return isfinite(pdf) && pdf > 0.0f;
    }
    case LK_INSTANCE: {
        const GObject O = S.objects[L.object];
        const GMesh M = S.meshes[L.mesh];
        if (L.area <= 0.0) return false;
        int32_t slot;
        if (L.uniform) {
            double selected;
            slot = mesh_pick(S, M, k, selected);
        } else {
            if (L.cdf_count <= 0) return false;
            const double* c = S.cdf + L.cdf_offset;
            const double target = sample1d(k, DIM_LIGHT_SURFACE_SELECTION) * L.area;
            int64_t idx = lower_bound_d(c, L.cdf_count, target);
            if (idx > L.cdf_count - 1) idx = L.cdf_count - 1;
            const double prev = idx == 0 ? 0.0 : c[idx - 1];
            if (c[idx] - prev <= 0.0) return false;
            slot = S.index_pool[M.slot_offset + idx];
        }
        if (slot < 0) return false;
        const F3 lp = tri_point(S, slot, k);
        const float4 fs = __ldg(reinterpret_cast<const float4*>(S.tri_shade + slot));
        const F3 sc = f3(O.f + 3);
        const F3 pos = fwd_rotate(O, lp * sc) + f3(O.f);
        const F3 nrm = transform_normal(O, F3{fs.x, fs.y, fs.z});
        if (!isfinite(pos.x) || !isfinite(pos.y) || !isfinite(pos.z) || len2(nrm) <= 0.0f) return false;
        const F3 dir = pos - origin;
        const float d2 = len2(dir);
        if (!isfinite(d2) || d2 <= 0.0f) return false;
        const float dist = sqrtf(d2);
        ls.dir = vdiv(dir, dist);
        const float c = fabsf(dot(ls.dir, nrm));
        if (!isfinite(c) || c <= 0.0f) return false;
        ls.pdf = (float)((double)d2 / ((double)c * L.area));
        ls.tmax = dist;
        return isfinite(ls.pdf) && ls.pdf > 0.0f && isfinite(ls.tmax) && ls.tmax > kTMin;
    }
    case LK_DIRECTIONAL: {
        const GObject O = S.objects[L.object];
        ls.dir = f3(O.f) * -1.0f;
        ls.pdf = 1.0f;
        ls.tmax = kInf;
        return len2(ls.dir) > 0.0f;
    }
    default:
        return false;
    }
}

// Hittable::pdfValue of light L toward direction vec from origin.
static __device__ __noinline__ float light_pdf_value(const DScene& S, const GLight& L, F3 origin, F3 vec)
{
    VolSample vs{nullptr, 0.0, true};
    switch (L.kind) {
    case LK_RECT: {
        const GObject O = S.objects[L.object];
        const GRect R = S.rects[O.aux];
        const TRay r = make_ray(origin, ray_dir_normalized(vec));
        float t;
        if (!rect_test(R, r, kTMin, kInf, t)) return 0.0f;
        const F3 n = dot(r.d, f3(R.n)) < 0.0f ? f3(R.n) : f3(R.n) * -1.0f;
        const float d2 = t * t * len2(vec);
        const float c = fabsf(dot(vec, n) / sqrtf(len2(vec)));
        return d2 / (c * (R.h * R.w));
    }
    case LK_SPHERE: {
        const GObject O = S.objects[L.object];
        const TRay r = make_ray(origin, ray_dir_normalized(vec));
        float t;
        if (!sphere_test(O, r, kTMin, kInf, t)) return 0.0f;
        const float rr2 = (O.f[3] * O.f[3]) / len2(f3(O.f) - origin);
        const float ctm = sqrtf(1.0f - rr2);
        return 1.0f / (2.0f * kPiF * (rr2 / (1.0f + ctm)));
    }
    case LK_MESH: {
        const GMesh M = S.meshes[L.mesh];
        if (M.tri_count <= 0 || M.total_area <= 0.0) return 0.0f;
        const TRay r = make_ray(origin, ray_dir_normalized(vec));
        float closest = kInf, u, v;
        int32_t slot;
        LocalStack<true> st;
        if (!mesh_closest<0u>(S, M, r, kTMin, closest, slot, u, v, -1, vs, st)) return 0.0f;
        F3 n, gn;
        bool front;
        float tu, tv;
        triangle_shading(S, M, slot, u, v, r.d, n, gn, front, tu, tv);
        const float d2 = closest * closest * len2(vec);
        const float c = fabsf(dot(vec, n) / sqrtf(len2(vec)));
        if (c <= 0.0f) return 0.0f;
        return (float)((double)d2 / ((double)c * M.total_area));
    }
    case LK_INSTANCE: {
        if (L.area <= 0.0) return 0.0f;
        const float vl = sqrtf(len2(vec));
        if (!isfinite(vl) || vl <= 0.0f) return 0.0f;
        const TRay r = make_ray(origin, ray_dir_normalized(vec));
        float closest = kInf;
        THit th{kInf, -1, 0, 0.f, 0.f};
        LocalStack<true> st;
        object_closest<TF_ALL>(S, L.object, r, kTMin, closest, th, vs, st);
        if (th.obj < 0) return 0.0f;
        const Hit h = make_hit(S, r, th);
        const float d2 = th.t * th.t * len2(vec);
        const float c = fabsf(dot(vec, h.gn) / vl);
        if (!isfinite(d2) || !isfinite(c) || c <= 0.0f) return 0.0f;
        return (float)((double)d2 / ((double)c * L.area));
    }
    default:
        return 0.0f;
    }
}

__device__ __forceinline__ float light_select_prob(const DScene& S, int32_t i)
{
    const int32_t n = S.k.light_count;
    if (n <= 0) return 0.0f;
    if (S.k.light_cdf_offset < 0) return (float)(1.0 / (double)n);
    const double* c = S.cdf + S.k.light_cdf_offset;
    const double prev = i == 0 ? 0.0 : c[i - 1];
    const double w = c[i] - prev;
    if (w <= 0.0 || S.k.light_total_weight <= 0.0) return 0.0f;
    return (float)(w / S.k.light_total_weight);
}
// lightPDFValue (ColorHelper.cpp:233-257)
static __device__ LUZ_LIGHT_ATTR float lights_pdf(const DScene& S, F3 origin, F3 dir)
{
    const int32_t n = S.k.light_count;
    if (n <= 0) return 0.0f;
    if (n == 1) return light_pdf_value(S, S.lights[0], origin, dir);
    float sum = 0.0f;
    for (int32_t i = 0; i < n; i++) sum += light_select_prob(S, i) * light_pdf_value(S, S.lights[i], origin, dir);
    return sum;
}
// selectLightIndex + sampleLight (ColorHelper.cpp:190-231, 925-971)
static __device__ LUZ_LIGHT_ATTR bool sample_light(const DScene& S, F3 origin, const Key& k, LightSample& ls)
{
    ls.valid = false;
    const int32_t n = S.k.light_count;
    if (n <= 0) return false;
    int32_t idx = 0;
    if (n > 1) {
        if (S.k.light_cdf_offset >= 0) {
            const double target = sample1d(k, DIM_LIGHT_SELECTION) * S.k.light_total_weight;
            idx = (int32_t)min(upper_bound_d(S.cdf + S.k.light_cdf_offset, n, target), (int64_t)n - 1);
        } else {
            idx = (int32_t)min((int64_t)(sample1d(k, DIM_LIGHT_SELECTION) * (double)n), (int64_t)n - 1);
        }
    }
    const float sel = light_select_prob(S, idx);
    if (sel <= 0.0f || !isfinite(sel)) return false;
    const GLight L = S.lights[idx];
    LightSample s;
    s.scale = 1.0f;
    if (!light_surface_sample(S, L, origin, k, s)) return false;
    ls.dir = s.dir;
    ls.pdf = s.pdf * sel;
    ls.tmax = s.tmax;
    if (ls.pdf <= 0.0f || ls.tmax <= kTMin || !isfinite(ls.pdf) || !(ls.tmax == ls.tmax)) return false;
    if (!isfinite(ls.tmax) && L.kind != LK_DIRECTIONAL) return false;
    ls.emitted = f3(L.emitted);
    if (L.ies >= 0) ls.emitted = ls.emitted * s.scale;
    if (maxc(ls.emitted) <= 0.0f) return false;
    ls.light = idx;
    ls.valid = true;
    return true;
}

}  // namespace luz
