// Caustic photon map on the device: photon emission and tracing
// (CausticPhotonMap::build, src/renderer/CausticPhotonMap.cpp:430-551), the
// grid-cell keys and table the map is looked up through, and the density
// estimate the path loop adds at diffuse hits (CausticPhotonMap::estimate,
// :553-618; called from ColorHelper.cpp:1263-1268).
//
// Layout: photons sorted by (cell, photon index), three float4 each
// (position + flux.r, normal + flux.g, incoming direction + flux.b); an
// open-addressing table maps a packed cell key to the cell's photon range, so
// a cell's photons are summed in the reference's per-cell order (photon index).
#pragma once

#include "shade.cuh"

namespace luz {

constexpr uint32_t kCausticSeedScramble = 0x6a09e667u;   // CAUSTIC_SEED_SCRAMBLE
constexpr uint32_t kCausticStream = 0x13579bdfu;         // CAUSTIC_STREAM
constexpr unsigned long long kEmptyCell = ~0ull;
constexpr double kCellBias = 1048576.0;                  // cells per axis in [-2^20, 2^20)

// gridKey (:403-410) packed into 63 bits: 21 bits per axis after a 2^20 bias.
// Returns false for a cell outside the packed range.
__host__ __device__ __forceinline__ bool pack_cell(double cx, double cy, double cz, unsigned long long& key)
{
    if (!(cx >= -kCellBias && cx < kCellBias && cy >= -kCellBias && cy < kCellBias && cz >= -kCellBias
          && cz < kCellBias))
        return false;
    key = ((unsigned long long)(int64_t)(cx + kCellBias) << 42) | ((unsigned long long)(int64_t)(cy + kCellBias) << 21)
        | (unsigned long long)(int64_t)(cz + kCellBias);
    return true;
}
__device__ __forceinline__ uint32_t cell_slot(unsigned long long key, uint32_t mask)
{
    return (uint32_t)(splitmix64(key) & mask);
}
// Photon range [begin, end) of a cell; empty when the cell holds none.
__device__ __forceinline__ uint2 cell_range(const DCaustics& C, unsigned long long key)
{
    uint32_t slot = cell_slot(key, C.mask);
    for (uint32_t probe = 0; probe <= C.mask; probe++) {
        const unsigned long long k = __ldg(C.cell_keys + slot);
        if (k == key) return __ldg(C.cell_ranges + slot);
        if (k == kEmptyCell) break;
        slot = (slot + 1) & C.mask;
    }
    return make_uint2(0u, 0u);
}

__device__ __forceinline__ bool valid_positive(F3 c)   // validPositiveColor (:29-37)
{
    return isfinite(c.x) && isfinite(c.y) && isfinite(c.z) && maxc(c) > 0.0f;
}
__device__ __forceinline__ bool receives_caustics(const GMaterial& m)   // materialReceivesCaustics (:225-232)
{
    return m.type != MT_EMISSIVE && !(m.flags & MF_TRANSPORT);
}

// HittableEmissionSample (include/luz/Hittables/Hittable.hpp:49-57).
struct Emission {
    F3 pos, n, dir, emitted;
    double power;
};

// Rectangle / Sphere / Triangle / MeshInstance / directional sampleEmission
// (Rectangle.cpp:421-454, Sphere.cpp:467-497, Mesh.cpp:942-985,
// Triangle.cpp:434-470, MeshInstance.cpp:549-582, CausticPhotonMap.cpp:279-326).
static __device__ __noinline__ bool light_emission(const DScene& S, const GLight& L, const Key& k, Emission& e)
{
    const F3 emitted = f3(L.emitted);
    switch (L.kind) {
    case LK_RECT: {
        const GObject O = S.objects[L.object];
        if (O.aux < 0) return false;
        const GRect R = S.rects[O.aux];
        const float area = R.h * R.w;
        if (area <= 0.0f || luminance(emitted) <= 0.0f) return false;
        const S2 s = sample2d(k, DIM_LIGHT_SURFACE_POINT);
        e.pos = (f3(R.p) + (f3(R.wa) * ((s.x - 0.5f) * R.w))) + (f3(R.ha) * ((s.y - 0.5f) * R.h));
        e.n = f3(R.n);
        if (sample1d(k, DIM_LIGHT_EMISSION_SIDE) < 0.5) e.n = e.n * -1.0f;
        e.dir = normalize(onb_local(make_onb(e.n), cosine_hemisphere(k, DIM_LIGHT_EMISSION_DIRECTION)));
        e.emitted = emitted;
        e.power = 2.0 * kPiD * (double)area;
        return len2(e.dir) > 0.0f;
    }
    case LK_SPHERE: {
        const GObject O = S.objects[L.object];
        const float r = O.f[3];
        if (r <= 0.0f || luminance(emitted) <= 0.0f) return false;
        const F3 out = normalize(sphere_direction(k, DIM_LIGHT_SURFACE_POINT));
        e.pos = f3(O.f) + out * r;
        e.n = out;
        e.dir = normalize(onb_local(make_onb(out), cosine_hemisphere(k, DIM_LIGHT_EMISSION_DIRECTION)));
        e.emitted = emitted;
        if (L.ies >= 0) e.emitted = e.emitted * ies_relative(S, L, e.dir);
        e.power = kPiD * 4.0 * kPiD * (double)r * (double)r;
        return luminance(e.emitted) > 0.0f && len2(e.dir) > 0.0f;
    }
    case LK_MESH: {
        const GMesh M = S.meshes[L.mesh];
        double selected;
        const int32_t slot = mesh_pick(S, M, k, selected);
        if (slot < 0) return false;
        const GTri T = load_tri(S.tris, (uint32_t)slot);
        if (T.area <= 0.0f || luminance(emitted) <= 0.0f) return false;
        e.pos = tri_point(S, slot, k);
        const float4 fs = __ldg(reinterpret_cast<const float4*>(S.tri_shade + slot));
        e.n = F3{fs.x, fs.y, fs.z};
        if (sample1d(k, DIM_LIGHT_EMISSION_SIDE) < 0.5) e.n = e.n * -1.0f;
        e.dir = normalize(onb_local(make_onb(e.n), cosine_hemisphere(k, DIM_LIGHT_EMISSION_DIRECTION)));
        e.emitted = emitted;
        e.power = 2.0 * kPiD * (double)T.area * (M.total_area / selected);
        return len2(e.dir) > 0.0f && isfinite(e.power) && e.power > 0.0;
    }
    case LK_INSTANCE: {
        if (luminance(emitted) <= 0.0f || L.area <= 0.0) return false;
        const GObject O = S.objects[L.object];
        const GMesh M = S.meshes[L.mesh];
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
        if (slot < 0 || load_tri(S.tris, (uint32_t)slot).area <= 0.0f) return false;
        const F3 lp = tri_point(S, slot, k);
        const float4 fs = __ldg(reinterpret_cast<const float4*>(S.tri_shade + slot));
        e.pos = fwd_rotate(O, lp * f3(O.f + 3)) + f3(O.f);
        e.n = transform_normal(O, F3{fs.x, fs.y, fs.z});
        if (!isfinite(e.pos.x) || !isfinite(e.pos.y) || !isfinite(e.pos.z) || len2(e.n) <= 0.0f) return false;
        if (sample1d(k, DIM_LIGHT_EMISSION_SIDE) < 0.5) e.n = e.n * -1.0f;
        F3 d = onb_local(make_onb(e.n), cosine_hemisphere(k, DIM_LIGHT_EMISSION_DIRECTION));
        const float dl2 = len2(d);
        e.dir = (isfinite(dl2) && dl2 > 0.0f) ? vdiv(d, sqrtf(dl2)) : F3{0.f, 0.f, 0.f};   // normalizedOrZero
        e.emitted = emitted;
        e.power = 2.0 * kPiD * L.area;
        return isfinite(e.power) && e.power > 0.0 && len2(e.dir) > 0.0f;
    }
    case LK_DIRECTIONAL: {
        const GCaustics& G = S.k.caustics;
        if (!valid_positive(emitted) || !G.has_bounds) return false;
        const GObject O = S.objects[L.object];
        const F3 dir = f3(O.f);
        const double R = G.disk_radius;
        float dx, dy;
        unit_disk(k, DIM_LIGHT_EMISSION_DIRECTION, dx, dy);
        const Onb b = make_onb(dir);
        const F3 off = onb_local(b, (float)(dx * R), (float)(dy * R), 0.0f);
        const double back = R + (double)kTMin;
        e.pos = F3{(float)(G.center[0] - dir.x * back), (float)(G.center[1] - dir.y * back),
                   (float)(G.center[2] - dir.z * back)} + off;
        e.n = dir * -1.0f;
        e.dir = dir;
        e.emitted = emitted;
        e.power = kPiD * R * R;
        return true;
    }
    default:
        return false;   // Hittable::sampleEmission
    }
}

// samplePhotonEmission (:328-354): light pick as selectLight / lightSelectionProbability.
__device__ __forceinline__ bool photon_emission(const DScene& S, const Key& k, Emission& e, double& sel)
{
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
    if (S.k.light_cdf_offset < 0) {
        sel = 1.0 / (double)n;
    } else {
        const double* c = S.cdf + S.k.light_cdf_offset;
        const double w = c[idx] - (idx == 0 ? 0.0 : c[idx - 1]);
        sel = w <= 0.0 ? 0.0 : w / S.k.light_total_weight;
    }
    if (!(sel > 0.0) || !isfinite(sel)) return false;
    return light_emission(S, S.lights[idx], k, e);
}

// applyRussianRoulette of the photon pass (:162-183).
__device__ __forceinline__ bool photon_roulette(F3& thr, int bounce, const Key& k)
{
    if (bounce < 3) return true;
    const float surv = fmaxf(0.05f, fminf(0.95f, maxc(thr)));
    if (sample1d(k, DIM_RUSSIAN_ROULETTE) > (double)surv) return false;
    thr = cdiv(thr, surv);
    return true;
}

// CausticPhotonMap::estimate (:553-618) at a diffuse hit with its scatter record.
static __device__ __noinline__ F3 caustic_estimate(const DScene& S, const Hit& h, const Scatter& sr, const GMaterial& m, F3 ray_d)
{
    const DCaustics& C = S.cm;
    const GCaustics& G = S.k.caustics;
    F3 sum{0.f, 0.f, 0.f};
    if (C.count == 0) return sum;
    const double r = G.radius_su;
    const double gx = floor((double)h.p.x / r), gy = floor((double)h.p.y / r), gz = floor((double)h.p.z / r);
    const float r2 = (float)(r * r);
    for (int z = -1; z <= 1; z++)
        for (int y = -1; y <= 1; y++)
            for (int x = -1; x <= 1; x++) {
                unsigned long long key;
                if (!pack_cell(gx + x, gy + y, gz + z, key)) continue;
                const uint2 rg = cell_range(C, key);
                for (uint32_t j = rg.x; j < rg.y; j++) {
                    const float4 a = __ldg(C.photons + 3 * (size_t)j);
                    const F3 off = F3{a.x, a.y, a.z} - h.p;
                    if (len2(off) > r2) continue;
                    const float4 b = __ldg(C.photons + 3 * (size_t)j + 1);
                    if (dot(h.n, F3{b.x, b.y, b.z}) <= 0.25f) continue;
                    const float4 c = __ldg(C.photons + 3 * (size_t)j + 2);
                    const F3 to_light = F3{c.x, c.y, c.z} * -1.0f;
                    const float cosine = fabsf(dot(h.n, to_light));
                    if (cosine <= 1e-6f) continue;
                    const F3 bc = scatter_bsdfcos(S, sr, m, h, ray_d, to_light);
                    if (!valid_positive(bc)) continue;
                    sum = sum + F3{a.w, b.w, c.w} * cdiv(bc, cosine);
                }
            }
    return cdiv(sum, (float)G.gather_area_m2);
}

}  // namespace luz
