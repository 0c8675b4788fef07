/*
 * restate.cpp — TEST INFRASTRUCTURE ONLY (the oracle's C restatement).
 *
 * A plain, single-threaded FP32 restatement of two pieces of the Luz reference,
 * written from the reference sources (not from the CUDA kernels):
 *   1. the Sampler stream            src/core/Sampler.cpp:31-237 (bit-exact: u64
 *      hashing and non-contracted double arithmetic, -ffp-contract=off);
 *   2. closest-hit / any-hit traversal of the packed scene arrays that the GPU
 *      library uploads (layout in luz_b200/csrc/layout.h), following
 *        Renderer::internal::_checkHits   src/renderer/HitHelper.cpp:5-32
 *        isShadowOccluded                 src/renderer/ColorHelper.cpp:801-829
 *        BVHNode::hit / hitAny            src/core/Hittables/BVHNode.cpp:221-380
 *        Mesh::hit / hitAny               src/core/Hittables/Mesh.cpp:578-735
 *        Triangle::hit                    src/core/Hittables/Triangle.cpp:196-305
 *        MeshInstance::_localRay / hit    src/core/Hittables/MeshInstance.cpp:245-327
 *        Rectangle/Sphere/Cube/Plane/ConstantVolume intersectors
 *      in FP32 with the reference's operation order. The GPU traversal must
 *      return the same (t, object, primitive, u, v) bit for bit on the same rays;
 *      this file in turn is checked against the reference's own hits (golden
 *      vectors from oracle/_ref) in tests/.
 * Only tests/ and __graft_entry__.smoke() use it, as the checker.
 */
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../luz_b200/csrc/layout.h"
#include "luz_gpu.h"

using namespace luz;

namespace {

/* ---------------------------------------------------------------- sampler */

uint64_t smix(uint64_t v)
{
    v += 0x9e3779b97f4a7c15ull;
    v = (v ^ (v >> 30)) * 0xbf58476d1ce4e5b9ull;
    v = (v ^ (v >> 27)) * 0x94d049bb133111ebull;
    return v ^ (v >> 31);
}
double u24(uint32_t h) { return (double)(h >> 8) * (1.0 / 16777216.0); }
double u53(uint64_t h) { return (double)(h >> 11) * (1.0 / 9007199254740992.0); }
uint32_t h32(uint64_t v) { return (uint32_t)(smix(v) >> 32); }
double frac(double v) { return v - std::floor(v); }

struct Ctx {
    uint64_t base;
    uint32_t sample, bounce;
};
Ctx begin(uint32_t seed, uint32_t x, uint32_t y, uint32_t s, uint32_t stream, uint32_t bounce)
{
    Ctx c;
    c.base = seed;
    c.base ^= ((uint64_t)x + 1ull) * 0xbf58476d1ce4e5b9ull;
    c.base ^= ((uint64_t)y + 1ull) * 0x94d049bb133111ebull;
    c.base ^= ((uint64_t)stream + 1ull) * 0xda942042e4dd58b5ull;
    c.sample = s;
    c.bounce = bounce;
    return c;
}
double step(uint32_t d, uint32_t c)
{
    const uint64_t key = ((uint64_t)d + 1ull) * 0x9e3779b97f4a7c15ull ^ ((uint64_t)c + 1ull) * 0xda942042e4dd58b5ull;
    double s = u24(h32(key));
    if (s < 0.05 || s > 0.95) s = frac(s + 0.6180339887498948);
    return s;
}
bool prog(uint32_t d)
{
    const uint32_t b = d % 32u;
    return b == 0 || b == 1 || b == 4 || b == 5 || b == 12 || b == 13 || b == 16;
}
uint64_t ckey(const Ctx& c, uint32_t dk) { return c.base ^ (((uint64_t)dk + 1ull) * 0x9e3779b97f4a7c15ull); }
double hsample(const Ctx& c, uint32_t dk, uint32_t comp)
{
    uint64_t k = ckey(c, dk);
    k ^= ((uint64_t)c.sample + 1ull) * 0x94d049bb133111ebull;
    k ^= ((uint64_t)comp + 1ull) * 0xbf58476d1ce4e5b9ull;
    return u53(smix(k));
}
double s1(const Ctx& c, uint32_t dim)
{
    const uint32_t dk = dim + c.bounce * 32u;
    if (!prog(dim)) return hsample(c, dk, 0);
    const double shift = u24(h32(ckey(c, dk)));
    return frac(0.5 + ((double)c.sample + 1.0) * step(dk, 0) + shift);
}
void s2(const Ctx& c, uint32_t dim, float* out)
{
    const uint32_t dk = dim + c.bounce * 32u;
    if (!prog(dim)) {
        out[0] = (float)hsample(c, dk, 0);
        out[1] = (float)hsample(c, dk, 1);
        return;
    }
    const uint64_t k = ckey(c, dk);
    const double sx = u24(h32(k)), sy = u24(h32(k ^ 0xda942042e4dd58b5ull));
    const double smp = (double)c.sample + 1.0;
    out[0] = (float)frac(0.5 + smp * step(dk, 0) + sx);
    out[1] = (float)frac(0.5 + smp * step(dk, 1) + sy);
}

/* ---------------------------------------------------------------- traversal */

struct Scene {
    const GTopNode* tn;
    const GTopChild* tc;
    const GObject* ob;
    const GNode* nd;
    const GTri* tr;
    const GMesh* me;
    const GRect* rc;
    const int32_t* pool;
    const GSceneConst* k;
};

struct Ray {
    float o[3], d[3], iv[3];
    bool zero;
};

const float TMIN = 0.001f;
const float INF = INFINITY;

float dotf(const float* a, const float* b) { return (a[0] * b[0]) + (a[1] * b[1]) + (a[2] * b[2]); }
void crossf(const float* a, const float* b, float* r)
{
    r[0] = (a[1] * b[2]) - (a[2] * b[1]);
    r[1] = (a[2] * b[0]) - (a[0] * b[2]);
    r[2] = (a[0] * b[1]) - (a[1] * b[0]);
}
float invc(float c)
{
    if (c == 0.0f || !std::isfinite(c)) return 0.0f;
    const float i = 1.0f / c;
    return std::isfinite(i) ? i : 0.0f;
}
Ray mkray(const float* o, const float* d)
{
    Ray r;
    for (int a = 0; a < 3; a++) {
        r.o[a] = o[a];
        r.d[a] = d[a];
        r.iv[a] = invc(d[a]);
    }
    r.zero = d[0] == 0.0f && d[1] == 0.0f && d[2] == 0.0f;
    return r;
}

/* boxHitDistance (Mesh.cpp:99-139) */
bool box(const float* mn, const float* mx, const Ray& r, float tmax, float* near)
{
    if (r.zero) return false;
    float tmin = TMIN;
    for (int a = 0; a < 3; a++) {
        const float iv = r.iv[a];
        if (iv == 0.0f) {
            if (r.o[a] < mn[a] || r.o[a] > mx[a]) return false;
            continue;
        }
        float t0 = (mn[a] - r.o[a]) * iv, t1 = (mx[a] - r.o[a]) * iv;
        if (iv < 0.0f) std::swap(t0, t1);
        tmin = t0 > tmin ? t0 : tmin;
        tmax = t1 < tmax ? t1 : tmax;
        if (tmax <= tmin) return false;
    }
    *near = tmin;
    return true;
}

/* The mesh-box slab test of the GPU traversal when the ray has no zero inverse
 * component, |o| < 4096 and the mesh lies within 8192 units of the origin:
 * t = fma(plane, inv, -(o * inv)); interval max(TMIN, mins) / min(tmax, maxes). */
struct Slabs {
    bool fast;
    float iv[3], noi[3];
};
Slabs mesh_slabs(const GMesh& M, const Ray& r)
{
    Slabs s{};
    float om = 0.f, mm = 0.f;
    bool axis0 = false;
    for (int a = 0; a < 3; a++) {
        om = std::fmax(om, std::fabs(r.o[a]));
        mm = std::fmax(mm, std::fmax(std::fabs(M.bmin[a]), std::fabs(M.bmax[a])));
        axis0 = axis0 || r.iv[a] == 0.0f;
        s.iv[a] = r.iv[a];
        s.noi[a] = -(r.o[a] * r.iv[a]);
    }
    s.fast = !r.zero && !axis0 && om < 4096.0f && mm < 8192.0f;
    return s;
}
bool mbox(const float* mn, const float* mx, const Ray& r, const Slabs& s, float tmax, float* near)
{
    if (!s.fast) return box(mn, mx, r, tmax, near);
    float lo = TMIN, hi = tmax;
    for (int a = 0; a < 3; a++) {
        const float t0 = std::fma(mn[a], s.iv[a], s.noi[a]), t1 = std::fma(mx[a], s.iv[a], s.noi[a]);
        lo = std::fmax(lo, std::fmin(t0, t1));
        hi = std::fmin(hi, std::fmax(t0, t1));
    }
    *near = lo;
    return !(hi <= lo);
}

/* Triangle::hit (Triangle.cpp:196-232) */
bool tri(const GTri& T, const Ray& r, float tmin, float tmax, float* t, float* u, float* v)
{
    float p[3], q[3], tv[3];
    crossf(r.d, T.e2, p);
    const float det = dotf(T.e1, p);
    if (std::fabs(det) < 1e-12f) return false;
    const float id = 1.0f / det;
    for (int a = 0; a < 3; a++) tv[a] = r.o[a] - T.v0[a];
    *u = dotf(tv, p) * id;
    if (*u < 0.0f || *u > 1.0f) return false;
    crossf(tv, T.e1, q);
    *v = dotf(r.d, q) * id;
    if (*v < 0.0f || *u + *v > 1.0f) return false;
    *t = dotf(T.e2, q) * id;
    return !(*t > tmax || *t < tmin);
}

struct Hit {
    float t;
    int32_t obj, prim;
    float u, v;
};

/* Mesh::hit (Mesh.cpp:578-660) */
bool mesh_hit(const Scene& S, const GMesh& M, const Ray& r, float tmin, float* closest, Hit* h, int32_t oi)
{
    float rn;
    const Slabs sl = mesh_slabs(M, r);
    if (!mbox(M.bmin, M.bmax, r, sl, *closest, &rn)) return false;
    std::vector<std::pair<uint32_t, float>> st;
    st.push_back({(uint32_t)M.root_ref, rn});
    bool any = false;
    while (!st.empty()) {
        const auto e = st.back();
        st.pop_back();
        if (e.second >= *closest) continue;
        if (e.first & kLeafBit) {
            const uint32_t first = (e.first & 0x7fffffffu) >> 3, cnt = (e.first & 7u) + 1u;
            for (uint32_t i = first; i < first + cnt; i++) {
                float t, u, v;
                if (tri(S.tr[i], r, tmin, *closest, &t, &u, &v)) {
                    *closest = t;
                    *h = Hit{t, oi, (int32_t)S.tr[i].orig, u, v};
                    any = true;
                }
            }
            continue;
        }
        const GNode& n = S.nd[e.first];
        float ln = 0.f, rnn = 0.f;
        const bool hl = mbox(n.lmin, n.lmax, r, sl, *closest, &ln);
        const bool hr = mbox(n.rmin, n.rmax, r, sl, *closest, &rnn);
        if (hl && hr) {
            if (ln < rnn) {
                st.push_back({n.rref, rnn});
                st.push_back({n.lref, ln});
            } else {
                st.push_back({n.lref, ln});
                st.push_back({n.rref, rnn});
            }
        } else if (hl) {
            st.push_back({n.lref, ln});
        } else if (hr) {
            st.push_back({n.rref, rnn});
        }
    }
    return any;
}

/* Mesh::hitAny (Mesh.cpp:662-735) */
bool mesh_any(const Scene& S, const GMesh& M, const Ray& r, float tmin, float tmax)
{
    float rn;
    const Slabs sl = mesh_slabs(M, r);
    if (!mbox(M.bmin, M.bmax, r, sl, tmax, &rn)) return false;
    std::vector<uint32_t> st{(uint32_t)M.root_ref};
    while (!st.empty()) {
        const uint32_t e = st.back();
        st.pop_back();
        if (e & kLeafBit) {
            const uint32_t first = (e & 0x7fffffffu) >> 3, cnt = (e & 7u) + 1u;
            for (uint32_t i = first; i < first + cnt; i++) {
                float t, u, v;
                if (tri(S.tr[i], r, tmin, tmax, &t, &u, &v)) return true;
            }
            continue;
        }
        const GNode& n = S.nd[e];
        float ln = 0.f, rnn = 0.f;
        const bool hl = mbox(n.lmin, n.lmax, r, sl, tmax, &ln), hr = mbox(n.rmin, n.rmax, r, sl, tmax, &rnn);
        if (hl && hr) {
            if (ln < rnn) {
                st.push_back(n.rref);
                st.push_back(n.lref);
            } else {
                st.push_back(n.lref);
                st.push_back(n.rref);
            }
        } else if (hl) {
            st.push_back(n.lref);
        } else if (hr) {
            st.push_back(n.rref);
        }
    }
    return false;
}

/* Rectangle::hit test (Rectangle.cpp:212-249) */
bool rect(const GRect& R, const Ray& r, float tmin, float tmax, float* t)
{
    if (R.w <= 0.0f || R.h <= 0.0f) return false;
    float op[3];
    for (int a = 0; a < 3; a++) op[a] = r.o[a] - R.p[a];
    const float a = dotf(op, R.n), b = dotf(r.d, R.n);
    if (b == 0.0f || (a < 0.0f && b < 0.0f) || (a > 0.0f && b > 0.0f)) return false;
    *t = -a / b;
    if (*t > tmax || *t < tmin) return false;
    float dd[3];
    for (int k = 0; k < 3; k++) dd[k] = (r.o[k] + (*t * r.d[k])) - R.p[k];
    return !(std::fabs(dotf(dd, R.wa)) > R.hw || std::fabs(dotf(dd, R.ha)) > R.hh);
}

/* Sphere::hit (Sphere.cpp:227-263) */
bool sphere(const GObject& O, const Ray& r, float tmin, float tmax, float* t)
{
    if (O.f[4] == 0.0f || r.zero) return false;
    float oc[3];
    for (int a = 0; a < 3; a++) oc[a] = r.o[a] - O.f[a];
    const float b = dotf(oc, r.d);
    float f[3];
    for (int a = 0; a < 3; a++) f[a] = oc[a] - b * r.d[a];
    const float disc = (O.f[3] * O.f[3]) - dotf(f, f);   // = b^2 - (|oc|^2 - r^2) for a unit direction
    if (disc < 0.0f) return false;
    const float sq = std::sqrt(disc);
    float root = -b - sq;
    if (root < tmin || root > tmax) {
        root = -b + sq;
        if (root < tmin || root > tmax) return false;
    }
    *t = root;
    return true;
}

bool plane(const GObject& O, const Ray& r, float tmin, float tmax, float* t)
{
    const float pos[3] = {0.0f, O.f[0], 0.0f};
    const float d = dotf(r.d, O.f + 1);
    if (d == 0.0f) return false;
    float pmo[3];
    for (int a = 0; a < 3; a++) pmo[a] = pos[a] - r.o[a];
    *t = dotf(pmo, O.f + 1) / d;
    return !(*t > tmax || *t < tmin);
}

/* MeshInstance::_localRay (MeshInstance.cpp:245-265) */
bool local_ray(const GObject& O, const Ray& r, Ray* lr, float* scale)
{
    const float cx = O.f[6], sx = O.f[7], cy = O.f[8], sy = O.f[9], cz = O.f[10], sz = O.f[11];
    if (!(std::fabs(O.f[3]) > 1e-12f && std::fabs(O.f[4]) > 1e-12f && std::fabs(O.f[5]) > 1e-12f)) return false;
    auto inv_rot = [&](const float* v, float* out) {
        float x = v[0], y = v[1], z = v[2];
        float nx = (x * cz) + (y * sz), ny = (-x * sz) + (y * cz);
        x = nx;
        y = ny;
        nx = (x * cy) - (z * sy);
        float nz = (x * sy) + (z * cy);
        x = nx;
        z = nz;
        ny = (y * cx) + (z * sx);
        nz = (-y * sx) + (z * cx);
        out[0] = x;
        out[1] = ny;
        out[2] = nz;
    };
    float ur[3], ld[3], om[3], uo[3], lo[3];
    inv_rot(r.d, ur);
    for (int a = 0; a < 3; a++) ld[a] = ur[a] / O.f[3 + a];
    *scale = std::sqrt((ld[0] * ld[0]) + (ld[1] * ld[1]) + (ld[2] * ld[2]));
    if (!std::isfinite(*scale) || *scale <= 0.0f) return false;
    for (int a = 0; a < 3; a++) om[a] = r.o[a] - O.f[a];
    inv_rot(om, uo);
    for (int a = 0; a < 3; a++) lo[a] = uo[a] / O.f[3 + a];
    if (!std::isfinite(lo[0]) || !std::isfinite(lo[1]) || !std::isfinite(lo[2])) return false;
    const float is = 1.0f / *scale;
    float nd[3] = {is * ld[0], is * ld[1], is * ld[2]};
    *lr = mkray(lo, nd);
    return true;
}

/* ConstantVolume::sampleScatteringDistance (ConstantVolume.cpp:62-105) */
bool volume(const GObject& O, const Ray& r, float tmin, float tmax, double u, float* t)
{
    float entry, exit;
    if (O.aux == LUZ_OBJ_CUBE) {
        float imin = -INF, imax = INF;
        for (int a = 0; a < 3; a++) {
            if (r.d[a] == 0.0f) {
                if (r.o[a] < O.f[a] || r.o[a] > O.f[3 + a]) return false;
                continue;
            }
            const float iv = 1.0f / r.d[a];
            float t0 = (O.f[a] - r.o[a]) * iv, t1 = (O.f[3 + a] - r.o[a]) * iv;
            if (t0 > t1) std::swap(t0, t1);
            imin = std::fmax(imin, t0);
            imax = std::fmin(imax, t1);
            if (imin >= imax) return false;
        }
        entry = imin;
        exit = imax;
    } else {
        if (r.zero) return false;
        float oc[3];
        for (int a = 0; a < 3; a++) oc[a] = r.o[a] - O.f[a];
        const float b = dotf(oc, r.d);
        float f[3];
        for (int a = 0; a < 3; a++) f[a] = oc[a] - b * r.d[a];
        const float disc = (O.f[3] * O.f[3]) - dotf(f, f);
        if (disc < 0.0f) return false;
        const float sq = std::sqrt(disc);
        float r0 = -b - sq, r1 = -b + sq;
        if (r0 > r1) std::swap(r0, r1);
        if (r0 >= r1) return false;
        entry = r0;
        exit = r1;
    }
    if (entry < tmin) entry = tmin;
    if (exit > tmax) exit = tmax;
    if (entry >= exit) return false;
    if (entry < 0.0f) entry = 0.0f;
    const float len = std::sqrt((r.d[0] * r.d[0]) + (r.d[1] * r.d[1]) + (r.d[2] * r.d[2]));
    if (len <= 0.0f || !std::isfinite(len)) return false;
    const float inside = (exit - entry) * len;
    const float hd = (float)((double)O.f[6] * std::log(std::fmax(u, 1e-12)));
    if (hd > inside) return false;
    *t = entry + hd / len;
    return true;
}

void obj_hit(const Scene& S, int32_t oi, const Ray& r, float tmin, float* closest, Hit* h, double vu)
{
    const GObject& O = S.ob[oi];
    float t;
    switch (O.kind) {
    case OK_RECT:
        if (rect(S.rc[O.aux], r, tmin, *closest, &t)) {
            *closest = t;
            *h = Hit{t, oi, 0, 0.f, 0.f};
        }
        break;
    case OK_CUBE:
        for (int f = 0; f < 6; f++)
            if (rect(S.rc[O.aux + f], r, tmin, *closest, &t)) {
                *closest = t;
                *h = Hit{t, oi, f, 0.f, 0.f};
            }
        break;
    case OK_SPHERE:
        if (sphere(O, r, tmin, *closest, &t)) {
            *closest = t;
            *h = Hit{t, oi, 0, 0.f, 0.f};
        }
        break;
    case OK_PLANE:
        if (plane(O, r, tmin, *closest, &t)) {
            *closest = t;
            *h = Hit{t, oi, 0, 0.f, 0.f};
        }
        break;
    case OK_MESH:
        mesh_hit(S, S.me[O.aux], r, tmin, closest, h, oi);
        break;
    case OK_INSTANCE: {
        Ray lr;
        float s;
        if (!local_ray(O, r, &lr, &s)) break;
        float lc = *closest * s;
        Hit lh{};
        if (!mesh_hit(S, S.me[O.aux], lr, tmin * s, &lc, &lh, oi)) break;
        const float wt = lc / s;
        if (!std::isfinite(wt) || wt < tmin || wt > *closest) break;
        *closest = wt;
        *h = Hit{wt, oi, lh.prim, lh.u, lh.v};
        break;
    }
    case OK_VOLUME:
        if (volume(O, r, tmin, *closest, vu, &t)) {
            *closest = t;
            *h = Hit{t, oi, 0, 0.f, 0.f};
        }
        break;
    default:
        break;
    }
}

bool obj_any(const Scene& S, int32_t oi, const Ray& r, float tmin, float tmax, double vu)
{
    const GObject& O = S.ob[oi];
    float t;
    switch (O.kind) {
    case OK_RECT:
        return rect(S.rc[O.aux], r, tmin, tmax, &t);
    case OK_CUBE:
        for (int f = 0; f < 6; f++)
            if (rect(S.rc[O.aux + f], r, tmin, tmax, &t)) return true;
        return false;
    case OK_SPHERE:
        return sphere(O, r, tmin, tmax, &t);
    case OK_PLANE:
        return plane(O, r, tmin, tmax, &t);
    case OK_MESH:
        return mesh_any(S, S.me[O.aux], r, tmin, tmax);
    case OK_INSTANCE: {
        Ray lr;
        float s;
        if (!local_ray(O, r, &lr, &s)) return false;
        return mesh_any(S, S.me[O.aux], lr, tmin * s, tmax * s);
    }
    case OK_VOLUME:
        return volume(O, r, tmin, tmax, vu, &t);
    default:
        return false;
    }
}

/* BVHNode::hit recursion (BVHNode.cpp:221-324), written recursively as in the reference. */
void top_hit(const Scene& S, int32_t node, const Ray& r, float tmin, float* closest, Hit* h, double vu)
{
    const GTopNode& N = S.tn[node];
    float dummy;
    if (!box(N.bmin, N.bmax, r, *closest, &dummy)) return;
    const int n = N.child_count;
    const GTopChild* C = S.tc + N.child_start;
    auto visit = [&](const GTopChild& c) {
        if (c.is_node) top_hit(S, c.ref, r, tmin, closest, h, vu);
        else obj_hit(S, c.ref, r, tmin, closest, h, vu);
    };
    if (n != 2 && n <= 3) {
        for (int i = 0; i < n; i++) visit(C[i]);
        return;
    }
    if (n == 2) {
        float n0 = 0.f, n1 = 0.f;
        const bool h0 = box(C[0].bmin, C[0].bmax, r, *closest, &n0);
        const bool h1 = box(C[1].bmin, C[1].bmax, r, *closest, &n1);
        int fi = 0, si = 1;
        float fn = n0, sn = n1;
        if (h0 && h1 && n1 < n0) {
            std::swap(fn, sn);
            std::swap(fi, si);
        }
        if (fi == 0 ? h0 : h1) visit(C[fi]);
        if ((si == 0 ? h0 : h1) && sn < *closest) visit(C[si]);
        return;
    }
    int ord[16];
    float on[16];
    int cnt = 0;
    for (int i = 0; i < n; i++) {
        float cn;
        if (!box(C[i].bmin, C[i].bmax, r, *closest, &cn)) continue;
        int j = cnt;
        while (j > 0 && on[j - 1] > cn) {
            on[j] = on[j - 1];
            ord[j] = ord[j - 1];
            j--;
        }
        on[j] = cn;
        ord[j] = i;
        cnt++;
    }
    for (int j = 0; j < cnt; j++) {
        if (on[j] >= *closest) continue;
        visit(C[ord[j]]);
    }
}

bool top_any(const Scene& S, int32_t node, const Ray& r, float tmin, float tmax, double vu)
{
    const GTopNode& N = S.tn[node];
    float dummy;
    if (!box(N.bmin, N.bmax, r, tmax, &dummy)) return false;
    const int n = N.child_count;
    const GTopChild* C = S.tc + N.child_start;
    const bool test = !(n != 2 && n <= 3);
    for (int i = 0; i < n; i++) {
        float cn;
        if (test && !box(C[i].bmin, C[i].bmax, r, tmax, &cn)) continue;
        if (C[i].is_node ? top_any(S, C[i].ref, r, tmin, tmax, vu) : obj_any(S, C[i].ref, r, tmin, tmax, vu))
            return true;
    }
    return false;
}

}  // namespace

extern "C" {

int restate_sample1d(uint32_t seed, int32_t x, int32_t y, int32_t s, uint32_t stream, uint32_t bounce, uint32_t dim,
                     double* out)
{
    *out = s1(begin(seed, (uint32_t)x, (uint32_t)y, (uint32_t)s, stream, bounce), dim);
    return 0;
}

int restate_sample2d(uint32_t seed, int32_t x, int32_t y, int32_t s, uint32_t stream, uint32_t bounce, uint32_t dim,
                     float* out)
{
    s2(begin(seed, (uint32_t)x, (uint32_t)y, (uint32_t)s, stream, bounce), dim, out);
    return 0;
}

/* rays: (ox,oy,oz,tmin,dx,dy,dz,tmax) float32; out: LuzHit with object = desc
 * object index, primitive = mesh triangle id / cube face. */
int restate_trace(const void* top_nodes, const void* top_children, const void* objects, const void* mesh_nodes,
                  const void* tris, const void* meshes, const void* rects, const void* index_pool, const void* consts,
                  const float* rays, int64_t n, int32_t any, uint32_t seed, const int32_t* vkey, LuzHit* out)
{
    Scene S{(const GTopNode*)top_nodes, (const GTopChild*)top_children, (const GObject*)objects,
            (const GNode*)mesh_nodes,   (const GTri*)tris,               (const GMesh*)meshes,
            (const GRect*)rects,        (const int32_t*)index_pool,      (const GSceneConst*)consts};
    const GSceneConst& K = *S.k;
    for (int64_t i = 0; i < n; i++) {
        const float* rr = rays + 8 * i;
        const Ray r = mkray(rr, rr + 4);
        const Ctx c = vkey ? begin(seed, (uint32_t)vkey[4 * i], (uint32_t)vkey[4 * i + 1], (uint32_t)vkey[4 * i + 2], 0,
                                   (uint32_t)vkey[4 * i + 3])
                           : begin(seed, 0, 0, 0, 0, 0);
        const double vu = s1(c, 10 /* DIM_VOLUME_DISTANCE */);
        if (any) {
            bool occ = false;
            if (rr[7] > TMIN) {
                if (K.accel_kind == 2) occ = obj_any(S, K.accel_object, r, rr[3], rr[7], vu);
                else if (K.accel_kind == 1) occ = top_any(S, 0, r, rr[3], rr[7], vu);
                for (int u = 0; !occ && u < K.unaccel_count; u++)
                    occ = obj_any(S, S.pool[K.unaccel_offset + u], r, rr[3], rr[7], vu);
            }
            out[i] = LuzHit{0.f, occ ? 0 : -1, 0, 0.f, 0.f};
            continue;
        }
        float closest = rr[7];
        Hit h{INF, -1, 0, 0.f, 0.f};
        if (K.accel_kind == 2) obj_hit(S, K.accel_object, r, rr[3], &closest, &h, vu);
        else if (K.accel_kind == 1) top_hit(S, 0, r, rr[3], &closest, &h, vu);
        for (int u = 0; u < K.unaccel_count; u++) obj_hit(S, S.pool[K.unaccel_offset + u], r, rr[3], &closest, &h, vu);
        if (h.obj < 0) out[i] = LuzHit{INF, -1, -1, 0.f, 0.f};
        else out[i] = LuzHit{h.t, S.ob[h.obj].id, h.prim, h.u, h.v};
    }
    return 0;
}

}  // extern "C"
