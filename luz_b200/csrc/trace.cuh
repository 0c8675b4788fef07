// trace.cuh — closest-hit and any-hit traversal of the two-level scene.
//
// Semantics follow the reference exactly (tie order included):
//   Renderer::internal::_checkHits          src/renderer/HitHelper.cpp:5-32
//   isShadowOccluded                        src/renderer/ColorHelper.cpp:801-829
//   BVHNode::hit / hitAny                   src/core/Hittables/BVHNode.cpp:221-380
//     1 or 3 children: index order, each child does its own test;
//     2 children: near-first, swap only on strict <, second needs near < closest;
//     >= 4 children: stable insertion sort by near, skip near >= closest.
//   Mesh::hit / hitAny                      src/core/Hittables/Mesh.cpp:578-735
//     explicit stack, prune near >= closest, ties push the right child last
//     (visited first); leaf triangles in order, later equal-t triangle wins.
//   Triangle::hit (Moller-Trumbore)         src/core/Hittables/Triangle.cpp:196-305
//   MeshInstance::hit / hitAny              src/core/Hittables/MeshInstance.cpp:251-327
//   Rectangle / Sphere / Cube / Plane / ConstantVolume intersectors.
// Arithmetic is FP32 with the reference's operation order (-fmad=false), so
// oracle/restate.cpp reproduces every hit bit for bit on the same packed arrays.
#pragma once
#include "dmath.cuh"

namespace luz {

// Caustic photon map of the current render (caustics.cuh): photons in grid-cell
// order, three float4 each, and an open-addressing table from packed cell key
// to the cell's [begin, end) photon range. count = 0: no map.
struct DCaustics {
    const float4* photons;
    const unsigned long long* cell_keys;
    const uint2* cell_ranges;
    uint32_t mask;
    uint32_t count;
};

struct DScene {
    const GRect* rects;
    const GObject* objects;
    const GTopNode* top_nodes;
    const GTopChild* top_children;
    const GNode4* nodes4;      // collapsed mesh BVH
    const GTri* tris;
    const GTriShade* tri_shade;
    const float* vnormals;
    const float* vuvs;
    const GMesh* meshes;
    const GMaterial* materials;
    const GTexture* textures;
    const float4* texels;
    const GLight* lights;
    const GIes* ies;
    const double* cdf;
    const int32_t* index_pool;
    const float4* env_texels;
    const uint8_t* obj_class;  // material type a hit on each object shades with (shade binning)
    uint32_t* error;          // device error word (bit flags)
    unsigned long long* counters;   // LUZ_RENDER_COUNT: ext nodes/tris/top, shadow nodes/tris/top,
                                    // ext / shadow binary-node visits (read by the counting
                                    // instantiations of the trace kernels only)
    int32_t mesh_stack_limit;       // traversal stack bounds enforced (<= kMeshStack4 / kTopStack;
    int32_t top_stack_limit;        // lowered only by luz_gpu_scene_set_traversal_limits)
    uint32_t top4_base;             // staged nodes: [top4_base, top4_base + top4_count) of nodes4, the
    uint32_t top4_count;            // breadth-first top of the scene's largest mesh (0: none)
    DCaustics cm;
    GSceneConst k;
};

enum ErrBits : uint32_t { ERR_TOP_STACK = 1u, ERR_MESH_STACK = 2u, ERR_CAUSTIC_GRID = 4u };

// Scene features a traversal kernel is instantiated for (GSceneConst.features).
// A kernel compiled without a feature never meets that object kind in its
// scene. (Analytic primitives are always compiled in: an instantiation with
// meshes as its only kind measured 2.3x slower in the any-hit kernel, at 2.4
// instead of 6.1 active threads per warp instruction.)
// TF_STAGED: the kernel has staged the scene's top collapsed nodes in shared
// memory (stage_top_nodes) and the mesh walks read them there.
enum TraceFeature : uint32_t { TF_INSTANCE = 1u, TF_VOLUME = 2u, TF_ALL = 3u, TF_STAGED = 4u };

// The staged nodes (kTopNodes4 x 160 B) of a trace kernel's block.
static __shared__ float4 s_top4[kTopNodes4 * 10];

// Copies the staged node range into shared memory; every thread of the block calls it
// once, before its first traversal.
__device__ __forceinline__ void stage_top_nodes(const DScene& S)
{
    const float4* src = reinterpret_cast<const float4*>(S.nodes4 + S.top4_base);
    for (uint32_t i = threadIdx.x; i < S.top4_count * 10u; i += blockDim.x) s_top4[i] = __ldg(src + i);
    __syncthreads();
}

// xobj / xprim name the primitive a secondary ray leaves from. A ray that
// starts on a planar primitive cannot meet it again at t > 0 in exact
// arithmetic (the reference's FP64 hits never do, they fall below T_MIN), so
// the FP32 traversal skips that primitive instead of re-hitting it through
// rounding error at grazing angles; for the source sphere an outgoing ray
// skips it and an entering ray keeps only the far root.
struct TRay {
    F3 o, d, inv;
    bool zero;
    bool axis0;      // some inverse-direction component is 0 (axis-parallel ray)
    int32_t xobj, xprim;
};

__device__ __forceinline__ float inv_component(float c)
{
    if (c == 0.0f || !isfinite(c)) return 0.0f;
    const float i = 1.0f / c;
    return isfinite(i) ? i : 0.0f;
}
__device__ __forceinline__ TRay make_ray(F3 o, F3 d)
{
    TRay r;
    r.o = o;
    r.d = d;
    r.inv = F3{inv_component(d.x), inv_component(d.y), inv_component(d.z)};
    r.zero = (d.x == 0.0f && d.y == 0.0f && d.z == 0.0f);
    r.axis0 = r.inv.x == 0.0f || r.inv.y == 0.0f || r.inv.z == 0.0f;
    r.xobj = -1;
    r.xprim = -1;
    return r;
}
__device__ __forceinline__ TRay make_ray_x(F3 o, F3 d, int32_t xobj, int32_t xprim)
{
    TRay r = make_ray(o, d);
    r.xobj = xobj;
    r.xprim = xprim;
    return r;
}

struct THit {
    float t;
    int32_t obj;     // GObject index, -1 = miss
    int32_t prim;    // mesh: leaf slot of the triangle; cube: face; else 0
    float u, v;
};

// Per-ray traversal context: the volume distance sample (evaluated once, on
// first use) and counts of the records read (mesh nodes, triangles, top-level
// nodes/children/objects), used for the algorithmic-bytes roofline.
struct VolSample {
    const Key* key;
    double u;
    bool have;
    uint32_t nodes = 0, tris = 0, top = 0;
    uint32_t bnodes = 0;   // binary-tree node visits the collapsed walk stands for
    __device__ __forceinline__ double get()
    {
        if (!have) {
            u = sample1d(*key, DIM_VOLUME_DISTANCE);
            have = true;
        }
        return u;
    }
};

// boxHitDistance / AABB::hit (Mesh.cpp:99-139, BVHNode.cpp:20-60, AABB.cpp:37-71).
// For a ray with no zero inverse component the per-axis swap and the running
// max/min are written as selects (same values as the reference's sequence: the
// early exit on tmax <= tmin is monotone, so testing once at the end is equal).
__device__ __forceinline__ bool box_hit(const float* mn, const float* mx, const TRay& r, float tmax, float& tnear)
{
    if (r.zero) return false;
    float tmin = kTMin;
    const float o[3] = {r.o.x, r.o.y, r.o.z};
    const float iv[3] = {r.inv.x, r.inv.y, r.inv.z};
    if (!r.axis0) {
#pragma unroll
        for (int a = 0; a < 3; a++) {
            const float t0 = (mn[a] - o[a]) * iv[a];
            const float t1 = (mx[a] - o[a]) * iv[a];
            tmin = fmaxf(tmin, fminf(t0, t1));
            tmax = fminf(tmax, fmaxf(t0, t1));
        }
        tnear = tmin;
        return !(tmax <= tmin);
    }
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const float inv = iv[a];
        if (inv == 0.0f) {
            if (o[a] < mn[a] || o[a] > mx[a]) return false;
            continue;
        }
        float t0 = (mn[a] - o[a]) * inv;
        float t1 = (mx[a] - o[a]) * inv;
        if (inv < 0.0f) {
            const float sw = t0;
            t0 = t1;
            t1 = sw;
        }
        tmin = t0 > tmin ? t0 : tmin;
        tmax = t1 < tmax ? t1 : tmax;
        if (tmax <= tmin) return false;
    }
    tnear = tmin;
    return true;
}

__device__ __forceinline__ float fmax3f(float a, float b, float c)
{
    float d;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}
__device__ __forceinline__ float fmin3f(float a, float b, float c)
{
    float d;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}

// Mesh-box slab test in the form t = plane * inv + noi with noi = -(o * inv)
// rounded once per ray: one FMA per plane instead of a subtraction and a
// product, and three-input min/max for the running interval. Equal to
// box_hit in real arithmetic; in FP32 each distance is off by less than
// 2^-24 (|o| + |t d|) / |d| along its axis, below the T_MIN padding of every
// mesh box (Triangle.cpp:114-125) while |o| < 4096 and the mesh lies within
// 8192 units of the origin: mesh_fast_slabs checks both.
__device__ __forceinline__ bool mesh_fast_slabs(const GMesh& M, const TRay& r)
{
    const float om = fmax3f(fabsf(r.o.x), fabsf(r.o.y), fabsf(r.o.z));
    const float mm = fmaxf(fmax3f(fabsf(M.bmin[0]), fabsf(M.bmin[1]), fabsf(M.bmin[2])),
                           fmax3f(fabsf(M.bmax[0]), fabsf(M.bmax[1]), fabsf(M.bmax[2])));
    return !r.zero && !r.axis0 && om < 4096.0f && mm < 8192.0f;
}
__device__ __forceinline__ F3 neg_o_inv(const TRay& r)
{
    return F3{-(r.o.x * r.inv.x), -(r.o.y * r.inv.y), -(r.o.z * r.inv.z)};
}
__device__ __forceinline__ bool box_hit_fast(const float* mn, const float* mx, const TRay& r, const F3& noi, float tmax,
                                             float& tnear)
{
    const float t0x = fmaf(mn[0], r.inv.x, noi.x), t1x = fmaf(mx[0], r.inv.x, noi.x);
    const float t0y = fmaf(mn[1], r.inv.y, noi.y), t1y = fmaf(mx[1], r.inv.y, noi.y);
    const float t0z = fmaf(mn[2], r.inv.z, noi.z), t1z = fmaf(mx[2], r.inv.z, noi.z);
    const float lo = fmax3f(fmaxf(kTMin, fminf(t0x, t1x)), fminf(t0y, t1y), fminf(t0z, t1z));
    const float hi = fmin3f(fminf(tmax, fmaxf(t0x, t1x)), fmaxf(t0y, t1y), fmaxf(t0z, t1z));
    tnear = lo;
    return !(hi <= lo);
}
// Mesh box test: the FMA form (FAST) or box_hit. noi = neg_o_inv(r) (FAST only).
template <bool FAST>
__device__ __forceinline__ bool mesh_box(const float* mn, const float* mx, const TRay& r, const F3& noi, float tmax,
                                         float& tnear)
{
    if constexpr (FAST) return box_hit_fast(mn, mx, r, noi, tmax, tnear);
    else return box_hit(mn, mx, r, tmax, tnear);
}

__device__ __forceinline__ bool tri_test(const GTri& T, const TRay& r, float tmin, float tmax, float& t, float& u, float& v)
{
    const F3 e1 = f3(T.e1), e2 = f3(T.e2), v0 = f3(T.v0);
    const F3 p = cross(r.d, e2);
    const float det = dot(e1, p);
    if (fabsf(det) < 1e-12f) return false;
    const float inv_det = 1.0f / det;
    const F3 tv = r.o - v0;
    u = dot(tv, p) * inv_det;
    if (u < 0.0f || u > 1.0f) return false;
    const F3 q = cross(tv, e1);
    v = dot(r.d, q) * inv_det;
    if (v < 0.0f || u + v > 1.0f) return false;
    t = dot(e2, q) * inv_det;
    return !(t > tmax || t < tmin);
}

__device__ __forceinline__ GTri load_tri(const GTri* tris, uint32_t i)
{
    const float4* p = reinterpret_cast<const float4*>(tris + i);
    const float4 a = ld4(p), b = ld4(p + 1), c = ld4(p + 2);
    GTri t;
    t.v0[0] = a.x; t.v0[1] = a.y; t.v0[2] = a.z; t.orig = __float_as_uint(a.w);
    t.e1[0] = b.x; t.e1[1] = b.y; t.e1[2] = b.z; t.area = b.w;
    t.e2[0] = c.x; t.e2[1] = c.y; t.e2[2] = c.z; t.pad = 0;
    return t;
}
__device__ __forceinline__ GNode4 load_node4(const GNode4* nodes, uint32_t i)
{
    const float4* p = reinterpret_cast<const float4*>(nodes + i);
    float4 v[10];
#pragma unroll
    for (int k = 0; k < 10; k++) v[k] = ld4(p + k);
    GNode4 n;
    float* f = reinterpret_cast<float*>(&n);
#pragma unroll
    for (int k = 0; k < 10; k++) {
        f[4 * k] = v[k].x;
        f[4 * k + 1] = v[k].y;
        f[4 * k + 2] = v[k].z;
        f[4 * k + 3] = v[k].w;
    }
    return n;
}

// The entry part of a GNode4 (its four entry boxes and refs, without the two
// side boxes): what the any-hit walk reads, seven of the ten 16-byte loads.
struct GNode4C {
    float cmin[4][3];
    float cmax[4][3];
    uint32_t ref[4];
};
static_assert(offsetof(GNode4, cmin) == 48 && offsetof(GNode4, ref) == 144 && sizeof(GNode4) == 160,
              "GNode4 layout: the entry loads start at byte 48");
static_assert(sizeof(GNode4C) == 112, "GNode4C is the last 112 bytes of a GNode4");
__device__ __forceinline__ GNode4C load_node4_entries(const GNode4* nodes, uint32_t i)
{
    const float4* p = reinterpret_cast<const float4*>(nodes + i) + 3;   // skips lmin..rmax (48 B)
    float4 v[7];
#pragma unroll
    for (int k = 0; k < 7; k++) v[k] = ld4(p + k);
    GNode4C n;
    float* f = reinterpret_cast<float*>(&n);
#pragma unroll
    for (int k = 0; k < 7; k++) {
        f[4 * k] = v[k].x;
        f[4 * k + 1] = v[k].y;
        f[4 * k + 2] = v[k].z;
        f[4 * k + 3] = v[k].w;
    }
    return n;
}

// Visit order of a collapsed node's entries, as the binary near-first
// traversal (Mesh::hit, Mesh.cpp:578-660) would reach them: the nearer of L
// and R first (ties: R), and within each the nearer child first (ties: the
// right one). mesh_closest_walk computes each accepted entry's position in
// this order.
//
// Testing all boxes at N's visit instead of at L's and R's gives the same
// visits: L is visited right after N (nothing changes `closest` in between),
// and an entry of R's side that the binary traversal would reject later,
// because `closest` shrank meanwhile, has near >= closest by then and is
// pruned when popped. Child boxes lie inside their parent's (the node boxes
// are unions of their triangles' boxes, rounded outward), so a grandchild's
// entry distance is never below its parent's and a grandchild of a rejected
// child is itself rejected.

// Mesh traversal stack in the thread's local memory: node or leaf reference
// and near distance per entry; NEAR = false drops the distances (any-hit never
// prunes on them). (A variant holding the top 8-32 entries in a shared-memory
// tile, one bank per thread, measured no faster on B200.)
template <bool NEAR>
struct LocalStack {
    uint32_t r[kMeshStack4];
    float n[NEAR ? kMeshStack4 : 1];
    __device__ __forceinline__ void set(int d, uint32_t ref, float near)
    {
        r[d] = ref;
        if constexpr (NEAR) n[d] = near;
    }
    __device__ __forceinline__ uint32_t ref(int d) const { return r[d]; }
    __device__ __forceinline__ float near(int d) const
    {
        if constexpr (NEAR) return n[d];
        else return 0.0f;
    }
};

// A collapsed node from the staged copy when it lies in the staged range, else from
// global memory (the same bytes either way).
template <uint32_t F>
__device__ __forceinline__ GNode4 fetch_node4(const DScene& S, uint32_t ref)
{
    if constexpr ((F & TF_STAGED) != 0) {
        const uint32_t j = ref - S.top4_base;
        if (j < S.top4_count) {
            GNode4 n;
            float4* d = reinterpret_cast<float4*>(&n);
#pragma unroll
            for (int k = 0; k < 10; k++) d[k] = s_top4[10 * j + k];
            return n;
        }
    }
    return load_node4(S.nodes4, ref);
}
template <uint32_t F>
__device__ __forceinline__ GNode4C fetch_node4_entries(const DScene& S, uint32_t ref)
{
    if constexpr ((F & TF_STAGED) != 0) {
        const uint32_t j = ref - S.top4_base;
        if (j < S.top4_count) {
            GNode4C n;
            float4* d = reinterpret_cast<float4*>(&n);
#pragma unroll
            for (int k = 0; k < 7; k++) d[k] = s_top4[10 * j + 3 + k];
            return n;
        }
    }
    return load_node4_entries(S.nodes4, ref);
}

// Mesh::hit — closest triangle; closest is updated in place.
template <bool FAST, uint32_t F, class Stk>
__device__ __forceinline__ bool mesh_closest_walk(const DScene& S, const GMesh& M, const TRay& r, float tmin,
                                                  float& closest, int32_t& slot, float& bu, float& bv, int32_t skip,
                                                  VolSample& vs, Stk& st)
{
    float root_near;
    if (!mesh_box<FAST>(M.bmin, M.bmax, r, neg_o_inv(r), closest, root_near)) return false;
    // Walks the collapsed BVH. The entry about to be visited stays in
    // registers (ref, near); a node visit pushes the other accepted entries in
    // reverse visit order. Pruning (near >= closest) happens when an entry is
    // reached, as in the reference.
    uint32_t ref = (uint32_t)M.root4_ref;
    float near = root_near;
    int sp = 0;
    bool hit = false;
    while (true) {
        if (!(near >= closest)) {
            if (ref & kLeafBit) {
                const uint32_t first = (ref & 0x7fffffffu) >> 3;
                const uint32_t cnt = (ref & 7u) + 1u;
                for (uint32_t i = first; i < first + cnt; i++) {
                    if ((int32_t)i == skip) continue;
                    const GTri T = load_tri(S.tris, i);
                    vs.tris++;
                    float t, u, v;
                    if (tri_test(T, r, tmin, closest, t, u, v)) {
                        closest = t;
                        slot = (int32_t)i;
                        bu = u;
                        bv = v;
                        hit = true;
                    }
                }
            } else {
                const GNode4 n = fetch_node4<F>(S, ref);
                vs.nodes++;
                float nl = 0.f, nr = 0.f;
                const F3 noi = FAST ? neg_o_inv(r) : F3{0.f, 0.f, 0.f};
                const bool hl = mesh_box<FAST>(n.lmin, n.lmax, r, noi, closest, nl);
                const bool hr = mesh_box<FAST>(n.rmin, n.rmax, r, noi, closest, nr);
                bool ha[4];
                float na[4];
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    na[k] = 0.f;
                    ha[k] = n.ref[k] != kEmptySlot && mesh_box<FAST>(n.cmin[k], n.cmax[k], r, noi, closest, na[k]);
                }
                // node4_order's visit order as a position per accepted entry
                // (side offset + place within the side), without appending to
                // arrays. An accepted entry implies an accepted side box (the
                // entry box lies inside it), so hl/hr only decide which side goes
                // first when both hold entries: the nearer (ties: R).
                const int cl = (int)ha[0] + (int)ha[1], cr = (int)ha[2] + (int)ha[3];
                const bool r_first = (cl > 0 && cr > 0) ? !(nl < nr) : (cr > 0);
                const int ne = cl + cr;
                // binary-node visits this node stands for: N itself, and each accepted
                // side that is an interior node (two entries) of the binary tree
                vs.bnodes += 1u + (uint32_t)(hl && n.ref[1] != kEmptySlot) + (uint32_t)(hr && n.ref[3] != kEmptySlot);
                if (sp + ne > S.mesh_stack_limit) {
                    atomicOr(S.error, ERR_MESH_STACK);
                    break;
                }
                if (ne > 0) {
                    uint32_t first_ref = 0;
                    float first_near = 0.f;
#pragma unroll
                    for (int k = 0; k < 4; k++) {
                        const int side = k >> 1;
                        const bool a_first = na[2 * side] < na[2 * side + 1];   // ties: the right entry first
                        const bool behind_partner = ha[k ^ 1] && ((k & 1) ? a_first : !a_first);
                        const bool side_second = side ? !r_first : r_first;
                        const int pos = (side_second ? (side ? cl : cr) : 0) + (behind_partner ? 1 : 0);
                        if (ha[k]) {
                            if (pos == 0) {
                                first_ref = n.ref[k];
                                first_near = na[k];
                            } else {
                                st.set(sp + ne - 1 - pos, n.ref[k], na[k]);
                            }
                        }
                    }
                    sp += ne - 1;
                    ref = first_ref;
                    near = first_near;
                    continue;
                }
            }
        }
        if (sp == 0) break;
        sp--;
        ref = st.ref(sp);
        near = st.near(sp);
    }
    return hit;
}

template <uint32_t F, class Stk>
__device__ __forceinline__ bool mesh_closest(const DScene& S, const GMesh& M, const TRay& r, float tmin, float& closest,
                                             int32_t& slot, float& bu, float& bv, int32_t skip, VolSample& vs, Stk& st)
{
    if (mesh_fast_slabs(M, r)) return mesh_closest_walk<true, F>(S, M, r, tmin, closest, slot, bu, bv, skip, vs, st);
    return mesh_closest_walk<false, F>(S, M, r, tmin, closest, slot, bu, bv, skip, vs, st);
}

// Mesh::hitAny
template <bool FAST, uint32_t F, class Stk>
__device__ __forceinline__ bool mesh_any_walk(const DScene& S, const GMesh& M, const TRay& r, float tmin, float tmax,
                                              int32_t skip, VolSample& vs, Stk& st)
{
    float root_near;
    if (!mesh_box<FAST>(M.bmin, M.bmax, r, neg_o_inv(r), tmax, root_near)) return false;
    // The walk of mesh_closest without pruning: any accepted entry may hold an
    // occluder and the first one found ends the walk, so the entries of a node are
    // taken in a fixed order (left side, then right) instead of nearest first; the
    // answer does not depend on the order.
    uint32_t ref = (uint32_t)M.root4_ref;
    int sp = 0;
    bool hit = false;
    while (true) {
        if (ref & kLeafBit) {
            const uint32_t first = (ref & 0x7fffffffu) >> 3;
            const uint32_t cnt = (ref & 7u) + 1u;
            for (uint32_t i = first; i < first + cnt; i++) {
                if ((int32_t)i == skip) continue;
                const GTri T = load_tri(S.tris, i);
                vs.tris++;
                float t, u, v;
                if (tri_test(T, r, tmin, tmax, t, u, v)) {
                    hit = true;
                    break;
                }
            }
            if (hit) break;
        } else {
            // Only the four entry boxes are tested. The two side boxes would
            // reject nothing more: an entry box lies inside its side's box (both
            // rounded outward from nested FP64 boxes), and every slab form here is
            // monotone in the plane coordinate, so a ray that misses a side box
            // misses the entry boxes inside it. The triangles tested, and so the
            // answer, are the same as with the side tests.
            const GNode4C n = fetch_node4_entries<F>(S, ref);
            vs.nodes++;
            const F3 noi = FAST ? neg_o_inv(r) : F3{0.f, 0.f, 0.f};
            bool ha[4];
#pragma unroll
            for (int k = 0; k < 4; k++) {
                float na;
                ha[k] = n.ref[k] != kEmptySlot && mesh_box<FAST>(n.cmin[k], n.cmax[k], r, noi, tmax, na);
            }
            // Entries in slot order; an entry's place is the number of accepted
            // entries before it (selects, no running index into an array).
            const int ne = (int)ha[0] + (int)ha[1] + (int)ha[2] + (int)ha[3];
            // binary-node visits: N, and each interior side with an accepted entry
            vs.bnodes += 1u + (uint32_t)(n.ref[1] != kEmptySlot && (ha[0] || ha[1]))
                         + (uint32_t)(n.ref[3] != kEmptySlot && (ha[2] || ha[3]));
            if (sp + ne > S.mesh_stack_limit) {
                atomicOr(S.error, ERR_MESH_STACK);
                break;
            }
            if (ne > 0) {
                uint32_t first_ref = 0;
                int pos = 0;
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    if (ha[k]) {
                        if (pos == 0) first_ref = n.ref[k];
                        else st.set(sp + ne - 1 - pos, n.ref[k], 0.f);
                        pos++;
                    }
                }
                sp += ne - 1;
                ref = first_ref;
                continue;
            }
        }
        if (sp == 0) break;
        ref = st.ref(--sp);
    }
    return hit;
}

template <uint32_t F, class Stk>
__device__ __forceinline__ bool mesh_any(const DScene& S, const GMesh& M, const TRay& r, float tmin, float tmax,
                                         int32_t skip, VolSample& vs, Stk& st)
{
    if (mesh_fast_slabs(M, r)) return mesh_any_walk<true, F>(S, M, r, tmin, tmax, skip, vs, st);
    return mesh_any_walk<false, F>(S, M, r, tmin, tmax, skip, vs, st);
}

// Rectangle::hit geometric test (Rectangle.cpp:212-249); returns t.
__device__ __forceinline__ bool rect_test(const GRect& R, const TRay& r, float tmin, float tmax, float& t)
{
    if (R.w <= 0.0f || R.h <= 0.0f) return false;
    const F3 p = f3(R.p), n = f3(R.n);
    const float a = dot(r.o - p, n);
    const float b = dot(r.d, n);
    if (b == 0.0f || (a < 0.0f && b < 0.0f) || (a > 0.0f && b > 0.0f)) return false;
    t = -a / b;
    if (t > tmax || t < tmin) return false;
    const F3 d = (r.o + (t * r.d)) - p;
    const float wd = dot(d, f3(R.wa));
    const float hd = dot(d, f3(R.ha));
    return !(fabsf(wd) > R.hw || fabsf(hd) > R.hh);
}

// Sphere::hit / hitAny root selection (Sphere.cpp:227-302).
__device__ __forceinline__ bool sphere_test(const GObject& O, const TRay& r, float tmin, float tmax, float& t,
                                            bool source = false)
{
    if (O.f[4] == 0.0f || r.zero) return false;
    const F3 c = f3(O.f);
    const float rad = O.f[3];
    const F3 oc = r.o - c;
    const float b = dot(oc, r.d);
    if (source && b >= 0.0f) return false;   // leaving the source sphere
    // b^2 - (|oc|^2 - r^2) as r^2 - |oc - b d|^2: equal for a unit direction, free of cancellation.
    const F3 f = oc - b * r.d;
    const float disc = (rad * rad) - len2(f);
    if (disc < 0.0f) return false;
    const float sq = sqrtf(disc);
    float root = -b - sq;
    if (source || root < tmin || root > tmax) {
        root = -b + sq;
        if (root < tmin || root > tmax) return false;
    }
    t = root;
    return true;
}

__device__ __forceinline__ bool plane_test(const GObject& O, const TRay& r, float tmin, float tmax, float& t)
{
    const F3 n = f3(O.f + 1);
    const F3 pos = F3{0.0f, O.f[0], 0.0f};
    const float d = dot(r.d, n);
    if (d == 0.0f) return false;
    t = dot(pos - r.o, n) / d;
    return !(t > tmax || t < tmin);
}

// MeshInstance::_localRay (MeshInstance.cpp:245-265) with InstanceTransform inverses.
__device__ __forceinline__ F3 inv_rotate(const GObject& O, F3 v)
{
    const float cx = O.f[6], sx = O.f[7], cy = O.f[8], sy = O.f[9], cz = O.f[10], sz = O.f[11];
    float x = v.x, y = v.y, z = v.z;
    float nx = (x * cz) + (y * sz);
    float ny = (-x * sz) + (y * cz);
    x = nx;
    y = ny;
    nx = (x * cy) - (z * sy);
    float nz = (x * sy) + (z * cy);
    x = nx;
    z = nz;
    ny = (y * cx) + (z * sx);
    nz = (-y * sx) + (z * cx);
    return F3{x, ny, nz};
}
__device__ __forceinline__ F3 fwd_rotate(const GObject& O, F3 v)
{
    const float cx = O.f[6], sx = O.f[7], cy = O.f[8], sy = O.f[9], cz = O.f[10], sz = O.f[11];
    float x = v.x, y = v.y, z = v.z;
    float ny = (y * cx) - (z * sx);
    float nz = (y * sx) + (z * cx);
    y = ny;
    z = nz;
    float nx = (x * cy) + (z * sy);
    nz = (-x * sy) + (z * cy);
    x = nx;
    z = nz;
    nx = (x * cz) - (y * sz);
    ny = (x * sz) + (y * cz);
    return F3{nx, ny, z};
}
__device__ __forceinline__ bool instance_invertible(const GObject& O)
{
    return fabsf(O.f[3]) > 1e-12f && fabsf(O.f[4]) > 1e-12f && fabsf(O.f[5]) > 1e-12f;
}
__device__ __forceinline__ bool local_ray(const GObject& O, const TRay& r, TRay& lr, float& scale)
{
    if (!instance_invertible(O)) return false;
    const F3 s = f3(O.f + 3);
    const F3 ur = inv_rotate(O, r.d);
    const F3 ld = F3{ur.x / s.x, ur.y / s.y, ur.z / s.z};
    scale = sqrtf(len2(ld));
    if (!isfinite(scale) || scale <= 0.0f) return false;
    const F3 uo = inv_rotate(O, r.o - f3(O.f));
    const F3 lo = F3{uo.x / s.x, uo.y / s.y, uo.z / s.z};
    if (!isfinite(lo.x) || !isfinite(lo.y) || !isfinite(lo.z)) return false;
    lr = make_ray_x(lo, vdiv(ld, scale), r.xobj, r.xprim);
    return true;
}

// ConstantVolume::sampleScatteringDistance (ConstantVolume.cpp:62-121) with the
// boundary's hitInterval(-T_MAX, T_MAX) (Cube.cpp:134-175, Sphere.cpp:304-343).
// Length (scene units along the ray) of the part of [tmin, tmax] inside the
// boundary of volume O: the interval volume_distance samples in.
static __device__ float volume_overlap(const GObject& O, F3 o, F3 d, float tmin, float tmax)
{
    float entry, exit;
    if (O.aux == 3 /* LUZ_OBJ_CUBE */) {
        float imin = -kInf, imax = kInf;
        const float oo[3] = {o.x, o.y, o.z}, dd[3] = {d.x, d.y, d.z};
        for (int a = 0; a < 3; a++) {
            if (dd[a] == 0.0f) {
                if (oo[a] < O.f[a] || oo[a] > O.f[3 + a]) return 0.0f;
                continue;
            }
            const float inv = 1.0f / dd[a];
            const float t0 = (O.f[a] - oo[a]) * inv, t1 = (O.f[3 + a] - oo[a]) * inv;
            imin = fmaxf(imin, fminf(t0, t1));
            imax = fminf(imax, fmaxf(t0, t1));
            if (imin >= imax) return 0.0f;
        }
        entry = imin;
        exit = imax;
    } else {
        if (d.x == 0.0f && d.y == 0.0f && d.z == 0.0f) return 0.0f;
        const F3 oc = o - f3(O.f);
        const float b = dot(oc, d);
        const F3 f = oc - b * d;
        const float disc = (O.f[3] * O.f[3]) - len2(f);
        if (disc < 0.0f) return 0.0f;
        const float sq = sqrtf(disc);
        entry = fminf(-b - sq, -b + sq);
        exit = fmaxf(-b - sq, -b + sq);
    }
    entry = fmaxf(fmaxf(entry, tmin), 0.0f);
    exit = fminf(exit, tmax);
    if (!(exit > entry)) return 0.0f;
    return (exit - entry) * sqrtf(len2(d));
}

static __device__ bool volume_distance(const GObject& O, const TRay& r, float tmin, float tmax, VolSample& vs, float& t)
{
    float entry, exit;
    if (O.aux == 3 /* LUZ_OBJ_CUBE */) {
        float imin = -kInf, imax = kInf;
        const float o[3] = {r.o.x, r.o.y, r.o.z};
        const float d[3] = {r.d.x, r.d.y, r.d.z};
#pragma unroll
        for (int a = 0; a < 3; a++) {
            if (d[a] == 0.0f) {
                if (o[a] < O.f[a] || o[a] > O.f[3 + a]) return false;
                continue;
            }
            const float inv = 1.0f / d[a];
            float t0 = (O.f[a] - o[a]) * inv;
            float t1 = (O.f[3 + a] - o[a]) * inv;
            if (t0 > t1) {
                const float s = t0;
                t0 = t1;
                t1 = s;
            }
            imin = fmaxf(imin, t0);
            imax = fminf(imax, t1);
            if (imin >= imax) return false;
        }
        entry = imin;
        exit = imax;
    } else {
        if (r.zero) return false;
        const F3 oc = r.o - f3(O.f);
        const float b = dot(oc, r.d);
        const F3 f = oc - b * r.d;
        const float disc = (O.f[3] * O.f[3]) - len2(f);
        if (disc < 0.0f) return false;
        const float sq = sqrtf(disc);
        float r0 = -b - sq, r1 = -b + sq;
        if (r0 > r1) {
            const float s = r0;
            r0 = r1;
            r1 = s;
        }
        if (r0 >= r1) return false;
        entry = r0;
        exit = r1;
    }
    if (entry < tmin) entry = tmin;
    if (exit > tmax) exit = tmax;
    if (entry >= exit) return false;
    if (entry < 0.0f) entry = 0.0f;
    const float len = sqrtf(len2(r.d));
    if (len <= 0.0f || !isfinite(len)) return false;
    const float inside = (exit - entry) * len;
    const float hd = (float)((double)O.f[6] * log(fmax(vs.get(), 1e-12)));
    if (hd > inside) return false;
    t = entry + hd / len;
    return true;
}

// One object's closest hit; updates closest/hit when it wins.
template <uint32_t F, class Stk>
__device__ __forceinline__ void object_closest(const DScene& S, int32_t oi, const TRay& r, float tmin, float& closest,
                                               THit& h, VolSample& vs, Stk& st)
{
    const GObject O = S.objects[oi];
    vs.top++;
    const bool src = oi == r.xobj;
    float t;
    switch (O.kind) {
    case OK_RECT:
        if (!src && rect_test(S.rects[O.aux], r, tmin, closest, t)) {
            closest = t;
            h = THit{t, oi, 0, 0.f, 0.f};
        }
        break;
    case OK_CUBE:
        for (int f = 0; f < 6; f++)
            if (!(src && f == r.xprim) && rect_test(S.rects[O.aux + f], r, tmin, closest, t)) {
                closest = t;
                h = THit{t, oi, f, 0.f, 0.f};
            }
        break;
    case OK_SPHERE:
        if (sphere_test(O, r, tmin, closest, t, src)) {
            closest = t;
            h = THit{t, oi, 0, 0.f, 0.f};
        }
        break;
    case OK_PLANE:
        if (!src && plane_test(O, r, tmin, closest, t)) {
            closest = t;
            h = THit{t, oi, 0, 0.f, 0.f};
        }
        break;
    case OK_MESH: {
        int32_t slot;
        float u, v;
        if (mesh_closest<F>(S, S.meshes[O.aux], r, tmin, closest, slot, u, v, src ? r.xprim : -1, vs, st))
            h = THit{closest, oi, slot, u, v};
        break;
    }
    case OK_INSTANCE: {
        if constexpr (!(F & TF_INSTANCE)) break;
        TRay lr;
        float s;
        if (!local_ray(O, r, lr, s)) break;
        float lc = closest * s;
        int32_t slot;
        float u, v;
        if (!mesh_closest<F>(S, S.meshes[O.aux], lr, tmin * s, lc, slot, u, v, src ? r.xprim : -1, vs, st)) break;
        const float wt = lc / s;
        if (!isfinite(wt) || wt < tmin || wt > closest) break;
        closest = wt;
        h = THit{wt, oi, slot, u, v};
        break;
    }
    case OK_VOLUME:
        if constexpr (!(F & TF_VOLUME)) break;
        if (volume_distance(O, r, tmin, closest, vs, t)) {
            closest = t;
            h = THit{t, oi, 0, 0.f, 0.f};
        }
        break;
    default:
        break;
    }
}

template <uint32_t F, class Stk>
__device__ __forceinline__ bool object_any(const DScene& S, int32_t oi, const TRay& r, float tmin, float tmax, VolSample& vs,
                                           Stk& st)
{
    const GObject O = S.objects[oi];
    vs.top++;
    const bool src = oi == r.xobj;
    float t;
    switch (O.kind) {
    case OK_RECT:
        return !src && rect_test(S.rects[O.aux], r, tmin, tmax, t);
    case OK_CUBE:
        for (int f = 0; f < 6; f++)
            if (!(src && f == r.xprim) && rect_test(S.rects[O.aux + f], r, tmin, tmax, t)) return true;
        return false;
    case OK_SPHERE:
        return sphere_test(O, r, tmin, tmax, t, src);
    case OK_PLANE:
        return !src && plane_test(O, r, tmin, tmax, t);
    case OK_MESH:
        return mesh_any<F>(S, S.meshes[O.aux], r, tmin, tmax, src ? r.xprim : -1, vs, st);
    case OK_INSTANCE: {
        if constexpr (!(F & TF_INSTANCE)) return false;
        TRay lr;
        float s;
        if (!local_ray(O, r, lr, s)) return false;
        return mesh_any<F>(S, S.meshes[O.aux], lr, tmin * s, tmax * s, src ? r.xprim : -1, vs, st);
    }
    case OK_VOLUME:
        if constexpr (!(F & TF_VOLUME)) return false;
        return volume_distance(O, r, tmin, tmax, vs, t);
    default:
        return false;
    }
}

// Top-level stack entries: ref | kind << 30; kind 0 = node (near check),
// 1 = node (own box test), 2 = object (near check), 3 = object (no check).
#define TOP_PUSH(ref_, kind_, near_)                       \
    do {                                                   \
        if (sp >= S.top_stack_limit) {                     \
            atomicOr(S.error, ERR_TOP_STACK);              \
            sp = 0;                                        \
            break;                                         \
        }                                                  \
        sref[sp] = (uint32_t)(ref_) | ((uint32_t)(kind_) << 30); \
        snear[sp] = (near_);                               \
        sp++;                                              \
    } while (0)

// Renderer::internal::_checkHits with explicit [tmin, tmax].
template <uint32_t F, class Stk>
__device__ __forceinline__ THit closest_hit(const DScene& S, const TRay& r, float tmin, float tmax, VolSample& vs, Stk& st)
{
    THit h{kInf, -1, 0, 0.f, 0.f};
    float closest = tmax;
    if (S.k.accel_kind == 2) {
        object_closest<F>(S, S.k.accel_object, r, tmin, closest, h, vs, st);
    } else if (S.k.accel_kind == 1) {
        uint32_t sref[kTopStack];
        float snear[kTopStack];
        int sp = 0;
        TOP_PUSH(0, 1, -kInf);
        while (sp > 0) {
            sp--;
            const uint32_t e = sref[sp];
            const float near = snear[sp];
            const uint32_t kind = e >> 30;
            const int32_t idx = (int32_t)(e & 0x3fffffffu);
            if (kind >= 2) {
                if (kind == 2 && near >= closest) continue;
                object_closest<F>(S, idx, r, tmin, closest, h, vs, st);
                continue;
            }
            const GTopNode N = S.top_nodes[idx];
            vs.top += 1 + (uint32_t)N.child_count;
            float dummy;
            if (kind == 1) {
                if (!box_hit(N.bmin, N.bmax, r, closest, dummy)) continue;
            } else if (near >= closest) {
                continue;
            }
            const int n = N.child_count;
            const GTopChild* C = S.top_children + N.child_start;
            if (n != 2 && n <= 3) {
                for (int i = n - 1; i >= 0; i--) {
                    if (C[i].is_node) TOP_PUSH(C[i].ref, 1, -kInf);
                    else TOP_PUSH(C[i].ref, 3, -kInf);
                }
            } else if (n == 2) {
                float na = 0.f, nb = 0.f;
                const bool ha = box_hit(C[0].bmin, C[0].bmax, r, closest, na);
                const bool hb = box_hit(C[1].bmin, C[1].bmax, r, closest, nb);
                int first = 0, second = 1;
                bool hf = ha, hs = hb;
                float nf = na, ns = nb;
                if (ha && hb && nb < na) {
                    first = 1;
                    second = 0;
                    hf = hb;
                    hs = ha;
                    nf = nb;
                    ns = na;
                }
                if (hs) TOP_PUSH(C[second].ref, C[second].is_node ? 0 : 2, ns);
                if (hf) TOP_PUSH(C[first].ref, C[first].is_node ? 0 : 2, nf);
            } else {
                int ord[16];
                float on[16];
                int cnt = 0;
                for (int i = 0; i < n && i < 16; i++) {
                    float cn;
                    if (!box_hit(C[i].bmin, C[i].bmax, r, closest, cn)) continue;
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
                for (int j = cnt - 1; j >= 0; j--) {
                    const GTopChild& c = C[ord[j]];
                    TOP_PUSH(c.ref, c.is_node ? 0 : 2, on[j]);
                }
            }
        }
    }
    for (int i = 0; i < S.k.unaccel_count; i++)
        object_closest<F>(S, S.index_pool[S.k.unaccel_offset + i], r, tmin, closest, h, vs, st);
    return h;
}

// isShadowOccluded body with explicit [tmin, tmax] (tmax <= T_MIN -> not occluded).
template <uint32_t F, class Stk>
__device__ __forceinline__ bool any_hit(const DScene& S, const TRay& r, float tmin, float tmax, VolSample& vs, Stk& st)
{
    if (tmax <= kTMin) return false;
    bool occ = false;
    if (S.k.accel_kind == 2) {
        occ = object_any<F>(S, S.k.accel_object, r, tmin, tmax, vs, st);
    } else if (S.k.accel_kind == 1) {
        uint32_t sref[kTopStack];
        float snear[kTopStack];
        int sp = 0;
        TOP_PUSH(0, 1, 0.f);
        while (sp > 0) {
            sp--;
            const uint32_t e = sref[sp];
            const uint32_t kind = e >> 30;
            const int32_t idx = (int32_t)(e & 0x3fffffffu);
            if (kind >= 2) {
                if (object_any<F>(S, idx, r, tmin, tmax, vs, st)) {
                    occ = true;
                    break;
                }
                continue;
            }
            const GTopNode N = S.top_nodes[idx];
            vs.top += 1 + (uint32_t)N.child_count;
            float dummy;
            if (kind == 1 && !box_hit(N.bmin, N.bmax, r, tmax, dummy)) continue;
            const int n = N.child_count;
            const GTopChild* C = S.top_children + N.child_start;
            const bool test_kids = !(n != 2 && n <= 3);
            for (int i = n - 1; i >= 0; i--) {
                if (test_kids) {
                    float cn;
                    if (!box_hit(C[i].bmin, C[i].bmax, r, tmax, cn)) continue;
                    TOP_PUSH(C[i].ref, C[i].is_node ? 1 : 3, 0.f);
                } else {
                    TOP_PUSH(C[i].ref, C[i].is_node ? 1 : 3, 0.f);
                }
            }
        }
    }
    for (int i = 0; i < S.k.unaccel_count && !occ; i++)
        occ = object_any<F>(S, S.index_pool[S.k.unaccel_offset + i], r, tmin, tmax, vs, st);
    return occ;
}

}  // namespace luz
