// layout.h — device-resident scene arena layout, shared by the host packer
// (pack.cpp) and the CUDA kernels. Everything is plain data in FP32 except the
// sampling CDFs, which stay FP64 so that discrete selections (light, triangle,
// environment texel) pick the same index as the reference's std::upper_bound /
// std::lower_bound over its double prefix sums.
#pragma once
#include <stdint.h>

#ifdef __CUDACC__
#define LUZ_HD __host__ __device__
#else
#define LUZ_HD
#endif

namespace luz {

// T_MIN of include/luz/Defaults.hpp:18 as the nearest float.
constexpr float kTMin = 0.001f;
constexpr int kMeshStack = 128;        // MESH_BVH_STACK_SIZE, src/core/Hittables/Mesh.cpp:17
// Device stack of the collapsed (4-wide) mesh BVH: a node visit pushes up to 3
// entries, for at most 63 collapsed levels of a depth-126 binary tree.
constexpr int kMeshStack4 = 192;
constexpr int kTopStack = 96;
constexpr uint32_t kLeafBit = 0x80000000u;

// Object kinds inside the top-level BVH / unaccelerated list.
enum ObjKind : int32_t {
    OK_RECT = 1, OK_SPHERE = 2, OK_CUBE = 3, OK_PLANE = 4, OK_MESH = 5, OK_INSTANCE = 6, OK_VOLUME = 7,
    OK_DIRECTIONAL = 8
};

// 64 B. Rectangle with its basis precomputed in double (Rectangle::_buildBasis,
// src/core/Hittables/Rectangle.cpp:127-152) and rounded to float.
struct alignas(16) GRect {
    float p[3];     // centre
    float hw;       // width / 2
    float n[3];     // normal
    float hh;       // height / 2
    float wa[3];    // width axis
    float w;        // width
    float ha[3];    // height axis
    float h;        // height
};

// 64 B top-level object record.
struct alignas(16) GObject {
    int32_t kind;
    int32_t material;
    int32_t aux;      // rect index (RECT/CUBE first face), mesh index (MESH/INSTANCE), boundary kind (VOLUME)
    int32_t id;       // index in LuzSceneDesc.objects
    // RECT: texture coordinates uv0..uv3 (x, y) in f[0..7], f[8] = 1 when set
    // SPHERE: c[3], r, visible
    // PLANE: y, n[3]
    // INSTANCE: pos[3], scale[3], cx, sx, cy, sy, cz, sz
    // VOLUME: cube bmin[3], bmax[3] | sphere c[3], r ; f[6] = negative inverse density
    // DIRECTIONAL: dir[3] (normalised light direction)
    float f[12];
};

// Top-level BVHNode (src/core/Hittables/BVHNode.cpp). 32 B each.
struct alignas(16) GTopNode {
    float bmin[3];
    int32_t child_start;
    float bmax[3];
    int32_t child_count;
};
struct alignas(16) GTopChild {
    float bmin[3];
    int32_t ref;       // top node index or object index
    float bmax[3];
    int32_t is_node;
};

// Mesh BVH interior node with both child boxes (64 B, one 128-B line holds 2).
// ref: interior child = node index; leaf child = kLeafBit | first << 3 | (count - 1).
struct alignas(16) GNode {
    float lmin[3];
    float lmax[3];
    float rmin[3];
    float rmax[3];
    uint32_t lref;
    uint32_t rref;
    uint32_t pad0, pad1;
};

// Collapsed mesh BVH node (160 B): a binary node N together with its two
// children L and R. It holds the boxes of L and R and of up to four
// grandchildren: slots 0-1 are L's children (or L itself, slot 1 empty, when L
// is a leaf), slots 2-3 are R's. A traversal step over it visits exactly the
// entries the binary near-first traversal would visit after N, L and R, in the
// same order (see trace.cuh). ref: node4 index, leaf ref, or kEmptySlot.
constexpr uint32_t kEmptySlot = 0xffffffffu;
// Collapsed nodes at the front of each mesh's node range in breadth-first order
// (the root and the next two collapsed levels: the nodes every ray of the mesh
// visits first); the trace kernels stage them in shared memory.
constexpr int kTopNodes4 = 21;
struct alignas(16) GNode4 {
    float lmin[3], lmax[3];
    float rmin[3], rmax[3];
    float cmin[4][3];
    float cmax[4][3];
    uint32_t ref[4];
};

// Triangle in leaf order: v0, e1 = v1 - v0, e2 = v2 - v0 (edges formed in double
// as Triangle::_updateCache does, src/core/Hittables/Triangle.cpp:94-126).
struct alignas(16) GTri {
    float v0[3];
    uint32_t orig;     // index into the mesh's surviving-triangle list (primitive id)
    float e1[3];
    float area;
    float e2[3];
    uint32_t pad;
};

// Per-triangle shading data (leaf order).
struct alignas(16) GTriShade {
    float fn[3];       // face normal (normalised in double)
    float pad;
};

struct alignas(16) GMesh {
    float bmin[3];
    int32_t node_offset;      // first GNode of this mesh; -1 when the root is a leaf
    float bmax[3];
    int32_t tri_offset;       // first GTri
    int32_t tri_count;
    int32_t root_ref;         // root reference (node index or leaf ref)
    int32_t normal_offset;    // -1 or first entry (3 float3 per tri) in vertex-normal pool
    int32_t uv_offset;        // -1 or first entry (3 float2 per tri) in uv pool
    int32_t cdf_offset;       // area prefix sums (double) in the CDF pool, original order
    int32_t slot_offset;      // original index -> leaf slot map
    int32_t material;
    int32_t depth;
    double total_area;
    int32_t node4_offset;     // first GNode4 of this mesh; -1 when the root is a leaf
    int32_t root4_ref;        // root reference in the collapsed BVH (node4 index or leaf ref)
};

// Materials (src/core/Materials/*). 160 B.
enum MatType : int32_t {
    MT_LAMBERTIAN = 1, MT_METAL = 2, MT_DIELECTRIC = 3, MT_EMISSIVE = 4, MT_ISOTROPIC = 5, MT_HG = 6,
    MT_PRINCIPLED = 7, MT_GLOSSY = 8, MT_DIFFUSE_GLOSSY = 9
};
enum MatFlags : int32_t {
    MF_CONDUCTOR = 1, MF_THIN = 2, MF_SMOOTH_FULL_TRANSMISSION = 4, MF_CAN_TRANSMIT = 8, MF_ABSORPTION = 16,
    MF_TRANSPORT = 32   // materialIsTransport (CausticPhotonMap.cpp:199-223): carries caustic photons
};
struct alignas(16) GMaterial {
    int32_t type;
    int32_t texture;
    int32_t flags;
    int32_t rtexture;         // Metal: roughness texture (red channel), -1 = the scalar roughness
    float color[3];
    float roughness;
    float alpha;              // BSDF::roughnessToAlpha(roughness)
    float clearcoat_alpha;
    float ior;
    float anisotropy;
    float metallic, transmission, clearcoat, clearcoat_roughness;
    float sheen, subsurface, f0_diel, pad2;
    float eta[3], pad3;
    float k[3], pad4;
    float absorption[3], pad5;
    float ss_radius_m[3], pad6;  // subsurface radius * scale (metres)
    float ss_color[3], pad7;     // clampColor01(subsurface colour)
    float gcolor[3];             // DiffuseGlossy glossy colour
    float gweight;               // DiffuseGlossy glossy weight
};

struct GTexture {
    int32_t width, height;
    int32_t offset;     // first texel (float4) in the texel pool
    int32_t pad;
};

// Lights (Scene::updateLights, src/scene/Scene.cpp:615-638).
enum LightKind : int32_t { LK_NONE = 0, LK_RECT = 1, LK_SPHERE = 2, LK_MESH = 3, LK_INSTANCE = 4, LK_DIRECTIONAL = 5 };
struct alignas(16) GLight {
    int32_t kind;
    int32_t object;          // GObject index (top-level object id)
    int32_t material;
    int32_t cdf_offset;      // INSTANCE with non-uniform scale: transformed-area prefix sums
    float emitted[3];
    int32_t cdf_count;
    double area;             // surface area used by pdfValue / sampleLight
    int32_t uniform;         // INSTANCE: uniform area scale
    int32_t mesh;
    int32_t ies;             // SPHERE: -1 or GIes index
    int32_t pad;
    double ies_axis[3];      // Sphere::setIESProfile vertical axis and horizontal rotation
    double ies_rotation;
};

// IES profile: angles and candela values in the double pool (vertical
// angles, then horizontal angles, then candela[h * nv + v]); mean candela
// = integrated flux / 4 pi (IESProfile::load, IESProfile.cpp:218-223).
struct alignas(16) GIes {
    int32_t nv, nh;
    int32_t offset;
    int32_t pad;
    double mean_candela;
};

// Camera prepared in double (Renderer::internal::_prepareRenderCamera,
// src/renderer/RayHelper.cpp:50-83); kept in double for ray generation.
struct GCamera {
    double position[3];
    double u[3], v[3];
    double horizontal[3], vertical[3], lower_left[3];
    double lens_radius;
    double inv_w1, inv_h1;
};

struct GEnv {
    int32_t width, height;
    int32_t present;          // hasVisibleEnvironment
    int32_t lighting;         // hasEnvironmentLight
    float strength;
    float pad;
    double rotation;
    double total_weight;
    int64_t texel_offset;     // float4 texels
    int64_t cdf_offset;       // double CDF (W*H)
    int64_t pdf_offset;       // double (weight/total)/solidAngle per texel
    int32_t guide_offset;     // CDF guide tables (lo[K], hi[K] in the index pool), -1 = none
    int32_t guide_count;
};

// Atmosphere::sampleSegment inputs (FP64, metres).
struct GAtmos {
    double sun_dir[3];
    double sun_rad[3];          // sun radiance * scale
    double earth_r, atmos_r;
    double inv_hr, inv_hm;
    double stars;
    int32_t samples, light_samples;
};

// Caustic photon map settings resolved on the host (CausticPhotonMap::build,
// src/renderer/CausticPhotonMap.cpp:430-450, and sampleDirectionalEmission,
// :287-326). enabled = caustics on, photons > 0 and at least one light.
struct GCaustics {
    int32_t enabled;
    int32_t photons;          // photon target
    int32_t passes;
    int32_t has_bounds;       // sceneBoundingBox found a box (directional-light emission)
    double radius_m;          // progressiveRadiusMeters
    double radius_su;         // radius_m / meters per unit (grid cell size)
    double gather_area_m2;    // pi radius_m^2
    double m2_per_area;       // meters per unit squared
    double center[3];         // scene box centre
    double disk_radius;       // |diagonal| / 2 (1 if not positive) + max(T_MIN, radius setting / meters per unit)
};

struct GSceneConst {
    int32_t accel_kind;       // 0 none, 1 top BVH (root node 0), 2 single object
    int32_t accel_object;
    int32_t unaccel_count;
    int32_t unaccel_offset;   // into the object-index pool
    int32_t light_count;
    int32_t sky;              // 0 none, 1 linear, 2 atmosphere, 3 environment
    int32_t has_constant_background_light;
    int32_t sampled_infinite_light;
    float background[3];
    float background_luminance;
    double light_total_weight;
    int32_t light_cdf_offset; // double cumulative weights; -1 = uniform selection
    int32_t features;         // traversal specialisation: 1 = has instances, 2 = has volumes
    double meters_per_unit;
    GCamera camera;
    GEnv env;
    GAtmos atmos;
    GCaustics caustics;
    float box_lo[3];          // box of every bounded object (radiance-cache position input)
    float box_inv[3];         // 1 / extent per axis (1 where the extent is 0 or there is no box)
    int32_t cube_cross_spheres;   // 1 when a sphere uses the cube-cross UV projection
};

}  // namespace luz
