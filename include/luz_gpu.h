/*
 * luz_gpu.h — C ABI of the B200 Monte Carlo integrator for Luz.
 *
 * The integrator replaces the per-pixel sample loop of the Luz CPU renderer:
 *   Renderer::internal::_manageThreads   (src/renderer/Threads.cpp:375)
 *   Renderer::internal::_threadRender    (src/renderer/Threads.cpp:551)
 *   calculateLightRaysColor              (src/renderer/ColorHelper.cpp:1136-1326)
 *   Renderer::internal::_checkHits       (src/renderer/HitHelper.cpp:5-32)
 *   isShadowOccluded                     (src/renderer/ColorHelper.cpp:801-829)
 * The C++20 host keeps the .luz loader, CLI, NFOR denoiser, post-processing
 * and image writers; it flattens its Scene into a LuzSceneDesc, calls
 * luz_gpu_render and copies the returned FP32 film into its Image.
 *
 * Conventions (mirroring the reference's error behaviour):
 *   - every entry point returns int status: 0 = ok, < 0 = error;
 *   - the last error message of the calling thread is available through
 *     luz_gpu_last_error (the host turns it into std::runtime_error, as
 *     src/cli/main.cpp:209-213 expects of the CPU renderer);
 *   - invalid scene parameters are rejected with LUZ_E_INVALID and the same
 *     wording as the reference's std::invalid_argument messages;
 *   - the caller owns every array it passes; the library copies what it keeps.
 *   - one host thread per scene handle; handles are independent.
 */
#ifndef LUZ_GPU_H
#define LUZ_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LUZ_GPU_ABI_VERSION 5   /* 5: LuzCacheParams.warm_steps */

/* status codes */
#define LUZ_OK            0
#define LUZ_E_INVALID    -1   /* bad argument / scene description            */
#define LUZ_E_CUDA       -2   /* CUDA runtime error (no device, OOM, launch)  */
#define LUZ_E_UNSUPPORTED -3  /* feature of the reference not on this path   */
#define LUZ_E_LIMIT      -4   /* BVH deeper than the traversal stack, etc.   */
#define LUZ_E_DEVICE     -5   /* a kernel reported a device-side error flag  */

/* Material types: values equal enum MaterialType (include/luz/Materials/MaterialTypes.hpp:3-15). */
#define LUZ_MAT_LAMBERTIAN         1
#define LUZ_MAT_METAL              2
#define LUZ_MAT_DIELECTRIC         3
#define LUZ_MAT_EMISSIVE           4
#define LUZ_MAT_ISOTROPIC          5
#define LUZ_MAT_HENYEY_GREENSTEIN  6
#define LUZ_MAT_PRINCIPLED         7
#define LUZ_MAT_GLOSSY             8
#define LUZ_MAT_DIFFUSE_GLOSSY     9

/* Sky types: values equal enum SkyTypes (include/luz/SkyTypes.hpp). */
#define LUZ_SKY_NONE         0
#define LUZ_SKY_LINEAR       1   /* white-to-blue gradient, Atmospherics.cpp:44-53 */
#define LUZ_SKY_ATMOSPHERE   2   /* single-scattering Rayleigh/Mie sky, Atmosphere.cpp */
#define LUZ_SKY_ENVIRONMENT  3

/* Scene object kinds (one per reference Hittable class on the path). */
#define LUZ_OBJ_RECTANGLE          1   /* src/core/Hittables/Rectangle.cpp        */
#define LUZ_OBJ_SPHERE             2   /* src/core/Hittables/Sphere.cpp           */
#define LUZ_OBJ_CUBE               3   /* src/core/Hittables/Cube.cpp             */
#define LUZ_OBJ_PLANE              4   /* src/core/Hittables/Plane.cpp            */
#define LUZ_OBJ_MESH               5   /* src/core/Hittables/Mesh.cpp             */
#define LUZ_OBJ_MESH_INSTANCE      6   /* src/core/Hittables/MeshInstance.cpp     */
#define LUZ_OBJ_VOLUME             7   /* src/core/Hittables/ConstantVolume.cpp   */
#define LUZ_OBJ_DIRECTIONAL_LIGHT  8   /* src/core/Hittables/DirectionalLight.cpp */

/* Material parameters; which fields are read depends on type, exactly as the
 * reference constructors/setters (Lambertian.cpp, Metal.cpp, Dielectric.cpp,
 * Emissive.cpp, Isotropic.cpp, HenyeyGreenstein.cpp, Principled.cpp,
 * Glossy.cpp, DiffuseGlossy.cpp). */
typedef struct LuzMaterialDesc {
    int32_t type;                 /* LUZ_MAT_*                                     */
    int32_t texture;              /* -1 or index into LuzSceneDesc.textures         */
    double  color[3];             /* albedo / base colour / emitted radiance       */
    double  roughness;            /* Metal fuzz, Dielectric/Principled roughness   */
    double  ior;                  /* Dielectric / Principled refractive index      */
    double  anisotropy;           /* Henyey-Greenstein g                            */
    int32_t conductor;            /* Metal: 1 = conductor Fresnel (eta, k)          */
    int32_t subsurface_method;    /* Principled: 0 = Burley, 1 = thin               */
    double  eta[3];               /* Metal conductor eta                            */
    double  k[3];                 /* Metal conductor extinction                     */
    double  absorption[3];        /* Dielectric/Principled absorption (1/m)         */
    double  metallic, transmission, clearcoat, clearcoat_roughness, sheen, subsurface;
    double  subsurface_radius[3];
    double  subsurface_scale;
    double  subsurface_color[3];
    double  glossy_color[3];      /* DiffuseGlossy glossy colour (color = diffuse colour) */
    double  glossy_weight;        /* DiffuseGlossy glossy weight; roughness = glossy roughness */
    int32_t has_roughness_texture;  /* Metal only, an extension (the reference's Metal roughness */
    int32_t roughness_texture;      /* is a scalar): roughness = red channel of this texture,   */
                                    /* bilinear at the hit's uv, clamped to [0, 1]              */
} LuzMaterialDesc;

/* Bilinear albedo texture (src/core/Texture.cpp:142-172): width*height RGB, row 0 = top. */
typedef struct LuzTextureDesc {
    int32_t width, height;
    const double* rgb;
} LuzTextureDesc;

/* Triangle soup of one Mesh (Mesh(position, material, std::vector<Triangle>),
 * src/core/Hittables/Mesh.cpp:343-350). Degenerate triangles are dropped as the
 * reference does (Mesh.cpp:353-365); primitive ids count surviving triangles. */
typedef struct LuzMeshDesc {
    int64_t triangle_count;
    const double* positions;      /* triangle_count * 9                             */
    const double* normals;        /* NULL or triangle_count * 9 (vertex normals)    */
    const double* uvs;            /* NULL or triangle_count * 6                     */
    int32_t material;             /* material of the triangles and of the mesh      */
    int32_t _pad;
} LuzMeshDesc;

typedef struct LuzObjectDesc {
    int32_t kind;                 /* LUZ_OBJ_*                                      */
    int32_t material;             /* VOLUME: phase-function material                */
    int32_t mesh;                 /* MESH / MESH_INSTANCE: index into meshes        */
    int32_t boundary_kind;        /* VOLUME: LUZ_OBJ_CUBE or LUZ_OBJ_SPHERE         */
    double  position[3];          /* centre / translation; PLANE: y = position[1]   */
    double  orientation[3];       /* rect normal, plane normal, light direction     */
    double  size[3];              /* rect (w,h,-), cube (w,h,d), sphere (r,-,-)     */
    double  width_axis[3];        /* rect: optional explicit axes                   */
    double  height_axis[3];
    int32_t has_axes;
    int32_t visible;              /* sphere: 0 = invisible (Sphere.cpp:229-232)     */
    double  rotation_degrees[3];  /* MESH_INSTANCE Euler X->Y->Z                    */
    double  scale[3];             /* MESH_INSTANCE                                  */
    double  density;              /* VOLUME                                         */
    int32_t has_uvs;              /* rect: optional uv0..uv3                        */
    int32_t _pad;
    double  uv[12];
    int32_t ies;                  /* sphere: -1 or index into LuzSceneDesc.ies      */
    int32_t uv_projection;        /* sphere: 0 = lat-long, 1 = cube cross           */
                                  /* (SphereUVProjection, Sphere.cpp:14-92)         */
    double  ies_direction[3];     /* Sphere::setIESProfile vertical axis            */
    double  ies_rotation_degrees; /* Sphere::setIESProfile horizontal rotation      */
} LuzObjectDesc;

/* IES photometric profile (IESProfile, src/core/IESProfile.cpp): angles in
 * degrees, each strictly increasing; candela[h * vertical_count + v], the
 * file's candela multiplier already applied. Scales the emission of the sphere
 * lights that use it when they are sampled for direct lighting
 * (Sphere::sampleLight, src/core/Hittables/Sphere.cpp:451-460). */
typedef struct LuzIesDesc {
    int32_t vertical_count;
    int32_t horizontal_count;
    const double* vertical_deg;
    const double* horizontal_deg;
    const double* candela;
} LuzIesDesc;

/* Camera (src/core/Camera.cpp); thin lens unless pinhole != 0. */
typedef struct LuzCameraDesc {
    double  position[3], direction[3], up[3];
    double  focal_length_m, sensor_width_m, sensor_height_m, f_number, focus_distance_m;
    int32_t pinhole;
    int32_t _pad;
} LuzCameraDesc;

/* Equirect environment (EnvironmentMap(width,height,pixels), src/core/EnvironmentMap.cpp:296). */
typedef struct LuzEnvironmentDesc {
    int32_t width, height;        /* 0 = no environment map                         */
    const double* rgb;            /* width*height*3                                 */
    double  strength;
    double  rotation_degrees;
    int32_t lighting;             /* Scene::setEnvironmentLighting                  */
    int32_t _pad;
} LuzEnvironmentDesc;

/* Atmosphere state as Renderer::render sees it after
 * Scene::syncAtmosphereSunDirection (src/scene/Scene.cpp:457-475): the sun
 * direction and radiance of the first directional light, or the atmosphere's
 * own. Read when sky = LUZ_SKY_ATMOSPHERE; meters per unit is the scene's. */
typedef struct LuzAtmosphereDesc {
    double  sun_direction[3];     /* towards the sun                                */
    double  sun_radiance[3];
    double  sun_radiance_scale;
    double  earth_radius, atmosphere_radius;   /* metres                        */
    double  h_r, h_m;             /* Rayleigh / Mie scale heights (metres)          */
    int32_t samples, light_samples;
    double  stars_brightness;
} LuzAtmosphereDesc;

/* Caustic photon map settings (Scene::setCausticsEnabled / setCausticPhotonCount
 * / setCausticPassCount / setCausticRadiusMeters / setCausticAlpha,
 * src/scene/Scene.cpp:302-360; defaults include/luz/Defaults.hpp:51-55: off,
 * 100000, 8, 0.05, 0.7). Read only when enabled != 0; then photons >= 0,
 * passes > 0, radius_meters finite > 0 and alpha in (0, 1], with the
 * reference's messages otherwise. The map (CausticPhotonMap::build,
 * src/renderer/CausticPhotonMap.cpp:430-551) is built on the device from the
 * render seed and max_bounces of each render call that needs it. */
typedef struct LuzCausticsDesc {
    int32_t enabled;
    int32_t photons;
    int32_t passes;
    int32_t reserved;
    double  radius_meters;
    double  alpha;
} LuzCausticsDesc;

typedef struct LuzSceneDesc {
    int32_t abi_version;          /* LUZ_GPU_ABI_VERSION                            */
    int32_t material_count;
    const LuzMaterialDesc* materials;
    int32_t texture_count;
    int32_t mesh_count;
    const LuzTextureDesc* textures;
    const LuzMeshDesc* meshes;
    int32_t object_count;         /* objects in Scene::addHittable order            */
    int32_t sky;                  /* LUZ_SKY_*                                      */
    const LuzObjectDesc* objects;
    LuzCameraDesc camera;
    LuzEnvironmentDesc environment;
    double  background[3];
    double  meters_per_unit;
    int32_t ies_count;
    int32_t _pad;
    const LuzIesDesc* ies;
    LuzAtmosphereDesc atmosphere;
    LuzCausticsDesc caustics;
} LuzSceneDesc;

/* Render settings: the parts of Scene that Renderer::render reads for the
 * sample loop (adaptive sampling and NFOR buffers: luz_gpu_render_ex);
 * stream selects the Sampler stream (0 = no denoise, Threads.cpp:565).
 * sample_offset shifts the sample indices (resume). flags may hold
 * LUZ_RENDER_PROFILE (per-stage device times) and LUZ_RENDER_COUNT (BVH node /
 * triangle visit counts); neither changes the image. */
#define LUZ_RENDER_PROFILE 0x100
#define LUZ_RENDER_COUNT   0x200
typedef struct LuzRenderParams {
    int32_t  width, height;
    int32_t  spp;
    int32_t  max_bounces;         /* Scene::getMaxLightBounces                      */
    uint32_t seed;                /* Sampler::setRenderSeed                         */
    uint32_t stream;
    int32_t  sample_offset;
    int32_t  flags;
} LuzRenderParams;

typedef struct LuzRenderStats {
    double   render_ms;           /* device time of the sample loop (CUDA events)   */
    double   samples;             /* rendered samples (width*height*spp)            */
    double   extension_rays;      /* closest-hit rays traced                        */
    double   shadow_rays;         /* any-hit rays traced                            */
    int64_t  kernel_launches;     /* kernels launched by this call                  */
    int64_t  waves;
    double   extend_ms, shade_ms, shadow_ms;   /* LUZ_RENDER_PROFILE: summed stage times */
    int64_t  extend_launches, shadow_launches;
    double   ext_nodes, ext_tris, ext_top;     /* LUZ_RENDER_COUNT: mesh nodes, triangles,  */
    double   sh_nodes, sh_tris, sh_top;        /* top-level records read (ext / shadow)     */
    double   denoise_ms;          /* luz_gpu_render_denoised: device time of NFOR    */
    double   caustic_photons;     /* photons stored in the caustic map (photonCount) */
    double   caustic_ms;          /* device time of the caustic map build            */
    double   ext_bnodes, sh_bnodes;   /* LUZ_RENDER_COUNT: binary mesh-BVH node visits the */
                                      /* collapsed walks stand for (ext / shadow)          */
} LuzRenderStats;

/* One closest-hit / any-hit result (luz_gpu_trace_rays). */
typedef struct LuzHit {
    float    t;                   /* world distance; +inf on miss                   */
    int32_t  object;              /* index into LuzSceneDesc.objects, -1 = miss     */
    int32_t  primitive;           /* triangle id (mesh/instance), cube face, else 0 */
    float    u, v;                /* barycentrics for triangles                     */
} LuzHit;

typedef struct LuzSceneInfo {
    int64_t  top_nodes;           /* BVHNode count (src/core/Hittables/BVHNode.cpp)  */
    int64_t  top_leaf_objects;
    int64_t  mesh_nodes;          /* packed mesh BVH nodes over all meshes          */
    int64_t  mesh_triangles;
    int64_t  device_bytes;        /* scene arena size on the device                 */
    int32_t  max_mesh_depth;
    int32_t  light_count;
} LuzSceneInfo;

/* Packed mesh BVH node as the reference builds it (Mesh::PackedBVHNode,
 * include/luz/Hittables/Mesh.hpp:37-45), in double, for layout parity. */
typedef struct LuzMeshNode64 {
    double   bmin[3], bmax[3];
    int64_t  left, right, start, count;
    int32_t  is_leaf;
    int32_t  _pad;
} LuzMeshNode64;

typedef struct luz_gpu_scene luz_gpu_scene;      /* device scene arena + queues */
typedef struct luz_scene_pack luz_scene_pack;    /* host-side packed scene      */

/* ---- errors / device ------------------------------------------------------ */
int luz_gpu_last_error(char* buffer, size_t length);
int luz_gpu_device_count(int32_t* count);

/* ---- host packing (no GPU needed) ----------------------------------------- */
/* Flattens the description: lights (Scene::updateLights, Scene.cpp:615-638),
 * top-level BVHNode (Scene::updateAccelerationStructure, Scene.cpp:655-688;
 * BVHNode.cpp:142-185), packed binned-SAH mesh BVHs (Mesh::_buildPackedBVH,
 * Mesh.cpp:383-521), environment CDF (EnvironmentMap::buildDistribution,
 * EnvironmentMap.cpp:627-671). */
int luz_pack_create(const LuzSceneDesc* desc, luz_scene_pack** out);
int luz_pack_destroy(luz_scene_pack* pack);
int luz_pack_info(const luz_scene_pack* pack, LuzSceneInfo* info);
/* Copies mesh `mesh`'s node array (node_capacity entries at most) and triangle
 * order (_triangleIndices) for comparison with the reference's own arrays. */
int luz_pack_mesh_bvh(const luz_scene_pack* pack, int32_t mesh,
                      LuzMeshNode64* nodes, int64_t node_capacity, int64_t* node_count,
                      int64_t* triangle_order, int64_t order_capacity);
/* Raw packed arrays (FP32 device layout) for a CPU traversal check.
 * name: "top_nodes", "top_children", "objects", "mesh_nodes", "mesh_tris",
 * "meshes", "rects". Returns pointer and byte size; valid until destroy. */
int luz_pack_array(const luz_scene_pack* pack, const char* name, const void** data, int64_t* bytes);

/* ---- device scene --------------------------------------------------------- */
int luz_gpu_scene_create(const LuzSceneDesc* desc, int32_t device, luz_gpu_scene** out);
int luz_gpu_scene_destroy(luz_gpu_scene* scene);
int luz_gpu_scene_info(const luz_gpu_scene* scene, LuzSceneInfo* info);
/* Caps the path state (the SoA arrays of one wave, 268 bytes per path, 316
 * with NFOR features) the handle may hold, in bytes; -1 restores the default,
 * a quarter of the device memory free (plus what the handle holds) when a
 * render allocates. Renders split into more, smaller waves under a lower cap
 * (the film does not depend on the wave size); when cudaMalloc refuses a wave
 * the render halves it, down to 2^20 paths, before it reports LUZ_E_CUDA. A
 * cap below what the handle holds releases the held state. No counterpart in
 * the reference (it keeps one sample's state per thread). */
int luz_gpu_scene_set_path_budget(luz_gpu_scene* scene, int64_t bytes);
/* Lowers the traversal stack bounds the kernels enforce: mesh_entries entries
 * of the collapsed mesh-BVH stack (compiled: 192) and top_entries of the
 * top-level stack (compiled: 96); 0 restores the compiled size. A ray that
 * needs more stops its walk, the kernel sets the scene's device error word and
 * the call reports LUZ_E_DEVICE; the next call starts clean. The compiled sizes
 * hold every BVH the packer accepts (Mesh.cpp's 128-entry stack bound is
 * checked at luz_gpu_scene_create); lower bounds exercise the overflow path.
 * The reference's counterpart is the fixed stack of Mesh::hit (Mesh.cpp:578-660). */
int luz_gpu_scene_set_traversal_limits(luz_gpu_scene* scene, int32_t mesh_entries, int32_t top_entries);

/* Launch tuning of a scene handle (zeros = defaults). None of it changes a film: the
 * image does not depend on the wave size, the grid or where nodes are read from.
 *   wave_paths:           paths per wave (default 64 Mi; 4 Mi for luz_gpu_render_cached, which
 *                         trains its cache between waves), capped by the path budget;
 *   staged_top_nodes:     1 = the trace kernels copy the breadth-first top of the scene's
 *                         largest collapsed mesh BVH (21 nodes) into shared memory per
 *                         block and read those nodes there;
 *   *_blocks_per_sm:      blocks per SM of the persistent closest-hit / any-hit grids and
 *                         of the shade grid (default: full occupancy; larger values are
 *                         capped at it);
 *   sort_rays, lanes:     see the fields.
 * No counterpart in the reference (its worker count is Scene::setRenderingThreads). */
typedef struct LuzTuneParams {
    int64_t wave_paths;
    int32_t staged_top_nodes;
    int32_t extend_blocks_per_sm;
    int32_t shadow_blocks_per_sm;
    int32_t shade_blocks_per_sm;
    int32_t sort_rays;            /* 1: extension rays of bounces >= 1 are traced in coherence
                                     order (direction octant, then the Morton cell of the ray
                                     origin in a 16^3 grid over the scene box)                 */
    int32_t lanes;                /* 0: a frame that takes more than one wave splits the path
                                     state in two halves and runs consecutive waves on two
                                     streams, the last bounces of one overlapping the first of
                                     the next (film accumulation stays in wave order);
                                     1: one wave at a time                                     */
} LuzTuneParams;
typedef struct LuzTuneTrial {
    LuzTuneParams params;
    double render_ms;             /* device time of the trial render */
} LuzTuneTrial;
int luz_gpu_scene_set_tuning(luz_gpu_scene* scene, const LuzTuneParams* tune);
int luz_gpu_scene_get_tuning(const luz_gpu_scene* scene, LuzTuneParams* tune);
/* Autotuner: times renders of `params` on the device (CUDA events; each trial rendered
 * twice, the second timed) while it changes one knob at a time from the handle's
 * current tuning (staged nodes on/off; ray sorting on/off; one or two wave lanes; waves of 4 Mi, 16 Mi and 64 Mi paths; the
 * closest-hit grid at full occupancy or one block fewer; the any-hit grid at full or
 * half occupancy), keeps every change that lowers the time, and leaves the best
 * tuning on the handle (also copied to `chosen` when not NULL). The trials (up to
 * trial_capacity) and their count go to trials / trial_count when not NULL. */
int luz_gpu_autotune(luz_gpu_scene* scene, const LuzRenderParams* params, LuzTuneParams* chosen,
                     LuzTuneTrial* trials, int32_t trial_capacity, int32_t* trial_count);

/* ---- hot path ------------------------------------------------------------- */
/* Full render: W*H*spp paths through the wavefront integrator; rgb_out is the
 * host film (W*H*3, row-major, y = 0 first) holding per-pixel means, exactly
 * what _threadRender stores with Image::setPixelUnchecked (Threads.cpp:581). */
int luz_gpu_render(luz_gpu_scene* scene, const LuzRenderParams* params,
                   float* rgb_out, LuzRenderStats* stats);
/* Same, device pointer film and caller stream (cudaStream_t as void*). */
int luz_gpu_render_device(luz_gpu_scene* scene, const LuzRenderParams* params,
                          float* d_rgb_out, void* stream, LuzRenderStats* stats);

/* Per-path radiance for explicit (x, y, sample) triples: the colour
 * calculateLightRaysColor returns for Sampler::beginPixelSample(x, y, s, stream)
 * (ColorHelper.cpp:1110-1115), before cleanColor. Host buffers. */
int luz_gpu_trace_paths(luz_gpu_scene* scene, const LuzRenderParams* params,
                        const int32_t* x, const int32_t* y, const int32_t* sample,
                        int64_t count, float* rgb_out);

/* Render without allocating device memory.
 * For callers that cannot call cudaMalloc while they render: a host whose
 * device memory is owned by its own allocator, or a per-frame loop that must
 * not take the implicit device synchronisation that cudaMalloc/cudaFree cause.
 * Same result as luz_gpu_render_device (same kernels, shading binned by hit
 * class, same FP64 film), but the path state, queues, shade bins and film live
 * in one file-scope device array of LUZ_STATIC_SCRATCH_BYTES that every GPU
 * loading this library holds until process exit; waves are
 * LUZ_STATIC_WAVE_PATHS paths. The caller passes the scene (created
 * beforehand), the device film and the stream. Limits: width*height <=
 * LUZ_STATIC_MAX_PIXELS, otherwise LUZ_E_LIMIT; flags must be 0. The call
 * returns once the render has finished on the stream (it waits for the
 * stream to read the ray totals and the error word into the handle's pinned
 * buffer), so the call itself cannot be captured into a CUDA graph. The first
 * call on a device resolves the array's device address (cudaGetSymbolAddress),
 * which other threads' global-mode stream captures forbid: make that first
 * call before such captures begin.
 * All calls share the array and it keeps the previous call's contents: calls
 * whose GPU work overlaps (other streams, other threads) race on it and must
 * be serialised by the caller.
 * No counterpart in the reference: the CPU renderer has no device memory. */
#define LUZ_STATIC_SCRATCH_BYTES (96u << 20)
#define LUZ_STATIC_WAVE_PATHS    131072
#define LUZ_STATIC_MAX_PIXELS    2800000
int luz_gpu_render_device_noalloc(luz_gpu_scene* scene, const LuzRenderParams* params,
                                  float* d_rgb_out, void* stream, LuzRenderStats* stats);

/* Many independent renders in one call (a batch of scenes and views of uneven size,
 * one result each). The scenes' arrays are copied into one geometry arena (kept for
 * later calls with the same scene contents) and their paths share the wavefront:
 * a wave packs runs of pixels of any scenes (every sample of a pixel in the same
 * wave), and each bounce runs one persistent closest-hit, one shade and one any-hit
 * launch over the rays of all scenes, every ray traversing its own scene. A wave's
 * launches are recorded once per call as a CUDA graph and replayed for every wave.
 * The wave size is autotuned per scene set: the first call times one wave at 4 Mi,
 * 16 Mi and 64 Mi paths and keeps the fastest rate for later calls. Each result
 * equals luz_gpu_render(scenes[i], &params[i], rgb_out[i], &stats[i]) bit for bit;
 * stats[i] counts scene i's samples and rays, with the batch's device time. All
 * handles on one device, each at most once; params[i].flags must be 0; stats may
 * be NULL. Calls on one device are serialised. The reference renders one scene
 * per process; its workers share an atomic block counter (Threads.cpp:410-451),
 * which the shared ray queues generalise to many scenes. */
int luz_gpu_batch_render(luz_gpu_scene* const* scenes, const LuzRenderParams* params, int32_t count,
                         float* const* rgb_out, LuzRenderStats* stats);
/* The same, with what the batch did: the wave size used (tuned or cached), the waves
 * and launches, the device time, and the autotuner's trials of this call (none when
 * the scene set's wave size was already tuned). */
typedef struct LuzBatchTrial {
    int64_t wave_paths;
    double  paths;                /* paths of the trial wave */
    double  ms;                   /* its device time */
} LuzBatchTrial;
typedef struct LuzBatchReport {
    int64_t wave_paths;
    int64_t waves;
    int64_t kernel_launches;
    double  render_ms;
    int32_t trial_count;
    int32_t reserved;
    LuzBatchTrial trials[8];
} LuzBatchReport;
int luz_gpu_batch_render_ex(luz_gpu_scene* const* scenes, const LuzRenderParams* params, int32_t count,
                            float* const* rgb_out, LuzRenderStats* stats, LuzBatchReport* report);

/* ---- differentiation (albedo textures) ------------------------------------
 * No counterpart in the reference (it has no gradients); the oracle is central
 * finite differences of renders with common random numbers. */
/* Replaces the texels of texture `texture` (its width*height*3 RGB, row 0 =
 * top, as in LuzTextureDesc) in the device scene. */
int luz_gpu_scene_set_texture(luz_gpu_scene* scene, int32_t texture, const double* rgb);
/* Forward pass: set the texture's texels, then luz_gpu_render. */
int luz_gpu_adjoint_forward(luz_gpu_scene* scene, const LuzRenderParams* params, int32_t texture,
                            const double* texels, float* rgb_out, LuzRenderStats* stats);
/* Backward pass: dLoss/dtexel (texture width*height*3, host) for the film of
 * `params` and dLoss/dpixel = adjoint_rgb (W*H*3, host), by path replay: the
 * paths are traced once for their radiance and once more to spread each
 * textured Lambertian vertex's share of it over the bilinear texel weights.
 * When the texture is a Metal roughness texture instead, the gradient is in the
 * red channel (green and blue 0): at every rough vertex of such a Metal the
 * light sample, the environment sample and the continuation each contribute
 * their radiance times d ln f / d roughness of their direction (a central
 * difference of the BSDF; each sample's density held fixed, so MIS weights and
 * sampling are not differentiated), spread over the texel weights; GGX samples
 * replaced by the mirror direction (half vector facing away or reflection below
 * the surface) and mirror-like vertices (roughness <= 1e-4) carry none.
 * Russian roulette's survival probabilities are treated as constants. A texture
 * may be differentiated as the albedo of Lambertian materials or the roughness
 * of Metal ones, not both, and no other material may use it as albedo (else
 * LUZ_E_UNSUPPORTED). stats->samples counts the paths replayed. */
int luz_gpu_adjoint_backward(luz_gpu_scene* scene, const LuzRenderParams* params, int32_t texture,
                             const float* adjoint_rgb, double* grad_out, LuzRenderStats* stats);
/* dLoss/d(emitted radiance) of every light (grad_out: light_count x 3, the
 * lights in Scene::updateLights order, LuzSceneInfo.light_count) for the film
 * of `params` and dLoss/dpixel = adjoint_rgb, by one path replay: every emitter
 * hit and every light sample adds adj * contribution / E per channel (both are
 * linear in E). The light-selection distribution, which weights lights by
 * area x luminance(E), is held fixed: with one light the result is exact up to
 * rounding, with several it omits the change in which light is sampled. No
 * counterpart in the reference (it has no gradients). */
int luz_gpu_adjoint_emission(luz_gpu_scene* scene, const LuzRenderParams* params, const float* adjoint_rgb,
                             double* grad_out, LuzRenderStats* stats);
/* dLoss/d(density) of the volume `object` (index into LuzSceneDesc.objects, a
 * LUZ_OBJ_VOLUME) for the film of `params` and dLoss/dpixel = adjoint_rgb, as
 * one replay with a score-function estimate: the distance a bounce's rays sample
 * in the medium, hd = -ln(u) / density (ConstantVolume.cpp:62-121), has score
 * 1 / density - hd, and each contribution is weighted by the scores of the
 * bounces whose rays crossed the medium before it. Unbiased while no ray meets a
 * second medium (media met by one ray share its u). No counterpart in the
 * reference (it has no gradients). */
int luz_gpu_adjoint_density(luz_gpu_scene* scene, const LuzRenderParams* params, int32_t object,
                            const float* adjoint_rgb, double* grad_out, LuzRenderStats* stats);

/* Adaptive sampling settings: Scene::setAdaptiveSampling / setAdaptiveMinSamples /
 * setAdaptiveCheckInterval / setAdaptiveThreshold (src/scene/Scene.cpp:183-222),
 * defaults include/luz/Defaults.hpp:12-15 (on, 128, 32, 0.03). */
typedef struct LuzAdaptiveParams {
    int32_t  enabled;
    int32_t  min_samples;         /* > 0 */
    int32_t  check_interval;      /* > 0 */
    int32_t  reserved;
    double   threshold;           /* finite, > 0: relative 95% confidence interval */
} LuzAdaptiveParams;

/* NFOR inputs (Denoise::NFORBuffers, include/luz/Denoise/NFOR.hpp:23-32), host
 * buffers, row-major, y = 0 first. Each pointer may be NULL to skip that buffer. */
#define LUZ_NFOR_FEATURES 11
typedef struct LuzNforBuffers {
    double*  color_a;             /* W*H*3: mean of the even samples (stream 1)      */
    double*  color_b;             /* W*H*3: mean of the odd samples (stream 2)       */
    double*  color_variance;      /* W*H: variance of the pixel mean, channel average */
    double*  features_a;          /* W*H*11 */
    double*  features_b;          /* W*H*11 */
    double*  feature_variance;    /* W*H*11 */
} LuzNforBuffers;

/* Render with adaptive sampling and/or NFOR buffers: the _threadRender loop
 * (src/renderer/Threads.cpp:551-641) with adaptiveSampleConverged (:194-265)
 * and storeDenoisePixel (:343-372).
 *   adaptive: NULL or enabled = 0 samples every pixel params->spp times; else a
 *             pixel stops at the first check point (min_samples, then every
 *             check_interval samples) where its luminance and RGB confidence
 *             intervals are within threshold (adaptiveSamplingCanStop, :267-273).
 *   nfor:     NULL renders on params->stream; else samples alternate between
 *             sampler streams 1 and 2 (the denoise half buffers, :593-598) and
 *             the buffers are filled.
 *   samples_out: NULL or W*H samples used per pixel.
 * rgb_out is the host film of per-pixel means; stats->samples is the sum of the
 * samples used (SceneRenderStats::renderedSamples). */
int luz_gpu_render_ex(luz_gpu_scene* scene, const LuzRenderParams* params,
                      const LuzAdaptiveParams* adaptive, float* rgb_out,
                      const LuzNforBuffers* nfor, int32_t* samples_out,
                      LuzRenderStats* stats);

/* Renders listed pixels only: the _threadRender loop (src/renderer/Threads.cpp:551-641,
 * adaptive sampling off) for each pixel index (y * width + x; distinct, inside the
 * image, else LUZ_E_INVALID), as the reference's block scheduler hands pixels to its
 * workers (Threads.cpp:410-451). rgb_out (count * 3 floats, host) receives each
 * listed pixel's mean over params->spp samples, the value luz_gpu_render writes for
 * it. stats->samples = count * spp. */
int luz_gpu_render_pixels(luz_gpu_scene* scene, const LuzRenderParams* params, const int32_t* pixels, int64_t count,
                          float* rgb_out, LuzRenderStats* stats);

/* ---- NFOR denoiser ----------------------------------------------------------
 * Denoise::applyNFOR (src/core/Denoise/NFOR.cpp:977-1102) on the GPU in FP64:
 * firefly suppression, cross-guided feature prefilter, two-bandwidth feature
 * regressions of each half buffer, MSE-driven bandwidth selection and a last
 * regression. Input: the NFOR buffers of a render (luz_gpu_render_ex), host
 * arrays; output: width*height*3 doubles (the denoised Image). settings NULL
 * = NFORSettings defaults (include/luz/Denoise/NFOR.hpp:39-47). A zero-sized
 * image returns LUZ_OK with nothing written. Errors: LUZ_E_INVALID with the
 * message of luz_gpu_nfor_error (e.g. "NFOR radii must be positive."). */
typedef struct LuzNforSettings {
    int32_t feature_prefilter_radius;   /* 1 */
    int32_t regression_radius;          /* 2 */
    int32_t patch_radius;               /* 1 */
    int32_t reserved;
    double  min_variance;               /* 1e-5 */
} LuzNforSettings;
int luz_gpu_nfor_denoise(int32_t device, const LuzNforBuffers* buffers, int32_t width, int32_t height,
                         const LuzNforSettings* settings, double* rgb_out);
int luz_gpu_nfor_error(char* buf, size_t len);

/* Render and denoise in one call, the NFOR buffers staying on the device: the
 * _manageThreads tail (src/renderer/Threads.cpp:514-536) that runs
 * Denoise::applyNFOR on the scene's denoise buffers after the sample loop.
 * Samples use the half-buffer streams 1 and 2 as in luz_gpu_render_ex with
 * nfor set. rgb_out (W*H*3 floats) is the film of per-pixel means, denoised_out
 * (W*H*3 doubles) the NFOR image; settings NULL = NFORSettings defaults.
 * stats->denoise_ms is the device time of the denoiser. Errors: those of
 * luz_gpu_render_ex, and LUZ_E_INVALID for bad settings (radii must be
 * positive) before any sample is rendered. */
int luz_gpu_render_denoised(luz_gpu_scene* scene, const LuzRenderParams* params,
                            const LuzAdaptiveParams* adaptive, const LuzNforSettings* settings,
                            float* rgb_out, double* denoised_out, int32_t* samples_out,
                            LuzRenderStats* stats);

/* ---- Learned radiance cache -------------------------------------------------
 * No counterpart in the reference. A small MLP (inputs: position normalised to
 * the scene box, outgoing direction, shading normal, roughness, each encoded as
 * sin/cos(2^k pi x) for k = 0..5; four hidden layers of 64 with ReLU; RGB out)
 * with FP16 weights and activations and FP32 accumulation on the tensor cores,
 * trained online with Adam on the relative L2 loss sum_c (y - t)^2 / (y^2 + 0.01)
 * (denominator held constant, per-row gradient clamped to +-2000).
 * luz_gpu_render_cached renders every pixel's first sample plain, every path
 * supplying a training row, and trains the cache on them (32 Adam steps). Later
 * samples stop at their first surface vertex at or after bounce `prefix` that
 * does not scatter specularly: the vertex's own emission and next-event
 * estimate stay explicit, and the cache's prediction times the path throughput
 * stands for the continuation (a biased estimate: the plain luz_gpu_render
 * stays the unbiased reference for it). One path in `train_every` instead continues
 * past that vertex and supplies a training row: its inputs at that vertex and the
 * radiance its continuation gathered divided by its throughput there, where the
 * continuation itself ends in the cache at its next such vertex (self-training:
 * short training paths, low-variance targets; the first sample's training paths run
 * to their end). Samples
 * run in waves as in luz_gpu_render; after each wave the cache takes one Adam
 * step per `batch` of that wave's rows (at most 16). Training rows are appended
 * in arrival order, so cached renders are not bit-reproducible. The cache
 * belongs to one device and one scene at a time
 * (the position input is normalised to the box of the scene it renders). */
typedef struct luz_gpu_cache luz_gpu_cache;
#define LUZ_CACHE_PARAMS 21504   /* FP32 weights: W0 128x64, W1..W3 64x64, W4 64x16, row-major [in][out] */
typedef struct LuzCacheParams {
    uint32_t seed;                /* weight initialisation (uniform +-sqrt(6 / fan_in))    */
    int32_t  batch;               /* training rows per step (16384); > 0                     */
    float    learning_rate;       /* Adam step size (1e-2); beta1 0.9, beta2 0.99, eps 1e-8 */
    int32_t  prefix;              /* first bounce whose vertex queries the cache (1); >= 0   */
    int32_t  train_every;         /* one training path in this many (32); >= 1               */
    float    min_roughness;       /* in [0, 1]: a surface vertex whose roughness is below this
                                     continues the path and a later vertex queries the cache
                                     (0: the first vertex at or after `prefix` always does);
                                     diffuse and phase-function materials count as 1          */
    int32_t  warm_steps;          /* Adam steps on the warm-up wave (the first sample of every
                                     pixel, rendered plain, every path a training row); 0 selects
                                     64, at most 4096. More steps lower the cache's error floor
                                     and cost ~45 us each on a 16,384-row batch               */
} LuzCacheParams;
int luz_gpu_cache_create(int32_t device, const LuzCacheParams* params, luz_gpu_cache** out);
int luz_gpu_cache_destroy(luz_gpu_cache* cache);
/* Reads (get != NULL) and/or replaces (set != NULL) the LUZ_CACHE_PARAMS FP32
 * weights; replacing resets the Adam moments and step count. */
int luz_gpu_cache_weights(luz_gpu_cache* cache, float* get, const float* set);
/* Predictions for n rows of 10 inputs (host arrays): rgb_out n x 3. */
int luz_gpu_cache_predict(luz_gpu_cache* cache, const float* inputs, int64_t n, float* rgb_out);
/* Gradient of the mean loss over n rows (targets n x 3) with respect to the
 * weights (grad_out LUZ_CACHE_PARAMS floats, or NULL) and the mean loss; no step. */
int luz_gpu_cache_gradient(luz_gpu_cache* cache, const float* inputs, const float* targets, int64_t n,
                           float* grad_out, double* loss_out);
/* `steps` Adam steps on the same n rows (n <= batch); loss_out (steps doubles,
 * or NULL) receives the mean loss before each step. */
int luz_gpu_cache_train(luz_gpu_cache* cache, const float* inputs, const float* targets, int64_t n, int32_t steps,
                        double* loss_out);
/* Renders with the cache (see above), training it as it goes: params as for
 * luz_gpu_render (flags 0); stats->samples counts the camera samples,
 * extension_rays / shadow_rays the rays traced. Caustic photon maps are not
 * combined with the cache (LUZ_E_UNSUPPORTED). */
int luz_gpu_render_cached(luz_gpu_scene* scene, luz_gpu_cache* cache, const LuzRenderParams* params,
                          float* rgb_out, LuzRenderStats* stats);


/* Ray batch traversal (test hook and building block): rays are
 * (ox, oy, oz, tmin, dx, dy, dz, tmax) * count, host buffers. any_hit != 0
 * runs the shadow traversal and reports object = 0 (occluded) / -1. The
 * stochastic volume sample uses (seed, pixel 0, sample 0, bounce 0) unless
 * the caller passes volume_key (x, y, sample, bounce) per ray (may be NULL). */
int luz_gpu_trace_rays(luz_gpu_scene* scene, const float* rays, int64_t count,
                       int32_t any_hit, uint32_t seed, const int32_t* volume_key,
                       LuzHit* out);

#ifdef __cplusplus
}
#endif
#endif /* LUZ_GPU_H */
