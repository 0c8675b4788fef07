/*
 * ref_harness.cpp — TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * A C entry layer over the UNMODIFIED Luz reference renderer, compiled from its
 * own sources by oracle/Makefile into oracle/_ref/libluzref*.so. Nothing in the
 * product links or calls this file; tests, the golden-fixture script and the
 * CPU-baseline leg of bench.py load it through ctypes as the checker.
 *
 * It builds a reference Scene from the same LuzSceneDesc the GPU library
 * consumes (include/luz_gpu.h) using only the reference's public classes, then
 * calls the reference's own code:
 *   - closest / any hit:   the body of Renderer::internal::_checkHits
 *                          (src/renderer/HitHelper.cpp:5-32) and isShadowOccluded
 *                          (src/renderer/ColorHelper.cpp:801-829) with explicit
 *                          t ranges, calling Hittable::hit / hitAny;
 *   - per-path radiance:   Sampler::beginPixelSample + _calculatePixelColor
 *                          (src/renderer/ColorHelper.cpp:1110-1115), the exact
 *                          sequence of _threadRender (src/renderer/Threads.cpp:563-566);
 *   - full render:         Renderer::render (src/renderer/Renderer.cpp:10) with
 *                          denoise/adaptive off and the Raw view transform;
 *   - mesh BVH layout:     Mesh::_packedBVHNodes / _triangleIndices, read with
 *                          private access in this translation unit only;
 *   - .luz scenes:         SceneFile::read (src/io/SceneFile/SceneFile.cpp:256-321)
 *                          into a reference Scene, and the reference-side scene
 *                          glue (luz_b200/glue/scene_glue.cpp) that packs such a
 *                          Scene into a LuzSceneDesc.
 *   - top-level BVH:       the BVHNode tree of Scene::updateAccelerationStructure
 *                          (src/scene/Scene.cpp:655-688, BVHNode.cpp:142-185) in
 *                          preorder, read with private access here only.
 * Hit identification: in "tag" mode every object (and every mesh triangle) gets
 * its own Lambertian-derived material so the HitRecord's material pointer names
 * the object and primitive; traversal does not depend on material values.
 *
 * FP32 ambiguity probe (parity build only, LUZREF_PERTURB): the Sampler's
 * exported functions are wrapped at link time (ld --wrap, oracle/Makefile) so
 * that, while a perturbation seed is set, every value the path loop draws is
 * moved by +-delta (a sign hashed from the seed, the dimension and the value,
 * so repeated draws of one dimension move together). A path whose radiance
 * changes by more than the parity tolerance under such moves depends on its
 * draws, and so on every quantity compared with them, finer than the FP32
 * arithmetic of the GPU can resolve; the fixtures mark it as ambiguous. The
 * mappings of cosineHemisphere, sphereDirection and unitDisk
 * (src/core/Sampler.cpp:239-290) are restated below on the moved draws,
 * because their internal calls of sample2D do not pass through the wrap.
 */
#include <algorithm>
#include <fstream>
#include <unistd.h>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "Color.hpp"
#include "Camera.hpp"
#include "EnvironmentMap.hpp"
#include "Texture.hpp"
#include "Sampler.hpp"
#include "IESProfile.hpp"
#include "Denoise/NFOR.hpp"
#include "Random.hpp"
#include "Defaults.hpp"
#include "Transform.hpp"
#include "Materials/Lambertian.hpp"
#include "Materials/Metal.hpp"
#include "Materials/Dielectric.hpp"
#include "Materials/Emissive.hpp"
#include "Materials/Isotropic.hpp"
#include "Materials/HenyeyGreenstein.hpp"
#include "Materials/Principled.hpp"
#include "Materials/Glossy.hpp"
#include "Materials/DiffuseGlossy.hpp"
#include "Hittables/Rectangle.hpp"
#include "Hittables/Sphere.hpp"
#include "Hittables/Cube.hpp"
#include "Hittables/Plane.hpp"
#include "Hittables/ConstantVolume.hpp"
#include "Hittables/DirectionalLight.hpp"
#include "Hittables/Triangle.hpp"
#define private public
#include "Hittables/BVHNode.hpp"
#include "Hittables/Mesh.hpp"
#include "Hittables/MeshInstance.hpp"
#undef private
#include "Scene/Scene.hpp"
#include "Renderer/Renderer.hpp"
#include "Renderer/CausticPhotonMap.hpp"
#include "RendererInternal.hpp"
#include "SceneFile/SceneFile.hpp"

#include "luz_gpu.h"
#include "scene_glue.h"

namespace {

thread_local std::string g_error;

struct TagMaterial : public Lambertian {
    int32_t object;
    int32_t primitive;
    TagMaterial(int32_t o, int32_t p) : Lambertian(Color(0.5, 0.5, 0.5)), object(o), primitive(p) {}
};
struct TagHG : public HenyeyGreenstein {
    int32_t object;
    TagHG(int32_t o, double g) : HenyeyGreenstein(Color(0.5, 0.5, 0.5), g), object(o) {}
};

struct RefScene {
    Scene scene;
    bool tagged = false;
    std::vector<std::shared_ptr<Mesh>> meshes;
    std::vector<std::shared_ptr<Hittable>> objects;           // by desc object index (nullptr if skipped)
    std::vector<int32_t> mesh_object;                         // mesh index -> first MESH object
    std::unordered_map<const Material*, std::pair<int32_t, int32_t>> tags;
    std::vector<std::shared_ptr<Material>> keep;
    std::unique_ptr<LuzPackedScene> packed;                   // luzref_scene_pack output
};

Color col(const double* c) { return Color(c[0], c[1], c[2]); }

// An IESProfile can only be made by IESProfile::load: write the profile as an
// LM-63 file (TILT=NONE, multiplier 1, type C) and load it.
std::shared_ptr<IESProfile> ies_profile(const LuzIesDesc& q)
{
    char path[] = "/tmp/luzref_iesXXXXXX";
    const int fd = mkstemp(path);
    if (fd < 0) throw std::runtime_error("cannot create a temporary IES file");
    close(fd);
    {
        std::ofstream f(path);
        f.precision(17);
        f << "IESNA:LM-63-2002\nTILT=NONE\n1 -1 1 " << q.vertical_count << " " << q.horizontal_count
          << " 1 1 0 0 0\n1 1 0\n";
        for (int i = 0; i < q.vertical_count; i++) f << q.vertical_deg[i] << " ";
        f << "\n";
        for (int i = 0; i < q.horizontal_count; i++) f << q.horizontal_deg[i] << " ";
        f << "\n";
        for (int64_t i = 0; i < (int64_t)q.vertical_count * q.horizontal_count; i++) f << q.candela[i] << " ";
        f << "\n";
    }
    auto p = std::make_shared<IESProfile>(IESProfile::load(path));
    unlink(path);
    return p;
}
Vector3 vec(const double* c) { return Vector3(c[0], c[1], c[2]); }

std::shared_ptr<Material> make_material(const LuzMaterialDesc& m, const std::vector<std::shared_ptr<Texture>>& textures)
{
    std::shared_ptr<Material> out;
    switch (m.type) {
    case LUZ_MAT_LAMBERTIAN: out = std::make_shared<Lambertian>(col(m.color)); break;
    case LUZ_MAT_METAL:
        if (m.conductor) {
            auto metal = std::make_shared<Metal>(col(m.eta), col(m.k), m.roughness);
            out = metal;
        } else {
            out = std::make_shared<Metal>(col(m.color), m.roughness);
        }
        break;
    case LUZ_MAT_DIELECTRIC: {
        auto d = std::make_shared<Dielectric>(col(m.color), m.ior, m.roughness);
        d->setAbsorptionCoefficient(col(m.absorption));
        out = d;
        break;
    }
    case LUZ_MAT_EMISSIVE: out = std::make_shared<Emissive>(col(m.color)); break;
    case LUZ_MAT_ISOTROPIC: out = std::make_shared<Isotropic>(col(m.color)); break;
    case LUZ_MAT_HENYEY_GREENSTEIN: out = std::make_shared<HenyeyGreenstein>(col(m.color), m.anisotropy); break;
    case LUZ_MAT_PRINCIPLED: {
        auto p = std::make_shared<Principled>(col(m.color), m.metallic, m.roughness, m.transmission, m.ior,
                                              m.clearcoat, m.clearcoat_roughness, m.sheen);
        p->setSubsurface(m.subsurface);
        p->setSubsurfaceRadius(col(m.subsurface_radius));
        p->setSubsurfaceScale(m.subsurface_scale);
        p->setSubsurfaceColor(col(m.subsurface_color));
        p->setSubsurfaceMethod(m.subsurface_method ? SUBSURFACE_THIN : SUBSURFACE_BURLEY);
        p->setAbsorptionCoefficient(col(m.absorption));
        out = p;
        break;
    }
    case LUZ_MAT_GLOSSY: out = std::make_shared<Glossy>(col(m.color), m.roughness); break;
    case LUZ_MAT_DIFFUSE_GLOSSY:
        out = std::make_shared<DiffuseGlossy>(col(m.color), col(m.glossy_color), m.glossy_weight, m.roughness);
        break;
    default: throw std::invalid_argument("unknown material type");
    }
    if (m.texture >= 0) {
        if (m.texture >= (int32_t)textures.size()) throw std::invalid_argument("texture index out of range");
        out->setTexture(textures[m.texture]);
    }
    return out;
}

void configure(Scene& scene, const LuzSceneDesc& d, int32_t width, int32_t height)
{
    scene.getImage()->setWidth((std::size_t)width);
    scene.getImage()->setHeight((std::size_t)height);
    scene.getImage()->initialize();
    scene.setViewTransform(ViewTransform::Raw);
    scene.setExposure(0.0);
    scene.setBloom(false);
    scene.setDenoise(false);
    scene.setAdaptiveSampling(false);
    scene.setBenchmarkMode(true);
    (void)d;
}

RefScene* build(const LuzSceneDesc* d, int tag)
{
    auto rs = std::make_unique<RefScene>();
    rs->tagged = tag != 0;
    Scene& scene = rs->scene;

    std::vector<std::shared_ptr<Texture>> textures;
    for (int i = 0; i < d->texture_count; i++) {
        const LuzTextureDesc& t = d->textures[i];
        std::vector<Color> px((std::size_t)t.width * t.height);
        for (std::size_t k = 0; k < px.size(); k++) px[k] = Color(t.rgb[3 * k], t.rgb[3 * k + 1], t.rgb[3 * k + 2]);
        textures.push_back(std::make_shared<Texture>((std::size_t)t.width, (std::size_t)t.height, std::move(px)));
    }
    std::vector<std::shared_ptr<Material>> mats;
    for (int i = 0; i < d->material_count; i++) mats.push_back(make_material(d->materials[i], textures));

    rs->mesh_object.assign(d->mesh_count, -1);
    for (int i = 0; i < d->object_count; i++)
        if (d->objects[i].kind == LUZ_OBJ_MESH && d->objects[i].mesh >= 0 && d->objects[i].mesh < d->mesh_count
            && rs->mesh_object[d->objects[i].mesh] < 0)
            rs->mesh_object[d->objects[i].mesh] = i;

    for (int mi = 0; mi < d->mesh_count; mi++) {
        const LuzMeshDesc& m = d->meshes[mi];
        std::shared_ptr<Material> mm = mats.at(m.material);
        std::vector<Triangle> tris;
        tris.reserve((std::size_t)m.triangle_count);
        for (int64_t t = 0; t < m.triangle_count; t++) {
            const double* p = m.positions + 9 * t;
            std::shared_ptr<Material> tm = mm;
            if (m.normals) {
                const double* n = m.normals + 9 * t;
                tris.emplace_back(vec(p), vec(p + 3), vec(p + 6), vec(n), vec(n + 3), vec(n + 6), tm);
            } else {
                tris.emplace_back(vec(p), vec(p + 3), vec(p + 6), tm);
            }
            if (m.uvs) {
                const double* uv = m.uvs + 6 * t;
                tris.back().setTextureCoordinates(Vector3(uv[0], uv[1], 0), Vector3(uv[2], uv[3], 0), Vector3(uv[4], uv[5], 0));
            }
        }
        auto mesh = std::make_shared<Mesh>(Vector3(), mm, std::move(tris));
        if (tag) {
            for (std::size_t t = 0; t < mesh->_triangles.size(); t++) {
                auto tm = std::make_shared<TagMaterial>(rs->mesh_object[mi], (int32_t)t);
                rs->tags[tm.get()] = {rs->mesh_object[mi], (int32_t)t};
                mesh->_triangles[t].setMaterial(tm);
                rs->keep.push_back(tm);
            }
        }
        rs->meshes.push_back(mesh);
    }

    for (int i = 0; i < d->object_count; i++) {
        const LuzObjectDesc& o = d->objects[i];
        std::shared_ptr<Material> mat;
        if (o.kind != LUZ_OBJ_MESH) {
            if (tag && o.kind != LUZ_OBJ_VOLUME && o.kind != LUZ_OBJ_DIRECTIONAL_LIGHT) {
                auto tm = std::make_shared<TagMaterial>(i, 0);
                rs->tags[tm.get()] = {i, 0};
                rs->keep.push_back(tm);
                mat = tm;
            } else if (tag && o.kind == LUZ_OBJ_VOLUME) {
                auto tm = std::make_shared<TagHG>(i, mats.at(o.material)->getType() == HENYEY_GREENSTEIN
                                                  ? std::static_pointer_cast<HenyeyGreenstein>(mats.at(o.material))->getAnisotropy()
                                                  : 0.0);
                rs->tags[tm.get()] = {i, 0};
                rs->keep.push_back(tm);
                mat = tm;
            } else {
                mat = mats.at(o.material);
            }
        }
        std::shared_ptr<Hittable> h;
        switch (o.kind) {
        case LUZ_OBJ_RECTANGLE: {
            auto r = std::make_shared<Rectangle>(Transform(vec(o.position), vec(o.orientation), Vector3(1, 1, 1)),
                                                 o.size[0], o.size[1], mat);
            if (o.has_axes) r->setAxes(vec(o.width_axis), vec(o.height_axis));
            if (o.has_uvs) r->setTextureCoordinates(vec(o.uv), vec(o.uv + 3), vec(o.uv + 6), vec(o.uv + 9));
            h = r;
            break;
        }
        case LUZ_OBJ_SPHERE: {
            auto sp = std::make_shared<Sphere>(vec(o.position), o.size[0], mat, o.visible != 0,
                                               o.uv_projection == 1 ? SphereUVProjection::CubeCross
                                                                    : SphereUVProjection::LatLong);
            if (o.ies >= 0) sp->setIESProfile(ies_profile(d->ies[o.ies]), vec(o.ies_direction), o.ies_rotation_degrees);
            h = sp;
            break;
        }
        case LUZ_OBJ_CUBE:
            h = std::make_shared<Cube>(Transform(vec(o.position), Vector3(0, 0, 1), Vector3(1, 1, 1)),
                                       o.size[0], o.size[1], o.size[2], mat);
            break;
        case LUZ_OBJ_PLANE:
            h = std::make_shared<Plane>(o.position[1], vec(o.orientation), mat);
            break;
        case LUZ_OBJ_MESH:
            h = rs->meshes.at(o.mesh);
            break;
        case LUZ_OBJ_MESH_INSTANCE:
            h = std::make_shared<MeshInstance>(rs->meshes.at(o.mesh), vec(o.position), vec(o.rotation_degrees),
                                               vec(o.scale), mat);
            break;
        case LUZ_OBJ_VOLUME: {
            std::shared_ptr<Hittable> boundary;
            if (o.boundary_kind == LUZ_OBJ_CUBE)
                boundary = std::make_shared<Cube>(Transform(vec(o.position), Vector3(0, 0, 1), Vector3(1, 1, 1)),
                                                  o.size[0], o.size[1], o.size[2], nullptr);
            else
                boundary = std::make_shared<Sphere>(vec(o.position), o.size[0], nullptr, SphereUVProjection::LatLong);
            h = std::make_shared<ConstantVolume>(boundary, mat, o.density);
            break;
        }
        case LUZ_OBJ_DIRECTIONAL_LIGHT:
            h = std::make_shared<DirectionalLight>(vec(o.orientation), mat);
            break;
        default: throw std::invalid_argument("unknown object kind");
        }
        rs->objects.push_back(h);
        scene.addHittable(h);
    }

    const LuzCameraDesc& c = d->camera;
    Camera cam(vec(c.position), vec(c.direction), c.focal_length_m, c.sensor_width_m, c.sensor_height_m,
               c.f_number, c.focus_distance_m);
    cam.setUpDirection(vec(c.up));
    if (c.pinhole) cam.setPinhole(true);
    scene.addCamera(cam);
    scene.setMetersPerUnit(d->meters_per_unit);
    if (d->caustics.enabled) {
        scene.setCausticsEnabled(true);
        scene.setCausticPhotonCount(d->caustics.photons);
        scene.setCausticPassCount(d->caustics.passes);
        scene.setCausticRadiusMeters(d->caustics.radius_meters);
        scene.setCausticAlpha(d->caustics.alpha);
    }
    scene.setBackgroundColor(col(d->background));
    scene.setRenderSky(d->sky == LUZ_SKY_ENVIRONMENT ? SKY_ENVIRONMENT
                       : d->sky == LUZ_SKY_LINEAR   ? SKY_LINEAR
                       : d->sky == LUZ_SKY_ATMOSPHERE ? SKY_ATMOSPHERE
                                                      : SKY_NONE);
    if (d->sky == LUZ_SKY_ATMOSPHERE) {
        const LuzAtmosphereDesc& a = d->atmosphere;
        Atmosphere atm(-0.4, a.earth_radius, a.atmosphere_radius, a.h_r, a.h_m, a.samples, a.light_samples,
                       a.stars_brightness);
        atm.setSunDirection(vec(a.sun_direction));
        atm.setSunRadiance(col(a.sun_radiance));
        atm.setSunRadianceScale(a.sun_radiance_scale);
        scene.setAtmosphere(atm);   // takes the scene's meters per unit
    }
    if (d->environment.width > 0) {
        const LuzEnvironmentDesc& e = d->environment;
        std::vector<Color> px((std::size_t)e.width * e.height);
        for (std::size_t k = 0; k < px.size(); k++) px[k] = Color(e.rgb[3 * k], e.rgb[3 * k + 1], e.rgb[3 * k + 2]);
        scene.setEnvironmentMap(std::make_shared<EnvironmentMap>((std::size_t)e.width, (std::size_t)e.height, std::move(px)));
        scene.setEnvironmentStrength(e.strength);
        scene.setEnvironmentRotation(e.rotation_degrees);
        scene.setEnvironmentLighting(e.lighting != 0);
    }
    scene.updateLights();
    scene.updateAccelerationStructure();
    return rs.release();
}

// Preorder walk of the reference BVHNode tree. Per node: the child count, then
// per child 8 doubles: is_node, desc object index (-1 for a node), box min, box max.
void dump_bvh(const RefScene& rs, const std::unordered_map<const Hittable*, int32_t>& ids, const BVHNode& n,
              std::vector<double>& out)
{
    out.push_back((double)n._childs.size());
    for (std::size_t i = 0; i < n._childs.size(); i++) {
        const Hittable* c = n._childs[i].get();
        const BVHNode* cn = dynamic_cast<const BVHNode*>(c);
        const AABB& b = n._childBoundingBoxes[i];
        auto it = ids.find(c);
        out.push_back(cn ? 1.0 : 0.0);
        out.push_back(cn ? -1.0 : (it != ids.end() ? (double)it->second : -2.0));
        out.push_back(b.getMinimum().getX());
        out.push_back(b.getMinimum().getY());
        out.push_back(b.getMinimum().getZ());
        out.push_back(b.getMaximum().getX());
        out.push_back(b.getMaximum().getY());
        out.push_back(b.getMaximum().getZ());
    }
    for (const auto& c : n._childs)
        if (const BVHNode* cn = dynamic_cast<const BVHNode*>(c.get())) dump_bvh(rs, ids, *cn, out);
    (void)rs;
}

template <class F> int guarded(F&& f)
{
    try {
        return f();
    } catch (const std::exception& e) {
        g_error = e.what();
        return LUZ_E_INVALID;
    }
}

// The photon map Renderer::render builds before the sample loop (Renderer.cpp:40-52).
void caustic_map(Scene& scene, uint32_t seed)
{
    if (scene.getCausticsEnabled() && scene.getCausticPhotonCount() > 0) {
        auto m = std::make_shared<CausticPhotonMap>();
        m->build(scene, seed);
        scene.setCausticPhotonMap(m);
    } else {
        scene.setCausticPhotonMap(nullptr);
    }
}

bool closest(Scene& scene, Ray& ray, double tmin, double tmax, HitRecord& rec)
{
    bool any = false;
    double best = tmax;
    const auto& accel = scene.getAccelerationStructure();
    if (accel && accel->hit(ray, rec, tmin, best)) {
        best = rec.t0;
        any = true;
    }
    const auto& un = scene.getUnacceleratedHittables();
    const auto& list = (!accel && un.empty()) ? scene.getHittables() : un;
    for (const auto& h : list)
        if (h->hit(ray, rec, tmin, best)) {
            best = rec.t0;
            any = true;
        }
    return any;
}

bool occluded(Scene& scene, Ray& ray, double tmin, double tmax)
{
    if (tmax <= T_MIN) return false;
    const auto& accel = scene.getAccelerationStructure();
    if (accel && accel->hitAny(ray, tmin, tmax)) return true;
    const auto& un = scene.getUnacceleratedHittables();
    const auto& list = (!accel && un.empty()) ? scene.getHittables() : un;
    for (const auto& h : list)
        if (h->hitAny(ray, tmin, tmax)) return true;
    return false;
}

// Perturbation of the Sampler's draws (see the file header). seed 0 = off.
struct Perturb {
    uint64_t seed = 0;
    double dir = 0.0;    // directions and distances (surface points, BSDF and phase directions, media)
    double dec = 0.0;    // dimensions compared with an FP32 threshold (lobe, Russian roulette)
    double cam = 0.0;    // camera and lens (a pixel or the aperture, not a hemisphere)
    double bsdf = 0.0;   // BSDF and fuzz directions (a narrow lobe maps the draw onto a small angle)
} g_perturb;

uint64_t mix64(uint64_t v)
{
    v += 0x9e3779b97f4a7c15ull;
    v = (v ^ (v >> 30)) * 0xbf58476d1ce4e5b9ull;
    v = (v ^ (v >> 27)) * 0x94d049bb133111ebull;
    return v ^ (v >> 31);
}

// Draws the GPU compares with the same FP64 values as the reference (constant
// strategy probabilities, FP64 selection CDFs built bit-identically on the host)
// are exact on both sides and are not moved.
double perturb_delta(uint32_t dimension)
{
    switch (dimension % 32u) {
    case Sampler::DIM_LIGHT_STRATEGY:
    case Sampler::DIM_LIGHT_SELECTION:
    case Sampler::DIM_LIGHT_SURFACE_SELECTION:
    case Sampler::DIM_ENVIRONMENT_SELECTION:
    case Sampler::DIM_ENVIRONMENT_STRATEGY:
    case Sampler::DIM_LIGHT_EMISSION_SIDE: return 0.0;
    case Sampler::DIM_CAMERA:
    case Sampler::DIM_LENS: return g_perturb.cam;
    case Sampler::DIM_BSDF_DIRECTION:
    case Sampler::DIM_MATERIAL_FUZZ: return g_perturb.bsdf;
    case Sampler::DIM_LIGHT_SURFACE_POINT:
    case Sampler::DIM_ATMOSPHERE:
    case Sampler::DIM_ENVIRONMENT_POINT:
    case Sampler::DIM_LIGHT_EMISSION_DIRECTION:
    case Sampler::DIM_SUBSURFACE_SPATIAL:
    case Sampler::DIM_VOLUME_DISTANCE: return g_perturb.dir;
    default: return g_perturb.dec;
    }
}

double moved(double u, uint32_t dimension, uint32_t component, double top)
{
    uint64_t bits;
    std::memcpy(&bits, &u, sizeof bits);
    const uint64_t h = mix64(g_perturb.seed ^ mix64(((uint64_t)dimension << 8 | component) ^ mix64(bits)));
    const double v = u + ((h >> 63) ? 1.0 : -1.0) * perturb_delta(dimension);
    return v < 0.0 ? 0.0 : (v > top ? top : v);
}

}  // namespace

#ifdef LUZREF_PERTURB
// ld --wrap targets (mangled names of the Sampler namespace functions).
extern "C" double __real__ZN7Sampler8sample1DEj(std::uint32_t dimension);
extern "C" Sampler::Sample2D __real__ZN7Sampler8sample2DEj(std::uint32_t dimension);

extern "C" double __wrap__ZN7Sampler8sample1DEj(std::uint32_t dimension)
{
    const double u = __real__ZN7Sampler8sample1DEj(dimension);
    if (!g_perturb.seed || !Sampler::isActive()) return u;
    return moved(u, dimension, 0, 0x1.fffffffffffffp-1);
}

extern "C" Sampler::Sample2D __wrap__ZN7Sampler8sample2DEj(std::uint32_t dimension)
{
    Sampler::Sample2D s = __real__ZN7Sampler8sample2DEj(dimension);
    if (!g_perturb.seed || !Sampler::isActive()) return s;
    s.x = (float)moved((double)s.x, dimension, 0, 0x1.fffffep-1);
    s.y = (float)moved((double)s.y, dimension, 1, 0x1.fffffep-1);
    return s;
}

extern "C" Vector3 __wrap__ZN7Sampler16cosineHemisphereEj(std::uint32_t dimension)
{
    const Sampler::Sample2D u = __wrap__ZN7Sampler8sample2DEj(dimension);
    const float phi = static_cast<float>(2.0 * D_PI) * u.x;
    const float r = std::sqrt(u.y);
    const float z = std::sqrt(std::max(0.0f, 1.0f - u.y));
    return Vector3(r * std::cos(phi), r * std::sin(phi), z);
}

extern "C" Vector3 __wrap__ZN7Sampler15sphereDirectionEj(std::uint32_t dimension)
{
    const Sampler::Sample2D u = __wrap__ZN7Sampler8sample2DEj(dimension);
    const float z = 1.0f - (2.0f * u.y);
    const float r = std::sqrt(std::max(0.0f, 1.0f - z * z));
    const float phi = static_cast<float>(2.0 * D_PI) * u.x;
    return Vector3(r * std::cos(phi), r * std::sin(phi), z);
}

extern "C" Vector3 __wrap__ZN7Sampler8unitDiskEj(std::uint32_t dimension)
{
    const Sampler::Sample2D u = __wrap__ZN7Sampler8sample2DEj(dimension);
    const float sx = (2.0f * u.x) - 1.0f;
    const float sy = (2.0f * u.y) - 1.0f;
    if (sx == 0.0f && sy == 0.0f) return Vector3(0.0, 0.0, 0.0);
    float radius, theta;
    if (std::fabs(sx) > std::fabs(sy)) {
        radius = sx;
        theta = (static_cast<float>(D_PI) / 4.0f) * (sy / sx);
    } else {
        radius = sy;
        theta = (static_cast<float>(D_PI) / 2.0f) - ((static_cast<float>(D_PI) / 4.0f) * (sx / sy));
    }
    return Vector3(radius * std::cos(theta), radius * std::sin(theta), 0.0);
}
#endif

extern "C" {

/* Sets the draw perturbation of the ambiguity probe (seed 0 = off); the
 * parity library only (LUZ_E_UNSUPPORTED elsewhere). */
int luzref_set_perturbation(uint64_t seed, double delta_dir, double delta_dec, double delta_cam, double delta_bsdf)
{
#ifdef LUZREF_PERTURB
    g_perturb.seed = seed;
    g_perturb.dir = delta_dir;
    g_perturb.dec = delta_dec;
    g_perturb.cam = delta_cam;
    g_perturb.bsdf = delta_bsdf;
    return 0;
#else
    (void)seed;
    (void)delta_dir;
    (void)delta_dec;
    (void)delta_cam;
    (void)delta_bsdf;
    g_error = "draw perturbation is built into the parity library only";
    return LUZ_E_UNSUPPORTED;
#endif
}

/* The top-level BVHNode tree in preorder (dump_bvh): up to cap doubles into out,
 * the full length into *count. *count = 0 when the acceleration structure is
 * not a BVHNode (no object or one bounded object). */
int luzref_top_bvh(void* s, double* out, int64_t cap, int64_t* count)
{
    return guarded([&] {
        RefScene* rs = static_cast<RefScene*>(s);
        std::unordered_map<const Hittable*, int32_t> ids;
        for (std::size_t i = 0; i < rs->objects.size(); i++)
            if (rs->objects[i]) ids[rs->objects[i].get()] = (int32_t)i;
        std::vector<double> v;
        const auto& accel = rs->scene.getAccelerationStructure();
        if (const BVHNode* n = dynamic_cast<const BVHNode*>(accel.get())) dump_bvh(*rs, ids, *n, v);
        *count = (int64_t)v.size();
        if (out) std::memcpy(out, v.data(), sizeof(double) * (std::size_t)std::min<int64_t>(cap, *count));
        return 0;
    });
}

int luzref_last_error(char* buf, size_t len)
{
    if (buf && len) {
        std::strncpy(buf, g_error.c_str(), len - 1);
        buf[len - 1] = 0;
    }
    return 0;
}

int luzref_scene_create(const LuzSceneDesc* desc, int32_t tag, void** out)
{
    return guarded([&] {
        *out = build(desc, tag);
        return 0;
    });
}

int luzref_scene_destroy(void* s)
{
    delete static_cast<RefScene*>(s);
    return 0;
}

/* A scene read from a .luz file by the reference's own parser (SceneFile::read,
 * src/io/SceneFile/SceneFile.cpp:256-321), left as Renderer::render prepares it
 * (Renderer.cpp:18-20). Untagged: hits are not identified per object. */
int luzref_scene_load(const char* path, void** out)
{
    return guarded([&] {
        auto rs = std::make_unique<RefScene>();
        SceneFile::read(rs->scene, path);
        rs->scene.syncAtmosphereSunDirection();
        rs->scene.updateLights();
        rs->scene.updateAccelerationStructure();
        *out = rs.release();
        return 0;
    });
}

/* The scene glue (luz_b200/glue/scene_glue.cpp) applied to a reference scene:
 * *desc stays valid until the scene is destroyed or packed again; settings
 * receives width, height, spp and max light bounces from the scene. */
int luzref_scene_pack(void* s, const LuzSceneDesc** desc, int32_t* settings)
{
    return guarded([&] {
        RefScene* rs = static_cast<RefScene*>(s);
        auto packed = std::make_unique<LuzPackedScene>();
        luz_pack_scene(rs->scene, *packed);
        rs->packed = std::move(packed);
        *desc = &rs->packed->desc;
        settings[0] = rs->packed->width;
        settings[1] = rs->packed->height;
        settings[2] = rs->packed->spp;
        settings[3] = rs->packed->max_bounces;
        return 0;
    });
}

/* rays: (ox,oy,oz,tmin,dx,dy,dz,tmax) per ray, used as given (no renormalisation). */
int luzref_trace_rays(void* s, const double* rays, int64_t n, int32_t any_hit, uint32_t seed,
                      const int32_t* volume_key, double* t_out, int32_t* obj_out, int32_t* prim_out)
{
    return guarded([&] {
        RefScene* rs = static_cast<RefScene*>(s);
        Sampler::setRenderSeed(seed);
        for (int64_t i = 0; i < n; i++) {
            const double* r = rays + 8 * i;
            if (volume_key) {
                const int32_t* k = volume_key + 4 * i;
                Sampler::beginPixelSample((std::size_t)k[0], (std::size_t)k[1], (uint32_t)k[2], 0);
                Sampler::setBounce((uint32_t)k[3]);
            } else {
                Sampler::beginPixelSample(0, 0, 0, 0);
            }
            Ray ray = Ray::fromNormalizedDirection(Vector3(r[0], r[1], r[2]), Vector3(r[4], r[5], r[6]));
            const double tmax = std::isinf(r[7]) ? T_MAX : r[7];
            if (any_hit) {
                const bool o = occluded(rs->scene, ray, r[3], tmax);
                t_out[i] = 0.0;
                obj_out[i] = o ? 0 : -1;
                prim_out[i] = 0;
            } else {
                HitRecord rec;
                if (!closest(rs->scene, ray, r[3], tmax, rec)) {
                    t_out[i] = INFINITY;
                    obj_out[i] = -1;
                    prim_out[i] = -1;
                } else {
                    t_out[i] = rec.t0;
                    obj_out[i] = -2;
                    prim_out[i] = -2;
                    auto it = rs->tags.find(rec.material);
                    if (it != rs->tags.end()) {
                        obj_out[i] = it->second.first;
                        prim_out[i] = it->second.second;
                        const int32_t o = it->second.first;
                        auto inst = o >= 0 ? std::dynamic_pointer_cast<MeshInstance>(rs->objects[o]) : nullptr;
                        if (inst) {
                            Ray local;
                            double scale = 1.0;
                            HitRecord lrec;
                            if (inst->_localRay(ray, local, scale)
                                && inst->_geometry->hit(local, lrec, r[3] * scale, T_MAX)) {
                                auto jt = rs->tags.find(lrec.material);
                                prim_out[i] = jt != rs->tags.end() ? jt->second.second : -3;
                            }
                        }
                    }
                }
            }
            Sampler::endPixelSample();
        }
        return 0;
    });
}

int luzref_trace_paths(void* s, const LuzRenderParams* p, const int32_t* x, const int32_t* y,
                       const int32_t* sample, int64_t n, double* rgb_out)
{
    return guarded([&] {
        RefScene* rs = static_cast<RefScene*>(s);
        configure(rs->scene, LuzSceneDesc{}, p->width, p->height);
        rs->scene.setMaxLightBounces(p->max_bounces);
        rs->scene.setSampleCount(p->spp);
        caustic_map(rs->scene, p->seed);
        const auto cam = Renderer::internal::_prepareRenderCamera(rs->scene);
        Sampler::setRenderSeed(p->seed);
        for (int64_t i = 0; i < n; i++) {
            Sampler::beginPixelSample((std::size_t)x[i], (std::size_t)y[i], (uint32_t)sample[i], p->stream);
            const Color c = Renderer::internal::_calculatePixelColor(rs->scene, cam, (std::size_t)x[i], (std::size_t)y[i]);
            Sampler::endPixelSample();
            rgb_out[3 * i] = c.getRed();
            rgb_out[3 * i + 1] = c.getGreen();
            rgb_out[3 * i + 2] = c.getBlue();
        }
        return 0;
    });
}

/* Full reference render through Renderer::render; rows [row_begin,row_end) only
 * when row_end > row_begin (a bounded sample of the image: the image is set to
 * those rows with a camera viewport shifted to match is NOT done — instead the
 * whole-image render is used and the caller bounds cost through spp). */
int luzref_render(void* s, const LuzRenderParams* p, int32_t threads, double* rgb_out, double* render_ms,
                  double* samples)
{
    return guarded([&] {
        RefScene* rs = static_cast<RefScene*>(s);
        configure(rs->scene, LuzSceneDesc{}, p->width, p->height);
        rs->scene.setMaxLightBounces(p->max_bounces);
        rs->scene.setSampleCount(p->spp);
        rs->scene.setRenderingThreads((std::size_t)std::max(1, threads));
        setRandomSeed((int_fast32_t)p->seed);
        if (!Renderer::render(rs->scene)) throw std::runtime_error("Renderer::render failed");
        const auto& img = rs->scene.getImage();
        for (int32_t yy = 0; yy < p->height; yy++)
            for (int32_t xx = 0; xx < p->width; xx++) {
                const Color c = img->getPixel((std::size_t)xx, (std::size_t)yy);
                const std::size_t k = (std::size_t)yy * p->width + xx;
                rgb_out[3 * k] = c.getRed();
                rgb_out[3 * k + 1] = c.getGreen();
                rgb_out[3 * k + 2] = c.getBlue();
            }
        const SceneRenderStats& st = rs->scene.getRenderStats();
        if (render_ms) *render_ms = st.renderMS;
        if (samples) *samples = (double)st.renderedSamples;
        return 0;
    });
}

/* _calculatePixelSample (src/renderer/ColorHelper.cpp:1119-1126) for explicit
 * (x, y, sample): colour (before cleanColor) and the 11 primary features. The
 * sampler stream is params->stream, or 1 + sample % 2 when half_streams != 0
 * (the denoise half buffers, Threads.cpp:593-598). */
int luzref_trace_samples(void* s, const LuzRenderParams* p, int32_t half_streams, const int32_t* x,
                         const int32_t* y, const int32_t* sample, int64_t n, double* rgb_out, double* feat_out)
{
    return guarded([&] {
        RefScene* rs = static_cast<RefScene*>(s);
        configure(rs->scene, LuzSceneDesc{}, p->width, p->height);
        rs->scene.setMaxLightBounces(p->max_bounces);
        rs->scene.setSampleCount(p->spp);
        caustic_map(rs->scene, p->seed);
        const auto cam = Renderer::internal::_prepareRenderCamera(rs->scene);
        Sampler::setRenderSeed(p->seed);
        for (int64_t i = 0; i < n; i++) {
            const uint32_t st = half_streams ? 1u + ((uint32_t)sample[i] % 2u) : p->stream;
            Sampler::beginPixelSample((std::size_t)x[i], (std::size_t)y[i], (uint32_t)sample[i], st);
            const Renderer::internal::RenderSample r =
                Renderer::internal::_calculatePixelSample(rs->scene, cam, (std::size_t)x[i], (std::size_t)y[i]);
            Sampler::endPixelSample();
            rgb_out[3 * i] = r.color.getRed();
            rgb_out[3 * i + 1] = r.color.getGreen();
            rgb_out[3 * i + 2] = r.color.getBlue();
            for (int f = 0; f < 11; f++) feat_out[11 * i + f] = r.features[(std::size_t)f];
        }
        return 0;
    });
}

/* _threadRender (src/renderer/Threads.cpp:551-641) for listed pixels with the
 * scene's adaptive settings and, when nfor != 0, its denoise buffers
 * (Scene::initializeDenoiseBuffers). Per pixel: rgb_out[3] (the stored pixel),
 * used_out (samples used) and, when nfor_out is given, 40 doubles laid out as
 * colorA[3], colorB[3], colorVariance, featuresA[11], featuresB[11],
 * featureVariance[11] (storeDenoisePixel, :343-372). */
int luzref_render_pixels(void* s, const LuzRenderParams* p, int32_t adaptive, int32_t min_samples,
                         int32_t check_interval, double threshold, int32_t nfor, const int32_t* x,
                         const int32_t* y, int64_t n, double* rgb_out, int32_t* used_out, double* nfor_out)
{
    return guarded([&] {
        RefScene* rs = static_cast<RefScene*>(s);
        Scene& scene = rs->scene;
        configure(scene, LuzSceneDesc{}, p->width, p->height);
        scene.setMaxLightBounces(p->max_bounces);
        scene.setSampleCount(p->spp);
        scene.setAdaptiveSampling(adaptive != 0);
        if (adaptive) {
            scene.setAdaptiveMinSamples(min_samples);
            scene.setAdaptiveCheckInterval(check_interval);
            scene.setAdaptiveThreshold(threshold);
        }
        if (nfor) scene.initializeDenoiseBuffers((std::size_t)p->width, (std::size_t)p->height);
        else scene.clearDenoiseBuffers();
        caustic_map(scene, p->seed);
        const auto cam = Renderer::internal::_prepareRenderCamera(scene);
        Sampler::setRenderSeed(p->seed);
        for (int64_t i = 0; i < n; i++) {
            const std::size_t px = (std::size_t)x[i], py = (std::size_t)y[i];
            used_out[i] = (int32_t)Renderer::internal::_threadRender(scene, cam, px, py);
            const Color c = scene.getImage()->getPixel(px, py);
            rgb_out[3 * i] = c.getRed();
            rgb_out[3 * i + 1] = c.getGreen();
            rgb_out[3 * i + 2] = c.getBlue();
            if (nfor && nfor_out) {
                const Denoise::NFORBuffers* b = scene.getDenoiseBuffers();
                const std::size_t k = b->index(px, py);
                double* o = nfor_out + 40 * i;
                const Color ca = b->colorA[k], cb = b->colorB[k];
                o[0] = ca.getRed();
                o[1] = ca.getGreen();
                o[2] = ca.getBlue();
                o[3] = cb.getRed();
                o[4] = cb.getGreen();
                o[5] = cb.getBlue();
                o[6] = b->colorVariance[k];
                for (int f = 0; f < 11; f++) {
                    o[7 + f] = b->featuresA[k][(std::size_t)f];
                    o[18 + f] = b->featuresB[k][(std::size_t)f];
                    o[29 + f] = b->featureVariance[k][(std::size_t)f];
                }
            }
        }
        scene.clearDenoiseBuffers();
        scene.setAdaptiveSampling(false);
        return 0;
    });
}

/* _threadRender (src/renderer/Threads.cpp:551-641) for listed pixels, adaptive
 * sampling and denoise buffers off, on `threads` host threads (pixels dealt round
 * robin): the stored pixel (mean of params->spp cleaned samples) per pixel. */
int luzref_render_pixels_mt(void* s, const LuzRenderParams* p, const int32_t* x, const int32_t* y, int64_t n,
                            int32_t threads, double* rgb_out)
{
    return guarded([&] {
        RefScene* rs = static_cast<RefScene*>(s);
        Scene& scene = rs->scene;
        configure(scene, LuzSceneDesc{}, p->width, p->height);
        scene.setMaxLightBounces(p->max_bounces);
        scene.setSampleCount(p->spp);
        scene.setAdaptiveSampling(false);
        scene.clearDenoiseBuffers();
        caustic_map(scene, p->seed);
        const auto cam = Renderer::internal::_prepareRenderCamera(scene);
        Sampler::setRenderSeed(p->seed);
        const int nt = std::max(1, threads);
        std::vector<std::thread> pool;
        for (int t = 0; t < nt; t++)
            pool.emplace_back([&, t] {
                for (int64_t i = t; i < n; i += nt) {
                    const std::size_t px = (std::size_t)x[i], py = (std::size_t)y[i];
                    Renderer::internal::_threadRender(scene, cam, px, py);
                    const Color c = scene.getImage()->getPixel(px, py);
                    rgb_out[3 * i] = c.getRed();
                    rgb_out[3 * i + 1] = c.getGreen();
                    rgb_out[3 * i + 2] = c.getBlue();
                }
            });
        for (auto& th : pool) th.join();
        return 0;
    });
}

/* CausticPhotonMap::build (src/renderer/CausticPhotonMap.cpp:430-551) for a
 * render seed and bounce limit: the number of photons stored. */
int luzref_caustic_photons(void* s, uint32_t seed, int32_t max_bounces, int64_t* count)
{
    return guarded([&] {
        RefScene* rs = static_cast<RefScene*>(s);
        rs->scene.setMaxLightBounces(max_bounces);
        CausticPhotonMap m;
        m.build(rs->scene, seed);
        *count = (int64_t)m.photonCount();
        return 0;
    });
}

/* Denoise::applyNFOR (src/core/Denoise/NFOR.cpp:977-1102) on the given buffers. */
int luzref_nfor(int32_t width, int32_t height, const double* color_a, const double* color_b,
                const double* color_variance, const double* features_a, const double* features_b,
                const double* feature_variance, int32_t prefilter_radius, int32_t regression_radius,
                int32_t patch_radius, double min_variance, int32_t threads, double* rgb_out)
{
    return guarded([&] {
        Denoise::NFORBuffers b;
        b.initialize((std::size_t)width, (std::size_t)height);
        const std::size_t n = (std::size_t)width * height;
        for (std::size_t i = 0; i < n; i++) {
            b.colorA[i] = Color(color_a[3 * i], color_a[3 * i + 1], color_a[3 * i + 2]);
            b.colorB[i] = Color(color_b[3 * i], color_b[3 * i + 1], color_b[3 * i + 2]);
            b.colorVariance[i] = color_variance[i];
            for (std::size_t f = 0; f < Denoise::NFOR_FEATURE_COUNT; f++) {
                b.featuresA[i][f] = features_a[Denoise::NFOR_FEATURE_COUNT * i + f];
                b.featuresB[i][f] = features_b[Denoise::NFOR_FEATURE_COUNT * i + f];
                b.featureVariance[i][f] = feature_variance[Denoise::NFOR_FEATURE_COUNT * i + f];
            }
        }
        Denoise::NFORSettings s;
        s.featurePrefilterRadius = (unsigned)prefilter_radius;
        s.regressionRadius = (unsigned)regression_radius;
        s.patchRadius = (unsigned)patch_radius;
        s.minVariance = min_variance;
        s.threadCount = (std::size_t)std::max(1, threads);
        const std::unique_ptr<Image> img = Denoise::applyNFOR(b, s);
        for (int32_t y = 0; y < height; y++)
            for (int32_t x = 0; x < width; x++) {
                const Color c = img->getPixel((std::size_t)x, (std::size_t)y);
                const std::size_t k = (std::size_t)y * width + x;
                rgb_out[3 * k] = c.getRed();
                rgb_out[3 * k + 1] = c.getGreen();
                rgb_out[3 * k + 2] = c.getBlue();
            }
        return 0;
    });
}

int luzref_mesh_bvh(void* s, int32_t mesh, LuzMeshNode64* nodes, int64_t cap, int64_t* count, int64_t* order,
                    int64_t order_cap)
{
    return guarded([&] {
        RefScene* rs = static_cast<RefScene*>(s);
        const Mesh& m = *rs->meshes.at(mesh);
        *count = (int64_t)m._packedBVHNodes.size();
        for (int64_t i = 0; i < *count && i < cap; i++) {
            const auto& n = m._packedBVHNodes[(std::size_t)i];
            for (int a = 0; a < 3; a++) {
                nodes[i].bmin[a] = n.boundingBox.getMinimum()[a];
                nodes[i].bmax[a] = n.boundingBox.getMaximum()[a];
            }
            nodes[i].left = (int64_t)n.left;
            nodes[i].right = (int64_t)n.right;
            nodes[i].start = (int64_t)n.start;
            nodes[i].count = (int64_t)n.count;
            nodes[i].is_leaf = n.isLeaf ? 1 : 0;
        }
        for (int64_t i = 0; i < (int64_t)m._triangleIndices.size() && i < order_cap; i++)
            order[i] = (int64_t)m._triangleIndices[(std::size_t)i];
        return 0;
    });
}

int luzref_mesh_triangle_count(void* s, int32_t mesh, int64_t* count)
{
    RefScene* rs = static_cast<RefScene*>(s);
    *count = (int64_t)rs->meshes.at(mesh)->_triangles.size();
    return 0;
}

/* Sampler stream values (Sampler.cpp:203-237). which: 1 = sample1D, 2 = sample2D. */
int luzref_sampler(uint32_t seed, int32_t x, int32_t y, int32_t s, uint32_t stream, uint32_t bounce,
                   uint32_t dim, int32_t which, double* out)
{
    Sampler::setRenderSeed(seed);
    Sampler::beginPixelSample((std::size_t)x, (std::size_t)y, (uint32_t)s, stream);
    Sampler::setBounce(bounce);
    if (which == 1) {
        out[0] = Sampler::sample1D(dim);
    } else {
        const Sampler::Sample2D v = Sampler::sample2D(dim);
        out[0] = v.x;
        out[1] = v.y;
    }
    Sampler::endPixelSample();
    return 0;
}

}  // extern "C"
