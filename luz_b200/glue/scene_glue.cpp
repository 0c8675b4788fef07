/*
 * scene_glue.cpp — Scene -> LuzSceneDesc (see scene_glue.h).
 *
 * Walks Scene::getHittables() in Scene::addHittable order and maps each
 * reference class onto one LuzObjectDesc:
 *   Rectangle        -> LUZ_OBJ_RECTANGLE  (src/core/Hittables/Rectangle.cpp)
 *   Sphere           -> LUZ_OBJ_SPHERE     (Sphere.cpp; IES profile included)
 *   Cube             -> LUZ_OBJ_CUBE       (Cube.cpp:79-103: axis-aligned faces)
 *   Plane            -> LUZ_OBJ_PLANE      (Plane.cpp)
 *   Mesh             -> LUZ_OBJ_MESH       (Mesh.cpp:343-382, packed or legacy triangles)
 *   Triangle         -> LUZ_OBJ_MESH of one triangle: Mesh::sampleLight picks the
 *                       triangle from its own dimension (DIM_LIGHT_SURFACE_SELECTION,
 *                       Mesh.cpp:895-935), so a one-triangle mesh samples, hits and
 *                       weighs as the lone Triangle does
 *   MeshInstance     -> LUZ_OBJ_MESH_INSTANCE (MeshInstance.cpp:48-94; Euler angles
 *                       recovered from the stored sines and cosines)
 *   ConstantVolume   -> LUZ_OBJ_VOLUME     (sphere or cube boundary)
 *   DirectionalLight -> LUZ_OBJ_DIRECTIONAL_LIGHT
 *   the scene file's deferred mesh loads (DeferredHittable,
 *   src/io/SceneFile/Objects.cpp:223-290) are resolved and mapped as what they
 *   wrap.
 * Materials and textures are shared by pointer, as in the reference, and
 * packed once each. Camera, sky, background, environment map, atmosphere (as
 * synchronised with the first directional light), meters per unit and the
 * caustic photon map settings come from the Scene's getters.
 */
#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <functional>
#include <future>
#include <iostream>
#include <map>
#include <memory>
#include <mutex>
#include <optional>
#include <random>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <typeinfo>
#include <unordered_map>
#include <vector>

// Private members are read in this translation unit only (the reference's
// classes expose few getters); nothing is written through this access.
#define private public
#define protected public
#include "Color.hpp"
#include "Camera.hpp"
#include "Atmosphere.hpp"
#include "EnvironmentMap.hpp"
#include "Texture.hpp"
#include "Transform.hpp"
#include "IESProfile.hpp"
#include "Materials/Material.hpp"
#include "Materials/MaterialTypes.hpp"
#include "Materials/Lambertian.hpp"
#include "Materials/Metal.hpp"
#include "Materials/Dielectric.hpp"
#include "Materials/Emissive.hpp"
#include "Materials/Isotropic.hpp"
#include "Materials/HenyeyGreenstein.hpp"
#include "Materials/Principled.hpp"
#include "Materials/Glossy.hpp"
#include "Materials/DiffuseGlossy.hpp"
#include "Hittables/Hittable.hpp"
#include "Hittables/Rectangle.hpp"
#include "Hittables/Sphere.hpp"
#include "Hittables/Cube.hpp"
#include "Hittables/Plane.hpp"
#include "Hittables/Triangle.hpp"
#include "Hittables/Mesh.hpp"
#include "Hittables/MeshInstance.hpp"
#include "Hittables/ConstantVolume.hpp"
#include "Hittables/DirectionalLight.hpp"
#include "Hittables/PerlinSphere.hpp"
#include "Scene/Scene.hpp"
#undef protected
#undef private

#include "scene_glue.h"

namespace {

// Same members, in the same order, as the scene file's deferred mesh wrapper
// (src/io/SceneFile/Objects.cpp:223-290), which lives in an anonymous
// namespace there; inside the Luz tree an accessor on that class replaces
// this mirror.
struct DeferredMirror : public Hittable {
    std::shared_future<std::shared_ptr<Hittable>> future;
    mutable std::once_flag once;
    mutable std::shared_ptr<Hittable> hittable;
};

[[noreturn]] void unsupported(const std::string& what)
{
    throw std::runtime_error("GPU scene packing: " + what + " is not supported by the GPU path.");
}

void put(double* dst, const Vector3& v)
{
    dst[0] = v.getX();
    dst[1] = v.getY();
    dst[2] = v.getZ();
}

void put(double* dst, const Color& c)
{
    dst[0] = c.getRed();
    dst[1] = c.getGreen();
    dst[2] = c.getBlue();
}

double degrees(double s, double c) { return std::atan2(s, c) * (180.0 / M_PI); }

struct Packer {
    LuzPackedScene& out;
    std::unordered_map<const Material*, int32_t> material_index;
    std::unordered_map<const Texture*, int32_t> texture_index;
    std::unordered_map<const Mesh*, int32_t> mesh_index;
    std::unordered_map<const IESProfile*, int32_t> ies_index;
    // Arrays are appended while packing; pointers into them are set by finish().

    explicit Packer(LuzPackedScene& o) : out(o) {}

    int32_t texture(const std::shared_ptr<Texture>& t)
    {
        if (!t) return -1;
        auto it = texture_index.find(t.get());
        if (it != texture_index.end()) return it->second;
        if (t->_width == 0 || t->_height == 0 || t->_pixels.size() != t->_width * t->_height)
            unsupported("an empty texture");
        std::vector<double> px(3 * t->_pixels.size());
        for (std::size_t k = 0; k < t->_pixels.size(); k++) put(&px[3 * k], t->_pixels[k]);
        LuzTextureDesc d{};
        d.width = (int32_t)t->_width;
        d.height = (int32_t)t->_height;
        out.texels.push_back(std::move(px));
        out.textures.push_back(d);
        const int32_t i = (int32_t)out.textures.size() - 1;
        texture_index[t.get()] = i;
        return i;
    }

    int32_t material(const Material* m)
    {
        if (!m) unsupported("a hittable without a material");
        auto it = material_index.find(m);
        if (it != material_index.end()) return it->second;
        LuzMaterialDesc d{};
        d.texture = -1;
        d.roughness_texture = -1;
        put(d.color, m->_color);
        switch (m->getType()) {
        case LAMBERTIAN: d.type = LUZ_MAT_LAMBERTIAN; break;
        case METAL: {
            auto* x = static_cast<const Metal*>(m);
            d.type = LUZ_MAT_METAL;
            d.roughness = x->_reflectionFuzziness;
            if (x->_useConductorFresnel) {
                // Metal(eta, k, fuzz) keeps a white tint (Metal.cpp:82-90); the
                // descriptor's conductor form has no tint to carry another one.
                const Color& c = x->_color;
                if (c.getRed() != 1.0 || c.getGreen() != 1.0 || c.getBlue() != 1.0)
                    unsupported("a conductor Metal with a non-white tint");
                d.conductor = 1;
                put(d.eta, x->_eta);
                put(d.k, x->_extinctionCoefficient);
            }
            break;
        }
        case DIELECTRIC: {
            auto* x = static_cast<const Dielectric*>(m);
            d.type = LUZ_MAT_DIELECTRIC;
            d.ior = x->_refractiveIndex;
            d.roughness = x->_roughness;
            put(d.absorption, x->_absorptionCoefficient);
            break;
        }
        case EMISSIVE: d.type = LUZ_MAT_EMISSIVE; break;
        case ISOTROPIC: d.type = LUZ_MAT_ISOTROPIC; break;
        case HENYEY_GREENSTEIN:
            d.type = LUZ_MAT_HENYEY_GREENSTEIN;
            d.anisotropy = static_cast<const HenyeyGreenstein*>(m)->_anisotropy;
            break;
        case PRINCIPLED: {
            auto* x = static_cast<const Principled*>(m);
            d.type = LUZ_MAT_PRINCIPLED;
            d.metallic = x->_metallic;
            d.roughness = x->_roughness;
            d.transmission = x->_transmission;
            d.ior = x->_refractiveIndex;
            d.clearcoat = x->_clearcoat;
            d.clearcoat_roughness = x->_clearcoatRoughness;
            d.sheen = x->_sheen;
            d.subsurface = x->_subsurface;
            put(d.subsurface_radius, x->_subsurfaceRadius);
            d.subsurface_scale = x->_subsurfaceScale;
            put(d.subsurface_color, x->_subsurfaceColor);
            d.subsurface_method = x->_subsurfaceMethod == SUBSURFACE_THIN ? 1 : 0;
            put(d.absorption, x->_absorptionCoefficient);
            break;
        }
        case GLOSSY:
            d.type = LUZ_MAT_GLOSSY;
            d.roughness = static_cast<const Glossy*>(m)->_roughness;
            break;
        case DIFFUSE_GLOSSY: {
            auto* x = static_cast<const DiffuseGlossy*>(m);
            d.type = LUZ_MAT_DIFFUSE_GLOSSY;
            put(d.glossy_color, x->_glossyColor);
            d.glossy_weight = x->_glossyWeight;
            d.roughness = x->_glossyRoughness;
            break;
        }
        default: unsupported("the base Material type");
        }
        d.texture = texture(m->_texture);
        out.materials.push_back(d);
        const int32_t i = (int32_t)out.materials.size() - 1;
        material_index[m] = i;
        return i;
    }

    static void add_triangle(const Triangle& t, std::vector<double>& pos, std::vector<double>& nrm,
                             std::vector<double>& uv, bool& has_normals, bool& has_uvs, bool first)
    {
        if (first) {
            has_normals = t._hasVertexNormals;
            has_uvs = t._hasTextureCoordinates;
        } else if (has_normals != t._hasVertexNormals || has_uvs != t._hasTextureCoordinates) {
            unsupported("a mesh whose triangles mix vertex normals or texture coordinates with none");
        }
        double v[9];
        put(v, t._vertex0);
        put(v + 3, t._vertex1);
        put(v + 6, t._vertex2);
        pos.insert(pos.end(), v, v + 9);
        if (has_normals) {
            put(v, t._normal0);
            put(v + 3, t._normal1);
            put(v + 6, t._normal2);
            nrm.insert(nrm.end(), v, v + 9);
        }
        if (has_uvs) {
            const double w[6] = {t._uv0.getX(), t._uv0.getY(), t._uv1.getX(), t._uv1.getY(), t._uv2.getX(),
                                 t._uv2.getY()};
            uv.insert(uv.end(), w, w + 6);
        }
    }

    // One LuzMeshDesc over `tris`; every triangle has to carry `mat`.
    int32_t mesh_from(const std::vector<const Triangle*>& tris, const Material* mat)
    {
        std::vector<double> pos, nrm, uv;
        bool has_normals = false, has_uvs = false;
        pos.reserve(9 * tris.size());
        for (std::size_t i = 0; i < tris.size(); i++) {
            if (tris[i]->_material.get() != mat) unsupported("a mesh with per-triangle materials");
            add_triangle(*tris[i], pos, nrm, uv, has_normals, has_uvs, i == 0);
        }
        LuzMeshDesc d{};
        d.triangle_count = (int64_t)tris.size();
        d.material = material(mat);
        out.positions.push_back(std::move(pos));
        out.normals.push_back(has_normals ? std::move(nrm) : std::vector<double>());
        out.uvs.push_back(has_uvs ? std::move(uv) : std::vector<double>());
        out.meshes.push_back(d);
        return (int32_t)out.meshes.size() - 1;
    }

    int32_t mesh(const Mesh* m)
    {
        auto it = mesh_index.find(m);
        if (it != mesh_index.end()) return it->second;
        std::vector<const Triangle*> tris;
        if (m->_usesPackedTriangles) {
            for (const Triangle& t : m->_triangles) tris.push_back(&t);
        } else {
            for (const auto& h : m->_legacyTriangles) {
                auto* t = dynamic_cast<const Triangle*>(h.get());
                if (!t) unsupported("a mesh built from non-triangle hittables");
                tris.push_back(t);
            }
        }
        if (tris.empty()) unsupported("an empty mesh");
        const int32_t i = mesh_from(tris, m->_material.get());
        mesh_index[m] = i;
        return i;
    }

    int32_t ies(const std::shared_ptr<IESProfile>& p)
    {
        auto it = ies_index.find(p.get());
        if (it != ies_index.end()) return it->second;
        LuzIesDesc d{};
        d.vertical_count = (int32_t)p->_verticalAngles.size();
        d.horizontal_count = (int32_t)p->_horizontalAngles.size();
        out.ies_data.push_back(p->_verticalAngles);
        out.ies_data.push_back(p->_horizontalAngles);
        out.ies_data.push_back(p->_candelaValues);
        out.ies.push_back(d);
        const int32_t i = (int32_t)out.ies.size() - 1;
        ies_index[p.get()] = i;
        return i;
    }

    static LuzObjectDesc object(int32_t kind)
    {
        LuzObjectDesc o{};
        o.kind = kind;
        o.mesh = -1;
        o.ies = -1;
        o.visible = 1;
        o.scale[0] = o.scale[1] = o.scale[2] = 1.0;
        return o;
    }

    void hittable(const std::shared_ptr<Hittable>& hp)
    {
        const Hittable* h = hp.get();
        if (!h) unsupported("a null hittable");
        if (std::strstr(typeid(*h).name(), "DeferredHittable")) {
            (void)h->getMaterial();   // resolves the pending load (call_once)
            hittable(static_cast<const DeferredMirror*>(h)->hittable);
            return;
        }
        if (auto* r = dynamic_cast<const Rectangle*>(h)) {
            LuzObjectDesc o = object(LUZ_OBJ_RECTANGLE);
            o.material = material(r->_material.get());
            put(o.position, r->_transform.getPosition());
            put(o.orientation, r->_transform.getOrientation());
            o.size[0] = r->_width;
            o.size[1] = r->_height;
            if (r->_hasAxes) {
                o.has_axes = 1;
                put(o.width_axis, r->_widthAxis);
                put(o.height_axis, r->_heightAxis);
            }
            if (r->_hasTextureCoordinates) {
                o.has_uvs = 1;
                put(o.uv, r->_uv0);
                put(o.uv + 3, r->_uv1);
                put(o.uv + 6, r->_uv2);
                put(o.uv + 9, r->_uv3);
            }
            out.objects.push_back(o);
        } else if (dynamic_cast<const PerlinSphere*>(h)) {
            // PerlinSphere::hit writes the shared material's colour on every hit
            // (PerlinSphere.cpp:112-117), a value that depends on which render
            // thread hit last; no scene file creates one.
            unsupported("PerlinSphere");
        } else if (auto* s = dynamic_cast<const Sphere*>(h)) {
            LuzObjectDesc o = object(LUZ_OBJ_SPHERE);
            o.material = material(s->_material.get());
            o.uv_projection = s->_uvProjection == SphereUVProjection::CubeCross ? 1 : 0;
            put(o.position, s->_position);
            o.size[0] = s->_radius;
            o.visible = s->_visible ? 1 : 0;
            if (s->_iesProfile) {
                o.ies = ies(s->_iesProfile);
                put(o.ies_direction, s->_iesDirection);
                o.ies_rotation_degrees = s->_iesRotationDegrees;
            }
            out.objects.push_back(o);
        } else if (auto* c = dynamic_cast<const Cube*>(h)) {
            LuzObjectDesc o = object(LUZ_OBJ_CUBE);
            o.material = material(c->_material.get());
            put(o.position, c->_transform.getPosition());
            o.size[0] = c->_width;
            o.size[1] = c->_height;
            o.size[2] = c->_depth;
            out.objects.push_back(o);
        } else if (auto* p = dynamic_cast<const Plane*>(h)) {
            LuzObjectDesc o = object(LUZ_OBJ_PLANE);
            o.material = material(p->_material.get());
            o.position[1] = p->_y;
            put(o.orientation, p->_orientation);
            out.objects.push_back(o);
        } else if (auto* t = dynamic_cast<const Triangle*>(h)) {
            if (t->_isDegenerate) return;   // never hit, never sampled (Triangle.cpp:94-126)
            LuzObjectDesc o = object(LUZ_OBJ_MESH);
            o.mesh = mesh_from({t}, t->_material.get());
            o.material = out.meshes[o.mesh].material;
            out.objects.push_back(o);
        } else if (auto* m = dynamic_cast<const Mesh*>(h)) {
            LuzObjectDesc o = object(LUZ_OBJ_MESH);
            o.mesh = mesh(m);
            o.material = out.meshes[o.mesh].material;
            out.objects.push_back(o);
        } else if (auto* mi = dynamic_cast<const MeshInstance*>(h)) {
            LuzObjectDesc o = object(LUZ_OBJ_MESH_INSTANCE);
            o.mesh = mesh(mi->_geometry.get());
            o.material = material(mi->_material.get());
            const auto& x = mi->_transform;
            put(o.position, x.position);
            put(o.scale, x.scale);
            o.rotation_degrees[0] = degrees(x.sinX, x.cosX);
            o.rotation_degrees[1] = degrees(x.sinY, x.cosY);
            o.rotation_degrees[2] = degrees(x.sinZ, x.cosZ);
            out.objects.push_back(o);
        } else if (auto* v = dynamic_cast<const ConstantVolume*>(h)) {
            LuzObjectDesc o = object(LUZ_OBJ_VOLUME);
            o.material = material(v->_phaseFunction.get());
            o.density = v->_density;
            const Hittable* b = v->_boundary.get();
            if (auto* bs = dynamic_cast<const Sphere*>(b)) {
                o.boundary_kind = LUZ_OBJ_SPHERE;
                put(o.position, bs->_position);
                o.size[0] = bs->_radius;
            } else if (auto* bc = dynamic_cast<const Cube*>(b)) {
                o.boundary_kind = LUZ_OBJ_CUBE;
                put(o.position, bc->_transform.getPosition());
                o.size[0] = bc->_width;
                o.size[1] = bc->_height;
                o.size[2] = bc->_depth;
            } else {
                unsupported("a volume whose boundary is neither a Sphere nor a Cube");
            }
            out.objects.push_back(o);
        } else if (auto* dl = dynamic_cast<const DirectionalLight*>(h)) {
            LuzObjectDesc o = object(LUZ_OBJ_DIRECTIONAL_LIGHT);
            o.material = material(dl->_material.get());
            put(o.orientation, dl->_direction);
            out.objects.push_back(o);
        } else {
            unsupported(std::string("the hittable class ") + typeid(*h).name());
        }
    }

    void settings(Scene& scene)
    {
        LuzSceneDesc& d = out.desc;
        if (!scene.hasCamera()) throw std::runtime_error("No camera on the Scene.");
        const Camera cam = scene.getActiveCamera();
        put(d.camera.position, cam.getPosition());
        put(d.camera.direction, cam.getDirection());
        put(d.camera.up, cam.getUpDirection());
        d.camera.focal_length_m = cam.getFocalLengthMeters();
        d.camera.sensor_width_m = cam.getSensorWidthMeters();
        d.camera.sensor_height_m = cam.getSensorHeightMeters();
        d.camera.f_number = cam.getFNumber();
        d.camera.focus_distance_m = cam.getFocusDistanceMeters();
        d.camera.pinhole = cam.getPinhole() ? 1 : 0;

        // The linear sky's horizon is fixed at 0.5 on the GPU (Atmospherics.cpp:44-53,
        // Scene.cpp:117); no scene file key changes it.
        if (scene.getSkyline() != 0.5) unsupported("a skyline other than 0.5");
        switch (scene.getRenderSky()) {
        case SKY_NONE: d.sky = LUZ_SKY_NONE; break;
        case SKY_LINEAR: d.sky = LUZ_SKY_LINEAR; break;
        case SKY_ATMOSPHERE: d.sky = LUZ_SKY_ATMOSPHERE; break;
        case SKY_ENVIRONMENT: d.sky = LUZ_SKY_ENVIRONMENT; break;
        default: unsupported("this sky type");
        }
        put(d.background, scene.getBackgroundColor());
        d.meters_per_unit = scene.getMetersPerUnit();

        const auto& env = scene.getEnvironmentMap();
        if (env) {
            out.environment.resize(3 * env->_pixels.size());
            for (std::size_t k = 0; k < env->_pixels.size(); k++) put(&out.environment[3 * k], env->_pixels[k]);
            d.environment.width = (int32_t)env->_width;
            d.environment.height = (int32_t)env->_height;
            d.environment.strength = scene.getEnvironmentStrength();
            d.environment.rotation_degrees = scene.getEnvironmentRotation();
            d.environment.lighting = scene.getEnvironmentLighting() ? 1 : 0;
        }
        if (d.sky == LUZ_SKY_ATMOSPHERE) {
            const Atmosphere& a = scene.getAtmosphere();
            LuzAtmosphereDesc& q = d.atmosphere;
            put(q.sun_direction, a.getSunDirection());
            put(q.sun_radiance, a.getSunRadiance());
            q.sun_radiance_scale = a.getSunRadianceScale();
            q.earth_radius = a.getEarthRadius();
            q.atmosphere_radius = a.getAtmosphereRadius();
            q.h_r = a._hR;
            q.h_m = a._hM;
            q.samples = a._samples;
            q.light_samples = a._lightSamples;
            q.stars_brightness = a.getStarsBrightness();
        }
        if (scene.getCausticsEnabled()) {
            d.caustics.enabled = 1;
            d.caustics.photons = scene.getCausticPhotonCount();
            d.caustics.passes = scene.getCausticPassCount();
            d.caustics.radius_meters = scene.getCausticRadiusMeters();
            d.caustics.alpha = scene.getCausticAlpha();
        }
        out.width = (int32_t)scene.getImage()->getWidth();
        out.height = (int32_t)scene.getImage()->getHeight();
        out.spp = scene.getSampleCount();
        out.max_bounces = scene.getMaxLightBounces();
    }

    void finish()
    {
        LuzSceneDesc& d = out.desc;
        for (std::size_t i = 0; i < out.textures.size(); i++) out.textures[i].rgb = out.texels[i].data();
        for (std::size_t i = 0; i < out.meshes.size(); i++) {
            out.meshes[i].positions = out.positions[i].data();
            out.meshes[i].normals = out.normals[i].empty() ? nullptr : out.normals[i].data();
            out.meshes[i].uvs = out.uvs[i].empty() ? nullptr : out.uvs[i].data();
        }
        for (std::size_t i = 0; i < out.ies.size(); i++) {
            out.ies[i].vertical_deg = out.ies_data[3 * i].data();
            out.ies[i].horizontal_deg = out.ies_data[3 * i + 1].data();
            out.ies[i].candela = out.ies_data[3 * i + 2].data();
        }
        d.abi_version = LUZ_GPU_ABI_VERSION;
        d.material_count = (int32_t)out.materials.size();
        d.materials = out.materials.data();
        d.texture_count = (int32_t)out.textures.size();
        d.textures = out.textures.data();
        d.mesh_count = (int32_t)out.meshes.size();
        d.meshes = out.meshes.data();
        d.object_count = (int32_t)out.objects.size();
        d.objects = out.objects.data();
        d.ies_count = (int32_t)out.ies.size();
        d.ies = out.ies.data();
        d.environment.rgb = out.environment.empty() ? nullptr : out.environment.data();
    }
};

}  // namespace

void luz_pack_scene(Scene& scene, LuzPackedScene& out)
{
    // The state Renderer::render traces (src/renderer/Renderer.cpp:18-20).
    scene.syncAtmosphereSunDirection();
    scene.updateLights();
    scene.updateAccelerationStructure();
    Packer p(out);
    for (const auto& h : scene.getHittables()) p.hittable(h);
    p.settings(scene);
    p.finish();
}
