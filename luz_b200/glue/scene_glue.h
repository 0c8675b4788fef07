/*
 * scene_glue.h — packs a Luz reference `Scene` into the LuzSceneDesc that
 * luz_gpu_scene_create (include/luz_gpu.h) takes.
 *
 * This is the reference-side half of the drop-in: the code a maintainer adds
 * to the Luz tree next to Renderer::render (src/renderer/Renderer.cpp:10) so
 * that any scene the reference can build — from a .luz file through
 * SceneFile::read (src/io/SceneFile/SceneFile.cpp) or from C++ — renders on
 * the GPU. It reads the scene after Scene::syncAtmosphereSunDirection,
 * Scene::updateLights and Scene::updateAccelerationStructure, as
 * Renderer::render leaves it (Renderer.cpp:18-20).
 *
 * It compiles only against the Luz headers (include/luz, src/renderer), and
 * reads fields the reference keeps private; inside the Luz tree a friend
 * declaration or getters on those classes stand in for the private access
 * used here.
 */
#pragma once

#include <cstdint>
#include <memory>
#include <vector>

#include "luz_gpu.h"

class Scene;

/* Owns every array behind one LuzSceneDesc. `desc` points into the vectors,
 * so the object is neither copied nor moved once packed. */
struct LuzPackedScene {
    std::vector<LuzMaterialDesc> materials;
    std::vector<LuzTextureDesc> textures;
    std::vector<std::vector<double>> texels;
    std::vector<LuzMeshDesc> meshes;
    std::vector<std::vector<double>> positions, normals, uvs;
    std::vector<LuzObjectDesc> objects;
    std::vector<LuzIesDesc> ies;
    std::vector<std::vector<double>> ies_data;
    std::vector<double> environment;
    LuzSceneDesc desc{};
    /* the scene's own render settings (Scene::getImage, getSampleCount,
     * getMaxLightBounces); the seed and stream stay the caller's */
    int32_t width = 0, height = 0, spp = 0, max_bounces = 0;

    LuzPackedScene() = default;
    LuzPackedScene(const LuzPackedScene&) = delete;
    LuzPackedScene& operator=(const LuzPackedScene&) = delete;
};

/* Fills `out` from `scene`. Throws std::runtime_error naming the first
 * hittable, material or setting that the GPU path does not implement. */
void luz_pack_scene(Scene& scene, LuzPackedScene& out);
