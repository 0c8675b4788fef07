// pack.h — host-side scene packer (C++, no CUDA calls).
#pragma once
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "layout.h"
#include "luz_gpu.h"

namespace luz {

struct Status : std::runtime_error {
    int code;
    Status(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void set_error(const std::string& message);
const std::string& get_error();

struct Box64 {
    double mn[3], mx[3];
};

struct MeshBuild {
    std::vector<LuzMeshNode64> nodes;        // reference layout (Mesh::_packedBVHNodes)
    std::vector<int64_t> order;              // Mesh::_triangleIndices
    std::vector<double> vtx;                 // v0 v1 v2 per surviving triangle (9 each)
    std::vector<double> v0, e1, e2;          // per surviving triangle (3 each)
    std::vector<double> fn;                  // face normal
    std::vector<double> area;
    std::vector<double> vn;                  // vertex normals (9 per tri) or empty
    std::vector<uint8_t> has_vn;
    std::vector<double> uv;                  // 6 per tri or empty
    double total_area = 0.0;
    Box64 box{};
    int depth = 0;
    int material = -1;
};

struct ScenePack {
    // device arrays (host copies)
    std::vector<GRect> rects;
    std::vector<GObject> objects;
    std::vector<GTopNode> top_nodes;
    std::vector<GTopChild> top_children;
    std::vector<GNode> nodes;                // binary mesh BVH (host: restatement and layout dumps)
    std::vector<GNode4> nodes4;              // collapsed 4-wide mesh BVH (device traversal)
    std::vector<GTri> tris;
    std::vector<GTriShade> tri_shade;
    std::vector<float> vnormals;             // 9 floats per tri (leaf order) for meshes with normals
    std::vector<float> vuvs;                 // 6 floats per tri (leaf order)
    std::vector<GMesh> meshes;
    std::vector<GMaterial> materials;
    std::vector<GTexture> textures;
    std::vector<float> texels;               // float4 per texel
    std::vector<GLight> lights;
    std::vector<GIes> ies;
    std::vector<double> cdf;                 // all double CDF / pdf pools
    std::vector<int32_t> index_pool;         // unaccelerated object list, slot maps
    std::vector<float> env_texels;           // float4 per texel
    std::vector<uint8_t> obj_class;          // per GObject: material type a hit on it shades (shade binning)
    GSceneConst consts{};
    LuzCameraDesc camera{};
    std::vector<int32_t> object_of_desc;     // desc object -> GObject index (-1 = none)
    std::vector<MeshBuild> builds;           // reference-layout BVHs (kept for parity dumps)
    int max_mesh_depth = 0;
    int64_t device_bytes() const;
};

ScenePack* pack_scene(const LuzSceneDesc* desc);
// Prepares the camera for a W x H image (Renderer::internal::_prepareRenderCamera).
GCamera prepare_camera(const LuzCameraDesc& cam, double meters_per_unit, int width, int height);

}  // namespace luz

struct luz_scene_pack {
    luz::ScenePack* p;
};
