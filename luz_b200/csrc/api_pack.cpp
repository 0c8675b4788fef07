// api_pack.cpp — C ABI of the host packer (usable without a GPU).
#include <cstring>
#include <functional>
#include <string>

#include "luz_gpu.h"
#include "pack.h"

using namespace luz;

namespace {
int guard(const std::function<int()>& f)
{
    try {
        return f();
    } catch (const Status& s) {
        set_error(s.what());
        return s.code;
    } catch (const std::exception& e) {
        set_error(e.what());
        return LUZ_E_INVALID;
    }
}
}  // namespace

extern "C" {

int luz_pack_create(const LuzSceneDesc* desc, luz_scene_pack** out)
{
    return guard([&] {
        if (!out) throw Status(LUZ_E_INVALID, "Output handle pointer is NULL.");
        *out = nullptr;
        ScenePack* p = pack_scene(desc);
        *out = new luz_scene_pack{p};
        return LUZ_OK;
    });
}

int luz_pack_destroy(luz_scene_pack* pack)
{
    if (pack) {
        delete pack->p;
        delete pack;
    }
    return LUZ_OK;
}

int luz_pack_info(const luz_scene_pack* pack, LuzSceneInfo* info)
{
    return guard([&] {
        if (!pack || !info) throw Status(LUZ_E_INVALID, "NULL argument.");
        const ScenePack& P = *pack->p;
        info->top_nodes = (int64_t)P.top_nodes.size();
        info->top_leaf_objects = (int64_t)P.objects.size();
        info->mesh_nodes = (int64_t)P.nodes.size();
        info->mesh_triangles = (int64_t)P.tris.size();
        info->device_bytes = P.device_bytes();
        info->max_mesh_depth = P.max_mesh_depth;
        info->light_count = P.consts.light_count;
        return LUZ_OK;
    });
}

int luz_pack_mesh_bvh(const luz_scene_pack* pack, int32_t mesh, LuzMeshNode64* nodes, int64_t node_capacity,
                      int64_t* node_count, int64_t* triangle_order, int64_t order_capacity)
{
    return guard([&] {
        if (!pack || !node_count) throw Status(LUZ_E_INVALID, "NULL argument.");
        const ScenePack& P = *pack->p;
        if (mesh < 0 || mesh >= (int32_t)P.builds.size()) throw Status(LUZ_E_INVALID, "Mesh index out of range.");
        const MeshBuild& b = P.builds[mesh];
        *node_count = (int64_t)b.nodes.size();
        if (nodes)
            for (int64_t i = 0; i < (int64_t)b.nodes.size() && i < node_capacity; i++) nodes[i] = b.nodes[(size_t)i];
        if (triangle_order)
            for (int64_t i = 0; i < (int64_t)b.order.size() && i < order_capacity; i++) triangle_order[i] = b.order[(size_t)i];
        return LUZ_OK;
    });
}

int luz_pack_array(const luz_scene_pack* pack, const char* name, const void** data, int64_t* bytes)
{
    return guard([&] {
        if (!pack || !name || !data || !bytes) throw Status(LUZ_E_INVALID, "NULL argument.");
        const ScenePack& P = *pack->p;
        const std::string n(name);
        auto put = [&](const void* d, std::size_t b) {
            *data = d;
            *bytes = (int64_t)b;
            return LUZ_OK;
        };
        if (n == "top_nodes") return put(P.top_nodes.data(), P.top_nodes.size() * sizeof(GTopNode));
        if (n == "top_children") return put(P.top_children.data(), P.top_children.size() * sizeof(GTopChild));
        if (n == "objects") return put(P.objects.data(), P.objects.size() * sizeof(GObject));
        if (n == "mesh_nodes") return put(P.nodes.data(), P.nodes.size() * sizeof(GNode));
        if (n == "mesh_tris") return put(P.tris.data(), P.tris.size() * sizeof(GTri));
        if (n == "meshes") return put(P.meshes.data(), P.meshes.size() * sizeof(GMesh));
        if (n == "rects") return put(P.rects.data(), P.rects.size() * sizeof(GRect));
        if (n == "index_pool") return put(P.index_pool.data(), P.index_pool.size() * sizeof(int32_t));
        if (n == "consts") return put(&P.consts, sizeof(GSceneConst));
        throw Status(LUZ_E_INVALID, "Unknown packed array '" + n + "'.");
    });
}

}  // extern "C"
