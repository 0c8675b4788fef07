"""Host BVH builders reproduce the reference node layout bit for bit
(Mesh::_buildPackedBVH, src/core/Hittables/Mesh.cpp:383-521): node boxes in
double, child/leaf indices and the triangle order (_triangleIndices)."""
import numpy as np
import pytest

from cases import BVH_CASES
from luz_b200 import native


@pytest.mark.parametrize("name", sorted(BVH_CASES))
def test_mesh_bvh_matches_reference(name, golden):
    g = golden("bvh_" + name)
    sc = BVH_CASES[name]()
    pk = native.Pack(sc.build())
    for mi in range(len(sc.meshes)):
        nodes, order = pk.mesh_bvh(mi)
        ref_nodes, ref_order = g[f"nodes{mi}"], g[f"order{mi}"]
        assert nodes.tobytes() == ref_nodes.tobytes()
        assert np.array_equal(order[:len(ref_order)], ref_order)


def test_degenerate_triangles_are_dropped():
    sc = BVH_CASES["degenerate"]()
    pk = native.Pack(sc.build())
    info = pk.info()
    assert info.mesh_triangles < sc.meshes[0]["positions"].shape[0]


def test_packed_boxes_contain_double_boxes(golden):
    sc = BVH_CASES["icosphere3"]()
    pk = native.Pack(sc.build())
    raw = pk.array("meshes")
    assert raw.size > 0
    nodes, _ = pk.mesh_bvh(0)
    mesh = np.frombuffer(raw[:48], np.float32)
    assert np.all(mesh[[0, 1, 2]].astype(np.float64) <= nodes[0]["bmin"])
    assert np.all(mesh[[4, 5, 6]].astype(np.float64) >= nodes[0]["bmax"])


def test_empty_scene_packs():
    from luz_b200.desc import Scene
    pk = native.Pack(Scene().build())
    assert pk.info().top_leaf_objects == 0
