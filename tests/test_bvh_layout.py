"""Host BVH builders reproduce the reference node layouts bit for bit.

* Mesh BVH (Mesh::_buildPackedBVH, src/core/Hittables/Mesh.cpp:383-521): node
  boxes in double, child/leaf indices and the triangle order (_triangleIndices),
  on small meshes and on the benchmarked 1,310,722-triangle mesh (sha256 of the
  reference's full arrays).
* Top-level tree (BVHNode::BVHNode, src/core/Hittables/BVHNode.cpp:142-185, built
  by Scene::updateAccelerationStructure, src/scene/Scene.cpp:655-688): node order,
  child order, child kinds and object ids exactly, child boxes as the reference's
  double boxes rounded outward to FP32; on every parity case and on the 1e5-instance
  benchmark frame.
"""
import hashlib

import numpy as np
import pytest

import oracle as O
from cases import BVH_CASES, CASES, FULL_CASES
from luz_b200 import native


def sha256(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


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


@pytest.mark.parametrize("name", sorted(CASES))
def test_top_level_tree_matches_reference(name, golden):
    ref = golden("hits_" + name)["top"]
    ours = O.top_tree_from_pack(native.Pack(CASES[name]().scene.build()))
    assert len(ours) == len(ref) and np.array_equal(ours, ref)


@pytest.mark.parametrize("name", sorted(FULL_CASES))
def test_full_size_layouts_match_reference(name, golden):
    """The benchmarked frames: every mesh BVH (the 1,310,722-triangle mesh has 448,391
    nodes) and the top-level tree (1e5 instances) equal the reference's arrays."""
    g = golden("full_" + name)
    w = FULL_CASES[name]()
    pk = native.Pack(w.scene.build())
    for mi in range(len(w.scene.meshes)):
        nodes, order = pk.mesh_bvh(mi)
        assert len(nodes) == int(g[f"mesh{mi}_nodes"])
        assert nodes[:64].tobytes() == g[f"mesh{mi}_head"].tobytes()
        assert sha256(nodes, order) == str(g[f"mesh{mi}_sha256"])
    top = O.top_tree_from_pack(pk)
    assert len(top) == int(g["top_len"]) and np.array_equal(top[:4096], g["top_head"])
    assert sha256(top) == str(g["top_sha256"])
