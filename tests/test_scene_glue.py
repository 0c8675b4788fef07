"""The reference-side scene glue (luz_b200/glue/scene_glue.cpp).

A .luz file is read by the reference's own parser (SceneFile::read,
src/io/SceneFile/SceneFile.cpp:256-321) and the glue packs the resulting Scene
into the LuzSceneDesc of include/luz_gpu.h: the drop-in path of a Luz program
that renders its scenes on the GPU.

CPU: the packed description, rebuilt into a reference scene by the oracle
harness, traces the same per-path radiance as the parsed scene (to 1e-12
relative: instance Euler angles are recovered from the stored sines and
cosines), and the GPU library's host packer accepts it.
GPU: the packed description renders per path as the reference renders the
parsed file.

The scenes under tests/golden/scenes are written for these tests; their assets
come from tests/golden/scenes/make_assets.py.
"""
import glob
import os

import numpy as np
import pytest

from luz_b200 import native

SCENE_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "scenes")
SCENES = sorted(os.path.basename(p) for p in glob.glob(os.path.join(SCENE_DIR, "*.luz")))


def _reference_tree():
    """The reference tree the oracle libraries were built from (oracle/Makefile records
    it in oracle/_ref/ref_root.txt), or LUZ_REFERENCE; None where neither is present."""
    root = os.environ.get("LUZ_REFERENCE")
    rec = os.path.join(os.path.dirname(SCENE_DIR), "..", "..", "oracle", "_ref", "ref_root.txt")
    if not root and os.path.exists(rec):
        root = open(rec).read().strip() or None
    return root
# bound on the fraction of paths the oracle's FP32-ambiguity probe may exclude
# (oracle.ambiguous_paths); every other path is within 1e-4 of the reference
GPU_AMBIGUOUS_MAX = 0.05


def _oracle():
    import oracle as O
    if not O.reference_available():
        pytest.fail("oracle/_ref/libluzref.so missing: run __graft_entry__.build()")
    return O.RefOracle()


def _paths(pk, n=400, seed=7):
    rng = np.random.default_rng(seed)
    return (rng.integers(0, pk.width, n), rng.integers(0, pk.height, n), rng.integers(0, max(1, pk.spp), n))


def test_scene_files_present():
    assert SCENES == ["glue_meshes.luz", "glue_planet.luz", "glue_room.luz", "glue_volumes.luz"]


@pytest.mark.parametrize("name", SCENES)
def test_packed_scene_traces_as_parsed_scene(name):
    o = _oracle()
    parsed = o.load_luz(os.path.join(SCENE_DIR, name))
    pk = parsed.pack()
    rebuilt = o.scene(pk)
    x, y, s = _paths(pk)
    p = native.params(pk.width, pk.height, pk.spp, pk.max_bounces, 20240611)
    a = parsed.trace_paths(p, x, y, s)
    b = rebuilt.trace_paths(p, x, y, s)
    assert (a.max(axis=1) > 0).mean() > 0.4           # the scene is lit where the camera looks
    rel = np.abs(a - b) / np.maximum(np.abs(a), 1e-3)
    assert rel.max() <= 1e-12, rel.max()


@pytest.mark.parametrize("name", SCENES)
def test_host_packer_accepts_packed_scene(name):
    o = _oracle()
    pk = o.load_luz(os.path.join(SCENE_DIR, name)).pack()
    info = native.Pack(pk).info()
    assert info.light_count >= 1
    assert info.top_leaf_objects >= 1


def test_packed_settings_and_objects():
    """Scene-level settings and object kinds survive the packing."""
    import ctypes as C
    from luz_b200 import desc as D
    o = _oracle()
    pk = o.load_luz(os.path.join(SCENE_DIR, "glue_meshes.luz")).pack()
    d = C.cast(C.c_void_p(pk.ptr()), C.POINTER(D.SceneDesc)).contents
    assert (pk.width, pk.height, pk.spp, pk.max_bounces) == (40, 30, 4, 5)
    assert d.sky == D.SKY_LINEAR
    kinds = [d.objects[i].kind for i in range(d.object_count)]
    # sun, two instances of the shared geometry, the baked zero-scale mesh, the textured instance, the plane
    assert kinds == [D.OBJ_DIRECTIONAL_LIGHT, D.OBJ_MESH_INSTANCE, D.OBJ_MESH_INSTANCE, D.OBJ_MESH,
                     D.OBJ_MESH_INSTANCE, D.OBJ_PLANE]
    assert d.objects[1].mesh == d.objects[2].mesh == d.objects[4].mesh
    assert np.allclose([d.objects[1].rotation_degrees[i] for i in range(3)], [20, 35, 10], atol=1e-9)
    pk = o.load_luz(os.path.join(SCENE_DIR, "glue_planet.luz")).pack()
    d = C.cast(C.c_void_p(pk.ptr()), C.POINTER(D.SceneDesc)).contents
    assert d.sky == D.SKY_ATMOSPHERE
    spheres = [d.objects[i] for i in range(d.object_count) if d.objects[i].kind == D.OBJ_SPHERE]
    assert len(spheres) == 1 and spheres[0].uv_projection == 1
    assert d.materials[spheres[0].material].texture >= 0
    pk = o.load_luz(os.path.join(SCENE_DIR, "glue_volumes.luz")).pack()
    d = C.cast(C.c_void_p(pk.ptr()), C.POINTER(D.SceneDesc)).contents
    assert d.caustics.enabled == 1 and d.caustics.photons == 20000 and d.caustics.passes == 2
    assert d.environment.width == 16 and d.environment.height == 8 and d.environment.lighting == 1
    vols = [d.objects[i].boundary_kind for i in range(d.object_count) if d.objects[i].kind == D.OBJ_VOLUME]
    assert vols == [D.OBJ_CUBE, D.OBJ_SPHERE]


def test_reference_example_scenes_pack():
    """Every example scene the reference ships packs, and its packed description
    traces as the parsed scene (runs only where the reference sources are)."""
    root = _reference_tree()
    examples = sorted(glob.glob(os.path.join(root, "examples", "scenes", "*.luz"))) if root else []
    if not examples:
        pytest.skip("the reference's example scenes are not on this machine")
    o = _oracle()
    for path in examples:
        parsed = o.load_luz(path)
        pk = parsed.pack()
        rebuilt = o.scene(pk)
        x, y, s = _paths(pk, n=64)
        p = native.params(pk.width, pk.height, pk.spp, min(pk.max_bounces, 6), 99)
        a = parsed.trace_paths(p, x, y, s)
        b = rebuilt.trace_paths(p, x, y, s)
        rel = np.abs(a - b) / np.maximum(np.abs(a), 1e-3)
        assert rel.max() <= 1e-12, (os.path.basename(path), rel.max())


@pytest.mark.gpu
@pytest.mark.parametrize("name", SCENES)
def test_gpu_renders_parsed_scene_as_reference(name):
    o = _oracle()
    parsed = o.load_luz(os.path.join(SCENE_DIR, name))
    pk = parsed.pack()
    g = native.GpuScene(pk)
    x, y, s = _paths(pk, n=1500, seed=11)
    p = native.params(pk.width, pk.height, pk.spp, pk.max_bounces, 31337)
    ref = parsed.trace_paths(p, x, y, s)
    import ctypes as C
    import oracle as O
    from luz_b200 import desc as D
    cam = C.cast(C.c_void_p(pk.ptr()), C.POINTER(D.SceneDesc)).contents.camera
    amb = O.ambiguous_paths(o, parsed, p, x, y, s, ref, O.path_deltas(pk.width, pk.height, cam))
    rgb = g.trace_paths(p, x, y, s).astype(np.float64)
    rel = (np.abs(rgb - ref) / np.maximum(np.abs(ref), 1e-3)).max(axis=1)
    print(f"{name}: {amb.mean():.4f} of paths ambiguous; {(rel <= 1e-4).mean():.4f} within 1e-4")
    assert amb.mean() <= GPU_AMBIGUOUS_MAX, amb.mean()
    # as test_gpu_parity.check_paths, at most 0.2% of the unflagged paths outside 1e-4; these
    # scenes also hold a mirror-like gold lobe (roughness 0.05) whose draws the probe moves by
    # too little to see every discrete outcome FP32 can flip (measured: one path in 1,477)
    bad = (rel > 1e-4) & ~amb
    assert bad.sum() <= max(1, int(0.002 * (~amb).sum())), np.flatnonzero(bad)[:10]
    assert abs(rgb.mean() - ref.mean()) <= 0.02 * max(ref.mean(), 1e-6) + 1e-6
    img, _ = g.render(native.params(pk.width, pk.height, pk.spp, pk.max_bounces, 31337))
    assert np.isfinite(img).all() and img.mean() > 0
