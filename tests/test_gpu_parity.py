"""GPU parity against the oracle (the reference's own outputs and the FP32 restatement).

- ray batches: GPU traversal == FP32 restatement bit for bit (t, object,
  primitive, u, v); against the reference, object and primitive ids are equal
  on every ray the oracle does not mark as FP32-ambiguous;
- per-path radiance under the reference Sampler stream: within 1e-4 relative
  (absolute below 1e-3) on the paths the oracle does not mark as ambiguous
  (oracle.ambiguous_paths: the reference's own radiance moves by more than the
  tolerance when its draws move by a few FP32 ulps of what they become: a draw
  within rounding of a lobe or Russian-roulette threshold, a very sharp lobe, a
  grazing vertex), all but at most 0.2% of them, which stay within 1e-3; the
  excluded fraction is bounded and printed per case;
- the same at the benchmarked sizes: the 1920x1080 frame over the
  1,310,722-triangle mesh and the 1280x720 frame over 1e5 instances;
- whole images against the reference film;
- full-size properties: determinism, sample additivity, finiteness.
"""
import numpy as np
import pytest

from cases import CASES, FULL_CASES, camera_rays
from luz_b200 import native, scenes
from luz_b200.desc import OBJ_MESH, OBJ_MESH_INSTANCE

pytestmark = pytest.mark.gpu

# upper bound on the fraction of paths the oracle may exclude as ambiguous, per case
# (measured: linear_sky 0.078 (f/16 thin lens, mirror spheres), glossy 0.010, ies 0.005,
# cornell 0.003, tiny 0.003, caustics 0.001, instancing 0.001, atmosphere 0)
AMBIGUOUS_MAX = {"linear_sky": 0.10}
REL_TOL = 1e-4
RESIDUAL_MAX = 0.002   # unflagged paths allowed between REL_TOL and 10 x REL_TOL (measured: 5 of 20,000)


def path_rel(rgb, ref):
    """max over channels of |gpu - ref| / max(|ref|, 1e-3)"""
    return (np.abs(rgb - ref) / np.maximum(np.abs(ref), 1e-3)).max(axis=1)


def check_paths(label, rgb, ref, amb, amb_max=0.02, photon=None):
    """photon: paths that gather caustic photons (compared in test_caustics), left out here."""
    rel = path_rel(rgb.astype(np.float64), ref)
    print(f"{label}: {amb.mean():.4f} of {len(amb)} paths ambiguous; "
          f"{(rel <= REL_TOL).mean():.4f} of all paths within {REL_TOL}"
          + ("" if photon is None else f"; {photon.mean():.4f} gather caustic photons"))
    assert amb.mean() <= amb_max, amb.mean()
    if photon is not None:
        amb = amb | photon
    bad = np.flatnonzero((rel > REL_TOL) & ~amb)
    # FP32 error the probe does not model (a few paths in 10^4: a narrow-lobe or near-tangent
    # refraction early in the path, metre-scale FP32 positions under the atmosphere) stays
    # within 10x the tolerance
    assert bad.size <= max(1, int(RESIDUAL_MAX * (~amb).sum())), (bad[:10], rel[bad[:10]])
    assert (rel[~amb] <= 10 * REL_TOL).all(), rel[~amb].max()
    ok = ~amb
    assert abs(rgb[ok].mean() - ref[ok].mean()) <= 1e-4 * max(ref[ok].mean(), 1e-6) + 1e-6


@pytest.fixture(scope="module")
def gpu_scenes():
    out = {}
    for name, fn in CASES.items():
        w = fn()
        b = w.scene.build()
        out[name] = (w, b, native.GpuScene(b))
    yield out
    for _, _, g in out.values():
        g.close()


@pytest.mark.parametrize("name", sorted(CASES))
def test_traversal_bit_exact_with_restatement(name, gpu_scenes, golden, restate):
    w, b, g = gpu_scenes[name]
    gd = golden("hits_" + name)
    hg = g.trace_rays(gd["rays"], seed=w.seed, volume_key=gd["vkey"])
    hr = restate.trace(native.Pack(b), gd["rays"], seed=w.seed, volume_key=gd["vkey"])
    assert hg.tobytes() == hr.tobytes()
    ag = g.trace_rays(gd["rays"], any_hit=True, seed=w.seed, volume_key=gd["vkey"])
    ar = restate.trace(native.Pack(b), gd["rays"], any_hit=True, seed=w.seed, volume_key=gd["vkey"])
    assert np.array_equal(ag["object"], ar["object"])


@pytest.mark.parametrize("name", sorted(CASES))
def test_hits_agree_with_reference(name, gpu_scenes, golden):
    w, b, g = gpu_scenes[name]
    gd = golden("hits_" + name)
    h = g.trace_rays(gd["rays"], seed=w.seed, volume_key=gd["vkey"])
    kinds = np.array([w.scene.objects[o]["kind"] if o >= 0 else 0 for o in gd["obj"]])
    meshy = np.isin(kinds, [OBJ_MESH, OBJ_MESH_INSTANCE])
    agree = (h["object"] == gd["obj"]) & (~meshy | (h["primitive"] == gd["prim"]))
    amb = gd["ambiguous"]
    assert amb.mean() <= 0.01 and agree[~amb].all(), np.flatnonzero(~agree & ~amb)[:10]
    a = g.trace_rays(gd["rays"], any_hit=True, seed=w.seed, volume_key=gd["vkey"])
    same = (a["object"] >= 0) == gd["occluded"]
    assert same[~gd["ambiguous_any"]].all()


@pytest.mark.parametrize("name", sorted(CASES))
def test_per_path_radiance_matches_reference(name, gpu_scenes, golden):
    w, b, g = gpu_scenes[name]
    gd = golden("paths_" + name)
    p = native.params(w.width, w.height, w.spp, w.max_bounces, w.seed)
    rgb = g.trace_paths(p, gd["x"], gd["y"], gd["s"])
    check_paths(name, rgb, gd["rgb"], gd["ambiguous"], AMBIGUOUS_MAX.get(name, 0.02),
                gd["photon"] if "photon" in gd.files else None)


@pytest.mark.parametrize("name", sorted(FULL_CASES))
def test_full_size_frame_parity(name, golden, restate):
    """The benchmarked frames at full size: 2,000 rays (bit for bit with the FP32
    restatement; ids equal to the reference's on unambiguous rays) and 4,096 paths
    (plus the lit paths of the mostly dark 1e5-instance frame) within 1e-4 of the
    reference on unambiguous paths."""
    w = FULL_CASES[name]()
    b = w.scene.build()
    gd = golden("full_" + name)
    g = native.GpuScene(b)
    try:
        rays, vkey = gd["hit_rays"], gd["hit_vkey"]
        h = g.trace_rays(rays, seed=w.seed, volume_key=vkey)
        hr = restate.trace(native.Pack(b), rays, seed=w.seed, volume_key=vkey)
        assert h.tobytes() == hr.tobytes()
        kinds = np.array([w.scene.objects[o]["kind"] if o >= 0 else 0 for o in gd["hit_obj"]])
        meshy = np.isin(kinds, [OBJ_MESH, OBJ_MESH_INSTANCE])
        agree = (h["object"] == gd["hit_obj"]) & (~meshy | (h["primitive"] == gd["hit_prim"]))
        amb = gd["hit_ambiguous"]
        assert amb.mean() <= 0.01 and agree[~amb].all(), np.flatnonzero(~agree & ~amb)[:10]
        a = g.trace_rays(rays, any_hit=True, seed=w.seed, volume_key=vkey)
        assert ((a["object"] >= 0) == gd["hit_occluded"])[~gd["hit_ambiguous_any"]].all()
        p = native.params(w.width, w.height, w.spp, w.max_bounces, w.seed)
        rgb = g.trace_paths(p, gd["path_x"], gd["path_y"], gd["path_s"])
        check_paths(name, rgb, gd["path_rgb"], gd["path_ambiguous"])
        assert (gd["path_rgb"].max(axis=1) > 0).sum() >= 50   # lit paths are part of the check
    finally:
        g.close()


@pytest.mark.parametrize("name", ["cornell", "tiny"])
def test_image_matches_reference_film(name, gpu_scenes, golden):
    w, b, g = gpu_scenes[name]
    gd = golden("image_" + name)
    img, st = g.render(native.params(w.width, w.height, w.spp, w.max_bounces, w.seed))
    ref = gd["rgb"]
    assert img.shape == ref.shape
    rel = np.abs(img - ref) / np.maximum(np.abs(ref), 1e-3)
    assert (rel <= 1e-4).mean() >= 0.98
    rel_mse = np.mean((img - ref) ** 2) / max(np.mean(ref ** 2), 1e-12)
    assert rel_mse < 1e-4
    assert st.kernel_launches > 0 and st.extension_rays >= w.width * w.height * w.spp


def test_render_is_deterministic_and_sample_additive(gpu_scenes):
    w, b, g = gpu_scenes["instancing"]
    p4 = native.params(w.width, w.height, 4, w.max_bounces, w.seed)
    a, _ = g.render(p4)
    a2, _ = g.render(p4)
    assert a.tobytes() == a2.tobytes()
    h0, _ = g.render(native.params(w.width, w.height, 2, w.max_bounces, w.seed, 0, 0))
    h1, _ = g.render(native.params(w.width, w.height, 2, w.max_bounces, w.seed, 0, 2))
    assert np.allclose((h0 + h1) / 2.0, a, rtol=1e-5, atol=1e-7)


def test_trace_paths_equals_render_for_one_sample(gpu_scenes):
    w, b, g = gpu_scenes["tiny"]
    p = native.params(w.width, w.height, 1, w.max_bounces, w.seed)
    img, _ = g.render(p)
    yy, xx = np.mgrid[0:w.height, 0:w.width]
    rgb = g.trace_paths(p, xx.ravel(), yy.ravel(), np.zeros(xx.size))
    rgb = np.where(np.isfinite(rgb), rgb, 0.0).reshape(img.shape)
    assert np.allclose(rgb, img, rtol=1e-6, atol=1e-7)


def test_invalid_render_arguments(gpu_scenes):
    w, b, g = gpu_scenes["tiny"]
    with pytest.raises(native.LuzError) as e:
        g.render(native.params(0, 10, 1, 4, 1))
    assert e.value.code == -1
    p = native.params(8, 8, 1, 4, 1)
    p.flags = 1
    with pytest.raises(native.LuzError) as e:
        g.render(p)
    assert e.value.code == -3
    with pytest.raises(native.LuzError):
        g.trace_paths(native.params(8, 8, 1, 4, 1), [9], [0], [0])


def test_full_size_glossy_frame_properties():
    """The benchmark workload at full size (1920x1080, 1.3M triangles) at 2 spp:
    finite, non-negative, deterministic; sample-range additivity holds."""
    w = scenes.mesh_glossy()
    g = native.GpuScene(w.scene.build())
    try:
        p = native.params(w.width, w.height, 2, w.max_bounces, w.seed)
        a, st = g.render(p)
        assert np.isfinite(a).all() and (a >= 0).all() and a.mean() > 0.1
        b2, _ = g.render(p)
        assert a.tobytes() == b2.tobytes()
        s0, _ = g.render(native.params(w.width, w.height, 1, w.max_bounces, w.seed, 0, 0))
        s1, _ = g.render(native.params(w.width, w.height, 1, w.max_bounces, w.seed, 0, 1))
        assert np.allclose((s0 + s1) / 2.0, a, rtol=1e-5, atol=1e-6)
        assert st.extension_rays > w.width * w.height * 2
    finally:
        g.close()


def test_full_size_instancing_frame_properties():
    """1e5 instances (2e7 instanced triangles) in an HG medium at 1280x720, 1 spp."""
    w = scenes.instancing_volumes(spp=1)
    g = native.GpuScene(w.scene.build())
    try:
        a, st = g.render(native.params(w.width, w.height, 1, w.max_bounces, w.seed))
        assert np.isfinite(a).all() and (a >= 0).all() and a.mean() > 0
        assert g.info().top_leaf_objects >= 100_000
    finally:
        g.close()


@pytest.mark.gpu
def test_batch_render_equals_individual_renders():
    """luz_gpu_batch_render: scenes of different sizes rendered concurrently give
    exactly the films and ray counts of one-at-a-time renders."""
    ws = [scenes.cornell(48, 40, 3, 8), scenes.tiny_mixed(24, 18, 5, 6),
          scenes.mesh_glossy(64, 36, 2, 12, level=4), scenes.instancing_volumes(40, 30, 2, 16, count=300)]
    gs = [native.GpuScene(w.scene.build()) for w in ws]
    ps = [native.params(w.width, w.height, w.spp, w.max_bounces, w.seed) for w in ws]
    imgs, stats = native.batch_render(gs, ps)
    for g, p, img, st in zip(gs, ps, imgs, stats):
        ref, rst = g.render(p)
        assert np.array_equal(img, ref)
        assert st.extension_rays == rst.extension_rays and st.shadow_rays == rst.shadow_rays
    with pytest.raises(native.LuzError) as e:
        native.batch_render([gs[0], gs[0]], [ps[0], ps[0]])
    assert e.value.code == -1
    assert native.batch_render([], []) == ([], [])
    for g in gs:
        g.close()


@pytest.mark.gpu
def test_batch_of_many_waves_with_caustics_equals_individual_renders():
    """A batch larger than the largest autotuned wave (75.5 M paths of one Cornell view, so
    at least two multi-scene waves replay the wave graph), with a caustic-map scene (the
    shade instantiation with the photon estimate) and a second view of the same geometry:
    every film equals its single render bit for bit, the autotuner reports its trials on
    the first call and its choice is reused on the second."""
    from cases import caustic_case
    ws = [scenes.cornell(1024, 1024, 72, 8), caustic_case(), scenes.cornell(200, 120, 9, 5),
          scenes.mesh_glossy(96, 64, 3, 12, level=5)]
    gs = [native.GpuScene(w.scene.build()) for w in ws]
    ps = [native.params(w.width, w.height, w.spp, w.max_bounces, w.seed) for w in ws]
    imgs, stats, rep = native.batch_render(gs, ps, report=True)
    assert rep["waves"] >= 2 and len(rep["trials"]) >= 2
    assert rep["wave_paths"] in [t["wave_paths"] for t in rep["trials"]]
    for g, p, img, st in zip(gs, ps, imgs, stats):
        ref, rst = g.render(p)
        assert np.array_equal(img, ref)
        assert st.extension_rays == rst.extension_rays and st.shadow_rays == rst.shadow_rays
        assert st.samples == p.width * p.height * p.spp
    imgs2, _, rep2 = native.batch_render(gs, ps, report=True)
    assert rep2["trials"] == [] and rep2["wave_paths"] == rep["wave_paths"]
    assert all(np.array_equal(a, b) for a, b in zip(imgs, imgs2))
    for g in gs:
        g.close()
