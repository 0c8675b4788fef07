"""Caustic photon map (CausticPhotonMap::build / estimate, src/renderer/CausticPhotonMap.cpp)
on the GPU against the reference, fixture tests/golden/caustics.npz made by make_golden.py
from the reference itself: stored-photon counts for several render seeds and bounce
limits, and the radiance of one-sample paths whose caustic estimate is non-zero.

The photon pass runs in FP32 like the path loop, so a photon whose Russian-roulette
or refraction decision sits on a rounding boundary can differ; counts agree to a few
photons and almost every gathering path to 1e-4 relative."""
import numpy as np
import pytest

from cases import CAUSTIC_COUNTS, caustic_case
from luz_b200 import native


def test_reference_fixture_reproducible(golden):
    """The oracle (the reference's photon map) reproduces the committed fixture."""
    import oracle as O
    if not O.reference_available():
        pytest.fail("oracle/_ref/libluzref.so missing: run __graft_entry__.build()")
    ref = golden("caustics")
    w = caustic_case()
    rs = O.RefOracle().scene(w.scene.build())
    assert [rs.caustic_photons(sd, mb) for sd, mb in CAUSTIC_COUNTS] == list(ref["counts"])
    p = native.params(w.width, w.height, w.spp, w.max_bounces, w.seed)
    assert np.array_equal(rs.trace_paths(p, ref["x"][:200], ref["y"][:200], ref["s"][:200]), ref["rgb"][:200])


@pytest.fixture(scope="module")
def caustic_gpu():
    w = caustic_case()
    g = native.GpuScene(w.scene.build())
    yield w, g
    g.close()


@pytest.mark.gpu
def test_photon_counts_match_reference(caustic_gpu, golden):
    w, g = caustic_gpu
    ref = golden("caustics")["counts"]
    for (seed, mb), n_ref in zip(CAUSTIC_COUNTS, ref):
        _, st = g.render(native.params(8, 8, 1, mb, seed))
        assert abs(st.caustic_photons - n_ref) <= 2 + 0.002 * n_ref, (seed, mb, st.caustic_photons, n_ref)
        assert st.caustic_ms > 0.0
    # the same seed and bounce limit reuse the map
    _, st = g.render(native.params(8, 8, 1, CAUSTIC_COUNTS[-1][1], CAUSTIC_COUNTS[-1][0]))
    assert st.caustic_ms == 0.0 and st.caustic_photons > 0


@pytest.mark.gpu
def test_gathering_paths_match_reference(caustic_gpu, golden):
    w, g = caustic_gpu
    ref = golden("caustics")
    p = native.params(w.width, w.height, w.spp, w.max_bounces, w.seed)
    rgb = g.trace_paths(p, ref["x"], ref["y"], ref["s"]).astype(np.float64)
    r = ref["rgb"]
    rel = np.abs(rgb - r) / np.maximum(np.abs(r), 1e-3)
    frac = (rel.max(axis=1) <= 1e-4).mean()
    assert frac >= 0.95, frac
    # the caustic term is present: the paths differ from their photon-map-free values
    assert (np.abs(rgb - ref["rgb_off"]).max(axis=1) > 1e-3 * np.maximum(np.abs(r).max(axis=1), 1e-3)).mean() > 0.9
    assert abs(rgb.mean() - r.mean()) <= 2e-3 * r.mean()


@pytest.mark.gpu
def test_caustic_render_deterministic_and_map_rebuilt(caustic_gpu):
    w, g = caustic_gpu
    p = native.params(w.width, w.height, 2, w.max_bounces, w.seed)
    a, sa = g.render(p)
    g.render(native.params(w.width, w.height, 2, w.max_bounces, 5))   # another seed: rebuild
    b, sb = g.render(p)                                                 # and back
    assert a.tobytes() == b.tobytes() and sb.caustic_ms > 0.0
    assert sa.caustic_photons == sb.caustic_photons
    img, used, _, st = g.render_ex(p)
    assert np.array_equal(img, a) and st.caustic_photons == sa.caustic_photons


@pytest.mark.gpu
def test_caustic_scene_unsupported_in_adjoint(caustic_gpu):
    w, g = caustic_gpu
    with pytest.raises(native.LuzError) as e:
        g.adjoint_backward(native.params(8, 8, 1, 4, 1), 0, np.zeros((8, 8, 3), np.float32), (2, 2, 3))
    assert e.value.code in (-1, -3)


@pytest.mark.gpu
def test_caustic_scene_in_batch_and_denoised_render(caustic_gpu):
    """Every render entry point builds the map: a batch of the caustic scene and a plain scene
    equals their one-at-a-time renders, and the render-and-denoise call films the same image."""
    from luz_b200 import scenes
    w, g = caustic_gpu
    p = native.params(w.width, w.height, 2, w.max_bounces, 31)
    t = scenes.tiny_mixed(24, 18, 2, 4)
    gt = native.GpuScene(t.scene.build())
    pt = native.params(t.width, t.height, t.spp, t.max_bounces, t.seed)
    a, _ = g.render(p)
    b, _ = gt.render(pt)
    outs, stats = native.batch_render([g, gt], [p, pt])
    assert np.array_equal(outs[0], a) and np.array_equal(outs[1], b)
    assert stats[0].caustic_photons > 0 and stats[1].caustic_photons == 0
    img, den, used, st = g.render_denoised(p)
    assert st.caustic_photons == stats[0].caustic_photons and np.isfinite(den).all()
    ref, _, _, _ = g.render_ex(native.params(w.width, w.height, 2, w.max_bounces, 31), None, True)
    assert np.array_equal(img, ref)
    gt.close()
