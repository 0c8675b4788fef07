"""Launch tuning and the autotuner (luz_gpu_scene_set_tuning, luz_gpu_autotune): no
tuning choice changes a film. Staged top BVH nodes (shared memory), the coherence sort
of the extension queue, wave sizes, one or two wave lanes and persistent grid sizes give
the same image bit for bit; the autotuner leaves its choice on the handle and reports its timed trials."""
import numpy as np
import pytest

from cases import CASES
from luz_b200 import native

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["glossy", "instancing"])
def test_tuning_choices_leave_the_film_unchanged(name):
    w = CASES[name]()
    g = native.GpuScene(w.scene.build())
    try:
        p = native.params(w.width, w.height, w.spp, w.max_bounces, w.seed)
        ref, _ = g.render(p)
        for kw in (dict(staged_top_nodes=1), dict(sort_rays=1), dict(wave_paths=4096),
                   dict(extend_blocks_per_sm=2, shadow_blocks_per_sm=3, shade_blocks_per_sm=1),
                   dict(staged_top_nodes=1, sort_rays=1, wave_paths=5000, extend_blocks_per_sm=1)):
            g.set_tuning(**kw)
            img, _ = g.render(p)
            assert np.array_equal(img, ref), kw
            assert all(g.tuning()[k] == v for k, v in kw.items())
        g.set_tuning()
        with pytest.raises(native.LuzError):
            g.set_tuning(staged_top_nodes=2)
        with pytest.raises(native.LuzError):
            g.set_tuning(lanes=2)
    finally:
        g.close()


def test_two_wave_lanes_equal_one():
    """A frame of several waves on two lanes (consecutive waves on two streams over the two
    halves of the path state) gives the one-lane film and ray totals bit for bit; 8 Mi paths
    of path state make two lanes of 4 Mi, four waves for this 16.8 M-path frame."""
    from luz_b200 import scenes
    w = scenes.mesh_glossy(256, 256, 256, 8, level=5)
    g = native.GpuScene(w.scene.build())
    try:
        p = native.params(w.width, w.height, w.spp, w.max_bounces, w.seed)
        g.set_tuning(wave_paths=1 << 23)
        two, s2 = g.render(p)
        g.set_tuning(wave_paths=1 << 23, lanes=1)
        one, s1 = g.render(p)
        g.set_tuning()
        ref, s0 = g.render(p)
        assert s2.waves == 4 and s1.waves == 2 and s0.waves == 1, (s2.waves, s1.waves, s0.waves)
        assert np.array_equal(two, one) and np.array_equal(two, ref)
        assert s2.extension_rays == s1.extension_rays == s0.extension_rays
        assert s2.shadow_rays == s1.shadow_rays == s0.shadow_rays
    finally:
        g.close()


def test_autotune_keeps_the_best_trial():
    w = CASES["glossy"]()
    g = native.GpuScene(w.scene.build())
    try:
        p = native.params(w.width, w.height, 16, w.max_bounces, w.seed)
        ref, _ = g.render(p)
        chosen, trials = g.autotune(p)
        assert len(trials) >= 4 and chosen == g.tuning()
        best = min(ms for _, ms in trials)
        assert any(t == chosen and ms == best for t, ms in trials)
        img, _ = g.render(p)
        assert np.array_equal(img, ref)
    finally:
        g.close()
