"""Device error words and path-state budgets (luz_gpu_scene_set_traversal_limits,
luz_gpu_scene_set_path_budget).

* A traversal that outgrows its stack stops its walk and sets the scene's device
  error word; the call reports LUZ_E_DEVICE. The tests lower the enforced stack
  bounds so that a real scene trips them (a bounded check: the walk breaks out, no
  access leaves the stack), then restore them: the next call on the same handle
  succeeds and renders the same film as a fresh handle.
* A cap on the path state splits a render into more, smaller waves; the film is the
  same bit for bit. With most of the device memory held elsewhere, a render whose
  default wave no longer fits falls back to smaller waves instead of failing.
"""
import numpy as np
import pytest

from cases import CASES, camera_rays
from luz_b200 import native, scenes

pytestmark = pytest.mark.gpu


def test_stack_overflow_is_reported_and_does_not_poison_the_handle():
    w = CASES["instancing"]()
    b = w.scene.build()
    g = native.GpuScene(b)
    fresh = native.GpuScene(b)
    try:
        p = native.params(w.width, w.height, w.spp, w.max_bounces, w.seed)
        want, _ = fresh.render(p)
        g.set_traversal_limits(mesh_entries=2)     # the collapsed mesh walk's stack
        with pytest.raises(native.LuzError) as e:
            g.render(p)
        assert e.value.code == -5 and "stack overflow" in str(e.value)
        g.set_traversal_limits(top_entries=1)      # the top-level stack (every ray pushes the root's children)
        with pytest.raises(native.LuzError) as e:
            g.render(p)
        assert e.value.code == -5
        with pytest.raises(native.LuzError) as e:
            g.trace_rays(camera_rays(w, 256, seed=5), seed=w.seed)
        assert e.value.code == -5
        g.set_traversal_limits(0, 0)
        got, st = g.render(p)
        assert np.array_equal(got, want) and st.extension_rays > 0
        got2, _ = g.render(p)
        assert np.array_equal(got2, want)
        with pytest.raises(native.LuzError) as e:
            g.set_traversal_limits(mesh_entries=100000)
        assert e.value.code == -1
    finally:
        g.close()
        fresh.close()


def test_path_budget_splits_waves_with_the_same_film():
    w = CASES["glossy"]()
    g = native.GpuScene(w.scene.build())
    try:
        p = native.params(w.width, w.height, w.spp, w.max_bounces, w.seed)
        ref, st0 = g.render(p)
        g.set_path_budget(268 * 4096)       # 4,096 paths per wave
        img, st1 = g.render(p)
        assert st1.waves > st0.waves and st1.waves == -(-w.width * w.height * w.spp // 4096)
        assert np.array_equal(img, ref)
        g.set_path_budget(-1)
        img2, st2 = g.render(p)
        assert st2.waves == st0.waves and np.array_equal(img2, ref)
        with pytest.raises(native.LuzError):
            g.set_path_budget(-2)
    finally:
        g.close()


def test_render_falls_back_to_smaller_waves_when_memory_is_held():
    """Another user of the device holds all but 2 GiB: the 1080p frame at 8 spp
    (16.6 M paths, one 4.4 GB wave on an otherwise empty device) still renders, in
    smaller waves, to the same film."""
    import torch
    w = scenes.mesh_glossy(spp=8)
    b = w.scene.build()
    p = native.params(w.width, w.height, w.spp, w.max_bounces, w.seed)
    g = native.GpuScene(b)
    ref, st0 = g.render(p)
    g.close()
    torch.cuda.empty_cache()
    free, _ = torch.cuda.mem_get_info()
    hog = torch.empty(max(0, free - (2 << 30)), dtype=torch.uint8, device="cuda")
    g = native.GpuScene(b)
    try:
        g.set_path_budget(1 << 40)          # the budget allows the full wave: cudaMalloc must refuse it
        img, st = g.render(p)
        assert st.waves > st0.waves
        assert np.array_equal(img, ref)
    finally:
        g.close()
        del hog
        torch.cuda.empty_cache()
