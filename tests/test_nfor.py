"""The NFOR denoiser on the GPU (luz_gpu_nfor_denoise) against the reference's
Denoise::applyNFOR (src/core/Denoise/NFOR.cpp:977-1102), fixture
tests/golden/nfor.npz made by make_golden.py from the reference itself.

The GPU runs the same FP64 statements in the same order; CUDA's exp may differ
from the host libm's in the last bit, so results agree to ~1e-12, checked at
1e-8 relative."""
import numpy as np
import pytest

from cases import nfor_synthetic
from luz_b200 import native

KEYS = ("color_a", "color_b", "color_variance", "features_a", "features_b", "feature_variance")


def _inputs(name, golden):
    if name.startswith("synthetic"):
        return nfor_synthetic()
    g = golden("adaptive_" + name)
    return {k: g[k] for k in KEYS}


SETTINGS = {"synthetic_r3": dict(prefilter_radius=2, regression_radius=3, patch_radius=2)}


def test_reference_fixture_reproducible(golden):
    """The oracle (reference NFOR) reproduces the committed fixture."""
    import oracle as O
    if not O.reference_available():
        pytest.fail("oracle/_ref/libluzref.so missing: run __graft_entry__.build()")
    ref = golden("nfor")
    out = O.RefOracle().nfor(nfor_synthetic())
    assert np.array_equal(out, ref["synthetic"])


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["tiny_nfor", "tiny_adaptive_nfor", "synthetic", "synthetic_r3"])
def test_gpu_nfor_matches_reference(name, golden):
    ref = golden("nfor")[name]
    out = native.nfor_denoise(_inputs(name, golden), **SETTINGS.get(name, {}))
    assert out.shape == ref.shape
    assert np.allclose(out, ref, rtol=1e-8, atol=1e-12), np.abs(out - ref).max()


@pytest.mark.gpu
def test_gpu_nfor_settings_rejected():
    with pytest.raises(native.LuzError) as e:
        native.nfor_denoise(nfor_synthetic(), regression_radius=0)
    assert e.value.code == -1 and "NFOR radii must be positive." in str(e.value)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["tiny_nfor", "tiny_adaptive_nfor"])
def test_render_denoised_equals_render_then_denoise(name):
    """luz_gpu_render_denoised (buffers stay on the device) gives the film of
    render_ex and exactly the image of luz_gpu_nfor_denoise on its buffers."""
    from cases import ADAPTIVE_CASES
    from luz_b200 import desc as D
    fn, ad, _ = ADAPTIVE_CASES[name]
    w = fn()
    g = native.GpuScene(w.scene.build())
    p = native.params(w.width, w.height, w.spp, w.max_bounces, w.seed)
    a = native.adaptive(**ad) if ad else None
    img, used, bufs, st = g.render_ex(p, a, True)
    img2, den, used2, st2 = g.render_denoised(p, a)
    assert np.array_equal(img, img2) and np.array_equal(used, used2)
    assert np.array_equal(den, native.nfor_denoise(bufs))
    assert st2.samples == st.samples and st2.denoise_ms > 0.0
    s3 = D.NforSettings(2, 3, 2, 0, 1e-5)
    _, den3, _, _ = g.render_denoised(p, a, s3)
    assert np.array_equal(den3, native.nfor_denoise(bufs, prefilter_radius=2, regression_radius=3, patch_radius=2))
    with pytest.raises(native.LuzError) as e:
        g.render_denoised(p, a, D.NforSettings(1, 0, 1, 0, 1e-5))
    assert e.value.code == -1 and "NFOR radii must be positive." in str(e.value)
