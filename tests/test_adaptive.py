"""Adaptive sampling and NFOR buffers (luz_gpu_render_ex).

Reference: _threadRender with adaptiveSampleConverged and storeDenoisePixel
(src/renderer/Threads.cpp:194-372, 551-641). The oracle is oracle/adaptive.py,
a numpy restatement of that loop, pinned here against the reference itself
(bit-exact on the reference's own per-sample colours); the GPU is then checked
(a) bit-exactly against the restatement fed with the GPU's own per-sample
colours, and (b) against the reference fixtures within tolerance (FP32 paths).
"""
import numpy as np
import pytest

import adaptive as A
from cases import ADAPTIVE_CASES
from luz_b200 import native


def _grid(w):
    yy, xx = np.mgrid[0:w.height, 0:w.width]
    P, S = w.width * w.height, w.spp
    return (np.repeat(xx.ravel(), S).astype(np.int32), np.repeat(yy.ravel(), S).astype(np.int32),
            np.tile(np.arange(S), P).astype(np.int32))


# ----------------------------------------------------------------------------- restatement (CPU)

def test_rule_constant_pixel_stops_at_min_samples():
    c = np.full((2, 64, 3), 0.5)
    _, used, _ = A.render_pixels(c, dict(min_samples=8, check_interval=4, threshold=0.03))
    # zero variance: converged at the first check point, which is min_samples
    assert used.tolist() == [8, 8]


def test_rule_dark_pixel_waits_for_dark_minimum():
    c = np.full((1, 400, 3), 0.001)
    _, used, _ = A.render_pixels(c, dict(min_samples=16, check_interval=16, threshold=0.5))
    # max luminance < 0.02: no stop before darkMinimumSamples = max(256, 16 + 48)
    assert used[0] == 256


def test_rule_nan_samples_are_cleaned_and_full_count_when_adaptive_off():
    c = np.full((1, 10, 3), 0.25)
    c[0, 3, 1] = np.nan
    c[0, 5, :] = np.inf
    rgb, used, _ = A.render_pixels(c, None)
    assert used[0] == 10
    assert np.allclose(rgb[0], [0.225, 0.2, 0.225])


def test_rule_half_buffers_alternate_samples():
    c = np.zeros((1, 6, 3))
    c[0, :, 0] = [1, 2, 3, 4, 5, 6]
    f = np.zeros((1, 6, 11))
    f[0, :, 3] = [1, 0, 1, 0, 1, 0]
    _, used, b = A.render_pixels(c, None, f)
    assert b["color_a"][0, 0] == 3.0 and b["color_b"][0, 0] == 4.0
    assert b["features_a"][0, 3] == 1.0 and b["features_b"][0, 3] == 0.0
    assert np.isclose(b["feature_variance"][0, 3], (0.25 * 6 / 5) / 6)


@pytest.mark.parametrize("name", list(ADAPTIVE_CASES))
def test_restatement_matches_reference(name, golden):
    """The numpy restatement reproduces the reference's _threadRender bit for bit
    when fed the reference's own per-sample colours and features."""
    import oracle as O
    if not O.reference_available():
        pytest.fail("oracle/_ref/libluzref.so missing: run __graft_entry__.build()")
    fn, ad, nfor = ADAPTIVE_CASES[name]
    w = fn()
    rs = O.RefOracle().scene(w.scene.build())
    p = native.params(w.width, w.height, w.spp, w.max_bounces, w.seed)
    x, y, s = _grid(w)
    rgb, feat = rs.trace_samples(p, x, y, s, half_streams=nfor)
    P, S = w.width * w.height, w.spp
    r, u, b = A.render_pixels(rgb.reshape(P, S, 3), ad, feat.reshape(P, S, 11) if nfor else None)
    g = golden("adaptive_" + name)
    assert np.array_equal(u, g["used"].ravel())
    assert np.array_equal(r, g["rgb"].reshape(P, 3))
    if nfor:
        for k, v in b.items():
            assert np.array_equal(v.reshape(g[k].shape), g[k]), k


# ----------------------------------------------------------------------------- GPU

def _gpu_samples(g, w, half_streams):
    x, y, s = _grid(w)
    P, S = w.width * w.height, w.spp
    rgb = np.zeros((x.shape[0], 3), np.float32)
    if half_streams:
        for st in (1, 2):
            sel = (s % 2) == (st - 1)
            rgb[sel] = g.trace_paths(native.params(w.width, w.height, w.spp, w.max_bounces, w.seed, stream=st),
                                     x[sel], y[sel], s[sel])
    else:
        rgb = g.trace_paths(native.params(w.width, w.height, w.spp, w.max_bounces, w.seed), x, y, s)
    return rgb.reshape(P, S, 3)


@pytest.fixture(scope="module")
def adaptive_runs():
    out = {}
    for name, (fn, ad, nfor) in ADAPTIVE_CASES.items():
        w = fn()
        g = native.GpuScene(w.scene.build())
        p = native.params(w.width, w.height, w.spp, w.max_bounces, w.seed)
        a = native.adaptive(**ad) if ad else None
        img, used, bufs, st = g.render_ex(p, a, nfor)
        out[name] = (w, g, img, used, bufs, st)
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(ADAPTIVE_CASES))
def test_gpu_decisions_match_restated_rule(name, adaptive_runs):
    """Stop decisions, films and colour buffers equal the restatement run on the
    GPU's own per-sample colours (same FP64 sums in the same order)."""
    w, g, img, used, bufs, st = adaptive_runs[name]
    _, ad, nfor = ADAPTIVE_CASES[name]
    P, S = w.width * w.height, w.spp
    c = _gpu_samples(g, w, nfor)
    r, u, b = A.render_pixels(c, ad, np.zeros((P, S, 11)) if nfor else None)
    assert np.array_equal(used.ravel(), u)
    assert np.array_equal(img.reshape(P, 3), r.astype(np.float32))
    assert st.samples == float(u.sum())
    if nfor:
        for k in ("color_a", "color_b", "color_variance"):
            assert np.array_equal(bufs[k].reshape(b[k].shape), b[k]), k


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(ADAPTIVE_CASES))
def test_gpu_matches_reference_fixture(name, adaptive_runs, golden):
    """Against the reference's own _threadRender output: FP32 paths change a few
    stop decisions and the low bits of the means, nothing more."""
    w, g, img, used, bufs, st = adaptive_runs[name]
    _, ad, nfor = ADAPTIVE_CASES[name]
    ref = golden("adaptive_" + name)
    same = used == ref["used"]
    assert same.mean() >= 0.97
    rel = np.abs(img - ref["rgb"]) / np.maximum(np.abs(ref["rgb"]), 1e-3)
    assert (rel.max(axis=-1)[same] <= 1e-3).mean() >= 0.98
    if nfor:
        for k in ("features_a", "features_b"):
            d = np.abs(bufs[k] - ref[k])
            assert (d.max(axis=-1)[same] <= 1e-4).mean() >= 0.98, k
        for k in ("color_a", "color_b"):
            rk = np.abs(bufs[k] - ref[k]) / np.maximum(np.abs(ref[k]), 1e-3)
            assert (rk.max(axis=-1)[same] <= 1e-3).mean() >= 0.98, k


@pytest.mark.gpu
def test_render_ex_without_options_equals_render(adaptive_runs):
    w, g, *_ = adaptive_runs["cornell_adaptive"]
    p = native.params(w.width, w.height, 8, w.max_bounces, w.seed)
    img, _ = g.render(p)
    img2, used, bufs, st = g.render_ex(p)
    assert np.array_equal(img, img2) and (used == 8).all() and bufs is None


@pytest.mark.gpu
def test_render_ex_invalid_adaptive_settings(adaptive_runs):
    w, g, *_ = adaptive_runs["cornell_adaptive"]
    p = native.params(8, 8, 4, 2, 1)
    for bad, msg in ((dict(min_samples=0), "minimum samples"), (dict(check_interval=0), "check interval"),
                     (dict(threshold=float("nan")), "threshold")):
        with pytest.raises(native.LuzError) as e:
            g.render_ex(p, native.adaptive(**bad))
        assert e.value.code == -1 and msg in str(e.value)
