"""Learned radiance cache (include/luz_gpu.h: luz_gpu_cache_*, luz_gpu_render_cached).

The reference renderer has no cache, so the oracle is the numpy restatement in
oracle/radiance_cache.py: its backward pass is checked against finite
differences in float64 (CPU), and the GPU kernels (FP16 tensor-core matmuls,
FP32 accumulation) against its FP16-rounded forward pass, gradient and Adam
step. Tolerances: FP16 rounding of inputs, weights and activations may differ
by one unit in the last place where the GPU's sinpi/cospi and numpy's sin(pi x)
or the accumulation order differ, so outputs agree to ~1e-2 relative."""
import numpy as np
import pytest

import radiance_cache as RC
from luz_b200 import desc as D
from luz_b200 import native


def rows(n, seed=5):
    rng = np.random.default_rng(seed)
    x = np.zeros((n, 10), np.float32)
    x[:, 0:3] = rng.uniform(0.0, 1.0, (n, 3))
    d = rng.normal(size=(n, 3))
    x[:, 3:6] = d / np.linalg.norm(d, axis=1, keepdims=True)
    nn = rng.normal(size=(n, 3))
    x[:, 6:9] = nn / np.linalg.norm(nn, axis=1, keepdims=True)
    x[:, 9] = rng.uniform(0.0, 1.0, n)
    return x


def smooth_target(x):
    """A smooth radiance field over the inputs (what training should fit)."""
    r = 1.0 + 0.5 * np.sin(3.0 * x[:, 0]) * np.cos(2.0 * x[:, 1]) + 0.3 * x[:, 4]
    return np.stack([r, 0.7 * r + 0.2 * x[:, 2], 0.5 + 0.4 * x[:, 9]], 1).astype(np.float32)


def test_restated_gradient_matches_finite_differences():
    rng = np.random.default_rng(1)
    w = RC.init_weights(3).astype(np.float64) * 0.5
    x = rows(6)
    t = np.abs(rng.normal(size=(6, 3))).astype(np.float64)
    loss, g = RC.gradient(w, x, t, exact=True)

    def L(wv):
        y, _ = RC.forward(wv, x, exact=True)
        yy = y[:, :3]
        return float(np.sum((yy - t) ** 2 / (yy * yy + RC.EPS_REL))) / x.shape[0]

    # the loss holds the denominator constant: differentiate with it frozen at w
    y0, _ = RC.forward(w, x, exact=True)
    den = y0[:, :3] ** 2 + RC.EPS_REL

    def Lf(wv):
        y, _ = RC.forward(wv, x, exact=True)
        return float(np.sum((y[:, :3] - t) ** 2 / den)) / x.shape[0]

    assert abs(L(w) - loss) < 1e-12
    for i in rng.choice(RC.N_PARAMS, 40, replace=False):
        h = 1e-6
        wp, wm = w.copy(), w.copy()
        wp[i] += h
        wm[i] -= h
        fd = (Lf(wp) - Lf(wm)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])


@pytest.fixture(scope="module")
def cache():
    c = native.RadianceCache(D.cache_params(seed=7, batch=4096))
    yield c
    c.close()


@pytest.mark.gpu
def test_initial_weights_match_restatement(cache):
    assert np.array_equal(cache.weights(), RC.init_weights(7))


@pytest.mark.gpu
def test_prediction_matches_restatement(cache):
    x = rows(1000)
    ref, _ = RC.forward(RC.init_weights(7), x)
    got = cache.predict(x)
    scale = np.abs(ref[:, :3]).max()
    assert np.allclose(got, ref[:, :3], rtol=2e-2, atol=2e-3 * scale), np.abs(got - ref[:, :3]).max()


@pytest.mark.gpu
def test_gradient_matches_restatement(cache):
    x = rows(1000, seed=9)
    t = smooth_target(x)
    w = RC.init_weights(7)
    loss_ref, g_ref = RC.gradient(w, x, t)
    g, loss = cache.gradient(x, t)
    assert abs(loss - loss_ref) <= 1e-3 * loss_ref
    assert np.linalg.norm(g - g_ref) <= 3e-2 * np.linalg.norm(g_ref)
    for l, ((k, n), off) in enumerate(zip(RC.LAYERS, RC.OFFSETS)):   # every layer, not only the largest
        a, b = g[off:off + k * n], g_ref[off:off + k * n]
        assert np.linalg.norm(a - b) <= 5e-2 * np.linalg.norm(b), l


@pytest.mark.gpu
def test_adam_step_matches_restatement(cache):
    x = rows(2000, seed=11)
    t = smooth_target(x)
    w0 = RC.init_weights(7)
    cache.set_weights(w0)
    cache.train(x, t, steps=1)
    _, g = RC.gradient(w0, x, t)
    w, m, v = w0.astype(np.float64), np.zeros(RC.N_PARAMS), np.zeros(RC.N_PARAMS)
    RC.adam(w, m, v, g.astype(np.float64), 1)
    got = cache.weights()
    # a first Adam step moves each weight by ~lr * sign(g): compare the moves
    moved, ref_moved = got - w0, w - w0
    agree = np.abs(moved - ref_moved) <= 1e-3 * 1e-2 + 0.05 * np.abs(ref_moved)
    assert agree.mean() >= 0.97, agree.mean()
    cache.set_weights(w0)


@pytest.mark.gpu
def test_training_fits_a_smooth_field(cache):
    cache.set_weights(RC.init_weights(7))
    x = rows(4096, seed=13)
    t = smooth_target(x)
    losses = cache.train(x, t, steps=400)
    assert np.isfinite(losses).all()
    assert losses[-1] < 0.05 * losses[0], (losses[0], losses[-1])
    xv = rows(2048, seed=17)
    pred = cache.predict(xv)
    rel = np.abs(pred - smooth_target(xv)) / smooth_target(xv)
    assert np.median(rel) < 0.15, np.median(rel)   # unseen rows of a 10-input field fit from 4096 rows
    cache.set_weights(RC.init_weights(7))


@pytest.mark.gpu
def test_invalid_arguments(cache):
    with pytest.raises(native.LuzError):
        native.RadianceCache(D.cache_params(batch=0))
    for bad in (-0.1, 1.5, float("nan")):
        with pytest.raises(native.LuzError):
            native.RadianceCache(D.cache_params(min_roughness=bad))
    for bad in (-1, 4097):
        with pytest.raises(native.LuzError):
            native.RadianceCache(D.cache_params(warm_steps=bad))
    with pytest.raises(native.LuzError):
        cache.train(rows(5000), smooth_target(rows(5000)), steps=1)   # more rows than the batch


def rmse(a, b):
    return float(np.sqrt(np.mean((a.astype(np.float64) - b) ** 2)))


@pytest.mark.gpu
def test_cached_render_against_plain():
    """Cornell 64 x 64, depth 8: after a training render, the cache's image at 32 spp is
    closer to the converged plain image (4096 spp) than the plain 32-spp image, it
    traces fewer rays, and its mean stays within 5% (the cache is biased; the plain
    renderer is the reference)."""
    from luz_b200 import scenes
    w = scenes.cornell(64, 64, 1, 8)
    g = native.GpuScene(w.scene.build())
    ref, _ = g.render(native.params(64, 64, 4096, 8, 5))
    plain, sp = g.render(native.params(64, 64, 32, 8, 11))
    c = native.RadianceCache(D.cache_params(seed=3, batch=4096, train_every=4))
    c.render(g, native.params(64, 64, 256, 8, 21))
    cached, sc = c.render(g, native.params(64, 64, 32, 8, 11))
    c.close()
    g.close()
    facts = dict(rays=(sc.extension_rays, sp.extension_rays), mean=(float(cached.mean()), float(ref.mean())),
                 rmse=(rmse(cached, ref), rmse(plain, ref)))
    assert np.isfinite(cached).all()
    assert sc.samples == sp.samples
    # one path in 4 trains and runs on to its next surface vertex; the rest stop at their second
    assert sc.extension_rays < 0.8 * sp.extension_rays, facts
    assert abs(cached.mean() - ref.mean()) < 0.05 * ref.mean(), facts
    assert rmse(cached, ref) < rmse(plain, ref), facts


@pytest.mark.gpu
def test_min_roughness_gate():
    """Glass (roughness 0.1) sphere over a metal (0.3) floor under an environment map: with
    min_roughness 0.5 no vertex is rough enough to query the cache, so the cached render
    traces every path to its end like the plain render (same rays, same image up to
    contraction differences between the two shading instantiations); with the gate at 0 the
    cache ends the paths that reach a second vertex there."""
    from luz_b200 import scenes
    w = scenes.mesh_glossy(64, 36, 1, 8, level=3)
    g = native.GpuScene(w.scene.build())
    p = native.params(64, 36, 16, 8, 5)
    plain, sp = g.render(p)
    c = native.RadianceCache(D.cache_params(seed=3, batch=4096, min_roughness=0.5))
    gated, sg = c.render(g, p)
    c.close()
    c = native.RadianceCache(D.cache_params(seed=3, batch=4096, min_roughness=0.0))
    _, so = c.render(g, p)
    c.close()
    g.close()
    assert sg.extension_rays == sp.extension_rays and sg.shadow_rays == sp.shadow_rays
    assert np.allclose(gated, plain, rtol=1e-4, atol=1e-5)
    assert so.extension_rays < 0.9 * sp.extension_rays   # most paths leave for the environment first
