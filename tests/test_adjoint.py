"""Albedo-texture gradients (luz_gpu_adjoint_forward / luz_gpu_adjoint_backward).

The reference has no gradients. The oracle is the derivative of the reference's
own film functional sum(adjoint * film) by central differences with common
random numbers (tests/golden/adjoint_cornell.npz, made by make_golden.py). At
depth 2 there is no Russian roulette, so the film is linear in each texel and
the differences are exact up to rounding (the fixture's h = 0.05 and h = 0.01
agree to 12 digits).
"""
import numpy as np
import pytest

from cases import adjoint_case
from luz_b200 import native


@pytest.fixture(scope="module")
def adjoint_run():
    w, adj, picks = adjoint_case()
    g = native.GpuScene(w.scene.build())
    p = native.params(w.width, w.height, w.spp, w.max_bounces, w.seed)
    tex = np.array(w.scene.textures[0])
    grad, st = g.adjoint_backward(p, 0, adj, tex.shape)
    return w, adj, picks, g, p, tex, grad, st


@pytest.mark.gpu
def test_gradient_matches_reference_finite_differences(adjoint_run, golden):
    w, adj, picks, g, p, tex, grad, st = adjoint_run
    ref = golden("adjoint_cornell")
    assert np.array_equal(ref["picks"], picks) and np.array_equal(ref["texture"], tex)
    got = np.array([grad[ty, tx, ch] for ty, tx, ch in picks])
    scale = np.abs(ref["fd"]).max()
    assert np.allclose(got, ref["fd"], rtol=2e-3, atol=1e-4 * scale), (got, ref["fd"])
    assert st.samples == w.width * w.height * w.spp


@pytest.mark.gpu
def test_gradient_matches_own_finite_differences(adjoint_run):
    """Same check against the GPU's own film (common random numbers)."""
    w, adj, picks, g, p, tex, grad, st = adjoint_run
    h = 0.05

    def loss(t):
        img, _ = g.adjoint_forward(p, 0, t)
        return float((adj.astype(np.float64) * img).sum())

    for ty, tx, ch in picks[:4]:
        tp, tm = tex.copy(), tex.copy()
        tp[ty, tx, ch] += h
        tm[ty, tx, ch] -= h
        fd = (loss(tp) - loss(tm)) / (2 * h)
        assert abs(fd - grad[ty, tx, ch]) <= 2e-3 * abs(fd) + 1e-5, (ty, tx, ch, fd, grad[ty, tx, ch])
    g.set_texture(0, tex)


@pytest.mark.gpu
def test_gradient_support_and_errors(adjoint_run):
    w, adj, picks, g, p, tex, grad, st = adjoint_run
    # texels the camera cannot see through any path keep a zero gradient; most receive some
    assert np.isfinite(grad).all() and (grad != 0).mean() > 0.5
    with pytest.raises(native.LuzError) as e:
        g.adjoint_backward(p, 3, adj, tex.shape)
    assert e.value.code == -1
    with pytest.raises(native.LuzError) as e:
        g.set_texture(1, tex)
    assert e.value.code == -1
