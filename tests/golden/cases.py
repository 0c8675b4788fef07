"""Named, seeded test cases shared by the fixture generator and the tests.

Each case is a small version of one benchmark configuration (same object
kinds, materials, light types and value distributions, fewer pixels/samples)
so the reference oracle computes its fixtures in seconds.
"""
from __future__ import annotations

import numpy as np

from luz_b200 import scenes
from luz_b200.desc import Scene


def degenerate_soup() -> Scene:
    """Triangle soup with degenerate and duplicate triangles (dropped / tied)."""
    rng = np.random.default_rng(17)
    s = Scene()
    m = s.lambertian((0.5, 0.5, 0.5))
    tris = rng.uniform(-1, 1, (300, 3, 3))
    tris[::25, 2] = tris[::25, 1]            # zero-area triangles
    tris[1::40] = tris[0::40][: len(tris[1::40])]   # exact duplicates -> equal-t ties
    tris[::7, :, 1] = np.round(tris[::7, :, 1], 1)  # equal centroids along y
    s.mesh(tris, m)
    s.camera.position = (0.0, 0.0, 4.0)
    return s


CASES = {
    "cornell": lambda: scenes.cornell(64, 64, 4, 8),
    "tiny": lambda: scenes.tiny_mixed(24, 18, 4, 6),
    "glossy": lambda: scenes.mesh_glossy(96, 54, 4, 12, level=4),
    "instancing": lambda: scenes.instancing_volumes(64, 36, 4, 16, count=500),
    "linear_sky": lambda: scenes.spheres_linear_sky(64, 36, 4, 12),
    "ies": lambda: scenes.ies_room(48, 36, 4, 6),
    "atmosphere": lambda: scenes.atmosphere_hills(48, 32, 4, 3),
    "caustics": lambda: scenes.caustic_pool(48, 36, 4, 8, photons=20000),
}

# The benchmarked frames at full size (1920x1080 over the 1,310,722-triangle mesh;
# 1280x720 over 1e5 instances in an HG medium): the mesh BVH and top-level BVHNode
# layouts (hashes of the full arrays), 2,000 ray hits and 4,096 paths, with the
# reference's FP32-ambiguity flags (oracle.ambiguous_rays / ambiguous_paths).
FULL_CASES = {
    "glossy_full": lambda: scenes.mesh_glossy(),
    "instancing_full": lambda: scenes.instancing_volumes(),
}

# Caustic photon map case (CausticPhotonMap): the scene with its map on, and the
# (render seed, max bounces) pairs whose stored-photon counts are pinned.
def caustic_case():
    return scenes.caustic_pool(64, 48, 2, 8)


# Converged-oracle cases: the reference's film at 65,536 spp.
ORACLE_64K = {
    "cornell": lambda: scenes.cornell(24, 24, 65536, 8),
    "tiny": lambda: scenes.tiny_mixed(24, 18, 65536, 6),
}

# The config-0 frame itself (Cornell box, 300x300, depth 8) at 65,536 spp: the whole
# converged image, against which GPU films at increasing spp are measured.
ORACLE_64K_FULL = {
    "cornell300": lambda: scenes.cornell(300, 300, 65536, 8),
}

# Seeded 4,096-pixel subsets of the full-size benchmarked frames, rendered by the reference
# at 65,536 spp (the converged oracle where a full 1080p or 720p frame at that count is out
# of reach on host cores).
ORACLE_64K_SUBSET = {
    "glossy_full": lambda: scenes.mesh_glossy(spp=65536),
    "instancing_full": lambda: scenes.instancing_volumes(spp=65536),
}


def oracle_subset_pixels(w, n=4096, seed=4242):
    rng = np.random.default_rng(seed)
    idx = np.sort(rng.choice(w.width * w.height, n, replace=False))
    return (idx % w.width).astype(np.int32), (idx // w.width).astype(np.int32)


CAUSTIC_COUNTS = [(424242424, 8), (7, 8), (424242424, 3), (99, 12)]

# Adaptive sampling / NFOR buffer cases: workload, adaptive settings (None = off), NFOR on.
ADAPTIVE_CASES = {
    "cornell_adaptive": (lambda: scenes.cornell(32, 32, 128, 8),
                         dict(min_samples=16, check_interval=16, threshold=0.25), False),
    "tiny_nfor": (lambda: scenes.tiny_mixed(24, 18, 8, 6), None, True),
    "tiny_adaptive_nfor": (lambda: scenes.tiny_mixed(24, 18, 48, 6),
                           dict(min_samples=8, check_interval=8, threshold=0.15), True),
}

# Differentiation case: textured Cornell box (texture 0 = back-wall albedo), depth 2
# (no Russian roulette, so finite differences with common random numbers are exact
# up to rounding), a seeded adjoint image and the texel channels checked.
def adjoint_case():
    w = scenes.cornell_textured(48, 48, 16, 2)
    rng = np.random.default_rng(77)
    adj = rng.normal(0.0, 1.0, (w.height, w.width, 3)).astype(np.float32)
    picks = np.stack([rng.integers(0, 32, 8), rng.integers(0, 32, 8), rng.integers(0, 3, 8)], 1)
    return w, adj, picks


# Differentiation at the C3 configuration: the 256 x 256 textured Cornell box at depth 8
# (Russian roulette from bounce 3), a seeded dLoss/dpixel image, and central differences of
# the reference's own film at 65,536 spp (common random numbers) along three directions:
# every back-wall texel scaled together (albedo), the light's emission scaled (emission), and
# the density of a fog cube in the same box (density). The GPU's replay gradients, projected
# on the same directions, must agree within 2%.
C3_H = 1e-3
C3_SPP_FD = 65536


def c3_case(spp=64):
    w = scenes.cornell_textured(256, 256, spp, 8)
    adj = np.random.default_rng(78).uniform(0.5, 1.5, (256, 256, 3)).astype(np.float32)
    return w, adj


def c3_fog_case(spp=64, density=0.0035):
    w = scenes.cornell_textured(256, 256, spp, 8)
    fog = w.scene.henyey_greenstein((0.8, 0.8, 0.8), 0.3)
    obj = w.scene.volume_cube((278.0, 250.0, 280.0), 300.0, 300.0, 300.0, fog, density)
    return w, obj


def nfor_synthetic(width: int = 40, height: int = 32, seed: int = 3) -> dict:
    """Seeded NFOR buffers with the structure of a render's: smooth colour with noise, a
    few fireflies, an edge in the features, small variances."""
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:height, 0:width]
    base = np.stack([0.3 + 0.4 * xx / width, 0.2 + 0.5 * yy / height, 0.4 + 0.1 * np.sin(xx / 5.0)], -1)
    base[:, width // 2:] *= 0.5                        # an edge the features also show
    def half():
        c = base + rng.normal(0.0, 0.05, base.shape)
        for _ in range(6):                             # fireflies
            c[rng.integers(2, height - 2), rng.integers(2, width - 2)] = rng.uniform(3.0, 9.0, 3)
        return np.clip(c, 0.0, None)
    feat = np.zeros((height, width, 11))
    feat[..., 0] = xx / (width - 1.0)
    feat[..., 1] = yy / (height - 1.0)
    feat[..., 2] = 1.0
    feat[..., 3] = 0.5 + 0.1 * (xx >= width // 2)
    feat[..., 4:7] = 0.5 + 0.3 * np.stack([np.cos(xx / 7.0), np.sin(yy / 6.0), np.full(xx.shape, 0.2)], -1)
    feat[..., 7:10] = np.where((xx >= width // 2)[..., None], 0.3, 0.7)
    feat[..., 10] = 1.0 / 7.0
    fa = feat + rng.normal(0.0, 0.01, feat.shape)
    fb = feat + rng.normal(0.0, 0.01, feat.shape)
    return {"color_a": half(), "color_b": half(), "color_variance": rng.uniform(1e-4, 3e-3, (height, width)),
            "features_a": fa, "features_b": fb, "feature_variance": rng.uniform(1e-6, 1e-4, (height, width, 11))}


BVH_CASES = {
    "box": lambda: scenes.cornell().scene,
    "icosphere3": lambda: scenes.mesh_glossy(level=3).scene,
    "torus": lambda: scenes.instancing_volumes(count=1).scene,
    "degenerate": degenerate_soup,
}


def camera_rays(w, n: int, seed: int) -> np.ndarray:
    """Rays from near the camera into the view cone: (ox,oy,oz,tmin,dx,dy,dz,tmax) float32."""
    rng = np.random.default_rng(seed)
    cam = w.scene.camera
    fwd = np.asarray(cam.direction, float)
    fwd /= np.linalg.norm(fwd)
    org = np.asarray(cam.position, float) + rng.normal(0.0, 0.01, (n, 3))
    d = rng.normal(0.0, 1.0, (n, 3)) + 2.5 * fwd
    d[: n // 20, 1] = 0.0                     # axis-parallel components (inverse = 0 branch)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = np.zeros((n, 8), np.float32)
    r[:, 0:3] = org
    r[:, 3] = 1e-3
    r[:, 4:7] = d
    r[:, 7] = np.inf
    r[n // 10: n // 5, 7] = rng.uniform(0.5, 20.0, n // 5 - n // 10)   # bounded segments
    return r


def path_keys(w, n: int, seed: int):
    rng = np.random.default_rng(seed)
    return (rng.integers(0, w.width, n).astype(np.int32), rng.integers(0, w.height, n).astype(np.int32),
            rng.integers(0, w.spp, n).astype(np.int32))
