"""Generates the golden fixtures in this folder from the Luz reference itself.

Runs in the build container only (it needs oracle/_ref/libluzref.so, built by
oracle/Makefile from the reference sources). Every value stored here is an
output of the unmodified reference code:
  sampler.npz        Sampler::sample1D / sample2D          (src/core/Sampler.cpp)
  bvh_<case>.npz     Mesh::_packedBVHNodes, _triangleIndices (src/core/Hittables/Mesh.cpp)
  hits_<case>.npz    _checkHits / isShadowOccluded results   (HitHelper.cpp, ColorHelper.cpp)
  paths_<case>.npz   per-path radiance, calculateLightRaysColor (ColorHelper.cpp)
  image_<case>.npz   Renderer::render film (Raw view, no denoise, no adaptive)
  adaptive_<case>.npz _threadRender with adaptive sampling and/or NFOR buffers
                     (src/renderer/Threads.cpp:551-641): film, samples used, NFORBuffers
  adjoint_cornell.npz central differences of the reference's film functional
                     sum(adjoint * film) with respect to chosen texel channels
                     (the reference has no gradients; common random numbers: same seed)
  nfor.npz           Denoise::applyNFOR outputs (src/core/Denoise/NFOR.cpp:977-1102)
  caustics.npz       CausticPhotonMap::build photon counts (src/renderer/CausticPhotonMap.cpp:430-551)
                     and per-path radiance of paths whose caustic estimate is non-zero
  oracle64k_<case>.npz Renderer::render films at 65,536 spp (the converged oracle images)
  full_<case>.npz    the benchmarked frames at full size: sha256 of the reference's mesh
                     BVH arrays and of its top-level BVHNode tree (BVHNode.cpp:142-185),
                     ray hits and per-path radiance with FP32-ambiguity flags
  The hits_ and paths_ files carry the same ambiguity flags (oracle/oracle.py).
Usage: python tests/golden/make_golden.py [adaptive | adjoint | nfor | caustics | oracle64k | cases <name>...]
"""
from __future__ import annotations

import os
import sys
import zlib

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, HERE)

from cases import (ADAPTIVE_CASES, BVH_CASES, C3_H, C3_SPP_FD, CASES, CAUSTIC_COUNTS, FULL_CASES,  # noqa: E402
                   ORACLE_64K, ORACLE_64K_FULL, ORACLE_64K_SUBSET, adjoint_case, c3_case, c3_fog_case,
                   oracle_subset_pixels,
                   camera_rays, caustic_case, nfor_synthetic, path_keys)
from luz_b200 import native  # noqa: E402
import oracle as O  # noqa: E402
from oracle import RefOracle  # noqa: E402


def adaptive_fixtures(o):
    for name, (fn, ad, nfor) in ADAPTIVE_CASES.items():
        w = fn()
        rs = o.scene(w.scene.build())
        p = native.params(w.width, w.height, w.spp, w.max_bounces, w.seed)
        yy, xx = np.mgrid[0:w.height, 0:w.width]
        rgb, used, bufs = rs.render_pixels(p, xx.ravel(), yy.ravel(), ad, nfor)
        out = {"rgb": rgb.reshape(w.height, w.width, 3), "used": used.reshape(w.height, w.width)}
        for k, v in (bufs or {}).items():
            out[k] = v.reshape((w.height, w.width) + v.shape[1:])
        np.savez_compressed(os.path.join(HERE, f"adaptive_{name}.npz"), **out)
        print("golden", name, flush=True)


def adjoint_fixture(o, h=0.05):
    w, adj, picks = adjoint_case()
    tex0 = np.array(w.scene.textures[0])
    p = native.params(w.width, w.height, w.spp, w.max_bounces, w.seed)
    yy, xx = np.mgrid[0:w.height, 0:w.width]
    S = w.spp
    x = np.repeat(xx.ravel(), S)
    y = np.repeat(yy.ravel(), S)
    s = np.tile(np.arange(S), w.width * w.height)

    def loss(tex):
        w.scene.textures[0] = tex
        rs = o.scene(w.scene.build())
        c = rs.trace_paths(p, x, y, s)
        c = np.where(np.isfinite(c), c, 0.0).reshape(w.height, w.width, S, 3).mean(axis=2)
        return float((adj.astype(np.float64) * c).sum())

    fd = []
    for ty, tx, ch in picks:
        tp, tm = tex0.copy(), tex0.copy()
        tp[ty, tx, ch] += h
        tm[ty, tx, ch] -= h
        fd.append((loss(tp) - loss(tm)) / (2.0 * h))
    w.scene.textures[0] = tex0
    np.savez_compressed(os.path.join(HERE, "adjoint_cornell.npz"), adj=adj, texture=tex0, picks=picks,
                        fd=np.array(fd), h=h)
    print("golden adjoint_cornell", flush=True)


def sha256(*arrays) -> str:
    import hashlib
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def ray_fixture(rt, w, name, rng, n=2000):
    """Rays, volume keys, the reference's closest / any hits and ambiguity flags."""
    rays = camera_rays(w, n, seed=len(name))
    vkey = np.stack([rng.integers(0, w.width, n), rng.integers(0, w.height, n),
                     rng.integers(0, w.spp, n), rng.integers(0, 4, n)], 1).astype(np.int32)
    r64 = rays.astype(np.float64)
    t, ob, pr = rt.trace_rays(r64, seed=w.seed, volume_key=vkey)
    _, occ, _ = rt.trace_rays(r64, any_hit=True, seed=w.seed, volume_key=vkey)
    amb = O.ambiguous_rays(rt, r64, ob, pr, seed=w.seed, volume_key=vkey)
    amb_any = np.zeros(n, bool)
    for k in O.RAY_PROBES:
        _, o2, _ = rt.trace_rays(O.perturbed_rays(r64, k), any_hit=True, seed=w.seed, volume_key=vkey)
        amb_any |= o2 != occ
    return dict(rays=rays, vkey=vkey, t=t, obj=ob, prim=pr, occluded=occ >= 0, ambiguous=amb,
                ambiguous_any=amb_any)


def path_fixture(o, rs, w, x, y, s):
    """Per-path radiance with its ambiguity flags; for a scene with a caustic photon map
    also `photon`: paths whose radiance changes when the map is switched off (they
    gather photons, whose FP32 tracing test_caustics compares on its own)."""
    p = native.params(w.width, w.height, w.spp, w.max_bounces, w.seed)
    rgb = rs.trace_paths(p, x, y, s)
    amb = O.ambiguous_paths(o, rs, p, x, y, s, rgb, O.path_deltas(w.width, w.height, w.scene.camera),
                            scene=w.scene)
    out = dict(x=x, y=y, s=s, rgb=rgb, ambiguous=amb)
    if w.scene.caustics.get("enabled"):
        import copy
        sc = copy.deepcopy(w.scene)
        sc.caustics["enabled"] = 0
        off = o.scene(sc.build()).trace_paths(p, x, y, s)
        out["photon"] = np.abs(off - rgb).max(axis=1) > 0
    return out


def full_fixtures(o, only=None):
    """full_<case>.npz for FULL_CASES."""
    for name, fn in FULL_CASES.items():
        if only and name not in only:
            continue
        rng = np.random.default_rng(zlib.crc32(name.encode()))
        w = fn()
        b = w.scene.build()
        rs = o.scene(b)
        out = {}
        for mi in range(len(w.scene.meshes)):
            nodes, order = rs.mesh_bvh(mi)
            out[f"mesh{mi}_sha256"] = sha256(nodes, order)
            out[f"mesh{mi}_nodes"] = len(nodes)
            out[f"mesh{mi}_head"] = nodes[:64]
        top = O.top_tree_from_reference(rs.top_bvh())
        out["top_sha256"] = sha256(top)
        out["top_len"] = len(top)
        out["top_head"] = top[:4096]
        rt = o.scene(b, tag=True)
        for k, v in ray_fixture(rt, w, name, rng).items():
            out["hit_" + k] = v
        rt.close()
        x, y, s = path_keys(w, 4096, seed=7 + len(name))
        p = native.params(w.width, w.height, w.spp, w.max_bounces, w.seed)
        lit = rs.trace_paths(p, x, y, s).max(axis=1) > 0
        if lit.mean() < 0.25:
            # a mostly dark frame (the 1e5-instance box is opaque a few units into it):
            # add the lit paths among 2^21 seeded candidates, up to 1,024 of them
            cx, cy, cs = path_keys(w, 1 << 21, seed=8 + len(name))
            nz = np.flatnonzero(rs.trace_paths(p, cx, cy, cs).max(axis=1) > 0)[:1024]
            x, y, s = np.concatenate([x, cx[nz]]), np.concatenate([y, cy[nz]]), np.concatenate([s, cs[nz]])
        for k, v in path_fixture(o, rs, w, x, y, s).items():
            out["path_" + k] = v
        np.savez_compressed(os.path.join(HERE, f"full_{name}.npz"), **out)
        print("golden", name, "ambiguous rays %.4f paths %.4f" % (out["hit_ambiguous"].mean(),
                                                                  out["path_ambiguous"].mean()), flush=True)


def case_fixtures(o, only=None):
    """hits_/paths_/image_<case>.npz; each case draws from its own seeded generator."""
    for name, fn in CASES.items():
        if only is not None and name not in only:
            continue
        rng = np.random.default_rng(zlib.crc32(name.encode()))
        w = fn()
        b = w.scene.build()
        rs = o.scene(b)
        rt = o.scene(b, tag=True)
        hits = ray_fixture(rt, w, name, rng)
        hits["top"] = O.top_tree_from_reference(rs.top_bvh())
        np.savez_compressed(os.path.join(HERE, f"hits_{name}.npz"), **hits)
        x, y, s = path_keys(w, 1500, seed=7 + len(name))
        np.savez_compressed(os.path.join(HERE, f"paths_{name}.npz"), **path_fixture(o, rs, w, x, y, s))
        p = native.params(w.width, w.height, w.spp, w.max_bounces, w.seed)
        if name in ("cornell", "tiny"):
            img, _, _ = rs.render(p, os.cpu_count() or 1)
            np.savez_compressed(os.path.join(HERE, f"image_{name}.npz"), rgb=img, spp=w.spp)
        print("golden", name, flush=True)


NFOR_KEYS = ("color_a", "color_b", "color_variance", "features_a", "features_b", "feature_variance")


def nfor_fixture(o):
    """nfor.npz: Denoise::applyNFOR outputs for the NFOR buffers of the adaptive fixtures and of
    cases.nfor_synthetic() (default settings)."""
    out = {}
    for name in ("tiny_nfor", "tiny_adaptive_nfor"):
        g = np.load(os.path.join(HERE, f"adaptive_{name}.npz"))
        out[name] = o.nfor({k: g[k] for k in NFOR_KEYS})
    out["synthetic"] = o.nfor(nfor_synthetic())
    out["synthetic_r3"] = o.nfor(nfor_synthetic(), prefilter_radius=2, regression_radius=3, patch_radius=2)
    np.savez_compressed(os.path.join(HERE, "nfor.npz"), **out)
    print("golden nfor", flush=True)


def caustic_fixture(o, n_paths=2000):
    """caustics.npz: photons stored for CAUSTIC_COUNTS (seed, max_bounces) pairs, and the
    reference radiance of up to n_paths one-sample paths whose value changes when the
    photon map is switched off (paths that gather caustic photons)."""
    w = caustic_case()
    rs = o.scene(w.scene.build())
    counts = np.array([rs.caustic_photons(sd, mb) for sd, mb in CAUSTIC_COUNTS], np.int64)
    p = native.params(w.width, w.height, w.spp, w.max_bounces, w.seed)
    yy, xx = np.mgrid[0:w.height, 0:w.width]
    x = np.repeat(xx.ravel(), w.spp).astype(np.int32)
    y = np.repeat(yy.ravel(), w.spp).astype(np.int32)
    s = np.tile(np.arange(w.spp), w.width * w.height).astype(np.int32)
    on = rs.trace_paths(p, x, y, s)
    w.scene.caustics["enabled"] = 0
    off = o.scene(w.scene.build()).trace_paths(p, x, y, s)
    sel = np.flatnonzero(np.abs(on - off).max(axis=1) > 0)
    rng = np.random.default_rng(zlib.crc32(b"caustics"))
    sel = np.sort(rng.choice(sel, min(n_paths, sel.size), replace=False))
    np.savez_compressed(os.path.join(HERE, "caustics.npz"), counts=counts, x=x[sel], y=y[sel], s=s[sel],
                        rgb=on[sel], rgb_off=off[sel])
    print("golden caustics", counts, sel.size, flush=True)


def oracle64k_fixtures(o):
    """oracle64k_<case>.npz: the reference's own film at 65,536 spp (all host threads)."""
    for name, fn in ORACLE_64K.items():
        w = fn()
        rs = o.scene(w.scene.build())
        img, ms, _ = rs.render(native.params(w.width, w.height, w.spp, w.max_bounces, w.seed), os.cpu_count() or 1)
        np.savez_compressed(os.path.join(HERE, f"oracle64k_{name}.npz"), rgb=img, spp=w.spp, seed=w.seed)
        print("golden oracle64k", name, f"{ms / 1000:.1f} s", flush=True)


def oracle64k_full_fixtures(o, threads=None):
    """oracle64k_<case>.npz for the full-size frames of ORACLE_64K_FULL (FP32 film: the
    oracle's own Monte Carlo noise at 65,536 spp is far above FP32 rounding)."""
    threads = threads or os.cpu_count() or 1
    for name, fn in ORACLE_64K_FULL.items():
        w = fn()
        rs = o.scene(w.scene.build())
        img, ms, _ = rs.render(native.params(w.width, w.height, w.spp, w.max_bounces, w.seed), threads)
        np.savez_compressed(os.path.join(HERE, f"oracle64k_{name}.npz"), rgb=img.astype(np.float32), spp=w.spp,
                            seed=w.seed, render_ms=ms, threads=threads)
        print("golden oracle64k", name, f"{ms / 1000:.1f} s", flush=True)


def oracle64k_subset_fixtures(o, threads=None, only=None):
    """oracle64k_<case>.npz for ORACLE_64K_SUBSET: the reference's pixel means at 65,536 spp
    on a seeded 4,096-pixel subset of the frame (_threadRender per pixel, host threads)."""
    import time
    threads = threads or os.cpu_count() or 1
    for name, fn in ORACLE_64K_SUBSET.items():
        if only and name not in only:
            continue
        w = fn()
        x, y = oracle_subset_pixels(w)
        rs = o.scene(w.scene.build())
        t0 = time.time()
        rgb = rs.render_pixels_mt(native.params(w.width, w.height, w.spp, w.max_bounces, w.seed), x, y, threads)
        np.savez_compressed(os.path.join(HERE, f"oracle64k_{name}.npz"), x=x, y=y, rgb=rgb.astype(np.float32),
                            spp=w.spp, seed=w.seed, seconds=time.time() - t0, threads=threads)
        print("golden oracle64k subset", name, f"{time.time() - t0:.0f} s", flush=True)


def adjoint_c3_fixture(o, threads=None, only=None):
    """adjoint_c3.npz: central differences of the reference's film functional
    L = sum(adj * film) at the C3 configuration (cases.c3_case), Renderer::render with
    common random numbers (one seed for both sides): 65,536 spp for the albedo (all
    back-wall texels scaled by 1 +- h) and for the density of the fog cube (c3_fog_case,
    density scaled by 1 +- h); 1,024 spp for the emission (the film is linear in it, and
    light selection does not depend on it with one light)."""
    threads = threads or os.cpu_count() or 1
    path = os.path.join(HERE, "adjoint_c3.npz")
    out = dict(np.load(path)) if os.path.exists(path) else {}
    w, adj = c3_case()
    out["adj"] = adj
    out["h"] = C3_H
    seed = 20261204
    out["seed"] = seed
    a64 = adj.astype(np.float64)

    def loss(workload, spp):
        rs = o.scene(workload.scene.build())
        img, ms, _ = rs.render(native.params(workload.width, workload.height, spp, workload.max_bounces, seed),
                               threads)
        rs.close()
        return float((a64 * img).sum()), ms

    jobs = [("albedo", C3_SPP_FD), ("emission", 1024), ("density", C3_SPP_FD)]
    for name, spp in jobs:
        if only and name not in only:
            continue
        vals = []
        for sgn in (1.0, -1.0):
            if name == "density":
                wk, obj = c3_fog_case(spp)
                wk.scene.objects[obj]["density"] *= 1.0 + sgn * C3_H
            else:
                wk, _ = c3_case()
                wk.spp = spp
                if name == "albedo":
                    wk.scene.textures[0] = wk.scene.textures[0] * (1.0 + sgn * C3_H)
                else:
                    light = [m for m in wk.scene.materials if m["type"] == 4][0]
                    light["color"] = tuple(np.array(light["color"]) * (1.0 + sgn * C3_H))
            v, ms = loss(wk, spp)
            vals.append(v)
            print("adjoint_c3", name, sgn, v, f"{ms / 1000:.0f} s", flush=True)
        out[f"fd_{name}"] = (vals[0] - vals[1]) / (2.0 * C3_H)
        out[f"spp_{name}"] = spp
        np.savez_compressed(path, **out)


def main():
    o = RefOracle()
    if sys.argv[1:] == ["adaptive"]:
        adaptive_fixtures(o)
        return
    if sys.argv[1:] == ["adjoint"]:
        adjoint_fixture(o)
        return
    if sys.argv[1:] == ["nfor"]:
        nfor_fixture(o)
        return
    if sys.argv[1:] == ["caustics"]:
        caustic_fixture(o)
        return
    if sys.argv[1:] == ["oracle64k"]:
        oracle64k_fixtures(o)
        return
    if sys.argv[1:2] == ["oracle64k_subset"]:
        oracle64k_subset_fixtures(o, only=sys.argv[2:] or None)
        return
    if sys.argv[1:2] == ["adjoint_c3"]:    # adjoint_c3 [albedo|emission|density ...]
        adjoint_c3_fixture(o, only=sys.argv[2:] or None)
        return
    if sys.argv[1:2] == ["full"]:      # full [name...]: the full-size frames
        full_fixtures(o, sys.argv[2:])
        return
    if sys.argv[1:2] == ["oracle64k_full"]:
        oracle64k_full_fixtures(o, int(sys.argv[2]) if len(sys.argv) > 2 else None)
        return
    if sys.argv[1:2] == ["cases"]:     # cases <name>...: only the per-case files of those cases
        case_fixtures(o, sys.argv[2:] or None)
        return
    rng = np.random.default_rng(20261203)
    n = 600
    keys = np.stack([rng.integers(0, 2**32, n), rng.integers(0, 4096, n), rng.integers(0, 4096, n),
                     rng.integers(0, 70000, n), rng.integers(0, 3, n), rng.integers(0, 20, n),
                     rng.integers(0, 20, n)], 1).astype(np.int64)
    s1 = np.array([o.sampler(*map(int, k), 1) for k in keys])
    s2 = np.array([o.sampler(*map(int, k), 2) for k in keys], np.float64).astype(np.float32)
    np.savez_compressed(os.path.join(HERE, "sampler.npz"), keys=keys, s1=s1, s2=s2)

    for name, fn in BVH_CASES.items():
        sc = fn()
        rs = o.scene(sc.build())
        out = {}
        for mi in range(len(sc.meshes)):
            nodes, order = rs.mesh_bvh(mi)
            out[f"nodes{mi}"] = nodes
            out[f"order{mi}"] = order
        np.savez_compressed(os.path.join(HERE, f"bvh_{name}.npz"), **out)

    case_fixtures(o)
    adaptive_fixtures(o)
    adjoint_fixture(o)
    nfor_fixture(o)
    caustic_fixture(o)
    oracle64k_fixtures(o)


if __name__ == "__main__":
    main()
