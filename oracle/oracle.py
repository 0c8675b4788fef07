"""TEST INFRASTRUCTURE ONLY — ctypes access to the oracle libraries.

  oracle/_ref/libluzref.so       the Luz reference itself (built by oracle/Makefile
                                 from the reference sources, -O2, no fast-math)
  oracle/_ref/libluzref_fast.so  same sources with release flags (timed CPU baseline)
  oracle/_ref/librestate.so      oracle/restate.cpp, the FP32 restatement of the
                                 sampler and the BVH traversal

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this
module, as the checker. The product (luz_b200) never does.
"""
from __future__ import annotations

import contextlib
import ctypes as C
import os
import sys
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")


def _path(name: str) -> str:
    return os.path.join(REF_DIR, name)


@contextlib.contextmanager
def stdout_to_stderr():
    """The reference's renderer prints its render statistics on stdout (std::cout); a
    caller whose stdout carries machine-read output moves them to stderr."""
    sys.stdout.flush()
    saved = os.dup(1)
    os.dup2(2, 1)
    try:
        yield
    finally:
        C.CDLL(None).fflush(None)
        os.dup2(saved, 1)
        os.close(saved)


def reference_available(fast: bool = False) -> bool:
    return os.path.exists(_path("libluzref_fast.so" if fast else "libluzref.so"))


def restate_available() -> bool:
    return os.path.exists(_path("librestate.so"))


class RefOracle:
    """The reference renderer behind the harness in oracle/ref_harness.cpp."""

    def __init__(self, fast: bool = False):
        self.lib = C.CDLL(_path("libluzref_fast.so" if fast else "libluzref.so"))
        L = self.lib
        vp = C.c_void_p
        L.luzref_scene_create.argtypes = [vp, C.c_int32, C.POINTER(vp)]
        L.luzref_scene_destroy.argtypes = [vp]
        L.luzref_trace_rays.argtypes = [vp, vp, C.c_int64, C.c_int32, C.c_uint32, vp, vp, vp, vp]
        L.luzref_trace_paths.argtypes = [vp, vp, vp, vp, vp, C.c_int64, vp]
        L.luzref_render.argtypes = [vp, vp, C.c_int32, vp, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.luzref_nfor.argtypes = [C.c_int32, C.c_int32, vp, vp, vp, vp, vp, vp, C.c_int32, C.c_int32, C.c_int32,
                                  C.c_double, C.c_int32, vp]
        L.luzref_trace_samples.argtypes = [vp, vp, C.c_int32, vp, vp, vp, C.c_int64, vp, vp]
        L.luzref_render_pixels.argtypes = [vp, vp, C.c_int32, C.c_int32, C.c_int32, C.c_double, C.c_int32, vp, vp,
                                           C.c_int64, vp, vp, vp]
        L.luzref_mesh_bvh.argtypes = [vp, C.c_int32, vp, C.c_int64, C.POINTER(C.c_int64), vp, C.c_int64]
        L.luzref_mesh_triangle_count.argtypes = [vp, C.c_int32, C.POINTER(C.c_int64)]
        L.luzref_caustic_photons.argtypes = [vp, C.c_uint32, C.c_int32, C.POINTER(C.c_int64)]
        L.luzref_sampler.argtypes = [C.c_uint32, C.c_int32, C.c_int32, C.c_int32, C.c_uint32, C.c_uint32,
                                     C.c_uint32, C.c_int32, vp]
        L.luzref_last_error.argtypes = [C.c_char_p, C.c_size_t]
        L.luzref_scene_load.argtypes = [C.c_char_p, C.POINTER(vp)]
        L.luzref_scene_pack.argtypes = [vp, C.POINTER(vp), vp]
        L.luzref_set_perturbation.argtypes = [C.c_uint64, C.c_double, C.c_double, C.c_double, C.c_double]
        L.luzref_top_bvh.argtypes = [vp, vp, C.c_int64, C.POINTER(C.c_int64)]
        L.luzref_render_pixels_mt.argtypes = [vp, vp, vp, vp, C.c_int64, C.c_int32, vp]

    def _check(self, rc):
        if rc != 0:
            buf = C.create_string_buffer(512)
            self.lib.luzref_last_error(buf, 512)
            raise RuntimeError("reference oracle: " + buf.value.decode())

    def scene(self, built, tag: bool = False) -> "RefScene":
        h = C.c_void_p()
        self._check(self.lib.luzref_scene_create(C.cast(built.ptr(), C.c_void_p), 1 if tag else 0, C.byref(h)))
        return RefScene(self, h, built)

    def load_luz(self, path: str) -> "RefScene":
        """A scene read from a .luz file by the reference's own parser (SceneFile::read)."""
        h = C.c_void_p()
        with stdout_to_stderr():
            rc = self.lib.luzref_scene_load(os.fsencode(path), C.byref(h))
        self._check(rc)
        return RefScene(self, h, None)

    def nfor(self, bufs: dict, prefilter_radius=1, regression_radius=2, patch_radius=1, min_variance=1e-5,
             threads=1):
        """Denoise::applyNFOR on NFOR buffers (dict of H x W x k arrays); returns H x W x 3."""
        h, w = bufs["color_variance"].shape[:2]
        a = {k: np.ascontiguousarray(v, np.float64) for k, v in bufs.items()}
        out = np.zeros((h, w, 3), np.float64)
        self._check(self.lib.luzref_nfor(w, h, a["color_a"].ctypes.data, a["color_b"].ctypes.data,
                                         a["color_variance"].ctypes.data, a["features_a"].ctypes.data,
                                         a["features_b"].ctypes.data, a["feature_variance"].ctypes.data,
                                         prefilter_radius, regression_radius, patch_radius, min_variance, threads,
                                         out.ctypes.data))
        return out

    def set_perturbation(self, seed: int, delta_dir: float = 0.0, delta_dec: float = 0.0, delta_cam: float = 0.0,
                         delta_bsdf: float = 0.0):
        """Moves every Sampler draw by +-delta while seed != 0 (the FP32 ambiguity probe,
        oracle/ref_harness.cpp); seed 0 turns it off."""
        self._check(self.lib.luzref_set_perturbation(int(seed), float(delta_dir), float(delta_dec), float(delta_cam),
                                                     float(delta_bsdf)))

    def sampler(self, seed, x, y, s, stream, bounce, dim, which=1):
        out = np.zeros(2, np.float64)
        self.lib.luzref_sampler(seed, x, y, s, stream, bounce, dim, which, out.ctypes.data)
        return out[0] if which == 1 else (out[0], out[1])


class PackedDesc:
    """A LuzSceneDesc owned by a reference scene (valid while that scene lives and
    is not packed again); .ptr() is what luz_gpu_scene_create and
    luzref_scene_create take, as for the Python-built descriptions."""

    def __init__(self, owner: "RefScene", address: int, width: int, height: int, spp: int, max_bounces: int):
        self.owner, self.address = owner, address
        self.width, self.height, self.spp, self.max_bounces = width, height, spp, max_bounces

    def ptr(self) -> int:
        return self.address


class RefScene:
    def __init__(self, oracle: RefOracle, handle, built):
        self.o, self.h, self.built = oracle, handle, built

    def close(self):
        if self.h:
            self.o.lib.luzref_scene_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def trace_rays(self, rays: np.ndarray, any_hit=False, seed=0, volume_key: Optional[np.ndarray] = None):
        rays = np.ascontiguousarray(rays, dtype=np.float64)
        n = rays.shape[0]
        t = np.zeros(n, np.float64)
        obj = np.zeros(n, np.int32)
        prim = np.zeros(n, np.int32)
        vk = None if volume_key is None else np.ascontiguousarray(volume_key, dtype=np.int32)
        self.o._check(self.o.lib.luzref_trace_rays(self.h, rays.ctypes.data, n, 1 if any_hit else 0, seed,
                                                   None if vk is None else vk.ctypes.data,
                                                   t.ctypes.data, obj.ctypes.data, prim.ctypes.data))
        return t, obj, prim

    def render_pixels_mt(self, params, x, y, threads: int) -> np.ndarray:
        """_threadRender for listed pixels on `threads` host threads: n x 3 pixel means."""
        x = np.ascontiguousarray(x, np.int32)
        y = np.ascontiguousarray(y, np.int32)
        out = np.zeros((len(x), 3), np.float64)
        self.o._check(self.o.lib.luzref_render_pixels_mt(self.h, C.byref(params), x.ctypes.data, y.ctypes.data,
                                                         len(x), int(threads), out.ctypes.data))
        return out

    def top_bvh(self) -> np.ndarray:
        """The reference's top-level BVHNode tree in preorder: per node its child count,
        then per child (is_node, object, min xyz, max xyz)."""
        n = C.c_int64(0)
        self.o._check(self.o.lib.luzref_top_bvh(self.h, None, 0, C.byref(n)))
        out = np.zeros(n.value, np.float64)
        self.o._check(self.o.lib.luzref_top_bvh(self.h, out.ctypes.data, n.value, C.byref(n)))
        return out

    def pack(self) -> "PackedDesc":
        """The scene glue (luz_b200/glue/scene_glue.cpp) applied to this scene."""
        d = C.c_void_p()
        st = np.zeros(4, np.int32)
        self.o._check(self.o.lib.luzref_scene_pack(self.h, C.byref(d), st.ctypes.data))
        return PackedDesc(self, d.value, *[int(v) for v in st])

    def caustic_photons(self, seed: int, max_bounces: int) -> int:
        """CausticPhotonMap::build for the render seed: photons stored."""
        n = C.c_int64()
        self.o._check(self.o.lib.luzref_caustic_photons(self.h, seed, max_bounces, C.byref(n)))
        return n.value

    def trace_paths(self, params, x, y, s) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.int32)
        y = np.ascontiguousarray(y, dtype=np.int32)
        s = np.ascontiguousarray(s, dtype=np.int32)
        out = np.zeros((x.shape[0], 3), np.float64)
        self.o._check(self.o.lib.luzref_trace_paths(self.h, C.addressof(params), x.ctypes.data, y.ctypes.data,
                                                    s.ctypes.data, x.shape[0], out.ctypes.data))
        return out

    def render(self, params, threads: int):
        out = np.zeros((params.height, params.width, 3), np.float64)
        ms = C.c_double()
        ns = C.c_double()
        with stdout_to_stderr():
            rc = self.o.lib.luzref_render(self.h, C.addressof(params), threads, out.ctypes.data, C.byref(ms),
                                          C.byref(ns))
        self.o._check(rc)
        return out, ms.value, ns.value

    def trace_samples(self, params, x, y, s, half_streams=False):
        """Per-sample colour (before cleanColor) and primary features (_calculatePixelSample)."""
        x = np.ascontiguousarray(x, dtype=np.int32)
        y = np.ascontiguousarray(y, dtype=np.int32)
        s = np.ascontiguousarray(s, dtype=np.int32)
        rgb = np.zeros((x.shape[0], 3), np.float64)
        feat = np.zeros((x.shape[0], 11), np.float64)
        self.o._check(self.o.lib.luzref_trace_samples(self.h, C.addressof(params), 1 if half_streams else 0,
                                                      x.ctypes.data, y.ctypes.data, s.ctypes.data, x.shape[0],
                                                      rgb.ctypes.data, feat.ctypes.data))
        return rgb, feat

    def render_pixels(self, params, x, y, adaptive=None, nfor=False):
        """_threadRender for the listed pixels (Threads.cpp:551-641). adaptive: None or a dict
        with min_samples, check_interval, threshold. Returns rgb (n,3), samples used (n,) and,
        with nfor, a dict of the NFORBuffers entries of each pixel."""
        x = np.ascontiguousarray(x, dtype=np.int32)
        y = np.ascontiguousarray(y, dtype=np.int32)
        n = x.shape[0]
        rgb = np.zeros((n, 3), np.float64)
        used = np.zeros(n, np.int32)
        nf = np.zeros((n, 40), np.float64)
        a = adaptive or {}
        self.o._check(self.o.lib.luzref_render_pixels(
            self.h, C.addressof(params), 1 if adaptive else 0, int(a.get("min_samples", 1)),
            int(a.get("check_interval", 1)), float(a.get("threshold", 1.0)), 1 if nfor else 0, x.ctypes.data,
            y.ctypes.data, n, rgb.ctypes.data, used.ctypes.data, nf.ctypes.data if nfor else None))
        bufs = None
        if nfor:
            bufs = {"color_a": nf[:, 0:3], "color_b": nf[:, 3:6], "color_variance": nf[:, 6],
                    "features_a": nf[:, 7:18], "features_b": nf[:, 18:29], "feature_variance": nf[:, 29:40]}
        return rgb, used, bufs

    def mesh_bvh(self, mesh: int):
        from luz_b200.desc import NODE64_DTYPE
        nt = C.c_int64()
        self.o._check(self.o.lib.luzref_mesh_triangle_count(self.h, mesh, C.byref(nt)))
        cap = max(1, 2 * nt.value)
        nodes = np.zeros(cap, NODE64_DTYPE)
        order = np.zeros(max(1, nt.value), np.int64)
        cnt = C.c_int64()
        self.o._check(self.o.lib.luzref_mesh_bvh(self.h, mesh, nodes.ctypes.data, cap, C.byref(cnt),
                                                 order.ctypes.data, order.shape[0]))
        return nodes[:cnt.value], order[:nt.value]


class Restate:
    """oracle/restate.cpp: FP32 restatement of the sampler and the traversal."""

    def __init__(self):
        self.lib = C.CDLL(_path("librestate.so"))
        vp = C.c_void_p
        self.lib.restate_sample1d.argtypes = [C.c_uint32, C.c_int32, C.c_int32, C.c_int32, C.c_uint32, C.c_uint32,
                                              C.c_uint32, vp]
        self.lib.restate_sample2d.argtypes = self.lib.restate_sample1d.argtypes
        self.lib.restate_trace.argtypes = [vp] * 9 + [vp, C.c_int64, C.c_int32, C.c_uint32, vp, vp]

    def sample1d(self, seed, x, y, s, stream, bounce, dim):
        out = np.zeros(1, np.float64)
        self.lib.restate_sample1d(seed, x, y, s, stream, bounce, dim, out.ctypes.data)
        return out[0]

    def sample2d(self, seed, x, y, s, stream, bounce, dim):
        out = np.zeros(2, np.float32)
        self.lib.restate_sample2d(seed, x, y, s, stream, bounce, dim, out.ctypes.data)
        return out

    def trace(self, pack, rays: np.ndarray, any_hit=False, seed=0, volume_key=None):
        """Traverses the packed arrays of a luz_b200.native.Pack on the CPU."""
        from luz_b200.desc import HIT_DTYPE
        names = ["top_nodes", "top_children", "objects", "mesh_nodes", "mesh_tris", "meshes", "rects", "index_pool",
                 "consts"]
        arrs = [np.ascontiguousarray(pack.array(n)) for n in names]
        ptrs = [a.ctypes.data if a.size else None for a in arrs]
        rays = np.ascontiguousarray(rays, np.float32)
        out = np.zeros(rays.shape[0], HIT_DTYPE)
        vk = None if volume_key is None else np.ascontiguousarray(volume_key, np.int32)
        self.lib.restate_trace(*ptrs, rays.ctypes.data, rays.shape[0], 1 if any_hit else 0, seed,
                               None if vk is None else vk.ctypes.data, out.ctypes.data)
        return out


# ---------------------------------------------------------------------------- FP32 ambiguity flags
#
# The GPU computes in FP32 what the reference computes in FP64. Where a result
# depends on its inputs more finely than FP32 resolves (a draw within FP32
# rounding of a lobe, Russian-roulette or light-selection threshold, a ray
# grazing a triangle edge, a very sharp lobe), the two may legitimately part.
# These probes mark such rays and paths from the reference alone, before any GPU
# result is seen: a ray or path is ambiguous when the reference's own answer
# changes under perturbations of the size of FP32 rounding: of the draws (a few
# FP32 ulps of what they become) and of the geometry (its FP32 storage).

# Draw perturbations (in units of the draw u in [0, 1)): 2^-21 for draws that
# become directions or distances (FP32 directions are good to ~1e-7), 2^-16 for
# draws compared with a threshold the GPU computes in FP32 from a long product of
# FP32 factors (throughput for Russian roulette, Fresnel and lobe weights), and
# for the camera and lens draws twice the FP32 rounding of the camera ray in
# pixels or aperture widths (path_deltas). Draws compared with FP64 values both sides share bit for bit (strategy
# probabilities, light / triangle / environment selection CDFs) are not moved.
def path_deltas(width: int, height: int, camera) -> dict:
    """Draw perturbations for a frame. The GPU rounds each FP64 camera ray to FP32:
    the direction by at most 2^-25 per component, the origin by half an FP32 ulp of
    its largest coordinate. The camera draw moves the ray by twice the former, in
    pixels (one pixel spans ~sensor_height / focal / height rad); the lens draw moves
    the origin by twice the latter, in units of the aperture diameter."""
    cam = 2.0 * 2.0 ** -25 * height * camera.focal_length_m / camera.sensor_height_m
    if not camera.pinhole and camera.f_number > 0:
        radius = camera.focal_length_m / (2.0 * camera.f_number)
        omax = max(1.0, max(abs(float(camera.position[i])) for i in range(3)))
        half_ulp = float(np.spacing(np.float32(omax))) / 2.0
        cam = max(cam, 2.0 * half_ulp / (2.0 * radius))
    return dict(delta_dir=2.0 ** -21, delta_dec=2.0 ** -16, delta_cam=min(cam, 2.0 ** -8), delta_bsdf=2.0 ** -21)


PATH_PROBES = (1, 2, 3)
# Ray perturbations: every origin coordinate by +-2^-20 of max(|o|, 1), every
# direction component by +-2^-20 (renormalised).
RAY_DELTA = 2.0 ** -20
RAY_PROBES = (11, 12, 13)


def path_rel(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Per-path relative difference as the parity tests measure it: max over channels
    of |a - b| / max(|b|, 1e-3); non-finite values count as different."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    r = np.abs(a - b) / np.maximum(np.abs(b), 1e-3)
    r = np.where(np.isfinite(r), r, np.inf)
    return r.max(axis=1)


def perturbed_geometry(scene, seed: int):
    """A copy of a luz_b200.desc.Scene whose geometry carries the GPU's FP32 storage error:
    every triangle translated rigidly by the FP32 rounding of its first vertex (the GPU keeps
    v0 in FP32 and the edges, formed in FP64, in FP32: a triangle moves as a whole), vertex
    normals and object parameters (centres, sizes, orientations) rounded to FP32; seeds other
    than 0 add a further +-1 FP32 ulp (relative 2^-24) of random sign. The camera is left
    alone: the GPU forms camera rays in FP64 (the camera draws carry that rounding)."""
    import copy
    sc = copy.deepcopy(scene)
    rng = np.random.default_rng(seed)

    def jitter(v):
        v = np.asarray(v, np.float64)
        return 0.0 if seed == 0 else rng.choice([-1.0, 1.0], v.shape) * 2.0 ** -24 * np.abs(v)

    def rounded(v):
        v = np.asarray(v, np.float64)
        return v.astype(np.float32).astype(np.float64) + jitter(v)

    for m in sc.meshes:
        tri = np.asarray(m["positions"], np.float64).reshape(-1, 3, 3)
        v0 = tri[:, 0, :]
        shift = v0.astype(np.float32).astype(np.float64) - v0 + jitter(v0)
        m["positions"] = np.ascontiguousarray((tri + shift[:, None, :]).reshape(-1, 9))
        if m["normals"] is not None:
            m["normals"] = np.ascontiguousarray(rounded(m["normals"]))
    for ob in sc.objects:
        for k in ("position", "size", "orientation", "width_axis", "height_axis"):
            ob[k] = tuple(rounded(ob[k]))
    return sc


GEOMETRY_PROBES = (0, 1, 2)


def ambiguous_paths(oracle: RefOracle, rs: "RefScene", params, x, y, s, base: np.ndarray, deltas: dict,
                    tol: float = 1e-4, scene=None):
    """True per path whose reference radiance moves by more than tol under any of the
    PATH_PROBES draw perturbations (deltas: path_deltas of the frame) or, when the
    luz_b200.desc.Scene is given, under any of the GEOMETRY_PROBES (perturbed_geometry)."""
    flags = np.zeros(len(x), bool)
    try:
        for seed in PATH_PROBES:
            oracle.set_perturbation(seed, **deltas)
            flags |= path_rel(rs.trace_paths(params, x, y, s), base) > tol
    finally:
        oracle.set_perturbation(0)
    if scene is not None:
        for seed in GEOMETRY_PROBES:
            rg = oracle.scene(perturbed_geometry(scene, seed).build())
            flags |= path_rel(rg.trace_paths(params, x, y, s), base) > tol
            rg.close()
    return flags


def perturbed_rays(rays: np.ndarray, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    r = np.array(rays, np.float64)
    o = r[:, 0:3]
    r[:, 0:3] = o + rng.choice([-1.0, 1.0], o.shape) * RAY_DELTA * np.maximum(np.abs(o), 1.0)
    d = r[:, 4:7] + rng.choice([-1.0, 1.0], (len(r), 3)) * RAY_DELTA
    r[:, 4:7] = d / np.linalg.norm(d, axis=1, keepdims=True)
    return r


def ambiguous_rays(rs_tagged: "RefScene", rays: np.ndarray, obj: np.ndarray, prim: np.ndarray, seed: int = 0,
                   volume_key=None):
    """True per ray whose reference closest hit (object, primitive) changes under any of
    the RAY_PROBES perturbations (edge grazes and near ties in t)."""
    flags = np.zeros(len(rays), bool)
    for k in RAY_PROBES:
        _, o2, p2 = rs_tagged.trace_rays(perturbed_rays(rays, k), seed=seed, volume_key=volume_key)
        flags |= (o2 != obj) | (p2 != prim)
    return flags


# ---------------------------------------------------------------------------- top-level BVH layout

def _round_out(lo: np.ndarray, hi: np.ndarray):
    """FP64 box bounds rounded outward to FP32 (the nearest float at or below the
    minimum, at or above the maximum), as float64 values."""
    f_lo = lo.astype(np.float32)
    f_lo = np.where(f_lo.astype(np.float64) > lo, np.nextafter(f_lo, np.float32(-np.inf)), f_lo)
    f_hi = hi.astype(np.float32)
    f_hi = np.where(f_hi.astype(np.float64) < hi, np.nextafter(f_hi, np.float32(np.inf)), f_hi)
    return f_lo.astype(np.float64), f_hi.astype(np.float64)


def top_tree_from_reference(dump: np.ndarray) -> np.ndarray:
    """RefScene.top_bvh() with every child box rounded outward to FP32: the form the
    GPU's top-level arrays take (node preorder, children in the reference's order)."""
    out = np.array(dump, np.float64)
    i = 0
    while i < len(out):
        n = int(out[i])
        rec = out[i + 1:i + 1 + 8 * n].reshape(n, 8)
        rec[:, 2:5], rec[:, 5:8] = _round_out(rec[:, 2:5].copy(), rec[:, 5:8].copy())
        out[i + 1:i + 1 + 8 * n] = rec.ravel()
        i += 1 + 8 * n
    return out


TOP_NODE = np.dtype([("bmin", "<f4", 3), ("child_start", "<i4"), ("bmax", "<f4", 3), ("child_count", "<i4")])
TOP_CHILD = np.dtype([("bmin", "<f4", 3), ("ref", "<i4"), ("bmax", "<f4", 3), ("is_node", "<i4")])
GOBJECT = np.dtype([("kind", "<i4"), ("material", "<i4"), ("aux", "<i4"), ("id", "<i4"), ("f", "<f4", 12)])


def top_tree_from_pack(pack) -> np.ndarray:
    """The packed top-level arrays (luz_pack_array "top_nodes", "top_children",
    "objects") walked in the order of top_tree_from_reference."""
    nodes = np.frombuffer(pack.array("top_nodes").tobytes(), TOP_NODE)
    kids = np.frombuffer(pack.array("top_children").tobytes(), TOP_CHILD)
    objs = np.frombuffer(pack.array("objects").tobytes(), GOBJECT)
    out = []
    if len(nodes) == 0:
        return np.zeros(0)
    stack = [0]
    order = []
    while stack:   # preorder over nodes, children in order
        k = stack.pop()
        order.append(k)
        c = kids[nodes[k]["child_start"]:nodes[k]["child_start"] + nodes[k]["child_count"]]
        stack.extend(int(r) for r in reversed(c["ref"][c["is_node"] != 0]))
    for k in order:
        c = kids[nodes[k]["child_start"]:nodes[k]["child_start"] + nodes[k]["child_count"]]
        out.append(float(len(c)))
        rec = np.zeros((len(c), 8))
        rec[:, 0] = c["is_node"] != 0
        rec[:, 1] = np.where(c["is_node"] != 0, -1, objs["id"][np.where(c["is_node"] != 0, 0, c["ref"])])
        rec[:, 2:5] = c["bmin"]
        rec[:, 5:8] = c["bmax"]
        out.extend(rec.ravel())
    return np.array(out)
