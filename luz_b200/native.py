"""ctypes binding of luz_b200/libluz_b200.so (include/luz_gpu.h).

The shared library is the product: the CUDA integrator and its host packer.
There is no fallback path: if the library is missing or the GPU call fails the
call raises, exactly as the reference's renderer throws std::runtime_error
(src/cli/main.cpp:209-213).
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional, Tuple

import numpy as np

from . import desc as D

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libluz_b200.so")

EXPORTED = [
    "luz_gpu_last_error", "luz_gpu_device_count", "luz_pack_create", "luz_pack_destroy", "luz_pack_info",
    "luz_pack_mesh_bvh", "luz_pack_array", "luz_gpu_scene_create", "luz_gpu_scene_destroy", "luz_gpu_scene_info",
    "luz_gpu_render", "luz_gpu_render_device", "luz_gpu_trace_paths", "luz_gpu_trace_rays",
    "luz_gpu_render_device_noalloc", "luz_gpu_render_ex", "luz_gpu_batch_render",
    "luz_gpu_scene_set_texture", "luz_gpu_adjoint_forward", "luz_gpu_adjoint_backward",
    "luz_gpu_nfor_denoise", "luz_gpu_nfor_error", "luz_gpu_render_denoised",
    "luz_gpu_cache_create", "luz_gpu_cache_destroy", "luz_gpu_cache_weights", "luz_gpu_cache_predict",
    "luz_gpu_cache_gradient", "luz_gpu_cache_train", "luz_gpu_render_cached", "luz_gpu_adjoint_emission",
    "luz_gpu_adjoint_density", "luz_gpu_scene_set_path_budget", "luz_gpu_scene_set_traversal_limits",
    "luz_gpu_render_pixels", "luz_gpu_scene_set_tuning", "luz_gpu_scene_get_tuning", "luz_gpu_autotune",
    "luz_gpu_batch_render_ex",
]

STATUS = {0: "ok", -1: "invalid argument", -2: "CUDA error", -3: "unsupported", -4: "limit exceeded",
          -5: "device error"}


class LuzError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"{message} [{STATUS.get(code, code)}]")
        self.code = code


_lib = None


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"luz_b200 native library not built: {LIB_PATH} (run __graft_entry__.build())")
    L = C.CDLL(LIB_PATH)
    vp, i32, i64 = C.c_void_p, C.c_int32, C.c_int64
    L.luz_gpu_last_error.argtypes = [C.c_char_p, C.c_size_t]
    L.luz_gpu_device_count.argtypes = [C.POINTER(i32)]
    L.luz_pack_create.argtypes = [vp, C.POINTER(vp)]
    L.luz_pack_destroy.argtypes = [vp]
    L.luz_pack_info.argtypes = [vp, C.POINTER(D.SceneInfo)]
    L.luz_pack_mesh_bvh.argtypes = [vp, i32, vp, i64, C.POINTER(i64), vp, i64]
    L.luz_pack_array.argtypes = [vp, C.c_char_p, C.POINTER(vp), C.POINTER(i64)]
    L.luz_gpu_scene_create.argtypes = [vp, i32, C.POINTER(vp)]
    L.luz_gpu_scene_destroy.argtypes = [vp]
    L.luz_gpu_scene_info.argtypes = [vp, C.POINTER(D.SceneInfo)]
    L.luz_gpu_scene_set_path_budget.argtypes = [vp, i64]
    L.luz_gpu_render_pixels.argtypes = [vp, C.POINTER(D.RenderParams), vp, i64, vp, C.POINTER(D.RenderStats)]
    L.luz_gpu_scene_set_tuning.argtypes = [vp, C.POINTER(D.TuneParams)]
    L.luz_gpu_scene_get_tuning.argtypes = [vp, C.POINTER(D.TuneParams)]
    L.luz_gpu_autotune.argtypes = [vp, C.POINTER(D.RenderParams), C.POINTER(D.TuneParams), vp, i32, C.POINTER(i32)]
    L.luz_gpu_scene_set_traversal_limits.argtypes = [vp, i32, i32]
    L.luz_gpu_render.argtypes = [vp, C.POINTER(D.RenderParams), vp, C.POINTER(D.RenderStats)]
    L.luz_gpu_render_device.argtypes = [vp, C.POINTER(D.RenderParams), vp, vp, C.POINTER(D.RenderStats)]
    L.luz_gpu_trace_paths.argtypes = [vp, C.POINTER(D.RenderParams), vp, vp, vp, i64, vp]
    L.luz_gpu_trace_rays.argtypes = [vp, vp, i64, i32, C.c_uint32, vp, vp]
    L.luz_gpu_render_device_noalloc.argtypes = [vp, C.POINTER(D.RenderParams), vp, vp, C.POINTER(D.RenderStats)]
    L.luz_gpu_render_ex.argtypes = [vp, C.POINTER(D.RenderParams), C.POINTER(D.AdaptiveParams), vp,
                                    C.POINTER(D.NforBuffers), vp, C.POINTER(D.RenderStats)]
    L.luz_gpu_batch_render.argtypes = [vp, vp, i32, vp, vp]
    L.luz_gpu_batch_render_ex.argtypes = [vp, vp, i32, vp, vp, C.POINTER(D.BatchReport)]
    L.luz_gpu_nfor_denoise.argtypes = [i32, C.POINTER(D.NforBuffers), i32, i32, C.POINTER(D.NforSettings), vp]
    L.luz_gpu_nfor_error.argtypes = [C.c_char_p, C.c_size_t]
    L.luz_gpu_render_denoised.argtypes = [vp, C.POINTER(D.RenderParams), C.POINTER(D.AdaptiveParams),
                                          C.POINTER(D.NforSettings), vp, vp, vp, C.POINTER(D.RenderStats)]
    L.luz_gpu_scene_set_texture.argtypes = [vp, i32, vp]
    L.luz_gpu_adjoint_forward.argtypes = [vp, C.POINTER(D.RenderParams), i32, vp, vp, C.POINTER(D.RenderStats)]
    L.luz_gpu_adjoint_backward.argtypes = [vp, C.POINTER(D.RenderParams), i32, vp, vp, C.POINTER(D.RenderStats)]
    L.luz_gpu_adjoint_emission.argtypes = [vp, C.POINTER(D.RenderParams), vp, vp, C.POINTER(D.RenderStats)]
    L.luz_gpu_adjoint_density.argtypes = [vp, C.POINTER(D.RenderParams), i32, vp, C.POINTER(C.c_double),
                                          C.POINTER(D.RenderStats)]
    L.luz_gpu_cache_create.argtypes = [i32, C.POINTER(D.CacheParams), C.POINTER(vp)]
    L.luz_gpu_cache_destroy.argtypes = [vp]
    L.luz_gpu_cache_weights.argtypes = [vp, vp, vp]
    L.luz_gpu_cache_predict.argtypes = [vp, vp, i64, vp]
    L.luz_gpu_cache_gradient.argtypes = [vp, vp, vp, i64, vp, C.POINTER(C.c_double)]
    L.luz_gpu_cache_train.argtypes = [vp, vp, vp, i64, i32, vp]
    L.luz_gpu_render_cached.argtypes = [vp, vp, C.POINTER(D.RenderParams), vp, C.POINTER(D.RenderStats)]
    for name in EXPORTED:
        getattr(L, name).restype = C.c_int
    _lib = L
    return L


def _check(rc: int):
    if rc != 0:
        buf = C.create_string_buffer(1024)
        lib().luz_gpu_last_error(buf, 1024)
        raise LuzError(rc, buf.value.decode(errors="replace"))


def device_count() -> int:
    n = C.c_int32(0)
    _check(lib().luz_gpu_device_count(C.byref(n)))
    return n.value


def adaptive(min_samples=128, check_interval=32, threshold=0.03, enabled=True) -> D.AdaptiveParams:
    """Adaptive sampling settings; the defaults are the reference's (include/luz/Defaults.hpp:12-15)."""
    return D.AdaptiveParams(1 if enabled else 0, int(min_samples), int(check_interval), 0, float(threshold))


def params(width, height, spp, max_bounces, seed, stream=0, sample_offset=0) -> D.RenderParams:
    return D.RenderParams(int(width), int(height), int(spp), int(max_bounces), int(seed) & 0xFFFFFFFF,
                          int(stream), int(sample_offset), 0)


class Pack:
    """Host-side packed scene (no GPU): BVH layouts and device arrays."""

    def __init__(self, built: D.BuiltDesc):
        self.built = built
        self.h = C.c_void_p()
        _check(lib().luz_pack_create(C.cast(built.ptr(), C.c_void_p), C.byref(self.h)))

    def close(self):
        if self.h:
            lib().luz_pack_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self) -> D.SceneInfo:
        i = D.SceneInfo()
        _check(lib().luz_pack_info(self.h, C.byref(i)))
        return i

    def mesh_bvh(self, mesh: int):
        cnt = C.c_int64()
        _check(lib().luz_pack_mesh_bvh(self.h, mesh, None, 0, C.byref(cnt), None, 0))
        nodes = np.zeros(max(1, cnt.value), D.NODE64_DTYPE)
        ntri = self.built.scene.meshes[mesh]["positions"].shape[0]
        order = np.zeros(max(1, ntri), np.int64)
        _check(lib().luz_pack_mesh_bvh(self.h, mesh, nodes.ctypes.data, nodes.shape[0], C.byref(cnt),
                                       order.ctypes.data, order.shape[0]))
        return nodes[:cnt.value], order

    def array(self, name: str) -> np.ndarray:
        p = C.c_void_p()
        n = C.c_int64()
        _check(lib().luz_pack_array(self.h, name.encode(), C.byref(p), C.byref(n)))
        if n.value == 0:
            return np.zeros(0, np.uint8)
        return np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_uint8)), shape=(n.value,)).copy()


class GpuScene:
    """Device scene arena (luz_gpu_scene). One host thread per handle."""

    def __init__(self, built: D.BuiltDesc, device: int = 0):
        self.built = built
        self.h = C.c_void_p()
        _check(lib().luz_gpu_scene_create(C.cast(built.ptr(), C.c_void_p), device, C.byref(self.h)))

    def close(self):
        if self.h:
            lib().luz_gpu_scene_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self) -> D.SceneInfo:
        i = D.SceneInfo()
        _check(lib().luz_gpu_scene_info(self.h, C.byref(i)))
        return i

    def render_pixels(self, p: D.RenderParams, x, y) -> Tuple[np.ndarray, D.RenderStats]:
        """luz_gpu_render_pixels: means of the listed pixels (n x 3)."""
        idx = np.ascontiguousarray(np.asarray(y, np.int64) * p.width + np.asarray(x, np.int64), np.int32)
        out = np.zeros((len(idx), 3), np.float32)
        st = D.RenderStats()
        _check(lib().luz_gpu_render_pixels(self.h, C.byref(p), idx.ctypes.data, len(idx), out.ctypes.data,
                                           C.byref(st)))
        return out, st

    def set_tuning(self, **kw):
        """luz_gpu_scene_set_tuning: fields of LuzTuneParams (unset = 0 = default)."""
        t = D.TuneParams(**kw)
        _check(lib().luz_gpu_scene_set_tuning(self.h, C.byref(t)))

    def tuning(self) -> dict:
        t = D.TuneParams()
        _check(lib().luz_gpu_scene_get_tuning(self.h, C.byref(t)))
        return {f: getattr(t, f) for f, _ in D.TuneParams._fields_}

    def autotune(self, p: D.RenderParams):
        """luz_gpu_autotune: (chosen tuning as a dict, [(tuning dict, render_ms) per trial])."""
        chosen = D.TuneParams()
        trials = (D.TuneTrial * 32)()
        n = C.c_int32(0)
        _check(lib().luz_gpu_autotune(self.h, C.byref(p), C.byref(chosen), trials, 32, C.byref(n)))
        as_dict = lambda t: {f: getattr(t, f) for f, _ in D.TuneParams._fields_}
        return as_dict(chosen), [(as_dict(trials[i].params), trials[i].render_ms) for i in range(n.value)]

    def set_path_budget(self, nbytes: int):
        """luz_gpu_scene_set_path_budget: cap on the path state held (bytes; -1 = default)."""
        _check(lib().luz_gpu_scene_set_path_budget(self.h, int(nbytes)))

    def set_traversal_limits(self, mesh_entries: int = 0, top_entries: int = 0):
        """luz_gpu_scene_set_traversal_limits (0 = the compiled stack size)."""
        _check(lib().luz_gpu_scene_set_traversal_limits(self.h, int(mesh_entries), int(top_entries)))

    def render(self, p: D.RenderParams, out: Optional[np.ndarray] = None) -> Tuple[np.ndarray, D.RenderStats]:
        """luz_gpu_render into `out` (H x W x 3 float32, C-contiguous, e.g. pinned) or a new array."""
        if out is None:
            out = np.zeros((p.height, p.width, 3), np.float32)
        elif out.dtype != np.float32 or out.shape != (p.height, p.width, 3) or not out.flags.c_contiguous:
            raise ValueError("out must be a C-contiguous float32 array of shape (height, width, 3)")
        st = D.RenderStats()
        _check(lib().luz_gpu_render(self.h, C.byref(p), out.ctypes.data, C.byref(st)))
        return out, st

    def render_ex(self, p: D.RenderParams, adaptive: Optional[D.AdaptiveParams] = None, nfor: bool = False):
        """luz_gpu_render_ex: film, samples used per pixel, NFOR buffers (dict, or None) and stats."""
        h, w = p.height, p.width
        out = np.zeros((h, w, 3), np.float32)
        used = np.zeros((h, w), np.int32)
        st = D.RenderStats()
        bufs = None
        nb = None
        if nfor:
            bufs = {"color_a": np.zeros((h, w, 3)), "color_b": np.zeros((h, w, 3)),
                    "color_variance": np.zeros((h, w)),
                    "features_a": np.zeros((h, w, D.NFOR_FEATURES)), "features_b": np.zeros((h, w, D.NFOR_FEATURES)),
                    "feature_variance": np.zeros((h, w, D.NFOR_FEATURES))}
            nb = D.NforBuffers(*[bufs[k].ctypes.data for k in ("color_a", "color_b", "color_variance", "features_a",
                                                                 "features_b", "feature_variance")])
        _check(lib().luz_gpu_render_ex(self.h, C.byref(p), C.byref(adaptive) if adaptive is not None else None,
                                       out.ctypes.data, C.byref(nb) if nb is not None else None, used.ctypes.data,
                                       C.byref(st)))
        return out, used, bufs, st

    def render_denoised(self, p: D.RenderParams, adaptive: Optional[D.AdaptiveParams] = None,
                        settings: Optional[D.NforSettings] = None):
        """luz_gpu_render_denoised: film, NFOR image (H x W x 3 float64), samples used per pixel and stats."""
        h, w = p.height, p.width
        out = np.zeros((h, w, 3), np.float32)
        den = np.zeros((h, w, 3), np.float64)
        used = np.zeros((h, w), np.int32)
        st = D.RenderStats()
        _check(lib().luz_gpu_render_denoised(self.h, C.byref(p), C.byref(adaptive) if adaptive is not None else None,
                                             C.byref(settings) if settings is not None else None, out.ctypes.data,
                                             den.ctypes.data, used.ctypes.data, C.byref(st)))
        return out, den, used, st

    def set_texture(self, texture: int, rgb: np.ndarray):
        rgb = np.ascontiguousarray(rgb, np.float64)
        _check(lib().luz_gpu_scene_set_texture(self.h, int(texture), rgb.ctypes.data))

    def adjoint_forward(self, p: D.RenderParams, texture: int, texels: np.ndarray):
        texels = np.ascontiguousarray(texels, np.float64)
        out = np.zeros((p.height, p.width, 3), np.float32)
        st = D.RenderStats()
        _check(lib().luz_gpu_adjoint_forward(self.h, C.byref(p), int(texture), texels.ctypes.data, out.ctypes.data,
                                             C.byref(st)))
        return out, st

    def adjoint_backward(self, p: D.RenderParams, texture: int, adjoint_rgb: np.ndarray, tex_shape):
        """dLoss/dtexel (tex_shape = (height, width, 3)) for dLoss/dpixel = adjoint_rgb (H x W x 3)."""
        adj = np.ascontiguousarray(adjoint_rgb, np.float32)
        grad = np.zeros(tex_shape, np.float64)
        st = D.RenderStats()
        _check(lib().luz_gpu_adjoint_backward(self.h, C.byref(p), int(texture), adj.ctypes.data, grad.ctypes.data,
                                              C.byref(st)))
        return grad, st

    def adjoint_emission(self, p: D.RenderParams, adjoint_rgb: np.ndarray):
        """dLoss/d(emitted radiance) per light (light_count x 3) for dLoss/dpixel = adjoint_rgb."""
        adj = np.ascontiguousarray(adjoint_rgb, np.float32)
        grad = np.zeros((max(self.info().light_count, 1), 3), np.float64)
        st = D.RenderStats()
        _check(lib().luz_gpu_adjoint_emission(self.h, C.byref(p), adj.ctypes.data, grad.ctypes.data, C.byref(st)))
        return grad[:self.info().light_count], st

    def adjoint_density(self, p: D.RenderParams, obj: int, adjoint_rgb: np.ndarray):
        """dLoss/d(density) of volume object `obj` for dLoss/dpixel = adjoint_rgb."""
        adj = np.ascontiguousarray(adjoint_rgb, np.float32)
        g = C.c_double()
        st = D.RenderStats()
        _check(lib().luz_gpu_adjoint_density(self.h, C.byref(p), int(obj), adj.ctypes.data, C.byref(g), C.byref(st)))
        return g.value, st

    def render_device(self, p: D.RenderParams, out_ptr: int, stream: int = 0) -> D.RenderStats:
        st = D.RenderStats()
        _check(lib().luz_gpu_render_device(self.h, C.byref(p), C.c_void_p(out_ptr), C.c_void_p(stream), C.byref(st)))
        return st

    def trace_paths(self, p: D.RenderParams, x, y, s) -> np.ndarray:
        x = np.ascontiguousarray(x, np.int32)
        y = np.ascontiguousarray(y, np.int32)
        s = np.ascontiguousarray(s, np.int32)
        out = np.zeros((x.shape[0], 3), np.float32)
        _check(lib().luz_gpu_trace_paths(self.h, C.byref(p), x.ctypes.data, y.ctypes.data, s.ctypes.data,
                                         x.shape[0], out.ctypes.data))
        return out

    def trace_rays(self, rays: np.ndarray, any_hit=False, seed=0, volume_key: Optional[np.ndarray] = None):
        rays = np.ascontiguousarray(rays, np.float32)
        out = np.zeros(rays.shape[0], D.HIT_DTYPE)
        vk = None if volume_key is None else np.ascontiguousarray(volume_key, np.int32)
        _check(lib().luz_gpu_trace_rays(self.h, rays.ctypes.data, rays.shape[0], 1 if any_hit else 0, seed,
                                        None if vk is None else vk.ctypes.data, out.ctypes.data))
        return out


def nfor_denoise(bufs: dict, device: int = 0, prefilter_radius=1, regression_radius=2, patch_radius=1,
                 min_variance=1e-5) -> np.ndarray:
    """luz_gpu_nfor_denoise on NFOR buffers (dict as GpuScene.render_ex returns); H x W x 3 float64."""
    h, w = bufs["color_variance"].shape[:2]
    a = {k: np.ascontiguousarray(v, np.float64) for k, v in bufs.items()}
    nb = D.NforBuffers(*[a[k].ctypes.data for k in ("color_a", "color_b", "color_variance", "features_a",
                                                    "features_b", "feature_variance")])
    st = D.NforSettings(int(prefilter_radius), int(regression_radius), int(patch_radius), 0, float(min_variance))
    out = np.zeros((h, w, 3), np.float64)
    rc = lib().luz_gpu_nfor_denoise(int(device), C.byref(nb), w, h, C.byref(st), out.ctypes.data)
    if rc != 0:
        buf = C.create_string_buffer(1024)
        lib().luz_gpu_nfor_error(buf, 1024)
        raise LuzError(rc, buf.value.decode(errors="replace"))
    return out


def batch_render(scenes, plist, report: bool = False):
    """luz_gpu_batch_render(_ex): renders every (scene, params) pair in shared multi-scene
    waves; returns the films (H x W x 3 each) and the per-scene stats (and the batch report
    as a dict when report=True)."""
    n = len(scenes)
    if len(plist) != n:
        raise ValueError("one RenderParams per scene")
    handles = (C.c_void_p * max(n, 1))(*[g.h.value for g in scenes])
    ps = (D.RenderParams * max(n, 1))(*plist)
    outs = [np.zeros((p.height, p.width, 3), np.float32) for p in plist]
    optrs = (C.c_void_p * max(n, 1))(*[o.ctypes.data for o in outs])
    stats = (D.RenderStats * max(n, 1))()
    rep = D.BatchReport()
    _check(lib().luz_gpu_batch_render_ex(handles, ps, n, optrs, stats, C.byref(rep)))
    if not report:
        return outs, list(stats)[:n]
    r = {"wave_paths": rep.wave_paths, "waves": rep.waves, "kernel_launches": rep.kernel_launches,
         "render_ms": rep.render_ms,
         "trials": [{"wave_paths": rep.trials[i].wave_paths, "paths": rep.trials[i].paths, "ms": rep.trials[i].ms}
                    for i in range(rep.trial_count)]}
    return outs, list(stats)[:n], r


def render(scene: D.Scene, width: int, height: int, spp: int, max_bounces: int, seed: int, device: int = 0,
           stream: int = 0):
    """Renderer::render (src/renderer/Renderer.cpp:10) for the sample loop: returns the
    W x H x 3 film of per-pixel means and the render stats."""
    g = GpuScene(scene.build(), device)
    try:
        return g.render(params(width, height, spp, max_bounces, seed, stream))
    finally:
        g.close()


class RadianceCache:
    """luz_gpu_cache: the learned radiance cache (FP16 tensor-core MLP trained online)."""

    def __init__(self, params: Optional[D.CacheParams] = None, device: int = 0):
        self.params = params if params is not None else D.cache_params()
        self.h = C.c_void_p()
        _check(lib().luz_gpu_cache_create(device, C.byref(self.params), C.byref(self.h)))

    def close(self):
        if self.h:
            lib().luz_gpu_cache_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def weights(self) -> np.ndarray:
        w = np.zeros(D.CACHE_PARAMS, np.float32)
        _check(lib().luz_gpu_cache_weights(self.h, w.ctypes.data, None))
        return w

    def set_weights(self, w: np.ndarray):
        w = np.ascontiguousarray(w, np.float32)
        _check(lib().luz_gpu_cache_weights(self.h, None, w.ctypes.data))

    def predict(self, inputs: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(inputs, np.float32)
        out = np.zeros((x.shape[0], 3), np.float32)
        _check(lib().luz_gpu_cache_predict(self.h, x.ctypes.data, x.shape[0], out.ctypes.data))
        return out

    def gradient(self, inputs: np.ndarray, targets: np.ndarray):
        x = np.ascontiguousarray(inputs, np.float32)
        t = np.ascontiguousarray(targets, np.float32)
        g = np.zeros(D.CACHE_PARAMS, np.float32)
        loss = C.c_double()
        _check(lib().luz_gpu_cache_gradient(self.h, x.ctypes.data, t.ctypes.data, x.shape[0], g.ctypes.data,
                                            C.byref(loss)))
        return g, loss.value

    def train(self, inputs: np.ndarray, targets: np.ndarray, steps: int = 1) -> np.ndarray:
        x = np.ascontiguousarray(inputs, np.float32)
        t = np.ascontiguousarray(targets, np.float32)
        losses = np.zeros(max(steps, 1), np.float64)
        _check(lib().luz_gpu_cache_train(self.h, x.ctypes.data, t.ctypes.data, x.shape[0], steps, losses.ctypes.data))
        return losses[:steps]

    def render(self, scene: "GpuScene", p: D.RenderParams):
        """luz_gpu_render_cached: film (H x W x 3) and stats; trains the cache as it renders."""
        out = np.zeros((p.height, p.width, 3), np.float32)
        st = D.RenderStats()
        _check(lib().luz_gpu_render_cached(scene.h, self.h, C.byref(p), out.ctypes.data, C.byref(st)))
        return out, st
