"""ctypes mirror of include/luz_gpu.h and a builder for LuzSceneDesc.

The builder plays the role of the C++ host-side packer a Luz maintainer adds to
Renderer::render: it turns a scene made of the reference's
object kinds (Rectangle, Sphere, Cube, Plane, Mesh, MeshInstance,
ConstantVolume, DirectionalLight; src/core/Hittables/*) and materials
(src/core/Materials/*) into the flat description both the GPU library and the
reference oracle consume. Defaults follow the reference constructors.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

ABI_VERSION = 5

MAT_LAMBERTIAN, MAT_METAL, MAT_DIELECTRIC, MAT_EMISSIVE = 1, 2, 3, 4
MAT_ISOTROPIC, MAT_HENYEY_GREENSTEIN, MAT_PRINCIPLED = 5, 6, 7
MAT_GLOSSY, MAT_DIFFUSE_GLOSSY = 8, 9

OBJ_RECTANGLE, OBJ_SPHERE, OBJ_CUBE, OBJ_PLANE = 1, 2, 3, 4
OBJ_MESH, OBJ_MESH_INSTANCE, OBJ_VOLUME, OBJ_DIRECTIONAL_LIGHT = 5, 6, 7, 8

SKY_NONE, SKY_LINEAR, SKY_ATMOSPHERE, SKY_ENVIRONMENT = 0, 1, 2, 3

D3 = C.c_double * 3
D12 = C.c_double * 12


class MaterialDesc(C.Structure):
    _fields_ = [
        ("type", C.c_int32), ("texture", C.c_int32),
        ("color", D3), ("roughness", C.c_double), ("ior", C.c_double), ("anisotropy", C.c_double),
        ("conductor", C.c_int32), ("subsurface_method", C.c_int32),
        ("eta", D3), ("k", D3), ("absorption", D3),
        ("metallic", C.c_double), ("transmission", C.c_double), ("clearcoat", C.c_double),
        ("clearcoat_roughness", C.c_double), ("sheen", C.c_double), ("subsurface", C.c_double),
        ("subsurface_radius", D3), ("subsurface_scale", C.c_double), ("subsurface_color", D3),
        ("glossy_color", D3), ("glossy_weight", C.c_double),
        ("has_roughness_texture", C.c_int32), ("roughness_texture", C.c_int32),
    ]


class TextureDesc(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("rgb", C.POINTER(C.c_double))]


class MeshDesc(C.Structure):
    _fields_ = [
        ("triangle_count", C.c_int64), ("positions", C.POINTER(C.c_double)),
        ("normals", C.POINTER(C.c_double)), ("uvs", C.POINTER(C.c_double)),
        ("material", C.c_int32), ("_pad", C.c_int32),
    ]


class ObjectDesc(C.Structure):
    _fields_ = [
        ("kind", C.c_int32), ("material", C.c_int32), ("mesh", C.c_int32), ("boundary_kind", C.c_int32),
        ("position", D3), ("orientation", D3), ("size", D3), ("width_axis", D3), ("height_axis", D3),
        ("has_axes", C.c_int32), ("visible", C.c_int32),
        ("rotation_degrees", D3), ("scale", D3), ("density", C.c_double),
        ("has_uvs", C.c_int32), ("_pad", C.c_int32), ("uv", D12),
        ("ies", C.c_int32), ("uv_projection", C.c_int32), ("ies_direction", D3), ("ies_rotation_degrees", C.c_double),
    ]


class IesDesc(C.Structure):
    _fields_ = [("vertical_count", C.c_int32), ("horizontal_count", C.c_int32),
                ("vertical_deg", C.POINTER(C.c_double)), ("horizontal_deg", C.POINTER(C.c_double)),
                ("candela", C.POINTER(C.c_double))]


class CameraDesc(C.Structure):
    _fields_ = [
        ("position", D3), ("direction", D3), ("up", D3),
        ("focal_length_m", C.c_double), ("sensor_width_m", C.c_double), ("sensor_height_m", C.c_double),
        ("f_number", C.c_double), ("focus_distance_m", C.c_double),
        ("pinhole", C.c_int32), ("_pad", C.c_int32),
    ]


class EnvironmentDesc(C.Structure):
    _fields_ = [
        ("width", C.c_int32), ("height", C.c_int32), ("rgb", C.POINTER(C.c_double)),
        ("strength", C.c_double), ("rotation_degrees", C.c_double),
        ("lighting", C.c_int32), ("_pad", C.c_int32),
    ]


class AtmosphereDesc(C.Structure):
    _fields_ = [("sun_direction", D3), ("sun_radiance", D3), ("sun_radiance_scale", C.c_double),
                ("earth_radius", C.c_double), ("atmosphere_radius", C.c_double), ("h_r", C.c_double),
                ("h_m", C.c_double), ("samples", C.c_int32), ("light_samples", C.c_int32),
                ("stars_brightness", C.c_double)]


class CausticsDesc(C.Structure):
    """LuzCausticsDesc: Scene caustic settings (src/scene/Scene.cpp:302-360)."""
    _fields_ = [("enabled", C.c_int32), ("photons", C.c_int32), ("passes", C.c_int32), ("reserved", C.c_int32),
                ("radius_meters", C.c_double), ("alpha", C.c_double)]


class SceneDesc(C.Structure):
    _fields_ = [
        ("abi_version", C.c_int32), ("material_count", C.c_int32), ("materials", C.POINTER(MaterialDesc)),
        ("texture_count", C.c_int32), ("mesh_count", C.c_int32),
        ("textures", C.POINTER(TextureDesc)), ("meshes", C.POINTER(MeshDesc)),
        ("object_count", C.c_int32), ("sky", C.c_int32), ("objects", C.POINTER(ObjectDesc)),
        ("camera", CameraDesc), ("environment", EnvironmentDesc),
        ("background", D3), ("meters_per_unit", C.c_double),
        ("ies_count", C.c_int32), ("_pad", C.c_int32), ("ies", C.POINTER(IesDesc)),
        ("atmosphere", AtmosphereDesc), ("caustics", CausticsDesc),
    ]


RENDER_PROFILE = 0x100
RENDER_COUNT = 0x200


class RenderParams(C.Structure):
    _fields_ = [
        ("width", C.c_int32), ("height", C.c_int32), ("spp", C.c_int32), ("max_bounces", C.c_int32),
        ("seed", C.c_uint32), ("stream", C.c_uint32), ("sample_offset", C.c_int32), ("flags", C.c_int32),
    ]


class RenderStats(C.Structure):
    _fields_ = [
        ("render_ms", C.c_double), ("samples", C.c_double), ("extension_rays", C.c_double),
        ("shadow_rays", C.c_double), ("kernel_launches", C.c_int64), ("waves", C.c_int64),
        ("extend_ms", C.c_double), ("shade_ms", C.c_double), ("shadow_ms", C.c_double),
        ("extend_launches", C.c_int64), ("shadow_launches", C.c_int64),
        ("ext_nodes", C.c_double), ("ext_tris", C.c_double), ("ext_top", C.c_double),
        ("sh_nodes", C.c_double), ("sh_tris", C.c_double), ("sh_top", C.c_double),
        ("denoise_ms", C.c_double), ("caustic_photons", C.c_double), ("caustic_ms", C.c_double),
        ("ext_bnodes", C.c_double), ("sh_bnodes", C.c_double),
    ]


class TuneParams(C.Structure):
    """LuzTuneParams: launch tuning of a scene handle (zeros = defaults)."""
    _fields_ = [("wave_paths", C.c_int64), ("staged_top_nodes", C.c_int32), ("extend_blocks_per_sm", C.c_int32),
                ("shadow_blocks_per_sm", C.c_int32), ("shade_blocks_per_sm", C.c_int32), ("sort_rays", C.c_int32),
                ("lanes", C.c_int32)]


class TuneTrial(C.Structure):
    _fields_ = [("params", TuneParams), ("render_ms", C.c_double)]


class BatchTrial(C.Structure):
    _fields_ = [("wave_paths", C.c_int64), ("paths", C.c_double), ("ms", C.c_double)]


class BatchReport(C.Structure):
    """LuzBatchReport: what luz_gpu_batch_render_ex did."""
    _fields_ = [("wave_paths", C.c_int64), ("waves", C.c_int64), ("kernel_launches", C.c_int64),
                ("render_ms", C.c_double), ("trial_count", C.c_int32), ("reserved", C.c_int32),
                ("trials", BatchTrial * 8)]


class AdaptiveParams(C.Structure):
    """LuzAdaptiveParams: Scene adaptive settings (src/scene/Scene.cpp:183-222)."""
    _fields_ = [("enabled", C.c_int32), ("min_samples", C.c_int32), ("check_interval", C.c_int32),
                ("reserved", C.c_int32), ("threshold", C.c_double)]


NFOR_FEATURES = 11


class NforBuffers(C.Structure):
    """LuzNforBuffers: host pointers of the Denoise::NFORBuffers arrays."""
    _fields_ = [("color_a", C.c_void_p), ("color_b", C.c_void_p), ("color_variance", C.c_void_p),
                ("features_a", C.c_void_p), ("features_b", C.c_void_p), ("feature_variance", C.c_void_p)]


class NforSettings(C.Structure):
    """LuzNforSettings (Denoise::NFORSettings)."""
    _fields_ = [("feature_prefilter_radius", C.c_int32), ("regression_radius", C.c_int32),
                ("patch_radius", C.c_int32), ("reserved", C.c_int32), ("min_variance", C.c_double)]


CACHE_PARAMS = 21504


class CacheParams(C.Structure):
    """LuzCacheParams: learned radiance cache settings."""
    _fields_ = [("seed", C.c_uint32), ("batch", C.c_int32), ("learning_rate", C.c_float), ("prefix", C.c_int32),
                ("train_every", C.c_int32), ("min_roughness", C.c_float), ("warm_steps", C.c_int32)]


def cache_params(seed=1, batch=16384, learning_rate=1e-2, prefix=1, train_every=32,
                 min_roughness=0.0, warm_steps=0) -> CacheParams:
    return CacheParams(seed, batch, learning_rate, prefix, train_every, min_roughness, warm_steps)


class Hit(C.Structure):
    _fields_ = [("t", C.c_float), ("object", C.c_int32), ("primitive", C.c_int32), ("u", C.c_float), ("v", C.c_float)]


class SceneInfo(C.Structure):
    _fields_ = [
        ("top_nodes", C.c_int64), ("top_leaf_objects", C.c_int64), ("mesh_nodes", C.c_int64),
        ("mesh_triangles", C.c_int64), ("device_bytes", C.c_int64),
        ("max_mesh_depth", C.c_int32), ("light_count", C.c_int32),
    ]


class MeshNode64(C.Structure):
    _fields_ = [
        ("bmin", D3), ("bmax", D3), ("left", C.c_int64), ("right", C.c_int64),
        ("start", C.c_int64), ("count", C.c_int64), ("is_leaf", C.c_int32), ("_pad", C.c_int32),
    ]


HIT_DTYPE = np.dtype([("t", "<f4"), ("object", "<i4"), ("primitive", "<i4"), ("u", "<f4"), ("v", "<f4")])
NODE64_DTYPE = np.dtype([("bmin", "<f8", 3), ("bmax", "<f8", 3), ("left", "<i8"), ("right", "<i8"),
                         ("start", "<i8"), ("count", "<i8"), ("is_leaf", "<i4"), ("_pad", "<i4")])


def _d3(v):
    return D3(*[float(x) for x in v])


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


@dataclass
class Camera:
    """Camera (src/core/Camera.cpp). Defaults: 50 mm lens, 36 x 20.25 mm sensor, f/8, 10 m focus."""
    position: tuple = (0.0, 0.0, 15.0)
    direction: tuple = (0.0, 0.0, -1.0)
    up: tuple = (0.0, 1.0, 0.0)
    focal_length_m: float = 0.050
    sensor_width_m: float = 0.036
    sensor_height_m: float = 0.02025
    f_number: float = 8.0
    focus_distance_m: float = 10.0
    pinhole: bool = False


@dataclass
class Scene:
    """Flat scene: materials, textures, meshes and objects in Scene::addHittable order."""
    materials: List[dict] = field(default_factory=list)
    textures: List[np.ndarray] = field(default_factory=list)
    ies: list = field(default_factory=list)
    # Atmosphere (sky = SKY_ATMOSPHERE): reference defaults (Defaults.hpp:21-24, Atmosphere.cpp:69-80);
    # sun direction/radiance as Scene::syncAtmosphereSunDirection leaves them.
    atmosphere: dict = field(default_factory=lambda: dict(
        sun_direction=(0.0, 0.3, -0.95), sun_radiance=(1.0, 1.0, 1.0), sun_radiance_scale=1.0,
        earth_radius=6360e3, atmosphere_radius=6420e3, h_r=7994.0, h_m=1200.0, samples=16, light_samples=8,
        stars_brightness=0.5))
    meshes: List[dict] = field(default_factory=list)
    objects: List[dict] = field(default_factory=list)
    camera: Camera = field(default_factory=Camera)
    background: tuple = (0.0, 0.0, 0.0)
    sky: int = SKY_NONE
    environment: Optional[np.ndarray] = None      # (H, W, 3) float64
    environment_strength: float = 1.0
    environment_rotation: float = 0.0
    environment_lighting: bool = True
    meters_per_unit: float = 1.0
    # Caustic photon map (Defaults.hpp:51-55); enabled by Scene.caustics(...)
    caustics: dict = field(default_factory=lambda: dict(enabled=0, photons=100000, passes=8, radius_meters=0.05,
                                                        alpha=0.7))

    # -- materials (defaults = reference constructors) --------------------------
    def _mat(self, **kw) -> int:
        m = dict(type=MAT_LAMBERTIAN, texture=-1, color=(0.6, 0.6, 0.6), roughness=0.0, ior=1.52,
                 anisotropy=0.0, conductor=0, subsurface_method=0, eta=(1.0, 1.0, 1.0), k=(0.0, 0.0, 0.0),
                 absorption=(0.0, 0.0, 0.0), metallic=0.0, transmission=0.0, clearcoat=0.0,
                 clearcoat_roughness=0.03, sheen=0.0, subsurface=0.0, subsurface_radius=(1.0, 1.0, 1.0),
                 subsurface_scale=0.001, subsurface_color=(1.0, 1.0, 1.0), glossy_color=(1.0, 1.0, 1.0),
                 glossy_weight=0.5)
        m.update(kw)
        self.materials.append(m)
        return len(self.materials) - 1

    def lambertian(self, color, texture=-1):
        return self._mat(type=MAT_LAMBERTIAN, color=color, texture=texture)

    def metal(self, color=(0.6, 0.6, 0.6), roughness=0.0, eta=None, k=None, roughness_texture=None):
        """roughness_texture: index of a texture whose red channel gives the roughness per hit
        (an extension: the reference's Metal roughness is a scalar)."""
        rt = {} if roughness_texture is None else dict(has_roughness_texture=1, roughness_texture=roughness_texture)
        if eta is not None:
            return self._mat(type=MAT_METAL, color=(1.0, 1.0, 1.0), roughness=roughness, conductor=1, eta=eta, k=k,
                             **rt)
        return self._mat(type=MAT_METAL, color=color, roughness=roughness, **rt)

    def glossy(self, color=(1.0, 1.0, 1.0), roughness=0.0):
        return self._mat(type=MAT_GLOSSY, color=color, roughness=roughness)

    def diffuse_glossy(self, diffuse=(0.6, 0.6, 0.6), glossy=(1.0, 1.0, 1.0), weight=0.5, roughness=0.0):
        return self._mat(type=MAT_DIFFUSE_GLOSSY, color=diffuse, glossy_color=glossy, glossy_weight=weight,
                         roughness=roughness)

    def dielectric(self, color=(1.0, 1.0, 1.0), ior=1.52, roughness=0.0, absorption=(0.0, 0.0, 0.0)):
        return self._mat(type=MAT_DIELECTRIC, color=color, ior=ior, roughness=roughness, absorption=absorption)

    def emissive(self, radiance):
        return self._mat(type=MAT_EMISSIVE, color=radiance)

    def isotropic(self, color):
        return self._mat(type=MAT_ISOTROPIC, color=color)

    def henyey_greenstein(self, color, g):
        return self._mat(type=MAT_HENYEY_GREENSTEIN, color=color, anisotropy=g)

    def principled(self, color, metallic=0.0, roughness=0.5, transmission=0.0, ior=1.52, clearcoat=0.0,
                   clearcoat_roughness=0.03, sheen=0.0, **kw):
        return self._mat(type=MAT_PRINCIPLED, color=color, metallic=metallic, roughness=roughness,
                         transmission=transmission, ior=ior, clearcoat=clearcoat,
                         clearcoat_roughness=clearcoat_roughness, sheen=sheen, **kw)

    def texture(self, rgb: np.ndarray) -> int:
        self.textures.append(np.ascontiguousarray(rgb, dtype=np.float64))
        return len(self.textures) - 1

    # -- geometry ----------------------------------------------------------------
    def _obj(self, **kw) -> int:
        o = dict(kind=0, material=-1, mesh=-1, boundary_kind=0, position=(0, 0, 0), orientation=(0, 0, 1),
                 size=(1, 1, 1), width_axis=(1, 0, 0), height_axis=(0, 1, 0), has_axes=0, visible=1,
                 rotation_degrees=(0, 0, 0), scale=(1, 1, 1), density=1.42, has_uvs=0, uv=(0,) * 12, ies=-1,
                 ies_direction=(0, -1, 0), ies_rotation_degrees=0.0)
        o.update(kw)
        self.objects.append(o)
        return len(self.objects) - 1

    def rectangle(self, position, normal, width, height, material, width_axis=None, height_axis=None, uvs=None):
        """uvs: optional corner texture coordinates ((u0,v0), (u1,v1), (u2,v2), (u3,v3))
        (Rectangle::setTextureCoordinates)."""
        kw = {}
        if width_axis is not None:
            kw = dict(has_axes=1, width_axis=width_axis, height_axis=height_axis)
        if uvs is not None:
            kw.update(has_uvs=1, uv=tuple(float(c) for uv in uvs for c in (uv[0], uv[1], 0.0)))
        return self._obj(kind=OBJ_RECTANGLE, position=position, orientation=normal, size=(width, height, 0),
                         material=material, **kw)

    def sphere(self, center, radius, material, visible=True, ies=-1, ies_direction=(0.0, -1.0, 0.0),
               ies_rotation=0.0, uv_projection=0):
        """ies: -1 or an index from ies_profile (Sphere::setIESProfile); uv_projection: 0 lat-long,
        1 cube cross (SphereUVProjection)."""
        return self._obj(kind=OBJ_SPHERE, position=center, size=(radius, 0, 0), material=material,
                         visible=1 if visible else 0, ies=ies, ies_direction=ies_direction,
                         ies_rotation_degrees=float(ies_rotation), uv_projection=int(uv_projection))

    def ies_profile(self, vertical_deg, horizontal_deg, candela) -> int:
        """candela: (len(horizontal), len(vertical)) array (IES file order, multiplier applied)."""
        c = np.ascontiguousarray(candela, dtype=np.float64)
        self.ies.append((np.ascontiguousarray(vertical_deg, np.float64), np.ascontiguousarray(horizontal_deg, np.float64),
                         c.reshape(-1)))
        return len(self.ies) - 1

    def cube(self, center, w, h, d, material):
        return self._obj(kind=OBJ_CUBE, position=center, size=(w, h, d), material=material)

    def plane(self, y, normal, material):
        return self._obj(kind=OBJ_PLANE, position=(0, y, 0), orientation=normal, material=material)

    def mesh(self, positions: np.ndarray, material: int, normals=None, uvs=None, add_object=True):
        """Adds a triangle soup (N, 3, 3); returns (mesh index, object index or -1)."""
        pos = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1, 9)
        m = dict(positions=pos, material=material,
                 normals=None if normals is None else np.ascontiguousarray(normals, dtype=np.float64).reshape(-1, 9),
                 uvs=None if uvs is None else np.ascontiguousarray(uvs, dtype=np.float64).reshape(-1, 6))
        self.meshes.append(m)
        mi = len(self.meshes) - 1
        oi = self._obj(kind=OBJ_MESH, mesh=mi, material=material) if add_object else -1
        return mi, oi

    def mesh_instance(self, mesh: int, position, rotation_degrees, scale, material):
        return self._obj(kind=OBJ_MESH_INSTANCE, mesh=mesh, position=position, rotation_degrees=rotation_degrees,
                         scale=scale, material=material)

    def volume_cube(self, center, w, h, d, phase_material, density):
        return self._obj(kind=OBJ_VOLUME, boundary_kind=OBJ_CUBE, position=center, size=(w, h, d),
                         material=phase_material, density=density)

    def volume_sphere(self, center, radius, phase_material, density):
        return self._obj(kind=OBJ_VOLUME, boundary_kind=OBJ_SPHERE, position=center, size=(radius, 0, 0),
                         material=phase_material, density=density)

    def directional_light(self, direction, material):
        return self._obj(kind=OBJ_DIRECTIONAL_LIGHT, orientation=direction, material=material)

    def set_environment(self, rgb: np.ndarray, strength=1.0, rotation=0.0, lighting=True):
        self.environment = np.ascontiguousarray(rgb, dtype=np.float64)
        self.environment_strength = strength
        self.environment_rotation = rotation
        self.environment_lighting = lighting
        self.sky = SKY_ENVIRONMENT

    def set_caustics(self, photons=100000, passes=8, radius_meters=0.05, alpha=0.7, enabled=True):
        """Scene::setCausticsEnabled / setCausticPhotonCount / setCausticPassCount /
        setCausticRadiusMeters / setCausticAlpha."""
        self.caustics = dict(enabled=1 if enabled else 0, photons=photons, passes=passes,
                             radius_meters=radius_meters, alpha=alpha)

    # -- C description -------------------------------------------------------
    def build(self) -> "BuiltDesc":
        return BuiltDesc(self)


class BuiltDesc:
    """Owns the ctypes arrays behind one LuzSceneDesc (keep it alive while in use)."""

    def __init__(self, s: Scene):
        self._keep = []
        mats = (MaterialDesc * max(1, len(s.materials)))()
        for i, m in enumerate(s.materials):
            md = mats[i]
            for k, v in m.items():
                setattr(md, k, _d3(v) if isinstance(v, (tuple, list)) else v)
        texs = (TextureDesc * max(1, len(s.textures)))()
        for i, t in enumerate(s.textures):
            t = np.ascontiguousarray(t, dtype=np.float64)
            self._keep.append(t)
            texs[i].height, texs[i].width = t.shape[0], t.shape[1]
            texs[i].rgb = _dptr(t)
        meshes = (MeshDesc * max(1, len(s.meshes)))()
        for i, m in enumerate(s.meshes):
            meshes[i].triangle_count = m["positions"].shape[0]
            meshes[i].positions = _dptr(m["positions"])
            self._keep.append(m["positions"])
            if m["normals"] is not None:
                meshes[i].normals = _dptr(m["normals"])
                self._keep.append(m["normals"])
            if m["uvs"] is not None:
                meshes[i].uvs = _dptr(m["uvs"])
                self._keep.append(m["uvs"])
            meshes[i].material = m["material"]
        objs = (ObjectDesc * max(1, len(s.objects)))()
        for i, o in enumerate(s.objects):
            od = objs[i]
            for k, v in o.items():
                if k == "uv":
                    od.uv = D12(*[float(x) for x in v])
                else:
                    setattr(od, k, _d3(v) if isinstance(v, (tuple, list, np.ndarray)) else v)
        d = SceneDesc()
        d.abi_version = ABI_VERSION
        d.material_count, d.materials = len(s.materials), mats
        d.texture_count, d.textures = len(s.textures), texs
        d.mesh_count, d.meshes = len(s.meshes), meshes
        d.object_count, d.objects = len(s.objects), objs
        cam = s.camera
        d.camera = CameraDesc(_d3(cam.position), _d3(cam.direction), _d3(cam.up), cam.focal_length_m,
                              cam.sensor_width_m, cam.sensor_height_m, cam.f_number, cam.focus_distance_m,
                              1 if cam.pinhole else 0, 0)
        if s.environment is not None:
            env = np.ascontiguousarray(s.environment, dtype=np.float64)
            self._keep.append(env)
            d.environment = EnvironmentDesc(env.shape[1], env.shape[0], _dptr(env), s.environment_strength,
                                            s.environment_rotation, 1 if s.environment_lighting else 0, 0)
        d.background = _d3(s.background)
        ies = (IesDesc * max(1, len(s.ies)))()
        for i, (va, ha, cd) in enumerate(s.ies):
            self._keep += [va, ha, cd]
            ies[i] = IesDesc(va.shape[0], ha.shape[0], _dptr(va), _dptr(ha), _dptr(cd))
        d.ies_count, d.ies = len(s.ies), ies
        a = s.atmosphere
        d.atmosphere = AtmosphereDesc(_d3(a["sun_direction"]), _d3(a["sun_radiance"]), a["sun_radiance_scale"],
                                      a["earth_radius"], a["atmosphere_radius"], a["h_r"], a["h_m"], a["samples"],
                                      a["light_samples"], a["stars_brightness"])
        c = s.caustics
        d.caustics = CausticsDesc(int(c["enabled"]), int(c["photons"]), int(c["passes"]), 0,
                                  float(c["radius_meters"]), float(c["alpha"]))
        d.sky = s.sky
        d.meters_per_unit = s.meters_per_unit
        self._keep += [mats, texs, meshes, objs]
        self.desc = d
        self.scene = s

    def ptr(self):
        return C.byref(self.desc)
