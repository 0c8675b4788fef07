"""Seeded synthetic scenes with the shapes of the five benchmark configurations.

No dataset or asset is read: every scene is generated from a seed, with the
sizes and value distributions of the workload it stands for. The same
description feeds the GPU integrator and the reference oracle.

  cornell()              300x300, 50 spp, depth 8: five 555 walls, 130x105 light,
                         two rotated boxes as instanced 12-triangle meshes.
  mesh_glossy()          1920x1080, 64 spp, depth 12: level-8 icosphere (1,310,720
                         triangles) displaced by 4-octave value noise (amplitude
                         0.1) over a ground quad; rough dielectric + GGX metal;
                         1024x512 equirect sky with a 0.5 degree sun lobe; f/2.8.
  instancing_volumes()   1280x720, 32 spp, depth 16: 1e5 instances of a 200-triangle
                         mesh, uniform random rotations, log-normal scales (sigma
                         0.3) in a 100^3 box filled with an HG medium (g 0.6,
                         sigma_t 0.05, albedo 0.8), two sphere lights and a
                         directional light.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .desc import SKY_LINEAR, Camera, Scene


@dataclass
class Workload:
    name: str
    scene: Scene
    width: int
    height: int
    spp: int
    max_bounces: int
    seed: int = 424242424


# ----------------------------------------------------------------------------- meshes

def box_mesh() -> np.ndarray:
    """Unit cube [0,1]^3 as 12 outward-wound triangles, shape (12, 3, 3)."""
    c = np.array([[x, y, z] for z in (0, 1) for y in (0, 1) for x in (0, 1)], np.float64)
    quads = [(0, 2, 3, 1), (4, 5, 7, 6), (0, 1, 5, 4), (2, 6, 7, 3), (0, 4, 6, 2), (1, 3, 7, 5)]
    tris = []
    for a, b, cc, d in quads:
        tris.append([c[a], c[b], c[cc]])
        tris.append([c[a], c[cc], c[d]])
    return np.array(tris, np.float64)


def icosphere(level: int):
    """Subdivided icosahedron on the unit sphere: (vertices (V,3), faces (F,3))."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
                  [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], np.float64)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4], [11, 10, 2],
                  [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5],
                  [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], np.int64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    for _ in range(level):
        e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
        e.sort(axis=1)
        uniq, inv = np.unique(e, axis=0, return_inverse=True)
        mid = v[uniq[:, 0]] + v[uniq[:, 1]]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        base = v.shape[0]
        v = np.concatenate([v, mid])
        nf = f.shape[0]
        m01, m12, m20 = (inv[:nf] + base, inv[nf:2 * nf] + base, inv[2 * nf:] + base)
        f = np.concatenate([np.stack([f[:, 0], m01, m20], 1), np.stack([f[:, 1], m12, m01], 1),
                            np.stack([f[:, 2], m20, m12], 1), np.stack([m01, m12, m20], 1)])
    return v, f


def value_noise(p: np.ndarray, seed: int, octaves: int = 4) -> np.ndarray:
    """Seeded 3-D value noise (smoothstep-trilinear over a hashed lattice), in [-1, 1]."""
    rng = np.random.default_rng(seed)
    table = rng.uniform(-1.0, 1.0, 4096)
    perm = rng.permutation(4096)

    def lattice(ix, iy, iz):
        h = perm[(ix * 73856093 ^ iy * 19349663 ^ iz * 83492791) & 4095]
        return table[h]

    out = np.zeros(p.shape[0])
    amp, freq, norm = 1.0, 2.0, 0.0
    for _ in range(octaves):
        q = p * freq
        i = np.floor(q).astype(np.int64)
        fr = q - i
        w = fr * fr * (3.0 - 2.0 * fr)
        acc = 0.0
        for dx in (0, 1):
            for dy in (0, 1):
                for dz in (0, 1):
                    wx = w[:, 0] if dx else 1 - w[:, 0]
                    wy = w[:, 1] if dy else 1 - w[:, 1]
                    wz = w[:, 2] if dz else 1 - w[:, 2]
                    acc = acc + wx * wy * wz * lattice(i[:, 0] + dx, i[:, 1] + dy, i[:, 2] + dz)
        out += amp * acc
        norm += amp
        amp *= 0.5
        freq *= 2.0
    return out / norm


def torus_mesh(segments: int = 10, rings: int = 10, major: float = 1.0, minor: float = 0.35) -> np.ndarray:
    """segments*rings*2 triangles (200 at the defaults)."""
    u = np.linspace(0, 2 * np.pi, segments, endpoint=False)
    w = np.linspace(0, 2 * np.pi, rings, endpoint=False)
    U, W = np.meshgrid(u, w, indexing="ij")
    P = np.stack([(major + minor * np.cos(W)) * np.cos(U), minor * np.sin(W), (major + minor * np.cos(W)) * np.sin(U)], -1)
    tris = []
    for a in range(segments):
        for b in range(rings):
            a1, b1 = (a + 1) % segments, (b + 1) % rings
            tris.append([P[a, b], P[a1, b], P[a1, b1]])
            tris.append([P[a, b], P[a1, b1], P[a, b1]])
    return np.array(tris, np.float64)


# ----------------------------------------------------------------------------- scenes

def _pinhole(position, look_at, vfov_deg, aspect):
    d = np.asarray(look_at, float) - np.asarray(position, float)
    f = 0.050
    sh = 2.0 * math.tan(math.radians(vfov_deg) / 2.0) * f
    return Camera(position=tuple(position), direction=tuple(d), up=(0.0, 1.0, 0.0), focal_length_m=f,
                  sensor_width_m=sh * aspect, sensor_height_m=sh, f_number=8.0, focus_distance_m=10.0, pinhole=True)


def cornell(width: int = 300, height: int = 300, spp: int = 50, max_bounces: int = 8, closed: bool = False) -> Workload:
    """The Cornell box; closed = True closes its open side with a white wall and puts the
    camera inside, so that paths stay in the room until Russian roulette or the depth limit
    ends them."""
    s = Scene()
    white = s.lambertian((0.73, 0.73, 0.73))
    red = s.lambertian((0.65, 0.05, 0.05))
    green = s.lambertian((0.12, 0.45, 0.15))
    light = s.emissive((15.0, 15.0, 15.0))
    s.rectangle((555.0, 277.5, 277.5), (1, 0, 0), 555.0, 555.0, red)       # image left
    s.rectangle((0.0, 277.5, 277.5), (-1, 0, 0), 555.0, 555.0, green)      # image right
    s.rectangle((277.5, 0.0, 277.5), (0, 1, 0), 555.0, 555.0, white)       # floor
    s.rectangle((277.5, 555.0, 277.5), (0, -1, 0), 555.0, 555.0, white)    # ceiling
    s.rectangle((277.5, 277.5, 555.0), (0, 0, -1), 555.0, 555.0, white)    # back
    s.rectangle((278.0, 554.0, 279.5), (0, -1, 0), 130.0, 105.0, light)
    cube, _ = s.mesh(box_mesh(), white, add_object=False)
    s.mesh_instance(cube, (265.0, 0.0, 295.0), (0.0, 15.0, 0.0), (165.0, 330.0, 165.0), white)
    s.mesh_instance(cube, (130.0, 0.0, 65.0), (0.0, -18.0, 0.0), (165.0, 165.0, 165.0), white)
    if closed:   # a front wall closes the box; the camera moves inside it
        s.rectangle((277.5, 277.5, 0.0), (0, 0, 1), 555.0, 555.0, white)
        s.camera = _pinhole((278.0, 278.0, 20.0), (278.0, 278.0, 555.0), 75.0, width / height)
    else:
        s.camera = _pinhole((278.0, 278.0, -800.0), (278.0, 278.0, 0.0), 40.0, width / height)
    s.background = (0.0, 0.0, 0.0)
    return Workload("cornell_closed" if closed else "cornell", s, width, height, spp, max_bounces)


def spheres_linear_sky(width: int = 64, height: int = 36, spp: int = 4, max_bounces: int = 12,
                       count: int = 40, seed: int = 9) -> Workload:
    """Spheres on a ground sphere under the linear sky (SKY_LINEAR), the kind of scene of
    the reference's ray-tracing-in-one-weekend example: Lambertian, Glossy, DiffuseGlossy,
    sharp and rough metal, smooth and rough glass, and a UV-mapped textured panel."""
    rng = np.random.default_rng(seed)
    s = Scene()
    s.sky = SKY_LINEAR
    s.sphere((0.0, -1000.0, 0.0), 1000.0, s.lambertian((0.5, 0.5, 0.5)))
    s.sphere((0.0, 1.0, 0.0), 1.0, s.dielectric((1.0, 1.0, 1.0), ior=1.5, roughness=0.0))
    s.sphere((-4.0, 1.0, 0.0), 1.0, s.lambertian((0.4, 0.2, 0.1)))
    s.sphere((4.0, 1.0, 0.0), 1.0, s.metal((0.7, 0.6, 0.5), roughness=0.0))
    # a textured panel with explicit corner texture coordinates (rotated, tiled mapping)
    tex = s.texture(checker_texture(16, 4, 0.15, 0.85) * np.array([1.0, 0.8, 0.6]))
    s.rectangle((-6.0, 2.0, -4.0), (0.6, 0.0, 0.8), 6.0, 4.0, s.lambertian((1.0, 1.0, 1.0), texture=tex),
                uvs=((0.0, 0.0), (2.0, 0.5), (1.5, 2.5), (-0.5, 2.0)))
    s.sphere((-2.0, 0.6, 2.5), 0.6, s.glossy((0.9, 0.7, 0.4), roughness=0.2))
    s.sphere((2.0, 0.6, 2.5), 0.6, s.diffuse_glossy((0.2, 0.4, 0.8), (1.0, 1.0, 1.0), weight=0.4, roughness=0.1))
    for _ in range(count):
        c = (rng.uniform(-8, 8), 0.2, rng.uniform(-8, 8))
        k = rng.random()
        if k < 0.4:
            m = s.lambertian(tuple(rng.uniform(0.05, 0.9, 3)))
        elif k < 0.55:
            m = s.glossy(tuple(rng.uniform(0.3, 1.0, 3)), roughness=float(rng.uniform(0.0, 0.6)))
        elif k < 0.7:
            m = s.diffuse_glossy(tuple(rng.uniform(0.05, 0.9, 3)), tuple(rng.uniform(0.5, 1.0, 3)),
                                 weight=float(rng.uniform(0.1, 0.9)), roughness=float(rng.uniform(0.0, 0.5)))
        elif k < 0.85:
            m = s.metal(tuple(rng.uniform(0.5, 1.0, 3)), roughness=float(rng.uniform(0.0, 0.5)))
        else:
            m = s.dielectric((1.0, 1.0, 1.0), ior=1.5, roughness=float(rng.choice([0.0, 0.1])))
        s.sphere(c, 0.2, m)
    s.camera = Camera(position=(13.0, 2.0, 3.0), direction=(-13.0, -2.0, -3.0), up=(0.0, 1.0, 0.0),
                      focal_length_m=0.050, sensor_width_m=0.036, sensor_height_m=0.02025, f_number=16.0,
                      focus_distance_m=10.0)
    s.background = (0.0, 0.0, 0.0)
    return Workload("spheres_linear_sky", s, width, height, spp, max_bounces)


def spot_ies_profile(power: float = 4.0, asym: float = 0.35):
    """A synthetic type-C photometric profile: a cos^power spot around the vertical axis
    (0..180 degrees in 10-degree steps) with a horizontal asymmetry over 0..270 degrees."""
    v = np.arange(0.0, 181.0, 10.0)
    h = np.array([0.0, 90.0, 180.0, 270.0])
    cd = 1000.0 * np.maximum(0.0, np.cos(np.radians(v)))[None, :] ** power * (1.0 + asym * np.cos(np.radians(h)))[:, None]
    return v, h, cd + 5.0


def ies_room(width: int = 48, height: int = 36, spp: int = 4, max_bounces: int = 6) -> Workload:
    """A room lit by two IES-profiled sphere lights (Sphere::setIESProfile) aimed at different
    directions and rotations, plus Lambertian, metal and glass objects."""
    s = Scene()
    white = s.lambertian((0.75, 0.75, 0.75))
    blue = s.lambertian((0.2, 0.3, 0.7))
    s.rectangle((0.0, 0.0, 0.0), (0, 1, 0), 10.0, 10.0, white)
    s.rectangle((0.0, 3.0, -4.0), (0, 0, 1), 10.0, 6.0, blue)
    s.rectangle((-4.5, 3.0, 0.0), (1, 0, 0), 10.0, 6.0, white)
    s.sphere((-1.0, 0.8, 0.0), 0.8, s.metal((0.9, 0.85, 0.8), roughness=0.2))
    s.sphere((1.3, 0.6, 0.8), 0.6, s.dielectric((1.0, 1.0, 1.0), ior=1.5, roughness=0.05))
    s.cube((1.5, 0.5, -1.5), 1.0, 1.0, 1.0, s.lambertian((0.8, 0.4, 0.2)))
    prof = s.ies_profile(*spot_ies_profile())
    s.sphere((-0.5, 3.5, 0.5), 0.2, s.emissive((30.0, 28.0, 24.0)), ies=prof, ies_direction=(0.2, -1.0, -0.1),
             ies_rotation=30.0)
    s.sphere((2.5, 2.5, 1.5), 0.15, s.emissive((25.0, 25.0, 30.0)), ies=prof, ies_direction=(-1.0, -1.0, -0.5),
             ies_rotation=-75.0)
    s.camera = _pinhole((0.0, 2.2, 7.0), (0.0, 1.0, 0.0), 45.0, width / height)
    s.background = (0.0, 0.0, 0.0)
    return Workload("ies_room", s, width, height, spp, max_bounces)


def atmosphere_hills(width: int = 48, height: int = 32, spp: int = 4, max_bounces: int = 3) -> Workload:
    """The atmosphere sky (SKY_ATMOSPHERE, metres as scene units) seen from 1.5 km above a
    6,360-km planet at a low sun: a sky gradient, in-scattering in front of distant hills
    (spheres near the ground), a directional-light sun that drives the atmosphere as
    Scene::syncAtmosphereSunDirection does, and procedural stars in the sky misses."""
    from .desc import SKY_ATMOSPHERE
    s = Scene()
    s.sky = SKY_ATMOSPHERE
    R = 6360e3
    base = np.array([0.0, R, 0.0])
    ground = s.lambertian((0.25, 0.3, 0.18))
    rock = s.lambertian((0.45, 0.4, 0.35))
    s.sphere(tuple(base + np.array([0.0, -1.0e6 + 2.0, 0.0])), 1.0e6, ground)
    for x, z, r in ((-3000.0, 9000.0, 1200.0), (1500.0, 14000.0, 2500.0), (5000.0, 7000.0, 900.0)):
        s.sphere(tuple(base + np.array([x, 0.0, z])), r, rock)
    sun_dir = np.array([-0.55, -0.12, -0.83])   # light travels this way: the sun is low, behind-left
    sun = s.emissive((4.0, 3.8, 3.4))
    s.directional_light(tuple(sun_dir), sun)
    s.atmosphere.update(sun_direction=tuple(-sun_dir), sun_radiance=(4.0, 3.8, 3.4), stars_brightness=0.6)
    s.camera = Camera(position=tuple(base + np.array([0.0, 1500.0, 0.0])), direction=(0.0, -0.02, 1.0),
                      up=(0.0, 1.0, 0.0), focal_length_m=0.024, sensor_width_m=0.036, sensor_height_m=0.024,
                      f_number=8.0, focus_distance_m=10.0, pinhole=True)
    s.meters_per_unit = 1.0
    s.background = (0.0, 0.0, 0.0)
    return Workload("atmosphere_hills", s, width, height, spp, max_bounces)


def checker_texture(size: int = 32, squares: int = 4, lo: float = 0.2, hi: float = 0.8) -> np.ndarray:
    """size x size x 3 checker of `squares` x `squares` cells (the target of the albedo fit)."""
    c = (np.arange(size) * squares // size)
    return np.where(((c[:, None] + c[None, :]) % 2)[..., None] == 0, hi, lo) * np.ones((1, 1, 3))


def cornell_textured(width: int = 256, height: int = 256, spp: int = 64, max_bounces: int = 8,
                     texture: np.ndarray = None, seed: int = 31) -> Workload:
    """The Cornell box with its back wall's albedo given by a 32 x 32 texture on a white
    (1, 1, 1) Lambertian (Material::setTexture): the differentiation workload. The
    texture starts uniform in [0.2, 0.8] unless given; it is texture 0 of the scene."""
    w = cornell(width, height, spp, max_bounces)
    s = w.scene
    if texture is None:
        texture = np.random.default_rng(seed).uniform(0.2, 0.8, (32, 32, 3))
    t = s.texture(texture)
    wall = s.lambertian((1.0, 1.0, 1.0), texture=t)
    back = [o for o in s.objects if tuple(o["position"]) == (277.5, 277.5, 555.0)]
    back[0]["material"] = wall
    return Workload("cornell_textured", s, width, height, spp, max_bounces)


def cornell_rough_panel(width: int = 64, height: int = 64, spp: int = 64, max_bounces: int = 8,
                        roughness: np.ndarray = None, seed: int = 41) -> Workload:
    """The textured Cornell box (texture 0: back-wall albedo) with a GGX Metal panel whose
    roughness comes from a 64 x 64 map (texture 1, red channel; U[0.08, 0.25] unless given),
    tilted to reflect the ceiling light toward the camera: the roughness-gradient workload
    (Metal roughness textures are an extension; the reference's Metal roughness is a scalar)."""
    w = cornell_textured(width, height, spp, max_bounces)
    s = w.scene
    if roughness is None:
        roughness = np.repeat(np.random.default_rng(seed).uniform(0.08, 0.25, (64, 64, 1)), 3, axis=2)
    t = s.texture(roughness)
    panel = s.metal((0.95, 0.9, 0.85), roughness=0.15, roughness_texture=t)
    n = np.array([-0.13, 0.49, -0.86])   # bisects the directions to the camera and to the light
    s.rectangle((330.0, 300.0, 420.0), tuple(n / np.linalg.norm(n)), 220.0, 260.0, panel)
    return Workload("cornell_rough_panel", s, width, height, spp, max_bounces)


def sky_environment(width: int = 1024, height: int = 512, seed: int = 7, sun_peak: float = 5.0e4,
                    sun_diameter_deg: float = 0.5):
    """Equirect RGB sky: zenith-to-horizon gradient, dark ground, seeded sun lobe.

    Texel (x, y) maps to direction through EnvironmentMap::uvToDirection
    (src/core/EnvironmentMap.cpp:616-623): u = (x+0.5)/W, v = 1-(y+0.5)/H.
    """
    rng = np.random.default_rng(seed)
    u = (np.arange(width) + 0.5) / width
    v = 1.0 - (np.arange(height) + 0.5) / height
    phi = (u - 0.5) * 2.0 * np.pi
    yy = np.sin((v - 0.5) * np.pi)
    r = np.sqrt(np.maximum(0.0, 1.0 - yy * yy))
    D = np.stack([np.outer(r, np.cos(phi)), np.repeat(yy[:, None], width, 1), np.outer(r, np.sin(phi))], -1)
    up = np.clip(D[..., 1], 0.0, 1.0)[..., None]
    zenith = np.array([0.25, 0.45, 0.95])
    horizon = np.array([0.95, 0.95, 1.0])
    ground = np.array([0.18, 0.16, 0.14])
    sky = horizon * (1 - up) + zenith * up
    img = np.where(D[..., 1:2] >= 0.0, sky, ground)
    elev = math.radians(rng.uniform(20.0, 50.0))
    azim = rng.uniform(0.0, 2.0 * math.pi)
    sun = np.array([math.cos(elev) * math.cos(azim), math.sin(elev), math.cos(elev) * math.sin(azim)])
    ang = np.degrees(np.arccos(np.clip(D @ sun, -1.0, 1.0)))
    lobe = np.exp(-0.5 * (ang / (sun_diameter_deg / 2.0)) ** 2)
    img = img + sun_peak * lobe[..., None] * np.array([1.0, 0.95, 0.85])
    return np.ascontiguousarray(img), sun


def mesh_glossy(width: int = 1920, height: int = 1080, spp: int = 64, max_bounces: int = 12,
                level: int = 8, seed: int = 11) -> Workload:
    s = Scene()
    glass = s.dielectric((1.0, 1.0, 1.0), ior=1.5, roughness=0.1)
    metal = s.metal((0.85, 0.8, 0.75), roughness=0.3)
    v, f = icosphere(level)
    disp = 1.0 + 0.1 * value_noise(v, seed)
    v = v * disp[:, None]
    s.mesh(v[f], glass)
    g = 12.0
    y = -1.15
    quad = np.array([[[-g, y, -g], [g, y, g], [g, y, -g]], [[-g, y, -g], [-g, y, g], [g, y, g]]], np.float64)
    s.mesh(quad, metal)
    env, _ = sky_environment(seed=seed + 1)
    s.set_environment(env, strength=1.0)
    s.camera = Camera(position=(0.0, 0.35, 4.2), direction=(0.0, -0.35 * 0.25, -4.2), up=(0.0, 1.0, 0.0),
                      focal_length_m=0.050, sensor_width_m=0.036, sensor_height_m=0.02025, f_number=2.8,
                      focus_distance_m=4.2)
    return Workload("mesh_glossy", s, width, height, spp, max_bounces)


def random_rotation_euler_xyz(rng, n):
    """Uniform random rotations (Shoemake quaternions) as Euler angles in degrees for
    MeshInstance's rotate(): R = Rz(z) Ry(y) Rx(x) (src/core/Hittables/MeshInstance.cpp:74-94)."""
    u1, u2, u3 = rng.random(n), rng.random(n), rng.random(n)
    q = np.stack([np.sqrt(1 - u1) * np.sin(2 * np.pi * u2), np.sqrt(1 - u1) * np.cos(2 * np.pi * u2),
                  np.sqrt(u1) * np.sin(2 * np.pi * u3), np.sqrt(u1) * np.cos(2 * np.pi * u3)], 1)
    x, y, z, w = q.T
    r20 = 2 * (x * z - w * y)
    r21 = 2 * (y * z + w * x)
    r22 = 1 - 2 * (x * x + y * y)
    r10 = 2 * (x * y + w * z)
    r00 = 1 - 2 * (y * y + z * z)
    ay = np.arcsin(np.clip(-r20, -1, 1))
    ax = np.arctan2(r21, r22)
    az = np.arctan2(r10, r00)
    return np.degrees(np.stack([ax, ay, az], 1))


def instancing_volumes(width: int = 1280, height: int = 720, spp: int = 32, max_bounces: int = 16,
                       count: int = 100_000, seed: int = 23) -> Workload:
    rng = np.random.default_rng(seed)
    s = Scene()
    palette = [s.lambertian(tuple(rng.uniform(0.2, 0.85, 3))) for _ in range(6)]
    palette.append(s.metal((0.9, 0.85, 0.7), roughness=0.3))
    palette.append(s.dielectric((1.0, 1.0, 1.0), ior=1.5, roughness=0.1))
    tor, _ = s.mesh(torus_mesh(), palette[0], add_object=False)
    pos = rng.uniform(-48.0, 48.0, (count, 3))
    rot = random_rotation_euler_xyz(rng, count)
    sc = np.exp(rng.normal(0.0, 0.3, count)) * 0.8
    mat = rng.integers(0, len(palette), count)
    for i in range(count):
        sv = float(sc[i])
        s.mesh_instance(tor, tuple(pos[i]), tuple(rot[i]), (sv, sv, sv), palette[int(mat[i])])
    hg = s.henyey_greenstein((0.8, 0.8, 0.8), 0.6)
    s.volume_cube((0.0, 0.0, 0.0), 100.0, 100.0, 100.0, hg, 0.05)
    s.sphere((-20.0, 30.0, -10.0), 3.0, s.emissive((40.0, 36.0, 30.0)))
    s.sphere((25.0, -10.0, 15.0), 2.0, s.emissive((20.0, 30.0, 45.0)))
    s.directional_light((-0.3, -1.0, -0.2), s.emissive((2.0, 2.0, 2.0)))
    s.camera = Camera(position=(0.0, 5.0, 49.0), direction=(0.0, -0.1, -1.0), up=(0.0, 1.0, 0.0),
                      focal_length_m=0.035, sensor_width_m=0.036, sensor_height_m=0.02025, f_number=8.0,
                      focus_distance_m=30.0, pinhole=True)
    return Workload("instancing_volumes", s, width, height, spp, max_bounces)


def tiny_mixed(width: int = 24, height: int = 18, spp: int = 4, max_bounces: int = 6) -> Workload:
    """Small scene touching every object kind and material on the path (parity tests)."""
    rng = np.random.default_rng(5)
    s = Scene()
    white = s.lambertian((0.73, 0.73, 0.73))
    red = s.lambertian((0.65, 0.05, 0.05))
    s.rectangle((0.0, -1.0, 0.0), (0, 1, 0), 8.0, 8.0, white)
    s.rectangle((0.0, 1.0, -3.0), (0, 0, 1), 8.0, 4.0, red)
    s.sphere((-1.2, -0.4, 0.0), 0.6, s.metal((0.9, 0.8, 0.6), roughness=0.25))
    s.sphere((0.2, -0.5, 0.6), 0.5, s.dielectric((1.0, 1.0, 1.0), ior=1.5, roughness=0.0))
    s.sphere((1.4, -0.5, -0.4), 0.5, s.principled((0.3, 0.6, 0.8), metallic=0.2, roughness=0.35, clearcoat=0.5,
                                                   sheen=0.3))
    s.cube((-0.2, -0.6, -1.4), 0.7, 0.8, 0.7, s.dielectric((0.9, 1.0, 0.9), ior=1.45, roughness=0.2))
    s.sphere((0.0, 2.2, 0.5), 0.35, s.emissive((12.0, 11.0, 9.0)))
    s.rectangle((1.5, 1.8, 1.0), (0, -1, 0), 0.8, 0.5, s.emissive((6.0, 6.0, 8.0)))
    tri = box_mesh() - 0.5
    m, _ = s.mesh(tri * 0.4 + np.array([1.0, 0.2, 1.2]), s.metal((0.8, 0.8, 0.8), roughness=0.0))
    s.mesh_instance(m, (-1.5, 0.2, 1.0), tuple(rng.uniform(-40, 40, 3)), (0.7, 1.2, 0.9), white)
    s.volume_sphere((1.0, -0.3, 1.4), 0.45, s.henyey_greenstein((0.8, 0.8, 0.8), 0.5), 1.5)
    s.directional_light((0.3, -1.0, -0.4), s.emissive((1.5, 1.4, 1.2)))
    s.camera = _pinhole((0.0, 0.5, 5.0), (0.0, -0.2, 0.0), 50.0, width / height)
    s.background = (0.05, 0.06, 0.08)
    return Workload("tiny_mixed", s, width, height, spp, max_bounces)


def caustic_pool(width: int = 64, height: int = 48, spp: int = 4, max_bounces: int = 8, photons: int = 40000,
                 passes: int = 4, radius_meters: float = 0.08, alpha: float = 0.7) -> Workload:
    """Caustics (CausticPhotonMap): smooth and rough glass, a rough metal torus, a transmissive
    Principled block and a rough-glass wavy sheet over Lambertian / diffuse-glossy receivers and
    a scattering volume, lit by every emitter kind the photon pass samples (rectangle, sphere,
    emissive mesh, emissive non-uniformly scaled instance, directional light)."""
    s = Scene()
    floor = s.lambertian((0.8, 0.78, 0.74))
    wall = s.lambertian((0.35, 0.55, 0.7))
    s.rectangle((0.0, 0.0, 0.0), (0, 1, 0), 8.0, 8.0, floor)
    s.rectangle((0.0, 2.0, -3.0), (0, 0, 1), 8.0, 4.0, wall)
    s.rectangle((3.0, 1.0, -1.5), (-1, 0, 0), 3.0, 2.0, s.diffuse_glossy((0.6, 0.5, 0.4), weight=0.3,
                                                                         roughness=0.4))
    s.sphere((0.0, 0.7, 0.0), 0.6, s.dielectric((1.0, 1.0, 1.0), ior=1.5, roughness=0.0))
    tor, _ = s.mesh(torus_mesh(24, 12, 0.5, 0.12), s.metal((0.95, 0.85, 0.6), roughness=0.1), add_object=False)
    s.mesh_instance(tor, (-1.6, 0.35, 0.6), (70.0, 20.0, 0.0), (1.0, 1.0, 1.0), s.metal((0.95, 0.85, 0.6),
                                                                                     roughness=0.1))
    s.cube((1.6, 0.4, 0.8), 0.6, 0.8, 0.6, s.principled((0.9, 0.95, 1.0), roughness=0.05, transmission=0.9,
                                                         ior=1.45))
    xs = np.linspace(-1.0, 1.0, 9)
    zs = np.linspace(-0.6, 0.6, 7)
    X, Z = np.meshgrid(xs, zs)
    Y = 1.6 + 0.08 * np.sin(3.0 * X) * np.cos(4.0 * Z)
    P = np.stack([X + 0.8, Y, Z - 1.4], -1)
    quads = []
    for i in range(len(zs) - 1):
        for j in range(len(xs) - 1):
            a, b, c, d = P[i, j], P[i, j + 1], P[i + 1, j + 1], P[i + 1, j]
            quads += [[a, b, c], [a, c, d]]
    s.mesh(np.array(quads), s.dielectric((0.85, 0.95, 1.0), ior=1.33, roughness=0.05))
    s.volume_sphere((-0.4, 0.5, 1.5), 0.4, s.henyey_greenstein((0.8, 0.85, 0.9), 0.4), 1.2)
    s.rectangle((0.0, 3.2, 0.0), (0, -1, 0), 0.6, 0.6, s.emissive((30.0, 29.0, 26.0)))
    s.sphere((1.8, 2.6, 1.2), 0.15, s.emissive((40.0, 36.0, 30.0)))
    panel = np.array([[[-0.3, 0.0, 0.0], [0.3, 0.0, 0.0], [0.3, 0.0, 0.3]],
                      [[-0.3, 0.0, 0.0], [0.3, 0.0, 0.3], [-0.3, 0.0, 0.3]]])
    s.mesh(panel + np.array([-1.8, 3.0, -1.0]), s.emissive((12.0, 14.0, 18.0)))
    pm, _ = s.mesh(panel, s.emissive((10.0, 9.0, 7.0)), add_object=False)
    s.mesh_instance(pm, (1.0, 3.1, -2.0), (180.0, 10.0, 0.0), (1.5, 1.0, 0.6), s.emissive((10.0, 9.0, 7.0)))
    s.directional_light((-0.3, -1.0, -0.2), s.emissive((1.2, 1.15, 1.0)))
    s.camera = _pinhole((0.0, 2.6, 4.6), (0.0, 0.4, 0.0), 50.0, width / height)
    s.background = (0.02, 0.025, 0.03)
    s.set_caustics(photons=photons, passes=passes, radius_meters=radius_meters, alpha=alpha)
    return Workload("caustic_pool", s, width, height, spp, max_bounces)


def batch_workloads(count: int = 48, seed: int = 4242, side_range=(128, 1024), spp_range=(4, 256)) -> list:
    """Many independent scenes for luz_gpu_batch_render: triangle counts log-uniform in
    [1e3, 1e6] (displaced icospheres of the nearest level), square images with sides
    log-uniform in side_range, spp log-uniform in spp_range, max depth uniform in [4, 16]."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        tris = float(np.exp(rng.uniform(np.log(1e3), np.log(1e6))))
        level = int(np.clip(np.round(np.log(tris / 20.0) / np.log(4.0)), 3, 8))
        side = int(np.exp(rng.uniform(np.log(side_range[0]), np.log(side_range[1]))))
        spp = int(np.exp(rng.uniform(np.log(spp_range[0]), np.log(spp_range[1]))))
        depth = int(rng.integers(4, 17))
        w = mesh_glossy(side, side, spp, depth, level=level, seed=seed + i)
        w.name = f"batch{i}"
        out.append(w)
    return out


WORKLOADS = {
    "cornell": cornell,
    "mesh_glossy": mesh_glossy,
    "instancing_volumes": instancing_volumes,
    "tiny_mixed": tiny_mixed,
}
