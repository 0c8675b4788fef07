"""Scene validation mirrors the reference's std::invalid_argument messages."""
import numpy as np
import pytest

from luz_b200 import native
from luz_b200.desc import Scene


def packs(sc):
    return native.Pack(sc.build())


@pytest.mark.parametrize("make,msg", [
    (lambda s: s.sphere((0, 0, 0), 1, s.metal((1, 1, 1), roughness=1.5)), "Metal roughness must be finite and in [0,1]."),
    (lambda s: s.sphere((0, 0, 0), 1, s.dielectric(ior=-1.0)), "Dielectric refractive index must be finite and positive."),
    (lambda s: s.volume_sphere((0, 0, 0), 1, s.henyey_greenstein((1, 1, 1), 0.995), 1.0),
     "Volume anisotropy must be finite and between -0.99 and 0.99."),
    (lambda s: s.volume_sphere((0, 0, 0), 1, s.isotropic((1, 1, 1)), 0.0), "Volume density must be finite and positive."),
    (lambda s: s.sphere((0, 0, 0), 1, s.principled((1, 1, 1), metallic=2.0)), "Principled metallic must be finite and in [0,1]."),
    (lambda s: s.sphere((0, 0, 0), 1, s.glossy((1, 1, 1), roughness=-0.1)), "Glossy roughness must be finite and in [0,1]."),
    (lambda s: s.sphere((0, 0, 0), 1, s.diffuse_glossy(weight=1.5)), "Diffuse-glossy weight must be finite and in [0,1]."),
    (lambda s: s.sphere((0, 0, 0), 1, s.diffuse_glossy(roughness=float("nan"))),
     "Diffuse-glossy roughness must be finite and in [0,1]."),
])
def test_invalid_parameters_rejected(make, msg):
    s = Scene()
    make(s)
    with pytest.raises(native.LuzError) as e:
        packs(s)
    assert msg in str(e.value) and e.value.code == -1


def _ies_scene(**kw):
    from luz_b200.scenes import spot_ies_profile
    s = Scene()
    v, h, c = spot_ies_profile()
    prof = s.ies_profile(kw.pop("v", v), h, kw.pop("c", c))
    s.sphere((0, 2, 0), 0.2, s.emissive((5, 5, 5)), ies=kw.pop("ies", prof), **kw)
    return s


@pytest.mark.parametrize("kw,msg", [
    (dict(ies_direction=(0, 0, 0)), "IES profile direction must be non-zero."),
    (dict(ies_rotation=float("inf")), "IES profile rotation must be finite."),
    (dict(ies=3), "IES profile index out of range."),
    (dict(v=[0.0, 10.0, 10.0] + list(range(20, 181, 10))), "IES vertical angles must be strictly increasing."),
    (dict(c=-1.0 * np.ones((4, 19))), "IES profile candela values must be finite and non-negative."),
    (dict(c=np.zeros((4, 19))), "IES profile has zero luminous flux."),
])
def test_ies_validation(kw, msg):
    with pytest.raises(native.LuzError) as e:
        packs(_ies_scene(**kw))
    assert msg in str(e.value) and e.value.code == -1


def test_unknown_sky_rejected():
    s = Scene()
    s.sky = 7
    with pytest.raises(native.LuzError) as e:
        packs(s)
    assert e.value.code == -1


@pytest.mark.parametrize("kw,msg", [
    (dict(earth_radius=-1.0), "Earth radius must be positive."),
    (dict(atmosphere_radius=6000e3), "Atmosphere radius must be larger than Earth radius."),
    (dict(h_r=0.0), "Atmosphere HR must be positive."),
    (dict(samples=0), "Atmosphere sample count must be positive."),
    (dict(sun_direction=(0.0, 0.0, 0.0)), "Atmosphere sun direction must be finite and non-zero."),
    (dict(sun_radiance=(1.0, -1.0, 1.0)), "Atmosphere sun radiance must be finite and non-negative."),
])
def test_atmosphere_validation(kw, msg):
    from luz_b200.desc import SKY_ATMOSPHERE
    s = Scene()
    s.sky = SKY_ATMOSPHERE
    s.atmosphere.update(kw)
    with pytest.raises(native.LuzError) as e:
        packs(s)
    assert msg in str(e.value) and e.value.code == -1


def test_camera_validation():
    s = Scene()
    s.camera.focal_length_m = 0.0
    with pytest.raises(native.LuzError) as e:
        packs(s)
    assert "focal length" in str(e.value)


def test_material_index_out_of_range():
    s = Scene()
    s.sphere((0, 0, 0), 1, 5)
    with pytest.raises(native.LuzError):
        packs(s)


def test_light_list_and_weights():
    s = Scene()
    e = s.emissive((1, 1, 1))
    s.rectangle((0, 0, 0), (0, 1, 0), 2, 3, e)
    s.sphere((0, 0, 0), 1, e)
    s.directional_light((0, -1, 0), e)
    s.sphere((3, 0, 0), 1, s.lambertian((1, 1, 1)))
    assert packs(s).info().light_count == 3


@pytest.mark.parametrize("kw,msg", [
    (dict(photons=-1), "Caustic photon count must be non-negative."),
    (dict(passes=0), "Caustic pass count must be positive."),
    (dict(radius_meters=0.0), "Caustic radius must be finite and positive."),
    (dict(radius_meters=float("inf")), "Caustic radius must be finite and positive."),
    (dict(alpha=1.5), "Caustic alpha must be finite and in (0,1]."),
    (dict(alpha=0.0), "Caustic alpha must be finite and in (0,1]."),
])
def test_caustic_settings_validation(kw, msg):
    """Scene::setCausticPhotonCount / PassCount / RadiusMeters / Alpha (src/scene/Scene.cpp:317-360)."""
    s = Scene()
    s.sphere((0, 2, 0), 0.2, s.emissive((5, 5, 5)))
    s.set_caustics(**kw)
    with pytest.raises(native.LuzError) as e:
        packs(s)
    assert msg in str(e.value) and e.value.code == -1
    s.caustics["enabled"] = 0          # settings are read only with caustics on
    packs(s)
