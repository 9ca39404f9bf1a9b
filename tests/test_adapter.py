"""The drop-in adapter's scene export (rainbow_b200/adapter/scene_export.cpp),
compiled against the reference's headers: a reference `scene` and
`perspective_camera` (built by the oracle harness) exported back to the C ABI
must describe the same scene: rb_bvh_build on the export gives the reference's
own tree (geometry, transforms and mesh sharing, so also the two-level case),
every entity keeps its material and emitter parameters, and the camera its
matrices."""
import numpy as np
import pytest

import rainbow_b200 as rb
from oracle import ref
from tests.helpers import (extra_materials_scene, layered_scene, mixture_scene, real_textured_scene, subsurface_scene,
                           textured_scene, two_level_scene)

pytestmark = pytest.mark.skipif(not ref.adapter_available(), reason="oracle/_ref/libadapter_check.so not built")


def _scene(name):
    if name == "box":
        return rb.generate_scene(rb.RB_SCENE_BOX, width=32, height=32)
    if name == "spheres_materials":
        return extra_materials_scene(rb.generate_scene(rb.RB_SCENE_SPHERES, seed=1, width=48, height=40, num_spheres=12,
                                                       subdivision=2))
    if name == "spheres_layered":
        return layered_scene(rb.generate_scene(rb.RB_SCENE_SPHERES, seed=1, width=48, height=40, num_spheres=12,
                                               subdivision=2))
    if name == "spheres_mixture":
        return mixture_scene(rb.generate_scene(rb.RB_SCENE_SPHERES, seed=1, width=48, height=40, num_spheres=12,
                                               subdivision=2))
    if name == "spheres_subsurface":
        return subsurface_scene(rb.generate_scene(rb.RB_SCENE_SPHERES, seed=1, width=48, height=40, num_spheres=12,
                                                  subdivision=2))
    if name == "fog":
        return rb.generate_scene(rb.RB_SCENE_FOG, seed=4, width=40, height=30, num_spheres=6, subdivision=2)
    return two_level_scene()


@pytest.mark.parametrize("name", ["box", "spheres_materials", "spheres_layered", "spheres_mixture", "spheres_subsurface",
                                  "fog", "two_level"])
def test_export_describes_the_reference_scene(name):
    scene = _scene(name)
    R = ref.RefScene(scene)
    (nodes, pe, pi), mats, ems, has, cam = ref.adapter_export(R, rb.MaterialDesc, rb._native.EmitterDesc, rb.CameraDesc)
    rn, rpe, rpi = R.bvh()
    assert np.array_equal(nodes.view(np.uint32), rn.view(np.uint32)) and np.array_equal(pe, rpe) and np.array_equal(pi, rpi)
    d = scene.desc
    for e in range(d.num_entities):
        ent = d.entities[e]
        assert bool(has[e, 0]) == (ent.material >= 0) and bool(has[e, 1]) == (ent.emitter >= 0), e
        if ent.material >= 0 and d.materials[ent.material].kind != rb.RB_MATERIAL_MIXTURE:
            assert bytes(mats[e]) == bytes(d.materials[ent.material]), f"entity {e}: material differs"
        if ent.emitter >= 0:
            assert bytes(ems[e]) == bytes(d.emitters[ent.emitter]), f"entity {e}: emitter differs"
    for field in ("raster_to_camera", "camera_to_world"):
        assert np.array_equal(np.array(getattr(cam, field)[:], np.float32), np.array(getattr(scene.camera, field)[:], np.float32))
    assert (cam.width, cam.height, cam.lens_radius) == (scene.camera.width, scene.camera.height, scene.camera.lens_radius)


def _expand(mats, k):
    """A material with its mixture components resolved (their indices replaced by the components themselves)."""
    m = mats[k]
    if m.kind != rb.RB_MATERIAL_MIXTURE:
        return bytes(m)
    own = rb.MaterialDesc.from_buffer_copy(bytes(m))
    own.components[0] = own.components[1] = 0
    return (bytes(own), _expand(mats, m.components[0]), _expand(mats, m.components[1]))


def test_export_keeps_mixtures():
    """Mixtures (nested too) are exported with their components, weights and
    the components' parameters; shared components stay shared."""
    scene = _scene("spheres_mixture")
    R = ref.RefScene(scene)
    mats, ent = ref.adapter_export_materials(R, rb.MaterialDesc)
    d = scene.desc
    assert ent.shape[0] == d.num_entities
    seen = 0
    for e in range(d.num_entities):
        k = d.entities[e].material
        assert (k >= 0) == (ent[e] >= 0)
        if k >= 0:
            assert _expand(mats, int(ent[e])) == _expand(d.materials, k), f"entity {e}"
            seen += d.materials[k].kind == rb.RB_MATERIAL_MIXTURE
    assert seen > 0


_TEX_FIELDS = ("diffuse_texture", "reflectance_texture", "transmission_texture", "specular_texture", "opacity_texture",
               "eta_texture", "k_texture", "mfp_texture")


def _resolve_texture(descs, texels, ref, channel0=False):
    """Texture ref (index + 1) with its inputs resolved: an image's shape and texel bytes (channel 0 alone for
    a mixture's real-valued alpha), or a composite's kind, resolved inputs and the constants it reads."""
    d = descs[ref - 1]
    if d.kind == rb.RB_TEXTURE_IMAGE:
        a = texels(ref - 1)
        return ("image", a.shape[:2], np.ascontiguousarray(a[..., 0] if channel0 else a).tobytes())
    mixture = d.kind == rb.RB_TEXTURE_MIXTURE
    out = [d.kind]
    for i in range(3 if mixture else 2):
        alpha = mixture and i == 2
        if d.inputs[i]:
            out.append(_resolve_texture(descs, texels, d.inputs[i], channel0=alpha))
        else:
            out.append((d.constants[i][0],) if alpha else tuple(d.constants[i]))
    return tuple(out)


_REAL_FIELDS = ("roughness_u_texture", "roughness_v_texture", "ior_texture", "sigma_texture")


@pytest.mark.parametrize("make", [textured_scene, real_textured_scene])
def test_export_keeps_image_textures(make):
    """Image, scale and mixture textures of material spectra, and image textures
    of real parameters (roughness, IOR, sigma: image_texture2d<real>, exported as
    RGB images read at channel 0), are exported with the same texels, inputs and
    constants, each texture once, and the material's other parameters kept."""
    scene = make(rb.generate_scene(rb.RB_SCENE_SPHERES, seed=1, width=48, height=40, num_spheres=12, subdivision=2))
    R = ref.RefScene(scene)
    mats, ent = ref.adapter_export_materials(R, rb.MaterialDesc)
    exported = ref.adapter_export_textures(R, rb.TextureDesc)
    d = scene.desc
    src_descs = [d.textures[t] for t in range(d.num_textures)]

    def src_texels(t):
        return np.ctypeslib.as_array(d.textures[t].rgb, (d.textures[t].height, d.textures[t].width, 3))

    exp_descs = [e[0] for e in exported]
    used = 0
    for e in range(d.num_entities):
        k = d.entities[e].material
        if k < 0:
            continue
        a = rb.MaterialDesc.from_buffer_copy(bytes(mats[int(ent[e])]))
        b = rb.MaterialDesc.from_buffer_copy(bytes(d.materials[k]))
        for f in _TEX_FIELDS:
            ra, rb_ = getattr(a, f), getattr(b, f)
            assert (ra == 0) == (rb_ == 0), (e, f)
            if ra:
                assert _resolve_texture(exp_descs, lambda t: exported[t][1], ra) == \
                    _resolve_texture(src_descs, src_texels, rb_), (e, f)
                used += 1
                value = f[:-len("_texture")]  # the constant the texture replaces is not read
                getattr(a, value)[:] = (0.0, 0.0, 0.0)
                getattr(b, value)[:] = (0.0, 0.0, 0.0)
            setattr(a, f, 0)
            setattr(b, f, 0)
        for f in _REAL_FIELDS:
            ra, rb_ = getattr(a, f), getattr(b, f)
            assert (ra == 0) == (rb_ == 0), (e, f)
            if ra:
                assert _resolve_texture(exp_descs, lambda t: exported[t][1], ra, channel0=True) == \
                    _resolve_texture(src_descs, src_texels, rb_, channel0=True), (e, f)
                used += 1
                setattr(a, f[:-len("_texture")], 0.0)  # the constant the texture replaces is not read
                setattr(b, f[:-len("_texture")], 0.0)
            setattr(a, f, 0)
            setattr(b, f, 0)
        if a.kind == rb.RB_MATERIAL_TRANSLUCENT:  # one roughness, exported as both
            a.roughness_v = b.roughness_v
        assert bytes(a) == bytes(b), f"entity {e}"
    kinds = {dd.kind for dd in exp_descs}
    assert used > 0
    if make is textured_scene:
        assert kinds == {rb.RB_TEXTURE_IMAGE, rb.RB_TEXTURE_SCALE, rb.RB_TEXTURE_MIXTURE}
