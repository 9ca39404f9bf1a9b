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
from tests.helpers import extra_materials_scene, layered_scene, two_level_scene

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
    if name == "fog":
        return rb.generate_scene(rb.RB_SCENE_FOG, seed=4, width=40, height=30, num_spheres=6, subdivision=2)
    return two_level_scene()


@pytest.mark.parametrize("name", ["box", "spheres_materials", "spheres_layered", "fog", "two_level"])
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
        if ent.material >= 0:
            assert bytes(mats[e]) == bytes(d.materials[ent.material]), f"entity {e}: material differs"
        if ent.emitter >= 0:
            assert bytes(ems[e]) == bytes(d.emitters[ent.emitter]), f"entity {e}: emitter differs"
    for field in ("raster_to_camera", "camera_to_world"):
        assert np.array_equal(np.array(getattr(cam, field)[:], np.float32), np.array(getattr(scene.camera, field)[:], np.float32))
    assert (cam.width, cam.height, cam.lens_radius) == (scene.camera.width, scene.camera.height, scene.camera.lens_radius)
