"""Host pieces of the boundary: the BVH builder reproduces the reference's own
tree, the scene generator is deterministic with the configured sizes, and the
camera matrices equal the reference camera's."""
import ctypes
import hashlib

import numpy as np
import pytest

import rainbow_b200 as rb
from oracle import ref
from tests import golden
from tests.helpers import scene_from_params


@pytest.mark.parametrize("name", ["box_rays", "spheres_rays"])
def test_bvh_equals_reference_tree(name):
    fx = golden.load(name)
    b = rb.build_bvh(scene_from_params(fx["params"]))
    assert np.array_equal(b.nodes.view(np.uint32), fx["bvh_nodes"].view(np.uint32))
    assert np.array_equal(b.prim_entity, fx["bvh_prim_entity"])
    assert np.array_equal(b.prim_index, fx["bvh_prim_index"])


def test_bvh_full_size_equals_reference_digest():
    fx = golden.load("bvh_c2")
    b = rb.build_bvh(scene_from_params(fx["params"]))
    assert b.nodes.shape[0] == int(fx["num_nodes"]) and b.prim_entity.shape[0] == int(fx["num_prims"]) == 1024010
    h = hashlib.sha256()
    for a in (b.nodes.astype(np.float32).view(np.uint32), b.prim_entity, b.prim_index):
        h.update(np.ascontiguousarray(a).tobytes())
    assert h.hexdigest() == str(fx["digest"])
    assert 18 <= b.depth <= 30


@pytest.mark.parametrize("name", ["box_rays", "spheres_rays"])
def test_camera_matrices_equal_reference(name):
    fx = golden.load(name)
    cam = scene_from_params(fx["params"]).camera
    assert np.array_equal(np.array(cam.raster_to_camera[:], np.float32).view(np.uint32), fx["raster_to_camera"].view(np.uint32))
    assert np.array_equal(np.array(cam.camera_to_world[:], np.float32).view(np.uint32), fx["camera_to_world"].view(np.uint32))


def test_scene_sizes_and_determinism():
    box = rb.generate_scene(rb.RB_SCENE_BOX, width=256, height=256)
    assert box.num_triangles == 32
    a = rb.generate_scene(rb.RB_SCENE_SPHERES, seed=1, width=64, height=64, num_spheres=200, subdivision=4)
    assert a.num_triangles == 200 * 5120 + 2 + 4 * 2
    b = rb.generate_scene(rb.RB_SCENE_SPHERES, seed=1, width=64, height=64, num_spheres=200, subdivision=4)
    for i in (0, 57, 199):
        ma, mb = a.desc.meshes[i], b.desc.meshes[i]
        pa = np.ctypeslib.as_array(ma.positions, (ma.num_vertices * 3,))
        pb = np.ctypeslib.as_array(mb.positions, (mb.num_vertices * 3,))
        assert np.array_equal(pa, pb)
    c = rb.generate_scene(rb.RB_SCENE_SPHERES, seed=2, width=64, height=64, num_spheres=200, subdivision=4)
    pc = np.ctypeslib.as_array(c.desc.meshes[0].positions, (c.desc.meshes[0].num_vertices * 3,))
    assert not np.array_equal(pc, np.ctypeslib.as_array(a.desc.meshes[0].positions, (a.desc.meshes[0].num_vertices * 3,)))
    room = rb.generate_scene(rb.RB_SCENE_SLIT_ROOM, seed=3, width=64, height=64, num_spheres=40, subdivision=3)
    assert room.desc.num_emitters == 1


def test_bvh_shared_mesh_is_two_level_and_bad_indices_rejected():
    s = rb.generate_scene(rb.RB_SCENE_BOX, width=16, height=16)
    d = rb.SceneDesc()
    ctypes.pointer(d)[0] = s.desc
    ents = (rb._native.EntityDesc * s.desc.num_entities)()
    for i in range(s.desc.num_entities):
        ents[i] = s.desc.entities[i]
    ents[1].mesh = ents[0].mesh  # one shape referenced twice: the reference builds a two-level tree
    d.entities = ctypes.cast(ents, ctypes.POINTER(rb._native.EntityDesc))
    h = ctypes.c_void_p()
    assert rb.lib().rb_bvh_build(ctypes.byref(d), ctypes.byref(h)) == 0
    count = ctypes.c_uint32()
    assert rb.lib().rb_bvh_mesh_tree_count(h, ctypes.byref(count)) == 0 and count.value == 1
    rb.lib().rb_bvh_free(h)
    assert rb.lib().rb_bvh_build(None, ctypes.byref(h)) == 1
    bad = (rb._native.MeshDesc * s.desc.num_meshes)()
    for i in range(s.desc.num_meshes):
        bad[i] = s.desc.meshes[i]
    idx = (ctypes.c_uint32 * 3)(0, 1, 10 ** 6)
    bad[0].indices = ctypes.cast(idx, ctypes.POINTER(ctypes.c_uint32))
    bad[0].num_triangles = 1
    d.meshes = ctypes.cast(bad, ctypes.POINTER(rb._native.MeshDesc))
    assert rb.lib().rb_bvh_build(ctypes.byref(d), ctypes.byref(h)) == 1


@pytest.mark.skipif(not ref.available(), reason="reference oracle not built")
def test_areas_equal_reference():
    fx = golden.load("spheres_rays")
    R = ref.RefScene(scene_from_params(fx["params"]))
    assert np.array_equal(R.areas(), fx["areas"])


@pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("kind,n,sub", [(rb.RB_SCENE_BOX, 0, 0), (rb.RB_SCENE_SPHERES, 20, 2), (rb.RB_SCENE_FOG, 6, 2)])
def test_oracle_generated_scene_equals_product_scene(kind, n, sub):
    """The timed CPU reference builds its scene with the generator compiled into
    the oracle library (so it loads nothing of the product); that scene must be
    the one the GPU arm renders: same reference BVH, camera and triangle count."""
    a = ref.RefScene.generated(kind, 5, 40, 30, n, sub)
    sc = rb.generate_scene(kind, seed=5, width=40, height=30, num_spheres=n, subdivision=sub)
    b = ref.RefScene(sc)
    assert a.triangles == sc.num_triangles
    for x, y in zip(a.bvh(), b.bvh()):
        assert np.array_equal(x.view(np.uint32), y.view(np.uint32))
    for x, y in zip(a.camera_matrices(), b.camera_matrices()):
        assert np.array_equal(x.view(np.uint32), y.view(np.uint32))
