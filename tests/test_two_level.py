"""The reference's two-level tree (scene::build_accelerator, scene.cpp:41-75;
mesh::build_accelerator, mesh.cpp:159-172): a mesh used by several entities,
or with more than 2^17 triangles, is held whole by one scene-tree leaf and
gets its own tree in local space. The builder must reproduce both levels bit
for bit, and the traversal (host build of the kernels' code) must hit what
scene::intersect hits: entity, triangle and the bits of t."""
import numpy as np
import pytest

import rainbow_b200 as rb
from oracle import ref
from tests.helpers import HostPaths, assert_hits_equal, random_rays, two_level_scene

pytestmark = pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")


@pytest.fixture(scope="module")
def scene():
    return two_level_scene()


@pytest.fixture(scope="module")
def reference(scene):
    return ref.RefScene(scene)


def test_scene_tree_and_mesh_trees_equal_reference(scene, reference):
    b = rb.build_bvh(scene)
    nodes, pe, pi = reference.bvh()
    assert np.array_equal(b.nodes.view(np.uint32), nodes.view(np.uint32))
    assert np.array_equal(b.prim_entity, pe) and np.array_equal(b.prim_index, pi)
    whole = np.flatnonzero(pi == rb.RB_BVH_ALL_TRIANGLES)
    assert whole.size == 3  # the two entities sharing a mesh, and the 327,680-triangle sphere
    assert len(b.mesh_trees) == 2
    d = scene.desc
    for e in pe[whole]:
        mesh = d.entities[int(e)].mesh
        tree = next(t for t in b.mesh_trees if t[0] == mesh)
        rn, rf = reference.mesh_bvh(int(e))
        assert np.array_equal(tree[1].view(np.uint32), rn.view(np.uint32)), f"entity {e}: mesh tree nodes differ"
        assert np.array_equal(tree[2], rf), f"entity {e}: mesh tree faces differ"
    # nesting depth: the scene tree's depth + 1 + the deepest mesh tree's (18+ levels for 327,680 faces)
    assert b.depth >= 20


def test_traversal_equals_reference(scene, reference):
    rays = random_rays(scene, 6000, 31)
    hp = HostPaths(scene)
    for shadow in (False, True):
        got, want = hp.trace(rays, shadow), reference.trace(rays, shadow)
        assert_hits_equal(got, want, f"shadow={shadow}")
        hit_ents = set(np.unique(want["entity"][want["entity"] >= 0]).tolist())
        whole = {int(e) for e, t in zip(*reference.bvh()[1:]) if t == rb.RB_BVH_ALL_TRIANGLES}
        assert whole <= hit_ents, "every whole-entity leaf should be hit by some ray"


def test_supplied_scene_tree_gets_its_mesh_trees(scene, reference):
    """A caller-supplied scene tree (the reference's own, exported) whose
    whole-entity prims name no mesh tree: the library builds the mesh trees
    with the reference's rules, and the hits are the same."""
    nodes, pe, pi = reference.bvh()
    sb = scene.with_bvh(rb.bvh_from_arrays(nodes, pe, pi))
    rays = random_rays(scene, 3000, 32)
    assert_hits_equal(HostPaths(sb).trace(rays), reference.trace(rays), "supplied tree")


def test_batch_with_two_level_scene(scene, reference):
    """Merged batch arrays relocate the mesh trees and the whole-entity slots:
    tracing the two-level scene inside a batch gives the reference's hits."""
    from tests.helpers import HostBatch
    other = rb.generate_scene(rb.RB_SCENE_BOX, width=32, height=32)
    hb = HostBatch([other, scene])
    rays = random_rays(scene, 3000, 34)
    assert_hits_equal(hb.trace(1, rays), reference.trace(rays), "batch")
