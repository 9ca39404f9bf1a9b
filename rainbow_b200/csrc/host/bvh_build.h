// Host BVH builder internals shared by the C ABI (rb_bvh_*) and the scene packer.
#pragma once

#include "../../../include/rbgpu.h"

#include <vector>

namespace rb {
namespace host {

// The reference's accelerator of one mesh (mesh::build_accelerator,
// rainbow-cpu/shapes/mesh.cpp:159-172): one leaf element per face, boxed in the
// mesh's local space, the same median-split build as the scene tree.
// nodes: 8 words per node (rb_bvh_desc layout, preorder); faces[p]: the face of
// leaf element p; depth: the deepest node's depth.
struct mesh_tree {
	int32_t mesh = -1;
	std::vector<float> nodes;
	std::vector<uint32_t> faces;
	uint32_t depth = 0;
};
rb_status build_mesh_tree(const rb_mesh_desc& mesh, int32_t mesh_index, mesh_tree& out);

// The mesh trees of a built rb_bvh (meshes that scene::build_accelerator gives
// their own accelerator), in order of first use.
const std::vector<mesh_tree>& bvh_mesh_trees(const rb_bvh* bvh);

} // namespace host
} // namespace rb
