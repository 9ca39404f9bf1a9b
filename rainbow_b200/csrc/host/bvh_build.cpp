// Host BVH builder: the reference's binary median-split tree, flattened.
//
// Follows scene::build_accelerator (rainbow-cpu/scenes/scene.cpp:30-80) and
// bounding_volume_hierarchy<T>::recursive_build / split_equal_count
// (rainbow-cpu/shared/accelerators/detail/bounding_volume_hierarchy.hpp:162-233):
//  - one leaf element per triangle of each shaped entity whose mesh is used by
//    that entity alone and has at most 2^17 triangles, in entity order, boxed in
//    world space (mesh::bounding_box(transform, index), mesh.cpp:45-62);
//  - one element for the whole entity otherwise (a mesh shared by several
//    entities, or a larger one), boxed by transform::operator()(bound3)
//    (transform.cpp:78-92) of the mesh's local box, with the mesh given its own
//    tree over its faces in local space (mesh::build_accelerator, mesh.cpp:159-172);
//  - a node over one element, or over elements whose centroids coincide on the
//    widest centroid axis, is a leaf;
//  - otherwise std::nth_element splits at (begin + end) / 2 on that axis.
// std::nth_element is implementation-defined; this file and the reference are
// both compiled against libstdc++, and with the same element order and
// comparator it makes the same permutation, hence the same tree.
#include "bvh_build.h"

#include "../rb_math.h"

#include <algorithm>
#include <cstring>
#include <new>
#include <vector>

using rb::vec3;

struct rb_bvh {
	std::vector<float> nodes;          // 8 words per node
	std::vector<uint32_t> prim_entity;
	std::vector<uint32_t> prim_index;  // RB_BVH_ALL_TRIANGLES: the entity's whole mesh (its own tree)
	uint32_t depth = 0;                // of the scene tree
	std::vector<rb::host::mesh_tree> meshes;
};

namespace {

struct box3 {
	vec3 min, max;
};

// bound_t(p0, p1) then union_it(p2) (rainbow-core/math/detail/bound.hpp:12-30)
box3 triangle_box(const float* l2w, vec3 p0, vec3 p1, vec3 p2) {
	p0 = rb::xform_point(l2w, p0);
	p1 = rb::xform_point(l2w, p1);
	p2 = rb::xform_point(l2w, p2);
	box3 b{rb::vmin(p0, p1), rb::vmax(p0, p1)};
	b.min = rb::vmin(b.min, p2);
	b.max = rb::vmax(b.max, p2);
	return b;
}

// transform::operator()(bound3) (transform.cpp:78-92): the box of min and
// max, then the other six corners in the reference's order.
box3 transform_box(const float* m, const box3& b) {
	const vec3 a = rb::xform_point(m, b.min), c = rb::xform_point(m, b.max);
	box3 r{rb::vmin(a, c), rb::vmax(a, c)};
	const vec3 corners[6] = {
		{b.min.x, b.min.y, b.max.z}, {b.min.x, b.max.y, b.min.z}, {b.min.x, b.max.y, b.max.z},
		{b.max.x, b.min.y, b.min.z}, {b.max.x, b.min.y, b.max.z}, {b.max.x, b.max.y, b.min.z}};
	for (const vec3& k : corners) {
		const vec3 p = rb::xform_point(m, k);
		r.min = rb::vmin(r.min, p);
		r.max = rb::vmax(r.max, p);
	}
	return r;
}

const float kIdentity[16] = {1.f, 0.f, 0.f, 0.f, 0.f, 1.f, 0.f, 0.f, 0.f, 0.f, 1.f, 0.f, 0.f, 0.f, 0.f, 1.f};

vec3 vertex(const rb_mesh_desc& m, uint32_t i) { return vec3{m.positions[3 * i], m.positions[3 * i + 1], m.positions[3 * i + 2]}; }

// Box of face t of mesh m under transform l2w (mesh::bounding_box(transform, index)).
box3 face_box(const float* l2w, const rb_mesh_desc& m, uint32_t t) {
	const uint32_t* idx = m.indices + 3 * t;
	return triangle_box(l2w, vertex(m, idx[0]), vertex(m, idx[1]), vertex(m, idx[2]));
}

bool faces_valid(const rb_mesh_desc& m) {
	for (uint64_t i = 0; i < 3ull * m.num_triangles; i++)
		if (m.indices[i] >= m.num_vertices) return false;
	return true;
}

struct element {
	box3 box;
	uint32_t entity;
	uint32_t triangle;
	vec3 centroid() const { return (box.min + box.max) * 0.5f; }
};

struct node {
	box3 box;
	int left = -1, right = -1;
	size_t begin = 0, end = 0, axis = 0;
};

struct builder {
	std::vector<element> elems;
	std::vector<node> nodes;
	uint32_t max_depth = 0;

	int build(size_t begin, size_t end, uint32_t depth) {
		if (depth > max_depth) max_depth = depth;
		const int id = static_cast<int>(nodes.size());
		nodes.emplace_back();

		box3 u = elems[begin].box;
		for (size_t i = begin + 1; i < end; i++) {
			u.min = rb::vmin(u.min, elems[i].box.min);
			u.max = rb::vmax(u.max, elems[i].box.max);
		}
		auto make_leaf = [&]() {
			nodes[id].box = u;
			nodes[id].begin = begin;
			nodes[id].end = end;
			return id;
		};
		if (end - begin == 1) return make_leaf();

		const vec3 c0 = elems[begin].centroid();
		box3 cb{rb::vmin(c0, c0), rb::vmax(c0, c0)};
		for (size_t i = begin + 1; i < end; i++) {
			const vec3 c = elems[i].centroid();
			cb.min = rb::vmin(cb.min, c);
			cb.max = rb::vmax(cb.max, c);
		}
		// bounding_box<T>::max_dimension (detail/accelerator.hpp:69-77)
		const vec3 len = cb.max - cb.min;
		size_t dim = 2;
		if (len.x > len.y && len.x > len.z) dim = 0;
		else if (len.y > len.z) dim = 1;
		if (rb::get(cb.max, static_cast<int>(dim)) == rb::get(cb.min, static_cast<int>(dim))) return make_leaf();

		const size_t middle = (begin + end) >> 1;
		const int d = static_cast<int>(dim);
		std::nth_element(elems.data() + begin, elems.data() + middle, elems.data() + end,
			[d](const element& a, const element& b) { return rb::get(a.centroid(), d) < rb::get(b.centroid(), d); });
		if (middle == begin || middle == end) return make_leaf();

		const int l = build(begin, middle, depth + 1);
		const int r = build(middle, end, depth + 1);
		// interior box = min/max of the two child boxes (bounding_box(box0, box1), detail/accelerator.hpp:20-25)
		nodes[id].box.min = rb::vmin(nodes[l].box.min, nodes[r].box.min);
		nodes[id].box.max = rb::vmax(nodes[l].box.max, nodes[r].box.max);
		nodes[id].left = l;
		nodes[id].right = r;
		nodes[id].begin = begin;
		nodes[id].end = end;
		nodes[id].axis = dim;
		return id;
	}
};

void put_u32(float* dst, uint32_t v) { std::memcpy(dst, &v, sizeof(v)); }

// Preorder flattening: the left child always directly follows its parent.
uint32_t flatten(const builder& b, int id, std::vector<float>& out) {
	const uint32_t index = static_cast<uint32_t>(out.size() / 8);
	out.resize(out.size() + 8);
	const node& n = b.nodes[id];
	float* w = out.data() + index * 8;
	w[0] = n.box.min.x; w[1] = n.box.min.y; w[2] = n.box.min.z;
	w[3] = n.box.max.x; w[4] = n.box.max.y; w[5] = n.box.max.z;
	if (n.left < 0) {
		put_u32(w + 6, static_cast<uint32_t>(n.begin));
		put_u32(w + 7, RB_BVH_LEAF_FLAG | static_cast<uint32_t>(n.end - n.begin));
		return index;
	}
	flatten(b, n.left, out);
	const uint32_t right = flatten(b, n.right, out);
	w = out.data() + index * 8;  // out may have grown
	put_u32(w + 6, right);
	put_u32(w + 7, static_cast<uint32_t>(n.axis));
	return index;
}

} // namespace

extern "C" rb_status rb_bvh_build(const rb_scene_desc* desc, rb_bvh** out) {
	if (desc == nullptr || out == nullptr) return RB_ERR_INVALID_ARGUMENT;
	*out = nullptr;
	if (desc->num_entities > 0 && desc->entities == nullptr) return RB_ERR_INVALID_ARGUMENT;

	// shape reference counts (scene.cpp:49-56)
	std::vector<uint32_t> refs(desc->num_meshes, 0);
	for (uint32_t e = 0; e < desc->num_entities; e++) {
		const int32_t m = desc->entities[e].mesh;
		if (m < 0) continue;
		if (static_cast<uint32_t>(m) >= desc->num_meshes) return RB_ERR_INVALID_ARGUMENT;
		refs[m]++;
	}

	builder b;
	std::vector<rb::host::mesh_tree> trees;
	std::vector<int32_t> tree_of(desc->num_meshes, -1);
	try {
		for (uint32_t e = 0; e < desc->num_entities; e++) {
			const rb_entity_desc& ent = desc->entities[e];
			if (ent.mesh < 0) continue;
			const rb_mesh_desc& mesh = desc->meshes[ent.mesh];
			if (mesh.positions == nullptr || mesh.indices == nullptr || !faces_valid(mesh)) return RB_ERR_INVALID_ARGUMENT;
			const uint64_t count = refs[ent.mesh];
			if (count <= 1 && count * mesh.num_triangles <= (1u << 17)) {
				for (uint32_t t = 0; t < mesh.num_triangles; t++)
					b.elems.push_back(element{face_box(ent.local_to_world, mesh, t), e, t});
				continue;
			}
			// the whole entity as one element, the mesh with its own tree (built once)
			if (tree_of[ent.mesh] < 0) {
				rb::host::mesh_tree tree;
				const rb_status st = rb::host::build_mesh_tree(mesh, ent.mesh, tree);
				if (st != RB_OK) return st;
				tree_of[ent.mesh] = static_cast<int32_t>(trees.size());
				trees.push_back(std::move(tree));
			}
			// the mesh's local box (mesh constructor, mesh.cpp:31-36), then entity::bounding_box
			box3 local = face_box(kIdentity, mesh, 0);
			for (uint32_t t = 1; t < mesh.num_triangles; t++) {
				const box3 f = face_box(kIdentity, mesh, t);
				local.min = rb::vmin(local.min, f.min);
				local.max = rb::vmax(local.max, f.max);
			}
			b.elems.push_back(element{transform_box(ent.local_to_world, local), e, RB_BVH_ALL_TRIANGLES});
		}
		if (b.elems.empty()) return RB_ERR_INVALID_ARGUMENT;
		b.nodes.reserve(2 * b.elems.size());
		const int root = b.build(0, b.elems.size(), 0);

		rb_bvh* bvh = new rb_bvh();
		bvh->nodes.reserve(b.nodes.size() * 8);
		flatten(b, root, bvh->nodes);
		bvh->prim_entity.resize(b.elems.size());
		bvh->prim_index.resize(b.elems.size());
		for (size_t i = 0; i < b.elems.size(); i++) {
			bvh->prim_entity[i] = b.elems[i].entity;
			bvh->prim_index[i] = b.elems[i].triangle;
		}
		bvh->depth = b.max_depth;
		bvh->meshes = std::move(trees);
		*out = bvh;
	} catch (const std::bad_alloc&) {
		return RB_ERR_OUT_OF_MEMORY;
	}
	return RB_OK;
}

namespace rb {
namespace host {

rb_status build_mesh_tree(const rb_mesh_desc& mesh, int32_t mesh_index, mesh_tree& out) {
	if (mesh.num_triangles == 0 || mesh.positions == nullptr || mesh.indices == nullptr || !faces_valid(mesh))
		return RB_ERR_INVALID_ARGUMENT;
	try {
		builder b;
		b.elems.reserve(mesh.num_triangles);
		for (uint32_t t = 0; t < mesh.num_triangles; t++) b.elems.push_back(element{face_box(kIdentity, mesh, t), 0u, t});
		b.nodes.reserve(2 * b.elems.size());
		const int root = b.build(0, b.elems.size(), 0);
		out = mesh_tree();
		out.mesh = mesh_index;
		out.nodes.reserve(b.nodes.size() * 8);
		flatten(b, root, out.nodes);
		out.faces.resize(b.elems.size());
		for (size_t i = 0; i < b.elems.size(); i++) out.faces[i] = b.elems[i].triangle;
		out.depth = b.max_depth;
	} catch (const std::bad_alloc&) {
		return RB_ERR_OUT_OF_MEMORY;
	}
	return RB_OK;
}

const std::vector<mesh_tree>& bvh_mesh_trees(const rb_bvh* bvh) { return bvh->meshes; }

} // namespace host
} // namespace rb

extern "C" rb_status rb_bvh_get(const rb_bvh* bvh, rb_bvh_desc* out) {
	if (bvh == nullptr || out == nullptr) return RB_ERR_INVALID_ARGUMENT;
	out->nodes = bvh->nodes.data();
	out->num_nodes = static_cast<uint32_t>(bvh->nodes.size() / 8);
	out->num_prims = static_cast<uint32_t>(bvh->prim_entity.size());
	out->prim_entity = bvh->prim_entity.data();
	out->prim_index = bvh->prim_index.data();
	return RB_OK;
}

extern "C" rb_status rb_bvh_depth(const rb_bvh* bvh, uint32_t* max_depth) {
	if (bvh == nullptr || max_depth == nullptr) return RB_ERR_INVALID_ARGUMENT;
	uint32_t deepest_mesh = 0;
	for (const auto& t : bvh->meshes) deepest_mesh = t.depth > deepest_mesh ? t.depth : deepest_mesh;
	// a walk into a mesh tree continues below the scene tree's entity leaf
	*max_depth = bvh->meshes.empty() ? bvh->depth : bvh->depth + 1 + deepest_mesh;
	return RB_OK;
}

extern "C" rb_status rb_bvh_mesh_tree_count(const rb_bvh* bvh, uint32_t* count) {
	if (bvh == nullptr || count == nullptr) return RB_ERR_INVALID_ARGUMENT;
	*count = static_cast<uint32_t>(bvh->meshes.size());
	return RB_OK;
}

extern "C" rb_status rb_bvh_get_mesh_tree(const rb_bvh* bvh, uint32_t k, int32_t* mesh, rb_bvh_desc* out) {
	if (bvh == nullptr || mesh == nullptr || out == nullptr || k >= bvh->meshes.size()) return RB_ERR_INVALID_ARGUMENT;
	const auto& t = bvh->meshes[k];
	*mesh = t.mesh;
	out->nodes = t.nodes.data();
	out->num_nodes = static_cast<uint32_t>(t.nodes.size() / 8);
	out->num_prims = static_cast<uint32_t>(t.faces.size());
	out->prim_entity = nullptr;
	out->prim_index = t.faces.data();
	return RB_OK;
}

extern "C" void rb_bvh_free(rb_bvh* bvh) { delete bvh; }
