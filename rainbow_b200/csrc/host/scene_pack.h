// Host packing of an rb_scene_desc into the flat record arrays the kernels read.
#pragma once

#include "../../../include/rbgpu.h"
#include "../pt/pt_types.h"

#include <vector>

namespace rb {
namespace host {

struct packed_scene {
	std::vector<float4> nodes;            // 2 per BVH node (reference layout, exact traversal)
	std::vector<pt::node4> wnodes;        // 4-wide nodes over the same tree (fast traversal)
	float4 root_a{}, root_b{};
	uint32_t root_ref = 0;
	bool wide_ok = false;                 // every leaf fits the 4-wide slot reference encoding
	std::vector<float4> tri_a, tri_b;     // per prim slot, entity-local p0 / e1 / e2
	std::vector<float2> tri_c;
	std::vector<uint32_t> prim_index;
	std::vector<uint32_t> prim_entity;
	std::vector<pt::entity_rec> entities;
	std::vector<pt::mesh_rec> meshes;
	std::vector<float> positions, normals, tangents, uvs;
	std::vector<uint32_t> indices;
	std::vector<pt::material_rec> materials;
	std::vector<pt::material_src> material_srcs;  // parameters of the MAT_TEXTURED records
	std::vector<pt::texture_rec> textures;
	std::vector<float> texels;
	std::vector<float> sss_table;                 // the normalized-diffusion inverse CDF when some material has a BSSRDF
	std::vector<pt::emitter_rec> emitters;
	std::vector<pt::medium_rec> mediums;
	std::vector<pt::media_rec> media;
	std::vector<int32_t> environments;
	pt::env_distribution env{};
	uint32_t bvh_depth = 0;
	bool instances = false;               // some prim slots are whole entities with their own mesh tree
};

// Validates and packs a scene. Builds the BVH with rb_bvh_build when the
// description carries none.
rb_status pack_scene(const rb_scene_desc* desc, packed_scene& out);

// Where one scene of a merged batch sits in the merged arrays.
struct scene_place {
	float4 root_a, root_b;
	uint32_t root_ref, root_node;
	uint32_t emitter_base, num_emitters;
	uint32_t env_base, num_environments;
	pt::env_distribution env;
};

// Concatenates packed scenes into one set of record arrays with every index
// (child nodes, prim slots, entities, meshes, vertices, materials, media)
// relocated, so that traversal from scene k's root only reaches scene k.
// Emitter indices (an entity's emitter, the environment list) stay relative to
// the scene: its view starts the emitter array at emitter_base.
// The merged scene has the wide nodes only if every part has them and all prim
// slots stay below 2^24.
rb_status merge_scenes(const std::vector<packed_scene>& parts, packed_scene& out, std::vector<scene_place>& places);

// A scene_view whose pointers are the host vectors of `p`.
pt::scene_view host_view(const packed_scene& p);

} // namespace host
} // namespace rb
