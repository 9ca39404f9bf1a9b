// Host packing of an rb_scene_desc into the kernels' record arrays.
//
// Derived quantities are computed here once, on the host, with the
// reference's formulas, so the kernels read exactly the reference's values:
//  - entity world areas: mesh::area(transform) (rainbow-cpu/shapes/mesh.cpp:131-150)
//  - Trowbridge-Reitz alphas: roughness_to_alpha (trowbridge_reitz_distribution.cpp:128-137)
//  - the environment's 2x2 sampling distribution (environment_light.cpp:20-36)
//  - local-space triangle edges e1 = p1 - p0, e2 = p2 - p0 (mesh.cpp:334-335)
#include "scene_pack.h"

#include "bvh_build.h"

#include "../pt/pt_bsdf.h"
#include "../pt/pt_geom.h"
#include "../pt/pt_material.h"
#include "../pt/pt_sss.h"

#include <cmath>
#include <cstring>
#include <new>

namespace rb {
namespace host {

namespace {

vec3 v3(const float* a, uint32_t i) { return vec3{a[3 * i], a[3 * i + 1], a[3 * i + 2]}; }

// A material's parameters with what derives from its reals applied
// (pt::derive_src: roughness_to_alpha, the smooth-glass test, Oren-Nayar's A
// and B). False for parameters the reference material would not take (a
// constant IOR of a plastic or uber material that is not positive) and for
// kinds it does not know.
bool make_src(const rb_material_desc& md, pt::material_src& p) {
	p = pt::material_src{};
	p.kind = md.kind;
	p.diffuse = v3(md.diffuse, 0);
	p.reflectance = v3(md.reflectance, 0);
	p.transmission = v3(md.transmission, 0);
	p.specular = v3(md.specular, 0);
	p.opacity = v3(md.opacity, 0);
	p.ior = md.ior;
	p.roughness_u = md.roughness_u;
	p.roughness_v = md.roughness_v;
	p.sigma = md.sigma;
	p.remap = md.remap_roughness ? 1u : 0u;
	p.tex[pt::TEX_DIFFUSE] = md.diffuse_texture;
	p.tex[pt::TEX_REFLECTANCE] = md.reflectance_texture;
	p.tex[pt::TEX_TRANSMISSION] = md.transmission_texture;
	p.tex[pt::TEX_SPECULAR] = md.specular_texture;
	p.tex[pt::TEX_OPACITY] = md.opacity_texture;
	p.tex[pt::TEX_ROUGHNESS_U] = md.roughness_u_texture;
	p.tex[pt::TEX_ROUGHNESS_V] = md.roughness_v_texture;
	p.tex[pt::TEX_IOR] = md.ior_texture;
	p.tex[pt::TEX_SIGMA] = md.sigma_texture;
	p.tex[pt::TEX_ETA] = md.eta_texture;
	p.tex[pt::TEX_K] = md.k_texture;
	p.tex[pt::TEX_MFP] = md.mfp_texture;
	switch (md.kind) {
	case RB_MATERIAL_METAL:
		p.cond_eta = v3(md.eta, 0);
		p.cond_k = v3(md.k, 0);
		break;
	case RB_MATERIAL_GLASS:
	case RB_MATERIAL_SUBSURFACE: p.mfp = v3(md.mfp, 0); break;
	case RB_MATERIAL_PLASTIC:
	case RB_MATERIAL_UBER:
		if (!md.ior_texture && !(md.ior > 0.f)) return false;
		break;
	case RB_MATERIAL_MATTE:
	case RB_MATERIAL_TRANSLUCENT:
	case RB_MATERIAL_SUBSTRATE:
	case RB_MATERIAL_MIRROR: break;
	default: return false;
	}
	pt::derive_src(p);
	return true;
}

bool textured(const rb_material_desc& md) {
	return md.diffuse_texture || md.reflectance_texture || md.transmission_texture || md.specular_texture ||
		md.opacity_texture || md.roughness_u_texture || md.roughness_v_texture || md.ior_texture || md.sigma_texture ||
		md.eta_texture || md.k_texture || md.mfp_texture;
}

// One material's record (pt::build_record), or with `scale` its scaled build.
rb_status pack_material(const rb_material_desc& md, const vec3* scale, pt::material_rec& r) {
	pt::material_src p;
	if (!make_src(md, p)) return RB_ERR_INVALID_ARGUMENT;
	return pt::build_record(p, scale, r) ? RB_OK : RB_ERR_INVALID_ARGUMENT;
}

// A lobe of a mixture: the component record it lives in and its index there.
struct mixture_lobe {
	uint32_t record, local, kind, type;
};

// The lobes that material k contributes, built with `scale`, in collection
// order; component records are appended to `records`. A mixture contributes
// its two components' lobes (mixture_material.cpp:29-43): material0 with
// alpha * scale, material1 with clamp(1 - alpha) * scale (without a scale,
// alpha and clamp(1 - alpha)). Mixtures nest up to 8 deep.
rb_status mixture_lobes(const rb_scene_desc* desc, uint32_t k, const vec3* scale, int depth,
	std::vector<pt::material_rec>& records, std::vector<mixture_lobe>& lobes) {
	const rb_material_desc& md = desc->materials[k];
	if (md.kind == RB_MATERIAL_MIXTURE) {
		if (depth >= 8) return RB_ERR_INVALID_ARGUMENT;
		for (int c = 0; c < 2; c++)
			if (md.components[c] < 0 || md.components[c] >= static_cast<int32_t>(desc->num_materials))
				return RB_ERR_INVALID_ARGUMENT;
		const vec3 alpha0 = v3(md.amount, 0);
		vec3 alpha1;
		alpha1.x = fclamp_ref(1.f - alpha0.x, 0.f, 1.f);
		alpha1.y = fclamp_ref(1.f - alpha0.y, 0.f, 1.f);
		alpha1.z = fclamp_ref(1.f - alpha0.z, 0.f, 1.f);
		const vec3 s0 = scale ? alpha0 * *scale : alpha0;
		const vec3 s1 = scale ? alpha1 * *scale : alpha1;
		rb_status st = mixture_lobes(desc, static_cast<uint32_t>(md.components[0]), &s0, depth + 1, records, lobes);
		if (st != RB_OK) return st;
		return mixture_lobes(desc, static_cast<uint32_t>(md.components[1]), &s1, depth + 1, records, lobes);
	}
	if (textured(md)) return RB_ERR_UNSUPPORTED;  // a mixture's components are built once, on the host
	pt::material_rec r;
	const rb_status st = pack_material(md, scale, r);
	if (st != RB_OK) return st;
	const pt::bsdf_t b = pt::make_bsdf(&r);
	if (b.count == 0) return RB_OK;
	const uint32_t index = static_cast<uint32_t>(records.size());
	records.push_back(r);
	for (uint32_t i = 0; i < b.count; i++) lobes.push_back(mixture_lobe{index, i, pt::lobe_kind(b, i), pt::lobe_type(b, i)});
	return RB_OK;
}

// Every material's record, in order, then the component records of mixtures;
// a material with image-textured spectra gets a MAT_TEXTURED record and its
// parameters in `srcs`.
rb_status pack_materials(const rb_scene_desc* desc, std::vector<pt::material_rec>& out,
	std::vector<pt::material_src>& srcs) {
	const uint32_t n = desc->num_materials;
	out.resize(n);
	std::vector<pt::material_rec> components;
	for (uint32_t k = 0; k < n; k++) {
		const rb_material_desc& md = desc->materials[k];
		if (md.kind != RB_MATERIAL_MIXTURE && textured(md)) {
			pt::material_src p;
			if (!make_src(md, p)) return RB_ERR_INVALID_ARGUMENT;
			for (uint32_t t = 0; t < pt::kNumTexSlots; t++)
				if (p.tex[t] > desc->num_textures) return RB_ERR_INVALID_ARGUMENT;
			out[k] = pt::material_rec{};
			out[k].kind = pt::MAT_TEXTURED;
			out[k].src = static_cast<uint32_t>(srcs.size());
			srcs.push_back(p);
			continue;
		}
		if (md.kind != RB_MATERIAL_MIXTURE) {
			const rb_status st = pack_material(md, nullptr, out[k]);
			if (st != RB_OK) return st;
			continue;
		}
		std::vector<pt::material_rec> recs;
		std::vector<mixture_lobe> lobes;
		const rb_status st = mixture_lobes(desc, k, nullptr, 0, recs, lobes);
		if (st != RB_OK) return st;
		if (lobes.size() > pt::kMaxLayeredLobes) return RB_ERR_UNSUPPORTED;
		pt::material_rec& r = out[k];
		r = pt::material_rec{};
		r.kind = pt::MAT_MIXTURE;
		r.blend_scale = vec3{1.f, 1.f, 1.f};
		const uint32_t base = n + static_cast<uint32_t>(components.size());  // index of recs[0]
		for (const mixture_lobe& l : lobes) {
			r.lobe_kinds |= l.kind << (4u * r.lobe_count);
			r.lobe_types |= l.type << (5u * r.lobe_count);
			r.lobe_ref[r.lobe_count] = ((base + l.record - k) << 4) | l.local;
			r.lobe_count++;
		}
		components.insert(components.end(), recs.begin(), recs.end());
	}
	out.insert(out.end(), components.begin(), components.end());
	return RB_OK;
}

// distribution1d over n values (distributions/detail/distribution.hpp:48-77)
void dist1(const float* values, int n, float* cdf, float& integral) {
	cdf[0] = 0.f;
	for (int i = 1; i <= n; i++) cdf[i] = cdf[i - 1] + values[i - 1] / static_cast<float>(n);
	integral = cdf[n];
	for (int i = 1; i <= n; i++) {
		if (integral != 0.f) cdf[i] = cdf[i] / integral;
		else cdf[i] = static_cast<float>(i) / static_cast<float>(n);
	}
}

void env_distribution_build(pt::env_distribution& d) {
	// constant map of 1: luminance(1, 1, 1) (color_spectrum.cpp:98-101)
	const float lum = 1.f * 0.212671f + 1.f * 0.715160f + 1.f * 0.072169f;
	for (int y = 0; y < 2; y++) {
		const float yp = (static_cast<float>(y) + 0.5f) / 2.f;
		const float st = sinf(yp * pt::kPi);
		for (int x = 0; x < 2; x++) d.value_row[y][x] = lum * st;
		dist1(d.value_row[y], 2, d.cdf_row[y], d.integral_row[y]);
	}
	d.value_marg[0] = d.integral_row[0];
	d.value_marg[1] = d.integral_row[1];
	dist1(d.value_marg, 2, d.cdf_marg, d.integral_marg);
}

} // namespace

rb_status pack_scene(const rb_scene_desc* desc, packed_scene& out) {
	if (desc == nullptr) return RB_ERR_INVALID_ARGUMENT;
	if ((desc->num_meshes && !desc->meshes) || (desc->num_entities && !desc->entities) ||
		(desc->num_materials && !desc->materials) || (desc->num_emitters && !desc->emitters))
		return RB_ERR_INVALID_ARGUMENT;
	try {
		out = packed_scene();
		// ---- meshes
		for (uint32_t m = 0; m < desc->num_meshes; m++) {
			const rb_mesh_desc& md = desc->meshes[m];
			if (md.num_triangles == 0 || md.positions == nullptr || md.indices == nullptr) return RB_ERR_INVALID_ARGUMENT;
			pt::mesh_rec r{};
			r.vertex_offset = static_cast<uint32_t>(out.positions.size() / 3);
			r.index_offset = static_cast<uint32_t>(out.indices.size());
			r.num_triangles = md.num_triangles;
			r.flags = (md.normals ? pt::MESH_HAS_NORMALS : 0u) | (md.tangents ? pt::MESH_HAS_TANGENTS : 0u) |
				(md.uvs ? pt::MESH_HAS_UVS : 0u) | (md.reverse_orientation ? pt::MESH_REVERSE : 0u);
			out.positions.insert(out.positions.end(), md.positions, md.positions + 3 * md.num_vertices);
			const size_t nv = 3ull * md.num_vertices;
			// optional attribute arrays stay aligned with the positions
			auto append = [&](std::vector<float>& dst, const float* src) {
				dst.resize(out.positions.size() - nv, 0.f);
				if (src) dst.insert(dst.end(), src, src + nv);
				else dst.resize(out.positions.size(), 0.f);
			};
			append(out.normals, md.normals);
			append(out.tangents, md.tangents);
			append(out.uvs, md.uvs);
			for (uint32_t i = 0; i < 3 * md.num_triangles; i++) {
				if (md.indices[i] >= md.num_vertices) return RB_ERR_INVALID_ARGUMENT;
				out.indices.push_back(md.indices[i]);
			}
			out.meshes.push_back(r);
		}
		// ---- image textures, then materials (records 0 .. n-1; component records of mixtures follow them)
		if (desc->num_textures > 0 && desc->textures == nullptr) return RB_ERR_INVALID_ARGUMENT;
		for (uint32_t t = 0; t < desc->num_textures; t++) {
			const rb_texture_desc& td = desc->textures[t];
			pt::texture_rec tr{};
			tr.kind = td.kind;
			if (td.kind == RB_TEXTURE_IMAGE) {
				if (td.rgb == nullptr || td.width == 0 || td.height == 0 || td.width > (1u << 15) || td.height > (1u << 15))
					return RB_ERR_INVALID_ARGUMENT;
				tr.offset = static_cast<uint32_t>(out.texels.size());
				tr.width = td.width;
				tr.height = td.height;
				if (out.texels.size() + 3ull * td.width * td.height > 0xffffffffull) return RB_ERR_INVALID_ARGUMENT;
				out.texels.insert(out.texels.end(), td.rgb, td.rgb + 3ull * td.width * td.height);
			} else if (td.kind == RB_TEXTURE_SCALE || td.kind == RB_TEXTURE_MIXTURE) {
				// inputs: images or constants (one level of composition)
				for (uint32_t i = 0; i < 3; i++) {
					const uint32_t in = td.inputs[i];
					if (in > desc->num_textures) return RB_ERR_INVALID_ARGUMENT;
					if (in && desc->textures[in - 1].kind != RB_TEXTURE_IMAGE) return RB_ERR_UNSUPPORTED;
					tr.inputs[i] = in;
					tr.constants[i] = v3(td.constants[i], 0);
				}
			} else {
				return RB_ERR_INVALID_ARGUMENT;
			}
			out.textures.push_back(tr);
		}
		{
			const rb_status st = pack_materials(desc, out.materials, out.material_srcs);
			if (st != RB_OK) return st;
			bool sss = false;
			for (const pt::material_rec& m : out.materials) sss = sss || m.sss;
			for (const pt::material_src& m : out.material_srcs) sss = sss || m.kind == RB_MATERIAL_SUBSURFACE;
			if (sss) {
				out.sss_table.resize(pt::kSssTableSize);
				pt::sss_build_table(out.sss_table.data());
			}
		}
		// ---- homogeneous media and media components
		if ((desc->num_mediums > 0 && desc->mediums == nullptr) || (desc->num_media > 0 && desc->media == nullptr))
			return RB_ERR_INVALID_ARGUMENT;
		for (uint32_t i = 0; i < desc->num_mediums; i++) {
			const rb_medium_desc& md = desc->mediums[i];
			pt::medium_rec r{};
			r.sigma_s = vec3{md.sigma_s[0], md.sigma_s[1], md.sigma_s[2]};
			r.sigma_t = vec3{md.sigma_a[0] + md.sigma_s[0], md.sigma_a[1] + md.sigma_s[1], md.sigma_a[2] + md.sigma_s[2]};
			r.g = md.g;
			out.mediums.push_back(r);
		}
		for (uint32_t i = 0; i < desc->num_media; i++) {
			const rb_media_desc& md = desc->media[i];
			const int32_t n = static_cast<int32_t>(desc->num_mediums);
			if (md.inside < -1 || md.inside >= n || md.outside < -1 || md.outside >= n) return RB_ERR_INVALID_ARGUMENT;
			out.media.push_back(pt::media_rec{md.inside, md.outside});
		}
		// ---- entities and the emitter list (scene::add_entity order, scene.cpp:16-28)
		for (uint32_t e = 0; e < desc->num_entities; e++) {
			const rb_entity_desc& ed = desc->entities[e];
			if (ed.medium < -1 || ed.medium >= static_cast<int32_t>(desc->num_media)) return RB_ERR_INVALID_ARGUMENT;
			if (ed.mesh >= static_cast<int32_t>(desc->num_meshes) || ed.material >= static_cast<int32_t>(desc->num_materials) ||
				ed.emitter >= static_cast<int32_t>(desc->num_emitters))
				return RB_ERR_INVALID_ARGUMENT;
			pt::entity_rec r{};
			std::memcpy(r.l2w, ed.local_to_world, sizeof(r.l2w));
			std::memcpy(r.w2l, ed.world_to_local, sizeof(r.w2l));
			r.mesh = ed.mesh;
			r.material = ed.material;
			r.emitter = -1;
			r.media = ed.medium;
			r.flags = (ed.mesh >= 0 ? pt::ENT_HAS_SHAPE : 0u) | (ed.material >= 0 ? pt::ENT_HAS_MATERIAL : 0u) |
				(ed.emitter >= 0 ? pt::ENT_HAS_EMITTER : 0u) | (ed.medium >= 0 ? pt::ENT_HAS_MEDIA : 0u);
			if (ed.mesh >= 0 && ed.material >= 0) r.flags |= pt::ENT_VISIBLE;
			if (ed.mesh >= 0) {
				// mesh::area(transform): sum of 0.5 |(p2 - p0) x (p2 - p1)| over world-space triangles
				const rb_mesh_desc& md = desc->meshes[ed.mesh];
				float area = 0.f;
				for (uint32_t t = 0; t < md.num_triangles; t++) {
					const uint32_t* idx = md.indices + 3 * t;
					const vec3 p0 = xform_point(r.l2w, v3(md.positions, idx[0]));
					const vec3 p1 = xform_point(r.l2w, v3(md.positions, idx[1]));
					const vec3 p2 = xform_point(r.l2w, v3(md.positions, idx[2]));
					area = area + 0.5f * length(cross(p2 - p0, p2 - p1));
				}
				r.area = area;
			}
			if (ed.emitter >= 0) {
				const rb_emitter_desc& em = desc->emitters[ed.emitter];
				pt::emitter_rec er{};
				er.kind = em.kind == RB_EMITTER_ENVIRONMENT ? pt::EMIT_ENVIRONMENT : pt::EMIT_SURFACE;
				if (em.kind != RB_EMITTER_ENVIRONMENT && em.kind != RB_EMITTER_SURFACE) return RB_ERR_INVALID_ARGUMENT;
				if (er.kind == pt::EMIT_SURFACE && ed.mesh < 0) return RB_ERR_INVALID_ARGUMENT;
				er.entity = static_cast<int32_t>(e);
				er.radiance = vec3{em.radiance[0], em.radiance[1], em.radiance[2]};
				er.radius = em.radius;
				r.emitter = static_cast<int32_t>(out.emitters.size());
				if (er.kind == pt::EMIT_ENVIRONMENT) out.environments.push_back(r.emitter);
				out.emitters.push_back(er);
			}
			out.entities.push_back(r);
		}
		if (out.emitters.empty()) return RB_ERR_INVALID_ARGUMENT;  // uniform_sample_one_emitter needs one
		env_distribution_build(out.env);

		// ---- BVH
		rb_bvh* built = nullptr;
		rb_bvh_desc bvh = desc->bvh;
		if (bvh.num_nodes == 0) {
			const rb_status st = rb_bvh_build(desc, &built);
			if (st != RB_OK) return st;
			rb_bvh_get(built, &bvh);
			rb_bvh_depth(built, &out.bvh_depth);
		}
		if (bvh.nodes == nullptr || bvh.prim_entity == nullptr || bvh.prim_index == nullptr) {
			rb_bvh_free(built);
			return RB_ERR_INVALID_ARGUMENT;
		}
		out.nodes.resize(2ull * bvh.num_nodes);
		for (uint32_t n = 0; n < bvh.num_nodes; n++) {
			const float* w = bvh.nodes + 8ull * n;
			out.nodes[2 * n] = float4{w[0], w[1], w[2], w[3]};
			out.nodes[2 * n + 1] = float4{w[4], w[5], w[6], w[7]};
		}
		if (built == nullptr) {
			// depth of a caller-supplied tree (iterative preorder walk with a validity check)
			std::vector<std::pair<uint32_t, uint32_t>> st{{0u, 0u}};
			uint32_t depth = 0;
			while (!st.empty()) {
				const auto [n, d] = st.back();
				st.pop_back();
				if (n >= bvh.num_nodes || d > 64) return RB_ERR_INVALID_ARGUMENT;
				depth = d > depth ? d : depth;
				uint32_t w0, w1;
				std::memcpy(&w0, bvh.nodes + 8ull * n + 6, 4);
				std::memcpy(&w1, bvh.nodes + 8ull * n + 7, 4);
				if (w1 & RB_BVH_LEAF_FLAG) {
					if (static_cast<uint64_t>(w0) + (w1 & ~RB_BVH_LEAF_FLAG) > bvh.num_prims) return RB_ERR_INVALID_ARGUMENT;
					continue;
				}
				if (w1 > 2) return RB_ERR_INVALID_ARGUMENT;
				st.push_back({n + 1, d + 1});
				st.push_back({w0, d + 1});
			}
			out.bvh_depth = depth;
		}
		// ---- mesh trees of entities that the scene tree holds whole (prim index
		// RB_BVH_ALL_TRIANGLES): the builder's, or built here with the same rules
		// for a caller-supplied scene tree. Appended after the scene's nodes;
		// their leaves are marked kMeshLeaf, with w0 relative to the first slot
		// of the instance being walked (each instance has its own copy of the
		// mesh's triangle slots, so a hit slot still names its entity).
		std::vector<host::mesh_tree> own_trees;
		std::vector<int32_t> tree_of(desc->num_meshes, -1);
		if (built != nullptr) {
			const auto& bt = host::bvh_mesh_trees(built);
			for (size_t k = 0; k < bt.size(); k++) tree_of[bt[k].mesh] = static_cast<int32_t>(k);
		} else {
			for (uint32_t s = 0; s < bvh.num_prims; s++) {
				if (bvh.prim_index[s] != RB_BVH_ALL_TRIANGLES) continue;
				const uint32_t e = bvh.prim_entity[s];
				if (e >= desc->num_entities || desc->entities[e].mesh < 0) return RB_ERR_INVALID_ARGUMENT;
				const int32_t m = desc->entities[e].mesh;
				if (tree_of[m] >= 0) continue;
				host::mesh_tree t;
				const rb_status st = host::build_mesh_tree(desc->meshes[m], m, t);
				if (st != RB_OK) return st;
				tree_of[m] = static_cast<int32_t>(own_trees.size());
				own_trees.push_back(std::move(t));
			}
		}
		const std::vector<host::mesh_tree>& trees = built != nullptr ? host::bvh_mesh_trees(built) : own_trees;
		std::vector<uint32_t> tree_root(trees.size(), 0);
		uint32_t deepest_tree = 0;
		for (size_t k = 0; k < trees.size(); k++) {
			const uint32_t base = static_cast<uint32_t>(out.nodes.size() / 2);
			tree_root[k] = base;
			deepest_tree = trees[k].depth > deepest_tree ? trees[k].depth : deepest_tree;
			const std::vector<float>& tn = trees[k].nodes;
			for (size_t n = 0; n < tn.size() / 8; n++) {
				const float* w = tn.data() + 8 * n;
				uint32_t w0, w1;
				std::memcpy(&w0, w + 6, 4);
				std::memcpy(&w1, w + 7, 4);
				if (w1 & RB_BVH_LEAF_FLAG) w1 |= pt::kMeshLeaf;
				else w0 += base;
				float f0, f1;
				std::memcpy(&f0, &w0, 4);
				std::memcpy(&f1, &w1, 4);
				out.nodes.push_back(float4{w[0], w[1], w[2], w[3]});
				out.nodes.push_back(float4{w[4], w[5], f0, f1});
			}
		}
		if (built == nullptr && !trees.empty()) out.bvh_depth += 1 + deepest_tree;
		out.instances = !trees.empty();
		// ---- 4-wide nodes: every binary node at an even depth with its
		// grandchildren as slots, numbered in preorder (the scene tree only)
		{
			const uint32_t nn = bvh.num_nodes;  // the scene tree's nodes (mesh trees follow them)
			auto word = [&](uint32_t n, int k) {
				uint32_t v;
				std::memcpy(&v, bvh.nodes + 8ull * n + k, 4);
				return v;
			};
			auto is_leaf = [&](uint32_t n) { return (word(n, 7) & RB_BVH_LEAF_FLAG) != 0; };
			bool ok = bvh.num_prims < (1u << 24) && nn > 0;
			auto leaf_ref = [&](uint32_t n) -> uint32_t {
				const uint32_t count = word(n, 7) & ~RB_BVH_LEAF_FLAG, first = word(n, 6);
				if (count == 0 || count > 127 || first >= (1u << 24)) ok = false;
				return pt::kRefLeaf | ((count & 0x7fu) << 24) | (first & 0x00ffffffu);
			};
			auto set_slot = [&](pt::node4& q, int k, uint32_t n, uint32_t ref) {
				const float* b = bvh.nodes + 8ull * n;
				reinterpret_cast<float*>(&q.lo_x)[k] = b[0];
				reinterpret_cast<float*>(&q.lo_y)[k] = b[1];
				reinterpret_cast<float*>(&q.lo_z)[k] = b[2];
				reinterpret_cast<float*>(&q.hi_x)[k] = b[3];
				reinterpret_cast<float*>(&q.hi_y)[k] = b[4];
				reinterpret_cast<float*>(&q.hi_z)[k] = b[5];
				reinterpret_cast<uint32_t*>(&q.ref)[k] = ref;
				q.meta.x |= 1u << (8 + k);
			};
			// depth-first with an explicit work list: (binary node, node4 index)
			std::vector<std::pair<uint32_t, uint32_t>> todo;
			if (ok && !is_leaf(0)) {
				out.wnodes.push_back(pt::node4{});
				todo.push_back({0u, 0u});
			}
			while (ok && !todo.empty()) {
				const auto [n, id] = todo.back();
				todo.pop_back();
				pt::node4 q{};
				q.meta.x = word(n, 7) & 3u;
				const uint32_t child[2] = {n + 1, word(n, 6)};
				std::vector<std::pair<uint32_t, uint32_t>> later;
				for (int p = 0; p < 2; p++) {
					const uint32_t x = child[p];
					if (x >= nn) { ok = false; break; }
					if (is_leaf(x)) {
						set_slot(q, 2 * p, x, leaf_ref(x));
						continue;
					}
					q.meta.x |= (word(x, 7) & 3u) << (2 + 2 * p);
					const uint32_t grand[2] = {x + 1, word(x, 6)};
					for (int g = 0; g < 2; g++) {
						const uint32_t y = grand[g];
						if (y >= nn) { ok = false; break; }
						if (is_leaf(y)) {
							set_slot(q, 2 * p + g, y, leaf_ref(y));
						} else {
							const uint32_t yid = static_cast<uint32_t>(out.wnodes.size());
							out.wnodes.push_back(pt::node4{});
							set_slot(q, 2 * p + g, y, yid);
							later.push_back({y, yid});
						}
					}
				}
				out.wnodes[id] = q;
				for (auto it = later.rbegin(); it != later.rend(); ++it) todo.push_back(*it);
			}
			out.root_a = float4{bvh.nodes[0], bvh.nodes[1], bvh.nodes[2], bvh.nodes[3]};
			out.root_b = float4{bvh.nodes[4], bvh.nodes[5], 0.f, 0.f};
			out.root_ref = nn > 0 ? (is_leaf(0) ? leaf_ref(0) : 0u) : 0u;
			out.wide_ok = ok;
			if (!ok) out.wnodes.clear();
		}
		// ---- prim slots: the scene tree's, then one block per whole-entity slot
		uint64_t total = bvh.num_prims;
		std::vector<uint32_t> block(bvh.num_prims, 0);
		for (uint32_t s = 0; s < bvh.num_prims; s++) {
			if (bvh.prim_index[s] != RB_BVH_ALL_TRIANGLES) continue;
			const uint32_t e = bvh.prim_entity[s];
			if (e >= desc->num_entities || desc->entities[e].mesh < 0) { rb_bvh_free(built); return RB_ERR_INVALID_ARGUMENT; }
			block[s] = static_cast<uint32_t>(total);
			total += trees[tree_of[desc->entities[e].mesh]].faces.size();
		}
		if (total >= (1ull << 31)) { rb_bvh_free(built); return RB_ERR_UNSUPPORTED; }
		out.tri_a.resize(total);
		out.tri_b.resize(total);
		out.tri_c.resize(total);
		out.prim_index.resize(total);
		out.prim_entity.resize(total);
		auto entity_word = [&](uint32_t e, uint32_t flags) {
			uint32_t word = e | flags;
			if (!(out.entities[e].flags & pt::ENT_VISIBLE)) word |= pt::kEntityInvisible;
			float wf;
			std::memcpy(&wf, &word, 4);
			return wf;
		};
		// entity-local p0, e1 = p1 - p0, e2 = p2 - p0 of face t of entity e's mesh in slot `slot`
		auto pack_triangle = [&](uint64_t slot, uint32_t e, uint32_t t) {
			const rb_mesh_desc& md = desc->meshes[desc->entities[e].mesh];
			const uint32_t* idx = md.indices + 3 * t;
			const vec3 p0 = v3(md.positions, idx[0]), p1 = v3(md.positions, idx[1]), p2 = v3(md.positions, idx[2]);
			const vec3 e1 = p1 - p0, e2 = p2 - p0;
			out.tri_a[slot] = float4{p0.x, p0.y, p0.z, e1.x};
			out.tri_b[slot] = float4{e1.y, e1.z, e2.x, e2.y};
			out.tri_c[slot] = float2{e2.z, entity_word(e, 0u)};
			out.prim_index[slot] = t;
			out.prim_entity[slot] = e;
		};
		for (uint32_t s = 0; s < bvh.num_prims; s++) {
			const uint32_t e = bvh.prim_entity[s];
			if (e >= desc->num_entities || desc->entities[e].mesh < 0) { rb_bvh_free(built); return RB_ERR_INVALID_ARGUMENT; }
			const rb_mesh_desc& md = desc->meshes[desc->entities[e].mesh];
			const uint32_t t = bvh.prim_index[s];
			if (t == RB_BVH_ALL_TRIANGLES) {
				// the whole entity: its mesh tree's root and its block of slots
				const int32_t k = tree_of[desc->entities[e].mesh];
				float root, first;
				std::memcpy(&root, &tree_root[k], 4);
				std::memcpy(&first, &block[s], 4);
				out.tri_a[s] = float4{root, first, 0.f, 0.f};
				out.tri_b[s] = float4{0.f, 0.f, 0.f, 0.f};
				out.tri_c[s] = float2{0.f, entity_word(e, pt::kEntityInstance)};
				out.prim_index[s] = RB_BVH_ALL_TRIANGLES;
				out.prim_entity[s] = e;
				const std::vector<uint32_t>& faces = trees[k].faces;
				for (size_t p = 0; p < faces.size(); p++) pack_triangle(block[s] + p, e, faces[p]);
				continue;
			}
			if (t >= md.num_triangles) { rb_bvh_free(built); return RB_ERR_INVALID_ARGUMENT; }
			pack_triangle(s, e, t);
		}
		rb_bvh_free(built);
	} catch (const std::bad_alloc&) {
		return RB_ERR_OUT_OF_MEMORY;
	}
	return RB_OK;
}

namespace {
uint32_t bits(float f) { uint32_t v; std::memcpy(&v, &f, 4); return v; }
float from_bits(uint32_t v) { float f; std::memcpy(&f, &v, 4); return f; }
template <typename T>
void append_vec(std::vector<T>& dst, const std::vector<T>& src) { dst.insert(dst.end(), src.begin(), src.end()); }
} // namespace

rb_status merge_scenes(const std::vector<packed_scene>& parts, packed_scene& out, std::vector<scene_place>& places) {
	try {
		out = packed_scene();
		places.clear();
		bool wide_ok = true;
		uint64_t slots = 0;
		for (const packed_scene& p : parts) {
			wide_ok = wide_ok && p.wide_ok;
			slots += p.tri_a.size();
		}
		if (slots >= (1ull << 31) || parts.empty()) return RB_ERR_UNSUPPORTED;
		wide_ok = wide_ok && slots < (1ull << 24);
		for (const packed_scene& p : parts) {
			const uint32_t node_base = static_cast<uint32_t>(out.nodes.size() / 2);
			const uint32_t wnode_base = static_cast<uint32_t>(out.wnodes.size());
			const uint32_t slot_base = static_cast<uint32_t>(out.tri_a.size());
			const uint32_t entity_base = static_cast<uint32_t>(out.entities.size());
			const uint32_t mesh_base = static_cast<uint32_t>(out.meshes.size());
			const uint32_t vertex_base = static_cast<uint32_t>(out.positions.size() / 3);
			const uint32_t index_base = static_cast<uint32_t>(out.indices.size());
			const uint32_t material_base = static_cast<uint32_t>(out.materials.size());
			const uint32_t emitter_base = static_cast<uint32_t>(out.emitters.size());
			const uint32_t env_base = static_cast<uint32_t>(out.environments.size());
			const int32_t medium_base = static_cast<int32_t>(out.mediums.size());
			const int32_t media_base = static_cast<int32_t>(out.media.size());
			// reference-layout nodes: interior w0 = right child, leaf w0 = first slot
			// (a mesh tree's leaf: relative to the instance's block, unchanged)
			for (size_t n = 0; n < p.nodes.size() / 2; n++) {
				float4 a = p.nodes[2 * n], b = p.nodes[2 * n + 1];
				const uint32_t w1 = bits(b.w);
				if (!(w1 & RB_BVH_LEAF_FLAG)) b.z = from_bits(bits(b.z) + node_base);
				else if (!(w1 & pt::kMeshLeaf)) b.z = from_bits(bits(b.z) + slot_base);
				out.nodes.push_back(a);
				out.nodes.push_back(b);
			}
			auto reloc_ref = [&](uint32_t r) {
				if (!(r & pt::kRefLeaf)) return r + wnode_base;
				const uint32_t first = (r & 0x00ffffffu) + slot_base;
				return (r & 0xff000000u) | (first & 0x00ffffffu);
			};
			if (wide_ok) {
				for (pt::node4 w : p.wnodes) {
					uint32_t* ref = reinterpret_cast<uint32_t*>(&w.ref);
					for (int k = 0; k < 4; k++)
						if (w.meta.x & (1u << (8 + k))) ref[k] = reloc_ref(ref[k]);
					out.wnodes.push_back(w);
				}
			}
			for (size_t k = 0; k < p.tri_a.size(); k++) {
				float2 c = p.tri_c[k];
				const uint32_t w = bits(c.y), flags = w & ~pt::kEntityMask;
				c.y = from_bits(((w & pt::kEntityMask) + entity_base) | flags);
				out.tri_c.push_back(c);
				out.prim_entity.push_back(p.prim_entity[k] + entity_base);
				float4 a = p.tri_a[k];
				if (w & pt::kEntityInstance) {  // a whole entity: its mesh tree's root and its block of slots
					a.x = from_bits(bits(a.x) + node_base);
					a.y = from_bits(bits(a.y) + slot_base);
				}
				out.tri_a.push_back(a);
			}
			append_vec(out.tri_b, p.tri_b);
			append_vec(out.prim_index, p.prim_index);
			for (pt::entity_rec e : p.entities) {
				if (e.mesh >= 0) e.mesh += static_cast<int32_t>(mesh_base);
				if (e.material >= 0) e.material += static_cast<int32_t>(material_base);
				// e.emitter stays scene-relative: a scene's view offsets the emitter array
				if (e.media >= 0) e.media += media_base;
				out.entities.push_back(e);
			}
			for (pt::mesh_rec m : p.meshes) {
				m.vertex_offset += vertex_base;
				m.index_offset += index_base;
				out.meshes.push_back(m);
			}
			append_vec(out.positions, p.positions);
			append_vec(out.normals, p.normals);
			append_vec(out.tangents, p.tangents);
			append_vec(out.uvs, p.uvs);
			append_vec(out.indices, p.indices);
			// materials: a textured record names its parameters, whose textures name their texels
			const uint32_t src_base = static_cast<uint32_t>(out.material_srcs.size());
			const uint32_t texture_base = static_cast<uint32_t>(out.textures.size());
			const uint32_t texel_base = static_cast<uint32_t>(out.texels.size());
			for (pt::material_rec m : p.materials) {
				if (m.kind == pt::MAT_TEXTURED) m.src += src_base;
				out.materials.push_back(m);
			}
			for (pt::material_src ms : p.material_srcs) {
				for (uint32_t t = 0; t < pt::kNumTexSlots; t++)
					if (ms.tex[t]) ms.tex[t] += texture_base;
				out.material_srcs.push_back(ms);
			}
			for (pt::texture_rec tr : p.textures) {
				if (tr.kind == pt::TEXK_IMAGE) tr.offset += texel_base;
				for (uint32_t i = 0; i < 3; i++)
					if (tr.inputs[i]) tr.inputs[i] += texture_base;
				out.textures.push_back(tr);
			}
			append_vec(out.texels, p.texels);
			if (!p.sss_table.empty()) out.sss_table = p.sss_table;
			for (pt::emitter_rec e : p.emitters) {
				e.entity += static_cast<int32_t>(entity_base);
				out.emitters.push_back(e);
			}
			append_vec(out.environments, p.environments);  // scene-relative emitter indices
			append_vec(out.mediums, p.mediums);
			for (pt::media_rec m : p.media) {
				if (m.inside >= 0) m.inside += medium_base;
				if (m.outside >= 0) m.outside += medium_base;
				out.media.push_back(m);
			}
			scene_place pl{};
			pl.root_a = p.root_a;
			pl.root_b = p.root_b;
			pl.root_ref = wide_ok ? reloc_ref(p.root_ref) : 0u;
			pl.root_node = node_base;
			pl.emitter_base = emitter_base;
			pl.num_emitters = static_cast<uint32_t>(p.emitters.size());
			pl.env_base = env_base;
			pl.num_environments = static_cast<uint32_t>(p.environments.size());
			pl.env = p.env;
			places.push_back(pl);
			out.bvh_depth = p.bvh_depth > out.bvh_depth ? p.bvh_depth : out.bvh_depth;
			out.instances = out.instances || p.instances;
		}
		out.wide_ok = wide_ok;
		if (!wide_ok) out.wnodes.clear();
		out.root_a = places[0].root_a;
		out.root_b = places[0].root_b;
		out.root_ref = places[0].root_ref;
		out.env = places[0].env;
	} catch (const std::bad_alloc&) {
		return RB_ERR_OUT_OF_MEMORY;
	}
	return RB_OK;
}

pt::scene_view host_view(const packed_scene& p) {
	pt::scene_view v{};
	v.wnodes = p.wide_ok ? p.wnodes.data() : nullptr;
	v.root_a = p.root_a;
	v.root_b = p.root_b;
	v.root_ref = p.root_ref;
	v.nodes = p.nodes.data();
	v.tri_a = p.tri_a.data();
	v.tri_b = p.tri_b.data();
	v.tri_c = p.tri_c.data();
	v.prim_index = p.prim_index.data();
	v.entities = p.entities.data();
	v.meshes = p.meshes.data();
	v.positions = p.positions.data();
	v.normals = p.normals.data();
	v.tangents = p.tangents.data();
	v.uvs = p.uvs.data();
	v.indices = p.indices.data();
	v.materials = p.materials.data();
	v.emitters = p.emitters.data();
	v.environments = p.environments.data();
	v.env = p.env;
	v.num_nodes = static_cast<uint32_t>(p.nodes.size() / 2);
	v.num_emitters = static_cast<uint32_t>(p.emitters.size());
	v.num_environments = static_cast<uint32_t>(p.environments.size());
	v.num_entities = static_cast<uint32_t>(p.entities.size());
	v.mediums = p.mediums.data();
	v.media = p.media.data();
	v.num_media = static_cast<uint32_t>(p.media.size());
	v.instances = p.instances ? 1u : 0u;
	v.material_srcs = p.material_srcs.data();
	v.textures = p.textures.data();
	v.texels = p.texels.data();
	v.num_textures = static_cast<uint32_t>(p.textures.size());
	v.sss_table = p.sss_table.empty() ? nullptr : p.sss_table.data();
	v.sss = p.sss_table.empty() ? 0u : 1u;
	return v;
}

} // namespace host
} // namespace rb
