// Host packing of an rb_scene_desc into the kernels' record arrays.
//
// Derived quantities are computed here once, on the host, with the
// reference's formulas, so the kernels read exactly the reference's values:
//  - entity world areas: mesh::area(transform) (rainbow-cpu/shapes/mesh.cpp:131-150)
//  - Trowbridge-Reitz alphas: roughness_to_alpha (trowbridge_reitz_distribution.cpp:128-137)
//  - the environment's 2x2 sampling distribution (environment_light.cpp:20-36)
//  - local-space triangle edges e1 = p1 - p0, e2 = p2 - p0 (mesh.cpp:334-335)
#include "scene_pack.h"

#include "../pt/pt_bsdf.h"

#include <cmath>
#include <cstring>
#include <new>

namespace rb {
namespace host {

namespace {

vec3 v3(const float* a, uint32_t i) { return vec3{a[3 * i], a[3 * i + 1], a[3 * i + 2]}; }
bool black3(const float* c) { return c[0] == 0.f && c[1] == 0.f && c[2] == 0.f; }

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
		// ---- materials
		for (uint32_t i = 0; i < desc->num_materials; i++) {
			const rb_material_desc& md = desc->materials[i];
			pt::material_rec r{};
			switch (md.kind) {
			case RB_MATERIAL_MATTE: {
				const float sigma = fclamp_ref(md.sigma, 0.f, 90.f);
				if (black3(md.diffuse)) r.kind = pt::MAT_BLACK;
				else if (sigma != 0.f) return RB_ERR_UNSUPPORTED;  // Oren-Nayar is outside the supported subset
				else r.kind = pt::MAT_LAMBERT;
				r.diffuse = vec3{md.diffuse[0], md.diffuse[1], md.diffuse[2]};
				break;
			}
			case RB_MATERIAL_METAL:
				r.kind = pt::MAT_METAL;
				r.alpha_x = md.remap_roughness ? pt::roughness_to_alpha(md.roughness_u) : md.roughness_u;
				r.alpha_y = md.remap_roughness ? pt::roughness_to_alpha(md.roughness_v) : md.roughness_v;
				r.cond_eta = vec3{md.eta[0], md.eta[1], md.eta[2]};
				r.cond_k = vec3{md.k[0], md.k[1], md.k[2]};
				break;
			case RB_MATERIAL_GLASS: {
				const bool specular = md.roughness_u == 0.f && md.roughness_v == 0.f;
				r.kind = specular ? pt::MAT_GLASS_SMOOTH : pt::MAT_GLASS_ROUGH;
				if (!specular) {
					r.alpha_x = md.remap_roughness ? pt::roughness_to_alpha(md.roughness_u) : md.roughness_u;
					r.alpha_y = md.remap_roughness ? pt::roughness_to_alpha(md.roughness_v) : md.roughness_v;
				}
				r.eta = md.ior;
				r.reflectance = vec3{md.reflectance[0], md.reflectance[1], md.reflectance[2]};
				r.transmission = vec3{md.transmission[0], md.transmission[1], md.transmission[2]};
				r.has_reflect = black3(md.reflectance) ? 0u : 1u;
				r.has_transmit = black3(md.transmission) ? 0u : 1u;
				break;
			}
			default: return RB_ERR_INVALID_ARGUMENT;
			}
			out.materials.push_back(r);
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
		// ---- wide nodes: interior nodes numbered in preorder, children's boxes inline
		{
			const uint32_t nn = bvh.num_nodes;
			auto word = [&](uint32_t n, int k) {
				uint32_t v;
				std::memcpy(&v, bvh.nodes + 8ull * n + k, 4);
				return v;
			};
			std::vector<uint32_t> wid(nn, 0xffffffffu);
			uint32_t next = 0;
			for (uint32_t n = 0; n < nn; n++)
				if (!(word(n, 7) & RB_BVH_LEAF_FLAG)) wid[n] = next++;
			bool ok = bvh.num_prims < (1u << 24);
			auto ref_of = [&](uint32_t n) -> uint32_t {
				const uint32_t w1 = word(n, 7);
				if (!(w1 & RB_BVH_LEAF_FLAG)) return wid[n];
				const uint32_t count = w1 & ~RB_BVH_LEAF_FLAG, first = word(n, 6);
				if (count == 0 || count > 127 || first >= (1u << 24)) ok = false;
				return pt::kRefLeaf | ((count & 0x7fu) << 24) | (first & 0x00ffffffu);
			};
			out.wnodes.resize(next);
			for (uint32_t n = 0; n < nn; n++) {
				if (wid[n] == 0xffffffffu) continue;
				const uint32_t l = n + 1, r = word(n, 6);
				const float* bl = bvh.nodes + 8ull * l;
				const float* br = bvh.nodes + 8ull * r;
				pt::wide_node& w = out.wnodes[wid[n]];
				w.a = float4{bl[0], bl[1], bl[2], bl[3]};
				w.b = float4{bl[4], bl[5], br[0], br[1]};
				w.c = float4{br[2], br[3], br[4], br[5]};
				w.d = uint4{ref_of(l), ref_of(r), word(n, 7), 0u};
			}
			out.root_a = float4{bvh.nodes[0], bvh.nodes[1], bvh.nodes[2], bvh.nodes[3]};
			out.root_b = float4{bvh.nodes[4], bvh.nodes[5], 0.f, 0.f};
			out.root_ref = nn > 0 ? ref_of(0) : 0u;
			out.wide_ok = ok && nn > 0;
		}
		out.tri_a.resize(bvh.num_prims);
		out.tri_b.resize(bvh.num_prims);
		out.tri_c.resize(bvh.num_prims);
		out.prim_index.assign(bvh.prim_index, bvh.prim_index + bvh.num_prims);
		out.prim_entity.assign(bvh.prim_entity, bvh.prim_entity + bvh.num_prims);
		for (uint32_t s = 0; s < bvh.num_prims; s++) {
			const uint32_t e = bvh.prim_entity[s];
			if (e >= desc->num_entities || desc->entities[e].mesh < 0) { rb_bvh_free(built); return RB_ERR_INVALID_ARGUMENT; }
			const rb_mesh_desc& md = desc->meshes[desc->entities[e].mesh];
			const uint32_t t = bvh.prim_index[s];
			if (t >= md.num_triangles) { rb_bvh_free(built); return RB_ERR_INVALID_ARGUMENT; }
			const uint32_t* idx = md.indices + 3 * t;
			const vec3 p0 = v3(md.positions, idx[0]), p1 = v3(md.positions, idx[1]), p2 = v3(md.positions, idx[2]);
			const vec3 e1 = p1 - p0, e2 = p2 - p0;
			uint32_t word = e;
			if (!(out.entities[e].flags & pt::ENT_VISIBLE)) word |= 0x80000000u;
			float wf;
			std::memcpy(&wf, &word, 4);
			out.tri_a[s] = float4{p0.x, p0.y, p0.z, e1.x};
			out.tri_b[s] = float4{e1.y, e1.z, e2.x, e2.y};
			out.tri_c[s] = float2{e2.z, wf};
		}
		rb_bvh_free(built);
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
	return v;
}

} // namespace host
} // namespace rb
