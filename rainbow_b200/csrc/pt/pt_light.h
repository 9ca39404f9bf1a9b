// Emitters of the path tracer: area lights on triangle meshes (surface_light)
// and the constant environment (environment_light with a constant map), with
// the entity transforms the reference applies around them
// (rainbow-cpu/scenes/detail/entity.hpp:32-71). Host- and device-compilable.
#pragma once

#include "pt_bsdf.h"
#include "pt_geom.h"

namespace rb {
namespace pt {

struct light_sample {
	vec3 p;            // world point on the emitter
	vec3 wi;           // world direction (transform_vector of the local one, not renormalised)
	spectrum L;
	float pdf;         // solid-angle pdf, before the emitter-choice pdf
};

// transform_interaction(W2L, reference) (transform.cpp:190-196): the reference
// point and normal in entity-local space.
RB_HD void reference_to_local(const entity_rec& e, vec3 p, vec3 n, vec3& pl, vec3& nl) {
	nl = xform_normal(e.l2w, n);  // transform_normal with the W2L transform, whose inverse is L2W
	pl = xform_point(e.w2l, p);
}

// ---- distribution1d / distribution2d sampling (distributions/detail/distribution.hpp:48-141)
RB_HD uint32_t find_interval2(const float* cdf, float u) {
	// upper_bound over 3 entries, minus one
	uint32_t i = 0;
	while (i < 3 && !(u < cdf[i])) i++;
	return i - 1;
}
RB_HD float dist1_sample(const float* cdf, const float* values, float integral, float u, uint32_t& offset, float& pdf) {
	offset = find_interval2(cdf, u);
	float du = u - cdf[offset];
	if (offset < 2 && cdf[offset + 1] - cdf[offset] > 0.f) du = du / (cdf[offset + 1] - cdf[offset]);
	pdf = integral > 0.f ? values[offset] / integral : 0.f;
	return (static_cast<float>(offset) + du) / 2.f;
}
RB_HD vec2 env_dist_sample(const env_distribution& d, vec2 u, float& pdf) {
	uint32_t oy, ox;
	float py, px;
	const float vy = dist1_sample(d.cdf_marg, d.value_marg, d.integral_marg, u.y, oy, py);
	const float vx = dist1_sample(d.cdf_row[oy], d.value_row[oy], d.integral_row[oy], u.x, ox, px);
	pdf = px * py;
	return vec2{vx, vy};
}
RB_HD float env_dist_pdf(const env_distribution& d, vec2 p) {
	uint32_t x = static_cast<uint32_t>(p.x * 2.f), y = static_cast<uint32_t>(p.y * 2.f);
	if (x > 1) x = 1;
	if (y > 1) y = 1;
	return d.value_row[y][x] / d.integral_marg;
}

// environment_light::pdf(properties, reference, wi) (environment_light.cpp:130-149)
RB_HD float env_pdf(const scene_view& s, vec3 wi) {
	const vec3 w = normalize(wi);
	const float theta = acosf(fclamp_ref(w.z, -1.f, 1.f));
	float phi = atan2f(w.y, w.x);
	phi = phi < 0.f ? phi + kTwoPi : phi;
	const float st = sinf(theta);
	if (st == 0.f) return 0.f;
	const float dp = env_dist_pdf(s.env, vec2{phi * kInvTwoPi, theta * kInvPi});
	return dp / (kTwoPi * kPi * st);
}

// Emitter sample towards a world reference point (uniform_sample_one_emitter's
// light half, integrator.cpp:126-133): entity::sample<emitter>(reference, u).
RB_HD light_sample sample_emitter(const scene_view& s, const emitter_rec& em, vec3 ref_p, vec3 ref_n, vec2 u) {
	light_sample out{};
	const entity_rec& e = s.entities[em.entity];
	vec3 pl, nl;
	reference_to_local(e, ref_p, ref_n, pl, nl);
	if (em.kind == EMIT_SURFACE) {
		// surface_light::sample -> shape::sample(properties, reference, u) -> mesh::sample (mesh.cpp:84-116)
		const mesh_rec& m = s.meshes[e.mesh];
		const float fc = static_cast<float>(m.num_triangles);
		uint32_t which = static_cast<uint32_t>(floorf(u.x * fc));
		if (which > m.num_triangles - 1) which = m.num_triangles - 1;
		const float rx = u.x * fc - static_cast<float>(which);
		const vec2 ur{(kOneMinusEps < rx) ? kOneMinusEps : rx, u.y};
		const uint32_t* idx = s.indices + m.index_offset + 3 * which;
		const uint32_t i0 = m.vertex_offset + idx[0], i1 = m.vertex_offset + idx[1], i2 = m.vertex_offset + idx[2];
		const vec3 p0 = load3(s.positions, i0), p1 = load3(s.positions, i1), p2 = load3(s.positions, i2);
		const float su = sqrtf(ur.x);
		const float b0 = 1.f - su, b1 = ur.y * su;
		const vec3 point = p0 * b0 + p1 * b1 + p2 * (1.f - b0 - b1);
		vec3 normal = normalize(cross(p1 - p0, p2 - p0));
		if (m.flags & MESH_HAS_NORMALS)
			normal = load3(s.normals, i0) * b0 + load3(s.normals, i1) * b1 + load3(s.normals, i2) * (1.f - b0 - b1);
		if (m.flags & MESH_REVERSE) normal = normal * -1.f;
		float pdf = 1.f / e.area;
		// shape::sample(properties, reference, sample) (shape.cpp:26-44)
		vec3 wi = point - pl;
		if (length_squared(wi) == 0.f) return out;
		wi = normalize(wi);
		pdf = pdf * distance_squared(pl, point) / fabs_ref(dot(normal, -wi));
		if (isinf(pdf)) return out;
		if (pdf == 0.f) return out;
		// surface_light::sample (surface_light.cpp:39-54)
		const vec3 wl = normalize(point - pl);
		const spectrum L = dot(normal, -wl) > 0.f ? em.radiance : spectrum{0.f, 0.f, 0.f};
		// emitter_sample::transform (emitter.cpp:26-34)
		out.p = xform_point(e.l2w, point);
		out.wi = xform_vector(e.l2w, wl);
		out.L = L;
		out.pdf = pdf;
		return out;
	}
	// environment_light::sample(properties, reference, u) (environment_light.cpp:85-107)
	float dpdf;
	const vec2 v = env_dist_sample(s.env, u, dpdf);
	if (dpdf == 0.f) return out;
	const float theta = v.y * kPi;
	const float phi = v.x * kTwoPi;
	const float ct = cosf(theta), st = sinf(theta);
	const float pdf = st != 0.f ? dpdf / (kTwoPi * kPi * st) : 0.f;
	const vec3 wi{st * cosf(phi), st * sinf(phi), ct};
	const vec3 point = pl + 2.f * em.radius * wi;
	out.p = xform_point(e.l2w, point);
	out.wi = xform_vector(e.l2w, wi);
	out.L = em.radiance;
	out.pdf = pdf;
	return out;
}

// entity::evaluate<emitter>(interaction, w) for a surface emitter: one-sided on
// the local geometric normal (surface_light.cpp:12-16).
RB_HD spectrum surface_emission(const entity_rec& e, const emitter_rec& em, vec3 n_world, vec3 w_world) {
	const vec3 nl = xform_normal(e.l2w, n_world);
	const vec3 wl = xform_vector(e.w2l, w_world);
	return dot(nl, wl) > 0.f ? em.radiance : spectrum{0.f, 0.f, 0.f};
}

// entity::pdf<emitter>(reference, wi) of a surface emitter: shape::pdf
// (shape.cpp:46-60), re-intersecting the emitter mesh in its local space.
RB_HD float surface_pdf(const scene_view& s, const entity_rec& e, vec3 ref_p, vec3 ref_n, vec3 wi_world) {
	vec3 pl, nl;
	reference_to_local(e, ref_p, ref_n, pl, nl);
	const vec3 wl = xform_vector(e.w2l, wi_world);
	const ray_t r = spawn_ray(pl, nl, wl);
	const mesh_rec& m = s.meshes[e.mesh];
	float len = r.len;
	int32_t best = -1;
	float bb1 = 0.f, bb2 = 0.f;
	for (uint32_t t = 0; t < m.num_triangles; t++) {
		const uint32_t* idx = s.indices + m.index_offset + 3 * t;
		const vec3 p0 = load3(s.positions, m.vertex_offset + idx[0]);
		const vec3 p1 = load3(s.positions, m.vertex_offset + idx[1]);
		const vec3 p2 = load3(s.positions, m.vertex_offset + idx[2]);
		float th, b1, b2;
		if (triangle_hit(r.o, r.d, len, p0, p1 - p0, p2 - p0, th, b1, b2)) {
			len = th;
			best = static_cast<int32_t>(t);
			bb1 = b1;
			bb2 = b2;
		}
	}
	if (best < 0) return 0.f;
	const local_surface ls = triangle_surface(s, m, static_cast<uint32_t>(best), bb1, bb2);
	const float pdf = distance_squared(pl, ls.p) / (fabs_ref(dot(ls.n, -wl)) * e.area);
	return isinf(pdf) ? 0.f : pdf;
}

// entity::pdf<emitter>(reference, wi) for either emitter kind (integrator.cpp:170).
RB_HD float emitter_pdf(const scene_view& s, const emitter_rec& em, vec3 ref_p, vec3 ref_n, vec3 wi_world) {
	const entity_rec& e = s.entities[em.entity];
	if (em.kind == EMIT_SURFACE) return surface_pdf(s, e, ref_p, ref_n, wi_world);
	return env_pdf(s, xform_vector(e.w2l, wi_world));
}

RB_HD float power_heuristic(float f, float g) { return (f * f) / (f * f + g * g); }

} // namespace pt
} // namespace rb
