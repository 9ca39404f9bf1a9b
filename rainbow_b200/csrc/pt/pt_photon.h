// Stochastic progressive photon mapping (rainbow-cpu/integrators/photon_mapping_integrator.cpp):
// per iteration, a visible point per pixel (trace_visible_point, :101-207),
// a hashed grid of the visible points' search spheres (build_visible_point_grid,
// :209-280), photons traced from the emitters that deposit flux at the visible
// points they land near (trace_photon / add_photon, :282-384), and the
// per-pixel radius and flux update (:512-537). The stage functions here are
// shared by the kernels (one thread per pixel or per photon) and the host
// build, which runs them in the reference's own order.
#pragma once

#include "pt_path.h"

namespace rb {
namespace pt {

// Streams of the kernels (the reference shares one stream per 16 x 16 tile of
// pixels and per chunk of 8192 photons, :418-451): pixel p of iteration i draws
// from stream_seed(p, i, seed) (bit 62 clear), photon j of iteration i from
// j | i << 32 | seed << 48 | 1 << 62, so the two never share a stream.
RB_HD uint64_t sppm_pixel_seed(uint32_t pixel, uint32_t iteration, uint32_t seed) {
	return stream_seed(pixel, iteration, seed & 0x3fffu);
}
RB_HD uint64_t sppm_photon_seed(uint32_t photon, uint32_t iteration, uint32_t seed) {
	return static_cast<uint64_t>(photon) | (static_cast<uint64_t>(iteration & 0xffffu) << 32) |
		(static_cast<uint64_t>(seed & 0x3fffu) << 48) | (1ull << 62);
}

// color_spectrum::luminance (shared/spectrums/color_spectrum.cpp:98-101).
RB_HD float luminance(const spectrum& c) { return c.x * 0.212671f + c.y * 0.715160f + c.z * 0.072169f; }

// A pixel's visible point: where its camera path met a diffuse surface (or a
// glossy one at its last bounce), with the path throughput there. The BSDF is
// rebuilt from the material and the texture coordinates when a photon lands.
struct visible_point {
	vec3 p;          // world point
	vec3 wo;         // world direction back along the camera path
	spectrum beta;
	uint32_t material;
	vec2 uv;
	uint32_t valid;  // found, with a non-black throughput (the grid's test, :217, :245)
};

// trace_visible_point (photon_mapping_integrator.cpp:101-207) for the path p
// starts: emission at the first hit and after specular bounces, the
// environment on every miss, uniform_sample_one_emitter at surfaces with a
// non-specular lobe, and BSDF continuations until a diffuse surface (or a
// glossy one at the last bounce) becomes the visible point. Radiance goes to
// p.L. trace(o, d, len, shadow): closest hit (shadow: visible entities only).
template <typename Trace>
RB_HD void sppm_visible(const scene_view& s, path_state& p, uint32_t max_depth, Trace&& trace, visible_point& vp) {
	vp.valid = 0u;
	bool specular = false;
	int guard = 0;
	for (int32_t bounces = 0; bounces < static_cast<int32_t>(max_depth) && guard < 4096; bounces++, guard++) {
		float len = p.len;
		const hit_t h = trace(p.o, p.d, len, false);
		if (h.slot < 0) {
			for (uint32_t i = 0; i < s.num_environments; i++) p.L = p.L + p.beta * s.emitters[s.environments[i]].radiance;
			break;
		}
		const surface_t si = make_surface(s, h.slot, h.b1, h.b2, p.o, p.d);
		const entity_rec& ent = s.entities[si.entity];
		if ((bounces == 0 || specular) && (ent.flags & ENT_HAS_EMITTER))
			p.L = p.L + p.beta * surface_emission(ent, s.emitters[ent.emitter], si.n, -p.d);
		if (!(ent.flags & ENT_HAS_MATERIAL)) {
			const ray_t r = spawn_ray(si.p, si.n, p.d);
			p.o = r.o;
			p.d = r.d;
			p.len = r.len;
			bounces--;
			continue;
		}
		const uint32_t material = static_cast<uint32_t>(ent.material);
		material_rec scratch;
		const bsdf_t b = make_bsdf(hit_material(s, material, si.uv, si.p, scratch));
		if (bsdf_count(b, ST_NON_SPECULAR) != 0) {
			shade_record rec;
			rec.si = si;
			rec.material = material;
			rec.pass_through = 0u;
			rec.guidable = 0u;
			rec.nee_entity = -1;
			rec.mis_valid = 0u;
			nee_sample<MAT_ANY>(s, p, si, b, rec);
			hit_t sh{-1, 0.f, 0.f}, mh{-1, 0.f, 0.f};
			if (rec.nee_entity >= 0) {
				float l = rec.shadow_ray.len;
				sh = trace(rec.shadow_ray.o, rec.shadow_ray.d, l, true);
			}
			if (rec.mis_valid) {
				float l = rec.mis_ray.len;
				mh = trace(rec.mis_ray.o, rec.mis_ray.d, l, true);
			}
			shade_b_direct<MAT_ANY>(s, p, rec, sh, mh);
		}
		const bool diffuse = bsdf_count(b, ST_DIFFUSE | ST_REFLECTION | ST_TRANSMISSION) > 0;
		const bool glossy = bsdf_count(b, ST_GLOSSY | ST_REFLECTION | ST_TRANSMISSION) > 0;
		if (diffuse || (glossy && bounces == static_cast<int32_t>(max_depth) - 1)) {
			vp.p = si.p;
			vp.wo = -p.d;
			vp.beta = p.beta;
			vp.material = material;
			vp.uv = si.uv;
			vp.valid = is_black(p.beta) ? 0u : 1u;
			break;
		}
		const lobe_sample bs = bsdf_sample<MAT_ANY>(b, to_local(si, si.wo), pcg_2d(p.rng), ST_ALL);
		if (is_black(bs.f) || bs.pdf == 0.f) break;
		const vec3 wi = to_world(si, bs.wi);
		p.beta = p.beta * (bs.f * fabs_ref(dot(wi, si.sz)) / bs.pdf);
		specular = type_match(bs.type, ST_SPECULAR);
		// Russian roulette below a luminance of 1/4 (:189-195)
		const float lum = luminance(p.beta);
		if (lum < 0.25f) {
			const float prob = (lum < 1.f) ? lum : 1.f;
			if (pcg_real(p.rng) > prob) break;
			p.beta = p.beta / prob;
		}
		const ray_t r = spawn_ray(si.p, si.n, wi);
		p.o = r.o;
		p.d = r.d;
		p.len = r.len;
	}
}

// A photon's first ray and throughput: uniform_sample_one_emitter(scene,
// samplers) (integrator.cpp:84-99) picks the emitter (1D), entity::sample<emitter>(u0, u1)
// samples the ray (surface_light.cpp:18-37: a point on the mesh, a cosine
// direction about its normal; environment_light.cpp:55-83: a direction from
// the map's distribution and a point on the disk of radius r facing it), and
// beta = Le |n . d| / (pick pdf * pdf_direction * pdf_position)
// (photon_mapping_integrator.cpp:332-343). The two 2D draws are arguments of
// one call; the reference as built here (g++) evaluates them right to left,
// so u1 is drawn before u0. Returns false when the photon carries nothing.
RB_HD bool sppm_emit(const scene_view& s, pcg32& rng, ray_t& ray, spectrum& beta) {
	if (s.num_emitters == 0) return false;
	const float n = static_cast<float>(s.num_emitters);
	uint32_t which = static_cast<uint32_t>(floorf(pcg_real(rng) * n));
	if (which > s.num_emitters - 1) which = s.num_emitters - 1;
	const float pick_pdf = 1.f / n;
	const vec2 u1 = pcg_2d(rng);
	const vec2 u0 = pcg_2d(rng);
	const emitter_rec& em = s.emitters[which];
	const entity_rec& e = s.entities[em.entity];
	spectrum Le;
	vec3 normal;
	ray_t r;
	float pdf_dir, pdf_pos;
	if (em.kind == EMIT_SURFACE) {
		// mesh::sample(properties, u0) (mesh.cpp:84-116): a triangle by index, a uniform point on it
		const mesh_rec& m = s.meshes[e.mesh];
		const float fc = static_cast<float>(m.num_triangles);
		uint32_t t = static_cast<uint32_t>(floorf(u0.x * fc));
		if (t > m.num_triangles - 1) t = m.num_triangles - 1;
		const float rx = u0.x * fc - static_cast<float>(t);
		const vec2 ur{(kOneMinusEps < rx) ? kOneMinusEps : rx, u0.y};
		const uint32_t* idx = s.indices + m.index_offset + 3 * t;
		const uint32_t i0 = m.vertex_offset + idx[0], i1 = m.vertex_offset + idx[1], i2 = m.vertex_offset + idx[2];
		const vec3 p0 = load3(s.positions, i0), p1 = load3(s.positions, i1), p2 = load3(s.positions, i2);
		const float su = sqrtf(ur.x);
		const float b0 = 1.f - su, b1 = ur.y * su;
		const vec3 point = p0 * b0 + p1 * b1 + p2 * (1.f - b0 - b1);
		normal = normalize(cross(p1 - p0, p2 - p0));
		if (m.flags & MESH_HAS_NORMALS)
			normal = load3(s.normals, i0) * b0 + load3(s.normals, i1) * b1 + load3(s.normals, i2) * (1.f - b0 - b1);
		if (m.flags & MESH_REVERSE) normal = normal * -1.f;
		pdf_pos = 1.f / e.area;
		const vec3 dir = cosine_hemisphere(u1);
		vec3 fx, fy, fz;
		frame_from_normal(normal, fx, fy, fz);
		const vec3 wl{fx.x * dir.x + fy.x * dir.y + fz.x * dir.z, fx.y * dir.x + fy.y * dir.y + fz.y * dir.z,
			fx.z * dir.x + fy.z * dir.y + fz.z * dir.z};
		r = spawn_ray(point, normal, wl);
		Le = dot(normal, r.d) > 0.f ? em.radiance : spectrum{0.f, 0.f, 0.f};
		pdf_dir = cosine_hemisphere_pdf(dir.z);
	} else {
		float dpdf;
		const vec2 v = env_dist_sample(s.env, u0, dpdf);
		if (dpdf == 0.f) return false;
		const float theta = v.y * kPi;
		const float phi = v.x * kTwoPi;
		const float ct = cosf(theta), st = sinf(theta);
		const vec3 dir = vec3{st * cosf(phi), st * sinf(phi), ct} * -1.f;
		vec3 fx, fy, fz;
		frame_from_normal(dir * -1.f, fx, fy, fz);
		const vec2 disk = concentric_disk(u1);
		const vec3 pl = (fx * disk.x + fy * disk.y) * em.radius;
		r.o = pl + (dir * -1.f) * em.radius;
		r.d = normalize(dir);
		r.len = kInf;
		normal = dir;
		Le = em.radiance;
		pdf_dir = st != 0.f ? dpdf / (kTwoPi * kPi * st) : 0.f;
		pdf_pos = 1.f / (kPi * em.radius * em.radius);
	}
	// emitter_ray_sample::transform (emitter.cpp:34-42) with the entity's local-to-world
	// transform; transform(ray) renormalises the direction and scales the length
	// (transform.cpp:94-105), and the ray's constructor normalises it once more
	const vec3 nw = xform_normal(e.w2l, normal);
	const vec3 dw = xform_vector(e.l2w, r.d);
	ray.d = normalize(normalize(dw));
	ray.o = xform_point(e.l2w, r.o);
	ray.len = r.len * length(dw);
	if (is_black(Le) || pdf_dir == 0.f || pdf_pos == 0.f) return false;
	beta = Le * fabs_ref(dot(nw, ray.d)) / (pick_pdf * pdf_dir * pdf_pos);
	return !is_black(beta);
}

// trace_photon (photon_mapping_integrator.cpp:326-384): the photon's path with
// importance transport; from its second hit on, every hit (invisible entities
// too) calls deposit(si, beta, d), d the direction the photon arrived along
// (add_photon). Continuation by BSDF sampling (2D) and a roulette (1D) that
// keeps the luminance of beta.
template <typename Trace, typename Deposit>
RB_HD void sppm_photon(const scene_view& s, pcg32& rng, uint32_t max_depth, Trace&& trace, Deposit&& deposit) {
	ray_t ray;
	spectrum beta;
	if (!sppm_emit(s, rng, ray, beta)) return;
	int guard = 0;
	for (int32_t bounces = 0; bounces < static_cast<int32_t>(max_depth) && guard < 4096; bounces++, guard++) {
		float len = ray.len;
		const hit_t h = trace(ray.o, ray.d, len, false);
		if (h.slot < 0) break;
		const surface_t si = make_surface(s, h.slot, h.b1, h.b2, ray.o, ray.d);
		if (bounces > 0) deposit(si, beta, ray.d);
		const entity_rec& ent = s.entities[si.entity];
		if (!(ent.flags & ENT_HAS_MATERIAL)) {
			const ray_t r = spawn_ray(si.p, si.n, ray.d);
			ray = r;
			bounces--;
			continue;
		}
		material_rec scratch;
		bsdf_t b = make_bsdf(hit_material(s, static_cast<uint32_t>(ent.material), si.uv, si.p, scratch));
		b.importance = 1u;
		const lobe_sample bs = bsdf_sample<MAT_ANY>(b, to_local(si, si.wo), pcg_2d(rng), ST_ALL);
		if (is_black(bs.f) || bs.pdf == 0.f) break;
		const vec3 wi = to_world(si, bs.wi);
		const spectrum next = beta * bs.f * fabs_ref(dot(wi, si.sz)) / bs.pdf;
		float q = 1.f - luminance(next) / luminance(beta);
		q = (q < 0.f) ? 0.f : q;
		if (pcg_real(rng) < q) break;
		beta = next / (1.f - q);
		ray = spawn_ray(si.p, si.n, wi);
	}
}

// The hashed grid of visible points (visible_point_grid, :41-47, 74-99): the
// bound of every search sphere, cells about the largest radius wide, and
// `pool` hash buckets (one per pixel).
struct sppm_grid {
	vec3 lo, hi;
	int32_t nx, ny, nz;
	uint32_t pool;
};

// position_in_grid (:74-81)
RB_HD bool sppm_inside(const sppm_grid& g, vec3 p) {
	if (p.x < g.lo.x || p.x > g.hi.x) return false;
	if (p.y < g.lo.y || p.y > g.hi.y) return false;
	if (p.z < g.lo.z || p.z > g.hi.z) return false;
	return true;
}
// position_to_grid (:83-92): the cell, truncated toward zero
RB_HD void sppm_cell(const sppm_grid& g, vec3 p, int32_t& x, int32_t& y, int32_t& z) {
	const vec3 o = p - g.lo;
	x = static_cast<int32_t>(o.x / (g.hi.x - g.lo.x) * static_cast<float>(g.nx));
	y = static_cast<int32_t>(o.y / (g.hi.y - g.lo.y) * static_cast<float>(g.ny));
	z = static_cast<int32_t>(o.z / (g.hi.z - g.lo.z) * static_cast<float>(g.nz));
}
// grid_to_index (:94-99): the cell's hash, in 32-bit wrapping arithmetic
RB_HD uint32_t sppm_bucket(const sppm_grid& g, int32_t x, int32_t y, int32_t z) {
	const uint32_t h = (static_cast<uint32_t>(x) * 73856093u) ^ (static_cast<uint32_t>(y) * 19349663u) ^
		(static_cast<uint32_t>(z) * 83492791u);
	return h % g.pool;
}
// The grid's cell counts from the bound and the largest radius (:213-241).
RB_HD void sppm_grid_size(sppm_grid& g, float max_radius) {
	const vec3 diag = g.hi - g.lo;
	const float md = fmax_ref(fmax_ref(diag.x, diag.y), diag.z);
	const int32_t base = static_cast<int32_t>(md / max_radius);
	const int32_t x = static_cast<int32_t>(static_cast<float>(base) * diag.x / md);
	const int32_t y = static_cast<int32_t>(static_cast<float>(base) * diag.y / md);
	const int32_t z = static_cast<int32_t>(static_cast<float>(base) * diag.z / md);
	g.nx = x > 1 ? x : 1;
	g.ny = y > 1 ? y : 1;
	g.nz = z > 1 ? z : 1;
}

// add_photon's flux at one visible point (:300-318): the visible point's BSDF
// at the photon's hit frame, beta times f(wo, wi) with wo the visible point's
// outgoing direction and wi back along the photon; zero outside the radius.
RB_HD bool sppm_flux(const scene_view& s, const surface_t& si, const spectrum& beta, vec3 d, const visible_point& vp,
	float radius, spectrum& flux) {
	if (distance_squared(vp.p, si.p) > radius * radius) return false;
	const vec3 wo = to_local(si, vp.wo);
	const vec3 wi = to_local(si, -d);
	material_rec scratch;
	const bsdf_t b = make_bsdf(hit_material(s, vp.material, vp.uv, vp.p, scratch));
	flux = beta * bsdf_f<MAT_ANY>(b, wo, wi, ST_ALL);
	return true;
}

// A pixel's state between iterations (mapping_pixel, :49-72).
struct sppm_pixel {
	spectrum tau, L;
	float radius, n;
};
// The update after the photon pass (:512-537): with m > 0 photons this
// iteration, n grows by 2/3 m, the radius shrinks by sqrt(n' / (n + m)), and
// tau takes the flux scaled to the new radius.
RB_HD void sppm_update(sppm_pixel& px, const spectrum& beta, const spectrum& phi, uint32_t m) {
	if (m == 0u) return;
	const float gamma = 2.f / 3.f;
	const float fm = static_cast<float>(m);
	const float n2 = px.n + gamma * fm;
	const float r2 = px.radius * sqrtf(n2 / (px.n + fm));
	px.tau = (px.tau + beta * phi) * (r2 * r2) / (px.radius * px.radius);
	px.radius = r2;
	px.n = n2;
}
// The pixel's value after all iterations (:545-550).
RB_HD spectrum sppm_value(const sppm_pixel& px, uint32_t iterations, uint64_t photons) {
	const float denom = static_cast<float>(static_cast<uint64_t>(iterations) * photons) * kPi * px.radius * px.radius;
	return px.L / static_cast<float>(iterations) + px.tau / denom;
}

} // namespace pt
} // namespace rb
