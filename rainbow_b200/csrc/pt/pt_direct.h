// Direct lighting: direct_integrator (rainbow-cpu/integrators/direct_integrator.cpp)
// for one camera sample, host and device.
//
// At the first visible surface the reference takes `emitter_samples` light
// samples and `bsdf_samples` BSDF samples, each weighted by the power heuristic
// over the two techniques' sample fractions (direct_integrator.cpp:5-18, 56-127).
// Random numbers are drawn in the reference's order: every light sample (emitter
// pick, then its point) before the first BSDF sample, and a BSDF sample's
// environment pick (find_emitter, integrator.cpp:49-82) after its own ray, before
// the next BSDF sample. Entities without a material, or whose material has no
// lobes, are passed through without a draw (direct_integrator.cpp:45-55).
#pragma once

#include "pt_path.h"

namespace rb {
namespace pt {

// direct_integrator's constructor constants (direct_integrator.cpp:5-18).
struct direct_cfg {
	uint32_t emitter_samples;
	uint32_t bsdf_samples;
	float weight_emitter;    // 1 / emitter_samples
	float weight_bsdf;       // 1 / bsdf_samples
	float frac_emitter;      // emitter_samples / (emitter_samples + bsdf_samples)
	float frac_bsdf;
};

RB_HD direct_cfg make_direct_cfg(uint32_t emitter_samples, uint32_t bsdf_samples) {
	direct_cfg c;
	c.emitter_samples = emitter_samples;
	c.bsdf_samples = bsdf_samples;
	const float sum = static_cast<float>(emitter_samples + bsdf_samples);
	c.weight_emitter = 1.f / static_cast<float>(emitter_samples);
	c.weight_bsdf = 1.f / static_cast<float>(bsdf_samples);
	c.frac_emitter = static_cast<float>(emitter_samples) / sum;
	c.frac_bsdf = static_cast<float>(bsdf_samples) / sum;
	return c;
}

// direct_integrator::trace (direct_integrator.cpp:20-127) of the camera ray in
// p (p.o, p.d, p.len, and p.rng after the camera's draws); the radiance goes
// to p.L. trace(o, d, len, shadow) returns the closest hit of the ray (shadow:
// invisible entities skipped, scene::intersect_with_shadow_ray) and shortens
// len to it.
template <typename Trace>
RB_HD void direct_radiance(const scene_view& s, const direct_cfg& cfg, path_state& p, Trace&& trace) {
	p.L = splat3(0.f);
	if (s.num_emitters == 0) return;
	vec3 o = p.o, d = p.d;
	float len = p.len;
	for (int guard = 0; guard < 4096; guard++) {
		float l = len;
		const hit_t h = trace(o, d, l, false);
		if (h.slot < 0) {
			for (uint32_t i = 0; i < s.num_environments; i++) p.L = p.L + s.emitters[s.environments[i]].radiance;
			return;
		}
		const surface_t si = make_surface(s, h.slot, h.b1, h.b2, o, d);
		const entity_rec& ent = s.entities[si.entity];
		if (ent.flags & ENT_HAS_EMITTER) p.L = p.L + surface_emission(ent, s.emitters[ent.emitter], si.n, -d);
		bsdf_t b;
		b.count = 0;
		material_rec mat_scratch;
		if (ent.flags & ENT_HAS_MATERIAL) b = make_bsdf(hit_material(s, static_cast<uint32_t>(ent.material), si.uv, si.p, mat_scratch));
		if (b.count == 0) {
			// no scattering functions: continue the ray through the surface
			const ray_t r = spawn_ray(si.p, si.n, d);
			o = r.o;
			d = r.d;
			len = r.len;
			continue;
		}
		const vec3 wo = to_local(si, si.wo);
		const float n_emitters = static_cast<float>(s.num_emitters);
		const float pick_pdf = 1.f / n_emitters;
		// emitter sampling (direct_integrator.cpp:58-101)
		for (uint32_t k = 0; k < cfg.emitter_samples; k++) {
			uint32_t which = static_cast<uint32_t>(floorf(pcg_real(p.rng) * n_emitters));
			if (which > s.num_emitters - 1) which = s.num_emitters - 1;
			const emitter_rec& em = s.emitters[which];
			light_sample ls = sample_emitter(s, em, si.p, si.n, pcg_2d(p.rng));
			ls.pdf = ls.pdf * pick_pdf;
			if (is_black(ls.L) || !(ls.pdf > 0.f)) continue;
			const vec3 wi = to_local(si, ls.wi);
			spectrum f = bsdf_f(b, wo, wi, ST_ALL);
			const float fpdf = bsdf_pdf(b, wo, wi, ST_ALL);
			f = f * fabs_ref(dot(ls.wi, si.sz));
			if (is_black(f) || fpdf <= 0.f) continue;
			const ray_t sr = spawn_ray_to(si.p, si.n, ls.p);
			float sl = sr.len;
			const hit_t sh = trace(sr.o, sr.d, sl, true);
			if (sh.slot < 0 || hit_entity(s, sh.slot) == static_cast<uint32_t>(em.entity)) {
				const float w = power_heuristic(ls.pdf * cfg.frac_emitter, fpdf * cfg.frac_bsdf) * cfg.weight_emitter;
				p.L = p.L + f * ls.L * w / ls.pdf;
			}
		}
		// BSDF sampling (direct_integrator.cpp:103-127) with find_emitter (integrator.cpp:49-82)
		for (uint32_t k = 0; k < cfg.bsdf_samples; k++) {
			const lobe_sample bs = bsdf_sample(b, wo, pcg_2d(p.rng), ST_ALL);
			const vec3 wi = bs.pdf > 0.f ? to_world(si, bs.wi) : vec3{0.f, 0.f, 0.f};
			const spectrum v = bs.f * fabs_ref(dot(wi, si.sz));
			if (is_black(v) || !(bs.pdf > 0.f)) continue;
			const ray_t er = spawn_ray(si.p, si.n, wi);
			float el = er.len;
			const hit_t eh = trace(er.o, er.d, el, true);
			spectrum Le = splat3(0.f);
			float epdf = 0.f;
			if (eh.slot >= 0) {
				const entity_rec& e2 = s.entities[hit_entity(s, eh.slot)];
				if (!(e2.flags & ENT_HAS_EMITTER)) continue;
				const surface_t es = make_surface(s, eh.slot, eh.b1, eh.b2, er.o, er.d);
				const emitter_rec& em = s.emitters[e2.emitter];
				Le = surface_emission(e2, em, es.n, -wi);
				epdf = emitter_pdf(s, em, si.p, si.n, wi) * pick_pdf;
			} else {
				if (s.num_environments == 0) continue;
				const float ne = static_cast<float>(s.num_environments);
				uint32_t which = static_cast<uint32_t>(floorf(pcg_real(p.rng) * ne));
				if (which > s.num_environments - 1) which = s.num_environments - 1;
				const emitter_rec& em = s.emitters[s.environments[which]];
				Le = em.radiance;
				epdf = emitter_pdf(s, em, si.p, si.n, wi) * pick_pdf;
			}
			if (is_black(Le) || epdf <= 0.f) continue;
			const float w = type_match(bs.type, ST_SPECULAR) ? 1.f
				: power_heuristic(bs.pdf * cfg.frac_bsdf, epdf * cfg.frac_emitter) * cfg.weight_bsdf;
			p.L = p.L + v * Le * w / bs.pdf;
		}
		return;
	}
}

// ------------------------------------------------------------ staged form
// The same sample in stages, for kernels that trace each stage's rays
// together: direct_surface at the camera ray's hit, direct_sample_lights (the
// light samples' shadow rays and the first BSDF sample's ray), then one
// direct_round per BSDF sample, each after its ray is traced. The draws and the
// additions to L happen in the order of direct_radiance.
constexpr uint32_t kDirectStagedLights = 8;  // light samples per surface the staged form holds

struct direct_record {
	surface_t si;
	uint32_t material;
	uint32_t round;                                 // BSDF samples resolved so far
	spectrum light_L[kDirectStagedLights];          // light sample k's term if its ray reaches its emitter
	int32_t light_entity[kDirectStagedLights];      // that emitter's entity, -1: no shadow ray
	spectrum bsdf_v;                                // pending BSDF sample: f |cos|, direction, pdf
	vec3 bsdf_wi;
	float bsdf_pdf;
	uint32_t bsdf_specular;
	uint32_t bsdf_valid;                            // 0: no ray for it
};

// At the hit h of the ray in p: 0 when the sample is done (p.L final), 1 when
// the ray continues through the surface (p.o / p.d / p.len updated), 2 when
// the surface is shaded (rec.si and rec.material set, its emission in p.L).
RB_HD int direct_surface(const scene_view& s, path_state& p, const hit_t& h, direct_record& rec) {
	if (s.num_emitters == 0) return 0;
	if (h.slot < 0) {
		for (uint32_t i = 0; i < s.num_environments; i++) p.L = p.L + s.emitters[s.environments[i]].radiance;
		return 0;
	}
	const surface_t si = make_surface(s, h.slot, h.b1, h.b2, p.o, p.d);
	const entity_rec& ent = s.entities[si.entity];
	if (ent.flags & ENT_HAS_EMITTER) p.L = p.L + surface_emission(ent, s.emitters[ent.emitter], si.n, -p.d);
	material_rec mat_scratch;
	if (!(ent.flags & ENT_HAS_MATERIAL) ||
		make_bsdf(hit_material(s, static_cast<uint32_t>(ent.material), si.uv, si.p, mat_scratch)).count == 0) {
		const ray_t r = spawn_ray(si.p, si.n, p.d);
		p.o = r.o;
		p.d = r.d;
		p.len = r.len;
		return 1;
	}
	rec.si = si;
	rec.material = static_cast<uint32_t>(ent.material);
	rec.round = 0u;
	return 2;
}

// Draws the next BSDF sample of a shaded surface; out: its ray when rec.bsdf_valid.
// MAT: the material kind when the caller knows it (a shading class), else MAT_ANY.
template <int MAT = MAT_ANY>
RB_HD void direct_next_bsdf(const scene_view& s, path_state& p, direct_record& rec, ray_t& out) {
	const surface_t& si = rec.si;
	material_rec mat_scratch;
	const bsdf_t b = make_bsdf(surface_material<MAT>(s, rec.material, si, mat_scratch));
	const lobe_sample bs = bsdf_sample<MAT>(b, to_local(si, si.wo), pcg_2d(p.rng), ST_ALL);
	const vec3 wi = bs.pdf > 0.f ? to_world(si, bs.wi) : vec3{0.f, 0.f, 0.f};
	const spectrum v = bs.f * fabs_ref(dot(wi, si.sz));
	rec.bsdf_valid = (!is_black(v) && bs.pdf > 0.f) ? 1u : 0u;
	rec.bsdf_v = v;
	rec.bsdf_wi = wi;
	rec.bsdf_pdf = bs.pdf;
	rec.bsdf_specular = type_match(bs.type, ST_SPECULAR) ? 1u : 0u;
	if (rec.bsdf_valid) out = spawn_ray(si.p, si.n, wi);
}

// The light samples (cfg.emitter_samples <= kDirectStagedLights): shadow ray k
// in out[k] where rec.light_entity[k] >= 0; then the first BSDF sample, its ray
// in out[cfg.emitter_samples].
template <int MAT = MAT_ANY>
RB_HD void direct_sample_lights(const scene_view& s, const direct_cfg& cfg, path_state& p, direct_record& rec,
	ray_t* out) {
	const surface_t& si = rec.si;
	material_rec mat_scratch;
	const bsdf_t b = make_bsdf(surface_material<MAT>(s, rec.material, si, mat_scratch));
	const vec3 wo = to_local(si, si.wo);
	const float n_emitters = static_cast<float>(s.num_emitters);
	const float pick_pdf = 1.f / n_emitters;
	for (uint32_t k = 0; k < cfg.emitter_samples; k++) {
		rec.light_entity[k] = -1;
		uint32_t which = static_cast<uint32_t>(floorf(pcg_real(p.rng) * n_emitters));
		if (which > s.num_emitters - 1) which = s.num_emitters - 1;
		const emitter_rec& em = s.emitters[which];
		light_sample ls = sample_emitter(s, em, si.p, si.n, pcg_2d(p.rng));
		ls.pdf = ls.pdf * pick_pdf;
		if (is_black(ls.L) || !(ls.pdf > 0.f)) continue;
		const vec3 wi = to_local(si, ls.wi);
		spectrum f = bsdf_f<MAT>(b, wo, wi, ST_ALL);
		const float fpdf = bsdf_pdf<MAT>(b, wo, wi, ST_ALL);
		f = f * fabs_ref(dot(ls.wi, si.sz));
		if (is_black(f) || fpdf <= 0.f) continue;
		out[k] = spawn_ray_to(si.p, si.n, ls.p);
		const float w = power_heuristic(ls.pdf * cfg.frac_emitter, fpdf * cfg.frac_bsdf) * cfg.weight_emitter;
		rec.light_L[k] = f * ls.L * w / ls.pdf;
		rec.light_entity[k] = em.entity;
	}
	direct_next_bsdf<MAT>(s, p, rec, out[cfg.emitter_samples]);
}

// After the traces of the pending rays: in round 0 first the light samples
// (light_hits[k], closest visible hit of shadow ray k), then the pending BSDF
// sample (hit bh of its ray); draws the next BSDF sample into out. Returns true
// while a BSDF sample is pending (rec.bsdf_valid: its ray needs tracing).
template <int MAT = MAT_ANY>
RB_HD bool direct_round(const scene_view& s, const direct_cfg& cfg, path_state& p, direct_record& rec,
	const hit_t* light_hits, const hit_t& bh, ray_t& out) {
	const surface_t& si = rec.si;
	if (rec.round == 0u)
		for (uint32_t k = 0; k < cfg.emitter_samples; k++) {
			const int32_t e = rec.light_entity[k];
			if (e >= 0 && (light_hits[k].slot < 0 || hit_entity(s, light_hits[k].slot) == static_cast<uint32_t>(e)))
				p.L = p.L + rec.light_L[k];
		}
	if (rec.bsdf_valid) {
		const vec3 wi = rec.bsdf_wi;
		const float pick_pdf = 1.f / static_cast<float>(s.num_emitters);
		spectrum Le = splat3(0.f);
		float epdf = 0.f;
		bool found = false;
		if (bh.slot >= 0) {
			const entity_rec& e2 = s.entities[hit_entity(s, bh.slot)];
			if (e2.flags & ENT_HAS_EMITTER) {
				const ray_t er = spawn_ray(si.p, si.n, wi);
				const surface_t es = make_surface(s, bh.slot, bh.b1, bh.b2, er.o, er.d);
				const emitter_rec& em = s.emitters[e2.emitter];
				Le = surface_emission(e2, em, es.n, -wi);
				epdf = emitter_pdf(s, em, si.p, si.n, wi) * pick_pdf;
				found = true;
			}
		} else if (s.num_environments > 0) {
			const float ne = static_cast<float>(s.num_environments);
			uint32_t which = static_cast<uint32_t>(floorf(pcg_real(p.rng) * ne));
			if (which > s.num_environments - 1) which = s.num_environments - 1;
			const emitter_rec& em = s.emitters[s.environments[which]];
			Le = em.radiance;
			epdf = emitter_pdf(s, em, si.p, si.n, wi) * pick_pdf;
			found = true;
		}
		if (found && !is_black(Le) && epdf > 0.f) {
			const float w = rec.bsdf_specular ? 1.f
				: power_heuristic(rec.bsdf_pdf * cfg.frac_bsdf, epdf * cfg.frac_emitter) * cfg.weight_bsdf;
			p.L = p.L + rec.bsdf_v * Le * w / rec.bsdf_pdf;
		}
	}
	rec.round++;
	if (rec.round >= cfg.bsdf_samples) return false;
	direct_next_bsdf<MAT>(s, p, rec, out);
	return true;
}

} // namespace pt
} // namespace rb
