// Per-path stages of path_integrator::trace (rainbow-cpu/integrators/path_integrator.cpp:15-47)
// split at the two points where the reference traces a ray in the middle of
// shading. One bounce is:
//   extend   closest hit of the path ray                    (scene::intersect)
//   shade_a  environment / emission / pass-through; when the BSDF has a
//            non-specular lobe: emitter pick (1D), light sample (2D) and the
//            MIS BSDF sample (2D) of uniform_sample_one_emitter
//            (integrator.cpp:101-201) -> a shadow ray and an MIS ray
//   trace    both secondary rays, visible entities only (intersect_with_shadow_ray)
//   shade_b  resolve the shadow test and find_emitter (integrator.cpp:49-82,
//            drawing the environment pick (1D) only when the MIS ray misses),
//            path BSDF sample (2D), throughput/eta update, spawn, Russian
//            roulette (1D) exactly as path_integrator::trace orders them.
// Splitting there keeps the reference's per-sample random-number order.
#pragma once

#include "pt_light.h"
#include "pt_material.h"

namespace rb {
namespace pt {

enum : uint32_t {
	PATH_SPECULAR = 1u << 0,
	PATH_SSS = 1u << 1  // the last BSDF sample transmitted into a subsurface material: the BSSRDF stage is next
};

struct path_state {
	vec3 o, d;
	float len;
	spectrum beta, L;
	float eta;
	uint32_t flags;
	int32_t bounces;
	pcg32 rng;
	int32_t medium;               // medium the path travels in (volume path tracing), -1: vacuum
};

// Everything shade_b needs from shade_a.
struct shade_record {
	surface_t si;
	uint32_t material;
	uint32_t pass_through;        // invisible entity: continue straight on
	uint32_t did_nee;             // uniform_sample_one_emitter was called
	uint32_t guidable;            // BSDF without specular lobes: a learned guide may sample here
	int32_t nee_entity;           // emitter entity of the shadow ray, -1: no shadow ray
	spectrum nee_L;               // its contribution if unoccluded
	uint32_t mis_valid;
	uint32_t mis_specular;
	vec3 mis_wi;                  // world direction of the MIS BSDF sample
	spectrum mis_f;               // f * |cos|
	float mis_pdf;
	ray_t shadow_ray, mis_ray;
};

// Volume path tracing keeps the factors of each light connection apart until
// the connection's transmittance is known, so that it enters the sum at the
// place the reference multiplies it in (integrator.cpp:139-146,180-191,226-232,263-271).
enum : uint32_t { VOL_MEDIUM_VERTEX = 1u, VOL_NEE = 2u, VOL_MIS = 4u };
struct vol_rec {
	spectrum nee_f;      // f * |cos| (surface) or the phase value (medium vertex)
	spectrum nee_Le;     // emitter_sample.intensity
	float nee_w, nee_pdf;
	vec3 nee_to;         // the sampled point on the emitter
	spectrum mis_Le;     // radiance found by the MIS sample
	float mis_w;
	vec3 mis_to;         // the point it was found at
	int32_t medium;      // medium of the path at this vertex
	uint32_t flags;      // VOL_*
	float g;             // phase asymmetry of a medium vertex
};

// perspective_camera::sample(position, u) (rainbow-cpu/cameras/perspective_camera.cpp:78-99)
// for pixel (x, y): position = (x, y) + film sample, then the lens sample.
RB_HD ray_t camera_ray(const float* r2c, const float* c2w, float lens, float focus, uint32_t x, uint32_t y, pcg32& rng) {
	const vec2 f = pcg_2d(rng);
	const vec2 lu = pcg_2d(rng);
	const float px = static_cast<float>(x) + f.x, py = static_cast<float>(y) + f.y;
	const vec3 target = xform_point(r2c, vec3{px, py, 0.f});
	vec3 o{0.f, 0.f, 0.f};
	vec3 d = normalize(normalize(target));
	if (lens > 0.f) {
		const vec3 fp = o + d * (focus / d.z);
		const vec2 l = concentric_disk(lu) * lens;
		o = vec3{l.x, l.y, 0.f};
		d = normalize(fp - o);
	}
	const vec3 dw = xform_vector(c2w, d);
	ray_t r;
	r.d = normalize(normalize(dw));
	r.o = xform_point(c2w, o);
	r.len = kInf * length(dw);
	return r;
}

RB_HD void path_begin(path_state& p, const float* r2c, const float* c2w, float lens, float focus, uint32_t x, uint32_t y,
	uint32_t pixel, uint32_t sample, uint32_t seed) {
	p.rng = pcg_seed(stream_seed(pixel, sample, seed));
	const ray_t r = camera_ray(r2c, c2w, lens, focus, x, y, p.rng);
	p.o = r.o;
	p.d = r.d;
	p.len = r.len;
	p.beta = splat3(1.f);
	p.L = splat3(0.f);
	p.eta = 1.f;
	p.flags = 0u;
	p.bounces = 0;
	p.medium = -1;
}

RB_HD uint32_t hit_entity(const scene_view& s, int32_t slot) {
	return float_as_u32(s.tri_c[slot].y) & ~kEntityInvisible;
}

// Shading classes: hits are queued by the material kind of the hit entity so
// that each shading kernel runs one BSDF's code on coherent warps.
// CLASS_MEDIUM: paths inside a medium (volume path tracing), whose next vertex
// is decided by free-flight sampling before any surface is shaded.
enum : uint32_t { CLASS_MISS = 0, CLASS_LAMBERT = 1, CLASS_METAL = 2, CLASS_GLASS_ROUGH = 3, CLASS_OTHER = 4, CLASS_MEDIUM = 5,
	NUM_CLASSES = 6 };
constexpr int class_material(uint32_t c) {
	return c == CLASS_LAMBERT ? static_cast<int>(MAT_LAMBERT)
		: c == CLASS_METAL ? static_cast<int>(MAT_METAL)
		: c == CLASS_GLASS_ROUGH ? static_cast<int>(MAT_GLASS_ROUGH) : MAT_ANY;
}
RB_HD uint32_t class_of_material(int32_t material, const scene_view& s) {
	if (material < 0 || s.materials[material].sss) return CLASS_OTHER;
	const uint32_t k = s.materials[material].kind;
	return k == MAT_LAMBERT ? CLASS_LAMBERT : k == MAT_METAL ? CLASS_METAL : k == MAT_GLASS_ROUGH ? CLASS_GLASS_ROUGH : CLASS_OTHER;
}
RB_HD uint32_t shade_class(const scene_view& s, int32_t slot) {
	if (slot < 0) return CLASS_MISS;
	const uint32_t e = float_as_u32(s.tri_c[slot].y) & ~kEntityInvisible;
	return class_of_material(s.entities[e].material, s);
}

// The miss branch of shade_a alone: environment radiance at bounce 0 or after
// a specular bounce (integrator.cpp:333-346); the path always ends.
RB_HD void shade_miss(const scene_view& s, path_state& p) {
	if (p.bounces == 0 || (p.flags & PATH_SPECULAR))
		for (uint32_t i = 0; i < s.num_environments; i++) p.L = p.L + p.beta * s.emitters[s.environments[i]].radiance;
}

template <int MAT = MAT_ANY>
RB_HD void nee_sample(const scene_view& s, path_state& p, const surface_t& si, const bsdf_t& b, shade_record& rec,
	vol_rec* vr = nullptr);

// Returns false when the path ends here (a miss). vr (volume path tracing
// only): receives the factors of the emitter-sampling connection.
template <int MAT = MAT_ANY>
RB_HD bool shade_a(const scene_view& s, path_state& p, const hit_t& h, shade_record& rec, vol_rec* vr = nullptr) {
	rec.pass_through = 0u;
	rec.did_nee = 0u;
	rec.guidable = 0u;
	rec.nee_entity = -1;
	rec.mis_valid = 0u;
	const bool count_emission = p.bounces == 0 || (p.flags & PATH_SPECULAR);
	if (h.slot < 0) {
		// sample_surface_interaction, miss branch (integrator.cpp:333-346)
		if (count_emission)
			for (uint32_t i = 0; i < s.num_environments; i++) p.L = p.L + p.beta * s.emitters[s.environments[i]].radiance;
		return false;
	}
	const surface_t si = make_surface(s, h.slot, h.b1, h.b2, p.o, p.d);
	rec.si = si;
	const entity_rec& ent = s.entities[si.entity];
	if (count_emission && (ent.flags & ENT_HAS_EMITTER))
		p.L = p.L + p.beta * surface_emission(ent, s.emitters[ent.emitter], si.n, -p.d);
	if (!(ent.flags & ENT_HAS_MATERIAL)) {
		const ray_t r = spawn_ray(si.p, si.n, p.d);
		p.o = r.o;
		p.d = r.d;
		p.len = r.len;
		p.bounces--;
		rec.pass_through = 1u;
		return true;
	}
	rec.material = static_cast<uint32_t>(ent.material);
	material_rec mat_scratch;
	const bsdf_t b = make_bsdf(surface_material<MAT>(s, rec.material, si, mat_scratch));
	if (bsdf_count(b, ST_NON_SPECULAR) == 0) return true;
	rec.guidable = bsdf_count(b, ST_SPECULAR) == 0 ? 1u : 0u;
	nee_sample<MAT>(s, p, si, b, rec, vr);
	return true;
}

// uniform_sample_one_emitter's draws and rays (integrator.cpp:101-201) at
// surface si with BSDF b: emitter pick (1D), light sample (2D) -> rec's shadow
// ray and its unoccluded contribution; the MIS BSDF sample (2D) -> rec's MIS
// ray. shade_b_direct adds what the two rays find.
template <int MAT>
RB_HD void nee_sample(const scene_view& s, path_state& p, const surface_t& si, const bsdf_t& b, shade_record& rec,
	vol_rec* vr) {
	rec.did_nee = 1u;
	const vec3 wo = to_local(si, si.wo);
	// emitter sampling half (integrator.cpp:121-159)
	const float n = static_cast<float>(s.num_emitters);
	uint32_t which = static_cast<uint32_t>(floorf(pcg_real(p.rng) * n));
	if (which > s.num_emitters - 1) which = s.num_emitters - 1;
	const float pick_pdf = 1.f / n;
	const emitter_rec& em = s.emitters[which];
	light_sample ls = sample_emitter(s, em, si.p, si.n, pcg_2d(p.rng));
	ls.pdf = ls.pdf * pick_pdf;
	if (!is_black(ls.L) && ls.pdf > 0.f) {
		const vec3 wi = to_local(si, ls.wi);
		spectrum f = bsdf_f<MAT>(b, wo, wi, ST_NON_SPECULAR);
		const float fpdf = bsdf_pdf<MAT>(b, wo, wi, ST_NON_SPECULAR);
		f = f * fabs_ref(dot(ls.wi, si.sz));
		if (!is_black(f) && fpdf > 0.f) {
			rec.shadow_ray = spawn_ray_to(si.p, si.n, ls.p);
			const float w = power_heuristic(ls.pdf, fpdf);
			rec.nee_L = f * ls.L * w / ls.pdf;
			rec.nee_entity = em.entity;
			if (vr != nullptr) {
				vr->nee_f = f;
				vr->nee_Le = ls.L;
				vr->nee_w = w;
				vr->nee_pdf = ls.pdf;
				vr->nee_to = ls.p;
			}
		}
	}
	// BSDF sampling half (integrator.cpp:161-198)
	const lobe_sample bs = bsdf_sample<MAT>(b, wo, pcg_2d(p.rng), ST_NON_SPECULAR);
	const vec3 wi_w = bs.pdf > 0.f ? to_world(si, bs.wi) : vec3{0.f, 0.f, 0.f};
	const spectrum v = bs.f * fabs_ref(dot(wi_w, si.sz));
	if (!is_black(v) && bs.pdf > 0.f) {
		rec.mis_valid = 1u;
		rec.mis_specular = type_match(bs.type, ST_SPECULAR) ? 1u : 0u;
		rec.mis_wi = wi_w;
		rec.mis_f = v;
		rec.mis_pdf = bs.pdf;
		rec.mis_ray = spawn_ray(si.p, si.n, wi_w);
	}
}

// Direct lighting half of shade_b: the unoccluded NEE sample and the MIS
// BSDF sample that found an emitter (integrator.cpp:121-198), added to the path.
// shadow / mis are the closest visible hits of rec.shadow_ray / rec.mis_ray.
template <int MAT = MAT_ANY>
RB_HD void shade_b_direct(const scene_view& s, path_state& p, const shade_record& rec, const hit_t& shadow, const hit_t& mis) {
	const surface_t& si = rec.si;
	spectrum Ls = splat3(0.f);
	if (rec.nee_entity >= 0 && (shadow.slot < 0 || hit_entity(s, shadow.slot) == static_cast<uint32_t>(rec.nee_entity)))
		Ls = Ls + rec.nee_L;
	if (rec.mis_valid) {
		// find_emitter (integrator.cpp:49-82) and the MIS term (:165-195)
		bool found = false;
		spectrum Le = splat3(0.f);
		float epdf = 0.f;
		const float pick_pdf = 1.f / static_cast<float>(s.num_emitters);
		if (mis.slot >= 0) {
			const uint32_t e = hit_entity(s, mis.slot);
			const entity_rec& ent = s.entities[e];
			if (ent.flags & ENT_HAS_EMITTER) {
				const surface_t es = make_surface(s, mis.slot, mis.b1, mis.b2, rec.mis_ray.o, rec.mis_ray.d);
				const emitter_rec& em = s.emitters[ent.emitter];
				Le = surface_emission(ent, em, es.n, -rec.mis_wi);
				epdf = emitter_pdf(s, em, si.p, si.n, rec.mis_wi) * pick_pdf;
				found = true;
			}
		} else if (s.num_environments > 0) {
			const float ne = static_cast<float>(s.num_environments);
			uint32_t which = static_cast<uint32_t>(floorf(pcg_real(p.rng) * ne));
			if (which > s.num_environments - 1) which = s.num_environments - 1;
			const emitter_rec& em = s.emitters[s.environments[which]];
			Le = em.radiance;
			epdf = emitter_pdf(s, em, si.p, si.n, rec.mis_wi) * pick_pdf;
			found = true;
		}
		if (found && !is_black(Le) && epdf > 0.f) {
			const float w = rec.mis_specular ? 1.f : power_heuristic(rec.mis_pdf, epdf);
			Ls = Ls + rec.mis_f * Le * w / rec.mis_pdf;
		}
	}
	p.L = p.L + p.beta * Ls;
}

// Path continuation by BSDF sampling (integrator.cpp:380-399). Returns false
// when the BSDF sample fails; otherwise updates beta, the specular flag, eta
// and the ray, and reports the world direction and its pdf.
template <int MAT = MAT_ANY>
RB_HD bool continue_bsdf(const scene_view& s, path_state& p, const shade_record& rec, vec3& wi_out, float& pdf_out) {
	const surface_t& si = rec.si;
	material_rec mat_scratch;
	const bsdf_t b = make_bsdf(surface_material<MAT>(s, rec.material, si, mat_scratch));
	const vec3 wo = to_local(si, si.wo);
	const lobe_sample bs = bsdf_sample<MAT>(b, wo, pcg_2d(p.rng), ST_ALL);
	if (is_black(bs.f) || bs.pdf == 0.f) return false;
	const vec3 wi = to_world(si, bs.wi);
	p.beta = p.beta * (bs.f * fabs_ref(dot(wi, si.sz)) / bs.pdf);
	p.flags = type_match(bs.type, ST_SPECULAR) ? (p.flags | PATH_SPECULAR) : (p.flags & ~PATH_SPECULAR);
	if (type_match(bs.type, ST_SPECULAR | ST_TRANSMISSION))
		p.eta = p.eta * ((dot(si.wo, si.n) > 0.f) ? (b.eta * b.eta) : (1.f / (b.eta * b.eta)));
	const ray_t r = spawn_ray(si.p, si.n, wi);
	p.o = r.o;
	p.d = r.d;
	p.len = r.len;
	// a transmission into a material with a BSSRDF (integrator.cpp:401-402)
	if constexpr (MAT == MAT_ANY)
		if (b.m->sss && type_match(bs.type, ST_TRANSMISSION)) p.flags |= PATH_SSS;
	wi_out = wi;
	pdf_out = bs.pdf;
	return true;
}

// Russian roulette (path_integrator.cpp:35-43) and the bounce count; false
// when the path ends.
RB_HD bool roulette(path_state& p, uint32_t max_depth, float rr_threshold) {
	const float mc = spectrum_max(p.beta * p.eta);
	if (mc < rr_threshold && p.bounces > 3) {
		const float q = fmax_ref(0.05f, 1.f - mc);
		if (pcg_real(p.rng) < q) return false;
		p.beta = p.beta / (1.f - q);
	}
	p.bounces++;
	return p.bounces < static_cast<int32_t>(max_depth);
}

// Returns false when the path ends (BSDF sample failed, Russian roulette, max depth).
// shadow / mis are the closest visible hits of rec.shadow_ray / rec.mis_ray.
template <int MAT = MAT_ANY>
RB_HD bool shade_b(const scene_view& s, path_state& p, const shade_record& rec, const hit_t& shadow, const hit_t& mis,
	uint32_t max_depth, float rr_threshold) {
	if (!rec.pass_through) {
		if (rec.did_nee) shade_b_direct<MAT>(s, p, rec, shadow, mis);
		vec3 wi;
		float pdf;
		if (!continue_bsdf<MAT>(s, p, rec, wi, pdf)) return false;
		if (p.flags & PATH_SSS) return true;  // the BSSRDF stage, then Russian roulette
	}
	return roulette(p, max_depth, rr_threshold);
}

// Run-time dispatch to the class-specialised stages (the host build uses it;
// the kernels launch one class at a time).
RB_HD bool shade_a_any(const scene_view& s, path_state& p, const hit_t& h, shade_record& rec) {
	switch (shade_class(s, h.slot)) {
	case CLASS_LAMBERT: return shade_a<class_material(CLASS_LAMBERT)>(s, p, h, rec);
	case CLASS_METAL: return shade_a<class_material(CLASS_METAL)>(s, p, h, rec);
	case CLASS_GLASS_ROUGH: return shade_a<class_material(CLASS_GLASS_ROUGH)>(s, p, h, rec);
	default: return shade_a<MAT_ANY>(s, p, h, rec);
	}
}
RB_HD bool shade_b_any(const scene_view& s, path_state& p, const shade_record& rec, const hit_t& shadow, const hit_t& mis,
	uint32_t max_depth, float rr_threshold) {
	const uint32_t c = rec.pass_through ? CLASS_OTHER : class_of_material(static_cast<int32_t>(rec.material), s);
	switch (c) {
	case CLASS_LAMBERT: return shade_b<class_material(CLASS_LAMBERT)>(s, p, rec, shadow, mis, max_depth, rr_threshold);
	case CLASS_METAL: return shade_b<class_material(CLASS_METAL)>(s, p, rec, shadow, mis, max_depth, rr_threshold);
	case CLASS_GLASS_ROUGH: return shade_b<class_material(CLASS_GLASS_ROUGH)>(s, p, rec, shadow, mis, max_depth, rr_threshold);
	default: return shade_b<MAT_ANY>(s, p, rec, shadow, mis, max_depth, rr_threshold);
	}
}

} // namespace pt
} // namespace rb
