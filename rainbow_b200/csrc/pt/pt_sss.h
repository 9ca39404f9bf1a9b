// Subsurface scattering of the path integrator: the normalized-diffusion
// BSSRDF (rainbow-cpu/scatterings/bssrdf/normalized_diffusion.cpp) sampled as
// separable_bidirectional_scattering_surface_distribution_function::sample
// (scatterings/scattering_surface_function.cpp:71-147) and used as
// sample_scattering_surface_function (integrators/integrator.cpp:290-327) does
// after a BSDF sample that transmits into a subsurface material.
#pragma once

#include "pt_path.h"

#if !defined(__CUDA_ARCH__)
#include <cmath>
#endif

namespace rb {
namespace pt {

// Knots of the inverse CDF of the normalized-diffusion radial profile for
// d = 1: knot k is r with cdf(r) = k / (kSssTableSize - 1), cdf(r) = 1 -
// e^-r / 4 - 3 e^(-r / 3) / 4 (Christensen and Burley 2015). The reference
// keeps these as a table (inv_normalized_diffusion_cdf_table); they are
// computed here by Newton's method in double and rounded to float, which
// gives the table's floats for every knot but the last, where the inverse is
// infinite and the table holds the finite value kSssTableEnd.
constexpr uint32_t kSssTableSize = 2048;
constexpr float kSssTableEnd = 111.686673513429369f;

#if !defined(__CUDA_ARCH__)
inline void sss_build_table(float* table) {
	const auto cdf = [](double r) { return 1.0 - std::exp(-r) / 4.0 - 0.75 * std::exp(-r / 3.0); };
	const auto dcdf = [](double r) { return std::exp(-r) / 4.0 + 0.25 * std::exp(-r / 3.0); };
	table[0] = 0.f;
	for (uint32_t k = 1; k + 1 < kSssTableSize; k++) {
		const double u = static_cast<double>(k) / static_cast<double>(kSssTableSize - 1);
		double r = 1.0;
		for (int it = 0; it < 200; it++) {
			double next = r - (cdf(r) - u) / dcdf(r);
			if (next < 0.0) next = r / 2.0;
			const bool done = std::fabs(next - r) < 1e-15 * (r > 1.0 ? r : 1.0);
			r = next;
			if (done) break;
		}
		table[k] = static_cast<float>(r);
	}
	table[kSssTableSize - 1] = kSssTableEnd;
}
#endif

// sample_from_inv_cdf_table (rainbow-core/sample_function.cpp:84-95) times d:
// the knot interval of u, a lerp s (1 - t) + e t inside it.
RB_HD float sss_sample_profile(const float* table, float d, float u) {
	const float size = static_cast<float>(kSssTableSize - 1);
	uint32_t which = static_cast<uint32_t>(u * size);
	if (which > kSssTableSize - 2) which = kSssTableSize - 2;
	const float t = u * size - static_cast<float>(which);
	const float r = table[which] * (1.f - t) + table[which + 1] * t;
	return r * d;
}

// normalized_diffusion::pdf_reflectance_profile (normalized_diffusion.cpp:397-407).
RB_HD float sss_pdf_profile(float d, float distance) {
	if (distance < 1e-6f) distance = 1e-6f;
	const float r = distance / d;
	return 0.25f * (expf(-r) + expf(-r / 3.f)) / (d * (2.f * kPi) * distance);
}

// normalized_diffusion::evaluate_reflectance_profile (normalized_diffusion.cpp:379-388).
RB_HD spectrum sss_eval_profile(spectrum A, spectrum D, float distance) {
	if (distance < 1e-6f) distance = 1e-6f;
	const auto channel = [&](float a, float d) {
		const float value = a * (expf(-distance / d) + expf(-distance / (d * 3.f)));
		return value / (d * kPi * 8.f * distance);
	};
	return spectrum{channel(A.x, D.x), channel(A.y, D.y), channel(A.z, D.z)};
}

// World dp/du of a hit (mesh.cpp:362-380 after transform_vector, transform.cpp:38-50).
RB_HD vec3 world_dpdu(const scene_view& s, int32_t slot, float b1, float b2) {
	const uint32_t ent = float_as_u32(s.tri_c[slot].y) & kEntityMask;
	const entity_rec& e = s.entities[ent];
	const local_surface ls = triangle_surface(s, s.meshes[e.mesh], s.prim_index[slot], b1, b2);
	return xform_vector(e.l2w, ls.dp_du);
}

constexpr int kSssMaxProbeHits = 64;  // probe-ray steps of one walk (the reference does not bound them)
constexpr uint32_t kSssProbeCache = 8;  // hits the first walk keeps, so that the second walk is needed only beyond them

// The hits of the subsurface material that a probe walk found, with their rays.
struct sss_probe_cache {
	hit_t hit[kSssProbeCache];
	vec3 o[kSssProbeCache], d[kSssProbeCache];
};

// The probe of a BSSRDF sample: walks from `from` toward `to` as the
// reference's loop does (scattering_surface_function.cpp:103-121): spawn_ray_to
// from the last hit (from the bare point, normal 0, at first), closest hit,
// repeat; hits on entities with `material` count. Returns their number (all
// of them when want < 0, else want + 1 once the want-th one, counted from 0,
// is reached) and that hit and its ray in hit_out / o_out / d_out.
// cache (not null, want < 0): receives the first kSssProbeCache hits counted.
template <typename Trace>
RB_HD uint32_t sss_probe(const scene_view& s, uint32_t material, vec3 from, vec3 to, int32_t want, Trace&& trace,
	hit_t& hit_out, vec3& o_out, vec3& d_out, sss_probe_cache* cache = nullptr) {
	vec3 bp = from, bn{0.f, 0.f, 0.f};
	uint32_t found = 0;
	for (int step = 0; step < kSssMaxProbeHits; step++) {
		const ray_t r = spawn_ray_to(bp, bn, to);
		if (r.d.x == 0.f && r.d.y == 0.f && r.d.z == 0.f) break;
		float len = r.len;
		const hit_t h = trace(r.o, r.d, len, false);
		if (h.slot < 0) break;
		const surface_t hs = make_surface(s, h.slot, h.b1, h.b2, r.o, r.d);
		const entity_rec& e = s.entities[hs.entity];
		if ((e.flags & ENT_HAS_MATERIAL) && static_cast<uint32_t>(e.material) == material) {
			if (static_cast<int32_t>(found) == want) {
				hit_out = h;
				o_out = r.o;
				d_out = r.d;
				return found + 1;
			}
			if (cache != nullptr && found < kSssProbeCache) {
				cache->hit[found] = h;
				cache->o[found] = r.o;
				cache->d[found] = r.d;
			}
			found++;
		}
		bp = hs.p;
		bn = hs.n;
	}
	return found;
}

// sample_scattering_surface_function (integrator.cpp:290-327) for a path
// whose BSDF sample at rec's surface (hit `entry`) transmitted into a
// subsurface material: the BSSRDF sample (an exit point on the same material
// and beta *= S / pdf), uniform_sample_one_emitter at the exit with the
// separable_bssrdf_reflection lobe, and the continuation sampled from it.
// trace(o, d, len, shadow): closest hit (shadow: visible entities only).
// Returns false when the path ends.
template <typename Trace>
RB_HD bool subsurface_walk(const scene_view& s, path_state& p, const shade_record& rec, const hit_t& entry, Trace&& trace) {
	const surface_t& si = rec.si;
	material_rec scratch;
	const material_rec* m = hit_material(s, rec.material, si.uv, si.p, scratch);
	// the BSSRDF's frame: shading z, x = normalize(dp/du), y = z x x (scattering_surface_function.cpp:63-69)
	const vec3 fz = si.sz;
	const vec3 fx = normalize(world_dpdu(s, entry.slot, entry.b1, entry.b2));
	const vec3 fy = cross(fz, fx);
	// bssrdf->sample(scene, vector3(sampler1d->next(), sampler2d->next())): the order of the two
	// draws is the compiler's; the reference as built here (g++) evaluates the constructor's
	// arguments right to left, so (y, z) are drawn first and then x
	const vec2 uyz = pcg_2d(p.rng);
	const float u0 = pcg_real(p.rng);
	// sample_axis_and_channel (scattering_surface_function.cpp:7-41)
	vec3 px, py, pz;
	float u = u0;
	if (u < 0.5f) {
		px = fx; py = fy; pz = fz;
		u = u * 2.f;
	} else if (u < 0.75f) {
		px = fy; py = fz; pz = fx;
		u = (u - 0.5f) * 4.f;
	} else {
		px = fz; py = fx; pz = fy;
		u = (u - 0.75f) * 4.f;
	}
	uint32_t channel = static_cast<uint32_t>(u * 3.f);
	if (channel > 2u) channel = 2u;
	u = u * 3.f - static_cast<float>(channel);
	const float d = channel == 0u ? m->sss_d.x : (channel == 1u ? m->sss_d.y : m->sss_d.z);
	const float r = sss_sample_profile(s.sss_table, d, uyz.x);
	if (r < 0.f) return false;
	const float phi = 2.f * kPi * uyz.y;
	const float max_r = sss_sample_profile(s.sss_table, d, 0.999f);
	if (r >= max_r) return false;
	const float l = 2.f * sqrtf(max_r * max_r - r * r);
	const vec3 from = si.p + r * (px * cosf(phi) + py * sinf(phi)) - l * pz * 0.5f;
	const vec3 to = from + l * pz;
	hit_t h{};
	vec3 o{}, dir{};
	sss_probe_cache cache;
	const uint32_t count = sss_probe(s, rec.material, from, to, -1, trace, h, o, dir, &cache);
	if (count == 0u) return false;
	uint32_t which = static_cast<uint32_t>(u * static_cast<float>(count));
	if (which > count - 1u) which = count - 1u;
	// the chosen hit (the reference walks the segment again up to it; the walk is deterministic)
	if (which < kSssProbeCache) {
		h = cache.hit[which];
		o = cache.o[which];
		dir = cache.d[which];
	} else {
		sss_probe(s, rec.material, from, to, static_cast<int32_t>(which), trace, h, o, dir);
	}
	surface_t sx = make_surface(s, h.slot, h.b1, h.b2, o, dir);
	sx.wo = sx.sz;
	const spectrum value = sss_eval_profile(m->sss_a, m->sss_d, length(si.p - sx.p));
	// separable_bidirectional_scattering_surface_distribution_function::pdf (:149-175) / count
	const vec3 dd = si.p - sx.p;
	const vec3 ld{dot(dd, fx), dot(dd, fy), dot(dd, fz)};
	const vec3 ln{dot(sx.n, fx), dot(sx.n, fy), dot(sx.n, fz)};
	const float proj[3] = {sqrtf(ld.y * ld.y + ld.z * ld.z), sqrtf(ld.z * ld.z + ld.x * ld.x), sqrtf(ld.x * ld.x + ld.y * ld.y)};
	const float lnabs[3] = {fabs_ref(ln.x), fabs_ref(ln.y), fabs_ref(ln.z)};
	const float axis_pdf[3] = {0.25f, 0.25f, 0.5f};
	const float channel_pdf = 1.f / 3.f;
	float pdf = 0.f;
	for (uint32_t c = 0; c < 3u; c++) {
		const float dc = c == 0u ? m->sss_d.x : (c == 1u ? m->sss_d.y : m->sss_d.z);
#if defined(__CUDA_ARCH__)
#pragma unroll
#endif
		for (int a = 0; a < 3; a++) pdf = pdf + sss_pdf_profile(dc, proj[a]) * lnabs[a] * channel_pdf * axis_pdf[a];
	}
	pdf = pdf / static_cast<float>(count);
	if (is_black(value) || pdf == 0.f) return false;
	p.beta = p.beta * (value / pdf);
	// uniform_sample_one_emitter at the exit with the separable_bssrdf_reflection lobe
	material_rec exit_rec{};
	exit_rec.kind = MAT_SSS_EXIT;
	exit_rec.eta = m->eta;
	const bsdf_t b = make_bsdf(&exit_rec);
	shade_record r2;
	r2.si = sx;
	r2.material = rec.material;
	r2.pass_through = 0u;
	r2.guidable = 0u;
	r2.nee_entity = -1;
	r2.mis_valid = 0u;
	nee_sample<MAT_ANY>(s, p, sx, b, r2);
	hit_t sh{-1, 0.f, 0.f}, mh{-1, 0.f, 0.f};
	if (r2.nee_entity >= 0) {
		float len = r2.shadow_ray.len;
		sh = trace(r2.shadow_ray.o, r2.shadow_ray.d, len, true);
	}
	if (r2.mis_valid) {
		float len = r2.mis_ray.len;
		mh = trace(r2.mis_ray.o, r2.mis_ray.d, len, true);
	}
	shade_b_direct<MAT_ANY>(s, p, r2, sh, mh);
	// the continuation from the exit (functions.sample with the lobe's cosine sampling)
	const lobe_sample bs = bsdf_sample<MAT_ANY>(b, to_local(sx, sx.wo), pcg_2d(p.rng), ST_ALL);
	if (is_black(bs.f) || bs.pdf == 0.f) return false;
	const vec3 wi = to_world(sx, bs.wi);
	p.beta = p.beta * (bs.f * fabs_ref(dot(wi, sx.sz)) / bs.pdf);
	p.flags = type_match(bs.type, ST_SPECULAR) ? (p.flags | PATH_SPECULAR) : (p.flags & ~PATH_SPECULAR);
	const ray_t nr = spawn_ray(sx.p, sx.n, wi);
	p.o = nr.o;
	p.d = nr.d;
	p.len = nr.len;
	return true;
}

} // namespace pt
} // namespace rb
