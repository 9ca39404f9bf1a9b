// BSDFs of the three supported materials and the lobe-collection rules of
// scattering_function_collection (rainbow-cpu/scatterings/scattering_function_collection.cpp:29-148).
// All directions are in the shading frame (z = shading normal). Host- and
// device-compilable, reference operation order throughout.
#pragma once

#include "pt_types.h"

namespace rb {
namespace pt {

constexpr float kPi = 3.14159265358979323846f;
constexpr float kTwoPi = 6.28318530717958647692f;
constexpr float kHalfPi = 1.57079632679489661923f;
constexpr float kQuarterPi = 0.785398163397448309616f;
constexpr float kInvPi = 0.318309886183790671538f;
constexpr float kInvTwoPi = 0.159154943091895335769f;
constexpr float kOneMinusEps = 1.f - FLT_EPSILON;

// scattering_type bits (rainbow-cpu/scatterings/scattering_function.hpp:26-34)
enum : uint32_t {
	ST_REFLECTION = 1u << 0,
	ST_TRANSMISSION = 1u << 1,
	ST_SPECULAR = 1u << 2,
	ST_DIFFUSE = 1u << 3,
	ST_GLOSSY = 1u << 4,
	ST_ALL = 31u,
	ST_NON_SPECULAR = ST_ALL ^ ST_SPECULAR
};
RB_HD bool type_match(uint32_t target, uint32_t flag) { return (target & flag) == flag; }

// ------------------------------------------------------------------ shading-frame trigonometry
// rainbow-core/shading_function.cpp:3-127
RB_HD float cos2_theta(vec3 w) { return w.z * w.z; }
RB_HD float sin2_theta(vec3 w) { return fmax_ref(0.f, 1.f - cos2_theta(w)); }
RB_HD float sin_theta(vec3 w) { return sqrtf(sin2_theta(w)); }
RB_HD float tan_theta(vec3 w) { return sin_theta(w) / w.z; }
RB_HD float tan2_theta(vec3 w) { return sin2_theta(w) / cos2_theta(w); }
RB_HD float cos_phi(vec3 w) {
	const float s = sin_theta(w);
	return s == 0.f ? 1.f : fclamp_ref(w.x / s, -1.f, 1.f);
}
RB_HD float sin_phi(vec3 w) {
	const float s = sin_theta(w);
	return s == 0.f ? 0.f : fclamp_ref(w.y / s, -1.f, 1.f);
}
RB_HD bool same_hemisphere(vec3 a, vec3 b) { return a.z * b.z > 0.f; }
RB_HD vec3 face_forward(vec3 v, vec3 f) { return dot(v, f) > 0.f ? v : -v; }
RB_HD vec3 reflect(vec3 wi, vec3 n) { return -wi + 2.f * dot(wi, n) * n; }
RB_HD vec3 refract(vec3 wi, vec3 n, float eta) {
	const float ci = dot(wi, n);
	const float s2i = fmax_ref(0.f, 1.f - ci * ci);
	const float s2o = s2i * eta * eta;
	if (s2o >= 1.f) return vec3{0.f, 0.f, 0.f};
	const float co = sqrtf(1.f - s2o);
	return -wi * eta + (ci * eta - co) * n;
}

// rainbow-core/sample_function.cpp:15-44
RB_HD vec2 concentric_disk(vec2 u) {
	const vec2 r = 2.f * u - vec2{1.f, 1.f};
	if (r.x == 0.f && r.y == 0.f) return vec2{0.f, 0.f};
	float theta, rad;
	if (fabs_ref(r.x) > fabs_ref(r.y)) {
		rad = r.x;
		theta = kQuarterPi * (r.y / r.x);
	} else {
		rad = r.y;
		theta = kHalfPi - kQuarterPi * (r.x / r.y);
	}
	return rad * vec2{cosf(theta), sinf(theta)};
}
RB_HD vec3 cosine_hemisphere(vec2 u) {
	const vec2 d = concentric_disk(u);
	const float z = sqrtf(fmax_ref(0.f, 1.f - dot(d, d)));
	return vec3{d.x, d.y, z};
}
RB_HD float cosine_hemisphere_pdf(float c) { return c * kInvPi; }

// ------------------------------------------------------------------ Trowbridge-Reitz
// rainbow-cpu/scatterings/distribution/trowbridge_reitz_distribution.cpp and
// microfacet_distribution.cpp (visible-normal sampling enabled).
RB_HD float tr_d(float ax, float ay, vec3 wh) {
	const float t2 = tan2_theta(wh);
	if (isinf(t2)) return 0.f;
	const float c4 = cos2_theta(wh) * cos2_theta(wh);
	const float cp = cos_phi(wh), sp = sin_phi(wh);
	const float e = (cp * cp / (ax * ax) + sp * sp / (ay * ay)) * t2;
	return 1.f / (kPi * ax * ay * c4 * (1.f + e) * (1.f + e));
}
RB_HD float tr_lambda(float ax, float ay, vec3 w) {
	const float at = fabs_ref(tan_theta(w));
	if (isinf(at)) return 0.f;
	const float cp = cos_phi(w), sp = sin_phi(w);
	const float alpha = sqrtf(cp * cp * ax * ax + sp * sp * ay * ay);
	const float a2 = (alpha * at) * (alpha * at);
	return (-1.f + sqrtf(1.f + a2)) / 2.f;
}
RB_HD float tr_g(float ax, float ay, vec3 wo, vec3 wi) { return 1.f / (1.f + tr_lambda(ax, ay, wo) + tr_lambda(ax, ay, wi)); }
RB_HD float tr_g1(float ax, float ay, vec3 w) { return 1.f / (1.f + tr_lambda(ax, ay, w)); }
RB_HD float tr_pdf(float ax, float ay, vec3 wo, vec3 wh) {
	return tr_d(ax, ay, wh) * tr_g1(ax, ay, wo) * fabs_ref(dot(wo, wh)) / fabs_ref(wo.z);
}

// trowbridge_reitz_sample(cos_theta, u1, u2): slope sampling of the isotropic
// distribution, including its rational approximation of the inverse CDF (:7-45).
RB_HD vec2 tr_sample11(float cos_t, float u1, float u2) {
	if (static_cast<double>(cos_t) > 0.9999) {
		const float r = sqrtf(u1 / (1.f - u1));
		const float phi = kTwoPi * u2;
		return vec2{r * cosf(phi), r * sinf(phi)};
	}
	const float sin_t = sqrtf(fmax_ref(0.f, 1.f - cos_t * cos_t));
	const float tan_t = sin_t / cos_t;
	const float a = 1.f / tan_t;
	const float g1 = 2.f / (1.f + sqrtf(1.f + 1.f / (a * a)));
	const float A = 2.f * u1 / g1 - 1.f;
	float tmp = 1.f / (A * A - 1.f);
	if (static_cast<double>(tmp) > 1e10) tmp = 1e10f;
	const float B = tan_t;
	const float D = sqrtf(fmax_ref(B * B * tmp * tmp - (A * A - B * B) * tmp, 0.f));
	const float sx1 = B * tmp - D;
	const float sx2 = B * tmp + D;
	vec2 slope;
	slope.x = (A < 0.f || sx2 > 1.f / tan_t) ? sx1 : sx2;
	float S;
	if (u2 > 0.5f) {
		S = 1.f;
		u2 = 2.f * (u2 - .5f);
	} else {
		S = -1.f;
		u2 = 2.f * (.5f - u2);
	}
	const float z = (u2 * (u2 * (u2 * 0.27385f - 0.73369f) + 0.46341f)) /
		(u2 * (u2 * (u2 * 0.093073f + 0.309420f) - 1.000000f) + 0.597999f);
	slope.y = S * z * sqrtf(1.f + slope.x * slope.x);
	return slope;
}
RB_HD vec3 tr_sample_visible(vec3 wi, float ax, float ay, float u1, float u2) {
	const vec3 ws = normalize(vec3{ax * wi.x, ay * wi.y, wi.z});
	vec2 slope = tr_sample11(ws.z, u1, u2);
	const float tmp = cos_phi(ws) * slope.x - sin_phi(ws) * slope.y;
	slope.y = sin_phi(ws) * slope.x + cos_phi(ws) * slope.y;
	slope.x = tmp;
	slope.x = ax * slope.x;
	slope.y = ay * slope.y;
	return normalize(vec3{-slope.x, -slope.y, 1.f});
}
RB_HD vec3 tr_sample(float ax, float ay, vec3 wo, vec2 u) {
	const bool flip = wo.z < 0.f;
	const vec3 wh = tr_sample_visible(flip ? -wo : wo, ax, ay, u.x, u.y);
	return flip ? -wh : wh;
}

// ------------------------------------------------------------------ Fresnel
// rainbow-cpu/scatterings/fresnel_effect.cpp:5-58
RB_HD float fresnel_dielectric(float cos_i, float eta_i, float eta_o) {
	cos_i = fclamp_ref(cos_i, -1.f, 1.f);
	if (cos_i < 0.f) {
		const float t = eta_i; eta_i = eta_o; eta_o = t;
		cos_i = fabs_ref(cos_i);
	}
	const float sin_i = sqrtf(fmax_ref(0.f, 1.f - cos_i * cos_i));
	const float sin_o = sin_i * eta_i / eta_o;
	const float cos_o = sqrtf(fmax_ref(0.f, 1.f - sin_o * sin_o));
	if (sin_o >= 1.f) return 1.f;
	const float r0 = (eta_o * cos_i - eta_i * cos_o) / (eta_o * cos_i + eta_i * cos_o);
	const float r1 = (eta_i * cos_i - eta_o * cos_o) / (eta_i * cos_i + eta_o * cos_o);
	return (r0 * r0 + r1 * r1) / 2.f;
}
// conductor with eta_i = 1 (metal_material.cpp:29), one channel
RB_HD float fresnel_conductor1(float cos_i, float eta, float k) {
	cos_i = fclamp_ref(cos_i, -1.f, 1.f);
	const float e = eta / 1.f, ek = k / 1.f;
	const float c2 = cos_i * cos_i;
	const float s2 = 1.f - c2;
	const float e2 = e * e, ek2 = ek * ek;
	const float t0 = e2 - ek2 - s2;
	const float ab = sqrtf(t0 * t0 + e2 * ek2 * 4.f);
	const float t1 = ab + c2;
	const float a = sqrtf((ab + t0) * 0.5f);
	const float t2 = a * 2.f * cos_i;
	const float t3 = ab * c2 + s2 * s2;
	const float t4 = t2 * s2;
	const float r0 = (t1 - t2) / (t1 + t2);
	const float r1 = r0 * (t3 - t4) / (t3 + t4);
	return (r0 + r1) * 0.5f;
}
RB_HD spectrum fresnel_conductor(float cos_i, spectrum eta, spectrum k) {
	const float c = fabs_ref(cos_i);
	return spectrum{fresnel_conductor1(c, eta.x, k.x), fresnel_conductor1(c, eta.y, k.y), fresnel_conductor1(c, eta.z, k.z)};
}

// ------------------------------------------------------------------ lobes
struct lobe_sample {
	uint32_t type;
	spectrum f;
	vec3 wi;
	float pdf;
};
RB_HD lobe_sample no_sample() { return lobe_sample{0u, spectrum{0.f, 0.f, 0.f}, vec3{0.f, 0.f, 0.f}, 0.f}; }

// Lobe kinds in collection order for each material. The LOBE_L_* kinds are
// the lobes of layered materials, whose spectrum (and specular transmission's
// IOR) is the material's per-lobe entry rather than a named field.
enum : uint32_t { LOBE_LAMBERT = 0, LOBE_MF_REFLECT = 1, LOBE_MF_TRANSMIT = 2, LOBE_FRESNEL_SPECULAR = 3,
	LOBE_SPECULAR_REFLECT = 4, LOBE_FRESNEL_BLEND = 5, LOBE_OREN_NAYAR = 6,
	LOBE_L_LAMBERT = 7,           // lambertian_reflection(R)
	LOBE_L_LAMBERT_TRANSMIT = 8,  // lambertian_transmission(T)
	LOBE_L_MF_REFLECT = 9,        // microfacet_reflection(TR, dielectric Fresnel (1, eta), R)
	LOBE_L_MF_TRANSMIT = 10,      // microfacet_transmission(TR, T, 1, eta)
	LOBE_L_SPECULAR_REFLECT = 11, // specular_reflection(dielectric Fresnel (1, eta), R)
	LOBE_L_SPECULAR_TRANSMIT = 12, // specular_transmission(T, 1, lobe_eta)
	LOBE_SSS_EXIT = 13            // separable_bssrdf_reflection(eta) at a subsurface walk's exit
};

// The lobe list: kinds (4 bits each) and scattering types (5 bits each) packed
// in two words, so that a lobe is selected by a shift and the record stays in
// registers whatever the lobe index.
struct bsdf_t {
	uint32_t kinds;
	uint32_t types;
	uint32_t count;
	const material_rec* m;
	float eta;     // collection eta (glass IOR, else 1)
	uint32_t mix;  // a mixture: each lobe reads its own component record (lobe_ref)
	uint32_t importance;  // transport_mode::important (photon paths): transmission without the (eta_i / eta_o)^2 of radiance
};
RB_HD uint32_t lobe_kind(const bsdf_t& b, uint32_t i) { return (b.kinds >> (4u * i)) & 15u; }
RB_HD uint32_t lobe_type(const bsdf_t& b, uint32_t i) { return (b.types >> (5u * i)) & 31u; }
RB_HD void add_lobe(bsdf_t& b, uint32_t kind, uint32_t type) {
	b.kinds |= kind << (4u * b.count);
	b.types |= type << (5u * b.count);
	b.count++;
}

RB_HD bsdf_t make_bsdf(const material_rec* m) {
	bsdf_t b;
	b.m = m;
	b.count = 0;
	b.kinds = 0;
	b.types = 0;
	b.eta = 1.f;
	b.mix = 0;
	b.importance = 0;
	switch (m->kind) {
	case MAT_LAMBERT:
		add_lobe(b, LOBE_LAMBERT, ST_DIFFUSE | ST_REFLECTION);
		break;
	case MAT_OREN_NAYAR:
		add_lobe(b, LOBE_OREN_NAYAR, ST_DIFFUSE | ST_REFLECTION);
		break;
	case MAT_METAL:
		add_lobe(b, LOBE_MF_REFLECT, ST_GLOSSY | ST_REFLECTION);
		break;
	case MAT_GLASS_ROUGH:
		b.eta = m->eta;
		if (m->has_reflect) add_lobe(b, LOBE_MF_REFLECT, ST_GLOSSY | ST_REFLECTION);
		if (m->has_transmit) add_lobe(b, LOBE_MF_TRANSMIT, ST_GLOSSY | ST_TRANSMISSION);
		break;
	case MAT_GLASS_SMOOTH:
		b.eta = m->eta;
		if (m->has_reflect || m->has_transmit) add_lobe(b, LOBE_FRESNEL_SPECULAR, ST_REFLECTION | ST_TRANSMISSION | ST_SPECULAR);
		break;
	case MAT_PLASTIC:
		// plastic_material::build_surface_properties (plastic_material.cpp:30-55): the
		// collection's eta, then the Lambert lobe, then the reflection lobe, each if not black
		b.eta = m->eta;
		if (!is_black(m->diffuse)) add_lobe(b, LOBE_LAMBERT, ST_DIFFUSE | ST_REFLECTION);
		if (m->has_reflect) add_lobe(b, LOBE_MF_REFLECT, ST_GLOSSY | ST_REFLECTION);
		break;
	case MAT_MIRROR:
		add_lobe(b, LOBE_SPECULAR_REFLECT, ST_SPECULAR | ST_REFLECTION);
		break;
	case MAT_SUBSTRATE:
		add_lobe(b, LOBE_FRESNEL_BLEND, ST_GLOSSY | ST_REFLECTION);
		break;
	case MAT_LAYERED:
		b.eta = m->collection_eta;
		b.kinds = m->lobe_kinds;
		b.types = m->lobe_types;
		b.count = m->lobe_count;
		break;
	case MAT_SSS_EXIT:
		// sample_scattering_surface_function's collection (scattering_surface_function.cpp:131-135)
		add_lobe(b, LOBE_SSS_EXIT, ST_DIFFUSE | ST_REFLECTION);
		break;
	case MAT_MIXTURE:
		// mixture_material::build_surface_properties (mixture_material.cpp:13-27): the
		// lobes of both components, the collection's eta left at its default of 1
		b.kinds = m->lobe_kinds;
		b.types = m->lobe_types;
		b.count = m->lobe_count;
		b.mix = 1;
		break;
	default: break;  // black matte: no lobes
	}
	return b;
}

// Material kind known at compile time (a shading class), or MAT_ANY for a
// run-time switch. Specialised code keeps each shading kernel small.
constexpr int MAT_ANY = -1;

// microfacet_reflection::evaluate (scatterings/reflection/microfacet_reflection.cpp):
// conductor Fresnel for metal, else dielectric Fresnel (1, m->eta), scaled by R
// (the material's reflectance field, or a layered lobe's own spectrum).
template <int MAT = MAT_ANY>
RB_HD spectrum mf_reflect_f(const material_rec* m, vec3 wo, vec3 wi, spectrum R) {
	const float co = fabs_ref(wo.z), ci = fabs_ref(wi.z);
	vec3 wh = wi + wo;
	if (co == 0.f || ci == 0.f) return spectrum{0.f, 0.f, 0.f};
	if (wh.x == 0.f && wh.y == 0.f && wh.z == 0.f) return spectrum{0.f, 0.f, 0.f};
	wh = face_forward(normalize(wh), vec3{0.f, 0.f, 1.f});
	spectrum F;
	const bool conductor = MAT == MAT_ANY ? (m->kind == MAT_METAL) : (MAT == static_cast<int>(MAT_METAL));
	if (conductor) F = fresnel_conductor(dot(wi, wh), m->cond_eta, m->cond_k);  // R: 1, or a mixture's weight
	else F = splat3(fresnel_dielectric(dot(wi, wh), 1.f, m->eta));
	const float G = tr_g(m->alpha_x, m->alpha_y, wo, wi);
	const float D = tr_d(m->alpha_x, m->alpha_y, wh);
	return R * (G * D) * F / (4.f * ci * co);
}
RB_HD float mf_reflect_pdf(const material_rec* m, vec3 wo, vec3 wi) {
	if (!same_hemisphere(wo, wi)) return 0.f;
	const vec3 wh = normalize(wo + wi);
	return tr_pdf(m->alpha_x, m->alpha_y, wo, wh) / (4.f * dot(wo, wh));
}
// microfacet_transmission::evaluate (scatterings/transmission/microfacet_transmission.cpp:14-37),
// eta (1, m->eta), scaled by T; importance transport drops the 1 / eta factor (:31).
RB_HD spectrum mf_transmit_f(const material_rec* m, vec3 wo, vec3 wi, spectrum T, uint32_t importance = 0u) {
	if (same_hemisphere(wo, wi)) return spectrum{0.f, 0.f, 0.f};
	const float co = wo.z, ci = wi.z;
	if (co == 0.f || ci == 0.f) return spectrum{0.f, 0.f, 0.f};
	const bool entering = co > 0.f;
	const float eta = entering ? (m->eta / 1.f) : (1.f / m->eta);
	const vec3 wh = face_forward(normalize(wo + wi * eta), vec3{0.f, 0.f, 1.f});
	const float F = fresnel_dielectric(dot(wo, wh), 1.f, m->eta);
	const float denom = dot(wo, wh) + eta * dot(wi, wh);
	const float factor = importance ? 1.f : 1.f / eta;
	const float D = tr_d(m->alpha_x, m->alpha_y, wh);
	const float G = tr_g(m->alpha_x, m->alpha_y, wo, wi);
	const float v = fabs_ref(D * G * eta * eta * fabs_ref(dot(wi, wh)) * fabs_ref(dot(wo, wh) * factor * factor) /
		(ci * co * denom * denom));
	return (splat3(1.f) - splat3(F)) * T * v;
}
RB_HD float mf_transmit_pdf(const material_rec* m, vec3 wo, vec3 wi) {
	if (same_hemisphere(wo, wi)) return 0.f;
	const bool entering = wo.z > 0.f;
	const float eta = entering ? (m->eta / 1.f) : (1.f / m->eta);
	const vec3 wh = normalize(wo + wi * eta);
	const float denom = dot(wo, wh) + eta * dot(wi, wh);
	return tr_pdf(m->alpha_x, m->alpha_y, wo, wh) * fabs_ref((eta * eta * dot(wi, wh)) / (denom * denom));
}

// fresnel_blend_reflection (scatterings/reflection/fresnel_blend_reflection.cpp):
// Rd (28 / (23 pi)) (1 - Rs) (1 - (1 - |cos_i| / 2)^5) (1 - (1 - |cos_o| / 2)^5)
// plus the Schlick-Fresnel glossy term F(wo . wh) D / (4 |wi . wh| max(|cos_i|, |cos_o|)).
RB_HD float pow5(float v) { return (v * v) * (v * v) * v; }
RB_HD spectrum fresnel_blend_f(const material_rec* m, vec3 wo, vec3 wi) {
	vec3 wh = wo + wi;
	if (wh.x == 0.f && wh.y == 0.f && wh.z == 0.f) return spectrum{0.f, 0.f, 0.f};
	wh = normalize(wh);
	const spectrum diffuse = m->diffuse * (28.f / (23.f * kPi)) * (splat3(1.f) - m->reflectance) *
		(1.f - pow5(1.f - 0.5f * fabs_ref(wi.z))) * (1.f - pow5(1.f - 0.5f * fabs_ref(wo.z)));
	const float D = tr_d(m->alpha_x, m->alpha_y, wh);
	const spectrum fresnel = m->reflectance + (splat3(1.f) - m->reflectance) * pow5(1.f - dot(wo, wh));
	const spectrum specular = fresnel * D / (4.f * fabs_ref(dot(wi, wh)) * fmax_ref(fabs_ref(wi.z), fabs_ref(wo.z)));
	return m->blend_scale * (specular + diffuse);  // the layer's scale: 1, or a mixture's weight
}
RB_HD float fresnel_blend_pdf(const material_rec* m, vec3 wo, vec3 wi) {
	if (!same_hemisphere(wo, wi)) return 0.f;
	const vec3 wh = normalize(wo + wi);
	const float pd = tr_pdf(m->alpha_x, m->alpha_y, wo, wh) / (4.f * dot(wo, wh));
	const float ph = cosine_hemisphere_pdf(fabs_ref(wi.z));
	return 0.5f * (pd + ph);
}

// oren_nayar_reflection::evaluate (scatterings/reflection/oren_nayar_reflection.cpp:18-47):
// R / pi * (A + B max(0, cos(phi_i - phi_o)) sin(alpha) tan(beta)), with A and B
// (the material's alpha_x / alpha_y) computed on the host from sigma. The
// 1e-4 threshold is a double literal in the reference, so the test is in double.
RB_HD spectrum oren_nayar_f(const material_rec* m, vec3 wo, vec3 wi) {
	const float sin_theta_i = sin_theta(wi), sin_theta_o = sin_theta(wo);
	float max_cos = 0.f;
	if (static_cast<double>(sin_theta_i) > 1e-4 && static_cast<double>(sin_theta_o) > 1e-4) {
		const float sin_phi_i = sin_phi(wi), sin_phi_o = sin_phi(wo);
		const float cos_phi_i = cos_phi(wi), cos_phi_o = cos_phi(wo);
		max_cos = fmax_ref(0.f, cos_phi_i * cos_phi_o + sin_phi_i * sin_phi_o);
	}
	float sin_alpha, tan_beta;
	if (fabs_ref(wi.z) > fabs_ref(wo.z)) {
		sin_alpha = sin_theta_o;
		tan_beta = sin_theta_i / fabs_ref(wi.z);
	} else {
		sin_alpha = sin_theta_i;
		tan_beta = sin_theta_o / fabs_ref(wo.z);
	}
	return m->diffuse * kInvPi * (m->alpha_x + m->alpha_y * max_cos * sin_alpha * tan_beta);
}

// fresnel_moment1 (scatterings/reflection/separable_bssrdf_reflection.cpp:7-20):
// the first moment of the dielectric Fresnel reflectance as a polynomial in
// eta, the published fit of d'Eon and Irving (2011), in float.
RB_HD float fresnel_moment1(float eta) {
	const float eta2 = eta * eta, eta3 = eta2 * eta, eta4 = eta3 * eta, eta5 = eta4 * eta;
	if (eta < 1.f)
		return 0.45966f - 1.73965f * eta + 3.37668f * eta2 - 3.904945f * eta3 + 2.49277f * eta4 - 0.68441f * eta5;
	return -4.61686f + 11.1136f * eta - 10.4646f * eta2 + 5.11455f * eta3 - 1.27198f * eta4 + 0.12746f * eta5;
}
// separable_bssrdf_reflection::evaluate (separable_bssrdf_reflection.cpp:27-34),
// radiance transport: (1 - Fr(cos theta_i)) / (c pi) eta^2, c = 1 - 2 moment1(1 / eta).
RB_HD float sss_exit_f(float eta, float cos_i) {
	const float c = 1.f - 2.f * fresnel_moment1(1.f / eta);
	const float value = (1.f - fresnel_dielectric(cos_i, 1.f, eta)) / (c * kPi);
	return value * (eta * eta);
}

// The record a lobe reads and the lobe's index in it: the material's own
// record, or for a mixture the component record the lobe came from.
template <int MAT = MAT_ANY>
RB_HD const material_rec* lobe_rec(const bsdf_t& b, uint32_t i) {
	if constexpr (MAT != MAT_ANY) return b.m;
	else return b.mix ? b.m + (b.m->lobe_ref[i] >> 4) : b.m;
}
RB_HD uint32_t lobe_local(const bsdf_t& b, uint32_t i) { return b.mix ? (b.m->lobe_ref[i] & 15u) : i; }
// A layered lobe's own spectrum.
RB_HD spectrum layered_r(const bsdf_t& b, uint32_t i) { return lobe_rec(b, i)->lobe_r[lobe_local(b, i)]; }

template <int MAT>
RB_HD spectrum lobe_f(const bsdf_t& b, uint32_t i, vec3 wo, vec3 wi) {
	if constexpr (MAT == static_cast<int>(MAT_LAMBERT)) return b.m->diffuse * kInvPi;
	else if constexpr (MAT == static_cast<int>(MAT_METAL)) return mf_reflect_f<MAT>(b.m, wo, wi, b.m->reflectance);
	else if constexpr (MAT == static_cast<int>(MAT_GLASS_ROUGH))
		return lobe_kind(b, i) == LOBE_MF_REFLECT ? mf_reflect_f<MAT>(b.m, wo, wi, b.m->reflectance)
		                                          : mf_transmit_f(b.m, wo, wi, b.m->transmission, b.importance);
	else {
		const material_rec* m = lobe_rec(b, i);
		switch (lobe_kind(b, i)) {
		case LOBE_LAMBERT: return m->diffuse * kInvPi;
		case LOBE_OREN_NAYAR: return oren_nayar_f(m, wo, wi);
		case LOBE_MF_REFLECT: return mf_reflect_f<MAT_ANY>(m, wo, wi, m->reflectance);
		case LOBE_MF_TRANSMIT: return mf_transmit_f(m, wo, wi, m->transmission, b.importance);
		case LOBE_FRESNEL_BLEND: return fresnel_blend_f(m, wo, wi);
		// lambertian_reflection / lambertian_transmission::evaluate: R / pi, T / pi
		case LOBE_L_LAMBERT:
		case LOBE_L_LAMBERT_TRANSMIT: return layered_r(b, i) * kInvPi;
		case LOBE_L_MF_REFLECT: return mf_reflect_f<MAT_ANY>(m, wo, wi, layered_r(b, i));
		case LOBE_L_MF_TRANSMIT: return mf_transmit_f(m, wo, wi, layered_r(b, i), b.importance);
		case LOBE_SSS_EXIT: return splat3(sss_exit_f(m->eta, wi.z));
		default: return spectrum{0.f, 0.f, 0.f};  // specular lobes evaluate to 0
		}
	}
}
template <int MAT>
RB_HD float lobe_pdf(const bsdf_t& b, uint32_t i, vec3 wo, vec3 wi) {
	if constexpr (MAT == static_cast<int>(MAT_LAMBERT)) return same_hemisphere(wo, wi) ? cosine_hemisphere_pdf(fabs_ref(wi.z)) : 0.f;
	else if constexpr (MAT == static_cast<int>(MAT_METAL)) return mf_reflect_pdf(b.m, wo, wi);
	else if constexpr (MAT == static_cast<int>(MAT_GLASS_ROUGH))
		return lobe_kind(b, i) == LOBE_MF_REFLECT ? mf_reflect_pdf(b.m, wo, wi) : mf_transmit_pdf(b.m, wo, wi);
	else {
		const material_rec* m = lobe_rec(b, i);
		switch (lobe_kind(b, i)) {
		case LOBE_LAMBERT:
		case LOBE_OREN_NAYAR:
		case LOBE_L_LAMBERT:
		case LOBE_SSS_EXIT: return same_hemisphere(wo, wi) ? cosine_hemisphere_pdf(fabs_ref(wi.z)) : 0.f;
		// transmission_function::pdf (scatterings/transmission/transmission_function.cpp:25-28)
		case LOBE_L_LAMBERT_TRANSMIT: return same_hemisphere(wo, wi) ? 0.f : cosine_hemisphere_pdf(fabs_ref(wi.z));
		case LOBE_MF_REFLECT:
		case LOBE_L_MF_REFLECT: return mf_reflect_pdf(m, wo, wi);
		case LOBE_MF_TRANSMIT:
		case LOBE_L_MF_TRANSMIT: return mf_transmit_pdf(m, wo, wi);
		case LOBE_FRESNEL_BLEND: return fresnel_blend_pdf(m, wo, wi);
		default: return 0.f;  // specular lobes: pdf 0
		}
	}
}

template <int MAT>
RB_HD lobe_sample sample_lambert(const bsdf_t& b, uint32_t i, vec3 wo, vec2 u) {
	vec3 wi = cosine_hemisphere(u);
	if (wo.z < 0.f) wi.z = -wi.z;
	return lobe_sample{lobe_type(b, i), lobe_f<MAT>(b, i, wo, wi), wi, lobe_pdf<MAT>(b, i, wo, wi)};
}
// transmission_function::sample (scatterings/transmission/transmission_function.cpp:11-23):
// the cosine hemisphere on the side opposite wo.
RB_HD lobe_sample sample_lambert_transmit(const bsdf_t& b, uint32_t i, vec3 wo, vec2 u) {
	vec3 wi = cosine_hemisphere(u);
	if (wo.z > 0.f) wi.z = -wi.z;
	return lobe_sample{lobe_type(b, i), lobe_f<MAT_ANY>(b, i, wo, wi), wi, lobe_pdf<MAT_ANY>(b, i, wo, wi)};
}
template <int MAT>
RB_HD lobe_sample sample_mf_reflect(const bsdf_t& b, uint32_t i, vec3 wo, vec2 u, spectrum R) {
	const material_rec* m = lobe_rec<MAT>(b, i);
	if (wo.z == 0.f) return no_sample();
	const vec3 wh = tr_sample(m->alpha_x, m->alpha_y, wo, u);
	if (dot(wo, wh) < 0.f) return no_sample();
	const vec3 wi = reflect(wo, wh);
	if (!same_hemisphere(wo, wi)) return no_sample();
	return lobe_sample{lobe_type(b, i), mf_reflect_f<MAT>(m, wo, wi, R), wi, tr_pdf(m->alpha_x, m->alpha_y, wo, wh) / (4.f * dot(wo, wh))};
}
template <int MAT>
RB_HD lobe_sample sample_mf_transmit(const bsdf_t& b, uint32_t i, vec3 wo, vec2 u, spectrum T) {
	const material_rec* m = lobe_rec<MAT>(b, i);
	if (wo.z == 0.f) return no_sample();
	const vec3 wh = tr_sample(m->alpha_x, m->alpha_y, wo, u);
	if (dot(wo, wh) < 0.f) return no_sample();
	const bool entering = wo.z > 0.f;
	const float eta = entering ? (1.f / m->eta) : (m->eta / 1.f);
	const vec3 wi = refract(wo, wh, eta);
	if (is_zero(wi)) return no_sample();
	return lobe_sample{lobe_type(b, i), mf_transmit_f(m, wo, wi, T, b.importance), wi, mf_transmit_pdf(m, wo, wi)};
}
// fresnel_specular::sample (rainbow-cpu/scatterings/mixture/fresnel_specular.cpp:25-54)
RB_HD lobe_sample sample_fresnel_specular(const material_rec* m, vec3 wo, vec2 u, uint32_t importance) {
	const float F = fresnel_dielectric(wo.z, 1.f, m->eta);
	if (u.x < F) {
		const vec3 wi{-wo.x, -wo.y, wo.z};
		return lobe_sample{ST_REFLECTION | ST_SPECULAR, m->reflectance * F / fabs_ref(wi.z), wi, F};
	}
	const bool entering = wo.z > 0.f;
	const float ei = entering ? 1.f : m->eta;
	const float eo = entering ? m->eta : 1.f;
	const vec3 wi = refract(wo, face_forward(vec3{0.f, 0.f, 1.f}, wo), ei / eo);
	if (is_zero(wi)) return no_sample();
	const float factor = importance ? 1.f : (ei * ei) / (eo * eo);
	const spectrum v = m->transmission * (splat3(1.f) - splat3(F)) * factor / fabs_ref(wi.z);
	return lobe_sample{ST_TRANSMISSION | ST_SPECULAR, v, wi, 1.f - F};
}

// fresnel_blend_reflection::sample: u.x below one half picks the cosine
// hemisphere, above it the Trowbridge-Reitz half vector, u.x remapped to [0, 1).
RB_HD lobe_sample sample_fresnel_blend(const material_rec* m, vec3 wo, vec2 u) {
	vec3 wi;
	if (u.x < 0.5f) {
		wi = cosine_hemisphere(vec2{fmin_ref(2.f * u.x, kOneMinusEps), u.y});
		if (wo.z < 0.f) wi.z = -wi.z;
	} else {
		const vec3 wh = tr_sample(m->alpha_x, m->alpha_y, wo, vec2{fmin_ref(2.f * (u.x - 0.5f), kOneMinusEps), u.y});
		wi = reflect(wo, wh);
		if (!same_hemisphere(wo, wi)) return no_sample();
	}
	return lobe_sample{ST_GLOSSY | ST_REFLECTION, fresnel_blend_f(m, wo, wi), wi, fresnel_blend_pdf(m, wo, wi)};
}

// specular_reflection::sample with fresnel_effect_nop (specular_reflection.cpp:16-31):
// the mirror direction, f = reflectance / |cos theta_i|, pdf 1.
RB_HD lobe_sample sample_specular_reflect(const material_rec* m, vec3 wo) {
	const vec3 wi{-wo.x, -wo.y, wo.z};
	return lobe_sample{ST_SPECULAR | ST_REFLECTION, m->reflectance / fabs_ref(wi.z), wi, 1.f};
}
// specular_reflection::sample with a dielectric Fresnel (1, m->eta):
// f = F(cos theta_i) R / |cos theta_i|, pdf 1.
RB_HD lobe_sample sample_layered_specular_reflect(const bsdf_t& b, uint32_t i, vec3 wo) {
	const vec3 wi{-wo.x, -wo.y, wo.z};
	const float F = fresnel_dielectric(wi.z, 1.f, lobe_rec(b, i)->eta);
	return lobe_sample{ST_SPECULAR | ST_REFLECTION, splat3(F) * layered_r(b, i) / fabs_ref(wi.z), wi, 1.f};
}
// specular_transmission::sample (scatterings/transmission/specular_transmission.cpp:17-46),
// radiance transport, eta (1, lobe_eta): refraction about the normal on wo's
// side, f = T (1 - F(cos theta_i)) (eta_i / eta_o)^2 / |cos theta_i|, pdf 1.
RB_HD lobe_sample sample_specular_transmit(const bsdf_t& b, uint32_t i, vec3 wo) {
	const float lobe_eta = lobe_rec(b, i)->lobe_eta[lobe_local(b, i)];
	const bool entering = wo.z > 0.f;
	const float ei = entering ? 1.f : lobe_eta;
	const float eo = entering ? lobe_eta : 1.f;
	const vec3 wi = refract(wo, face_forward(vec3{0.f, 0.f, 1.f}, wo), ei / eo);
	if (is_zero(wi)) return no_sample();
	const float F = fresnel_dielectric(wi.z, 1.f, lobe_eta);
	const float factor = b.importance ? 1.f : (ei * ei) / (eo * eo);
	const spectrum v = layered_r(b, i) * (splat3(1.f) - splat3(F)) * factor / fabs_ref(wi.z);
	return lobe_sample{ST_SPECULAR | ST_TRANSMISSION, v, wi, 1.f};
}

template <int MAT>
RB_HD lobe_sample lobe_sample_dir(const bsdf_t& b, uint32_t i, vec3 wo, vec2 u) {
	if constexpr (MAT == static_cast<int>(MAT_LAMBERT)) return sample_lambert<MAT>(b, i, wo, u);
	else if constexpr (MAT == static_cast<int>(MAT_METAL)) return sample_mf_reflect<MAT>(b, i, wo, u, b.m->reflectance);
	else if constexpr (MAT == static_cast<int>(MAT_GLASS_ROUGH))
		return lobe_kind(b, i) == LOBE_MF_REFLECT ? sample_mf_reflect<MAT>(b, i, wo, u, b.m->reflectance)
		                                          : sample_mf_transmit<MAT>(b, i, wo, u, b.m->transmission);
	else {
		const material_rec* m = lobe_rec(b, i);
		switch (lobe_kind(b, i)) {
		case LOBE_LAMBERT:
		case LOBE_OREN_NAYAR:
		case LOBE_L_LAMBERT:
		case LOBE_SSS_EXIT: return sample_lambert<MAT_ANY>(b, i, wo, u);  // reflection_function::sample, cosine
		case LOBE_L_LAMBERT_TRANSMIT: return sample_lambert_transmit(b, i, wo, u);
		case LOBE_MF_REFLECT: return sample_mf_reflect<MAT_ANY>(b, i, wo, u, m->reflectance);
		case LOBE_L_MF_REFLECT: return sample_mf_reflect<MAT_ANY>(b, i, wo, u, layered_r(b, i));
		case LOBE_MF_TRANSMIT: return sample_mf_transmit<MAT_ANY>(b, i, wo, u, m->transmission);
		case LOBE_L_MF_TRANSMIT: return sample_mf_transmit<MAT_ANY>(b, i, wo, u, layered_r(b, i));
		case LOBE_FRESNEL_SPECULAR: return sample_fresnel_specular(m, wo, u, b.importance);
		case LOBE_SPECULAR_REFLECT: return sample_specular_reflect(m, wo);
		case LOBE_L_SPECULAR_REFLECT: return sample_layered_specular_reflect(b, i, wo);
		case LOBE_L_SPECULAR_TRANSMIT: return sample_specular_transmit(b, i, wo);
		case LOBE_FRESNEL_BLEND: return sample_fresnel_blend(m, wo, u);
		default: return no_sample();
		}
	}
}

// ------------------------------------------------------------------ collection
// scattering_function_collection::evaluate (:29-46)
template <int MAT = MAT_ANY>
RB_HD spectrum bsdf_f(const bsdf_t& b, vec3 wo, vec3 wi, uint32_t include) {
	if (wo.z == 0.f) return spectrum{0.f, 0.f, 0.f};
	const uint32_t rt = same_hemisphere(wo, wi) ? ST_REFLECTION : ST_TRANSMISSION;
	spectrum f{0.f, 0.f, 0.f};
	for (uint32_t i = 0; i < b.count; i++)
		if (type_match(include, lobe_type(b, i)) && type_match(lobe_type(b, i), rt)) f = f + lobe_f<MAT>(b, i, wo, wi);
	return f;
}
// scattering_function_collection::pdf (:131-148)
template <int MAT = MAT_ANY>
RB_HD float bsdf_pdf(const bsdf_t& b, vec3 wo, vec3 wi, uint32_t include) {
	if (b.count == 0 || wo.z == 0.f) return 0.f;
	uint32_t n = 0;
	float pdf = 0.f;
	for (uint32_t i = 0; i < b.count; i++)
		if (type_match(include, lobe_type(b, i))) {
			pdf = pdf + lobe_pdf<MAT>(b, i, wo, wi);
			n++;
		}
	return n != 0 ? pdf / static_cast<float>(n) : 0.f;
}
RB_HD uint32_t bsdf_count(const bsdf_t& b, uint32_t include) {
	uint32_t n = 0;
	for (uint32_t i = 0; i < b.count; i++)
		if (type_match(include, lobe_type(b, i))) n++;
	return n;
}
// scattering_function_collection::sample (:48-100) with wo already in the
// shading frame; the returned wi is in the shading frame too.
template <int MAT = MAT_ANY>
RB_HD lobe_sample bsdf_sample(const bsdf_t& b, vec3 wo, vec2 u, uint32_t include) {
	const uint32_t n = bsdf_count(b, include);
	if (n == 0) return no_sample();
	const float fn = static_cast<float>(n);
	uint32_t which = static_cast<uint32_t>(floorf(u.x * fn));
	if (which > n - 1) which = n - 1;
	const float rx = u.x * fn - static_cast<float>(which);
	const vec2 ur{(kOneMinusEps < rx) ? kOneMinusEps : rx, u.y};
	if (wo.z == 0.f) return no_sample();
	// the which-th lobe matching include, in collection order
	uint32_t pick = 0;
	for (uint32_t i = 0, k = 0; i < b.count; i++)
		if (type_match(include, lobe_type(b, i))) {
			if (k == which) pick = i;
			k++;
		}
	lobe_sample s = lobe_sample_dir<MAT>(b, pick, wo, ur);
	if (s.pdf == 0.f) return no_sample();
	if (!type_match(s.type, ST_SPECULAR)) {
		const uint32_t rt = same_hemisphere(wo, s.wi) ? ST_REFLECTION : ST_TRANSMISSION;
		s.f = spectrum{0.f, 0.f, 0.f};
		s.pdf = 0.f;
		for (uint32_t i = 0; i < b.count; i++) {
			if (!type_match(include, lobe_type(b, i))) continue;
			if (type_match(lobe_type(b, i), rt)) s.f = s.f + lobe_f<MAT>(b, i, wo, s.wi);
			s.pdf = s.pdf + lobe_pdf<MAT>(b, i, wo, s.wi);
		}
	}
	s.pdf = s.pdf / fn;
	return s;
}

// trowbridge_reitz_distribution::roughness_to_alpha (:128-137); host-side use.
RB_HD float roughness_to_alpha(float roughness) {
	roughness = fmax_ref(roughness, 1e-3f);
	const float x = logf(roughness);
	return 1.62142f + 0.819955f * x + 0.1734f * x * x + 0.0171201f * x * x * x + 0.000640711f * x * x * x * x;
}

} // namespace pt
} // namespace rb
