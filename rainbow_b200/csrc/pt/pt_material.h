// Material records from material parameters, and image textures.
//
// build_record does what each reference material's build_surface_properties
// does for the parameters it is given (constant textures, or image textures
// already sampled at the hit): which lobes, with which spectra, in which
// order. The host calls it once per material at upload; for a material with
// image-textured spectra the shading code calls it at every hit (hit_material)
// with the texels at the hit's uv, so both give the reference's lobes.
#pragma once

#include "../../../include/rbgpu.h"
#include "pt_bsdf.h"
#include "pt_geom.h"

namespace rb {
namespace pt {

RB_HD bool is_black3(vec3 c) { return c.x == 0.f && c.y == 0.f && c.z == 0.f; }

RB_HD void layered_lobe(material_rec& r, uint32_t kind, uint32_t type, vec3 spectrum, float eta = 1.f) {
	r.lobe_kinds |= kind << (4u * r.lobe_count);
	r.lobe_types |= type << (5u * r.lobe_count);
	r.lobe_r[r.lobe_count] = spectrum;
	r.lobe_eta[r.lobe_count] = eta;
	r.lobe_count++;
}

// The lobe lists of uber_material::build_surface_properties (uber_material.cpp:26-75)
// and translucent_material::build_surface_properties (translucent_material.cpp:23-69),
// radiance transport: the same lobes, spectra and order. scale (not null): the
// overloads with a scale (uber_material.cpp:77-126, translucent_material.cpp:71-117),
// which multiply in different places.
RB_HD void build_layered(const material_src& p, const vec3* scale, material_rec& r) {
	r.kind = MAT_LAYERED;
	r.alpha_x = p.alpha_x;
	r.alpha_y = p.alpha_y;
	if (p.kind == RB_MATERIAL_UBER) {
		const float eta = p.ior;
		r.eta = r.collection_eta = eta;
		const vec3 reflectance = p.opacity * p.reflectance;
		const vec3 transmission = p.opacity * p.transmission;
		const vec3 specular = p.opacity * p.specular;
		const vec3 diffuse = p.opacity * p.diffuse;
		// clamp(spectrum(1) - opacity) to [0, 1]
		vec3 invert;
		invert.x = fclamp_ref(1.f - p.opacity.x, 0.f, 1.f);
		invert.y = fclamp_ref(1.f - p.opacity.y, 0.f, 1.f);
		invert.z = fclamp_ref(1.f - p.opacity.z, 0.f, 1.f);
		// the black tests are on the unscaled spectra, the lobes take them times scale
		const vec3 one{1.f, 1.f, 1.f};
		const bool sc = scale != nullptr;
		const vec3 s = sc ? *scale : one;
		if (!is_black3(invert)) layered_lobe(r, LOBE_L_SPECULAR_TRANSMIT, ST_SPECULAR | ST_TRANSMISSION, sc ? invert * s : invert, 1.f);
		if (!is_black3(diffuse)) layered_lobe(r, LOBE_L_LAMBERT, ST_DIFFUSE | ST_REFLECTION, sc ? diffuse * s : diffuse);
		if (!is_black3(specular)) layered_lobe(r, LOBE_L_MF_REFLECT, ST_GLOSSY | ST_REFLECTION, sc ? specular * s : specular);
		if (!is_black3(reflectance))
			layered_lobe(r, LOBE_L_SPECULAR_REFLECT, ST_SPECULAR | ST_REFLECTION, sc ? reflectance * s : reflectance);
		if (!is_black3(transmission))
			layered_lobe(r, LOBE_L_SPECULAR_TRANSMIT, ST_SPECULAR | ST_TRANSMISSION, sc ? transmission * s : transmission, eta);
		return;
	}
	// translucent: IOR 1.5, one isotropic roughness; the scaled build scales
	// specular and diffuse before its black tests and products
	const float eta = 1.5f;
	r.eta = r.collection_eta = eta;
	const vec3 R = p.reflectance, T = p.transmission;
	const vec3 S = scale ? p.specular * *scale : p.specular;
	const vec3 D = scale ? p.diffuse * *scale : p.diffuse;
	const bool has_r = !is_black3(R), has_t = !is_black3(T);
	if (!has_r && !has_t) return;
	if (!is_black3(D)) {
		if (has_r) layered_lobe(r, LOBE_L_LAMBERT, ST_DIFFUSE | ST_REFLECTION, D * R);
		if (has_t) layered_lobe(r, LOBE_L_LAMBERT_TRANSMIT, ST_DIFFUSE | ST_TRANSMISSION, D * T);
	}
	if (!is_black3(S)) {
		if (has_r) layered_lobe(r, LOBE_L_MF_REFLECT, ST_GLOSSY | ST_REFLECTION, S * R);
		if (has_t) layered_lobe(r, LOBE_L_MF_TRANSMIT, ST_GLOSSY | ST_TRANSMISSION, S * T);
	}
}

// One material's record: build_surface_properties, or with `scale` (not null)
// its overload with a scale, as a mixture calls it: matte, glass, plastic and
// mirror multiply their spectra before their tests (matte_material.cpp:31-47,
// glass_material.cpp:66-108, plastic_material.cpp:57-84, mirror_material.cpp:28-44),
// metal's microfacet reflection takes the scale as its spectrum
// (metal_material.cpp:39-59), the substrate's Fresnel-blend layer takes it as its
// scale (substrate_material.cpp:38-58). False for a kind it does not build.
// The fields of a material source that derive from its reals, as the
// reference's materials derive them in build_surface_properties: the
// Trowbridge-Reitz alphas (roughness_to_alpha when the material maps
// roughness, trowbridge_reitz_distribution.cpp:128-137; plastic and
// translucent take roughness u for both), glass and subsurface smooth when
// both roughnesses are 0, and the matte's sigma clamped to [0, 90] with
// oren_nayar_reflection's A and B (oren_nayar_reflection.cpp:5-16: radians in
// float, then A and B in double, rounded to float). Called once on the host
// for constant reals, at every hit for textured ones.
RB_HD void derive_src(material_src& p) {
	const auto alpha = [&](float v) { return p.remap ? roughness_to_alpha(v) : v; };
	switch (p.kind) {
	case RB_MATERIAL_MATTE: {
		const float sigma = fclamp_ref(p.sigma, 0.f, 90.f);
		p.oren_nayar = sigma != 0.f ? 1u : 0u;
		if (p.oren_nayar) {
			const float sr = sigma * 0.01745329251994329576923690768489f;
			const float s2 = sr * sr;
			p.on_a = static_cast<float>(1. - (s2 / (2 * (s2 + 0.33))));
			p.on_b = static_cast<float>(0.45 * s2 / (s2 + 0.09));
		}
		return;
	}
	case RB_MATERIAL_METAL:
	case RB_MATERIAL_SUBSTRATE:
	case RB_MATERIAL_UBER:
		p.alpha_x = alpha(p.roughness_u);
		p.alpha_y = alpha(p.roughness_v);
		return;
	case RB_MATERIAL_GLASS:
	case RB_MATERIAL_SUBSURFACE:
		p.smooth = (p.roughness_u == 0.f && p.roughness_v == 0.f) ? 1u : 0u;
		if (!p.smooth) {
			p.alpha_x = alpha(p.roughness_u);
			p.alpha_y = alpha(p.roughness_v);
		}
		return;
	case RB_MATERIAL_PLASTIC:
	case RB_MATERIAL_TRANSLUCENT:
		p.alpha_x = p.alpha_y = alpha(p.roughness_u);
		return;
	default: return;
	}
}

RB_HD bool build_record(const material_src& p, const vec3* scale, material_rec& r) {
	r = material_rec{};
	r.blend_scale = vec3{1.f, 1.f, 1.f};
	const auto sc = [&](vec3 v) { return scale ? v * *scale : v; };
	switch (p.kind) {
	case RB_MATERIAL_MATTE: {
		const vec3 diffuse = sc(p.diffuse);
		if (is_black3(diffuse)) r.kind = MAT_BLACK;
		else if (p.oren_nayar) {
			r.kind = MAT_OREN_NAYAR;
			r.alpha_x = p.on_a;
			r.alpha_y = p.on_b;
		} else r.kind = MAT_LAMBERT;
		r.diffuse = diffuse;
		return true;
	}
	case RB_MATERIAL_METAL:
		r.kind = MAT_METAL;
		r.alpha_x = p.alpha_x;
		r.alpha_y = p.alpha_y;
		r.cond_eta = p.cond_eta;
		r.cond_k = p.cond_k;
		r.reflectance = scale ? *scale : vec3{1.f, 1.f, 1.f};
		return true;
	case RB_MATERIAL_GLASS: {
		const vec3 reflectance = sc(p.reflectance), transmission = sc(p.transmission);
		r.kind = p.smooth ? MAT_GLASS_SMOOTH : MAT_GLASS_ROUGH;
		if (!p.smooth) {
			r.alpha_x = p.alpha_x;
			r.alpha_y = p.alpha_y;
		}
		r.eta = p.ior;
		r.reflectance = reflectance;
		r.transmission = transmission;
		r.has_reflect = is_black3(reflectance) ? 0u : 1u;
		r.has_transmit = is_black3(transmission) ? 0u : 1u;
		return true;
	}
	case RB_MATERIAL_PLASTIC:
		r.kind = MAT_PLASTIC;
		r.alpha_x = r.alpha_y = p.alpha_x;
		r.eta = p.ior;
		r.diffuse = sc(p.diffuse);
		r.reflectance = sc(p.reflectance);
		r.has_reflect = is_black3(r.reflectance) ? 0u : 1u;
		return true;
	case RB_MATERIAL_SUBSTRATE:
		r.kind = (is_black3(p.reflectance) && is_black3(p.diffuse)) ? MAT_BLACK : MAT_SUBSTRATE;
		r.alpha_x = p.alpha_x;
		r.alpha_y = p.alpha_y;
		r.diffuse = p.diffuse;
		r.reflectance = p.reflectance;
		if (scale) r.blend_scale = *scale;
		return true;
	case RB_MATERIAL_MIRROR:
		r.reflectance = sc(p.reflectance);
		r.kind = is_black3(r.reflectance) ? MAT_BLACK : MAT_MIRROR;
		return true;
	case RB_MATERIAL_UBER:
	case RB_MATERIAL_TRANSLUCENT:
		build_layered(p, scale, r);
		return true;
	case RB_MATERIAL_SUBSURFACE: {
		// subsurface_material::build_surface_properties (subsurface_material.cpp:24-66):
		// nothing when transmission or reflectance is black, nor in the overload with a
		// scale (:68-73); else glass lobes and the normalized-diffusion BSSRDF, whose
		// constructor (normalized_diffusion.cpp:358-377) sets s = 1.85 - A + 7 |A - 0.8|^3
		// and d = mfp / s
		if (scale != nullptr || is_black3(p.transmission) || is_black3(p.reflectance)) {
			r.kind = MAT_BLACK;
			return true;
		}
		r.kind = p.smooth ? MAT_GLASS_SMOOTH : MAT_GLASS_ROUGH;
		if (!p.smooth) {
			r.alpha_x = p.alpha_x;
			r.alpha_y = p.alpha_y;
		}
		r.eta = p.ior;
		r.reflectance = p.reflectance;
		r.transmission = p.transmission;
		r.has_reflect = 1u;
		r.has_transmit = 1u;
		r.sss = 1u;
		r.sss_a = p.diffuse;
		vec3 t;
		t.x = fabs_ref(p.diffuse.x - 0.8f);
		t.y = fabs_ref(p.diffuse.y - 0.8f);
		t.z = fabs_ref(p.diffuse.z - 0.8f);
		const vec3 sd = (splat3(1.85f) - p.diffuse) + t * t * t * 7.f;
		r.sss_d = p.mfp / sd;
		return true;
	}
	default: return false;
	}
}

// image_texture_t<2, T>::sample(uv) (textures/detail/image_texture.hpp:44-75):
// uv wrapped to [0, 1) (glm::mod(x, 1) = x - floor(x)), scaled to texels and
// shifted by half a texel, the four neighbours clamped to the image, and two
// lerps s (1 - x) + t x along u then one along v.
RB_HD spectrum sample_image(const scene_view& s, const texture_rec& tr, vec2 uv) {
	const float* px = s.texels + tr.offset;
	const float fw = static_cast<float>(tr.width), fh = static_cast<float>(tr.height);
	const float x = (uv.x - floorf(uv.x)) * fw - 0.5f;
	const float y = (uv.y - floorf(uv.y)) * fh - 0.5f;
	const int32_t mx = static_cast<int32_t>(tr.width) - 1, my = static_cast<int32_t>(tr.height) - 1;
	const auto clampi = [](int32_t v, int32_t lo, int32_t hi) { return v < lo ? lo : (v > hi ? hi : v); };
	const int32_t x0 = clampi(static_cast<int32_t>(floorf(x)), 0, mx), y0 = clampi(static_cast<int32_t>(floorf(y)), 0, my);
	const int32_t x1 = clampi(x0 + 1, 0, mx), y1 = clampi(y0 + 1, 0, my);
	const float du = fclamp_ref(x - static_cast<float>(x0), 0.f, 1.f);
	const float dv = fclamp_ref(y - static_cast<float>(y0), 0.f, 1.f);
	const auto texel = [&](int32_t xi, int32_t yi) {
		const float* q = px + 3u * (static_cast<uint32_t>(yi) * tr.width + static_cast<uint32_t>(xi));
		return vec3{q[0], q[1], q[2]};
	};
	const vec3 v0 = texel(x0, y0) * (1.f - du) + texel(x1, y0) * du;
	const vec3 v1 = texel(x0, y1) * (1.f - du) + texel(x1, y1) * du;
	return v0 * (1.f - dv) + v1 * dv;
}

// Input i of a composite texture at coordinates c: its image, or its constant.
RB_HD spectrum texture_input(const scene_view& s, const texture_rec& tr, uint32_t i, vec2 c) {
	return tr.inputs[i] ? sample_image(s, s.textures[tr.inputs[i] - 1u], c) : tr.constants[i];
}

// Texture t at a hit with texture coordinates uv and world point p, as
// texture_t::sample(surface_interaction) does: an image samples uv; a scale
// texture samples its inputs at uv and gives base * scale
// (textures/detail/scale_texture.hpp:33-43); a mixture samples its inputs at
// (p.x, p.y), the interaction's point converted to a 2D coordinate
// (textures/detail/mixture_texture.hpp:36-48), and gives t0 a + t1 clamp(1 - a)
// with a = clamp(alpha, 0, 1).
RB_HD spectrum sample_texture(const scene_view& s, uint32_t t, vec2 uv, vec3 p) {
	const texture_rec& tr = s.textures[t];
	switch (tr.kind) {
	case TEXK_SCALE: return texture_input(s, tr, 1u, uv) * texture_input(s, tr, 0u, uv);
	case TEXK_MIXTURE: {
		const vec2 c{p.x, p.y};
		const float a0 = fclamp_ref(texture_input(s, tr, 2u, c).x, 0.f, 1.f);
		const float a1 = fclamp_ref(1.f - a0, 0.f, 1.f);
		return texture_input(s, tr, 0u, c) * a0 + texture_input(s, tr, 1u, c) * a1;
	}
	default: return sample_image(s, tr, uv);
	}
}

// The record of material `index` at a hit with texture coordinates uv and
// world point p: the uploaded record, or for MAT_TEXTURED one built into
// `scratch` from the material's parameters with its textured spectra sampled.
RB_HD const material_rec* hit_material(const scene_view& s, uint32_t index, vec2 uv, vec3 p, material_rec& scratch) {
	const material_rec* m = s.materials + index;
	if (m->kind != MAT_TEXTURED) return m;
	material_src q = s.material_srcs[m->src];
	if (q.tex[TEX_DIFFUSE]) q.diffuse = sample_texture(s, q.tex[TEX_DIFFUSE] - 1u, uv, p);
	if (q.tex[TEX_REFLECTANCE]) q.reflectance = sample_texture(s, q.tex[TEX_REFLECTANCE] - 1u, uv, p);
	if (q.tex[TEX_TRANSMISSION]) q.transmission = sample_texture(s, q.tex[TEX_TRANSMISSION] - 1u, uv, p);
	if (q.tex[TEX_SPECULAR]) q.specular = sample_texture(s, q.tex[TEX_SPECULAR] - 1u, uv, p);
	if (q.tex[TEX_OPACITY]) q.opacity = sample_texture(s, q.tex[TEX_OPACITY] - 1u, uv, p);
	// real parameters: channel 0 of their textures (texture2d<real>)
	const bool reals = q.tex[TEX_ROUGHNESS_U] | q.tex[TEX_ROUGHNESS_V] | q.tex[TEX_IOR] | q.tex[TEX_SIGMA];
	if (q.tex[TEX_ROUGHNESS_U]) q.roughness_u = sample_texture(s, q.tex[TEX_ROUGHNESS_U] - 1u, uv, p).x;
	if (q.tex[TEX_ROUGHNESS_V]) q.roughness_v = sample_texture(s, q.tex[TEX_ROUGHNESS_V] - 1u, uv, p).x;
	if (q.tex[TEX_IOR]) q.ior = sample_texture(s, q.tex[TEX_IOR] - 1u, uv, p).x;
	if (q.tex[TEX_SIGMA]) q.sigma = sample_texture(s, q.tex[TEX_SIGMA] - 1u, uv, p).x;
	if (reals) derive_src(q);
	if (q.tex[TEX_ETA]) q.cond_eta = sample_texture(s, q.tex[TEX_ETA] - 1u, uv, p);
	if (q.tex[TEX_K]) q.cond_k = sample_texture(s, q.tex[TEX_K] - 1u, uv, p);
	if (q.tex[TEX_MFP]) q.mfp = sample_texture(s, q.tex[TEX_MFP] - 1u, uv, p);
	build_record(q, nullptr, scratch);
	return &scratch;
}

// The record a shading stage uses at a hit: a shading class's material kind
// (MAT) is never textured (textured records are shaded as MAT_ANY).
template <int MAT>
RB_HD const material_rec* surface_material(const scene_view& s, uint32_t index, const surface_t& si,
	material_rec& scratch) {
	if constexpr (MAT != MAT_ANY) return s.materials + index;
	else return hit_material(s, index, si.uv, si.p, scratch);
}

} // namespace pt
} // namespace rb
