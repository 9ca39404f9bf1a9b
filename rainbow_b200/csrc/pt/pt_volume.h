// Participating media of the volume path integrator: homogeneous medium
// sampling and transmittance, the Henyey-Greenstein phase function, and the
// medium switch at a surface. Rounding order follows the reference.
#pragma once

#include "pt_bsdf.h"
#include "pt_geom.h"

namespace rb {
namespace pt {

constexpr float kOneOverFourPi = 0.0795774715459476678f;  // math::one_over_four_pi<float>
constexpr float kFloatMax = 3.402823466e+38f;             // std::numeric_limits<float>::max()

// e^(-sigma_t * min(len, FLT_MAX)) per channel (homogeneous_medium::evaluate,
// media/homogeneous_medium.cpp:13-17); vacuum (medium < 0) gives 1.
RB_HD spectrum transmittance(const scene_view& s, int32_t medium, float len) {
	if (medium < 0) return splat3(1.f);
	const vec3 st = s.mediums[medium].sigma_t;
	const float l = len < kFloatMax ? len : kFloatMax;
	return vec3{expf(-st.x * l), expf(-st.y * l), expf(-st.z * l)};
}

// homogeneous_medium::sample (homogeneous_medium.cpp:19-58): one channel picked
// uniformly (uniform_sample_one_from_range, sample_function.cpp:97-102), a free
// flight t = -ln(1 - u) / sigma_t[channel] clamped to the ray length, and the
// spectral-MIS pdf averaged over the channels.
struct medium_event {
	bool scattered;     // a medium interaction at distance t (otherwise the surface at len)
	float t;
	spectrum weight;    // value / pdf (surface) or value * sigma_s / pdf (medium)
};

RB_HD medium_event sample_medium(const medium_rec& m, float len, float u_channel, float u_distance) {
	size_t channel = static_cast<size_t>(u_channel * 3.f);
	if (channel > 2) channel = 2;
	const float st[3] = {m.sigma_t.x, m.sigma_t.y, m.sigma_t.z};
	const float tf = -logf(1.f - u_distance) / st[channel];
	const float t = (len < tf) ? len : tf;  // min(a, b) = (b < a) ? b : a
	medium_event e;
	e.scattered = t < len;
	e.t = t;
	const float tc = t < kFloatMax ? t : kFloatMax;
	const vec3 value{expf(-m.sigma_t.x * tc), expf(-m.sigma_t.y * tc), expf(-m.sigma_t.z * tc)};
	const vec3 density = e.scattered ? (m.sigma_t * value) : value;
	float pdf = 0.f;
	pdf = pdf + density.x;
	pdf = pdf + density.y;
	pdf = pdf + density.z;
	pdf = pdf / 3.f;
	if (pdf == 0.f) pdf = 1.f;
	e.weight = e.scattered ? (value * m.sigma_s / pdf) : (value / pdf);
	return e;
}

// henyey_greenstein_phase_function (rainbow-core/utilities.cpp:46-51).
RB_HD float hg_phase(float cos_theta, float g) {
	const float denominator = 1.f + g * g + 2.f * g * cos_theta;
	return kOneOverFourPi * (1.f - g * g) / (denominator * sqrtf(denominator));
}

// henyey_greenstein::sample (shared/phases/henyey_greenstein.cpp:17-50): the
// direction in the frame coordinate_system(wo) with its z axis replaced by -wo,
// and its phase value (which is also its pdf).
RB_HD float hg_sample(vec3 wo, float g, vec2 u, vec3& wi) {
	float cos_theta;
	if (fabs_ref(g) >= 1e-3f) {
		const float sqr_term = (1.f - g * g) / (1.f - g + 2.f * g * u.x);
		cos_theta = (1.f + g * g - sqr_term * sqr_term) / (2.f * g);
	} else {
		cos_theta = 1.f - 2.f * u.x;
	}
	const float sin_theta = sqrtf(fmax_ref(0.f, 1.f - cos_theta * cos_theta));
	const float phi = kTwoPi * u.y;
	const vec3 l{sin_theta * cosf(phi), sin_theta * sinf(phi), cos_theta};  // spherical_direction
	vec3 x, y, z;
	frame_from_normal(wo, x, y, z);
	z = -wo;
	// local_to_world (shared/coordinate_system.cpp:71-78)
	wi = vec3{x.x * l.x + y.x * l.y + z.x * l.z, x.y * l.x + y.y * l.y + z.y * l.z, x.z * l.x + y.z * l.y + z.z * l.z};
	return hg_phase(-cos_theta, g);
}

// medium_info(entity, normal, wi) (media/medium.cpp:27-35): the medium on the
// side of the entity's surface that a ray in direction wi enters.
RB_HD int32_t medium_after(const scene_view& s, const entity_rec& e, vec3 normal, vec3 wi) {
	const media_rec& m = s.media[e.media];
	return dot(normal, wi) > 0.f ? m.outside : m.inside;
}

} // namespace pt
} // namespace rb
