// Reference scene and camera -> rb_scene_desc / rb_camera_desc.
//
// The reference's classes keep every parameter private and offer no getters
// (e.g. matte_material::mDiffuse, materials/matte_material.hpp:26-28;
// surface_light::mRadiance, emitters/surface_light.hpp:24-25;
// projective_camera::mRasterToCamera, cameras/camera.hpp:73-80). This file reads
// them through member pointers formed in explicit template instantiations, where
// the language does not apply access checks, and carried out by a friend
// function of a tag type. A maintainer adding this adapter inside the
// reference would give those classes const accessors instead and drop the
// access_bind lines; nothing else here would change.
#include "scene_export.hpp"

#include "rainbow-cpu/cameras/perspective_camera.hpp"
#include "rainbow-cpu/emitters/environment_light.hpp"
#include "rainbow-cpu/emitters/surface_light.hpp"
#include "rainbow-cpu/materials/glass_material.hpp"
#include "rainbow-cpu/materials/matte_material.hpp"
#include "rainbow-cpu/materials/metal_material.hpp"
#include "rainbow-cpu/materials/mirror_material.hpp"
#include "rainbow-cpu/materials/mixture_material.hpp"
#include "rainbow-cpu/materials/plastic_material.hpp"
#include "rainbow-cpu/materials/substrate_material.hpp"
#include "rainbow-cpu/materials/subsurface_material.hpp"
#include "rainbow-cpu/materials/translucent_material.hpp"
#include "rainbow-cpu/materials/uber_material.hpp"
#include "rainbow-cpu/media/homogeneous_medium.hpp"
#include "rainbow-cpu/shapes/mesh.hpp"
#include "rainbow-cpu/textures/constant_texture.hpp"
#include "rainbow-cpu/textures/texture.hpp"

// image_texture_t<2, T>::sample (textures/detail/image_texture.hpp:65-66) calls
// clamp(float, real, real) unqualified; under standard two-phase lookup (g++)
// the spectrum clamp made visible by a using-directive hides the scalar one of
// rainbow-core, so the reference's header only compiles with the scalar clamp
// declared in the textures namespace first. It changes nothing the header computes.
namespace rainbow::cpus::textures {
using rainbow::core::math::clamp;
}
#include "rainbow-cpu/textures/image_texture.hpp"
#include "rainbow-cpu/textures/mixture_texture.hpp"
#include "rainbow-cpu/textures/scale_texture.hpp"

#include <functional>
#include <unordered_map>

using namespace rainbow::cpus;

namespace rb {
namespace adapter {
namespace {

template <auto Member, typename Tag>
struct access_bind {
	friend constexpr auto member_of(Tag) { return Member; }
};
#define COMMA ,
#define RB_PRIVATE_MEMBER(tag, member)                              \
	struct tag { friend constexpr auto member_of(tag); };          \
	template struct access_bind<&member, tag>

RB_PRIVATE_MEMBER(mesh_positions, shapes::mesh::mPositions);
RB_PRIVATE_MEMBER(mesh_normals, shapes::mesh::mNormals);
RB_PRIVATE_MEMBER(mesh_tangents, shapes::mesh::mTangents);
RB_PRIVATE_MEMBER(mesh_uvs, shapes::mesh::mUVs);
RB_PRIVATE_MEMBER(mesh_indices, shapes::mesh::mIndices);
RB_PRIVATE_MEMBER(mesh_mask, shapes::mesh::mMask);
RB_PRIVATE_MEMBER(matte_diffuse, materials::matte_material::mDiffuse);
RB_PRIVATE_MEMBER(matte_sigma, materials::matte_material::mSigma);
RB_PRIVATE_MEMBER(metal_eta, materials::metal_material::mEta);
RB_PRIVATE_MEMBER(metal_k, materials::metal_material::mK);
RB_PRIVATE_MEMBER(metal_ru, materials::metal_material::mRoughnessU);
RB_PRIVATE_MEMBER(metal_rv, materials::metal_material::mRoughnessV);
RB_PRIVATE_MEMBER(metal_remap, materials::metal_material::mMapRoughnessToAlpha);
RB_PRIVATE_MEMBER(glass_reflectance, materials::glass_material::mReflectance);
RB_PRIVATE_MEMBER(glass_transmission, materials::glass_material::mTransmission);
RB_PRIVATE_MEMBER(glass_ru, materials::glass_material::mRoughnessU);
RB_PRIVATE_MEMBER(glass_rv, materials::glass_material::mRoughnessV);
RB_PRIVATE_MEMBER(glass_eta, materials::glass_material::mEta);
RB_PRIVATE_MEMBER(glass_remap, materials::glass_material::mMapRoughnessToAlpha);
RB_PRIVATE_MEMBER(plastic_specular, materials::plastic_material::mSpecular);
RB_PRIVATE_MEMBER(plastic_diffuse, materials::plastic_material::mDiffuse);
RB_PRIVATE_MEMBER(plastic_roughness, materials::plastic_material::mRoughness);
RB_PRIVATE_MEMBER(plastic_eta, materials::plastic_material::mEta);
RB_PRIVATE_MEMBER(plastic_remap, materials::plastic_material::mMapRoughnessToAlpha);
RB_PRIVATE_MEMBER(mirror_reflectance, materials::mirror_material::mReflectance);
RB_PRIVATE_MEMBER(substrate_specular, materials::substrate_material::mSpecular);
RB_PRIVATE_MEMBER(substrate_diffuse, materials::substrate_material::mDiffuse);
RB_PRIVATE_MEMBER(substrate_ru, materials::substrate_material::mRoughnessU);
RB_PRIVATE_MEMBER(substrate_rv, materials::substrate_material::mRoughnessV);
RB_PRIVATE_MEMBER(substrate_remap, materials::substrate_material::mMapRoughnessToAlpha);
RB_PRIVATE_MEMBER(uber_transmission, materials::uber_material::mTransmission);
RB_PRIVATE_MEMBER(uber_reflectance, materials::uber_material::mReflectance);
RB_PRIVATE_MEMBER(uber_specular, materials::uber_material::mSpecular);
RB_PRIVATE_MEMBER(uber_diffuse, materials::uber_material::mDiffuse);
RB_PRIVATE_MEMBER(uber_opacity, materials::uber_material::mOpacity);
RB_PRIVATE_MEMBER(uber_ru, materials::uber_material::mRoughnessU);
RB_PRIVATE_MEMBER(uber_rv, materials::uber_material::mRoughnessV);
RB_PRIVATE_MEMBER(uber_eta, materials::uber_material::mEta);
RB_PRIVATE_MEMBER(uber_remap, materials::uber_material::mMapRoughnessToAlpha);
RB_PRIVATE_MEMBER(translucent_transmission, materials::translucent_material::mTransmission);
RB_PRIVATE_MEMBER(translucent_reflectance, materials::translucent_material::mReflectance);
RB_PRIVATE_MEMBER(translucent_specular, materials::translucent_material::mSpecular);
RB_PRIVATE_MEMBER(translucent_diffuse, materials::translucent_material::mDiffuse);
RB_PRIVATE_MEMBER(translucent_roughness, materials::translucent_material::mRoughness);
RB_PRIVATE_MEMBER(translucent_remap, materials::translucent_material::mMapRoughnessToAlpha);
RB_PRIVATE_MEMBER(subsurface_transmission, materials::subsurface_material::mTransmission);
RB_PRIVATE_MEMBER(subsurface_reflectance, materials::subsurface_material::mReflectance);
RB_PRIVATE_MEMBER(subsurface_diffuse, materials::subsurface_material::mDiffuse);
RB_PRIVATE_MEMBER(subsurface_mfp, materials::subsurface_material::mMFP);
RB_PRIVATE_MEMBER(subsurface_ru, materials::subsurface_material::mRoughnessU);
RB_PRIVATE_MEMBER(subsurface_rv, materials::subsurface_material::mRoughnessV);
RB_PRIVATE_MEMBER(subsurface_eta, materials::subsurface_material::mEta);
RB_PRIVATE_MEMBER(subsurface_remap, materials::subsurface_material::mMapRoughnessToAlpha);
RB_PRIVATE_MEMBER(mixture_alpha, materials::mixture_material::mAlpha);
RB_PRIVATE_MEMBER(mixture_materials, materials::mixture_material::mMaterials);
RB_PRIVATE_MEMBER(scale_scale, textures::scale_texture_t<2 COMMA shared::spectrums::spectrum>::mScale);
RB_PRIVATE_MEMBER(scale_base, textures::scale_texture_t<2 COMMA shared::spectrums::spectrum>::mBase);
RB_PRIVATE_MEMBER(mixture_t0, textures::mixture_texture_t<2 COMMA shared::spectrums::spectrum>::mTexture0);
RB_PRIVATE_MEMBER(mixture_t1, textures::mixture_texture_t<2 COMMA shared::spectrums::spectrum>::mTexture1);
RB_PRIVATE_MEMBER(mixture_alpha_texture, textures::mixture_texture_t<2 COMMA shared::spectrums::spectrum>::mAlpha);
RB_PRIVATE_MEMBER(real_scale_scale, textures::scale_texture_t<2 COMMA rainbow::core::real>::mScale);
RB_PRIVATE_MEMBER(real_scale_base, textures::scale_texture_t<2 COMMA rainbow::core::real>::mBase);
RB_PRIVATE_MEMBER(real_mixture_t0, textures::mixture_texture_t<2 COMMA rainbow::core::real>::mTexture0);
RB_PRIVATE_MEMBER(real_mixture_t1, textures::mixture_texture_t<2 COMMA rainbow::core::real>::mTexture1);
RB_PRIVATE_MEMBER(real_mixture_alpha, textures::mixture_texture_t<2 COMMA rainbow::core::real>::mAlpha);
RB_PRIVATE_MEMBER(surface_radiance, emitters::surface_light::mRadiance);
RB_PRIVATE_MEMBER(environment_map, emitters::environment_light::mEnvironmentMap);
RB_PRIVATE_MEMBER(environment_intensity, emitters::environment_light::mIntensity);
RB_PRIVATE_MEMBER(environment_radius, emitters::environment_light::mRadius);
RB_PRIVATE_MEMBER(medium_sigma_a, media::homogeneous_medium::mSigmaA);
RB_PRIVATE_MEMBER(medium_sigma_s, media::homogeneous_medium::mSigmaS);
RB_PRIVATE_MEMBER(medium_g, media::homogeneous_medium::mG);
RB_PRIVATE_MEMBER(camera_raster_to_camera, cameras::projective_camera::mRasterToCamera);
RB_PRIVATE_MEMBER(camera_focus, cameras::projective_camera::mFocus);
RB_PRIVATE_MEMBER(camera_lens, cameras::projective_camera::mLens);
RB_PRIVATE_MEMBER(camera_to_world, cameras::camera::mCameraToWorld);
#undef RB_PRIVATE_MEMBER
#undef COMMA

template <typename Tag, typename Object>
const auto& read(const Object& o, Tag tag) { return o.*member_of(tag); }

// The value of a constant texture (constant_texture_t::sample returns it
// anywhere); false for any other texture.
template <typename T>
bool constant_value(const std::shared_ptr<textures::texture2d<T>>& t, T& out) {
	const auto c = std::dynamic_pointer_cast<textures::constant_texture2d<T>>(t);
	if (c == nullptr) return false;
	out = c->sample(rainbow::core::math::vector2(0));
	return true;
}
bool constant_rgb(const std::shared_ptr<textures::texture2d<shared::spectrums::spectrum>>& t, float* rgb) {
	shared::spectrums::spectrum v;
	if (!constant_value(t, v)) return false;
	rgb[0] = v[0]; rgb[1] = v[1]; rgb[2] = v[2];
	return true;
}
bool constant_real(const std::shared_ptr<textures::texture2d<rainbow::core::real>>& t, float& v) { return constant_value(t, v); }

void put_rgb(const shared::spectrums::spectrum& s, float* rgb) { rgb[0] = s[0]; rgb[1] = s[1]; rgb[2] = s[2]; }

// glm's column-major storage, element (row r, column c) at [c * 4 + r].
void put_matrix(const rainbow::core::math::matrix4x4& m, float* out) {
	for (int c = 0; c < 4; c++)
		for (int r = 0; r < 4; r++) out[c * 4 + r] = m[c][r];
}

// The scene's image textures (image_texture2d<spectrum>), each exported once.
struct texture_registry {
	exported_scene& out;
	std::unordered_map<const void*, uint32_t> ref_of;
	// A spectrum parameter: a constant texture's value in rgb (ref 0), or an
	// image texture's reference (index + 1 into out.textures); false for
	// other textures.
	bool spectrum(const std::shared_ptr<textures::texture2d<shared::spectrums::spectrum>>& t, float* rgb, uint32_t& ref) {
		ref = 0;
		if (constant_rgb(t, rgb)) return true;
		if (image(t, ref)) return true;
		return composite(t, ref);
	}
	// A scale or mixture texture whose inputs are images or constants.
	bool composite(const std::shared_ptr<textures::texture2d<shared::spectrums::spectrum>>& t, uint32_t& ref) {
		using S = shared::spectrums::spectrum;
		const auto it = ref_of.find(t.get());
		if (it != ref_of.end()) {
			ref = it->second;
			return true;
		}
		rb_texture_desc td{};
		const auto input = [&](const std::shared_ptr<textures::texture2d<S>>& in, uint32_t i) {
			return constant_rgb(in, td.constants[i]) || image(in, td.inputs[i]);
		};
		if (const auto x = std::dynamic_pointer_cast<textures::scale_texture_t<2, S>>(t)) {
			td.kind = RB_TEXTURE_SCALE;
			if (!input(read(*x, scale_scale{}), 0) || !input(read(*x, scale_base{}), 1)) return false;
		} else if (const auto x = std::dynamic_pointer_cast<textures::mixture_texture_t<2, S>>(t)) {
			td.kind = RB_TEXTURE_MIXTURE;
			if (!input(read(*x, mixture_t0{}), 0) || !input(read(*x, mixture_t1{}), 1)) return false;
			// the real-valued alpha: a constant, or a real image exported as an RGB image (channel 0)
			const auto& alpha = read(*x, mixture_alpha_texture{});
			if (!constant_real(alpha, td.constants[2][0])) {
				const auto img = std::dynamic_pointer_cast<textures::image_texture2d<rainbow::core::real>>(alpha);
				if (img == nullptr || !add_image(img.get(), img->size().x, img->size().y,
						[&](size_t i, float* c) { c[0] = c[1] = c[2] = img->value(i); }, td.inputs[2]))
					return false;
			}
		} else {
			return false;
		}
		out.texels.emplace_back();
		out.textures.push_back(td);
		ref = static_cast<uint32_t>(out.textures.size());
		ref_of.emplace(t.get(), ref);
		return true;
	}
	// A real parameter: a constant texture's value in v (ref 0), or a real image
	// texture exported as an RGB image whose channels all hold its values (the
	// core reads channel 0); false for other textures.
	bool real(const std::shared_ptr<textures::texture2d<rainbow::core::real>>& t, float& v, uint32_t& ref) {
		ref = 0;
		if (constant_real(t, v)) return true;
		if (real_image(t, ref)) return true;
		return real_composite(t, ref);
	}
	bool real_image(const std::shared_ptr<textures::texture2d<rainbow::core::real>>& t, uint32_t& ref) {
		const auto img = std::dynamic_pointer_cast<textures::image_texture2d<rainbow::core::real>>(t);
		return img != nullptr && add_image(img.get(), img->size().x, img->size().y,
			[&](size_t i, float* c) { c[0] = c[1] = c[2] = img->value(i); }, ref);
	}
	// A scale or mixture texture of reals whose inputs are real images or
	// constants (constants in every channel; the core reads channel 0).
	bool real_composite(const std::shared_ptr<textures::texture2d<rainbow::core::real>>& t, uint32_t& ref) {
		using R = rainbow::core::real;
		const auto it = ref_of.find(t.get());
		if (it != ref_of.end()) {
			ref = it->second;
			return true;
		}
		rb_texture_desc td{};
		const auto input = [&](const std::shared_ptr<textures::texture2d<R>>& in, uint32_t i) {
			float v = 0.f;
			if (constant_real(in, v)) {
				td.constants[i][0] = td.constants[i][1] = td.constants[i][2] = v;
				return true;
			}
			return real_image(in, td.inputs[i]);
		};
		if (const auto x = std::dynamic_pointer_cast<textures::scale_texture_t<2, R>>(t)) {
			td.kind = RB_TEXTURE_SCALE;
			if (!input(read(*x, real_scale_scale{}), 0) || !input(read(*x, real_scale_base{}), 1)) return false;
		} else if (const auto x = std::dynamic_pointer_cast<textures::mixture_texture_t<2, R>>(t)) {
			td.kind = RB_TEXTURE_MIXTURE;
			if (!input(read(*x, real_mixture_t0{}), 0) || !input(read(*x, real_mixture_t1{}), 1) ||
				!input(read(*x, real_mixture_alpha{}), 2))
				return false;
		} else {
			return false;
		}
		out.texels.emplace_back();
		out.textures.push_back(td);
		ref = static_cast<uint32_t>(out.textures.size());
		ref_of.emplace(t.get(), ref);
		return true;
	}
	// An RGB image texture, exported once.
	bool image(const std::shared_ptr<textures::texture2d<shared::spectrums::spectrum>>& t, uint32_t& ref) {
		const auto img = std::dynamic_pointer_cast<textures::image_texture2d<shared::spectrums::spectrum>>(t);
		if (img == nullptr) return false;
		return add_image(img.get(), img->size().x, img->size().y, [&](size_t i, float* c) {
			const auto v = img->value(i);
			c[0] = v[0]; c[1] = v[1]; c[2] = v[2];
		}, ref);
	}
	template <typename Texel>
	bool add_image(const void* key, size_t w, size_t h, Texel texel, uint32_t& ref) {
		const auto it = ref_of.find(key);
		if (it != ref_of.end()) {
			ref = it->second;
			return true;
		}
		if (w == 0 || h == 0 || w > (1u << 15) || h > (1u << 15)) return false;
		std::vector<float> texels(3 * w * h);
		for (size_t i = 0; i < w * h; i++) texel(i, texels.data() + 3 * i);
		out.texels.push_back(std::move(texels));
		rb_texture_desc td{};
		td.kind = RB_TEXTURE_IMAGE;
		td.width = static_cast<uint32_t>(w);
		td.height = static_cast<uint32_t>(h);
		out.textures.push_back(td);
		ref = static_cast<uint32_t>(out.textures.size());
		ref_of.emplace(key, ref);
		return true;
	}
};

rb_status export_material(const std::shared_ptr<materials::material>& m, rb_material_desc& d, texture_registry& tex) {
	d = rb_material_desc{};
	bool ok = true;
	// a spectrum parameter that may be an image texture
	const auto spec = [&](const std::shared_ptr<textures::texture2d<shared::spectrums::spectrum>>& t, float* rgb,
		uint32_t& ref) { return tex.spectrum(t, rgb, ref); };
	if (const auto x = std::dynamic_pointer_cast<materials::matte_material>(m)) {
		d.kind = RB_MATERIAL_MATTE;
		ok = spec(read(*x, matte_diffuse{}), d.diffuse, d.diffuse_texture) && tex.real(read(*x, matte_sigma{}), d.sigma, d.sigma_texture);
	} else if (const auto x = std::dynamic_pointer_cast<materials::metal_material>(m)) {
		d.kind = RB_MATERIAL_METAL;
		d.remap_roughness = read(*x, metal_remap{}) ? 1 : 0;
		ok = spec(read(*x, metal_eta{}), d.eta, d.eta_texture) && spec(read(*x, metal_k{}), d.k, d.k_texture) &&
			tex.real(read(*x, metal_ru{}), d.roughness_u, d.roughness_u_texture) && tex.real(read(*x, metal_rv{}), d.roughness_v, d.roughness_v_texture);
	} else if (const auto x = std::dynamic_pointer_cast<materials::glass_material>(m)) {
		d.kind = RB_MATERIAL_GLASS;
		d.remap_roughness = read(*x, glass_remap{}) ? 1 : 0;
		ok = spec(read(*x, glass_reflectance{}), d.reflectance, d.reflectance_texture) &&
			spec(read(*x, glass_transmission{}), d.transmission, d.transmission_texture) &&
			tex.real(read(*x, glass_ru{}), d.roughness_u, d.roughness_u_texture) && tex.real(read(*x, glass_rv{}), d.roughness_v, d.roughness_v_texture) &&
			tex.real(read(*x, glass_eta{}), d.ior, d.ior_texture);
	} else if (const auto x = std::dynamic_pointer_cast<materials::plastic_material>(m)) {
		d.kind = RB_MATERIAL_PLASTIC;
		d.remap_roughness = read(*x, plastic_remap{}) ? 1 : 0;
		ok = spec(read(*x, plastic_specular{}), d.reflectance, d.reflectance_texture) &&
			spec(read(*x, plastic_diffuse{}), d.diffuse, d.diffuse_texture) &&
			tex.real(read(*x, plastic_roughness{}), d.roughness_u, d.roughness_u_texture) && tex.real(read(*x, plastic_eta{}), d.ior, d.ior_texture);
	} else if (const auto x = std::dynamic_pointer_cast<materials::mirror_material>(m)) {
		d.kind = RB_MATERIAL_MIRROR;
		ok = spec(read(*x, mirror_reflectance{}), d.reflectance, d.reflectance_texture);
	} else if (const auto x = std::dynamic_pointer_cast<materials::substrate_material>(m)) {
		d.kind = RB_MATERIAL_SUBSTRATE;
		d.remap_roughness = read(*x, substrate_remap{}) ? 1 : 0;
		ok = spec(read(*x, substrate_specular{}), d.reflectance, d.reflectance_texture) &&
			spec(read(*x, substrate_diffuse{}), d.diffuse, d.diffuse_texture) && tex.real(read(*x, substrate_ru{}), d.roughness_u, d.roughness_u_texture) &&
			tex.real(read(*x, substrate_rv{}), d.roughness_v, d.roughness_v_texture);
	} else if (const auto x = std::dynamic_pointer_cast<materials::uber_material>(m)) {
		d.kind = RB_MATERIAL_UBER;
		d.remap_roughness = read(*x, uber_remap{}) ? 1 : 0;
		ok = spec(read(*x, uber_transmission{}), d.transmission, d.transmission_texture) &&
			spec(read(*x, uber_reflectance{}), d.reflectance, d.reflectance_texture) &&
			spec(read(*x, uber_specular{}), d.specular, d.specular_texture) &&
			spec(read(*x, uber_diffuse{}), d.diffuse, d.diffuse_texture) && spec(read(*x, uber_opacity{}), d.opacity, d.opacity_texture) &&
			tex.real(read(*x, uber_ru{}), d.roughness_u, d.roughness_u_texture) && tex.real(read(*x, uber_rv{}), d.roughness_v, d.roughness_v_texture) &&
			tex.real(read(*x, uber_eta{}), d.ior, d.ior_texture);
	} else if (const auto x = std::dynamic_pointer_cast<materials::translucent_material>(m)) {
		d.kind = RB_MATERIAL_TRANSLUCENT;
		d.remap_roughness = read(*x, translucent_remap{}) ? 1 : 0;
		ok = spec(read(*x, translucent_transmission{}), d.transmission, d.transmission_texture) &&
			spec(read(*x, translucent_reflectance{}), d.reflectance, d.reflectance_texture) &&
			spec(read(*x, translucent_specular{}), d.specular, d.specular_texture) &&
			spec(read(*x, translucent_diffuse{}), d.diffuse, d.diffuse_texture) &&
			tex.real(read(*x, translucent_roughness{}), d.roughness_u, d.roughness_u_texture);
		d.roughness_v = d.roughness_u;
	} else if (const auto x = std::dynamic_pointer_cast<materials::subsurface_material>(m)) {
		d.kind = RB_MATERIAL_SUBSURFACE;
		d.remap_roughness = read(*x, subsurface_remap{}) ? 1 : 0;
		ok = spec(read(*x, subsurface_transmission{}), d.transmission, d.transmission_texture) &&
			spec(read(*x, subsurface_reflectance{}), d.reflectance, d.reflectance_texture) &&
			spec(read(*x, subsurface_diffuse{}), d.diffuse, d.diffuse_texture) &&
			spec(read(*x, subsurface_mfp{}), d.mfp, d.mfp_texture) && tex.real(read(*x, subsurface_ru{}), d.roughness_u, d.roughness_u_texture) &&
			tex.real(read(*x, subsurface_rv{}), d.roughness_v, d.roughness_v_texture) && tex.real(read(*x, subsurface_eta{}), d.ior, d.ior_texture);
	} else {
		return RB_ERR_UNSUPPORTED;  // a material kind outside these (a mixture is exported by export_scene)
	}
	return ok ? RB_OK : RB_ERR_UNSUPPORTED;  // a texture that is neither constant nor an RGB image
}

rb_status export_emitter(const std::shared_ptr<emitters::emitter>& e, rb_emitter_desc& d) {
	d = rb_emitter_desc{};
	if (const auto x = std::dynamic_pointer_cast<emitters::surface_light>(e)) {
		d.kind = RB_EMITTER_SURFACE;
		put_rgb(read(*x, surface_radiance{}), d.radiance);
		return RB_OK;
	}
	if (const auto x = std::dynamic_pointer_cast<emitters::environment_light>(e)) {
		// the core renders the constant map of 1 that environment_light(intensity, radius) makes
		shared::spectrums::spectrum map;
		if (!constant_value(read(*x, environment_map{}), map) || map[0] != 1.f || map[1] != 1.f || map[2] != 1.f)
			return RB_ERR_UNSUPPORTED;
		d.kind = RB_EMITTER_ENVIRONMENT;
		put_rgb(read(*x, environment_intensity{}), d.radiance);
		d.radius = read(*x, environment_radius{});
		return RB_OK;
	}
	return RB_ERR_UNSUPPORTED;  // point and directional lights
}

template <typename T>
std::vector<float> flat(const std::vector<T>& v) {
	std::vector<float> out;
	out.reserve(3 * v.size());
	for (const auto& p : v) { out.push_back(p.x); out.push_back(p.y); out.push_back(p.z); }
	return out;
}

} // namespace

rb_status export_scene(const scenes::scene& s, exported_scene& out) {
	out = exported_scene();
	std::unordered_map<const void*, int32_t> mesh_of, material_of, medium_of;
	texture_registry tex{out, {}};
	// a material's index in out.materials, exported on first use; a mixture's
	// two materials are exported before it (mixture_material.hpp: mAlpha, mMaterials)
	std::function<rb_status(const std::shared_ptr<materials::material>&, int, int32_t&)> material_index =
		[&](const std::shared_ptr<materials::material>& mat, int depth, int32_t& index) -> rb_status {
		if (mat == nullptr || depth > 8) return RB_ERR_UNSUPPORTED;
		const auto it = material_of.find(mat.get());
		if (it != material_of.end()) {
			index = it->second;
			return RB_OK;
		}
		rb_material_desc md{};
		if (const auto x = std::dynamic_pointer_cast<materials::mixture_material>(mat)) {
			md.kind = RB_MATERIAL_MIXTURE;
			if (!constant_rgb(read(*x, mixture_alpha{}), md.amount)) return RB_ERR_UNSUPPORTED;
			const auto& parts = read(*x, mixture_materials{});
			for (int c = 0; c < 2; c++) {
				const rb_status st = material_index(parts[c], depth + 1, md.components[c]);
				if (st != RB_OK) return st;
			}
		} else {
			const rb_status st = export_material(mat, md, tex);
			if (st != RB_OK) return st;
		}
		out.materials.push_back(md);
		index = static_cast<int32_t>(out.materials.size() - 1);
		material_of.emplace(mat.get(), index);
		return RB_OK;
	};
	try {
		for (const auto& ent : s.entities()) {
			rb_entity_desc ed{};
			ed.mesh = ed.material = ed.emitter = ed.medium = -1;
			put_matrix(ent->transform().matrix(), ed.local_to_world);
			put_matrix(ent->transform().inverse_matrix(), ed.world_to_local);
			if (ent->has_component<shapes::shape>()) {
				const auto shape = ent->component<shapes::shape>();
				const auto m = std::dynamic_pointer_cast<shapes::mesh>(shape);
				if (m == nullptr || read(*m, mesh_mask{}) != nullptr) return RB_ERR_UNSUPPORTED;  // sphere, disk, curve; alpha masks
				auto it = mesh_of.find(shape.get());
				if (it == mesh_of.end()) {
					const auto& idx = read(*m, mesh_indices{});
					out.positions.push_back(flat(read(*m, mesh_positions{})));
					out.normals.push_back(flat(read(*m, mesh_normals{})));
					out.tangents.push_back(flat(read(*m, mesh_tangents{})));
					out.uvs.push_back(flat(read(*m, mesh_uvs{})));
					out.indices.emplace_back(idx.begin(), idx.end());
					rb_mesh_desc md{};
					md.num_vertices = static_cast<uint32_t>(read(*m, mesh_positions{}).size());
					md.num_triangles = static_cast<uint32_t>(idx.size() / 3);
					md.reverse_orientation = m->reverse_orientation() ? 1 : 0;
					out.meshes.push_back(md);
					it = mesh_of.emplace(shape.get(), static_cast<int32_t>(out.meshes.size() - 1)).first;
				}
				ed.mesh = it->second;
			}
			if (ent->has_component<materials::material>()) {
				const rb_status st = material_index(ent->component<materials::material>(), 0, ed.material);
				if (st != RB_OK) return st;
			}
			if (ent->has_component<emitters::emitter>()) {
				rb_emitter_desc em;
				const rb_status st = export_emitter(ent->component<emitters::emitter>(), em);
				if (st != RB_OK) return st;
				out.emitters.push_back(em);
				ed.emitter = static_cast<int32_t>(out.emitters.size() - 1);
			}
			if (ent->has_component<media::media>()) {
				const auto md = ent->component<media::media>();
				auto medium_index = [&](const std::shared_ptr<media::medium>& m, int32_t& index) -> rb_status {
					index = -1;
					if (m == nullptr) return RB_OK;
					auto it = medium_of.find(m.get());
					if (it == medium_of.end()) {
						const auto h = std::dynamic_pointer_cast<media::homogeneous_medium>(m);
						if (h == nullptr) return RB_ERR_UNSUPPORTED;  // heterogeneous media
						rb_medium_desc r{};
						put_rgb(read(*h, medium_sigma_a{}), r.sigma_a);
						put_rgb(read(*h, medium_sigma_s{}), r.sigma_s);
						r.g = read(*h, medium_g{});
						out.mediums.push_back(r);
						it = medium_of.emplace(m.get(), static_cast<int32_t>(out.mediums.size() - 1)).first;
					}
					index = it->second;
					return RB_OK;
				};
				rb_media_desc r{};
				rb_status st = medium_index(md->inside(), r.inside);
				if (st == RB_OK) st = medium_index(md->outside(), r.outside);
				if (st != RB_OK) return st;
				out.media.push_back(r);
				ed.medium = static_cast<int32_t>(out.media.size() - 1);
			}
			out.entities.push_back(ed);
		}
	} catch (const std::bad_alloc&) {
		return RB_ERR_OUT_OF_MEMORY;
	}
	for (size_t i = 0; i < out.meshes.size(); i++) {
		rb_mesh_desc& md = out.meshes[i];
		md.positions = out.positions[i].data();
		md.normals = out.normals[i].empty() ? nullptr : out.normals[i].data();
		md.tangents = out.tangents[i].empty() ? nullptr : out.tangents[i].data();
		md.uvs = out.uvs[i].empty() ? nullptr : out.uvs[i].data();
		md.indices = out.indices[i].data();
	}
	rb_scene_desc& d = out.desc;
	d = rb_scene_desc{};
	d.meshes = out.meshes.data();
	d.num_meshes = static_cast<uint32_t>(out.meshes.size());
	d.entities = out.entities.data();
	d.num_entities = static_cast<uint32_t>(out.entities.size());
	d.materials = out.materials.data();
	d.num_materials = static_cast<uint32_t>(out.materials.size());
	d.emitters = out.emitters.data();
	d.num_emitters = static_cast<uint32_t>(out.emitters.size());
	d.mediums = out.mediums.data();
	d.num_mediums = static_cast<uint32_t>(out.mediums.size());
	d.media = out.media.data();
	d.num_media = static_cast<uint32_t>(out.media.size());
	for (size_t t = 0; t < out.textures.size(); t++)
		out.textures[t].rgb = out.texels[t].empty() ? nullptr : out.texels[t].data();
	d.textures = out.textures.data();
	d.num_textures = static_cast<uint32_t>(out.textures.size());
	return RB_OK;
}

rb_status export_camera(const cameras::camera& c, rb_camera_desc& out) {
	const auto* p = dynamic_cast<const cameras::perspective_camera*>(&c);
	if (p == nullptr) return RB_ERR_UNSUPPORTED;  // other camera models
	out = rb_camera_desc{};
	const auto& c2w = read(*p, camera_to_world{});
	put_matrix(read(*p, camera_raster_to_camera{}).matrix(), out.raster_to_camera);
	put_matrix(c2w.matrix(), out.camera_to_world);
	out.eye[0] = out.camera_to_world[12];
	out.eye[1] = out.camera_to_world[13];
	out.eye[2] = out.camera_to_world[14];
	out.lens_radius = read(*p, camera_lens{});
	out.focus_distance = read(*p, camera_focus{});
	const auto res = c.film()->resolution();
	out.width = res.x;
	out.height = res.y;
	return RB_OK;
}

} // namespace adapter
} // namespace rb
