// Oracle harness over the reference renderer itself (TEST INFRASTRUCTURE).
//
// Compiled together with the unmodified reference sources (rainbow-core,
// rainbow-cpu) into oracle/_ref/liboracle_ref.so by oracle/Makefile. Only the
// tests, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it, as the
// checker. It exposes C entry points that:
//  - build a reference `scene` (entity / mesh / material / emitter objects, then
//    scene::build_accelerator) and a `perspective_camera` from an rb_scene_desc,
//    or from the seeded scene generator of the benchmark configurations;
//  - export the reference's own BVH, camera matrices and emitter areas;
//  - trace rays through scene::intersect / intersect_with_shadow_ray;
//  - render through path_integrator::trace with one PCG32 stream per
//    (pixel, sample), on a std::thread pool, accumulating FP64 sums;
//  - run sampler_integrator::render as shipped;
//  - evaluate PCG32 and BSDF known-answer vectors.
// Private members are reached through the explicit-instantiation access idiom:
// names in an explicit instantiation are exempt from access checking, and the
// member pointer is carried out through a friend function of a tag type.
#include "../../include/rbgpu.h"

#include "rainbow-cpu/integrators/path_integrator.hpp"
#include "rainbow-cpu/integrators/volume_path_integrator.hpp"
#include "rainbow-cpu/integrators/direct_integrator.hpp"
#include "rainbow-cpu/integrators/photon_mapping_integrator.hpp"
#include "rainbow-cpu/media/homogeneous_medium.hpp"
#include "rainbow-cpu/cameras/perspective_camera.hpp"
#include "rainbow-cpu/filters/box_filter.hpp"
#include "rainbow-cpu/samplers/random_sampler.hpp"
#include "rainbow-cpu/shapes/mesh.hpp"
#include "rainbow-cpu/materials/matte_material.hpp"
#include "rainbow-cpu/materials/metal_material.hpp"
#include "rainbow-cpu/materials/mixture_material.hpp"
#include "rainbow-cpu/materials/glass_material.hpp"
#include "rainbow-cpu/materials/mirror_material.hpp"
#include "rainbow-cpu/materials/plastic_material.hpp"
#include "rainbow-cpu/materials/substrate_material.hpp"
#include "rainbow-cpu/materials/subsurface_material.hpp"
#include "rainbow-cpu/materials/translucent_material.hpp"
#include "rainbow-cpu/materials/uber_material.hpp"
#include "rainbow-cpu/emitters/surface_light.hpp"
#include "rainbow-cpu/emitters/environment_light.hpp"
#include "rainbow-cpu/textures/constant_texture.hpp"
#include "texture_lookup.hpp"  // before the image texture definitions (shim/)
#include "rainbow-cpu/textures/image_texture.hpp"
#include "rainbow-cpu/textures/mixture_texture.hpp"
#include "rainbow-cpu/textures/scale_texture.hpp"
#include "rainbow-cpu/shared/accelerators/bounding_volume_hierarchy.hpp"
#include "rainbow-core/sample_function.hpp"

#include <atomic>
#include <chrono>
#include <cstring>
#include <thread>
#include <unordered_map>

using namespace rainbow::cpus;
using namespace rainbow::cpus::shared;
using namespace rainbow::cpus::scenes;
using namespace rainbow::cpus::cameras;
using namespace rainbow::cpus::integrators;
using namespace rainbow::cpus::materials;
using namespace rainbow::cpus::emitters;
using namespace rainbow::cpus::textures;
using namespace rainbow::cpus::shapes;
using namespace rainbow::cpus::samplers;
using namespace rainbow::cpus::shared::accelerators;
using rainbow::core::real;
using rainbow::core::math::vector2;
using rainbow::core::math::vector3;
using rainbow::core::math::vector2i;
using rainbow::core::math::matrix4x4;

// ------------------------------------------------------------------ private-member access
template <auto Member, typename Tag>
struct access_bind {
	friend constexpr auto member_of(Tag) { return Member; }
};
struct scene_accelerator_tag { friend constexpr auto member_of(scene_accelerator_tag); };
struct bvh_root_tag { friend constexpr auto member_of(bvh_root_tag); };
struct bvh_boxes_tag { friend constexpr auto member_of(bvh_boxes_tag); };
struct entity_instance_tag { friend constexpr auto member_of(entity_instance_tag); };
struct camera_raster_to_camera_tag { friend constexpr auto member_of(camera_raster_to_camera_tag); };
struct camera_to_world_tag { friend constexpr auto member_of(camera_to_world_tag); };
struct film_pixels_tag { friend constexpr auto member_of(film_pixels_tag); };
struct mesh_accelerator_tag { friend constexpr auto member_of(mesh_accelerator_tag); };
struct mesh_bvh_root_tag { friend constexpr auto member_of(mesh_bvh_root_tag); };
struct mesh_bvh_boxes_tag { friend constexpr auto member_of(mesh_bvh_boxes_tag); };
struct entity_world_to_local_tag { friend constexpr auto member_of(entity_world_to_local_tag); };

template struct access_bind<&scene::mAccelerator, scene_accelerator_tag>;
template struct access_bind<&bounding_volume_hierarchy<scene::entity_reference>::mRoot, bvh_root_tag>;
template struct access_bind<&accelerator<scene::entity_reference>::mBoundingBoxes, bvh_boxes_tag>;
template struct access_bind<&entity::mShapeInstanceProperties, entity_instance_tag>;
template struct access_bind<&projective_camera::mRasterToCamera, camera_raster_to_camera_tag>;
template struct access_bind<&camera::mCameraToWorld, camera_to_world_tag>;
template struct access_bind<&film::mPixels, film_pixels_tag>;
template struct access_bind<&mesh::mAccelerator, mesh_accelerator_tag>;
template struct access_bind<&bounding_volume_hierarchy<mesh::mesh_reference>::mRoot, mesh_bvh_root_tag>;
template struct access_bind<&accelerator<mesh::mesh_reference>::mBoundingBoxes, mesh_bvh_boxes_tag>;
template struct access_bind<&entity::mWorldToLocal, entity_world_to_local_tag>;

namespace {

struct orc_scene_impl {
	std::shared_ptr<scene> world;
	std::vector<std::shared_ptr<entity>> entities;
	std::shared_ptr<film> film_ptr;
	std::shared_ptr<perspective_camera> cam;
	int width = 0, height = 0;
	rb_camera_desc desc{};
	std::unordered_map<const entity*, int32_t> ordinal;
	bool volume = false;  // trace with volume_path_integrator instead of path_integrator
	uint32_t direct_emitter = 0, direct_bsdf = 0;  // > 0: trace with direct_integrator(emitter, bsdf samples)

	std::shared_ptr<perspective_camera> make_camera(const std::shared_ptr<film>& f) const {
		const vector3 eye(desc.eye[0], desc.eye[1], desc.eye[2]);
		const vector3 target(desc.target[0], desc.target[1], desc.target[2]);
		const vector3 up(desc.up[0], desc.up[1], desc.up[2]);
		return std::make_shared<perspective_camera>(f, camera_system::right_hand, bound2(vector2(-1), vector2(1)),
			perspective_right_hand(rainbow::core::math::radians(desc.fov_degrees), static_cast<real>(desc.width),
				static_cast<real>(desc.height)),
			look_at_right_hand(eye, target, up).inverse(), 1e6f, desc.lens_radius);
	}
	std::shared_ptr<film> make_film() const {
		return std::make_shared<film>(std::make_shared<filters::box_filter>(), vector2i(desc.width, desc.height),
			bound2(vector2(0), vector2(1)));
	}
};

std::shared_ptr<constant_texture2d<spectrum>> spectrum_texture(const float* v) {
	return std::make_shared<constant_texture2d<spectrum>>(spectrum(v[0], v[1], v[2]));
}
std::shared_ptr<constant_texture2d<real>> real_texture(float v) {
	return std::make_shared<constant_texture2d<real>>(v);
}

// The scene's image textures as reference image_texture2d<spectrum>s, made once
// each (materials that name the same texture share it).
struct texture_set {
	const rb_texture_desc* descs = nullptr;
	uint32_t count = 0;
	std::vector<std::shared_ptr<texture2d<spectrum>>> made;
	// a constant texture of v, or with ref > 0 texture ref - 1: an image, or a
	// scale_texture_t / mixture_texture_t of images and constants
	std::shared_ptr<texture2d<spectrum>> spectrum_of(const float* v, uint32_t ref, int depth = 0) {
		if (ref == 0) return spectrum_texture(v);
		if (ref > count || depth > 1) return nullptr;
		if (made.size() < count) made.resize(count);
		auto& t = made[ref - 1];
		if (t) return t;
		const rb_texture_desc& d = descs[ref - 1];
		if (d.kind == RB_TEXTURE_IMAGE) {
			std::vector<spectrum> values;
			values.reserve(static_cast<size_t>(d.width) * d.height);
			for (size_t i = 0; i < static_cast<size_t>(d.width) * d.height; i++)
				values.emplace_back(d.rgb[3 * i], d.rgb[3 * i + 1], d.rgb[3 * i + 2]);
			t = std::make_shared<image_texture2d<spectrum>>(rainbow::core::math::vector_t<2, size_t>(d.width, d.height), values);
		} else if (d.kind == RB_TEXTURE_SCALE) {
			const auto scale = spectrum_of(d.constants[0], d.inputs[0], depth + 1);
			const auto base = spectrum_of(d.constants[1], d.inputs[1], depth + 1);
			if (!scale || !base) return nullptr;
			t = std::make_shared<scale_texture_t<2, spectrum>>(scale, base);
		} else if (d.kind == RB_TEXTURE_MIXTURE) {
			const auto t0 = spectrum_of(d.constants[0], d.inputs[0], depth + 1);
			const auto t1 = spectrum_of(d.constants[1], d.inputs[1], depth + 1);
			if (!t0 || !t1) return nullptr;
			t = std::make_shared<mixture_texture_t<2, spectrum>>(t0, t1, real_of(d.constants[2][0], d.inputs[2]));
		} else {
			return nullptr;
		}
		return t;
	}
	// a real texture: a constant, or with ref > 0 texture ref - 1 read at channel
	// 0: an image_texture2d<real>, or a scale / mixture texture of real images
	// and constants
	std::shared_ptr<texture2d<real>> real_of(float v, uint32_t ref, int depth = 0) {
		if (ref == 0 || ref > count || depth > 1) return real_texture(v);
		const rb_texture_desc& d = descs[ref - 1];
		if (d.kind == RB_TEXTURE_SCALE)
			return std::make_shared<scale_texture_t<2, real>>(real_of(d.constants[0][0], d.inputs[0], depth + 1),
				real_of(d.constants[1][0], d.inputs[1], depth + 1));
		if (d.kind == RB_TEXTURE_MIXTURE)
			return std::make_shared<mixture_texture_t<2, real>>(real_of(d.constants[0][0], d.inputs[0], depth + 1),
				real_of(d.constants[1][0], d.inputs[1], depth + 1), real_of(d.constants[2][0], d.inputs[2], depth + 1));
		std::vector<real> values;
		for (size_t i = 0; i < static_cast<size_t>(d.width) * d.height; i++) values.push_back(d.rgb[3 * i]);
		return std::make_shared<image_texture2d<real>>(rainbow::core::math::vector_t<2, size_t>(d.width, d.height), values);
	}
};

// Material k of the array `all` (count entries); a mixture's components are
// indices into the same array (nesting up to 8 deep).
std::shared_ptr<material> make_material(const rb_material_desc* all, uint32_t count, uint32_t k, texture_set& tex,
	int depth = 0) {
	if (k >= count || depth > 8) return nullptr;
	const rb_material_desc& m = all[k];
	const auto diffuse = tex.spectrum_of(m.diffuse, m.diffuse_texture);
	const auto reflectance = tex.spectrum_of(m.reflectance, m.reflectance_texture);
	const auto transmission = tex.spectrum_of(m.transmission, m.transmission_texture);
	const auto specular = tex.spectrum_of(m.specular, m.specular_texture);
	const auto opacity = tex.spectrum_of(m.opacity, m.opacity_texture);
	if (!diffuse || !reflectance || !transmission || !specular || !opacity) return nullptr;
	switch (m.kind) {
	case RB_MATERIAL_MATTE: return std::make_shared<matte_material>(diffuse, tex.real_of(m.sigma, m.sigma_texture));
	case RB_MATERIAL_METAL:
		return std::make_shared<metal_material>(tex.spectrum_of(m.eta, m.eta_texture), tex.spectrum_of(m.k, m.k_texture),
			tex.real_of(m.roughness_u, m.roughness_u_texture),
			tex.real_of(m.roughness_v, m.roughness_v_texture), m.remap_roughness != 0);
	case RB_MATERIAL_GLASS:
		return std::make_shared<glass_material>(reflectance, transmission, tex.real_of(m.roughness_u, m.roughness_u_texture),
			tex.real_of(m.roughness_v, m.roughness_v_texture), tex.real_of(m.ior, m.ior_texture), m.remap_roughness != 0);
	case RB_MATERIAL_PLASTIC:
		return std::make_shared<plastic_material>(reflectance, diffuse, tex.real_of(m.roughness_u, m.roughness_u_texture), tex.real_of(m.ior, m.ior_texture),
			m.remap_roughness != 0);
	case RB_MATERIAL_MIRROR: return std::make_shared<mirror_material>(reflectance);
	case RB_MATERIAL_SUBSTRATE:
		return std::make_shared<substrate_material>(reflectance, diffuse, tex.real_of(m.roughness_u, m.roughness_u_texture),
			tex.real_of(m.roughness_v, m.roughness_v_texture), m.remap_roughness != 0);
	case RB_MATERIAL_UBER:
		return std::make_shared<uber_material>(transmission, reflectance, specular, diffuse, opacity,
			tex.real_of(m.roughness_u, m.roughness_u_texture), tex.real_of(m.roughness_v, m.roughness_v_texture), tex.real_of(m.ior, m.ior_texture), m.remap_roughness != 0);
	case RB_MATERIAL_TRANSLUCENT:
		return std::make_shared<translucent_material>(transmission, reflectance, specular, diffuse,
			tex.real_of(m.roughness_u, m.roughness_u_texture), m.remap_roughness != 0);
	case RB_MATERIAL_SUBSURFACE:
		return std::make_shared<subsurface_material>(transmission, reflectance, diffuse, tex.spectrum_of(m.mfp, m.mfp_texture),
			tex.real_of(m.roughness_u, m.roughness_u_texture), tex.real_of(m.roughness_v, m.roughness_v_texture), tex.real_of(m.ior, m.ior_texture), m.remap_roughness != 0);
	case RB_MATERIAL_MIXTURE: {
		if (m.components[0] < 0 || m.components[1] < 0) return nullptr;
		const auto m0 = make_material(all, count, static_cast<uint32_t>(m.components[0]), tex, depth + 1);
		const auto m1 = make_material(all, count, static_cast<uint32_t>(m.components[1]), tex, depth + 1);
		if (!m0 || !m1) return nullptr;
		return std::make_shared<mixture_material>(spectrum_texture(m.amount), m0, m1);
	}
	default: return nullptr;
	}
}

matrix4x4 to_matrix(const float* m) {
	matrix4x4 r;
	for (int c = 0; c < 4; c++)
		for (int row = 0; row < 4; row++) r[c][row] = m[c * 4 + row];
	return r;
}
void from_matrix(const matrix4x4& m, float* out) {
	for (int c = 0; c < 4; c++)
		for (int row = 0; row < 4; row++) out[c * 4 + row] = m[c][row];
}

std::vector<vector3> to_vec3(const float* p, uint32_t n) {
	std::vector<vector3> v;
	if (p == nullptr) return v;
	v.reserve(n);
	for (uint32_t i = 0; i < n; i++) v.emplace_back(p[3 * i], p[3 * i + 1], p[3 * i + 2]);
	return v;
}

// Seed of the PCG32 stream of one (pixel, sample): pixel index in bits 0-23,
// sample index in bits 24-47, the render seed in bits 48-62.
uint64_t stream_seed(uint32_t pixel, uint32_t sample, uint32_t seed) {
	return static_cast<uint64_t>(pixel & 0xffffffu) | (static_cast<uint64_t>(sample & 0xffffffu) << 24) |
		(static_cast<uint64_t>(seed & 0x7fffu) << 48);
}

struct sample_driver {
	std::shared_ptr<sampler_integrator> integrator;
	std::shared_ptr<sampler1d> proto1;
	std::shared_ptr<sampler2d> proto2;
	sample_driver(uint32_t max_depth, float rr, bool volume, uint32_t direct_emitter = 0, uint32_t direct_bsdf = 0) {
		proto1 = std::make_shared<random_sampler1d>(1);
		proto2 = std::make_shared<random_sampler2d>(1);
		if (direct_emitter > 0 && direct_bsdf > 0)
			integrator = std::make_shared<direct_integrator>(proto2, proto1, direct_emitter, direct_bsdf);
		else if (volume) integrator = std::make_shared<volume_path_integrator>(proto2, proto1, max_depth, rr);
		else integrator = std::make_shared<path_integrator>(proto2, proto1, max_depth, rr);
	}
	// One sample of the body of sampler_integrator::render (sampler_integrator.cpp:102-130),
	// with samplers seeded per (pixel, sample).
	spectrum run(orc_scene_impl& s, int x, int y, uint32_t sample, uint32_t seed) {
		const uint32_t pixel = static_cast<uint32_t>(y) * static_cast<uint32_t>(s.width) + static_cast<uint32_t>(x);
		const auto generator = std::make_shared<random_generator>(stream_seed(pixel, sample, seed));
		const sampler_group samplers(proto1->clone(generator), proto2->clone(generator));
		const auto position = vector2(x, y) + samplers.sampler2d->next();
		const auto ray = s.cam->sample(position, samplers.sampler2d->next());
		return integrator->trace(s.world, integrator_debug_info(vector2i(x, y), sample), samplers, ray, 0);
	}
};

} // namespace

struct orc_scene : orc_scene_impl {};

extern "C" {

int orc_scene_build(const rb_scene_desc* desc, const rb_camera_desc* cam, orc_scene** out) {
	if (desc == nullptr || cam == nullptr || out == nullptr) return RB_ERR_INVALID_ARGUMENT;
	auto* s = new orc_scene();
	std::vector<std::shared_ptr<mesh>> meshes;
	for (uint32_t i = 0; i < desc->num_meshes; i++) {
		const rb_mesh_desc& m = desc->meshes[i];
		std::vector<unsigned> idx(m.indices, m.indices + 3 * m.num_triangles);
		meshes.push_back(std::make_shared<mesh>(to_vec3(m.positions, m.num_vertices), to_vec3(m.tangents, m.num_vertices),
			to_vec3(m.normals, m.num_vertices), to_vec3(m.uvs, m.num_vertices), idx, m.reverse_orientation != 0));
	}
	std::vector<std::shared_ptr<material>> materials;
	texture_set tex{desc->textures, desc->num_textures, {}};
	for (uint32_t i = 0; i < desc->num_materials; i++)
		materials.push_back(make_material(desc->materials, desc->num_materials, i, tex));
	std::vector<std::shared_ptr<emitter>> emitter_list;
	for (uint32_t i = 0; i < desc->num_emitters; i++) {
		const rb_emitter_desc& e = desc->emitters[i];
		const spectrum L(e.radiance[0], e.radiance[1], e.radiance[2]);
		if (e.kind == RB_EMITTER_SURFACE) emitter_list.push_back(std::make_shared<surface_light>(L));
		else emitter_list.push_back(std::make_shared<environment_light>(L, e.radius));
	}
	std::vector<std::shared_ptr<rainbow::cpus::media::medium>> mediums;
	for (uint32_t i = 0; i < desc->num_mediums; i++) {
		const rb_medium_desc& m = desc->mediums[i];
		mediums.push_back(std::make_shared<rainbow::cpus::media::homogeneous_medium>(spectrum(m.sigma_a[0], m.sigma_a[1], m.sigma_a[2]),
			spectrum(m.sigma_s[0], m.sigma_s[1], m.sigma_s[2]), m.g));
	}
	std::vector<std::shared_ptr<rainbow::cpus::media::media>> media_list;
	for (uint32_t i = 0; i < desc->num_media; i++) {
		const rb_media_desc& m = desc->media[i];
		media_list.push_back(std::make_shared<rainbow::cpus::media::media>(m.outside >= 0 ? mediums[m.outside] : nullptr,
			m.inside >= 0 ? mediums[m.inside] : nullptr));
	}
	s->world = std::make_shared<scene>();
	for (uint32_t i = 0; i < desc->num_entities; i++) {
		const rb_entity_desc& e = desc->entities[i];
		const transform xf(to_matrix(e.local_to_world), to_matrix(e.world_to_local));
		auto ent = std::make_shared<entity>(e.material >= 0 ? materials[e.material] : nullptr,
			e.emitter >= 0 ? emitter_list[e.emitter] : nullptr, e.mesh >= 0 ? meshes[e.mesh] : nullptr,
			e.medium >= 0 ? media_list[e.medium] : nullptr, xf);
		s->ordinal[ent.get()] = static_cast<int32_t>(i);
		s->entities.push_back(ent);
		s->world->add_entity(ent);
	}
	s->world->build_accelerator();

	s->width = cam->width;
	s->height = cam->height;
	s->desc = *cam;
	s->film_ptr = s->make_film();
	s->cam = s->make_camera(s->film_ptr);
	*out = s;
	return RB_OK;
}

void orc_scene_free(orc_scene* s) { delete s; }

// The reference scene and camera of a harness scene (pointers to their
// shared_ptrs), for other test libraries that drive reference objects.
int orc_scene_objects(orc_scene* s, const void** world, const void** cam) {
	if (s == nullptr || world == nullptr || cam == nullptr) return RB_ERR_INVALID_ARGUMENT;
	*world = &s->world;
	*cam = &s->cam;
	return RB_OK;
}

// The camera's film as an integrator left it: pixel::spectrum() of every pixel
// (film.cpp:19-24), W * H * 3 floats; 0 for a pixel nothing has written yet
// (pixel::spectrum asserts a non-zero filter weight).
int orc_film_read(orc_scene* s, float* rgb) {
	const auto& pixels = (*s->film_ptr).*member_of(film_pixels_tag{});
	for (size_t i = 0; i < pixels.size(); i++) {
		const spectrum L = pixels[i].filter_weight != 0 ? pixels[i].spectrum() : spectrum(0);
		rgb[3 * i] = L[0]; rgb[3 * i + 1] = L[1]; rgb[3 * i + 2] = L[2];
	}
	return RB_OK;
}

// The seeded synthetic scene of the benchmark configurations
// (rb_scene_generate, compiled into this library from the same source file as
// the product's generator), built directly as a reference scene and camera, so
// that a CPU-only caller needs nothing but this library. *triangles: the
// scene's triangle count.
int orc_scene_generate(const rb_scene_gen_params* params, orc_scene** out, uint32_t* triangles) {
	if (params == nullptr || out == nullptr) return RB_ERR_INVALID_ARGUMENT;
	rb_scene* gen = nullptr;
	int st = rb_scene_generate(params, &gen);
	if (st != RB_OK) return st;
	rb_scene_desc desc{};
	rb_camera_desc cam{};
	st = rb_scene_get(gen, &desc, &cam);
	if (st == RB_OK && triangles != nullptr) {
		uint64_t n = 0;
		for (uint32_t i = 0; i < desc.num_entities; i++)
			if (desc.entities[i].mesh >= 0) n += desc.meshes[desc.entities[i].mesh].num_triangles;
		*triangles = static_cast<uint32_t>(n);
	}
	if (st == RB_OK) st = orc_scene_build(&desc, &cam, out);
	rb_scene_free(gen);
	return st;
}

// Selects the integrator of the tracing entry points: path_integrator (0) or
// volume_path_integrator (1).
void orc_set_volume(orc_scene* s, int volume) { s->volume = volume != 0; }

// Selects direct_integrator(sampler2d, sampler1d, emitter_samples, bsdf_samples)
// for the tracing entry points (both > 0), or clears that choice (either 0).
void orc_set_direct(orc_scene* s, uint32_t emitter_samples, uint32_t bsdf_samples) {
	s->direct_emitter = emitter_samples;
	s->direct_bsdf = bsdf_samples;
}



} // extern "C"

namespace {

template <typename T>
const bounding_volume_hierarchy_node<T>* bvh_root(const accelerator<T>& acc) {
	const auto& bvh = dynamic_cast<const bounding_volume_hierarchy<T>&>(acc);
	return bvh.*member_of(bvh_root_tag{});
}
template <typename T>
const std::vector<bounding_box<T>>& bvh_boxes(const accelerator<T>& acc) {
	return acc.*member_of(bvh_boxes_tag{});
}
// mesh::mesh_reference is a private type: it is recovered from the type of the
// mAccelerator member pointer (types carry no access checks, names do).
template <typename> struct member_type;
template <typename C, typename M> struct member_type<M C::*> { using type = M; };
template <typename> struct accelerator_element;
template <typename T> struct accelerator_element<accelerator<T>> { using type = T; };
using mesh_ref = typename accelerator_element<
	typename member_type<decltype(member_of(mesh_accelerator_tag{}))>::type::element_type>::type;
const bounding_volume_hierarchy_node<mesh_ref>* bvh_root(const accelerator<mesh_ref>& acc) {
	const auto& bvh = dynamic_cast<const bounding_volume_hierarchy<mesh_ref>&>(acc);
	return bvh.*member_of(mesh_bvh_root_tag{});
}
const std::vector<bounding_box<mesh_ref>>& bvh_boxes(const accelerator<mesh_ref>& acc) {
	return acc.*member_of(mesh_bvh_boxes_tag{});
}
// The accelerator of an entity's mesh (built by scene::build_accelerator in the
// two-level case), or null.
const accelerator<mesh_ref>* mesh_accelerator(const entity& e) {
	const auto m = std::dynamic_pointer_cast<mesh>(e.component<shape>());
	return m ? ((*m).*member_of(mesh_accelerator_tag{})).get() : nullptr;
}

void put_u32(float* dst, uint32_t v) { std::memcpy(dst, &v, sizeof(v)); }

template <typename T>
void flatten(const orc_scene* s, const bounding_volume_hierarchy_node<T>* n, std::vector<float>& out) {
	const size_t index = out.size() / 8;
	out.resize(out.size() + 8);
	const auto& b = n->box.box;
	float* w = out.data() + index * 8;
	w[0] = b.min.x; w[1] = b.min.y; w[2] = b.min.z; w[3] = b.max.x; w[4] = b.max.y; w[5] = b.max.z;
	if (n->is_leaf()) {
		put_u32(w + 6, static_cast<uint32_t>(n->begin));
		put_u32(w + 7, RB_BVH_LEAF_FLAG | static_cast<uint32_t>(n->end - n->begin));
		return;
	}
	flatten(s, n->left, out);
	const uint32_t right = static_cast<uint32_t>(out.size() / 8);
	flatten(s, n->right, out);
	w = out.data() + index * 8;
	put_u32(w + 6, right);
	put_u32(w + 7, static_cast<uint32_t>(n->axis));
}

// The walk of mesh::intersect over a mesh's own tree (the reference's
// bounding_volume_hierarchy<mesh_reference>::intersect order) on a local ray,
// calling the reference's triangle test; *face: the last face that hit.
void mesh_walk(const accelerator<mesh_ref>& acc, const ray& r, int32_t* face) {
	const auto* root = bvh_root(acc);
	const auto& boxes = bvh_boxes(acc);
	std::vector<const bounding_volume_hierarchy_node<mesh_ref>*> stack{root};
	const auto inv = static_cast<real>(1) / r.direction;
	const bool neg[3] = {inv.x < 0, inv.y < 0, inv.z < 0};
	while (!stack.empty()) {
		const auto* n = stack.back();
		stack.pop_back();
		if (!n->box.intersect(r)) continue;
		if (n->is_leaf()) {
			for (auto i = n->begin; i < n->end; i++)
				if (boxes[i].entity->intersect(r).has_value()) *face = static_cast<int32_t>(boxes[i].entity->face);
			continue;
		}
		if (neg[n->axis]) { stack.push_back(n->left); stack.push_back(n->right); }
		else { stack.push_back(n->right); stack.push_back(n->left); }
	}
}

// Closest-hit walk over the reference's tree in the order of
// bounding_volume_hierarchy<T>::intersect (detail/bounding_volume_hierarchy.hpp:60-108),
// calling the reference's own leaf test, to learn which triangle was hit (the
// returned surface_interaction does not carry the triangle index).
template <typename T>
void walk(const accelerator<T>& acc, const ray& r, bool shadow, const orc_scene* s, int32_t* ent, int32_t* tri) {
	const auto* root = bvh_root(acc);
	const auto& boxes = bvh_boxes(acc);
	std::vector<const bounding_volume_hierarchy_node<T>*> stack{root};
	const auto inv = static_cast<real>(1) / r.direction;
	const bool neg[3] = {inv.x < 0, inv.y < 0, inv.z < 0};
	*ent = -1;
	*tri = -1;
	while (!stack.empty()) {
		const auto* n = stack.back();
		stack.pop_back();
		if (!n->box.intersect(r)) continue;
		if (n->is_leaf()) {
			for (auto i = n->begin; i < n->end; i++) {
				const auto& ref = *boxes[i].entity;
				if (shadow && !ref.entity->visible()) continue;
				if (ref.index == std::numeric_limits<size_t>::max()) {
					// the whole entity: entity::intersect walks its mesh's tree with the
					// local ray; the same walk on a copy of that local ray names the face
					const ray local = ((*ref.entity).*member_of(entity_world_to_local_tag{}))(r);
					int32_t face = -1;
					mesh_walk(*mesh_accelerator(*ref.entity), local, &face);
					if (ref.intersect(r).has_value()) {
						*ent = s->ordinal.at(ref.entity.get());
						*tri = face;
					}
					continue;
				}
				if (ref.intersect(r).has_value()) {
					*ent = s->ordinal.at(ref.entity.get());
					*tri = static_cast<int32_t>(ref.index);
				}
			}
			continue;
		}
		if (neg[n->axis]) { stack.push_back(n->left); stack.push_back(n->right); }
		else { stack.push_back(n->right); stack.push_back(n->left); }
	}
}

} // namespace

extern "C" {

// Flattened copy of the reference's own BVH (rb_bvh_desc layout). Call with
// NULL arrays first to get the sizes.
int orc_export_bvh(orc_scene* s, float* nodes, uint32_t* prim_entity, uint32_t* prim_index, uint32_t* num_nodes, uint32_t* num_prims) {
	const auto& acc = *((*s->world).*member_of(scene_accelerator_tag{}));
	const auto& boxes = bvh_boxes(acc);
	std::vector<float> flat;
	flatten(s, bvh_root(acc), flat);
	*num_nodes = static_cast<uint32_t>(flat.size() / 8);
	*num_prims = static_cast<uint32_t>(boxes.size());
	if (nodes == nullptr) return RB_OK;
	std::memcpy(nodes, flat.data(), flat.size() * sizeof(float));
	for (size_t i = 0; i < boxes.size(); i++) {
		const auto& ref = *boxes[i].entity;
		prim_entity[i] = static_cast<uint32_t>(s->ordinal.at(ref.entity.get()));
		prim_index[i] = ref.index == std::numeric_limits<size_t>::max() ? RB_BVH_ALL_TRIANGLES : static_cast<uint32_t>(ref.index);
	}
	return RB_OK;
}

// Flattened copy of the reference's own tree of entity `entity`'s mesh (the
// two-level case: mesh::build_accelerator); faces[p] is the face of leaf
// element p. RB_ERR_UNSUPPORTED when the mesh has no tree. NULL arrays: sizes only.
int orc_export_mesh_bvh(orc_scene* s, uint32_t entity, float* nodes, uint32_t* faces, uint32_t* num_nodes, uint32_t* num_prims) {
	if (entity >= s->entities.size()) return RB_ERR_INVALID_ARGUMENT;
	const auto* acc = mesh_accelerator(*s->entities[entity]);
	if (acc == nullptr) return RB_ERR_UNSUPPORTED;
	const auto& boxes = bvh_boxes(*acc);
	std::vector<float> flat;
	flatten(s, bvh_root(*acc), flat);
	*num_nodes = static_cast<uint32_t>(flat.size() / 8);
	*num_prims = static_cast<uint32_t>(boxes.size());
	if (nodes == nullptr) return RB_OK;
	std::memcpy(nodes, flat.data(), flat.size() * sizeof(float));
	for (size_t i = 0; i < boxes.size(); i++) faces[i] = static_cast<uint32_t>(boxes[i].entity->face);
	return RB_OK;
}

int orc_export_camera(orc_scene* s, float* raster_to_camera, float* camera_to_world) {
	const transform& r2c = (*s->cam).*member_of(camera_raster_to_camera_tag{});
	const transform& c2w = (*s->cam).*member_of(camera_to_world_tag{});
	from_matrix(r2c.matrix(), raster_to_camera);
	from_matrix(c2w.matrix(), camera_to_world);
	return RB_OK;
}

// World-space area of each entity's shape (shape_instance_properties::area), 0 without a shape.
int orc_export_areas(orc_scene* s, float* areas) {
	for (size_t i = 0; i < s->entities.size(); i++) areas[i] = ((*s->entities[i]).*member_of(entity_instance_tag{})).area;
	return RB_OK;
}

// scene::intersect (shadow = 0) or scene::intersect_with_shadow_ray (shadow = 1)
// of each ray, taken as the reference ray holds it (no renormalisation).
// points (3 per ray, may be NULL) receives the world hit point.
int orc_trace(orc_scene* s, const rb_ray* rays, uint32_t n, int shadow, rb_hit* hits, float* points) {
	const auto& acc = *((*s->world).*member_of(scene_accelerator_tag{}));
	int status = RB_OK;
	for (uint32_t i = 0; i < n; i++) {
		ray r;
		r.origin = vector3(rays[i].origin[0], rays[i].origin[1], rays[i].origin[2]);
		r.direction = vector3(rays[i].direction[0], rays[i].direction[1], rays[i].direction[2]);
		r.length = rays[i].length;
		const auto hit = shadow ? s->world->intersect_with_shadow_ray(r) : s->world->intersect(r);
		rb_hit& h = hits[i];
		h.t = r.length;
		h.b1 = h.b2 = std::numeric_limits<float>::quiet_NaN();
		ray w;
		w.origin = vector3(rays[i].origin[0], rays[i].origin[1], rays[i].origin[2]);
		w.direction = vector3(rays[i].direction[0], rays[i].direction[1], rays[i].direction[2]);
		w.length = rays[i].length;
		walk(acc, w, shadow != 0, s, &h.entity, &h.triangle);
		const int32_t e = hit.has_value() ? s->ordinal.at(hit->entity.get()) : -1;
		if (e != h.entity || !(w.length == r.length || (std::isnan(w.length) && std::isnan(r.length)))) status = RB_ERR_CHECKPOINT;
		if (points != nullptr) {
			const vector3 p = hit.has_value() ? hit->point : vector3(0);
			points[3 * i] = p.x; points[3 * i + 1] = p.y; points[3 * i + 2] = p.z;
		}
	}
	return status;
}

// Seeded ray batch: for each ray a random (pixel, sample) camera ray, then
// `bounces` (0, 1 or 2, chosen per ray) cosine-distributed continuations spawned
// with interaction::spawn_ray from the reference's own hit points.
int orc_make_rays(orc_scene* s, uint32_t n, uint64_t seed, rb_ray* out) {
	pcg32 rng(seed);
	for (uint32_t i = 0; i < n; i++) {
		const int x = static_cast<int>(rng.uniform_uint32() % static_cast<uint32_t>(s->width));
		const int y = static_cast<int>(rng.uniform_uint32() % static_cast<uint32_t>(s->height));
		const vector2 pos = vector2(x, y) + vector2(rng.uniform_real(), rng.uniform_real());
		ray r = s->cam->sample(pos, vector2(rng.uniform_real(), rng.uniform_real()));
		const uint32_t bounces = rng.uniform_uint32() % 3u;
		for (uint32_t b = 0; b < bounces; b++) {
			ray probe = r;
			const auto hit = s->world->intersect(probe);
			if (!hit.has_value()) break;
			const coordinate_system frame(hit->normal);
			auto d = rainbow::core::cosine_sample_hemisphere(vector2(rng.uniform_real(), rng.uniform_real()));
			if (dot(hit->normal, r.direction) > 0) d.z = -d.z;
			r = hit->spawn_ray(local_to_world(frame, d));
		}
		rb_ray& o = out[i];
		o.origin[0] = r.origin.x; o.origin[1] = r.origin.y; o.origin[2] = r.origin.z;
		o.direction[0] = r.direction.x; o.direction[1] = r.direction.y; o.direction[2] = r.direction.z;
		o.length = r.length;
	}
	return RB_OK;
}

// Camera ray of each (pixel, sample) exactly as the per-sample driver makes it.
int orc_camera_rays(orc_scene* s, const uint32_t* pixels, const uint32_t* samples, uint32_t n, uint32_t seed, rb_ray* out) {
	for (uint32_t i = 0; i < n; i++) {
		const int x = static_cast<int>(pixels[i] % static_cast<uint32_t>(s->width));
		const int y = static_cast<int>(pixels[i] / static_cast<uint32_t>(s->width));
		random_generator gen(stream_seed(pixels[i], samples[i], seed));
		const vector2 pos = vector2(x, y) + vector2(gen.uniform_real(), gen.uniform_real());
		const vector2 lens(gen.uniform_real(), gen.uniform_real());
		const ray r = s->cam->sample(pos, lens);
		rb_ray& o = out[i];
		o.origin[0] = r.origin.x; o.origin[1] = r.origin.y; o.origin[2] = r.origin.z;
		o.direction[0] = r.direction.x; o.direction[1] = r.direction.y; o.direction[2] = r.direction.z;
		o.length = r.length;
	}
	return RB_OK;
}

// Radiance of individual (pixel, sample) pairs through path_integrator::trace.
int orc_trace_samples(orc_scene* s, const uint32_t* pixels, const uint32_t* samples, uint32_t n, uint32_t max_depth, float rr,
	uint32_t seed, float* radiance) {
	sample_driver d(max_depth, rr, s->volume, s->direct_emitter, s->direct_bsdf);
	for (uint32_t i = 0; i < n; i++) {
		const int x = static_cast<int>(pixels[i] % static_cast<uint32_t>(s->width));
		const int y = static_cast<int>(pixels[i] / static_cast<uint32_t>(s->width));
		const spectrum L = d.run(*s, x, y, samples[i], seed);
		radiance[3 * i] = L[0]; radiance[3 * i + 1] = L[1]; radiance[3 * i + 2] = L[2];
	}
	return RB_OK;
}

// Render samples [first_sample, first_sample + spp) of rows [row_begin, row_end)
// on `threads` std::threads, FP64 per-pixel sums of L and L^2 (3 per pixel,
// full image layout; rows outside the range are left untouched).
int orc_render(orc_scene* s, uint32_t spp, uint32_t first_sample, uint32_t max_depth, float rr, uint32_t seed, int threads,
	int row_begin, int row_end, double* sum, double* sum_sq, double* seconds) {
	if (threads <= 0) threads = static_cast<int>(std::max(1u, std::thread::hardware_concurrency()));
	if (row_end <= 0 || row_end > s->height) row_end = s->height;
	std::atomic<int> next_row(row_begin);
	const auto t0 = std::chrono::steady_clock::now();
	auto work = [&]() {
		sample_driver d(max_depth, rr, s->volume, s->direct_emitter, s->direct_bsdf);
		for (int y = next_row++; y < row_end; y = next_row++) {
			for (int x = 0; x < s->width; x++) {
				const size_t p = static_cast<size_t>(y) * s->width + x;
				double acc[3] = {0, 0, 0}, acc2[3] = {0, 0, 0};
				for (uint32_t k = 0; k < spp; k++) {
					const spectrum L = d.run(*s, x, y, first_sample + k, seed);
					for (int c = 0; c < 3; c++) {
						acc[c] += L[c];
						acc2[c] += static_cast<double>(L[c]) * L[c];
					}
				}
				for (int c = 0; c < 3; c++) {
					if (sum) sum[3 * p + c] += acc[c];
					if (sum_sq) sum_sq[3 * p + c] += acc2[c];
				}
			}
		}
	};
	std::vector<std::thread> pool;
	for (int t = 0; t < threads; t++) pool.emplace_back(work);
	for (auto& t : pool) t.join();
	if (seconds) *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
	return RB_OK;
}

// sampler_integrator::render as shipped (per-tile seeds, std::execution::par),
// then the film's per-pixel mean (W * H * 3 floats).
int orc_render_shipped(orc_scene* s, uint32_t spp, uint32_t max_depth, float rr, float* rgb, double* seconds) {
	const auto f = s->make_film();
	const auto cam = s->make_camera(f);
	path_integrator integrator(std::make_shared<random_sampler2d>(spp), std::make_shared<random_sampler1d>(spp), max_depth, rr);
	const auto t0 = std::chrono::steady_clock::now();
	integrator.render(cam, s->world);
	if (seconds) *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
	const auto& pixels = (*f).*member_of(film_pixels_tag{});
	for (size_t i = 0; i < pixels.size(); i++) {
		const spectrum L = pixels[i].spectrum();
		rgb[3 * i] = L[0]; rgb[3 * i + 1] = L[1]; rgb[3 * i + 2] = L[2];
	}
	return RB_OK;
}

// photon_mapping_integrator::render as shipped (stochastic progressive photon
// mapping: per-tile and per-chunk seeds; the parallel loops run in order with
// libstdc++'s serial backend), then the film (W * H * 3 floats, set_pixel values).
int orc_render_photons(orc_scene* s, uint32_t iterations, uint32_t max_depth, uint32_t photons, float radius, float* rgb,
	double* seconds) {
	const auto f = s->make_film();
	const auto cam = s->make_camera(f);
	photon_mapping_integrator integrator(std::make_shared<random_sampler2d>(1), std::make_shared<random_sampler1d>(1),
		iterations, max_depth, photons, radius);
	const auto t0 = std::chrono::steady_clock::now();
	integrator.render(cam, s->world);
	if (seconds) *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
	const auto& pixels = (*f).*member_of(film_pixels_tag{});
	for (size_t i = 0; i < pixels.size(); i++) {
		const spectrum L = pixels[i].spectrum();
		rgb[3 * i] = L[0]; rgb[3 * i + 1] = L[1]; rgb[3 * i + 2] = L[2];
	}
	return RB_OK;
}

// PCG32 known answers: n outputs of uniform_uint32 from pcg32(seed), and n of
// uniform_real from a second pcg32(seed).
int orc_pcg32(uint64_t seed, uint32_t n, uint32_t* u32, float* reals) {
	pcg32 a(seed), b(seed);
	for (uint32_t i = 0; i < n; i++) {
		u32[i] = a.uniform_uint32();
		reals[i] = b.uniform_real();
	}
	return RB_OK;
}

// image_texture2d<spectrum>(size, texels).sample(uv) for n texture coordinates.
int orc_texture_sample(const float* rgb, uint32_t width, uint32_t height, uint32_t n, const float* uv, float* out) {
	if (rgb == nullptr || width == 0 || height == 0) return RB_ERR_INVALID_ARGUMENT;
	rb_texture_desc d{rgb, width, height};
	texture_set tex{&d, 1u, {}};
	const float zero[3] = {0.f, 0.f, 0.f};
	const auto t = tex.spectrum_of(zero, 1u);
	for (uint32_t i = 0; i < n; i++) {
		const auto v = t->sample(vector2(uv[2 * i], uv[2 * i + 1]));
		out[3 * i] = v[0];
		out[3 * i + 1] = v[1];
		out[3 * i + 2] = v[2];
	}
	return RB_OK;
}

// BSDF known answers on the shading frame = world axes: for each (wo, u)
// scattering_function_collection::sample(interaction, u, include); for each
// (wo, wi) evaluate and pdf with `include`.
// m[0] is the material; a mixture's components index m[0 .. num_materials).
int orc_bsdf(const rb_material_desc* m, uint32_t num_materials, uint32_t n, const float* wo, const float* u,
	const float* wi_eval, uint32_t include, float* wi_out, float* f_out, float* pdf_out, uint32_t* type_out, float* f_eval,
	float* pdf_eval) {
	texture_set tex;
	const auto mat = make_material(m, num_materials, 0, tex);
	if (!mat) return RB_ERR_INVALID_ARGUMENT;
	for (uint32_t i = 0; i < n; i++) {
		surface_interaction si;
		si.wo = vector3(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]);
		si.normal = vector3(0, 0, 1);
		const auto props = mat->build_surface_properties(si);
		const auto type = static_cast<scatterings::scattering_type>(include);
		const auto smp = props.functions.sample(si, vector2(u[2 * i], u[2 * i + 1]), type);
		wi_out[3 * i] = smp.wi.x; wi_out[3 * i + 1] = smp.wi.y; wi_out[3 * i + 2] = smp.wi.z;
		f_out[3 * i] = smp.value[0]; f_out[3 * i + 1] = smp.value[1]; f_out[3 * i + 2] = smp.value[2];
		pdf_out[i] = smp.pdf;
		type_out[i] = static_cast<uint32_t>(smp.type);
		const vector3 wie(wi_eval[3 * i], wi_eval[3 * i + 1], wi_eval[3 * i + 2]);
		const auto fe = props.functions.evaluate(si.wo, wie, type);
		f_eval[3 * i] = fe[0]; f_eval[3 * i + 1] = fe[1]; f_eval[3 * i + 2] = fe[2];
		pdf_eval[i] = props.functions.pdf(si.wo, wie, type);
	}
	return RB_OK;
}

} // extern "C"
