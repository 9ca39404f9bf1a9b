// Test entry points over the drop-in adapter (TEST INFRASTRUCTURE).
//
// Built by oracle/Makefile into _ref/libadapter_check.so from
// rainbow_b200/adapter/*.cpp (the wavefront_path_integrator a maintainer adds
// to the reference) and this file, against the reference's headers, linked with
// liboracle_ref.so (the reference itself and the harness's scenes) and
// librbgpu.so. Only the tests load it.
#include "../../rainbow_b200/adapter/scene_export.hpp"
#include "../../rainbow_b200/adapter/wavefront_path_integrator.hpp"
#include "../../rainbow_b200/adapter/wavefront_photon_mapping_integrator.hpp"

#include "rainbow-cpu/cameras/perspective_camera.hpp"
#include "rainbow-cpu/samplers/random_sampler.hpp"

#include <cstring>
#include <exception>

using namespace rainbow::cpus;

struct orc_scene;
extern "C" int orc_scene_objects(orc_scene* s, const void** world, const void** cam);

namespace {
bool objects(orc_scene* s, std::shared_ptr<scenes::scene>& world, std::shared_ptr<cameras::camera>& cam) {
	const void *w = nullptr, *c = nullptr;
	if (orc_scene_objects(s, &w, &c) != RB_OK) return false;
	world = *static_cast<const std::shared_ptr<scenes::scene>*>(w);
	cam = *static_cast<const std::shared_ptr<cameras::perspective_camera>*>(c);
	return true;
}
} // namespace

extern "C" {

// wavefront_path_integrator(random_sampler2d(spp), random_sampler1d(spp),
// max_depth, threshold).render(camera, scene) on a harness scene; the result is
// in the camera's film (orc_film_read). Returns 0, or -1 when render threw.
int adp_render(orc_scene* s, uint32_t spp, uint32_t max_depth, float threshold, uint32_t seed, char* error, uint32_t error_size) {
	std::shared_ptr<scenes::scene> world;
	std::shared_ptr<cameras::camera> cam;
	if (!objects(s, world, cam)) return RB_ERR_INVALID_ARGUMENT;
	try {
		integrators::wavefront_path_integrator integrator(std::make_shared<samplers::random_sampler2d>(spp),
			std::make_shared<samplers::random_sampler1d>(spp), max_depth, threshold);
		integrator.set_seed(seed);
		integrator.render(cam, world);
	} catch (const std::exception& e) {
		if (error != nullptr && error_size > 0) {
			std::strncpy(error, e.what(), error_size - 1);
			error[error_size - 1] = '\0';
		}
		return -1;
	}
	return RB_OK;
}

// The adapter's export of a harness scene: the tree rb_bvh_build makes of it
// (sizes first with NULL arrays) and, per entity, its material and emitter
// descriptions (has[2 e] / has[2 e + 1]: 1 when present).
// wavefront_photon_mapping_integrator(random_sampler2d(1), random_sampler1d(1),
// iterations, max_depth, photons, radius).render(camera, scene) on a harness
// scene; the result is in the camera's film. Returns 0, or -1 when render threw.
int adp_render_photons(orc_scene* s, uint32_t iterations, uint32_t max_depth, uint32_t photons, float radius,
	uint32_t seed, char* error, uint32_t error_size) {
	std::shared_ptr<scenes::scene> world;
	std::shared_ptr<cameras::camera> cam;
	if (!objects(s, world, cam)) return RB_ERR_INVALID_ARGUMENT;
	try {
		integrators::wavefront_photon_mapping_integrator integrator(std::make_shared<samplers::random_sampler2d>(1),
			std::make_shared<samplers::random_sampler1d>(1), iterations, max_depth, photons, radius);
		integrator.set_seed(seed);
		integrator.render(cam, world);
	} catch (const std::exception& e) {
		if (error != nullptr && error_size > 0) {
			std::strncpy(error, e.what(), error_size - 1);
			error[error_size - 1] = 0;
		}
		return -1;
	}
	return 0;
}

int adp_export(orc_scene* s, float* nodes, uint32_t* prim_entity, uint32_t* prim_index, uint32_t* num_nodes,
	uint32_t* num_prims, rb_material_desc* materials, rb_emitter_desc* emitters, int32_t* has, rb_camera_desc* camera) {
	std::shared_ptr<scenes::scene> world;
	std::shared_ptr<cameras::camera> cam;
	if (!objects(s, world, cam)) return RB_ERR_INVALID_ARGUMENT;
	rb::adapter::exported_scene ex;
	rb_status st = rb::adapter::export_scene(*world, ex);
	if (st != RB_OK) return st;
	rb_bvh* bvh = nullptr;
	st = rb_bvh_build(&ex.desc, &bvh);
	if (st != RB_OK) return st;
	rb_bvh_desc d;
	rb_bvh_get(bvh, &d);
	*num_nodes = d.num_nodes;
	*num_prims = d.num_prims;
	if (nodes != nullptr) {
		std::memcpy(nodes, d.nodes, 8ull * d.num_nodes * sizeof(float));
		std::memcpy(prim_entity, d.prim_entity, d.num_prims * sizeof(uint32_t));
		std::memcpy(prim_index, d.prim_index, d.num_prims * sizeof(uint32_t));
		for (size_t e = 0; e < ex.entities.size(); e++) {
			const rb_entity_desc& ed = ex.entities[e];
			has[2 * e] = ed.material >= 0;
			has[2 * e + 1] = ed.emitter >= 0;
			if (ed.material >= 0) materials[e] = ex.materials[ed.material];
			if (ed.emitter >= 0) emitters[e] = ex.emitters[ed.emitter];
		}
		st = rb::adapter::export_camera(*cam, *camera);
	}
	rb_bvh_free(bvh);
	return st;
}

// The adapter's material list of a harness scene (sizes first with NULL
// arrays) and each entity's index into it (-1: none).
int adp_export_materials(orc_scene* s, rb_material_desc* materials, uint32_t* count, int32_t* entity_material,
	uint32_t* num_entities) {
	std::shared_ptr<scenes::scene> world;
	std::shared_ptr<cameras::camera> cam;
	if (!objects(s, world, cam)) return RB_ERR_INVALID_ARGUMENT;
	rb::adapter::exported_scene ex;
	const rb_status st = rb::adapter::export_scene(*world, ex);
	if (st != RB_OK) return st;
	*count = static_cast<uint32_t>(ex.materials.size());
	*num_entities = static_cast<uint32_t>(ex.entities.size());
	if (materials != nullptr) {
		for (size_t k = 0; k < ex.materials.size(); k++) materials[k] = ex.materials[k];
		for (size_t e = 0; e < ex.entities.size(); e++) entity_material[e] = ex.entities[e].material;
	}
	return RB_OK;
}

// Texture t of the adapter's export of a harness scene: its size (and the
// number of textures) first with rgb NULL, then its texels.
// desc (not NULL): the texture's description, its rgb pointer cleared.
int adp_export_texture(orc_scene* s, uint32_t t, float* rgb, uint32_t* width, uint32_t* height, uint32_t* count,
	rb_texture_desc* desc) {
	std::shared_ptr<scenes::scene> world;
	std::shared_ptr<cameras::camera> cam;
	if (!objects(s, world, cam)) return RB_ERR_INVALID_ARGUMENT;
	rb::adapter::exported_scene ex;
	const rb_status st = rb::adapter::export_scene(*world, ex);
	if (st != RB_OK) return st;
	*count = static_cast<uint32_t>(ex.textures.size());
	if (t >= ex.textures.size()) return RB_OK;
	*width = ex.textures[t].width;
	*height = ex.textures[t].height;
	if (desc != nullptr) {
		*desc = ex.textures[t];
		desc->rgb = nullptr;
	}
	if (rgb != nullptr && ex.textures[t].rgb != nullptr)
		std::memcpy(rgb, ex.textures[t].rgb, 3ull * *width * *height * sizeof(float));
	return RB_OK;
}

} // extern "C"
