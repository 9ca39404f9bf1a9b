// Reference scene and camera -> rb_scene_desc / rb_camera_desc (include/rbgpu.h).
//
// The C++ side of the drop-in: reads a rainbow `scene` (rainbow-cpu/scenes/scene.hpp)
// and its `perspective_camera` and describes them to the C ABI. Compiled against
// the reference's own headers (the include root is the reference checkout).
//
// Supported, as the wavefront core renders them: triangle meshes without alpha
// masks; matte, metal, glass, plastic, mirror, substrate, uber, translucent and
// mixture materials with constant textures, and RGB image textures for their
// spectra (not inside a mixture); surface lights and constant environment
// lights; homogeneous media. Anything else returns RB_ERR_UNSUPPORTED, so a caller can
// fall back to the reference integrator for that scene.
#pragma once

#include "../../include/rbgpu.h"

#include "rainbow-cpu/cameras/camera.hpp"
#include "rainbow-cpu/scenes/scene.hpp"

#include <memory>
#include <vector>

namespace rb {
namespace adapter {

// An rb_scene_desc with the arrays it points into.
struct exported_scene {
	std::vector<std::vector<float>> positions, normals, tangents, uvs;
	std::vector<std::vector<uint32_t>> indices;
	std::vector<rb_mesh_desc> meshes;
	std::vector<rb_entity_desc> entities;
	std::vector<rb_material_desc> materials;
	std::vector<rb_emitter_desc> emitters;
	std::vector<rb_medium_desc> mediums;
	std::vector<rb_media_desc> media;
	std::vector<std::vector<float>> texels;
	std::vector<rb_texture_desc> textures;
	rb_scene_desc desc{};  // valid while this object lives and is not copied
};

// Entities in the scene's order; meshes, materials and mediums shared by
// pointer stay shared (so a mesh used by several entities keeps the
// reference's two-level tree).
rb_status export_scene(const rainbow::cpus::scenes::scene& s, exported_scene& out);

// A perspective_camera's raster-to-camera and camera-to-world matrices, lens,
// focus and film resolution.
rb_status export_camera(const rainbow::cpus::cameras::camera& c, rb_camera_desc& out);

} // namespace adapter
} // namespace rb
