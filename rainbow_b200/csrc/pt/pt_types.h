// Scene records, the PCG32 sampler stream and spectrum helpers of the
// wavefront path tracer. Host- and device-compilable.
#pragma once

#include "../rb_math.h"

#include <vector_types.h>  // float2 / float4 (CUDA headers, also usable from host C++)

#include <float.h>
#include <stdint.h>

namespace rb {
namespace pt {

using spectrum = vec3;  // RGB color_spectrum (rainbow-cpu/shared/spectrums/color_spectrum.cpp:58-70)

RB_HD bool is_black(spectrum s) { return s.x == 0.f && s.y == 0.f && s.z == 0.f; }
// coefficient_spectrum::max_component: m = max(m, c) with glm's max.
RB_HD float spectrum_max(spectrum s) { return fmax_ref(fmax_ref(s.x, s.y), s.z); }

// ------------------------------------------------------------------ PCG32
// pcg32 (rainbow-cpu/shared/random_generator.cpp:41-85): seed -> inc = seed << 1 | 1,
// state = 0, step, state += default state, step. XSH-RR output.
struct pcg32 {
	uint64_t state;
	uint64_t inc;
};
constexpr uint64_t kPcgDefaultState = 0x853c49e6748fea9bULL;
constexpr uint64_t kPcgMult = 0x5851f42d4c957f2dULL;

RB_HD uint32_t pcg_next(pcg32& g) {
	const uint64_t old = g.state;
	g.state = old * kPcgMult + g.inc;
	const uint32_t xs = static_cast<uint32_t>(((old >> 18u) ^ old) >> 27u);
	const uint32_t rot = static_cast<uint32_t>(old >> 59u);
	return (xs >> rot) | (xs << ((~rot + 1u) & 31u));
}
RB_HD pcg32 pcg_seed(uint64_t seed) {
	pcg32 g;
	g.state = 0u;
	g.inc = (seed << 1u) | 1u;
	pcg_next(g);
	g.state += kPcgDefaultState;
	pcg_next(g);
	return g;
}
// uniform_real: min(1 - eps, float(u32) * 2^-32), with std::min's (b < a) ? b : a.
RB_HD float pcg_real(pcg32& g) {
	const float v = static_cast<float>(pcg_next(g)) * 2.3283064365386963e-10f;
	const float one_minus_eps = 1.f - FLT_EPSILON;
	return (v < one_minus_eps) ? v : one_minus_eps;
}
RB_HD vec2 pcg_2d(pcg32& g) {
	const float a = pcg_real(g);
	const float b = pcg_real(g);
	return vec2{a, b};
}

// Seed of the stream of one (pixel, sample): pixel in bits 0-23, sample in
// bits 24-47, render seed in bits 48-62. The reference instead shares one
// stream across a 16x16 tile (sampler_integrator.cpp:94-96); per-sample streams
// make every sample independent of the launch order.
RB_HD uint64_t stream_seed(uint32_t pixel, uint32_t sample, uint32_t seed) {
	return static_cast<uint64_t>(pixel & 0xffffffu) | (static_cast<uint64_t>(sample & 0xffffffu) << 24) |
		(static_cast<uint64_t>(seed & 0x7fffu) << 48);
}

// ------------------------------------------------------------------ scene records
enum : uint32_t {
	ENT_HAS_SHAPE = 1u << 0,
	ENT_HAS_MATERIAL = 1u << 1,
	ENT_HAS_EMITTER = 1u << 2,
	ENT_VISIBLE = 1u << 3, // shape and material (entity::visible, entity.cpp:80-83)
	ENT_HAS_MEDIA = 1u << 4
};

struct entity_rec {
	float l2w[16];
	float w2l[16];
	int32_t mesh;
	int32_t material;
	int32_t emitter;      // index into the emitter table, -1 if none
	uint32_t flags;
	float area;           // shape_instance_properties::area (world-space area)
	int32_t media;        // index into the media table, -1 if none
	int32_t pad[2];
};

// homogeneous_medium (media/homogeneous_medium.cpp:7-11): sigma_t = sigma_a + sigma_s,
// Henyey-Greenstein asymmetry g.
struct medium_rec {
	vec3 sigma_s;
	vec3 sigma_t;
	float g;
	float pad;
};

// media(outside, inside) (media/medium.hpp:82-101): medium indices, -1 for vacuum.
struct media_rec {
	int32_t inside;
	int32_t outside;
};

enum : uint32_t {
	MESH_HAS_NORMALS = 1u << 0,
	MESH_HAS_TANGENTS = 1u << 1,
	MESH_HAS_UVS = 1u << 2,
	MESH_REVERSE = 1u << 3
};

struct mesh_rec {
	uint32_t vertex_offset;   // into the vertex arrays (in vertices)
	uint32_t index_offset;    // into the index array (in indices)
	uint32_t num_triangles;
	uint32_t flags;
};

enum : uint32_t { MAT_LAMBERT = 0, MAT_METAL = 1, MAT_GLASS_ROUGH = 2, MAT_GLASS_SMOOTH = 3, MAT_BLACK = 4, MAT_PLASTIC = 5,
	MAT_MIRROR = 6, MAT_SUBSTRATE = 7, MAT_OREN_NAYAR = 8, MAT_LAYERED = 9, MAT_MIXTURE = 10, MAT_TEXTURED = 11,
	MAT_SSS_EXIT = 12 };  // the exit point of a subsurface walk: one separable_bssrdf_reflection lobe

// Lobes of a layered material (uber, translucent) or of a mixture: at most
// kMaxLayeredLobes.
constexpr uint32_t kMaxLayeredLobes = 6;

struct material_rec {
	uint32_t kind;
	float alpha_x, alpha_y;   // Trowbridge-Reitz alphas (roughness_to_alpha applied on the host);
	                          // Oren-Nayar (matte with sigma != 0): its A and B
	float eta;                // glass / plastic IOR
	spectrum diffuse;         // lambert reflectance (matte, plastic Kd)
	spectrum reflectance;     // glass reflectance, plastic Ks, mirror reflectance; metal: the
	                          // microfacet reflection's scale (1, or a mixture's weight)
	spectrum transmission;    // glass transmission
	spectrum cond_eta;        // conductor eta
	spectrum cond_k;          // conductor k
	uint32_t has_reflect;     // glass: reflectance not black
	uint32_t has_transmit;    // glass: transmission not black
	// layered materials (MAT_LAYERED: uber, translucent), whose lobe list is
	// built on the host: the lobe kinds (4 bits each) and scattering types (5
	// bits each) in collection order, their count, each lobe's spectrum and the
	// outer IOR of its specular transmission, and the collection's eta (eta is
	// the IOR of the dielectric Fresnel of its reflection lobes)
	uint32_t lobe_kinds, lobe_types, lobe_count;
	float collection_eta;
	spectrum lobe_r[kMaxLayeredLobes];
	float lobe_eta[kMaxLayeredLobes];
	// mixtures (MAT_MIXTURE): the lobe list of both components in order, each
	// lobe a lobe of a component record built with the mixture's weight on the
	// host: (record offset from this record << 4) | the lobe's index there
	uint32_t lobe_ref[kMaxLayeredLobes];
	spectrum blend_scale;     // substrate: the Fresnel-blend layer's scale (1, or a mixture's weight)
	// MAT_TEXTURED: a material with image-textured spectra, built at every hit
	// from material_src[src] and its textures at the hit's uv
	uint32_t src;
	// subsurface (a glass-kind record with a BSSRDF): the normalized-diffusion
	// profile's A (diffuse) and d (mfp / s(A)) per channel; eta is the IOR
	uint32_t sss;
	spectrum sss_a, sss_d;
};

// Textured parameters of a material: the spectra diffuse, reflectance,
// transmission, specular, opacity, the reals roughness u and v, IOR and
// Oren-Nayar sigma (channel 0 of a texture), then the spectra conductor eta
// and k and the subsurface mean free path.
enum : uint32_t { TEX_DIFFUSE = 0, TEX_REFLECTANCE = 1, TEX_TRANSMISSION = 2, TEX_SPECULAR = 3, TEX_OPACITY = 4,
	TEX_ROUGHNESS_U = 5, TEX_ROUGHNESS_V = 6, TEX_IOR = 7, TEX_SIGMA = 8, TEX_ETA = 9, TEX_K = 10, TEX_MFP = 11,
	kNumTexSlots = 12 };

// A material's parameters with what only the host computes already applied
// (roughness_to_alpha, Oren-Nayar's A and B), from which its record is built
// (pt_material.h): once on the host for constant textures, at every hit for
// image-textured spectra.
struct material_src {
	uint32_t kind;            // RB_MATERIAL_* of its description
	float alpha_x, alpha_y;   // Trowbridge-Reitz alphas (metal, rough glass, plastic, substrate, uber, translucent)
	float ior;                // glass, plastic, uber
	uint32_t smooth;          // glass: both roughnesses 0 (Fresnel-specular)
	uint32_t oren_nayar;      // matte: sigma != 0
	float on_a, on_b;         // matte: Oren-Nayar's A and B
	spectrum diffuse, reflectance, transmission, specular, opacity;
	spectrum cond_eta, cond_k;
	spectrum mfp;             // subsurface: mean free path
	float roughness_u, roughness_v, sigma;  // the description's reals, from which the fields above derive
	uint32_t remap;           // roughness_to_alpha applies
	uint32_t tex[kNumTexSlots];  // 0: the constant above; k > 0: texture k - 1 of the scene
};

enum : uint32_t { TEXK_IMAGE = 0, TEXK_SCALE = 1, TEXK_MIXTURE = 2 };

// A texture: an RGB image (texels row-major, (x, y) at texels[offset + 3 (y
// width + x)]), or a scale / mixture of inputs that are images (inputs[i] =
// image index + 1) or constants (inputs[i] = 0: constants[i]).
struct texture_rec {
	uint32_t kind;
	uint32_t offset;          // image: in floats
	uint32_t width, height;
	uint32_t inputs[3];
	spectrum constants[3];
};

enum : uint32_t { EMIT_SURFACE = 0, EMIT_ENVIRONMENT = 1 };

struct emitter_rec {
	uint32_t kind;
	int32_t entity;           // owning entity ordinal
	spectrum radiance;        // surface radiance / environment intensity
	float radius;             // environment radius
};

// 2x2 piecewise-constant distribution of a constant environment map
// (environment_light.cpp:20-36, distribution.hpp:48-141), precomputed on the host.
struct env_distribution {
	float cdf_row[2][3];      // conditional CDFs of the two rows
	float value_row[2][2];
	float integral_row[2];
	float cdf_marg[3];        // marginal CDF
	float value_marg[2];
	float integral_marg;
};

// Interior node of the 4-wide traversal tree (128 bytes): binary node N of the
// reference's tree with its grandchildren as slots [L0, L1, R0, R1] (L, R: N's
// left and right child; X0, X1: X's left and right child). A child that is a
// leaf takes its pair's first slot itself and leaves the second one empty.
// Boxes are stored per coordinate, one float4 across the four slots.
// Slot reference: interior -> its index in this array; leaf ->
// kRefLeaf | count << 24 | first prim slot (count 1..127, slot < 2^24).
struct node4 {
	float4 lo_x, lo_y, lo_z;
	float4 hi_x, hi_y, hi_z;
	uint4 ref;
	uint4 meta;  // x: split axis of N (bits 0-1), of L (bits 2-3), of R (bits 4-5); valid slots (bits 8-11)
};
constexpr uint32_t kRefLeaf = 0x80000000u;

// Flat view of an uploaded scene; pointers are device pointers in kernels and
// host pointers in host-side use.
struct scene_view {
	const node4* wnodes;          // 4-wide nodes (fast traversal); null: the reference-order traversal only
	float4 root_a, root_b;        // root box, (min.xyz, max.x), (max.y, max.z, -, -)
	uint32_t root_ref;
	uint32_t root_node;           // index of the root in `nodes` (non-zero for a scene of a merged batch)
	const float4* nodes;          // 2 per node: (min.xyz, max.x), (max.y, max.z, w0, w1)
	const float4* tri_a;          // per prim slot: (p0.xyz, e1.x)        entity-local space
	const float4* tri_b;          // (e1.y, e1.z, e2.x, e2.y)
	const float2* tri_c;          // (e2.z, entity as bits)
	const uint32_t* prim_index;   // triangle index within its mesh
	const entity_rec* entities;
	const mesh_rec* meshes;
	const float* positions;       // 3 per vertex
	const float* normals;
	const float* tangents;
	const float* uvs;
	const uint32_t* indices;
	const material_rec* materials;
	const emitter_rec* emitters;  // scene->emitters() order
	const int32_t* environments;  // emitter indices of the environment emitters
	env_distribution env;
	uint32_t num_nodes;
	uint32_t num_emitters;
	uint32_t num_environments;
	uint32_t num_entities;
	const medium_rec* mediums;
	const media_rec* media;
	uint32_t num_media;
	uint32_t instances;           // non-zero: some prim slots hold a whole entity walked in its mesh's own tree
	const float* sss_table;             // the normalized-diffusion inverse CDF (kSssTableSize knots), or null
	uint32_t sss;                       // non-zero: some material has a BSSRDF
	uint32_t pad3;
	const material_src* material_srcs;  // parameters of the MAT_TEXTURED records
	const texture_rec* textures;
	const float* texels;
	uint32_t num_textures;
	uint32_t pad2;
};

} // namespace pt
} // namespace rb
