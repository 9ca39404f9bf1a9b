/*
 * rbgpu.h - C ABI of the B200 wavefront path-tracing core (librbgpu.so).
 *
 * The core is a drop-in for the unidirectional path integrator of the C++
 * renderer LinkClinton/rainbow. The reference has no C ABI: its extension
 * point is the C++ class `integrator` (rainbow-cpu/integrators/integrator.hpp:58-71)
 * and `path_integrator(sampler2d, sampler1d, max_depth = 5, threshold = 1)`
 * (rainbow-cpu/integrators/path_integrator.hpp:9-12). Each entry point below
 * names the reference interface whose work it takes over. A C++ adapter class
 * deriving from `integrator` exports the reference scene into these structures
 * and writes the result back through film::set_pixel (rainbow-cpu/cameras/film.cpp:202-205).
 *
 * Conventions
 *  - Every call returns rb_status; no exception crosses this boundary.
 *  - Matrices are 4x4 float, column-major, element (row r, column c) at [c * 4 + r]
 *    (the glm layout the reference uses, rainbow-core/math/matrix4x4.hpp:15).
 *  - Vectors are float triples. Colours are linear RGB (the reference's
 *    color_spectrum, rainbow-cpu/shared/spectrums/color_spectrum.cpp:58-70).
 *  - Host pointers passed in are read during the call only and never retained.
 *  - One host thread per context; calls on one context are serialised.
 */
#ifndef RBGPU_H
#define RBGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RBGPU_ABI_VERSION 10

/* ------------------------------------------------------------------ status */
typedef int32_t rb_status;
enum {
	RB_OK = 0,
	RB_ERR_INVALID_ARGUMENT = 1,
	RB_ERR_CUDA = 2,             /* a CUDA runtime call failed */
	RB_ERR_OUT_OF_MEMORY = 3,
	RB_ERR_NO_SCENE = 4,         /* render/trace before rb_scene_upload */
	RB_ERR_STACK_OVERFLOW = 5,   /* device traversal stack limit reached (reported, never trapped) */
	RB_ERR_QUEUE_OVERFLOW = 6,   /* a wavefront queue exceeded its capacity */
	RB_ERR_UNSUPPORTED = 7,      /* scene feature outside the supported subset */
	RB_ERR_IO = 8,               /* checkpoint file could not be read or written */
	RB_ERR_CHECKPOINT = 9,       /* checkpoint does not match the context */
	RB_ERR_DEVICE_TIMEOUT = 10,  /* a bounded device wait gave up */
	RB_ERR_NO_DEVICE = 11,       /* no CUDA device is visible */
	RB_ERR_TOO_LARGE = 12        /* more work than rb_render_noalloc's fixed scratch holds */
};

/* Human-readable name of a status code. Never NULL. */
const char* rb_status_string(rb_status status);

/* ------------------------------------------------------------------ scene description */

/* Indexed triangle mesh. Replaces rainbow-cpu/shapes/mesh.hpp:16-108
 * (mesh(positions, tangents, normals, uvs, indices, reverse_orientation)).
 * uvs are triples because the reference stores them as vector3. */
typedef struct rb_mesh_desc {
	const float* positions;     /* 3 * num_vertices, local space */
	const float* normals;       /* 3 * num_vertices or NULL */
	const float* tangents;      /* 3 * num_vertices or NULL */
	const float* uvs;           /* 3 * num_vertices or NULL (defaults (0,0),(1,0),(1,1) per face) */
	const uint32_t* indices;    /* 3 * num_triangles */
	uint32_t num_vertices;
	uint32_t num_triangles;
	int32_t reverse_orientation;
	int32_t reserved;
} rb_mesh_desc;

enum {
	RB_MATERIAL_MATTE = 0,  /* rainbow-cpu/materials/matte_material.cpp:13-29 (Lambert when sigma == 0, else
	                           Oren-Nayar, scatterings/reflection/oren_nayar_reflection.cpp) */
	RB_MATERIAL_METAL = 1,  /* rainbow-cpu/materials/metal_material.cpp:17-37 */
	RB_MATERIAL_GLASS = 2,  /* rainbow-cpu/materials/glass_material.cpp:25-64 */
	RB_MATERIAL_PLASTIC = 3, /* rainbow-cpu/materials/plastic_material.cpp:9-55: diffuse = Kd (Lambert lobe),
	                            reflectance = Ks (Trowbridge-Reitz reflection with a dielectric Fresnel
	                            of ior, 1.49 in the reference's default constructor), roughness_u the
	                            isotropic roughness */
	RB_MATERIAL_MIRROR = 4,  /* rainbow-cpu/materials/mirror_material.cpp:9-26: reflectance (specular
	                            reflection, no Fresnel term) */
	RB_MATERIAL_SUBSTRATE = 5, /* rainbow-cpu/materials/substrate_material.cpp: the Fresnel-blend
	                            layer (scatterings/reflection/fresnel_blend_reflection.cpp) of
	                            reflectance = specular Rs over diffuse = Rd, Trowbridge-Reitz
	                            roughness_u / roughness_v */
	RB_MATERIAL_UBER = 6,    /* rainbow-cpu/materials/uber_material.cpp:26-75: with O = opacity, the lobes
	                            specular transmission of clamp(1 - O) (eta 1 / 1), Lambert of O diffuse,
	                            Trowbridge-Reitz reflection of O specular (dielectric Fresnel of ior,
	                            roughness_u / roughness_v), specular reflection of O reflectance
	                            (dielectric Fresnel of ior) and specular transmission of
	                            O transmission (eta 1 / ior), each if not black */
	RB_MATERIAL_TRANSLUCENT = 7, /* rainbow-cpu/materials/translucent_material.cpp:23-69: IOR 1.5; no lobes
	                            when reflectance and transmission are both black; else Lambert
	                            reflection of diffuse reflectance and Lambert transmission of diffuse
	                            transmission (if diffuse is not black), Trowbridge-Reitz reflection of
	                            specular reflectance and transmission of specular transmission (if
	                            specular is not black), isotropic roughness_u */
	RB_MATERIAL_SUBSURFACE = 9, /* rainbow-cpu/materials/subsurface_material.cpp:24-66: glass lobes of
	                            reflectance / transmission (Fresnel-specular when both roughnesses are
	                            0, else Trowbridge-Reitz reflection and transmission, IOR ior) and a
	                            normalized-diffusion BSSRDF (scatterings/bssrdf/normalized_diffusion.cpp)
	                            of albedo diffuse and mean free path mfp; nothing when reflectance or
	                            transmission is black, and nothing inside a mixture. Plain path tracing
	                            and direct lighting only (guided and volume renders return
	                            RB_ERR_UNSUPPORTED) */
	RB_MATERIAL_MIXTURE = 8  /* rainbow-cpu/materials/mixture_material.cpp:13-43: the lobes of material
	                            components[0] built with the weight amount and of components[1] with
	                            clamp(1 - amount), each by its material's build with a scale (mixtures
	                            nest up to 8 deep; at most 6 lobes in all, else RB_ERR_UNSUPPORTED) */
};

enum {
	RB_TEXTURE_IMAGE = 0,    /* image_texture_t<2, spectrum> (textures/detail/image_texture.hpp) */
	RB_TEXTURE_SCALE = 1,    /* scale_texture_t<2, spectrum> (textures/detail/scale_texture.hpp):
	                            base * scale, inputs[0] the scale, inputs[1] the base */
	RB_TEXTURE_MIXTURE = 2   /* mixture_texture_t<2, spectrum> (textures/detail/mixture_texture.hpp):
	                            t0 a + t1 clamp(1 - a) with a = clamp(alpha) to [0, 1]; inputs[0] t0,
	                            inputs[1] t1, inputs[2] alpha (a real texture: channel 0). Like the
	                            reference, it samples its inputs at the hit point's world x and y */
};

/* A texture for a material's spectrum. RB_TEXTURE_IMAGE: width * height RGB
 * texels, row-major, texel (x, y) at rgb[3 * (y * width + x)], sampled at a
 * hit's uv (the triangle's vertex uvs, or (0, 0), (1, 0), (1, 1) without them)
 * with the uv wrapped to [0, 1) and bilinear filtering between the four nearest
 * texels. RB_TEXTURE_SCALE / MIXTURE combine inputs: inputs[i] = k > 0 is
 * texture k - 1 (an image), 0 the constant constants[i]. */
typedef struct rb_texture_desc {
	const float* rgb;
	uint32_t width;
	uint32_t height;
	uint32_t kind;
	uint32_t inputs[3];
	float constants[3][3];
} rb_texture_desc;

/* Material parameters: constant textures (constant_texture_t,
 * textures/detail/constant_texture.hpp:25-35), and for the spectra named by the
 * *_texture fields image textures instead. */
typedef struct rb_material_desc {
	uint32_t kind;
	int32_t remap_roughness;    /* metal/glass: apply trowbridge_reitz_distribution::roughness_to_alpha */
	float diffuse[3];           /* matte */
	float sigma;                /* matte: Oren-Nayar sigma in degrees, clamped to [0, 90]; 0 gives Lambert */
	float eta[3];               /* metal: conductor eta (RGB) */
	float k[3];                 /* metal: conductor absorption k (RGB) */
	float reflectance[3];       /* glass, plastic, mirror, substrate, uber, translucent */
	float transmission[3];      /* glass, uber, translucent */
	float ior;                  /* glass, plastic, uber */
	float roughness_u;          /* metal, glass (glass with both zero -> fresnel_specular) */
	float roughness_v;
	float specular[3];          /* uber, translucent: the glossy reflection's spectrum */
	float opacity[3];           /* uber */
	int32_t components[2];      /* mixture: indices of its two materials in rb_scene_desc.materials */
	float amount[3];            /* mixture: the weight of components[0] (mixture_material's alpha) */
	/* 0: the constant spectrum above; k > 0: image texture rb_scene_desc.textures[k - 1] instead
	 * (for the spectra the material reads; not inside a mixture) */
	uint32_t diffuse_texture;
	uint32_t reflectance_texture;
	uint32_t transmission_texture;
	uint32_t specular_texture;
	uint32_t opacity_texture;
	float mfp[3];               /* subsurface: mean free path (RGB) */
	/* real parameters from textures: 0 the constant above; k > 0: channel 0 of
	 * texture rb_scene_desc.textures[k - 1] (an image_texture2d<real>, or a scale /
	 * mixture texture of real images and constants; not inside a mixture);
	 * roughness_to_alpha, the smooth-glass test and Oren-Nayar's A and B then
	 * follow the texel at every hit */
	uint32_t roughness_u_texture;
	uint32_t roughness_v_texture;
	uint32_t ior_texture;
	uint32_t sigma_texture;
	/* spectra from textures, as the *_texture fields above: metal eta and k, subsurface mfp */
	uint32_t eta_texture;
	uint32_t k_texture;
	uint32_t mfp_texture;
} rb_material_desc;

enum {
	RB_EMITTER_SURFACE = 0,      /* rainbow-cpu/emitters/surface_light.cpp (one-sided on the geometric normal) */
	RB_EMITTER_ENVIRONMENT = 1   /* rainbow-cpu/emitters/environment_light.cpp with a constant map of 1 */
};

/* Homogeneous participating medium: rainbow-cpu/media/homogeneous_medium.cpp:7-58
 * (homogeneous_medium(sigma_a, sigma_s, g)) with the Henyey-Greenstein phase
 * function of asymmetry g (shared/phases/henyey_greenstein.cpp). */
typedef struct rb_medium_desc {
	float sigma_a[3];
	float sigma_s[3];
	float g;
	uint32_t reserved;
} rb_medium_desc;

/* The media component of an entity: media(outside, inside) (media/medium.hpp:82-101),
 * indices into rb_scene_desc.mediums, -1 for vacuum. A ray leaving a surface
 * of the entity along +normal continues in `outside`, otherwise in `inside`. */
typedef struct rb_media_desc {
	int32_t inside;
	int32_t outside;
} rb_media_desc;

typedef struct rb_emitter_desc {
	uint32_t kind;
	float radiance[3];          /* surface radiance, or environment intensity */
	float radius;               /* environment: the radius passed to environment_light(intensity, radius) */
} rb_emitter_desc;

/* One scene entity: rainbow-cpu/scenes/entity.hpp:22-70,
 * entity(material, emitter, shape, media, transform). -1 means the component is absent.
 * An entity without a material is invisible (entity.cpp:80-83). */
typedef struct rb_entity_desc {
	int32_t mesh;
	int32_t material;
	int32_t emitter;
	int32_t medium;             /* index of the entity's media component (rb_media_desc), -1: none */
	float local_to_world[16];
	float world_to_local[16];
} rb_entity_desc;

/* Flattened binary BVH over (entity, triangle) leaves, the layout of the
 * reference's bounding_volume_hierarchy<entity_reference>
 * (rainbow-cpu/shared/accelerators/bounding_volume_hierarchy.hpp:45-80) in preorder.
 * Node i is 8 words: min.xyz, max.xyz (float), then w0, w1 (uint32 bit patterns):
 *   interior: left child = i + 1, w0 = right child index, w1 = split axis (0..2)
 *   leaf:     w0 = first prim slot, w1 = RB_BVH_LEAF_FLAG | count
 * Prim slot s refers to triangle prim_index[s] of entity prim_entity[s], or,
 * when prim_index[s] is RB_BVH_ALL_TRIANGLES, to the whole entity: its mesh has
 * a tree of its own in local space (the reference's two-level case,
 * scene::build_accelerator, scene.cpp:41-75, for a mesh used by several
 * entities or with more than 2^17 triangles; rb_bvh_get_mesh_tree). */
#define RB_BVH_LEAF_FLAG 0x80000000u
#define RB_BVH_ALL_TRIANGLES 0xffffffffu
typedef struct rb_bvh_desc {
	const float* nodes;         /* 8 * num_nodes words */
	uint32_t num_nodes;
	uint32_t num_prims;
	const uint32_t* prim_entity;
	const uint32_t* prim_index;
} rb_bvh_desc;

/* Scene: rainbow-cpu/scenes/scene.hpp:24-44. Entities are kept in add order;
 * the emitter list is the entities with an emitter, in that order
 * (scene::add_entity, scene.cpp:16-28). */
typedef struct rb_scene_desc {
	const rb_mesh_desc* meshes;
	uint32_t num_meshes;
	uint32_t num_entities;
	const rb_entity_desc* entities;
	const rb_material_desc* materials;
	uint32_t num_materials;
	uint32_t num_emitters;
	const rb_emitter_desc* emitters;
	rb_bvh_desc bvh;            /* num_nodes == 0: rb_scene_upload builds it (rb_bvh_build); a supplied
	                               tree's RB_BVH_ALL_TRIANGLES prims get their mesh trees built */
	const rb_medium_desc* mediums;
	uint32_t num_mediums;
	uint32_t num_media;
	const rb_media_desc* media;
	const rb_texture_desc* textures;  /* image textures that materials refer to (*_texture fields) */
	uint32_t num_textures;
	uint32_t reserved;
} rb_scene_desc;

/* Pinhole / thin-lens perspective camera: rainbow-cpu/cameras/perspective_camera.cpp:78-99.
 * raster_to_camera is projective_camera::mRasterToCamera (camera.cpp:21-52),
 * camera_to_world is camera::mCameraToWorld. The eye/target/up/fov fields
 * record how the matrices were made; the kernels read only the matrices. */
typedef struct rb_camera_desc {
	float raster_to_camera[16];
	float camera_to_world[16];
	float eye[3];
	float target[3];
	float up[3];
	float fov_degrees;
	float lens_radius;          /* 0: pinhole */
	float focus_distance;
	int32_t width;
	int32_t height;
} rb_camera_desc;

/* ------------------------------------------------------------------ rays and hits */

/* A reference `ray` (rainbow-cpu/shared/ray.hpp:13-28): direction as the ray
 * holds it (the constructor normalises it), origin, and the current length. */
typedef struct rb_ray {
	float origin[3];
	float direction[3];
	float length;
} rb_ray;

/* Closest hit: entity ordinal and triangle index within the entity's mesh
 * (-1, -1 on a miss), world ray length after the hit (the value the reference
 * leaves in ray.length), and the barycentrics b1, b2 of the hit triangle. */
typedef struct rb_hit {
	int32_t entity;
	int32_t triangle;
	float t;
	float b1;
	float b2;
} rb_hit;

/* ------------------------------------------------------------------ context */
typedef struct rb_context rb_context;

/* Create a context on CUDA device `device`. Replaces nothing in the reference
 * (which has no device); holds device memory, streams and captured graphs. */
rb_status rb_context_create(rb_context** out, int device);
rb_status rb_context_destroy(rb_context* ctx);

/* Upload a scene (copied; the caller keeps ownership of the description).
 * Replaces scene::build_accelerator (rainbow-cpu/scenes/scene.cpp:30-80): when
 * desc->bvh.num_nodes == 0 the tree is built with the reference's rules. */
rb_status rb_scene_upload(rb_context* ctx, const rb_scene_desc* desc);

/* Closest hit of each ray over all entities: scene::intersect (scene.cpp:82-95). */
rb_status rb_trace_closest(rb_context* ctx, const rb_ray* rays, uint32_t count, rb_hit* hits);
/* Closest hit over visible entities only: scene::intersect_with_shadow_ray (scene.cpp:97-112). */
rb_status rb_trace_shadow(rb_context* ctx, const rb_ray* rays, uint32_t count, rb_hit* hits);
/* Same as the two calls above on device-resident arrays, enqueued on `stream`
 * (a cudaStream_t, NULL for the context's stream); returns once enqueued. */
rb_status rb_trace_closest_device(rb_context* ctx, const rb_ray* d_rays, uint32_t count, rb_hit* d_hits, void* stream);
rb_status rb_trace_shadow_device(rb_context* ctx, const rb_ray* d_rays, uint32_t count, rb_hit* d_hits, void* stream);

/* ------------------------------------------------------------------ rendering */
enum {
	RB_RENDER_RESET = 1u << 0,     /* clear the film accumulators before adding these samples */
	RB_RENDER_GUIDE = 1u << 1,     /* learned guiding: sample path continuations from the guide (below) */
	RB_RENDER_TRAIN = 1u << 2,     /* learned guiding: collect training samples and train after every wave */
	RB_RENDER_VOLUME = 1u << 3,    /* volume_path_integrator::trace (volume_path_integrator.cpp:13-79) instead
	                                  of path_integrator::trace: free-flight sampling in the media of the
	                                  path, Henyey-Greenstein scattering, transmittance on every light
	                                  connection; with learned guiding, medium vertices use a second
	                                  guide network (rb_guide_medium_stats_get) */
	RB_RENDER_DIRECT = 1u << 4     /* direct_integrator::trace (direct_integrator.cpp:20-127) instead of
	                                  path_integrator::trace: at the first visible surface, light samples
	                                  and BSDF samples combined by the power heuristic (direct_samples
	                                  below); max_depth and rr_threshold are unused; not combined with
	                                  RB_RENDER_GUIDE, RB_RENDER_TRAIN or RB_RENDER_VOLUME */
};

/* One render call: path_integrator::trace (rainbow-cpu/integrators/path_integrator.cpp:15-47)
 * for samples [first_sample, first_sample + spp) of every pixel, driven the way
 * sampler_integrator::render (sampler_integrator.cpp:19-144) drives it, with one
 * PCG32 stream per (pixel, sample) instead of one per 16x16 tile. */
typedef struct rb_render_params {
	rb_camera_desc camera;
	uint32_t spp;
	uint32_t first_sample;
	uint32_t max_depth;         /* reference default 5 */
	float rr_threshold;         /* reference default 1 */
	uint32_t seed;              /* mixed into every per-sample stream (15 bits used) */
	uint32_t flags;             /* RB_RENDER_* */
	uint32_t paths_per_wave;    /* 0: library default */
	uint32_t direct_samples;    /* RB_RENDER_DIRECT: emitter samples in bits 0-15, BSDF samples in bits
	                               16-31 (direct_integrator(sampler2d, sampler1d, emitter_samples,
	                               bsdf_samples), direct_integrator.hpp:9-13); 0: the reference's
	                               defaults, 4 and 4; both must be non-zero otherwise */
} rb_render_params;

/* Render and write the per-pixel mean radiance (box filter, film::add_tile +
 * pixel::spectrum, film.cpp:11-21,207-223) of everything accumulated since the
 * last reset into rgb_out (caller-owned, width * height * 3 floats, row-major,
 * pixel (x, y) at (y * width + x) * 3). rgb_out may be NULL. When rgb_out is
 * page-locked memory, each slice of it is copied as soon as its pixels have all
 * of the call's samples, while later waves still run; if the call then fails,
 * part of rgb_out may already be written. */
rb_status rb_render(rb_context* ctx, const rb_render_params* params, float* rgb_out);

/* rb_render without waiting: returns once the call's work is enqueued, so that
 * consecutive calls overlap on the GPU (the late bounces of one call with the
 * first waves of the next: the calls' waves take the wave lanes in turn, so a
 * call of one wave runs beside the previous call) while the film still adds
 * their samples in call order. No counterpart in the reference, whose render() is
 * synchronous. Plain path tracing only: flags other than RB_RENDER_RESET return
 * RB_ERR_UNSUPPORTED. rgb_out, if not NULL, must be page-locked; its slices are
 * written as the call's pixels complete, and it must not be read or reused
 * before rb_render_wait. A call whose camera, spp, max_depth, rr_threshold or
 * paths_per_wave differs from the pending calls', or that sets RB_RENDER_RESET,
 * first waits for them; so does every other entry point on the context.
 * rb_render_wait returns once every pending call has finished, with the first
 * device error of any of them; rb_render_stats_get then covers all of them
 * (samples, rays, elapsed time from the first call's start). */
rb_status rb_render_async(rb_context* ctx, const rb_render_params* params, float* rgb_out);
rb_status rb_render_wait(rb_context* ctx);

/* Read back the accumulators: per-pixel sums of radiance (double, 3 per pixel),
 * of squared radiance (double, 3 per pixel) and the sample count per pixel.
 * Any output may be NULL. */
rb_status rb_film_read(rb_context* ctx, double* sum_rgb, double* sum_sq_rgb, uint32_t* sample_count);

/* The film accumulators (layout as rb_film_read) copied to, or replaced from,
 * device memory the caller owns, enqueued on `stream` (a cudaStream_t, NULL: the
 * context's stream). No counterpart in the reference, which renders on one
 * machine. For renders over several GPUs: every rank's context renders its own
 * range of sample indices of the same image, copies its film out, the ranks sum
 * the buffers (an all-reduce, e.g. NCCL over NVLink), and each copies the sums
 * back, after which its film holds the union of the ranges.
 * rb_film_to_device returns once the copies are enqueued (after the context's
 * own pending work); rb_film_from_device waits for its copies, needs the film
 * of the same size to exist (a render made it) and records samples_per_pixel as
 * the film's sample count. */
rb_status rb_film_to_device(rb_context* ctx, double* d_sum_rgb, double* d_sum_sq_rgb, uint32_t* d_count, void* stream);
rb_status rb_film_from_device(rb_context* ctx, const double* d_sum_rgb, const double* d_sum_sq_rgb, const uint32_t* d_count,
	uint64_t samples_per_pixel, void* stream);

/* Render without allocating: for callers that must not call cudaMalloc at
 * render time (code that runs inside a framework which owns the device memory
 * pool, or a real-time loop where an allocation's implicit synchronisation is
 * not allowed). No counterpart in the reference, which has no device.
 * The plain path integrator only: the same work as rb_render without flags for
 * samples [first_sample, first_sample + spp) of every pixel (scenes with
 * invisible entities included: paths keep bouncing past max_depth until done,
 * with a host read of the active count between those bounces). Any flag but
 * RB_RENDER_RESET returns RB_ERR_UNSUPPORTED; RESET clears the caller's
 * accumulators first. All per-path state, queues and counters live in one
 * static device array of RB_NOALLOC_SCRATCH_BYTES that every GPU loading the
 * library keeps until exit; at most RB_NOALLOC_MAX_PATHS = width * height * spp
 * paths per call (larger requests return RB_ERR_TOO_LARGE). Results are ADDED
 * to the caller's device accumulators d_sum_rgb / d_sum_sq_rgb (3 doubles per
 * pixel) and d_count (one uint32 per pixel), which the caller zeroes before the
 * first call (or clears with RB_RENDER_RESET). The scene must have been
 * uploaded with rb_scene_upload beforehand. The first call on a device looks up
 * the scratch array's device address, so make it before any stream capture.
 * Every call shares the one scratch array: calls that overlap on the GPU (other
 * streams, other threads) race, so serialise them; the call also reads its
 * counters through the context's page-locked buffer, so serialise it with every
 * other call on the same context too. `stream` is a cudaStream_t (NULL: the
 * context's stream); the call waits for its work to finish and returns the
 * first device error, if any. */
#define RB_NOALLOC_MAX_PATHS 16384u
#define RB_NOALLOC_SCRATCH_BYTES (8u << 20)
rb_status rb_render_noalloc(rb_context* ctx, const rb_render_params* params, double* d_sum_rgb, double* d_sum_sq_rgb,
	uint32_t* d_count, void* stream);

/* Stochastic progressive photon mapping:
 * photon_mapping_integrator(sampler2d, sampler1d, iterations, max_depth,
 * photons, radius)::render (rainbow-cpu/integrators/photon_mapping_integrator.hpp:9-13,
 * photon_mapping_integrator.cpp:386-560). Each iteration traces a visible point
 * per pixel, hashes the visible points' search spheres into a grid, traces
 * `photons` photons (0: one per pixel) that deposit flux at the visible points
 * they land near, and shrinks each pixel's radius by the photons it received.
 * The image (W * H * 3 floats into rgb_out, host memory) is the reference's
 * film value: L / iterations + tau / (iterations * photons * pi * r^2). Each
 * pixel and each photon draws from its own PCG32 stream (pixel, iteration,
 * seed) / (photon, iteration, seed), where the reference shares one stream per
 * 16 x 16 tile and per chunk of 8192 photons. Media and BSSRDFs are ignored, as
 * in the reference. The call allocates its buffers (about 270 bytes per pixel),
 * waits for its work and returns the first device error, if any. */
typedef struct rb_photon_params {
	rb_camera_desc camera;
	uint32_t iterations;  /* 1 .. 65535 (the reference's default: 64) */
	uint32_t max_depth;   /* 1 .. 64 (5) */
	uint32_t photons;     /* per iteration; 0: width * height (the reference's default) */
	float radius;         /* initial search radius (1) */
	uint32_t seed;        /* stream seed, 14 bits */
	uint32_t reserved;
} rb_photon_params;
rb_status rb_render_photons(rb_context* ctx, const rb_photon_params* params, float* rgb_out);

/* Counters of the last rb_render call. */
typedef struct rb_render_stats {
	uint64_t samples;
	uint64_t extend_rays;       /* closest-hit rays of the path (one per bounce) */
	uint64_t shadow_rays;       /* NEE shadow rays */
	uint64_t mis_rays;          /* BSDF-sampled emitter-search rays of the MIS step */
	uint64_t node_visits;       /* box tests (filled only when counting is enabled) */
	uint64_t triangle_tests;    /* (filled only when counting is enabled) */
	uint32_t device_error;      /* rb_status raised inside a kernel, RB_OK if none */
	uint32_t kernel_launches;
	float elapsed_ms;           /* device time of the call, CUDA events */
	float extend_ms;            /* device time of the extend (closest-hit) launches */
	float secondary_ms;         /* device time of the shadow / MIS traversal launches */
	uint32_t extend_launches;   /* traversal launches timed: with rb_set_profiling, by CUDA events around each
	                               launch; otherwise by the device clock inside the kernels (from the first
	                               warp's start to the last warp's end of each launch), on every lane */
	uint32_t secondary_launches;
} rb_render_stats;
rb_status rb_render_stats_get(rb_context* ctx, rb_render_stats* out);

/* Enable node-visit / triangle-test counting in the traversal kernels (slower). */
rb_status rb_set_counting(rb_context* ctx, int enabled);
/* Time every traversal launch with CUDA events on the launching stream
 * (stats extend_ms / secondary_ms). Launches then run without graph replay. */
rb_status rb_set_profiling(rb_context* ctx, int enabled);

/* Checkpoint / resume of the film accumulators and sample counter. */
rb_status rb_checkpoint_save(rb_context* ctx, const char* path);
rb_status rb_checkpoint_load(rb_context* ctx, const char* path);

/* ------------------------------------------------------------------ launch tuning and autotuner
 * No counterpart in the reference (its only knob is the 16x16 tile of
 * sampler_integrator.cpp:30). The wavefront's launch shapes: paths per wave
 * (queue capacity), threads per block of the traversal and shading kernels,
 * blocks per SM of the grid-stride launches, and the sort key of the hit
 * queues. Every setting gives the same image; only the speed changes. */
enum {
	RB_SORT_MATERIAL = 0,       /* one hit queue per material class (coherent shading warps) */
	RB_SORT_NONE = 1,           /* one hit queue for every surface hit (no sorting) */
	RB_SORT_RAYS = 2            /* material-class hit queues, and before every bounce's traversal the active
	                               paths binned by ray direction octant and a Morton cell of the origin
	                               (coherent traversal warps) */
};
enum {
	RB_SHADOW_CLOSEST = 0,       /* NEE shadow rays find their closest visible hit, as scene::intersect_with_shadow_ray */
	RB_SHADOW_FIRST_OCCLUDER = 1 /* NEE shadow rays of plain path tracing: the sampled emitter's own triangles first,
	                                then the traversal stops at the first visible hit closer than the emitter's (the
	                                reference's accept rule, integrator.cpp:131-136, needs no more); the same
	                                visibility except where an occluder and the emitter are hit at distances equal
	                                to float rounding */
};
enum {
	RB_TRAVERSAL_PER_THREAD = 0, /* one ray per thread, traced to the end (grid-stride) */
	RB_TRAVERSAL_REFILL = 1      /* persistent lanes advance their ray one node at a time and take the next ray
	                                from the queue as soon as theirs is done */
};
typedef struct rb_tuning {
	uint32_t paths_per_wave;    /* queue capacity, 0: library default (2^21); a render's own
	                               rb_render_params.paths_per_wave takes precedence */
	uint32_t block_trace;       /* 32..256, a multiple of 32; 0: 128 */
	uint32_t block_shade;       /* 32..256, a multiple of 32; 0: 128 */
	uint32_t grid_per_sm;       /* 1..64; 0: 8 */
	uint32_t sort;              /* RB_SORT_* */
	uint32_t tail_bounce;       /* bounces run as separate wavefront stages before one kernel carries
	                               every surviving path to its end (one thread per path, the same
	                               stage code); 0: library default (64: none), >= max_depth: none */
	uint32_t lanes;             /* wave lanes (1..8, 0: 1): each lane has its own path buffers, stream and
	                               graph, so the late bounces of one wave overlap the next wave's early
	                               ones; the film still adds the waves in order (every render kind;
	                               guided waves sample the weights their lane saw after its previous
	                               wave trained) */
	uint32_t traversal;         /* RB_TRAVERSAL_*: how the traversal kernels take rays */
	uint32_t smem_carveout;     /* traversal kernels' shared-memory share of the L1 / shared storage, in
	                               percent + 1 (1..101); 0: the largest share (4 blocks of 256 threads with
	                               their stacks); smaller shares leave more L1 for tree nodes */
	uint32_t shadow_test;       /* RB_SHADOW_* */
	uint32_t reserved[2];
} rb_tuning;
/* Use `tuning` (NULL: defaults) for the context's later render calls. */
rb_status rb_set_tuning(rb_context* ctx, const rb_tuning* tuning);
rb_status rb_get_tuning(rb_context* ctx, rb_tuning* tuning);
/* Autotuner: times renders of `probe_spp` samples per pixel of `params`
 * (its camera, depth, seed, and RB_RENDER_VOLUME or RB_RENDER_DIRECT with its
 * direct_samples; guiding is refused; the film is left cleared) under candidate
 * tunings by coordinate descent over the settings above (CUDA events, best of
 * repeats), keeps the fastest for the context and returns it with its time. */
rb_status rb_tune_render(rb_context* ctx, const rb_render_params* params, uint32_t probe_spp, rb_tuning* best,
	float* best_ms);

/* ------------------------------------------------------------------ batched rendering
 * No counterpart in the reference, which renders one scene per
 * integrator::render call (integrator.hpp:64-66). Many scenes of uneven size
 * are uploaded together and rendered by one sequence of wavefront launches:
 * their samples share waves and queues, every path carries its scene, and each
 * scene's film is its own range of one merged film. Scene k's samples are the
 * ones rb_render would make for it with the same camera, spp, first_sample and
 * seed (same per-sample streams), so a batch and the scenes' separate renders
 * give the same films up to the order of FP64 additions. Learned guiding and
 * volumes are not available in batches. */
typedef struct rb_batch_view {
	rb_camera_desc camera;
	uint32_t spp;
	uint32_t first_sample;
	uint32_t seed;
	uint32_t reserved;
} rb_batch_view;
typedef struct rb_batch_params {
	const rb_batch_view* views; /* one per uploaded scene, in upload order */
	uint32_t count;             /* number of uploaded scenes */
	uint32_t max_depth;         /* shared by every scene */
	float rr_threshold;
	uint32_t flags;             /* RB_RENDER_RESET only */
	const uint32_t* order;      /* order in which scenes are started (a permutation), NULL: upload order */
} rb_batch_params;
/* Upload `count` scenes into the context, replacing any scene or batch there.
 * Afterwards rb_render, rb_trace_* and rb_render_noalloc refuse the context
 * until an rb_scene_upload. */
rb_status rb_batch_upload(rb_context* ctx, const rb_scene_desc* scenes, uint32_t count);
/* Render every scene of the batch. scene_ms (may be NULL, `count` floats):
 * device time from the start of the call until the wave that completed each
 * scene had finished (the scene's latency within the batch). */
rb_status rb_batch_render(rb_context* ctx, const rb_batch_params* params, float* scene_ms);
/* Film of scene `scene` of the last batch render (layout as rb_film_read / rb_render). */
rb_status rb_batch_film_read(rb_context* ctx, uint32_t scene, double* sum_rgb, double* sum_sq_rgb, uint32_t* sample_count);
rb_status rb_batch_image(rb_context* ctx, uint32_t scene, float* rgb_out);
/* The autotuner on a batch: probes render the batch's first `probe_items`
 * work items (scene order as in params). */
rb_status rb_tune_batch(rb_context* ctx, const rb_batch_params* params, uint64_t probe_items, rb_tuning* best,
	float* best_ms);

/* ------------------------------------------------------------------ learned path guiding
 * No counterpart in the reference renderer, which samples path continuations
 * from the BSDF only (integrator.cpp:380-399). A small network maps a surface
 * vertex (position normalised to the scene box, shading normal and outgoing
 * direction, each mapped to [0, 1]) through a 12-frequency sin/cos encoding and
 * 4 hidden ReLU layers of width 64 (BF16 weights, FP32 accumulation on the
 * tensor cores) to 8 von Mises-Fisher lobes (mean, concentration, weight) and a
 * mixing fraction alpha. With RB_RENDER_GUIDE a non-specular vertex samples its
 * continuation from the guide with probability alpha and from the BSDF
 * otherwise, and weights it by f cos / (alpha q + (1 - alpha) p_bsdf) (one-sample
 * MIS, unbiased for any network); until the first training step every vertex
 * samples the BSDF alone, exactly as without the flag. With RB_RENDER_TRAIN
 * each finished wave turns its recorded vertices into training samples
 * (direction, BSDF pdf and weight = luminance of the radiance the continuation
 * brought back over the throughput at the vertex), appends them to a replay
 * ring that keeps the samples of earlier waves, and runs steps_per_wave Adam
 * steps on batches drawn from the whole ring, of the loss
 * -weight * (log q + log(alpha q + (1 - alpha) p_bsdf)). */
#define RB_GUIDE_NUM_PARAMS 30000u  /* flat W1[64][224] b1[64] W2[64][64] b2 W3 b3 W4 b4 W5[48][64] b5[48] */
#define RB_GUIDE_INPUTS 9u
#define RB_GUIDE_OUTPUTS 48u        /* raw outputs: lobe i at 5i..5i+4 (mean xyz, log kappa, weight logit), alpha logit at 40 */
typedef struct rb_guide_config {
	uint32_t seed;              /* weight initialisation */
	float learning_rate;        /* Adam step size, 0: 1e-3 */
	uint32_t batch_size;        /* rows per training step, 0: 2^18 */
	uint32_t steps_per_wave;    /* training steps after each wave of a RB_RENDER_TRAIN render, 0: 8 */
	uint32_t max_samples;       /* replay ring of training samples (rounded up to a power of two), 0: 2^21 */
	uint32_t min_rows;          /* steps with fewer collected samples are skipped, 0: 4096 */
	float weight_clip;          /* rendering-time training clips each weight at this multiple of the
	                               running mean weight (fewer steps dominated by rare paths), 0: 16,
	                               < 0: no clipping */
	uint32_t warmup_steps;      /* RB_RENDER_GUIDE samples the guide only after this many Adam steps
	                               (until then continuations come from the BSDF alone), 0: 1 */
} rb_guide_config;
/* One training sample (64 bytes). */
typedef struct rb_guide_sample {
	float inputs[9];
	float direction[3];         /* unit world direction of the continuation */
	float bsdf_pdf;             /* BSDF pdf of that direction (solid angle) */
	float weight;               /* integrand over sampling pdf, >= 0 */
	float reserved[2];
} rb_guide_sample;
typedef struct rb_guide_stats {
	uint32_t steps;             /* Adam steps taken */
	uint32_t samples_last_wave; /* training samples stored by the last wave */
	uint32_t candidates_last_wave; /* vertices with a positive weight in the last wave */
	uint32_t device_error;      /* rb_status of a failed bounded device wait, RB_OK if none */
	float last_loss;
	uint32_t rows_last_step;
	uint32_t reserved[2];
} rb_guide_stats;
enum {
	RB_GUIDE_SEQUENTIAL = 1u << 0  /* rb_guide_train: every step uses all samples in order (full batch) */
};
/* (Re)create the network with fresh weights and zero Adam moments; config may be NULL (defaults). */
rb_status rb_guide_init(rb_context* ctx, const rb_guide_config* config);
/* FP32 master weights in the flat order of RB_GUIDE_NUM_PARAMS. W1 columns
 * 216..223 (padding features) are always zero; set ignores them. Set also
 * clears the Adam moments and step count. */
rb_status rb_guide_get_params(rb_context* ctx, float* params, uint32_t count);
rb_status rb_guide_set_params(rb_context* ctx, const float* params, uint32_t count);
/* Raw outputs (RB_GUIDE_OUTPUTS per row) of the tensor-core forward pass. */
rb_status rb_guide_forward(rb_context* ctx, const float* inputs, uint32_t n, float* outputs);
/* `steps` training steps on host samples (batch: config batch_size rows drawn
 * by a hash of (step, row), or all n in order with RB_GUIDE_SEQUENTIAL).
 * gradient (may be NULL): the batch gradient of the last step, flat order. */
rb_status rb_guide_train(rb_context* ctx, const rb_guide_sample* samples, uint32_t n, uint32_t steps, uint32_t flags,
	float* gradient, float* loss);
/* Decode raw outputs (RB_GUIDE_OUTPUTS per row) and draw one direction per row
 * from the guide density with the uniforms u (3 per row: lobe pick, two for the
 * lobe); writes the unit direction (3 per row) and the guide pdf q at it. */
rb_status rb_guide_sample_dirs(rb_context* ctx, const float* outputs, const float* u, uint32_t n, float* directions,
	float* pdfs);
rb_status rb_guide_stats_get(rb_context* ctx, rb_guide_stats* out);
/* Guided volume renders (RB_RENDER_VOLUME with RB_RENDER_GUIDE / RB_RENDER_TRAIN)
 * guide medium vertices with a second network of the same shape (its own
 * weights, Adam moments and replay ring), fed the vertex position, a zero
 * normal and the outgoing direction, and mixed with the Henyey-Greenstein
 * phase function by the same one-sample MIS; its counters: */
rb_status rb_guide_medium_stats_get(rb_context* ctx, rb_guide_stats* out);

/* ------------------------------------------------------------------ host-side helpers (no GPU) */

/* Build the flattened BVH of a scene with the reference's rules
 * (scene::build_accelerator, scene.cpp:30-80): one leaf per triangle of each
 * entity whose mesh is used by that entity only and has at most 2^17
 * triangles, one leaf for the whole entity otherwise (prim_index
 * RB_BVH_ALL_TRIANGLES), whose mesh then gets its own tree over its faces in
 * local space (mesh::build_accelerator, mesh.cpp:159-172); median split on the
 * widest centroid axis with std::nth_element (detail/bounding_volume_hierarchy.hpp:162-233).
 * rb_bvh_depth: the deepest nesting, a mesh tree's levels counted below the
 * scene tree's entity leaf. */
typedef struct rb_bvh rb_bvh;
rb_status rb_bvh_build(const rb_scene_desc* desc, rb_bvh** out);
rb_status rb_bvh_get(const rb_bvh* bvh, rb_bvh_desc* out);
rb_status rb_bvh_depth(const rb_bvh* bvh, uint32_t* max_depth);
/* The mesh trees of the two-level case (mesh::mAccelerator), in order of first
 * use: tree k belongs to mesh *mesh; in *out, prim slot p is face prim_index[p]
 * of that mesh and prim_entity is NULL. */
rb_status rb_bvh_mesh_tree_count(const rb_bvh* bvh, uint32_t* count);
rb_status rb_bvh_get_mesh_tree(const rb_bvh* bvh, uint32_t k, int32_t* mesh, rb_bvh_desc* out);
void rb_bvh_free(rb_bvh* bvh);

/* Seeded synthetic scenes of the benchmark configurations. */
enum {
	RB_SCENE_BOX = 0,          /* closed box room: 32 triangles, one 0.25 x 0.25 quad light */
	RB_SCENE_SPHERES = 1,      /* displaced icospheres over a ground plane, 4 quad lights + environment */
	RB_SCENE_SLIT_ROOM = 2,    /* glossy room, light behind a wall with a slit (hard indirect) */
	RB_SCENE_FOG = 3           /* displaced icospheres in a homogeneous medium box, 16 quad lights */
};
typedef struct rb_scene_gen_params {
	uint32_t kind;
	uint32_t seed;
	uint32_t num_spheres;      /* RB_SCENE_SPHERES / RB_SCENE_SLIT_ROOM clutter count */
	uint32_t subdivision;      /* icosphere subdivision level */
	int32_t width;
	int32_t height;
} rb_scene_gen_params;
typedef struct rb_scene rb_scene;
rb_status rb_scene_generate(const rb_scene_gen_params* params, rb_scene** out);
/* Pointers stay valid until rb_scene_free. bvh is left empty (num_nodes == 0). */
rb_status rb_scene_get(const rb_scene* scene, rb_scene_desc* desc, rb_camera_desc* camera);
void rb_scene_free(rb_scene* scene);

/* ------------------------------------------------------------------ failure detection (no reference counterpart)
 * Device waits in this library are bounded: a wait that runs out sets an error
 * word and returns, and the context stays usable. rb_check_bounded_wait runs
 * one such wait (an mbarrier that nothing arrives on, the wait of the guide
 * kernels) with a limit of limit_us microseconds and reports what the wait
 * returned in *status (RB_ERR_DEVICE_TIMEOUT when it ran out). */
rb_status rb_check_bounded_wait(rb_context* ctx, uint32_t limit_us, rb_status* status);
/* Host-side fault injection: the `after`-th device allocation from now on
 * fails as if the device were out of memory (after < 0: off). */
void rb_inject_allocation_failure(int32_t after);

/* Library ABI version (RBGPU_ABI_VERSION at build time). */
int32_t rb_abi_version(void);

#ifdef __cplusplus
}
#endif

#endif /* RBGPU_H */
