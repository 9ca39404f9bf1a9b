// Test-only host build of the kernels' per-path functions (rainbow_b200/csrc/pt/*.h).
//
// The device code of the path tracer is written as __host__ __device__
// functions. This file compiles them for the CPU, with glibc's libm (the same
// library the compiled reference uses), and drives them one sample at a time,
// so a test can check the stage logic and its random-number order against the
// reference bit for bit without a GPU. It is not reachable from the library:
// librbgpu.so has no CPU path.
#include "../../include/rbgpu.h"
#include "../../rainbow_b200/csrc/host/scene_pack.h"
#include "../../rainbow_b200/csrc/kernels.cuh"
#include "../../rainbow_b200/csrc/pt/pt_path.h"
#include "../../rainbow_b200/csrc/pt/pt_sss.h"
#include "../../rainbow_b200/csrc/pt/pt_photon.h"

#include <algorithm>
#include <cmath>
#include <limits>
#include <new>
#include <vector>

using namespace rb;
using namespace rb::pt;

namespace {

struct host_stack {
	uint32_t data[128];
	float te[128];
	uint32_t sp = 0;
	void reset() { sp = 0; }
	void push(uint32_t v) { data[sp++] = v; }
	uint32_t pop() { return data[--sp]; }
	void push(uint32_t v, float t) { data[sp] = v; te[sp] = t; sp++; }
	void pop(uint32_t& v, float& t) { sp--; v = data[sp]; t = te[sp]; }
	bool empty() const { return sp == 0; }
	bool full() const { return sp + 2 > 128; }
	uint32_t size() const { return sp; }
	raw_stack raw() { return raw_stack{data, 1u, sp, 128u}; }
};

struct hp_scene {
	host::packed_scene packed;
	scene_view view;
};

// mode 0: the kernels' dispatch (child-box traversal, exact path on NaN);
// mode 1: the reference-order traversal only.
int g_mode = 0;

hit_t trace(const scene_view& v, vec3 o, vec3 d, float& len, bool shadow) {
	host_stack st;
	trace_counters c{0, 0};
	hit_t h;
	if (g_mode == 0 && v.wnodes != nullptr && !std::isnan(len)) {
		const float len0 = len;
		const int r = shadow ? closest_hit_fast<true>(v, o, d, len, h, st) : closest_hit_fast<false>(v, o, d, len, h, st);
		if (r >= 0) return h;
		len = len0;
	}
	if (shadow) closest_hit<true, false>(v, o, d, len, h, st, c);
	else closest_hit<false, false>(v, o, d, len, h, st, c);
	return h;
}

} // namespace

extern "C" {

void hp_set_mode(int mode) { g_mode = mode; }

int hp_create(const rb_scene_desc* desc, void** out) {
	auto* s = new (std::nothrow) hp_scene();
	if (!s) return RB_ERR_OUT_OF_MEMORY;
	const rb_status st = host::pack_scene(desc, s->packed);
	if (st != RB_OK) {
		delete s;
		return st;
	}
	s->view = host::host_view(s->packed);
	*out = s;
	return RB_OK;
}

void hp_free(void* s) { delete static_cast<hp_scene*>(s); }

} // extern "C"

namespace {

// entity_base: subtracted from reported entity ordinals (a scene of a merged batch).
void trace_batch(const host::packed_scene& packed, const scene_view& view, uint32_t entity_base, const rb_ray* rays,
	uint32_t n, int shadow, rb_hit* hits) {
	for (uint32_t i = 0; i < n; i++) {
		float len = rays[i].length;
		const hit_t h = trace(view, vec3{rays[i].origin[0], rays[i].origin[1], rays[i].origin[2]},
			vec3{rays[i].direction[0], rays[i].direction[1], rays[i].direction[2]}, len, shadow != 0);
		hits[i].entity = h.slot >= 0 ? static_cast<int32_t>(packed.prim_entity[h.slot] - entity_base) : -1;
		hits[i].triangle = h.slot >= 0 ? static_cast<int32_t>(packed.prim_index[h.slot]) : -1;
		hits[i].t = len;
		hits[i].b1 = h.slot >= 0 ? h.b1 : 0.f;
		hits[i].b2 = h.slot >= 0 ? h.b2 : 0.f;
	}
}

// Radiance of (pixel, sample) pairs through the same stage sequence the
// kernels run: camera, then per bounce extend -> shade_a -> secondary rays -> shade_b.
void samples_view(const scene_view& view, const rb_camera_desc* cam, const uint32_t* pixels, const uint32_t* samples,
	uint32_t n, uint32_t max_depth, float rr, uint32_t seed, float* out) {
	for (uint32_t i = 0; i < n; i++) {
		const uint32_t pixel = pixels[i];
		const uint32_t x = pixel % static_cast<uint32_t>(cam->width), y = pixel / static_cast<uint32_t>(cam->width);
		path_state p;
		path_begin(p, cam->raster_to_camera, cam->camera_to_world, cam->lens_radius, cam->focus_distance, x, y, pixel,
			samples[i], seed);
		for (int guard = 0; guard < 4096; guard++) {
			float len = p.len;
			const hit_t h = trace(view, p.o, p.d, len, false);
			shade_record rec;
			if (!shade_a_any(view, p, h, rec)) break;
			hit_t sh{-1, 0.f, 0.f}, mh{-1, 0.f, 0.f};
			if (rec.nee_entity >= 0) {
				float l = rec.shadow_ray.len;
				sh = trace(view, rec.shadow_ray.o, rec.shadow_ray.d, l, true);
			}
			if (rec.mis_valid) {
				float l = rec.mis_ray.len;
				mh = trace(view, rec.mis_ray.o, rec.mis_ray.d, l, true);
			}
			if (!shade_b_any(view, p, rec, sh, mh, max_depth, rr)) break;
			if (p.flags & PATH_SSS) {
				// the BSSRDF stage (k_subsurface), then Russian roulette
				p.flags &= ~PATH_SSS;
				auto tracer = [&view](vec3 o, vec3 d, float& l, bool shadow) { return trace(view, o, d, l, shadow); };
				if (!subsurface_walk(view, p, rec, h, tracer)) break;
				if (!roulette(p, max_depth, rr)) break;
			}
		}
		out[3 * i] = p.L.x;
		out[3 * i + 1] = p.L.y;
		out[3 * i + 2] = p.L.z;
	}
}

// Radiance of (pixel, sample) pairs through direct_integrator (pt::direct_radiance),
// rays traced with the kernels' traversal dispatch.
void direct_samples_view(const scene_view& view, const rb_camera_desc* cam, const uint32_t* pixels, const uint32_t* samples,
	uint32_t n, uint32_t emitter_samples, uint32_t bsdf_samples, uint32_t seed, float* out) {
	const direct_cfg dc = make_direct_cfg(emitter_samples, bsdf_samples);
	auto tracer = [&view](vec3 o, vec3 d, float& len, bool shadow) { return trace(view, o, d, len, shadow); };
	for (uint32_t i = 0; i < n; i++) {
		const uint32_t pixel = pixels[i];
		const uint32_t x = pixel % static_cast<uint32_t>(cam->width), y = pixel / static_cast<uint32_t>(cam->width);
		path_state p;
		path_begin(p, cam->raster_to_camera, cam->camera_to_world, cam->lens_radius, cam->focus_distance, x, y, pixel,
			samples[i], seed);
		direct_radiance(view, dc, p, tracer);
		out[3 * i] = p.L.x;
		out[3 * i + 1] = p.L.y;
		out[3 * i + 2] = p.L.z;
	}
}

// A merged batch (host::merge_scenes) with the per-scene views the kernels
// build from their batch_scene records (gpu::batch_view).
struct hp_batch {
	host::packed_scene packed;
	std::vector<scene_view> views;
	std::vector<uint32_t> entity_base;
};

} // namespace

extern "C" {

// The lobe list that the packed record of material 0 of `mds` (count materials,
// a mixture's components among them) gives make_bsdf: the lobe kinds (LOBE_*)
// in collection order. Returns the packing status.
int hp_material_set_lobes(const rb_material_desc* mds, uint32_t num, uint32_t* kinds, uint32_t* count);
int hp_material_lobes(const rb_material_desc* md, uint32_t* kinds, uint32_t* count) {
	return hp_material_set_lobes(md, 1, kinds, count);
}
int hp_material_set_lobes(const rb_material_desc* mds, uint32_t num, uint32_t* kinds, uint32_t* count) {
	// one triangle with the material, and an environment emitter (a scene needs one)
	const float pos[9] = {0.f, 0.f, 0.f, 1.f, 0.f, 0.f, 0.f, 1.f, 0.f};
	const uint32_t idx[3] = {0, 1, 2};
	rb_mesh_desc mesh{};
	mesh.positions = pos;
	mesh.indices = idx;
	mesh.num_vertices = 3;
	mesh.num_triangles = 1;
	rb_emitter_desc em{};
	em.kind = RB_EMITTER_ENVIRONMENT;
	em.radius = 1.f;
	rb_entity_desc ents[2]{};
	for (int e = 0; e < 2; e++) {
		ents[e].mesh = e == 0 ? 0 : -1;
		ents[e].material = e == 0 ? 0 : -1;
		ents[e].emitter = e == 0 ? -1 : 0;
		ents[e].medium = -1;
		for (int i = 0; i < 16; i++) ents[e].local_to_world[i] = ents[e].world_to_local[i] = (i % 5 == 0) ? 1.f : 0.f;
	}
	rb_scene_desc d{};
	d.meshes = &mesh;
	d.num_meshes = 1;
	d.materials = mds;
	d.num_materials = num;
	d.emitters = &em;
	d.num_emitters = 1;
	d.entities = ents;
	d.num_entities = 2;
	host::packed_scene p;
	const rb_status st = host::pack_scene(&d, p);
	if (st != RB_OK) return st;
	const bsdf_t b = make_bsdf(p.materials.data());
	*count = b.count;
	for (uint32_t i = 0; i < b.count; i++) kinds[i] = lobe_kind(b, i);
	return RB_OK;
}

// The kernels' image texture lookup (pt::sample_texture) at n texture coordinates.
int hp_texture_sample(const float* rgb, uint32_t width, uint32_t height, uint32_t n, const float* uv, float* out) {
	texture_rec tr{};
	tr.kind = TEXK_IMAGE;
	tr.width = width;
	tr.height = height;
	scene_view v{};
	v.textures = &tr;
	v.texels = rgb;
	v.num_textures = 1;
	for (uint32_t i = 0; i < n; i++) {
		const vec3 c = sample_texture(v, 0u, vec2{uv[2 * i], uv[2 * i + 1]}, vec3{0.f, 0.f, 0.f});
		out[3 * i] = c.x;
		out[3 * i + 1] = c.y;
		out[3 * i + 2] = c.z;
	}
	return 0;
}

// The normalized-diffusion inverse CDF table (kSssTableSize knots) the scene
// packer builds, and sss_sample_profile(table, d, u) at n (d, u) pairs.
int hp_sss_table(float* table, uint32_t n, const float* du, float* r) {
	std::vector<float> t(kSssTableSize);
	sss_build_table(t.data());
	for (uint32_t i = 0; i < kSssTableSize; i++) table[i] = t[i];
	for (uint32_t i = 0; i < n; i++) r[i] = sss_sample_profile(t.data(), du[2 * i], du[2 * i + 1]);
	return static_cast<int>(kSssTableSize);
}

// photon_mapping_integrator::render (photon_mapping_integrator.cpp:386-560)
// through the photon stage functions. streams 0: the reference's own order and
// streams (one pcg32 per 16 x 16 tile of pixels, seeded by the tile's index,
// and one per chunk of 8192 photons, seeded by the chunk's index, each kept
// across iterations; pixels and photons in order), so the image is the
// reference's bit for bit; streams 1: the kernels' per-pixel and per-photon
// streams (sppm_pixel_seed, sppm_photon_seed). The grid is built as the
// reference builds it (a pixel appears in a bucket once per cell of its box
// that hashes there). out: W * H * 3 floats, the film's set_pixel values.
int hp_photon_render(void* hs, const rb_camera_desc* cam, uint32_t iterations, uint32_t max_depth, uint32_t photons,
	float radius, int streams, uint32_t seed, float* out) {
	const scene_view& view = static_cast<hp_scene*>(hs)->view;
	const uint32_t W = static_cast<uint32_t>(cam->width), H = static_cast<uint32_t>(cam->height);
	const uint32_t npix = W * H;
	const uint64_t nphot = photons == 0 ? npix : photons;
	std::vector<sppm_pixel> px(npix);
	for (auto& q : px) {
		q.tau = splat3(0.f);
		q.L = splat3(0.f);
		q.radius = radius;
		q.n = 0.f;
	}
	std::vector<visible_point> vp(npix);
	std::vector<spectrum> phi(npix);
	std::vector<uint32_t> m(npix);
	auto tracer = [&view](vec3 o, vec3 d, float& len, bool shadow) { return trace(view, o, d, len, shadow); };
	// the reference's streams: tiles in row order, chunks in order
	const uint32_t tiles_x = (W + 15) / 16, tiles_y = (H + 15) / 16;
	std::vector<pcg32> tile_rng(static_cast<size_t>(tiles_x) * tiles_y);
	for (size_t t = 0; t < tile_rng.size(); t++) tile_rng[t] = pcg_seed(t);
	const uint64_t chunks = (nphot + 8191) / 8192;
	std::vector<pcg32> chunk_rng(chunks);
	for (uint64_t c = 0; c < chunks; c++) chunk_rng[c] = pcg_seed(c);
	for (uint32_t it = 0; it < iterations; it++) {
		// visible points
		for (uint32_t ty = 0; ty < tiles_y; ty++)
			for (uint32_t tx = 0; tx < tiles_x; tx++)
				for (uint32_t y = ty * 16; y < std::min(H, ty * 16 + 16); y++)
					for (uint32_t x = tx * 16; x < std::min(W, tx * 16 + 16); x++) {
						const uint32_t pixel = y * W + x;
						path_state p;
						pcg32& g = tile_rng[ty * tiles_x + tx];
						p.rng = streams == 0 ? g : pcg_seed(sppm_pixel_seed(pixel, it, seed));
						const ray_t r = camera_ray(cam->raster_to_camera, cam->camera_to_world, cam->lens_radius,
							cam->focus_distance, x, y, p.rng);
						p.o = r.o;
						p.d = r.d;
						p.len = r.len;
						p.beta = splat3(1.f);
						p.L = splat3(0.f);
						p.eta = 1.f;
						p.flags = 0u;
						p.bounces = 0;
						p.medium = -1;
						sppm_visible(view, p, max_depth, tracer, vp[pixel]);
						if (streams == 0) g = p.rng;
						px[pixel].L = px[pixel].L + p.L;
					}
		// the grid (build_visible_point_grid)
		sppm_grid g;
		g.lo = splat3(std::numeric_limits<float>::max());
		g.hi = splat3(std::numeric_limits<float>::min());
		g.pool = npix;
		float max_r = 0.f;
		bool any = false;
		for (uint32_t i = 0; i < npix; i++) {
			if (!vp[i].valid) continue;
			any = true;
			const vec3 a = vp[i].p - splat3(px[i].radius), b = vp[i].p + splat3(px[i].radius);
			g.lo = vec3{std::min(g.lo.x, a.x), std::min(g.lo.y, a.y), std::min(g.lo.z, a.z)};
			g.hi = vec3{std::max(g.hi.x, b.x), std::max(g.hi.y, b.y), std::max(g.hi.z, b.z)};
			max_r = std::max(max_r, px[i].radius);
		}
		std::vector<std::vector<uint32_t>> bucket(npix);
		if (any) {
			sppm_grid_size(g, max_r);
			for (uint32_t i = 0; i < npix; i++) {
				if (!vp[i].valid) continue;
				int32_t x0, y0, z0, x1, y1, z1;
				sppm_cell(g, vp[i].p - splat3(px[i].radius), x0, y0, z0);
				sppm_cell(g, vp[i].p + splat3(px[i].radius), x1, y1, z1);
				for (int32_t z = z0; z <= z1; z++)
					for (int32_t y = y0; y <= y1; y++)
						for (int32_t x = x0; x <= x1; x++) bucket[sppm_bucket(g, x, y, z)].push_back(i);
			}
		}
		// photons
		std::fill(phi.begin(), phi.end(), splat3(0.f));
		std::fill(m.begin(), m.end(), 0u);
		auto deposit = [&](const surface_t& si, const spectrum& beta, vec3 d) {
			if (!any || !sppm_inside(g, si.p)) return;
			int32_t x, y, z;
			sppm_cell(g, si.p, x, y, z);
			const auto& list = bucket[sppm_bucket(g, x, y, z)];
			for (size_t k = list.size(); k-- > 0;) {  // the reference pushes at the list's head
				const uint32_t i = list[k];
				spectrum flux;
				if (!sppm_flux(view, si, beta, d, vp[i], px[i].radius, flux)) continue;
				phi[i] = phi[i] + flux;
				m[i]++;
			}
		};
		for (uint64_t j = 0; j < nphot; j++) {
			pcg32& c = chunk_rng[j / 8192];
			pcg32 rng = streams == 0 ? c : pcg_seed(sppm_photon_seed(static_cast<uint32_t>(j), it, seed));
			sppm_photon(view, rng, max_depth, tracer, deposit);
			if (streams == 0) c = rng;
		}
		for (uint32_t i = 0; i < npix; i++) sppm_update(px[i], vp[i].beta, phi[i], m[i]);
	}
	for (uint32_t i = 0; i < npix; i++) {
		const spectrum v = sppm_value(px[i], iterations, nphot);
		out[3 * i] = v.x;
		out[3 * i + 1] = v.y;
		out[3 * i + 2] = v.z;
	}
	return RB_OK;
}

int hp_trace(void* hs, const rb_ray* rays, uint32_t n, int shadow, rb_hit* hits) {
	const hp_scene& s = *static_cast<hp_scene*>(hs);
	trace_batch(s.packed, s.view, 0u, rays, n, shadow, hits);
	return RB_OK;
}

int hp_samples(void* hs, const rb_camera_desc* cam, const uint32_t* pixels, const uint32_t* samples, uint32_t n,
	uint32_t max_depth, float rr, uint32_t seed, float* out) {
	samples_view(static_cast<hp_scene*>(hs)->view, cam, pixels, samples, n, max_depth, rr, seed, out);
	return RB_OK;
}

int hp_direct_samples(void* hs, const rb_camera_desc* cam, const uint32_t* pixels, const uint32_t* samples, uint32_t n,
	uint32_t emitter_samples, uint32_t bsdf_samples, uint32_t seed, float* out) {
	if (emitter_samples == 0 || bsdf_samples == 0) return RB_ERR_INVALID_ARGUMENT;
	direct_samples_view(static_cast<hp_scene*>(hs)->view, cam, pixels, samples, n, emitter_samples, bsdf_samples, seed, out);
	return RB_OK;
}

// The staged form of the same samples, stage by stage as the staged kernels
// run them: camera ray (and pass-throughs), light samples and the first BSDF
// ray, their traces, then one round per BSDF sample.
int hp_direct_staged_samples(void* hs, const rb_camera_desc* cam, const uint32_t* pixels, const uint32_t* samples,
	uint32_t n, uint32_t emitter_samples, uint32_t bsdf_samples, uint32_t seed, float* out) {
	if (emitter_samples == 0 || bsdf_samples == 0 || emitter_samples > kDirectStagedLights) return RB_ERR_INVALID_ARGUMENT;
	const scene_view& view = static_cast<hp_scene*>(hs)->view;
	const direct_cfg dc = make_direct_cfg(emitter_samples, bsdf_samples);
	for (uint32_t i = 0; i < n; i++) {
		const uint32_t pixel = pixels[i];
		const uint32_t x = pixel % static_cast<uint32_t>(cam->width), y = pixel / static_cast<uint32_t>(cam->width);
		path_state p;
		path_begin(p, cam->raster_to_camera, cam->camera_to_world, cam->lens_radius, cam->focus_distance, x, y, pixel,
			samples[i], seed);
		direct_record rec;
		int state = 1;
		for (int guard = 0; guard < 4096 && state == 1; guard++) {
			float len = p.len;
			const hit_t h = trace(view, p.o, p.d, len, false);
			state = direct_surface(view, p, h, rec);
		}
		if (state == 2) {
			ray_t rays[kDirectStagedLights + 1];
			direct_sample_lights(view, dc, p, rec, rays);
			hit_t lh[kDirectStagedLights];
			for (uint32_t k = 0; k < emitter_samples; k++) {
				lh[k] = hit_t{-1, 0.f, 0.f};
				if (rec.light_entity[k] >= 0) {
					float l = rays[k].len;
					lh[k] = trace(view, rays[k].o, rays[k].d, l, true);
				}
			}
			ray_t br = rays[emitter_samples];
			for (;;) {
				hit_t bh{-1, 0.f, 0.f};
				if (rec.bsdf_valid) {
					float l = br.len;
					bh = trace(view, br.o, br.d, l, true);
				}
				if (!direct_round(view, dc, p, rec, lh, bh, br)) break;
			}
		}
		out[3 * i] = p.L.x;
		out[3 * i + 1] = p.L.y;
		out[3 * i + 2] = p.L.z;
	}
	return RB_OK;
}

int hp_batch_create(const rb_scene_desc* descs, uint32_t count, void** out) {
	auto* b = new (std::nothrow) hp_batch();
	if (!b) return RB_ERR_OUT_OF_MEMORY;
	std::vector<host::packed_scene> parts(count);
	uint32_t ent = 0;
	for (uint32_t k = 0; k < count; k++) {
		const rb_status st = host::pack_scene(descs + k, parts[k]);
		if (st != RB_OK) { delete b; return st; }
		b->entity_base.push_back(ent);
		ent += static_cast<uint32_t>(parts[k].entities.size());
	}
	std::vector<host::scene_place> places;
	const rb_status st = host::merge_scenes(parts, b->packed, places);
	if (st != RB_OK) { delete b; return st; }
	const scene_view merged = host::host_view(b->packed);
	for (const host::scene_place& pl : places) {
		gpu::batch_scene r{};
		r.root_a = pl.root_a;
		r.root_b = pl.root_b;
		r.root_ref = pl.root_ref;
		r.root_node = pl.root_node;
		r.emitter_base = pl.emitter_base;
		r.num_emitters = pl.num_emitters;
		r.env_base = pl.env_base;
		r.num_environments = pl.num_environments;
		r.env = pl.env;
		b->views.push_back(gpu::batch_view(merged, r));
	}
	*out = b;
	return RB_OK;
}

void hp_batch_free(void* b) { delete static_cast<hp_batch*>(b); }

int hp_batch_trace(void* hb, uint32_t scene, const rb_ray* rays, uint32_t n, int shadow, rb_hit* hits) {
	const hp_batch& b = *static_cast<hp_batch*>(hb);
	if (scene >= b.views.size()) return RB_ERR_INVALID_ARGUMENT;
	trace_batch(b.packed, b.views[scene], b.entity_base[scene], rays, n, shadow, hits);
	return RB_OK;
}

int hp_batch_samples(void* hb, uint32_t scene, const rb_camera_desc* cam, const uint32_t* pixels, const uint32_t* samples,
	uint32_t n, uint32_t max_depth, float rr, uint32_t seed, float* out) {
	const hp_batch& b = *static_cast<hp_batch*>(hb);
	if (scene >= b.views.size()) return RB_ERR_INVALID_ARGUMENT;
	samples_view(b.views[scene], cam, pixels, samples, n, max_depth, rr, seed, out);
	return RB_OK;
}

} // extern "C"
