// Wavefront path-tracing kernels for sm_100a.
//
// Traversal kernels keep each thread's DFS stack in shared memory, laid out
// [entry][thread] so a warp's pushes and pops hit 32 distinct banks. Queues
// are compacted with one atomic per warp: __ballot_sync collects the lanes
// that push, the lowest such lane reserves popc(mask) slots, and every lane
// writes at base + popc(mask & lanes_below_me). All loops are grid-stride loops
// over counts that live in device memory, so the launches can be captured in a
// CUDA graph once and replayed for every wave.
#include "device_common.cuh"
#include "kernels.cuh"
#include "pt/pt_volume.h"

namespace rb {
namespace gpu {

using namespace rb::pt;

namespace {

// Warp-aggregated push of `value` into queue (when `pred`); all lanes of the
// warp must call it together.
__device__ __forceinline__ void warp_push(bool pred, uint32_t value, uint32_t* queue, uint32_t* counter) {
	const uint32_t mask = __ballot_sync(0xffffffffu, pred);
	if (mask == 0) return;
	const uint32_t lane = threadIdx.x & 31u;
	const uint32_t leader = __ffs(mask) - 1;
	uint32_t base = 0;
	if (lane == leader) base = atomicAdd(counter, static_cast<uint32_t>(__popc(mask)));
	base = __shfl_sync(0xffffffffu, base, leader);
	if (pred) queue[base + __popc(mask & lanemask_lt())] = value;
}

// Warp-aggregated push into one of several queues: lanes with the same key are
// grouped with __match_any_sync, one lane per group reserves the group's slots.
// key == 0xffffffff: nothing to push. All lanes of the warp must call it together.
__device__ __forceinline__ void warp_push_keyed(uint32_t key, uint32_t value, uint32_t* queues, uint32_t stride,
	uint32_t* counters) {
	const uint32_t peers = __match_any_sync(0xffffffffu, key);
	const uint32_t lane = threadIdx.x & 31u;
	const uint32_t leader = __ffs(peers) - 1;
	uint32_t base = 0;
	if (lane == leader && key != 0xffffffffu) base = atomicAdd(counters + key, static_cast<uint32_t>(__popc(peers)));
	base = __shfl_sync(0xffffffffu, base, leader);
	if (key != 0xffffffffu) queues[key * stride + base + __popc(peers & lanemask_lt())] = value;
}

__device__ __forceinline__ void add64(uint32_t* counters, uint32_t word, uint64_t v) {
	atomicAdd(reinterpret_cast<unsigned long long*>(counters + word), static_cast<unsigned long long>(v));
}

__device__ __forceinline__ void warp_add64(uint32_t* counters, uint32_t word, uint32_t v) {
	for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
	if ((threadIdx.x & 31u) == 0 && v) add64(counters, word, v);
}


// Device-clock time of a launch, measured inside it: every warp marks its
// start and its end with %globaltimer, and the last warp to finish adds the
// span from the earliest start to the latest end to the timer's total and
// counts the launch. The timer's words (kernels.cuh) live in the counters of
// the launching lane, so launches of one timer never overlap. Every warp of the
// launch must call launch_timer_end exactly once, after all its work.
__device__ __forceinline__ uint64_t global_time_ns() {
	uint64_t t;
	asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
	return t;
}
__device__ __forceinline__ unsigned long long* timer_u64(uint32_t* counters, uint32_t word) {
	return reinterpret_cast<unsigned long long*>(counters + word);
}
__device__ __forceinline__ void launch_timer_begin(uint32_t* counters, uint32_t timer) {
	if ((threadIdx.x & 31u) == 0) atomicMax(timer_u64(counters, timer + TIMER_START), ~global_time_ns());
}
__device__ __forceinline__ void launch_timer_end(uint32_t* counters, uint32_t timer) {
	__syncwarp();
	if ((threadIdx.x & 31u) != 0) return;
	atomicMax(timer_u64(counters, timer + TIMER_END), global_time_ns());
	__threadfence();
	const uint32_t warps = gridDim.x * ((blockDim.x + 31u) / 32u);
	if (atomicAdd(counters + timer + TIMER_WARPS, 1u) != warps - 1u) return;
	// the last warp: every other warp's marks are in place
	__threadfence();
	const uint64_t start = ~atomicExch(timer_u64(counters, timer + TIMER_START), 0ull);
	const uint64_t end = atomicExch(timer_u64(counters, timer + TIMER_END), 0ull);
	atomicExch(counters + timer + TIMER_WARPS, 0u);
	atomicAdd(timer_u64(counters, timer + TIMER_TOTAL_NS), static_cast<unsigned long long>(end > start ? end - start : 0ull));
	atomicAdd(counters + timer + TIMER_LAUNCHES, 1u);
}

__device__ __forceinline__ hit_t to_hit(float4 h) {
	hit_t r;
	r.slot = static_cast<int32_t>(__float_as_uint(h.x));
	r.b1 = h.z;
	r.b2 = h.w;
	return r;
}

// ------------------------------------------------------------------ ray batches
template <bool SHADOW, bool COUNT>
__global__ void __launch_bounds__(256) k_trace_rays(scene_view s, const uint32_t* __restrict__ prim_entity,
	const rb_ray* __restrict__ rays, uint32_t n, rb_hit* __restrict__ hits, uint32_t stack_cap, uint32_t* counters) {
	extern __shared__ uint32_t smem[];
	smem_stack st = make_stack(smem, stack_cap);
	uint32_t nodes = 0, tris = 0;
	for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
		const uint32_t i = base + threadIdx.x;
		if (i < n) {
			const rb_ray r = rays[i];
			float len = r.length;
			hit_t h;
			const vec3 o{r.origin[0], r.origin[1], r.origin[2]};
			const vec3 d{r.direction[0], r.direction[1], r.direction[2]};
			if (!trace_one<SHADOW, COUNT>(s, o, d, len, h, st, nodes, tris)) set_error(counters, RB_ERR_STACK_OVERFLOW);
			rb_hit out;
			if (h.slot >= 0) {
				out.entity = static_cast<int32_t>(prim_entity[h.slot]);
				out.triangle = static_cast<int32_t>(s.prim_index[h.slot]);
				out.b1 = h.b1;
				out.b2 = h.b2;
			} else {
				out.entity = -1;
				out.triangle = -1;
				out.b1 = out.b2 = 0.f;
			}
			out.t = len;
			hits[i] = out;
		}
	}
	if (COUNT) {
		warp_add64(counters, CNT_NODE_VISITS, nodes);
		warp_add64(counters, CNT_TRI_TESTS, tris);
	}
}

// ------------------------------------------------------------------ learned guiding
// The guide's 9 inputs of a surface vertex: position in the scene box, shading
// normal and outgoing direction, each mapped to [0, 1].
__device__ __forceinline__ void write_guide_query(const wave_params& p, const surface_t& si, float4* out) {
	float x[9] = {(si.p.x - p.box_min[0]) * p.box_inv[0], (si.p.y - p.box_min[1]) * p.box_inv[1],
		(si.p.z - p.box_min[2]) * p.box_inv[2], 0.5f * (si.sz.x + 1.f), 0.5f * (si.sz.y + 1.f), 0.5f * (si.sz.z + 1.f),
		0.5f * (si.wo.x + 1.f), 0.5f * (si.wo.y + 1.f), 0.5f * (si.wo.z + 1.f)};
	for (int j = 0; j < 9; j++) x[j] = fminf(1.f, fmaxf(0.f, x[j]));
	out[0] = make_float4(x[0], x[1], x[2], x[3]);
	out[1] = make_float4(x[4], x[5], x[6], x[7]);
	out[2] = make_float4(x[8], 0.f, 0.f, 0.f);
}

// The medium guide's 9 inputs of a medium vertex: position in the scene box,
// a zero normal (mapped to 0.5) and the outgoing direction.
__device__ __forceinline__ void write_guide_query_medium(const wave_params& p, vec3 pos, vec3 wo, float4* out) {
	float x[9] = {(pos.x - p.box_min[0]) * p.box_inv[0], (pos.y - p.box_min[1]) * p.box_inv[1],
		(pos.z - p.box_min[2]) * p.box_inv[2], 0.5f, 0.5f, 0.5f, 0.5f * (wo.x + 1.f), 0.5f * (wo.y + 1.f), 0.5f * (wo.z + 1.f)};
	for (int j = 0; j < 9; j++) x[j] = fminf(1.f, fmaxf(0.f, x[j]));
	out[0] = make_float4(x[0], x[1], x[2], x[3]);
	out[1] = make_float4(x[4], x[5], x[6], x[7]);
	out[2] = make_float4(x[8], 0.f, 0.f, 0.f);
}

// One training vertex of path i (the wave_guide's layout): the guide inputs,
// the continuation direction and the pdf of the method that could also have
// drawn it (BSDF or phase function), the throughput before the continuation
// and the path radiance after the vertex's direct lighting.
__device__ __forceinline__ void record_vertex(const guide::wave_guide& g, uint32_t i, vec3 wi, float pb, spectrum beta0,
	spectrum L0) {
	const uint32_t nv = g.vertex_count[i];
	if (nv >= g.depth) return;
	float4* r = g.vertices + (static_cast<size_t>(i) * g.depth + nv) * guide::kVertexFloat4;
	const float4* x = g.query_in + 3 * i;
	r[0] = x[0];
	r[1] = x[1];
	r[2] = make_float4(x[2].x, wi.x, wi.y, wi.z);
	r[3] = make_float4(pb, beta0.x, beta0.y, beta0.z);
	r[4] = make_float4(L0.x, L0.y, L0.z, 0.f);
	g.vertex_count[i] = nv + 1u;
}

// Path continuation by one-sample MIS of the guide q (probability alpha) and
// the BSDF: the direction comes from either, and beta is multiplied by
// f cos / (alpha q + (1 - alpha) p_bsdf), which is unbiased for any guide.
// g: the decoded guide of this vertex (48 floats in device memory).
template <int MAT>
__device__ bool continue_guided(const scene_view& s, path_state& p, const shade_record& rec, const float* g, vec3& wi_out,
	float& pb_out) {
	const surface_t& si = rec.si;
	material_rec mat_scratch;
	const bsdf_t b = make_bsdf(surface_material<MAT>(s, rec.material, si, mat_scratch));
	const vec3 wo = to_local(si, si.wo);
	const float alpha = g[guide::kAlphaOff];
	const float u_sel = pcg_real(p.rng);
	const vec2 u = pcg_2d(p.rng);
	vec3 wi;
	spectrum f;
	float pb;
	if (u_sel < alpha) {
		float d[3];
		guide::guide_sample(g, u_sel / alpha, u.x, u.y, d);
		wi = vec3{d[0], d[1], d[2]};
		const vec3 wl = to_local(si, wi);
		f = bsdf_f<MAT>(b, wo, wl, ST_ALL);
		pb = bsdf_pdf<MAT>(b, wo, wl, ST_ALL);
	} else {
		const lobe_sample bs = bsdf_sample<MAT>(b, wo, u, ST_ALL);
		if (bs.pdf == 0.f) return false;
		wi = to_world(si, bs.wi);
		f = bs.f;
		pb = bs.pdf;
	}
	const float pdf = alpha * guide::guide_pdf(g, wi.x, wi.y, wi.z) + (1.f - alpha) * pb;
	if (is_black(f) || !(pdf > 0.f)) return false;
	p.beta = p.beta * (f * fabs_ref(dot(wi, si.sz)) / pdf);
	p.flags &= ~PATH_SPECULAR;
	const ray_t r = spawn_ray(si.p, si.n, wi);
	p.o = r.o;
	p.d = r.d;
	p.len = r.len;
	wi_out = wi;
	pb_out = pb;
	return true;
}

// shade_b of a guided or training render: direct lighting as always, the
// continuation from the guide where it applies (else from the BSDF, with the
// same random numbers as plain path tracing), and one recorded training vertex
// per guidable continuation.
template <int MAT>
__device__ bool shade_b_guided(const scene_view& s, const wave_buffers& w, const wave_params& p, uint32_t i, path_state& st,
	const shade_record& rec, const hit_t& sh, const hit_t& mh) {
	if (!rec.pass_through) {
		if (rec.did_nee) shade_b_direct<MAT>(s, st, rec, sh, mh);
		const spectrum beta0 = st.beta, L0 = st.L;
		vec3 wi;
		float pb;
		const bool use_guide = (p.guide_flags & GUIDE_SAMPLE) && rec.guidable && *w.guide.usable != 0u;
		const bool ok = use_guide
			? continue_guided<MAT>(s, st, rec, reinterpret_cast<const float*>(w.guide.query_out + 12 * i), wi, pb)
			: continue_bsdf<MAT>(s, st, rec, wi, pb);
		if (!ok) return false;
		if ((p.guide_flags & GUIDE_TRAIN) && rec.guidable && st.bounces + 1 < static_cast<int32_t>(p.max_depth)) {
			const uint32_t nv = w.guide.vertex_count[i];
			if (nv < w.guide.depth) {
				float4* r = w.guide.vertices + (static_cast<size_t>(i) * w.guide.depth + nv) * guide::kVertexFloat4;
				const float4* x = w.guide.query_in + 3 * i;
				r[0] = x[0];
				r[1] = x[1];
				r[2] = make_float4(x[2].x, wi.x, wi.y, wi.z);
				r[3] = make_float4(pb, beta0.x, beta0.y, beta0.z);
				r[4] = make_float4(L0.x, L0.y, L0.z, 0.f);
				w.guide.vertex_count[i] = nv + 1u;
			}
		}
	}
	return roulette(st, p.max_depth, p.rr_threshold);
}

__device__ bool shade_b_guided_any(const scene_view& s, const wave_buffers& w, const wave_params& p, uint32_t i,
	path_state& st, const shade_record& rec, const hit_t& sh, const hit_t& mh) {
	const uint32_t c = rec.pass_through ? CLASS_OTHER : class_of_material(static_cast<int32_t>(rec.material), s);
	switch (c) {
	case CLASS_LAMBERT: return shade_b_guided<class_material(CLASS_LAMBERT)>(s, w, p, i, st, rec, sh, mh);
	case CLASS_METAL: return shade_b_guided<class_material(CLASS_METAL)>(s, w, p, i, st, rec, sh, mh);
	case CLASS_GLASS_ROUGH: return shade_b_guided<class_material(CLASS_GLASS_ROUGH)>(s, w, p, i, st, rec, sh, mh);
	default: return shade_b_guided<MAT_ANY>(s, w, p, i, st, rec, sh, mh);
	}
}

// ------------------------------------------------------------------ wavefront
template <bool BATCH = false>
__device__ __forceinline__ pcg32 load_rng(const wave_buffers& w, const wave_params& p, uint32_t i) {
	pcg32 g;
	g.state = w.rng[i];
	const uint32_t seed = BATCH ? w.batch[w.scene[i]].seed : p.seed;
	g.inc = (stream_seed(w.pixel[i], w.sample[i], seed) << 1u) | 1u;
	return g;
}

// Scene of work item `item` of a batch: the last scene whose first item is <= item.
__device__ __forceinline__ uint32_t batch_scene_of_item(const wave_buffers& w, uint64_t item) {
	uint32_t lo = 0, hi = w.num_scenes;
	while (hi - lo > 1) {
		const uint32_t mid = (lo + hi) >> 1;
		if (w.batch[mid].item_base <= item) lo = mid;
		else hi = mid;
	}
	return lo;
}

// Scene of merged-film pixel g of a batch.
__device__ __forceinline__ uint32_t batch_scene_of_pixel(const wave_buffers& w, uint32_t g) {
	uint32_t lo = 0, hi = w.num_scenes;
	while (hi - lo > 1) {
		const uint32_t mid = (lo + hi) >> 1;
		if (w.batch[mid].pixel_base <= g) lo = mid;
		else hi = mid;
	}
	return lo;
}

template <bool BATCH = false>
__device__ __forceinline__ path_state load_path(const wave_buffers& w, const wave_params& p, uint32_t i) {
	path_state st;
	const float4 o = w.ray_o[i], d = w.ray_d[i], b = w.beta[i], L = w.radiance[i];
	st.o = vec3{o.x, o.y, o.z};
	st.len = o.w;
	st.d = vec3{d.x, d.y, d.z};
	st.beta = vec3{b.x, b.y, b.z};
	st.eta = b.w;
	st.L = vec3{L.x, L.y, L.z};
	st.flags = __float_as_uint(L.w);
	st.bounces = w.bounces[i];
	st.rng = load_rng<BATCH>(w, p, i);
	st.medium = w.medium != nullptr ? w.medium[i] : -1;
	return st;
}

__device__ __forceinline__ void store_path(const wave_buffers& w, uint32_t i, const path_state& st) {
	w.ray_o[i] = make_float4(st.o.x, st.o.y, st.o.z, st.len);
	w.ray_d[i] = make_float4(st.d.x, st.d.y, st.d.z, 0.f);
	w.beta[i] = make_float4(st.beta.x, st.beta.y, st.beta.z, st.eta);
	w.radiance[i] = make_float4(st.L.x, st.L.y, st.L.z, __uint_as_float(st.flags));
	w.bounces[i] = st.bounces;
	w.rng[i] = st.rng.state;
	if (w.medium != nullptr) w.medium[i] = st.medium;
}

// Queue of the paths of the subsurface stage: the medium class's segment of
// the class queues, which only volume renders use (those refuse subsurface
// materials).
__device__ __forceinline__ uint32_t* sss_queue(const wave_buffers& w) { return w.class_queue + CLASS_MEDIUM * w.capacity; }

__device__ __forceinline__ void finish(const wave_buffers& w, uint32_t i, vec3 L) {
	w.result[i] = make_float4(L.x, L.y, L.z, 1.f);
}

// Adds the finished samples of one wave to the film: one thread per pixel sums
// that pixel's paths of the wave in path order (plain adds, no atomics, so the
// accumulators do not depend on the launch order). Item k of the render is
// pixel k mod (width * height); path i of a wave is item first_item + i.
__global__ void __launch_bounds__(256) k_film_resolve(wave_buffers w, film_buffers f) {
	const wave_params& p = *w.params;
	const uint64_t pixels = static_cast<uint64_t>(p.width) * p.height;
	const uint64_t left = p.total_items > p.first_item ? p.total_items - p.first_item : 0;
	const uint32_t n = static_cast<uint32_t>(left < w.capacity ? left : w.capacity);
	const uint64_t shift = p.first_item % pixels;
	for (uint64_t px = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; px < pixels;
		 px += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
		double s0 = 0, s1 = 0, s2 = 0, q0 = 0, q1 = 0, q2 = 0;
		uint32_t c = 0;
		for (uint64_t i = (px + pixels - shift) % pixels; i < n; i += pixels) {
			const float4 L = w.result[i];
			if (L.w == 0.f) continue;
			s0 += L.x; s1 += L.y; s2 += L.z;
			q0 += static_cast<double>(L.x) * L.x;
			q1 += static_cast<double>(L.y) * L.y;
			q2 += static_cast<double>(L.z) * L.z;
			c++;
		}
		if (c == 0) continue;
		double* sp = f.sum + 3 * px;
		double* qp = f.sum_sq + 3 * px;
		sp[0] += s0; sp[1] += s1; sp[2] += s2;
		qp[0] += q0; qp[1] += q1; qp[2] += q2;
		f.count[px] += c;
	}
}

// k_film_resolve for a batch: merged-film pixel g of scene k has the items
// item_base + s * pixels + (g - pixel_base), s = 0 .. spp - 1; one thread per
// pixel of the scenes the wave overlaps sums that pixel's paths of the wave in
// path order (no atomics, as above).
__global__ void __launch_bounds__(256) k_film_resolve_batch(wave_buffers w, film_buffers f) {
	const wave_params& p = *w.params;
	const uint64_t first = p.first_item;
	const uint64_t left = p.total_items > first ? p.total_items - first : 0;
	const uint64_t n = left < w.capacity ? left : w.capacity;
	if (n == 0) return;
	const batch_scene& b0 = w.batch[batch_scene_of_item(w, first)];
	const batch_scene& b1 = w.batch[batch_scene_of_item(w, first + n - 1)];
	const uint32_t g0 = b0.pixel_base, g1 = b1.pixel_base + b1.width * b1.height;
	for (uint32_t g = g0 + blockIdx.x * blockDim.x + threadIdx.x; g < g1; g += gridDim.x * blockDim.x) {
		const batch_scene& b = w.batch[batch_scene_of_pixel(w, g)];
		const uint64_t px = static_cast<uint64_t>(b.width) * b.height;
		const uint64_t base = b.item_base + (g - b.pixel_base);  // the pixel's item of sample 0
		uint64_t s = base >= first ? 0 : (first - base + px - 1) / px;
		double s0 = 0, s1 = 0, s2 = 0, q0 = 0, q1 = 0, q2 = 0;
		uint32_t c = 0;
		for (; s < b.spp; s++) {
			const uint64_t item = base + s * px;
			if (item >= first + n) break;
			const float4 L = w.result[item - first];
			if (L.w == 0.f) continue;
			s0 += L.x; s1 += L.y; s2 += L.z;
			q0 += static_cast<double>(L.x) * L.x;
			q1 += static_cast<double>(L.y) * L.y;
			q2 += static_cast<double>(L.z) * L.z;
			c++;
		}
		if (c == 0) continue;
		double* sp = f.sum + 3 * static_cast<size_t>(g);
		double* qp = f.sum_sq + 3 * static_cast<size_t>(g);
		sp[0] += s0; sp[1] += s1; sp[2] += s2;
		qp[0] += q0; qp[1] += q1; qp[2] += q2;
		f.count[g] += c;
	}
}

// Per-pixel mean of the film (film::set_pixel's value after film::add_tile):
// rgb = sum / count in FP64, rounded once to float; 0 for a pixel without samples.
__global__ void __launch_bounds__(256) k_film_mean(film_buffers f, uint32_t pixels, float* __restrict__ rgb) {
	for (uint32_t px = blockIdx.x * blockDim.x + threadIdx.x; px < pixels; px += gridDim.x * blockDim.x) {
		const uint32_t c = f.count[px];
		const double* sp = f.sum + 3 * static_cast<size_t>(px);
		float* o = rgb + 3 * static_cast<size_t>(px);
		o[0] = c ? static_cast<float>(sp[0] / c) : 0.f;
		o[1] = c ? static_cast<float>(sp[1] / c) : 0.f;
		o[2] = c ? static_cast<float>(sp[2] / c) : 0.f;
	}
}

// sampler_integrator::render's per-sample set-up (sampler_integrator.cpp:102-126) for
// every work item of the wave; all of them enter the active queue.
// Batch: item -> (scene, sample, pixel) through the scene records, and the
// path remembers its scene.
template <bool BATCH>
__global__ void __launch_bounds__(256) k_camera(wave_buffers w, uint32_t queue_out) {
	const wave_params& p = *w.params;
	const uint64_t pixels = static_cast<uint64_t>(p.width) * p.height;
	for (uint32_t base = blockIdx.x * blockDim.x; base < w.capacity; base += gridDim.x * blockDim.x) {
		const uint32_t i = base + threadIdx.x;
		const uint64_t item = p.first_item + i;
		const bool valid = i < w.capacity && item < p.total_items;
		if (valid) {
			path_state st;
			uint32_t pixel, sample;
			if (BATCH) {
				const uint32_t k = batch_scene_of_item(w, item);
				const batch_scene& b = w.batch[k];
				const uint64_t local = item - b.item_base;
				const uint64_t px = static_cast<uint64_t>(b.width) * b.height;
				pixel = static_cast<uint32_t>(local % px);
				sample = b.first_sample + static_cast<uint32_t>(local / px);
				path_begin(st, b.r2c, b.c2w, b.lens, b.focus, pixel % b.width, pixel / b.width, pixel, sample, b.seed);
				w.scene[i] = k;
			} else {
				pixel = static_cast<uint32_t>(item % pixels);
				sample = p.first_sample + static_cast<uint32_t>(item / pixels);
				path_begin(st, p.r2c, p.c2w, p.lens, p.focus, pixel % p.width, pixel / p.width, pixel, sample, p.seed);
			}
			w.pixel[i] = pixel;
			w.sample[i] = sample;
			w.result[i] = make_float4(0.f, 0.f, 0.f, 0.f);
			if (p.guide_flags & GUIDE_TRAIN) {
				w.guide.vertex_count[i] = 0u;
				if (w.guide_medium.vertex_count != nullptr) w.guide_medium.vertex_count[i] = 0u;
			}
			store_path(w, i, st);
		}
		warp_push(valid, i, w.queue[queue_out], w.counters + CNT_ACTIVE);
	}
}

// The tracer pt::direct_radiance calls: the kernels' traversal on this
// thread's shared-memory stack; a full stack marks the sample failed.
template <bool COUNT>
struct thread_tracer {
	const scene_view* s;
	smem_stack* st;
	uint32_t* nodes;
	uint32_t* tris;
	uint32_t* rays;
	bool* ok;
	RB_HD hit_t operator()(vec3 o, vec3 d, float& len, bool shadow) const {
		hit_t h{-1, 0.f, 0.f};
#if defined(__CUDA_ARCH__)
		(*rays)++;
		const bool r = shadow ? trace_one<true, COUNT>(*s, o, d, len, h, *st, *nodes, *tris)
			: trace_one<false, COUNT>(*s, o, d, len, h, *st, *nodes, *tris);
		if (!r) {
			*ok = false;
			h.slot = -1;
		}
#endif
		return h;
	}
};

// direct_integrator (pt::direct_radiance) for every item of the wave, one
// thread per camera sample; the sample's radiance goes to w.result for the
// film resolve. Traced rays are counted as extension rays.
template <bool COUNT>
__global__ void __launch_bounds__(256) k_direct(scene_view s, wave_buffers w, direct_cfg dc, uint32_t stack_cap) {
	extern __shared__ uint32_t smem[];
	smem_stack st = make_stack(smem, stack_cap);
	const wave_params& p = *w.params;
	const uint64_t pixels = static_cast<uint64_t>(p.width) * p.height;
	uint32_t nodes = 0, tris = 0, rays = 0;
	bool ok = true;
	const thread_tracer<COUNT> tracer{&s, &st, &nodes, &tris, &rays, &ok};
	for (uint32_t base = blockIdx.x * blockDim.x; base < w.capacity; base += gridDim.x * blockDim.x) {
		const uint32_t i = base + threadIdx.x;
		const uint64_t item = p.first_item + i;
		if (i < w.capacity && item < p.total_items) {
			const uint32_t pixel = static_cast<uint32_t>(item % pixels);
			const uint32_t sample = p.first_sample + static_cast<uint32_t>(item / pixels);
			path_state ps;
			path_begin(ps, p.r2c, p.c2w, p.lens, p.focus, pixel % p.width, pixel / p.width, pixel, sample, p.seed);
			direct_radiance(s, dc, ps, tracer);
			w.result[i] = make_float4(ps.L.x, ps.L.y, ps.L.z, 1.f);
		}
	}
	if (!ok) set_error(w.counters, RB_ERR_STACK_OVERFLOW);
	warp_add64(w.counters, CNT_EXTEND_RAYS, rays);
	if (COUNT) {
		warp_add64(w.counters, CNT_NODE_VISITS, nodes);
		warp_add64(w.counters, CNT_TRI_TESTS, tris);
	}
}

__device__ __forceinline__ void put_ray(const direct_buffers& db, uint32_t slot, const ray_t& r) {
	db.ray_o[slot] = make_float4(r.o.x, r.o.y, r.o.z, r.len);
	db.ray_d[slot] = make_float4(r.d.x, r.d.y, r.d.z, 0.f);
}

// Staged direct lighting, first stage: the camera ray of every item of the
// wave (and its passes through lobeless surfaces) traced in the thread; a
// sample with a shaded surface is queued by the surface's material class for
// the light-sampling kernels, the others are finished here.
template <bool COUNT>
__global__ void __launch_bounds__(256) k_direct_surface(scene_view s, wave_buffers w, direct_buffers db, uint32_t stack_cap) {
	extern __shared__ uint32_t smem[];
	smem_stack st = make_stack(smem, stack_cap);
	const wave_params& p = *w.params;
	const uint64_t pixels = static_cast<uint64_t>(p.width) * p.height;
	uint32_t nodes = 0, tris = 0, rays = 0;
	bool ok = true;
	for (uint32_t base = blockIdx.x * blockDim.x; base < w.capacity; base += gridDim.x * blockDim.x) {
		const uint32_t i = base + threadIdx.x;
		const uint64_t item = p.first_item + i;
		uint32_t cls = CLASS_MISS;  // CLASS_MISS: nothing to queue
		if (i < w.capacity && item < p.total_items) {
			const uint32_t pixel = static_cast<uint32_t>(item % pixels);
			const uint32_t sample = p.first_sample + static_cast<uint32_t>(item / pixels);
			path_state ps;
			path_begin(ps, p.r2c, p.c2w, p.lens, p.focus, pixel % p.width, pixel / p.width, pixel, sample, p.seed);
			direct_record rec;
			int state = 1;
			for (int guard = 0; guard < 4096 && state == 1; guard++) {
				float len = ps.len;
				hit_t h;
				rays++;
				if (!trace_one<false, COUNT>(s, ps.o, ps.d, len, h, st, nodes, tris)) {
					ok = false;
					h.slot = -1;
				}
				state = direct_surface(s, ps, h, rec);
			}
			if (state == 2) {
				db.rec[i].si = rec.si;
				db.rec[i].material = rec.material;
				db.rec[i].round = 0u;
				store_path(w, i, ps);
				w.pixel[i] = pixel;  // the later stages rebuild the stream's increment from these
				w.sample[i] = sample;
				cls = class_of_material(static_cast<int32_t>(rec.material), s);
			} else {
				w.result[i] = make_float4(ps.L.x, ps.L.y, ps.L.z, 1.f);
			}
		}
#pragma unroll
		for (uint32_t c = CLASS_LAMBERT; c <= CLASS_OTHER; c++)
			warp_push(cls == c, i, w.class_queue + c * w.capacity, w.counters + CNT_CLASS + c);
	}
	if (!ok) set_error(w.counters, RB_ERR_STACK_OVERFLOW);
	warp_add64(w.counters, CNT_EXTEND_RAYS, rays);
	if (COUNT) {
		warp_add64(w.counters, CNT_NODE_VISITS, nodes);
		warp_add64(w.counters, CNT_TRI_TESTS, tris);
	}
}

// Staged direct lighting, second stage, for the shaded surfaces of one
// material class: the light samples and the first BSDF sample, their rays
// queued for the traversal kernel.
template <uint32_t CLASS>
__global__ void __launch_bounds__(256) k_direct_lights(scene_view s, wave_buffers w, direct_buffers db, direct_cfg dc) {
	const wave_params& p = *w.params;
	const uint32_t n = w.counters[CNT_CLASS + CLASS];
	const uint32_t* q = w.class_queue + CLASS * w.capacity;
	uint32_t rays = 0;
	for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
		const uint32_t k = base + threadIdx.x;
		uint32_t i = 0, push = 0u;  // bit j: slot j queued
		if (k < n) {
			i = q[k];
			path_state ps = load_path<false>(w, p, i);
			direct_record rec;
			rec.si = db.rec[i].si;
			rec.material = db.rec[i].material;
			rec.round = 0u;
			ray_t out[kDirectSlots];
			direct_sample_lights<class_material(CLASS)>(s, dc, ps, rec, out);
			for (uint32_t j = 0; j < dc.emitter_samples; j++)
				if (rec.light_entity[j] >= 0) {
					put_ray(db, i * kDirectSlots + j, out[j]);
					push |= 1u << j;
				}
			if (rec.bsdf_valid) {
				put_ray(db, i * kDirectSlots + dc.emitter_samples, out[dc.emitter_samples]);
				push |= 1u << dc.emitter_samples;
			}
			db.rec[i] = rec;
			store_path(w, i, ps);
		}
		for (uint32_t j = 0; j <= dc.emitter_samples; j++)
			warp_push((push >> j) & 1u, i * kDirectSlots + j, db.ray_queue, w.counters + CNT_SECONDARY);
		rays += __popc(push);
	}
	warp_add64(w.counters, CNT_EXTEND_RAYS, rays);
}

// Staged direct lighting, one round per BSDF sample over one material class's
// shaded paths: the traced hits of the pending rays (in the first round also
// the light samples'), then the next BSDF sample's ray queued, or the sample
// finished.
template <uint32_t CLASS>
__global__ void __launch_bounds__(256) k_direct_round(scene_view s, wave_buffers w, direct_buffers db, direct_cfg dc) {
	const wave_params& p = *w.params;
	const uint32_t n = w.counters[CNT_CLASS + CLASS];
	const uint32_t* q = w.class_queue + CLASS * w.capacity;
	uint32_t rays = 0;
	for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
		const uint32_t k = base + threadIdx.x;
		bool push = false;
		uint32_t i = 0;
		if (k < n) {
			i = q[k];
			path_state ps = load_path<false>(w, p, i);
			direct_record rec = db.rec[i];
			const uint32_t slot0 = i * kDirectSlots;
			hit_t lh[kDirectStagedLights];
			for (uint32_t j = 0; j < kDirectStagedLights; j++) {
				lh[j] = hit_t{-1, 0.f, 0.f};
				if (rec.round == 0u && j < dc.emitter_samples && rec.light_entity[j] >= 0) lh[j] = to_hit(db.ray_hit[slot0 + j]);
			}
			const hit_t bh = rec.bsdf_valid ? to_hit(db.ray_hit[slot0 + dc.emitter_samples]) : hit_t{-1, 0.f, 0.f};
			ray_t out;
			if (direct_round<class_material(CLASS)>(s, dc, ps, rec, lh, bh, out)) {
				if (rec.bsdf_valid) {
					put_ray(db, slot0 + dc.emitter_samples, out);
					push = true;
				}
				db.rec[i] = rec;
				store_path(w, i, ps);
			} else {
				w.result[i] = make_float4(ps.L.x, ps.L.y, ps.L.z, 1.f);
			}
		}
		warp_push(push, i * kDirectSlots + dc.emitter_samples, db.ray_queue, w.counters + CNT_SECONDARY);
		rays += push ? 1u : 0u;
	}
	warp_add64(w.counters, CNT_EXTEND_RAYS, rays);
}

template <bool COUNT, bool VOL, bool BATCH, bool INST>
__global__ void __launch_bounds__(256) k_extend(scene_view s, wave_buffers w, uint32_t queue_in, uint32_t stack_cap,
	uint32_t sort) {
	extern __shared__ uint32_t smem[];
	launch_timer_begin(w.counters, CNT_TIMER_EXTEND);
	smem_stack st = make_stack(smem, stack_cap);
	const uint32_t n = w.counters[CNT_ACTIVE];
	const uint32_t* q = w.queue[queue_in];
	uint32_t nodes = 0, tris = 0;
	for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
		const uint32_t k = base + threadIdx.x;
		uint32_t key = 0xffffffffu, i = 0;
		if (k < n) {
			i = q[k];
			const float4 o = w.ray_o[i], d = w.ray_d[i];
			float len = o.w;
			hit_t h;
			bool ok;
			if (BATCH) {
				const scene_view sv = batch_view(s, w.batch[w.scene[i]]);
				ok = trace_one<false, COUNT, INST>(sv, vec3{o.x, o.y, o.z}, vec3{d.x, d.y, d.z}, len, h, st, nodes, tris);
			} else {
				ok = trace_one<false, COUNT, INST>(s, vec3{o.x, o.y, o.z}, vec3{d.x, d.y, d.z}, len, h, st, nodes, tris);
			}
			if (!ok) {
				set_error(w.counters, RB_ERR_STACK_OVERFLOW);
				h.slot = -1;
			}
			w.hit[i] = make_float4(__uint_as_float(static_cast<uint32_t>(h.slot)), len, h.b1, h.b2);
			key = (VOL && w.medium[i] >= 0) ? static_cast<uint32_t>(CLASS_MEDIUM) : shade_class(s, h.slot);
			if (sort == RB_SORT_NONE && key != CLASS_MISS && key != CLASS_MEDIUM) key = CLASS_OTHER;
		}
		warp_push_keyed(key, i, w.class_queue, w.capacity, w.counters + CNT_CLASS);
	}
	if (COUNT) {
		warp_add64(w.counters, CNT_NODE_VISITS, nodes);
		warp_add64(w.counters, CNT_TRI_TESTS, tris);
	}
	launch_timer_end(w.counters, CNT_TIMER_EXTEND);
}

// ------------------------------------------------------------------ ray binning
// RB_SORT_RAYS: before a bounce's traversal the active queue is reordered by a
// 12-bit key, the ray direction's octant over an 8x8x8 Morton cell of its
// origin in the scene box, with a counting sort (per-block histograms, one scan,
// warp-aggregated scatter). Rays of a warp then start near each other in the
// same direction, which keeps their traversals together and their nodes in
// cache. Only the order of the queue changes, never a path's arithmetic.
__device__ __forceinline__ uint32_t ray_bin(const wave_params& p, float4 o, float4 d) {
	const uint32_t oct = (d.x < 0.f ? 1u : 0u) | (d.y < 0.f ? 2u : 0u) | (d.z < 0.f ? 4u : 0u);
	const float v[3] = {o.x, o.y, o.z};
	uint32_t morton = 0;
	for (int j = 0; j < 3; j++) {
		const float u = (v[j] - p.box_min[j]) * p.box_inv[j] * 8.f;
		const uint32_t c = u > 0.f ? (u < 7.f ? static_cast<uint32_t>(u) : 7u) : 0u;  // NaN and negatives: cell 0
		for (int b = 0; b < 3; b++) morton |= ((c >> b) & 1u) << (3 * b + j);
	}
	return (oct << 9) | morton;
}

__global__ void __launch_bounds__(256) k_bin_count(wave_buffers w, uint32_t queue_in) {
	__shared__ uint32_t hist[kSortBins];
	for (uint32_t b = threadIdx.x; b < kSortBins; b += blockDim.x) hist[b] = 0u;
	__syncthreads();
	const wave_params& p = *w.params;
	const uint32_t n = w.counters[CNT_ACTIVE];
	const uint32_t* q = w.queue[queue_in];
	for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
		const uint32_t i = q[k];
		const uint32_t key = ray_bin(p, w.ray_o[i], w.ray_d[i]);
		w.sort_keys[k] = key;
		atomicAdd(&hist[key], 1u);
	}
	__syncthreads();
	for (uint32_t b = threadIdx.x; b < kSortBins; b += blockDim.x)
		if (hist[b] != 0u) atomicAdd(w.sort_bins + b, hist[b]);
}

// One block of 1024 threads: exclusive prefix of the bin counts into the
// cursors, counts cleared for the next bounce.
__global__ void __launch_bounds__(1024) k_bin_scan(wave_buffers w) {
	__shared__ uint32_t part[1024];
	constexpr uint32_t per = kSortBins / 1024;
	const uint32_t t = threadIdx.x;
	uint32_t c[per], sum = 0;
	for (uint32_t j = 0; j < per; j++) {
		c[j] = w.sort_bins[t * per + j];
		sum += c[j];
	}
	part[t] = sum;
	__syncthreads();
	for (uint32_t off = 1; off < 1024; off <<= 1) {  // inclusive Hillis-Steele scan of the per-thread sums
		const uint32_t v = t >= off ? part[t - off] : 0u;
		__syncthreads();
		part[t] += v;
		__syncthreads();
	}
	uint32_t run = part[t] - sum;
	for (uint32_t j = 0; j < per; j++) {
		w.sort_bins[kSortBins + t * per + j] = run;
		w.sort_bins[t * per + j] = 0u;
		run += c[j];
	}
}

__global__ void __launch_bounds__(256) k_bin_scatter(wave_buffers w, uint32_t queue_in) {
	const uint32_t n = w.counters[CNT_ACTIVE];
	const uint32_t* q = w.queue[queue_in];
	uint32_t* cursor = w.sort_bins + kSortBins;
	for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
		const uint32_t k = base + threadIdx.x;
		const uint32_t key = k < n ? w.sort_keys[k] : 0xffffffffu;
		const uint32_t peers = __match_any_sync(0xffffffffu, key);
		const uint32_t leader = __ffs(peers) - 1;
		uint32_t pos = 0;
		if ((threadIdx.x & 31u) == leader && key != 0xffffffffu) pos = atomicAdd(cursor + key, static_cast<uint32_t>(__popc(peers)));
		pos = __shfl_sync(0xffffffffu, pos, leader);
		if (k < n) w.sort_tmp[pos + __popc(peers & lanemask_lt())] = q[k];
	}
}

__global__ void __launch_bounds__(256) k_bin_copy(wave_buffers w, uint32_t queue_in) {
	const uint32_t n = w.counters[CNT_ACTIVE];
	uint32_t* q = w.queue[queue_in];
	for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) q[k] = w.sort_tmp[k];
}

// ------------------------------------------------------------------ persistent traversal
// Lanes take rays one at a time from a queue (one atomic per warp for all the
// lanes that need a ray) and advance them one node or leaf per iteration, so a
// warp stays full until the queue is empty instead of idling while its longest
// ray finishes. Each ray sees exactly the operations of closest_hit_fast.
struct ray_fetch {
	bool exhausted = false;
	// Gives lanes without a ray the next queue positions; k >= n: none left.
	__device__ __forceinline__ bool take(bool need_ray, uint32_t* counter, uint32_t n, uint32_t& k) {
		const uint32_t need = __ballot_sync(0xffffffffu, need_ray);
		if (need == 0u || exhausted) return false;
		const uint32_t lane = threadIdx.x & 31u, leader = __ffs(need) - 1;
		uint32_t base = 0;
		if (lane == leader) base = atomicAdd(counter, static_cast<uint32_t>(__popc(need)));
		base = __shfl_sync(0xffffffffu, base, leader);
		if (base + static_cast<uint32_t>(__popc(need)) >= n) exhausted = true;
		k = base + __popc(need & lanemask_lt());
		return need_ray && k < n;
	}
};

// The reference-order redo of a ray the 4-wide walk gave up on.
template <bool SHADOW>
__device__ __forceinline__ bool trace_exact(const scene_view& sv, vec3 o, vec3 d, float& len, hit_t& h, smem_stack& st) {
	trace_counters c{0u, 0u};
	return closest_hit<SHADOW, false>(sv, o, d, len, h, st, c);
}

template <bool VOL, bool BATCH>
__global__ void __launch_bounds__(256) k_extend_refill(scene_view s, wave_buffers w, uint32_t queue_in, uint32_t stack_cap,
	uint32_t sort) {
	extern __shared__ uint32_t smem[];
	launch_timer_begin(w.counters, CNT_TIMER_EXTEND);
	smem_stack st = make_stack(smem, stack_cap);
	const uint32_t n = w.counters[CNT_ACTIVE];
	const uint32_t* q = w.queue[queue_in];
	ray_fetch fetch;
	trav_state t;
	uint32_t i = 0;
	float len0 = 0.f;
	bool active = false;
	for (;;) {
		bool finished = false, ok = true;
		hit_t h{-1, 0.f, 0.f};
		float len = 0.f;
		uint32_t k;
		if (fetch.take(!active, w.counters + CNT_FETCH_EXTEND, n, k)) {
			i = q[k];
			const float4 o = w.ray_o[i], d = w.ray_d[i];
			const vec3 o3{o.x, o.y, o.z}, d3{d.x, d.y, d.z};
			len0 = o.w;
			const scene_view sv = BATCH ? batch_view(s, w.batch[w.scene[i]]) : s;
			if (isnan(len0) || sv.wnodes == nullptr) {
				len = len0;
				ok = trace_exact<false>(sv, o3, d3, len, h, st);
				finished = true;
			} else if (trav_begin(sv, t, o3, d3, len0, st)) {
				active = true;
			} else {
				len = len0;
				finished = true;
			}
		}
		if (active) {
			const int r = trav_step<false>(s, t, st);
			if (r != 0) {
				active = false;
				finished = true;
				if (r > 0) {
					h = t.hit;
					len = t.len;
				} else {
					const scene_view sv = BATCH ? batch_view(s, w.batch[w.scene[i]]) : s;
					len = len0;
					ok = trace_exact<false>(sv, t.o, t.d, len, h, st);
				}
			}
		}
		uint32_t key = 0xffffffffu;
		if (finished) {
			if (!ok) {
				set_error(w.counters, RB_ERR_STACK_OVERFLOW);
				h.slot = -1;
			}
			w.hit[i] = make_float4(__uint_as_float(static_cast<uint32_t>(h.slot)), len, h.b1, h.b2);
			key = (VOL && w.medium[i] >= 0) ? static_cast<uint32_t>(CLASS_MEDIUM) : shade_class(s, h.slot);
			if (sort == RB_SORT_NONE && key != CLASS_MISS && key != CLASS_MEDIUM) key = CLASS_OTHER;
		}
		if (__any_sync(0xffffffffu, finished)) warp_push_keyed(key, i, w.class_queue, w.capacity, w.counters + CNT_CLASS);
		if (fetch.exhausted && !__any_sync(0xffffffffu, active)) break;
	}
	launch_timer_end(w.counters, CNT_TIMER_EXTEND);
}

template <bool BATCH>
__global__ void __launch_bounds__(256) k_secondary_refill(scene_view s, wave_buffers w, uint32_t stack_cap) {
	extern __shared__ uint32_t smem[];
	launch_timer_begin(w.counters, CNT_TIMER_SECONDARY);
	smem_stack st = make_stack(smem, stack_cap);
	const uint32_t n = w.counters[CNT_SECONDARY];
	ray_fetch fetch;
	trav_state t;
	uint32_t j = 0;
	float len0 = 0.f;
	bool active = false;
	for (;;) {
		bool finished = false, ok = true;
		hit_t h{-1, 0.f, 0.f};
		float len = 0.f;
		uint32_t k;
		if (fetch.take(!active, w.counters + CNT_FETCH_SECONDARY, n, k)) {
			j = w.sec_queue[k];
			const float4 o = w.sec_o[j], d = w.sec_d[j];
			const vec3 o3{o.x, o.y, o.z}, d3{d.x, d.y, d.z};
			len0 = o.w;
			const scene_view sv = BATCH ? batch_view(s, w.batch[w.scene[j >> 1]]) : s;
			if (isnan(len0) || sv.wnodes == nullptr) {
				len = len0;
				ok = trace_exact<true>(sv, o3, d3, len, h, st);
				finished = true;
			} else if (trav_begin(sv, t, o3, d3, len0, st)) {
				active = true;
			} else {
				len = len0;
				finished = true;
			}
		}
		if (active) {
			const int r = trav_step<true>(s, t, st);
			if (r != 0) {
				active = false;
				finished = true;
				if (r > 0) {
					h = t.hit;
					len = t.len;
				} else {
					const scene_view sv = BATCH ? batch_view(s, w.batch[w.scene[j >> 1]]) : s;
					len = len0;
					ok = trace_exact<true>(sv, t.o, t.d, len, h, st);
				}
			}
		}
		if (finished) {
			if (!ok) {
				set_error(w.counters, RB_ERR_STACK_OVERFLOW);
				h.slot = -1;
			}
			w.sec_hit[j] = make_float4(__uint_as_float(static_cast<uint32_t>(h.slot)), len, h.b1, h.b2);
		}
		if (fetch.exhausted && !__any_sync(0xffffffffu, active)) break;
	}
	launch_timer_end(w.counters, CNT_TIMER_SECONDARY);
}

template <uint32_t CLASS, bool VOL, bool BATCH>
__global__ void __launch_bounds__(256) k_shade_a(scene_view s_all, wave_buffers w) {
	const wave_params& p = *w.params;
	const uint32_t n = w.counters[CNT_CLASS + CLASS];
	const uint32_t* q = w.class_queue + CLASS * w.capacity;
	for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
		const uint32_t k = base + threadIdx.x;
		bool push_shadow = false, push_mis = false, push_guide = false;
		uint32_t i = 0;
		if (k < n) {
			i = q[k];
			path_state st = load_path<BATCH>(w, p, i);
			const scene_view s = BATCH ? batch_view(s_all, w.batch[w.scene[i]]) : s_all;
			if (CLASS == CLASS_MISS) {
				shade_miss(s, st);
				finish(w, i, st.L);
				st.flags |= 0x80000000u;  // ended in shade_a; shade_b skips it
			} else {
				shade_record& r = w.rec[i];
				vol_rec* vr = nullptr;
				if (VOL) {
					vr = w.vrec + i;
					vr->flags = 0u;
					vr->medium = st.medium;
				}
				const bool alive = shade_a<class_material(CLASS)>(s, st, to_hit(w.hit[i]), r, vr);
				if (!alive) {
					finish(w, i, st.L);
					st.flags |= 0x80000000u;
				} else {
					push_shadow = r.nee_entity >= 0;
					push_mis = r.mis_valid != 0;
					if (push_shadow) {
						const ray_t& sr = r.shadow_ray;
						w.sec_o[2 * i] = make_float4(sr.o.x, sr.o.y, sr.o.z, sr.len);
						w.sec_d[2 * i] = make_float4(sr.d.x, sr.d.y, sr.d.z, 0.f);
					}
					if (push_mis) {
						const ray_t& mr = r.mis_ray;
						w.sec_o[2 * i + 1] = make_float4(mr.o.x, mr.o.y, mr.o.z, mr.len);
						w.sec_d[2 * i + 1] = make_float4(mr.d.x, mr.d.y, mr.d.z, 0.f);
					}
					if (p.guide_flags != 0u && r.guidable && !r.pass_through) {
						write_guide_query(p, r.si, w.guide.query_in + 3 * i);
						push_guide = (p.guide_flags & GUIDE_SAMPLE) && *w.guide.usable != 0u;
					}
				}
			}
			store_path(w, i, st);
		}
		warp_push(push_shadow, 2 * i, w.sec_queue, w.counters + CNT_SECONDARY);
		warp_push(push_mis, 2 * i + 1, w.sec_queue, w.counters + CNT_SECONDARY);
		if (CLASS != CLASS_MISS && p.guide_flags != 0u) warp_push(push_guide, i, w.guide.queue, w.counters + CNT_GUIDE);
		const uint32_t ns = __popc(__ballot_sync(0xffffffffu, push_shadow));
		const uint32_t nm = __popc(__ballot_sync(0xffffffffu, push_mis));
		if ((threadIdx.x & 31u) == 0) {
			if (ns) add64(w.counters, CNT_SHADOW_RAYS, ns);
			if (nm) add64(w.counters, CNT_MIS_RAYS, nm);
		}
	}
}

// Secondary rays: 2 i is path i's NEE shadow ray, 2 i + 1 its MIS ray (closest
// visible hits). shadow_first (plain path-tracing bounces only): the shadow ray
// is answered as an occlusion query. The reference accepts it when its closest
// visible hit is the sampled emitter or nothing (integrator.cpp:131-136), that
// is, when no other visible hit lies closer than the emitter's own closest hit;
// so the emitter's triangles are tested first, the ray is cut at that hit, and
// the traversal stops at the first occluder found before it (shade_b needs only
// whether the hit slot is the emitter, nothing or something else). Emitters of
// more than kShadowFirstTris triangles keep the closest-hit query.
constexpr uint32_t kShadowFirstTris = 64;
template <bool COUNT, bool BATCH, bool INST>
__global__ void __launch_bounds__(256) k_trace_secondary(scene_view s, wave_buffers w, uint32_t stack_cap,
	uint32_t shadow_first) {
	extern __shared__ uint32_t smem[];
	launch_timer_begin(w.counters, CNT_TIMER_SECONDARY);
	smem_stack st = make_stack(smem, stack_cap);
	const uint32_t n = w.counters[CNT_SECONDARY];
	uint32_t nodes = 0, tris = 0;
	for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
		const uint32_t k = base + threadIdx.x;
		if (k < n) {
			const uint32_t j = w.sec_queue[k];
			const float4 o = w.sec_o[j], d = w.sec_d[j];
			float len = o.w;
			hit_t h;
			bool ok;
			const scene_view sv = BATCH ? batch_view(s, w.batch[w.scene[j >> 1]]) : s;
			const vec3 o3{o.x, o.y, o.z}, d3{d.x, d.y, d.z};
			bool first = false;
			if (!COUNT && shadow_first && !(j & 1u)) {
				const int32_t e = w.rec[j >> 1].nee_entity;
				float cut;
				if (e >= 0 && entity_closest_length(sv, static_cast<uint32_t>(e), o3, d3, len, kShadowFirstTris, cut)) {
					len = cut;
					first = true;
				}
			}
			ok = trace_one<true, COUNT, INST>(sv, o3, d3, len, h, st, nodes, tris, first);
			if (!ok) {
				set_error(w.counters, RB_ERR_STACK_OVERFLOW);
				h.slot = -1;
			}
			w.sec_hit[j] = make_float4(__uint_as_float(static_cast<uint32_t>(h.slot)), len, h.b1, h.b2);
		}
	}
	if (COUNT) {
		warp_add64(w.counters, CNT_NODE_VISITS, nodes);
		warp_add64(w.counters, CNT_TRI_TESTS, tris);
	}
	launch_timer_end(w.counters, CNT_TIMER_SECONDARY);
}

template <uint32_t CLASS, bool BATCH>
__global__ void __launch_bounds__(256) k_shade_b(scene_view s_all, wave_buffers w, uint32_t queue_in) {
	const wave_params& p = *w.params;
	const uint32_t n = w.counters[CNT_CLASS + CLASS];
	const uint32_t* q = w.class_queue + CLASS * w.capacity;
	uint32_t* qn = w.queue[queue_in ^ 1u];
	for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
		const uint32_t k = base + threadIdx.x;
		bool alive = false, sss = false;
		uint32_t i = 0;
		if (k < n) {
			i = q[k];
			path_state st = load_path<BATCH>(w, p, i);
			if (!(st.flags & 0x80000000u)) {
				const scene_view s = BATCH ? batch_view(s_all, w.batch[w.scene[i]]) : s_all;
				const shade_record& rec = w.rec[i];
				const hit_t sh = to_hit(w.sec_hit[2 * i]);
				const hit_t mh = to_hit(w.sec_hit[2 * i + 1]);
				if (!BATCH && p.guide_flags != 0u)
					alive = CLASS == CLASS_OTHER ? shade_b_guided_any(s, w, p, i, st, rec, sh, mh)
						: shade_b_guided<class_material(CLASS)>(s, w, p, i, st, rec, sh, mh);
				else
					alive = CLASS == CLASS_OTHER ? shade_b_any(s, st, rec, sh, mh, p.max_depth, p.rr_threshold)
						: shade_b<class_material(CLASS)>(s, st, rec, sh, mh, p.max_depth, p.rr_threshold);
				if (!alive) finish(w, i, st.L);
				store_path(w, i, st);
				// paths whose BSDF sample entered a subsurface material go on in k_subsurface
				sss = CLASS == CLASS_OTHER && alive && (st.flags & PATH_SSS);
			}
		}
		if (CLASS == CLASS_OTHER) {
			warp_push(sss, i, sss_queue(w), w.counters + CNT_SSS);
			alive = alive && !sss;
		}
		warp_push(alive, i, qn, w.counters + CNT_NEXT);
	}
}

// ------------------------------------------------------------------ subsurface
// The BSSRDF stage of the paths that k_shade_b<CLASS_OTHER> queued: a path
// whose BSDF sample transmitted into a subsurface material takes its exit
// point, the light sample there and its continuation
// (sample_scattering_surface_function, integrator.cpp:290-327), then Russian
// roulette, as path_integrator::trace orders them (path_integrator.cpp:30-43).
// The probe rays and the exit's shadow and MIS rays are traced in the thread:
// few paths reach this stage, and each needs two probe walks whose lengths
// depend on the geometry.
// Counting passes count the stage's rays but not their box and triangle tests.
template <bool BATCH, bool INST>
__global__ void __launch_bounds__(256) k_subsurface(scene_view s_all, wave_buffers w, uint32_t queue_in, uint32_t stack_cap) {
	extern __shared__ uint32_t smem[];
	smem_stack stk = make_stack(smem, stack_cap);
	const wave_params& p = *w.params;
	const uint32_t n = w.counters[CNT_SSS];
	const uint32_t* q = sss_queue(w);
	uint32_t* qn = w.queue[queue_in ^ 1u];
	uint32_t nprobe = 0, nshadow = 0;
	for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
		const uint32_t k = base + threadIdx.x;
		bool alive = false;
		uint32_t i = 0;
		if (k < n) {
			i = q[k];
			path_state st = load_path<BATCH>(w, p, i);
			const scene_view s = BATCH ? batch_view(s_all, w.batch[w.scene[i]]) : s_all;
			bool failed = false;
			auto trace = [&](vec3 o, vec3 d, float& len, bool shadow) {
				if (shadow) nshadow++;
				else nprobe++;
				return trace_out_of_line<INST>(s, o, d, len, shadow, stk, failed);
			};
			st.flags &= ~PATH_SSS;
			alive = subsurface_walk(s, st, w.rec[i], to_hit(w.hit[i]), trace) && roulette(st, p.max_depth, p.rr_threshold);
			if (failed) set_error(w.counters, RB_ERR_STACK_OVERFLOW);
			if (!alive) finish(w, i, st.L);
			store_path(w, i, st);
		}
		warp_push(alive, i, qn, w.counters + CNT_NEXT);
	}
	warp_add64(w.counters, CNT_EXTEND_RAYS, nprobe);
	warp_add64(w.counters, CNT_SHADOW_RAYS, nshadow);
}

// ------------------------------------------------------------------ tail
// The rest of every active path in one launch. Late bounces hold few paths,
// and their per-bounce launches cost more than their work, so from bounce
// `tail` on one thread carries each surviving path through all its remaining
// bounces with the same stage functions as the wavefront (extend -> shade_a ->
// shadow and MIS rays -> shade_b) and the same random-number order, so every
// sample's radiance is the same as without the tail. Lanes whose path ends
// take the next path from the active queue (one atomic per warp for all lanes
// that need one), so long paths do not idle the rest of their warp.
template <bool COUNT, bool BATCH>
__global__ void __launch_bounds__(256) k_tail(scene_view s_all, wave_buffers w, uint32_t queue_in, uint32_t stack_cap) {
	extern __shared__ uint32_t smem[];
	smem_stack stk = make_stack(smem, stack_cap);
	const wave_params& p = *w.params;
	const uint32_t n = w.counters[CNT_ACTIVE];
	const uint32_t* q = w.queue[queue_in];
	const uint32_t lane = threadIdx.x & 31u;
	uint32_t nodes = 0, tris = 0, ext = 0, nshadow = 0, nmis = 0;
	bool have = false, exhausted = false, first = false;
	uint32_t i = 0;
	int guard = 0;
	path_state st;
	for (;;) {
		const uint32_t need = __ballot_sync(0xffffffffu, !have);
		if (need != 0u && !exhausted) {
			const uint32_t leader = __ffs(need) - 1;
			uint32_t base = 0;
			if (lane == leader) base = atomicAdd(w.counters + CNT_TAIL, static_cast<uint32_t>(__popc(need)));
			base = __shfl_sync(0xffffffffu, base, leader);
			if (base + static_cast<uint32_t>(__popc(need)) >= n) exhausted = true;
			if (!have) {
				const uint32_t k = base + __popc(need & lanemask_lt());
				if (k < n) {
					i = q[k];
					st = load_path<BATCH>(w, p, i);
					have = true;
					first = true;
					guard = 0;
				}
			}
		}
		if (!__any_sync(0xffffffffu, have)) break;
		if (have) {
			const scene_view s = BATCH ? batch_view(s_all, w.batch[w.scene[i]]) : s_all;
			bool alive = false;
			float len = st.len;
			hit_t h;
			if (!first) ext++;  // the first extend ray of each path is counted with the queue (k_advance)
			first = false;
			if (!trace_one<false, COUNT>(s, st.o, st.d, len, h, stk, nodes, tris)) {
				set_error(w.counters, RB_ERR_STACK_OVERFLOW);
			} else {
				shade_record rec;
				if (shade_a_any(s, st, h, rec)) {
					hit_t sh{-1, 0.f, 0.f}, mh{-1, 0.f, 0.f};
					bool ok = true;
					if (rec.nee_entity >= 0) {
						float l = rec.shadow_ray.len;
						nshadow++;
						ok = trace_one<true, COUNT>(s, rec.shadow_ray.o, rec.shadow_ray.d, l, sh, stk, nodes, tris);
					}
					if (ok && rec.mis_valid) {
						float l = rec.mis_ray.len;
						nmis++;
						ok = trace_one<true, COUNT>(s, rec.mis_ray.o, rec.mis_ray.d, l, mh, stk, nodes, tris);
					}
					if (!ok) set_error(w.counters, RB_ERR_STACK_OVERFLOW);
					else alive = shade_b_any(s, st, rec, sh, mh, p.max_depth, p.rr_threshold) && ++guard < 4096;
				}
			}
			if (!alive) {
				finish(w, i, st.L);
				have = false;
			}
		}
	}
	warp_add64(w.counters, CNT_EXTEND_RAYS, ext);
	warp_add64(w.counters, CNT_SHADOW_RAYS, nshadow);
	warp_add64(w.counters, CNT_MIS_RAYS, nmis);
	if (COUNT) {
		warp_add64(w.counters, CNT_NODE_VISITS, nodes);
		warp_add64(w.counters, CNT_TRI_TESTS, tris);
	}
}

// ------------------------------------------------------------------ volume path tracing
// volume_path_integrator::trace (volume_path_integrator.cpp:13-79) per bounce:
// extend -> shade_a (surface classes, and CLASS_MEDIUM: free-flight sampling,
// then a medium vertex or the surface reached) -> shadow / MIS rays ->
// k_vol_direct (what each light connection found) -> k_beam (transmittance of
// each connection through invisible medium boundaries) -> k_vol_continue
// (accumulate, continue by BSDF or phase function, switch media, roulette).
// The random numbers are drawn in the reference's order; the transmittance
// walks draw none.

// Emitter sampling and phase sampling at a medium vertex, the first half of
// uniform_sample_one_emitter for a medium_interaction (integrator.cpp:203-288).
__device__ void medium_vertex_a(const scene_view& s, path_state& p, shade_record& rec, vol_rec& vr, const medium_rec& m,
	float t) {
	const vec3 point = p.o + p.d * t;
	const vec3 wo = -p.d;
	const vec3 zero{0.f, 0.f, 0.f};
	vr.flags = VOL_MEDIUM_VERTEX;
	vr.g = m.g;
	rec.pass_through = 0u;
	rec.did_nee = 1u;
	rec.guidable = 0u;
	rec.nee_entity = -1;
	rec.mis_valid = 0u;
	rec.si.p = point;
	rec.si.n = zero;
	rec.si.wo = wo;
	rec.si.entity = -1;
	const float n = static_cast<float>(s.num_emitters);
	uint32_t which = static_cast<uint32_t>(floorf(pcg_real(p.rng) * n));
	if (which > s.num_emitters - 1) which = s.num_emitters - 1;
	const emitter_rec& em = s.emitters[which];
	light_sample ls = sample_emitter(s, em, point, zero, pcg_2d(p.rng));
	ls.pdf = ls.pdf * (1.f / n);
	if (!is_black(ls.L) && ls.pdf > 0.f) {
		const float ph = hg_phase(dot(wo, ls.wi), m.g);
		const spectrum fv = splat3(ph);
		if (!is_black(fv) && ph > 0.f) {
			rec.shadow_ray = spawn_ray_to(point, zero, ls.p);
			rec.nee_entity = em.entity;
			vr.nee_f = fv;
			vr.nee_Le = ls.L;
			vr.nee_w = power_heuristic(ls.pdf, ph);
			vr.nee_pdf = ls.pdf;
			vr.nee_to = ls.p;
		}
	}
	vec3 wi;
	const float ph = hg_sample(wo, m.g, pcg_2d(p.rng), wi);
	const spectrum fv = splat3(ph);
	if (!is_black(fv) && ph > 0.f) {
		rec.mis_valid = 1u;
		rec.mis_specular = 0u;
		rec.mis_wi = wi;
		rec.mis_f = fv;
		rec.mis_pdf = ph;
		rec.mis_ray = spawn_ray(point, zero, wi);
	}
}

// Paths inside a medium: homogeneous_medium::sample over the segment to the
// closest hit (or to infinity on a miss), then a medium vertex or the surface.
__global__ void __launch_bounds__(256) k_shade_a_medium(scene_view s, wave_buffers w) {
	const wave_params& p = *w.params;
	const uint32_t n = w.counters[CNT_CLASS + CLASS_MEDIUM];
	const uint32_t* q = w.class_queue + CLASS_MEDIUM * w.capacity;
	for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
		const uint32_t k = base + threadIdx.x;
		bool push_shadow = false, push_mis = false, push_guide = false, push_guide_m = false;
		uint32_t i = 0;
		if (k < n) {
			i = q[k];
			path_state st = load_path(w, p, i);
			shade_record& r = w.rec[i];
			vol_rec& vr = w.vrec[i];
			vr.flags = 0u;
			vr.medium = st.medium;
			const float4 hv = w.hit[i];
			const medium_rec& m = s.mediums[st.medium];
			const float u_channel = pcg_real(st.rng);
			const float u_distance = pcg_real(st.rng);
			const medium_event ev = sample_medium(m, hv.y, u_channel, u_distance);
			st.beta = st.beta * ev.weight;
			bool alive;
			if (is_black(st.beta)) {
				alive = false;
			} else if (ev.scattered) {
				medium_vertex_a(s, st, r, vr, m, ev.t);
				alive = true;
			} else {
				alive = shade_a<MAT_ANY>(s, st, to_hit(hv), r, &vr);
			}
			if (!alive) {
				finish(w, i, st.L);
				st.flags |= 0x80000000u;
			} else {
				push_shadow = r.nee_entity >= 0;
				push_mis = r.mis_valid != 0;
				if (push_shadow) {
					const ray_t& sr = r.shadow_ray;
					w.sec_o[2 * i] = make_float4(sr.o.x, sr.o.y, sr.o.z, sr.len);
					w.sec_d[2 * i] = make_float4(sr.d.x, sr.d.y, sr.d.z, 0.f);
				}
				if (push_mis) {
					const ray_t& mr = r.mis_ray;
					w.sec_o[2 * i + 1] = make_float4(mr.o.x, mr.o.y, mr.o.z, mr.len);
					w.sec_d[2 * i + 1] = make_float4(mr.d.x, mr.d.y, mr.d.z, 0.f);
				}
				if (p.guide_flags != 0u && !r.pass_through) {
					if (vr.flags & VOL_MEDIUM_VERTEX) {
						if (w.guide_medium.query_in != nullptr) {
							write_guide_query_medium(p, r.si.p, r.si.wo, w.guide_medium.query_in + 3 * i);
							push_guide_m = (p.guide_flags & GUIDE_SAMPLE) && *w.guide_medium.usable != 0u;
						}
					} else if (r.guidable) {
						write_guide_query(p, r.si, w.guide.query_in + 3 * i);
						push_guide = (p.guide_flags & GUIDE_SAMPLE) && *w.guide.usable != 0u;
					}
				}
			}
			store_path(w, i, st);
		}
		warp_push(push_shadow, 2 * i, w.sec_queue, w.counters + CNT_SECONDARY);
		warp_push(push_mis, 2 * i + 1, w.sec_queue, w.counters + CNT_SECONDARY);
		if (p.guide_flags != 0u) {
			warp_push(push_guide, i, w.guide.queue, w.counters + CNT_GUIDE);
			warp_push(push_guide_m, i, w.guide_medium.queue, w.counters + CNT_GUIDE_MEDIUM);
		}
		const uint32_t ns = __popc(__ballot_sync(0xffffffffu, push_shadow));
		const uint32_t nm = __popc(__ballot_sync(0xffffffffu, push_mis));
		if ((threadIdx.x & 31u) == 0) {
			if (ns) add64(w.counters, CNT_SHADOW_RAYS, ns);
			if (nm) add64(w.counters, CNT_MIS_RAYS, nm);
		}
	}
}

// What the two light connections found (integrator.cpp:136-160,166-197 for a
// surface, :218-241,249-284 for a medium vertex): the unoccluded emitter sample,
// the emitter or environment found by the MIS sample (with find_emitter's
// environment pick, :49-82), and the point each connection ends at. Scenes
// without media skip the transmittance walks.
__global__ void __launch_bounds__(256) k_vol_direct(scene_view s, wave_buffers w, uint32_t queue_in) {
	const wave_params& p = *w.params;
	const uint32_t n = w.counters[CNT_ACTIVE];
	const uint32_t* q = w.queue[queue_in];
	for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
		const uint32_t k = base + threadIdx.x;
		bool push_nee = false, push_mis = false;
		uint32_t i = 0;
		if (k < n) {
			i = q[k];
			const uint32_t flags = __float_as_uint(w.radiance[i].w);
			const shade_record& rec = w.rec[i];
			if (!(flags & 0x80000000u) && !rec.pass_through && rec.did_nee) {
				vol_rec& vr = w.vrec[i];
				pcg32 rng = load_rng(w, p, i);
				const surface_t& si = rec.si;
				const hit_t sh = to_hit(w.sec_hit[2 * i]);
				if (rec.nee_entity >= 0 && (sh.slot < 0 || hit_entity(s, sh.slot) == static_cast<uint32_t>(rec.nee_entity)))
					vr.flags |= VOL_NEE;
				if (rec.mis_valid) {
					const hit_t mh = to_hit(w.sec_hit[2 * i + 1]);
					bool found = false;
					spectrum Le = splat3(0.f);
					float epdf = 0.f;
					vec3 to{0.f, 0.f, 0.f};
					const float pick_pdf = 1.f / static_cast<float>(s.num_emitters);
					if (mh.slot >= 0) {
						const entity_rec& ent = s.entities[hit_entity(s, mh.slot)];
						if (ent.flags & ENT_HAS_EMITTER) {
							const surface_t es = make_surface(s, mh.slot, mh.b1, mh.b2, rec.mis_ray.o, rec.mis_ray.d);
							const emitter_rec& em = s.emitters[ent.emitter];
							Le = surface_emission(ent, em, es.n, -rec.mis_wi);
							epdf = emitter_pdf(s, em, si.p, si.n, rec.mis_wi) * pick_pdf;
							to = es.p;
							found = true;
						}
					} else if (s.num_environments > 0) {
						const float ne = static_cast<float>(s.num_environments);
						uint32_t which = static_cast<uint32_t>(floorf(pcg_real(rng) * ne));
						if (which > s.num_environments - 1) which = s.num_environments - 1;
						const emitter_rec& em = s.emitters[s.environments[which]];
						Le = em.radiance;
						epdf = emitter_pdf(s, em, si.p, si.n, rec.mis_wi) * pick_pdf;
						to = si.p + (2.f * rec.mis_wi) * em.radius;
						found = true;
					}
					if (found && !is_black(Le) && epdf > 0.f) {
						vr.flags |= VOL_MIS;
						vr.mis_Le = Le;
						vr.mis_w = rec.mis_specular ? 1.f : power_heuristic(rec.mis_pdf, epdf);
						vr.mis_to = to;
					}
				}
				w.rng[i] = rng.state;
				if (s.num_media == 0) {
					w.beam[2 * i] = make_float4(1.f, 1.f, 1.f, 0.f);
					w.beam[2 * i + 1] = make_float4(1.f, 1.f, 1.f, 0.f);
				} else {
					push_nee = (vr.flags & VOL_NEE) != 0u;
					push_mis = (vr.flags & VOL_MIS) != 0u;
				}
			}
		}
		warp_push(push_nee, 2 * i, w.beam_queue, w.counters + CNT_BEAM);
		warp_push(push_mis, 2 * i + 1, w.beam_queue, w.counters + CNT_BEAM);
	}
}

// scene::evaluate_media_beam (scenes/scene.cpp:114-148): from the vertex to the
// connection's end point, closest hits over all entities; every segment
// multiplies the transmittance of the medium it runs in, an invisible entity
// with media switches the medium, a visible one blocks the connection.
constexpr uint32_t kMaxBeamSegments = 256;
template <bool COUNT>
__global__ void __launch_bounds__(256) k_beam(scene_view s, wave_buffers w, uint32_t stack_cap) {
	extern __shared__ uint32_t smem[];
	smem_stack stk = make_stack(smem, stack_cap);
	const uint32_t n = w.counters[CNT_BEAM];
	uint32_t nodes = 0, tris = 0, queries = 0;
	for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
		const uint32_t k = base + threadIdx.x;
		if (k >= n) continue;
		const uint32_t j = w.beam_queue[k];
		const uint32_t i = j >> 1;
		const shade_record& rec = w.rec[i];
		const vol_rec& vr = w.vrec[i];
		const vec3 target = (j & 1u) ? vr.mis_to : vr.nee_to;
		int32_t medium = vr.medium;
		spectrum L = splat3(1.f);
		ray_t r = spawn_ray_to(rec.si.p, rec.si.n, target);
		bool blocked = false, done = false;
		for (uint32_t seg = 0; seg < kMaxBeamSegments; seg++) {
			float len = r.len;
			hit_t h;
			queries++;
			if (!trace_one<false, COUNT>(s, r.o, r.d, len, h, stk, nodes, tris)) {
				set_error(w.counters, RB_ERR_STACK_OVERFLOW);
				blocked = true;
				break;
			}
			if (h.slot < 0) {
				done = true;
				break;
			}
			L = L * transmittance(s, medium, len);
			const entity_rec& ent = s.entities[hit_entity(s, h.slot)];
			if (ent.flags & ENT_VISIBLE) {
				blocked = true;
				break;
			}
			const surface_t si = make_surface(s, h.slot, h.b1, h.b2, r.o, r.d);
			r = spawn_ray_to(si.p, si.n, target);
			if (ent.flags & ENT_HAS_MEDIA) medium = medium_after(s, ent, si.n, r.d);
		}
		if (!done && !blocked) {
			set_error(w.counters, RB_ERR_STACK_OVERFLOW);  // more boundary crossings than the walk allows
			blocked = true;
		}
		if (!blocked) L = L * transmittance(s, medium, r.len);
		else L = splat3(0.f);
		w.beam[j] = make_float4(L.x, L.y, L.z, 0.f);
	}
	if (COUNT) {
		warp_add64(w.counters, CNT_NODE_VISITS, nodes);
		warp_add64(w.counters, CNT_TRI_TESTS, tris);
	}
	warp_add64(w.counters, CNT_BEAM_RAYS, queries);
}

// The rest of the bounce: the light connections with their transmittance
// (the reference's association of each product), then the continuation by the
// BSDF (surface) or the phase function (medium vertex), the medium switch when
// the entity carries media (volume_path_integrator.cpp:50-64), and roulette.
__device__ bool vol_continue(const scene_view& s, const wave_buffers& w, const wave_params& p, uint32_t i, path_state& st) {
	const shade_record& rec = w.rec[i];
	const vol_rec& vr = w.vrec[i];
	const bool medium_vertex = (vr.flags & VOL_MEDIUM_VERTEX) != 0u;
	if (!rec.pass_through) {
		if (rec.did_nee) {
			spectrum L = splat3(0.f);
			if (vr.flags & VOL_NEE) {
				const float4 b4 = w.beam[2 * i];
				const spectrum b{b4.x, b4.y, b4.z};
				if (medium_vertex) L = L + vr.nee_f * vr.nee_Le * b * vr.nee_w / vr.nee_pdf;
				else L = L + (vr.nee_f * b) * vr.nee_Le * vr.nee_w / vr.nee_pdf;
			}
			if (vr.flags & VOL_MIS) {
				const float4 b4 = w.beam[2 * i + 1];
				const spectrum b{b4.x, b4.y, b4.z};
				if (medium_vertex) L = L + rec.mis_f * vr.mis_Le * b * vr.mis_w / rec.mis_pdf;
				else L = L + (rec.mis_f * b) * vr.mis_Le * vr.mis_w / rec.mis_pdf;
			}
			st.L = st.L + st.beta * L;
		}
		const spectrum beta0 = st.beta, L0 = st.L;
		vec3 wi;
		float pb;
		if (medium_vertex) {
			// sample_medium_interaction (integrator.cpp:408-421): the phase value is its pdf, beta stays;
			// guided: one-sample MIS of the medium guide and the phase function
			const bool use_guide = (p.guide_flags & GUIDE_SAMPLE) && w.guide_medium.query_out != nullptr &&
				*w.guide_medium.usable != 0u;
			if (use_guide) {
				const float* g = reinterpret_cast<const float*>(w.guide_medium.query_out + 12 * i);
				const float alpha = g[guide::kAlphaOff];
				const float u_sel = pcg_real(st.rng);
				const vec2 u = pcg_2d(st.rng);
				if (u_sel < alpha) {
					float d[3];
					guide::guide_sample(g, u_sel / alpha, u.x, u.y, d);
					wi = vec3{d[0], d[1], d[2]};
					pb = hg_phase(dot(rec.si.wo, wi), vr.g);
				} else {
					pb = hg_sample(rec.si.wo, vr.g, u, wi);
				}
				const float pdf = alpha * guide::guide_pdf(g, wi.x, wi.y, wi.z) + (1.f - alpha) * pb;
				if (!(pdf > 0.f) || !(pb > 0.f)) return false;
				st.beta = st.beta * (pb / pdf);
			} else {
				pb = hg_sample(rec.si.wo, vr.g, pcg_2d(st.rng), wi);
			}
			st.flags &= ~PATH_SPECULAR;
			const ray_t r = spawn_ray(rec.si.p, vec3{0.f, 0.f, 0.f}, wi);
			st.o = r.o;
			st.d = r.d;
			st.len = r.len;
			if ((p.guide_flags & GUIDE_TRAIN) && w.guide_medium.vertices != nullptr && st.bounces + 1 < static_cast<int32_t>(p.max_depth))
				record_vertex(w.guide_medium, i, wi, pb, beta0, L0);
		} else {
			const bool use_guide = (p.guide_flags & GUIDE_SAMPLE) && rec.guidable && w.guide.query_out != nullptr &&
				*w.guide.usable != 0u;
			const bool ok = use_guide
				? continue_guided<MAT_ANY>(s, st, rec, reinterpret_cast<const float*>(w.guide.query_out + 12 * i), wi, pb)
				: continue_bsdf<MAT_ANY>(s, st, rec, wi, pb);
			if (!ok) return false;
			if ((p.guide_flags & GUIDE_TRAIN) && rec.guidable && w.guide.vertices != nullptr &&
				st.bounces + 1 < static_cast<int32_t>(p.max_depth))
				record_vertex(w.guide, i, wi, pb, beta0, L0);
		}
	}
	if (!medium_vertex) {
		const entity_rec& ent = s.entities[rec.si.entity];
		if (ent.flags & ENT_HAS_MEDIA) st.medium = medium_after(s, ent, rec.si.n, st.d);
	}
	return roulette(st, p.max_depth, p.rr_threshold);
}

__global__ void __launch_bounds__(256) k_vol_continue(scene_view s, wave_buffers w, uint32_t queue_in) {
	const wave_params& p = *w.params;
	const uint32_t n = w.counters[CNT_ACTIVE];
	const uint32_t* q = w.queue[queue_in];
	uint32_t* qn = w.queue[queue_in ^ 1u];
	for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
		const uint32_t k = base + threadIdx.x;
		bool alive = false;
		uint32_t i = 0;
		if (k < n) {
			i = q[k];
			path_state st = load_path(w, p, i);
			if (!(st.flags & 0x80000000u)) {
				alive = vol_continue(s, w, p, i, st);
				if (!alive) finish(w, i, st.L);
				store_path(w, i, st);
			}
		}
		warp_push(alive, i, qn, w.counters + CNT_NEXT);
	}
}

__global__ void k_advance(uint32_t* counters);

// Traversal kernels keep their stacks in dynamic shared memory; above 48 KB a
// block needs the kernel's opt-in.
// They also set their preferred shared-memory carve-out (percent of the
// combined L1 / shared storage): the largest share fits four blocks of 256
// threads with their stacks, smaller shares leave more L1 for tree nodes.
template <typename Kernel>
cudaError_t allow_smem(Kernel kernel, size_t bytes, int carveout = 100) {
	cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, carveout);
	if (e != cudaSuccess || bytes <= 48u * 1024u) return e;
	return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes));
}

template <bool COUNT, bool INST>
cudaError_t volume_bounce(const scene_view& s, const wave_buffers& w, uint32_t queue_in, const launch_cfg& cfg,
	cudaStream_t stream) {
	const size_t smem = 2 * static_cast<size_t>(cfg.stack_depth) * cfg.block_trace * sizeof(uint32_t);
	const bool refill = !COUNT && cfg.refill;
	cudaError_t e = allow_smem(k_extend<COUNT, true, false, INST>, smem, cfg.carveout);
	if (e == cudaSuccess) e = allow_smem(k_trace_secondary<COUNT, false, INST>, smem, cfg.carveout);
	if (e == cudaSuccess) e = allow_smem(k_beam<COUNT>, smem, cfg.carveout);
	if (e == cudaSuccess && refill) e = allow_smem(k_extend_refill<true, false>, smem, cfg.carveout);
	if (e == cudaSuccess && refill) e = allow_smem(k_secondary_refill<false>, smem, cfg.carveout);
	if (e != cudaSuccess) return e;
	if (refill) k_extend_refill<true, false><<<cfg.grid_trace, cfg.block_trace, smem, stream>>>(s, w, queue_in, cfg.stack_depth, cfg.sort);
	else k_extend<COUNT, true, false, INST><<<cfg.grid_trace, cfg.block_trace, smem, stream>>>(s, w, queue_in, cfg.stack_depth, cfg.sort);
	k_shade_a<CLASS_LAMBERT, true, false><<<cfg.grid_shade, cfg.block_shade, 0, stream>>>(s, w);
	k_shade_a<CLASS_METAL, true, false><<<cfg.grid_shade, cfg.block_shade, 0, stream>>>(s, w);
	k_shade_a<CLASS_GLASS_ROUGH, true, false><<<cfg.grid_shade, cfg.block_shade, 0, stream>>>(s, w);
	k_shade_a<CLASS_OTHER, true, false><<<cfg.grid_shade, cfg.block_shade, 0, stream>>>(s, w);
	k_shade_a<CLASS_MISS, true, false><<<cfg.grid_shade, cfg.block_shade, 0, stream>>>(s, w);
	k_shade_a_medium<<<cfg.grid_shade, cfg.block_shade, 0, stream>>>(s, w);
	if (cfg.guide != nullptr && (cfg.guide_mode & GUIDE_SAMPLE)) {
		e = guide::launch_forward_queue(*cfg.guide, w.guide, w.counters + CNT_GUIDE, stream);
		if (e == cudaSuccess && cfg.guide_medium != nullptr)
			e = guide::launch_forward_queue(*cfg.guide_medium, w.guide_medium, w.counters + CNT_GUIDE_MEDIUM, stream);
		if (e != cudaSuccess) return e;
	}
	if (refill) k_secondary_refill<false><<<cfg.grid_trace, cfg.block_trace, smem, stream>>>(s, w, cfg.stack_depth);
	else k_trace_secondary<COUNT, false, INST><<<cfg.grid_trace, cfg.block_trace, smem, stream>>>(s, w, cfg.stack_depth, 0u);
	k_vol_direct<<<cfg.grid_shade, cfg.block_shade, 0, stream>>>(s, w, queue_in);
	k_beam<COUNT><<<cfg.grid_trace, cfg.block_trace, smem, stream>>>(s, w, cfg.stack_depth);
	k_vol_continue<<<cfg.grid_shade, cfg.block_shade, 0, stream>>>(s, w, queue_in);
	k_advance<<<1, 1, 0, stream>>>(w.counters);
	return cudaGetLastError();
}

// Moves the next queue's count into place and accumulates the extend-ray count.
__global__ void k_advance(uint32_t* counters) {
	add64(counters, CNT_EXTEND_RAYS, counters[CNT_ACTIVE]);
	counters[CNT_ACTIVE] = counters[CNT_NEXT];
	counters[CNT_NEXT] = 0u;
	counters[CNT_SECONDARY] = 0u;
	counters[CNT_GUIDE] = 0u;
	counters[CNT_GUIDE_MEDIUM] = 0u;
	counters[CNT_BEAM] = 0u;
	for (uint32_t c = 0; c < NUM_CLASSES; c++) counters[CNT_CLASS + c] = 0u;
	counters[CNT_TAIL] = 0u;
	counters[CNT_SSS] = 0u;
	counters[CNT_FETCH_EXTEND] = 0u;
	counters[CNT_FETCH_SECONDARY] = 0u;
}

// Moves the wave window forward so the next replay of the same graph renders
// the following work items.
__global__ void k_next_wave(wave_params* p, uint32_t capacity) { p->first_item += capacity; }

// The first work item of the next wave of a lane (several lanes take turns).
__global__ void k_set_first(wave_params* p, uint64_t first) { p->first_item = first; }

// Writes a lane's parameter block from a kernel argument, so that no host
// buffer has to outlive the enqueued call.
__global__ void k_set_params(wave_params p, wave_params* dst) { *dst = p; }

// INST: the scene holds instance slots (scene_view::instances); the traversal
// kernels of single-level scenes are instantiated without that branch.
template <bool COUNT, bool BATCH, bool INST>
cudaError_t bounce(const scene_view& s, const wave_buffers& w, const film_buffers& f, uint32_t queue_in,
	const launch_cfg& cfg, cudaStream_t stream) {
	if (!BATCH && cfg.volume) return volume_bounce<COUNT, INST>(s, w, queue_in, cfg, stream);
	const size_t smem = 2 * static_cast<size_t>(cfg.stack_depth) * cfg.block_trace * sizeof(uint32_t);
	const bool refill = !COUNT && cfg.refill;
	cudaError_t e = allow_smem(k_extend<COUNT, false, BATCH, INST>, smem, cfg.carveout);
	if (e == cudaSuccess) e = allow_smem(k_trace_secondary<COUNT, BATCH, INST>, smem, cfg.carveout);
	if (e == cudaSuccess && refill) e = allow_smem(k_extend_refill<false, BATCH>, smem, cfg.carveout);
	if (e == cudaSuccess && refill) e = allow_smem(k_secondary_refill<BATCH>, smem, cfg.carveout);
	if (e != cudaSuccess) return e;
	const bool timed = cfg.events != nullptr && *cfg.next_event + 2 <= cfg.max_events;
	uint32_t ev = timed ? *cfg.next_event : 0u;
	if (timed) { cudaEventRecord(cfg.events[2 * ev], stream); cfg.event_kind[ev] = 0; }
	if (refill) k_extend_refill<false, BATCH><<<cfg.grid_trace, cfg.block_trace, smem, stream>>>(s, w, queue_in, cfg.stack_depth, cfg.sort);
	else k_extend<COUNT, false, BATCH, INST><<<cfg.grid_trace, cfg.block_trace, smem, stream>>>(s, w, queue_in, cfg.stack_depth, cfg.sort);
	if (timed) cudaEventRecord(cfg.events[2 * ev + 1], stream);
	if (cfg.sort != RB_SORT_NONE) {
		k_shade_a<CLASS_LAMBERT, false, BATCH><<<cfg.grid_shade, cfg.block_shade, 0, stream>>>(s, w);
		k_shade_a<CLASS_METAL, false, BATCH><<<cfg.grid_shade, cfg.block_shade, 0, stream>>>(s, w);
		k_shade_a<CLASS_GLASS_ROUGH, false, BATCH><<<cfg.grid_shade, cfg.block_shade, 0, stream>>>(s, w);
	}
	k_shade_a<CLASS_OTHER, false, BATCH><<<cfg.grid_shade, cfg.block_shade, 0, stream>>>(s, w);
	k_shade_a<CLASS_MISS, false, BATCH><<<cfg.grid_shade, cfg.block_shade, 0, stream>>>(s, w);
	if (!BATCH && cfg.guide != nullptr && (cfg.guide_mode & GUIDE_SAMPLE)) {
		e = guide::launch_forward_queue(*cfg.guide, w.guide, w.counters + CNT_GUIDE, stream);
		if (e != cudaSuccess) return e;
	}
	if (timed) { ev++; cudaEventRecord(cfg.events[2 * ev], stream); cfg.event_kind[ev] = 1; }
	if (refill) k_secondary_refill<BATCH><<<cfg.grid_trace, cfg.block_trace, smem, stream>>>(s, w, cfg.stack_depth);
	else k_trace_secondary<COUNT, BATCH, INST><<<cfg.grid_trace, cfg.block_trace, smem, stream>>>(s, w, cfg.stack_depth,
		cfg.shadow_first ? 1u : 0u);
	if (timed) { cudaEventRecord(cfg.events[2 * ev + 1], stream); *cfg.next_event = ev + 1; }
	if (cfg.sort != RB_SORT_NONE) {
		k_shade_b<CLASS_LAMBERT, BATCH><<<cfg.grid_shade, cfg.block_shade, 0, stream>>>(s, w, queue_in);
		k_shade_b<CLASS_METAL, BATCH><<<cfg.grid_shade, cfg.block_shade, 0, stream>>>(s, w, queue_in);
		k_shade_b<CLASS_GLASS_ROUGH, BATCH><<<cfg.grid_shade, cfg.block_shade, 0, stream>>>(s, w, queue_in);
	}
	k_shade_b<CLASS_OTHER, BATCH><<<cfg.grid_shade, cfg.block_shade, 0, stream>>>(s, w, queue_in);
	if (cfg.sss) {
		e = allow_smem(k_subsurface<BATCH, INST>, smem, cfg.carveout);
		if (e != cudaSuccess) return e;
		k_subsurface<BATCH, INST><<<cfg.grid_trace, cfg.block_trace, smem, stream>>>(s, w, queue_in, cfg.stack_depth);
	}
	k_advance<<<1, 1, 0, stream>>>(w.counters);
	return cudaGetLastError();
}

} // namespace

cudaError_t launch_trace_rays(const scene_view& s, const uint32_t* prim_entity, const rb_ray* rays, uint32_t n, rb_hit* hits,
	bool shadow, const launch_cfg& cfg, uint32_t* counters, cudaStream_t stream) {
	if (n == 0) return cudaSuccess;
	const size_t smem = 2 * static_cast<size_t>(cfg.stack_depth) * cfg.block_trace * sizeof(uint32_t);
	const uint32_t blocks_needed = (n + cfg.block_trace - 1) / cfg.block_trace;
	const int grid = static_cast<int>(blocks_needed < static_cast<uint32_t>(cfg.grid_trace) ? blocks_needed : cfg.grid_trace);
	cudaError_t e = allow_smem(k_trace_rays<true, true>, smem);
	if (e == cudaSuccess) e = allow_smem(k_trace_rays<true, false>, smem);
	if (e == cudaSuccess) e = allow_smem(k_trace_rays<false, true>, smem);
	if (e == cudaSuccess) e = allow_smem(k_trace_rays<false, false>, smem);
	if (e != cudaSuccess) return e;
	if (shadow) {
		if (cfg.count) k_trace_rays<true, true><<<grid, cfg.block_trace, smem, stream>>>(s, prim_entity, rays, n, hits, cfg.stack_depth, counters);
		else k_trace_rays<true, false><<<grid, cfg.block_trace, smem, stream>>>(s, prim_entity, rays, n, hits, cfg.stack_depth, counters);
	} else {
		if (cfg.count) k_trace_rays<false, true><<<grid, cfg.block_trace, smem, stream>>>(s, prim_entity, rays, n, hits, cfg.stack_depth, counters);
		else k_trace_rays<false, false><<<grid, cfg.block_trace, smem, stream>>>(s, prim_entity, rays, n, hits, cfg.stack_depth, counters);
	}
	return cudaGetLastError();
}

template <bool INST>
cudaError_t bounce_inst(const scene_view& s, const wave_buffers& w, const film_buffers& f, uint32_t queue_in,
	const launch_cfg& cfg, cudaStream_t stream) {
	if (cfg.batch)
		return cfg.count ? bounce<true, true, INST>(s, w, f, queue_in, cfg, stream)
			: bounce<false, true, INST>(s, w, f, queue_in, cfg, stream);
	return cfg.count ? bounce<true, false, INST>(s, w, f, queue_in, cfg, stream)
		: bounce<false, false, INST>(s, w, f, queue_in, cfg, stream);
}

cudaError_t launch_bounce(const scene_view& s, const wave_buffers& w, const film_buffers& f, uint32_t queue_in,
	const launch_cfg& cfg, cudaStream_t stream) {
	return s.instances ? bounce_inst<true>(s, w, f, queue_in, cfg, stream) : bounce_inst<false>(s, w, f, queue_in, cfg, stream);
}

// The secondary traversal of the staged direct-lighting rounds.
template <bool COUNT>
void direct_secondary(const scene_view& s, const wave_buffers& wr, const launch_cfg& cfg, size_t smem, cudaStream_t stream) {
	if (s.instances) k_trace_secondary<COUNT, false, true><<<cfg.grid_trace, cfg.block_trace, smem, stream>>>(s, wr, cfg.stack_depth, 0u);
	else k_trace_secondary<COUNT, false, false><<<cfg.grid_trace, cfg.block_trace, smem, stream>>>(s, wr, cfg.stack_depth, 0u);
}

// Whether a wave ends with the tail kernel after cfg.tail bounces (plain
// surface path tracing only: guided and volume paths keep their stages).
// Scenes with subsurface materials run every bounce staged: their BSSRDF
// stage is a kernel of its own (k_subsurface), not part of the tail.
bool uses_tail(uint32_t max_depth, const launch_cfg& cfg) {
	return cfg.tail < max_depth && !cfg.volume && cfg.guide == nullptr && !cfg.sss;
}

template <bool BATCH>
cudaError_t launch_tail(const scene_view& s, const wave_buffers& w, uint32_t queue_in, const launch_cfg& cfg,
	cudaStream_t stream) {
	const size_t smem = 2 * static_cast<size_t>(cfg.stack_depth) * cfg.block_trace * sizeof(uint32_t);
	cudaError_t e;
	if (cfg.count) {
		e = allow_smem(k_tail<true, BATCH>, smem, cfg.carveout);
		if (e == cudaSuccess) k_tail<true, BATCH><<<cfg.grid_trace, cfg.block_trace, smem, stream>>>(s, w, queue_in, cfg.stack_depth);
	} else {
		e = allow_smem(k_tail<false, BATCH>, smem, cfg.carveout);
		if (e == cudaSuccess) k_tail<false, BATCH><<<cfg.grid_trace, cfg.block_trace, smem, stream>>>(s, w, queue_in, cfg.stack_depth);
	}
	if (e != cudaSuccess) return e;
	k_advance<<<1, 1, 0, stream>>>(w.counters);
	return cudaGetLastError();
}

cudaError_t launch_wave(const scene_view& s, const wave_buffers& w, const film_buffers& f, uint32_t max_depth,
	uint32_t first_queue, const launch_cfg& cfg, cudaStream_t stream) {
	if (cfg.batch) k_camera<true><<<cfg.grid_shade, 256, 0, stream>>>(w, first_queue);
	else k_camera<false><<<cfg.grid_shade, 256, 0, stream>>>(w, first_queue);
	cudaError_t err = cudaGetLastError();
	uint32_t qi = first_queue;
	const bool tail = uses_tail(max_depth, cfg);
	const uint32_t staged = tail ? cfg.tail : max_depth;
	const bool bin = cfg.sort == RB_SORT_RAYS && w.sort_keys != nullptr;
	for (uint32_t b = 0; b < staged && err == cudaSuccess; b++) {
		if (bin && b > 0) {  // camera rays arrive in pixel order, already coherent
			k_bin_count<<<cfg.grid_shade, 256, 0, stream>>>(w, qi);
			k_bin_scan<<<1, 1024, 0, stream>>>(w);
			k_bin_scatter<<<cfg.grid_shade, 256, 0, stream>>>(w, qi);
			k_bin_copy<<<cfg.grid_shade, 256, 0, stream>>>(w, qi);
			err = cudaGetLastError();
			if (err != cudaSuccess) break;
		}
		err = launch_bounce(s, w, f, qi, cfg, stream);
		qi ^= 1u;
	}
	if (tail && err == cudaSuccess) err = cfg.batch ? launch_tail<true>(s, w, qi, cfg, stream) : launch_tail<false>(s, w, qi, cfg, stream);
	return err;
}

cudaError_t launch_next_wave(const wave_buffers& w, const film_buffers& f, int grid, cudaStream_t stream) {
	if (w.batch != nullptr) k_film_resolve_batch<<<grid, 256, 0, stream>>>(w, f);
	else k_film_resolve<<<grid, 256, 0, stream>>>(w, f);
	k_next_wave<<<1, 1, 0, stream>>>(w.params, w.capacity);
	return cudaGetLastError();
}

cudaError_t launch_direct_wave(const scene_view& s, const wave_buffers& w, const film_buffers& f, const direct_cfg& dc,
	const launch_cfg& cfg, int resolve_grid, cudaStream_t stream) {
	const size_t smem = 2 * static_cast<size_t>(cfg.stack_depth) * cfg.block_trace * sizeof(uint32_t);
	cudaError_t e;
	if (cfg.count) {
		e = allow_smem(k_direct<true>, smem, cfg.carveout);
		if (e == cudaSuccess) k_direct<true><<<cfg.grid_trace, cfg.block_trace, smem, stream>>>(s, w, dc, cfg.stack_depth);
	} else {
		e = allow_smem(k_direct<false>, smem, cfg.carveout);
		if (e == cudaSuccess) k_direct<false><<<cfg.grid_trace, cfg.block_trace, smem, stream>>>(s, w, dc, cfg.stack_depth);
	}
	if (e == cudaSuccess) e = cudaGetLastError();
	if (e == cudaSuccess) e = launch_next_wave(w, f, resolve_grid, stream);
	return e;
}

cudaError_t launch_direct_staged_wave(const scene_view& s, const wave_buffers& w, const film_buffers& f,
	const direct_buffers& db, const direct_cfg& dc, const launch_cfg& cfg, int resolve_grid, cudaStream_t stream) {
	const size_t smem = 2 * static_cast<size_t>(cfg.stack_depth) * cfg.block_trace * sizeof(uint32_t);
	cudaError_t e = cfg.count ? allow_smem(k_direct_surface<true>, smem, cfg.carveout)
		: allow_smem(k_direct_surface<false>, smem, cfg.carveout);
	if (e == cudaSuccess) e = allow_smem(k_trace_secondary<false, false, false>, smem, cfg.carveout);
	if (e == cudaSuccess) e = allow_smem(k_trace_secondary<true, false, false>, smem, cfg.carveout);
	if (e == cudaSuccess) e = allow_smem(k_trace_secondary<false, false, true>, smem, cfg.carveout);
	if (e == cudaSuccess) e = allow_smem(k_trace_secondary<true, false, true>, smem, cfg.carveout);
	if (e != cudaSuccess) return e;
	// the traversal kernel reads the queued slots through the secondary-ray fields
	wave_buffers wr = w;
	wr.sec_o = db.ray_o;
	wr.sec_d = db.ray_d;
	wr.sec_hit = db.ray_hit;
	wr.sec_queue = db.ray_queue;
	e = cudaMemsetAsync(w.counters + CNT_SECONDARY, 0, sizeof(uint32_t), stream);
	if (e == cudaSuccess) e = cudaMemsetAsync(w.counters + CNT_CLASS, 0, NUM_CLASSES * sizeof(uint32_t), stream);
	if (e != cudaSuccess) return e;
	if (cfg.count) k_direct_surface<true><<<cfg.grid_trace, cfg.block_trace, smem, stream>>>(s, w, db, cfg.stack_depth);
	else k_direct_surface<false><<<cfg.grid_trace, cfg.block_trace, smem, stream>>>(s, w, db, cfg.stack_depth);
	k_direct_lights<CLASS_LAMBERT><<<cfg.grid_shade, cfg.block_shade, 0, stream>>>(s, w, db, dc);
	k_direct_lights<CLASS_METAL><<<cfg.grid_shade, cfg.block_shade, 0, stream>>>(s, w, db, dc);
	k_direct_lights<CLASS_GLASS_ROUGH><<<cfg.grid_shade, cfg.block_shade, 0, stream>>>(s, w, db, dc);
	k_direct_lights<CLASS_OTHER><<<cfg.grid_shade, cfg.block_shade, 0, stream>>>(s, w, db, dc);
	for (uint32_t r = 0; r < dc.bsdf_samples && e == cudaSuccess; r++) {
		if (cfg.count) direct_secondary<true>(s, wr, cfg, smem, stream);
		else direct_secondary<false>(s, wr, cfg, smem, stream);
		e = cudaMemsetAsync(w.counters + CNT_SECONDARY, 0, sizeof(uint32_t), stream);
		if (e != cudaSuccess) break;
		k_direct_round<CLASS_LAMBERT><<<cfg.grid_shade, cfg.block_shade, 0, stream>>>(s, w, db, dc);
		k_direct_round<CLASS_METAL><<<cfg.grid_shade, cfg.block_shade, 0, stream>>>(s, w, db, dc);
		k_direct_round<CLASS_GLASS_ROUGH><<<cfg.grid_shade, cfg.block_shade, 0, stream>>>(s, w, db, dc);
		k_direct_round<CLASS_OTHER><<<cfg.grid_shade, cfg.block_shade, 0, stream>>>(s, w, db, dc);
	}
	if (e == cudaSuccess) e = cudaGetLastError();
	if (e == cudaSuccess) e = launch_next_wave(w, f, resolve_grid, stream);
	return e;
}

cudaError_t launch_set_params(const wave_params& p, wave_params* dst, cudaStream_t stream) {
	k_set_params<<<1, 1, 0, stream>>>(p, dst);
	return cudaGetLastError();
}

cudaError_t launch_set_first(wave_params* params, uint64_t first, cudaStream_t stream) {
	k_set_first<<<1, 1, 0, stream>>>(params, first);
	return cudaGetLastError();
}

cudaError_t launch_film_mean(const film_buffers& f, uint32_t pixels, float* rgb, int grid, cudaStream_t stream) {
	if (pixels == 0) return cudaSuccess;
	k_film_mean<<<grid, 256, 0, stream>>>(f, pixels, rgb);
	return cudaGetLastError();
}

cudaError_t launch_wave_end(const wave_buffers& w, const film_buffers& f, int grid, const launch_cfg& cfg,
	cudaStream_t stream) {
	const bool train = cfg.guide != nullptr && (cfg.guide_mode & GUIDE_TRAIN);
	const guide::guide_state* guides[2] = {cfg.guide, cfg.guide_medium};
	const guide::wave_guide* wgs[2] = {&w.guide, &w.guide_medium};
	cudaError_t e = cudaSuccess;
	for (int k = 0; k < 2; k++)
		if (train && guides[k] != nullptr && e == cudaSuccess)
			e = guide::launch_collect(*guides[k], *wgs[k], w.result, &w.params->first_item, &w.params->total_items, w.capacity,
				stream);
	if (e == cudaSuccess) e = launch_next_wave(w, f, grid, stream);
	for (const guide::guide_state* g : guides)
		if (train && g != nullptr)
			for (uint32_t k = 0; k < g->cfg.steps_per_wave && e == cudaSuccess; k++)
				e = guide::launch_train_step(*g, g->samples, &g->dstate->ring_filled, g->sample_cap, g->cfg.batch_size,
					g->cfg.min_rows, false, true, stream);
	return e;
}

namespace {

__global__ void k_drain_begin(cudaGraphConditionalHandle h, uint32_t* counters) {
	counters[CNT_DRAIN_WAVE] = 0u;
	cudaGraphSetConditional(h, counters[CNT_ACTIVE] != 0u ? 1u : 0u);
}

__global__ void k_drain_step(cudaGraphConditionalHandle h, uint32_t* counters) {
	const uint32_t it = counters[CNT_DRAIN_WAVE] + 1u;
	counters[CNT_DRAIN_WAVE] = it;
	counters[CNT_DRAIN_TOTAL] += 1u;
	cudaGraphSetConditional(h, counters[CNT_ACTIVE] != 0u && it < kMaxDrainIterations ? 1u : 0u);
}

} // namespace

cudaError_t launch_drain_begin(cudaGraphConditionalHandle h, uint32_t* counters, cudaStream_t stream) {
	k_drain_begin<<<1, 1, 0, stream>>>(h, counters);
	return cudaGetLastError();
}

cudaError_t launch_drain_step(cudaGraphConditionalHandle h, uint32_t* counters, cudaStream_t stream) {
	k_drain_step<<<1, 1, 0, stream>>>(h, counters);
	return cudaGetLastError();
}

uint32_t bounce_launches(const launch_cfg& cfg) {
	const bool sample = cfg.guide != nullptr && (cfg.guide_mode & GUIDE_SAMPLE);
	if (cfg.volume) return 12u + (sample ? (cfg.guide_medium != nullptr ? 2u : 1u) : 0u);
	return (cfg.sort == RB_SORT_NONE ? 7u : 12u) + (sample ? 1u : 0u) + (cfg.sss ? 1u : 0u);
}

uint32_t drain_launches(const launch_cfg& cfg) { return 2u * bounce_launches(cfg) + 1u; }

uint32_t wave_launches_unbinned(uint32_t max_depth, const launch_cfg& cfg);

uint32_t wave_launches(uint32_t max_depth, const launch_cfg& cfg) {
	const uint32_t staged = uses_tail(max_depth, cfg) ? cfg.tail : max_depth;
	return wave_launches_unbinned(max_depth, cfg) + (cfg.sort == RB_SORT_RAYS && staged > 1 ? 4u * (staged - 1) : 0u);
}

uint32_t wave_launches_unbinned(uint32_t max_depth, const launch_cfg& cfg) {
	if (cfg.volume) {
		const bool sample = cfg.guide != nullptr && (cfg.guide_mode & GUIDE_SAMPLE);
		const bool train = cfg.guide != nullptr && (cfg.guide_mode & GUIDE_TRAIN);
		const uint32_t nets = cfg.guide_medium != nullptr ? 2u : 1u;
		uint32_t n = 3u + (12u + (sample ? nets : 0u)) * max_depth;
		if (train) n += nets * (3u + 2u * cfg.guide->cfg.steps_per_wave);
		return n;
	}
	if (uses_tail(max_depth, cfg)) return 3u + (cfg.sort == RB_SORT_NONE ? 7u : 12u) * cfg.tail + 2u;
	const uint32_t sss = cfg.sss ? 1u : 0u;
	if (cfg.sort == RB_SORT_NONE && cfg.guide == nullptr) return 3u + (7u + sss) * max_depth;
	const bool sample = cfg.guide != nullptr && (cfg.guide_mode & GUIDE_SAMPLE);
	const bool train = cfg.guide != nullptr && (cfg.guide_mode & GUIDE_TRAIN);
	uint32_t n = 3u + (12u + sss + (sample ? 1u : 0u)) * max_depth;
	if (train) n += 3u + 2u * cfg.guide->cfg.steps_per_wave;
	return n;
}

} // namespace gpu
} // namespace rb
