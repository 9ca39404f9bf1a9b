// Batched rendering of many scenes in one wavefront, and the launch-shape
// autotuner (include/rbgpu.h).
//
// A batch is uploaded as one merged set of scene arrays (host::merge_scenes):
// each scene keeps its own BVH, entities, materials and emitters at an offset,
// and a table of batch_scene records says where. A render call lays the
// scenes' work items end to end in the order the caller asks for (scene k's
// items are its pixels x spp), so one wave may hold the tail of one scene and
// the head of the next; every path carries its scene index, the traversal
// starts at that scene's root and shading picks its emitters. Each scene's
// film is a range of one merged film.
//
// The autotuner times the same work under different launch shapes (paths per
// wave, block sizes, grid size, hit-queue sort key) by coordinate descent and
// keeps the fastest for the context.
#include "context.h"

#include <algorithm>
#include <vector>

namespace {

constexpr uint32_t kMaxBatchScenes = 4096;

// Renders the batch's first `max_items` work items (all of them when 0).
rb_status batch_render(rb_context* c, const rb_batch_params* prm, float* scene_ms, uint64_t max_items) {
	if (c == nullptr || prm == nullptr || prm->views == nullptr) return RB_ERR_INVALID_ARGUMENT;
	if (!c->is_batch) return RB_ERR_NO_SCENE;
	const uint32_t n = static_cast<uint32_t>(c->batch_scenes.size());
	if (prm->count != n || prm->max_depth == 0 || prm->max_depth > 64 || (prm->flags & ~RB_RENDER_RESET) != 0)
		return RB_ERR_INVALID_ARGUMENT;
	std::vector<uint32_t> order(n);
	if (prm->order != nullptr) {
		std::vector<uint8_t> seen(n, 0);
		for (uint32_t k = 0; k < n; k++) {
			const uint32_t s = prm->order[k];
			if (s >= n || seen[s]) return RB_ERR_INVALID_ARGUMENT;
			seen[s] = 1;
			order[k] = s;
		}
	} else {
		for (uint32_t k = 0; k < n; k++) order[k] = k;
	}
	// Records in render order: the kernels binary-search item_base and
	// pixel_base over them, so both increase; the merged film therefore holds
	// the scenes in render order, and batch_range maps upload order to it.
	std::vector<std::pair<uint32_t, uint32_t>> range(n);
	std::vector<uint64_t> item_base(n, 0), item_end(n, 0);
	std::vector<gpu::batch_scene> recs(n);
	uint64_t total = 0, film_px = 0;
	for (uint32_t r = 0; r < n; r++) {
		const uint32_t k = order[r];
		const rb_batch_view& v = prm->views[k];
		if (!host_is_valid_camera(v.camera) || v.spp == 0) return RB_ERR_INVALID_ARGUMENT;
		if (static_cast<uint64_t>(v.first_sample) + v.spp > (1u << 24)) return RB_ERR_INVALID_ARGUMENT;
		const uint64_t px = static_cast<uint64_t>(v.camera.width) * v.camera.height;
		gpu::batch_scene b = c->batch_scenes[k];
		std::memcpy(b.r2c, v.camera.raster_to_camera, sizeof(b.r2c));
		std::memcpy(b.c2w, v.camera.camera_to_world, sizeof(b.c2w));
		b.lens = v.camera.lens_radius;
		b.focus = v.camera.focus_distance;
		b.width = static_cast<uint32_t>(v.camera.width);
		b.height = static_cast<uint32_t>(v.camera.height);
		b.first_sample = v.first_sample;
		b.seed = v.seed;
		b.spp = v.spp;
		b.pixel_base = static_cast<uint32_t>(film_px);
		b.item_base = total;
		recs[r] = b;
		range[k] = {static_cast<uint32_t>(film_px), static_cast<uint32_t>(px)};
		item_base[k] = total;
		total += px * v.spp;
		item_end[k] = total;
		film_px += px;
		if (film_px >= (1ull << 31)) return RB_ERR_TOO_LARGE;
	}
	if (max_items != 0 && max_items < total) total = max_items;

	RB_CUDA(cudaSetDevice(c->device));
	const bool relayout = c->batch_range != range;
	rb_status st = ensure_film(c, static_cast<int32_t>(film_px), 1, (prm->flags & RB_RENDER_RESET) != 0 || relayout);
	if (st != RB_OK) return st;
	c->batch_range = range;
	uint64_t capacity = c->tuning.paths_per_wave ? c->tuning.paths_per_wave : (1ull << 21);
	if (capacity > total) capacity = total;
	if (capacity == 0) capacity = 1;
	st = ensure_wave(c, static_cast<uint32_t>(capacity));
	if (st != RB_OK) return st;
	if (c->batch_path_alloc < c->wave_alloc) {
		c->release_graph();
		dev_free(c->batch_path_scene);
		c->batch_path_alloc = 0;
		RB_CUDA(dev_alloc(&c->batch_path_scene, c->wave_alloc));
		c->batch_path_alloc = c->wave_alloc;
	}
	c->wave.scene = c->batch_path_scene;
	c->wave.batch = c->batch_dev;
	c->wave.num_scenes = n;
	c->guide_mode = 0u;
	c->wave.guide = guide::wave_guide{};
	c->volume = false;
	c->wave.medium = nullptr;
	RB_CUDA(cudaMemcpyAsync(c->batch_dev, recs.data(), n * sizeof(gpu::batch_scene), cudaMemcpyHostToDevice, c->stream));

	gpu::wave_params& hp = *c->params_host;
	hp = gpu::wave_params{};
	hp.total_items = total;
	hp.max_depth = prm->max_depth;
	hp.rr_threshold = prm->rr_threshold;
	hp.guide_flags = 0u;

	st = run_waves(c, total, prm->max_depth, true);
	if (st != RB_OK) return st;
	if (c->stats.device_error != 0) return static_cast<rb_status>(c->stats.device_error);
	if (scene_ms != nullptr) {
		for (uint32_t k = 0; k < n; k++) {
			if (item_base[k] >= total) { scene_ms[k] = -1.f; continue; }  // not reached by a truncated probe
			const uint64_t last = (item_end[k] < total ? item_end[k] : total) - 1;
			float ms = 0.f;
			cudaEventElapsedTime(&ms, c->ev_begin, c->wave_events[last / c->wave_capacity]);
			scene_ms[k] = ms;
		}
	}
	return RB_OK;
}

// One timed probe under tuning t: the probe runs three times (the first run
// also records the wave graph) and the faster of the last two counts.
template <typename Probe>
rb_status time_probe(rb_context* c, const rb_tuning& t, Probe&& probe, float* ms) {
	if (std::memcmp(&t, &c->tuning, sizeof(t)) != 0) c->release_graph();
	c->tuning = t;
	float best = 0.f;
	for (int r = 0; r < 3; r++) {
		const rb_status st = probe();
		if (st != RB_OK) return st;
		if (r == 1 || (r > 1 && c->stats.elapsed_ms < best)) best = c->stats.elapsed_ms;
	}
	*ms = best;
	return RB_OK;
}

// Coordinate descent over the launch shapes (paths per wave with lanes,
// block sizes, grid size, sort key, tail bounce, traversal kind, shared-memory
// carve-out), two passes, starting from the context's current tuning. A change
// is kept when it is at least 1% faster.
template <typename Probe>
rb_status autotune(rb_context* c, uint64_t work_items, Probe&& probe, rb_tuning* best_out, float* best_ms_out) {
	const rb_tuning start = c->tuning;
	rb_tuning best = resolved_tuning(c->tuning);
	if (best.paths_per_wave == 0) best.paths_per_wave = 1u << 21;
	best.lanes = resolved_tuning(best).lanes;
	float best_ms = 0.f;
	rb_status st = time_probe(c, best, probe, &best_ms);
	if (st != RB_OK) { c->tuning = start; return st; }
	const uint32_t waves[] = {1u << 18, 1u << 19, 1u << 20, 1u << 21, 1u << 22};
	const uint32_t blocks[] = {64u, 128u, 256u};
	const uint32_t grids[] = {2u, 4u, 8u, 16u};
	const uint32_t sorts[] = {RB_SORT_MATERIAL, RB_SORT_NONE, RB_SORT_RAYS};
	const uint32_t tails[] = {1u, 2u, 3u, 4u, 6u, 64u};
	const uint32_t lane_counts[] = {1u, 2u, 3u, 4u, 6u, 8u};
	const uint32_t traversals[] = {RB_TRAVERSAL_PER_THREAD, RB_TRAVERSAL_REFILL};
	const uint32_t carveouts[] = {0u, 26u, 51u, 76u};  // largest, 25%, 50%, 75% (stored as percent + 1)
	auto try_value = [&](uint32_t rb_tuning::*field, uint32_t value) -> rb_status {
		if (best.*field == value) return RB_OK;
		rb_tuning t = best;
		t.*field = value;
		float ms = 0.f;
		const rb_status s = time_probe(c, t, probe, &ms);
		if (s != RB_OK) return s;
		if (ms < 0.99f * best_ms) {
			best = t;
			best_ms = ms;
		}
		return RB_OK;
	};
	// wave size and lanes interact (lanes only help with several waves), so
	// they are searched together
	auto try_waves_lanes = [&]() -> rb_status {
		const rb_tuning base = best;
		for (uint32_t v : waves) {
			// capacities above the work of a probe all run as one wave of that size
			if (v > work_items && v != waves[0] && (v >> 1) >= work_items) continue;
			for (uint32_t l : lane_counts) {
				if (l > 1 && v >= work_items) continue;  // a single wave has nothing to overlap
				rb_tuning t = base;
				t.paths_per_wave = v;
				t.lanes = l;
				if (std::memcmp(&t, &best, sizeof(t)) == 0) continue;
				float ms = 0.f;
				const rb_status s = time_probe(c, t, probe, &ms);
				if (s != RB_OK) return s;
				if (ms < 0.99f * best_ms) {
					best = t;
					best_ms = ms;
				}
			}
		}
		return RB_OK;
	};
	for (int pass = 0; pass < 2 && st == RB_OK; pass++) {
		st = try_waves_lanes();
		for (uint32_t v : blocks) if (st == RB_OK) st = try_value(&rb_tuning::block_trace, v);
		for (uint32_t v : blocks) if (st == RB_OK) st = try_value(&rb_tuning::block_shade, v);
		for (uint32_t v : grids) if (st == RB_OK) st = try_value(&rb_tuning::grid_per_sm, v);
		for (uint32_t v : sorts) if (st == RB_OK) st = try_value(&rb_tuning::sort, v);
		for (uint32_t v : tails) if (st == RB_OK) st = try_value(&rb_tuning::tail_bounce, v);
		for (uint32_t v : traversals) if (st == RB_OK) st = try_value(&rb_tuning::traversal, v);
		for (uint32_t v : carveouts) if (st == RB_OK) st = try_value(&rb_tuning::smem_carveout, v);
	}
	if (st != RB_OK) {
		c->release_graph();
		c->tuning = start;
		return st;
	}
	if (std::memcmp(&best, &c->tuning, sizeof(best)) != 0) c->release_graph();
	c->tuning = best;
	if (best_out) *best_out = best;
	if (best_ms_out) *best_ms_out = best_ms;
	return RB_OK;
}

} // namespace

extern "C" {

rb_status rb_set_tuning(rb_context* c, const rb_tuning* t) {
	if (c == nullptr) return RB_ERR_INVALID_ARGUMENT;
	const rb_status pending = async_finish(c);  // its graphs may be released below
	if (pending != RB_OK) return pending;
	rb_tuning v{};
	if (t != nullptr) v = *t;
	if (!valid_tuning(v)) return RB_ERR_INVALID_ARGUMENT;
	if (std::memcmp(&v, &c->tuning, sizeof(v)) != 0) c->release_graph();
	c->tuning = v;
	return RB_OK;
}

rb_status rb_get_tuning(rb_context* c, rb_tuning* t) {
	if (c == nullptr || t == nullptr) return RB_ERR_INVALID_ARGUMENT;
	*t = c->tuning;
	return RB_OK;
}

rb_status rb_tune_render(rb_context* c, const rb_render_params* params, uint32_t probe_spp, rb_tuning* best, float* best_ms) {
	if (c == nullptr || params == nullptr || probe_spp == 0) return RB_ERR_INVALID_ARGUMENT;
	if (!c->has_scene || c->is_batch) return RB_ERR_NO_SCENE;
	if (params->flags & (RB_RENDER_GUIDE | RB_RENDER_TRAIN)) return RB_ERR_INVALID_ARGUMENT;
	rb_render_params p = *params;
	p.spp = probe_spp;
	p.paths_per_wave = 0;  // the tuning's
	p.flags = (params->flags & (RB_RENDER_VOLUME | RB_RENDER_DIRECT)) | RB_RENDER_RESET;
	const uint64_t items = static_cast<uint64_t>(p.camera.width > 0 ? p.camera.width : 0) *
		static_cast<uint64_t>(p.camera.height > 0 ? p.camera.height : 0) * probe_spp;
	return autotune(c, items, [&]() { return rb_render(c, &p, nullptr); }, best, best_ms);
}

rb_status rb_batch_upload(rb_context* c, const rb_scene_desc* scenes, uint32_t count) {
	if (c == nullptr || scenes == nullptr || count == 0 || count > kMaxBatchScenes) return RB_ERR_INVALID_ARGUMENT;
	host::packed_scene merged;
	std::vector<host::scene_place> places;
	bool invisible = false;
	{
		std::vector<host::packed_scene> parts(count);
		for (uint32_t k = 0; k < count; k++) {
			const rb_status st = host::pack_scene(scenes + k, parts[k]);
			if (st != RB_OK) return st;
		}
		const rb_status st = host::merge_scenes(parts, merged, places);
		if (st != RB_OK) return st;
	}
	rb_status st = upload_packed(c, merged);
	if (st != RB_OK) return st;
	for (const auto& e : merged.entities)
		if ((e.flags & pt::ENT_HAS_SHAPE) && !(e.flags & pt::ENT_HAS_MATERIAL)) invisible = true;
	c->has_invisible = invisible;
	c->batch_scenes.assign(count, gpu::batch_scene{});
	for (uint32_t k = 0; k < count; k++) {
		gpu::batch_scene& b = c->batch_scenes[k];
		const host::scene_place& pl = places[k];
		b.root_a = pl.root_a;
		b.root_b = pl.root_b;
		b.root_ref = pl.root_ref;
		b.root_node = pl.root_node;
		b.emitter_base = pl.emitter_base;
		b.num_emitters = pl.num_emitters;
		b.env_base = pl.env_base;
		b.num_environments = pl.num_environments;
		b.env = pl.env;
	}
	RB_CUDA(dev_alloc(&c->batch_dev, count));
	c->wave.batch = c->batch_dev;
	c->wave.num_scenes = count;
	c->is_batch = true;
	c->batch_range.clear();
	c->release_film();
	return RB_OK;
}

rb_status rb_batch_render(rb_context* c, const rb_batch_params* params, float* scene_ms) {
	return batch_render(c, params, scene_ms, 0);
}

rb_status rb_batch_film_read(rb_context* c, uint32_t scene, double* sum_rgb, double* sum_sq_rgb, uint32_t* count) {
	if (c == nullptr) return RB_ERR_INVALID_ARGUMENT;
	if (!c->is_batch || c->batch_range.empty()) return RB_ERR_NO_SCENE;
	if (scene >= c->batch_range.size()) return RB_ERR_INVALID_ARGUMENT;
	RB_CUDA(cudaSetDevice(c->device));
	RB_CUDA(cudaStreamSynchronize(c->stream));
	const size_t g0 = c->batch_range[scene].first;
	const size_t px = c->batch_range[scene].second;
	if (sum_rgb) RB_CUDA(cudaMemcpy(sum_rgb, c->film.sum + 3 * g0, 3 * px * sizeof(double), cudaMemcpyDeviceToHost));
	if (sum_sq_rgb) RB_CUDA(cudaMemcpy(sum_sq_rgb, c->film.sum_sq + 3 * g0, 3 * px * sizeof(double), cudaMemcpyDeviceToHost));
	if (count) RB_CUDA(cudaMemcpy(count, c->film.count + g0, px * sizeof(uint32_t), cudaMemcpyDeviceToHost));
	return RB_OK;
}

rb_status rb_batch_image(rb_context* c, uint32_t scene, float* rgb_out) {
	if (c == nullptr || rgb_out == nullptr) return RB_ERR_INVALID_ARGUMENT;
	if (!c->is_batch || c->batch_range.empty()) return RB_ERR_NO_SCENE;
	if (scene >= c->batch_range.size()) return RB_ERR_INVALID_ARGUMENT;
	RB_CUDA(cudaSetDevice(c->device));
	const uint32_t g0 = c->batch_range[scene].first, px = c->batch_range[scene].second;
	const gpu::film_buffers f{c->film.sum + 3 * static_cast<size_t>(g0), c->film.sum_sq + 3 * static_cast<size_t>(g0),
		c->film.count + g0};
	RB_CUDA(gpu::launch_film_mean(f, px, c->film_mean + 3 * static_cast<size_t>(g0), c->num_sms * 4, c->stream));
	RB_CUDA(cudaMemcpyAsync(rgb_out, c->film_mean + 3 * static_cast<size_t>(g0), 3 * static_cast<size_t>(px) * sizeof(float),
		cudaMemcpyDeviceToHost, c->stream));
	RB_CUDA(cudaStreamSynchronize(c->stream));
	return RB_OK;
}

rb_status rb_tune_batch(rb_context* c, const rb_batch_params* params, uint64_t probe_items, rb_tuning* best, float* best_ms) {
	if (c == nullptr || params == nullptr || probe_items == 0) return RB_ERR_INVALID_ARGUMENT;
	if (!c->is_batch) return RB_ERR_NO_SCENE;
	rb_batch_params p = *params;
	p.flags = RB_RENDER_RESET;
	return autotune(c, probe_items, [&]() { return batch_render(c, &p, nullptr, probe_items); }, best, best_ms);
}

} // extern "C"
