// C ABI of the wavefront path-tracing core (include/rbgpu.h).
//
// A context owns one device's memory: the packed scene, the wave buffers, the
// film accumulators (FP64 sums and squared sums, sample counts) and one CUDA
// graph per (wave capacity, depth, counting) configuration. A render call
// splits its pixels x spp work items into waves; each wave is one replay of the
// captured graph (camera rays plus max_depth bounces), with the wave's first
// work item written to a device-side parameter block before the replay.
#include "context.h"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

using namespace rb;

using namespace rb::ctx;

namespace {
constexpr uint32_t kCheckpointMagic = 0x52424350u;  // "RBCP"
} // namespace

namespace rb {
namespace ctx {

cudaError_t alloc_wave_buffers(gpu::wave_buffers& w, size_t n) {
	cudaError_t e = cudaSuccess;
	auto take = [&](auto** p, size_t count) {
		if (e == cudaSuccess) e = dev_alloc(p, count);
	};
	take(&w.ray_o, n); take(&w.ray_d, n); take(&w.beta, n); take(&w.radiance, n); take(&w.bounces, n);
	take(&w.rng, n); take(&w.pixel, n); take(&w.sample, n); take(&w.hit, n); take(&w.rec, n); take(&w.result, n);
	take(&w.sec_o, 2 * n); take(&w.sec_d, 2 * n); take(&w.sec_hit, 2 * n); take(&w.queue[0], n); take(&w.queue[1], n);
	take(&w.sec_queue, 2 * n);
	take(&w.class_queue, static_cast<size_t>(pt::NUM_CLASSES) * n);
	take(&w.sort_keys, n);
	take(&w.sort_tmp, n);
	take(&w.sort_bins, 2 * gpu::kSortBins);
	if (e == cudaSuccess) e = cudaMemset(w.sort_bins, 0, 2 * gpu::kSortBins * sizeof(uint32_t));
	return e;
}

void free_wave_buffers(gpu::wave_buffers& w) {
	dev_free(w.ray_o); dev_free(w.ray_d); dev_free(w.beta); dev_free(w.radiance); dev_free(w.bounces);
	dev_free(w.rng); dev_free(w.pixel); dev_free(w.sample); dev_free(w.hit); dev_free(w.rec); dev_free(w.result);
	dev_free(w.sec_o); dev_free(w.sec_d); dev_free(w.sec_hit); dev_free(w.queue[0]); dev_free(w.queue[1]);
	dev_free(w.sec_queue);
	dev_free(w.class_queue);
	dev_free(w.sort_keys);
	dev_free(w.sort_tmp);
	dev_free(w.sort_bins);
}

std::atomic<int32_t>& allocation_countdown() {
	static std::atomic<int32_t> countdown{-1};
	return countdown;
}

rb_status ensure_wave(rb_context* c, uint32_t capacity) {
	if (c->wave_alloc >= capacity) {
		// same buffers, smaller waves: the kernels read the wave size from wave.capacity
		if (c->wave_capacity != capacity) c->release_graph();
		c->wave.capacity = capacity;
		c->wave_capacity = capacity;
		return RB_OK;
	}
	c->release_graph();
	c->release_wave();
	RB_CUDA(alloc_wave_buffers(c->wave, capacity));
	gpu::wave_buffers& w = c->wave;
	w.capacity = capacity;
	w.counters = c->counters;
	c->wave_capacity = capacity;
	c->wave_alloc = capacity;
	return RB_OK;
}

rb_status ensure_lanes(rb_context* c, uint32_t count) {
	if (count > kMaxLanes) return RB_ERR_INVALID_ARGUMENT;
	while (c->lanes.size() + 1 < count) c->lanes.emplace_back();
	for (uint32_t k = 0; k + 1 < count; k++) {
		wave_lane& l = c->lanes[k];
		if (l.stream == nullptr) {
			RB_CUDA(cudaStreamCreateWithFlags(&l.stream, cudaStreamNonBlocking));
			RB_CUDA(cudaEventCreateWithFlags(&l.done, cudaEventDisableTiming));
			RB_CUDA(dev_alloc(&l.counters, gpu::CNT_WORDS));
			RB_CUDA(dev_alloc(&l.params, 1));
		}
		if (l.alloc < c->wave_capacity) {
			l.release_graph();
			free_wave_buffers(l.wave);
			dev_free(l.path_scene);
			l.alloc = 0;
			RB_CUDA(alloc_wave_buffers(l.wave, c->wave_capacity));
			RB_CUDA(dev_alloc(&l.path_scene, c->wave_capacity));
			l.alloc = c->wave_capacity;
		}
		l.wave.capacity = c->wave_capacity;
		l.wave.counters = l.counters;
		l.wave.params = l.params;
		l.wave.guide = guide::wave_guide{};
		l.wave.guide_medium = guide::wave_guide{};
		if (c->volume && l.vol_alloc < c->wave_capacity) {
			l.release_graph();
			dev_free(l.vol_medium); dev_free(l.vol_rec); dev_free(l.vol_beam); dev_free(l.vol_beam_queue);
			l.vol_alloc = 0;
			RB_CUDA(dev_alloc(&l.vol_medium, c->wave_capacity));
			RB_CUDA(dev_alloc(&l.vol_rec, c->wave_capacity));
			RB_CUDA(dev_alloc(&l.vol_beam, 2 * static_cast<size_t>(c->wave_capacity)));
			RB_CUDA(dev_alloc(&l.vol_beam_queue, 2 * static_cast<size_t>(c->wave_capacity)));
			l.vol_alloc = c->wave_capacity;
		}
		l.wave.medium = c->volume ? l.vol_medium : nullptr;
		l.wave.vrec = c->volume ? l.vol_rec : nullptr;
		l.wave.beam = c->volume ? l.vol_beam : nullptr;
		l.wave.beam_queue = c->volume ? l.vol_beam_queue : nullptr;
		l.wave.batch = c->wave.batch;
		l.wave.num_scenes = c->wave.num_scenes;
		l.wave.scene = l.path_scene;
	}
	return RB_OK;
}

rb_status ensure_film(rb_context* c, int32_t width, int32_t height, bool reset) {
	if (c->film_w != width || c->film_h != height) {
		c->release_film();
		const size_t px = static_cast<size_t>(width) * height;
		RB_CUDA(dev_alloc(&c->film.sum, 3 * px));
		RB_CUDA(dev_alloc(&c->film.sum_sq, 3 * px));
		RB_CUDA(dev_alloc(&c->film.count, px));
		RB_CUDA(dev_alloc(&c->film_mean, 3 * px));
		c->film_w = width;
		c->film_h = height;
		reset = true;
	}
	if (reset) {
		const size_t px = static_cast<size_t>(width) * height;
		RB_CUDA(cudaMemsetAsync(c->film.sum, 0, 3 * px * sizeof(double), c->stream));
		RB_CUDA(cudaMemsetAsync(c->film.sum_sq, 0, 3 * px * sizeof(double), c->stream));
		RB_CUDA(cudaMemsetAsync(c->film.count, 0, px * sizeof(uint32_t), c->stream));
		c->film_samples = 0;
	}
	return RB_OK;
}

// Records one wave of buffers `w` on stream `s` into a graph: counter reset,
// camera rays and bounces, and with_end the film resolve / guide training that
// close the wave. Kept while the configuration is unchanged.
// Appends the drain loop to the graph being captured on `s`: a kernel that sets
// the loop condition from the active count, then a conditional WHILE node whose
// body (captured on `body`) is two bounces and the condition update. The first
// body bounce reads the queue the host-driven loop would read after max_depth
// bounces; a second bounce on an emptied queue launches kernels that find no
// work.
cudaError_t capture_drain(rb_context* c, const gpu::wave_buffers& w, cudaStream_t s, cudaStream_t body, uint32_t* counters,
	uint32_t max_depth, const gpu::launch_cfg& cfg) {
	cudaStreamCaptureStatus status;
	cudaGraph_t graph = nullptr;
	const cudaGraphNode_t* deps = nullptr;
	size_t ndeps = 0;
	cudaError_t e = cudaStreamGetCaptureInfo(s, &status, nullptr, &graph, &deps, &ndeps);
	if (e != cudaSuccess) return e;
	if (status != cudaStreamCaptureStatusActive) return cudaErrorStreamCaptureInvalidated;
	cudaGraphConditionalHandle h;
	e = cudaGraphConditionalHandleCreate(&h, graph, 0u, cudaGraphCondAssignDefault);
	if (e == cudaSuccess) e = gpu::launch_drain_begin(h, counters, s);
	if (e == cudaSuccess) e = cudaStreamGetCaptureInfo(s, &status, nullptr, &graph, &deps, &ndeps);
	if (e != cudaSuccess) return e;
	cudaGraphNodeParams np{};
	np.type = cudaGraphNodeTypeConditional;
	np.conditional.handle = h;
	np.conditional.type = cudaGraphCondTypeWhile;
	np.conditional.size = 1;
	cudaGraphNode_t node;
	e = cudaGraphAddNode(&node, graph, deps, ndeps, &np);
	if (e != cudaSuccess) return e;
	cudaGraph_t body_graph = np.conditional.phGraph_out[0];
	e = cudaStreamBeginCaptureToGraph(body, body_graph, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
	if (e != cudaSuccess) return e;
	const uint32_t q = max_depth & 1u;
	e = gpu::launch_bounce(c->view, w, c->film, q, cfg, body);
	if (e == cudaSuccess) e = gpu::launch_bounce(c->view, w, c->film, q ^ 1u, cfg, body);
	if (e == cudaSuccess) e = gpu::launch_drain_step(h, counters, body);
	cudaGraph_t captured = nullptr;
	const cudaError_t e2 = cudaStreamEndCapture(body, &captured);
	if (e != cudaSuccess) return e;
	if (e2 != cudaSuccess) return e2;
	return cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies);
}

rb_status capture_into(rb_context* c, const gpu::wave_buffers& w, cudaStream_t s, uint32_t* counters, uint32_t max_depth,
	bool with_end, cudaGraphExec_t& graph, graph_key& current) {
	const gpu::launch_cfg cfg = c->cfg();
	graph_key key;
	key.capacity = c->wave_capacity;
	key.max_depth = max_depth;
	key.stack = static_cast<uint32_t>(cfg.stack_depth);
	key.count = cfg.count;
	key.guide_mode = cfg.guide_mode;
	key.volume = cfg.volume;
	key.batch = cfg.batch;
	key.with_end = with_end;
	key.block_trace = static_cast<uint32_t>(cfg.block_trace);
	key.block_shade = static_cast<uint32_t>(cfg.block_shade);
	key.grid_trace = static_cast<uint32_t>(cfg.grid_trace);
	key.grid_shade = static_cast<uint32_t>(cfg.grid_shade);
	key.sort = cfg.sort;
	key.tail = cfg.tail;
	key.refill = cfg.refill;
	key.shadow_first = cfg.shadow_first;
	key.sss = cfg.sss;
	key.carveout = cfg.carveout;
	if (cfg.guide) {
		key.guide_steps = cfg.guide->cfg.steps_per_wave;
		key.guide_batch = cfg.guide->cfg.batch_size;
	}
	if (graph && current == key) return RB_OK;
	if (graph) cudaGraphExecDestroy(graph);
	graph = nullptr;
	current = graph_key();
	// scenes with invisible entities: the drain loop's body is captured on a
	// second stream into the conditional node's child graph
	const bool drain = c->has_invisible;
	cudaStream_t body_stream = nullptr;
	if (drain) RB_CUDA(cudaStreamCreateWithFlags(&body_stream, cudaStreamNonBlocking));
	cudaGraph_t g = nullptr;
	cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
	if (e != cudaSuccess) {
		if (body_stream) cudaStreamDestroy(body_stream);
		return from_cuda(e);
	}
	e = cudaMemsetAsync(counters, 0, gpu::kWaveCounterWords * sizeof(uint32_t), s);
	if (e == cudaSuccess) e = gpu::launch_wave(c->view, w, c->film, max_depth, 0u, cfg, s);
	if (e == cudaSuccess && drain) e = capture_drain(c, w, s, body_stream, counters, max_depth, cfg);
	if (e == cudaSuccess && with_end) e = gpu::launch_wave_end(w, c->film, c->num_sms * 4, cfg, s);
	const cudaError_t e2 = cudaStreamEndCapture(s, &g);
	if (body_stream) cudaStreamDestroy(body_stream);
	if (e != cudaSuccess || e2 != cudaSuccess) {
		if (g) cudaGraphDestroy(g);
		if (drain) c->drain_graph_failed = true;
		return from_cuda(e != cudaSuccess ? e : e2);
	}
	e = cudaGraphInstantiate(&graph, g, 0);
	cudaGraphDestroy(g);
	RB_CUDA(e);
	current = key;
	return RB_OK;
}

rb_status capture_wave(rb_context* c, uint32_t max_depth) {
	return capture_into(c, c->wave, c->stream, c->counters, max_depth, true, c->graph, c->graph_cfg);
}

// Learned guiding for one render call: the guide (default configuration on
// first use), its per-path buffers for this wave size and depth, and the
// pointers the kernels read. A plain render leaves the guide untouched.
// A guided volume render also prepares the medium guide (created from the
// surface guide's configuration with seed + 1 on first use).
rb_status prepare_guide(rb_context* c, const rb_render_params* prm) {
	c->guide_mode = 0u;
	c->wave.guide = guide::wave_guide{};
	c->wave.guide_medium = guide::wave_guide{};
	if (!(prm->flags & (RB_RENDER_GUIDE | RB_RENDER_TRAIN))) return RB_OK;
	if (!c->guide.ready) {
		const rb_status st = rb_guide_init(c, nullptr);
		if (st != RB_OK) return st;
	}
	auto attach = [&](guide::guide_state& g, guide::wave_guide& w) -> rb_status {
		const float4* before = g.query_in;
		RB_CUDA(guide::allocate_wave(g, c->wave_capacity, prm->max_depth));
		if (g.query_in != before) c->release_graph();
		w = guide::state_view(g);
		return RB_OK;
	};
	rb_status st = attach(c->guide, c->wave.guide);
	if (st != RB_OK) return st;
	if (prm->flags & RB_RENDER_VOLUME) {
		if (!c->guide_medium.ready) {
			c->release_graph();
			rb_guide_config mc = c->guide.cfg;
			mc.seed += 1u;
			st = guide::init_state(c->guide_medium, &mc, c->num_sms, c->stream);
			if (st != RB_OK) return st;
		}
		st = attach(c->guide_medium, c->wave.guide_medium);
		if (st != RB_OK) return st;
	}
	c->guide_mode = ((prm->flags & RB_RENDER_GUIDE) ? gpu::GUIDE_SAMPLE : 0u) | ((prm->flags & RB_RENDER_TRAIN) ? gpu::GUIDE_TRAIN : 0u);
	return RB_OK;
}

// Volume path tracing: per-path medium, light-connection records and
// transmittance buffers, allocated with the wave on first use.
rb_status prepare_volume(rb_context* c, const rb_render_params* prm) {
	c->volume = (prm->flags & RB_RENDER_VOLUME) != 0;
	if (!c->volume) {
		c->wave.medium = nullptr;  // plain kernels see no media
		return RB_OK;
	}
	if (c->vol_alloc < c->wave_alloc) {
		c->release_graph();
		dev_free(c->vol_medium); dev_free(c->wave.vrec); dev_free(c->wave.beam); dev_free(c->wave.beam_queue);
		c->vol_alloc = 0;
		const size_t n = c->wave_alloc;
		RB_CUDA(dev_alloc(&c->vol_medium, n));
		RB_CUDA(dev_alloc(&c->wave.vrec, n));
		RB_CUDA(dev_alloc(&c->wave.beam, 2 * n));
		RB_CUDA(dev_alloc(&c->wave.beam_queue, 2 * n));
		c->vol_alloc = c->wave_alloc;
	}
	c->wave.medium = c->vol_medium;
	return RB_OK;
}

// Wave lanes a render call can use: more than one for any render replayed
// from graphs (not while profiling), with at least two waves.
// async: calls that overlap on the GPU take their waves on the lanes in turn
// across calls (a call of one wave runs beside the previous call's), so they
// get every lane the tuning asks for.
uint32_t lanes_for(const rb_context* c, uint64_t total, const gpu::launch_cfg& cfg, bool async = false) {
	const uint32_t want = resolved_tuning(c->tuning).lanes;
	if (want <= 1 || c->profiling || (c->has_invisible && c->drain_graph_failed)) return 1;
	if (async) return want;
	const uint64_t waves = (total + c->wave_capacity - 1) / c->wave_capacity;
	return static_cast<uint32_t>(waves < want ? waves : want);
}

// Traversal time of a render call: with profiling, CUDA events around each
// launch; otherwise the device-clock timers the traversal kernels keep in the
// counters of each lane (the span of each launch from its first warp's start to
// its last warp's end), summed over the lanes.
void traversal_times(rb_context* c, uint32_t nlanes, rb_render_stats& s) {
	s.extend_ms = s.secondary_ms = 0.f;
	s.extend_launches = s.secondary_launches = 0;
	if (c->profiling) {
		for (uint32_t k = 0; k < c->next_event; k++) {
			float ms = 0.f;
			cudaEventElapsedTime(&ms, c->events[2 * k], c->events[2 * k + 1]);
			if (c->event_kind[k] == 0) { s.extend_ms += ms; s.extend_launches++; }
			else { s.secondary_ms += ms; s.secondary_launches++; }
		}
		return;
	}
	auto u64 = [](const uint32_t* a, uint32_t w) { return static_cast<uint64_t>(a[w]) | (static_cast<uint64_t>(a[w + 1]) << 32); };
	uint64_t ext_ns = 0, sec_ns = 0;
	for (uint32_t k = 0; k < nlanes; k++) {
		const uint32_t* a = c->counters_host + k * gpu::CNT_WORDS;
		ext_ns += u64(a, gpu::CNT_TIMER_EXTEND + gpu::TIMER_TOTAL_NS);
		sec_ns += u64(a, gpu::CNT_TIMER_SECONDARY + gpu::TIMER_TOTAL_NS);
		s.extend_launches += a[gpu::CNT_TIMER_EXTEND + gpu::TIMER_LAUNCHES];
		s.secondary_launches += a[gpu::CNT_TIMER_SECONDARY + gpu::TIMER_LAUNCHES];
	}
	s.extend_ms = static_cast<float>(ext_ns * 1e-6);
	s.secondary_ms = static_cast<float>(sec_ns * 1e-6);
}

// Runs the waves of one render call, whose parameters are in c->params_host
// (first_item is set here): one graph replay per wave, or direct launches when
// profiling or when invisible entities make paths outlive max_depth
// iterations. With several lanes, wave j runs on lane j mod lanes (own buffers
// and stream) and its film resolve waits for wave j - 1's, so the waves'
// bounces overlap while the film adds them in order. record_waves: event
// c->wave_events[j] after wave j's resolve. Fills the call's statistics.
bool is_page_locked(const void* p) {
	cudaPointerAttributes a{};
	if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
		cudaGetLastError();  // unknown pointers are plain host memory here
		return false;
	}
	return a.type == cudaMemoryTypeHost;
}

// Means of the pixels made final by the items resolved so far, copied to the
// caller's buffer on stream s (see image_readback).
rb_status readback_after(rb_context* c, image_readback* r, uint64_t resolved_items, cudaStream_t s) {
	if (r == nullptr || resolved_items <= r->final_from) return RB_OK;
	const uint64_t upto = std::min<uint64_t>(r->pixels, resolved_items - r->final_from);
	if (upto <= r->done) return RB_OK;
	const size_t first = static_cast<size_t>(r->done), n = static_cast<size_t>(upto - r->done);
	const gpu::film_buffers f{c->film.sum + 3 * first, c->film.sum_sq + 3 * first, c->film.count + first};
	RB_CUDA(gpu::launch_film_mean(f, static_cast<uint32_t>(n), c->film_mean + 3 * first, c->num_sms, s));
	RB_CUDA(cudaMemcpyAsync(r->host + 3 * first, c->film_mean + 3 * first, 3 * n * sizeof(float), cudaMemcpyDeviceToHost, s));
	r->done = upto;
	return RB_OK;
}

// The statistics of the waves that ran since the counters were last cleared:
// lane 0's counters, with the other lanes' statistics and first error added.
void take_stats(rb_context* c, uint32_t nlanes, uint64_t samples, uint32_t launches, bool use_graph,
	const gpu::launch_cfg& cfg) {
	uint32_t* h = c->counters_host;
	auto u64 = [&](const uint32_t* a, uint32_t w) { return static_cast<uint64_t>(a[w]) | (static_cast<uint64_t>(a[w + 1]) << 32); };
	rb_render_stats& s = c->stats;
	s = rb_render_stats{};
	for (uint32_t k = 0; k < nlanes; k++) {
		const uint32_t* a = h + k * gpu::CNT_WORDS;
		s.extend_rays += u64(a, gpu::CNT_EXTEND_RAYS);
		s.shadow_rays += u64(a, gpu::CNT_SHADOW_RAYS);
		s.mis_rays += u64(a, gpu::CNT_MIS_RAYS);
		s.node_visits += u64(a, gpu::CNT_NODE_VISITS);
		s.triangle_tests += u64(a, gpu::CNT_TRI_TESTS);
		if (s.device_error == 0) s.device_error = a[gpu::CNT_ERROR];
		if (use_graph) launches += a[gpu::CNT_DRAIN_TOTAL] * gpu::drain_launches(cfg);
	}
	h[gpu::CNT_ERROR] = s.device_error;
	s.samples = samples;
	s.kernel_launches = launches;
	cudaEventElapsedTime(&s.elapsed_ms, c->ev_begin, c->ev_end);
	traversal_times(c, nlanes, s);
}

rb_status async_finish(rb_context* c) {
	if (c->async.pending == 0) return RB_OK;
	const uint32_t nlanes = c->async.lanes;
	for (uint32_t k = 0; k + 1 < nlanes; k++) RB_CUDA(cudaStreamWaitEvent(c->stream, c->lanes[k].done, 0));
	RB_CUDA(cudaEventRecord(c->ev_end, c->stream));
	const cudaError_t e = cudaStreamSynchronize(c->stream);
	const rb_context::async_state a = c->async;
	c->async = rb_context::async_state{};
	RB_CUDA(e);
	take_stats(c, nlanes, a.samples, a.launches, a.use_graph, c->profiled_cfg());
	return c->counters_host[gpu::CNT_ERROR] != 0 ? static_cast<rb_status>(c->counters_host[gpu::CNT_ERROR]) : RB_OK;
}

rb_status run_waves(rb_context* c, uint64_t total, uint32_t max_depth, bool record_waves, image_readback* readback,
	bool async) {
	gpu::wave_params& hp = *c->params_host;
	rb_status st = RB_OK;
	const gpu::launch_cfg cfg = c->profiled_cfg();
	// a later async call of the same configuration: no clearing, no start
	// barrier across the lanes; its counters add to the pending calls'
	const bool continuing = async && c->async.pending > 0;
	const uint32_t nlanes = lanes_for(c, total, cfg, async);
	const uint64_t waves = (total + c->wave_capacity - 1) / c->wave_capacity;
	// the lane of the call's first wave: the one after the previous async call's last wave
	const uint32_t first_lane = continuing ? c->async.next_lane % nlanes : 0u;
	if (record_waves || nlanes > 1) {
		while (c->wave_events.size() < waves) {
			cudaEvent_t e;
			RB_CUDA(cudaEventCreate(&e));
			c->wave_events.push_back(e);
		}
	}
	if (!continuing) RB_CUDA(cudaMemsetAsync(c->counters, 0, gpu::CNT_WORDS * sizeof(uint32_t), c->stream));
	// scenes with invisible entities replay graphs too (their drain loop is a
	// conditional node) unless the runtime refused that node
	const bool use_graph = !c->profiling && !(c->has_invisible && c->drain_graph_failed);
	const uint32_t drain_begin = c->has_invisible ? 1u : 0u;  // launches of the drain set-up per graph wave
	c->next_event = 0;
	const bool guided = nlanes > 1 && cfg.guide != nullptr;
	const bool training = guided && (cfg.guide_mode & gpu::GUIDE_TRAIN);
	if (nlanes > 1) {
		st = ensure_lanes(c, nlanes);
		// guided waves on lanes: each lane's own guide buffers and its snapshot of the
		// weights, taken after the lane's previous wave trained (a fixed lag of
		// nlanes - 1 waves behind the newest weights, independent of timing)
		for (uint32_t k = 0; k < nlanes && st == RB_OK && guided; k++) {
			guide::lane_guide& lg = c->lane_guides[k];
			const float4* before = lg.query_in;
			const cudaError_t e = guide::allocate_lane(lg, c->wave_capacity, max_depth);
			if (e != cudaSuccess) st = from_cuda(e);
			else if (lg.query_in != before) c->release_graph();
			const guide::wave_guide wg = guide::lane_view(c->guide, lg);
			if (k == 0) c->wave.guide = wg;
			else c->lanes[k - 1].wave.guide = wg;
			if (st != RB_OK || cfg.guide_medium == nullptr) continue;
			// guided volume renders: the medium guide's lane buffers and snapshot alike
			guide::lane_guide& lm = c->lane_guides_medium[k];
			const float4* before_m = lm.query_in;
			const cudaError_t em = guide::allocate_lane(lm, c->wave_capacity, max_depth);
			if (em != cudaSuccess) st = from_cuda(em);
			else if (lm.query_in != before_m) c->release_graph();
			const guide::wave_guide wm = guide::lane_view(c->guide_medium, lm);
			if (k == 0) c->wave.guide_medium = wm;
			else c->lanes[k - 1].wave.guide_medium = wm;
		}
		if (st == RB_OK) st = capture_into(c, c->wave, c->stream, c->counters, max_depth, false, c->graph, c->graph_cfg);
		for (uint32_t k = 0; k + 1 < nlanes && st == RB_OK; k++) {
			wave_lane& l = c->lanes[k];
			st = capture_into(c, l.wave, l.stream, l.counters, max_depth, false, l.graph, l.key);
		}
		if (st != RB_OK && c->has_invisible && c->drain_graph_failed)
			return run_waves(c, total, max_depth, record_waves, readback, async);
		if (st != RB_OK) return st;
	} else if (use_graph) {
		st = capture_wave(c, max_depth);
		if (st != RB_OK && c->has_invisible && c->drain_graph_failed)
			return run_waves(c, total, max_depth, record_waves, readback, async);
		if (st != RB_OK) return st;
	}
	uint32_t launches = 0;
	hp.first_item = 0;
	RB_CUDA(gpu::launch_set_params(hp, c->wave.params, c->stream));
	for (uint32_t k = 0; guided && k < nlanes; k++) {
		RB_CUDA(guide::launch_snapshot(c->guide, c->lane_guides[k], c->stream));
		if (cfg.guide_medium != nullptr)
			RB_CUDA(guide::launch_snapshot(*cfg.guide_medium, c->lane_guides_medium[k], c->stream));
	}
	if (!continuing) RB_CUDA(cudaEventRecord(c->ev_begin, c->stream));
	if (nlanes > 1) {
		for (uint32_t k = 0; k + 1 < nlanes; k++) {
			wave_lane& l = c->lanes[k];
			if (!continuing) {
				RB_CUDA(cudaStreamWaitEvent(l.stream, c->ev_begin, 0));
				RB_CUDA(cudaMemsetAsync(l.counters, 0, gpu::CNT_WORDS * sizeof(uint32_t), l.stream));
			}
			RB_CUDA(gpu::launch_set_params(hp, l.params, l.stream));
		}
		for (uint64_t j = 0; j < waves; j++) {
			const uint32_t lane = static_cast<uint32_t>((first_lane + j) % nlanes);
			const cudaStream_t s = lane == 0 ? c->stream : c->lanes[lane - 1].stream;
			const gpu::wave_buffers& w = lane == 0 ? c->wave : c->lanes[lane - 1].wave;
			const cudaGraphExec_t g = lane == 0 ? c->graph : c->lanes[lane - 1].graph;
			RB_CUDA(gpu::launch_set_first(w.params, j * c->wave_capacity, s));
			RB_CUDA(cudaGraphLaunch(g, s));
			if (j > 0) RB_CUDA(cudaStreamWaitEvent(s, c->wave_events[j - 1], 0));
			else if (continuing) RB_CUDA(cudaStreamWaitEvent(s, c->wave_events[c->async.waves - 1], 0));  // the previous call's last wave
			// in wave order: training-sample collection, film resolve, training, then this lane's snapshot
			RB_CUDA(gpu::launch_wave_end(w, c->film, c->num_sms * 4, cfg, s));
			if (training) RB_CUDA(guide::launch_snapshot(c->guide, c->lane_guides[lane], s));
			if (training && cfg.guide_medium != nullptr)
				RB_CUDA(guide::launch_snapshot(*cfg.guide_medium, c->lane_guides_medium[lane], s));
			// the image slice this wave completes is read back before the wave's event, so that
			// the next wave to resolve into the film (of this call or the next, on any lane)
			// waits for the read
			st = readback_after(c, readback, std::min<uint64_t>(total, (j + 1) * c->wave_capacity), s);
			if (st != RB_OK) return st;
			RB_CUDA(cudaEventRecord(c->wave_events[j], s));
			launches += gpu::wave_launches(max_depth, cfg) + 1u + drain_begin;
		}
		for (uint32_t k = 0; k + 1 < nlanes; k++) {
			wave_lane& l = c->lanes[k];
			RB_CUDA(cudaMemcpyAsync(c->counters_host + (k + 1) * gpu::CNT_WORDS, l.counters, gpu::CNT_WORDS * sizeof(uint32_t),
				cudaMemcpyDeviceToHost, l.stream));
			RB_CUDA(cudaEventRecord(l.done, l.stream));
			if (!async) RB_CUDA(cudaStreamWaitEvent(c->stream, l.done, 0));
		}
	} else {
		uint64_t wave = 0;
		for (uint64_t first = 0; first < total; first += c->wave_capacity, wave++) {
			if (use_graph) {
				// the graph's last node moves params->first_item to the next wave
				RB_CUDA(cudaGraphLaunch(c->graph, c->stream));
				launches += gpu::wave_launches(max_depth, cfg) + drain_begin;
			} else {
				// direct launches: profiling, or invisible entities (a pass-through
				// does not count as a bounce, so keep bouncing until the queue drains)
				RB_CUDA(cudaMemsetAsync(c->counters, 0, gpu::kWaveCounterWords * sizeof(uint32_t), c->stream));
				RB_CUDA(gpu::launch_wave(c->view, c->wave, c->film, max_depth, 0u, cfg, c->stream));
				launches += gpu::wave_launches(max_depth, cfg) - 2u;
				uint32_t q = max_depth & 1u;
				for (int guard = 0; guard < 4096 && c->has_invisible; guard++) {
					RB_CUDA(cudaMemcpyAsync(c->counters_host, c->counters, sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
					RB_CUDA(cudaStreamSynchronize(c->stream));
					if (c->counters_host[gpu::CNT_ACTIVE] == 0) break;
					RB_CUDA(gpu::launch_bounce(c->view, c->wave, c->film, q, cfg, c->stream));
					launches += (cfg.sort == RB_SORT_NONE ? 7u : 12u) + ((cfg.guide_mode & gpu::GUIDE_SAMPLE) ? 1u : 0u);
					q ^= 1u;
				}
				RB_CUDA(gpu::launch_wave_end(c->wave, c->film, c->num_sms * 4, cfg, c->stream));
			}
			if (record_waves) RB_CUDA(cudaEventRecord(c->wave_events[wave], c->stream));
			st = readback_after(c, readback, std::min<uint64_t>(total, first + c->wave_capacity), c->stream);
			if (st != RB_OK) return st;
		}
	}
	if (async) {
		// lane 0's counters follow its last wave; the host reads them at rb_render_wait
		RB_CUDA(cudaMemcpyAsync(c->counters_host, c->counters, gpu::CNT_WORDS * sizeof(uint32_t), cudaMemcpyDeviceToHost,
			c->stream));
		c->async.pending++;
		c->async.waves = waves;
		c->async.lanes = nlanes;
		c->async.next_lane = static_cast<uint32_t>((first_lane + waves) % nlanes);
		c->async.samples += total;
		c->async.launches += launches;
		c->async.use_graph = use_graph;
		return RB_OK;
	}
	RB_CUDA(cudaEventRecord(c->ev_end, c->stream));
	RB_CUDA(cudaMemcpyAsync(c->counters_host, c->counters, gpu::CNT_WORDS * sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
	RB_CUDA(cudaStreamSynchronize(c->stream));
	take_stats(c, nlanes, total, launches, use_graph, cfg);
	return RB_OK;
}

// Waves of a RB_RENDER_DIRECT call: one k_direct launch per wave, then its
// film resolve (in wave order, as in run_waves).
rb_status run_direct(rb_context* c, uint64_t total, const pt::direct_cfg& dc, image_readback* readback) {
	gpu::wave_params& hp = *c->params_host;
	const gpu::launch_cfg cfg = c->cfg();
	// the staged kernels when the light samples fit their records, else one thread per sample;
	// their buffers are allocated before the timed region
	const bool staged = dc.emitter_samples <= pt::kDirectStagedLights;
	if (staged && c->direct_alloc < c->wave_capacity) {
		gpu::direct_buffers& db = c->direct;
		dev_free(db.rec); dev_free(db.ray_o); dev_free(db.ray_d); dev_free(db.ray_hit);
		dev_free(db.ray_queue); dev_free(db.shade_queue);
		c->direct_alloc = 0;
		const size_t n = c->wave_capacity, slots = n * gpu::kDirectSlots;
		RB_CUDA(dev_alloc(&db.rec, n));
		RB_CUDA(dev_alloc(&db.ray_o, slots));
		RB_CUDA(dev_alloc(&db.ray_d, slots));
		RB_CUDA(dev_alloc(&db.ray_hit, slots));
		RB_CUDA(dev_alloc(&db.ray_queue, slots));
		RB_CUDA(dev_alloc(&db.shade_queue, n));
		c->direct_alloc = c->wave_capacity;
	}
	RB_CUDA(cudaMemsetAsync(c->counters, 0, gpu::CNT_WORDS * sizeof(uint32_t), c->stream));
	hp.first_item = 0;
	RB_CUDA(gpu::launch_set_params(hp, c->wave.params, c->stream));
	RB_CUDA(cudaEventRecord(c->ev_begin, c->stream));
	uint32_t launches = 0;
	for (uint64_t first = 0; first < total; first += c->wave_capacity) {
		if (staged) {
			RB_CUDA(gpu::launch_direct_staged_wave(c->view, c->wave, c->film, c->direct, dc, cfg, c->num_sms * 4, c->stream));
			launches += 7u + 5u * dc.bsdf_samples;
		} else {
			RB_CUDA(gpu::launch_direct_wave(c->view, c->wave, c->film, dc, cfg, c->num_sms * 4, c->stream));
			launches += 3u;
		}
		const rb_status st = readback_after(c, readback, std::min<uint64_t>(total, first + c->wave_capacity), c->stream);
		if (st != RB_OK) return st;
	}
	RB_CUDA(cudaEventRecord(c->ev_end, c->stream));
	RB_CUDA(cudaMemcpyAsync(c->counters_host, c->counters, gpu::CNT_WORDS * sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
	RB_CUDA(cudaStreamSynchronize(c->stream));
	const uint32_t* h = c->counters_host;
	auto u64 = [&](uint32_t w) { return static_cast<uint64_t>(h[w]) | (static_cast<uint64_t>(h[w + 1]) << 32); };
	rb_render_stats& s = c->stats;
	s = rb_render_stats{};
	s.extend_rays = u64(gpu::CNT_EXTEND_RAYS);
	s.node_visits = u64(gpu::CNT_NODE_VISITS);
	s.triangle_tests = u64(gpu::CNT_TRI_TESTS);
	s.device_error = h[gpu::CNT_ERROR];
	s.samples = total;
	s.kernel_launches = launches;
	cudaEventElapsedTime(&s.elapsed_ms, c->ev_begin, c->ev_end);
	traversal_times(c, 1u, s);
	return RB_OK;
}

// Replaces the context's scene (or batch) with the packed arrays of `p`.
rb_status upload_packed(rb_context* c, const host::packed_scene& p) {
	if (p.bvh_depth + 3 > 64) return RB_ERR_UNSUPPORTED;
	const rb_status pending = async_finish(c);
	if (pending != RB_OK) return pending;
	RB_CUDA(cudaSetDevice(c->device));
	RB_CUDA(cudaStreamSynchronize(c->stream));
	c->release_graph();
	c->scene.release();
	c->release_batch();
	c->has_scene = false;
	device_scene& d = c->scene;
	RB_CUDA(dev_upload(&d.nodes, p.nodes, c->stream));
	if (p.wide_ok) RB_CUDA(dev_upload(&d.wnodes, p.wnodes, c->stream));
	RB_CUDA(dev_upload(&d.tri_a, p.tri_a, c->stream));
	RB_CUDA(dev_upload(&d.tri_b, p.tri_b, c->stream));
	RB_CUDA(dev_upload(&d.tri_c, p.tri_c, c->stream));
	RB_CUDA(dev_upload(&d.prim_index, p.prim_index, c->stream));
	RB_CUDA(dev_upload(&d.prim_entity, p.prim_entity, c->stream));
	RB_CUDA(dev_upload(&d.entities, p.entities, c->stream));
	RB_CUDA(dev_upload(&d.meshes, p.meshes, c->stream));
	RB_CUDA(dev_upload(&d.positions, p.positions, c->stream));
	RB_CUDA(dev_upload(&d.normals, p.normals, c->stream));
	RB_CUDA(dev_upload(&d.tangents, p.tangents, c->stream));
	RB_CUDA(dev_upload(&d.uvs, p.uvs, c->stream));
	RB_CUDA(dev_upload(&d.indices, p.indices, c->stream));
	RB_CUDA(dev_upload(&d.materials, p.materials, c->stream));
	RB_CUDA(dev_upload(&d.emitters, p.emitters, c->stream));
	RB_CUDA(dev_upload(&d.environments, p.environments, c->stream));
	RB_CUDA(dev_upload(&d.mediums, p.mediums, c->stream));
	RB_CUDA(dev_upload(&d.media, p.media, c->stream));
	RB_CUDA(dev_upload(&d.material_srcs, p.material_srcs, c->stream));
	RB_CUDA(dev_upload(&d.textures, p.textures, c->stream));
	RB_CUDA(dev_upload(&d.texels, p.texels, c->stream));
	RB_CUDA(dev_upload(&d.sss_table, p.sss_table, c->stream));
	RB_CUDA(cudaStreamSynchronize(c->stream));
	pt::scene_view v{};
	v.wnodes = p.wide_ok ? d.wnodes : nullptr;
	v.root_a = p.root_a;
	v.root_b = p.root_b;
	v.root_ref = p.root_ref;
	v.nodes = d.nodes; v.tri_a = d.tri_a; v.tri_b = d.tri_b; v.tri_c = d.tri_c; v.prim_index = d.prim_index;
	v.entities = d.entities; v.meshes = d.meshes; v.positions = d.positions; v.normals = d.normals;
	v.tangents = d.tangents; v.uvs = d.uvs; v.indices = d.indices; v.materials = d.materials; v.emitters = d.emitters;
	v.environments = d.environments; v.env = p.env;
	v.num_nodes = static_cast<uint32_t>(p.nodes.size() / 2);
	v.num_emitters = static_cast<uint32_t>(p.emitters.size());
	v.num_environments = static_cast<uint32_t>(p.environments.size());
	v.num_entities = static_cast<uint32_t>(p.entities.size());
	v.mediums = d.mediums;
	v.media = d.media;
	v.num_media = static_cast<uint32_t>(p.media.size());
	v.instances = p.instances ? 1u : 0u;
	v.material_srcs = d.material_srcs;
	v.textures = d.textures;
	v.texels = d.texels;
	v.num_textures = static_cast<uint32_t>(p.textures.size());
	v.sss_table = p.sss_table.empty() ? nullptr : d.sss_table;
	v.sss = p.sss_table.empty() ? 0u : 1u;
	c->view = v;
	c->bvh_depth = p.bvh_depth;
	c->num_entities = v.num_entities;
	c->has_invisible = false;
	for (const auto& e : p.entities)
		if ((e.flags & pt::ENT_HAS_SHAPE) && !(e.flags & pt::ENT_HAS_MATERIAL)) c->has_invisible = true;
	c->has_scene = true;
	return RB_OK;
}

bool host_is_valid_camera(const rb_camera_desc& cam) {
	return cam.width > 0 && cam.height > 0 && cam.width <= 16384 && cam.height <= 16384 &&
		static_cast<uint64_t>(cam.width) * cam.height < (1ull << 24);
}

} // namespace ctx
} // namespace rb

namespace rb {
namespace gpu {
// Scene view, launch configuration of a plain surface render (no counting, no
// guide, no media: whatever the context's last rb_render used), stream, device,
// pinned counter buffer and whether the scene has invisible entities, for entry
// points defined in other files of the library.
bool context_view(rb_context* c, pt::scene_view* view, launch_cfg* cfg, cudaStream_t* stream, int* device,
	uint32_t** counters_host, bool* has_invisible) {
	if (c == nullptr || !c->has_scene || c->is_batch) return false;
	if (async_finish(c) != RB_OK) return false;
	*view = c->view;
	*cfg = c->cfg();
	cfg->count = false;
	cfg->guide = nullptr;
	cfg->guide_medium = nullptr;
	cfg->guide_mode = 0u;
	cfg->volume = false;
	*stream = c->stream;
	*device = c->device;
	*counters_host = c->counters_host;
	*has_invisible = c->has_invisible;
	return true;
}

// The guide of a context with its stream, device and SM count, for the
// rb_guide_* entry points (guide_api.cu).
guide::guide_state* context_guide(rb_context* c, cudaStream_t* stream, int* device, int* num_sms) {
	if (c == nullptr) return nullptr;
	async_finish(c);  // the guide entry points use the context's stream and buffers
	*stream = c->stream;
	*device = c->device;
	*num_sms = c->num_sms;
	return &c->guide;
}

// Drops the captured wave graph (its launches bake in guide buffer addresses).
void context_drop_graph(rb_context* c) { c->release_graph(); }

// The medium guide of guided volume renders.
guide::guide_state* context_guide_medium(rb_context* c) { return &c->guide_medium; }
} // namespace gpu
} // namespace rb

extern "C" {

int32_t rb_abi_version(void) { return RBGPU_ABI_VERSION; }

void rb_inject_allocation_failure(int32_t after) { allocation_countdown().store(after < 0 ? -1 : after); }

const char* rb_status_string(rb_status s) {
	switch (s) {
	case RB_OK: return "ok";
	case RB_ERR_INVALID_ARGUMENT: return "invalid argument";
	case RB_ERR_CUDA: return "CUDA runtime error";
	case RB_ERR_OUT_OF_MEMORY: return "out of device memory";
	case RB_ERR_NO_SCENE: return "no scene uploaded";
	case RB_ERR_STACK_OVERFLOW: return "traversal stack overflow";
	case RB_ERR_QUEUE_OVERFLOW: return "wavefront queue overflow";
	case RB_ERR_UNSUPPORTED: return "scene feature not supported";
	case RB_ERR_IO: return "checkpoint I/O error";
	case RB_ERR_CHECKPOINT: return "checkpoint does not match the context";
	case RB_ERR_DEVICE_TIMEOUT: return "device wait timed out";
	case RB_ERR_NO_DEVICE: return "no CUDA device";
	case RB_ERR_TOO_LARGE: return "work exceeds the fixed scratch capacity of rb_render_noalloc";
	default: return "unknown status";
	}
}

rb_status rb_context_create(rb_context** out, int device) {
	if (out == nullptr) return RB_ERR_INVALID_ARGUMENT;
	*out = nullptr;
	int count = 0;
	if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
		cudaGetLastError();
		return RB_ERR_NO_DEVICE;
	}
	if (device < 0 || device >= count) return RB_ERR_INVALID_ARGUMENT;
	rb_context* c = new (std::nothrow) rb_context();
	if (c == nullptr) return RB_ERR_OUT_OF_MEMORY;
	c->device = device;
	rb_status st = RB_OK;
	do {
		if (cudaSetDevice(device) != cudaSuccess) { st = RB_ERR_CUDA; break; }
		cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device);
		if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) { st = RB_ERR_CUDA; break; }
		if (cudaEventCreate(&c->ev_begin) != cudaSuccess || cudaEventCreate(&c->ev_end) != cudaSuccess) { st = RB_ERR_CUDA; break; }
		if (cudaMalloc(&c->counters, gpu::CNT_WORDS * sizeof(uint32_t)) != cudaSuccess) { st = RB_ERR_OUT_OF_MEMORY; break; }
		if (cudaMemset(c->counters, 0, gpu::CNT_WORDS * sizeof(uint32_t)) != cudaSuccess) { st = RB_ERR_CUDA; break; }
		if (cudaMallocHost(&c->counters_host, kMaxLanes * gpu::CNT_WORDS * sizeof(uint32_t)) != cudaSuccess) { st = RB_ERR_OUT_OF_MEMORY; break; }
		if (cudaMallocHost(&c->params_host, sizeof(gpu::wave_params)) != cudaSuccess) { st = RB_ERR_OUT_OF_MEMORY; break; }
		if (cudaMalloc(&c->wave.params, sizeof(gpu::wave_params)) != cudaSuccess) { st = RB_ERR_OUT_OF_MEMORY; break; }
	} while (false);
	if (st != RB_OK) {
		rb_context_destroy(c);
		return st;
	}
	*out = c;
	return RB_OK;
}

rb_status rb_context_destroy(rb_context* c) {
	if (c == nullptr) return RB_ERR_INVALID_ARGUMENT;
	cudaSetDevice(c->device);
	async_finish(c);
	if (c->stream) cudaStreamSynchronize(c->stream);
	c->release_graph();
	c->release_lanes();
	c->release_wave();
	c->release_film();
	c->scene.release();
	c->release_batch();
	for (cudaEvent_t e : c->wave_events) cudaEventDestroy(e);
	guide::release(c->guide);
	guide::release(c->guide_medium);
	dev_free(c->trace_rays);
	dev_free(c->trace_hits);
	dev_free(c->counters);
	dev_free(c->wave.params);
	if (c->counters_host) cudaFreeHost(c->counters_host);
	if (c->params_host) cudaFreeHost(c->params_host);
	for (cudaEvent_t e : c->events) cudaEventDestroy(e);
	if (c->ev_begin) cudaEventDestroy(c->ev_begin);
	if (c->ev_end) cudaEventDestroy(c->ev_end);
	if (c->stream) cudaStreamDestroy(c->stream);
	delete c;
	return RB_OK;
}

rb_status rb_scene_upload(rb_context* c, const rb_scene_desc* desc) {
	if (c == nullptr || desc == nullptr) return RB_ERR_INVALID_ARGUMENT;
	const rb_status pending = async_finish(c);
	if (pending != RB_OK) return pending;
	host::packed_scene p;
	const rb_status st = host::pack_scene(desc, p);
	if (st != RB_OK) return st;
	return upload_packed(c, p);
}

static rb_status trace_device(rb_context* c, const rb_ray* d_rays, uint32_t n, rb_hit* d_hits, bool shadow, cudaStream_t s) {
	gpu::launch_cfg cfg = c->cfg();
	RB_CUDA(gpu::launch_trace_rays(c->view, c->scene.prim_entity, d_rays, n, d_hits, shadow, cfg, c->counters, s));
	return RB_OK;
}

static rb_status trace_host(rb_context* c, const rb_ray* rays, uint32_t n, rb_hit* hits, bool shadow) {
	if (c == nullptr || (n > 0 && (rays == nullptr || hits == nullptr))) return RB_ERR_INVALID_ARGUMENT;
	if (!c->has_scene) return RB_ERR_NO_SCENE;
	if (c->is_batch) return RB_ERR_INVALID_ARGUMENT;
	if (n == 0) return RB_OK;
	RB_CUDA(cudaSetDevice(c->device));
	if (c->trace_cap < n) {
		dev_free(c->trace_rays);
		dev_free(c->trace_hits);
		c->trace_cap = 0;
		RB_CUDA(dev_alloc(&c->trace_rays, n));
		RB_CUDA(dev_alloc(&c->trace_hits, n));
		c->trace_cap = n;
	}
	RB_CUDA(cudaMemsetAsync(c->counters + gpu::CNT_ERROR, 0, sizeof(uint32_t), c->stream));
	RB_CUDA(cudaMemcpyAsync(c->trace_rays, rays, n * sizeof(rb_ray), cudaMemcpyHostToDevice, c->stream));
	const rb_status st = trace_device(c, c->trace_rays, n, c->trace_hits, shadow, c->stream);
	if (st != RB_OK) return st;
	RB_CUDA(cudaMemcpyAsync(hits, c->trace_hits, n * sizeof(rb_hit), cudaMemcpyDeviceToHost, c->stream));
	RB_CUDA(cudaMemcpyAsync(c->counters_host, c->counters, gpu::CNT_WORDS * sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
	RB_CUDA(cudaStreamSynchronize(c->stream));
	if (c->counters_host[gpu::CNT_ERROR] != 0) return static_cast<rb_status>(c->counters_host[gpu::CNT_ERROR]);
	return RB_OK;
}

rb_status rb_trace_closest(rb_context* c, const rb_ray* rays, uint32_t n, rb_hit* hits) { return trace_host(c, rays, n, hits, false); }
rb_status rb_trace_shadow(rb_context* c, const rb_ray* rays, uint32_t n, rb_hit* hits) { return trace_host(c, rays, n, hits, true); }

rb_status rb_trace_closest_device(rb_context* c, const rb_ray* d_rays, uint32_t n, rb_hit* d_hits, void* stream) {
	if (c == nullptr || (n > 0 && (d_rays == nullptr || d_hits == nullptr))) return RB_ERR_INVALID_ARGUMENT;
	if (!c->has_scene) return RB_ERR_NO_SCENE;
	if (c->is_batch) return RB_ERR_INVALID_ARGUMENT;
	RB_CUDA(cudaSetDevice(c->device));
	return trace_device(c, d_rays, n, d_hits, false, stream ? static_cast<cudaStream_t>(stream) : c->stream);
}
rb_status rb_trace_shadow_device(rb_context* c, const rb_ray* d_rays, uint32_t n, rb_hit* d_hits, void* stream) {
	if (c == nullptr || (n > 0 && (d_rays == nullptr || d_hits == nullptr))) return RB_ERR_INVALID_ARGUMENT;
	if (!c->has_scene) return RB_ERR_NO_SCENE;
	if (c->is_batch) return RB_ERR_INVALID_ARGUMENT;
	RB_CUDA(cudaSetDevice(c->device));
	return trace_device(c, d_rays, n, d_hits, true, stream ? static_cast<cudaStream_t>(stream) : c->stream);
}

rb_status rb_set_counting(rb_context* c, int enabled) {
	if (c == nullptr) return RB_ERR_INVALID_ARGUMENT;
	const rb_status pending = async_finish(c);
	if (pending != RB_OK) return pending;
	if (c->counting != (enabled != 0)) c->release_graph();
	c->counting = enabled != 0;
	return RB_OK;
}

rb_status rb_set_profiling(rb_context* c, int enabled) {
	if (c == nullptr) return RB_ERR_INVALID_ARGUMENT;
	const rb_status pending = async_finish(c);
	if (pending != RB_OK) return pending;
	c->profiling = enabled != 0;
	if (c->profiling && c->events.empty()) {
		RB_CUDA(cudaSetDevice(c->device));
		c->events.resize(2 * rb_context::kMaxEvents);
		c->event_kind.resize(rb_context::kMaxEvents);
		for (auto& e : c->events) RB_CUDA(cudaEventCreate(&e));
	}
	return RB_OK;
}

static rb_status render_call(rb_context* c, const rb_render_params* prm, float* rgb_out, bool async);

rb_status rb_render(rb_context* c, const rb_render_params* prm, float* rgb_out) {
	if (c == nullptr || prm == nullptr) return RB_ERR_INVALID_ARGUMENT;
	const rb_status pending = async_finish(c);
	if (pending != RB_OK) return pending;
	return render_call(c, prm, rgb_out, false);
}

rb_status rb_render_async(rb_context* c, const rb_render_params* prm, float* rgb_out) {
	if (c == nullptr || prm == nullptr) return RB_ERR_INVALID_ARGUMENT;
	if (prm->flags & ~static_cast<uint32_t>(RB_RENDER_RESET)) return RB_ERR_UNSUPPORTED;  // plain path tracing only
	if (rgb_out != nullptr && !is_page_locked(rgb_out)) return RB_ERR_INVALID_ARGUMENT;
	// what later calls must share with the pending ones to continue them
	struct signature {
		rb_camera_desc camera;
		uint32_t spp, max_depth, paths_per_wave;
		float rr_threshold;
		rb_tuning tuning;
		uint32_t counting, profiling;
	} sig;
	std::memset(&sig, 0, sizeof(sig));
	sig.camera = prm->camera;
	sig.spp = prm->spp;
	sig.max_depth = prm->max_depth;
	sig.paths_per_wave = prm->paths_per_wave;
	sig.rr_threshold = prm->rr_threshold;
	sig.tuning = c->tuning;
	sig.counting = c->counting;
	sig.profiling = c->profiling;
	static_assert(sizeof(signature) <= sizeof(c->async.signature), "async signature too large");
	const bool same = c->async.signature_size == sizeof(sig) && std::memcmp(c->async.signature, &sig, sizeof(sig)) == 0;
	if (c->async.pending > 0 && (!same || (prm->flags & RB_RENDER_RESET) || c->profiling)) {
		const rb_status st = async_finish(c);
		if (st != RB_OK) return st;
	}
	std::memcpy(c->async.signature, &sig, sizeof(sig));
	c->async.signature_size = sizeof(sig);
	const rb_status st = render_call(c, prm, rgb_out, !c->profiling);
	if (st != RB_OK) c->async = rb_context::async_state{};  // (the failed call was synchronised or never enqueued)
	return st;
}

rb_status rb_render_wait(rb_context* c) {
	if (c == nullptr) return RB_ERR_INVALID_ARGUMENT;
	RB_CUDA(cudaSetDevice(c->device));
	return async_finish(c);
}

static rb_status render_call(rb_context* c, const rb_render_params* prm, float* rgb_out, bool async) {
	if (!c->has_scene) return RB_ERR_NO_SCENE;
	if (c->is_batch) return RB_ERR_INVALID_ARGUMENT;
	const rb_camera_desc& cam = prm->camera;
	if (!host_is_valid_camera(cam) || prm->max_depth == 0 || prm->max_depth > 64) return RB_ERR_INVALID_ARGUMENT;
	if (static_cast<uint64_t>(prm->first_sample) + prm->spp > (1u << 24)) return RB_ERR_INVALID_ARGUMENT;
	const bool direct = (prm->flags & RB_RENDER_DIRECT) != 0;
	uint32_t direct_emitter = 4u, direct_bsdf = 4u;  // direct_integrator's defaults (direct_integrator.hpp:9-13)
	if (direct) {
		if (prm->flags & (RB_RENDER_GUIDE | RB_RENDER_TRAIN | RB_RENDER_VOLUME)) return RB_ERR_INVALID_ARGUMENT;
		if (prm->direct_samples != 0) {
			direct_emitter = prm->direct_samples & 0xffffu;
			direct_bsdf = prm->direct_samples >> 16;
			if (direct_emitter == 0 || direct_bsdf == 0) return RB_ERR_INVALID_ARGUMENT;
		}
	}
	// the BSSRDF stage runs in the plain path tracer only
	if (c->view.sss && (prm->flags & (RB_RENDER_GUIDE | RB_RENDER_TRAIN | RB_RENDER_VOLUME))) return RB_ERR_UNSUPPORTED;
	RB_CUDA(cudaSetDevice(c->device));
	rb_status st = ensure_film(c, cam.width, cam.height, (prm->flags & RB_RENDER_RESET) != 0);
	if (st != RB_OK) return st;
	const uint64_t pixels = static_cast<uint64_t>(cam.width) * cam.height;
	const uint64_t total = pixels * prm->spp;
	uint64_t capacity = prm->paths_per_wave ? prm->paths_per_wave : c->tuning.paths_per_wave ? c->tuning.paths_per_wave : (1ull << 21);
	if (capacity > total) capacity = total;
	if (capacity > (1ull << 24)) return RB_ERR_INVALID_ARGUMENT;
	if (capacity == 0) capacity = 1;
	st = ensure_wave(c, static_cast<uint32_t>(capacity));
	if (st != RB_OK) return st;
	st = prepare_guide(c, prm);
	if (st != RB_OK) return st;
	st = prepare_volume(c, prm);
	if (st != RB_OK) return st;

	gpu::wave_params& hp = *c->params_host;
	std::memcpy(hp.r2c, cam.raster_to_camera, sizeof(hp.r2c));
	std::memcpy(hp.c2w, cam.camera_to_world, sizeof(hp.c2w));
	hp.lens = cam.lens_radius;
	hp.focus = cam.focus_distance;
	hp.width = static_cast<uint32_t>(cam.width);
	hp.height = static_cast<uint32_t>(cam.height);
	hp.total_items = total;
	hp.first_sample = prm->first_sample;
	hp.seed = prm->seed;
	hp.max_depth = prm->max_depth;
	hp.rr_threshold = prm->rr_threshold;
	hp.guide_flags = c->guide_mode;
	{
		// scene box of the guide inputs: the root box of the BVH
		const float lo[3] = {c->view.root_a.x, c->view.root_a.y, c->view.root_a.z};
		const float hi[3] = {c->view.root_a.w, c->view.root_b.x, c->view.root_b.y};
		for (int k = 0; k < 3; k++) {
			const float ext = hi[k] - lo[k];
			hp.box_min[k] = lo[k];
			hp.box_inv[k] = ext > 0.f ? 1.f / ext : 0.f;
		}
	}

	// a page-locked output buffer receives each slice of the image as soon as
	// its pixels are final, overlapped with the waves still running
	image_readback overlap;
	const bool overlapped = rgb_out != nullptr && is_page_locked(rgb_out);
	if (overlapped) {
		overlap.host = rgb_out;
		overlap.pixels = pixels;
		overlap.final_from = total - pixels;
	}
	st = direct ? run_direct(c, total, pt::make_direct_cfg(direct_emitter, direct_bsdf), overlapped ? &overlap : nullptr)
		: run_waves(c, total, prm->max_depth, false, overlapped ? &overlap : nullptr, async);
	if (st != RB_OK) return st;
	c->film_samples += prm->spp;
	if (async) return RB_OK;  // the page-locked image arrives slice by slice; rb_render_wait ends the calls
	const uint32_t* h = c->counters_host;
	if (h[gpu::CNT_ERROR] != 0) return static_cast<rb_status>(h[gpu::CNT_ERROR]);

	if (rgb_out != nullptr && !(overlapped && overlap.done == pixels)) {
		// means on the device, then one copy of 3 floats per pixel (at full speed
		// when the caller's buffer is page-locked)
		const size_t first = overlapped ? static_cast<size_t>(overlap.done) : 0u, n = static_cast<size_t>(pixels) - first;
		const gpu::film_buffers f{c->film.sum + 3 * first, c->film.sum_sq + 3 * first, c->film.count + first};
		RB_CUDA(gpu::launch_film_mean(f, static_cast<uint32_t>(n), c->film_mean + 3 * first, c->num_sms * 4, c->stream));
		RB_CUDA(cudaMemcpyAsync(rgb_out + 3 * first, c->film_mean + 3 * first, 3 * n * sizeof(float), cudaMemcpyDeviceToHost,
			c->stream));
		RB_CUDA(cudaStreamSynchronize(c->stream));
	}
	return RB_OK;
}

rb_status rb_film_read(rb_context* c, double* sum_rgb, double* sum_sq_rgb, uint32_t* count) {
	if (c == nullptr) return RB_ERR_INVALID_ARGUMENT;
	const rb_status pending = async_finish(c);
	if (pending != RB_OK) return pending;
	if (c->film_w == 0) return RB_ERR_NO_SCENE;
	RB_CUDA(cudaSetDevice(c->device));
	RB_CUDA(cudaStreamSynchronize(c->stream));
	const size_t px = static_cast<size_t>(c->film_w) * c->film_h;
	if (sum_rgb) RB_CUDA(cudaMemcpy(sum_rgb, c->film.sum, 3 * px * sizeof(double), cudaMemcpyDeviceToHost));
	if (sum_sq_rgb) RB_CUDA(cudaMemcpy(sum_sq_rgb, c->film.sum_sq, 3 * px * sizeof(double), cudaMemcpyDeviceToHost));
	if (count) RB_CUDA(cudaMemcpy(count, c->film.count, px * sizeof(uint32_t), cudaMemcpyDeviceToHost));
	return RB_OK;
}

rb_status rb_film_to_device(rb_context* c, double* d_sum, double* d_sum_sq, uint32_t* d_count, void* stream) {
	if (c == nullptr || d_sum == nullptr || d_sum_sq == nullptr || d_count == nullptr) return RB_ERR_INVALID_ARGUMENT;
	const rb_status pending = async_finish(c);
	if (pending != RB_OK) return pending;
	if (c->film_w == 0) return RB_ERR_NO_SCENE;
	RB_CUDA(cudaSetDevice(c->device));
	const cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : c->stream;
	if (s != c->stream) RB_CUDA(cudaStreamSynchronize(c->stream));  // the film's last writes are on the context's stream
	const size_t px = static_cast<size_t>(c->film_w) * c->film_h;
	RB_CUDA(cudaMemcpyAsync(d_sum, c->film.sum, 3 * px * sizeof(double), cudaMemcpyDeviceToDevice, s));
	RB_CUDA(cudaMemcpyAsync(d_sum_sq, c->film.sum_sq, 3 * px * sizeof(double), cudaMemcpyDeviceToDevice, s));
	RB_CUDA(cudaMemcpyAsync(d_count, c->film.count, px * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
	return RB_OK;
}

rb_status rb_film_from_device(rb_context* c, const double* d_sum, const double* d_sum_sq, const uint32_t* d_count,
	uint64_t samples_per_pixel, void* stream) {
	if (c == nullptr || d_sum == nullptr || d_sum_sq == nullptr || d_count == nullptr) return RB_ERR_INVALID_ARGUMENT;
	const rb_status pending = async_finish(c);
	if (pending != RB_OK) return pending;
	if (c->film_w == 0) return RB_ERR_NO_SCENE;
	RB_CUDA(cudaSetDevice(c->device));
	const cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : c->stream;
	const size_t px = static_cast<size_t>(c->film_w) * c->film_h;
	RB_CUDA(cudaMemcpyAsync(c->film.sum, d_sum, 3 * px * sizeof(double), cudaMemcpyDeviceToDevice, s));
	RB_CUDA(cudaMemcpyAsync(c->film.sum_sq, d_sum_sq, 3 * px * sizeof(double), cudaMemcpyDeviceToDevice, s));
	RB_CUDA(cudaMemcpyAsync(c->film.count, d_count, px * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
	RB_CUDA(cudaStreamSynchronize(s));  // later calls run on the context's stream
	c->film_samples = samples_per_pixel;
	return RB_OK;
}

rb_status rb_render_stats_get(rb_context* c, rb_render_stats* out) {
	if (c == nullptr || out == nullptr) return RB_ERR_INVALID_ARGUMENT;
	const rb_status pending = async_finish(c);
	if (pending != RB_OK) return pending;
	*out = c->stats;
	return RB_OK;
}

// Checkpoint layout: magic, version, width, height, samples per pixel so far,
// then the FP64 sums, FP64 squared sums and uint32 counts.
rb_status rb_checkpoint_save(rb_context* c, const char* path) {
	if (c == nullptr || path == nullptr) return RB_ERR_INVALID_ARGUMENT;
	if (c->film_w == 0) return RB_ERR_NO_SCENE;
	const size_t px = static_cast<size_t>(c->film_w) * c->film_h;
	std::vector<double> sum(3 * px), sq(3 * px);
	std::vector<uint32_t> cnt(px);
	const rb_status st = rb_film_read(c, sum.data(), sq.data(), cnt.data());
	if (st != RB_OK) return st;
	FILE* f = std::fopen(path, "wb");
	if (f == nullptr) return RB_ERR_IO;
	const uint32_t head[4] = {kCheckpointMagic, 1u, static_cast<uint32_t>(c->film_w), static_cast<uint32_t>(c->film_h)};
	const uint64_t spp = c->film_samples;
	bool ok = std::fwrite(head, sizeof(head), 1, f) == 1 && std::fwrite(&spp, sizeof(spp), 1, f) == 1 &&
		std::fwrite(sum.data(), sizeof(double), sum.size(), f) == sum.size() &&
		std::fwrite(sq.data(), sizeof(double), sq.size(), f) == sq.size() &&
		std::fwrite(cnt.data(), sizeof(uint32_t), cnt.size(), f) == cnt.size();
	ok = (std::fclose(f) == 0) && ok;
	return ok ? RB_OK : RB_ERR_IO;
}

rb_status rb_checkpoint_load(rb_context* c, const char* path) {
	if (c == nullptr || path == nullptr) return RB_ERR_INVALID_ARGUMENT;
	const rb_status pending = async_finish(c);
	if (pending != RB_OK) return pending;
	FILE* f = std::fopen(path, "rb");
	if (f == nullptr) return RB_ERR_IO;
	uint32_t head[4];
	uint64_t spp = 0;
	if (std::fread(head, sizeof(head), 1, f) != 1 || std::fread(&spp, sizeof(spp), 1, f) != 1 || head[0] != kCheckpointMagic ||
		head[1] != 1u || head[2] == 0 || head[3] == 0 || static_cast<uint64_t>(head[2]) * head[3] >= (1ull << 24)) {
		std::fclose(f);
		return RB_ERR_CHECKPOINT;
	}
	const size_t px = static_cast<size_t>(head[2]) * head[3];
	std::vector<double> sum(3 * px), sq(3 * px);
	std::vector<uint32_t> cnt(px);
	const bool ok = std::fread(sum.data(), sizeof(double), sum.size(), f) == sum.size() &&
		std::fread(sq.data(), sizeof(double), sq.size(), f) == sq.size() &&
		std::fread(cnt.data(), sizeof(uint32_t), cnt.size(), f) == cnt.size();
	std::fclose(f);
	if (!ok) return RB_ERR_CHECKPOINT;
	RB_CUDA(cudaSetDevice(c->device));
	const rb_status st = ensure_film(c, static_cast<int32_t>(head[2]), static_cast<int32_t>(head[3]), true);
	if (st != RB_OK) return st;
	RB_CUDA(cudaMemcpyAsync(c->film.sum, sum.data(), sum.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
	RB_CUDA(cudaMemcpyAsync(c->film.sum_sq, sq.data(), sq.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
	RB_CUDA(cudaMemcpyAsync(c->film.count, cnt.data(), cnt.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, c->stream));
	RB_CUDA(cudaStreamSynchronize(c->stream));
	c->film_samples = spp;
	return RB_OK;
}

} // extern "C"
