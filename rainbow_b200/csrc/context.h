// Internal: the rb_context of the C ABI and the helpers its entry points
// share (api.cu, batch.cu). Not part of the public interface.
#pragma once

#include "../../include/rbgpu.h"
#include "host/scene_pack.h"
#include "kernels.cuh"

#include <atomic>
#include <cstring>
#include <utility>
#include <vector>

namespace rb {
namespace ctx {


// Host-side allocation-failure injection (rb_inject_allocation_failure): the
// countdown of device allocations until one fails, < 0 when off.
std::atomic<int32_t>& allocation_countdown();

template <typename T>
inline cudaError_t dev_alloc(T** p, size_t count) {
	*p = nullptr;
	if (count == 0) return cudaSuccess;
	std::atomic<int32_t>& fail = allocation_countdown();
	if (fail.load() >= 0 && fail.fetch_sub(1) == 0) return cudaErrorMemoryAllocation;
	return cudaMalloc(reinterpret_cast<void**>(p), count * sizeof(T));
}
template <typename T>
inline cudaError_t dev_upload(T** p, const std::vector<T>& v, cudaStream_t s) {
	cudaError_t e = dev_alloc(p, v.size());
	if (e != cudaSuccess || v.empty()) return e;
	return cudaMemcpyAsync(*p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s);
}
template <typename T>
inline void dev_free(T*& p) {
	if (p) cudaFree(p);
	p = nullptr;
}

inline rb_status from_cuda(cudaError_t e) {
	if (e == cudaSuccess) return RB_OK;
	if (e == cudaErrorMemoryAllocation) return RB_ERR_OUT_OF_MEMORY;
	if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return RB_ERR_NO_DEVICE;
	return RB_ERR_CUDA;
}

#define RB_CUDA(call)                                   \
	do {                                                \
		const cudaError_t rb_e_ = (call);               \
		if (rb_e_ != cudaSuccess) return from_cuda(rb_e_); \
	} while (0)

struct device_scene {
	pt::node4* wnodes = nullptr;
	float4* nodes = nullptr;
	float4* tri_a = nullptr;
	float4* tri_b = nullptr;
	float2* tri_c = nullptr;
	uint32_t* prim_index = nullptr;
	uint32_t* prim_entity = nullptr;
	pt::entity_rec* entities = nullptr;
	pt::mesh_rec* meshes = nullptr;
	float* positions = nullptr;
	float* normals = nullptr;
	float* tangents = nullptr;
	float* uvs = nullptr;
	uint32_t* indices = nullptr;
	pt::material_rec* materials = nullptr;
	pt::emitter_rec* emitters = nullptr;
	int32_t* environments = nullptr;
	pt::medium_rec* mediums = nullptr;
	pt::media_rec* media = nullptr;
	pt::material_src* material_srcs = nullptr;
	pt::texture_rec* textures = nullptr;
	float* texels = nullptr;
	float* sss_table = nullptr;
	void release() {
		dev_free(wnodes); dev_free(nodes); dev_free(tri_a); dev_free(tri_b); dev_free(tri_c); dev_free(prim_index); dev_free(prim_entity);
		dev_free(entities); dev_free(meshes); dev_free(positions); dev_free(normals); dev_free(tangents); dev_free(uvs);
		dev_free(indices); dev_free(materials); dev_free(emitters); dev_free(environments);
		dev_free(mediums); dev_free(media); dev_free(material_srcs); dev_free(textures); dev_free(texels); dev_free(sss_table);
	}
};

struct graph_key {
	uint32_t capacity = 0, max_depth = 0, stack = 0;
	bool count = false;
	uint32_t guide_mode = 0, guide_steps = 0, guide_batch = 0;
	bool volume = false;
	bool batch = false;
	bool with_end = true;  // the graph ends with the film resolve (one lane) or stops after the bounces
	uint32_t block_trace = 0, block_shade = 0, grid_trace = 0, grid_shade = 0, sort = 0, tail = 0;
	bool refill = false;
	bool shadow_first = false;
	bool sss = false;
	int carveout = 0;
	bool operator==(const graph_key& o) const {
		return capacity == o.capacity && max_depth == o.max_depth && stack == o.stack && count == o.count &&
			guide_mode == o.guide_mode && guide_steps == o.guide_steps && guide_batch == o.guide_batch &&
			volume == o.volume && batch == o.batch && block_trace == o.block_trace && block_shade == o.block_shade &&
			grid_trace == o.grid_trace && grid_shade == o.grid_shade && sort == o.sort && tail == o.tail &&
			with_end == o.with_end && refill == o.refill && carveout == o.carveout && shadow_first == o.shadow_first &&
			sss == o.sss;
	}
};

constexpr uint32_t kMaxLanes = 8;  // wave lanes of a context

// Launch shapes of a tuning with the defaults filled in.
inline rb_tuning resolved_tuning(const rb_tuning& t) {
	rb_tuning r = t;
	if (r.block_trace == 0) r.block_trace = 128;
	if (r.block_shade == 0) r.block_shade = 128;
	if (r.grid_per_sm == 0) r.grid_per_sm = 8;
	if (r.tail_bounce == 0) r.tail_bounce = 64;
	if (r.lanes == 0) r.lanes = 1;
	return r;
}
inline bool valid_tuning(const rb_tuning& t) {
	auto block_ok = [](uint32_t b) { return b == 0 || (b >= 32 && b <= 256 && b % 32 == 0); };
	return block_ok(t.block_trace) && block_ok(t.block_shade) && t.grid_per_sm <= 64 && t.sort <= RB_SORT_RAYS &&
		t.paths_per_wave <= (1u << 24) && t.tail_bounce <= 64 && t.lanes <= kMaxLanes && t.traversal <= RB_TRAVERSAL_REFILL &&
		t.smem_carveout <= 101 && t.shadow_test <= RB_SHADOW_FIRST_OCCLUDER;
}

// Path state of one wave: the buffers of wave_buffers for `n` paths.
cudaError_t alloc_wave_buffers(gpu::wave_buffers& w, size_t n);
void free_wave_buffers(gpu::wave_buffers& w);

// A further wave lane of a context: its own path buffers, counters, parameter
// block, stream and wave graph, so that the waves of one render call overlap.
struct wave_lane {
	gpu::wave_buffers wave{};
	uint32_t alloc = 0;              // paths its buffers hold
	uint32_t* counters = nullptr;    // device
	gpu::wave_params* params = nullptr;  // device
	uint32_t* path_scene = nullptr;  // batch renders: scene of each path
	uint32_t vol_alloc = 0;          // volume renders: paths the lane's medium / beam buffers hold
	int32_t* vol_medium = nullptr;
	pt::vol_rec* vol_rec = nullptr;
	float4* vol_beam = nullptr;
	uint32_t* vol_beam_queue = nullptr;
	cudaStream_t stream = nullptr;
	cudaGraphExec_t graph = nullptr;
	graph_key key;
	cudaEvent_t done = nullptr;
	void release_graph() {
		if (graph) cudaGraphExecDestroy(graph);
		graph = nullptr;
		key = graph_key();
	}
	void release() {
		release_graph();
		free_wave_buffers(wave);
		dev_free(counters);
		dev_free(params);
		dev_free(path_scene);
		dev_free(vol_medium); dev_free(vol_rec); dev_free(vol_beam); dev_free(vol_beam_queue);
		vol_alloc = 0;
		if (done) cudaEventDestroy(done);
		if (stream) cudaStreamDestroy(stream);
		done = nullptr;
		stream = nullptr;
		alloc = 0;
	}
};


} // namespace ctx
} // namespace rb

using namespace rb;
using namespace rb::ctx;

struct rb_context {
	int device = 0;
	int num_sms = 148;
	cudaStream_t stream = nullptr;
	cudaEvent_t ev_begin = nullptr, ev_end = nullptr;

	bool has_scene = false;
	bool has_invisible = false;
	bool drain_graph_failed = false;  // the runtime refused the drain loop's conditional node: host-driven drain
	uint32_t bvh_depth = 0;
	uint32_t num_entities = 0;
	device_scene scene;
	pt::scene_view view{};

	gpu::wave_buffers wave{};
	uint32_t wave_capacity = 0;  // paths per wave of the current render call (<= wave_alloc)
	uint32_t wave_alloc = 0;     // paths the wave buffers hold
	gpu::wave_params* params_host = nullptr;  // pinned
	gpu::film_buffers film{};
	float* film_mean = nullptr;  // per-pixel means of the film, 3 floats per pixel (rb_render's output)
	int32_t film_w = 0, film_h = 0;
	uint64_t film_samples = 0;  // samples per pixel accumulated since the last reset

	cudaGraphExec_t graph = nullptr;
	graph_key graph_cfg;

	rb_ray* trace_rays = nullptr;
	rb_hit* trace_hits = nullptr;
	size_t trace_cap = 0;

	uint32_t* counters = nullptr;
	uint32_t* counters_host = nullptr;  // pinned, kMaxLanes * CNT_WORDS (lane k's at k * CNT_WORDS)
	bool counting = false;
	bool profiling = false;
	static constexpr uint32_t kMaxEvents = 4096;  // event pairs per render call when profiling
	std::vector<cudaEvent_t> events;
	std::vector<uint8_t> event_kind;
	uint32_t next_event = 0;
	rb_render_stats stats{};
	guide::guide_state guide;        // learned path guide (allocated on first use)
	guide::guide_state guide_medium; // guide of medium vertices in guided volume renders
	guide::lane_guide lane_guides[kMaxLanes];  // per-lane guide buffers and weight snapshots (guided renders on lanes)
	guide::lane_guide lane_guides_medium[kMaxLanes];  // the same for the medium guide (guided volume renders)
	uint32_t guide_mode = 0;         // gpu::GUIDE_* of the current render call
	rb_tuning tuning{};              // launch shapes of render calls (zeros: defaults)
	// batched rendering: the uploaded scenes (geometry part of their records;
	// the view part is filled per render call), the device copy of the
	// records, the per-path scene buffer, and one event per wave for latencies
	bool is_batch = false;
	std::vector<gpu::batch_scene> batch_scenes;
	gpu::batch_scene* batch_dev = nullptr;
	uint32_t* batch_path_scene = nullptr;
	uint32_t batch_path_alloc = 0;
	std::vector<std::pair<uint32_t, uint32_t>> batch_range;  // film (first pixel, pixels) of each scene, upload order
	std::vector<cudaEvent_t> wave_events;  // recorded after each wave's film resolve
	std::vector<wave_lane> lanes;    // wave lanes beyond the context's own (lane 0: wave, stream, graph above)
	bool volume = false;             // the current render call uses the volume path integrator
	gpu::direct_buffers direct{};    // staged direct lighting (RB_RENDER_DIRECT), allocated on first use
	uint32_t direct_alloc = 0;       // paths the direct buffers hold
	int32_t* vol_medium = nullptr;   // per-path medium buffer (wave.medium points here in volume renders)
	uint32_t vol_alloc = 0;          // paths the volume buffers hold
	// rb_render_async calls enqueued since the last wait: their count, the
	// configuration they share, the waves and lanes of each (the first wave of
	// the next call waits for the last of the previous one), and the samples and
	// launches to report at rb_render_wait
	struct async_state {
		uint32_t pending = 0;
		uint64_t waves = 0;
		uint32_t lanes = 0;
		uint32_t next_lane = 0;  // lane of the next continuing call's first wave
		uint64_t samples = 0;
		uint32_t launches = 0;
		unsigned char signature[512];
		size_t signature_size = 0;
		bool use_graph = true;
	} async;

	gpu::launch_cfg cfg() const {
		gpu::launch_cfg c;
		const rb_tuning t = resolved_tuning(tuning);
		c.block_trace = static_cast<int>(t.block_trace);
		c.block_shade = static_cast<int>(t.block_shade);
		c.grid_trace = num_sms * static_cast<int>(t.grid_per_sm);
		c.grid_shade = num_sms * static_cast<int>(t.grid_per_sm);
		c.sort = t.sort;
		c.tail = t.tail_bounce;
		c.refill = t.traversal == RB_TRAVERSAL_REFILL;
		c.shadow_first = t.shadow_test == RB_SHADOW_FIRST_OCCLUDER;
		c.carveout = t.smem_carveout == 0 ? 100 : static_cast<int>(t.smem_carveout) - 1;
		c.batch = is_batch;
		// the reference-order traversal holds at most depth + 2 entries; the
		// 4-wide one falls back to it when its stack is full
		c.stack_depth = static_cast<int>((bvh_depth + 3 + 3) / 4 * 4);
		if (c.stack_depth < 16) c.stack_depth = 16;
		c.count = counting;
		if (guide_mode != 0u && guide.ready) {
			c.guide = &guide;
			c.guide_mode = guide_mode;
			if (volume && guide_medium.ready) c.guide_medium = &guide_medium;
		}
		c.volume = volume;
		c.sss = view.sss != 0u;
		return c;
	}
	gpu::launch_cfg profiled_cfg() {
		gpu::launch_cfg c = cfg();
		if (profiling) c.tail = 0xffffffffu;  // every bounce as separate stages, each traversal launch timed
		if (profiling && !events.empty()) {
			c.events = events.data();
			c.next_event = &next_event;
			c.max_events = static_cast<uint32_t>(events.size() / 2);
			c.event_kind = event_kind.data();
		}
		return c;
	}

	void release_wave() {
		free_wave_buffers(wave);
		dev_free(vol_medium); dev_free(wave.vrec); dev_free(wave.beam); dev_free(wave.beam_queue);
		wave.medium = nullptr;
		vol_alloc = 0;
		dev_free(direct.rec); dev_free(direct.ray_o); dev_free(direct.ray_d); dev_free(direct.ray_hit);
		dev_free(direct.ray_queue); dev_free(direct.shade_queue);
		direct_alloc = 0;
		dev_free(batch_path_scene);
		wave.scene = nullptr;
		batch_path_alloc = 0;
		wave_capacity = 0;
		wave_alloc = 0;
	}
	void release_batch() {
		dev_free(batch_dev);
		wave.batch = nullptr;
		wave.num_scenes = 0;
		batch_scenes.clear();
		is_batch = false;
	}
	void release_graph() {
		if (graph) cudaGraphExecDestroy(graph);
		graph = nullptr;
		graph_cfg = graph_key();
		for (wave_lane& l : lanes) l.release_graph();
	}
	void release_lanes() {
		for (wave_lane& l : lanes) l.release();
		lanes.clear();
		for (guide::lane_guide& g : lane_guides) guide::release_lane(g);
		for (guide::lane_guide& g : lane_guides_medium) guide::release_lane(g);
	}
	void release_film() {
		dev_free(film.sum); dev_free(film.sum_sq); dev_free(film.count); dev_free(film_mean);
		film_w = film_h = 0;
		film_samples = 0;
	}
};

namespace rb {
namespace ctx {

// Wave buffers for `capacity` paths (kept when large enough).
rb_status ensure_wave(rb_context* c, uint32_t capacity);
// Film accumulators of width x height pixels, cleared when reset or resized.
rb_status ensure_film(rb_context* c, int32_t width, int32_t height, bool reset);
// The wave graph of the current configuration (recorded when it changed).
rb_status capture_wave(rb_context* c, uint32_t max_depth);
// Extra lanes 1..count-1, each with buffers for c->wave_capacity paths.
rb_status ensure_lanes(rb_context* c, uint32_t count);
rb_status prepare_guide(rb_context* c, const rb_render_params* prm);
rb_status prepare_volume(rb_context* c, const rb_render_params* prm);
bool host_is_valid_camera(const rb_camera_desc& cam);
// Copy-out of rb_render's image while the call's later waves still run: film
// resolves add the waves in order and items are sample-major, so once the wave
// holding item final_from + p has resolved, pixel p has all of the call's
// samples; its mean then goes to the caller's page-locked buffer on that wave's
// stream.
struct image_readback {
	float* host = nullptr;     // page-locked, 3 floats per pixel
	uint64_t pixels = 0;
	uint64_t final_from = 0;   // first item of the call's last sample
	uint64_t done = 0;         // pixels already copied (or enqueued)
};
// async: an rb_render_async call, which returns once its work is enqueued and
// continues the film order of the pending async calls (statistics are taken at
// rb_render_wait by async_finish).
rb_status run_waves(rb_context* c, uint64_t total, uint32_t max_depth, bool record_waves,
	image_readback* readback = nullptr, bool async = false);
// Waits for the pending rb_render_async calls and takes their statistics.
rb_status async_finish(rb_context* c);
// Replaces the context's scene arrays with a packed scene (single or merged).
rb_status upload_packed(rb_context* c, const host::packed_scene& p);

} // namespace ctx
} // namespace rb
