// Kernel launchers of the wavefront path tracer (kernels.cu).
#pragma once

#include "../../include/rbgpu.h"
#include "guide/guide_host.h"
#include "pt/pt_path.h"

#include <cuda_runtime.h>

namespace rb {
namespace gpu {

// Device-side counters of one context. Indices into device_counters::c.
enum : uint32_t {
	CNT_ACTIVE = 0,      // paths in the current active queue
	CNT_NEXT = 1,        // paths pushed to the next active queue
	CNT_SECONDARY = 2,   // secondary rays queued this bounce
	CNT_ERROR = 3,       // first device error (rb_status), 0 if none
	CNT_CLASS = 4,       // paths per shading class this bounce (pt::NUM_CLASSES words)
	CNT_GUIDE = 10,      // paths queued for a guide evaluation this bounce
	CNT_BEAM = 11,       // light connections queued for a transmittance walk this bounce
	CNT_EXTEND_RAYS = 12, // 64-bit stats, two words each (lo, hi) from here on
	CNT_SHADOW_RAYS = 14,
	CNT_MIS_RAYS = 16,
	CNT_NODE_VISITS = 18,
	CNT_TRI_TESTS = 20,
	CNT_BEAM_RAYS = 22,  // closest-hit queries of the transmittance walks
	CNT_WORDS = 24
};
static_assert(CNT_CLASS + pt::NUM_CLASSES <= CNT_GUIDE, "class counters overlap");
// words cleared at the start of a wave: everything before the 64-bit stats
constexpr uint32_t kWaveCounterWords = CNT_EXTEND_RAYS;

// Per-launch wave parameters, read by the kernels from device memory so a
// captured graph can be replayed for every wave.
struct wave_params {
	float r2c[16];
	float c2w[16];
	float lens, focus;
	uint32_t width, height;
	uint64_t first_item;     // first work item of the wave (item = sample_offset * pixels + pixel)
	uint64_t total_items;    // pixels * spp of this render call
	uint32_t first_sample;
	uint32_t seed;
	uint32_t max_depth;
	float rr_threshold;
	uint32_t guide_flags;    // GUIDE_SAMPLE | GUIDE_TRAIN, 0 for plain path tracing
	float box_min[3];        // scene box, maps vertex positions to the guide's [0, 1] inputs
	float box_inv[3];
};

// wave_params::guide_flags
enum : uint32_t {
	GUIDE_SAMPLE = 1u,       // continuations sample the guide once it has been trained (one-sample MIS)
	GUIDE_TRAIN = 2u         // record vertices for training
};

// Path state of one wave, structure of arrays over `capacity` paths.
struct wave_buffers {
	uint32_t capacity;
	float4* ray_o;           // o.xyz, length
	float4* ray_d;           // d.xyz, unused
	float4* beta;            // beta.xyz, eta
	float4* radiance;        // L.xyz, flags (bits)
	int32_t* bounces;
	unsigned long long* rng; // PCG32 state; the increment is rebuilt from the stream seed
	uint32_t* pixel;
	uint32_t* sample;
	float4* hit;             // slot (bits), t, b1, b2
	float4* result;          // L.xyz of a finished path, w = 1 once it finished
	pt::shade_record* rec;
	float4* sec_o;           // 2 per path: shadow ray, MIS ray
	float4* sec_d;
	float4* sec_hit;
	uint32_t* queue[2];      // active queues (ping-pong)
	uint32_t* class_queue;   // NUM_CLASSES queues of `capacity` entries: paths by shading class
	uint32_t* sec_queue;
	uint32_t* counters;
	wave_params* params;
	guide::wave_guide guide;  // null pointers unless a guided render allocated them
	// volume path tracing (null unless a volume render allocated them)
	int32_t* medium;         // medium of each path, -1: vacuum
	pt::vol_rec* vrec;       // light-connection factors of the current vertex
	float4* beam;            // 2 per path: transmittance of the NEE and MIS connections
	uint32_t* beam_queue;    // connections (2 i, 2 i + 1) waiting for their transmittance
};

struct film_buffers {
	double* sum;             // 3 per pixel
	double* sum_sq;          // 3 per pixel
	uint32_t* count;         // samples per pixel
};

struct launch_cfg {
	int grid_trace, grid_shade;
	int block_trace, block_shade;
	int stack_depth;         // traversal stack entries per thread (32 or 64)
	bool count;              // node / triangle counting
	// optional CUDA events recorded around every traversal launch (profiling);
	// event pairs [2k, 2k + 1], k counted by *next_event, up to max_events pairs
	cudaEvent_t* events = nullptr;
	uint32_t* next_event = nullptr;
	uint32_t max_events = 0;
	uint8_t* event_kind = nullptr;  // 0 extend, 1 secondary
	// learned guiding: the guide state and the host-side mode (GUIDE_SAMPLE |
	// GUIDE_TRAIN) deciding which guide kernels are launched
	const guide::guide_state* guide = nullptr;
	uint32_t guide_mode = 0;
	bool volume = false;     // volume_path_integrator instead of path_integrator
};

// Ray batches for rb_trace_closest / rb_trace_shadow.
cudaError_t launch_trace_rays(const pt::scene_view& s, const uint32_t* prim_entity, const rb_ray* rays, uint32_t n,
	rb_hit* hits, bool shadow, const launch_cfg& cfg, uint32_t* counters, cudaStream_t stream);

// One wave: camera rays then `max_depth` bounces of
// extend -> shade_a -> secondary trace -> shade_b -> advance.
cudaError_t launch_wave(const pt::scene_view& s, const wave_buffers& w, const film_buffers& f, uint32_t max_depth,
	uint32_t first_queue, const launch_cfg& cfg, cudaStream_t stream);

// Adds the wave's finished samples to the film, then advances
// params->first_item by the wave capacity (the last nodes of a wave).
cudaError_t launch_next_wave(const wave_buffers& w, const film_buffers& f, int grid, cudaStream_t stream);

// Wave end with learned guiding: training-sample collection, film resolve,
// next-wave advance, then the training steps (cfg.guide_mode & GUIDE_TRAIN).
cudaError_t launch_wave_end(const wave_buffers& w, const film_buffers& f, int grid, const launch_cfg& cfg,
	cudaStream_t stream);

// Kernel launches of one wave for a given configuration (for the stats).
uint32_t wave_launches(uint32_t max_depth, const launch_cfg& cfg);

// One extra bounce (used when invisible entities make paths outlive max_depth iterations).
cudaError_t launch_bounce(const pt::scene_view& s, const wave_buffers& w, const film_buffers& f, uint32_t queue_in,
	const launch_cfg& cfg, cudaStream_t stream);

} // namespace gpu
} // namespace rb
