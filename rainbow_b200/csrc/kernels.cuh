// Kernel launchers of the wavefront path tracer (kernels.cu).
#pragma once

#include "../../include/rbgpu.h"
#include "guide/guide_host.h"
#include "pt/pt_direct.h"
#include "pt/pt_path.h"
#include "pt/pt_sss.h"

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
	CNT_TAIL = 24,       // paths taken from the active queue by the tail kernel (reset after it)
	CNT_GUIDE_MEDIUM = 25,  // medium vertices queued for a medium-guide evaluation this bounce
	CNT_FETCH_EXTEND = 26,  // rays taken from the active queue by the persistent extend kernel
	CNT_FETCH_SECONDARY = 27,  // rays taken from the secondary queue by the persistent secondary kernel
	CNT_DRAIN_WAVE = 28,    // drain-loop iterations of the current wave (below)
	CNT_DRAIN_TOTAL = 29,   // drain-loop iterations of the render call
	// device-clock timers of the traversal launches (launch_timer in kernels.cu),
	// kTimerWords words each from these (even, so the 64-bit words are aligned)
	CNT_TIMER_EXTEND = 30,
	CNT_TIMER_SECONDARY = 40,
	CNT_SSS = 50,           // paths queued for the subsurface stage this bounce
	CNT_WORDS = 52          // even, so that each lane's 64-bit words stay aligned
};
// launch timer layout, offsets from its first word: the complement of the
// earliest warp start (64-bit, so that an atomic max keeps the minimum), the
// latest warp end (64-bit), warps finished in the current launch, the total
// nanoseconds of the finished launches (64-bit) and their count
enum : uint32_t { TIMER_START = 0, TIMER_END = 2, TIMER_WARPS = 4, TIMER_TOTAL_NS = 6, TIMER_LAUNCHES = 8, kTimerWords = 10 };
static_assert(CNT_TIMER_EXTEND % 2 == 0 && CNT_TIMER_SECONDARY % 2 == 0, "64-bit timer words must be aligned");
static_assert(CNT_TIMER_EXTEND >= CNT_DRAIN_TOTAL + 1 && CNT_TIMER_SECONDARY >= CNT_TIMER_EXTEND + kTimerWords &&
	CNT_SSS >= CNT_TIMER_SECONDARY + kTimerWords && CNT_WORDS > CNT_SSS && CNT_WORDS % 2 == 0, "counter words overlap");
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

// One scene of a batched render (rb_batch_render): where its records sit in
// the merged scene arrays, and its view for this render call. Item k of the
// batch belongs to the scene with item_base <= k < the next scene's item_base;
// within it, local item j is sample first_sample + j / pixels of pixel j % pixels.
struct batch_scene {
	float4 root_a, root_b;   // the scene's root box (scene_view::root_a / root_b)
	uint32_t root_ref;       // its root in the wide-node array
	uint32_t root_node;      // its root in the reference-layout node array
	uint32_t emitter_base, num_emitters;
	uint32_t env_base, num_environments;
	uint32_t pixel_base;     // first film pixel of the scene in the merged film
	uint32_t spp;
	uint64_t item_base;      // first work item of the scene in this render call
	pt::env_distribution env;
	float r2c[16];
	float c2w[16];
	float lens, focus;
	uint32_t width, height;
	uint32_t first_sample;
	uint32_t seed;
};

// The scene_view of one scene of a batch: the merged arrays with the scene's
// root, emitter list and environments.
RB_HD pt::scene_view batch_view(const pt::scene_view& merged, const batch_scene& b) {
	pt::scene_view v = merged;
	v.root_a = b.root_a;
	v.root_b = b.root_b;
	v.root_ref = b.root_ref;
	v.root_node = b.root_node;
	v.emitters = merged.emitters + b.emitter_base;
	v.num_emitters = b.num_emitters;
	v.environments = merged.environments + b.env_base;
	v.num_environments = b.num_environments;
	v.env = b.env;
	return v;
}

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
	guide::wave_guide guide_medium;  // medium vertices of guided volume renders (else null pointers)
	// volume path tracing (null unless a volume render allocated them)
	int32_t* medium;         // medium of each path, -1: vacuum
	pt::vol_rec* vrec;       // light-connection factors of the current vertex
	float4* beam;            // 2 per path: transmittance of the NEE and MIS connections
	uint32_t* beam_queue;    // connections (2 i, 2 i + 1) waiting for their transmittance
	// ray binning before traversal (RB_SORT_RAYS)
	uint32_t* sort_keys;     // key of every active-queue entry
	uint32_t* sort_tmp;      // the binned queue before it is copied back
	uint32_t* sort_bins;     // kSortBins counts, then kSortBins cursors
	// batched rendering (null unless a batch render allocated them)
	uint32_t* scene;         // scene of each path
	const batch_scene* batch;  // num_scenes records
	uint32_t num_scenes;
};

constexpr uint32_t kSortBins = 4096;  // 3 direction-octant bits, 9 bits of an 8x8x8 Morton cell of the origin

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
	const guide::guide_state* guide_medium = nullptr;  // guided volume renders
	uint32_t guide_mode = 0;
	bool volume = false;     // volume_path_integrator instead of path_integrator
	bool batch = false;      // many scenes per wave (wave_buffers::batch)
	uint32_t sort = 0;       // hit queues: 0 one per material class, 1 a single queue (no sorting)
	uint32_t tail = 0xffffffffu;  // bounces of separate stages before the tail kernel (>= max_depth: none)
	bool refill = false;     // traversal kernels: persistent lanes that take a new ray when theirs is done
	bool shadow_first = false;  // NEE shadow rays of plain path tracing as occlusion queries (k_trace_secondary)
	bool sss = false;        // subsurface materials: a k_subsurface launch after shade_b, every bounce staged
	int carveout = 100;      // traversal kernels' preferred shared-memory carve-out, percent
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

// Writes the parameter block `dst` from `p` (passed by value at launch time).
cudaError_t launch_set_params(const wave_params& p, wave_params* dst, cudaStream_t stream);

// Sets params->first_item (the wave window of a lane).
cudaError_t launch_set_first(wave_params* params, uint64_t first, cudaStream_t stream);

// Per-pixel means of the film into `rgb` (3 floats per pixel, device memory).
cudaError_t launch_film_mean(const film_buffers& f, uint32_t pixels, float* rgb, int grid, cudaStream_t stream);

// Wave end with learned guiding: training-sample collection, film resolve,
// next-wave advance, then the training steps (cfg.guide_mode & GUIDE_TRAIN).
cudaError_t launch_wave_end(const wave_buffers& w, const film_buffers& f, int grid, const launch_cfg& cfg,
	cudaStream_t stream);

// Kernel launches of one wave for a given configuration (for the stats).
uint32_t wave_launches(uint32_t max_depth, const launch_cfg& cfg);

// One wave of direct_integrator samples (RB_RENDER_DIRECT): one thread per
// camera sample traces its light and BSDF rays itself, then the film resolve
// and the move to the next wave (3 launches).
cudaError_t launch_direct_wave(const pt::scene_view& s, const wave_buffers& w, const film_buffers& f,
	const pt::direct_cfg& dc, const launch_cfg& cfg, int resolve_grid, cudaStream_t stream);

// Buffers of the staged direct-lighting kernels (at most pt::kDirectStagedLights
// light samples): per path its record and kDirectSlots ray slots (the light
// samples, then the pending BSDF sample in slot emitter_samples) with their hits.
constexpr uint32_t kDirectSlots = pt::kDirectStagedLights + 1;
struct direct_buffers {
	pt::direct_record* rec;
	float4* ray_o;            // kDirectSlots per path: o.xyz, length
	float4* ray_d;
	float4* ray_hit;
	uint32_t* ray_queue;      // slots to trace (path * kDirectSlots + slot), count in CNT_SECONDARY
	uint32_t* shade_queue;    // unused (the shaded paths wait in the wave's material-class queues)
};
// One wave of direct_integrator samples in stages: camera rays, then per
// material class the light samples, then per BSDF sample a traversal of the
// queued rays and one round kernel per class, then the film resolve
// (7 + 5 * bsdf_samples launches).
cudaError_t launch_direct_staged_wave(const pt::scene_view& s, const wave_buffers& w, const film_buffers& f,
	const direct_buffers& db, const pt::direct_cfg& dc, const launch_cfg& cfg, int resolve_grid, cudaStream_t stream);

// Drain loop of scenes with invisible entities. A pass through an invisible
// boundary is not a bounce, so paths can outlive max_depth iterations; after
// them a wave keeps bouncing until its active queue is empty. Inside a wave's
// graph this loop is a conditional WHILE node: launch_drain_begin sets its
// condition from the active count, and each iteration runs two bounces, then
// launch_drain_step, which sets the condition again (at most
// kMaxDrainIterations iterations per wave: 4096 bounces).
constexpr uint32_t kMaxDrainIterations = 2048;
cudaError_t launch_drain_begin(cudaGraphConditionalHandle h, uint32_t* counters, cudaStream_t stream);
cudaError_t launch_drain_step(cudaGraphConditionalHandle h, uint32_t* counters, cudaStream_t stream);
uint32_t bounce_launches(const launch_cfg& cfg);  // kernels of one launch_bounce
uint32_t drain_launches(const launch_cfg& cfg);   // kernels of one drain iteration

// One extra bounce (used when invisible entities make paths outlive max_depth iterations).
cudaError_t launch_bounce(const pt::scene_view& s, const wave_buffers& w, const film_buffers& f, uint32_t queue_in,
	const launch_cfg& cfg, cudaStream_t stream);

} // namespace gpu
} // namespace rb
