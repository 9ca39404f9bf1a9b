// Host-side state and kernel launchers of the learned path guide.
#pragma once

#include "../../../include/rbgpu.h"
#include "guide_net.h"

#include <cuda_runtime.h>
#include <stdint.h>

namespace rb {
namespace guide {

// Device-resident counters of the guide (one per context).
struct device_state {
	uint32_t step;             // Adam steps taken
	uint32_t ticket;           // blocks of the running Adam launch that finished
	uint32_t ring_head;        // training samples written since the guide was created (ring index, mod 2^32)
	uint32_t candidates;       // vertices with a positive training weight this wave
	uint32_t candidates_last;  // the same for the previous wave (sets the keep probability)
	uint32_t error;            // rb_status of a failed bounded wait, RB_OK if none
	float last_loss;           // loss of the last step
	uint32_t rows_last;        // rows of the last step
	uint32_t usable;           // weights trained or loaded: the renderer may sample the guide
	uint32_t wave_written;     // training samples written by the current wave
	uint32_t ring_filled;      // samples in the ring (<= capacity); the training steps draw from all of them
	uint32_t wave_budget;      // training steps to run after this wave (the launches beyond it return at once)
	uint32_t wave_step;        // training steps run after this wave so far
	float wave_weight;         // sum of the weights written by this wave
	float weight_mean;         // running mean of the training weights (exponential over waves)
	uint32_t pad;
};

// One recorded path vertex (5 float4): inputs x0..x8, the continuation
// direction, the BSDF pdf of that direction, the throughput at the vertex and
// the path radiance after the vertex's direct lighting.
constexpr int kVertexFloat4 = 5;
// One training sample (4 float4): x0..x8, direction, bsdf_pdf, weight.
constexpr int kSampleFloat4 = 4;

struct guide_state {
	bool ready = false;              // buffers allocated
	rb_guide_config cfg{};
	float weight_clip = 16.f;        // training weights clipped at this multiple of their running mean
	device_state* dstate = nullptr;
	float* master = nullptr;         // FP32 weights, device layout (kAugParams)
	float* adam_m = nullptr;
	float* adam_v = nullptr;
	uint8_t* image = nullptr;        // bf16 image of the weights (kImageBytes)
	float* grad = nullptr;           // summed gradient of the last step (kAugParams), device layout
	float* partial = nullptr;        // per-CTA gradient partials [ctas][kAugParams]
	float* partial_loss = nullptr;   // [ctas]
	int ctas = 0;
	float4* samples = nullptr;       // replay ring of training samples, filled by every training wave
	uint32_t sample_cap = 0;         // ring capacity, a power of two
	float4* host_samples = nullptr;  // rb_guide_train upload buffer (device)
	uint32_t host_sample_cap = 0;
	uint32_t* host_count = nullptr;  // its sample count (device)
	// per-wave path buffers (sized with the wave)
	float4* query_in = nullptr;      // 3 per path: the 9 inputs
	float4* query_out = nullptr;     // 12 per path: decoded guide
	uint32_t* queue = nullptr;       // paths that need a guide this bounce
	float4* vertices = nullptr;      // kVertexFloat4 per record, `depth` records per path
	uint32_t* vertex_count = nullptr;
	uint32_t wave_capacity = 0;
	uint32_t depth = 0;
};

// Pointers the wavefront kernels use (a plain copy inside wave_buffers).
struct wave_guide {
	const device_state* dstate;
	float4* query_in;
	float4* query_out;
	uint32_t* queue;
	float4* vertices;
	uint32_t* vertex_count;
	uint32_t depth;
	const uint32_t* usable;  // the guide may be sampled: the device_state's flag, or a lane's snapshot of it
	const uint8_t* image;    // bf16 weights this wave's forward passes read: the training image, or a lane's snapshot
};

// Per-wave guide buffers of one wave lane, with the lane's snapshot of the
// weights and of the usable flag (taken after the lane's own wave trained), so
// that overlapping waves read weights fixed by the wave order alone.
struct lane_guide {
	float4* query_in = nullptr;
	float4* query_out = nullptr;
	uint32_t* queue = nullptr;
	float4* vertices = nullptr;
	uint32_t* vertex_count = nullptr;
	uint32_t capacity = 0, depth = 0;
	uint8_t* image = nullptr;
	uint32_t* usable = nullptr;
};
cudaError_t allocate_lane(lane_guide& l, uint32_t capacity, uint32_t depth);
void release_lane(lane_guide& l);
// The guide's own buffers, weights and flag (one lane).
wave_guide state_view(const guide_state& g);
// A lane's buffers and snapshots.
wave_guide lane_view(const guide_state& g, const lane_guide& l);
// One bounded mbarrier wait that nothing completes (failure-detection check).
cudaError_t launch_bounded_wait(uint64_t limit_ns, uint32_t* status, cudaStream_t s);
// Copies the training image and the usable flag into the lane's snapshots.
cudaError_t launch_snapshot(const guide_state& g, const lane_guide& l, cudaStream_t s);

void release(guide_state& g);
// (Re)creates a guide with fresh weights (guide_api.cu); config may be null (defaults).
rb_status init_state(guide_state& g, const rb_guide_config* config, int sms, cudaStream_t stream);
cudaError_t allocate(guide_state& g, int ctas);
cudaError_t allocate_wave(guide_state& g, uint32_t capacity, uint32_t depth);

// Launchers (guide.cu).
cudaError_t launch_init_image(const guide_state& g, cudaStream_t s);
cudaError_t launch_forward_raw(const guide_state& g, const float* x, uint32_t n, float* out, cudaStream_t s);
// Forward pass of the queued vertices of a wave (wg: its buffers and weights).
cudaError_t launch_forward_queue(const guide_state& g, const wave_guide& wg, const uint32_t* count, cudaStream_t s);
// One training step over min(batch, *count, count_cap) samples: the gradient kernel then
// the reduction + Adam kernel. sequential: row r uses sample r, else rows draw
// samples by a hash of (step, row). budgeted: the step runs only while the
// wave's step budget (device_state::wave_budget) is not used up.
cudaError_t launch_train_step(const guide_state& g, const float4* samples, const uint32_t* count, uint32_t count_cap,
	uint32_t batch, uint32_t min_rows, bool sequential, bool budgeted, cudaStream_t s);
cudaError_t launch_decode_sample(const float* raw, const float* u, uint32_t n, float* dirs, float* pdfs, cudaStream_t s);
// Wave end: training samples from the recorded vertices (wg) of the wave's paths.
cudaError_t launch_collect(const guide_state& g, const wave_guide& wg, const float4* result, const uint64_t* first_item,
	const uint64_t* total_items, uint32_t capacity, cudaStream_t s);

} // namespace guide
} // namespace rb
