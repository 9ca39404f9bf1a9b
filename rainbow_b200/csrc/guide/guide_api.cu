// C ABI of the learned path guide (the rb_guide_* entry points of rbgpu.h).
// The guide lives in the context; rb_render with RB_RENDER_GUIDE /
// RB_RENDER_TRAIN drives it inside the wave graph, these calls expose the
// network on host data: initialisation, parameters, the forward pass, training
// steps and the sampler.
#include "../../../include/rbgpu.h"
#include "guide_host.h"

#include <cmath>
#include <cstring>
#include <vector>

namespace rb {
namespace gpu {
guide::guide_state* context_guide(rb_context* c, cudaStream_t* stream, int* device, int* num_sms);
guide::guide_state* context_guide_medium(rb_context* c);
void context_drop_graph(rb_context* c);
} // namespace gpu
} // namespace rb

using namespace rb;
using namespace rb::guide;

namespace {

rb_status from_cuda(cudaError_t e) {
	if (e == cudaSuccess) return RB_OK;
	if (e == cudaErrorMemoryAllocation) return RB_ERR_OUT_OF_MEMORY;
	return RB_ERR_CUDA;
}

#define RB_CUDA(call)                                      \
	do {                                                   \
		const cudaError_t rb_e_ = (call);                  \
		if (rb_e_ != cudaSuccess) return from_cuda(rb_e_); \
	} while (0)

// splitmix64 (Steele, Lea, Flood 2014), for a seeded, portable initialisation.
struct splitmix {
	uint64_t s;
	uint64_t next() {
		uint64_t z = (s += 0x9E3779B97F4A7C15ull);
		z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
		z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
		return z ^ (z >> 31);
	}
	float uniform() { return static_cast<float>(next() >> 40) * (1.f / 16777216.f); }
};

// He-uniform weights over the live inputs, zero biases; the output layer is
// scaled by 0.1 (an almost uniform untrained guide) and its unused rows are
// zero. First-layer weights of encoding octave k > 3 start 2^-(k-3) smaller:
// at 2^k pi with k near 11 a feature changes sign every few millimetres of the
// scene, so the untrained network starts smooth and sharpens where the
// training data asks for it.
std::vector<float> default_params(uint32_t seed) {
	std::vector<float> p(kNumParams, 0.f);
	splitmix rng{0x5EEDull ^ (static_cast<uint64_t>(seed) << 20)};
	for (int l = 0; l < kLayers; l++) {
		const int in = layer_in(l), out = layer_out(l), live = l == 0 ? kFeatures : in;
		const float lim = std::sqrt(6.f / static_cast<float>(live)) * (l == kLayers - 1 ? 0.1f : 1.f);
		float* w = p.data() + flat_offset(l);
		for (int o = 0; o < out; o++)
			for (int i = 0; i < in; i++) {
				const float u = rng.uniform();
				const int octave = (i % 24) / 2;  // feature 24 j + 2 k + s
				const float scale = (l == 0 && octave > 3) ? std::ldexp(1.f, 3 - octave) : 1.f;
				w[o * in + i] = (i < live && !(l == kLayers - 1 && o > 40)) ? (2.f * u - 1.f) * lim * scale : 0.f;
			}
	}
	return p;
}

std::vector<float> to_device_layout(const float* flat) {
	std::vector<float> a(kAugParams, 0.f);
	for (int i = 0; i < kAugParams; i++) {
		int l, o, k;
		aug_coords(i, l, o, k);
		const int f = aug_to_flat(l, o, k);
		a[i] = f >= 0 ? flat[f] : 0.f;
	}
	return a;
}

void to_flat_layout(const float* aug, float* flat) {
	std::memset(flat, 0, sizeof(float) * kNumParams);
	for (int i = 0; i < kAugParams; i++) {
		int l, o, k;
		aug_coords(i, l, o, k);
		const int f = aug_to_flat(l, o, k);
		if (f >= 0) flat[f] = aug[i];
	}
}

struct guide_ctx {
	guide_state* g = nullptr;
	cudaStream_t stream = nullptr;
	int device = 0, sms = 0;
};

rb_status open_guide(rb_context* ctx, guide_ctx& gc, bool need_ready) {
	if (ctx == nullptr) return RB_ERR_INVALID_ARGUMENT;
	gc.g = gpu::context_guide(ctx, &gc.stream, &gc.device, &gc.sms);
	if (gc.g == nullptr) return RB_ERR_INVALID_ARGUMENT;
	RB_CUDA(cudaSetDevice(gc.device));
	if (need_ready && !gc.g->ready) {
		const rb_status st = rb_guide_init(ctx, nullptr);
		if (st != RB_OK) return st;
	}
	return RB_OK;
}

rb_status upload_params(guide_ctx& gc, const float* flat) {
	const std::vector<float> a = to_device_layout(flat);
	guide_state& g = *gc.g;
	RB_CUDA(cudaMemcpyAsync(g.master, a.data(), sizeof(float) * kAugParams, cudaMemcpyHostToDevice, gc.stream));
	RB_CUDA(cudaMemsetAsync(g.adam_m, 0, sizeof(float) * kAugParams, gc.stream));
	RB_CUDA(cudaMemsetAsync(g.adam_v, 0, sizeof(float) * kAugParams, gc.stream));
	RB_CUDA(launch_init_image(g, gc.stream));
	RB_CUDA(cudaStreamSynchronize(gc.stream));
	return RB_OK;
}

rb_status device_error(guide_ctx& gc) {
	device_state s{};
	RB_CUDA(cudaMemcpy(&s, gc.g->dstate, sizeof(s), cudaMemcpyDeviceToHost));
	return s.error != 0u ? static_cast<rb_status>(s.error) : RB_OK;
}

template <typename T>
struct scratch {
	T* p = nullptr;
	~scratch() {
		if (p) cudaFree(p);
	}
	cudaError_t alloc(size_t n) { return cudaMalloc(reinterpret_cast<void**>(&p), n * sizeof(T)); }
};

} // namespace

namespace rb {
namespace guide {

// (Re)creates guide `g` with fresh weights and zero Adam moments for `config`
// (defaults filled in for zero fields).
rb_status init_state(guide_state& g, const rb_guide_config* config, int sms, cudaStream_t stream) {
	release(g);
	rb_guide_config cfg{};
	if (config) cfg = *config;
	if (!(cfg.learning_rate > 0.f)) cfg.learning_rate = 1e-3f;
	if (cfg.batch_size == 0) cfg.batch_size = 1u << 18;
	if (cfg.steps_per_wave == 0) cfg.steps_per_wave = 8;
	if (cfg.max_samples == 0) cfg.max_samples = 1u << 21;
	if (cfg.min_rows == 0) cfg.min_rows = 4096;
	if (cfg.warmup_steps == 0) cfg.warmup_steps = 1;
	if (cfg.batch_size > (1u << 24) || cfg.max_samples > (1u << 26) || cfg.steps_per_wave > 64) return RB_ERR_INVALID_ARGUMENT;
	uint32_t ring = 1024u;
	while (ring < cfg.max_samples) ring <<= 1;  // the replay ring holds a power of two
	cfg.max_samples = ring;
	g.cfg = cfg;
	g.sample_cap = cfg.max_samples;
	g.weight_clip = cfg.weight_clip == 0.f ? 16.f : (cfg.weight_clip < 0.f ? 0.f : cfg.weight_clip);
	const cudaError_t e = allocate(g, sms);
	if (e != cudaSuccess) {
		release(g);
		return from_cuda(e);
	}
	guide_ctx gc;
	gc.g = &g;
	gc.stream = stream;
	gc.sms = sms;
	const std::vector<float> p = default_params(cfg.seed);
	const rb_status st = upload_params(gc, p.data());
	if (st != RB_OK) {
		release(g);
		return st;
	}
	g.ready = true;
	return RB_OK;
}

} // namespace guide
} // namespace rb

extern "C" {

// Creates the surface guide; the medium guide of volume renders is released
// here and created again, from the same configuration with seed + 1, by the
// next guided volume render.
rb_status rb_guide_init(rb_context* ctx, const rb_guide_config* config) {
	guide_ctx gc;
	rb_status st = open_guide(ctx, gc, false);
	if (st != RB_OK) return st;
	RB_CUDA(cudaStreamSynchronize(gc.stream));
	gpu::context_drop_graph(ctx);
	release(*gpu::context_guide_medium(ctx));
	return init_state(*gc.g, config, gc.sms, gc.stream);
}

rb_status rb_check_bounded_wait(rb_context* ctx, uint32_t limit_us, rb_status* status) {
	if (status == nullptr || limit_us == 0 || limit_us > 10000000u) return RB_ERR_INVALID_ARGUMENT;
	guide_ctx gc;
	const rb_status st = open_guide(ctx, gc, false);
	if (st != RB_OK) return st;
	scratch<uint32_t> d;
	RB_CUDA(d.alloc(1));
	RB_CUDA(cudaMemsetAsync(d.p, 0xff, sizeof(uint32_t), gc.stream));
	RB_CUDA(launch_bounded_wait(static_cast<uint64_t>(limit_us) * 1000ull, d.p, gc.stream));
	uint32_t h = 0;
	RB_CUDA(cudaMemcpyAsync(&h, d.p, sizeof(h), cudaMemcpyDeviceToHost, gc.stream));
	RB_CUDA(cudaStreamSynchronize(gc.stream));
	*status = static_cast<rb_status>(h);
	return RB_OK;
}

rb_status rb_guide_medium_stats_get(rb_context* ctx, rb_guide_stats* out) {
	if (ctx == nullptr || out == nullptr) return RB_ERR_INVALID_ARGUMENT;
	guide_ctx gc;
	const rb_status st = open_guide(ctx, gc, false);
	if (st != RB_OK) return st;
	*out = rb_guide_stats{};
	guide_state* g = gpu::context_guide_medium(ctx);
	if (!g->ready) return RB_OK;
	RB_CUDA(cudaStreamSynchronize(gc.stream));
	device_state s{};
	RB_CUDA(cudaMemcpy(&s, g->dstate, sizeof(s), cudaMemcpyDeviceToHost));
	out->steps = s.step;
	out->samples_last_wave = s.wave_written;
	out->candidates_last_wave = s.candidates;
	out->device_error = s.error;
	out->last_loss = s.last_loss;
	out->rows_last_step = s.rows_last;
	return RB_OK;
}

rb_status rb_guide_get_params(rb_context* ctx, float* params, uint32_t count) {
	if (params == nullptr || count < kNumParams) return RB_ERR_INVALID_ARGUMENT;
	guide_ctx gc;
	const rb_status st = open_guide(ctx, gc, true);
	if (st != RB_OK) return st;
	std::vector<float> a(kAugParams);
	RB_CUDA(cudaStreamSynchronize(gc.stream));
	RB_CUDA(cudaMemcpy(a.data(), gc.g->master, sizeof(float) * kAugParams, cudaMemcpyDeviceToHost));
	to_flat_layout(a.data(), params);
	return RB_OK;
}

rb_status rb_guide_set_params(rb_context* ctx, const float* params, uint32_t count) {
	if (params == nullptr || count < kNumParams) return RB_ERR_INVALID_ARGUMENT;
	guide_ctx gc;
	rb_status st = open_guide(ctx, gc, true);
	if (st != RB_OK) return st;
	RB_CUDA(cudaStreamSynchronize(gc.stream));
	st = upload_params(gc, params);
	if (st != RB_OK) return st;
	device_state s{};
	RB_CUDA(cudaMemcpy(&s, gc.g->dstate, sizeof(s), cudaMemcpyDeviceToHost));
	s.step = 0u;
	s.usable = 1u;
	RB_CUDA(cudaMemcpy(gc.g->dstate, &s, sizeof(s), cudaMemcpyHostToDevice));
	return RB_OK;
}

rb_status rb_guide_forward(rb_context* ctx, const float* inputs, uint32_t n, float* outputs) {
	if (n > 0 && (inputs == nullptr || outputs == nullptr)) return RB_ERR_INVALID_ARGUMENT;
	if (n > (1u << 26)) return RB_ERR_INVALID_ARGUMENT;
	guide_ctx gc;
	const rb_status st = open_guide(ctx, gc, true);
	if (st != RB_OK || n == 0) return st;
	scratch<float> x, out;
	RB_CUDA(x.alloc(static_cast<size_t>(n) * kInputs));
	RB_CUDA(out.alloc(static_cast<size_t>(n) * kOutputs));
	RB_CUDA(cudaMemcpyAsync(x.p, inputs, sizeof(float) * kInputs * n, cudaMemcpyHostToDevice, gc.stream));
	RB_CUDA(launch_forward_raw(*gc.g, x.p, n, out.p, gc.stream));
	RB_CUDA(cudaMemcpyAsync(outputs, out.p, sizeof(float) * kOutputs * n, cudaMemcpyDeviceToHost, gc.stream));
	RB_CUDA(cudaStreamSynchronize(gc.stream));
	return device_error(gc);
}

rb_status rb_guide_train(rb_context* ctx, const rb_guide_sample* samples, uint32_t n, uint32_t steps, uint32_t flags,
	float* gradient, float* loss) {
	if (n > 0 && samples == nullptr) return RB_ERR_INVALID_ARGUMENT;
	if (n > (1u << 24) || steps > 4096) return RB_ERR_INVALID_ARGUMENT;
	static_assert(sizeof(rb_guide_sample) == 16 * kSampleFloat4, "rb_guide_sample is four float4");
	guide_ctx gc;
	const rb_status st = open_guide(ctx, gc, true);
	if (st != RB_OK) return st;
	guide_state& g = *gc.g;
	RB_CUDA(cudaStreamSynchronize(gc.stream));
	if (g.host_sample_cap < n) {
		if (g.host_samples) cudaFree(g.host_samples);
		g.host_samples = nullptr;
		g.host_sample_cap = 0;
		RB_CUDA(cudaMalloc(reinterpret_cast<void**>(&g.host_samples), sizeof(rb_guide_sample) * n));
		g.host_sample_cap = n;
	}
	if (n > 0) RB_CUDA(cudaMemcpyAsync(g.host_samples, samples, sizeof(rb_guide_sample) * n, cudaMemcpyHostToDevice, gc.stream));
	RB_CUDA(cudaMemcpyAsync(g.host_count, &n, sizeof(uint32_t), cudaMemcpyHostToDevice, gc.stream));
	const bool sequential = (flags & RB_GUIDE_SEQUENTIAL) != 0;
	const uint32_t batch = sequential ? (n > 0 ? n : 1u) : g.cfg.batch_size;
	for (uint32_t k = 0; k < steps; k++)
		RB_CUDA(launch_train_step(g, g.host_samples, g.host_count, n, batch, 1u, sequential, false, gc.stream));
	RB_CUDA(cudaStreamSynchronize(gc.stream));
	if (gradient) {
		std::vector<float> a(kAugParams);
		RB_CUDA(cudaMemcpy(a.data(), g.grad, sizeof(float) * kAugParams, cudaMemcpyDeviceToHost));
		to_flat_layout(a.data(), gradient);
	}
	device_state s{};
	RB_CUDA(cudaMemcpy(&s, g.dstate, sizeof(s), cudaMemcpyDeviceToHost));
	if (loss) *loss = s.last_loss;
	return s.error != 0u ? static_cast<rb_status>(s.error) : RB_OK;
}

rb_status rb_guide_sample_dirs(rb_context* ctx, const float* outputs, const float* u, uint32_t n, float* directions,
	float* pdfs) {
	if (n > 0 && (outputs == nullptr || u == nullptr || directions == nullptr || pdfs == nullptr)) return RB_ERR_INVALID_ARGUMENT;
	if (n > (1u << 26)) return RB_ERR_INVALID_ARGUMENT;
	guide_ctx gc;
	const rb_status st = open_guide(ctx, gc, false);
	if (st != RB_OK || n == 0) return st;
	scratch<float> raw, uu, d, pd;
	RB_CUDA(raw.alloc(static_cast<size_t>(n) * kOutputs));
	RB_CUDA(uu.alloc(static_cast<size_t>(n) * 3));
	RB_CUDA(d.alloc(static_cast<size_t>(n) * 3));
	RB_CUDA(pd.alloc(n));
	RB_CUDA(cudaMemcpyAsync(raw.p, outputs, sizeof(float) * kOutputs * n, cudaMemcpyHostToDevice, gc.stream));
	RB_CUDA(cudaMemcpyAsync(uu.p, u, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, gc.stream));
	RB_CUDA(launch_decode_sample(raw.p, uu.p, n, d.p, pd.p, gc.stream));
	RB_CUDA(cudaMemcpyAsync(directions, d.p, sizeof(float) * 3 * n, cudaMemcpyDeviceToHost, gc.stream));
	RB_CUDA(cudaMemcpyAsync(pdfs, pd.p, sizeof(float) * n, cudaMemcpyDeviceToHost, gc.stream));
	RB_CUDA(cudaStreamSynchronize(gc.stream));
	return RB_OK;
}

rb_status rb_guide_stats_get(rb_context* ctx, rb_guide_stats* out) {
	if (out == nullptr) return RB_ERR_INVALID_ARGUMENT;
	guide_ctx gc;
	const rb_status st = open_guide(ctx, gc, false);
	if (st != RB_OK) return st;
	*out = rb_guide_stats{};
	if (!gc.g->ready) return RB_OK;
	RB_CUDA(cudaStreamSynchronize(gc.stream));
	device_state s{};
	RB_CUDA(cudaMemcpy(&s, gc.g->dstate, sizeof(s), cudaMemcpyDeviceToHost));
	out->steps = s.step;
	out->samples_last_wave = s.wave_written;
	out->candidates_last_wave = s.candidates;
	out->device_error = s.error;
	out->last_loss = s.last_loss;
	out->rows_last_step = s.rows_last;
	return RB_OK;
}

} // extern "C"
