// rb_render_noalloc: the wavefront render with its scratch in a static device array.
//
// For callers that cannot allocate device memory when they render (a host
// framework that owns the whole memory pool, or a loop where cudaMalloc's
// implicit device synchronisation is not acceptable). rb_render allocates its
// wave buffers, film and graph on first use; this entry point allocates
// nothing: per-path state, queues, counters and the wave parameter block are
// carved out of g_noalloc_scratch below, and the film is the caller's.
//
// Only the plain path integrator is available here (RB_RENDER_RESET is the one
// flag accepted): the volume, direct-lighting and guided renders need buffers
// that the scratch array does not hold. Scenes with invisible entities get the
// same bounded drain loop as rb_render's direct launches (a pass through a
// shape without a material is not a bounce, so paths can outlive max_depth
// iterations), with a host read of the active count between bounces.
//
// g_noalloc_scratch is a file-scope __device__ array, so every GPU that loads
// the library holds its RB_NOALLOC_SCRATCH_BYTES until the process exits. In
// host code its name only stands in for the device object: the device address
// comes from cudaGetSymbolAddress, looked up once per device with that device
// current, on the first call there (make that call before any stream capture).
// Every call reuses the same array and finds the previous call's contents in
// it; the counters and parameter block are rewritten by each call, so calls
// that overlap on the GPU race and must be serialised by the caller. The call
// also reads its counters back through the context's page-locked counter
// buffer, so it must be serialised with every other call on the same context.
#include "context.h"

#include <mutex>

namespace rb {
namespace gpu {
bool context_view(rb_context* c, pt::scene_view* view, launch_cfg* cfg, cudaStream_t* stream, int* device,
	uint32_t** counters_host, bool* has_invisible);
} // namespace gpu
} // namespace rb

namespace {

using rb::gpu::wave_buffers;
using rb::gpu::wave_params;

static __device__ __align__(256) unsigned char g_noalloc_scratch[RB_NOALLOC_SCRATCH_BYTES];

constexpr size_t kAlign = 256;
constexpr size_t round_up(size_t v) { return (v + kAlign - 1) / kAlign * kAlign; }

// Byte layout of the scratch array for n paths.
struct scratch_layout {
	size_t counters, params, ray_o, ray_d, beta, radiance, bounces, rng, pixel, sample, hit, result, rec, sec_o, sec_d,
		sec_hit, queue0, queue1, sec_queue, class_queue, end;
};
constexpr scratch_layout layout_for(size_t n) {
	scratch_layout l{};
	size_t o = 0;
	auto take = [&o](size_t bytes) { const size_t at = o; o = round_up(o + bytes); return at; };
	l.counters = take(rb::gpu::CNT_WORDS * sizeof(uint32_t));
	l.params = take(sizeof(wave_params));
	l.ray_o = take(n * sizeof(float4));
	l.ray_d = take(n * sizeof(float4));
	l.beta = take(n * sizeof(float4));
	l.radiance = take(n * sizeof(float4));
	l.bounces = take(n * sizeof(int32_t));
	l.rng = take(n * sizeof(unsigned long long));
	l.pixel = take(n * sizeof(uint32_t));
	l.sample = take(n * sizeof(uint32_t));
	l.hit = take(n * sizeof(float4));
	l.result = take(n * sizeof(float4));
	l.rec = take(n * sizeof(rb::pt::shade_record));
	l.sec_o = take(2 * n * sizeof(float4));
	l.sec_d = take(2 * n * sizeof(float4));
	l.sec_hit = take(2 * n * sizeof(float4));
	l.queue0 = take(n * sizeof(uint32_t));
	l.queue1 = take(n * sizeof(uint32_t));
	l.sec_queue = take(2 * n * sizeof(uint32_t));
	l.class_queue = take(rb::pt::NUM_CLASSES * n * sizeof(uint32_t));
	l.end = o;
	return l;
}
static_assert(layout_for(RB_NOALLOC_MAX_PATHS).end <= RB_NOALLOC_SCRATCH_BYTES, "no-alloc scratch too small");

// Writes the parameter block from a kernel argument, so no host buffer has to
// outlive the call.
__global__ void k_noalloc_params(wave_params p, wave_params* dst) { *dst = p; }

constexpr int kMaxDevices = 64;
std::mutex g_lock;
unsigned char* g_scratch_address[kMaxDevices] = {};

// The scratch array's device address on `device` (which must be current).
rb_status scratch_address(int device, unsigned char** out) {
	if (device < 0 || device >= kMaxDevices) return RB_ERR_INVALID_ARGUMENT;
	std::lock_guard<std::mutex> guard(g_lock);
	if (g_scratch_address[device] == nullptr) {
		void* p = nullptr;
		const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
		if (e != cudaSuccess || p == nullptr) return RB_ERR_CUDA;
		g_scratch_address[device] = static_cast<unsigned char*>(p);
	}
	*out = g_scratch_address[device];
	return RB_OK;
}

} // namespace

extern "C" rb_status rb_render_noalloc(rb_context* ctx, const rb_render_params* prm, double* d_sum_rgb, double* d_sum_sq_rgb,
	uint32_t* d_count, void* stream) {
	if (ctx == nullptr || prm == nullptr || d_sum_rgb == nullptr || d_sum_sq_rgb == nullptr || d_count == nullptr)
		return RB_ERR_INVALID_ARGUMENT;
	rb::pt::scene_view view;
	rb::gpu::launch_cfg cfg;
	cudaStream_t own = nullptr;
	int device = 0;
	uint32_t* counters_host = nullptr;
	bool has_invisible = false;
	if (!rb::gpu::context_view(ctx, &view, &cfg, &own, &device, &counters_host, &has_invisible)) return RB_ERR_NO_SCENE;
	if (prm->flags & ~static_cast<uint32_t>(RB_RENDER_RESET)) return RB_ERR_UNSUPPORTED;  // plain path tracing only
	const rb_camera_desc& cam = prm->camera;
	if (!rb::ctx::host_is_valid_camera(cam) || prm->spp == 0 || prm->max_depth == 0 || prm->max_depth > 64)
		return RB_ERR_INVALID_ARGUMENT;
	if (static_cast<uint64_t>(prm->first_sample) + prm->spp > (1u << 24)) return RB_ERR_INVALID_ARGUMENT;
	// both factors are below 2^24 here, so the product cannot wrap
	const uint64_t pixels = static_cast<uint64_t>(cam.width) * static_cast<uint64_t>(cam.height);
	const uint64_t paths = pixels * prm->spp;
	if (paths > RB_NOALLOC_MAX_PATHS) return RB_ERR_TOO_LARGE;
	const cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : own;

	if (cudaSetDevice(device) != cudaSuccess) return RB_ERR_CUDA;
	unsigned char* base = nullptr;
	const rb_status st = scratch_address(device, &base);
	if (st != RB_OK) return st;

	const uint32_t n = static_cast<uint32_t>(paths);
	const scratch_layout l = layout_for(n);
	wave_buffers w{};
	w.capacity = n;
	w.counters = reinterpret_cast<uint32_t*>(base + l.counters);
	w.params = reinterpret_cast<wave_params*>(base + l.params);
	w.ray_o = reinterpret_cast<float4*>(base + l.ray_o);
	w.ray_d = reinterpret_cast<float4*>(base + l.ray_d);
	w.beta = reinterpret_cast<float4*>(base + l.beta);
	w.radiance = reinterpret_cast<float4*>(base + l.radiance);
	w.bounces = reinterpret_cast<int32_t*>(base + l.bounces);
	w.rng = reinterpret_cast<unsigned long long*>(base + l.rng);
	w.pixel = reinterpret_cast<uint32_t*>(base + l.pixel);
	w.sample = reinterpret_cast<uint32_t*>(base + l.sample);
	w.hit = reinterpret_cast<float4*>(base + l.hit);
	w.result = reinterpret_cast<float4*>(base + l.result);
	w.rec = reinterpret_cast<rb::pt::shade_record*>(base + l.rec);
	w.sec_o = reinterpret_cast<float4*>(base + l.sec_o);
	w.sec_d = reinterpret_cast<float4*>(base + l.sec_d);
	w.sec_hit = reinterpret_cast<float4*>(base + l.sec_hit);
	w.queue[0] = reinterpret_cast<uint32_t*>(base + l.queue0);
	w.queue[1] = reinterpret_cast<uint32_t*>(base + l.queue1);
	w.sec_queue = reinterpret_cast<uint32_t*>(base + l.sec_queue);
	w.class_queue = reinterpret_cast<uint32_t*>(base + l.class_queue);
	rb::gpu::film_buffers f{d_sum_rgb, d_sum_sq_rgb, d_count};

	wave_params p{};
	for (int i = 0; i < 16; i++) {
		p.r2c[i] = cam.raster_to_camera[i];
		p.c2w[i] = cam.camera_to_world[i];
	}
	p.lens = cam.lens_radius;
	p.focus = cam.focus_distance;
	p.width = static_cast<uint32_t>(cam.width);
	p.height = static_cast<uint32_t>(cam.height);
	p.first_item = 0;
	p.total_items = paths;
	p.first_sample = prm->first_sample;
	p.seed = prm->seed;
	p.max_depth = prm->max_depth;
	p.rr_threshold = prm->rr_threshold;

	// the call's own slot of the context's page-locked counter buffer (the last
	// lane's; rb_render only touches it while it runs and returns synchronised)
	uint32_t* h = counters_host + (rb::ctx::kMaxLanes - 1) * rb::gpu::CNT_WORDS;
	cudaError_t e = cudaSuccess;
	if (prm->flags & RB_RENDER_RESET) {  // the caller's accumulators, as rb_render clears its film
		e = cudaMemsetAsync(d_sum_rgb, 0, 3 * pixels * sizeof(double), s);
		if (e == cudaSuccess) e = cudaMemsetAsync(d_sum_sq_rgb, 0, 3 * pixels * sizeof(double), s);
		if (e == cudaSuccess) e = cudaMemsetAsync(d_count, 0, pixels * sizeof(uint32_t), s);
	}
	// everything that must start at zero: counters (queues, error word, stats)
	if (e == cudaSuccess) e = cudaMemsetAsync(w.counters, 0, rb::gpu::CNT_WORDS * sizeof(uint32_t), s);
	if (e != cudaSuccess) return RB_ERR_CUDA;
	k_noalloc_params<<<1, 1, 0, s>>>(p, w.params);
	e = cudaGetLastError();
	if (e == cudaSuccess) e = rb::gpu::launch_wave(view, w, f, prm->max_depth, 0u, cfg, s);
	// scenes with invisible entities: keep bouncing until the active queue is
	// empty, at most 4096 more bounces (rb_render's direct-launch drain)
	uint32_t q = prm->max_depth & 1u;
	for (int guard = 0; guard < 4096 && has_invisible && e == cudaSuccess; guard++) {
		e = cudaMemcpyAsync(h, w.counters, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
		if (e == cudaSuccess) e = cudaStreamSynchronize(s);
		if (e != cudaSuccess || h[rb::gpu::CNT_ACTIVE] == 0) break;
		e = rb::gpu::launch_bounce(view, w, f, q, cfg, s);
		q ^= 1u;
	}
	if (e == cudaSuccess) e = rb::gpu::launch_next_wave(w, f, cfg.grid_shade, s);
	if (e == cudaSuccess) e = cudaMemcpyAsync(h, w.counters, rb::gpu::CNT_WORDS * sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
	if (e == cudaSuccess) e = cudaStreamSynchronize(s);
	if (e != cudaSuccess) return RB_ERR_CUDA;
	return h[rb::gpu::CNT_ERROR] != 0 ? static_cast<rb_status>(h[rb::gpu::CNT_ERROR]) : RB_OK;
}
