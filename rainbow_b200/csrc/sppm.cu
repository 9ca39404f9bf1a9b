// rb_render_photons: stochastic progressive photon mapping
// (photon_mapping_integrator::render, rainbow-cpu/integrators/photon_mapping_integrator.cpp:386-560)
// on the GPU. One iteration is a fixed sequence of launches on the context's
// stream:
//   k_sppm_visible   one thread per pixel: camera path to its visible point
//                    (direct light on the way added to the pixel), and the
//                    bound of the search spheres and the largest radius by
//                    warp reductions and atomics on order-preserving keys
//   k_sppm_grid      one thread: the grid's cell counts from that bound
//   k_sppm_cells<0>  one thread per visible point: entries per hash bucket
//   k_scan_*         exclusive prefix sum of the bucket counts (bucket offsets)
//   k_sppm_cells<1>  the bucket entries (pixel indices), a pixel once per cell
//                    of its sphere's box that hashes to the bucket, as the
//                    reference's lists hold it
//   k_sppm_photons   one thread per photon: its path with importance
//                    transport; at each landing, the bucket's visible points
//                    within their radius receive beta f (atomic adds)
//   k_sppm_update    one thread per pixel: radius, photon count and flux
// and k_sppm_image writes the pixel values after the last iteration. Rays are
// traced in the thread (shared-memory stacks, the out-of-line traversal);
// pixels and photons draw from their own streams (sppm_pixel_seed,
// sppm_photon_seed) instead of the reference's per-tile and per-chunk ones.
#include "context.h"
#include "device_common.cuh"
#include "pt/pt_photon.h"

#include <cfloat>

namespace rb {
namespace gpu {
bool context_view(rb_context* c, pt::scene_view* view, launch_cfg* cfg, cudaStream_t* stream, int* device,
	uint32_t** counters_host, bool* has_invisible);
} // namespace gpu
} // namespace rb

namespace rb {
namespace gpu {
namespace {

using namespace rb::pt;

// Per-pixel and grid state of one render call (device pointers).
struct sppm_buffers {
	uint32_t npix, width;
	float4* vp_p;      // visible point: p, uv.y
	float4* vp_wo;     // wo, material bits (0xffffffff: no visible point)
	float4* vp_beta;   // beta, uv.x
	float4* tau;       // tau, n
	float4* L;         // L, radius
	float* phi;        // 3 per pixel
	uint32_t* m;       // photons found this iteration
	uint32_t* counts;  // per bucket
	uint32_t* offsets; // per bucket, exclusive prefix sum
	uint32_t* block_sums;
	uint32_t* entries;
	uint32_t capacity; // entries
	uint32_t* bounds;  // order keys: lo xyz, hi xyz, max radius; then the grid (sppm_grid) and the error word
	float* image;      // 3 per pixel
};
constexpr uint32_t kBoundWords = 7;
constexpr uint32_t kGridWords = 16;  // room for sppm_grid
constexpr uint32_t kErrorWord = kBoundWords + kGridWords;
constexpr uint32_t kStateWords = kErrorWord + 1;
constexpr uint32_t kMaxCellsPerAxis = 4;  // a sphere's box spans at most 3 cells (cells are >= the largest radius)

struct sppm_params {
	float r2c[16], c2w[16];
	float lens, focus;
	uint32_t width, height;
	uint32_t iteration, seed, max_depth;
	uint32_t photons;
	uint32_t stack_cap;
};

// Order-preserving keys of floats, so that atomicMin / atomicMax on the keys
// give the float minimum / maximum.
__device__ __forceinline__ uint32_t fkey(float f) {
	const uint32_t b = __float_as_uint(f);
	return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float funkey(uint32_t k) { return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k); }

__device__ __forceinline__ sppm_grid* grid_of(const sppm_buffers& b) { return reinterpret_cast<sppm_grid*>(b.bounds + kBoundWords); }

__global__ void k_sppm_init(sppm_buffers b, float radius) {
	for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < b.npix; i += gridDim.x * blockDim.x) {
		b.tau[i] = make_float4(0.f, 0.f, 0.f, 0.f);
		b.L[i] = make_float4(0.f, 0.f, 0.f, radius);
		b.phi[3 * i] = 0.f;
		b.phi[3 * i + 1] = 0.f;
		b.phi[3 * i + 2] = 0.f;
		b.m[i] = 0u;
	}
	if (blockIdx.x == 0 && threadIdx.x == 0) b.bounds[kErrorWord] = 0u;
}

// The bound starts as the reference's does: lo at the largest float, hi at
// the smallest positive normal float (numeric_limits<real>::min(), :213-214).
__global__ void k_sppm_begin(sppm_buffers b) {
	const uint32_t t = threadIdx.x;
	if (t < 3) b.bounds[t] = fkey(FLT_MAX);
	else if (t < 6) b.bounds[t] = fkey(FLT_MIN);
	else if (t == 6) b.bounds[t] = fkey(0.f);
}

template <bool INST>
__global__ void __launch_bounds__(128) k_sppm_visible(scene_view s, sppm_buffers b, sppm_params prm) {
	extern __shared__ uint32_t smem[];
	smem_stack stk = make_stack(smem, prm.stack_cap);
	float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {FLT_MIN, FLT_MIN, FLT_MIN}, rmax = 0.f;
	bool failed = false;
	for (uint32_t base = blockIdx.x * blockDim.x; base < b.npix; base += gridDim.x * blockDim.x) {
		const uint32_t i = base + threadIdx.x;
		if (i < b.npix) {
			const uint32_t x = i % prm.width, y = i / prm.width;
			path_state p;
			p.rng = pcg_seed(sppm_pixel_seed(i, prm.iteration, prm.seed));
			const ray_t r = camera_ray(prm.r2c, prm.c2w, prm.lens, prm.focus, x, y, p.rng);
			p.o = r.o;
			p.d = r.d;
			p.len = r.len;
			p.beta = splat3(1.f);
			p.L = splat3(0.f);
			p.eta = 1.f;
			p.flags = 0u;
			p.bounces = 0;
			p.medium = -1;
			visible_point vp;
			auto trace = [&](vec3 o, vec3 d, float& len, bool shadow) {
				return trace_out_of_line<INST>(s, o, d, len, shadow, stk, failed);
			};
			sppm_visible(s, p, prm.max_depth, trace, vp);
			float4 L = b.L[i];
			L.x += p.L.x;
			L.y += p.L.y;
			L.z += p.L.z;
			b.L[i] = L;
			b.vp_p[i] = make_float4(vp.p.x, vp.p.y, vp.p.z, vp.uv.y);
			b.vp_wo[i] = make_float4(vp.wo.x, vp.wo.y, vp.wo.z, __uint_as_float(vp.valid ? vp.material : 0xffffffffu));
			b.vp_beta[i] = make_float4(vp.beta.x, vp.beta.y, vp.beta.z, vp.uv.x);
			if (vp.valid) {
				const float rad = L.w;
				lo[0] = fminf(lo[0], vp.p.x - rad);
				lo[1] = fminf(lo[1], vp.p.y - rad);
				lo[2] = fminf(lo[2], vp.p.z - rad);
				hi[0] = fmaxf(hi[0], vp.p.x + rad);
				hi[1] = fmaxf(hi[1], vp.p.y + rad);
				hi[2] = fmaxf(hi[2], vp.p.z + rad);
				rmax = fmaxf(rmax, rad);
			}
		}
	}
	if (failed) atomicCAS(b.bounds + kErrorWord, 0u, static_cast<uint32_t>(RB_ERR_STACK_OVERFLOW));
	for (int o = 16; o > 0; o >>= 1) {
		for (int k = 0; k < 3; k++) {
			lo[k] = fminf(lo[k], __shfl_down_sync(0xffffffffu, lo[k], o));
			hi[k] = fmaxf(hi[k], __shfl_down_sync(0xffffffffu, hi[k], o));
		}
		rmax = fmaxf(rmax, __shfl_down_sync(0xffffffffu, rmax, o));
	}
	if ((threadIdx.x & 31u) == 0) {
		for (int k = 0; k < 3; k++) {
			atomicMin(b.bounds + k, fkey(lo[k]));
			atomicMax(b.bounds + 3 + k, fkey(hi[k]));
		}
		atomicMax(b.bounds + 6, fkey(rmax));
	}
}

// The grid from the bound (:209-241); pool 0: no visible point this iteration.
__global__ void k_sppm_grid(sppm_buffers b) {
	sppm_grid g;
	g.lo = vec3{funkey(b.bounds[0]), funkey(b.bounds[1]), funkey(b.bounds[2])};
	g.hi = vec3{funkey(b.bounds[3]), funkey(b.bounds[4]), funkey(b.bounds[5])};
	const float max_r = funkey(b.bounds[6]);
	g.pool = max_r > 0.f ? b.npix : 0u;
	g.nx = g.ny = g.nz = 1;
	if (g.pool) sppm_grid_size(g, max_r);
	*grid_of(b) = g;
}

// The cells of visible point i's sphere box (:254-272); false when its box is
// wider than kMaxCellsPerAxis cells along an axis (not reached: cells are at
// least the largest radius wide).
__device__ __forceinline__ bool sphere_cells(const sppm_grid& g, vec3 p, float r, int32_t* c0, int32_t* c1) {
	sppm_cell(g, p - splat3(r), c0[0], c0[1], c0[2]);
	sppm_cell(g, p + splat3(r), c1[0], c1[1], c1[2]);
	for (int k = 0; k < 3; k++)
		if (c1[k] - c0[k] + 1 > static_cast<int32_t>(kMaxCellsPerAxis)) return false;
	return true;
}

// pass 0: count the entries per bucket; pass 1: write them at the bucket's
// offset (counts reset to 0 in between serve as cursors).
template <int PASS>
__global__ void k_sppm_cells(sppm_buffers b) {
	const sppm_grid g = *grid_of(b);
	if (g.pool == 0u) return;
	for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < b.npix; i += gridDim.x * blockDim.x) {
		const float4 wo = b.vp_wo[i];
		if (__float_as_uint(wo.w) == 0xffffffffu) continue;
		const float4 pp = b.vp_p[i];
		int32_t c0[3], c1[3];
		if (!sphere_cells(g, vec3{pp.x, pp.y, pp.z}, b.L[i].w, c0, c1)) {
			atomicCAS(b.bounds + kErrorWord, 0u, static_cast<uint32_t>(RB_ERR_QUEUE_OVERFLOW));
			continue;
		}
		for (int32_t z = c0[2]; z <= c1[2]; z++)
			for (int32_t y = c0[1]; y <= c1[1]; y++)
				for (int32_t x = c0[0]; x <= c1[0]; x++) {
					const uint32_t k = sppm_bucket(g, x, y, z);
					if (PASS == 0) {
						atomicAdd(b.counts + k, 1u);
					} else {
						const uint32_t at = b.offsets[k] + atomicAdd(b.counts + k, 1u);
						if (at < b.capacity) b.entries[at] = i;
						else atomicCAS(b.bounds + kErrorWord, 0u, static_cast<uint32_t>(RB_ERR_QUEUE_OVERFLOW));
					}
				}
	}
}

// Exclusive prefix sum of n words, in blocks of 1024 (one word per thread):
// each block scans its words and writes its total, one block scans the totals,
// then every block adds its total's prefix.
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t& total) {
	__shared__ uint32_t warp_sums[32];
	const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
	uint32_t incl = v;
	for (int o = 1; o < 32; o <<= 1) {
		const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
		if (lane >= static_cast<uint32_t>(o)) incl += t;
	}
	if (lane == 31u) warp_sums[warp] = incl;
	__syncthreads();
	if (warp == 0) {
		const uint32_t nw = blockDim.x >> 5;
		uint32_t w = lane < nw ? warp_sums[lane] : 0u;
		for (int o = 1; o < 32; o <<= 1) {
			const uint32_t t = __shfl_up_sync(0xffffffffu, w, o);
			if (lane >= static_cast<uint32_t>(o)) w += t;
		}
		if (lane < nw) warp_sums[lane] = w;
	}
	__syncthreads();
	const uint32_t before = warp == 0 ? 0u : warp_sums[warp - 1];
	total = warp_sums[(blockDim.x >> 5) - 1];
	__syncthreads();
	return before + incl - v;
}

__global__ void __launch_bounds__(1024) k_scan_blocks(const uint32_t* in, uint32_t* out, uint32_t* block_sums, uint32_t n) {
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	uint32_t total;
	const uint32_t e = block_exclusive_scan(i < n ? in[i] : 0u, total);
	if (i < n) out[i] = e;
	if (threadIdx.x == 0) block_sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(1024) k_scan_sums(uint32_t* block_sums, uint32_t nblocks) {
	uint32_t carry = 0;
	for (uint32_t base = 0; base < nblocks; base += blockDim.x) {
		const uint32_t i = base + threadIdx.x;
		uint32_t total;
		const uint32_t e = block_exclusive_scan(i < nblocks ? block_sums[i] : 0u, total);
		if (i < nblocks) block_sums[i] = e + carry;
		carry += total;
	}
}

__global__ void __launch_bounds__(1024) k_scan_add(uint32_t* out, const uint32_t* block_sums, uint32_t n) {
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) out[i] += block_sums[blockIdx.x];
}

template <bool INST>
__global__ void __launch_bounds__(128) k_sppm_photons(scene_view s, sppm_buffers b, sppm_params prm) {
	extern __shared__ uint32_t smem[];
	smem_stack stk = make_stack(smem, prm.stack_cap);
	const sppm_grid g = *grid_of(b);
	if (g.pool == 0u) return;
	bool failed = false;
	for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < prm.photons; j += gridDim.x * blockDim.x) {
		pcg32 rng = pcg_seed(sppm_photon_seed(j, prm.iteration, prm.seed));
		auto trace = [&](vec3 o, vec3 d, float& len, bool shadow) {
			return trace_out_of_line<INST>(s, o, d, len, shadow, stk, failed);
		};
		// add_photon (:282-324)
		auto deposit = [&](const surface_t& si, const spectrum& beta, vec3 d) {
			if (!sppm_inside(g, si.p)) return;
			int32_t x, y, z;
			sppm_cell(g, si.p, x, y, z);
			const uint32_t k = sppm_bucket(g, x, y, z);
			const uint32_t first = b.offsets[k], last = first + b.counts[k];
			for (uint32_t e = first; e < last && e < b.capacity; e++) {
				const uint32_t i = b.entries[e];
				const float4 pp = b.vp_p[i], wo = b.vp_wo[i], bt = b.vp_beta[i];
				visible_point vp;
				vp.p = vec3{pp.x, pp.y, pp.z};
				vp.wo = vec3{wo.x, wo.y, wo.z};
				vp.beta = vec3{bt.x, bt.y, bt.z};
				vp.material = __float_as_uint(wo.w);
				vp.uv = vec2{bt.w, pp.w};
				vp.valid = 1u;
				spectrum flux;
				if (!sppm_flux(s, si, beta, d, vp, b.L[i].w, flux)) continue;
				atomicAdd(b.phi + 3 * i, flux.x);
				atomicAdd(b.phi + 3 * i + 1, flux.y);
				atomicAdd(b.phi + 3 * i + 2, flux.z);
				atomicAdd(b.m + i, 1u);
			}
		};
		sppm_photon(s, rng, prm.max_depth, trace, deposit);
	}
	if (failed) atomicCAS(b.bounds + kErrorWord, 0u, static_cast<uint32_t>(RB_ERR_STACK_OVERFLOW));
}

__global__ void k_sppm_update(sppm_buffers b) {
	for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < b.npix; i += gridDim.x * blockDim.x) {
		const uint32_t m = b.m[i];
		if (m == 0u) continue;
		const float4 t = b.tau[i], L = b.L[i], bt = b.vp_beta[i];
		sppm_pixel px;
		px.tau = vec3{t.x, t.y, t.z};
		px.n = t.w;
		px.L = vec3{L.x, L.y, L.z};
		px.radius = L.w;
		const spectrum phi{b.phi[3 * i], b.phi[3 * i + 1], b.phi[3 * i + 2]};
		sppm_update(px, vec3{bt.x, bt.y, bt.z}, phi, m);
		b.tau[i] = make_float4(px.tau.x, px.tau.y, px.tau.z, px.n);
		b.L[i].w = px.radius;
		b.phi[3 * i] = 0.f;
		b.phi[3 * i + 1] = 0.f;
		b.phi[3 * i + 2] = 0.f;
		b.m[i] = 0u;
	}
}

__global__ void k_sppm_image(sppm_buffers b, uint32_t iterations, uint64_t photons) {
	for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < b.npix; i += gridDim.x * blockDim.x) {
		const float4 t = b.tau[i], L = b.L[i];
		sppm_pixel px;
		px.tau = vec3{t.x, t.y, t.z};
		px.n = t.w;
		px.L = vec3{L.x, L.y, L.z};
		px.radius = L.w;
		const spectrum v = sppm_value(px, iterations, photons);
		b.image[3 * i] = v.x;
		b.image[3 * i + 1] = v.y;
		b.image[3 * i + 2] = v.z;
	}
}

template <typename Kernel>
cudaError_t allow_stack_smem(Kernel kernel, size_t bytes) {
	if (bytes <= 48u * 1024u) return cudaSuccess;
	return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes));
}

// One iteration's launches.
template <bool INST>
cudaError_t sppm_iteration(const scene_view& s, const sppm_buffers& b, const sppm_params& prm, int grid, cudaStream_t st) {
	const size_t smem = 2 * static_cast<size_t>(prm.stack_cap) * 128 * sizeof(uint32_t);
	cudaError_t e = allow_stack_smem(k_sppm_visible<INST>, smem);
	if (e == cudaSuccess) e = allow_stack_smem(k_sppm_photons<INST>, smem);
	if (e != cudaSuccess) return e;
	const uint32_t scan_blocks = (b.npix + 1023) / 1024;
	k_sppm_begin<<<1, 32, 0, st>>>(b);
	k_sppm_visible<INST><<<grid, 128, smem, st>>>(s, b, prm);
	k_sppm_grid<<<1, 1, 0, st>>>(b);
	e = cudaMemsetAsync(b.counts, 0, b.npix * sizeof(uint32_t), st);
	if (e != cudaSuccess) return e;
	k_sppm_cells<0><<<grid, 256, 0, st>>>(b);
	k_scan_blocks<<<scan_blocks, 1024, 0, st>>>(b.counts, b.offsets, b.block_sums, b.npix);
	k_scan_sums<<<1, 1024, 0, st>>>(b.block_sums, scan_blocks);
	k_scan_add<<<scan_blocks, 1024, 0, st>>>(b.offsets, b.block_sums, b.npix);
	e = cudaMemsetAsync(b.counts, 0, b.npix * sizeof(uint32_t), st);
	if (e != cudaSuccess) return e;
	k_sppm_cells<1><<<grid, 256, 0, st>>>(b);
	k_sppm_photons<INST><<<grid, 128, smem, st>>>(s, b, prm);
	k_sppm_update<<<grid, 256, 0, st>>>(b);
	return cudaGetLastError();
}

} // namespace
} // namespace gpu
} // namespace rb

extern "C" rb_status rb_render_photons(rb_context* c, const rb_photon_params* prm, float* rgb_out) {
	using namespace rb;
	using namespace rb::gpu;
	if (c == nullptr || prm == nullptr || rgb_out == nullptr) return RB_ERR_INVALID_ARGUMENT;
	const rb_camera_desc& cam = prm->camera;
	if (cam.width <= 0 || cam.height <= 0 || prm->iterations == 0 || prm->max_depth == 0 || prm->max_depth > 64 ||
		!(prm->radius > 0.f) || prm->iterations > 0xffffu)
		return RB_ERR_INVALID_ARGUMENT;
	const uint64_t npix64 = static_cast<uint64_t>(cam.width) * static_cast<uint64_t>(cam.height);
	if (npix64 > (1u << 24)) return RB_ERR_INVALID_ARGUMENT;
	const uint32_t npix = static_cast<uint32_t>(npix64);
	const uint32_t photons = prm->photons == 0 ? npix : prm->photons;
	pt::scene_view view;
	launch_cfg cfg;
	cudaStream_t st;
	int device;
	uint32_t* counters_host;
	bool has_invisible;
	if (!context_view(c, &view, &cfg, &st, &device, &counters_host, &has_invisible)) return RB_ERR_NO_SCENE;
	if (cudaSetDevice(device) != cudaSuccess) return RB_ERR_CUDA;
	sppm_buffers b{};
	b.npix = npix;
	b.width = static_cast<uint32_t>(cam.width);
	const uint32_t scan_blocks = (npix + 1023) / 1024;
	b.capacity = 27u * npix;
	// one allocation, carved up (256-byte aligned pieces)
	size_t off = 0;
	const auto take = [&](size_t bytes) {
		const size_t at = off;
		off += (bytes + 255) & ~static_cast<size_t>(255);
		return at;
	};
	const size_t o_p = take(16ull * npix), o_wo = take(16ull * npix), o_beta = take(16ull * npix), o_tau = take(16ull * npix),
		o_L = take(16ull * npix), o_phi = take(12ull * npix), o_m = take(4ull * npix), o_counts = take(4ull * npix),
		o_offsets = take(4ull * npix), o_sums = take(4ull * scan_blocks), o_entries = take(4ull * b.capacity),
		o_bounds = take(4ull * kStateWords), o_image = take(12ull * npix);
	unsigned char* base = nullptr;
	if (cudaMalloc(&base, off) != cudaSuccess) return RB_ERR_OUT_OF_MEMORY;
	b.vp_p = reinterpret_cast<float4*>(base + o_p);
	b.vp_wo = reinterpret_cast<float4*>(base + o_wo);
	b.vp_beta = reinterpret_cast<float4*>(base + o_beta);
	b.tau = reinterpret_cast<float4*>(base + o_tau);
	b.L = reinterpret_cast<float4*>(base + o_L);
	b.phi = reinterpret_cast<float*>(base + o_phi);
	b.m = reinterpret_cast<uint32_t*>(base + o_m);
	b.counts = reinterpret_cast<uint32_t*>(base + o_counts);
	b.offsets = reinterpret_cast<uint32_t*>(base + o_offsets);
	b.block_sums = reinterpret_cast<uint32_t*>(base + o_sums);
	b.entries = reinterpret_cast<uint32_t*>(base + o_entries);
	b.bounds = reinterpret_cast<uint32_t*>(base + o_bounds);
	b.image = reinterpret_cast<float*>(base + o_image);
	sppm_params p{};
	std::memcpy(p.r2c, cam.raster_to_camera, sizeof(p.r2c));
	std::memcpy(p.c2w, cam.camera_to_world, sizeof(p.c2w));
	p.lens = cam.lens_radius;
	p.focus = cam.focus_distance;
	p.width = static_cast<uint32_t>(cam.width);
	p.height = static_cast<uint32_t>(cam.height);
	p.seed = prm->seed;
	p.max_depth = prm->max_depth;
	p.photons = photons;
	p.stack_cap = static_cast<uint32_t>(cfg.stack_depth);
	const int grid = cfg.grid_shade > 0 ? cfg.grid_shade : 148 * 8;
	k_sppm_init<<<grid, 256, 0, st>>>(b, prm->radius);
	cudaError_t e = cudaGetLastError();
	for (uint32_t it = 0; it < prm->iterations && e == cudaSuccess; it++) {
		p.iteration = it;
		e = view.instances ? sppm_iteration<true>(view, b, p, grid, st) : sppm_iteration<false>(view, b, p, grid, st);
	}
	if (e == cudaSuccess) {
		k_sppm_image<<<grid, 256, 0, st>>>(b, prm->iterations, photons);
		e = cudaGetLastError();
	}
	uint32_t err = 0;
	if (e == cudaSuccess) e = cudaMemcpyAsync(rgb_out, b.image, 12ull * npix, cudaMemcpyDeviceToHost, st);
	if (e == cudaSuccess) e = cudaMemcpyAsync(&err, b.bounds + kErrorWord, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
	if (e == cudaSuccess) e = cudaStreamSynchronize(st);
	cudaFree(base);
	if (e != cudaSuccess) return RB_ERR_CUDA;
	return static_cast<rb_status>(err);
}
