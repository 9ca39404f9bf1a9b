// Tensor-core kernels of the learned path guide (sm_100a): the network's
// forward pass (inference for the path queue, raw outputs for tests), one
// fused forward + backward training kernel, the gradient reduction + Adam
// step, and the wave-end collection of training samples.
//
// Every layer is a 128-row tile product on tcgen05: operands in shared memory
// in the no-swizzle core-matrix layout (see umma.cuh), the FP32 accumulator in
// tensor memory, issued by one thread and completed through an mbarrier that
// every waiting thread polls with a wall-time bound. Epilogues run one thread
// per row (TMEM lane), so a CTA's 128 threads own the tile's 128 rows.
//
// Training kernel, per 128-row tile and all in one CTA:
//   forward:  X1 = relu(X0 W1^T) ... X4 = relu(X3 W4^T), O = X4 W5^T     (K-major x K-major)
//   output:   G = dL/dO per row (thread per row, FP32, stored BF16)
//   backward: dW5^T += X4^T G (accumulated in TMEM across tiles),          (MN-major x MN-major)
//             dX4 = G W5 (the same weight tile read MN-major), G = dX4 * [X4 > 0], ... down to dW1^T += X0^T G.
// Biases are weight columns against a constant-1 feature, so their gradient
// comes out of the same products. Per-CTA gradients go to a partial buffer
// that the Adam kernel sums in a fixed order (deterministic).
#include "guide_host.h"
#include "umma.cuh"

#include <cuda_bf16.h>

#include <cstddef>

namespace rb {
namespace guide {
namespace {

constexpr uint64_t kWaitNs = 2000000000ull;                        // bound of every device wait (2 s)
constexpr uint32_t kActBytes = kTileRows * kK1 * 2;                // 57,344: encoded input tile
constexpr uint32_t kHidBytes = kTileRows * kHiddenK * 2;           // 20,480: hidden activation tile
constexpr uint32_t kSigBytes = kTileRows * kHidden * 2;            // 16,384: back-propagated signal tile
constexpr uint32_t kSboIn = kK1 * 16;                              // 8-row group stride, encoded tile
constexpr uint32_t kSboHid = kHiddenK * 16;                        // 8-row group stride, hidden tile
constexpr uint32_t kCopyChunk = kImageBytes / 4;                   // 16,768 bytes per bulk copy
static_assert(kCopyChunk % 16 == 0, "bulk copies move multiples of 16 bytes");

// Forward kernel: four warpgroups per CTA, each with its own 32 KB tile. The
// encoded input (224 features) goes through layer 1 in two K parts that take
// turns in that tile: inputs 0..3 (features 0..95, 6 K-steps), then inputs
// 4..8 and the bias chunk (features 96..223, 8 K-steps). The hidden tiles
// (80 features, 20 KB) reuse it.
constexpr uint32_t kFwdGroups = 4;
constexpr int kPartAInputs = 4;
constexpr uint32_t kPartAChunks = 3 * kPartAInputs;                 // 12 chunks of 8 features
constexpr uint32_t kPartBChunks = 3 * (kInputs - kPartAInputs) + 1; // 16 (with the bias chunk)
constexpr uint32_t kSboPartA = kPartAChunks * 128;
constexpr uint32_t kSboPartB = kPartBChunks * 128;
constexpr uint32_t kFwdTile = kTileRows / 8 * kSboPartB;           // 32,768
static_assert(kPartAChunks % 2 == 0 && kPartBChunks % 2 == 0, "each part is whole K-steps of 16 features");
static_assert(kPartAChunks + kPartBChunks == kK1 / 8, "the two parts cover the encoded input");
static_assert(kFwdTile >= kTileRows / 8 * kSboPartA && kFwdTile >= kHidBytes, "the tile holds every operand");
constexpr uint32_t kFwdAct = kImageBytes;
constexpr uint32_t kFwdBars = kFwdAct + kFwdGroups * kFwdTile;
constexpr uint32_t kFwdSmem = kFwdBars + 128 + 128;
static_assert(kFwdSmem <= 232448, "forward kernel exceeds 227 KB of shared memory");
// training kernel: weight image, X0, X1..X4, signal tile, barriers. A weight-
// gradient product reads 128 feature rows of an activation tile, past the end
// of the 80 (or 224) stored ones; those extra rows land in the next buffer and
// only produce TMEM lanes that are never read.
constexpr uint32_t kTrX0 = kImageBytes;
constexpr uint32_t kTrX1 = kTrX0 + kActBytes;
constexpr uint32_t kTrSig = kTrX1 + 4 * kHidBytes;
constexpr uint32_t kTrBars = kTrSig + kSigBytes;
constexpr uint32_t kTrSmem = kTrBars + 64 + 128;
static_assert(kTrSmem <= 232448, "training kernel exceeds 227 KB of shared memory");
static_assert(kImageBytes % 128 == 0 && kActBytes % 128 == 0 && kHidBytes % 128 == 0, "128-byte aligned tiles");

// TMEM columns of the training kernel
constexpr uint32_t kColS = 0;      // layer outputs / back-propagated activations (80 columns)
// dW^T of layer l (0-based) at col_w(l); col_w(kLayers): features 128..255 of layer 1
__device__ __forceinline__ uint32_t col_w(int r) {
	return r == 0 ? 128u : r == kLayers ? 192u : 256u + 64u * static_cast<uint32_t>(r - 1);
}

__device__ __forceinline__ uint8_t* align128(uint8_t* p) {
	return reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(p) + 127u) & ~static_cast<uintptr_t>(127u));
}

__device__ __forceinline__ uint32_t pack2(float a, float b) {
	const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
	return *reinterpret_cast<const uint32_t*>(&h);
}

__device__ __forceinline__ float relu(float z) { return z > 0.f ? z : 0.f; }

__device__ __forceinline__ void set_error(uint32_t* e, uint32_t code) { atomicCAS(e, 0u, code); }

// MurmurHash3's 32-bit finaliser.
__device__ __forceinline__ uint32_t mix32(uint32_t h) {
	h ^= h >> 16; h *= 0x85ebca6bu; h ^= h >> 13; h *= 0xc2b2ae35u; h ^= h >> 16;
	return h;
}

// Inputs J0..J1-1 of one row of an encoded tile, from `base` (the row's first
// core-matrix line): 3 chunks of 8 features (4 sin/cos pairs) per input.
// sin/cos(2^k pi x) by the double-angle recurrence, restarted exactly at k = 4
// and k = 8 so that the error stays near 1e-6.
template <int J0, int J1>
__device__ __forceinline__ void encode_inputs(const float (&x)[kInputs], uint8_t* base) {
#pragma unroll
	for (int j = J0; j < J1; j++) {
		float s[kFreqs], c[kFreqs];
		sincospif(x[j], &s[0], &c[0]);
#pragma unroll
		for (int k = 1; k < kFreqs; k++) {
			if (k == 4 || k == 8) {
				sincospif(fmodf(x[j] * static_cast<float>(1 << k), 2.f), &s[k], &c[k]);
			} else {
				s[k] = 2.f * s[k - 1] * c[k - 1];
				c[k] = 1.f - 2.f * s[k - 1] * s[k - 1];
			}
		}
#pragma unroll
		for (int q = 0; q < 3; q++) {
			uint4 v;
			v.x = pack2(s[4 * q], c[4 * q]);
			v.y = pack2(s[4 * q + 1], c[4 * q + 1]);
			v.z = pack2(s[4 * q + 2], c[4 * q + 2]);
			v.w = pack2(s[4 * q + 3], c[4 * q + 3]);
			*reinterpret_cast<uint4*>(base + (3 * (j - J0) + q) * 128) = v;
		}
	}
}

// Row `row` of an encoded tile (K = 224): 27 chunks of 8 features, then the
// constant-1 bias feature and 7 zeros.
__device__ __forceinline__ void encode_row(const float (&x)[kInputs], uint8_t* tile, uint32_t row) {
	uint8_t* base = tile + (row >> 3) * kSboIn + (row & 7u) * 16u;
	encode_inputs<0, kInputs>(x, base);
	*reinterpret_cast<uint4*>(base + 27 * 128) = make_uint4(pack2(1.f, 0.f), 0u, 0u, 0u);
}

// Four of the eight value chunks of a hidden-tile row (chunks c0 .. c0 + 3: the
// relu of 32 values); with c0 == 4 also the constant-1 chunk and the zero chunk.
__device__ __forceinline__ void store_hidden_half(uint8_t* tile, uint32_t row, const float* v, int c0) {
	uint8_t* base = tile + (row >> 3) * kSboHid + (row & 7u) * 16u;
#pragma unroll
	for (int c = 0; c < 4; c++) {
		uint4 u;
		u.x = pack2(relu(v[8 * c]), relu(v[8 * c + 1]));
		u.y = pack2(relu(v[8 * c + 2]), relu(v[8 * c + 3]));
		u.z = pack2(relu(v[8 * c + 4]), relu(v[8 * c + 5]));
		u.w = pack2(relu(v[8 * c + 6]), relu(v[8 * c + 7]));
		*reinterpret_cast<uint4*>(base + (c0 + c) * 128) = u;
	}
	if (c0 == 4) {
		*reinterpret_cast<uint4*>(base + 8 * 128) = make_uint4(pack2(1.f, 0.f), 0u, 0u, 0u);
		*reinterpret_cast<uint4*>(base + 9 * 128) = make_uint4(0u, 0u, 0u, 0u);
	}
}

// Row of a hidden tile (K = 80): relu of 64 values, the constant 1, 15 zeros.
__device__ __forceinline__ void store_hidden_row(uint8_t* tile, uint32_t row, const float* v) {
	uint8_t* base = tile + (row >> 3) * kSboHid + (row & 7u) * 16u;
#pragma unroll
	for (int c = 0; c < 8; c++) {
		uint4 u;
		u.x = pack2(relu(v[8 * c]), relu(v[8 * c + 1]));
		u.y = pack2(relu(v[8 * c + 2]), relu(v[8 * c + 3]));
		u.z = pack2(relu(v[8 * c + 4]), relu(v[8 * c + 5]));
		u.w = pack2(relu(v[8 * c + 6]), relu(v[8 * c + 7]));
		*reinterpret_cast<uint4*>(base + c * 128) = u;
	}
	*reinterpret_cast<uint4*>(base + 8 * 128) = make_uint4(pack2(1.f, 0.f), 0u, 0u, 0u);
	*reinterpret_cast<uint4*>(base + 9 * 128) = make_uint4(0u, 0u, 0u, 0u);
}

// Row of a signal tile with N columns (K-major for the activation-gradient
// product, MN-major for the weight-gradient product).
template <int N>
__device__ __forceinline__ void store_signal_row(uint8_t* tile, uint32_t row, const float* v) {
	uint8_t* base = tile + (row >> 3) * (N * 16) + (row & 7u) * 16u;
#pragma unroll
	for (int c = 0; c < N / 8; c++) {
		uint4 u;
		u.x = pack2(v[8 * c], v[8 * c + 1]);
		u.y = pack2(v[8 * c + 2], v[8 * c + 3]);
		u.z = pack2(v[8 * c + 4], v[8 * c + 5]);
		u.w = pack2(v[8 * c + 6], v[8 * c + 7]);
		*reinterpret_cast<uint4*>(base + c * 128) = u;
	}
}

// v[c] = 0 where the stored activation of this row is not positive (relu').
__device__ __forceinline__ void relu_mask(const uint8_t* tile, uint32_t row, float* v) {
	const uint8_t* base = tile + (row >> 3) * kSboHid + (row & 7u) * 16u;
#pragma unroll
	for (int c = 0; c < 8; c++) {
		const uint4 u = *reinterpret_cast<const uint4*>(base + c * 128);
		const uint32_t w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
		for (int e = 0; e < 4; e++) {
			const uint32_t lo = w[e] & 0xffffu, hi = w[e] >> 16;
			if (lo == 0u || (lo & 0x8000u)) v[8 * c + 2 * e] = 0.f;
			if (hi == 0u || (hi & 0x8000u)) v[8 * c + 2 * e + 1] = 0.f;
		}
	}
}

// ---------------------------------------------------------------- MMA issue (one thread)
// D[128 x n] (+)= A[128 x K] B[n x K]^T, both K-major, K = 16 * ksteps.
__device__ __forceinline__ void mma_kk(uint32_t d, uint32_t a, uint32_t a_sbo, uint32_t b, uint32_t b_sbo, uint32_t n,
	uint32_t ksteps, bool accumulate = false) {
	const uint32_t id = idesc_bf16(128, n, false, false);
	for (uint32_t ks = 0; ks < ksteps; ks++)
		umma_bf16(d, sdesc(a + ks * 256u, 128u, a_sbo), sdesc(b + ks * 256u, 128u, b_sbo), id,
			(accumulate || ks > 0) ? 1u : 0u);
}
// D[128 x n] = A[128 x K] (K-major) B[K x n] with B MN-major (8-row K groups b_lbo apart).
__device__ __forceinline__ void mma_km(uint32_t d, uint32_t a, uint32_t a_sbo, uint32_t b, uint32_t b_lbo, uint32_t n,
	uint32_t ksteps) {
	const uint32_t id = idesc_bf16(128, n, false, true);
	for (uint32_t ks = 0; ks < ksteps; ks++)
		umma_bf16(d, sdesc(a + ks * 256u, 128u, a_sbo), sdesc(b + ks * 2u * b_lbo, b_lbo, 128u), id, ks > 0 ? 1u : 0u);
}
// D[128 x n] (+)= A^T B over the tile's 128 rows: A MN-major (128 features,
// row groups a_lbo apart), B MN-major (n columns, row groups b_lbo apart).
__device__ __forceinline__ void mma_mm(uint32_t d, uint32_t a, uint32_t a_lbo, uint32_t b, uint32_t b_lbo, uint32_t n,
	bool accumulate) {
	const uint32_t id = idesc_bf16(128, n, true, true);
	for (uint32_t ks = 0; ks < kTileRows / 16; ks++)
		umma_bf16(d, sdesc(a + ks * 2u * a_lbo, a_lbo, 128u), sdesc(b + ks * 2u * b_lbo, b_lbo, 128u), id,
			(accumulate || ks > 0) ? 1u : 0u);
}

// Bounded wait on an MMA barrier by every thread of a warpgroup, with a
// uniform outcome: false if any thread gave up.
__device__ __forceinline__ bool group_wait(uint64_t* bar, uint32_t& phase, volatile uint32_t* fail, uint32_t barrier_id) {
	const bool ok = mbar_wait(bar, phase, kWaitNs);
	if (!ok) *fail = 1u;
	named_barrier(barrier_id, 128);
	if (*fail != 0u) return false;
	phase ^= 1u;
	tc_fence_after();
	return true;
}

// Hands the tile just written by this warpgroup to the MMA issuer.
__device__ __forceinline__ void publish(uint32_t barrier_id) {
	fence_proxy_async_smem();
	tc_fence_before();
	named_barrier(barrier_id, 128);
}

// Shared start: TMEM allocation by warp 0, barrier set-up, weight image by bulk copy.
__device__ __forceinline__ bool kernel_begin(uint8_t* img, const uint8_t* image, uint64_t* bars, uint32_t nbars,
	uint32_t* tptr, volatile uint32_t* fail, uint32_t nfail, uint32_t ncols, uint32_t* error) {
	const uint32_t tid = threadIdx.x;
	if ((tid >> 5) == 0) {
		tmem_alloc(tptr, ncols);
		tmem_relinquish();
	}
	if (tid == 0) {
		for (uint32_t i = 0; i < nbars; i++) mbar_init(&bars[i], 1);
		for (uint32_t i = 0; i < nfail; i++) fail[i] = 0u;
		fence_mbar_init();
	}
	tc_fence_before();
	__syncthreads();
	tc_fence_after();
	if (tid == 0) {
		mbar_arrive_expect_tx(&bars[0], kImageBytes);
		for (uint32_t c = 0; c < 4; c++) bulk_g2s(img + c * kCopyChunk, image + c * kCopyChunk, kCopyChunk, &bars[0]);
	}
	const bool ok = __syncthreads_and(mbar_wait(&bars[0], 0, kWaitNs) ? 1 : 0) != 0;
	if (!ok) {
		if (tid == 0) set_error(error, RB_ERR_DEVICE_TIMEOUT);
		mbar_wait(&bars[0], 0, kWaitNs);  // let the copy in flight land before the CTA exits
	}
	return ok;
}

__device__ __forceinline__ void kernel_end(uint32_t tmem, uint32_t ncols) {
	tc_fence_before();
	__syncthreads();
	tc_fence_after();
	if ((threadIdx.x >> 5) == 0) tmem_dealloc(tmem, ncols);
}

// ---------------------------------------------------------------- forward
struct fwd_args {
	const uint8_t* image;
	uint32_t n;                 // rows (raw mode)
	const uint32_t* count;      // rows (queue mode)
	const float* x;             // raw mode: n x 9 inputs
	float* out;                 // raw mode: n x 48 raw outputs
	const uint32_t* queue;      // queue mode: path of each row
	const float4* in4;          // queue mode: 3 float4 of inputs per path
	float4* out4;               // queue mode: 12 float4 of decoded guide per path
	uint32_t* error;
};

// Four warpgroups per CTA, each running its own tiles through the 5 layers
// (TMEM columns 64 g .. 64 g + 63), sharing the weight image.
template <bool QUEUE>
__global__ void __launch_bounds__(kFwdGroups * 128, 1) k_forward(fwd_args a) {
	extern __shared__ uint8_t smem_raw[];
	uint8_t* sm = align128(smem_raw);
	const uint32_t tid = threadIdx.x, grp = tid >> 7, t = tid & 127u, warp = tid >> 5;
	uint8_t* img = sm;
	uint8_t* act = sm + kFwdAct + grp * kFwdTile;
	uint64_t* bars = reinterpret_cast<uint64_t*>(sm + kFwdBars);                       // 1 + kFwdGroups
	uint32_t* tptr = reinterpret_cast<uint32_t*>(sm + kFwdBars + 64);
	volatile uint32_t* fail = reinterpret_cast<volatile uint32_t*>(sm + kFwdBars + 80); // kFwdGroups
	const bool loaded = kernel_begin(img, a.image, bars, 1 + kFwdGroups, tptr, fail, kFwdGroups, kFwdGroups * 64, a.error);
	const uint32_t tmem = *tptr;
	if (loaded) {
		const uint32_t n = QUEUE ? *a.count : a.n;
		const uint32_t tiles = (n + kTileRows - 1) / kTileRows;
		const uint32_t dcol = tmem + grp * 64u;
		const uint32_t lane = dcol + ((32u * (warp & 3u)) << 16);
		const uint32_t bid = 1u + grp;
		uint64_t* bar = &bars[1 + grp];
		uint32_t phase = 0;
		const uint32_t act_s = smem_u32(act), img_s = smem_u32(img);
		uint8_t* base_a = act + (t >> 3) * kSboPartA + (t & 7u) * 16u;
		uint8_t* base_b = act + (t >> 3) * kSboPartB + (t & 7u) * 16u;
		bool failed = false;
		for (uint32_t tile = blockIdx.x * kFwdGroups + grp; tile < tiles; tile += gridDim.x * kFwdGroups) {
			const uint32_t row = tile * kTileRows + t;
			const bool valid = row < n;
			uint32_t path = 0;
			float x[kInputs];
#pragma unroll
			for (int j = 0; j < kInputs; j++) x[j] = 0.f;
			if (valid) {
				if (QUEUE) {
					path = a.queue[row];
					const float4 p0 = a.in4[3 * path], p1 = a.in4[3 * path + 1], p2 = a.in4[3 * path + 2];
					x[0] = p0.x; x[1] = p0.y; x[2] = p0.z; x[3] = p0.w;
					x[4] = p1.x; x[5] = p1.y; x[6] = p1.z; x[7] = p1.w; x[8] = p2.x;
				} else {
#pragma unroll
					for (int j = 0; j < kInputs; j++) x[j] = a.x[static_cast<size_t>(row) * kInputs + j];
				}
			}
			// layer 1, first K part
			encode_inputs<0, kPartAInputs>(x, base_a);
			publish(bid);
			if (t == 0) {
				tc_fence_after();
				mma_kk(dcol, act_s, kSboPartA, img_s, kSboIn, kHidden, kPartAChunks / 2);
				umma_commit(bar);
			}
			if (!group_wait(bar, phase, fail + grp, bid)) { failed = true; break; }
			// layer 1, second K part (accumulating), in the same tile
			encode_inputs<kPartAInputs, kInputs>(x, base_b);
			*reinterpret_cast<uint4*>(base_b + (kPartBChunks - 1) * 128) = make_uint4(pack2(1.f, 0.f), 0u, 0u, 0u);
			publish(bid);
			if (t == 0) {
				tc_fence_after();
				mma_kk(dcol, act_s, kSboPartB, img_s + kPartAChunks * 128u, kSboIn, kHidden, kPartBChunks / 2, true);
				umma_commit(bar);
			}
			if (!group_wait(bar, phase, fail + grp, bid)) { failed = true; break; }
#pragma unroll 1
			for (int l = 1; l < kLayers; l++) {
				float v[32];
				tmem_ld32(lane, v);
				store_hidden_half(act, t, v, 0);
				tmem_ld32(lane + 32u, v);
				store_hidden_half(act, t, v, 4);
				publish(bid);
				if (t == 0) {
					tc_fence_after();
					mma_kk(dcol, act_s, kSboHid, img_s + 2u * aug_offset(l), kSboHid, layer_out(l), kHiddenK / 16);
					umma_commit(bar);
				}
				if (!group_wait(bar, phase, fail + grp, bid)) { failed = true; break; }
			}
			if (failed) break;
			float v[kOutputs];
			tmem_ld32(lane, v);
			tmem_ld16(lane + 32u, v + 32);
			if (valid) {
				if (QUEUE) {
					float g[kOutputs];
					decode_outputs(v, g);
					float4* o = a.out4 + 12u * path;
#pragma unroll
					for (int c = 0; c < 12; c++) o[c] = make_float4(g[4 * c], g[4 * c + 1], g[4 * c + 2], g[4 * c + 3]);
				} else {
					float4* o = reinterpret_cast<float4*>(a.out + static_cast<size_t>(row) * kOutputs);
#pragma unroll
					for (int c = 0; c < 12; c++) o[c] = make_float4(v[4 * c], v[4 * c + 1], v[4 * c + 2], v[4 * c + 3]);
				}
			}
		}
		if (failed) {
			if (t == 0) set_error(a.error, RB_ERR_DEVICE_TIMEOUT);
			mbar_wait(bar, phase, kWaitNs);  // the MMAs in flight finish before TMEM is released
		}
	}
	kernel_end(tmem, kFwdGroups * 64);
}

// ---------------------------------------------------------------- training
struct train_args {
	const uint8_t* image;
	const float4* samples;      // kSampleFloat4 per sample
	const uint32_t* count;      // samples stored (may exceed count_cap)
	uint32_t count_cap;
	uint32_t batch;
	uint32_t min_rows;
	uint32_t sequential;
	uint32_t budgeted;
	float weight_clip;          // > 0: weights clipped at weight_clip * state->weight_mean
	const device_state* state;
	float* partial;             // [gridDim.x][kAugParams]
	float* partial_loss;        // [gridDim.x]
	uint32_t* error;
};

__device__ __forceinline__ uint32_t step_rows(uint32_t count, uint32_t batch, uint32_t min_rows) {
	return count < min_rows || count == 0u ? 0u : (count < batch ? count : batch);
}

__global__ void __launch_bounds__(128, 1) k_train(train_args a) {
	if (a.budgeted && a.state->wave_step >= a.state->wave_budget) return;
	extern __shared__ uint8_t smem_raw[];
	uint8_t* sm = align128(smem_raw);
	const uint32_t t = threadIdx.x, warp = t >> 5;
	uint8_t* img = sm;
	uint8_t* X0 = sm + kTrX0;
	uint8_t* sig = sm + kTrSig;
	uint64_t* bars = reinterpret_cast<uint64_t*>(sm + kTrBars);
	uint32_t* tptr = reinterpret_cast<uint32_t*>(sm + kTrBars + 32);
	volatile uint32_t* fail = reinterpret_cast<volatile uint32_t*>(sm + kTrBars + 40);
	float* red = reinterpret_cast<float*>(sm + kTrBars + 48);
	const bool loaded = kernel_begin(img, a.image, bars, 2, tptr, fail, 2, 512, a.error);
	const uint32_t tmem = *tptr;
	const uint32_t lane_off = (32u * warp) << 16;
	const uint32_t img_s = smem_u32(img), x0_s = smem_u32(X0), sig_s = smem_u32(sig);
	uint32_t xs[kLayers];
	xs[0] = x0_s;
	for (int l = 1; l < kLayers; l++) xs[l] = smem_u32(sm + kTrX1 + (l - 1) * kHidBytes);
	uint8_t* Xh[kLayers] = {X0, sm + kTrX1, sm + kTrX1 + kHidBytes, sm + kTrX1 + 2 * kHidBytes, sm + kTrX1 + 3 * kHidBytes};
	const uint32_t cnt = min(*a.count, a.count_cap);
	const uint32_t rows = step_rows(cnt, a.batch, a.min_rows);
	const float inv_n = rows ? 1.f / static_cast<float>(rows) : 0.f;
	const uint32_t tiles = (rows + kTileRows - 1) / kTileRows;
	const uint32_t step = a.state->step;
	const float wmax = a.weight_clip > 0.f && a.state->weight_mean > 0.f ? a.weight_clip * a.state->weight_mean : INFINITY;
	uint64_t* bar = &bars[1];
	uint32_t phase = 0;
	bool first = true, failed = !loaded;
	float loss = 0.f;
	for (uint32_t tile = blockIdx.x; loaded && tile < tiles; tile += gridDim.x) {
		const uint32_t row = tile * kTileRows + t;
		const bool valid = row < rows;
		float x[kInputs], dx = 0.f, dy = 0.f, dz = 1.f, pb = 1.f, wgt = 0.f;
#pragma unroll
		for (int j = 0; j < kInputs; j++) x[j] = 0.f;
		if (valid) {
			const uint32_t idx = a.sequential ? row : mix32(row * 0x9E3779B9u ^ mix32(step + 0x632BE5ABu)) % cnt;
			const float4* s = a.samples + static_cast<size_t>(kSampleFloat4) * idx;
			const float4 s0 = s[0], s1 = s[1], s2 = s[2], s3 = s[3];
			x[0] = s0.x; x[1] = s0.y; x[2] = s0.z; x[3] = s0.w;
			x[4] = s1.x; x[5] = s1.y; x[6] = s1.z; x[7] = s1.w; x[8] = s2.x;
			dx = s2.y; dy = s2.z; dz = s2.w;
			pb = s3.x; wgt = fminf(s3.y, wmax);
		}
		encode_row(x, X0, t);
		// forward
		float v[kHiddenK];
#pragma unroll 1
		for (int l = 0; l < kLayers; l++) {
			if (l > 0) {
				tmem_ld32(tmem + lane_off + kColS, v);
				tmem_ld32(tmem + lane_off + kColS + 32u, v + 32);
				store_hidden_row(Xh[l], t, v);
			}
			publish(1);
			if (t == 0) {
				tc_fence_after();
				const uint32_t sbo = l == 0 ? kSboIn : kSboHid;
				mma_kk(tmem + kColS, xs[l], sbo, img_s + 2u * aug_offset(l), sbo, layer_out(l), layer_k(l) / 16);
				umma_commit(bar);
			}
			if (!group_wait(bar, phase, fail, 1)) { failed = true; break; }
		}
		if (failed) break;
		// output gradient
		tmem_ld32(tmem + lane_off + kColS, v);
		tmem_ld16(tmem + lane_off + kColS + 32u, v + 32);
		float g[kOutputs];
		loss += output_grad(v, dx, dy, dz, wgt, pb, inv_n, g);
		store_signal_row<kOutputs>(sig, t, g);
		// backward, layer 5 down to layer 2
#pragma unroll 1
		for (int l = kLayers - 1; l >= 1; l--) {
			publish(1);
			if (t == 0) {
				tc_fence_after();
				const uint32_t n = layer_out(l);
				mma_mm(tmem + col_w(l), xs[l], kSboHid, sig_s, n * 16u, n, !first);
				mma_km(tmem + kColS, sig_s, n * 16u, img_s + 2u * aug_offset(l), kSboHid, kHiddenK, n / 16);
				umma_commit(bar);
			}
			if (!group_wait(bar, phase, fail, 1)) { failed = true; break; }
			tmem_ld32(tmem + lane_off + kColS, v);
			tmem_ld32(tmem + lane_off + kColS + 32u, v + 32);
			relu_mask(Xh[l], t, v);
			store_signal_row<kHidden>(sig, t, v);
		}
		if (failed) break;
		// layer 1: weight gradient only, features 0..127 and 128..255 (224.. unused)
		publish(1);
		if (t == 0) {
			tc_fence_after();
			mma_mm(tmem + col_w(0), x0_s, kSboIn, sig_s, kHidden * 16u, kHidden, !first);
			mma_mm(tmem + col_w(kLayers), x0_s + 16u * 128u, kSboIn, sig_s, kHidden * 16u, kHidden, !first);
			umma_commit(bar);
		}
		if (!group_wait(bar, phase, fail, 1)) { failed = true; break; }
		first = false;
	}
	if (failed && loaded) {
		if (t == 0) set_error(a.error, RB_ERR_DEVICE_TIMEOUT);
		mbar_wait(bar, phase, kWaitNs);
	}
	// per-CTA gradient partials, device parameter order [out][K]
	float* part = a.partial + static_cast<size_t>(blockIdx.x) * kAugParams;
	if (first || failed) {
		for (uint32_t i = t; i < static_cast<uint32_t>(kAugParams); i += blockDim.x) part[i] = 0.f;
	} else {
		float w[16];
#pragma unroll 1
		for (int region = 0; region < kLayers + 1; region++) {
			const int l = region == kLayers ? 0 : region;
			const uint32_t m = region == kLayers ? 128u + t : t;  // input feature of this lane
			const int K = layer_k(l);
			const bool keep = static_cast<int>(m) < K;
			const int nout = layer_out(l);
			for (int c = 0; c < nout; c += 16) {
				tmem_ld16(tmem + lane_off + col_w(region) + static_cast<uint32_t>(c), w);
				if (keep) {
#pragma unroll
					for (int j = 0; j < 16; j++) part[aug_offset(l) + (c + j) * K + static_cast<int>(m)] = w[j];
				}
			}
		}
	}
	// batch loss of this CTA
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) loss += __shfl_xor_sync(0xffffffffu, loss, o);
	if ((t & 31u) == 0) red[warp] = loss;
	kernel_end(tmem, 512);
	if (t == 0) a.partial_loss[blockIdx.x] = (red[0] + red[1]) + (red[2] + red[3]);
}

// ---------------------------------------------------------------- Adam
struct adam_args {
	float* master;
	float* m;
	float* v;
	__nv_bfloat16* image;
	const float* partial;
	const float* partial_loss;
	int parts;
	float* grad;
	device_state* state;
	const uint32_t* count;
	uint32_t count_cap;
	uint32_t batch;
	uint32_t min_rows;
	uint32_t budgeted;
	float lr;
	uint32_t warmup_steps;      // the guide becomes usable for sampling at this step count
};

// Sums the per-CTA partials in CTA order, then one Adam step (beta1 0.9,
// beta2 0.999, eps 1e-8, bias-corrected) on the FP32 master weights and a
// fresh BF16 image. The last block to finish advances the step counter.
__global__ void __launch_bounds__(256) k_adam(adam_args a) {
	if (a.budgeted && a.state->wave_step >= a.state->wave_budget) return;
	const uint32_t rows = step_rows(min(*a.count, a.count_cap), a.batch, a.min_rows);
	if (rows == 0u) return;
	const uint32_t t_step = a.state->step + 1u;
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i < kAugParams) {
		float g = 0.f;
		for (int c = 0; c < a.parts; c++) g += a.partial[static_cast<size_t>(c) * kAugParams + i];
		int l, o, k;
		aug_coords(i, l, o, k);
		if (aug_to_flat(l, o, k) < 0) g = 0.f;
		a.grad[i] = g;
		const float m = __fadd_rn(__fmul_rn(0.9f, a.m[i]), __fmul_rn(0.1f, g));
		const float v = __fadd_rn(__fmul_rn(0.999f, a.v[i]), __fmul_rn(__fmul_rn(0.001f, g), g));
		const float c1 = static_cast<float>(1.0 - pow(0.9, static_cast<double>(t_step)));
		const float c2 = static_cast<float>(1.0 - pow(0.999, static_cast<double>(t_step)));
		const float mh = __fdiv_rn(m, c1), vh = __fdiv_rn(v, c2);
		const float p = __fsub_rn(a.master[i], __fdiv_rn(__fmul_rn(a.lr, mh), __fadd_rn(__fsqrt_rn(vh), 1e-8f)));
		a.m[i] = m;
		a.v[i] = v;
		a.master[i] = p;
		a.image[image_index(l, o, k)] = __float2bfloat16_rn(p);
	}
	if (blockIdx.x == 0 && threadIdx.x == 0) {
		float s = 0.f;
		for (int c = 0; c < a.parts; c++) s += a.partial_loss[c];
		a.state->last_loss = s;
		a.state->rows_last = rows;
	}
	__syncthreads();
	if (threadIdx.x == 0) {
		__threadfence();
		if (atomicAdd(&a.state->ticket, 1u) == gridDim.x - 1u) {
			a.state->step = t_step;
			if (t_step >= a.warmup_steps) a.state->usable = 1u;
			a.state->wave_step += 1u;
			a.state->ticket = 0u;
			__threadfence();
		}
	}
}

__global__ void k_image(const float* master, __nv_bfloat16* image) {
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= kAugParams) return;
	int l, o, k;
	aug_coords(i, l, o, k);
	image[image_index(l, o, k)] = __float2bfloat16_rn(master[i]);
}

__global__ void k_decode_sample(const float* raw, const float* u, uint32_t n, float* dirs, float* pdfs) {
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	float o[kOutputs], d[3];
	alignas(16) float g[kOutputs];
	for (int c = 0; c < kOutputs; c++) o[c] = raw[static_cast<size_t>(i) * kOutputs + c];
	decode_outputs(o, g);
	guide_sample(g, u[3 * i], u[3 * i + 1], u[3 * i + 2], d);
	dirs[3 * i] = d[0];
	dirs[3 * i + 1] = d[1];
	dirs[3 * i + 2] = d[2];
	pdfs[i] = guide_pdf(g, d[0], d[1], d[2]);
}

// ---------------------------------------------------------------- collection
struct collect_args {
	const float4* result;
	const uint64_t* first_item;
	const uint64_t* total_items;
	uint32_t capacity;
	const float4* vertices;
	const uint32_t* vertex_count;
	uint32_t depth;
	float4* samples;
	uint32_t cap;
	device_state* state;
};

__global__ void k_collect_begin(device_state* s) {
	s->candidates_last = s->candidates;
	s->candidates = 0u;
	s->wave_written = 0u;
	s->wave_weight = 0.f;
}

// Ring fill, running mean of the weights (an exponential average over waves,
// weight 1/4 for the newest), and this wave's training budget (steps_per_wave steps).
__global__ void k_collect_end(device_state* s, uint32_t cap, uint32_t steps) {
	const uint32_t f = s->ring_filled + s->wave_written;
	s->ring_filled = f < cap ? f : cap;
	if (s->wave_written > 0u) {
		const float m = s->wave_weight / static_cast<float>(s->wave_written);
		s->weight_mean = s->weight_mean > 0.f ? 0.75f * s->weight_mean + 0.25f * m : m;
	}
	s->wave_budget = steps;
	s->wave_step = 0u;
}

// One thread per path of the wave: every recorded vertex with a positive
// weight is a candidate; candidates are kept with probability
// min(1, 0.9 cap / candidates of the previous wave), so that one wave never
// fills the ring with the first part of the image only, and written into the
// replay ring over its oldest samples. Every sample carries the pdf its
// direction was drawn with, so samples of older guides stay valid.
__global__ void __launch_bounds__(256) k_collect(collect_args a) {
	const uint64_t first = *a.first_item, total = *a.total_items;
	const uint64_t left = total > first ? total - first : 0;
	const uint32_t n = static_cast<uint32_t>(left < a.capacity ? left : a.capacity);
	const uint32_t cl = a.state->candidates_last;
	const float keep = cl == 0u ? 1.f : fminf(1.f, 0.9f * static_cast<float>(a.cap) / static_cast<float>(cl));
	const uint32_t lane = threadIdx.x & 31u;
	for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
		const uint32_t i = base + threadIdx.x;
		const uint32_t nv = i < n ? a.vertex_count[i] : 0u;
		const uint32_t nmax = __reduce_max_sync(0xffffffffu, nv);
		float4 L = make_float4(0.f, 0.f, 0.f, 0.f);
		if (nv > 0u) L = a.result[i];
		for (uint32_t vtx = 0; vtx < nmax; vtx++) {
			bool cand = false, kept = false;
			float4 r0, r1, r2, r3;
			float wgt = 0.f;
			if (vtx < nv) {
				const float4* r = a.vertices + (static_cast<size_t>(i) * a.depth + vtx) * kVertexFloat4;
				r0 = r[0]; r1 = r[1]; r2 = r[2]; r3 = r[3];
				const float4 r4 = r[4];
				const float b[3] = {r3.y, r3.z, r3.w};
				const float dl[3] = {L.x - r4.x, L.y - r4.y, L.z - r4.z};
				const float lum[3] = {0.2126f, 0.7152f, 0.0722f};
				for (int c = 0; c < 3; c++)
					if (b[c] > 0.f) wgt += lum[c] * (dl[c] / b[c]);
				cand = wgt > 0.f && isfinite(wgt);
				if (cand) {
					const uint32_t h = mix32(static_cast<uint32_t>(first + i) * 0x9E3779B9u ^ mix32(vtx * 0x85ebca6bu + static_cast<uint32_t>(first >> 32)));
					kept = static_cast<float>(h >> 8) * (1.f / 16777216.f) < keep;
				}
			}
			const uint32_t cmask = __ballot_sync(0xffffffffu, cand);
			const uint32_t kmask = __ballot_sync(0xffffffffu, kept);
			uint32_t slot0 = 0;
			if (lane == 0) {
				if (cmask) atomicAdd(&a.state->candidates, static_cast<uint32_t>(__popc(cmask)));
				if (kmask) {
					slot0 = atomicAdd(&a.state->ring_head, static_cast<uint32_t>(__popc(kmask)));
					atomicAdd(&a.state->wave_written, static_cast<uint32_t>(__popc(kmask)));
				}
			}
			slot0 = __shfl_sync(0xffffffffu, slot0, 0);
			float wsum = kept ? wgt : 0.f;
#pragma unroll
			for (int o = 16; o > 0; o >>= 1) wsum += __shfl_xor_sync(0xffffffffu, wsum, o);
			if (lane == 0 && kmask) atomicAdd(&a.state->wave_weight, wsum);
			if (kept) {
				const uint32_t slot = (slot0 + __popc(kmask & ((1u << lane) - 1u))) & (a.cap - 1u);
				float4* s = a.samples + static_cast<size_t>(kSampleFloat4) * slot;
				s[0] = r0;
				s[1] = r1;
				s[2] = r2;                                      // x8, direction
				s[3] = make_float4(r3.x, wgt, 0.f, 0.f);        // bsdf pdf, weight
			}
		}
	}
}

} // namespace

// ---------------------------------------------------------------- host side
void release(guide_state& g) {
	void* ptrs[] = {g.dstate, g.master, g.adam_m, g.adam_v, g.image, g.grad, g.partial, g.partial_loss, g.samples,
		g.host_samples, g.host_count, g.query_in, g.query_out, g.queue, g.vertices, g.vertex_count};
	for (void* p : ptrs)
		if (p) cudaFree(p);
	g = guide_state{};
}

cudaError_t allocate(guide_state& g, int ctas) {
	cudaError_t e = cudaSuccess;
	auto get = [&](void** p, size_t bytes) {
		if (e == cudaSuccess) e = cudaMalloc(p, bytes);
	};
	g.ctas = ctas;
	get(reinterpret_cast<void**>(&g.dstate), sizeof(device_state));
	get(reinterpret_cast<void**>(&g.master), sizeof(float) * kAugParams);
	get(reinterpret_cast<void**>(&g.adam_m), sizeof(float) * kAugParams);
	get(reinterpret_cast<void**>(&g.adam_v), sizeof(float) * kAugParams);
	get(reinterpret_cast<void**>(&g.image), kImageBytes);
	get(reinterpret_cast<void**>(&g.grad), sizeof(float) * kAugParams);
	get(reinterpret_cast<void**>(&g.partial), sizeof(float) * kAugParams * static_cast<size_t>(ctas));
	get(reinterpret_cast<void**>(&g.partial_loss), sizeof(float) * static_cast<size_t>(ctas));
	get(reinterpret_cast<void**>(&g.samples), sizeof(float4) * kSampleFloat4 * static_cast<size_t>(g.sample_cap));
	get(reinterpret_cast<void**>(&g.host_count), sizeof(uint32_t));
	if (e == cudaSuccess) e = cudaMemset(g.dstate, 0, sizeof(device_state));
	if (e == cudaSuccess) e = cudaFuncSetAttribute(k_forward<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kFwdSmem);
	if (e == cudaSuccess) e = cudaFuncSetAttribute(k_forward<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kFwdSmem);
	if (e == cudaSuccess) e = cudaFuncSetAttribute(k_train, cudaFuncAttributeMaxDynamicSharedMemorySize, kTrSmem);
	return e;
}

cudaError_t allocate_wave(guide_state& g, uint32_t capacity, uint32_t depth) {
	if (g.wave_capacity >= capacity && g.depth >= depth && g.query_in) return cudaSuccess;
	void* ptrs[] = {g.query_in, g.query_out, g.queue, g.vertices, g.vertex_count};
	for (void* p : ptrs)
		if (p) cudaFree(p);
	g.query_in = g.query_out = g.vertices = nullptr;
	g.queue = g.vertex_count = nullptr;
	g.wave_capacity = 0;
	g.depth = 0;
	cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&g.query_in), sizeof(float4) * 3 * static_cast<size_t>(capacity));
	if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&g.query_out), sizeof(float4) * 12 * static_cast<size_t>(capacity));
	if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&g.queue), sizeof(uint32_t) * static_cast<size_t>(capacity));
	if (e == cudaSuccess)
		e = cudaMalloc(reinterpret_cast<void**>(&g.vertices), sizeof(float4) * kVertexFloat4 * static_cast<size_t>(capacity) * depth);
	if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&g.vertex_count), sizeof(uint32_t) * static_cast<size_t>(capacity));
	if (e == cudaSuccess) e = cudaMemset(g.vertex_count, 0, sizeof(uint32_t) * static_cast<size_t>(capacity));
	if (e == cudaSuccess) {
		g.wave_capacity = capacity;
		g.depth = depth;
	}
	return e;
}

cudaError_t allocate_lane(lane_guide& l, uint32_t capacity, uint32_t depth) {
	if (l.capacity >= capacity && l.depth >= depth && l.query_in) return cudaSuccess;
	release_lane(l);
	cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&l.query_in), sizeof(float4) * 3 * static_cast<size_t>(capacity));
	if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&l.query_out), sizeof(float4) * 12 * static_cast<size_t>(capacity));
	if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&l.queue), sizeof(uint32_t) * static_cast<size_t>(capacity));
	if (e == cudaSuccess)
		e = cudaMalloc(reinterpret_cast<void**>(&l.vertices), sizeof(float4) * kVertexFloat4 * static_cast<size_t>(capacity) * depth);
	if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&l.vertex_count), sizeof(uint32_t) * static_cast<size_t>(capacity));
	if (e == cudaSuccess) e = cudaMemset(l.vertex_count, 0, sizeof(uint32_t) * static_cast<size_t>(capacity));
	if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&l.image), kImageBytes);
	if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&l.usable), sizeof(uint32_t));
	if (e == cudaSuccess) e = cudaMemset(l.usable, 0, sizeof(uint32_t));
	if (e != cudaSuccess) {
		release_lane(l);
		return e;
	}
	l.capacity = capacity;
	l.depth = depth;
	return cudaSuccess;
}

void release_lane(lane_guide& l) {
	void* ptrs[] = {l.query_in, l.query_out, l.queue, l.vertices, l.vertex_count, l.image, l.usable};
	for (void* p : ptrs)
		if (p) cudaFree(p);
	l = lane_guide{};
}

wave_guide state_view(const guide_state& g) {
	const uint32_t* usable = g.dstate == nullptr ? nullptr
		: reinterpret_cast<const uint32_t*>(reinterpret_cast<const char*>(g.dstate) + offsetof(device_state, usable));
	return wave_guide{g.dstate, g.query_in, g.query_out, g.queue, g.vertices, g.vertex_count, g.depth, usable, g.image};
}

wave_guide lane_view(const guide_state& g, const lane_guide& l) {
	return wave_guide{g.dstate, l.query_in, l.query_out, l.queue, l.vertices, l.vertex_count, l.depth, l.usable, l.image};
}

__global__ void k_snapshot(const uint4* __restrict__ image, uint4* __restrict__ lane_image, uint32_t n16,
	const device_state* s, uint32_t* usable) {
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n16) lane_image[i] = image[i];
	if (i == 0) *usable = s->usable;
}

// A bounded wait that is meant to run out: an mbarrier that nothing arrives
// on, waited for with mbar_wait (the wait of every guide kernel). Writes the
// status the wait leads to.
__global__ void k_bounded_wait(uint64_t limit_ns, uint32_t* status) {
	__shared__ __align__(8) uint64_t bar;
	if (threadIdx.x == 0) {
		mbar_init(&bar, 1);
		fence_mbar_init();
	}
	__syncthreads();
	const bool arrived = mbar_wait(&bar, 0, limit_ns);
	if (threadIdx.x == 0) *status = arrived ? RB_OK : RB_ERR_DEVICE_TIMEOUT;
}

cudaError_t launch_bounded_wait(uint64_t limit_ns, uint32_t* status, cudaStream_t s) {
	k_bounded_wait<<<1, 32, 0, s>>>(limit_ns, status);
	return cudaGetLastError();
}

cudaError_t launch_snapshot(const guide_state& g, const lane_guide& l, cudaStream_t s) {
	static_assert(kImageBytes % 16 == 0, "the image is copied in 16-byte units");
	const uint32_t n16 = kImageBytes / 16;
	k_snapshot<<<(n16 + 255) / 256, 256, 0, s>>>(reinterpret_cast<const uint4*>(g.image), reinterpret_cast<uint4*>(l.image),
		n16, g.dstate, l.usable);
	return cudaGetLastError();
}

cudaError_t launch_init_image(const guide_state& g, cudaStream_t s) {
	k_image<<<(kAugParams + 255) / 256, 256, 0, s>>>(g.master, reinterpret_cast<__nv_bfloat16*>(g.image));
	return cudaGetLastError();
}

cudaError_t launch_forward_raw(const guide_state& g, const float* x, uint32_t n, float* out, cudaStream_t s) {
	if (n == 0) return cudaSuccess;
	fwd_args a{};
	a.image = g.image;
	a.n = n;
	a.x = x;
	a.out = out;
	a.error = &g.dstate->error;
	const uint32_t tiles = (n + kTileRows - 1) / kTileRows;
	const uint32_t want = (tiles + kFwdGroups - 1) / kFwdGroups;
	const uint32_t grid = want < static_cast<uint32_t>(g.ctas) ? want : static_cast<uint32_t>(g.ctas);
	k_forward<false><<<grid, kFwdGroups * 128, kFwdSmem, s>>>(a);
	return cudaGetLastError();
}

cudaError_t launch_forward_queue(const guide_state& g, const wave_guide& wg, const uint32_t* count, cudaStream_t s) {
	fwd_args a{};
	a.image = wg.image;
	a.count = count;
	a.queue = wg.queue;
	a.in4 = wg.query_in;
	a.out4 = wg.query_out;
	a.error = &g.dstate->error;
	k_forward<true><<<g.ctas, kFwdGroups * 128, kFwdSmem, s>>>(a);
	return cudaGetLastError();
}

cudaError_t launch_train_step(const guide_state& g, const float4* samples, const uint32_t* count, uint32_t count_cap,
	uint32_t batch, uint32_t min_rows, bool sequential, bool budgeted, cudaStream_t s) {
	train_args t{};
	t.image = g.image;
	t.samples = samples;
	t.count = count;
	t.count_cap = count_cap;
	t.batch = batch;
	t.min_rows = min_rows;
	t.sequential = sequential ? 1u : 0u;
	t.budgeted = budgeted ? 1u : 0u;
	t.weight_clip = budgeted ? g.weight_clip : 0.f;
	t.state = g.dstate;
	t.partial = g.partial;
	t.partial_loss = g.partial_loss;
	t.error = &g.dstate->error;
	k_train<<<g.ctas, 128, kTrSmem, s>>>(t);
	adam_args a{};
	a.master = g.master;
	a.m = g.adam_m;
	a.v = g.adam_v;
	a.image = reinterpret_cast<__nv_bfloat16*>(g.image);
	a.partial = g.partial;
	a.partial_loss = g.partial_loss;
	a.parts = g.ctas;
	a.grad = g.grad;
	a.state = g.dstate;
	a.count = count;
	a.count_cap = count_cap;
	a.batch = batch;
	a.min_rows = min_rows;
	a.budgeted = budgeted ? 1u : 0u;
	a.lr = g.cfg.learning_rate;
	a.warmup_steps = g.cfg.warmup_steps;
	k_adam<<<(kAugParams + 255) / 256, 256, 0, s>>>(a);
	return cudaGetLastError();
}

cudaError_t launch_decode_sample(const float* raw, const float* u, uint32_t n, float* dirs, float* pdfs, cudaStream_t s) {
	if (n == 0) return cudaSuccess;
	k_decode_sample<<<(n + 127) / 128, 128, 0, s>>>(raw, u, n, dirs, pdfs);
	return cudaGetLastError();
}

cudaError_t launch_collect(const guide_state& g, const wave_guide& wg, const float4* result, const uint64_t* first_item,
	const uint64_t* total_items, uint32_t capacity, cudaStream_t s) {
	k_collect_begin<<<1, 1, 0, s>>>(g.dstate);
	collect_args a{};
	a.result = result;
	a.first_item = first_item;
	a.total_items = total_items;
	a.capacity = capacity;
	a.vertices = wg.vertices;
	a.vertex_count = wg.vertex_count;
	a.depth = wg.depth;
	a.samples = g.samples;
	a.cap = g.sample_cap;
	a.state = g.dstate;
	k_collect<<<g.ctas * 8, 256, 0, s>>>(a);
	k_collect_end<<<1, 1, 0, s>>>(g.dstate, g.sample_cap, g.cfg.steps_per_wave);
	return cudaGetLastError();
}

} // namespace guide
} // namespace rb
