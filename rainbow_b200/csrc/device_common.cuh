// Device helpers shared by the kernel files: the per-thread traversal stack
// in shared memory, one ray's traversal with the 4-wide fast path and its
// reference-order fallback, and the error word.
#pragma once

#include "kernels.cuh"

namespace rb {
namespace gpu {

using namespace rb::pt;

// Per-thread traversal stack in shared memory, [entry][thread]: node
// references, and for the child-box traversal the entry distance of each entry.
struct smem_stack {
	uint32_t* base;
	float* te;
	uint32_t stride;
	uint32_t sp;
	uint32_t cap;
	__device__ void reset() { sp = 0; }
	__device__ void push(uint32_t v) { base[sp * stride] = v; sp++; }
	__device__ uint32_t pop() { sp--; return base[sp * stride]; }
	__device__ void push(uint32_t v, float t) { base[sp * stride] = v; te[sp * stride] = t; sp++; }
	__device__ void pop(uint32_t& v, float& t) { sp--; v = base[sp * stride]; t = te[sp * stride]; }
	__device__ bool empty() const { return sp == 0; }
	__device__ bool full() const { return sp + 2 > cap; }
	__device__ uint32_t size() const { return sp; }
	__device__ raw_stack raw() const { return raw_stack{base, stride, sp, cap}; }
};

__device__ __forceinline__ smem_stack make_stack(uint32_t* smem, uint32_t cap) {
	return smem_stack{smem + threadIdx.x, reinterpret_cast<float*>(smem + cap * blockDim.x) + threadIdx.x, blockDim.x, 0u, cap};
}

__device__ __forceinline__ uint32_t lanemask_lt() {
	uint32_t m;
	asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
	return m;
}

__device__ __forceinline__ void set_error(uint32_t* counters, uint32_t code) { atomicCAS(counters + CNT_ERROR, 0u, code); }

// first: an occlusion query (any hit accepted at len will do) on the 4-wide
// path; its reference-order fallback finds the closest hit, which answers the
// same question.
// INST: instantiated without the instance-slot branch for single-level scenes.
template <bool SHADOW, bool COUNT, bool INST = true>
__device__ __forceinline__ bool trace_one(const scene_view& s, vec3 o, vec3 d, float& len, hit_t& h, smem_stack& st,
	uint32_t& nodes, uint32_t& tris, bool first = false) {
	trace_counters c{0u, 0u};
	bool ok;
	if (!COUNT && s.wnodes != nullptr && !isnan(len)) {
		const float len0 = len;
		const int r = closest_hit_fast<SHADOW, INST>(s, o, d, len, h, st, first);
		ok = r == 1;
		if (r < 0) {  // a NaN length or a full stack: redo the ray in the reference's own visiting order
			len = len0;
			ok = closest_hit<SHADOW, COUNT, INST>(s, o, d, len, h, st, c);
		}
	} else {
		// counting passes count the box and triangle tests of the reference's traversal
		ok = closest_hit<SHADOW, COUNT, INST>(s, o, d, len, h, st, c);
	}
	nodes += c.nodes;
	tris += c.tris;
	return ok;
}

// One ray, closest hit (shadow: visible entities only), out of line so that a
// stage with several call sites (the subsurface walk, the photon mapping
// passes) holds one copy of the traversal. A full stack sets `failed` and
// reports no hit.
template <bool INST>
__device__ __noinline__ hit_t trace_out_of_line(const scene_view& s, vec3 o, vec3 d, float& len, bool shadow, smem_stack& stk,
	bool& failed) {
	hit_t h{-1, 0.f, 0.f};
	uint32_t nodes = 0, tris = 0;
	const bool ok = shadow ? trace_one<true, false, INST>(s, o, d, len, h, stk, nodes, tris)
		: trace_one<false, false, INST>(s, o, d, len, h, stk, nodes, tris);
	if (!ok) {
		failed = true;
		h.slot = -1;
	}
	return h;
}

} // namespace gpu
} // namespace rb
