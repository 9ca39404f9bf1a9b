// Ray/scene geometry of the wavefront path tracer: world<->entity ray
// transforms, slab and triangle tests, the closest-hit traversal in the
// reference's visiting order, surface-interaction construction and ray spawning.
// Host- and device-compilable; every float operation keeps the reference's order.
#pragma once

#include "pt_types.h"

namespace rb {
namespace pt {

#if defined(__CUDA_ARCH__)
#define RB_LDG(p) __ldg(p)
#else
#define RB_LDG(p) (*(p))
#endif

struct ray_t {
	vec3 o, d;
	float len;
};

// ray_epsilon / shadow_epsilon (rainbow-cpu/shared/ray.hpp:10-11)
constexpr float kRayEpsilon = FLT_EPSILON / 2 * 1500;
constexpr float kShadowEpsilon = kRayEpsilon * 10;
constexpr float kInf = __builtin_huge_valf();

// ------------------------------------------------------------------ entity frames
// The ray as entity::intersect sees it (rainbow-cpu/scenes/entity.cpp:18-37 with
// transform::operator()(ray), transform.cpp:94-105): direction normalised twice
// (once by the transform, once by the ray constructor), local length = world
// length * |W2L d|, and back: world length = local t * |L2W d_local|.
struct local_ray {
	vec3 o, d;
	float to_local;   // |W2L d|
	float to_world;   // |L2W d_local|
};

RB_HD local_ray make_local_ray(const float* w2l, const float* l2w, vec3 o, vec3 d) {
	local_ray r;
	const vec3 dl = xform_vector(w2l, d);
	r.to_local = length(dl);
	r.d = normalize(normalize(dl));
	r.o = xform_point(w2l, o);
	r.to_world = length(xform_vector(l2w, r.d));
	return r;
}

// ------------------------------------------------------------------ tests
// Slab test of bounding_box<T>::intersect (detail/accelerator.hpp:29-53) with
// t1 = the ray's current length. inv = 1 / direction per axis.
// fminf/fmaxf give the same outcome as glm's ternary min/max here: t0 and t1
// are never NaN, and a NaN slab bound is ignored by both.
RB_HD bool slab_hit(float4 a, float4 b, vec3 o, vec3 inv, float len) {
	float t0 = 0.f, t1 = len;
	float n = (a.x - o.x) * inv.x, f = (a.w - o.x) * inv.x;
	if (n > f) { const float t = n; n = f; f = t; }
	t0 = fmaxf(t0, n); t1 = fminf(t1, f);
	if (t0 > t1) return false;
	n = (a.y - o.y) * inv.y; f = (b.x - o.y) * inv.y;
	if (n > f) { const float t = n; n = f; f = t; }
	t0 = fmaxf(t0, n); t1 = fminf(t1, f);
	if (t0 > t1) return false;
	n = (a.z - o.z) * inv.z; f = (b.y - o.z) * inv.z;
	if (n > f) { const float t = n; n = f; f = t; }
	t0 = fmaxf(t0, n); t1 = fminf(t1, f);
	return !(t0 > t1);
}

// Moller-Trumbore of mesh::intersect_with_triangle (rainbow-cpu/shapes/mesh.cpp:328-348).
RB_HD bool triangle_hit(vec3 o, vec3 d, float len, vec3 p0, vec3 e1, vec3 e2, float& t, float& b1, float& b2) {
	const vec3 pv = cross(d, e2);
	const vec3 tv = o - p0;
	const vec3 qv = cross(tv, e1);
	const float inv_det = 1.f / dot(e1, pv);
	b1 = dot(tv, pv) * inv_det;
	b2 = dot(d, qv) * inv_det;
	const float b0 = 1.f - b1 - b2;
	t = dot(e2, qv) * inv_det;
	if (t <= 0.f || t >= len) return false;
	if (b0 < 0.f || b0 > 1.f) return false;
	if (b1 < 0.f || b1 > 1.f) return false;
	if (b2 < 0.f || b2 > 1.f) return false;
	return true;
}

// ------------------------------------------------------------------ closest hit
struct hit_t {
	int32_t slot;  // prim slot, -1 on a miss
	float b1, b2;
};

struct trace_counters {
	uint32_t nodes, tris;
};

constexpr uint32_t kEntityInvisible = 0x80000000u;  // flag in the tri_c entity word
// flag in the tri_c entity word: the slot stands for a whole entity whose mesh
// has its own tree (tri_a.x = the tree's root node, tri_a.y = the first slot of
// the entity's copy of the mesh's triangles, in the tree's leaf order)
constexpr uint32_t kEntityInstance = 0x40000000u;
constexpr uint32_t kEntityMask = 0x3fffffffu;
// flag in a mesh tree leaf's w1: w0 counts from the walked instance's first slot
constexpr uint32_t kMeshLeaf = 0x40000000u;

RB_HD float u32_as_float(uint32_t v) {
#if defined(__CUDA_ARCH__)
	return __uint_as_float(v);
#else
	float f;
	__builtin_memcpy(&f, &v, 4);
	return f;
#endif
}
RB_HD uint32_t float_as_u32(float f) {
#if defined(__CUDA_ARCH__)
	return __float_as_uint(f);
#else
	uint32_t v;
	__builtin_memcpy(&v, &f, 4);
	return v;
#endif
}

// A traversal stack as raw words (entry i at base[i * stride], at most cap):
// what the mesh-tree walk below gets by value from its caller's stack.
struct raw_stack {
	uint32_t* base;
	uint32_t stride;
	uint32_t sp;
	uint32_t cap;
	RB_HD void push(uint32_t v) { base[sp * stride] = v; sp++; }
	RB_HD uint32_t pop() { sp--; return base[sp * stride]; }
	RB_HD bool full() const { return sp + 2 > cap; }
};

struct instance_result {
	uint32_t status;  // 0: no hit, 1: a hit (len, slot, b1, b2), 2: the stack overflowed
	float len;        // world length of the hit
	int32_t slot;
	float b1, b2;
	uint32_t nodes, tris;  // box and triangle tests (counting passes)
};

// entity::intersect(ray) for an entity held whole by the scene tree
// (rainbow-cpu/scenes/entity.cpp:39-58 with mesh::intersect, mesh.cpp:45-57):
// the ray goes to local space once, the mesh's own tree is walked in the
// reference's visiting order with the local ray and the local length (which
// every hit shortens), and if anything was hit the world length becomes local
// length * |L2W d_local|. The walk uses the stack above the caller's entries.
// occlusion: stop at the first hit.
template <bool COUNT>
RB_HD instance_result instance_walk(const float4* nodes, const float4* tri_a, const float4* tri_b,
	const float2* tri_c, const entity_rec* ent, uint32_t slot, vec3 o, vec3 d, float len, raw_stack stack, bool occlusion) {
	instance_result r{0u, len, -1, 0.f, 0.f, 0u, 0u};
	const float4 ia = RB_LDG(tri_a + slot);
	const uint32_t root = float_as_u32(ia.x), first = float_as_u32(ia.y);
	const local_ray lr = make_local_ray(ent->w2l, ent->l2w, o, d);
	const vec3 inv = 1.f / lr.d;
	const uint32_t neg = (inv.x < 0.f ? 1u : 0u) | (inv.y < 0.f ? 2u : 0u) | (inv.z < 0.f ? 4u : 0u);
	float llen = len * lr.to_local;
	const uint32_t base = stack.sp;
	if (stack.full()) { r.status = 2u; return r; }
	stack.push(root);
	while (stack.sp > base) {
		const uint32_t n = stack.pop();
		const float4 a = RB_LDG(nodes + 2 * n);
		const float4 b = RB_LDG(nodes + 2 * n + 1);
		if (COUNT) r.nodes++;
		if (!slab_hit(a, b, lr.o, inv, llen)) continue;
		const uint32_t w0 = float_as_u32(b.z), w1 = float_as_u32(b.w);
		if (w1 & RB_BVH_LEAF_FLAG) {
			const uint32_t count = w1 & ~(RB_BVH_LEAF_FLAG | kMeshLeaf);
			for (uint32_t k = 0; k < count; k++) {
				const uint32_t sl = first + w0 + k;
				const float4 ta = RB_LDG(tri_a + sl);
				const float4 tb = RB_LDG(tri_b + sl);
				const float2 tc = RB_LDG(tri_c + sl);
				if (COUNT) r.tris++;
				float t, b1, b2;
				if (triangle_hit(lr.o, lr.d, llen, vec3{ta.x, ta.y, ta.z}, vec3{ta.w, tb.x, tb.y}, vec3{tb.z, tb.w, tc.x}, t,
						b1, b2)) {
					llen = t;
					r.slot = static_cast<int32_t>(sl);
					r.b1 = b1;
					r.b2 = b2;
					r.status = 1u;
					if (occlusion) {  // any hit will do
						stack.sp = base;
						break;
					}
				}
			}
			continue;
		}
		if (stack.full()) { r.status = 2u; return r; }
		if ((neg >> w1) & 1u) { stack.push(n + 1); stack.push(w0); }
		else { stack.push(w0); stack.push(n + 1); }
	}
	if (r.status == 1u) r.len = llen * lr.to_world;
	return r;
}

// The walk above for a caller's stack (which provides raw()); false when the
// stack overflowed. The caller's entries and stack pointer are left as they were.
template <bool COUNT, typename Stack>
RB_HD bool instance_hit(const scene_view& s, uint32_t slot, uint32_t ent, vec3 o, vec3 d, float& len, hit_t& hit,
	Stack& stack, trace_counters& cnt, bool occlusion = false) {
	const instance_result r =
		instance_walk<COUNT>(s.nodes, s.tri_a, s.tri_b, s.tri_c, s.entities + ent, slot, o, d, len, stack.raw(), occlusion);
	if (COUNT) {
		cnt.nodes += r.nodes;
		cnt.tris += r.tris;
	}
	if (r.status == 2u) return false;
	if (r.status == 1u) {
		len = r.len;
		hit.slot = r.slot;
		hit.b1 = r.b1;
		hit.b2 = r.b2;
	}
	return true;
}

// Closest hit in the visiting order of bounding_volume_hierarchy<T>::intersect
// (detail/bounding_volume_hierarchy.hpp:60-108): pop a node, slab-test it
// against the current length, test a leaf's triangles in order, otherwise push
// the far child then the near child (near = right when the ray's direction is
// negative on the split axis). SHADOW skips invisible entities
// (intersect_with_shadow_ray, :110-160). `len` is updated in place like the
// reference's mutable ray.length. Stack provides push/pop/empty/full.
// Returns false when the stack overflowed (the hit is then incomplete).
// INST: the scene may hold instance slots (scene_view::instances); kernels for
// single-level scenes instantiate the traversals without that branch.
template <bool SHADOW, bool COUNT, bool INST = true, typename Stack>
RB_HD bool closest_hit(const scene_view& s, vec3 o, vec3 d, float& len, hit_t& hit, Stack& stack, trace_counters& cnt) {
	const vec3 inv = 1.f / d;
	const uint32_t neg = (inv.x < 0.f ? 1u : 0u) | (inv.y < 0.f ? 2u : 0u) | (inv.z < 0.f ? 4u : 0u);
	hit.slot = -1;
	uint32_t cur_entity = 0xffffffffu;
	local_ray lr{};
	stack.reset();
	stack.push(s.root_node);
	while (!stack.empty()) {
		const uint32_t n = stack.pop();
		const float4 a = RB_LDG(s.nodes + 2 * n);
		const float4 b = RB_LDG(s.nodes + 2 * n + 1);
		if (COUNT) cnt.nodes++;
		if (!slab_hit(a, b, o, inv, len)) continue;
		const uint32_t w0 = float_as_u32(b.z), w1 = float_as_u32(b.w);
		if (w1 & RB_BVH_LEAF_FLAG) {
			const uint32_t count = w1 & ~RB_BVH_LEAF_FLAG;
			for (uint32_t k = 0; k < count; k++) {
				const uint32_t slot = w0 + k;
				const float2 tc = RB_LDG(s.tri_c + slot);
				const uint32_t ew = float_as_u32(tc.y);
				if (SHADOW && (ew & kEntityInvisible)) continue;
				const uint32_t ent = ew & kEntityMask;
				if (INST && (ew & kEntityInstance)) {
					if (!instance_hit<COUNT>(s, slot, ent, o, d, len, hit, stack, cnt)) return false;
					continue;
				}
				const float4 ta = RB_LDG(s.tri_a + slot);
				const float4 tb = RB_LDG(s.tri_b + slot);
				if (ent != cur_entity) {
					cur_entity = ent;
					lr = make_local_ray(s.entities[ent].w2l, s.entities[ent].l2w, o, d);
				}
				if (COUNT) cnt.tris++;
				float t, b1, b2;
				if (triangle_hit(lr.o, lr.d, len * lr.to_local, vec3{ta.x, ta.y, ta.z}, vec3{ta.w, tb.x, tb.y},
						vec3{tb.z, tb.w, tc.x}, t, b1, b2)) {
					len = t * lr.to_world;
					hit.slot = static_cast<int32_t>(slot);
					hit.b1 = b1;
					hit.b2 = b2;
				}
			}
			continue;
		}
		const uint32_t left = n + 1, right = w0;
		if (stack.full()) return false;
		if ((neg >> w1) & 1u) { stack.push(left); stack.push(right); }
		else { stack.push(right); stack.push(left); }
	}
	return true;
}

// ------------------------------------------------------------------ closest hit, 4-wide traversal
// The same visiting decisions as closest_hit above, over the 4-wide collapse
// of the same tree (node4): expanding binary node N tests the boxes of its
// grandchildren directly (a child that is a leaf is tested itself), with one
// 128-byte node load instead of three dependent levels of pops.
//
// Why the decisions are identical. The reference pushes both children (far,
// then near), pops a node and slab-tests it against the ray length at pop time.
// For a box, let te be the reference's t0 after the three axes (it does not
// depend on the length) and tx the minimum of the far distances; with a
// length that is not NaN the box passes iff te <= min(len, tx), and the early
// exits after each axis do not change the outcome because t0 only grows and t1
// only shrinks. Float subtraction and multiplication are monotonic and a
// parent's box contains its children's, so a child that passes implies that its
// parent passes at the same length (te_parent <= te_child, tx_parent >= tx_child).
// Hence, at the length of N's expansion:
//  - the near child X of N is expanded by the reference at once, at the same
//    length: its children pass there iff they pass now, and they can be tested
//    without testing X (a passing child implies X passes);
//  - every other slot that fails now also fails when the reference reaches it
//    (the length only shrinks);
//  - a slot that passes now is pushed with te; when the reference reaches it
//    (popping it, or popping and expanding its parent first) its test, and its
//    parent's, reduce to te <= len, checked as !(te > len) at the pop.
// Slots are visited in the reference's order: the pair of N's near child
// first, each pair near child first (near = the right one when the ray's
// direction is negative on the split axis). Box tests are not counted here;
// counting passes use closest_hit. A NaN length (only reachable through a
// degenerate triangle hit) or a full stack returns -1 so the caller can redo
// the ray on the reference-order path.
RB_HD bool slab_pass(float ax, float ay, float az, float bx, float by, float bz, vec3 o, vec3 inv, float len, float& te) {
	float t0 = 0.f, t1 = len;
	float n = (ax - o.x) * inv.x, f = (bx - o.x) * inv.x;
	if (n > f) { const float t = n; n = f; f = t; }
	t0 = fmaxf(t0, n); t1 = fminf(t1, f);
	n = (ay - o.y) * inv.y; f = (by - o.y) * inv.y;
	if (n > f) { const float t = n; n = f; f = t; }
	t0 = fmaxf(t0, n); t1 = fminf(t1, f);
	n = (az - o.z) * inv.z; f = (bz - o.z) * inv.z;
	if (n > f) { const float t = n; n = f; f = t; }
	t0 = fmaxf(t0, n); t1 = fminf(t1, f);
	te = t0;
	return !(t0 > t1);
}

template <typename T>
RB_HD T pick4(T a, T b, T c, T d, uint32_t i) { return i == 0 ? a : i == 1 ? b : i == 2 ? c : d; }

// Traversal state of one ray, so that a thread can advance it a step at a
// time (and take a new ray as soon as its ray is done).
struct trav_state {
	vec3 o, d, inv;
	uint32_t neg;        // direction sign bits (x: 1, y: 2, z: 4)
	float len;
	hit_t hit;
	uint32_t cur;        // next node or leaf to visit
	uint32_t cur_entity;
	local_ray lr;
	bool first;          // stop at the first accepted hit (occlusion only)
};

// Starts a ray: the root box test of the reference. Returns false when the ray
// is already done (the root box is missed).
template <typename Stack>
RB_HD bool trav_begin(const scene_view& s, trav_state& t, vec3 o, vec3 d, float len, Stack& stack, bool first = false) {
	t.first = first;
	t.o = o;
	t.d = d;
	t.inv = 1.f / d;
	t.neg = (t.inv.x < 0.f ? 1u : 0u) | (t.inv.y < 0.f ? 2u : 0u) | (t.inv.z < 0.f ? 4u : 0u);
	t.len = len;
	t.hit.slot = -1;
	t.hit.b1 = t.hit.b2 = 0.f;
	t.cur_entity = 0xffffffffu;
	t.lr = local_ray{};
	stack.reset();
	float te;
	if (!slab_pass(s.root_a.x, s.root_a.y, s.root_a.z, s.root_a.w, s.root_b.x, s.root_b.y, o, t.inv, len, te)) return false;
	t.cur = s.root_ref;
	return true;
}

// One step of a started ray: the current leaf's triangles or the current
// node's four slots, then the next node (descent or pop). Returns 0 while the
// ray goes on, 1 when it is done, -1 when it must be redone in the reference's
// order (a NaN length or a full stack).
template <bool SHADOW, bool INST = true, typename Stack>
RB_HD int trav_step(const scene_view& s, trav_state& t, Stack& stack) {
	if (t.cur & kRefLeaf) {
		const uint32_t first = t.cur & 0x00ffffffu, count = (t.cur >> 24) & 0x7fu;
		for (uint32_t k = 0; k < count; k++) {
			const uint32_t slot = first + k;
			const float2 tc = RB_LDG(s.tri_c + slot);
			const uint32_t ew = float_as_u32(tc.y);
			if (SHADOW && (ew & kEntityInvisible)) continue;
			const uint32_t ent = ew & kEntityMask;
			if (INST && (ew & kEntityInstance)) {
				trace_counters none{0u, 0u};
				if (!instance_hit<false>(s, slot, ent, t.o, t.d, t.len, t.hit, stack, none, t.first)) return -1;
				if (isnan(t.len)) return -1;
				if (t.first && t.hit.slot >= 0) return 1;
				continue;
			}
			const float4 ta = RB_LDG(s.tri_a + slot);
			const float4 tb = RB_LDG(s.tri_b + slot);
			if (ent != t.cur_entity) {
				t.cur_entity = ent;
				t.lr = make_local_ray(s.entities[ent].w2l, s.entities[ent].l2w, t.o, t.d);
			}
			float th, b1, b2;
			if (triangle_hit(t.lr.o, t.lr.d, t.len * t.lr.to_local, vec3{ta.x, ta.y, ta.z}, vec3{ta.w, tb.x, tb.y},
					vec3{tb.z, tb.w, tc.x}, th, b1, b2)) {
				t.len = th * t.lr.to_world;
				t.hit.slot = static_cast<int32_t>(slot);
				t.hit.b1 = b1;
				t.hit.b2 = b2;
				if (isnan(t.len)) return -1;
				if (t.first) return 1;
			}
		}
	} else {
		const node4* nd = s.wnodes + t.cur;
		const float4 lx = RB_LDG(&nd->lo_x), ly = RB_LDG(&nd->lo_y), lz = RB_LDG(&nd->lo_z);
		const float4 hx = RB_LDG(&nd->hi_x), hy = RB_LDG(&nd->hi_y), hz = RB_LDG(&nd->hi_z);
		const uint4 rf = RB_LDG(&nd->ref);
		const uint32_t meta = RB_LDG(&nd->meta.x);
		float t0, t1, t2, t3;
		uint32_t pass = 0;
		if ((meta & 0x100u) && slab_pass(lx.x, ly.x, lz.x, hx.x, hy.x, hz.x, t.o, t.inv, t.len, t0)) pass |= 1u;
		if ((meta & 0x200u) && slab_pass(lx.y, ly.y, lz.y, hx.y, hy.y, hz.y, t.o, t.inv, t.len, t1)) pass |= 2u;
		if ((meta & 0x400u) && slab_pass(lx.z, ly.z, lz.z, hx.z, hy.z, hz.z, t.o, t.inv, t.len, t2)) pass |= 4u;
		if ((meta & 0x800u) && slab_pass(lx.w, ly.w, lz.w, hx.w, hy.w, hz.w, t.o, t.inv, t.len, t3)) pass |= 8u;
		if (pass != 0u) {
			// the reference's order: near pair first, near slot first within each pair
			const uint32_t pf = (t.neg >> (meta & 3u)) & 1u;
			const uint32_t ax_first = (meta >> (2u + 2u * pf)) & 3u, ax_second = (meta >> (2u + 2u * (pf ^ 1u))) & 3u;
			const uint32_t o0 = 2u * pf + ((t.neg >> ax_first) & 1u);
			const uint32_t o2 = 2u * (pf ^ 1u) + ((t.neg >> ax_second) & 1u);
			const uint32_t order = o0 | ((o0 ^ 1u) << 2) | (o2 << 4) | ((o2 ^ 1u) << 6);
			// walk the order backwards: every passing slot but the first is pushed,
			// later ones first, so they pop in order
			uint32_t next = 0xffffffffu;
			float next_te = 0.f;
#if defined(__CUDA_ARCH__)
#pragma unroll
#endif
			for (int k = 3; k >= 0; k--) {
				const uint32_t sl = (order >> (2 * k)) & 3u;
				if (!((pass >> sl) & 1u)) continue;
				if (next != 0xffffffffu) {
					if (stack.full()) return -1;
					stack.push(next, next_te);
				}
				next = pick4(rf.x, rf.y, rf.z, rf.w, sl);
				next_te = pick4(t0, t1, t2, t3, sl);
			}
			t.cur = next;
			return 0;
		}
	}
	// pop the next slot whose box still passes at the current length
	while (!stack.empty()) {
		uint32_t ref;
		float tent;
		stack.pop(ref, tent);
		if (!(tent > t.len)) {
			t.cur = ref;
			return 0;
		}
	}
	return 1;
}

// first: stop at the first hit accepted at the ray's length (an occlusion
// query), instead of the closest.
template <bool SHADOW, bool INST = true, typename Stack>
RB_HD int closest_hit_fast(const scene_view& s, vec3 o, vec3 d, float& len, hit_t& hit, Stack& stack, bool first = false) {
	trav_state t;
	int r = 1;
	if (trav_begin(s, t, o, d, len, stack, first)) {
		do r = trav_step<SHADOW, INST>(s, t, stack);
		while (r == 0);
	}
	len = t.len;
	hit = t.hit;
	return r;
}

// World length of the closest hit of ray (o, d) on entity ent's own triangles
// within len (len when none), with the arithmetic entity::intersect uses; false
// when the entity has more than max_tris triangles (then it is not worth it).
RB_HD bool entity_closest_length(const scene_view& s, uint32_t ent, vec3 o, vec3 d, float len, uint32_t max_tris,
	float& out) {
	const entity_rec& e = s.entities[ent];
	if (e.mesh < 0) return false;
	const mesh_rec& m = s.meshes[e.mesh];
	if (m.num_triangles > max_tris) return false;
	const local_ray lr = make_local_ray(e.w2l, e.l2w, o, d);
	float llen = len * lr.to_local;
	bool any = false;
	for (uint32_t k = 0; k < m.num_triangles; k++) {
		const uint32_t* idx = s.indices + m.index_offset + 3 * k;
		const float* p = s.positions;
		const uint32_t i0 = 3 * (m.vertex_offset + idx[0]), i1 = 3 * (m.vertex_offset + idx[1]), i2 = 3 * (m.vertex_offset + idx[2]);
		const vec3 p0{p[i0], p[i0 + 1], p[i0 + 2]}, p1{p[i1], p[i1 + 1], p[i1 + 2]}, p2{p[i2], p[i2 + 1], p[i2 + 2]};
		float t, b1, b2;
		if (triangle_hit(lr.o, lr.d, llen, p0, p1 - p0, p2 - p0, t, b1, b2)) {
			llen = t;
			any = true;
		}
	}
	out = any ? llen * lr.to_world : len;
	return true;
}

// ------------------------------------------------------------------ surface interaction
// World-space surface interaction of a hit: mesh::intersect_with_triangle's
// interaction (mesh.cpp:350-441) taken to world space by
// transform::operator()(surface_interaction) (transform.cpp:38-50).
struct surface_t {
	vec3 p;        // point
	vec3 n;        // geometric normal, face-forwarded to the shading normal
	vec3 sx, sy, sz;
	vec3 wo;
	int32_t entity;
	vec2 uv;       // texture coordinates (mesh.cpp:355)
};

RB_HD vec3 load3(const float* a, uint32_t i) { return vec3{a[3 * i], a[3 * i + 1], a[3 * i + 2]}; }

// coordinate_system(normal) (rainbow-cpu/shared/coordinate_system.cpp:8-23)
RB_HD void frame_from_normal(vec3 normal, vec3& x, vec3& y, vec3& z) {
	z = normalize(normal);
	if (fabs_ref(z.x) > fabs_ref(z.y)) x = vec3{-z.z, 0.f, z.x} / sqrtf(z.x * z.x + z.z * z.z);
	else x = vec3{0.f, z.z, -z.y} / sqrtf(z.y * z.y + z.z * z.z);
	y = cross(z, x);
}

// Local interaction pieces of one triangle at barycentrics (b1, b2).
struct local_surface {
	vec3 p, n, sx, sy, sz;
	vec2 uv;
	vec3 dp_du;    // local dp/du (after the degenerate-uv fallback)
};

RB_HD local_surface triangle_surface(const scene_view& s, const mesh_rec& m, uint32_t tri, float b1, float b2) {
	const uint32_t* idx = s.indices + m.index_offset + 3 * tri;
	const uint32_t i0 = m.vertex_offset + idx[0], i1 = m.vertex_offset + idx[1], i2 = m.vertex_offset + idx[2];
	const vec3 p0 = load3(s.positions, i0), p1 = load3(s.positions, i1), p2 = load3(s.positions, i2);
	vec3 uv0{0.f, 0.f, 0.f}, uv1{1.f, 0.f, 0.f}, uv2{1.f, 1.f, 0.f};
	if (m.flags & MESH_HAS_UVS) { uv0 = load3(s.uvs, i0); uv1 = load3(s.uvs, i1); uv2 = load3(s.uvs, i2); }
	const bool reverse = (m.flags & MESH_REVERSE) != 0;
	const vec3 e1 = p1 - p0, e2 = p2 - p0;
	const float b0 = 1.f - b1 - b2;
	local_surface out;
	out.p = p0 * b0 + p1 * b1 + p2 * b2;
	const vec3 uv = uv0 * b0 + uv1 * b1 + uv2 * b2;
	out.uv = vec2{uv.x, uv.y};
	const vec3 normal = reverse ? -normalize(cross(e1, e2)) : normalize(cross(e1, e2));
	const vec3 duv02 = uv0 - uv2, duv12 = uv1 - uv2;
	const vec3 dp02 = p0 - p2, dp12 = p1 - p2;
	const float determinant = duv02.x * duv12.y - duv02.y * duv12.x;
	const float inv_determinant = 1.f / determinant;
	vec3 dp_du = (duv12.y * dp02 - duv02.y * dp12) * inv_determinant;
	vec3 dp_dv = (-duv12.x * dp02 + duv02.x * dp12) * inv_determinant;
	// abs(determinant) < 1e-8 compares in double (a double literal in mesh.cpp:385)
	if (static_cast<double>(fabs_ref(determinant)) < 1e-8 || length(cross(dp_du, dp_dv)) == 0.f) {
		vec3 fx, fy, fz;
		frame_from_normal(normal, fx, fy, fz);
		dp_du = fx;
		dp_dv = fy;
	}
	vec3 z = normal;
	if (m.flags & MESH_HAS_NORMALS) {
		z = b0 * load3(s.normals, i0) + b1 * load3(s.normals, i1) + b2 * load3(s.normals, i2);
		if (reverse) z = z * -1.f;
		if (length_squared(z) <= 0.f) z = normal;
	}
	vec3 x = dp_du;
	if (m.flags & MESH_HAS_TANGENTS) {
		x = b0 * load3(s.tangents, i0) + b1 * load3(s.tangents, i1) + b2 * load3(s.tangents, i2);
		if (reverse) x = x * -1.f;
		if (length_squared(x) <= 0.f) x = dp_du;
	}
	x = normalize(x);
	z = normalize(z);
	vec3 y = cross(z, x);
	if (length_squared(y) > 0.f) {
		y = normalize(y);
		x = normalize(cross(y, z));
	} else {
		frame_from_normal(z, x, y, z);
	}
	out.sx = x;
	out.sy = y;
	out.sz = z;
	out.n = dot(normal, z) > 0.f ? normal : -normal;  // face_forward(normal, shading z)
	out.dp_du = dp_du;
	return out;
}

// World interaction of hit (slot, b1, b2) on a ray with world direction d.
RB_HD surface_t make_surface(const scene_view& s, int32_t slot, float b1, float b2, vec3 o, vec3 d) {
	const float2 tc = s.tri_c[slot];
	const uint32_t ent = float_as_u32(tc.y) & ~kEntityInvisible;
	const entity_rec& e = s.entities[ent];
	const local_ray lr = make_local_ray(e.w2l, e.l2w, o, d);
	const local_surface ls = triangle_surface(s, s.meshes[e.mesh], s.prim_index[slot], b1, b2);
	surface_t out;
	// transform::operator()(coordinate_system) (transform.cpp:62-76)
	vec3 x = xform_vector(e.l2w, ls.sx);
	vec3 y = xform_vector(e.l2w, ls.sy);
	const vec3 z = normalize(cross(x, y));
	x = normalize(x);
	y = normalize(cross(z, x));
	out.sx = x;
	out.sy = y;
	out.sz = z;
	out.n = xform_normal(e.w2l, ls.n);
	out.p = xform_point(e.l2w, ls.p);
	out.wo = normalize(xform_vector(e.l2w, -lr.d));
	out.entity = static_cast<int32_t>(ent);
	out.uv = ls.uv;
	return out;
}

// ------------------------------------------------------------------ spawning
RB_HD float next_toward(float x, bool up) {
	// std::nextafter(x, up ? FLT_MAX : FLT_MIN): FLT_MIN is the smallest positive
	// normal, so a value below it moves up (interaction.cpp:40-42).
	return nextafterf(x, up ? FLT_MAX : FLT_MIN);
}

// offset_ray_origin (rainbow-cpu/shared/interactions/interaction.cpp:25-46)
RB_HD vec3 offset_origin(vec3 p, vec3 n, vec3 dir) {
	const float scale = kRayEpsilon * (1.f + max_component(vabs(p)));
	vec3 off = scale * n;
	if (dot(n, dir) < 0.f) off = -off;
	vec3 q = p + off;
	q.x = next_toward(q.x, off.x > 0.f);
	q.y = next_toward(q.y, off.y > 0.f);
	q.z = next_toward(q.z, off.z > 0.f);
	return q;
}

// interaction::spawn_ray: ray(direction, offset origin) -> the constructor normalises.
RB_HD ray_t spawn_ray(vec3 p, vec3 n, vec3 dir) {
	ray_t r;
	r.o = offset_origin(p, n, dir);
	r.d = normalize(dir);
	r.len = kInf;
	return r;
}

// interaction::spawn_ray_to (interaction.cpp:17-23)
RB_HD ray_t spawn_ray_to(vec3 p, vec3 n, vec3 target) {
	ray_t r;
	r.o = offset_origin(p, n, normalize(target - p));
	const vec3 dir = target - r.o;
	r.d = normalize(normalize(dir));
	r.len = length(dir) - kShadowEpsilon;
	return r;
}

// world_to_local / local_to_world of a coordinate_system (coordinate_system.cpp:66-78)
RB_HD vec3 to_local(const surface_t& si, vec3 v) { return vec3{dot(v, si.sx), dot(v, si.sy), dot(v, si.sz)}; }
RB_HD vec3 to_world(const surface_t& si, vec3 l) {
	return vec3{si.sx.x * l.x + si.sy.x * l.y + si.sz.x * l.z, si.sx.y * l.x + si.sy.y * l.y + si.sz.y * l.z,
		si.sx.z * l.x + si.sy.z * l.y + si.sz.z * l.z};
}

} // namespace pt
} // namespace rb
