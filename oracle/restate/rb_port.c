/*
 * Plain-C restatement of the reference path integrator (TEST INFRASTRUCTURE).
 *
 * A CPU re-statement of rainbow's unidirectional path tracer, written straight
 * from the reference sources and used only as a checker by the tests and as the
 * "port" CPU baseline: closest-hit traversal of the reference's flattened BVH,
 * entity transforms, Moller-Trumbore, surface interactions, the Lambert /
 * Trowbridge-Reitz conductor and dielectric / Fresnel-specular BSDFs, quad and
 * constant-environment emitters, next-event estimation with MIS, Russian
 * roulette and the PCG32 sampler. It reads the same rb_scene_desc (with its
 * flattened tree) the GPU library takes. Float operations follow the
 * reference's order (with its glm replacement's documented associations);
 * it is compiled without FMA contraction, so with glibc's libm its results
 * equal the compiled reference's bit for bit (checked by the tests).
 *
 * Parity pinning: tests/test_oracle_pin.py compares this file's output with
 * the compiled reference and with the committed golden fixtures.
 */
#include "../../include/rbgpu.h"

#include <float.h>
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

/* ------------------------------------------------------------------ vectors (rainbow-core/math/detail/vector.hpp) */
typedef struct { float x, y, z; } v3;
static v3 V(float x, float y, float z) { v3 r = {x, y, z}; return r; }
static v3 add(v3 a, v3 b) { return V(a.x + b.x, a.y + b.y, a.z + b.z); }
static v3 sub(v3 a, v3 b) { return V(a.x - b.x, a.y - b.y, a.z - b.z); }
static v3 mul(v3 a, v3 b) { return V(a.x * b.x, a.y * b.y, a.z * b.z); }
static v3 muls(v3 a, float s) { return V(a.x * s, a.y * s, a.z * s); }
static v3 divs(v3 a, float s) { return V(a.x / s, a.y / s, a.z / s); }
static v3 neg(v3 a) { return V(-a.x, -a.y, -a.z); }
static float dot3(v3 a, v3 b) { float px = a.x * b.x, py = a.y * b.y, pz = a.z * b.z; return px + py + pz; }
static v3 cross3(v3 a, v3 b) { return V(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y); }
static float len3(v3 a) { return sqrtf(dot3(a, a)); }
static v3 norm3(v3 a) { return muls(a, 1.f / sqrtf(dot3(a, a))); }
static float gmax(float a, float b) { return (a < b) ? b : a; } /* glm max */
static float gmin(float a, float b) { return (b < a) ? b : a; } /* glm min */
static float gabs(float a) { return a >= 0.f ? a : -a; }
static float gclamp(float x, float lo, float hi) { return gmin(gmax(x, lo), hi); }
static int is_black(v3 a) { return a.x == 0.f && a.y == 0.f && a.z == 0.f; }
static float vmaxc(v3 a) { float m = a.x; if (m < a.y) m = a.y; if (m < a.z) m = a.z; return m; }
static v3 ld3(const float* p, uint32_t i) { return V(p[3 * i], p[3 * i + 1], p[3 * i + 2]); }

/* transform_point / transform_vector / transform_normal (rainbow-cpu/shared/transform.cpp:172-188)
 * with the glm replacement's M * v = (M0 x + M1 y) + (M2 z + M3 w). */
static float row4(const float* m, int r, float x, float y, float z, float w) {
	float a0 = m[r] * x + m[4 + r] * y;
	float a1 = m[8 + r] * z + m[12 + r] * w;
	return a0 + a1;
}
static v3 xpoint(const float* m, v3 p) { return V(row4(m, 0, p.x, p.y, p.z, 1.f), row4(m, 1, p.x, p.y, p.z, 1.f), row4(m, 2, p.x, p.y, p.z, 1.f)); }
static v3 xvector(const float* m, v3 p) { return V(row4(m, 0, p.x, p.y, p.z, 0.f), row4(m, 1, p.x, p.y, p.z, 0.f), row4(m, 2, p.x, p.y, p.z, 0.f)); }
/* transpose(inverse) * (n, 0): row r of the transpose is column r of the inverse */
static v3 xnormal(const float* inv, v3 n) {
	float o[3];
	for (int r = 0; r < 3; r++) {
		float a0 = inv[r * 4 + 0] * n.x + inv[r * 4 + 1] * n.y;
		float a1 = inv[r * 4 + 2] * n.z + inv[r * 4 + 3] * 0.f;
		o[r] = a0 + a1;
	}
	return norm3(V(o[0], o[1], o[2]));
}

/* ------------------------------------------------------------------ PCG32 (rainbow-cpu/shared/random_generator.cpp:41-85) */
typedef struct { uint64_t state, inc; } pcg;
static uint32_t pcg_u32(pcg* g) {
	uint64_t old = g->state;
	g->state = old * 0x5851f42d4c957f2dULL + g->inc;
	uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
	uint32_t rot = (uint32_t)(old >> 59u);
	return (xs >> rot) | (xs << ((~rot + 1u) & 31u));
}
static pcg pcg_new(uint64_t seed) {
	pcg g;
	g.state = 0u;
	g.inc = (seed << 1u) | 1u;
	pcg_u32(&g);
	g.state += 0x853c49e6748fea9bULL;
	pcg_u32(&g);
	return g;
}
static float pcg_f(pcg* g) {
	float v = (float)pcg_u32(g) * 2.3283064365386963e-10f;
	float m = 1.f - FLT_EPSILON;
	return (v < m) ? v : m;
}

/* ------------------------------------------------------------------ scene */
typedef struct {
	const rb_scene_desc* d;
	float* area;          /* per entity: mesh::area(transform) */
	int32_t* emitters;    /* entity ordinals with an emitter, in add order */
	int32_t* envs;        /* entity ordinals with an environment emitter */
	uint32_t n_emit, n_env;
	float env_val[2][2], env_cdf[2][3], env_int[2], marg_val[2], marg_cdf[3], marg_int;
} port_scene;

static const rb_mesh_desc* emesh(const port_scene* s, int32_t e) { return &s->d->meshes[s->d->entities[e].mesh]; }
static int visible(const port_scene* s, int32_t e) { return s->d->entities[e].mesh >= 0 && s->d->entities[e].material >= 0; }

static void dist1(const float* v, int n, float* cdf, float* integral) {
	cdf[0] = 0.f;
	for (int i = 1; i <= n; i++) cdf[i] = cdf[i - 1] + v[i - 1] / (float)n;
	*integral = cdf[n];
	for (int i = 1; i <= n; i++) cdf[i] = *integral != 0.f ? cdf[i] / *integral : (float)i / (float)n;
}

static int scene_init(port_scene* s, const rb_scene_desc* d) {
	memset(s, 0, sizeof(*s));
	s->d = d;
	s->area = calloc(d->num_entities + 1, sizeof(float));
	s->emitters = calloc(d->num_entities + 1, sizeof(int32_t));
	s->envs = calloc(d->num_entities + 1, sizeof(int32_t));
	if (!s->area || !s->emitters || !s->envs) return RB_ERR_OUT_OF_MEMORY;
	for (uint32_t e = 0; e < d->num_entities; e++) {
		const rb_entity_desc* ed = &d->entities[e];
		if (ed->mesh >= 0) { /* mesh::area(transform) (rainbow-cpu/shapes/mesh.cpp:131-150) */
			const rb_mesh_desc* m = &d->meshes[ed->mesh];
			float a = 0.f;
			for (uint32_t t = 0; t < m->num_triangles; t++) {
				v3 p0 = xpoint(ed->local_to_world, ld3(m->positions, m->indices[3 * t]));
				v3 p1 = xpoint(ed->local_to_world, ld3(m->positions, m->indices[3 * t + 1]));
				v3 p2 = xpoint(ed->local_to_world, ld3(m->positions, m->indices[3 * t + 2]));
				a = a + 0.5f * len3(cross3(sub(p2, p0), sub(p2, p1)));
			}
			s->area[e] = a;
		}
		if (ed->emitter >= 0) {
			s->emitters[s->n_emit++] = (int32_t)e;
			if (d->emitters[ed->emitter].kind == RB_EMITTER_ENVIRONMENT) s->envs[s->n_env++] = (int32_t)e;
		}
	}
	/* environment_light with a constant map (environment_light.cpp:20-36) */
	const float lum = 1.f * 0.212671f + 1.f * 0.715160f + 1.f * 0.072169f;
	for (int y = 0; y < 2; y++) {
		float st = sinf((((float)y + 0.5f) / 2.f) * 3.14159265358979323846f);
		s->env_val[y][0] = s->env_val[y][1] = lum * st;
		dist1(s->env_val[y], 2, s->env_cdf[y], &s->env_int[y]);
	}
	s->marg_val[0] = s->env_int[0];
	s->marg_val[1] = s->env_int[1];
	dist1(s->marg_val, 2, s->marg_cdf, &s->marg_int);
	return s->n_emit ? RB_OK : RB_ERR_INVALID_ARGUMENT;
}
static void scene_free(port_scene* s) { free(s->area); free(s->emitters); free(s->envs); }

/* ------------------------------------------------------------------ intersection */
typedef struct { v3 o, d; float len; } ray;

/* mesh::intersect_with_triangle's test (rainbow-cpu/shapes/mesh.cpp:328-348) */
static int tri_test(v3 o, v3 d, float len, v3 p0, v3 p1, v3 p2, float* t, float* b1, float* b2) {
	v3 e1 = sub(p1, p0), e2 = sub(p2, p0);
	v3 pv = cross3(d, e2), tv = sub(o, p0), qv = cross3(tv, e1);
	float inv_det = 1.f / dot3(e1, pv);
	*b1 = dot3(tv, pv) * inv_det;
	*b2 = dot3(d, qv) * inv_det;
	float b0 = 1.f - *b1 - *b2;
	*t = dot3(e2, qv) * inv_det;
	if (*t <= 0.f || *t >= len) return 0;
	if (b0 < 0.f || b0 > 1.f) return 0;
	if (*b1 < 0.f || *b1 > 1.f) return 0;
	if (*b2 < 0.f || *b2 > 1.f) return 0;
	return 1;
}

static void tri_points(const rb_mesh_desc* m, uint32_t t, v3* p0, v3* p1, v3* p2) {
	*p0 = ld3(m->positions, m->indices[3 * t]);
	*p1 = ld3(m->positions, m->indices[3 * t + 1]);
	*p2 = ld3(m->positions, m->indices[3 * t + 2]);
}

/* entity::intersect(ray, index) (rainbow-cpu/scenes/entity.cpp:18-37): world -> local ray
 * (direction normalised by the transform and again by the ray constructor), test,
 * world length = local t * |L2W d_local|. Returns 1 and updates r->len on a hit. */
static int entity_tri(const port_scene* s, int32_t e, uint32_t t, ray* r, float* b1, float* b2) {
	const rb_entity_desc* ed = &s->d->entities[e];
	v3 dl = xvector(ed->world_to_local, r->d);
	v3 d = norm3(norm3(dl));
	v3 o = xpoint(ed->world_to_local, r->o);
	float llen = r->len * len3(dl);
	v3 p0, p1, p2;
	tri_points(emesh(s, e), t, &p0, &p1, &p2);
	float th;
	if (!tri_test(o, d, llen, p0, p1, p2, &th, b1, b2)) return 0;
	r->len = th * len3(xvector(ed->local_to_world, d));
	return 1;
}

/* bounding_box<T>::intersect (rainbow-cpu/shared/accelerators/detail/accelerator.hpp:29-53) */
static int box_test(const float* nd, const ray* r) {
	float t0 = 0.f, t1 = r->len;
	const float o[3] = {r->o.x, r->o.y, r->o.z}, dd[3] = {r->d.x, r->d.y, r->d.z};
	for (int k = 0; k < 3; k++) {
		float inv = 1.f / dd[k];
		float nn = (nd[k] - o[k]) * inv, ff = (nd[3 + k] - o[k]) * inv;
		if (nn > ff) { float t = nn; nn = ff; ff = t; }
		t0 = gmax(t0, nn);
		t1 = gmin(t1, ff);
		if (t0 > t1) return 0;
	}
	return 1;
}

typedef struct { int32_t ent, tri; float b1, b2; } hitrec;

/* bounding_volume_hierarchy<T>::intersect / _with_shadow_ray
 * (rainbow-cpu/shared/accelerators/detail/bounding_volume_hierarchy.hpp:60-160) */
static hitrec bvh_hit(const port_scene* s, ray* r, int shadow) {
	const rb_bvh_desc* b = &s->d->bvh;
	hitrec h = {-1, -1, 0.f, 0.f};
	uint32_t stack[256];
	int sp = 0;
	stack[sp++] = 0;
	v3 inv = V(1.f / r->d.x, 1.f / r->d.y, 1.f / r->d.z);
	int negd[3] = {inv.x < 0.f, inv.y < 0.f, inv.z < 0.f};
	while (sp > 0) {
		uint32_t n = stack[--sp];
		const float* nd = b->nodes + 8ull * n;
		if (!box_test(nd, r)) continue;
		uint32_t w0, w1;
		memcpy(&w0, nd + 6, 4);
		memcpy(&w1, nd + 7, 4);
		if (w1 & RB_BVH_LEAF_FLAG) {
			for (uint32_t k = 0; k < (w1 & ~RB_BVH_LEAF_FLAG); k++) {
				int32_t e = (int32_t)b->prim_entity[w0 + k];
				uint32_t t = b->prim_index[w0 + k];
				if (shadow && !visible(s, e)) continue;
				float b1, b2;
				if (entity_tri(s, e, t, r, &b1, &b2)) { h.ent = e; h.tri = (int32_t)t; h.b1 = b1; h.b2 = b2; }
			}
			continue;
		}
		if (sp + 2 > 256) break;
		if (negd[w1]) { stack[sp++] = n + 1; stack[sp++] = w0; }
		else { stack[sp++] = w0; stack[sp++] = n + 1; }
	}
	return h;
}

/* ------------------------------------------------------------------ surface interaction */
typedef struct { v3 p, n, x, y, z, wo; int32_t ent; } surf;

/* coordinate_system(normal) (rainbow-cpu/shared/coordinate_system.cpp:8-23) */
static void frame_of(v3 nrm, v3* x, v3* y, v3* z) {
	*z = norm3(nrm);
	if (gabs(z->x) > gabs(z->y)) *x = divs(V(-z->z, 0.f, z->x), sqrtf(z->x * z->x + z->z * z->z));
	else *x = divs(V(0.f, z->z, -z->y), sqrtf(z->y * z->y + z->z * z->z));
	*y = cross3(*z, *x);
}

/* mesh::intersect_with_triangle's interaction (mesh.cpp:350-441), in local space */
static void local_surface(const rb_mesh_desc* m, uint32_t t, float b1, float b2, v3 ray_d, surf* out) {
	uint32_t i0 = m->indices[3 * t], i1 = m->indices[3 * t + 1], i2 = m->indices[3 * t + 2];
	v3 p0 = ld3(m->positions, i0), p1 = ld3(m->positions, i1), p2 = ld3(m->positions, i2);
	v3 u0 = V(0, 0, 0), u1 = V(1, 0, 0), u2 = V(1, 1, 0);
	if (m->uvs) { u0 = ld3(m->uvs, i0); u1 = ld3(m->uvs, i1); u2 = ld3(m->uvs, i2); }
	v3 e1 = sub(p1, p0), e2 = sub(p2, p0);
	float b0 = 1.f - b1 - b2;
	out->p = add(add(muls(p0, b0), muls(p1, b1)), muls(p2, b2));
	v3 normal = m->reverse_orientation ? neg(norm3(cross3(e1, e2))) : norm3(cross3(e1, e2));
	v3 duv02 = sub(u0, u2), duv12 = sub(u1, u2), dp02 = sub(p0, p2), dp12 = sub(p1, p2);
	float det = duv02.x * duv12.y - duv02.y * duv12.x;
	float inv = 1.f / det;
	v3 dpdu = muls(sub(muls(dp02, duv12.y), muls(dp12, duv02.y)), inv);
	v3 dpdv = muls(add(muls(dp02, -duv12.x), muls(dp12, duv02.x)), inv);
	if ((double)gabs(det) < 1e-8 || len3(cross3(dpdu, dpdv)) == 0.f) {
		v3 fx, fy, fz;
		frame_of(normal, &fx, &fy, &fz);
		dpdu = fx;
	}
	v3 z = normal, x = dpdu;
	if (m->normals) {
		z = add(add(muls(ld3(m->normals, i0), b0), muls(ld3(m->normals, i1), b1)), muls(ld3(m->normals, i2), b2));
		if (m->reverse_orientation) z = muls(z, -1.f);
		if (dot3(z, z) <= 0.f) z = normal;
	}
	if (m->tangents) {
		x = add(add(muls(ld3(m->tangents, i0), b0), muls(ld3(m->tangents, i1), b1)), muls(ld3(m->tangents, i2), b2));
		if (m->reverse_orientation) x = muls(x, -1.f);
		if (dot3(x, x) <= 0.f) x = dpdu;
	}
	x = norm3(x);
	z = norm3(z);
	v3 y = cross3(z, x);
	if (dot3(y, y) > 0.f) { y = norm3(y); x = norm3(cross3(y, z)); }
	else frame_of(z, &x, &y, &z);
	out->x = x; out->y = y; out->z = z;
	out->n = dot3(normal, z) > 0.f ? normal : neg(normal);
	out->wo = neg(ray_d);
}

/* the world interaction: transform::operator()(surface_interaction) (transform.cpp:38-76) */
static surf world_surface(const port_scene* s, hitrec h, v3 ray_o, v3 ray_d) {
	const rb_entity_desc* ed = &s->d->entities[h.ent];
	v3 dl = norm3(norm3(xvector(ed->world_to_local, ray_d)));
	surf l, w;
	local_surface(emesh(s, h.ent), (uint32_t)h.tri, h.b1, h.b2, dl, &l);
	v3 x = xvector(ed->local_to_world, l.x), y = xvector(ed->local_to_world, l.y);
	w.z = norm3(cross3(x, y));
	w.x = norm3(x);
	w.y = norm3(cross3(w.z, w.x));
	w.n = xnormal(ed->world_to_local, l.n);
	w.p = xpoint(ed->local_to_world, l.p);
	w.wo = norm3(xvector(ed->local_to_world, l.wo));
	w.ent = h.ent;
	(void)ray_o;
	return w;
}

static v3 to_local(const surf* si, v3 v) { return V(dot3(v, si->x), dot3(v, si->y), dot3(v, si->z)); }
static v3 to_world(const surf* si, v3 l) {
	return V(si->x.x * l.x + si->y.x * l.y + si->z.x * l.z, si->x.y * l.x + si->y.y * l.y + si->z.y * l.z,
		si->x.z * l.x + si->y.z * l.y + si->z.z * l.z);
}

/* offset_ray_origin / spawn_ray / spawn_ray_to (rainbow-cpu/shared/interactions/interaction.cpp:12-46) */
static const float RAY_EPS = FLT_EPSILON / 2 * 1500;
static v3 offset_origin(v3 p, v3 n, v3 dir) {
	float sc = RAY_EPS * (1.f + vmaxc(V(gabs(p.x), gabs(p.y), gabs(p.z))));
	v3 off = muls(n, sc);
	off = V(sc * n.x, sc * n.y, sc * n.z);
	if (dot3(n, dir) < 0.f) off = neg(off);
	v3 q = add(p, off);
	q.x = nextafterf(q.x, off.x > 0.f ? FLT_MAX : FLT_MIN);
	q.y = nextafterf(q.y, off.y > 0.f ? FLT_MAX : FLT_MIN);
	q.z = nextafterf(q.z, off.z > 0.f ? FLT_MAX : FLT_MIN);
	return q;
}
static ray spawn(v3 p, v3 n, v3 dir) { ray r; r.o = offset_origin(p, n, dir); r.d = norm3(dir); r.len = INFINITY; return r; }
static ray spawn_to(v3 p, v3 n, v3 target) {
	ray r;
	r.o = offset_origin(p, n, norm3(sub(target, p)));
	v3 dir = sub(target, r.o);
	r.d = norm3(norm3(dir));
	r.len = len3(dir) - RAY_EPS * 10;
	return r;
}

/* ------------------------------------------------------------------ BSDFs (rainbow-cpu/scatterings/) */
enum { T_REFL = 1, T_TRANS = 2, T_SPEC = 4, T_DIFF = 8, T_GLOSSY = 16, T_ALL = 31 };
enum { L_LAMBERT, L_MFR, L_MFT, L_FSPEC };
typedef struct { int kind[2], type[2], n; float ax, ay, eta; const rb_material_desc* m; } bsdf;
typedef struct { int type; v3 f, wi; float pdf; } bsample;
static int tmatch(int t, int f) { return (t & f) == f; }

static float roughness_alpha(float r) { /* trowbridge_reitz_distribution.cpp:128-137 */
	r = gmax(r, 1e-3f);
	float x = logf(r);
	return 1.62142f + 0.819955f * x + 0.1734f * x * x + 0.0171201f * x * x * x + 0.000640711f * x * x * x * x;
}

/* materials: matte_material.cpp:13-29, metal_material.cpp:17-37, glass_material.cpp:25-64 */
static bsdf make_bsdf(const rb_material_desc* m) {
	bsdf b;
	memset(&b, 0, sizeof(b));
	b.m = m;
	b.eta = 1.f;
	if (m->kind == RB_MATERIAL_MATTE) {
		if (!(m->diffuse[0] == 0.f && m->diffuse[1] == 0.f && m->diffuse[2] == 0.f)) {
			b.kind[0] = L_LAMBERT; b.type[0] = T_DIFF | T_REFL; b.n = 1;
		}
	} else if (m->kind == RB_MATERIAL_METAL) {
		b.ax = m->remap_roughness ? roughness_alpha(m->roughness_u) : m->roughness_u;
		b.ay = m->remap_roughness ? roughness_alpha(m->roughness_v) : m->roughness_v;
		b.kind[0] = L_MFR; b.type[0] = T_GLOSSY | T_REFL; b.n = 1;
	} else {
		b.eta = m->ior;
		int rb = !(m->reflectance[0] == 0.f && m->reflectance[1] == 0.f && m->reflectance[2] == 0.f);
		int tb = !(m->transmission[0] == 0.f && m->transmission[1] == 0.f && m->transmission[2] == 0.f);
		if (!rb && !tb) return b;
		if (m->roughness_u == 0.f && m->roughness_v == 0.f) {
			b.kind[0] = L_FSPEC; b.type[0] = T_REFL | T_TRANS | T_SPEC; b.n = 1;
			return b;
		}
		b.ax = m->remap_roughness ? roughness_alpha(m->roughness_u) : m->roughness_u;
		b.ay = m->remap_roughness ? roughness_alpha(m->roughness_v) : m->roughness_v;
		if (rb) { b.kind[b.n] = L_MFR; b.type[b.n] = T_GLOSSY | T_REFL; b.n++; }
		if (tb) { b.kind[b.n] = L_MFT; b.type[b.n] = T_GLOSSY | T_TRANS; b.n++; }
	}
	return b;
}

/* shading_function.cpp */
static float cos2t(v3 w) { return w.z * w.z; }
static float sin2t(v3 w) { return gmax(0.f, 1.f - cos2t(w)); }
static float sint(v3 w) { return sqrtf(sin2t(w)); }
static float tant(v3 w) { return sint(w) / w.z; }
static float tan2t(v3 w) { return sin2t(w) / cos2t(w); }
static float cosp(v3 w) { float s = sint(w); return s == 0.f ? 1.f : gclamp(w.x / s, -1.f, 1.f); }
static float sinp(v3 w) { float s = sint(w); return s == 0.f ? 0.f : gclamp(w.y / s, -1.f, 1.f); }
static int same_hemi(v3 a, v3 b) { return a.z * b.z > 0.f; }
static v3 ffwd(v3 v, v3 f) { return dot3(v, f) > 0.f ? v : neg(v); }
static v3 reflectv(v3 wi, v3 n) { return add(neg(wi), muls(n, 2.f * dot3(wi, n))); }
static v3 refractv(v3 wi, v3 n, float eta) {
	float ci = dot3(wi, n);
	float s2o = gmax(0.f, 1.f - ci * ci) * eta * eta;
	if (s2o >= 1.f) return V(0, 0, 0);
	float co = sqrtf(1.f - s2o);
	return add(muls(neg(wi), eta), muls(n, ci * eta - co));
}
/* sample_function.cpp:15-44 */
static void disk(float ux, float uy, float* dx, float* dy) {
	float rx = 2.f * ux - 1.f, ry = 2.f * uy - 1.f, th, r;
	if (rx == 0.f && ry == 0.f) { *dx = 0.f; *dy = 0.f; return; }
	if (gabs(rx) > gabs(ry)) { r = rx; th = 0.785398163397448309616f * (ry / rx); }
	else { r = ry; th = 1.57079632679489661923f - 0.785398163397448309616f * (rx / ry); }
	*dx = r * cosf(th);
	*dy = r * sinf(th);
}
static v3 cos_hemi(float ux, float uy) {
	float dx, dy;
	disk(ux, uy, &dx, &dy);
	float pdx = dx * dx, pdy = dy * dy;
	return V(dx, dy, sqrtf(gmax(0.f, 1.f - (pdx + pdy))));
}

/* trowbridge_reitz_distribution.cpp, microfacet_distribution.cpp */
static float tr_D(float ax, float ay, v3 wh) {
	float t2 = tan2t(wh);
	if (isinf(t2)) return 0.f;
	float c4 = cos2t(wh) * cos2t(wh);
	float cp = cosp(wh), sp = sinp(wh);
	float e = (cp * cp / (ax * ax) + sp * sp / (ay * ay)) * t2;
	return 1.f / (3.14159265358979323846f * ax * ay * c4 * (1.f + e) * (1.f + e));
}
static float tr_L(float ax, float ay, v3 w) {
	float at = gabs(tant(w));
	if (isinf(at)) return 0.f;
	float cp = cosp(w), sp = sinp(w);
	float al = sqrtf(cp * cp * ax * ax + sp * sp * ay * ay);
	float a2 = (al * at) * (al * at);
	return (-1.f + sqrtf(1.f + a2)) / 2.f;
}
static float tr_G(float ax, float ay, v3 wo, v3 wi) { return 1.f / (1.f + tr_L(ax, ay, wo) + tr_L(ax, ay, wi)); }
static float tr_pdf(float ax, float ay, v3 wo, v3 wh) {
	return tr_D(ax, ay, wh) * (1.f / (1.f + tr_L(ax, ay, wo))) * gabs(dot3(wo, wh)) / gabs(wo.z);
}
static void tr_slope(float ct, float u1, float u2, float* sx, float* sy) {
	if ((double)ct > 0.9999) {
		float r = sqrtf(u1 / (1.f - u1)), phi = 6.28318530717958647692f * u2;
		*sx = r * cosf(phi); *sy = r * sinf(phi);
		return;
	}
	float st = sqrtf(gmax(0.f, 1.f - ct * ct)), tt = st / ct, a = 1.f / tt;
	float g1 = 2.f / (1.f + sqrtf(1.f + 1.f / (a * a)));
	float A = 2.f * u1 / g1 - 1.f;
	float tmp = 1.f / (A * A - 1.f);
	if ((double)tmp > 1e10) tmp = 1e10f;
	float B = tt;
	float D = sqrtf(gmax(B * B * tmp * tmp - (A * A - B * B) * tmp, 0.f));
	float x1 = B * tmp - D, x2 = B * tmp + D;
	*sx = (A < 0.f || x2 > 1.f / tt) ? x1 : x2;
	float S;
	if (u2 > 0.5f) { S = 1.f; u2 = 2.f * (u2 - .5f); } else { S = -1.f; u2 = 2.f * (.5f - u2); }
	float z = (u2 * (u2 * (u2 * 0.27385f - 0.73369f) + 0.46341f)) / (u2 * (u2 * (u2 * 0.093073f + 0.309420f) - 1.000000f) + 0.597999f);
	*sy = S * z * sqrtf(1.f + *sx * *sx);
}
static v3 tr_sample(float ax, float ay, v3 wo, float u1, float u2) {
	int flip = wo.z < 0.f;
	v3 wi = flip ? neg(wo) : wo;
	v3 ws = norm3(V(ax * wi.x, ay * wi.y, wi.z));
	float sx, sy;
	tr_slope(ws.z, u1, u2, &sx, &sy);
	float tmp = cosp(ws) * sx - sinp(ws) * sy;
	sy = sinp(ws) * sx + cosp(ws) * sy;
	sx = tmp;
	sx = ax * sx;
	sy = ay * sy;
	v3 wh = norm3(V(-sx, -sy, 1.f));
	return flip ? neg(wh) : wh;
}
/* fresnel_effect.cpp */
static float fr_diel(float ci, float ei, float eo) {
	ci = gclamp(ci, -1.f, 1.f);
	if (ci < 0.f) { float t = ei; ei = eo; eo = t; ci = gabs(ci); }
	float si = sqrtf(gmax(0.f, 1.f - ci * ci));
	float so = si * ei / eo;
	float co = sqrtf(gmax(0.f, 1.f - so * so));
	if (so >= 1.f) return 1.f;
	float r0 = (eo * ci - ei * co) / (eo * ci + ei * co);
	float r1 = (ei * ci - eo * co) / (ei * ci + eo * co);
	return (r0 * r0 + r1 * r1) / 2.f;
}
static float fr_cond1(float ci, float eta, float k) {
	ci = gclamp(ci, -1.f, 1.f);
	float e = eta / 1.f, ek = k / 1.f, c2 = ci * ci, s2 = 1.f - c2, e2 = e * e, ek2 = ek * ek;
	float t0 = e2 - ek2 - s2;
	float ab = sqrtf(t0 * t0 + e2 * ek2 * 4.f);
	float t1 = ab + c2, a = sqrtf((ab + t0) * 0.5f), t2 = a * 2.f * ci;
	float t3 = ab * c2 + s2 * s2, t4 = t2 * s2;
	float r0 = (t1 - t2) / (t1 + t2);
	float r1 = r0 * (t3 - t4) / (t3 + t4);
	return (r0 + r1) * 0.5f;
}

static v3 mfr_f(const bsdf* b, v3 wo, v3 wi) { /* microfacet_reflection.cpp:13-36 */
	float co = gabs(wo.z), ci = gabs(wi.z);
	v3 wh = add(wi, wo);
	if (co == 0.f || ci == 0.f) return V(0, 0, 0);
	if (wh.x == 0.f && wh.y == 0.f && wh.z == 0.f) return V(0, 0, 0);
	wh = ffwd(norm3(wh), V(0, 0, 1));
	v3 F, R;
	if (b->m->kind == RB_MATERIAL_METAL) {
		float c = gabs(dot3(wi, wh));
		F = V(fr_cond1(c, b->m->eta[0], b->m->k[0]), fr_cond1(c, b->m->eta[1], b->m->k[1]), fr_cond1(c, b->m->eta[2], b->m->k[2]));
		R = V(1, 1, 1);
	} else {
		float f = fr_diel(dot3(wi, wh), 1.f, b->eta);
		F = V(f, f, f);
		R = V(b->m->reflectance[0], b->m->reflectance[1], b->m->reflectance[2]);
	}
	float G = tr_G(b->ax, b->ay, wo, wi), D = tr_D(b->ax, b->ay, wh);
	return divs(mul(muls(R, G * D), F), 4.f * ci * co);
}
static float mfr_pdf(const bsdf* b, v3 wo, v3 wi) {
	if (!same_hemi(wo, wi)) return 0.f;
	v3 wh = norm3(add(wo, wi));
	return tr_pdf(b->ax, b->ay, wo, wh) / (4.f * dot3(wo, wh));
}
static v3 mft_f(const bsdf* b, v3 wo, v3 wi) { /* microfacet_transmission.cpp:14-39 */
	if (same_hemi(wo, wi)) return V(0, 0, 0);
	float co = wo.z, ci = wi.z;
	if (co == 0.f || ci == 0.f) return V(0, 0, 0);
	float eta = co > 0.f ? (b->eta / 1.f) : (1.f / b->eta);
	v3 wh = ffwd(norm3(add(wo, muls(wi, eta))), V(0, 0, 1));
	float F = fr_diel(dot3(wo, wh), 1.f, b->eta);
	float den = dot3(wo, wh) + eta * dot3(wi, wh);
	float fac = 1.f / eta;
	float D = tr_D(b->ax, b->ay, wh), G = tr_G(b->ax, b->ay, wo, wi);
	float v = gabs(D * G * eta * eta * gabs(dot3(wi, wh)) * gabs(dot3(wo, wh) * fac * fac) / (ci * co * den * den));
	v3 one_minus_F = V(1.f - F, 1.f - F, 1.f - F);
	return muls(mul(one_minus_F, V(b->m->transmission[0], b->m->transmission[1], b->m->transmission[2])), v);
}
static float mft_pdf(const bsdf* b, v3 wo, v3 wi) {
	if (same_hemi(wo, wi)) return 0.f;
	float eta = wo.z > 0.f ? (b->eta / 1.f) : (1.f / b->eta);
	v3 wh = norm3(add(wo, muls(wi, eta)));
	float den = dot3(wo, wh) + eta * dot3(wi, wh);
	return tr_pdf(b->ax, b->ay, wo, wh) * gabs((eta * eta * dot3(wi, wh)) / (den * den));
}
static v3 lobe_f(const bsdf* b, int i, v3 wo, v3 wi) {
	if (b->kind[i] == L_LAMBERT) return muls(V(b->m->diffuse[0], b->m->diffuse[1], b->m->diffuse[2]), 0.318309886183790671538f);
	if (b->kind[i] == L_MFR) return mfr_f(b, wo, wi);
	if (b->kind[i] == L_MFT) return mft_f(b, wo, wi);
	return V(0, 0, 0);
}
static float lobe_pdf(const bsdf* b, int i, v3 wo, v3 wi) {
	if (b->kind[i] == L_LAMBERT) return same_hemi(wo, wi) ? gabs(wi.z) * 0.318309886183790671538f : 0.f;
	if (b->kind[i] == L_MFR) return mfr_pdf(b, wo, wi);
	if (b->kind[i] == L_MFT) return mft_pdf(b, wo, wi);
	return 0.f;
}
static bsample none(void) { bsample s; memset(&s, 0, sizeof(s)); return s; }
static bsample lobe_sample(const bsdf* b, int i, v3 wo, float ux, float uy) {
	bsample s = none();
	s.type = b->type[i];
	if (b->kind[i] == L_LAMBERT) { /* reflection_function::sample (reflection_function.cpp:12-24) */
		v3 wi = cos_hemi(ux, uy);
		if (wo.z < 0.f) wi.z = -wi.z;
		s.wi = wi; s.f = lobe_f(b, i, wo, wi); s.pdf = lobe_pdf(b, i, wo, wi);
		return s;
	}
	if (b->kind[i] == L_MFR) { /* microfacet_reflection::sample (:38-62) */
		if (wo.z == 0.f) return none();
		v3 wh = tr_sample(b->ax, b->ay, wo, ux, uy);
		if (dot3(wo, wh) < 0.f) return none();
		v3 wi = reflectv(wo, wh);
		if (!same_hemi(wo, wi)) return none();
		s.wi = wi; s.f = mfr_f(b, wo, wi); s.pdf = tr_pdf(b->ax, b->ay, wo, wh) / (4.f * dot3(wo, wh));
		return s;
	}
	if (b->kind[i] == L_MFT) { /* microfacet_transmission::sample (:41-63) */
		if (wo.z == 0.f) return none();
		v3 wh = tr_sample(b->ax, b->ay, wo, ux, uy);
		if (dot3(wo, wh) < 0.f) return none();
		float eta = wo.z > 0.f ? (1.f / b->eta) : (b->eta / 1.f);
		v3 wi = refractv(wo, wh, eta);
		if (is_black(wi)) return none();
		s.wi = wi; s.f = mft_f(b, wo, wi); s.pdf = mft_pdf(b, wo, wi);
		return s;
	}
	/* fresnel_specular::sample (fresnel_specular.cpp:25-54) */
	float F = fr_diel(wo.z, 1.f, b->eta);
	if (ux < F) {
		v3 wi = V(-wo.x, -wo.y, wo.z);
		s.type = T_REFL | T_SPEC;
		s.wi = wi;
		s.f = divs(muls(V(b->m->reflectance[0], b->m->reflectance[1], b->m->reflectance[2]), F), gabs(wi.z));
		s.pdf = F;
		return s;
	}
	int entering = wo.z > 0.f;
	float ei = entering ? 1.f : b->eta, eo = entering ? b->eta : 1.f;
	v3 wi = refractv(wo, ffwd(V(0, 0, 1), wo), ei / eo);
	if (is_black(wi)) return none();
	float fac = (ei * ei) / (eo * eo);
	s.type = T_TRANS | T_SPEC;
	s.wi = wi;
	s.f = divs(muls(mul(V(b->m->transmission[0], b->m->transmission[1], b->m->transmission[2]), V(1.f - F, 1.f - F, 1.f - F)), fac), gabs(wi.z));
	s.pdf = 1.f - F;
	return s;
}

/* scattering_function_collection (scattering_function_collection.cpp:29-148) */
static v3 coll_f(const bsdf* b, v3 wo, v3 wi, int include) {
	if (wo.z == 0.f) return V(0, 0, 0);
	int rt = same_hemi(wo, wi) ? T_REFL : T_TRANS;
	v3 f = V(0, 0, 0);
	for (int i = 0; i < b->n; i++)
		if (tmatch(include, b->type[i]) && tmatch(b->type[i], rt)) f = add(f, lobe_f(b, i, wo, wi));
	return f;
}
static float coll_pdf(const bsdf* b, v3 wo, v3 wi, int include) {
	if (b->n == 0 || wo.z == 0.f) return 0.f;
	int c = 0;
	float pdf = 0.f;
	for (int i = 0; i < b->n; i++)
		if (tmatch(include, b->type[i])) { pdf = pdf + lobe_pdf(b, i, wo, wi); c++; }
	return c ? pdf / (float)c : 0.f;
}
static int coll_count(const bsdf* b, int include) {
	int c = 0;
	for (int i = 0; i < b->n; i++) c += tmatch(include, b->type[i]);
	return c;
}
/* sample with wo already in the shading frame; wi returned in the shading frame */
static bsample coll_sample(const bsdf* b, v3 wo, float ux, float uy, int include) {
	int idx[2], n = 0;
	for (int i = 0; i < b->n; i++) if (tmatch(include, b->type[i])) idx[n++] = i;
	if (n == 0) return none();
	uint32_t which = (uint32_t)floorf(ux * (float)n);
	if (which > (uint32_t)n - 1) which = (uint32_t)n - 1;
	float rx = ux * (float)n - (float)which;
	float m = 1.f - FLT_EPSILON;
	rx = (m < rx) ? m : rx;
	if (wo.z == 0.f) return none();
	bsample s = lobe_sample(b, idx[which], wo, rx, uy);
	if (s.pdf == 0.f) return none();
	if (!tmatch(s.type, T_SPEC)) {
		int rt = same_hemi(wo, s.wi) ? T_REFL : T_TRANS;
		s.f = V(0, 0, 0);
		s.pdf = 0.f;
		for (int k = 0; k < n; k++) {
			int i = idx[k];
			if (tmatch(b->type[i], rt)) s.f = add(s.f, lobe_f(b, i, wo, s.wi));
			s.pdf = s.pdf + lobe_pdf(b, i, wo, s.wi);
		}
	}
	s.pdf = s.pdf / (float)n;
	return s;
}

/* ------------------------------------------------------------------ emitters */
static float env_dist_sample1(const float* cdf, const float* val, float integral, float u, int* off, float* pdf) {
	int i = 0;
	while (i < 3 && !(u < cdf[i])) i++;
	*off = i - 1;
	float du = u - cdf[*off];
	if (*off < 2 && cdf[*off + 1] - cdf[*off] > 0.f) du = du / (cdf[*off + 1] - cdf[*off]);
	*pdf = integral > 0.f ? val[*off] / integral : 0.f;
	return ((float)*off + du) / 2.f;
}
/* environment_light::pdf(properties, reference, wi) (environment_light.cpp:130-149) */
static float env_pdf(const port_scene* s, v3 wi) {
	v3 w = norm3(wi);
	float th = acosf(gclamp(w.z, -1.f, 1.f));
	float ph = atan2f(w.y, w.x);
	ph = ph < 0.f ? ph + 6.28318530717958647692f : ph;
	float st = sinf(th);
	if (st == 0.f) return 0.f;
	uint32_t x = (uint32_t)(ph * 0.159154943091895335769f * 2.f), y = (uint32_t)(th * 0.318309886183790671538f * 2.f);
	if (x > 1) x = 1;
	if (y > 1) y = 1;
	return (s->env_val[y][x] / s->marg_int) / (6.28318530717958647692f * 3.14159265358979323846f * st);
}

typedef struct { v3 p, wi, L; float pdf; } lsample;

/* entity::sample<emitter>(reference, u) (scenes/detail/entity.hpp:52-61) with
 * surface_light::sample -> shape::sample -> mesh::sample (surface_light.cpp:39-54,
 * shape.cpp:26-44, mesh.cpp:84-116) or environment_light::sample (:85-107). */
static lsample sample_light(const port_scene* s, int32_t e, v3 rp, v3 rn, float u0, float u1) {
	lsample out;
	memset(&out, 0, sizeof(out));
	const rb_entity_desc* ed = &s->d->entities[e];
	const rb_emitter_desc* em = &s->d->emitters[ed->emitter];
	v3 pl = xpoint(ed->world_to_local, rp);
	(void)rn;
	if (em->kind == RB_EMITTER_SURFACE) {
		const rb_mesh_desc* m = emesh(s, e);
		float fc = (float)m->num_triangles;
		uint32_t which = (uint32_t)floorf(u0 * fc);
		if (which > m->num_triangles - 1) which = m->num_triangles - 1;
		float rx = u0 * fc - (float)which, mx = 1.f - FLT_EPSILON;
		rx = (mx < rx) ? mx : rx;
		v3 p0, p1, p2;
		tri_points(m, which, &p0, &p1, &p2);
		float su = sqrtf(rx), b0 = 1.f - su, b1 = u1 * su;
		v3 pt = add(add(muls(p0, b0), muls(p1, b1)), muls(p2, 1.f - b0 - b1));
		v3 nrm = norm3(cross3(sub(p1, p0), sub(p2, p0)));
		if (m->normals) {
			uint32_t i0 = m->indices[3 * which], i1 = m->indices[3 * which + 1], i2 = m->indices[3 * which + 2];
			nrm = add(add(muls(ld3(m->normals, i0), b0), muls(ld3(m->normals, i1), b1)), muls(ld3(m->normals, i2), 1.f - b0 - b1));
		}
		if (m->reverse_orientation) nrm = muls(nrm, -1.f);
		float pdf = 1.f / s->area[e];
		v3 wi = sub(pt, pl);
		if (dot3(wi, wi) == 0.f) return out;
		wi = norm3(wi);
		v3 dd = sub(pl, pt);
		pdf = pdf * dot3(dd, dd) / gabs(dot3(nrm, neg(wi)));
		if (isinf(pdf) || pdf == 0.f) return out;
		v3 wl = norm3(sub(pt, pl));
		out.L = dot3(nrm, neg(wl)) > 0.f ? V(em->radiance[0], em->radiance[1], em->radiance[2]) : V(0, 0, 0);
		out.p = xpoint(ed->local_to_world, pt);
		out.wi = xvector(ed->local_to_world, wl);
		out.pdf = pdf;
		return out;
	}
	int oy, ox;
	float py, px;
	float vy = env_dist_sample1(s->marg_cdf, s->marg_val, s->marg_int, u1, &oy, &py);
	float vx = env_dist_sample1(s->env_cdf[oy], s->env_val[oy], s->env_int[oy], u0, &ox, &px);
	float dp = px * py;
	if (dp == 0.f) return out;
	float th = vy * 3.14159265358979323846f, ph = vx * 6.28318530717958647692f;
	float ct = cosf(th), st = sinf(th);
	float pdf = st != 0.f ? dp / (6.28318530717958647692f * 3.14159265358979323846f * st) : 0.f;
	v3 wi = V(st * cosf(ph), st * sinf(ph), ct);
	v3 pt = add(pl, muls(wi, 2.f * em->radius));
	out.p = xpoint(ed->local_to_world, pt);
	out.wi = xvector(ed->local_to_world, wi);
	out.L = V(em->radiance[0], em->radiance[1], em->radiance[2]);
	out.pdf = pdf;
	return out;
}

/* entity::evaluate<emitter> for a surface light (surface_light.cpp:12-16) */
static v3 surface_Le(const port_scene* s, int32_t e, v3 n_world, v3 w_world) {
	const rb_entity_desc* ed = &s->d->entities[e];
	const rb_emitter_desc* em = &s->d->emitters[ed->emitter];
	v3 nl = xnormal(ed->local_to_world, n_world);
	v3 wl = xvector(ed->world_to_local, w_world);
	return dot3(nl, wl) > 0.f ? V(em->radiance[0], em->radiance[1], em->radiance[2]) : V(0, 0, 0);
}

/* entity::pdf<emitter>(reference, wi) (scenes/detail/entity.hpp:63-71) */
static float emitter_pdf(const port_scene* s, int32_t e, v3 rp, v3 rn, v3 wi_world) {
	const rb_entity_desc* ed = &s->d->entities[e];
	const rb_emitter_desc* em = &s->d->emitters[ed->emitter];
	v3 wl = xvector(ed->world_to_local, wi_world);
	if (em->kind == RB_EMITTER_ENVIRONMENT) return env_pdf(s, wl);
	/* shape::pdf (shape.cpp:46-60): re-intersect the emitter mesh in local space */
	v3 pl = xpoint(ed->world_to_local, rp), nl = xnormal(ed->local_to_world, rn);
	ray r = spawn(pl, nl, wl);
	const rb_mesh_desc* m = emesh(s, e);
	int32_t best = -1;
	float bb1 = 0.f, bb2 = 0.f;
	for (uint32_t t = 0; t < m->num_triangles; t++) {
		v3 p0, p1, p2;
		tri_points(m, t, &p0, &p1, &p2);
		float th, b1, b2;
		if (tri_test(r.o, r.d, r.len, p0, p1, p2, &th, &b1, &b2)) { r.len = th; best = (int32_t)t; bb1 = b1; bb2 = b2; }
	}
	if (best < 0) return 0.f;
	surf ls;
	local_surface(m, (uint32_t)best, bb1, bb2, r.d, &ls);
	v3 dd = sub(pl, ls.p);
	float pdf = dot3(dd, dd) / (gabs(dot3(ls.n, neg(wl))) * s->area[e]);
	return isinf(pdf) ? 0.f : pdf;
}

static float power_h(float f, float g) { return (f * f) / (f * f + g * g); }

/* ------------------------------------------------------------------ integrator */
/* uniform_sample_one_emitter for a surface interaction (integrator.cpp:101-201),
 * with find_emitter (:49-82); returns the estimate to be scaled by beta. */
static v3 sample_one_emitter(const port_scene* s, pcg* g, const surf* si, const bsdf* b) {
	v3 L = V(0, 0, 0);
	const int type = T_ALL ^ T_SPEC;
	float ne = (float)s->n_emit;
	uint32_t which = (uint32_t)floorf(pcg_f(g) * ne);
	if (which > s->n_emit - 1) which = s->n_emit - 1;
	float pick = 1.f / ne;
	int32_t em = s->emitters[which];
	float u0 = pcg_f(g), u1 = pcg_f(g);
	lsample ls = sample_light(s, em, si->p, si->n, u0, u1);
	ls.pdf = ls.pdf * pick;
	v3 wo = to_local(si, si->wo);
	if (!is_black(ls.L) && ls.pdf > 0.f) {
		v3 wi = to_local(si, ls.wi);
		v3 f = coll_f(b, wo, wi, type);
		float fp = coll_pdf(b, wo, wi, type);
		f = muls(f, gabs(dot3(ls.wi, si->z)));
		if (!is_black(f) && fp > 0.f) {
			ray sr = spawn_to(si->p, si->n, ls.p);
			hitrec h = bvh_hit(s, &sr, 1);
			if (h.ent < 0 || h.ent == em) L = add(L, divs(muls(mul(f, ls.L), power_h(ls.pdf, fp)), ls.pdf));
		}
	}
	float v0 = pcg_f(g), v1 = pcg_f(g);
	bsample bs = coll_sample(b, wo, v0, v1, type);
	v3 wiw = bs.pdf > 0.f ? to_world(si, bs.wi) : V(0, 0, 0);
	v3 val = muls(bs.f, gabs(dot3(wiw, si->z)));
	if (!is_black(val) && bs.pdf > 0.f) {
		ray mr = spawn(si->p, si->n, wiw);
		ray probe = mr;
		hitrec h = bvh_hit(s, &probe, 1);
		int found = 0;
		v3 Le = V(0, 0, 0);
		float epdf = 0.f;
		if (h.ent >= 0 && s->d->entities[h.ent].emitter >= 0) {
			surf es = world_surface(s, h, mr.o, mr.d);
			Le = surface_Le(s, h.ent, es.n, neg(wiw));
			epdf = emitter_pdf(s, h.ent, si->p, si->n, wiw) * pick;
			found = 1;
		} else if (h.ent < 0 && s->n_env > 0) {
			float nv = (float)s->n_env;
			uint32_t w = (uint32_t)floorf(pcg_f(g) * nv);
			if (w > s->n_env - 1) w = s->n_env - 1;
			int32_t env = s->envs[w];
			const rb_emitter_desc* ee = &s->d->emitters[s->d->entities[env].emitter];
			Le = V(ee->radiance[0], ee->radiance[1], ee->radiance[2]);
			epdf = emitter_pdf(s, env, si->p, si->n, wiw) * pick;
			found = 1;
		}
		if (found && !is_black(Le) && epdf > 0.f) {
			float w = tmatch(bs.type, T_SPEC) ? 1.f : power_h(bs.pdf, epdf);
			L = add(L, divs(muls(mul(val, Le), w), bs.pdf));
		}
	}
	return L;
}

/* perspective_camera::sample(position, u) (rainbow-cpu/cameras/perspective_camera.cpp:78-99) */
static ray camera_ray(const rb_camera_desc* c, uint32_t x, uint32_t y, pcg* g) {
	float fx = pcg_f(g), fy = pcg_f(g);
	float lx = pcg_f(g), ly = pcg_f(g);
	v3 target = xpoint(c->raster_to_camera, V((float)x + fx, (float)y + fy, 0.f));
	v3 o = V(0, 0, 0), d = norm3(norm3(target));
	if (c->lens_radius > 0.f) {
		v3 fp = add(o, muls(d, c->focus_distance / d.z));
		float dx, dy;
		disk(lx, ly, &dx, &dy);
		o = V(dx * c->lens_radius, dy * c->lens_radius, 0.f);
		d = norm3(sub(fp, o));
	}
	v3 dw = xvector(c->camera_to_world, d);
	ray r;
	r.d = norm3(norm3(dw));
	r.o = xpoint(c->camera_to_world, o);
	r.len = INFINITY * len3(dw);
	return r;
}

static uint64_t stream_seed(uint32_t pixel, uint32_t sample, uint32_t seed) {
	return (uint64_t)(pixel & 0xffffffu) | ((uint64_t)(sample & 0xffffffu) << 24) | ((uint64_t)(seed & 0x7fffu) << 48);
}

/* path_integrator::trace (path_integrator.cpp:15-47) with sample_surface_interaction
 * (integrator.cpp:329-404), for one (pixel, sample) seeded like the GPU path */
static v3 trace_sample(const port_scene* s, const rb_camera_desc* c, uint32_t pixel, uint32_t sample, uint32_t max_depth,
	float rr, uint32_t seed) {
	pcg g = pcg_new(stream_seed(pixel, sample, seed));
	ray r = camera_ray(c, pixel % (uint32_t)c->width, pixel / (uint32_t)c->width, &g);
	v3 beta = V(1, 1, 1), L = V(0, 0, 0);
	float eta = 1.f;
	int specular = 0;
	for (int bounces = 0; bounces < (int)max_depth; bounces++) {
		ray probe = r;
		hitrec h = bvh_hit(s, &probe, 0);
		if (h.ent < 0) {
			if (bounces == 0 || specular)
				for (uint32_t k = 0; k < s->n_env; k++) {
					const rb_emitter_desc* ee = &s->d->emitters[s->d->entities[s->envs[k]].emitter];
					L = add(L, mul(beta, V(ee->radiance[0], ee->radiance[1], ee->radiance[2])));
				}
			break;
		}
		surf si = world_surface(s, h, r.o, r.d);
		const rb_entity_desc* ed = &s->d->entities[h.ent];
		if ((bounces == 0 || specular) && ed->emitter >= 0) L = add(L, mul(beta, surface_Le(s, h.ent, si.n, neg(r.d))));
		int alive = 1;
		if (ed->material < 0) {
			r = spawn(si.p, si.n, r.d);
			bounces--;
		} else {
			bsdf b = make_bsdf(&s->d->materials[ed->material]);
			if (coll_count(&b, T_ALL ^ T_SPEC) != 0) L = add(L, mul(beta, sample_one_emitter(s, &g, &si, &b)));
			float u0 = pcg_f(&g), u1 = pcg_f(&g);
			bsample bs = coll_sample(&b, to_local(&si, si.wo), u0, u1, T_ALL);
			if (is_black(bs.f) || bs.pdf == 0.f) { alive = 0; }
			else {
				v3 wi = to_world(&si, bs.wi);
				beta = mul(beta, divs(muls(bs.f, gabs(dot3(wi, si.z))), bs.pdf));
				specular = tmatch(bs.type, T_SPEC);
				if (tmatch(bs.type, T_SPEC | T_TRANS))
					eta = eta * ((dot3(si.wo, si.n) > 0.f) ? (b.eta * b.eta) : (1.f / (b.eta * b.eta)));
				r = spawn(si.p, si.n, wi);
			}
		}
		if (!alive) break;
		v3 be = muls(beta, eta);
		float mc = gmax(gmax(be.x, be.y), be.z);
		if (mc < rr && bounces > 3) {
			float q = gmax(0.05f, 1.f - mc);
			if (pcg_f(&g) < q) break;
			beta = divs(beta, 1.f - q);
		}
	}
	return L;
}

/* ------------------------------------------------------------------ C entry points */
int port_pcg32(uint64_t seed, uint32_t n, uint32_t* u32, float* reals) {
	pcg a = pcg_new(seed), b = pcg_new(seed);
	for (uint32_t i = 0; i < n; i++) { u32[i] = pcg_u32(&a); reals[i] = pcg_f(&b); }
	return RB_OK;
}

int port_trace(const rb_scene_desc* d, const rb_ray* rays, uint32_t n, int shadow, rb_hit* hits) {
	port_scene s;
	int st = scene_init(&s, d);
	if (st != RB_OK && st != RB_ERR_INVALID_ARGUMENT) { scene_free(&s); return st; }
	for (uint32_t i = 0; i < n; i++) {
		ray r;
		r.o = V(rays[i].origin[0], rays[i].origin[1], rays[i].origin[2]);
		r.d = V(rays[i].direction[0], rays[i].direction[1], rays[i].direction[2]);
		r.len = rays[i].length;
		hitrec h = bvh_hit(&s, &r, shadow);
		hits[i].entity = h.ent;
		hits[i].triangle = h.tri;
		hits[i].t = r.len;
		hits[i].b1 = h.ent >= 0 ? h.b1 : 0.f;
		hits[i].b2 = h.ent >= 0 ? h.b2 : 0.f;
	}
	scene_free(&s);
	return RB_OK;
}

int port_samples(const rb_scene_desc* d, const rb_camera_desc* c, const uint32_t* pixels, const uint32_t* samples,
	uint32_t n, uint32_t max_depth, float rr, uint32_t seed, float* out) {
	port_scene s;
	int st = scene_init(&s, d);
	if (st != RB_OK) { scene_free(&s); return st; }
	for (uint32_t i = 0; i < n; i++) {
		v3 L = trace_sample(&s, c, pixels[i], samples[i], max_depth, rr, seed);
		out[3 * i] = L.x; out[3 * i + 1] = L.y; out[3 * i + 2] = L.z;
	}
	scene_free(&s);
	return RB_OK;
}

typedef struct {
	const port_scene* s;
	const rb_camera_desc* c;
	uint32_t spp, first, depth, seed;
	float rr;
	int row_end;
	double *sum, *sq;
	int* next;
	pthread_mutex_t* lock;
} job;

static void* worker(void* arg) {
	job* j = (job*)arg;
	for (;;) {
		pthread_mutex_lock(j->lock);
		int y = (*j->next)++;
		pthread_mutex_unlock(j->lock);
		if (y >= j->row_end) break;
		for (int x = 0; x < j->c->width; x++) {
			uint32_t p = (uint32_t)y * (uint32_t)j->c->width + (uint32_t)x;
			double a[3] = {0, 0, 0}, q[3] = {0, 0, 0};
			for (uint32_t k = 0; k < j->spp; k++) {
				v3 L = trace_sample(j->s, j->c, p, j->first + k, j->depth, j->rr, j->seed);
				a[0] += L.x; a[1] += L.y; a[2] += L.z;
				q[0] += (double)L.x * L.x; q[1] += (double)L.y * L.y; q[2] += (double)L.z * L.z;
			}
			for (int k = 0; k < 3; k++) { j->sum[3 * p + k] += a[k]; j->sq[3 * p + k] += q[k]; }
		}
	}
	return NULL;
}

/* FP64 per-pixel sums of L and L^2 for rows [row_begin, row_end) on `threads` pthreads. */
int port_render(const rb_scene_desc* d, const rb_camera_desc* c, uint32_t spp, uint32_t first, uint32_t max_depth, float rr,
	uint32_t seed, int threads, int row_begin, int row_end, double* sum, double* sq, double* seconds) {
	port_scene s;
	int st = scene_init(&s, d);
	if (st != RB_OK) { scene_free(&s); return st; }
	if (threads <= 0) threads = 1;
	if (threads > 256) threads = 256;
	if (row_end <= 0 || row_end > c->height) row_end = c->height;
	int next = row_begin;
	pthread_mutex_t lock = PTHREAD_MUTEX_INITIALIZER;
	job j = {&s, c, spp, first, max_depth, seed, rr, row_end, sum, sq, &next, &lock};
	pthread_t tid[256];
	struct timespec t0, t1;
	clock_gettime(CLOCK_MONOTONIC, &t0);
	for (int t = 0; t < threads; t++) pthread_create(&tid[t], NULL, worker, &j);
	for (int t = 0; t < threads; t++) pthread_join(tid[t], NULL);
	clock_gettime(CLOCK_MONOTONIC, &t1);
	if (seconds) *seconds = (double)(t1.tv_sec - t0.tv_sec) + 1e-9 * (double)(t1.tv_nsec - t0.tv_nsec);
	scene_free(&s);
	return RB_OK;
}
