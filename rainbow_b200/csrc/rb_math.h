// Float vector / matrix arithmetic of the path-tracing core, usable from host
// C++ and CUDA device code.
//
// Every operation keeps the rounding order of the reference renderer's math
// layer (rainbow-core/math/detail/vector.hpp:9-105 and
// rainbow-core/math/detail/matrix4x4.hpp:15-73, which forward to glm):
//   dot(a, b)      = (a.x * b.x + a.y * b.y) + a.z * b.z
//   cross(a, b)    = (a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y)
//   length(v)      = sqrt(dot(v, v))
//   normalize(v)   = v * (1 / sqrt(dot(v, v)))
//   M * (x,y,z,w)  = (M[0] * x + M[1] * y) + (M[2] * z + M[3] * w)   (columns M[i])
//   min(a, b)      = (b < a) ? b : a,  max(a, b) = (a < b) ? b : a
// Device code is compiled without FMA contraction (-fmad=false) and with IEEE
// division and square root, so these produce the same bits on host and device.
#pragma once

#include <math.h>
#include <stdint.h>

#if defined(__CUDACC__)
#define RB_HD __host__ __device__ __forceinline__
#else
#define RB_HD inline
#endif

namespace rb {

struct vec2 {
	float x, y;
};

struct vec3 {
	float x, y, z;
};

RB_HD vec3 make3(float x, float y, float z) { return vec3{x, y, z}; }
RB_HD vec3 splat3(float s) { return vec3{s, s, s}; }
RB_HD vec2 make2(float x, float y) { return vec2{x, y}; }

RB_HD vec3 operator+(vec3 a, vec3 b) { return vec3{a.x + b.x, a.y + b.y, a.z + b.z}; }
RB_HD vec3 operator-(vec3 a, vec3 b) { return vec3{a.x - b.x, a.y - b.y, a.z - b.z}; }
RB_HD vec3 operator*(vec3 a, vec3 b) { return vec3{a.x * b.x, a.y * b.y, a.z * b.z}; }
RB_HD vec3 operator/(vec3 a, vec3 b) { return vec3{a.x / b.x, a.y / b.y, a.z / b.z}; }
RB_HD vec3 operator*(vec3 a, float s) { return vec3{a.x * s, a.y * s, a.z * s}; }
RB_HD vec3 operator*(float s, vec3 a) { return vec3{s * a.x, s * a.y, s * a.z}; }
RB_HD vec3 operator/(vec3 a, float s) { return vec3{a.x / s, a.y / s, a.z / s}; }
RB_HD vec3 operator/(float s, vec3 a) { return vec3{s / a.x, s / a.y, s / a.z}; }
RB_HD vec3 operator-(vec3 a) { return vec3{-a.x, -a.y, -a.z}; }
RB_HD vec2 operator+(vec2 a, vec2 b) { return vec2{a.x + b.x, a.y + b.y}; }
RB_HD vec2 operator-(vec2 a, vec2 b) { return vec2{a.x - b.x, a.y - b.y}; }
RB_HD vec2 operator*(vec2 a, float s) { return vec2{a.x * s, a.y * s}; }
RB_HD vec2 operator*(float s, vec2 a) { return vec2{s * a.x, s * a.y}; }

RB_HD bool equal(vec3 a, vec3 b) { return a.x == b.x && a.y == b.y && a.z == b.z; }
RB_HD bool is_zero(vec3 a) { return a.x == 0.f && a.y == 0.f && a.z == 0.f; }

RB_HD float dot(vec3 a, vec3 b) {
	const float px = a.x * b.x, py = a.y * b.y, pz = a.z * b.z;
	return px + py + pz;
}
RB_HD float dot(vec2 a, vec2 b) {
	const float px = a.x * b.x, py = a.y * b.y;
	return px + py;
}
RB_HD vec3 cross(vec3 a, vec3 b) {
	return vec3{a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}
RB_HD float length(vec3 v) { return sqrtf(dot(v, v)); }
RB_HD float length_squared(vec3 v) {
	// dot(v - 0, v - 0): subtracting +0 turns a -0 component into +0, which the
	// square does not see, so dot(v, v) gives the same bits.
	return dot(v, v);
}
RB_HD float distance_squared(vec3 a, vec3 b) { return dot(a - b, a - b); }
RB_HD vec3 normalize(vec3 v) { return v * (1.f / sqrtf(dot(v, v))); }

RB_HD float fmin_ref(float a, float b) { return (b < a) ? b : a; }
RB_HD float fmax_ref(float a, float b) { return (a < b) ? b : a; }
RB_HD float fabs_ref(float x) { return x >= 0.f ? x : -x; }
RB_HD float fclamp_ref(float x, float lo, float hi) { return fmin_ref(fmax_ref(x, lo), hi); }
RB_HD vec3 vmin(vec3 a, vec3 b) { return vec3{fmin_ref(a.x, b.x), fmin_ref(a.y, b.y), fmin_ref(a.z, b.z)}; }
RB_HD vec3 vmax(vec3 a, vec3 b) { return vec3{fmax_ref(a.x, b.x), fmax_ref(a.y, b.y), fmax_ref(a.z, b.z)}; }
RB_HD vec3 vabs(vec3 a) { return vec3{fabs_ref(a.x), fabs_ref(a.y), fabs_ref(a.z)}; }
RB_HD float max_component(vec3 v) {
	// vector max_component (rainbow-core/math/detail/vector.hpp:47-55)
	float m = v.x;
	if (m < v.y) m = v.y;
	if (m < v.z) m = v.z;
	return m;
}
RB_HD float get(vec3 v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }

// 4x4 column-major matrix, element (row r, column c) at m[c * 4 + r].
struct mat4 {
	float m[16];
};

// Column c times scalar s, summed as (c0 x + c1 y) + (c2 z + c3 w), one row at a time.
RB_HD float mat_row(const float* m, int r, float x, float y, float z, float w) {
	const float a0 = m[0 + r] * x + m[4 + r] * y;
	const float a1 = m[8 + r] * z + m[12 + r] * w;
	return a0 + a1;
}
// transform_point (rainbow-cpu/shared/transform.cpp:172-177): M * (p, 1), no divide.
RB_HD vec3 xform_point(const float* m, vec3 p) {
	return vec3{mat_row(m, 0, p.x, p.y, p.z, 1.f), mat_row(m, 1, p.x, p.y, p.z, 1.f), mat_row(m, 2, p.x, p.y, p.z, 1.f)};
}
// transform_vector (transform.cpp:179-182): M * (v, 0).
RB_HD vec3 xform_vector(const float* m, vec3 v) {
	return vec3{mat_row(m, 0, v.x, v.y, v.z, 0.f), mat_row(m, 1, v.x, v.y, v.z, 0.f), mat_row(m, 2, v.x, v.y, v.z, 0.f)};
}
// transform_normal (transform.cpp:184-188): normalize(transpose(Minv) * (n, 0)),
// where Minv is the transform's inverse matrix. Row r of transpose(Minv) is
// column r of Minv, so element (r, c) of the transpose is minv[r * 4 + c].
RB_HD vec3 xform_normal(const float* minv, vec3 n) {
	float out[3];
	for (int r = 0; r < 3; r++) {
		const float a0 = minv[r * 4 + 0] * n.x + minv[r * 4 + 1] * n.y;
		const float a1 = minv[r * 4 + 2] * n.z + minv[r * 4 + 3] * 0.f;
		out[r] = a0 + a1;
	}
	return normalize(vec3{out[0], out[1], out[2]});
}

// mat * mat: column i = ((A0 * B[i].x + A1 * B[i].y) + A2 * B[i].z) + A3 * B[i].w
RB_HD mat4 mat_mul(const mat4& a, const mat4& b) {
	mat4 r;
	for (int i = 0; i < 4; i++)
		for (int row = 0; row < 4; row++) {
			float s = a.m[0 * 4 + row] * b.m[i * 4 + 0] + a.m[1 * 4 + row] * b.m[i * 4 + 1];
			s = s + a.m[2 * 4 + row] * b.m[i * 4 + 2];
			s = s + a.m[3 * 4 + row] * b.m[i * 4 + 3];
			r.m[i * 4 + row] = s;
		}
	return r;
}

RB_HD mat4 mat_identity() {
	mat4 r;
	for (int i = 0; i < 16; i++) r.m[i] = (i % 5 == 0) ? 1.f : 0.f;
	return r;
}

} // namespace rb
