// Host construction of the perspective camera matrices.
//
// Reproduces what projective_camera's constructor computes
// (rainbow-cpu/cameras/camera.cpp:21-52) for a camera built from
// perspective_right_hand(fov, width, height) (rainbow-cpu/shared/transform.cpp:144-149,
// near 0.01, far 1000) and the camera-to-world transform
// look_at_right_hand(eye, target, up).inverse(), with screen window [-1, 1]^2:
//   screen_to_raster = scale(res) * scale(1 / (sw.max.x - sw.min.x), 1 / (sw.min.y - sw.max.y)) * translate(-sw.min.x, -sw.max.y)
//   raster_to_camera = camera_to_screen.inverse() * screen_to_raster.inverse()
// transform::operator* multiplies the matrices left to right and the inverses
// in reverse order (transform.cpp:19-25). The matrix inverse is the adjugate
// form (2x2 sub-determinants of the upper and lower row pairs) used by the
// glm replacement the reference is compiled against for the oracle.
#pragma once

#include "../rb_math.h"

namespace rb {
namespace host {

inline float elem(const mat4& m, int r, int c) { return m.m[c * 4 + r]; }

inline mat4 inverse4(const mat4& mm) {
	auto a = [&](int r, int c) { return elem(mm, r, c); };
	const float s0 = a(0, 0) * a(1, 1) - a(1, 0) * a(0, 1);
	const float s1 = a(0, 0) * a(1, 2) - a(1, 0) * a(0, 2);
	const float s2 = a(0, 0) * a(1, 3) - a(1, 0) * a(0, 3);
	const float s3 = a(0, 1) * a(1, 2) - a(1, 1) * a(0, 2);
	const float s4 = a(0, 1) * a(1, 3) - a(1, 1) * a(0, 3);
	const float s5 = a(0, 2) * a(1, 3) - a(1, 2) * a(0, 3);
	const float c5 = a(2, 2) * a(3, 3) - a(3, 2) * a(2, 3);
	const float c4 = a(2, 1) * a(3, 3) - a(3, 1) * a(2, 3);
	const float c3 = a(2, 1) * a(3, 2) - a(3, 1) * a(2, 2);
	const float c2 = a(2, 0) * a(3, 3) - a(3, 0) * a(2, 3);
	const float c1 = a(2, 0) * a(3, 2) - a(3, 0) * a(2, 2);
	const float c0 = a(2, 0) * a(3, 1) - a(3, 0) * a(2, 1);
	const float det = s0 * c5 - s1 * c4 + s2 * c3 + s3 * c2 - s4 * c1 + s5 * c0;
	const float inv = 1.f / det;
	mat4 r;
	auto set = [&](int row, int col, float v) { r.m[col * 4 + row] = v; };
	set(0, 0, (a(1, 1) * c5 - a(1, 2) * c4 + a(1, 3) * c3) * inv);
	set(0, 1, (-a(0, 1) * c5 + a(0, 2) * c4 - a(0, 3) * c3) * inv);
	set(0, 2, (a(3, 1) * s5 - a(3, 2) * s4 + a(3, 3) * s3) * inv);
	set(0, 3, (-a(2, 1) * s5 + a(2, 2) * s4 - a(2, 3) * s3) * inv);
	set(1, 0, (-a(1, 0) * c5 + a(1, 2) * c2 - a(1, 3) * c1) * inv);
	set(1, 1, (a(0, 0) * c5 - a(0, 2) * c2 + a(0, 3) * c1) * inv);
	set(1, 2, (-a(3, 0) * s5 + a(3, 2) * s2 - a(3, 3) * s1) * inv);
	set(1, 3, (a(2, 0) * s5 - a(2, 2) * s2 + a(2, 3) * s1) * inv);
	set(2, 0, (a(1, 0) * c4 - a(1, 1) * c2 + a(1, 3) * c0) * inv);
	set(2, 1, (-a(0, 0) * c4 + a(0, 1) * c2 - a(0, 3) * c0) * inv);
	set(2, 2, (a(3, 0) * s4 - a(3, 1) * s2 + a(3, 3) * s0) * inv);
	set(2, 3, (-a(2, 0) * s4 + a(2, 1) * s2 - a(2, 3) * s0) * inv);
	set(3, 0, (-a(1, 0) * c3 + a(1, 1) * c1 - a(1, 2) * c0) * inv);
	set(3, 1, (a(0, 0) * c3 - a(0, 1) * c1 + a(0, 2) * c0) * inv);
	set(3, 2, (-a(3, 0) * s3 + a(3, 1) * s1 - a(3, 2) * s0) * inv);
	set(3, 3, (a(2, 0) * s3 - a(2, 1) * s1 + a(2, 2) * s0) * inv);
	return r;
}

// scale(identity, v): column c = identity column c * v[c]
inline mat4 scale4(vec3 v) {
	const mat4 id = mat_identity();
	mat4 r = id;
	const float s[3] = {v.x, v.y, v.z};
	for (int c = 0; c < 3; c++)
		for (int row = 0; row < 4; row++) r.m[c * 4 + row] = id.m[c * 4 + row] * s[c];
	return r;
}

// translate(identity, v): column 3 = ((I0 * v.x + I1 * v.y) + I2 * v.z) + I3
inline mat4 translate4(vec3 v) {
	const mat4 id = mat_identity();
	mat4 r = id;
	for (int row = 0; row < 4; row++) {
		float s = id.m[0 * 4 + row] * v.x + id.m[1 * 4 + row] * v.y;
		s = s + id.m[2 * 4 + row] * v.z;
		s = s + id.m[3 * 4 + row];
		r.m[12 + row] = s;
	}
	return r;
}

struct xform {
	mat4 m, inv;
};
inline xform compose(const xform& a, const xform& b) { return xform{mat_mul(a.m, b.m), mat_mul(b.inv, a.inv)}; }
inline xform scale_xf(vec3 v) { return xform{scale4(v), scale4(vec3{1.f / v.x, 1.f / v.y, 1.f / v.z})}; }
inline xform translate_xf(vec3 v) { return xform{translate4(v), translate4(-v)}; }

inline mat4 perspective_rh(float fov_radians, float width, float height, float znear, float zfar) {
	const float h = cosf(0.5f * fov_radians) / sinf(0.5f * fov_radians);
	const float w = h * height / width;
	mat4 r;
	for (float& x : r.m) x = 0.f;
	r.m[0] = w;
	r.m[5] = h;
	r.m[10] = -(zfar + znear) / (zfar - znear);
	r.m[11] = -1.f;
	r.m[14] = -(2.f * zfar * znear) / (zfar - znear);
	return r;
}

inline mat4 look_at_rh(vec3 eye, vec3 center, vec3 up) {
	const vec3 f = normalize(center - eye);
	const vec3 s = normalize(cross(f, up));
	const vec3 u = cross(s, f);
	mat4 r = mat_identity();
	r.m[0] = s.x; r.m[4] = s.y; r.m[8] = s.z;
	r.m[1] = u.x; r.m[5] = u.y; r.m[9] = u.z;
	r.m[2] = -f.x; r.m[6] = -f.y; r.m[10] = -f.z;
	r.m[12] = -dot(s, eye);
	r.m[13] = -dot(u, eye);
	r.m[14] = dot(f, eye);
	return r;
}

// Fills the matrices of a camera description from eye/target/up/fov/size.
inline void camera_matrices(rb_camera_desc& cam) {
	const float fov_rad = cam.fov_degrees * static_cast<float>(0.01745329251994329576923690768489);
	const mat4 p = perspective_rh(fov_rad, static_cast<float>(cam.width), static_cast<float>(cam.height), 0.01f, 1000.f);
	const xform camera_to_screen{p, inverse4(p)};
	// screen window [-1, 1] x [-1, 1]
	const float sw_min_x = -1.f, sw_min_y = -1.f, sw_max_x = 1.f, sw_max_y = 1.f;
	xform screen_to_raster = scale_xf(vec3{static_cast<float>(cam.width), static_cast<float>(cam.height), 1.f});
	screen_to_raster = compose(screen_to_raster, scale_xf(vec3{1.0f / (sw_max_x - sw_min_x), 1.0f / (sw_min_y - sw_max_y), 1.0f}));
	screen_to_raster = compose(screen_to_raster, translate_xf(vec3{-sw_min_x, -sw_max_y, 0.f}));
	const xform raster_to_screen{screen_to_raster.inv, screen_to_raster.m};
	const xform screen_to_camera{camera_to_screen.inv, camera_to_screen.m};
	const xform raster_to_camera = compose(screen_to_camera, raster_to_screen);
	const mat4 view = look_at_rh(vec3{cam.eye[0], cam.eye[1], cam.eye[2]}, vec3{cam.target[0], cam.target[1], cam.target[2]},
		vec3{cam.up[0], cam.up[1], cam.up[2]});
	const mat4 camera_to_world = inverse4(view);
	for (int i = 0; i < 16; i++) {
		cam.raster_to_camera[i] = raster_to_camera.m.m[i];
		cam.camera_to_world[i] = camera_to_world.m[i];
	}
}

} // namespace host
} // namespace rb
