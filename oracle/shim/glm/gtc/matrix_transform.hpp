// Project-written stand-in for glm/gtc/matrix_transform.hpp (oracle build only).
// Restates the standard transform constructors the reference calls from
// rainbow-core/math/detail/matrix4x4.hpp:15-73. Angles are radians here; the
// reference converts degrees with glm::radians before calling rotate.
#pragma once

#include "../glm.hpp"

namespace glm {

// translate(m, v): column 3 becomes m[0]*v.x + m[1]*v.y + m[2]*v.z + m[3]
template <typename T> mat<4, 4, T> translate(const mat<4, 4, T>& m, const vec<3, T>& v) {
	mat<4, 4, T> r = m;
	r[3] = m[0] * v.x + m[1] * v.y + m[2] * v.z + m[3];
	return r;
}

template <typename T> mat<4, 4, T> scale(const mat<4, 4, T>& m, const vec<3, T>& v) {
	mat<4, 4, T> r;
	r[0] = m[0] * v.x;
	r[1] = m[1] * v.y;
	r[2] = m[2] * v.z;
	r[3] = m[3];
	return r;
}

// Axis-angle rotation (Rodrigues form) about the normalised axis, then m * R.
template <typename T> mat<4, 4, T> rotate(const mat<4, 4, T>& m, T angle, const vec<3, T>& v) {
	const T c = std::cos(angle);
	const T s = std::sin(angle);
	const vec<3, T> axis = normalize(v);
	const vec<3, T> t = axis * (static_cast<T>(1) - c);
	mat<4, 4, T> rot;
	rot[0][0] = c + t.x * axis.x;
	rot[0][1] = t.x * axis.y + s * axis.z;
	rot[0][2] = t.x * axis.z - s * axis.y;
	rot[1][0] = t.y * axis.x - s * axis.z;
	rot[1][1] = c + t.y * axis.y;
	rot[1][2] = t.y * axis.z + s * axis.x;
	rot[2][0] = t.z * axis.x + s * axis.y;
	rot[2][1] = t.z * axis.y - s * axis.x;
	rot[2][2] = c + t.z * axis.z;
	mat<4, 4, T> r;
	r[0] = m[0] * rot[0][0] + m[1] * rot[0][1] + m[2] * rot[0][2];
	r[1] = m[0] * rot[1][0] + m[1] * rot[1][1] + m[2] * rot[1][2];
	r[2] = m[0] * rot[2][0] + m[1] * rot[2][1] + m[2] * rot[2][2];
	r[3] = m[3];
	return r;
}

// OpenGL-style perspective with clip-space depth in [-1, 1].
// h = cot(fov / 2), w = h * height / width.
template <typename T> mat<4, 4, T> perspectiveFovRH(T fov, T width, T height, T zNear, T zFar) {
	const T rad = fov;
	const T h = std::cos(static_cast<T>(0.5) * rad) / std::sin(static_cast<T>(0.5) * rad);
	const T w = h * height / width;
	mat<4, 4, T> r(static_cast<T>(0));
	r[0][0] = w;
	r[1][1] = h;
	r[2][2] = -(zFar + zNear) / (zFar - zNear);
	r[2][3] = -static_cast<T>(1);
	r[3][2] = -(static_cast<T>(2) * zFar * zNear) / (zFar - zNear);
	return r;
}

template <typename T> mat<4, 4, T> perspectiveFovLH(T fov, T width, T height, T zNear, T zFar) {
	const T rad = fov;
	const T h = std::cos(static_cast<T>(0.5) * rad) / std::sin(static_cast<T>(0.5) * rad);
	const T w = h * height / width;
	mat<4, 4, T> r(static_cast<T>(0));
	r[0][0] = w;
	r[1][1] = h;
	r[2][2] = (zFar + zNear) / (zFar - zNear);
	r[2][3] = static_cast<T>(1);
	r[3][2] = -(static_cast<T>(2) * zFar * zNear) / (zFar - zNear);
	return r;
}

template <typename T> mat<4, 4, T> lookAtRH(const vec<3, T>& eye, const vec<3, T>& center, const vec<3, T>& up) {
	const vec<3, T> f = normalize(center - eye);
	const vec<3, T> s = normalize(cross(f, up));
	const vec<3, T> u = cross(s, f);
	mat<4, 4, T> r(static_cast<T>(1));
	r[0][0] = s.x; r[1][0] = s.y; r[2][0] = s.z;
	r[0][1] = u.x; r[1][1] = u.y; r[2][1] = u.z;
	r[0][2] = -f.x; r[1][2] = -f.y; r[2][2] = -f.z;
	r[3][0] = -dot(s, eye);
	r[3][1] = -dot(u, eye);
	r[3][2] = dot(f, eye);
	return r;
}

template <typename T> mat<4, 4, T> lookAtLH(const vec<3, T>& eye, const vec<3, T>& center, const vec<3, T>& up) {
	const vec<3, T> f = normalize(center - eye);
	const vec<3, T> s = normalize(cross(up, f));
	const vec<3, T> u = cross(f, s);
	mat<4, 4, T> r(static_cast<T>(1));
	r[0][0] = s.x; r[1][0] = s.y; r[2][0] = s.z;
	r[0][1] = u.x; r[1][1] = u.y; r[2][1] = u.z;
	r[0][2] = f.x; r[1][2] = f.y; r[2][2] = f.z;
	r[3][0] = -dot(s, eye);
	r[3][1] = -dot(u, eye);
	r[3][2] = -dot(f, eye);
	return r;
}

} // namespace glm
