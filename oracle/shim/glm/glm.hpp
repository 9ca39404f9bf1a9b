// Minimal, project-written stand-in for the glm vector/matrix library.
//
// TEST INFRASTRUCTURE ONLY (oracle build). The reference renderer includes
// <glm/glm.hpp> (rainbow-core/math/vector.hpp:7) and
// <glm/gtc/matrix_transform.hpp> (rainbow-core/math/detail/matrix4x4.hpp:9),
// but glm is not vendored and no version is pinned anywhere in the reference.
// This header implements only the subset the reference calls, restated from
// glm's published semantics (column-major matrices, component-wise vector
// operators). The floating-point association chosen for each reduction is
// documented beside it; the GPU kernels and the C restatement follow the same
// association, so "bit-exact" parity means "bit-exact against this shim".
#pragma once

#include <cassert>
#include <cmath>
#include <cstddef>
#include <limits>
#include <type_traits>

namespace glm {

using length_t = int;

template <std::size_t L, typename T> struct vec;

// ---------------------------------------------------------------- storage
template <typename T> struct vec<1, T> {
	using value_type = T;
	using length_type = length_t;
	T x = T(0);
	constexpr vec() = default;
	constexpr explicit vec(T s) : x(s) {}
	template <typename U> constexpr vec(const vec<1, U>& v) : x(static_cast<T>(v.x)) {}
	template <typename U> constexpr explicit vec(const vec<2, U>& v) : x(static_cast<T>(v.x)) {}
	template <typename U> constexpr explicit vec(const vec<3, U>& v) : x(static_cast<T>(v.x)) {}
	template <typename U> constexpr explicit vec(const vec<4, U>& v) : x(static_cast<T>(v.x)) {}
	static constexpr length_t length() { return 1; }
	T& operator[](length_t) { return x; }
	const T& operator[](length_t) const { return x; }
};

template <typename T> struct vec<2, T> {
	using value_type = T;
	using length_type = length_t;
	T x = T(0), y = T(0);
	constexpr vec() = default;
	constexpr explicit vec(T s) : x(s), y(s) {}
	template <typename A, typename B> constexpr vec(A a, B b) : x(static_cast<T>(a)), y(static_cast<T>(b)) {}
	template <typename U> constexpr vec(const vec<2, U>& v) : x(static_cast<T>(v.x)), y(static_cast<T>(v.y)) {}
	template <typename U> constexpr vec(const vec<3, U>& v) : x(static_cast<T>(v.x)), y(static_cast<T>(v.y)) {}
	template <typename U> constexpr vec(const vec<4, U>& v) : x(static_cast<T>(v.x)), y(static_cast<T>(v.y)) {}
	static constexpr length_t length() { return 2; }
	T& operator[](length_t i) { return i == 0 ? x : y; }
	const T& operator[](length_t i) const { return i == 0 ? x : y; }
};

template <typename T> struct vec<3, T> {
	using value_type = T;
	using length_type = length_t;
	T x = T(0), y = T(0), z = T(0);
	constexpr vec() = default;
	constexpr explicit vec(T s) : x(s), y(s), z(s) {}
	template <typename A, typename B, typename C>
	constexpr vec(A a, B b, C c) : x(static_cast<T>(a)), y(static_cast<T>(b)), z(static_cast<T>(c)) {}
	template <typename A, typename B>
	constexpr vec(const vec<2, A>& xy, B c) : x(static_cast<T>(xy.x)), y(static_cast<T>(xy.y)), z(static_cast<T>(c)) {}
	template <typename A, typename B>
	constexpr vec(const vec<1, A>& a, const vec<2, B>& yz) : x(static_cast<T>(a.x)), y(static_cast<T>(yz.x)), z(static_cast<T>(yz.y)) {}
	template <typename U> constexpr vec(const vec<3, U>& v) : x(static_cast<T>(v.x)), y(static_cast<T>(v.y)), z(static_cast<T>(v.z)) {}
	template <typename U> constexpr vec(const vec<4, U>& v) : x(static_cast<T>(v.x)), y(static_cast<T>(v.y)), z(static_cast<T>(v.z)) {}
	static constexpr length_t length() { return 3; }
	T& operator[](length_t i) { return i == 0 ? x : (i == 1 ? y : z); }
	const T& operator[](length_t i) const { return i == 0 ? x : (i == 1 ? y : z); }
};

template <typename T> struct vec<4, T> {
	using value_type = T;
	using length_type = length_t;
	T x = T(0), y = T(0), z = T(0), w = T(0);
	constexpr vec() = default;
	constexpr explicit vec(T s) : x(s), y(s), z(s), w(s) {}
	template <typename A, typename B, typename C, typename D>
	constexpr vec(A a, B b, C c, D d) : x(static_cast<T>(a)), y(static_cast<T>(b)), z(static_cast<T>(c)), w(static_cast<T>(d)) {}
	template <typename A, typename B>
	constexpr vec(const vec<3, A>& xyz, B d) : x(static_cast<T>(xyz.x)), y(static_cast<T>(xyz.y)), z(static_cast<T>(xyz.z)), w(static_cast<T>(d)) {}
	template <typename U> constexpr vec(const vec<4, U>& v) : x(static_cast<T>(v.x)), y(static_cast<T>(v.y)), z(static_cast<T>(v.z)), w(static_cast<T>(v.w)) {}
	static constexpr length_t length() { return 4; }
	T& operator[](length_t i) { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
	const T& operator[](length_t i) const { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
};

using vec2 = vec<2, float>;
using vec3 = vec<3, float>;
using vec4 = vec<4, float>;

// ---------------------------------------------------------------- component-wise operators
#define RB_SHIM_BINOP(OP)                                                                         \
	template <std::size_t L, typename T>                                                          \
	vec<L, T> operator OP(const vec<L, T>& a, const vec<L, T>& b) {                               \
		vec<L, T> r;                                                                              \
		for (length_t i = 0; i < static_cast<length_t>(L); i++) r[i] = a[i] OP b[i];              \
		return r;                                                                                 \
	}                                                                                             \
	template <std::size_t L, typename T, typename U,                                              \
		typename = std::enable_if_t<std::is_arithmetic<U>::value>>                                \
	vec<L, T> operator OP(const vec<L, T>& a, U s) {                                              \
		vec<L, T> r;                                                                              \
		for (length_t i = 0; i < static_cast<length_t>(L); i++) r[i] = a[i] OP static_cast<T>(s); \
		return r;                                                                                 \
	}                                                                                             \
	template <std::size_t L, typename T, typename U,                                              \
		typename = std::enable_if_t<std::is_arithmetic<U>::value>>                                \
	vec<L, T> operator OP(U s, const vec<L, T>& a) {                                              \
		vec<L, T> r;                                                                              \
		for (length_t i = 0; i < static_cast<length_t>(L); i++) r[i] = static_cast<T>(s) OP a[i]; \
		return r;                                                                                 \
	}                                                                                             \
	template <std::size_t L, typename T>                                                          \
	vec<L, T>& operator OP##=(vec<L, T>& a, const vec<L, T>& b) { return a = a OP b; }            \
	template <std::size_t L, typename T, typename U,                                              \
		typename = std::enable_if_t<std::is_arithmetic<U>::value>>                                \
	vec<L, T>& operator OP##=(vec<L, T>& a, U s) { return a = a OP s; }

RB_SHIM_BINOP(+)
RB_SHIM_BINOP(-)
RB_SHIM_BINOP(*)
RB_SHIM_BINOP(/)
#undef RB_SHIM_BINOP

template <std::size_t L, typename T>
vec<L, T> operator-(const vec<L, T>& a) {
	vec<L, T> r;
	for (length_t i = 0; i < static_cast<length_t>(L); i++) r[i] = -a[i];
	return r;
}

template <std::size_t L, typename T>
bool operator==(const vec<L, T>& a, const vec<L, T>& b) {
	for (length_t i = 0; i < static_cast<length_t>(L); i++)
		if (!(a[i] == b[i])) return false;
	return true;
}

template <std::size_t L, typename T>
bool operator!=(const vec<L, T>& a, const vec<L, T>& b) { return !(a == b); }

// ---------------------------------------------------------------- scalar functions
// min/max follow glm's ternary definitions: max(a, b) = (a < b) ? b : a and
// min(a, b) = (b < a) ? b : a. With a NaN in b both return a.
template <typename T, typename = std::enable_if_t<std::is_arithmetic<T>::value>>
constexpr T min(T a, T b) { return (b < a) ? b : a; }
template <typename T, typename = std::enable_if_t<std::is_arithmetic<T>::value>>
constexpr T max(T a, T b) { return (a < b) ? b : a; }
template <typename T, typename = std::enable_if_t<std::is_arithmetic<T>::value>>
constexpr T clamp(T x, T lo, T hi) { return min(max(x, lo), hi); }
// abs(x) = x >= 0 ? x : -x (keeps the sign of a negative zero, as glm does).
template <typename T, typename = std::enable_if_t<std::is_arithmetic<T>::value>>
constexpr T abs(T x) { return x >= T(0) ? x : -x; }

template <typename T> using if_arith = std::enable_if_t<std::is_arithmetic<T>::value, int>;
template <typename T, if_arith<T> = 0> T sqrt(T x) { return std::sqrt(x); }
template <typename T, if_arith<T> = 0> T sin(T x) { return std::sin(x); }
template <typename T, if_arith<T> = 0> T cos(T x) { return std::cos(x); }
template <typename T, if_arith<T> = 0> T tan(T x) { return std::tan(x); }
template <typename T, if_arith<T> = 0> T acos(T x) { return std::acos(x); }
template <typename T, if_arith<T> = 0> T atan(T y, T x) { return std::atan2(y, x); }
template <typename T, if_arith<T> = 0> T log(T x) { return std::log(x); }
template <typename T, if_arith<T> = 0> T exp(T x) { return std::exp(x); }
template <typename T, if_arith<T> = 0> T pow(T x, T y) { return std::pow(x, y); }
template <typename T, if_arith<T> = 0> T floor(T x) { return std::floor(x); }
template <typename T, if_arith<T> = 0> T ceil(T x) { return std::ceil(x); }
template <typename T, if_arith<T> = 0> T mod(T x, T y) { return x - y * std::floor(x / y); }
template <typename T, if_arith<T> = 0> bool isnan(T x) { return std::isnan(x); }
template <typename T, if_arith<T> = 0> constexpr T radians(T degrees) { return degrees * static_cast<T>(0.01745329251994329576923690768489); }

template <typename T> constexpr T pi() { return static_cast<T>(3.14159265358979323846264338327950288); }
template <typename T> constexpr T two_pi() { return static_cast<T>(6.28318530717958647692528676655900576); }
template <typename T> constexpr T half_pi() { return static_cast<T>(1.57079632679489661923132169163975144); }
template <typename T> constexpr T quarter_pi() { return static_cast<T>(0.785398163397448309615660845819875721); }
template <typename T> constexpr T one_over_pi() { return static_cast<T>(0.318309886183790671537767526745028724); }
template <typename T> constexpr T one_over_two_pi() { return static_cast<T>(0.159154943091895335768883763372514362); }

// ---------------------------------------------------------------- vector functions
// The vector overloads are written as constrained templates over the whole
// vector type, so the reference's own wrappers in rainbow::core::math (which
// take vector_t<L, T> and forward here qualified) stay the better match when
// a call inside the reference finds both through argument-dependent lookup.
template <typename V> struct is_vec : std::false_type {};
template <std::size_t L, typename T> struct is_vec<vec<L, T>> : std::true_type {};
template <typename V> using if_vec = std::enable_if_t<is_vec<V>::value, int>;

namespace detail {
template <std::size_t L, typename T, typename F> vec<L, T> map(const vec<L, T>& a, F f) {
	vec<L, T> r;
	for (length_t i = 0; i < static_cast<length_t>(L); i++) r[i] = f(a[i]);
	return r;
}
template <std::size_t L, typename T, typename F> vec<L, T> zip(const vec<L, T>& a, const vec<L, T>& b, F f) {
	vec<L, T> r;
	for (length_t i = 0; i < static_cast<length_t>(L); i++) r[i] = f(a[i], b[i]);
	return r;
}
// dot: products are formed first, then summed left to right:
// vec2 = p.x + p.y, vec3 = (p.x + p.y) + p.z, vec4 = (p.x + p.y) + (p.z + p.w).
template <typename T> T dot(const vec<1, T>& a, const vec<1, T>& b) { return a.x * b.x; }
template <typename T> T dot(const vec<2, T>& a, const vec<2, T>& b) {
	const vec<2, T> p = a * b;
	return p.x + p.y;
}
template <typename T> T dot(const vec<3, T>& a, const vec<3, T>& b) {
	const vec<3, T> p = a * b;
	return p.x + p.y + p.z;
}
template <typename T> T dot(const vec<4, T>& a, const vec<4, T>& b) {
	const vec<4, T> p = a * b;
	return (p.x + p.y) + (p.z + p.w);
}
} // namespace detail

template <typename V, if_vec<V> = 0> V abs(const V& a) { return detail::map(a, [](auto v) { return glm::abs(v); }); }
template <typename V, if_vec<V> = 0> V floor(const V& a) { return detail::map(a, [](auto v) { return std::floor(v); }); }
template <typename V, if_vec<V> = 0> V ceil(const V& a) { return detail::map(a, [](auto v) { return std::ceil(v); }); }
template <typename V, if_vec<V> = 0> V min(const V& a, const V& b) { return detail::zip(a, b, [](auto x, auto y) { return glm::min(x, y); }); }
template <typename V, if_vec<V> = 0> V max(const V& a, const V& b) { return detail::zip(a, b, [](auto x, auto y) { return glm::max(x, y); }); }
template <std::size_t L, typename T> vec<L, T> clamp(const vec<L, T>& x, const vec<L, T>& lo, const vec<L, T>& hi) {
	return glm::min(glm::max(x, lo), hi);
}

template <typename V, if_vec<V> = 0> typename V::value_type dot(const V& a, const V& b) { return detail::dot(a, b); }

template <typename V, if_vec<V> = 0> V cross(const V& a, const V& b) {
	return V(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}

template <typename V, if_vec<V> = 0> typename V::value_type length(const V& v) { return std::sqrt(detail::dot(v, v)); }
template <typename V, if_vec<V> = 0> typename V::value_type distance(const V& a, const V& b) { return glm::length(b - a); }
// normalize(v) = v * (1 / sqrt(dot(v, v)))
template <typename V, if_vec<V> = 0> V normalize(const V& v) {
	using T = typename V::value_type;
	return v * (static_cast<T>(1) / std::sqrt(detail::dot(v, v)));
}

// ---------------------------------------------------------------- 4x4 column-major matrix
template <std::size_t C, std::size_t R, typename T> struct mat;

template <typename T> struct mat<4, 4, T> {
	using col_type = vec<4, T>;
	using length_type = length_t;
	col_type value[4];

	mat() : mat(static_cast<T>(1)) {}
	explicit mat(T s) {
		value[0] = col_type(s, 0, 0, 0);
		value[1] = col_type(0, s, 0, 0);
		value[2] = col_type(0, 0, s, 0);
		value[3] = col_type(0, 0, 0, s);
	}
	mat(const col_type& c0, const col_type& c1, const col_type& c2, const col_type& c3) {
		value[0] = c0; value[1] = c1; value[2] = c2; value[3] = c3;
	}
	static constexpr length_t length() { return 4; }
	col_type& operator[](length_t i) { return value[i]; }
	const col_type& operator[](length_t i) const { return value[i]; }
};

using mat4 = mat<4, 4, float>;

// m * v = (m[0] * v.x + m[1] * v.y) + (m[2] * v.z + m[3] * v.w)
template <typename T> vec<4, T> operator*(const mat<4, 4, T>& m, const vec<4, T>& v) {
	const vec<4, T> a0 = m[0] * v.x + m[1] * v.y;
	const vec<4, T> a1 = m[2] * v.z + m[3] * v.w;
	return a0 + a1;
}

// (a * b)[i] = ((a[0] * b[i].x + a[1] * b[i].y) + a[2] * b[i].z) + a[3] * b[i].w
template <typename T> mat<4, 4, T> operator*(const mat<4, 4, T>& a, const mat<4, 4, T>& b) {
	mat<4, 4, T> r;
	for (length_t i = 0; i < 4; i++)
		r[i] = a[0] * b[i].x + a[1] * b[i].y + a[2] * b[i].z + a[3] * b[i].w;
	return r;
}

template <typename T> bool operator==(const mat<4, 4, T>& a, const mat<4, 4, T>& b) {
	for (length_t i = 0; i < 4; i++) if (a[i] != b[i]) return false;
	return true;
}
template <typename T> bool operator!=(const mat<4, 4, T>& a, const mat<4, 4, T>& b) { return !(a == b); }

template <typename M> struct is_mat : std::false_type {};
template <typename T> struct is_mat<mat<4, 4, T>> : std::true_type {};
template <typename M> using if_mat = std::enable_if_t<is_mat<M>::value, int>;

// transpose and inverse are constrained templates for the same lookup reason
// as the vector functions above.
template <typename M, if_mat<M> = 0> M transpose(const M& m) {
	M r;
	for (length_t c = 0; c < 4; c++)
		for (length_t row = 0; row < 4; row++) r[c][row] = m[row][c];
	return r;
}

// Inverse by the adjugate: the 2x2 sub-determinants of the lower and upper
// row pairs are formed once, every cofactor is built from them, and the
// adjugate is scaled by 1 / det (det expanded along the first column).
template <typename M, if_mat<M> = 0> M inverse(const M& m) {
	using T = typename M::col_type::value_type;
	// a(r, c) = element at row r, column c
	auto a = [&](int r, int c) { return m[c][r]; };
	const T s0 = a(0, 0) * a(1, 1) - a(1, 0) * a(0, 1);
	const T s1 = a(0, 0) * a(1, 2) - a(1, 0) * a(0, 2);
	const T s2 = a(0, 0) * a(1, 3) - a(1, 0) * a(0, 3);
	const T s3 = a(0, 1) * a(1, 2) - a(1, 1) * a(0, 2);
	const T s4 = a(0, 1) * a(1, 3) - a(1, 1) * a(0, 3);
	const T s5 = a(0, 2) * a(1, 3) - a(1, 2) * a(0, 3);
	const T c5 = a(2, 2) * a(3, 3) - a(3, 2) * a(2, 3);
	const T c4 = a(2, 1) * a(3, 3) - a(3, 1) * a(2, 3);
	const T c3 = a(2, 1) * a(3, 2) - a(3, 1) * a(2, 2);
	const T c2 = a(2, 0) * a(3, 3) - a(3, 0) * a(2, 3);
	const T c1 = a(2, 0) * a(3, 2) - a(3, 0) * a(2, 2);
	const T c0 = a(2, 0) * a(3, 1) - a(3, 0) * a(2, 1);
	const T det = s0 * c5 - s1 * c4 + s2 * c3 + s3 * c2 - s4 * c1 + s5 * c0;
	const T inv = static_cast<T>(1) / det;
	M r;
	// r(row, col) stored as r[col][row]
	r[0][0] = (a(1, 1) * c5 - a(1, 2) * c4 + a(1, 3) * c3) * inv;
	r[1][0] = (-a(0, 1) * c5 + a(0, 2) * c4 - a(0, 3) * c3) * inv;
	r[2][0] = (a(3, 1) * s5 - a(3, 2) * s4 + a(3, 3) * s3) * inv;
	r[3][0] = (-a(2, 1) * s5 + a(2, 2) * s4 - a(2, 3) * s3) * inv;
	r[0][1] = (-a(1, 0) * c5 + a(1, 2) * c2 - a(1, 3) * c1) * inv;
	r[1][1] = (a(0, 0) * c5 - a(0, 2) * c2 + a(0, 3) * c1) * inv;
	r[2][1] = (-a(3, 0) * s5 + a(3, 2) * s2 - a(3, 3) * s1) * inv;
	r[3][1] = (a(2, 0) * s5 - a(2, 2) * s2 + a(2, 3) * s1) * inv;
	r[0][2] = (a(1, 0) * c4 - a(1, 1) * c2 + a(1, 3) * c0) * inv;
	r[1][2] = (-a(0, 0) * c4 + a(0, 1) * c2 - a(0, 3) * c0) * inv;
	r[2][2] = (a(3, 0) * s4 - a(3, 1) * s2 + a(3, 3) * s0) * inv;
	r[3][2] = (-a(2, 0) * s4 + a(2, 1) * s2 - a(2, 3) * s0) * inv;
	r[0][3] = (-a(1, 0) * c3 + a(1, 1) * c1 - a(1, 2) * c0) * inv;
	r[1][3] = (a(0, 0) * c3 - a(0, 1) * c1 + a(0, 2) * c0) * inv;
	r[2][3] = (-a(3, 0) * s3 + a(3, 1) * s1 - a(3, 2) * s0) * inv;
	r[3][3] = (a(2, 0) * s3 - a(2, 1) * s1 + a(2, 2) * s0) * inv;
	return r;
}

} // namespace glm

// The reference calls isinf/isnan unqualified (shapes/shape.cpp:41,57,
// spectrums/detail/coefficient_specturm.hpp:33), which MSVC's <cmath> exposes
// in the global namespace; libstdc++ only declares them in std.
using std::isinf;
using std::isnan;
