// Seeded synthetic scenes for the benchmark configurations.
//
// The reference ships no scene loader (its front-end lives in another
// repository), so scenes are generated here and handed to the core, and to
// the oracle, as one rb_scene_desc:
//   RB_SCENE_BOX      closed box room, 32 triangles: a unit room with the +z face
//                     open (10), two inner boxes without bottoms rotated by 15 and
//                     -18 degrees about y (2 x 10) and a 0.25 x 0.25 quad light (2);
//                     Lambert 0.73 grey, red (0.65, 0.05, 0.05), green (0.12, 0.45, 0.15);
//                     light radiance (17, 12, 4); camera 40 degrees.
//   RB_SCENE_SPHERES  num_spheres displaced icospheres (radius U[0.05, 0.5], centre
//                     U[0, 10]^3, radial gradient-noise displacement of relative
//                     amplitude 0.1) over a ground quad; 40% Lambert, 30% rough
//                     conductor, 30% dielectric (IOR 1.5, roughness U[0, 0.3], values
//                     below 0.03 snapped to 0 = smooth); 4 quad lights and a constant
//                     environment of 0.5.
//   RB_SCENE_SLIT_ROOM glossy room whose only light sits behind a wall with a slit,
//                     filled with displaced-sphere clutter.
// Random numbers come from a PCG32 of this file (not the renderer's sampler).
#include "../../../include/rbgpu.h"
#include "../rb_math.h"
#include "camera_math.h"

#include <cmath>
#include <cstring>
#include <map>
#include <new>
#include <utility>
#include <vector>

using rb::vec3;

namespace {

struct gen_rng {
	uint64_t state, inc;
	explicit gen_rng(uint64_t seed, uint64_t stream = 0x9e3779b97f4a7c15ull) : state(0), inc((stream << 1u) | 1u) {
		next();
		state += seed;
		next();
	}
	uint32_t next() {
		const uint64_t old = state;
		state = old * 6364136223846793005ull + inc;
		const uint32_t xs = static_cast<uint32_t>(((old >> 18u) ^ old) >> 27u);
		const uint32_t rot = static_cast<uint32_t>(old >> 59u);
		return (xs >> rot) | (xs << ((32u - rot) & 31u));
	}
	float uniform() { return static_cast<float>(next() >> 8) * (1.f / 16777216.f); }
	float range(float a, float b) { return a + (b - a) * uniform(); }
};

// Gradient noise on an integer lattice with a seeded permutation (Perlin's
// improved-noise construction: quintic fade, 12 edge gradients).
struct gradient_noise {
	int perm[512];
	explicit gradient_noise(uint64_t seed) {
		gen_rng r(seed, 0x5851f42d4c957f2dull);
		for (int i = 0; i < 256; i++) perm[i] = i;
		for (int i = 255; i > 0; i--) {
			const int j = static_cast<int>(r.next() % static_cast<uint32_t>(i + 1));
			std::swap(perm[i], perm[j]);
		}
		for (int i = 0; i < 256; i++) perm[256 + i] = perm[i];
	}
	static double fade(double t) { return t * t * t * (t * (t * 6 - 15) + 10); }
	static double grad(int h, double x, double y, double z) {
		static const int g[12][3] = {{1, 1, 0}, {-1, 1, 0}, {1, -1, 0}, {-1, -1, 0}, {1, 0, 1}, {-1, 0, 1},
			{1, 0, -1}, {-1, 0, -1}, {0, 1, 1}, {0, -1, 1}, {0, 1, -1}, {0, -1, -1}};
		const int* v = g[h % 12];
		return v[0] * x + v[1] * y + v[2] * z;
	}
	static double lerp(double t, double a, double b) { return a + t * (b - a); }
	double operator()(double x, double y, double z) const {
		const double fx = std::floor(x), fy = std::floor(y), fz = std::floor(z);
		const int X = static_cast<int>(fx) & 255, Y = static_cast<int>(fy) & 255, Z = static_cast<int>(fz) & 255;
		x -= fx; y -= fy; z -= fz;
		const double u = fade(x), v = fade(y), w = fade(z);
		const int A = perm[X] + Y, AA = perm[A] + Z, AB = perm[A + 1] + Z;
		const int B = perm[X + 1] + Y, BA = perm[B] + Z, BB = perm[B + 1] + Z;
		return lerp(w,
			lerp(v, lerp(u, grad(perm[AA], x, y, z), grad(perm[BA], x - 1, y, z)),
				lerp(u, grad(perm[AB], x, y - 1, z), grad(perm[BB], x - 1, y - 1, z))),
			lerp(v, lerp(u, grad(perm[AA + 1], x, y, z - 1), grad(perm[BA + 1], x - 1, y, z - 1)),
				lerp(u, grad(perm[AB + 1], x, y - 1, z - 1), grad(perm[BB + 1], x - 1, y - 1, z - 1))));
	}
};

struct mesh_data {
	std::vector<float> positions, normals, uvs;
	std::vector<uint32_t> indices;
	int32_t reverse = 0;
	void add_vertex(vec3 p) { positions.insert(positions.end(), {p.x, p.y, p.z}); }
	uint32_t vertex_count() const { return static_cast<uint32_t>(positions.size() / 3); }
	void add_quad(vec3 a, vec3 b, vec3 c, vec3 d) {
		// triangles (a, b, c) and (a, c, d); geometric normal along (b - a) x (c - a)
		const uint32_t base = vertex_count();
		add_vertex(a); add_vertex(b); add_vertex(c); add_vertex(d);
		indices.insert(indices.end(), {base, base + 1, base + 2, base, base + 2, base + 3});
	}
};

rb_material_desc matte(float r, float g, float b) {
	rb_material_desc m{};
	m.kind = RB_MATERIAL_MATTE;
	m.diffuse[0] = r; m.diffuse[1] = g; m.diffuse[2] = b;
	m.sigma = 0.f;
	return m;
}

rb_material_desc metal(float roughness) {
	// Copper-like RGB conductor constants chosen for the synthetic scenes.
	rb_material_desc m{};
	m.kind = RB_MATERIAL_METAL;
	m.remap_roughness = 1;
	m.eta[0] = 0.200438f; m.eta[1] = 0.924033f; m.eta[2] = 1.102212f;
	m.k[0] = 3.912949f; m.k[1] = 2.452848f; m.k[2] = 2.142188f;
	m.roughness_u = m.roughness_v = roughness;
	return m;
}

rb_material_desc glass(float roughness, float ior) {
	rb_material_desc m{};
	m.kind = RB_MATERIAL_GLASS;
	m.remap_roughness = 1;
	for (int i = 0; i < 3; i++) m.reflectance[i] = m.transmission[i] = 1.f;
	m.ior = ior;
	m.roughness_u = m.roughness_v = roughness;
	return m;
}

void set_identity(float* m) {
	for (int i = 0; i < 16; i++) m[i] = (i % 5 == 0) ? 1.f : 0.f;
}

} // namespace

struct rb_scene {
	std::vector<mesh_data> meshes;
	std::vector<rb_mesh_desc> mesh_descs;
	std::vector<rb_entity_desc> entities;
	std::vector<rb_material_desc> materials;
	std::vector<rb_emitter_desc> emitters;
	std::vector<rb_medium_desc> mediums;
	std::vector<rb_media_desc> media;
	rb_camera_desc camera{};

	int32_t add_material(const rb_material_desc& m) {
		materials.push_back(m);
		return static_cast<int32_t>(materials.size() - 1);
	}
	int32_t add_emitter(uint32_t kind, float r, float g, float b, float radius = 0.f) {
		rb_emitter_desc e{};
		e.kind = kind;
		e.radiance[0] = r; e.radiance[1] = g; e.radiance[2] = b;
		e.radius = radius;
		emitters.push_back(e);
		return static_cast<int32_t>(emitters.size() - 1);
	}
	// Adds an entity over a new mesh with the given local-to-world transform.
	void add_entity(mesh_data&& mesh, int32_t material, int32_t emitter, const rb::host::xform& xf) {
		meshes.push_back(std::move(mesh));
		rb_entity_desc e{};
		e.mesh = static_cast<int32_t>(meshes.size() - 1);
		e.material = material;
		e.emitter = emitter;
		e.medium = -1;
		std::memcpy(e.local_to_world, xf.m.m, sizeof(e.local_to_world));
		std::memcpy(e.world_to_local, xf.inv.m, sizeof(e.world_to_local));
		entities.push_back(e);
	}
	void add_shapeless_emitter(int32_t emitter) {
		rb_entity_desc e{};
		e.mesh = -1;
		e.material = -1;
		e.emitter = emitter;
		e.medium = -1;
		set_identity(e.local_to_world);
		set_identity(e.world_to_local);
		entities.push_back(e);
	}
	void finalize() {
		mesh_descs.clear();
		for (const mesh_data& m : meshes) {
			rb_mesh_desc d{};
			d.positions = m.positions.data();
			d.normals = m.normals.empty() ? nullptr : m.normals.data();
			d.tangents = nullptr;
			d.uvs = m.uvs.empty() ? nullptr : m.uvs.data();
			d.indices = m.indices.data();
			d.num_vertices = m.vertex_count();
			d.num_triangles = static_cast<uint32_t>(m.indices.size() / 3);
			d.reverse_orientation = m.reverse;
			mesh_descs.push_back(d);
		}
	}
};

namespace {

rb::host::xform identity_xf() { return rb::host::xform{rb::mat_identity(), rb::mat_identity()}; }

// Rotation about +y by `degrees`, composed after a translation: L2W = T(c) * R(a).
rb::host::xform translate_rotate_y(vec3 c, float degrees) {
	const double a = degrees * 3.14159265358979323846 / 180.0;
	const float cs = static_cast<float>(std::cos(a)), sn = static_cast<float>(std::sin(a));
	rb::mat4 r = rb::mat_identity(), rt = rb::mat_identity();
	r.m[0] = cs; r.m[2] = -sn; r.m[8] = sn; r.m[10] = cs;
	rt.m[0] = cs; rt.m[2] = sn; rt.m[8] = -sn; rt.m[10] = cs;
	const rb::host::xform rot{r, rt};
	return rb::host::compose(rb::host::translate_xf(c), rot);
}

// Open-bottom box centred on the origin in x/z, standing on y = 0.
mesh_data open_box(float w, float h, float d) {
	mesh_data m;
	const float x0 = -0.5f * w, x1 = 0.5f * w, z0 = -0.5f * d, z1 = 0.5f * d;
	m.add_quad(vec3{x0, h, z0}, vec3{x0, h, z1}, vec3{x1, h, z1}, vec3{x1, h, z0});  // top, +y
	m.add_quad(vec3{x0, 0, z1}, vec3{x1, 0, z1}, vec3{x1, h, z1}, vec3{x0, h, z1});  // +z
	m.add_quad(vec3{x1, 0, z0}, vec3{x0, 0, z0}, vec3{x0, h, z0}, vec3{x1, h, z0});  // -z
	m.add_quad(vec3{x0, 0, z0}, vec3{x0, 0, z1}, vec3{x0, h, z1}, vec3{x0, h, z0});  // -x
	m.add_quad(vec3{x1, 0, z1}, vec3{x1, 0, z0}, vec3{x1, h, z0}, vec3{x1, h, z1});  // +x
	return m;
}

void build_box_scene(rb_scene& s, int width, int height) {
	const int32_t white = s.add_material(matte(0.73f, 0.73f, 0.73f));
	const int32_t red = s.add_material(matte(0.65f, 0.05f, 0.05f));
	const int32_t green = s.add_material(matte(0.12f, 0.45f, 0.15f));
	const int32_t black = s.add_material(matte(0.f, 0.f, 0.f));
	const int32_t light = s.add_emitter(RB_EMITTER_SURFACE, 17.f, 12.f, 4.f);

	// room [0,1]^3, open at z = 1, faces turned inward
	mesh_data room;
	room.add_quad(vec3{0, 0, 0}, vec3{0, 0, 1}, vec3{1, 0, 1}, vec3{1, 0, 0});  // floor, normal +y
	room.add_quad(vec3{0, 1, 0}, vec3{1, 1, 0}, vec3{1, 1, 1}, vec3{0, 1, 1});  // ceiling, -y
	room.add_quad(vec3{0, 0, 0}, vec3{1, 0, 0}, vec3{1, 1, 0}, vec3{0, 1, 0});  // back, +z
	s.add_entity(std::move(room), white, -1, identity_xf());
	mesh_data left;
	left.add_quad(vec3{0, 0, 0}, vec3{0, 1, 0}, vec3{0, 1, 1}, vec3{0, 0, 1});  // x = 0, +x
	s.add_entity(std::move(left), red, -1, identity_xf());
	mesh_data right;
	right.add_quad(vec3{1, 0, 0}, vec3{1, 0, 1}, vec3{1, 1, 1}, vec3{1, 1, 0});  // x = 1, -x
	s.add_entity(std::move(right), green, -1, identity_xf());

	s.add_entity(open_box(0.3f, 0.3f, 0.3f), white, -1, translate_rotate_y(vec3{0.67f, 0.f, 0.64f}, 15.f));
	s.add_entity(open_box(0.3f, 0.6f, 0.3f), white, -1, translate_rotate_y(vec3{0.33f, 0.f, 0.36f}, -18.f));

	// light quad just under the ceiling, emitting downwards
	mesh_data lq;
	const float a = 0.5f - 0.125f, b = 0.5f + 0.125f, y = 0.998f;
	lq.add_quad(vec3{a, y, a}, vec3{b, y, a}, vec3{b, y, b}, vec3{a, y, b});
	s.add_entity(std::move(lq), black, light, identity_xf());

	rb_camera_desc& c = s.camera;
	c.eye[0] = 0.5f; c.eye[1] = 0.5f; c.eye[2] = 2.4f;
	c.target[0] = 0.5f; c.target[1] = 0.5f; c.target[2] = 0.f;
	c.up[0] = 0.f; c.up[1] = 1.f; c.up[2] = 0.f;
	c.fov_degrees = 40.f;
	c.width = width;
	c.height = height;
}

// Unit icosphere of subdivision `level` (20 * 4^level faces), vertices shared.
void icosphere(int level, std::vector<vec3>& verts, std::vector<uint32_t>& faces) {
	const double t = (1.0 + std::sqrt(5.0)) / 2.0;
	const double base[12][3] = {{-1, t, 0}, {1, t, 0}, {-1, -t, 0}, {1, -t, 0}, {0, -1, t}, {0, 1, t},
		{0, -1, -t}, {0, 1, -t}, {t, 0, -1}, {t, 0, 1}, {-t, 0, -1}, {-t, 0, 1}};
	std::vector<double> dv;
	for (const auto& v : base) {
		const double l = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
		dv.insert(dv.end(), {v[0] / l, v[1] / l, v[2] / l});
	}
	faces = {0, 11, 5, 0, 5, 1, 0, 1, 7, 0, 7, 10, 0, 10, 11, 1, 5, 9, 5, 11, 4, 11, 10, 2, 10, 7, 6, 7, 1, 8,
		3, 9, 4, 3, 4, 2, 3, 2, 6, 3, 6, 8, 3, 8, 9, 4, 9, 5, 2, 4, 11, 6, 2, 10, 8, 6, 7, 9, 8, 1};
	for (int l = 0; l < level; l++) {
		std::map<std::pair<uint32_t, uint32_t>, uint32_t> mids;
		auto mid = [&](uint32_t a, uint32_t b) {
			const auto key = a < b ? std::make_pair(a, b) : std::make_pair(b, a);
			auto it = mids.find(key);
			if (it != mids.end()) return it->second;
			double m[3] = {dv[3 * a] + dv[3 * b], dv[3 * a + 1] + dv[3 * b + 1], dv[3 * a + 2] + dv[3 * b + 2]};
			const double len = std::sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
			const uint32_t id = static_cast<uint32_t>(dv.size() / 3);
			dv.insert(dv.end(), {m[0] / len, m[1] / len, m[2] / len});
			mids.emplace(key, id);
			return id;
		};
		std::vector<uint32_t> nf;
		nf.reserve(faces.size() * 4);
		for (size_t f = 0; f < faces.size(); f += 3) {
			const uint32_t a = faces[f], b = faces[f + 1], c = faces[f + 2];
			const uint32_t ab = mid(a, b), bc = mid(b, c), ca = mid(c, a);
			nf.insert(nf.end(), {a, ab, ca, b, bc, ab, c, ca, bc, ab, bc, ca});
		}
		faces.swap(nf);
	}
	verts.clear();
	for (size_t i = 0; i < dv.size(); i += 3)
		verts.push_back(vec3{static_cast<float>(dv[i]), static_cast<float>(dv[i + 1]), static_cast<float>(dv[i + 2])});
}

// Displaced unit sphere: vertex v -> v * (1 + amplitude * noise(v * frequency + offset)).
mesh_data displaced_sphere(const std::vector<vec3>& unit, const std::vector<uint32_t>& faces,
	const gradient_noise& noise, vec3 offset, float amplitude, float frequency) {
	mesh_data m;
	m.positions.reserve(unit.size() * 3);
	for (const vec3& v : unit) {
		const double n = noise(v.x * frequency + offset.x, v.y * frequency + offset.y, v.z * frequency + offset.z);
		const float s = static_cast<float>(1.0 + amplitude * n);
		m.add_vertex(vec3{v.x * s, v.y * s, v.z * s});
	}
	m.indices = faces;
	return m;
}

rb::host::xform translate_scale(vec3 c, float r) {
	return rb::host::compose(rb::host::translate_xf(c), rb::host::scale_xf(vec3{r, r, r}));
}

int32_t random_material(rb_scene& s, gen_rng& rng) {
	const float pick = rng.uniform();
	if (pick < 0.4f) {
		const float a = rng.range(0.1f, 0.9f), b = rng.range(0.1f, 0.9f), c = rng.range(0.1f, 0.9f);
		return s.add_material(matte(a, b, c));
	}
	if (pick < 0.7f) return s.add_material(metal(rng.range(0.05f, 0.8f)));
	float rough = rng.range(0.f, 0.3f);
	if (rough < 0.03f) rough = 0.f;
	return s.add_material(glass(rough, 1.5f));
}

void build_sphere_scene(rb_scene& s, uint32_t seed, uint32_t count, int level, int width, int height) {
	gen_rng rng(0x1234567ull + seed);
	const gradient_noise noise(seed * 7919ull + 13ull);
	std::vector<vec3> unit;
	std::vector<uint32_t> faces;
	icosphere(level, unit, faces);

	const int32_t black = s.add_material(matte(0.f, 0.f, 0.f));
	for (uint32_t i = 0; i < count; i++) {
		const float r = rng.range(0.05f, 0.5f);
		const vec3 c{rng.range(0.f, 10.f), rng.range(0.f, 10.f), rng.range(0.f, 10.f)};
		const vec3 off{rng.range(0.f, 100.f), rng.range(0.f, 100.f), rng.range(0.f, 100.f)};
		const int32_t mat = random_material(s, rng);
		s.add_entity(displaced_sphere(unit, faces, noise, off, 0.1f, 2.5f), mat, -1, translate_scale(c, r));
	}
	// ground quad at y = -0.5
	mesh_data ground;
	ground.add_quad(vec3{-20, -0.5f, -20}, vec3{-20, -0.5f, 30}, vec3{30, -0.5f, 30}, vec3{30, -0.5f, -20});
	s.add_entity(std::move(ground), s.add_material(matte(0.5f, 0.5f, 0.5f)), -1, identity_xf());
	// four 2 x 2 quad lights at y = 13 facing down
	for (int i = 0; i < 4; i++) {
		const float cx = (i & 1) ? 7.5f : 2.5f, cz = (i & 2) ? 7.5f : 2.5f;
		mesh_data q;
		q.add_quad(vec3{cx - 1, 13, cz - 1}, vec3{cx + 1, 13, cz - 1}, vec3{cx + 1, 13, cz + 1}, vec3{cx - 1, 13, cz + 1});
		const int32_t e = s.add_emitter(RB_EMITTER_SURFACE, rng.range(4.f, 12.f), rng.range(4.f, 12.f), rng.range(4.f, 12.f));
		s.add_entity(std::move(q), black, e, identity_xf());
	}
	// constant environment; radius encloses the ground quad
	s.add_shapeless_emitter(s.add_emitter(RB_EMITTER_ENVIRONMENT, 0.5f, 0.5f, 0.5f, 40.f));

	rb_camera_desc& c = s.camera;
	c.eye[0] = 5.f; c.eye[1] = 9.f; c.eye[2] = 25.f;
	c.target[0] = 5.f; c.target[1] = 3.5f; c.target[2] = 5.f;
	c.up[0] = 0.f; c.up[1] = 1.f; c.up[2] = 0.f;
	c.fov_degrees = 40.f;
	c.width = width;
	c.height = height;
}

// Sphere field inside a homogeneous medium (sigma_a 0.02, sigma_s 0.1,
// Henyey-Greenstein g = 0.6): the medium is the inside of an invisible box
// entity (no material) around the spheres, the ground and 16 quad lights of
// seeded radiance U[5, 40]; the camera looks in from outside the box, where
// rays travel in vacuum.
void build_fog_scene(rb_scene& s, uint32_t seed, uint32_t count, int level, int width, int height) {
	gen_rng rng(0xf09f09ull + seed);
	const gradient_noise noise(seed * 6151ull + 29ull);
	std::vector<vec3> unit;
	std::vector<uint32_t> faces;
	icosphere(level, unit, faces);
	const int32_t black = s.add_material(matte(0.f, 0.f, 0.f));
	for (uint32_t i = 0; i < count; i++) {
		const float r = rng.range(0.05f, 0.5f);
		const vec3 c{rng.range(0.f, 10.f), rng.range(0.f, 10.f), rng.range(0.f, 10.f)};
		const vec3 off{rng.range(0.f, 100.f), rng.range(0.f, 100.f), rng.range(0.f, 100.f)};
		const int32_t mat = random_material(s, rng);
		s.add_entity(displaced_sphere(unit, faces, noise, off, 0.1f, 2.5f), mat, -1, translate_scale(c, r));
	}
	mesh_data ground;
	ground.add_quad(vec3{-20, -0.5f, -20}, vec3{-20, -0.5f, 30}, vec3{30, -0.5f, 30}, vec3{30, -0.5f, -20});
	s.add_entity(std::move(ground), s.add_material(matte(0.5f, 0.5f, 0.5f)), -1, identity_xf());
	// 16 quad lights of 0.6 x 0.6 on a 4 x 4 grid at y = 11.5, facing down
	for (int i = 0; i < 16; i++) {
		const float cx = 1.25f + 2.5f * static_cast<float>(i & 3), cz = 1.25f + 2.5f * static_cast<float>(i >> 2);
		mesh_data q;
		q.add_quad(vec3{cx - 0.3f, 11.5f, cz - 0.3f}, vec3{cx + 0.3f, 11.5f, cz - 0.3f}, vec3{cx + 0.3f, 11.5f, cz + 0.3f},
			vec3{cx - 0.3f, 11.5f, cz + 0.3f});
		const float L = rng.range(5.f, 40.f);
		s.add_entity(std::move(q), black, s.add_emitter(RB_EMITTER_SURFACE, L, L, L), identity_xf());
	}
	// the medium box [-1, 11] x [-1, 12.5] x [-1, 11], faces wound outwards
	rb_medium_desc fog{};
	for (int c = 0; c < 3; c++) { fog.sigma_a[c] = 0.02f; fog.sigma_s[c] = 0.1f; }
	fog.g = 0.6f;
	s.mediums.push_back(fog);
	s.media.push_back(rb_media_desc{0, -1});
	const float x0 = -1.f, x1 = 11.f, y0 = -1.f, y1 = 12.5f, z0 = -1.f, z1 = 11.f;
	mesh_data box;
	box.add_quad(vec3{x0, y0, z0}, vec3{x1, y0, z0}, vec3{x1, y0, z1}, vec3{x0, y0, z1});  // -y
	box.add_quad(vec3{x0, y1, z0}, vec3{x0, y1, z1}, vec3{x1, y1, z1}, vec3{x1, y1, z0});  // +y
	box.add_quad(vec3{x0, y0, z0}, vec3{x0, y0, z1}, vec3{x0, y1, z1}, vec3{x0, y1, z0});  // -x
	box.add_quad(vec3{x1, y0, z0}, vec3{x1, y1, z0}, vec3{x1, y1, z1}, vec3{x1, y0, z1});  // +x
	box.add_quad(vec3{x0, y0, z0}, vec3{x0, y1, z0}, vec3{x1, y1, z0}, vec3{x1, y0, z0});  // -z
	box.add_quad(vec3{x0, y0, z1}, vec3{x1, y0, z1}, vec3{x1, y1, z1}, vec3{x0, y1, z1});  // +z
	s.add_entity(std::move(box), -1, -1, identity_xf());
	s.entities.back().medium = 0;

	rb_camera_desc& c = s.camera;
	c.eye[0] = 5.f; c.eye[1] = 8.f; c.eye[2] = 26.f;
	c.target[0] = 5.f; c.target[1] = 3.5f; c.target[2] = 5.f;
	c.up[0] = 0.f; c.up[1] = 1.f; c.up[2] = 0.f;
	c.fov_degrees = 45.f;
	c.width = width;
	c.height = height;
}

void build_slit_room(rb_scene& s, uint32_t seed, uint32_t count, int level, int width, int height) {
	gen_rng rng(0xabcdefull + seed);
	const gradient_noise noise(seed * 104729ull + 7ull);
	std::vector<vec3> unit;
	std::vector<uint32_t> faces;
	icosphere(level, unit, faces);
	const int32_t black = s.add_material(matte(0.f, 0.f, 0.f));
	const int32_t white = s.add_material(matte(0.7f, 0.7f, 0.7f));
	// room [0,10] x [0,5] x [0,10]; glossy floor and walls
	mesh_data floor_m, walls;
	floor_m.add_quad(vec3{0, 0, 0}, vec3{0, 0, 10}, vec3{10, 0, 10}, vec3{10, 0, 0});
	s.add_entity(std::move(floor_m), s.add_material(metal(rng.range(0.1f, 0.3f))), -1, identity_xf());
	walls.add_quad(vec3{0, 5, 0}, vec3{10, 5, 0}, vec3{10, 5, 10}, vec3{0, 5, 10});     // ceiling
	walls.add_quad(vec3{0, 0, 0}, vec3{0, 5, 0}, vec3{0, 5, 10}, vec3{0, 0, 10});       // x = 0
	walls.add_quad(vec3{10, 0, 0}, vec3{10, 0, 10}, vec3{10, 5, 10}, vec3{10, 5, 0});   // x = 10
	walls.add_quad(vec3{0, 0, 10}, vec3{0, 5, 10}, vec3{10, 5, 10}, vec3{10, 0, 10});   // z = 10 (behind camera)
	s.add_entity(std::move(walls), s.add_material(metal(rng.range(0.1f, 0.3f))), -1, identity_xf());
	// dividing wall at z = 2 with a 0.3-wide horizontal slit at y in [2.35, 2.65]
	mesh_data divider;
	divider.add_quad(vec3{0, 0, 2}, vec3{0, 2.35f, 2}, vec3{10, 2.35f, 2}, vec3{10, 0, 2});
	divider.add_quad(vec3{0, 2.65f, 2}, vec3{0, 5, 2}, vec3{10, 5, 2}, vec3{10, 2.65f, 2});
	s.add_entity(std::move(divider), white, -1, identity_xf());
	// back wall of the light chamber
	mesh_data back;
	back.add_quad(vec3{0, 0, 0}, vec3{10, 0, 0}, vec3{10, 5, 0}, vec3{0, 5, 0});
	s.add_entity(std::move(back), white, -1, identity_xf());
	// 0.5 x 0.5 light, radiance 50, facing the back wall of its chamber (-z):
	// no point of the room sees it, all light enters the room through the slit
	// after at least one bounce in the chamber (hard indirect lighting)
	mesh_data lq;
	lq.add_quad(vec3{4.75f, 2.25f, 0.5f}, vec3{4.75f, 2.75f, 0.5f}, vec3{5.25f, 2.75f, 0.5f}, vec3{5.25f, 2.25f, 0.5f});
	s.add_entity(std::move(lq), black, s.add_emitter(RB_EMITTER_SURFACE, 50.f, 50.f, 50.f), identity_xf());
	// clutter
	for (uint32_t i = 0; i < count; i++) {
		const float r = rng.range(0.1f, 0.45f);
		const vec3 c{rng.range(0.5f, 9.5f), r, rng.range(3.f, 9.f)};
		const vec3 off{rng.range(0.f, 100.f), rng.range(0.f, 100.f), rng.range(0.f, 100.f)};
		s.add_entity(displaced_sphere(unit, faces, noise, off, 0.1f, 2.5f), random_material(s, rng), -1, translate_scale(c, r));
	}
	rb_camera_desc& c = s.camera;
	c.eye[0] = 5.f; c.eye[1] = 2.5f; c.eye[2] = 9.8f;
	c.target[0] = 5.f; c.target[1] = 1.5f; c.target[2] = 2.f;
	c.up[0] = 0.f; c.up[1] = 1.f; c.up[2] = 0.f;
	c.fov_degrees = 60.f;
	c.width = width;
	c.height = height;
}

} // namespace

extern "C" rb_status rb_scene_generate(const rb_scene_gen_params* params, rb_scene** out) {
	if (params == nullptr || out == nullptr) return RB_ERR_INVALID_ARGUMENT;
	*out = nullptr;
	if (params->width <= 0 || params->height <= 0 || params->width > 16384 || params->height > 16384) return RB_ERR_INVALID_ARGUMENT;
	if (params->subdivision > 7) return RB_ERR_INVALID_ARGUMENT;
	try {
		rb_scene* s = new rb_scene();
		switch (params->kind) {
		case RB_SCENE_BOX: build_box_scene(*s, params->width, params->height); break;
		case RB_SCENE_SPHERES:
			build_sphere_scene(*s, params->seed, params->num_spheres, static_cast<int>(params->subdivision), params->width, params->height);
			break;
		case RB_SCENE_SLIT_ROOM:
			build_slit_room(*s, params->seed, params->num_spheres, static_cast<int>(params->subdivision), params->width, params->height);
			break;
		case RB_SCENE_FOG:
			build_fog_scene(*s, params->seed, params->num_spheres, static_cast<int>(params->subdivision), params->width, params->height);
			break;
		default: delete s; return RB_ERR_INVALID_ARGUMENT;
		}
		s->finalize();
		rb::host::camera_matrices(s->camera);
		*out = s;
	} catch (const std::bad_alloc&) {
		return RB_ERR_OUT_OF_MEMORY;
	}
	return RB_OK;
}

extern "C" rb_status rb_scene_get(const rb_scene* s, rb_scene_desc* desc, rb_camera_desc* camera) {
	if (s == nullptr) return RB_ERR_INVALID_ARGUMENT;
	if (desc != nullptr) {
		std::memset(desc, 0, sizeof(*desc));
		desc->meshes = s->mesh_descs.data();
		desc->num_meshes = static_cast<uint32_t>(s->mesh_descs.size());
		desc->entities = s->entities.data();
		desc->num_entities = static_cast<uint32_t>(s->entities.size());
		desc->materials = s->materials.data();
		desc->num_materials = static_cast<uint32_t>(s->materials.size());
		desc->emitters = s->emitters.data();
		desc->num_emitters = static_cast<uint32_t>(s->emitters.size());
		desc->mediums = s->mediums.data();
		desc->num_mediums = static_cast<uint32_t>(s->mediums.size());
		desc->media = s->media.data();
		desc->num_media = static_cast<uint32_t>(s->media.size());
	}
	if (camera != nullptr) *camera = s->camera;
	return RB_OK;
}

extern "C" void rb_scene_free(rb_scene* s) { delete s; }
