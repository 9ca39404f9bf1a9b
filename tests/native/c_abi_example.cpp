// C++ host program on the C ABI alone (include/rbgpu.h): what an integrator
// adapter in the reference renderer does, without Python. Generates the box
// room, uploads it, renders 16 spp through rb_render, then two scenes through
// one batched render, and prints one line of results. Exit code 0 on success;
// on a machine without a GPU it prints the status and exits 0 as well (the
// library reports RB_ERR_NO_DEVICE instead of falling back to the CPU).
#include "../../include/rbgpu.h"

#include <cmath>
#include <cstdio>
#include <vector>

namespace {

int fail(const char* what, rb_status st) {
	std::printf("%s: %s\n", what, rb_status_string(st));
	return 1;
}

struct scene_handle {
	rb_scene* s = nullptr;
	rb_scene_desc desc{};
	rb_camera_desc camera{};
	~scene_handle() { rb_scene_free(s); }
};

rb_status make_scene(uint32_t kind, uint32_t seed, int32_t w, int32_t h, scene_handle& out) {
	rb_scene_gen_params p{};
	p.kind = kind;
	p.seed = seed;
	p.num_spheres = 12;
	p.subdivision = 2;
	p.width = w;
	p.height = h;
	rb_status st = rb_scene_generate(&p, &out.s);
	if (st == RB_OK) st = rb_scene_get(out.s, &out.desc, &out.camera);
	return st;
}

double mean(const std::vector<float>& v) {
	double s = 0;
	for (float x : v) s += x;
	return v.empty() ? 0.0 : s / static_cast<double>(v.size());
}

} // namespace

int main() {
	if (rb_abi_version() != RBGPU_ABI_VERSION) return fail("abi", RB_ERR_INVALID_ARGUMENT);
	rb_context* ctx = nullptr;
	rb_status st = rb_context_create(&ctx, 0);
	if (st == RB_ERR_NO_DEVICE) {
		std::printf("no device: %s\n", rb_status_string(st));
		return 0;
	}
	if (st != RB_OK) return fail("rb_context_create", st);
	scene_handle box, spheres;
	if ((st = make_scene(RB_SCENE_BOX, 0, 64, 64, box)) != RB_OK) return fail("box", st);
	if ((st = make_scene(RB_SCENE_SPHERES, 5, 48, 32, spheres)) != RB_OK) return fail("spheres", st);

	// path_integrator(sampler2d(16), sampler1d, max_depth 5, threshold 1)::render
	if ((st = rb_scene_upload(ctx, &box.desc)) != RB_OK) return fail("rb_scene_upload", st);
	rb_render_params p{};
	p.camera = box.camera;
	p.spp = 16;
	p.max_depth = 5;
	p.rr_threshold = 1.f;
	p.flags = RB_RENDER_RESET;
	std::vector<float> rgb(3ull * box.camera.width * box.camera.height);
	if ((st = rb_render(ctx, &p, rgb.data())) != RB_OK) return fail("rb_render", st);
	rb_render_stats stats{};
	rb_render_stats_get(ctx, &stats);

	// two scenes in one batched render
	const rb_scene_desc scenes[2] = {box.desc, spheres.desc};
	if ((st = rb_batch_upload(ctx, scenes, 2)) != RB_OK) return fail("rb_batch_upload", st);
	rb_batch_view views[2] = {};
	views[0].camera = box.camera;
	views[0].spp = 16;
	views[1].camera = spheres.camera;
	views[1].spp = 8;
	views[1].seed = 3;
	rb_batch_params bp{views, 2, 5, 1.f, RB_RENDER_RESET, nullptr};
	float done_ms[2] = {0.f, 0.f};
	if ((st = rb_batch_render(ctx, &bp, done_ms)) != RB_OK) return fail("rb_batch_render", st);
	std::vector<float> batch_box(rgb.size());
	if ((st = rb_batch_image(ctx, 0, batch_box.data())) != RB_OK) return fail("rb_batch_image", st);
	// the batch renders the box with the same per-sample streams as rb_render did
	double max_diff = 0;
	for (size_t i = 0; i < rgb.size(); i++) max_diff = std::fmax(max_diff, std::fabs(static_cast<double>(rgb[i]) - batch_box[i]));
	rb_context_destroy(ctx);
	std::printf("ok mean=%.6f samples=%llu extend_rays=%llu batch_max_diff=%.3g done_ms=%.3f,%.3f\n", mean(rgb),
		static_cast<unsigned long long>(stats.samples), static_cast<unsigned long long>(stats.extend_rays), max_diff,
		done_ms[0], done_ms[1]);
	return max_diff <= 1e-6 * (1.0 + mean(rgb)) ? 0 : 2;
}
