// wavefront_path_integrator::render: export, one rb_render call, write-back.
#include "wavefront_path_integrator.hpp"

#include "scene_export.hpp"

#include <stdexcept>
#include <string>
#include <vector>

namespace rainbow::cpus::integrators {

	namespace {
		void check(rb_status st, const char* what) {
			if (st != RB_OK) throw std::runtime_error(std::string(what) + ": " + rb_status_string(st));
		}
	}

	wavefront_path_integrator::wavefront_path_integrator(
		const std::shared_ptr<sampler2d>& sampler2d,
		const std::shared_ptr<sampler1d>& sampler1d,
		size_t max_depth, real threshold) :
		mSampler2D(sampler2d), mSampler1D(sampler1d), mMaxDepth(max_depth), mThreshold(threshold)
	{
	}

	wavefront_path_integrator::~wavefront_path_integrator()
	{
		if (mContext != nullptr) rb_context_destroy(mContext);
	}

	void wavefront_path_integrator::set_device(int device) noexcept
	{
		if (device != mDevice && mContext != nullptr) {
			rb_context_destroy(mContext);
			mContext = nullptr;
		}
		mDevice = device;
	}

	void wavefront_path_integrator::set_seed(uint32_t seed) noexcept { mSeed = seed; }

	void wavefront_path_integrator::render(
		const std::shared_ptr<camera>& camera,
		const std::shared_ptr<scene>& scene)
	{
		rb::adapter::exported_scene exported;
		check(rb::adapter::export_scene(*scene, exported), "scene export");
		rb_render_params params{};
		check(rb::adapter::export_camera(*camera, params.camera), "camera export");
		if (mContext == nullptr) check(rb_context_create(&mContext, mDevice), "rb_context_create");
		check(rb_scene_upload(mContext, &exported.desc), "rb_scene_upload");

		params.spp = static_cast<uint32_t>(mSampler2D->samples_per_pixel());
		params.first_sample = 0;
		params.max_depth = static_cast<uint32_t>(mMaxDepth);
		params.rr_threshold = mThreshold;
		params.seed = mSeed;
		params.flags = RB_RENDER_RESET;
		const int width = params.camera.width, height = params.camera.height;
		std::vector<float> rgb(static_cast<size_t>(width) * height * 3);
		check(rb_render(mContext, &params, rgb.data()), "rb_render");

		// the film's pixels (its crop window, film::pixels_bound) get their means
		const auto film = camera->film();
		const auto bound = film->pixels_bound();
		for (int y = bound.min.y; y < bound.max.y; y++) {
			for (int x = bound.min.x; x < bound.max.x; x++) {
				const float* p = rgb.data() + 3 * (static_cast<size_t>(y) * width + x);
				film->set_pixel(vector2i(x, y), spectrum(p[0], p[1], p[2]));
			}
		}
	}

}
