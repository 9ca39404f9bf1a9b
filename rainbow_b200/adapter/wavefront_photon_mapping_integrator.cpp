// wavefront_photon_mapping_integrator::render: export, one rb_render_photons call, write-back.
#include "wavefront_photon_mapping_integrator.hpp"

#include "scene_export.hpp"

#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

namespace rainbow::cpus::integrators {

	namespace {
		void check(rb_status st, const char* what) {
			if (st != RB_OK) throw std::runtime_error(std::string(what) + ": " + rb_status_string(st));
		}
	}

	wavefront_photon_mapping_integrator::wavefront_photon_mapping_integrator(
		const std::shared_ptr<sampler2d>& sampler2d,
		const std::shared_ptr<sampler1d>& sampler1d,
		size_t iterations, size_t max_depth, size_t photons, real radius) :
		mSampler2D(sampler2d), mSampler1D(sampler1d), mIterations(iterations), mMaxDepth(max_depth),
		mPhotons(photons), mRadius(radius)
	{
	}

	wavefront_photon_mapping_integrator::~wavefront_photon_mapping_integrator()
	{
		if (mContext != nullptr) rb_context_destroy(mContext);
	}

	void wavefront_photon_mapping_integrator::set_device(int device) noexcept
	{
		if (device != mDevice && mContext != nullptr) {
			rb_context_destroy(mContext);
			mContext = nullptr;
		}
		mDevice = device;
	}

	void wavefront_photon_mapping_integrator::set_seed(uint32_t seed) noexcept { mSeed = seed; }

	void wavefront_photon_mapping_integrator::render(
		const std::shared_ptr<camera>& camera,
		const std::shared_ptr<scene>& scene)
	{
		if (mPhotons > std::numeric_limits<uint32_t>::max() || mIterations > std::numeric_limits<uint32_t>::max())
			check(RB_ERR_INVALID_ARGUMENT, "photon counts");
		rb::adapter::exported_scene exported;
		check(rb::adapter::export_scene(*scene, exported), "scene export");
		rb_photon_params params{};
		check(rb::adapter::export_camera(*camera, params.camera), "camera export");
		if (mContext == nullptr) check(rb_context_create(&mContext, mDevice), "rb_context_create");
		check(rb_scene_upload(mContext, &exported.desc), "rb_scene_upload");

		params.iterations = static_cast<uint32_t>(mIterations);
		params.max_depth = static_cast<uint32_t>(mMaxDepth);
		params.photons = static_cast<uint32_t>(mPhotons);
		params.radius = mRadius;
		params.seed = mSeed;
		const size_t pixels = static_cast<size_t>(params.camera.width) * params.camera.height;
		std::vector<float> rgb(pixels * 3);
		check(rb_render_photons(mContext, &params, rgb.data()), "rb_render_photons");

		const auto film = camera->film();
		for (size_t i = 0; i < pixels; i++)
			film->set_pixel(i, spectrum(rgb[3 * i], rgb[3 * i + 1], rgb[3 * i + 2]));
	}

}
