// wavefront_path_integrator: the reference's path integrator on the B200
// wavefront core, as a rainbow `integrator`.
//
// A drop-in for rainbow::cpus::integrators::path_integrator
// (rainbow-cpu/integrators/path_integrator.hpp:9-12): same constructor
// (sampler2d, sampler1d, max_depth = 5, threshold = 1), same render(camera,
// scene) entry point (integrator.hpp:64-66). render() exports the scene and the
// perspective camera to the C ABI (include/rbgpu.h), renders
// sampler2d->samples_per_pixel() samples of every pixel of the film with
// path_integrator::trace's estimator on the GPU, and writes each pixel's mean
// back through film::set_pixel (cameras/film.cpp:197-205), as the reference's
// film would hold it after sampler_integrator::render with the box filter.
// Samples use one PCG32 stream per (pixel, sample) instead of the reference's
// one per 16 x 16 tile, so images agree statistically, not sample for sample.
//
// Compiled against the reference's headers (include root: the reference
// checkout) and linked with librbgpu.so.
#pragma once

#include "rainbow-cpu/integrators/integrator.hpp"

struct rb_context;

namespace rainbow::cpus::integrators {

	class wavefront_path_integrator final : public integrator {
	public:
		explicit wavefront_path_integrator(
			const std::shared_ptr<sampler2d>& sampler2d,
			const std::shared_ptr<sampler1d>& sampler1d,
			size_t max_depth = 5, real threshold = 1);

		~wavefront_path_integrator();

		// Throws std::runtime_error (with rb_status_string's text) when the scene
		// holds something the core does not render (then the caller can fall
		// back to path_integrator) or the device fails; the film is left as it was.
		void render(
			const std::shared_ptr<camera>& camera,
			const std::shared_ptr<scene>& scene) override;

		// CUDA device of the next render (default 0) and the seed mixed into every
		// per-sample stream (default 0).
		void set_device(int device) noexcept;
		void set_seed(uint32_t seed) noexcept;
	private:
		std::shared_ptr<sampler2d> mSampler2D;
		std::shared_ptr<sampler1d> mSampler1D;
		size_t mMaxDepth = 5;
		real mThreshold = 1;
		int mDevice = 0;
		uint32_t mSeed = 0;
		rb_context* mContext = nullptr;
	};

}
