// wavefront_photon_mapping_integrator: the reference's stochastic progressive
// photon mapping on the B200 core, as a rainbow `integrator`.
//
// A drop-in for rainbow::cpus::integrators::photon_mapping_integrator
// (rainbow-cpu/integrators/photon_mapping_integrator.hpp:9-13): same
// constructor (sampler2d, sampler1d, iterations = 64, max_depth = 5,
// photons = 0, radius = 1), same render(camera, scene) entry point
// (integrator.hpp:64-66). render() exports the scene and the perspective camera
// to the C ABI (include/rbgpu.h), runs rb_render_photons, and writes every
// pixel's value through film::set_pixel(index, value) as the reference's
// render does (photon_mapping_integrator.cpp:545-551). Pixels and photons draw
// from their own PCG32 streams instead of the reference's per-tile and
// per-chunk ones, so images agree statistically, not pixel for pixel. The
// samplers only fix the random-number kind (uniform), as in the reference,
// which clones them for its streams.
#pragma once

#include "rainbow-cpu/integrators/integrator.hpp"

struct rb_context;

namespace rainbow::cpus::integrators {

	class wavefront_photon_mapping_integrator final : public integrator {
	public:
		explicit wavefront_photon_mapping_integrator(
			const std::shared_ptr<sampler2d>& sampler2d,
			const std::shared_ptr<sampler1d>& sampler1d,
			size_t iterations = 64, size_t max_depth = 5,
			size_t photons = 0, real radius = 1);

		~wavefront_photon_mapping_integrator();

		// Throws std::runtime_error (with rb_status_string's text) when the scene
		// holds something the core does not render or the device fails; the film
		// is left as it was.
		void render(
			const std::shared_ptr<camera>& camera,
			const std::shared_ptr<scene>& scene) override;

		// CUDA device of the next render (default 0) and the stream seed (default 0).
		void set_device(int device) noexcept;
		void set_seed(uint32_t seed) noexcept;
	private:
		std::shared_ptr<sampler2d> mSampler2D;
		std::shared_ptr<sampler1d> mSampler1D;
		size_t mIterations = 64;
		size_t mMaxDepth = 5;
		size_t mPhotons = 0;
		real mRadius = 1;
		int mDevice = 0;
		uint32_t mSeed = 0;
		rb_context* mContext = nullptr;
	};

}
