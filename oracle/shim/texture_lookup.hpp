// Shim for compiling the reference's image textures with g++ (test
// infrastructure, part of the oracle build).
//
// image_texture_t<2, T>::sample (textures/detail/image_texture.hpp:65-66) calls
// clamp(float, real, real) unqualified from namespace rainbow::cpus::textures.
// With standard two-phase name lookup the spectrum overload
// (shared/spectrums/detail/coefficient_specturm.hpp:253) made visible by a
// using-directive hides rainbow::core::math::clamp, and the call does not
// compile; the reference means the scalar clamp of rainbow-core. This
// using-declaration makes that clamp the one the call finds, with no change to
// what it computes.
#pragma once

#include "rainbow-core/math/math.hpp"
#include "rainbow-cpu/textures/texture.hpp"

namespace rainbow::cpus::textures {
using rainbow::core::math::clamp;
}
