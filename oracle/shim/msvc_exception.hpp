// Force-included (g++ -include) into rainbow-cpu/scatterings/scattering_function.cpp
// only. That file throws std::exception("..."), a constructor that exists in
// MSVC's standard library but not in libstdc++ (scattering_function.cpp:49,55).
// Every standard header the file reaches is included first, then a
// function-like macro maps that one construct to std::runtime_error. The
// throwing functions (rho) are never called on the path-tracing path.
#pragma once
#include <algorithm>
#include <array>
#include <atomic>
#include <cassert>
#include <cmath>
#include <cstddef>
#include <exception>
#include <limits>
#include <memory>
#include <optional>
#include <stdexcept>
#include <string>
#include <tuple>
#include <type_traits>
#include <vector>
#define exception(message) runtime_error(message)
