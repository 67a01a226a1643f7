/*
 * Force-included ahead of the reference headers when oracle/build_ref.sh
 * compiles the reference renderer on Linux (test infrastructure only).
 *
 * The reference is written for MSVC, where `abs`, `sqrt` and `pow` called
 * unqualified on a float resolve to the float overloads.  GCC's <cmath>
 * leaves only `int abs(int)` / `double sqrt(double)` in the global
 * namespace, which turns `abs(float)` into an integer truncation
 * (core/texture.h:109, renderer/surface_shader.h:76,250).  Pulling the
 * std overloads into the global namespace restores the float semantics
 * the reference's own GPU build (CUDA device overloads) and MSVC build use.
 */
#pragma once
#include <cmath>
#include <cstdlib>
using std::abs;
using std::sqrt;
using std::pow;
