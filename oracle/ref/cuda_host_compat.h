/*
 * Test infrastructure for the oracle: the few CUDA spellings the reference's
 * src/cuda/render.cu uses, mapped onto host C++ so that file compiles unchanged
 * with g++ and runs the reference's own per-voice render math on the CPU.
 *
 * Rounding follows the CUDA intrinsics' definitions: *_rd rounds toward -inf,
 * *_rn to nearest even (the host default rounding mode).  No FMA contraction is
 * requested (-ffp-contract=off), so only the explicit fmaf calls fuse.
 */
#pragma once

#include <algorithm>
#include <cmath>

#define __device__
#define __global__
#define __host__
#define __forceinline__ inline

struct float2 { float x, y; };
struct short2 { short x, y; };
inline float2 make_float2(float x, float y) { return {x, y}; }
inline short2 make_short2(short x, short y) { return {x, y}; }
inline int __double2int_rd(double v) { return static_cast<int>(std::floor(v)); }
inline int __double2int_rn(double v) { return static_cast<int>(std::nearbyint(v)); }
inline int __float2int_rn(float v) { return static_cast<int>(std::nearbyintf(v)); }

struct HostDim3 { unsigned x = 0, y = 0, z = 0; };
extern thread_local HostDim3 threadIdx, blockIdx, blockDim;

using std::max;
using std::min;
