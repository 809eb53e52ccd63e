// Seeded synthetic rectified stereo pairs for tests and benchmarks.
//
// Not part of the SGM boundary (it has no counterpart in vx-vision): the
// reference tests and benches build their own inputs
// (vx-vision/tests/test_kernels.rs:790-812, benches/kernel_benchmarks.rs:14-24).
// Convention: a left pixel (x, y) with disparity d appears in the right image at
// (x - d, y), i.e. R(x - d, y) = L(x, y), which is what the SGM shader matches
// (vx-vision/shaders/SGMStereo.metal:133-141).
#pragma once
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum vx_synth_scene {
    VX_SYNTH_PLANES = 0,   // piecewise-constant fronto-parallel planes, integer d
    VX_SYNTH_SLANTED = 1,  // slanted planes, |grad d| <= 0.2 px/px, real-valued d
    VX_SYNTH_SURFACE = 2,  // planes + sinusoidal surface (20 px amplitude) + 10% textureless
};

// Fills left/right (w*h u8, row pitch w) and, if non-null, the ground-truth left
// disparity (w*h f32). Disparities lie in [d_lo, d_hi]. Returns 0 or -1.
int vx_synth_pair(int scene, int w, int h, float d_lo, float d_hi, uint64_t seed, uint8_t* left,
                  uint8_t* right, float* gt_disparity);

#ifdef __cplusplus
}
#endif
