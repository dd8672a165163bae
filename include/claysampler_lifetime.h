/*
 * claysampler_b200 note-lifetime predictor — a small MLP that predicts, from a
 * note's region parameters, velocity, key and held time, how long the note stays
 * audible and how loud it peaks.  No render path reads it: the plain tail
 * detection judges every job, so output PCM is the same with or without the
 * predictor.  Its predictions size per-note lifetime reservations on the host
 * side (claysampler_b200/lifetime.py), which report how much a renderer that ends
 * voices at their audible end could save.
 *
 * No counterpart in the reference: ClaySampler decides every length after
 * rendering (the natural endpoint search, src/cuda/tail.cu:83-139) and sizes its
 * scratch from the plans (src/cuda/renderer.cpp:864-932).  The training labels
 * come from the renderer's own single-note renders (cs_note_labels).
 *
 * Network: CS_LIFETIME_FEATURES -> 64 -> 64 -> 2, ReLU, BF16 weights (the float32
 * master copy is rounded to bfloat16, nearest-even, wherever a kernel reads a
 * weight) with float32 accumulation and float32 biases.  Inputs are standardised
 * and outputs de-standardised with the `norm` vector.
 *
 * Parameter vector (float32, device, CS_LIFETIME_PARAMS entries):
 *   [W1_AT, B1_AT)  W1, 64 x 16, one row of 16 input weights per hidden unit
 *   [B1_AT, W2_AT)  b1[64]
 *   [W2_AT, B2_AT)  W2, 64 x 64, one row of 64 weights per second-layer unit
 *   [B2_AT, W3_AT)  b2[64]
 *   [W3_AT, B3_AT)  W3, 2 x 64
 *   [B3_AT, PARAMS) b3[2]
 * Normalisation (float32, device, CS_LIFETIME_NORM entries): feature mean[16],
 * feature 1/std[16], target mean[2], target std[2].
 *
 * Loss: L = 1/(2n) * sum over samples and both outputs of (y - t')^2, where y is
 * the standardised output and t' = (t - target mean) / target std.
 *
 * All pointers are device pointers; every call is enqueued on `stream` (a
 * cudaStream_t, NULL = the legacy default stream) and returns 0 once enqueued, or
 * nonzero with a message from cs_lifetime_last_error().
 */
#ifndef CLAYSAMPLER_LIFETIME_H
#define CLAYSAMPLER_LIFETIME_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CS_LIFETIME_FEATURES 16
#define CS_LIFETIME_HIDDEN 64
#define CS_LIFETIME_OUTPUTS 2
#define CS_LIFETIME_W1_AT 0
#define CS_LIFETIME_B1_AT (CS_LIFETIME_W1_AT + CS_LIFETIME_HIDDEN * CS_LIFETIME_FEATURES)
#define CS_LIFETIME_W2_AT (CS_LIFETIME_B1_AT + CS_LIFETIME_HIDDEN)
#define CS_LIFETIME_B2_AT (CS_LIFETIME_W2_AT + CS_LIFETIME_HIDDEN * CS_LIFETIME_HIDDEN)
#define CS_LIFETIME_W3_AT (CS_LIFETIME_B2_AT + CS_LIFETIME_HIDDEN)
#define CS_LIFETIME_B3_AT (CS_LIFETIME_W3_AT + CS_LIFETIME_OUTPUTS * CS_LIFETIME_HIDDEN)
#define CS_LIFETIME_PARAMS (CS_LIFETIME_B3_AT + CS_LIFETIME_OUTPUTS)
#define CS_LIFETIME_NORM (2 * CS_LIFETIME_FEATURES + 2 * CS_LIFETIME_OUTPUTS)
/* Samples per block of the fused gradient kernel; one partial row per block. */
#define CS_LIFETIME_BLOCK_SAMPLES 128

/* Predictions for `count` feature rows (row-major, CS_LIFETIME_FEATURES floats
 * each): `predictions` receives CS_LIFETIME_OUTPUTS floats per row, in target
 * units (log audible frames, peak dBFS). */
int cs_lifetime_forward(const float* params, const float* norm, const float* features, int count,
                        float* predictions, void* stream);

/* Floats of `partials` scratch the two calls below need for `count` samples:
 * one row of CS_LIFETIME_PARAMS + 1 floats per CS_LIFETIME_BLOCK_SAMPLES samples. */
size_t cs_lifetime_partial_floats(int count);

/* Fused forward + backward over `count` samples: `gradient` (CS_LIFETIME_PARAMS + 1
 * floats) receives dL/dparams followed by the loss L.  Per-block partial sums go to
 * `partials` and are added in block order, so results are deterministic. */
int cs_lifetime_gradient(const float* params, const float* norm, const float* features,
                         const float* targets, int count, float* partials, float* gradient, void* stream);

/* One Adam step (beta1 0.9, beta2 0.999, eps 1e-8) on a minibatch of `count`
 * samples: the fused forward + backward above, then the update of `params` and of
 * the moment vectors `moment1` / `moment2` (CS_LIFETIME_PARAMS floats each, zero
 * before step 1).  `step` counts from 1; `loss` (one float) receives the
 * minibatch loss before the update. */
int cs_lifetime_train_step(float* params, float* moment1, float* moment2, const float* norm,
                           const float* features, const float* targets, int count, float* partials,
                           int step, float learning_rate, float* loss, void* stream);

/* Training labels from a rendered float mix (float2 per frame, as the renderer's
 * natural mix): for each of `count` frame windows [windows[2i], windows[2i+1])
 * `peak[i]` receives the largest |sample| over both channels, and `last[i]` the
 * offset from the window's start of the last frame whose larger channel magnitude
 * is at least `threshold` (-1 when none is). */
int cs_note_labels(const float* mix, const int64_t* windows, int count, float threshold, float* peak,
                   int32_t* last, void* stream);

const char* cs_lifetime_last_error(void);

#ifdef __cplusplus
}
#endif

#endif
